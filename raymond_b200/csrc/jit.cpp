// NVRTC driver for the material module.
#include "jit.h"

#include <nvrtc.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <sys/stat.h>
#include <vector>

namespace rmdhost {

// device/*.cuh as string literals, generated at build time (embed_headers.py)
struct EmbeddedHeader {
    const char *name;
    const char *source;
};
extern const EmbeddedHeader kEmbeddedHeaders[];
extern const int kNumEmbeddedHeaders;

namespace {

uint64_t fnv1a(const std::string &s, uint64_t h = 1469598103934665603ull) {
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

std::string cacheDir() {
    if (const char *d = std::getenv("RMD_JIT_CACHE")) return d;
    const char *home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/raymond_b200";
}

void mkdirs(const std::string &path) {
    std::string cur;
    std::stringstream ss(path);
    std::string part;
    if (!path.empty() && path[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        mkdir(cur.c_str(), 0755);
    }
}

// RMD_JIT_FMAD=0 compiles the shading module without multiply-add
// contraction (NVRTC contracts by default), the evaluation order of the
// oracle's host build.
const std::vector<const char *> &options() {
    static std::vector<const char *> o = [] {
        std::vector<const char *> v = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "-DRMD_JIT=1",
                                       "--device-as-default-execution-space"};
        const char *f = std::getenv("RMD_JIT_FMAD");
        if (f && std::string(f) == "0") v.push_back("--fmad=false");
        return v;
    }();
    return o;
}

}  // namespace

std::string compileModule(const std::string &source, JitModule &out, const std::vector<std::string> &extraDefines) {
    std::vector<char> cubin;
    const auto t0 = std::chrono::steady_clock::now();
    std::string err = compileCubin(source, cubin, out.log, out.fromCache, extraDefines);
    if (!err.empty()) return err;
    cudaError_t e = cudaLibraryLoadData(&out.library, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess) return std::string("cudaLibraryLoadData: ") + cudaGetErrorString(e);
    if ((e = cudaLibraryGetKernel(&out.shade, out.library, "rmd_shade")) != cudaSuccess ||
        (e = cudaLibraryGetKernel(&out.envmapBuild, out.library, "rmd_envmap_build")) != cudaSuccess ||
        (e = cudaLibraryGetKernel(&out.materialEval, out.library, "rmd_material_eval")) != cudaSuccess)
        return std::string("cudaLibraryGetKernel: ") + cudaGetErrorString(e);
    out.compileMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return "";
}

std::string compileCubin(const std::string &source, std::vector<char> &cubin, std::string &logOut, bool &fromCache,
                         const std::vector<std::string> &extraDefines) {
    fromCache = false;
    int major = 0, minor = 0;
    nvrtcVersion(&major, &minor);
    std::string key = source;
    for (auto o : options()) key += o;
    for (const std::string &d : extraDefines) key += d;
    key += std::to_string(major) + "." + std::to_string(minor);
    for (int i = 0; i < kNumEmbeddedHeaders; i++) key += kEmbeddedHeaders[i].source;
    char hex[32];
    std::snprintf(hex, sizeof(hex), "%016llx", (unsigned long long)fnv1a(key));
    const std::string dir = cacheDir();
    const std::string path = dir + "/mat_" + hex + ".cubin";
    const bool useCache = std::getenv("RMD_JIT_NOCACHE") == nullptr;

    cubin.clear();
    if (useCache) {
        std::ifstream f(path, std::ios::binary);
        if (f) {
            cubin.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
            fromCache = !cubin.empty();
        }
    }
    if (cubin.empty()) {
        std::vector<const char *> names, srcs;
        for (int i = 0; i < kNumEmbeddedHeaders; i++) {
            // reachable both as "device/x.cuh" and, from inside device/, as "x.cuh"
            names.push_back(kEmbeddedHeaders[i].name);
            srcs.push_back(kEmbeddedHeaders[i].source);
            const char *slash = std::strrchr(kEmbeddedHeaders[i].name, '/');
            if (slash) {
                names.push_back(slash + 1);
                srcs.push_back(kEmbeddedHeaders[i].source);
            }
        }
        nvrtcProgram prog;
        nvrtcResult r = nvrtcCreateProgram(&prog, source.c_str(), "materials.cu", (int)names.size(), srcs.data(),
                                           names.data());
        if (r != NVRTC_SUCCESS) return std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(r);
        std::vector<const char *> opts = options();
        if (std::getenv("RMD_JIT_VERBOSE")) opts.push_back("--ptxas-options=-v");
        for (const std::string &d : extraDefines) opts.push_back(d.c_str());
        r = nvrtcCompileProgram(prog, (int)opts.size(), opts.data());
        size_t logSize = 0;
        nvrtcGetProgramLogSize(prog, &logSize);
        std::string log(logSize, '\0');
        if (logSize) nvrtcGetProgramLog(prog, &log[0]);
        logOut = log;
        if (r != NVRTC_SUCCESS) {
            nvrtcDestroyProgram(&prog);
            return std::string("NVRTC compile failed: ") + nvrtcGetErrorString(r) + "\n" + log;
        }
        size_t size = 0;
        nvrtcGetCUBINSize(prog, &size);
        cubin.resize(size);
        nvrtcGetCUBIN(prog, cubin.data());
        nvrtcDestroyProgram(&prog);
        if (useCache) {
            mkdirs(dir);
            const std::string tmp = path + ".tmp" + std::to_string((long long)std::rand());
            std::ofstream f(tmp, std::ios::binary);
            f.write(cubin.data(), (std::streamsize)cubin.size());
            f.close();
            std::rename(tmp.c_str(), path.c_str());
        }
    }
    return "";
}

void unloadModule(JitModule &m) {
    if (m.library) cudaLibraryUnload(m.library);
    m = JitModule();
}

}  // namespace rmdhost
