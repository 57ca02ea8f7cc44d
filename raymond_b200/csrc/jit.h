// NVRTC compilation of the generated material module to an sm_100a cubin,
// cached on disk by content hash, loaded through the CUDA runtime's library
// API (the reference compiled its generated Metal with device.makeLibrary,
// MaterialBuilder.swift:322-324).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace rmdhost {

struct JitModule {
    cudaLibrary_t library = nullptr;
    cudaKernel_t shade = nullptr;
    cudaKernel_t envmapBuild = nullptr;
    cudaKernel_t materialEval = nullptr;
    double compileMs = 0;
    bool fromCache = false;
    std::string log;
};

// Returns an empty string on success, else the error (NVRTC log included).
// extraDefines: "-DNAME=VALUE" options (launch-bound and tile choices of the autotuner)
std::string compileModule(const std::string &source, JitModule &out, const std::vector<std::string> &extraDefines = {});
void unloadModule(JitModule &m);
// NVRTC only (no device needed): source -> sm_100a cubin, through the disk cache.
std::string compileCubin(const std::string &source, std::vector<char> &cubin, std::string &log, bool &fromCache,
                         const std::vector<std::string> &extraDefines = {});

}  // namespace rmdhost
