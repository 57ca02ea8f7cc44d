// Node graph -> CUDA source: MaterialBuilder.swift's Codegen
// (raymond/host/scene/MaterialBuilder.swift:32-826) re-targeted at NVRTC.
//
// Kept from the reference: output nodes are visited in sorted-name order and
// emitted depth-first with inputs in sorted-name order (:684-691, :793-825);
// cycles and multi-input links are errors (:45-51); unlinked inputs take
// their literal wrapped in the socket's coercion, `TYPE(value)` (:110-121);
// links become `TYPE(n_src.output)` (:124-129); a few inputs default to
// shading.uv / shading.generated / shading.normal (provideDefaults,
// :762-791); kernel template parameters follow makeKernelInvocation
// (:327-661) and enum values are `k<Kernel>::<NS>_<VALUE>` (:147-150); the
// per-material functions are dispatched by shadeSurface / shadeLight switch
// tables (:289-300).
//
// Added for the GPU: node variables are numbered instead of named, and with
// `hoist` every literal becomes a load P[k] from the material's parameter
// block, so materials whose graphs have the same structure share one
// function (one code path for a warp that shades several of them).
#include "codegen.h"

#include "sky.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <map>
#include <set>

namespace rmdhost {

std::string makeIdentifier(const std::string &name) {
    size_t a = 0, b = name.size();
    while (a < b && name[a] == ' ') a++;
    while (b > a && name[b - 1] == ' ') b--;
    const std::string trimmed = name.substr(a, b - a);
    if (trimmed.empty()) return "";
    std::string cap;
    bool wordStart = true;
    for (char c : trimmed) {
        if (std::isalpha((unsigned char)c)) {
            cap += wordStart ? (char)std::toupper((unsigned char)c) : (char)std::tolower((unsigned char)c);
            wordStart = false;
        } else {
            cap += c;
            wordStart = !std::isdigit((unsigned char)c);
        }
    }
    std::string nospace;
    for (char c : cap)
        if (c != ' ') nospace += c;
    std::string out(1, (char)std::tolower((unsigned char)trimmed[0]));
    out += nospace.substr(1);
    for (auto &c : out)
        if (!(std::isalnum((unsigned char)c) || c == '_')) c = '_';
    return out;
}

namespace {

enum Kind { F1 = 1, F2 = 2, F3 = 3, F4 = 4, SH = 5, BOOL = 6 };

struct KernelDesc {
    std::map<std::string, Kind> fields;
};

const std::map<std::string, KernelDesc> &kernelTable() {
    static std::map<std::string, KernelDesc> t = [] {
        std::map<std::string, KernelDesc> m;
        auto add = [&](const char *k, std::initializer_list<std::pair<const char *, Kind>> f) {
            KernelDesc d;
            for (auto &p : f) d.fields[p.first] = p.second;
            m[k] = d;
        };
        add("TextureCoordinate", {{"generated", F3}, {"uv", F3}, {"object", F3}, {"normal", F3}, {"reflection", F3}});
        add("UVMapCoordinate", {{"uv", F3}});
        add("NewGeometry", {{"normal", F3}, {"trueNormal", F3}, {"tangent", F3}, {"position", F3}, {"parametric", F3},
                            {"incoming", F3}, {"randomPerIsland", F3}, {"backfacing", BOOL}});
        add("LightPath", {{"isCameraRay", BOOL}, {"isReflectionRay", BOOL}, {"isTransmissionRay", BOOL},
                          {"isShadowRay", BOOL}, {"isDiffuseRay", BOOL}, {"isGlossyRay", BOOL},
                          {"isSingularRay", BOOL}, {"rayLength", F1}});
        add("TexChecker", {{"scale", F1}, {"color1", F4}, {"color2", F4}, {"vector", F3}, {"fac", F1}, {"color", F4}});
        add("TexNoise", {{"detail", F1}, {"distortion", F1}, {"roughness", F1}, {"scale", F1}, {"w", F1},
                         {"vector", F3}, {"fac", F1}, {"color", F4}});
        add("ColorRamp", {{"fac", F1}, {"color", F4}});
        add("ColorMix", {{"color1", F4}, {"color2", F4}, {"fac", F1}, {"color", F4}});
        add("Mix", {{"a_Color", F4}, {"b_Color", F4}, {"result_Color", F4}, {"a_Float", F1}, {"b_Float", F1},
                    {"result_Float", F1}, {"a_Vector", F3}, {"b_Vector", F3}, {"result_Vector", F3},
                    {"factor_Float", F1}, {"factor_Vector", F3}});
        add("Math", {{"value", F1}, {"value_001", F1}, {"value_002", F1}});
        add("VectorMath", {{"scale", F1}, {"value", F1}, {"vector", F3}, {"vector_001", F3}, {"vector_002", F3}});
        add("SeparateVector", {{"vector", F3}, {"x", F1}, {"y", F1}, {"z", F1}});
        add("CombineVector", {{"x", F1}, {"y", F1}, {"z", F1}, {"vector", F3}});
        add("MapRange", {{"fromMin", F1}, {"fromMax", F1}, {"toMin", F1}, {"toMax", F1}, {"steps", F1},
                         {"steps_Float3", F3}, {"from_Min_Float3", F3}, {"from_Max_Float3", F3},
                         {"to_Min_Float3", F3}, {"to_Max_Float3", F3}, {"value", F1}, {"vector", F3}, {"result", F1}});
        add("Value", {{"value", F1}});
        add("RGB", {{"color", F4}});
        add("RGBToBW", {{"color", F4}, {"val", F1}});
        add("ColorInvert", {{"color", F4}, {"fac", F1}});
        add("Gamma", {{"color", F4}, {"gamma", F1}});
        add("TexImage", {{"vector", F3}, {"color", F4}, {"alpha", F1}});
        add("TexNishita", {{"vector", F3}, {"color", F4}});
        add("Mapping", {{"scale", F3}, {"rotation", F3}, {"location", F3}, {"vector", F3}});
        add("NormalMap", {{"color", F4}, {"strength", F1}, {"normal", F3}});
        add("HueSaturation", {{"color", F4}, {"fac", F1}, {"hue", F1}, {"saturation", F1}, {"value", F1}});
        add("BrightnessContrast", {{"bright", F1}, {"contrast", F1}, {"color", F4}});
        add("Blackbody", {{"temperature", F1}, {"color", F4}});
        add("Fresnel", {{"ior", F1}, {"normal", F3}, {"fac", F1}});
        add("LayerWeight", {{"blend", F1}, {"normal", F3}, {"fresnel", F1}, {"facing", F1}});
        add("Emission", {{"color", F4}, {"strength", F1}, {"weight", F1}, {"emission", SH}});
        add("Background", {{"color", F4}, {"strength", F1}, {"weight", F1}, {"background", SH}});
        add("BsdfPrincipled",
            {{"weight", F1}, {"emission", F4}, {"sheenTint", F1}, {"emissionStrength", F1}, {"transmission", F1},
             {"clearcoatNormal", F3}, {"alpha", F1}, {"specularTint", F1}, {"tangent", F3}, {"roughness", F1},
             {"subsurfaceIor", F1}, {"anisotropic", F1}, {"sheen", F1}, {"subsurfaceRadius", F3}, {"normal", F3},
             {"subsurfaceAnisotropy", F1}, {"baseColor", F4}, {"transmissionRoughness", F1}, {"metallic", F1},
             {"specular", F1}, {"clearcoatRoughness", F1}, {"subsurfaceColor", F4}, {"subsurface", F1},
             {"ior", F1}, {"anisotropicRotation", F1}, {"clearcoat", F1}, {"bsdf", SH}});
        add("BsdfDiffuse", {{"color", F4}, {"normal", F3}, {"roughness", F1}, {"weight", F1}, {"bsdf", SH}});
        add("BsdfGlossy", {{"color", F4}, {"normal", F3}, {"roughness", F1}, {"weight", F1}, {"bsdf", SH}});
        add("BsdfGlass", {{"color", F4}, {"ior", F1}, {"normal", F3}, {"roughness", F1}, {"weight", F1}, {"bsdf", SH}});
        add("BsdfTransparent", {{"color", F4}, {"weight", F1}, {"bsdf", SH}});
        add("AddShader", {{"shader", SH}, {"shader_001", SH}});
        add("MixShader", {{"fac", F1}, {"shader", SH}, {"shader_001", SH}});
        add("OutputMaterial", {{"displacement", F3}, {"thickness", F1}, {"surface", SH}, {"volume", SH}});
        add("OutputWorld", {{"thickness", F1}, {"surface", SH}});
        add("OutputLight", {{"surface", SH}});
        return m;
    }();
    return t;
}

const rmd_node_param *findParam(const rmd_node &n, const char *key) {
    for (int i = 0; i < n.num_params; i++)
        if (n.params[i].key && std::string(n.params[i].key) == key) return &n.params[i];
    return nullptr;
}
std::string paramString(const rmd_node &n, const char *key, const char *fb) {
    auto p = findParam(n, key);
    return (p && p->string_value) ? std::string(p->string_value) : std::string(fb);
}
bool paramBool(const rmd_node &n, const char *key, bool fb) {
    auto p = findParam(n, key);
    return p ? p->number_value != 0 : fb;
}
float paramNumber(const rmd_node &n, const char *key, float fb) {
    auto p = findParam(n, key);
    return (p && (p->kind == RMD_PARAM_NUMBER || p->kind == RMD_PARAM_BOOL)) ? (float)p->number_value : fb;
}

// The sky of a TEX_SKY node as MaterialBuilder.swift:329-349 resolves it: a
// Hosek-Wilkie sky becomes a Nishita sky of the same sun direction (no disc,
// air 2, dust 0.5, ozone 1, the sun at least 5 degrees up, radiance scaled by
// 0.08); other types than Nishita are unsupported.  Missing parameters take
// Blender's defaults.
rmdsky::SkyOptions skyOptionsOf(const rmd_node &n) {
    rmdsky::SkyOptions o;
    std::string type = paramString(n, "sky_type", "NISHITA");
    o.sunElevation = paramNumber(n, "sun_elevation", 15.0f * (float)M_PI / 180.0f);
    o.sunRotation = paramNumber(n, "sun_rotation", 0.0f);
    o.sunDisc = paramBool(n, "sun_disc", true);
    o.sunSize = paramNumber(n, "sun_size", 0.545f * (float)M_PI / 180.0f);
    o.sunIntensity = paramNumber(n, "sun_intensity", 1.0f);
    o.altitude = paramNumber(n, "altitude", 0.0f);
    o.airDensity = paramNumber(n, "air_density", 1.0f);
    o.dustDensity = paramNumber(n, "dust_density", 1.0f);
    o.ozoneDensity = paramNumber(n, "ozone_density", 1.0f);
    o.scale = 1.0f;
    if (type == "HOSEK_WILKIE") {
        float dir[3] = {0.0f, 0.0f, 1.0f};
        auto p = findParam(n, "sun_direction");
        if (p && p->num_numbers >= 3)
            for (int i = 0; i < 3; i++) dir[i] = p->numbers[i];
        const float rotation = std::atan2(dir[0], dir[1]);
        const float elevation = std::asin(dir[2]);
        type = "NISHITA";
        o.sunDisc = false;
        o.airDensity = 2.0f;
        o.dustDensity = 0.5f;
        o.ozoneDensity = 1.0f;
        o.sunElevation = std::max(elevation, 5.0f * (float)M_PI / 180.0f);
        o.sunRotation = rotation;
        o.scale = 0.08f;
    }
    if (type != "NISHITA") throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "TexSky: unsupported sky type '" + type + "'"};
    return o;
}

// MaterialBuilder.swift:147-149
std::string enumValue(const std::string &kernel, const std::string &ns, const std::string &v,
                      const std::vector<std::string> &known) {
    std::string e;
    for (char c : v) e += (std::isalnum((unsigned char)c) || c == '_') ? (char)std::toupper((unsigned char)c) : '_';
    if (std::find(known.begin(), known.end(), e) == known.end())
        throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, kernel + ": unsupported " + ns + " '" + v + "'"};
    return "k" + kernel + "::" + ns + "_" + e;
}

std::string ftoa(float v) {
    char buf[64];
    if (v != v) return "__int_as_float(0x7fc00000)";
    if (v == INFINITY) return "__int_as_float(0x7f800000)";
    if (v == -INFINITY) return "__int_as_float(0xff800000)";
    std::snprintf(buf, sizeof(buf), "%.9gf", v);
    std::string s(buf);
    if (s.find_first_of(".en") == std::string::npos) s.insert(s.size() - 1, ".0");
    return s;
}

// Literals are emitted as placeholders `@L<k>@`; emitTable later replaces each
// one by a constant (no hoisting, or the same value in every material of the
// structure group) or by a load P[j] from the material's parameter block.
struct Emitter {
    bool hoist;
    std::vector<float> literals;  // this material's literals in emission order
    std::string lit(float v) {
        if (!hoist) return ftoa(v);
        literals.push_back(v);
        return "@L" + std::to_string(literals.size() - 1) + "@";
    }
    std::string vec(const float *v, int n) {
        if (n == 1) return lit(v[0]);
        std::string s = "make_float" + std::to_string(n) + "(";
        for (int i = 0; i < n; i++) s += (i ? ", " : "") + lit(v[i]);
        return s + ")";
    }
};

struct Invocation {
    std::string kernel;      // struct name used for the field table
    std::string type;        // full C++ type (with template parameters)
    std::string var;
    std::vector<std::string> lines;
};

Kind coercedKind(const std::string &type) {
    if (type == "VALUE") return F1;
    if (type == "RGBA") return F4;
    if (type == "VECTOR") return F3;
    if (type == "SHADER") return SH;
    throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "unsupported socket type '" + type + "'"};
}

// `dst = TYPE(expr)` with Metal's implicit scalar-to-vector widening
std::string assignment(const std::string &var, const std::string &field, Kind fieldKind, const std::string &type,
                       const std::string &expr) {
    const Kind k = coercedKind(type);
    std::string value = type + "(" + expr + ")";
    if (k != fieldKind) {
        if (k == F1 && fieldKind == F3) value = "f3(" + value + ")";
        else if (k == F1 && fieldKind == F4) value = "f4(" + value + ")";
        else
            throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED,
                               "cannot assign " + type + " to field '" + field + "' of " + var};
    }
    return var + "." + field + " = " + value + ";";
}

// makeKernelInvocation (MaterialBuilder.swift:327-661) for the kernels of device/nodes.cuh
Invocation makeInvocation(const rmd_node &n, Emitter &em, const TextureTable &textures) {
    const std::string t = n.type ? n.type : "";
    Invocation inv;
    auto plain = [&](const char *k) {
        inv.kernel = k;
        inv.type = k;
    };
    if (t == "TEX_COORD") plain("TextureCoordinate");
    else if (t == "UVMAP") plain("UVMapCoordinate");
    else if (t == "NEW_GEOMETRY") plain("NewGeometry");
    else if (t == "LIGHT_PATH") plain("LightPath");
    else if (t == "TEX_CHECKER") plain("TexChecker");
    else if (t == "TEX_NOISE") {
        inv.kernel = "TexNoise";
        inv.type = "TexNoise<" + enumValue("TexNoise", "DIMENSION", paramString(n, "noise_dimensions", "3D"),
                                           {"1D", "2D", "3D", "4D"}) + ">";
    } else if (t == "VALTORGB") {
        auto p = findParam(n, "elements");
        if (!p || p->num_numbers < 5 || p->num_numbers % 5 != 0 || p->num_numbers / 5 > 32)
            throw CodegenError{RMD_ERROR_INVALID_ARGUMENT, "ColorRamp needs 1..32 elements"};
        const int ne = p->num_numbers / 5;
        inv.kernel = "ColorRamp";
        inv.type = "ColorRamp<" + std::to_string(ne) + ">";
        for (int i = 0; i < ne; i++)
            inv.lines.push_back("@.elements[" + std::to_string(i) + "] = ColorRampElement{" +
                                em.lit(p->numbers[5 * i]) + ", " + em.vec(p->numbers + 5 * i + 1, 4) + "};");
    } else if (t == "MIX_RGB") {
        inv.kernel = "ColorMix";
        inv.type = "ColorMix<" +
                   enumValue("ColorMix", "BLEND_TYPE", paramString(n, "blend_type", "MIX"),
                             {"MIX", "ADD", "MULTIPLY", "SCREEN", "OVERLAY", "SUB", "COLOR", "LIGHTEN", "DARKEN",
                              "VALUE"}) +
                   ", " + (paramBool(n, "use_clamp", false) ? "true" : "false") + ">";
    } else if (t == "MIX") {
        inv.kernel = "Mix";
        inv.type = std::string("Mix<") + (paramBool(n, "clamp_factor", true) ? "true" : "false") + ", " +
                   (paramBool(n, "clamp_result", false) ? "true" : "false") + ", " +
                   enumValue("Mix", "FACTOR_MODE", paramString(n, "factor_mode", "UNIFORM"), {"UNIFORM", "NON_UNIFORM"}) +
                   ">";
    } else if (t == "MATH") {
        inv.kernel = "Math";
        inv.type = "Math<" +
                   enumValue("Math", "OPERATION", paramString(n, "operation", "ADD"),
                             {"ADD", "SUBTRACT", "MULTIPLY", "DIVIDE", "MULTIPLY_ADD", "POWER", "MINIMUM", "MAXIMUM",
                              "TANGENT", "LESS_THAN", "GREATER_THAN", "MODULO"}) +
                   ", " + (paramBool(n, "use_clamp", false) ? "true" : "false") + ">";
    } else if (t == "VECT_MATH") {
        inv.kernel = "VectorMath";
        inv.type = "VectorMath<" +
                   enumValue("VectorMath", "OPERATION", paramString(n, "operation", "ADD"),
                             {"ADD", "SUBTRACT", "MULTIPLY", "MULTIPLY_ADD", "NORMALIZE", "SCALE", "MINIMUM", "LENGTH",
                              "DOT_PRODUCT"}) +
                   ">";
    } else if (t == "SEPXYZ") plain("SeparateVector");
    else if (t == "COMBXYZ") plain("CombineVector");
    else if (t == "MAP_RANGE") {
        inv.kernel = "MapRange";
        inv.type = std::string("MapRange<") + (paramBool(n, "clamp", true) ? "true" : "false") + ", " +
                   enumValue("MapRange", "DATA_TYPE", paramString(n, "data_type", "FLOAT"), {"FLOAT"}) + ", " +
                   enumValue("MapRange", "INTERPOLATION_TYPE", paramString(n, "interpolation_type", "LINEAR"),
                             {"LINEAR"}) +
                   ">";
    } else if (t == "VALUE") {
        plain("Value");
        auto p = findParam(n, "value");
        float v = p ? (float)p->number_value : 0.0f;
        inv.lines.push_back("@.value = " + em.lit(v) + ";");  // MaterialBuilder.swift:565-567
    } else if (t == "RGB") {
        plain("RGB");
        auto p = findParam(n, "value");
        float v[4] = {0, 0, 0, 0};
        if (p && p->num_numbers >= 4)
            for (int i = 0; i < 4; i++) v[i] = p->numbers[i];
        inv.lines.push_back("@.color = " + em.vec(v, 4) + ";");  // :568-575
    } else if (t == "RGBTOBW") plain("RGBToBW");
    else if (t == "INVERT") plain("ColorInvert");
    else if (t == "GAMMA") plain("Gamma");
    else if (t == "MAPPING") {  // :507-510
        inv.kernel = "Mapping";
        inv.type = "Mapping<" + enumValue("Mapping", "TYPE", paramString(n, "type", "MAPPING"), {"MAPPING"}) + ">";
    } else if (t == "NORMAL_MAP") {  // :517-523 (UV maps are ignored there too)
        inv.kernel = "NormalMap";
        inv.type = "NormalMap<" + enumValue("NormalMap", "SPACE", paramString(n, "space", "TANGENT"), {"TANGENT", "WORLD"}) +
                   ">";
    } else if (t == "TEX_IMAGE" || t == "TEX_ENVIRONMENT") {  // :387-433
        uint32_t slot, channels;
        textures.lookup(paramString(n, "filepath", ""), slot, channels);
        inv.kernel = "TexImage";
        inv.type = "TexImage<" + std::to_string(slot) + ", " +
                   enumValue("TexImage", "INTERPOLATION", paramString(n, "interpolation", "Linear"), {"LINEAR"}) + ", " +
                   enumValue("TexImage", "PROJECTION",
                             paramString(n, "projection", t == "TEX_IMAGE" ? "FLAT" : "EQUIRECTANGULAR"),
                             {"FLAT", "BOX", "EQUIRECTANGULAR", "MIRROR_BALL"}) +
                   ", kTexImage::EXTENSION_REPEAT, kTexImage::ALPHA_STRAIGHT, " +
                   enumValue("TexImage", "COLOR_SPACE", paramString(n, "colorspace", "sRGB"),
                             {"LINEAR", "SRGB", "NON_COLOR", "RAW", "XYZ", "FILMIC_LOG"}) +
                   ", kTexImage::PIXEL_FORMAT_" + (channels == 1 ? "R" : "RGBA") + ">";
    } else if (t == "TEX_SKY") {  // MaterialBuilder.swift:329-388
        const rmdsky::SkyOptions o = skyOptionsOf(n);
        uint32_t slot, channels;
        textures.lookup(skyTextureName(o.sunElevation, o.altitude, o.airDensity, o.dustDensity, o.ozoneDensity), slot,
                        channels);
        float data[10];
        rmdsky::skyNodeData(o, data);
        inv.kernel = "TexNishita";
        inv.type = "TexNishita<" + std::to_string(slot) + ">";
        for (int i = 0; i < 10; i++) inv.lines.push_back("@.data[" + std::to_string(i) + "] = " + em.lit(data[i]) + ";");
        inv.lines.push_back("@.scale = " + em.lit(o.scale) + ";");
    } else if (t == "HUE_SAT") plain("HueSaturation");
    else if (t == "BRIGHTCONTRAST") plain("BrightnessContrast");
    else if (t == "BLACKBODY") plain("Blackbody");
    else if (t == "FRESNEL") plain("Fresnel");
    else if (t == "LAYER_WEIGHT") plain("LayerWeight");
    else if (t == "EMISSION") plain("Emission");
    else if (t == "BACKGROUND") plain("Background");
    else if (t == "BSDF_PRINCIPLED") {
        inv.kernel = "BsdfPrincipled";
        inv.type = "BsdfPrincipled<kBsdfPrincipled::DISTRIBUTION_GGX, " +
                   enumValue("BsdfPrincipled", "SUBSURFACE_METHOD", paramString(n, "subsurface_method", "RANDOM_WALK"),
                             {"BURLEY", "RANDOM_WALK", "RANDOM_WALK_FIXED_RADIUS"}) +
                   ">";
    } else if (t == "BSDF_DIFFUSE") plain("BsdfDiffuse");
    else if (t == "BSDF_GLOSSY") {
        inv.kernel = "BsdfGlossy";
        inv.type = "BsdfGlossy<kBsdfGlossy::DISTRIBUTION_GGX>";
    } else if (t == "BSDF_GLASS") {
        inv.kernel = "BsdfGlass";
        inv.type = "BsdfGlass<kBsdfGlass::DISTRIBUTION_GGX>";
    } else if (t == "BSDF_TRANSPARENT") plain("BsdfTransparent");
    else if (t == "ADD_SHADER") plain("AddShader");
    else if (t == "MIX_SHADER") plain("MixShader");
    else if (t == "OUTPUT_MATERIAL") plain("OutputMaterial");
    else if (t == "OUTPUT_WORLD") plain("OutputWorld");
    else if (t == "OUTPUT_LIGHT") plain("OutputLight");
    else throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "unsupported node type '" + t + "'"};
    return inv;
}

bool isOutput(const char *t) {
    const std::string s = t ? t : "";
    return s == "OUTPUT_MATERIAL" || s == "OUTPUT_LIGHT" || s == "OUTPUT_WORLD";
}

struct MaterialCode {
    std::string body;  // function body; identical text = identical structure
    std::vector<float> literals;
    bool emissive = false;
};

// Codegen.add(material:named:), MaterialBuilder.swift:676-711 + emitNode :793-825
MaterialCode emitMaterial(const rmd_material &m, bool hoist, const TextureTable &textures) {
    std::map<std::string, const rmd_node *> nodes;
    for (int i = 0; i < m.num_nodes; i++) nodes[m.nodes[i].name ? m.nodes[i].name : ""] = &m.nodes[i];
    std::map<std::string, int> state;  // 1 pending, 2 emitted
    std::map<std::string, std::pair<std::string, std::string>> varOf;  // node -> (var, kernel)
    Emitter em{hoist, {}};
    std::string body;
    int counter = 0;
    MaterialCode out;

    std::function<void(const std::string &)> emit = [&](const std::string &key) {
        auto st = state.find(key);
        if (st != state.end()) {
            if (st->second == 2) return;
            throw CodegenError{RMD_ERROR_CODEGEN_CYCLE, "cycle detected at node '" + key + "'"};
        }
        auto it = nodes.find(key);
        if (it == nodes.end()) throw CodegenError{RMD_ERROR_INVALID_ARGUMENT, "link to unknown node '" + key + "'"};
        state[key] = 1;
        const rmd_node &node = *it->second;
        Invocation inv = makeInvocation(node, em, textures);
        const std::string var = "n" + std::to_string(counter++);
        const KernelDesc &desc = kernelTable().at(inv.kernel);
        const std::string t = node.type;
        if (t == "EMISSION") out.emissive = true;

        // provideDefaults (MaterialBuilder.swift:762-791)
        std::string defaultInput, defaultExpr;
        if (t == "TEX_IMAGE") {
            defaultInput = "Vector";
            defaultExpr = "shading.uv";
        } else if (t == "TEX_CHECKER" || t == "TEX_NOISE" || t == "TEX_ENVIRONMENT") {
            defaultInput = "Vector";
            defaultExpr = "shading.generated";
        } else if (t == "FRESNEL" || t == "LAYER_WEIGHT" || t == "BSDF_GLASS" || t == "BSDF_GLOSSY" ||
                   t == "BSDF_DIFFUSE" || t == "BSDF_PRINCIPLED" || t == "BSDF_TRANSLUCENT" ||
                   t == "BSDF_REFRACTION" || t == "BSDF_ANISOTROPIC" || t == "BSDF_VELVET" || t == "BUMP") {
            defaultInput = "Normal";
            defaultExpr = "shading.normal";
        }
        std::map<std::string, std::string> assigns;  // field -> statement (sorted like Swift's `inputs`)
        if (!defaultInput.empty()) {
            bool found = false;
            for (int i = 0; i < node.num_inputs; i++)
                if (node.inputs[i].name && defaultInput == node.inputs[i].name) found = true;
            if (!found)
                throw CodegenError{RMD_ERROR_INVALID_ARGUMENT, "node '" + key + "' lacks input '" + defaultInput + "'"};
            const std::string f = makeIdentifier(defaultInput);
            assigns[f] = assignment(var, f, desc.fields.at(f), "VECTOR", defaultExpr);
        }
        std::vector<const rmd_node_input *> sorted;
        for (int i = 0; i < node.num_inputs; i++) sorted.push_back(&node.inputs[i]);
        std::sort(sorted.begin(), sorted.end(), [](const rmd_node_input *a, const rmd_node_input *b) {
            return std::string(a->name) < std::string(b->name);
        });
        // literals are hoisted in the order the statements are finally emitted, so
        // build them in a second pass; first resolve links (emitting sources)
        struct Pending {
            std::string field;
            const rmd_node_input *in;
            bool link;
        };
        std::vector<Pending> pend;
        for (const rmd_node_input *in : sorted) {
            const std::string field = makeIdentifier(in->name);
            const bool linked = in->link_node != nullptr || in->num_links > 0;
            if (in->num_links > 1) throw CodegenError{RMD_ERROR_CODEGEN_MULTI_INPUT, "multi-input link detected"};
            if (!linked) {
                if (defaultInput == in->name || in->num_values <= 0) continue;
            } else {
                emit(in->link_node);
            }
            if (!desc.fields.count(field))
                throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED,
                                   inv.kernel + " (node '" + key + "') has no input '" + field + "'"};
            pend.push_back({field, in, linked});
        }
        std::map<std::string, const Pending *> byField;
        for (auto &p : pend) byField[p.field] = &p;
        for (auto &kv : byField) {
            const Pending &p = *kv.second;
            const std::string type = p.in->type ? p.in->type : "VALUE";
            if (p.link) {
                const auto &src = varOf.at(p.in->link_node);
                const std::string outField = makeIdentifier(p.in->link_socket ? p.in->link_socket : "");
                const KernelDesc &sd = kernelTable().at(src.second);
                if (!sd.fields.count(outField))
                    throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED,
                                       "node '" + std::string(p.in->link_node) + "' has no output '" + outField + "'"};
                if (type == "VALUE" && sd.fields.at(outField) == F2)
                    throw CodegenError{RMD_ERROR_CODEGEN_UNSUPPORTED, "VALUE() of a float2 output"};
                assigns[p.field] = assignment(var, p.field, desc.fields.at(p.field), type, src.first + "." + outField);
            } else {
                coercedKind(type);
                assigns[p.field] = assignment(var, p.field, desc.fields.at(p.field), type,
                                              em.vec(p.in->values, std::min(4, p.in->num_values)));
            }
        }
        std::string code = "    " + inv.type + " " + var + "{};\n";
        for (auto &l : inv.lines) {
            std::string s = l;
            s.replace(s.find('@'), 1, var);
            code += "    " + s + "\n";
        }
        for (auto &kv : assigns) code += "    " + kv.second + "\n";
        code += "    " + var + ".compute(ctx, shading);\n";
        body += code;
        varOf[key] = {var, inv.kernel};
        state[key] = 2;
    };
    for (auto &kv : nodes)
        if (isOutput(kv.second->type)) emit(kv.first);

    // Principled emission counts as surface emission when colour and strength are live
    for (auto &kv : varOf) {
        const rmd_node &n = *nodes[kv.first];
        if (std::string(n.type) != "BSDF_PRINCIPLED") continue;
        bool colorOn = false, strengthOn = false;
        for (int i = 0; i < n.num_inputs; i++) {
            const rmd_node_input &in = n.inputs[i];
            const std::string nm = in.name;
            const bool linked = in.link_node != nullptr;
            if (nm == "Emission")
                colorOn = linked || (in.num_values >= 3 && (in.values[0] != 0 || in.values[1] != 0 || in.values[2] != 0));
            if (nm == "Emission Strength") strengthOn = linked || (in.num_values >= 1 && in.values[0] != 0);
        }
        if (colorOn && strengthOn) out.emissive = true;
    }
    out.body = body;
    out.literals = em.literals;
    return out;
}

void emitTable(const rmd_material *mats, int n, bool hoist, const std::string &prefix, GeneratedModule &mod,
               MaterialTable &table, std::string &functions, int &groups, std::vector<bool> *emissive,
               const TextureTable &textures, const std::vector<const TextureTable *> &perMaterial) {
    std::map<std::string, int> groupOf;
    std::vector<std::string> groupBodies;
    std::vector<std::vector<std::string>> groupNames;
    std::vector<std::vector<int>> groupMembers;
    std::vector<MaterialCode> codes;
    for (int i = 0; i < n; i++) {
        codes.push_back(emitMaterial(mats[i], hoist, i < (int)perMaterial.size() ? *perMaterial[i] : textures));
        const MaterialCode &mc = codes.back();
        if (emissive) emissive->push_back(mc.emissive);
        int g;
        auto it = groupOf.find(mc.body);
        if (it == groupOf.end()) {
            g = (int)groupBodies.size();
            groupOf[mc.body] = g;
            groupBodies.push_back(mc.body);
            groupNames.push_back({});
            groupMembers.push_back({});
        } else {
            g = it->second;
        }
        groupNames[g].push_back(mats[i].name ? mats[i].name : "");
        groupMembers[g].push_back(i);
        table.group.push_back((uint32_t)g);
    }
    table.offset.assign(n, 0);
    groups = (int)groupBodies.size();
    const bool inlineFns = groups <= 8;
    for (int g = 0; g < groups; g++) {
        // literals equal in every member become constants; the rest are hoisted
        const std::vector<int> &mem = groupMembers[g];
        const size_t nl = codes[mem[0]].literals.size();
        std::vector<int> slot(nl, -1);
        int varying = 0;
        for (size_t k = 0; k < nl; k++) {
            const float v0 = codes[mem[0]].literals[k];
            bool uniform = true;
            for (int m : mem) {
                const float v = codes[m].literals[k];
                if (!(v == v0 || (v != v && v0 != v0)) || std::signbit(v) != std::signbit(v0)) uniform = false;
            }
            if (!uniform) slot[k] = varying++;
        }
        for (int m : mem) {
            table.offset[m] = (uint32_t)mod.params.size();
            for (size_t k = 0; k < nl; k++)
                if (slot[k] >= 0) mod.params.push_back(codes[m].literals[k]);
        }
        std::string body;
        const std::string &tpl = groupBodies[g];
        for (size_t i = 0; i < tpl.size();) {
            if (tpl[i] == '@' && i + 1 < tpl.size() && tpl[i + 1] == 'L') {
                const size_t end = tpl.find('@', i + 2);
                const size_t k = std::stoul(tpl.substr(i + 2, end - i - 2));
                body += slot[k] >= 0 ? "P[" + std::to_string(slot[k]) + "]" : ftoa(codes[mem[0]].literals[k]);
                i = end + 1;
            } else {
                body += tpl[i++];
            }
        }
        functions += "// materials:";
        for (size_t k = 0; k < groupNames[g].size() && k < 8; k++) functions += " " + groupNames[g][k];
        if (groupNames[g].size() > 8) functions += " ... (" + std::to_string(groupNames[g].size()) + ")";
        functions += "\n";
        functions += std::string("__device__ ") + (inlineFns ? "__forceinline__" : "__noinline__") + " void " + prefix +
                     std::to_string(g) + "(const float *__restrict__ P, const Context &ctx, ShadingContext &shading) {\n" +
                     body + "}\n\n";
    }
}

}  // namespace

std::string skyTextureName(float sunElevation, float altitude, float air, float dust, float ozone) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "@nishita:%a,%a,%a,%a,%a", (double)sunElevation, (double)altitude, (double)air,
                  (double)dust, (double)ozone);
    return buf;
}

bool parseSkyTextureName(const std::string &name, float v[5]) {
    if (name.rfind("@nishita:", 0) != 0) return false;
    const char *p = name.c_str() + 9;
    for (int i = 0; i < 5; i++) {
        char *end = nullptr;
        v[i] = std::strtof(p, &end);
        if (end == p) return false;
        p = end;
        if (i < 4) {
            if (*p != ',') return false;
            p++;
        }
    }
    return *p == 0;
}

SceneTextures sceneTextures(const rmd_scene_desc *d) {
    SceneTextures out;
    for (int i = 0; i < d->num_textures; i++) out.list.push_back(d->textures[i]);
    auto scan = [&](const rmd_material *mats, int count) {
        for (int m = 0; m < count; m++)
            for (int k = 0; k < mats[m].num_nodes; k++) {
                const rmd_node &n = mats[m].nodes[k];
                if (!n.type || std::string(n.type) != "TEX_SKY") continue;
                const rmdsky::SkyOptions o = skyOptionsOf(n);
                const std::string name =
                    skyTextureName(o.sunElevation, o.altitude, o.airDensity, o.dustDensity, o.ozoneDensity);
                if (std::find(out.generatedNames.begin(), out.generatedNames.end(), name) == out.generatedNames.end())
                    out.generatedNames.push_back(name);
            }
    };
    scan(d->surface_materials, d->num_surface_materials);
    scan(d->light_materials, d->num_light_materials);
    for (const std::string &name : out.generatedNames) {
        rmd_texture t{};
        t.name = name.c_str();
        t.width = t.height = rmdsky::kSkyTextureSize;
        t.channels = 4;
        t.format = RMD_TEXTURE_F32;
        t.data = nullptr;
        out.list.push_back(t);
    }
    return out;
}

TextureTable TextureTable::of(const rmd_texture *textures, int count) {
    TextureTable t;
    for (int i = 0; i < count; i++) {
        t.names.push_back(textures[i].name ? textures[i].name : "");
        t.channels.push_back(textures[i].channels);
    }
    return t;
}

void TextureTable::lookup(const std::string &name, uint32_t &slot, uint32_t &numChannels) const {
    for (size_t i = 0; i < names.size(); i++)
        if (names[i] == name) {
            slot = slots.empty() ? (uint32_t)i : slots[i];
            numChannels = channels[i];
            return;
        }
    slot = slots.empty() ? (uint32_t)names.size() : missingSlot;
    numChannels = 1;
}

GeneratedModule generateModule(const rmd_material *surface, int numSurface, const rmd_material *light, int numLight,
                               bool hoist, const TextureTable &textures,
                               const std::vector<const TextureTable *> &surfaceTables,
                               const std::vector<const TextureTable *> &lightTables) {
    GeneratedModule mod;
    std::string fns;
    emitTable(surface, numSurface, hoist, "s_", mod, mod.surface, fns, mod.surfaceGroups, &mod.surfaceEmissive,
              textures, surfaceTables);
    emitTable(light, numLight, hoist, "l_", mod, mod.light, fns, mod.lightGroups, nullptr, textures, lightTables);

    std::string src;
    src += "// generated by raymond_b200 codegen (shader graphs -> CUDA)\n";
    src += "#include \"device/integrator.cuh\"\n\nnamespace rmd {\n\n";
    src += fns;
    auto table = [&](const char *name, const char *prefix, int groups, int count) {
        std::string s = std::string("__device__ void ") + name +
                        "(uint32_t index, const Context &ctx, ShadingContext &shading) {\n";
        s += "    if (index >= " + std::to_string(count) + "u) return;\n";
        s += std::string("    const uint2 e = ctx.") + (prefix[0] == 's' ? "surfaceTable" : "lightTable") + "[index];\n";
        s += "    const float *P = ctx.materialParams + e.y;\n";
        s += "    switch (e.x) {\n";
        for (int g = 0; g < groups; g++)
            s += "    case " + std::to_string(g) + ": " + prefix + std::to_string(g) + "(P, ctx, shading); break;\n";
        s += "    default: break;\n    }\n}\n\n";
        return s;
    };
    src += table("shadeSurface", "s_", mod.surfaceGroups, numSurface);
    src += table("shadeLight", "l_", mod.lightGroups, numLight);
    src += "}  // namespace rmd\n";
    mod.source = src;
    return mod;
}

}  // namespace rmdhost
