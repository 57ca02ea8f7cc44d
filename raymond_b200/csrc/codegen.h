// Node graph -> CUDA source for the NVRTC material module.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/raymond.h"

namespace rmdhost {

struct CodegenError {
    int status;
    std::string message;
};

// Swift `camelCase` + non-word replacement of MaterialBuilder.swift:19-30,41-43.
std::string makeIdentifier(const std::string &name);

struct MaterialTable {
    // per material: (function group, offset into params)
    std::vector<uint32_t> group, offset;
};

struct GeneratedModule {
    std::string source;                  // CUDA source (includes device/integrator.cuh)
    std::vector<float> params;           // hoisted literals of all materials
    MaterialTable surface, light;
    std::vector<bool> surfaceEmissive;   // Material.hasSurfaceEmission per surface material
    int surfaceGroups = 0, lightGroups = 0;
};

// The scene's textures as the codegen sees them: image-texture nodes name a
// file, which becomes the slot of the texture of that name (channels decide
// the pixel format); an unknown file reads slot names.size(), a 1 x 1 zero
// texture (MaterialBuilder.swift:224-234, where a file that fails to load
// becomes a 1 x 1 single-channel texture).
struct TextureTable {
    std::vector<std::string> names;
    std::vector<uint32_t> channels;
    std::vector<uint32_t> slots;  // slot of each name (empty: the name's index)
    uint32_t missingSlot = 0;     // slot of unknown names (names.size() when slots is empty)
    static TextureTable of(const rmd_texture *textures, int count);
    // the slot a file name reads and that texture's channel count (1 for the zero texture)
    void lookup(const std::string &name, uint32_t &slot, uint32_t &numChannels) const;
};

// The textures a scene's materials read: the scene's own images, then one
// generated 512 x 512 sky texture per distinct Nishita sky of its TEX_SKY
// nodes (MaterialBuilder.swift:350-372, where SkyLoader fills the texture on
// the host).  A generated entry has data == NULL and a name that encodes the
// five parameters the texture depends on (skyTextureName); the library fills
// its texels on the device.  Throws CodegenError for an unsupported sky type.
struct SceneTextures {
    std::vector<rmd_texture> list;
    std::vector<std::string> generatedNames;
};
SceneTextures sceneTextures(const rmd_scene_desc *d);
// "@nishita:" and the sun elevation, altitude, air, dust and ozone densities
// as hexadecimal floats
std::string skyTextureName(float sunElevation, float altitude, float air, float dust, float ozone);
// parses a name made by skyTextureName; false for any other name
bool parseSkyTextureName(const std::string &name, float v[5]);

// Emits one function per distinct graph structure; literal inputs become
// loads from a per-material parameter block when `hoist` is set, or inline
// constants (the reference's code shape) otherwise.  Throws CodegenError.
// `surfaceTables` / `lightTables`, when given, hold one texture table per
// material (the scenes of a batch share a module but not their textures).
GeneratedModule generateModule(const rmd_material *surface, int numSurface, const rmd_material *light, int numLight,
                               bool hoist, const TextureTable &textures = TextureTable(),
                               const std::vector<const TextureTable *> &surfaceTables = {},
                               const std::vector<const TextureTable *> &lightTables = {});

}  // namespace rmdhost
