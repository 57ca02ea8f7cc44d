// Oracle (test infrastructure only): the reference's Cycles node library
// (raymond/device/nodes/nodes.hpp) and the semantics of its shader JIT
// (raymond/host/scene/MaterialBuilder.swift:32-826), executed by an
// interpreter instead of generated code.  The interpreter keeps the JIT's
// observable rules: nodes are emitted by a depth-first walk from every
// output node (nodes visited in sorted-name order, inputs in sorted-name
// order), cycles and multi-input links are errors, unlinked inputs take
// their literal, a few inputs take dynamic defaults (provideDefaults), and
// links pass through the VECTOR/RGBA/VALUE/SHADER coercions.
#pragma once
#include <cstddef>
#include <map>
#include <memory>
#include <string>
#include <vector>
#include "../../include/raymond.h"
#include "scene.h"

namespace orc {

enum Kind { K_F1 = 1, K_F2 = 2, K_F3 = 3, K_F4 = 4, K_SHADER = 5 };

struct FieldDesc {
    std::string name;
    Kind kind;
    size_t offset;
};

struct NodeImpl {
    virtual ~NodeImpl() = default;
    virtual void compute(const SceneData &ctx, ShadingContext &shading) = 0;
    virtual std::unique_ptr<NodeImpl> clone() const = 0;
    virtual void copy_from(const NodeImpl &other) = 0;
    virtual void *base() = 0;
    virtual const std::vector<FieldDesc> &fields() const = 0;
    const FieldDesc *field(const std::string &name) const {
        for (auto &f : fields())
            if (f.name == name) return &f;
        return nullptr;
    }
};

// Rayjay/Swift identifier rule, MaterialBuilder.swift:19-30,41-43
std::string makeIdentifier(const std::string &name);

struct CodegenError {
    int status;
    std::string message;
};

// One material = one compiled node program (Codegen.add(material:)).
class MaterialProgram {
public:
    // throws CodegenError
    // textures: the scene's texture names and channel counts (an image node's
    // file selects the slot; an unknown file the slot after the last)
    MaterialProgram(const rmd_material &m, const std::vector<std::string> &textureNames = {},
                    const std::vector<int> &textureChannels = {});
    // Runs the node chain (s_<material> of MaterialBuilder.swift:696-707).
    void run(const SceneData &ctx, ShadingContext &shading) const;
    bool hasSurfaceEmission() const { return hasEmission_; }
    const std::string &name() const { return name_; }

    struct Binding {
        enum Src { CONST, LINK, SHADING_UV, SHADING_GENERATED, SHADING_NORMAL } src;
        size_t dst_offset;
        Kind dst_kind;
        std::string in_type;  // coercion: VALUE/RGBA/VECTOR/SHADER
        int src_node = -1;
        size_t src_offset = 0;
        Kind src_kind = K_F1;
    };
    struct Step {
        std::unique_ptr<NodeImpl> proto;
        std::vector<Binding> links;  // CONST bindings are baked into proto
    };

private:
    std::string name_;
    std::vector<Step> steps_;
    bool hasEmission_ = false;
    uint64_t serial_ = 0;  // unique per program ever built: keys the per-thread node scratch
};

// TEX_SKY as MaterialBuilder.swift:329-349 resolves it: a Hosek-Wilkie sky
// becomes a Nishita sky of its sun direction (no disc, air 2, dust 0.5,
// ozone 1, sun at least 5 degrees up, scale 0.08); other types are
// unsupported (throws CodegenError).  Missing parameters: Blender's defaults.
struct SkyParams {
    float elevation, rotation, size, intensity, altitude, air, dust, ozone, scale;
    bool disc;
};
SkyParams skyParams(const rmd_node &n);
// the name under which the scene's texture table holds the sky texture of
// these parameters (the texture depends on elevation, altitude and densities)
std::string skyTextureKey(const SkyParams &p);

}  // namespace orc
