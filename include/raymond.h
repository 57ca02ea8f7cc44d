/*
 * raymond.h — C ABI of the B200 wavefront path tracer.
 *
 * This is the drop-in boundary for the rendering path of iRath96/raymond
 * (Swift host + Metal device library).  Every entry point below names the
 * reference interface it replaces (paths are relative to the reference
 * project).  The header is plain C99 so that a Swift host can import it
 * through a module map, and so that Python reaches it through ctypes.
 *
 * Ownership: callers own every host array they pass; the library copies
 * what it needs during the call (the reference copied into shared
 * MTLBuffers, raymond/host/scene/ShapeBuilder.swift:259-268).  Device memory
 * is owned by the library behind opaque handles and released by the
 * matching *_destroy call.
 *
 * Errors: every function returns an rmd_status.  rmd_last_error() returns a
 * thread-local description of the last failure on the calling thread
 * (the reference threw CodegenError / MeshLoaderError, or returned nil,
 * raymond/host/scene/MaterialBuilder.swift:45-51, Renderer.swift:319-330).
 *
 * Threading: calls on one handle must be serialised by the caller (the
 * reference kept one frame in flight, Renderer.swift:285); distinct
 * renderers are independent.
 */
#ifndef RAYMOND_H
#define RAYMOND_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Alignment of a struct member.  The host-facing records below keep the
 * memory layout of the reference's DEVICE_STRUCTs (raymond/bridge/ *.hpp) as
 * Swift and Metal see them: simd float3 takes 16 bytes with 16-byte
 * alignment (its 4th float is padding), float2 8 with 8, float4x4 64 and
 * float3x3 / float3x4 48 with 16, bool one byte. */
#if defined(__cplusplus)
#define RMD_ALIGN(n) alignas(n)
#else
#define RMD_ALIGN(n) _Alignas(n)
#endif

/* ------------------------------------------------------------------ status */

typedef int32_t rmd_status;
#define RMD_OK                         0
#define RMD_ERROR_INVALID_ARGUMENT     1
#define RMD_ERROR_CUDA                 2
#define RMD_ERROR_NVRTC                3
/* Codegen errors, MaterialBuilder.swift:45-51 */
#define RMD_ERROR_CODEGEN_CYCLE        4
#define RMD_ERROR_CODEGEN_MULTI_INPUT  5
#define RMD_ERROR_CODEGEN_UNSUPPORTED  6
#define RMD_ERROR_OUT_OF_MEMORY        7
/* a device queue was too small for the work pushed into it */
#define RMD_ERROR_QUEUE_OVERFLOW       8
/* a bounded device-side wait ran out */
#define RMD_ERROR_WATCHDOG             9
#define RMD_ERROR_NO_DEVICE           10

/* Thread-local message for the last failing call on this thread. */
const char *rmd_last_error(void);
/* Library version string. */
const char *rmd_version(void);

/* --------------------------------------------------------------- constants */

/* RayFlags, raymond/bridge/Ray.hpp:6-15 (entity visibility uses the same bits) */
#define RMD_RAY_CAMERA        (1u << 0)
#define RMD_RAY_REFLECTION    (1u << 1)
#define RMD_RAY_TRANSMISSION  (1u << 2)
#define RMD_RAY_SHADOW        (1u << 3)
#define RMD_RAY_VOLUME        (1u << 4)
#define RMD_RAY_DIFFUSE       (1u << 5)
#define RMD_RAY_GLOSSY        (1u << 6)
#define RMD_RAY_SINGULAR      (1u << 7)

/* SamplingMode, raymond/bridge/Uniforms.hpp:5-9 */
#define RMD_SAMPLING_BSDF  0
#define RMD_SAMPLING_NEE   1
#define RMD_SAMPLING_MIS   2

/* Tonemapping, raymond/bridge/Uniforms.hpp:11-15 */
#define RMD_TONEMAP_LINEAR 0
#define RMD_TONEMAP_HABLE  1
#define RMD_TONEMAP_ACES   2

/* Random number generators.  RMD_RNG_TEA is the reference's PrngState
 * (raymond/device/PrngState.metal:20-93) seeded per frame exactly as
 * generateRays does (kernels/shading/generate.metal:88-94).  RMD_RNG_PCG32
 * keeps the PrngState interface with a PCG32 body: one stream per path,
 * sequence = sampleIndex * width * height + y * width + x. */
#define RMD_RNG_PCG32 0
#define RMD_RNG_TEA   1

/* ---------------------------------------------------------- shader graphs */
/*
 * A material is the node graph the reference's Blender exporter writes
 * (scripts/blender_exporter/raymond_blender/materials.py:273-547) and the
 * Rayjay package parsed into Material/Node/Kernel types before
 * MaterialBuilder.swift turned it into Metal (Codegen.add(material:),
 * MaterialBuilder.swift:676-711).  Here the host passes it as plain structs.
 */

#define RMD_PARAM_STRING  0
#define RMD_PARAM_NUMBER  1
#define RMD_PARAM_BOOL    2
#define RMD_PARAM_NUMBERS 3   /* flat float list, e.g. ColorRamp elements as
                                 [pos, r, g, b, a, pos, r, g, b, a, ...] */

typedef struct rmd_node_param {
    const char *key;           /* e.g. "noise_dimensions", "blend_type" */
    int32_t kind;              /* RMD_PARAM_* */
    const char *string_value;  /* RMD_PARAM_STRING */
    double number_value;       /* RMD_PARAM_NUMBER / RMD_PARAM_BOOL */
    const float *numbers;      /* RMD_PARAM_NUMBERS */
    int32_t num_numbers;
} rmd_node_param;

typedef struct rmd_node_input {
    const char *name;          /* Blender socket identifier, e.g. "Base Color" */
    const char *type;          /* "VALUE", "RGBA", "VECTOR", "SHADER", ... */
    int32_t num_values;        /* 0: no literal; 1: scalar; 2..4: vector */
    float values[4];
    const char *link_node;     /* NULL when unlinked */
    const char *link_socket;   /* output socket identifier of link_node */
    int32_t num_links;         /* >1 reproduces CodegenError.multiInputDetected */
} rmd_node_input;

typedef struct rmd_node {
    const char *name;          /* unique within the material */
    const char *type;          /* Blender node type, e.g. "BSDF_PRINCIPLED" */
    int32_t num_inputs;
    const rmd_node_input *inputs;
    int32_t num_params;
    const rmd_node_param *params;
} rmd_node;

typedef struct rmd_material {
    const char *name;
    int32_t num_nodes;
    const rmd_node *nodes;
} rmd_material;

/* ---------------------------------------------------------------- geometry */

/* One shape = one PLY mesh of the reference (ShapeBuilder.swift:259-298). */
typedef struct rmd_shape {
    uint32_t num_vertices;
    uint32_t num_faces;
    const float *vertices;     /* 3 floats per vertex (packed float3, bridge/common.hpp:56) */
    const float *normals;      /* 3 floats per vertex */
    const float *texcoords;    /* 2 floats per vertex */
    const uint32_t *indices;   /* 3 per face (IndexTriplet, bridge/common.hpp:66-75) */
    const uint16_t *materials; /* per face: index into rmd_scene_desc.surface_materials */
} rmd_shape;

/* One entity = one instance of a shape (EntityBuilder.swift:66-77). */
typedef struct rmd_entity {
    uint32_t shape;
    uint32_t visibility;       /* RMD_RAY_* mask (EntityBuilder.swift:55-64) */
    float matrix[16];          /* column-major float4x4 point transform */
} rmd_entity;

/* --------------------------------------------------------------- lights */
/* The device records of raymond/bridge/lights/ *.hpp, with their layout
 * (sizes and field offsets as in Swift / Metal; checked by static_assert in
 * the library and by a C test program), as LightBuilder.build fills them
 * (LightBuilder.swift:187-223): colours already multiplied by power, spot
 * angles already as cosines.  A float3 field is float[4]; its [3] is
 * padding and ignored. */

typedef struct rmd_light_info {             /* bridge/lights/LightInfo.hpp:5-9, 4 bytes */
    uint16_t shader_index;                  /* index into light_materials */
    uint8_t casts_shadows;                  /* bool */
    uint8_t uses_mis;                       /* bool; the reference forces 0 (LightBuilder.swift:45) */
} rmd_light_info;

typedef struct rmd_area_light {             /* bridge/lights/AreaLight.hpp:6-16, 96 bytes */
    rmd_light_info info;                    /* offset 0 */
    RMD_ALIGN(16) float transform[12];      /* offset 16: float3x4, three float4 columns =
                                               the first three rows of the world matrix */
    RMD_ALIGN(16) float color[4];           /* offset 64: float3 */
    uint8_t is_circular;                    /* offset 80: bool */
} rmd_area_light;

typedef struct rmd_point_light {            /* bridge/lights/PointLight.hpp:6-16, 64 bytes */
    rmd_light_info info;                    /* offset 0 */
    RMD_ALIGN(16) float location[4];        /* offset 16: float3 */
    float radius;                           /* offset 32 */
    RMD_ALIGN(16) float color[4];           /* offset 48: float3 */
} rmd_point_light;

typedef struct rmd_sun_light {              /* bridge/lights/SunLight.hpp:6-16, 64 bytes */
    rmd_light_info info;                    /* offset 0 */
    RMD_ALIGN(16) float direction[4];       /* offset 16: float3 */
    float cos_angle;                        /* offset 32 */
    RMD_ALIGN(16) float color[4];           /* offset 48: float3 */
} rmd_sun_light;

typedef struct rmd_spot_light {             /* bridge/lights/SpotLight.hpp:6-19, 96 bytes */
    rmd_light_info info;                    /* offset 0 */
    RMD_ALIGN(16) float location[4];        /* offset 16: float3 */
    RMD_ALIGN(16) float direction[4];       /* offset 32: float3 */
    float radius;                           /* offset 48 */
    RMD_ALIGN(16) float color[4];           /* offset 64: float3 */
    float spot_size;                        /* offset 80: cos(size / 2) */
    float spot_blend;                       /* offset 84: (1 - spot_size) * blend */
} rmd_spot_light;

/* ---------------------------------------------------------------- camera */

typedef struct rmd_camera {                 /* bridge/Camera.hpp:5-11, 96 bytes */
    RMD_ALIGN(16) float transform[16];      /* offset 0: float4x4, column-major camera-to-world */
    float near_clip;                        /* offset 64 */
    float far_clip;                         /* offset 68 */
    float focal_length;                     /* offset 72: lens_mm / (sensor_width / 2), SceneLoader.swift:135-136 */
    RMD_ALIGN(8) float shift[2];            /* offset 80: float2 */
} rmd_camera;

/* ------------------------------------------------------ instance records */

/* bridge/PerInstanceData.hpp:6-20 (192 bytes): what EntityBuilder computes
 * per entity (EntityBuilder.swift:66-146) and the device reads in
 * ShadingContext::build.  rmd_scene_instance_data returns the library's
 * records in this layout. */
typedef struct rmd_per_instance_data {
    uint32_t vertex_offset;                 /* offset 0: first vertex of the shape in the scene's vertex array */
    uint32_t face_offset;                   /* offset 4: first face of the shape */
    uint32_t light_face_offset;             /* offset 8: the shape light's face CDF (shape lights only) */
    uint32_t light_face_count;              /* offset 12 */
    uint32_t light_index;                   /* offset 16: its shape light among the scene's shape
                                               lights (LightBuilder.swift:169-177), or 0xffffffff */
    RMD_ALIGN(16) float bounds_min[4];      /* offset 32: float3, object space */
    RMD_ALIGN(16) float bounds_size[4];     /* offset 48: float3 */
    RMD_ALIGN(16) float point_transform[16]; /* offset 64: float4x4, column-major */
    RMD_ALIGN(16) float normal_transform[12]; /* offset 128: float3x3, three float3 columns */
    uint8_t visibility;                     /* offset 176: RayFlags (RMD_RAY_*) */
} rmd_per_instance_data;

/* --------------------------------------------------------------- uniforms */

/* OutputChannel and RussianRoulette, raymond/bridge/Uniforms.hpp:17-26 */
#define RMD_OUTPUT_IMAGE 0
#define RMD_RR_NONE 0
#define RMD_RR_THROUGHPUT 1

/* bridge/Uniforms.hpp:29-47 (64 bytes): the per-frame settings the
 * reference's host writes and its kernels read (Renderer.swift:331-349,
 * 438-443).  rmd_render_frame and rmd_film_normalize take them. */
typedef struct rmd_uniforms {
    uint32_t num_lens_surfaces;             /* offset 0: must be 0 (pinhole camera) */
    uint32_t frame_index;                   /* offset 4: frames accumulated before this one */
    uint32_t random_seed;                   /* offset 8: PrngState seed of the frame (>= 1) */
    uint8_t accumulate;                     /* offset 12: bool; 0 clears the film first */
    uint8_t lens_spectral;                  /* offset 13: bool, lens only (ignored) */
    float sensor_scale;                     /* offset 16: lens only (ignored) */
    float camera_scale;                     /* offset 20: lens only (ignored) */
    float focus;                            /* offset 24: lens only (ignored) */
    float exposure;                         /* offset 28 */
    int32_t stop_index;                     /* offset 32: lens only (ignored) */
    float relative_stop;                    /* offset 36: lens only (ignored) */
    int32_t num_aperture_blades;            /* offset 40: lens only (ignored) */
    uint32_t sampling_mode;                 /* offset 44: RMD_SAMPLING_* */
    uint32_t tonemapping;                   /* offset 48: RMD_TONEMAP_* */
    uint32_t rr;                            /* offset 52: RMD_RR_* (the device code reads neither rr */
    int32_t rr_depth;                       /* offset 56:  nor rr_depth; ignored) */
    uint32_t output_channel;                /* offset 60: RMD_OUTPUT_IMAGE */
} rmd_uniforms;

/* ----------------------------------------------------------------- scene */

#define RMD_TEXTURE_U8 0u  /* unsigned bytes, value / 255 */
#define RMD_TEXTURE_U16 1u /* unsigned shorts, value / 65535 */
#define RMD_TEXTURE_F32 2u /* floats */

/* The image of an image or environment texture node, found by the node's
 * `filepath` parameter (MaterialBuilder.registerTexture,
 * MaterialBuilder.swift:719-735, where MTKTextureLoader reads the file).
 * Rows from the top of the image, channels interleaved: 1 (a single-channel
 * texture, sampled as (r, 0, 0, 1)), 3 (RGB, alpha 1) or 4 (RGBA).  A node
 * whose file is not among the textures reads a 1 x 1 zero texture, as the
 * reference does when a file fails to load (:224-234). */
typedef struct rmd_texture {
    const char *name;
    uint32_t width, height, channels, format;
    const void *data;
} rmd_texture;

typedef struct rmd_scene_desc {
    int32_t num_surface_materials;          /* shadeSurface table */
    const rmd_material *surface_materials;
    int32_t num_light_materials;            /* shadeLight table */
    const rmd_material *light_materials;

    int32_t num_shapes;
    const rmd_shape *shapes;
    int32_t num_entities;
    const rmd_entity *entities;

    uint16_t world_shader;                  /* light material of the world (LightBuilder.swift:247-248) */
    int32_t envmap_exponent;                /* envmap resolution 2^e; the reference uses 11 */

    int32_t num_area_lights;
    const rmd_area_light *area_lights;
    int32_t num_point_lights;
    const rmd_point_light *point_lights;
    int32_t num_sun_lights;
    const rmd_sun_light *sun_lights;
    int32_t num_spot_lights;
    const rmd_spot_light *spot_lights;

    rmd_camera camera;

    int32_t num_textures;
    const rmd_texture *textures;
} rmd_scene_desc;

/* -------------------------------------------------------------- renderer */

typedef struct rmd_render_settings {
    uint32_t spp;              /* samples per pixel added by this call (one
                                  reference frame per sample) */
    uint32_t max_depth;        /* shade passes per path (Renderer.swift:290) */
    uint32_t sampling_mode;    /* RMD_SAMPLING_* (Uniforms.samplingMode) */
    uint32_t rng;              /* RMD_RNG_* */
    uint64_t seed;             /* PCG32 initstate */
    int64_t first_sample;      /* <0: continue after the highest sample index
                                  rendered since the last reset; >=0: start at
                                  this sample index */
    uint32_t film_fp64;        /* accumulate the film in double precision */
    uint32_t reserved;
} rmd_render_settings;

typedef struct rmd_stats {
    uint64_t paths;            /* camera samples traced to termination */
    uint64_t segments;         /* closest-hit rays that hit a surface and were shaded */
    uint64_t shadow_rays;      /* shadow rays traced */
    uint64_t iterations;       /* wavefront iterations of the last render */
    double   ms_total;         /* device time of the last render */
    double   ms_trace;         /* closest-hit traversal */
    double   ms_shade;         /* shading, NEE and BSDF sampling */
    double   ms_shadow;        /* any-hit traversal + shadow resolve */
    double   ms_film;          /* film accumulation and path regeneration */
    uint32_t pool_size;        /* path slots in flight */
    uint32_t errors;           /* device error flags (queue overflow, watchdog) */
    uint64_t rays;             /* closest-hit rays traced (segments + misses) */
    double   ms_guide;         /* guide inference and training (0 without guiding) */
    double   ms_guide_train;   /* of which training (gradient and Adam steps) */
    uint64_t invalid_samples;  /* light and BSDF samples dropped for a non-finite weight (the
                                  reference drops them without a count) */
} rmd_stats;

/* ------------------------------------------------ acceleration structures */

#define RMD_BVH_HOST 0u /* binned SAH on the host (OpenMP), the default */
#define RMD_BVH_GPU 1u  /* on the device: Morton order, locally-ordered clustering, 8-wide collapse */

typedef struct rmd_bvh_stats {
    uint32_t builder;  /* RMD_BVH_* that built the scene's BVH */
    uint32_t levels;   /* levels of the 8-wide tree */
    uint64_t nodes;    /* 8-wide nodes */
    double build_ms;   /* host wall-clock time of the build, uploads included */
    double sah_cost;   /* surface-area cost relative to the root: per node the area of its box
                          (its parent's quantised slot; 1 for the root), plus per leaf the area of
                          its slot times its triangles */
    uint32_t cluster_iterations; /* RMD_BVH_GPU: clustering passes until one cluster was left */
    uint32_t reserved;
} rmd_bvh_stats;

typedef struct rmd_context rmd_context;
typedef struct rmd_scene rmd_scene;
typedef struct rmd_renderer rmd_renderer;

/* Device selection and stream.  Replaces MTLCreateSystemDefaultDevice and
 * the command queue of Renderer.init (Renderer.swift:319-325). */
rmd_status rmd_context_create(int32_t device, rmd_context **out);
void rmd_context_destroy(rmd_context *ctx);

/* Upload geometry, build the BVH, JIT-compile every material through NVRTC,
 * build shape lights and the environment importance map.  Replaces
 * SceneLoader.loadScene (SceneLoader.swift:46-143) with its
 * MaterialBuilder / ShapeBuilder / EntityBuilder / LightBuilder stages. */
rmd_status rmd_scene_create(rmd_context *ctx, const rmd_scene_desc *desc, rmd_scene **out);
void rmd_scene_destroy(rmd_scene *scene);
/* Builder of the acceleration structure of the scenes this context creates
 * from now on (RMD_BVH_HOST or RMD_BVH_GPU).  Replaces the choice of Metal's
 * acceleration-structure builder in ShapeBuilder.swift:7-94,302-319 and
 * EntityBuilder.swift:148-165 (the reference has one builder, Apple's).  Both
 * produce the same 8-wide node format, so rendering is unchanged. */
rmd_status rmd_context_set_bvh_builder(rmd_context *ctx, uint32_t builder);
/* Builder, build time, size and surface-area cost of a scene's BVH (the cost
 * is computed on the host on the first call).  No counterpart in the
 * reference, whose acceleration structures are opaque. */
rmd_status rmd_scene_bvh_stats(rmd_scene *scene, rmd_bvh_stats *out);
/* The per-instance records the library computed (EntityBuilder.build,
 * EntityBuilder.swift:79-127), one per entity in entity order, in the
 * bridge layout.  Writes min(capacity, entities) records; *count receives the
 * number of entities. */
rmd_status rmd_scene_instance_data(const rmd_scene *scene, rmd_per_instance_data *out, int32_t capacity,
                                   int32_t *count);
/* Number of triangles after instancing, and BVH nodes. */
rmd_status rmd_scene_info(const rmd_scene *scene, uint64_t *triangles, uint64_t *bvh_nodes,
                          int32_t *num_lights_total);

/* Renderer.init (Renderer.swift:319-390). pool_size 0 = autotuned. */
rmd_status rmd_renderer_create(rmd_scene *scene, uint32_t width, uint32_t height,
                               uint32_t pool_size, rmd_renderer **out);
void rmd_renderer_destroy(rmd_renderer *r);
/* Renderer.setSize (Renderer.swift:757-798); clears the film. */
rmd_status rmd_renderer_set_size(rmd_renderer *r, uint32_t width, uint32_t height);
/* Renderer.reset (Renderer.swift:729-732). */
rmd_status rmd_renderer_reset(rmd_renderer *r);
/* Renderer.updateProjection / scene.camera (Renderer.swift:749-755); resets. */
rmd_status rmd_renderer_set_camera(rmd_renderer *r, const rmd_camera *camera);

/* Renderer.execute(in:) (Renderer.swift:480-696), settings->spp times:
 * raygen, maxDepth shade passes with NEE shadow rays, film accumulation.
 * Runs on the renderer's stream; returns when the work is enqueued and
 * finished (blocking), with device error flags checked. */
rmd_status rmd_render(rmd_renderer *r, const rmd_render_settings *settings);

/* One frame of Renderer.execute(in:) (Renderer.swift:480-696) driven by the
 * reference's Uniforms: the reference's TEA generator seeded with
 * uniforms->random_seed per ray (generate.metal:88-94), sampling mode
 * uniforms->sampling_mode, `max_depth` shade passes (the reference hard-codes
 * 8, Renderer.swift:290), and, when uniforms->accumulate is 0, the film
 * cleared first (generate.metal:103-106).  The host advances frame_index and
 * random_seed between frames as updateState does (Renderer.swift:438-443).
 * Lens cameras (num_lens_surfaces > 0) are rejected. */
rmd_status rmd_render_frame(rmd_renderer *r, const rmd_uniforms *uniforms, uint32_t max_depth);
/* normalizeImage (kernels/utils/normalizeImage.metal:39-59) with the
 * reference's Uniforms: per pixel exposure * film, divided by frame_index + 1
 * when accumulate is set, then the Hable or ACES tonemap; W*H*4 floats
 * (RGB and alpha 1), row-major from the top-left pixel. */
rmd_status rmd_film_normalize(rmd_renderer *r, const rmd_uniforms *uniforms, float *rgba);

/* Copy the film to host memory: W*H*3 floats, row-major from the top-left
 * pixel.  With normalize != 0 the normalizeImage kernel math is applied
 * (exposure * L / samples, then the tonemap; normalizeImage.metal:39-59). */
rmd_status rmd_film_read(rmd_renderer *r, float *rgb, int32_t normalize, uint32_t tonemapping,
                         float exposure);
#define RMD_EXR_AUTO 0u /* ZIP, or none when width and height are both below 16 (the reference's choice) */
#define RMD_EXR_NONE 1u
#define RMD_EXR_ZIP 2u
/* MTLTexture.saveEXR(at:normalizedBy:) (utils/Metal.swift:75-126, called by
 * Renderer.saveFrame, Renderer.swift:804-807): writes the film to an OpenEXR
 * file of four 32-bit float channels stored A, B, G, R (alpha 1), each colour
 * the accumulated film times normalized_by (<= 0: 1 / samples, the mean).
 * The reference wrote it with tinyexr's SaveEXR; this writer is the
 * library's own (zlib for ZIP). */
rmd_status rmd_film_save_exr(rmd_renderer *r, const char *path, float normalized_by, uint32_t compression);
/* The double-precision film (settings.film_fp64), raw sums. */
rmd_status rmd_film_read_f64(rmd_renderer *r, double *rgb);
/* Samples accumulated in the film since the last reset, whatever their
 * indices (frameIndex of Renderer.swift:288); what normalisation divides by. */
rmd_status rmd_film_samples(const rmd_renderer *r, uint64_t *samples);
/* Device address of the renderer's film: width * height float4 (RGB radiance
 * sums and a path count per pixel), row-major from the top-left pixel, on the
 * renderer's device; valid until the renderer is resized or destroyed.  For
 * collectives that sum the films of renderers on several GPUs (one image's
 * samples split over ranks) without a round trip through host memory.  The
 * film is complete when rmd_render returns; a writer on another stream must
 * finish before the next call on this renderer.  No counterpart in the
 * reference (one GPU, Renderer.swift:285). */
rmd_status rmd_film_device(rmd_renderer *r, float **film, uint64_t *num_pixels);
/* Set the sample count of the film (what rmd_film_read divides by) after
 * other renderers' films were summed into it. */
rmd_status rmd_film_set_samples(rmd_renderer *r, uint64_t samples);

/* Launch choices picked by rmd_renderer_autotune. */
typedef struct rmd_tune_result {
    uint32_t shade_min_blocks;     /* register budget of the shading kernel (blocks of 128 per SM) */
    uint32_t trace_blocks_per_sm;  /* persistent traversal blocks per SM */
    uint32_t pool_size;            /* paths in flight (queue sizes) */
    uint32_t calibration_spp;
    double ms_default;             /* calibration render with the previous choices */
    double ms_best;                /* with the chosen ones */
} rmd_tune_result;

/* Autotuner.  No counterpart in the reference, which dispatched fixed
 * 64-thread threadgroups (Renderer.swift:471-474, 616-619).  Times short
 * calibration renders of this renderer's scene and size with `settings`
 * (depth, sampling mode, RNG) and keeps the fastest shading-kernel register
 * budget (1 to 16 blocks of 128 per SM), traversal grid and path-pool size
 * (half, twice or four times the current pool, memory permitting); the
 * calibration covers several generations of the largest pool tried, at most
 * settings->spp samples.  Compiles the shading-kernel variants it needs
 * (NVRTC, cached on disk): with the guide's code when guiding is switched on
 * for this renderer, without it otherwise.  Clears the film. */
rmd_status rmd_renderer_autotune(rmd_renderer *r, const rmd_render_settings *settings, rmd_tune_result *out);
/* Apply launch choices found earlier (by rmd_renderer_autotune, possibly in
 * another process): shade_min_blocks 1..16, trace_blocks_per_sm 1..32,
 * pool_size 0 (keep) or >= 1024.  The timing fields are ignored.  Results do
 * not depend on these choices. */
rmd_status rmd_renderer_set_tuning(rmd_renderer *r, const rmd_tune_result *tuning);

/* Per-stage device timings and counters of the last rmd_render
 * (RendererCounters, Renderer.swift:13-268). */
rmd_status rmd_renderer_stats(const rmd_renderer *r, rmd_stats *out);

/* ----------------------------------------------------- learned path guiding */
/* No counterpart in the reference.  A small MLP (160 one-blob inputs from
 * position, normal and view; 3 hidden layers of 64; BF16 weights, FP32
 * accumulation, on the tensor cores) maps each shading point to a mixture of
 * 8 von Mises-Fisher lobes and a selection probability.  Directions are drawn
 * from the BSDF or the mixture by one-sample MIS, so the estimator stays
 * unbiased whatever the network says.  The network trains online with Adam
 * on the radiance the tracer itself gathers: each path contributes one
 * sample (a vertex chosen uniformly among its eligible ones, with the
 * radiance that arrived through its sampled direction) and every light
 * sample one more; the samples with a nonzero target go to a replay ring from
 * which each step draws its records. */
typedef struct rmd_guide_settings {
    uint32_t sampling;       /* 1: sample directions from the guide as well as the BSDF */
    uint32_t training;       /* 1: collect records and take Adam steps during rmd_render */
    uint32_t batch_size;     /* tracer samples (paths) per Adam step; 0 = 1 << 20 */
    float learning_rate;     /* 0 = 1e-3 */
    uint32_t reset;          /* 1: re-initialise the network from `seed` */
    uint32_t seed;
    uint32_t step_records;   /* records each step trains on, drawn from the replay ring; 0 = 1 << 13 */
    uint32_t replay_records; /* ring of the latest nonzero-target records; power of two, 0 = 1 << 18 */
    uint32_t steps_per_batch; /* Adam steps per `batch_size` samples; 0 = 8 */
    uint32_t skip_light_records; /* 1: train on the paths' samples only, not on the light samples */
    uint32_t guided_depth;   /* guide the vertices of path depth below this; 0 = all */
} rmd_guide_settings;

typedef struct rmd_guide_stats {
    uint64_t steps;          /* Adam steps taken */
    uint64_t samples;        /* training samples consumed (one per path with an eligible vertex) */
    uint64_t records;        /* records with a nonzero target written to the replay ring so far */
    float last_loss;         /* mean loss of the last step (normalised targets) */
    float reserved;
} rmd_guide_stats;

/* A renderer that neither samples from nor trains the guide runs a shading
 * kernel compiled without the guide's code; the first rmd_render after
 * guiding is switched on takes (and, once per scene and register budget,
 * compiles with NVRTC, cached on disk) the kernel with it, and the plain one
 * again after both are switched off. */
rmd_status rmd_renderer_set_guide(rmd_renderer *r, const rmd_guide_settings *settings);
rmd_status rmd_renderer_guide_stats(const rmd_renderer *r, rmd_guide_stats *out);
/* Read (write = 0) or replace (write = 1) the network's FP32 parameters:
 * rmd_guide_param_count() floats, layers W1 [64][160], b1, W2 [64][64], b2,
 * W3 [64][64], b3, W4 [48][64], b4 (row-major, output-major). */
int32_t rmd_guide_param_count(void);
rmd_status rmd_renderer_guide_params(rmd_renderer *r, float *params, int32_t write);

/* ------------------------------------------------------------------ batches */
/* Many scenes and views traced by one wavefront: the paths of every view share
 * one pool and every stage is one launch over all of them (each path carries
 * its view; traversal and shading use that view's scene), and the render is
 * one CUDA-graph launch whose loop the device drives (a conditional while
 * node).  Each view renders as it would alone (same camera ray, same PCG
 * stream of its own pixel index).  The scenes' materials share one NVRTC
 * module.  No counterpart in the reference (one scene, one view per frame,
 * Renderer.swift:480-696). */
typedef struct rmd_batch rmd_batch;

typedef struct rmd_batch_view {
    int32_t scene;            /* index into the batch's scene descriptions */
    uint32_t width, height;
    rmd_camera camera;
} rmd_batch_view;

#define RMD_BATCH_NO_GRAPH 1u /* flags: host-driven loop (counter checks) instead of the graph */

rmd_status rmd_batch_create(rmd_context *ctx, const rmd_scene_desc *scenes, int32_t num_scenes,
                            const rmd_batch_view *views, int32_t num_views, uint32_t pool_size, uint32_t flags,
                            rmd_batch **out);  /* pool_size <= 2^22 (0: 2^21) */
void rmd_batch_destroy(rmd_batch *batch);
rmd_status rmd_batch_reset(rmd_batch *batch);
/* settings->spp samples of every view (sample indices below 2^24) */
rmd_status rmd_batch_render(rmd_batch *batch, const rmd_render_settings *settings);
rmd_status rmd_batch_film_read(rmd_batch *batch, int32_t view, float *rgb, int32_t normalize, uint32_t tonemapping,
                               float exposure);
rmd_status rmd_batch_film_read_f64(rmd_batch *batch, int32_t view, double *rgb);
/* rmd_film_save_exr for one view of a batch */
rmd_status rmd_batch_film_save_exr(rmd_batch *batch, int32_t view, const char *path, float normalized_by,
                                   uint32_t compression);
/* aggregate over the views (per-stage times are not taken inside the graph) */
rmd_status rmd_batch_stats(const rmd_batch *batch, rmd_stats *out);
rmd_status rmd_batch_autotune(rmd_batch *batch, const rmd_render_settings *settings, rmd_tune_result *out);
/* Learned path guiding of a batch whose views all show one scene (one
 * network for the scene; rmd_guide_settings as for a renderer).  While
 * training, the batch renders with the host-driven loop, since the Adam
 * steps run between its counter checks. */
rmd_status rmd_batch_set_guide(rmd_batch *batch, const rmd_guide_settings *settings);
rmd_status rmd_batch_guide_stats(const rmd_batch *batch, rmd_guide_stats *out);

/* ----------------------------------------------------- allocation-free render */
/*
 * No counterpart in the reference.  For callers that cannot allocate GPU
 * memory at render time (a plug-in whose host application owns every device
 * allocation, a real-time loop that must not pay allocation latency, a
 * process held to a fixed memory budget): renders like rmd_render but keeps
 * its path pool, queues and counters in one fixed device array compiled into
 * the library (RMD_NOALLOC_MAX_PATHS paths, about 8.1 MB) and never calls
 * cudaMalloc, cudaFree or any other allocating routine.  The array is
 * reserved on a GPU when the first rmd_context for that GPU is created
 * (rmd_context_create looks up its device address, which loads the module
 * holding it) and stays reserved until the library is unloaded.
 *
 * film: caller-owned DEVICE memory of width * height float4 (RGB radiance
 * sums and a path count per pixel, row-major from the top-left pixel); the
 * call adds to it, so clear it first for a fresh image.  settings->first_sample
 * must be >= 0 and film_fp64 must be 0.  pool_size: paths in flight, 0 for
 * RMD_NOALLOC_MAX_PATHS; larger values are rejected with
 * RMD_ERROR_INVALID_ARGUMENT.  All calls share the array, which keeps what
 * the last call left in it (each call clears its counters and queues before
 * use): calls whose GPU work overlaps (several streams or threads) race and
 * corrupt each other, so serialise them.  The call is synchronous: it runs on
 * the scene's stream and returns when the frame is finished.  A device reset
 * invalidates every scene; a context created after it refreshes the array's
 * address.
 */
#define RMD_NOALLOC_MAX_PATHS 32768
rmd_status rmd_render_noalloc(rmd_scene *scene, const rmd_camera *camera, uint32_t width, uint32_t height,
                              const rmd_render_settings *settings, float *film, uint32_t pool_size);

#ifdef __cplusplus
}
#endif

#endif /* RAYMOND_H */
