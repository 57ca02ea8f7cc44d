/*
 * oracle.h — CPU restatement of the reference's rendering path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the parity tests,
 * smoke() and the bench's CPU-baseline leg compare the CUDA path against; the
 * product never links, loads or calls it.
 *
 * It restates iRath96/raymond's Metal device library (raymond/device/ **) and
 * the host logic around it (Renderer.execute, LightBuilder, EntityBuilder,
 * MaterialBuilder) as host C++ with OpenMP, each function citing the
 * reference file:line it follows.  Apple's closed ray-tracing intersector is
 * replaced by a CPU BVH with a watertight triangle test.
 *
 * Parity of this oracle against the reference itself is pinned by
 * oracle/ref/ (the reference's own Metal sources compiled for the host
 * through a shim) where that build is available; see the oracle tests.
 */
#ifndef RAYMOND_ORACLE_H
#define RAYMOND_ORACLE_H

#include <stdint.h>
#include "../include/raymond.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_scene oracle_scene;

typedef struct oracle_settings {
    uint32_t width, height;
    uint32_t spp;
    uint32_t max_depth;
    uint32_t sampling_mode; /* RMD_SAMPLING_* */
    uint32_t rng;           /* RMD_RNG_* */
    uint64_t seed;
    int64_t first_sample;   /* sample index of the first frame */
    int32_t threads;        /* 0 = all */
    int32_t film_fp64;      /* accumulate in double */
    /* NULL: every pixel.  Otherwise trace only these pixels (y * width + x,
     * each at most once); their paths keep the full image's PRNG streams and
     * ray indices, and the other pixels of the film stay zero. */
    const uint32_t *pixels;
    uint64_t num_pixels;
} oracle_settings;

/* returns 0 or an RMD_ERROR_* code; err receives a message */
int oracle_scene_create(const rmd_scene_desc *desc, oracle_scene **out, char *err, int errlen);
void oracle_scene_destroy(oracle_scene *s);
/* per surface material: 1 if it emits; returns the number of materials */
int oracle_surface_emissive(const oracle_scene *s, uint8_t *out);
/* replace the scene's camera (the reference's Renderer.updateProjection) */
int oracle_scene_set_camera(oracle_scene *s, const rmd_camera *camera);
int oracle_scene_info(const oracle_scene *s, uint64_t *triangles, int32_t *num_lights_total, int32_t *num_shape_lights);

/* Film sums (W*H*3, row-major from the top-left pixel) of `spp` frames;
 * stats[0..2] = paths, segments (closest-hit rays shaded), shadow rays. */
int oracle_render(oracle_scene *s, const oracle_settings *st, double *film_rgb, uint64_t *stats);

/* normalizeImage (kernels/utils/normalizeImage.metal:11-59): per pixel of a
 * W*H float4 film, exposure * rgb, divided by frame_index + 1 when
 * accumulating, then the Hable or ACES tonemap; out W*H float4 with alpha 1. */
void oracle_normalize_image(const float *film, uint32_t width, uint32_t height, float exposure, int32_t accumulate,
                            uint32_t frame_index, uint32_t tonemapping, float *out);

/* The Nishita sky restated (host/sky/sky_nishita.cpp): the width x height
 * RGBA float texture (XYZ in rgb) and the TEX_SKY node's ten data values. */
void oracle_sky_texture(int32_t width, int32_t height, float sun_elevation, float altitude, float air, float dust,
                        float ozone, float *rgba);
void oracle_sky_data(float sun_elevation, float sun_rotation, int32_t sun_disc, float sun_size, float sun_intensity,
                     float altitude, float air, float dust, float *data10);

/* Unit hooks. */
/* n values of PrngState.sample() for the stream (a, b): TEA(a, b) or PCG32(seed=a, seq=b). */
void oracle_prng(int32_t mode, uint64_t a, uint64_t b, int32_t n, float *out);
/* rays: n x 8 floats (origin, tmin, direction, tmax); out: n x 4 (t, b0, b1, as-float prim)
 * plus n instance ids; any = 1 runs the occlusion query (t = 1 occluded, -1 not); any = 2 the
 * closest-hit query without culling against the best hit so far (every box the ray enters). */
int oracle_trace(const oracle_scene *s, const float *rays, int32_t n, int32_t any, float *out, uint32_t *instances);
/* Perlin/fractal noise of utils/noise.hpp at n points (x,y,z): out[i] = fractal_noise(p, detail, roughness). */
void oracle_fractal_noise3(const float *p, int32_t n, float detail, float roughness, float *out);
/* Evaluate a surface material and its BSDF: see tests for the record layout. */
int oracle_material_eval(const oracle_scene *s, int32_t material, const float *records, int32_t n, float *out);

#ifdef __cplusplus
}
#endif
#endif
