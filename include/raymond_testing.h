/*
 * raymond_testing.h — test hooks of the B200 path tracer.
 *
 * These entry points have no counterpart in the reference: they expose single
 * device-side building blocks (random numbers, BVH queries, one material's
 * BSDF) so that the parity tests can compare them with the CPU oracle on the
 * same inputs.  They allocate and free scratch memory per call and are not
 * meant for rendering.
 */
#ifndef RAYMOND_TESTING_H
#define RAYMOND_TESTING_H

#include "raymond.h"

#ifdef __cplusplus
extern "C" {
#endif

/* n values of PrngState.sample() for one stream: TEA(a, b) (mode 1) or
 * PCG32 with initstate a and sequence b (mode 0). */
rmd_status rmd_test_prng(uint32_t mode, uint64_t a, uint64_t b, int32_t n, float *out);

/* rays: n x 8 floats (origin.xyz, tmin, direction.xyz, tmax).  Closest hit:
 * out n x 4 = (t or -1, weight of v0, weight of v1, primitive index bits),
 * instances[n].  any != 0: occlusion query, out[4i] = 1 occluded / -1 not. */
rmd_status rmd_test_trace(const rmd_scene *scene, const float *rays, int32_t n, int32_t any, float *out,
                          uint32_t *instances);

/* The EXR writer of rmd_film_save_exr applied to a host image (width x
 * height x 3 floats) as if it were a film of one sample; needs no GPU. */
rmd_status rmd_test_exr_write(const char *path, const float *rgb, int32_t width, int32_t height, float normalized_by,
                              uint32_t compression);

/* The scene's BVH as the traversal kernels read it: max_nodes x 80-byte
 * nodes (the layout of device/traverse.cuh) and max_triangles x 12 floats
 * (v0, instance bits, v1, primitive bits, v2, 0) in leaf order.  Either
 * output may be NULL. */
rmd_status rmd_test_bvh_read(const rmd_scene *scene, void *nodes, uint64_t max_nodes, float *tris,
                             uint64_t max_triangles);

/* Shade n records with surface material `material` and evaluate / sample its
 * BSDF as handleIntersections does.  Record: position, normal, trueNormal,
 * generated, uv, wo, wi, rnd (float3 each), rayFlags, tangent tu (3; the bitangent
 * is normal x tu) = 28 floats.
 * Output: emission(3), eval(3), eval pdf, sampled wi(3), sampled weight(3),
 * sampled pdf, sampled flags, alpha (16 floats). */
rmd_status rmd_test_material_eval(const rmd_scene *scene, int32_t material, const float *records, int32_t n,
                                  float *out);

/* The CUDA source the material JIT generates for a scene description
 * (hoist != 0: literals hoisted into per-material parameter blocks).  Writes
 * at most buflen bytes (NUL-terminated) and the full size to *needed.  Needs
 * no GPU. */
rmd_status rmd_test_generate_source(const rmd_scene_desc *desc, int32_t hoist, char *buf, int64_t buflen,
                                    int64_t *needed);

/* Generate and NVRTC-compile the material module of a scene description for
 * sm_100a without loading it (no GPU needed).  The compile log (or the error)
 * goes to `log`, the cubin size to *cubin_bytes. */
rmd_status rmd_test_jit_compile(const rmd_scene_desc *desc, int32_t hoist, char *log, int64_t loglen,
                                int64_t *cubin_bytes);

/* Path-guiding network test hooks (no counterpart in the reference).
 * Forward pass of explicit features (n x 7) with FP32 parameters, raw
 * outputs (n x 48). */
rmd_status rmd_test_guide_forward(const float *params, const float *features, int32_t n, float *out);
/* Gradient of the mean training loss over n records of 12 floats (features
 * 7, direction 3, BSDF pdf, target), and the loss. */
rmd_status rmd_test_guide_gradient(const float *params, const float *records, int32_t n, float *grad, float *loss);
/* Packed mixture of one output vector (48): a direction and its pdf per row
 * of u (n x 3, into dirs_pdf n x 4), and the pdf at m query directions. */
/* One Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected for `step` >= 1)
 * of the guide's parameters on a given gradient and moments: the new FP32
 * parameters and moments, and the BF16 weight copy the tensor cores read
 * (rmd_guide_param_count() floats each; weights only in bf16_out). */
rmd_status rmd_test_guide_adam(const float *params, const float *grad, const float *m, const float *v, int32_t step,
                               float lr, float *params_out, float *m_out, float *v_out, uint16_t *bf16_out);
rmd_status rmd_test_guide_mixture(const float *outputs, const float *u, int32_t n, float *dirs_pdf,
                                  const float *queries, int32_t m, float *pdfs);

#ifdef __cplusplus
}
#endif

#endif
