/*
 * CPU oracle for the diffuse path-tracing hot path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of ProtoRay's scalar diffuse renderer, used by the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark as the
 * checker of the CUDA library. Nothing in the product links or calls it.
 *
 * Every path is re-evaluated in FP64: the random numbers are the reference's
 * 32-bit Murmur3/LCG stream converted to float exactly as the reference CPU
 * code does (round to nearest), and everything after that — camera ray,
 * closest-hit query (watertight FP64 ray/triangle test over an FP64 BVH),
 * hit point, geometric normal, shading frame, cosine-weighted bounce,
 * throughput — is computed in double precision.
 *
 * Reference functions restated (paths relative to the ProtoRay tree):
 *   sampling/random_sampler.h:44-73, math/hash.h:23-72, math/math.h:179
 *   camera/pinhole_camera.h:34-60, camera/thin_lens_camera.h:38-52
 *   math/basis3.h:63-80,128-145, math/vec3.h:409-412
 *   render/renderer_single.h:107-131, render/diffuse_integrator_single.h:41-69,
 *   render/diffuse2_integrator_single.h:41-90
 *   geometry/triangle_mesh.cpp:59-153, core/ray.h:40-76
 *   sampling/shape_sampler.h:50-74,114-124
 *   image/accum_buffer.h:130-173 (sum + weight accumulation)
 */
#ifndef PRT_ORACLE_H
#define PRT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* View record, main/render/view.h:25-33 */
typedef struct {
    float pos[3];
    float angleX, angleY, fovY, radius, focus;
} or_view;

/* Camera as the reference builds it on the host (float arithmetic). */
typedef struct {
    float origin[3];
    float U[3], V[3], N[3];
    float imageO[3], imageDx[3], imageDy[3];
    float lensRadius, focalDistance;
    int thinLens;
} or_camera;

typedef struct {
    double t;
    int primId;
    double u, v;
    int grazing;   /* 1: within 1e-5 (relative) of an edge, or a near-tie in t */
} or_hit;

typedef struct or_scene or_scene;

/* RNG (sampling/random_sampler.h:44-73, math/hash.h:23-72) */
uint32_t or_rng_seed(int pass, int pixelIndex);
uint32_t or_lcg_next(uint32_t s);
float or_unorm(uint32_t s);

/* Camera (main/render/render_window.cpp:307-325 makeCamera; camera/pinhole_camera.h, camera/thin_lens_camera.h) */
void or_camera_from_view(const or_view* view, float aspectRatio, or_camera* cam);

/* Scene: mesh + FP64 BVH.  Returns NULL on invalid input. */
or_scene* or_scene_create(const float* positions, int vertexCount, const int* indices, int triangleCount);
void or_scene_destroy(or_scene* s);
int or_scene_tri_count(const or_scene* s);

/* FP64 closest hit on (org + t dir), t in (tnear, tfar].  Returns 1 on hit. */
int or_intersect(const or_scene* s, const double org[3], const double dir[3],
                 double tnear, double tfar, or_hit* hit);
/* FP64 any hit: returns 1 if some triangle is hit with t in (tnear, tfar]. */
int or_occluded(const or_scene* s, const double org[3], const double dir[3], double tnear, double tfar);

/* Batched closest-hit over 32-byte ray records {org.xyz, tnear, dir.xyz, tfar}
 * (core/ray_cuda.cuh:23-80 layout).  Writes 16-byte hit records
 * {t, primId, u, v}; a miss has t = -1.  flags[i] = grazing flag (nullable). */
void or_intersect_rays(const or_scene* s, const float* rays, int n, float* hits, int* flags, int nthreads);
/* Batched any-hit; out[i] = t of some hit or -1 (AnyHitCuda layout). */
void or_occluded_rays(const or_scene* s, const float* rays, int n, float* out, int nthreads);

/* Primary rays of pass `pass` in float arithmetic, one 32-byte record per
 * pixel in raster order (RendererSingle::renderTile pixel loop). */
void or_primary_rays(const or_camera* cam, int width, int height, int pass, float* rays);

/* FP64 path re-evaluation.  accum: width*height*4 doubles (r,g,b,weight),
 * accumulated in pass order (pass0 .. pass0+npass-1).  albedo: per-triangle
 * albedo or NULL (constant 0.8, render/diffuse_integrator_single.h:43).
 * sky: escaped-path radiance (1 in the reference).  Returns the number of
 * closest-hit queries (the reference's ray count). */
int64_t or_render(const or_scene* s, const or_camera* cam, int width, int height,
                  int pass0, int npass, int maxDepth, const float* albedo, float sky,
                  double* accum, int nthreads);

/* As or_render; nee = 1 evaluates the next-event-estimation integrator of
 * render/diffuse2_integrator_single.h:41-90 (shadow rays count as rays). */
int64_t or_render_ex(const or_scene* s, const or_camera* cam, int width, int height,
                     int pass0, int npass, int maxDepth, const float* albedo, float sky,
                     double* accum, int nthreads, int nee);

/* As or_render_ex at the n pixels listed in pixels[] (x + y * width) of a
 * width x height frame only: out receives n * 4 doubles, the accumulation of
 * those pixels exactly as or_render_ex would leave it, and rays_out (n
 * entries, nullable) each pixel's closest-hit (and shadow) query count.
 * Lets a full-resolution frame be checked at a sample of its pixels. */
int64_t or_render_pixels(const or_scene* s, const or_camera* cam, int width, int height,
                         const int* pixels, int n, int pass0, int npass, int maxDepth,
                         const float* albedo, float sky, double* out, int64_t* rays_out,
                         int nthreads, int nee);

/* FP64 adjoint of or_render with respect to per-triangle albedo and sky.
 * dL_dsum: width*height*3 doubles, the gradient of the loss with respect to
 * the accumulated rgb sums.  d_albedo (triangleCount doubles) and d_sky are
 * overwritten. */
void or_render_backward(const or_scene* s, const or_camera* cam, int width, int height,
                        int pass0, int npass, int maxDepth, const float* albedo, float sky,
                        const double* dL_dsum, double* d_albedo, double* d_sky, int nthreads);

/* Kernels of the path exposed for known-answer tests. */
void or_cosine_sample_hemisphere(double sx, double sy, double out[3]);
void or_make_frame(const double N[3], double U[3], double V[3]);
/* Post-intersection shading of a hit on triangle primId: hit point, eps,
 * geometric normal flipped towards the ray (geometry/triangle_mesh.cpp:59-100). */
void or_post_intersect(const or_scene* s, const double org[3], const double dir[3], double t, int primId,
                       double p[3], double* eps, double Ng[3]);

#ifdef __cplusplus
}
#endif

#endif
