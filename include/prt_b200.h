/*
 * prt_b200 — C ABI of the B200 wavefront diffuse path tracer.
 *
 * This is the drop-in boundary for ProtoRay's GPU rendering path.  Each
 * entry point names the reference interface it replaces (paths relative to
 * the ProtoRay tree).  The signatures use only plain C types, pointers and
 * sizes; CUDA streams are passed as `void*` (a cudaStream_t, or NULL for the
 * context's own stream).
 *
 * Memory: bulk buffers given to prt_read_accum, prt_set_albedo,
 * prt_render_backward and prt_request.accum may be host or device pointers
 * (resolved with cudaPointerGetAttributes); device pointers are used in
 * place.  prt_intersect / prt_occluded take device pointers and borrow them
 * for the call only.
 *
 * Errors: every entry point returns a prt_status; prt_last_error() returns
 * the message of the last failure on that context.  The reference reports the
 * same conditions with C++ exceptions (render/device_cuda.cpp:63,92,
 * render/diffuse_renderer_cuda.cu:161-162, sys/memory_cuda.h:115-116).
 *
 * Threading: a context belongs to one host thread at a time; it owns one
 * CUDA stream on its device.
 */
#ifndef PRT_B200_H
#define PRT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PRT_OK = 0,
    PRT_EINVAL = 1,     /* invalid argument (std::invalid_argument / std::logic_error in the reference) */
    PRT_ENOMEM = 2,     /* device allocation failed (std::runtime_error, sys/memory_cuda.h:115-116) */
    PRT_ECUDA = 3,      /* CUDA runtime or launch error */
    PRT_ETIMEOUT = 4,   /* a bounded device wait expired */
    PRT_EINTERNAL = 5,  /* internal consistency check failed */
    PRT_EIO = 6,        /* file missing, truncated or with a wrong blob id (sys/blob.h:26-38) */
    PRT_ESTATE = 7      /* call out of order (e.g. render before build) */
} prt_status;

typedef struct prt_ctx prt_ctx;

/* View record of a .view file (main/render/view.h:25-33). */
typedef struct {
    float pos[3];
    float angleX, angleY, fovY;
    float radius;   /* lens radius; 0 = pinhole */
    float focus;    /* focal distance */
} prt_view;

/* Camera fields of ThinLensCameraCuda (camera/thin_lens_camera_cuda.h:23-30,
 * camera/pinhole_camera_cuda.h). lensRadius == 0 selects the pinhole camera. */
typedef struct {
    float origin[3];
    float basisU[3], basisV[3];
    float imageO[3], imageDx[3], imageDy[3];
    float lensRadius, focalDistance;
} prt_camera;

/* RayCuda (core/ray_cuda.cuh:47-80): 32 bytes. */
typedef struct {
    float org[3];
    float tnear;
    float dir[3];
    float tfar;
} prt_ray;

/* HitCuda (core/ray_cuda.cuh:23-35): 16 bytes; a miss has t < 0. */
typedef struct {
    float t;
    int primId;
    float u, v;
} prt_hit;

/* Stats of the acceleration build: the reference reports buildMs/buildMprim
 * (accel/optix/optix_intersector_stream_cuda.cpp:62-70). */
typedef struct {
    double buildMs;
    double buildMprim;
    int nodeCount;   /* 8-wide nodes */
    int levels;      /* tree depth in 8-wide levels */
} prt_build_stats;

/* Stats of one render call: ray = closest-hit queries, counted as the
 * reference counts them (render/diffuse_renderer_cuda.cu:185-186);
 * mray = rays / 1e6 / seconds of device time (render/device_cuda.cpp:99-105). */
typedef struct {
    long long rays;
    double ms;
    double mray;
    int passes;
} prt_render_stats;

/* One request of a batched render (no reference counterpart; see prt_render_batch). */
typedef struct {
    prt_ctx* scene;     /* context whose mesh and acceleration structure are rendered */
    prt_camera camera;
    int width, height;
    int spp;            /* passes, starting at pass 0 */
    int maxDepth;
    float* accum;       /* width*height*4 floats (sum r, g, b, weight), host or device, overwritten */
} prt_request;

/* Autotuned launch configuration. */
typedef struct {
    int blockSize;        /* threads per block of the bounce kernel (32..128) */
    int blocksPerSM;      /* resident blocks per SM of the persistent grid */
    int pathsPerWave;     /* queue capacity (paths in flight per wave); 0 = automatic */
    int concurrentWaves;  /* waves in flight at once, 1..4 (0 keeps the current value) */
    int primaryPackets;   /* 1: primary rays traced as warp packets (faster for fine pixels,
                             e.g. 1080p views; slower for coarse ones); 2: warp packets
                             traversed with interval bounds of the packet (one child test per
                             node; faster still where a packet's rays stay close, slower for
                             long, often missing rays); 0: per-lane (default) */
    double mray;          /* throughput measured for the winner */
} prt_tune;

/* --- context (DeviceCuda construction, render/device_cuda.cpp:31-49) --- */
int prt_create(int device, prt_ctx** out);
int prt_destroy(prt_ctx* ctx);
const char* prt_last_error(const prt_ctx* ctx);
/* Device name, as Device::getInfo (render/device.h:34). */
int prt_get_info(prt_ctx* ctx, char* buf, int len);

/* --- scene (DeviceCuda::initScene, render/device_cuda.cpp:121-168) --- */
/* Copies a triangle mesh: indices int32[triCount][3], positions float[vertCount][3]. */
int prt_load_mesh(prt_ctx* ctx, const int* indices, int triCount, const float* positions, int vertCount);
/* Loads a .mesh blob (geometry/triangle_mesh.cpp:305-320, sys/blob.h:26-38);
 * bounds (nullable) receive the stored scene box. */
int prt_load_mesh_file(prt_ctx* ctx, const char* path, float boundsLo[3], float boundsHi[3]);
/* Scene bounds (Device::getSceneBounds, render/device.h:38). */
int prt_get_scene_bounds(prt_ctx* ctx, float lo[3], float hi[3]);
/* Per-triangle diffuse albedo (NULL restores the constant 0.8 of
 * render/diffuse_integrator_single.h:43) and sky radiance (1 in the reference). */
int prt_set_albedo(prt_ctx* ctx, const float* albedo, int triCount);
int prt_set_sky(prt_ctx* ctx, float sky);

/* Integrator of prt_render (render/device_cuda.cpp:51-93 picks the CUDA
 * renderer by the same names):
 *   PRT_INTEGRATOR_DIFFUSE   diffuse path tracing (render/diffuse_integrator_single.h:41-69)
 *   PRT_INTEGRATOR_DIFFUSE2  diffuse path tracing with a shadow ray toward the sky at every
 *                            bounce and fixed 0.5 MIS weights (render/diffuse2_integrator_single.h:41-90)
 * The batched, replay/adjoint and allocation-free entry points use PRT_INTEGRATOR_DIFFUSE. */
enum { PRT_INTEGRATOR_DIFFUSE = 0, PRT_INTEGRATOR_DIFFUSE2 = 1 };
int prt_set_integrator(prt_ctx* ctx, int integrator);

/* --- acceleration structure (OptixIntersectorStreamCuda ctor, accel/optix/optix_intersector_stream_cuda.cpp:23-75) --- */
/* The context keeps the build's device scratch (about 160 bytes per triangle)
 * for its later builds and mesh builds; prt_destroy frees it. */
int prt_build_accel(prt_ctx* ctx, prt_build_stats* stats);
/* Largest leaf of the 8-wide tree, 1..3 triangles, for the next build. */
int prt_set_leaf_size(prt_ctx* ctx, int maxTrianglesPerLeaf);
/* Build quality for the next build, the reference's high-quality switch
 * (`-no-sbvh` turns it off, accel/embree/embree_intersector.cpp:24,56-57):
 * high (1, the default) builds a full SAH binary tree and groups it into
 * 8-wide nodes by the SAH dynamic program; low (0) builds the Morton LBVH and
 * opens the largest child greedily, which is several times faster to build
 * and traces slower (more, emptier nodes over a lower-quality tree). */
int prt_set_build_quality(prt_ctx* ctx, int high);

/* --- camera (DeviceCuda::initCamera, render/device_cuda.cpp:175-200) --- */
/* Builds the camera of a view for an image of width x height, as the
 * reference viewer does (main/render/render_window.cpp:307-325 with
 * camera/pinhole_camera.h:34-47). */
int prt_camera_from_view(const prt_view* view, int width, int height, prt_camera* cam);
int prt_set_camera(prt_ctx* ctx, const prt_camera* cam);

/* --- frame (DeviceCuda::initFrame / clearFrame / blitFrame, render/device_cuda.cpp:202-230) --- */
int prt_init_frame(prt_ctx* ctx, int width, int height);
int prt_clear(prt_ctx* ctx);
/* Accumulation buffer, width*height*4 floats (sum r, g, b, weight) in raster
 * order (AccumBufferCuda, image/accum_buffer_cuda.h:23-29). */
int prt_read_accum(prt_ctx* ctx, float* rgbw);
/* Gamma-2.2 BGRA8 resolve (accumBufferUpdateKernel, image/accum_buffer_cuda.cu:22-37). */
int prt_read_ldr(prt_ctx* ctx, uint32_t* bgra);

/* --- rendering (DiffuseRendererCuda::render, render/diffuse_renderer_cuda.cu:159-212) --- */
/* Renders `spp` passes of the diffuse path tracer (one path per pixel per
 * pass, up to maxDepth bounces).  accumulate = 0 clears the frame first (the
 * "Fast" renderers' overwrite, render/renderer_factory_single.cpp:58-59).
 * Passes continue from the previous call until prt_clear / prt_set_pass. */
int prt_render(prt_ctx* ctx, int spp, int maxDepth, int accumulate, prt_render_stats* stats);
/* Same work as prt_render without graph capture, with CUDA events around
 * every bounce launch: msPerDepth[d] / raysPerDepth[d] (maxDepth + 1 entries)
 * receive the device time and closest-hit queries of bounce d, summed over
 * waves.  The frame is cleared first. */
int prt_render_profile(prt_ctx* ctx, int spp, int maxDepth, double* msPerDepth, long long* raysPerDepth);
/* Pass counter of the next render (RendererSingle::pass, render/renderer_single.h:97-98). */
int prt_set_pass(prt_ctx* ctx, int pass);
int prt_get_pass(prt_ctx* ctx, int* pass);

/* --- queries (Renderer::queryRay, render/renderer_single.h:137-163;
 *     DeviceCuda::queryRay returns nothing in the reference, render/device_cuda.cpp:111-119) --- */
/* p and Ng (nullable) receive the hit point and the geometric normal facing the ray. */
int prt_query_ray(prt_ctx* ctx, const prt_ray* ray, prt_hit* hit, float p[3], float Ng[3]);

/* Primary rays of pass `pass` for every pixel of the frame (width*height ray
 * records, row-major, device pointer): the camera rays the renderer traces
 * first, with the pixel jitter and lens samples of RandomSampler.init(pass,
 * pixel) (generateRaysKernel, render/diffuse_renderer_cuda.cu:27-59;
 * RendererSingle::renderTile, render/renderer_single.h:107-124); tnear 0,
 * tfar FLT_MAX.  Needs a camera and a frame. */
int prt_primary_rays(prt_ctx* ctx, int pass, prt_ray* rays, void* stream);

/* --- intersector seam (IntersectorStreamCuda, core/intersector_stream_cuda.h:32-33) --- */
/* Closest hit for n rays (device pointers); misses get t = -1. */
int prt_intersect(prt_ctx* ctx, const prt_ray* rays, prt_hit* hits, int n, void* stream);
/* Any hit for n rays (device pointers); out[i] = t of some hit, or -1 (AnyHitCuda). */
int prt_occluded(prt_ctx* ctx, const prt_ray* rays, float* out, int n, void* stream);

/* --- differentiation (no reference counterpart) --- */
/* Path-replay adjoint of the last prt_render configuration: given
 * dL/dsum (width*height*3 floats, gradient of the loss with respect to the
 * accumulated r,g,b sums of passes [pass0, pass0+spp)), writes
 * d_albedo (triCount floats) and d_sky (1 float).  Paths are recomputed from
 * their (pixel, pass) seeds; nothing from the forward pass is stored. */
int prt_render_backward(prt_ctx* ctx, int pass0, int spp, int maxDepth, const float* dL_dsum, float* d_albedo,
                        float* d_sky);
/* Forward render of passes [pass0, pass0+spp) with the same path code as
 * prt_render_backward (for gradient checks); adds into the frame. */
int prt_render_replay(prt_ctx* ctx, int pass0, int spp, int maxDepth, prt_render_stats* stats);

/* --- batching (no reference counterpart) --- */
/* Renders n requests of uneven resolution, spp and scene in shared waves of
 * one persistent kernel per bounce (CUDA-graph captured), on ctx's device. */
int prt_render_batch(prt_ctx* ctx, const prt_request* reqs, int n, prt_render_stats* stats);

/* --- inspection --- */
/* Copies the acceleration structure to host memory: 80-byte 8-wide nodes
 * and 48-byte leaf triangles (layouts in csrc/prt_device.cuh).  Either
 * buffer may be NULL; counts (nullable) receive the sizes.  Used by the
 * structural tests. */
int prt_read_accel(prt_ctx* ctx, void* nodes, int nodeCapacity, void* tris, int triCapacity, int* nodeCount,
                   int* triCount);

/* Traversal counters of the bounce kernel since the last reset, in a build
 * compiled with -DPRT_COUNTERS=1 (the reference's RayStats nodeCount and
 * primCount, core/ray_stats.h:23-28): out[0] node visits, [1] triangle tests,
 * [2] rays, [3] warp traversal steps, [4] running lanes summed over steps,
 * [5] warp triangle-loop iterations.  n >= 6.  Other builds return PRT_ESTATE. */
int prt_read_counters(prt_ctx* ctx, long long* out, int n, int reset);

/* Failure injection for tests: the (afterCount+1)-th device or pinned-host
 * allocation made by the library from now on fails as if the GPU were out of
 * memory (the call reports PRT_ENOMEM); a negative count switches it off.
 * Process-wide. */
int prt_debug_fail_allocations(long long afterCount);

/* --- launch configuration --- */
/* Tunes the bounce kernels' launch configuration (primary rays per lane or as
 * warp packets, paths per wave = queue size, concurrent waves, resident blocks
 * per SM, block size) for the current scene, frame and camera by timing
 * renders of `spp` passes at `maxDepth`: coordinate descent from the current
 * configuration, one parameter at a time, a candidate replacing the incumbent
 * only when it is more than 0.3% faster.
 * Keeps the winner for later renders (see prt_get_tune), frees the path
 * queues the candidates grew (up to 4 chains of 64M-path waves; the next
 * render allocates what the winner needs), then clears the frame and the pass
 * counter.  The renders it times are the caller's workload, so a call costs
 * about 60 to 170 renders of it. */
int prt_autotune(prt_ctx* ctx, int spp, int maxDepth, prt_tune* best);
int prt_set_tune(prt_ctx* ctx, const prt_tune* tune);
int prt_get_tune(prt_ctx* ctx, prt_tune* tune);

/* --- rendering without device allocation (no counterpart in the reference) --- */
/* Renders passes [pass0, pass0+spp) of ctx's built scene through `cam` into
 * the caller's device buffer `accum` (width*height*4 floats: sum r, g, b,
 * weight; added to, not cleared) and returns the closest-hit query count in
 * `rays` (nullable).  It uses the context's integrator (diffuse or diffuse2),
 * sky and per-triangle albedo, like prt_render.  It allocates nothing: for
 * callers that cannot allocate device memory at render time (an application
 * that owns the GPU's memory through its own pool, or a frame loop that cannot
 * afford cudaMalloc's implicit synchronisation).  Its path queues live in one
 * fixed 40 MiB device array per GPU, so frames are limited to 524288 pixels
 * after rounding up to 8x8 tiles (larger ones return PRT_EINVAL).  `accum`
 * must be 16-byte aligned device (or managed) memory of the context's GPU,
 * else PRT_EINVAL.  All calls on a device share that array: calls that overlap
 * on the GPU race, so serialise them.  The first call in a CUDA context of a
 * device resolves the array's address there; make it before any stream
 * capture.  The caller's current device is restored on return. */
int prt_render_noalloc(prt_ctx* ctx, const prt_camera* cam, int width, int height, int pass0, int spp, int maxDepth,
                       float* accum, long long* rays);

/* Kernel launches issued by this context since creation (for accounting). */
long long prt_launch_count(prt_ctx* ctx);

/* ---- `protoray build`: OBJ -> triangle soup -> indexed .mesh ------------- */

/* One soup vertex and triangle: the reference's FatVertex / FatTriangle
 * (geometry/vertex.h:23-28, geometry/triangle.h:54-57), 32 and 100 bytes. */
typedef struct prt_soup_vertex {
    float pos[3];
    float normal[3];   /* all zero: none given */
    float tex[2];      /* all zero: none given */
} prt_soup_vertex;

typedef struct prt_soup_triangle {
    prt_soup_vertex v[3];
    int matId;
} prt_soup_triangle;

/* A parsed soup: triangles plus material names (geometry/triangle_soup.h:25-29). */
typedef struct prt_soup prt_soup;

/* Replaces ObjLoader::load (main/build/obj_loader.cpp:35-53): parses an OBJ
 * file on `threads` host threads (0: all cores).  Same grammar and results as
 * the reference: v / vn / vt / f / usemtl lines, 1-based and negative
 * (relative) indices, faces fan-triangulated, triangles with two equal
 * position indices dropped, material 0 named "" and "Default" added for faces
 * before the first usemtl.  Host code only (no device is touched).  On a
 * malformed file returns PRT_EIO and writes the reason into err. */
int prt_soup_load_obj(const char* path, int threads, prt_soup** soup, char* err, int errlen);
/* Counts of a soup; any output pointer may be NULL.  degenerateCount is the
 * number of triangles the OBJ loader dropped. */
int prt_soup_info(const prt_soup* soup, int* triCount, int* materialCount, int* degenerateCount);
const prt_soup_triangle* prt_soup_triangles(const prt_soup* soup);
const char* prt_soup_material_name(const prt_soup* soup, int i);
void prt_soup_free(prt_soup* soup);

/* Description of a mesh built by prt_build_mesh. */
typedef struct prt_mesh_info {
    int triCount;
    int vertCount;       /* unique vertices */
    int hasNormals;
    int hasTexcoords;
    int hasMaterials;    /* some matId != 0; otherwise all material ids are stored as 0 */
    float boundsLo[3];
    float boundsHi[3];
    double buildMs;      /* device time of the build kernels */
    double totalMs;      /* host soup in -> device mesh ready, copies included */
} prt_mesh_info;

/* Replaces TriangleMeshBuilder (geometry/triangle_mesh_builder.cpp:23-263) on
 * the GPU: zero normals are replaced by the triangle's cross product when
 * the soup has normals (:92-96), vertices equal in position, normal and
 * texcoord are merged (:98-112), and the vertices and triangles are put in
 * Morton order of their positions and centroids (the reference uses a median
 * split, :143-201; both are locality orders, so the mesh holds the same
 * vertices and triangles in a different order).  The mesh stays on the device
 * of ctx until the next call; material names are kept with it. */
int prt_build_mesh(prt_ctx* ctx, const prt_soup_triangle* tris, int triCount, const char* const* materialNames,
                   int materialCount, prt_mesh_info* info);
/* prt_build_mesh for a soup from prt_soup_load_obj, with the same result as
 * prt_build_mesh on prt_soup_triangles(soup) and the soup's material names:
 * uploads the soup's indexed form (the OBJ's vertex lists and each
 * triangle's corner indices: 12 bytes per triangle plus 12 per vertex for a
 * positions-only file, instead of 100 per triangle) and expands it on the GPU. */
int prt_build_mesh_soup(prt_ctx* ctx, const prt_soup* soup, prt_mesh_info* info);
/* Both mesh builders keep their device buffers (the uploaded lists, the
 * scratch, the built mesh's block) in the context for the next mesh build,
 * which allocates only when it needs more; prt_destroy frees them. */
/* Copies the built mesh to host arrays: indices[3*triCount],
 * materialIds[triCount], positions[3*vertCount]; normals[3*vertCount] and
 * texcoords[2*vertCount] only when present (else pass NULL). */
int prt_read_built_mesh(prt_ctx* ctx, int* indices, int* materialIds, float* positions, float* normals, float* texcoords);
/* Writes the built mesh as a .mesh blob (saveBlob + operator<<,
 * sys/blob.h:40-50, geometry/triangle_mesh.cpp:322-337). */
int prt_save_built_mesh(prt_ctx* ctx, const char* path);

#ifdef __cplusplus
}
#endif

#endif
