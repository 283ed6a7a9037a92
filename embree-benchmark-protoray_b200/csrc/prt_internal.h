// Internal host-side declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/prt_b200.h"
#include "prt_device.cuh"
#include "soup_view.h"

namespace prt_b200 {

// Every device allocation of the library goes through dev_malloc, so that an
// out-of-memory condition can be injected on the host (prt_debug_fail_allocations)
// and every error path tested without exhausting a real GPU.
extern long long g_allocFailAfter;   // < 0: off; n >= 0: the (n+1)-th allocation from now fails

template <class T>
inline cudaError_t dev_malloc(T** p, size_t bytes)
{
    if (g_allocFailAfter == 0)
    {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    if (g_allocFailAfter > 0) --g_allocFailAfter;
    return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}

inline cudaError_t host_pinned_alloc(char** p, size_t bytes)
{
    if (g_allocFailAfter == 0)
    {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    if (g_allocFailAfter > 0) --g_allocFailAfter;
    return cudaHostAlloc(reinterpret_cast<void**>(p), bytes, cudaHostAllocDefault);
}

// The 8-wide nodes and the leaf triangles live in one allocation (nodes
// first, 256-byte aligned).
struct Bvh8Device
{
    Bvh8Node* nodes = nullptr;
    TriRec* tris = nullptr;
    void* block = nullptr;   // the allocation holding both
    size_t bytes = 0;        // its size
    int nodeCount = 0;
    int triCount = 0;
    int levels = 0;
    int leafMax = 1;   // most triangles per leaf

    void release()
    {
        if (block) cudaFree(block);
        block = nullptr;
        nodes = nullptr;
        tris = nullptr;
        bytes = 0;
        nodeCount = triCount = levels = 0;
    }
};

// Buffers carved from one allocation, each 256-byte aligned: a dry run with a
// null base measures the block, a second run with the block hands them out.
struct Carve
{
    char* base;
    size_t off = 0;
    template <class T>
    T* take(size_t count)
    {
        off = (off + 255) & ~(size_t)255;
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += sizeof(T) * count;
        return p;
    }
};

// Device scratch kept between calls (a context's BVH and mesh builds): grows
// to the largest request and is reused, so a rebuild allocates only its output.
struct DeviceScratch
{
    void* p = nullptr;
    size_t bytes = 0;

    cudaError_t reserve(size_t need)
    {
        if (need <= bytes) return cudaSuccess;
        release();
        char* q = nullptr;
        cudaError_t e = dev_malloc(&q, need);
        if (e != cudaSuccess) return e;
        p = q;
        bytes = need;
        return cudaSuccess;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

struct BuildInfo
{
    double buildMs = 0;
    int nodeCount = 0;
    int levels = 0;
};

// scratch: kept by the caller between builds, or nullptr for a temporary one
int build_bvh8(const float* dPos, int nv, const int* dIdx, int nt, Bvh8Device& out, cudaStream_t stream,
               std::string& err, BuildInfo* info, int leafMax, bool sahGrouping = true,
               DeviceScratch* scratch = nullptr);

// Full SAH binary tree for the high-quality build (sah_build.cu): scratch
// carved by sah_tree_carve (tmp: n free words the caller supplies), then
// sah_build_tree writes child / range / parent of the n - 1 internal nodes
// (root 0, leaves ~p for position p of perm) and reorders perm.
struct TopTask;
struct TopSplit;
struct SahTreeBuffers
{
    TopTask* task[2];
    TopSplit* splits;
    uint32_t* bins;
    uint32_t* leftCount;   // per chunk, then its exclusive scan
    uint32_t* scanSums;
    int* small;
    int* counters;
    int4* chunks;
    uint32_t* tmp;
    int maxTasks, maxChunks;
};
void sah_tree_carve(Carve& c, int n, SahTreeBuffers& B);
cudaError_t sah_build_tree(int n, const float* triBox, const float* cbounds, uint32_t* perm, int2* child, int2* range,
                           int* parent, const SahTreeBuffers& B, int numSMs, cudaStream_t stream);

// Sort and scan primitives (sort_scan.cu).  radix_sort_pairs sorts (key, value)
// pairs stably on key bits [0, bits); the sorted pairs end in keys/vals (the
// pointers are swapped with the temporaries as needed).  hist needs
// radix_sort_hist_entries(n) words.  exclusive_scan_u32 writes the exclusive
// prefix sums of in[0, n) to out (in == out allowed) and the total to
// sums[scan_sums_entries(n) - 1].
// Both return the number of launches.
size_t radix_sort_hist_entries(int n);
int radix_sort_pairs(uint32_t*& keys, uint32_t*& vals, uint32_t*& keysTmp, uint32_t*& valsTmp, uint32_t* hist, int n,
                     int bits, cudaStream_t stream);
size_t scan_sums_entries(int n);
int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t* sums, int n, cudaStream_t stream);

// An indexed mesh built from a triangle soup on the device (mesh_build.cu).
struct BuiltMesh
{
    void* block = nullptr;  // the allocation holding idx, mat and attr (kept by the next build if large enough)
    size_t blockBytes = 0;
    int* idx = nullptr;     // [3 * triCount]
    int* mat = nullptr;     // [triCount]
    float* attr = nullptr;  // [vertCount * stride]: position [, normal] [, texcoord], as in the .mesh blob
    int triCount = 0, vertCount = 0, stride = 3;
    bool hasNormals = false, hasTexcoords = false, hasMaterials = false;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    std::vector<std::string> names;
    bool valid = false;

    // forget the mesh, keep the allocation
    void reset()
    {
        idx = mat = nullptr;
        attr = nullptr;
        triCount = vertCount = 0;
        valid = false;
        names.clear();
    }
    void release()
    {
        reset();
        if (block) cudaFree(block);
        block = nullptr;
        blockBytes = 0;
    }
};

// TriangleMeshBuilder on the device; hostTris may be host or device memory
// (soupOnDevice: device memory the builder may read in place).  On success
// `out` owns the mesh (names are left to the caller).
// scratch: kept by the caller between builds, or nullptr for a temporary one.
int build_mesh_gpu(const prt_soup_triangle* hostTris, int n, cudaStream_t stream, BuiltMesh& out, std::string& err,
                   double* buildMs, long long* launches, bool soupOnDevice = false, DeviceScratch* scratch = nullptr);
// The same for a parsed OBJ soup: uploads its indexed form and expands the
// triangle records on the device.
// upload: kept by the caller for the uploaded lists, or nullptr for a temporary block.
int build_mesh_gpu_indexed(const SoupIndexed& soup, cudaStream_t stream, BuiltMesh& out, std::string& err,
                           double* buildMs, long long* launches, DeviceScratch* scratch = nullptr,
                           DeviceScratch* upload = nullptr);

// Arguments of one wave of the wavefront renderer.
struct WaveArgs
{
    SceneDev scene;
    CameraDev cam;
    float4* accum;             // width*height sums (r,g,b,weight)
    PathRec* qin;              // input queue (depth >= 1)
    PathRec* qout;             // output queue
    float* thrIn;              // per-path throughput (albedo mode), or nullptr
    float* thrOut;
    int* counts;               // counts[d]: paths entering bounce d (d >= 1)
    int* fetch;                // fetch[d]: work counters of the persistent loop
    unsigned long long* rays;  // running total of closest-hit queries
    const int* passBase;       // device pass counter
    int passOffset;            // first pass of this wave relative to *passBase
    int passes;                // passes in this wave
    int tilesX, tilesY;        // 8x8 pixel tiles covering the frame
    int maxDepth;
    float thrConst;            // throughput at this depth when albedo is constant
    float sky;
    float* Lin = nullptr;      // next-event estimation: radiance gathered so far, per path
    float* Lout = nullptr;     // (nullptr for the plain diffuse integrator)
};

// Per-request table entry of the batched renderer.
struct BatchReq
{
    SceneDev scene;
    CameraDev cam;
    float4* accum;
    long long pathBegin;   // first global path index of this request
    int tilesX, tilesY;
    int spp;
    int maxDepth;
};

struct BatchArgs
{
    const BatchReq* reqs;
    int nreq;
    long long waveBegin;   // global path index range of this wave
    long long waveEnd;
    PathRec* qin;
    PathRec* qout;
    int* counts;
    int* fetch;
    unsigned long long* rays;
    int maxDepth;          // largest maxDepth of the batch
    float sky;
    int leaf1;             // every request's scene uses deferred triangle tests (one-triangle leaves)
    int packet;            // depth 0 as warp packets: one-triangle leaves everywhere, waves start at multiples of 32
};

struct LaunchCfg
{
    int block = 128;
    int blocksPerSM = 0;    // 0 = as many as stay resident
    int pathsPerWave = 0;   // 0 = automatic
    int chains = 2;         // waves in flight at once (concurrent graph branches)
    int packet = 0;         // primary rays as warp packets (one-triangle-leaf trees); 2: interval traversal
};

// Kernel launchers (render.cu).  Each returns the number of launches issued.
int launch_bounce(const WaveArgs& a, int depth, const LaunchCfg& cfg, int numSMs, cudaStream_t s);
// fetch: a zeroed work counter on the device, used by this launch only
int launch_intersect(const SceneDev& sc, const RayRec* rays, HitRec* hits, int n, bool anyHit, float* anyOut,
                     int* fetch, int numSMs, cudaStream_t s);
int launch_resolve_ldr(const float4* accum, uint32_t* out, int n, cudaStream_t s);
int launch_advance_pass(int* passBase, int spp, cudaStream_t s);
// primary rays of pass `pass` for every pixel of cam's frame (row-major)
int launch_primary_rays(const CameraDev& cam, int pass, RayRec* out, cudaStream_t s);
int launch_query(const SceneDev& sc, const RayRec* ray, HitRec* hit, float* pNg, cudaStream_t s);
// fetch: a zeroed 64-bit work counter on the device
int launch_replay(const SceneDev& sc, const CameraDev& cam, float4* accum, int pass0, int spp, int maxDepth, float sky,
                  const float* dL, float* dAlbedo, float* dSky, unsigned long long* rays, int* fetch, bool backward,
                  int numSMs, cudaStream_t s);
int launch_batch_bounce(const BatchArgs& a, int depth, const LaunchCfg& cfg, int numSMs, cudaStream_t s);
int launch_fill(float4* p, size_t n, cudaStream_t s);

} // namespace prt_b200
