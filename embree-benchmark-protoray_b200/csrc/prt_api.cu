// C ABI of the B200 diffuse path tracer (declared in include/prt_b200.h).
//
// Host-side runtime: context and device memory, .mesh loading, camera set-up,
// CUDA-graph capture of whole render calls, batched rendering, the path-replay
// adjoint and the launch-configuration autotuner.  All device work runs on the
// context's own stream; the only host synchronisations are at the end of a
// render call (ray-count read-back) and in the build's level loop.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <memory>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "prt_internal.h"

using namespace prt_b200;

long long prt_b200::g_allocFailAfter = -1;

namespace prt_b200 {
int replay_max_depth();
int read_counters(unsigned long long* out, bool reset, cudaStream_t s);
}

constexpr int kMaxChains = 4;
// Triangles per 8-wide-node leaf.  Box tests of a node run with the whole
// warp, triangle tests only with the lanes that reached a leaf, so smaller
// leaves move filtering work into the efficient part of the traversal:
// one-triangle leaves measured 1.98 / 1.84 / 1.69 Grays/s for leaves of
// 1 / 2 / 3 triangles on the 1.4M-triangle terrain at 1080p (and +14-16% on
// the 82K- and 10M-triangle sphere scenes).
#ifndef PRT_LEAF_MAX
#define PRT_LEAF_MAX 1
#endif
constexpr int kDefaultLeafMax = PRT_LEAF_MAX;
constexpr int kCounterStride = 64 + 2;   // counters per chain: one per bounce depth (<= 64) + 2

struct prt_ctx
{
    int device = 0;
    int numSMs = 148;
    cudaStream_t stream = nullptr;
    std::string err;
    std::string name;

    // mesh
    float* dPos = nullptr;
    int* dIdx = nullptr;
    int nv = 0, nt = 0;
    bool haveMesh = false;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    float* dAlbedo = nullptr;
    float sky = 1.0f;

    // acceleration structure
    Bvh8Device bvh;
    DeviceScratch buildScratch;   // BVH and mesh build scratch, reused by later builds
    DeviceScratch uploadScratch;  // a parsed OBJ's lists on the device, reused by later mesh builds
    bool built = false;
    int leafMax = kDefaultLeafMax;
    bool highQuality = true;   // SAH grouping into 8-wide nodes

    // camera / frame
    prt_camera cam{};
    bool haveCamera = false;
    int W = 0, H = 0;
    float4* dAccum = nullptr;

    // render state
    int* dPass = nullptr;                 // device pass counter
    unsigned long long* dRays = nullptr;  // rays of the current call
    int* dCounts = nullptr;               // [kMaxChains][kMaxDepthCap + 2]
    int* dFetch = nullptr;                // [kMaxChains][kMaxDepthCap + 2]
    PathRec* q[kMaxChains][2] = {};       // ping-pong path queues of each concurrent wave chain
    float* thr[kMaxChains][2] = {};
    float* Lq[kMaxChains][2] = {};        // next-event estimation: gathered radiance per path
    long long queueCap = 0;
    bool queueL = false;
    int integrator = PRT_INTEGRATOR_DIFFUSE;
    int queueChains = 0;
    bool queueThr = false;
    cudaStream_t side[kMaxChains] = {};   // streams of the concurrent wave chains (captured into graphs)
    cudaEvent_t forkEv = nullptr;
    cudaEvent_t joinEv[kMaxChains] = {};

    // work counters of prt_intersect / prt_occluded calls: a ring, so that
    // calls issued on different streams do not share one
    static constexpr int kIsectSlots = 64;
    int* dIsect = nullptr;
    int isectNext = 0;

    // query scratch
    RayRec* dRay = nullptr;
    HitRec* dHit = nullptr;
    float* dPNg = nullptr;

    // batch scratch
    BatchReq* dReqs = nullptr;
    int reqCap = 0;

    // mesh built from a triangle soup (prt_build_mesh)
    BuiltMesh builtMesh;

    LaunchCfg cfg;
    long long launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    struct GraphEntry
    {
        std::string key;
        cudaGraphExec_t exec = nullptr;
        int launches = 0;
    };
    std::vector<GraphEntry> graphs;

    ~prt_ctx();
};

namespace {

constexpr int kMaxDepthCap = kCounterStride - 2;

int fail(prt_ctx* c, int status, const std::string& msg)
{
    if (c) c->err = msg;
    return status;
}

#define CK(call)                                                                                                 \
    do                                                                                                           \
    {                                                                                                            \
        cudaError_t e_ = (call);                                                                                 \
        if (e_ != cudaSuccess)                                                                                   \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? PRT_ENOMEM : PRT_ECUDA,                          \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                                     \
    } while (0)

bool is_device_ptr(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes attr;
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

void clear_graphs(prt_ctx* ctx)
{
    for (auto& g : ctx->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    ctx->graphs.clear();
}

SceneDev scene_dev(const prt_ctx* ctx)
{
    SceneDev s;
    s.nodes = ctx->bvh.nodes;
    s.tris = ctx->bvh.tris;
    s.albedo = ctx->dAlbedo;
    s.triCount = ctx->nt;
    s.hasRoot = ctx->bvh.nodeCount > 0 ? 1 : 0;
    s.leafTris = ctx->bvh.leafMax;
    s.deferTris = ctx->bvh.leafMax == 1 && ctx->nt < kDeferMaxTris ? 1 : 0;
    return s;
}

CameraDev camera_dev(const prt_camera& c, int W, int H)
{
    CameraDev d;
    d.origin = make_float3(c.origin[0], c.origin[1], c.origin[2]);
    d.basisU = make_float3(c.basisU[0], c.basisU[1], c.basisU[2]);
    d.basisV = make_float3(c.basisV[0], c.basisV[1], c.basisV[2]);
    d.imageO = make_float3(c.imageO[0], c.imageO[1], c.imageO[2]);
    d.imageDx = make_float3(c.imageDx[0], c.imageDx[1], c.imageDx[2]);
    d.imageDy = make_float3(c.imageDy[0], c.imageDy[1], c.imageDy[2]);
    d.lensRadius = c.lensRadius;
    d.focalDistance = c.focalDistance;
    d.invW = 1.0f / (float)W;
    d.invH = 1.0f / (float)H;
    d.width = W;
    d.height = H;
    return d;
}

// Counts indices outside [0, nv): 16-byte loads over the bulk of the array
// (cudaMalloc memory is 256-byte aligned), scalar loads for the tail.
__global__ void k_check_indices(const int* __restrict__ idx, long long n3, int nv, int* bad)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long n4 = n3 >> 2;
    const unsigned unv = (unsigned)nv;
    int count = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride)
    {
        int4 v = __ldcs(reinterpret_cast<const int4*>(idx) + i);
        count += ((unsigned)v.x >= unv) + ((unsigned)v.y >= unv) + ((unsigned)v.z >= unv) + ((unsigned)v.w >= unv);
    }
    for (long long i = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += stride)
        count += (unsigned)idx[i] >= unv;
    count = __reduce_add_sync(0xffffffffu, count);
    if ((threadIdx.x & 31) == 0 && count) atomicAdd(bad, count);
}

// Frees the path queues (the next render allocates what it needs).
void release_queues(prt_ctx* ctx)
{
    for (int c = 0; c < kMaxChains; ++c)
        for (int i = 0; i < 2; ++i)
        {
            cudaFree(ctx->q[c][i]);
            cudaFree(ctx->thr[c][i]);
            cudaFree(ctx->Lq[c][i]);
            ctx->q[c][i] = nullptr;
            ctx->thr[c][i] = nullptr;
            ctx->Lq[c][i] = nullptr;
        }
    clear_graphs(ctx);
    ctx->queueCap = 0;
    ctx->queueChains = 0;
    ctx->queueThr = false;
    ctx->queueL = false;
}

int ensure_queues(prt_ctx* ctx, long long paths, bool withThr, int chains = 1, bool withL = false)
{
    if (paths <= ctx->queueCap && chains <= ctx->queueChains && (!withThr || ctx->queueThr) && (!withL || ctx->queueL))
        return PRT_OK;
    for (int c = 0; c < kMaxChains; ++c)
        for (int i = 0; i < 2; ++i)
        {
            cudaFree(ctx->q[c][i]);
            cudaFree(ctx->thr[c][i]);
            cudaFree(ctx->Lq[c][i]);
            ctx->q[c][i] = nullptr;
            ctx->thr[c][i] = nullptr;
            ctx->Lq[c][i] = nullptr;
        }
    clear_graphs(ctx);
    long long cap = std::max(paths, ctx->queueCap);
    int nch = std::max(chains, ctx->queueChains);
    bool thr = withThr || ctx->queueThr;
    bool lq = withL || ctx->queueL;
    ctx->queueCap = 0;
    ctx->queueChains = 0;
    for (int c = 0; c < nch; ++c)
        for (int i = 0; i < 2; ++i)
        {
            CK(dev_malloc(&ctx->q[c][i], sizeof(PathRec) * (size_t)cap));
            if (thr) CK(dev_malloc(&ctx->thr[c][i], sizeof(float) * (size_t)cap));
            if (lq) CK(dev_malloc(&ctx->Lq[c][i], sizeof(float) * (size_t)cap));
        }
    ctx->queueCap = cap;
    ctx->queueChains = nch;
    ctx->queueThr = thr;
    ctx->queueL = lq;
    return PRT_OK;
}

long long default_paths_per_wave(const prt_ctx* ctx)
{
    // Enough paths in flight that even the last bounce keeps every SM busy
    // and the per-launch tail stays small: 16M paths (8 passes of 1080p,
    // 1 GB of queues) measured 1.2x faster than 2M on the 1.4M-triangle
    // terrain scene.
    return std::max<long long>(1 << 24, (long long)ctx->numSMs * 8192);
}

// Throughput after `depth` non-final bounces with the constant albedo 0.8,
// multiplied in float as the reference does (render/diffuse_renderer_cuda.cu:182,209).
float const_throughput(int depth)
{
    float t = 1.0f;
    for (int d = 0; d < depth; ++d) t *= 0.8f;
    return t;
}

int chains_for(const prt_ctx* ctx) { return std::max(1, std::min(kMaxChains, ctx->cfg.chains)); }

int passes_per_wave(const prt_ctx* ctx, int spp)
{
    const long long perPass = (long long)((ctx->W + 7) / 8) * ((ctx->H + 7) / 8) * 64;
    long long ppw = ctx->cfg.pathsPerWave > 0 ? ctx->cfg.pathsPerWave : default_paths_per_wave(ctx);
    return (int)std::max<long long>(1, std::min<long long>(spp, ppw / perPass));
}

// Records every device operation of one render call on ctx->stream (the
// queues are allocated beforehand: no allocation happens during capture).
int record_render(prt_ctx* ctx, int spp, int maxDepth, int accumulate, int& launches)
{
    const int W = ctx->W, H = ctx->H;
    const int tilesX = (W + 7) / 8, tilesY = (H + 7) / 8;
    const long long perPass = (long long)tilesX * tilesY * 64;
    const int passesPerWave = passes_per_wave(ctx, spp);
    const bool albedo = ctx->dAlbedo != nullptr;
    const int waves = (spp + passesPerWave - 1) / passesPerWave;
    const int chains = std::max(1, std::min(chains_for(ctx), waves));
    const bool nee = ctx->integrator == PRT_INTEGRATOR_DIFFUSE2;
    if (ctx->queueCap < (long long)passesPerWave * perPass || ctx->queueChains < chains ||
        (albedo && !ctx->queueThr) || (nee && !ctx->queueL))
        return fail(ctx, PRT_EINTERNAL, "path queues too small");

    launches = 0;
    if (!accumulate) CK(cudaMemsetAsync(ctx->dAccum, 0, sizeof(float4) * (size_t)W * H, ctx->stream));
    CK(cudaMemsetAsync(ctx->dRays, 0, sizeof(unsigned long long), ctx->stream));
    // waves are dealt round-robin to `chains` streams, so the tail of one
    // wave's bounce kernel overlaps the work of another wave
    if (chains > 1)
    {
        CK(cudaEventRecord(ctx->forkEv, ctx->stream));
        for (int c = 0; c < chains; ++c) CK(cudaStreamWaitEvent(ctx->side[c], ctx->forkEv, 0));
    }
    WaveArgs a;
    a.scene = scene_dev(ctx);
    a.cam = camera_dev(ctx->cam, W, H);
    a.accum = ctx->dAccum;
    a.rays = ctx->dRays;
    a.passBase = ctx->dPass;
    a.tilesX = tilesX;
    a.tilesY = tilesY;
    a.maxDepth = maxDepth;
    a.sky = ctx->sky;
    for (int w = 0; w < waves; ++w)
    {
        const int c = w % chains;
        cudaStream_t s = chains > 1 ? ctx->side[c] : ctx->stream;
        int* counts = ctx->dCounts + c * kCounterStride;
        int* fetch = ctx->dFetch + c * kCounterStride;
        a.counts = counts;
        a.fetch = fetch;
        a.passOffset = w * passesPerWave;
        a.passes = std::min(passesPerWave, spp - w * passesPerWave);
        CK(cudaMemsetAsync(counts, 0, sizeof(int) * kCounterStride, s));
        CK(cudaMemsetAsync(fetch, 0, sizeof(int) * kCounterStride, s));
        for (int d = 0; d <= maxDepth; ++d)
        {
            a.qin = d == 0 ? nullptr : ctx->q[c][(d - 1) & 1];
            a.qout = ctx->q[c][d & 1];
            a.thrIn = albedo && d > 0 ? ctx->thr[c][(d - 1) & 1] : nullptr;
            a.thrOut = albedo ? ctx->thr[c][d & 1] : nullptr;
            a.Lin = nee && d > 0 ? ctx->Lq[c][(d - 1) & 1] : nullptr;
            a.Lout = nee ? ctx->Lq[c][d & 1] : nullptr;
            a.thrConst = const_throughput(d);
            launches += launch_bounce(a, d, ctx->cfg, ctx->numSMs, s);
        }
    }
    if (chains > 1)
        for (int c = 0; c < chains; ++c)
        {
            CK(cudaEventRecord(ctx->joinEv[c], ctx->side[c]));
            CK(cudaStreamWaitEvent(ctx->stream, ctx->joinEv[c], 0));
        }
    launches += launch_advance_pass(ctx->dPass, spp, ctx->stream);
    CK(cudaGetLastError());
    return PRT_OK;
}

int run_graph(prt_ctx* ctx, const std::string& key, const std::function<int(int&)>& record, int& launches)
{
    for (auto& g : ctx->graphs)
        if (g.key == key)
        {
            CK(cudaGraphLaunch(g.exec, ctx->stream));
            launches = g.launches;
            return PRT_OK;
        }
    if (ctx->graphs.size() >= 16) clear_graphs(ctx);
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int st = record(launches);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (st != PRT_OK)
    {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return fail(ctx, PRT_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ctx, PRT_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    prt_ctx::GraphEntry ge;
    ge.key = key;
    ge.exec = exec;
    ge.launches = launches;
    ctx->graphs.push_back(ge);
    CK(cudaGraphLaunch(exec, ctx->stream));
    return PRT_OK;
}

int finish_stats(prt_ctx* ctx, prt_render_stats* stats, int passes)
{
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaEventSynchronize(ctx->ev1));
    unsigned long long rays = 0;
    CK(cudaMemcpy(&rays, ctx->dRays, sizeof(rays), cudaMemcpyDeviceToHost));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (stats)
    {
        stats->rays = (long long)rays;
        stats->ms = ms;
        stats->mray = ms > 0 ? (double)rays / 1e6 / (ms / 1e3) : 0.0;
        stats->passes = passes;
    }
    return PRT_OK;
}

int check_ready(prt_ctx* ctx, bool needFrame)
{
    if (!ctx) return PRT_EINVAL;
    if (!ctx->built) return fail(ctx, PRT_ESTATE, "acceleration structure not built (prt_build_accel)");
    if (needFrame && !ctx->dAccum) return fail(ctx, PRT_ESTATE, "frame not initialised (prt_init_frame)");
    if (needFrame && !ctx->haveCamera) return fail(ctx, PRT_ESTATE, "camera not set (prt_set_camera)");
    return PRT_OK;
}

__global__ void k_deinterleave(const float* __restrict__ attrs, int stride, int nv, float* __restrict__ pos)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 3LL * nv;
         i += (long long)gridDim.x * blockDim.x)
    {
        long long v = i / 3;
        int k = (int)(i - 3 * v);
        pos[i] = attrs[v * stride + k];
    }
}

// Per-warp position bounds: each thread reads 4 vertices as three 16-byte
// loads (48 bytes), the last nv % 4 vertices with scalar loads.
__global__ void k_bounds_partial(const float* __restrict__ pos, int nv, float* __restrict__ partial)
{
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    const int quads = nv >> 2;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < quads; q += gridDim.x * blockDim.x)
    {
        const float4* p4 = reinterpret_cast<const float4*>(pos) + 3 * (size_t)q;
        const float4 a = __ldcs(p4), b = __ldcs(p4 + 1), c = __ldcs(p4 + 2);
        const float f[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
#pragma unroll
        for (int j = 0; j < 12; ++j)
        {
            lo[j % 3] = fminf(lo[j % 3], f[j]);
            hi[j % 3] = fmaxf(hi[j % 3], f[j]);
        }
    }
    for (int v = 4 * quads + blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
        for (int k = 0; k < 3; ++k)
        {
            float x = pos[3 * (size_t)v + k];
            lo[k] = fminf(lo[k], x);
            hi[k] = fmaxf(hi[k], x);
        }
    for (int k = 0; k < 3; ++k)
        for (int off = 16; off > 0; off >>= 1)
        {
            lo[k] = fminf(lo[k], __shfl_down_sync(0xffffffffu, lo[k], off));
            hi[k] = fmaxf(hi[k], __shfl_down_sync(0xffffffffu, hi[k], off));
        }
    if ((threadIdx.x & 31) == 0)
    {
        int w = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
        for (int k = 0; k < 3; ++k)
        {
            partial[6 * w + k] = lo[k];
            partial[6 * w + 3 + k] = hi[k];
        }
    }
}

// Takes ownership of device arrays dIdx (3*nt ints) and dPos (3*nv floats):
// checks every index, then makes them the context's mesh.  lo/hi: the stored
// scene box, or nullptr to compute it on the device.
int install_mesh(prt_ctx* ctx, int* dIdx, float* dPos, int nt, int nv, const float* lo, const float* hi)
{
    auto drop = [&]() {
        cudaFree(dIdx);
        cudaFree(dPos);
    };
    int* dBad = nullptr;
    float* dPart = nullptr;
    const int blocks = 4 * ctx->numSMs, threads = 256, warps = blocks * threads / 32;
    cudaError_t e = dev_malloc(&dBad, sizeof(int));
    if (e == cudaSuccess) e = dev_malloc(&dPart, sizeof(float) * 6 * warps);
    if (e == cudaSuccess) e = cudaMemsetAsync(dBad, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess && nt)
    {
        // every index must name a vertex: the kernels gather positions unchecked
        k_check_indices<<<blocks, threads, 0, ctx->stream>>>(dIdx, 3LL * nt, nv, dBad);
        ctx->launches++;
    }
    if (e == cudaSuccess && nv && !lo)
    {
        k_bounds_partial<<<blocks, threads, 0, ctx->stream>>>(dPos, nv, dPart);
        ctx->launches++;
    }
    int bad = 0;
    std::vector<float> part((size_t)6 * warps);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, dBad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && nv && !lo)
        e = cudaMemcpyAsync(part.data(), dPart, sizeof(float) * part.size(), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(dBad);
    cudaFree(dPart);
    if (e != cudaSuccess)
    {
        drop();
        return fail(ctx, e == cudaErrorMemoryAllocation ? PRT_ENOMEM : PRT_ECUDA, cudaGetErrorString(e));
    }
    if (bad)
    {
        drop();
        return fail(ctx, PRT_EINVAL, "triangle index out of range");
    }
    float blo[3] = {0, 0, 0}, bhi[3] = {0, 0, 0};
    if (lo)
    {
        std::memcpy(blo, lo, sizeof(blo));
        std::memcpy(bhi, hi, sizeof(bhi));
    }
    else if (nv)
    {
        for (int k = 0; k < 3; ++k)
        {
            blo[k] = FLT_MAX;
            bhi[k] = -FLT_MAX;
        }
        for (int w = 0; w < warps; ++w)
            for (int k = 0; k < 3; ++k)
            {
                blo[k] = std::min(blo[k], part[6 * (size_t)w + k]);
                bhi[k] = std::max(bhi[k], part[6 * (size_t)w + 3 + k]);
            }
    }
    clear_graphs(ctx);
    ctx->bvh.release();
    ctx->built = false;
    cudaFree(ctx->dPos);
    cudaFree(ctx->dIdx);
    cudaFree(ctx->dAlbedo);
    ctx->dAlbedo = nullptr;
    ctx->dPos = dPos;
    ctx->dIdx = dIdx;
    ctx->nt = nt;
    ctx->nv = nv;
    std::memcpy(ctx->lo, blo, sizeof(blo));
    std::memcpy(ctx->hi, bhi, sizeof(bhi));
    ctx->haveMesh = true;
    return PRT_OK;
}

// .mesh blob loader (geometry/triangle_mesh.cpp:305-320, sys/blob.h:26-38).
// The layout is validated against the file length first; the index and
// vertex-attribute blocks are then read straight into pinned host memory,
// copied to the device asynchronously, and the interleaved attributes
// (position [+ normal] [+ uv], geometry/triangle_mesh.cpp:29-56) are
// de-interleaved on the GPU.
int load_mesh_file(prt_ctx* ctx, const char* path, float outLo[3], float outHi[3])
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(ctx, PRT_EIO, std::string("cannot open ") + path);
    struct Closer
    {
        FILE* f;
        ~Closer() { std::fclose(f); }
    } closer{f};
    std::fseek(f, 0, SEEK_END);
    const long long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    unsigned char head[38];
    if (size < 38 || std::fread(head, 1, 38, f) != 38) return fail(ctx, PRT_EIO, "unexpected end of stream");
    int id, tri, vert;
    float b[6];
    std::memcpy(&id, head, 4);
    if (id != 0x04df8666) return fail(ctx, PRT_EIO, std::string("file has wrong blob ID: ") + path);
    std::memcpy(b, head + 4, 24);
    std::memcpy(&tri, head + 28, 4);
    std::memcpy(&vert, head + 32, 4);
    const bool hasN = head[36] != 0, hasT = head[37] != 0;
    if (tri < 0 || vert < 0) return fail(ctx, PRT_EIO, "negative element count");
    const int stride = 3 + (hasN ? 3 : 0) + (hasT ? 2 : 0);
    const size_t idxBytes = 12 * (size_t)tri, matBytes = 4 * (size_t)tri, attrBytes = 4 * (size_t)vert * stride;
    const long long namesAt = 38 + (long long)(idxBytes + matBytes + attrBytes);
    if (namesAt + 4 > size) return fail(ctx, PRT_EIO, "unexpected end of stream");
    // material names: int count + (int length + bytes) each (sys/array.h:357-392)
    {
        std::fseek(f, (long)namesAt, SEEK_SET);
        int n = 0;
        if (std::fread(&n, 4, 1, f) != 1 || n < 0) return fail(ctx, PRT_EIO, "unexpected end of stream");
        long long at = namesAt + 4;
        for (int i = 0; i < n; ++i)
        {
            int len = 0;
            if (std::fread(&len, 4, 1, f) != 1 || len < 0 || at + 4 + len > size)
                return fail(ctx, PRT_EIO, "unexpected end of stream");
            at += 4 + len;
            std::fseek(f, (long)at, SEEK_SET);
        }
    }
    char* pinned = nullptr;
    int* dIdx = nullptr;
    float* dPos = nullptr;
    float* dAttr = nullptr;
    auto cleanup = [&]() {
        if (pinned) cudaFreeHost(pinned);
        if (dAttr && dAttr != dPos) cudaFree(dAttr);
    };
    cudaError_t e = host_pinned_alloc(&pinned, std::max<size_t>(idxBytes + attrBytes, 16));
    if (e != cudaSuccess) return fail(ctx, PRT_ENOMEM, "cannot allocate pinned staging memory");
    std::fseek(f, 38, SEEK_SET);
    bool ok = std::fread(pinned, 1, idxBytes, f) == idxBytes;
    ok = ok && std::fseek(f, (long)(38 + idxBytes + matBytes), SEEK_SET) == 0;
    ok = ok && std::fread(pinned + idxBytes, 1, attrBytes, f) == attrBytes;
    if (!ok)
    {
        cleanup();
        return fail(ctx, PRT_EIO, std::string("read error: ") + path);
    }
    e = dev_malloc(&dIdx, std::max<size_t>(idxBytes, 12));
    if (e == cudaSuccess) e = dev_malloc(&dPos, sizeof(float) * 3 * (size_t)std::max(vert, 1));
    if (e == cudaSuccess)
    {
        if (stride == 3) dAttr = dPos;
        else e = dev_malloc(&dAttr, std::max<size_t>(attrBytes, 4));
    }
    if (e == cudaSuccess && idxBytes) e = cudaMemcpyAsync(dIdx, pinned, idxBytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && attrBytes)
        e = cudaMemcpyAsync(dAttr, pinned + idxBytes, attrBytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && stride != 3 && vert)
    {
        k_deinterleave<<<512, 256, 0, ctx->stream>>>(dAttr, stride, vert, dPos);
        ctx->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cleanup();
    if (e != cudaSuccess)
    {
        cudaFree(dIdx);
        cudaFree(dPos);
        return fail(ctx, e == cudaErrorMemoryAllocation ? PRT_ENOMEM : PRT_ECUDA, cudaGetErrorString(e));
    }
    float lo[3] = {b[0], b[1], b[2]}, hi[3] = {b[3], b[4], b[5]};
    int st = install_mesh(ctx, dIdx, dPos, tri, vert, lo, hi);
    if (st != PRT_OK) return st;
    if (outLo) std::memcpy(outLo, lo, sizeof(lo));
    if (outHi) std::memcpy(outHi, hi, sizeof(hi));
    return PRT_OK;
}

// A zeroed work counter for one prt_intersect / prt_occluded launch on stream s.
int isect_counter(prt_ctx* ctx, cudaStream_t s, int** out)
{
    if (!ctx->dIsect) CK(dev_malloc(&ctx->dIsect, sizeof(int) * prt_ctx::kIsectSlots));
    int* c = ctx->dIsect + (ctx->isectNext++ % prt_ctx::kIsectSlots);
    CK(cudaMemsetAsync(c, 0, sizeof(int), s));
    *out = c;
    return PRT_OK;
}

} // namespace

prt_ctx::~prt_ctx()
{
    cudaSetDevice(device);
    clear_graphs(this);
    bvh.release();
    buildScratch.release();
    uploadScratch.release();
    cudaFree(dPos);
    cudaFree(dIdx);
    cudaFree(dAlbedo);
    cudaFree(dAccum);
    cudaFree(dPass);
    cudaFree(dRays);
    cudaFree(dCounts);
    cudaFree(dFetch);
    for (int c = 0; c < kMaxChains; ++c)
    {
        for (int i = 0; i < 2; ++i)
        {
            cudaFree(q[c][i]);
            cudaFree(thr[c][i]);
            cudaFree(Lq[c][i]);
        }
        if (side[c]) cudaStreamDestroy(side[c]);
        if (joinEv[c]) cudaEventDestroy(joinEv[c]);
    }
    if (forkEv) cudaEventDestroy(forkEv);
    cudaFree(dIsect);
    cudaFree(dRay);
    cudaFree(dHit);
    cudaFree(dPNg);
    cudaFree(dReqs);
    builtMesh.release();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
}

extern "C" {

int prt_create(int device, prt_ctx** out)
{
    if (!out) return PRT_EINVAL;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return PRT_ECUDA;
    if (device < 0 || device >= count) return PRT_EINVAL;
    std::unique_ptr<prt_ctx> c(new prt_ctx);
    prt_ctx* ctx = c.get();
    ctx->device = device;
    CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    ctx->numSMs = prop.multiProcessorCount;
    ctx->name = prop.name;
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ctx->ev0));
    CK(cudaEventCreate(&ctx->ev1));
    CK(dev_malloc(&ctx->dPass, sizeof(int)));
    CK(cudaMemset(ctx->dPass, 0, sizeof(int)));
    CK(dev_malloc(&ctx->dRays, sizeof(unsigned long long)));
    CK(dev_malloc(&ctx->dCounts, sizeof(int) * kCounterStride * kMaxChains));
    CK(dev_malloc(&ctx->dFetch, sizeof(int) * kCounterStride * kMaxChains));
    CK(cudaEventCreateWithFlags(&ctx->forkEv, cudaEventDisableTiming));
    for (int c = 0; c < kMaxChains; ++c)
    {
        CK(cudaStreamCreateWithFlags(&ctx->side[c], cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->joinEv[c], cudaEventDisableTiming));
    }
    CK(dev_malloc(&ctx->dRay, sizeof(RayRec)));
    CK(dev_malloc(&ctx->dHit, sizeof(HitRec)));
    CK(dev_malloc(&ctx->dPNg, sizeof(float) * 6));
    *out = c.release();
    return PRT_OK;
}

int prt_destroy(prt_ctx* ctx)
{
    if (!ctx) return PRT_EINVAL;
    delete ctx;
    return PRT_OK;
}

const char* prt_last_error(const prt_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int prt_get_info(prt_ctx* ctx, char* buf, int len)
{
    if (!ctx || !buf || len <= 0) return PRT_EINVAL;
    std::snprintf(buf, (size_t)len, "%s", ctx->name.c_str());
    return PRT_OK;
}

long long prt_launch_count(prt_ctx* ctx) { return ctx ? ctx->launches : 0; }

int prt_load_mesh(prt_ctx* ctx, const int* indices, int triCount, const float* positions, int vertCount)
{
    if (!ctx) return PRT_EINVAL;
    if (triCount < 0 || vertCount < 0) return fail(ctx, PRT_EINVAL, "negative element count");
    if ((triCount > 0 && !indices) || (vertCount > 0 && !positions)) return fail(ctx, PRT_EINVAL, "null mesh array");
    CK(cudaSetDevice(ctx->device));
    int* dIdx = nullptr;
    float* dPos = nullptr;
    cudaError_t e = dev_malloc(&dPos, sizeof(float) * 3 * (size_t)std::max(vertCount, 1));
    if (e == cudaSuccess) e = dev_malloc(&dIdx, sizeof(int) * 3 * (size_t)std::max(triCount, 1));
    if (e == cudaSuccess && vertCount)
        e = cudaMemcpyAsync(dPos, positions, sizeof(float) * 3 * (size_t)vertCount, cudaMemcpyDefault, ctx->stream);
    if (e == cudaSuccess && triCount)
        e = cudaMemcpyAsync(dIdx, indices, sizeof(int) * 3 * (size_t)triCount, cudaMemcpyDefault, ctx->stream);
    if (e != cudaSuccess)
    {
        cudaFree(dPos);
        cudaFree(dIdx);
        return fail(ctx, e == cudaErrorMemoryAllocation ? PRT_ENOMEM : PRT_ECUDA, cudaGetErrorString(e));
    }
    return install_mesh(ctx, dIdx, dPos, triCount, vertCount, nullptr, nullptr);
}

int prt_load_mesh_file(prt_ctx* ctx, const char* path, float boundsLo[3], float boundsHi[3])
{
    if (!ctx || !path) return PRT_EINVAL;
    CK(cudaSetDevice(ctx->device));
    return load_mesh_file(ctx, path, boundsLo, boundsHi);
}

int prt_get_scene_bounds(prt_ctx* ctx, float lo[3], float hi[3])
{
    if (!ctx || !lo || !hi) return PRT_EINVAL;
    if (!ctx->haveMesh) return fail(ctx, PRT_ESTATE, "no scene loaded");
    std::memcpy(lo, ctx->lo, sizeof(ctx->lo));
    std::memcpy(hi, ctx->hi, sizeof(ctx->hi));
    return PRT_OK;
}

int prt_set_albedo(prt_ctx* ctx, const float* albedo, int triCount)
{
    if (!ctx) return PRT_EINVAL;
    if (!ctx->haveMesh) return fail(ctx, PRT_ESTATE, "no scene loaded");
    CK(cudaSetDevice(ctx->device));
    clear_graphs(ctx);
    if (!albedo)
    {
        cudaFree(ctx->dAlbedo);
        ctx->dAlbedo = nullptr;
        return PRT_OK;
    }
    if (triCount != ctx->nt) return fail(ctx, PRT_EINVAL, "albedo count differs from the triangle count");
    if (!ctx->dAlbedo) CK(dev_malloc(&ctx->dAlbedo, sizeof(float) * (size_t)std::max(ctx->nt, 1)));
    if (ctx->nt)
        CK(cudaMemcpyAsync(ctx->dAlbedo, albedo, sizeof(float) * (size_t)ctx->nt, cudaMemcpyDefault, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

int prt_set_integrator(prt_ctx* ctx, int integrator)
{
    if (!ctx) return PRT_EINVAL;
    if (integrator != PRT_INTEGRATOR_DIFFUSE && integrator != PRT_INTEGRATOR_DIFFUSE2)
        return fail(ctx, PRT_EINVAL, "unknown integrator");
    if (integrator != ctx->integrator) clear_graphs(ctx);
    ctx->integrator = integrator;
    return PRT_OK;
}

int prt_set_sky(prt_ctx* ctx, float sky)
{
    if (!ctx) return PRT_EINVAL;
    if (!std::isfinite(sky)) return fail(ctx, PRT_EINVAL, "sky radiance must be finite");
    ctx->sky = sky;
    clear_graphs(ctx);
    return PRT_OK;
}

int prt_set_leaf_size(prt_ctx* ctx, int maxTrianglesPerLeaf)
{
    if (!ctx) return PRT_EINVAL;
    if (maxTrianglesPerLeaf < 1 || maxTrianglesPerLeaf > 3) return fail(ctx, PRT_EINVAL, "leaf size must be 1..3");
    ctx->leafMax = maxTrianglesPerLeaf;
    return PRT_OK;
}

int prt_set_build_quality(prt_ctx* ctx, int high)
{
    if (!ctx) return PRT_EINVAL;
    if (high != 0 && high != 1) return fail(ctx, PRT_EINVAL, "build quality must be 0 (low) or 1 (high)");
    ctx->highQuality = high == 1;
    return PRT_OK;
}

int prt_build_accel(prt_ctx* ctx, prt_build_stats* stats)
{
    if (!ctx) return PRT_EINVAL;
    if (!ctx->haveMesh) return fail(ctx, PRT_ESTATE, "no scene loaded");
    CK(cudaSetDevice(ctx->device));
    clear_graphs(ctx);
    ctx->built = false;
    BuildInfo info;
    std::string err;
    int st = build_bvh8(ctx->dPos, ctx->nv, ctx->dIdx, ctx->nt, ctx->bvh, ctx->stream, err, &info, ctx->leafMax,
                        ctx->highQuality, &ctx->buildScratch);
    if (st != PRT_OK) return fail(ctx, st, err);
    ctx->built = true;
    if (stats)
    {
        stats->buildMs = info.buildMs;
        stats->buildMprim = info.buildMs > 0 ? (double)ctx->nt / 1e6 / (info.buildMs / 1e3) : 0.0;
        stats->nodeCount = ctx->bvh.nodeCount;
        stats->levels = ctx->bvh.levels;
    }
    return PRT_OK;
}

int prt_camera_from_view(const prt_view* v, int width, int height, prt_camera* cam)
{
    if (!v || !cam || width <= 0 || height <= 0) return PRT_EINVAL;
    // Basis3f(one).rotateV(angleY).rotateU(angleX) (math/basis3.h:63-79) with
    // rotate() of math/vec3.h:409-412, then PinholeCamera's image plane
    // (camera/pinhole_camera.h:40-47), all in float in the reference's order.
    struct V3 { float x, y, z; };
    auto vadd = [](V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; };
    auto vmul = [](V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; };
    auto vdot = [](V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; };
    auto vcross = [](V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; };
    auto rotate = [&](V3 vec, V3 axis, float ang) {
        float c = std::cos(ang), s = std::sin(ang);
        return vadd(vadd(vmul(vec, c), vmul(vmul(axis, vdot(axis, vec)), 1.0f - c)), vmul(vcross(vec, axis), s));
    };
    V3 V0{0, 1, 0}, N0{0, 0, 1};
    V3 N1 = rotate(N0, V0, v->angleY);
    V3 U1 = vcross(V0, N1);
    V3 V2 = rotate(V0, U1, v->angleX);
    V3 N2 = vcross(U1, V2);
    float aspect = (float)width / (float)height;
    float hh = std::tan(0.5f * v->fovY);
    float hw = hh * aspect;
    auto basis = [&](float ax, float ay, float az) { return vadd(vadd(vmul(U1, ax), vmul(V2, ay)), vmul(N2, az)); };
    V3 O = basis(-hw, hh, -1.0f);
    V3 Dx = basis(2.0f * hw, 0.0f, 0.0f);
    V3 Dy = basis(0.0f, (float)(-2.0 * (double)hh), 0.0f);
    auto put = [](float* d, V3 a) { d[0] = a.x; d[1] = a.y; d[2] = a.z; };
    cam->origin[0] = v->pos[0];
    cam->origin[1] = v->pos[1];
    cam->origin[2] = v->pos[2];
    put(cam->basisU, U1);
    put(cam->basisV, V2);
    put(cam->imageO, O);
    put(cam->imageDx, Dx);
    put(cam->imageDy, Dy);
    cam->lensRadius = v->radius;
    cam->focalDistance = v->focus;
    return PRT_OK;
}

int prt_set_camera(prt_ctx* ctx, const prt_camera* cam)
{
    if (!ctx || !cam) return PRT_EINVAL;
    // captured render graphs bake the camera into their kernel arguments
    if (!ctx->haveCamera || std::memcmp(&ctx->cam, cam, sizeof(prt_camera)) != 0) clear_graphs(ctx);
    ctx->cam = *cam;
    ctx->haveCamera = true;
    return PRT_OK;
}

int prt_init_frame(prt_ctx* ctx, int width, int height)
{
    if (!ctx) return PRT_EINVAL;
    if (width <= 0 || height <= 0 || (long long)width * height > (1LL << 28))
        return fail(ctx, PRT_EINVAL, "invalid frame size");
    CK(cudaSetDevice(ctx->device));
    clear_graphs(ctx);
    cudaFree(ctx->dAccum);
    ctx->dAccum = nullptr;
    CK(dev_malloc(&ctx->dAccum, sizeof(float4) * (size_t)width * height));
    ctx->W = width;
    ctx->H = height;
    return prt_clear(ctx);
}

int prt_clear(prt_ctx* ctx)
{
    if (!ctx) return PRT_EINVAL;
    if (!ctx->dAccum) return fail(ctx, PRT_ESTATE, "frame not initialised (prt_init_frame)");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemsetAsync(ctx->dAccum, 0, sizeof(float4) * (size_t)ctx->W * ctx->H, ctx->stream));
    CK(cudaMemsetAsync(ctx->dPass, 0, sizeof(int), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

int prt_set_pass(prt_ctx* ctx, int pass)
{
    if (!ctx || pass < 0) return PRT_EINVAL;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(ctx->dPass, &pass, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

int prt_get_pass(prt_ctx* ctx, int* pass)
{
    if (!ctx || !pass) return PRT_EINVAL;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(pass, ctx->dPass, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

int prt_read_accum(prt_ctx* ctx, float* rgbw)
{
    if (!ctx || !rgbw) return PRT_EINVAL;
    if (!ctx->dAccum) return fail(ctx, PRT_ESTATE, "frame not initialised (prt_init_frame)");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(rgbw, ctx->dAccum, sizeof(float4) * (size_t)ctx->W * ctx->H, cudaMemcpyDefault, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

int prt_read_ldr(prt_ctx* ctx, uint32_t* bgra)
{
    if (!ctx || !bgra) return PRT_EINVAL;
    if (!ctx->dAccum) return fail(ctx, PRT_ESTATE, "frame not initialised (prt_init_frame)");
    CK(cudaSetDevice(ctx->device));
    size_t n = (size_t)ctx->W * ctx->H;
    uint32_t* dOut = nullptr;
    bool dev = is_device_ptr(bgra);
    if (dev) dOut = bgra;
    else CK(dev_malloc(&dOut, sizeof(uint32_t) * n));
    ctx->launches += launch_resolve_ldr(ctx->dAccum, dOut, (int)n, ctx->stream);
    CK(cudaGetLastError());
    if (!dev) CK(cudaMemcpyAsync(bgra, dOut, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (!dev) cudaFree(dOut);
    return PRT_OK;
}

int prt_render(prt_ctx* ctx, int spp, int maxDepth, int accumulate, prt_render_stats* stats)
{
    int st = check_ready(ctx, true);
    if (st != PRT_OK) return st;
    if (spp < 0 || maxDepth < 0 || maxDepth > kMaxDepthCap) return fail(ctx, PRT_EINVAL, "invalid spp or maxDepth");
    CK(cudaSetDevice(ctx->device));
    if (spp > 0)
    {
        const long long perPass = (long long)((ctx->W + 7) / 8) * ((ctx->H + 7) / 8) * 64;
        const int ppw = passes_per_wave(ctx, spp);
        const int waves = (spp + ppw - 1) / ppw;
        st = ensure_queues(ctx, (long long)ppw * perPass, ctx->dAlbedo != nullptr,
                           std::max(1, std::min(chains_for(ctx), waves)),
                           ctx->integrator == PRT_INTEGRATOR_DIFFUSE2);
        if (st != PRT_OK) return st;
    }
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (spp > 0)
    {
        std::ostringstream key;
        key << "render:" << ctx->integrator << ":" << spp << ":" << maxDepth << ":" << accumulate << ":" << ctx->cfg.block << ":"
            << ctx->cfg.blocksPerSM << ":" << ctx->cfg.pathsPerWave;
        int launches = 0;
        st = run_graph(ctx, key.str(), [&](int& l) { return record_render(ctx, spp, maxDepth, accumulate, l); },
                       launches);
        if (st != PRT_OK) return st;
        ctx->launches += launches;
    }
    else
    {
        CK(cudaMemsetAsync(ctx->dRays, 0, sizeof(unsigned long long), ctx->stream));
    }
    return finish_stats(ctx, stats, spp);
}

int prt_render_profile(prt_ctx* ctx, int spp, int maxDepth, double* msPerDepth, long long* raysPerDepth)
{
    int st = check_ready(ctx, true);
    if (st != PRT_OK) return st;
    if (spp <= 0 || maxDepth < 0 || maxDepth > kMaxDepthCap || !msPerDepth || !raysPerDepth)
        return fail(ctx, PRT_EINVAL, "invalid spp, maxDepth or output arrays");
    CK(cudaSetDevice(ctx->device));
    const int W = ctx->W, H = ctx->H;
    const int tilesX = (W + 7) / 8, tilesY = (H + 7) / 8;
    const long long perPass = (long long)tilesX * tilesY * 64;
    const int ppw = passes_per_wave(ctx, spp);
    const bool albedo = ctx->dAlbedo != nullptr;
    const bool nee = ctx->integrator == PRT_INTEGRATOR_DIFFUSE2;
    st = ensure_queues(ctx, (long long)ppw * perPass, albedo, 1, nee);
    if (st != PRT_OK) return st;
    for (int d = 0; d <= maxDepth; ++d)
    {
        msPerDepth[d] = 0;
        raysPerDepth[d] = 0;
    }
    std::vector<cudaEvent_t> ev((size_t)maxDepth + 2);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    WaveArgs a;
    a.scene = scene_dev(ctx);
    a.cam = camera_dev(ctx->cam, W, H);
    a.accum = ctx->dAccum;
    a.counts = ctx->dCounts;
    a.fetch = ctx->dFetch;
    a.rays = ctx->dRays;
    a.passBase = ctx->dPass;
    a.tilesX = tilesX;
    a.tilesY = tilesY;
    a.maxDepth = maxDepth;
    a.sky = ctx->sky;
    CK(cudaMemsetAsync(ctx->dAccum, 0, sizeof(float4) * (size_t)W * H, ctx->stream));
    for (int p0 = 0; p0 < spp; p0 += ppw)
    {
        a.passOffset = p0;
        a.passes = std::min(ppw, spp - p0);
        CK(cudaMemsetAsync(ctx->dCounts, 0, sizeof(int) * (kMaxDepthCap + 2), ctx->stream));
        CK(cudaMemsetAsync(ctx->dFetch, 0, sizeof(int) * (kMaxDepthCap + 2), ctx->stream));
        CK(cudaEventRecord(ev[0], ctx->stream));
        for (int d = 0; d <= maxDepth; ++d)
        {
            a.qin = d == 0 ? nullptr : ctx->q[0][(d - 1) & 1];
            a.qout = ctx->q[0][d & 1];
            a.thrIn = albedo && d > 0 ? ctx->thr[0][(d - 1) & 1] : nullptr;
            a.thrOut = albedo ? ctx->thr[0][d & 1] : nullptr;
            a.Lin = nee && d > 0 ? ctx->Lq[0][(d - 1) & 1] : nullptr;
            a.Lout = nee ? ctx->Lq[0][d & 1] : nullptr;
            a.thrConst = const_throughput(d);
            ctx->launches += launch_bounce(a, d, ctx->cfg, ctx->numSMs, ctx->stream);
            CK(cudaEventRecord(ev[(size_t)d + 1], ctx->stream));
        }
        CK(cudaGetLastError());
        std::vector<int> counts((size_t)maxDepth + 2);
        CK(cudaMemcpyAsync(counts.data(), ctx->dCounts, sizeof(int) * counts.size(), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (int d = 0; d <= maxDepth; ++d)
        {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, ev[(size_t)d], ev[(size_t)d + 1]));
            msPerDepth[d] += ms;
            raysPerDepth[d] += d == 0 ? (long long)a.passes * W * H : counts[(size_t)d];
        }
    }
    launch_advance_pass(ctx->dPass, spp, ctx->stream);
    ctx->launches++;
    CK(cudaStreamSynchronize(ctx->stream));
    for (auto& e : ev) cudaEventDestroy(e);
    return PRT_OK;
}

int prt_query_ray(prt_ctx* ctx, const prt_ray* ray, prt_hit* hit, float p[3], float Ng[3])
{
    int st = check_ready(ctx, false);
    if (st != PRT_OK) return st;
    if (!ray || !hit) return fail(ctx, PRT_EINVAL, "null ray or hit");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(ctx->dRay, ray, sizeof(RayRec), cudaMemcpyHostToDevice, ctx->stream));
    ctx->launches += launch_query(scene_dev(ctx), ctx->dRay, ctx->dHit, ctx->dPNg, ctx->stream);
    CK(cudaGetLastError());
    float png[6];
    CK(cudaMemcpyAsync(hit, ctx->dHit, sizeof(HitRec), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(png, ctx->dPNg, sizeof(png), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (hit->t >= 0.f)
    {
        if (p) std::memcpy(p, png, 12);
        if (Ng) std::memcpy(Ng, png + 3, 12);
    }
    return PRT_OK;
}

int prt_intersect(prt_ctx* ctx, const prt_ray* rays, prt_hit* hits, int n, void* stream)
{
    int st = check_ready(ctx, false);
    if (st != PRT_OK) return st;
    if (n < 0 || (n > 0 && (!rays || !hits))) return fail(ctx, PRT_EINVAL, "invalid ray buffers");
    if (n > 0 && (!is_device_ptr(rays) || !is_device_ptr(hits)))
        return fail(ctx, PRT_EINVAL, "prt_intersect takes device pointers");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    int* fetch = nullptr;
    st = isect_counter(ctx, s, &fetch);
    if (st != PRT_OK) return st;
    ctx->launches += launch_intersect(scene_dev(ctx), (const RayRec*)rays, (HitRec*)hits, n, false, nullptr, fetch, ctx->numSMs, s);
    CK(cudaGetLastError());
    if (!stream) CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

int prt_primary_rays(prt_ctx* ctx, int pass, prt_ray* rays, void* stream)
{
    int st = check_ready(ctx, true);
    if (st != PRT_OK) return st;
    if (pass < 0 || !rays) return fail(ctx, PRT_EINVAL, "invalid pass or ray buffer");
    if (!is_device_ptr(rays)) return fail(ctx, PRT_EINVAL, "prt_primary_rays takes a device pointer");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    ctx->launches += launch_primary_rays(camera_dev(ctx->cam, ctx->W, ctx->H), pass, (RayRec*)rays, s);
    CK(cudaGetLastError());
    if (!stream) CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

int prt_occluded(prt_ctx* ctx, const prt_ray* rays, float* out, int n, void* stream)
{
    int st = check_ready(ctx, false);
    if (st != PRT_OK) return st;
    if (n < 0 || (n > 0 && (!rays || !out))) return fail(ctx, PRT_EINVAL, "invalid ray buffers");
    if (n > 0 && (!is_device_ptr(rays) || !is_device_ptr(out)))
        return fail(ctx, PRT_EINVAL, "prt_occluded takes device pointers");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    int* fetch = nullptr;
    st = isect_counter(ctx, s, &fetch);
    if (st != PRT_OK) return st;
    ctx->launches += launch_intersect(scene_dev(ctx), (const RayRec*)rays, nullptr, n, true, out, fetch, ctx->numSMs, s);
    CK(cudaGetLastError());
    if (!stream) CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

int prt_render_replay(prt_ctx* ctx, int pass0, int spp, int maxDepth, prt_render_stats* stats)
{
    int st = check_ready(ctx, true);
    if (st != PRT_OK) return st;
    if (pass0 < 0 || spp < 0 || maxDepth < 0 || maxDepth > replay_max_depth())
        return fail(ctx, PRT_EINVAL, "invalid pass range or maxDepth (replay supports maxDepth <= 16)");
    CK(cudaSetDevice(ctx->device));
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    CK(cudaMemsetAsync(ctx->dRays, 0, sizeof(unsigned long long), ctx->stream));
    CK(cudaMemsetAsync(ctx->dFetch, 0, sizeof(unsigned long long), ctx->stream));
    ctx->launches += launch_replay(scene_dev(ctx), camera_dev(ctx->cam, ctx->W, ctx->H), ctx->dAccum, pass0, spp,
                                   maxDepth, ctx->sky, nullptr, nullptr, nullptr, ctx->dRays, ctx->dFetch, false,
                                   ctx->numSMs, ctx->stream);
    CK(cudaGetLastError());
    return finish_stats(ctx, stats, spp);
}

int prt_render_backward(prt_ctx* ctx, int pass0, int spp, int maxDepth, const float* dL_dsum, float* d_albedo,
                        float* d_sky)
{
    int st = check_ready(ctx, true);
    if (st != PRT_OK) return st;
    if (!dL_dsum || !d_albedo || !d_sky) return fail(ctx, PRT_EINVAL, "null gradient buffer");
    if (pass0 < 0 || spp < 0 || maxDepth < 0 || maxDepth > replay_max_depth())
        return fail(ctx, PRT_EINVAL, "invalid pass range or maxDepth (replay supports maxDepth <= 16)");
    CK(cudaSetDevice(ctx->device));
    const size_t npix = (size_t)ctx->W * ctx->H;
    const bool devL = is_device_ptr(dL_dsum), devA = is_device_ptr(d_albedo), devS = is_device_ptr(d_sky);
    float* gL = nullptr;
    float* gA = nullptr;
    float* gS = nullptr;
    if (devL) gL = const_cast<float*>(dL_dsum);
    else
    {
        CK(dev_malloc(&gL, sizeof(float) * 3 * npix));
        CK(cudaMemcpyAsync(gL, dL_dsum, sizeof(float) * 3 * npix, cudaMemcpyHostToDevice, ctx->stream));
    }
    if (devA) gA = d_albedo;
    else CK(dev_malloc(&gA, sizeof(float) * (size_t)std::max(ctx->nt, 1)));
    if (devS) gS = d_sky;
    else CK(dev_malloc(&gS, sizeof(float)));
    CK(cudaMemsetAsync(gA, 0, sizeof(float) * (size_t)ctx->nt, ctx->stream));
    CK(cudaMemsetAsync(gS, 0, sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(ctx->dFetch, 0, sizeof(unsigned long long), ctx->stream));
    ctx->launches += launch_replay(scene_dev(ctx), camera_dev(ctx->cam, ctx->W, ctx->H), ctx->dAccum, pass0, spp,
                                   maxDepth, ctx->sky, gL, gA, gS, nullptr, ctx->dFetch, true, ctx->numSMs,
                                   ctx->stream);
    CK(cudaGetLastError());
    if (!devA) CK(cudaMemcpyAsync(d_albedo, gA, sizeof(float) * (size_t)ctx->nt, cudaMemcpyDeviceToHost, ctx->stream));
    if (!devS) CK(cudaMemcpyAsync(d_sky, gS, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (!devL) cudaFree(gL);
    if (!devA) cudaFree(gA);
    if (!devS) cudaFree(gS);
    return PRT_OK;
}

int prt_render_batch(prt_ctx* ctx, const prt_request* reqs, int n, prt_render_stats* stats)
{
    if (!ctx) return PRT_EINVAL;
    if (n < 0 || n > 255 || (n > 0 && !reqs)) return fail(ctx, PRT_EINVAL, "batch size must be 0..255");
    CK(cudaSetDevice(ctx->device));
    std::vector<BatchReq> table((size_t)n);
    std::vector<float4*> tmp((size_t)n, nullptr);
    long long total = 0;
    int maxDepth = 0;
    int leaf1 = 1, leafOne = 1;
    std::ostringstream key;
    key << "batch:" << n << ":" << ctx->cfg.block << ":" << ctx->cfg.blocksPerSM << ":" << ctx->cfg.pathsPerWave;
    for (int r = 0; r < n; ++r)
    {
        const prt_request& q = reqs[r];
        if (!q.scene || !q.scene->built) return fail(ctx, PRT_ESTATE, "batch request scene not built");
        if (q.scene->device != ctx->device) return fail(ctx, PRT_EINVAL, "batch request scene on another device");
        if (q.scene->dAlbedo) return fail(ctx, PRT_EINVAL, "batched rendering uses the constant albedo");
        if (q.width <= 0 || q.height <= 0 || (long long)q.width * q.height > (1LL << 24) || q.spp < 0 ||
            q.maxDepth < 0 || q.maxDepth > kMaxDepthCap || !q.accum)
            return fail(ctx, PRT_EINVAL, "invalid batch request");
        BatchReq& b = table[(size_t)r];
        b.scene = scene_dev(q.scene);
        b.cam = camera_dev(q.camera, q.width, q.height);
        b.tilesX = (q.width + 7) / 8;
        b.tilesY = (q.height + 7) / 8;
        b.spp = q.spp;
        b.maxDepth = q.maxDepth;
        b.pathBegin = total;
        total += (long long)b.tilesX * b.tilesY * 64 * q.spp;
        if (!b.scene.deferTris) leaf1 = 0;
        if (b.scene.leafTris != 1) leafOne = 0;
        maxDepth = std::max(maxDepth, q.maxDepth);
        key << ":" << (const void*)q.scene << "," << q.width << "x" << q.height << "," << q.spp << "," << q.maxDepth
            << "," << (const void*)q.accum;
        for (int k = 0; k < 3; ++k)
            key << "," << q.camera.origin[k] << "," << q.camera.imageO[k] << "," << q.camera.imageDx[k] << ","
                << q.camera.imageDy[k] << "," << q.camera.basisU[k] << "," << q.camera.basisV[k];
        key << "," << q.camera.lensRadius << "," << q.camera.focalDistance;
    }
    key << ":sky" << ctx->sky << ":leaf1" << leaf1;
    // device accumulation buffers (caller's device memory in place)
    bool anyTmp = false;
    for (int r = 0; r < n; ++r)
    {
        const prt_request& q = reqs[r];
        size_t bytes = sizeof(float4) * (size_t)q.width * q.height;
        if (is_device_ptr(q.accum)) table[(size_t)r].accum = (float4*)q.accum;
        else
        {
            CK(dev_malloc(&tmp[(size_t)r], bytes));
            table[(size_t)r].accum = tmp[(size_t)r];
            anyTmp = true;
        }
    }
    if (anyTmp) key << ":tmp";   // temporary buffers change per call: do not reuse a graph
    if (n > ctx->reqCap)
    {
        cudaFree(ctx->dReqs);
        ctx->dReqs = nullptr;
        CK(dev_malloc(&ctx->dReqs, sizeof(BatchReq) * (size_t)n));
        ctx->reqCap = n;
        clear_graphs(ctx);
    }
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (n > 0)
        CK(cudaMemcpyAsync(ctx->dReqs, table.data(), sizeof(BatchReq) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    for (int r = 0; r < n; ++r)
        CK(cudaMemsetAsync(table[(size_t)r].accum, 0, sizeof(float4) * (size_t)reqs[r].width * reqs[r].height,
                           ctx->stream));
    long long ppw = ctx->cfg.pathsPerWave > 0 ? ctx->cfg.pathsPerWave : default_paths_per_wave(ctx);
    const long long waves = total > 0 ? (total + ppw - 1) / ppw : 0;
    // waves are dealt round-robin to concurrent chains, as record_render does,
    // so the tail of one wave's bounce launch overlaps another wave's work
    const int chains = (int)std::max<long long>(1, std::min<long long>(chains_for(ctx), waves));
    key << ":chains" << chains;
    int st = ensure_queues(ctx, std::min<long long>(ppw, std::max<long long>(total, 1)), false, chains);
    if (st != PRT_OK) return st;
    auto record = [&](int& launches) -> int {
        launches = 0;
        CK(cudaMemsetAsync(ctx->dRays, 0, sizeof(unsigned long long), ctx->stream));
        if (chains > 1)
        {
            CK(cudaEventRecord(ctx->forkEv, ctx->stream));
            for (int c = 0; c < chains; ++c) CK(cudaStreamWaitEvent(ctx->side[c], ctx->forkEv, 0));
        }
        BatchArgs a;
        a.reqs = ctx->dReqs;
        a.nreq = n;
        a.rays = ctx->dRays;
        a.maxDepth = maxDepth;
        a.sky = ctx->sky;
        a.leaf1 = leaf1;
        a.packet = leafOne && ppw % 32 == 0;
        long long w = 0;
        for (long long w0 = 0; w0 < total; w0 += ppw, ++w)
        {
            const int c = (int)(w % chains);
            cudaStream_t s = chains > 1 ? ctx->side[c] : ctx->stream;
            a.counts = ctx->dCounts + c * kCounterStride;
            a.fetch = ctx->dFetch + c * kCounterStride;
            a.waveBegin = w0;
            a.waveEnd = std::min(total, w0 + ppw);
            CK(cudaMemsetAsync(a.counts, 0, sizeof(int) * kCounterStride, s));
            CK(cudaMemsetAsync(a.fetch, 0, sizeof(int) * kCounterStride, s));
            for (int d = 0; d <= maxDepth; ++d)
            {
                a.qin = d == 0 ? nullptr : ctx->q[c][(d - 1) & 1];
                a.qout = ctx->q[c][d & 1];
                launches += launch_batch_bounce(a, d, ctx->cfg, ctx->numSMs, s);
            }
        }
        if (chains > 1)
            for (int c = 0; c < chains; ++c)
            {
                CK(cudaEventRecord(ctx->joinEv[c], ctx->side[c]));
                CK(cudaStreamWaitEvent(ctx->stream, ctx->joinEv[c], 0));
            }
        CK(cudaGetLastError());
        return PRT_OK;
    };
    int launches = 0;
    if (n > 0 && total > 0)
    {
        st = run_graph(ctx, key.str(), record, launches);
        if (st != PRT_OK) return st;
        ctx->launches += launches;
    }
    else
    {
        CK(cudaMemsetAsync(ctx->dRays, 0, sizeof(unsigned long long), ctx->stream));
    }
    st = finish_stats(ctx, stats, 0);
    for (int r = 0; r < n; ++r)
        if (tmp[(size_t)r])
        {
            CK(cudaMemcpy(reqs[r].accum, tmp[(size_t)r], sizeof(float4) * (size_t)reqs[r].width * reqs[r].height,
                          cudaMemcpyDeviceToHost));
            cudaFree(tmp[(size_t)r]);
        }
    if (anyTmp)
    {
        // graphs that captured the temporary buffers are stale now
        auto& g = ctx->graphs;
        for (auto it = g.begin(); it != g.end();)
            if (it->key == key.str()) { cudaGraphExecDestroy(it->exec); it = g.erase(it); }
            else ++it;
    }
    return st;
}

int prt_read_accel(prt_ctx* ctx, void* nodes, int nodeCapacity, void* tris, int triCapacity, int* nodeCount,
                   int* triCount)
{
    int st = check_ready(ctx, false);
    if (st != PRT_OK) return st;
    if (nodeCount) *nodeCount = ctx->bvh.nodeCount;
    if (triCount) *triCount = ctx->bvh.triCount;
    CK(cudaSetDevice(ctx->device));
    if (nodes && nodeCapacity >= ctx->bvh.nodeCount && ctx->bvh.nodeCount > 0)
        CK(cudaMemcpy(nodes, ctx->bvh.nodes, sizeof(Bvh8Node) * (size_t)ctx->bvh.nodeCount, cudaMemcpyDeviceToHost));
    if (tris && triCapacity >= ctx->bvh.triCount && ctx->bvh.triCount > 0)
        CK(cudaMemcpy(tris, ctx->bvh.tris, sizeof(TriRec) * (size_t)ctx->bvh.triCount, cudaMemcpyDeviceToHost));
    return PRT_OK;
}

int prt_read_counters(prt_ctx* ctx, long long* out, int n, int reset)
{
    if (!ctx || !out || n < 6) return PRT_EINVAL;
    CK(cudaSetDevice(ctx->device));
    unsigned long long c[8];
    int r = read_counters(c, reset != 0, ctx->stream);
    if (r < 0) return fail(ctx, PRT_ESTATE, "library built without traversal counters (-DPRT_COUNTERS=1)");
    if (r > 0) return fail(ctx, PRT_ECUDA, "counter read-back failed");
    for (int i = 0; i < 6; ++i) out[i] = (long long)c[i];
    return PRT_OK;
}

int prt_debug_fail_allocations(long long afterCount)
{
    prt_b200::g_allocFailAfter = afterCount < 0 ? -1 : afterCount;
    return PRT_OK;
}

int prt_set_tune(prt_ctx* ctx, const prt_tune* t)
{
    if (!ctx || !t) return PRT_EINVAL;
    if (t->blockSize < 32 || t->blockSize > 128 || (t->blockSize & 31) || t->blocksPerSM < 0 || t->blocksPerSM > 64 ||
        t->pathsPerWave < 0 || t->concurrentWaves < 0 || t->primaryPackets < 0 || t->primaryPackets > 2)
        return fail(ctx, PRT_EINVAL, "invalid launch configuration");
    ctx->cfg.packet = t->primaryPackets;
    ctx->cfg.block = t->blockSize;
    ctx->cfg.blocksPerSM = t->blocksPerSM;
    ctx->cfg.pathsPerWave = t->pathsPerWave;
    ctx->cfg.chains = t->concurrentWaves > 0 ? std::min(t->concurrentWaves, kMaxChains) : ctx->cfg.chains;
    clear_graphs(ctx);
    return PRT_OK;
}

int prt_get_tune(prt_ctx* ctx, prt_tune* t)
{
    if (!ctx || !t) return PRT_EINVAL;
    t->blockSize = ctx->cfg.block;
    t->blocksPerSM = ctx->cfg.blocksPerSM;
    t->pathsPerWave = ctx->cfg.pathsPerWave;
    t->concurrentWaves = ctx->cfg.chains;
    t->primaryPackets = ctx->cfg.packet;
    t->mray = 0;
    return PRT_OK;
}

int prt_autotune(prt_ctx* ctx, int spp, int maxDepth, prt_tune* best)
{
    int st = check_ready(ctx, true);
    if (st != PRT_OK) return st;
    if (spp <= 0 || maxDepth < 0 || maxDepth > kMaxDepthCap)
        return fail(ctx, PRT_EINVAL, "autotune needs spp > 0 and 0 <= maxDepth <= 64");
    CK(cudaSetDevice(ctx->device));
    const long long perPass = (long long)((ctx->W + 7) / 8) * ((ctx->H + 7) / 8) * 64;
    const LaunchCfg saved = ctx->cfg;

    // Throughput of one configuration: the best of three timed renders of the
    // caller's workload after one untimed render (which also records and
    // instantiates the configuration's graph).  Repeated renders of the same
    // work vary by well under 0.1%.
    auto measure = [&](const LaunchCfg& cfg, double* mray) -> int {
        ctx->cfg = cfg;
        clear_graphs(ctx);
        *mray = 0;
        for (int rep = 0; rep < 4; ++rep)
        {
            prt_render_stats rs;
            CK(cudaMemsetAsync(ctx->dPass, 0, sizeof(int), ctx->stream));
            int s2 = prt_render(ctx, spp, maxDepth, 0, &rs);
            if (s2 != PRT_OK) return s2;
            if (rep > 0) *mray = std::max(*mray, rs.mray);
        }
        return PRT_OK;
    };

    // Candidate values per parameter.  Wave sizes: the automatic size and 1..16
    // passes of this frame (at least 64K and at most 64M paths).
    std::vector<long long> waveOpts = {0};
    for (long long k : {1, 2, 4, 8, 16})
    {
        long long ppw = std::min<long long>(std::max<long long>(perPass * k, 1 << 16), 1LL << 26);
        if (std::find(waveOpts.begin(), waveOpts.end(), ppw) == waveOpts.end()) waveOpts.push_back(ppw);
    }
    const int chainOpts[] = {1, 2, 3, 4};
    const int perSMOpts[] = {0, 4, 6};
    const int blockOpts[] = {64, 128};

    // Coordinate descent from the current configuration: one parameter at a
    // time (traversal mode, wave size, concurrent waves, blocks per SM, block
    // size), a candidate replaces the incumbent only if it is more than 0.3%
    // faster, at most three sweeps.
    LaunchCfg cur = saved;
    double curM = 0;
    st = measure(cur, &curM);
    for (int sweep = 0; sweep < 3 && st == PRT_OK; ++sweep)
    {
        bool improved = false;
        auto consider = [&](LaunchCfg c) -> int {
            if (c.block == cur.block && c.blocksPerSM == cur.blocksPerSM && c.pathsPerWave == cur.pathsPerWave &&
                c.chains == cur.chains && c.packet == cur.packet)
                return PRT_OK;
            double m = 0;
            int s2 = measure(c, &m);
            if (s2 == PRT_OK && m > curM * 1.003)
            {
                cur = c;
                curM = m;
                improved = true;
            }
            return s2;
        };
        for (int pk = 0; pk <= 2 && st == PRT_OK; ++pk)
        {
            LaunchCfg c = cur;
            c.packet = pk;
            st = consider(c);
        }
        for (long long w : waveOpts)
        {
            if (st != PRT_OK) break;
            LaunchCfg c = cur;
            c.pathsPerWave = (int)w;
            st = consider(c);
        }
        for (int ch : chainOpts)
        {
            if (st != PRT_OK) break;
            LaunchCfg c = cur;
            c.chains = ch;
            st = consider(c);
        }
        for (int b : perSMOpts)
        {
            if (st != PRT_OK) break;
            LaunchCfg c = cur;
            c.blocksPerSM = b;
            st = consider(c);
        }
        for (int b : blockOpts)
        {
            if (st != PRT_OK) break;
            LaunchCfg c = cur;
            c.block = b;
            st = consider(c);
        }
        if (!improved) break;
    }
    if (st != PRT_OK)
    {
        ctx->cfg = saved;
        clear_graphs(ctx);
        return st;
    }
    ctx->cfg = cur;
    // the candidates may have grown the queues beyond what the winner needs
    // (up to 4 chains of 64M-path waves): free them, the next render
    // allocates its own
    CK(cudaStreamSynchronize(ctx->stream));
    release_queues(ctx);
    st = prt_clear(ctx);
    if (st != PRT_OK) return st;
    if (best)
    {
        best->blockSize = cur.block;
        best->blocksPerSM = cur.blocksPerSM;
        best->pathsPerWave = cur.pathsPerWave;
        best->concurrentWaves = cur.chains;
        best->primaryPackets = cur.packet;
        best->mray = curM;
    }
    return PRT_OK;
}

int prt_build_mesh(prt_ctx* ctx, const prt_soup_triangle* tris, int triCount, const char* const* materialNames,
                   int materialCount, prt_mesh_info* info)
{
    if (!ctx) return PRT_EINVAL;
    if (triCount < 0 || (triCount > 0 && !tris)) return fail(ctx, PRT_EINVAL, "invalid soup");
    if (materialCount < 0 || (materialCount > 0 && !materialNames)) return fail(ctx, PRT_EINVAL, "invalid material names");
    for (int i = 0; i < materialCount; ++i)
        if (!materialNames[i]) return fail(ctx, PRT_EINVAL, "null material name");
    CK(cudaSetDevice(ctx->device));
    const auto t0 = std::chrono::steady_clock::now();
    double buildMs = 0;
    int st = build_mesh_gpu(tris, triCount, ctx->stream, ctx->builtMesh, ctx->err, &buildMs, &ctx->launches, false,
                            &ctx->buildScratch);
    if (st != PRT_OK) return st;
    const auto t1 = std::chrono::steady_clock::now();
    BuiltMesh& m = ctx->builtMesh;
    m.names.assign(materialNames, materialNames + materialCount);
    if (info)
    {
        info->triCount = m.triCount;
        info->vertCount = m.vertCount;
        info->hasNormals = m.hasNormals;
        info->hasTexcoords = m.hasTexcoords;
        info->hasMaterials = m.hasMaterials;
        std::memcpy(info->boundsLo, m.lo, sizeof(m.lo));
        std::memcpy(info->boundsHi, m.hi, sizeof(m.hi));
        info->buildMs = buildMs;
        info->totalMs = std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    return PRT_OK;
}

int prt_build_mesh_soup(prt_ctx* ctx, const prt_soup* soup, prt_mesh_info* info)
{
    if (!ctx) return PRT_EINVAL;
    SoupIndexed s;
    if (!soup_indexed(soup, &s)) return fail(ctx, PRT_EINVAL, "null soup");
    CK(cudaSetDevice(ctx->device));
    const auto t0 = std::chrono::steady_clock::now();
    double buildMs = 0;
    int st = build_mesh_gpu_indexed(s, ctx->stream, ctx->builtMesh, ctx->err, &buildMs, &ctx->launches,
                                    &ctx->buildScratch, &ctx->uploadScratch);
    if (st != PRT_OK) return st;
    const auto t1 = std::chrono::steady_clock::now();
    BuiltMesh& m = ctx->builtMesh;
    int names = 0;
    prt_soup_info(soup, nullptr, &names, nullptr);
    m.names.clear();
    for (int i = 0; i < names; ++i) m.names.push_back(prt_soup_material_name(soup, i));
    if (info)
    {
        info->triCount = m.triCount;
        info->vertCount = m.vertCount;
        info->hasNormals = m.hasNormals;
        info->hasTexcoords = m.hasTexcoords;
        info->hasMaterials = m.hasMaterials;
        std::memcpy(info->boundsLo, m.lo, sizeof(m.lo));
        std::memcpy(info->boundsHi, m.hi, sizeof(m.hi));
        info->buildMs = buildMs;
        info->totalMs = std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    return PRT_OK;
}

int prt_read_built_mesh(prt_ctx* ctx, int* indices, int* materialIds, float* positions, float* normals, float* texcoords)
{
    if (!ctx) return PRT_EINVAL;
    const BuiltMesh& m = ctx->builtMesh;
    if (!m.valid) return fail(ctx, PRT_ESTATE, "no mesh has been built");
    if ((m.triCount && (!indices || !materialIds)) || (m.vertCount && !positions) ||
        (m.vertCount && m.hasNormals && !normals) || (m.vertCount && m.hasTexcoords && !texcoords))
        return fail(ctx, PRT_EINVAL, "null output array");
    CK(cudaSetDevice(ctx->device));
    if (m.triCount)
    {
        CK(cudaMemcpyAsync(indices, m.idx, sizeof(int) * 3 * (size_t)m.triCount, cudaMemcpyDefault, ctx->stream));
        CK(cudaMemcpyAsync(materialIds, m.mat, sizeof(int) * (size_t)m.triCount, cudaMemcpyDefault, ctx->stream));
    }
    if (m.vertCount)
    {
        // de-interleave with strided copies: position, normal and texcoord columns
        const size_t pitch = sizeof(float) * m.stride;
        CK(cudaMemcpy2DAsync(positions, 12, m.attr, pitch, 12, m.vertCount, cudaMemcpyDefault, ctx->stream));
        if (m.hasNormals)
            CK(cudaMemcpy2DAsync(normals, 12, m.attr + 3, pitch, 12, m.vertCount, cudaMemcpyDefault, ctx->stream));
        if (m.hasTexcoords)
            CK(cudaMemcpy2DAsync(texcoords, 8, m.attr + (m.hasNormals ? 6 : 3), pitch, 8, m.vertCount,
                                 cudaMemcpyDefault, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return PRT_OK;
}

int prt_save_built_mesh(prt_ctx* ctx, const char* path)
{
    if (!ctx || !path) return PRT_EINVAL;
    const BuiltMesh& m = ctx->builtMesh;
    if (!m.valid) return fail(ctx, PRT_ESTATE, "no mesh has been built");
    CK(cudaSetDevice(ctx->device));
    // the blob in one host buffer: header, indices, material ids, attributes,
    // names (ordinary memory: pinning a buffer for one copy costs more than
    // the pageable copy saves)
    const size_t idxBytes = 12 * (size_t)m.triCount, matBytes = 4 * (size_t)m.triCount;
    const size_t attrBytes = sizeof(float) * m.stride * (size_t)m.vertCount;
    size_t namesBytes = 4;
    for (const std::string& s : m.names) namesBytes += 4 + s.size();
    const size_t total = 38 + idxBytes + matBytes + attrBytes + namesBytes;
    std::unique_ptr<char[]> owner(new (std::nothrow) char[total]);
    char* buf = owner.get();
    if (!buf) return fail(ctx, PRT_ENOMEM, "cannot allocate the host blob buffer");
    const int id = 0x04df8666, tri = m.triCount, vert = m.vertCount;
    std::memcpy(buf, &id, 4);
    std::memcpy(buf + 4, m.lo, 12);
    std::memcpy(buf + 16, m.hi, 12);
    std::memcpy(buf + 28, &tri, 4);
    std::memcpy(buf + 32, &vert, 4);
    buf[36] = m.hasNormals ? 1 : 0;
    buf[37] = m.hasTexcoords ? 1 : 0;
    char* at = buf + 38;
    if (idxBytes) CK(cudaMemcpyAsync(at, m.idx, idxBytes, cudaMemcpyDeviceToHost, ctx->stream));
    at += idxBytes;
    if (matBytes) CK(cudaMemcpyAsync(at, m.mat, matBytes, cudaMemcpyDeviceToHost, ctx->stream));
    at += matBytes;
    if (attrBytes) CK(cudaMemcpyAsync(at, m.attr, attrBytes, cudaMemcpyDeviceToHost, ctx->stream));
    at += attrBytes;
    const int count = (int)m.names.size();
    std::memcpy(at, &count, 4);
    at += 4;
    for (const std::string& s : m.names)
    {
        const int len = (int)s.size();
        std::memcpy(at, &len, 4);
        std::memcpy(at + 4, s.data(), s.size());
        at += 4 + s.size();
    }
    CK(cudaStreamSynchronize(ctx->stream));
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(ctx, PRT_EIO, std::string("cannot create ") + path);
    const bool ok = std::fwrite(buf, 1, total, f) == total;
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) return fail(ctx, PRT_EIO, std::string("write error: ") + path);
    return PRT_OK;
}

} // extern "C"

namespace prt_b200 {

// Read-only view of a context for prt_render_noalloc (noalloc.cu).
int ctx_noalloc_view(prt_ctx* ctx, SceneDev* scene, int* device, cudaStream_t* stream, int* numSMs, LaunchCfg* cfg,
                     float* sky, bool* albedo, bool* nee)
{
    if (!ctx->built) return fail(ctx, PRT_ESTATE, "acceleration structure not built (prt_build_accel)");
    *scene = scene_dev(ctx);
    *device = ctx->device;
    *stream = ctx->stream;
    *numSMs = ctx->numSMs;
    *cfg = ctx->cfg;
    *sky = ctx->sky;
    *albedo = ctx->dAlbedo != nullptr;
    *nee = ctx->integrator == PRT_INTEGRATOR_DIFFUSE2;
    return PRT_OK;
}

int ctx_fail(prt_ctx* ctx, int status, const char* msg) { return fail(ctx, status, msg); }

} // namespace prt_b200
