// prt_render_noalloc: the wavefront render with its scratch memory in a
// fixed, file-scope device array instead of memory allocated per context.
//
// Some callers cannot allocate device memory when they render: a host
// application that has already reserved (nearly) the whole GPU for its own
// memory pool, where cudaMalloc would fail or fragment that pool, or a frame
// loop with a hard latency budget, where cudaMalloc's implicit device
// synchronisation is not acceptable.  This entry point serves them: it calls
// no cudaMalloc, cudaFree or other allocating routine.  The caller passes the
// inputs (a context whose scene and acceleration structure are already built,
// and a camera) and the output (a device accumulation buffer it owns); the
// path queues and counters live in g_scratch below.
//
// Limits and sharing rules:
//   * the frame may hold at most kNoAllocMaxPaths pixels after rounding up to
//     8x8 tiles (524288, e.g. 1024x512 or 960x544); larger frames are
//     rejected with PRT_EINVAL;
//   * g_scratch occupies 40 MiB on every GPU that loads the library, until the
//     process exits;
//   * all calls on a device share g_scratch, which keeps the last call's
//     contents: each call clears the counters it needs before using them, and
//     calls that overlap on the GPU (concurrent streams or host threads) race
//     on the shared queues — serialise them;
//   * the first call in a CUDA context of a device looks up the array's device
//     address in that context (with that device current) and caches it; make
//     that first call before any stream capture on the calling thread.  A
//     later context on the same device (after cudaDeviceReset, for example)
//     is recognised by its context id and looked up again;
//   * the caller's current device is restored before the call returns.
#include <cuda.h>

#include <cstdint>
#include <mutex>

#include "prt_internal.h"

namespace prt_b200 {

namespace {

constexpr long long kNoAllocMaxPaths = 1LL << 19;
constexpr int kNoAllocCounters = 64 + 2;   // one slot per bounce depth (max depth 64) + 2

struct NoAllocScratch
{
    PathRec queue[2][kNoAllocMaxPaths];
    float thr[2][kNoAllocMaxPaths];   // per-path throughput (per-triangle albedo)
    float L[2][kNoAllocMaxPaths];     // radiance gathered so far (next-event estimation)
    int counts[kNoAllocCounters];
    int fetch[kNoAllocCounters];
    unsigned long long rays;
    int passBase;
};

static __device__ __align__(256) NoAllocScratch g_scratch;

constexpr int kMaxDevices = 64;

struct AddressCache
{
    unsigned long long ctxId = 0;   // CUDA context the address belongs to (0: none yet)
    NoAllocScratch* addr = nullptr;
};

std::mutex g_lock;
AddressCache g_cache[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the CUDA context current on this thread, through the driver entry
// points the runtime hands out (no link against libcuda needed).
cudaError_t current_context_id(unsigned long long* id)
{
    static CtxGetCurrentFn getCurrent = nullptr;
    static CtxGetIdFn getId = nullptr;
    if (!getCurrent || !getId)
    {
        void* f0 = nullptr;
        void* f1 = nullptr;
        cudaDriverEntryPointQueryResult q0, q1;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0);
        if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1);
        if (e != cudaSuccess) return e;
        if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
            return cudaErrorSymbolNotFound;
        getCurrent = reinterpret_cast<CtxGetCurrentFn>(f0);
        getId = reinterpret_cast<CtxGetIdFn>(f1);
    }
    CUcontext c = nullptr;
    if (getCurrent(&c) != CUDA_SUCCESS || !c) return cudaErrorDeviceUninitialized;
    if (getId(c, id) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
    return cudaSuccess;
}

// Device address of g_scratch in the current context of `device` (which is
// current); looked up once per context.
cudaError_t scratch_address(int device, NoAllocScratch** out)
{
    unsigned long long id = 0;
    cudaError_t e = current_context_id(&id);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> guard(g_lock);
    AddressCache& c = g_cache[device];
    if (c.ctxId != id || !c.addr)
    {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return e;
        c.addr = static_cast<NoAllocScratch*>(p);
        c.ctxId = id;
    }
    *out = c.addr;
    return cudaSuccess;
}

// Restores the caller's current device when the call returns.
struct DeviceRestore
{
    int prev = -1;
    DeviceRestore()
    {
        if (cudaGetDevice(&prev) != cudaSuccess)
        {
            cudaGetLastError();
            prev = -1;
        }
    }
    ~DeviceRestore()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// accum must be device (or managed) memory of `device`, 16-byte aligned (the
// kernels add float4 records to it).
bool accum_usable(const float* accum, int device)
{
    if (reinterpret_cast<uintptr_t>(accum) % 16 != 0) return false;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, accum) != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    if (attr.type == cudaMemoryTypeManaged) return true;
    return attr.type == cudaMemoryTypeDevice && attr.device == device;
}

} // namespace

// Scene/camera/stream accessors of the context (prt_api.cu).
int ctx_noalloc_view(prt_ctx* ctx, SceneDev* scene, int* device, cudaStream_t* stream, int* numSMs, LaunchCfg* cfg,
                     float* sky, bool* albedo, bool* nee);
int ctx_fail(prt_ctx* ctx, int status, const char* msg);

} // namespace prt_b200

using namespace prt_b200;

extern "C" int prt_render_noalloc(prt_ctx* ctx, const prt_camera* cam, int width, int height, int pass0, int spp,
                                  int maxDepth, float* accum, long long* rays)
{
    if (!ctx) return PRT_EINVAL;
    SceneDev scene;
    int device = 0, numSMs = 0;
    cudaStream_t stream = nullptr;
    LaunchCfg cfg;
    float sky = 1.0f;
    bool albedo = false, nee = false;
    int st = ctx_noalloc_view(ctx, &scene, &device, &stream, &numSMs, &cfg, &sky, &albedo, &nee);
    if (st != PRT_OK) return st;
    if (!cam || !accum || width <= 0 || height <= 0 || pass0 < 0 || spp < 0 || maxDepth < 0 ||
        maxDepth > kNoAllocCounters - 2)
        return ctx_fail(ctx, PRT_EINVAL, "prt_render_noalloc: invalid argument");
    const int tilesX = (width + 7) / 8, tilesY = (height + 7) / 8;
    const long long perPass = (long long)tilesX * tilesY * 64;
    if (perPass > kNoAllocMaxPaths)
        return ctx_fail(ctx, PRT_EINVAL,
                        "prt_render_noalloc: frame too large (at most 524288 pixels after rounding to 8x8 tiles)");
    if (device < 0 || device >= kMaxDevices) return ctx_fail(ctx, PRT_EINVAL, "prt_render_noalloc: device index");
    DeviceRestore restore;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return ctx_fail(ctx, PRT_ECUDA, cudaGetErrorString(e));
    if (!accum_usable(accum, device))
        return ctx_fail(ctx, PRT_EINVAL,
                        "prt_render_noalloc: accum must be 16-byte aligned device memory of the context's GPU");
    NoAllocScratch* s = nullptr;
    e = scratch_address(device, &s);
    if (e != cudaSuccess) return ctx_fail(ctx, PRT_ECUDA, cudaGetErrorString(e));

    const int passesPerWave = (int)std::max<long long>(1, kNoAllocMaxPaths / perPass);
    WaveArgs a;
    a.scene = scene;
    a.cam.origin = make_float3(cam->origin[0], cam->origin[1], cam->origin[2]);
    a.cam.basisU = make_float3(cam->basisU[0], cam->basisU[1], cam->basisU[2]);
    a.cam.basisV = make_float3(cam->basisV[0], cam->basisV[1], cam->basisV[2]);
    a.cam.imageO = make_float3(cam->imageO[0], cam->imageO[1], cam->imageO[2]);
    a.cam.imageDx = make_float3(cam->imageDx[0], cam->imageDx[1], cam->imageDx[2]);
    a.cam.imageDy = make_float3(cam->imageDy[0], cam->imageDy[1], cam->imageDy[2]);
    a.cam.lensRadius = cam->lensRadius;
    a.cam.focalDistance = cam->focalDistance;
    a.cam.invW = 1.0f / (float)width;
    a.cam.invH = 1.0f / (float)height;
    a.cam.width = width;
    a.cam.height = height;
    a.accum = reinterpret_cast<float4*>(accum);
    a.counts = s->counts;
    a.fetch = s->fetch;
    a.rays = &s->rays;
    a.passBase = &s->passBase;
    a.tilesX = tilesX;
    a.tilesY = tilesY;
    a.maxDepth = maxDepth;
    a.sky = sky;

    // the pass base stays 0: the kernels get pass0 + offset as the wave offset
    e = cudaMemsetAsync(&s->rays, 0, sizeof(unsigned long long) + sizeof(int), stream);
    for (int p0 = 0; p0 < spp && e == cudaSuccess; p0 += passesPerWave)
    {
        a.passOffset = pass0 + p0;
        a.passes = std::min(passesPerWave, spp - p0);
        e = cudaMemsetAsync(s->counts, 0, sizeof(int) * 2 * kNoAllocCounters, stream);
        for (int d = 0; d <= maxDepth && e == cudaSuccess; ++d)
        {
            a.qin = d == 0 ? nullptr : s->queue[(d - 1) & 1];
            a.qout = s->queue[d & 1];
            a.thrIn = albedo && d > 0 ? s->thr[(d - 1) & 1] : nullptr;
            a.thrOut = albedo ? s->thr[d & 1] : nullptr;
            a.Lin = nee && d > 0 ? s->L[(d - 1) & 1] : nullptr;
            a.Lout = nee ? s->L[d & 1] : nullptr;
            float t = 1.0f;
            for (int k = 0; k < d; ++k) t *= 0.8f;
            a.thrConst = t;
            launch_bounce(a, d, cfg, numSMs, stream);
            e = cudaGetLastError();
        }
    }
    unsigned long long total = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, &s->rays, sizeof(total), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return ctx_fail(ctx, PRT_ECUDA, cudaGetErrorString(e));
    if (rays) *rays = (long long)total;
    return PRT_OK;
}
