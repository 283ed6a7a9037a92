// Kernels of the wavefront diffuse path tracer.
//
// The reference GPU path (render/diffuse_renderer_cuda.cu:159-212) runs, per
// pass: generateRaysKernel -> { OptiX Prime closest hit -> cudaMemcpy(counter)
// -> shadeRaysKernel -> cudaMemcpy(count) } per bounce.  Here one persistent
// kernel per bounce does traversal, shading, queue compaction and
// accumulation together; primary rays are generated inside the first bounce
// kernel; queue sizes stay on the device, so a whole render is launched
// without host synchronisation (and is captured as a CUDA graph by the API).
#include <algorithm>

#include "prt_internal.h"

namespace prt_b200 {

#ifndef PRT_COUNTERS
#define PRT_COUNTERS 0
#endif

// Traversal counters of the bounce kernel, compiled in with -DPRT_COUNTERS=1
// (the reference's RayStats nodeCount/primCount, core/ray_stats.h:23-28):
//   [0] node visits  [1] triangle tests  [2] rays  [3] warp traversal steps
//   [4] running lanes summed over steps  [5] warp triangle-loop iterations
//   (max over the running lanes of a step, summed)
__device__ unsigned long long g_counters[8];

namespace {

__device__ __forceinline__ void morton8x8(int m, int& x, int& y)
{
    // same order as the reference's mortonTableX/Y (image/morton.cpp)
    x = (m & 1) | ((m >> 1) & 2) | ((m >> 2) & 4);
    y = ((m >> 1) & 1) | ((m >> 2) & 2) | ((m >> 3) & 4);
}

// Pixel of item rr (< tilesX * tilesY * 64) of one pass of a wave: 8x8 tiles
// in row order, Morton order inside a tile (image/morton.cpp's tables).
// Returns false for items past the frame's right or bottom edge.
__device__ __forceinline__ bool wave_item_pixel(int rr, int tilesX, int W, int H, int& x, int& y)
{
    int tile = rr >> 6;
    int mx, my;
    morton8x8(rr & 63, mx, my);
    x = (tile % tilesX) * 8 + mx;
    y = (tile / tilesX) * 8 + my;
    return x < W && y < H;
}

__device__ __forceinline__ PathRec load_path(const PathRec* q, int i)
{
    const float4* p = reinterpret_cast<const float4*>(q + i);
    PathRec r;
    r.w0 = __ldcs(p);
    r.w1 = __ldcs(p + 1);
    return r;
}

__device__ __forceinline__ void store_path(PathRec* q, int i, float3 org, int tag, float3 dir, uint32_t rng)
{
    float4* p = reinterpret_cast<float4*>(q + i);
    __stcs(p, make_float4(org.x, org.y, org.z, __int_as_float(tag)));
    __stcs(p + 1, make_float4(dir.x, dir.y, dir.z, __uint_as_float(rng)));
}

// Warp-aggregated append: one atomic per warp, survivors keep lane order.
__device__ __forceinline__ int warp_append(bool pred, int* counter)
{
    const unsigned lane = threadIdx.x & 31u;
    unsigned m = __ballot_sync(0xffffffffu, pred);
    int base = 0;
    if (lane == 0 && m) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    return base + __popc(m & ((1u << lane) - 1u));
}

// Deferred triangle tests per kernel (see warp_trav_deferred): the path-replay
// megakernel, the intersector seam and the diffuse2 bounce have their own switches.
#ifndef PRT_DEFER_REPLAY
#define PRT_DEFER_REPLAY PRT_DEFER_TRIS
#endif
#ifndef PRT_DEFER_ISECT
#define PRT_DEFER_ISECT PRT_DEFER_TRIS
#endif
#ifndef PRT_DEFER_NEE
#define PRT_DEFER_NEE PRT_DEFER_TRIS
#endif

// Lanes refill once at least this many of a warp's 32 lanes are idle
// (persistent threads with dynamic ray fetch, Aila & Laine, HPG 2009).
#ifndef PRT_REFILL_MIN
#define PRT_REFILL_MIN 12
#endif
constexpr int kRefillMin = PRT_REFILL_MIN;

// Paired FP32 FMAs in the node test (node_hits1<true>): the six plane FMAs of
// two children become three fma.rn.f32x2.  First-bounce kernels, per-lane and
// packet: depth 0 of the terrain 4% / 7% faster, of the 10M field 6% / 8%.
#ifndef PRT_PAIRED_FIRST
#define PRT_PAIRED_FIRST 1
#endif
#ifndef PRT_PAIRED_PACKET
#define PRT_PAIRED_PACKET 1
#endif

// Later bounces keep only a path's origin and its traversal terms in registers
// while the warp traverses: the pixel, RNG state and direction are read again
// from the input queue when the lane shades.  That frees the registers the
// paired node test needs there (with the path kept in registers it spilled and
// ran 2-3% slower); with both, bounces 1-5 of the terrain run 3% faster.
#ifndef PRT_RELOAD_PATH
#define PRT_RELOAD_PATH 1
#endif
#ifndef PRT_PAIRED_LATER
#define PRT_PAIRED_LATER 1
#endif

// Paired node test in the later bounces of the next-event-estimation kernel
// (k_bounce_nee; diffuse2 on the terrain frame at 16 spp 2281 -> 2319 Mrays/s);
// its first bounce keeps single FMAs (paired, it spills 128 bytes).
#ifndef PRT_PAIRED_NEE
#define PRT_PAIRED_NEE 1
#endif

// Paired node test in the any-hit ray-query kernel (k_intersect<true>): 4M
// incoherent occlusion queries on the terrain 1.085 -> 1.024 ms; closest-hit
// queries keep single FMAs (paired, they spill and took 1.358 instead of 1.305).
#ifndef PRT_PAIRED_QUERY
#define PRT_PAIRED_QUERY 1
#endif

// Minimum resident 128-thread blocks per SM requested from the compiler for
// the bounce kernel (8 caps it at 64 registers per thread).
#ifndef PRT_BOUNCE_MIN_BLOCKS
#define PRT_BOUNCE_MIN_BLOCKS 8
#endif

// One bounce of the wavefront over the queue of paths entering `depth`.
// kFirst: the queue is implicit — item i is (pass, 8x8 tile, Morton index)
// and the primary ray is generated in registers.
//
// Each warp keeps 32 rays in flight.  Traversal advances one 8-wide node per
// step; as soon as kRefillMin lanes have finished, the finished lanes shade
// their hit (or accumulate), append survivors to the next queue with one
// atomic per warp, and fetch fresh rays, so a few long rays do not idle the
// rest of the warp.
template <bool kFirst, bool kAlbedo>
__global__ void __launch_bounds__(128, PRT_BOUNCE_MIN_BLOCKS) k_bounce(WaveArgs a, int depth)
{
    extern __shared__ uint2 s_stack[];
    TravStack st;
    st.sh = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    st.overflow = false;
    // this warp's triangle queue, after the block's stack columns
    TriQueue* tq = reinterpret_cast<TriQueue*>(s_stack + kShared * blockDim.x) + (threadIdx.x >> 5);
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned ltMask = (1u << lane) - 1u;
    const int W = a.cam.width, H = a.cam.height;
    const int perPass = a.tilesX * a.tilesY * 64;
    int total;
    int pass0 = 0;
    if (kFirst)
    {
        total = a.passes * perPass;
        pass0 = *a.passBase + a.passOffset;
    }
    else
    {
        total = *(volatile int*)&a.counts[depth];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicAdd(a.rays, kFirst ? (unsigned long long)a.passes * (unsigned long long)W * (unsigned long long)H
                                 : (unsigned long long)total);
    const bool final = depth == a.maxDepth;

    bool has = false;         // this lane holds a ray
    bool exhausted = false;   // warp-uniform: every queue entry has been claimed
    uint32_t cNodes = 0, cTris = 0, cRays = 0;                          // per lane (PRT_COUNTERS)
    unsigned long long cSteps = 0, cLaneSteps = 0, cTriIters = 0;       // per warp (PRT_COUNTERS)
    int pixel = 0;
    uint32_t rng = 0;
    int qi = 0;               // input-queue index of this lane's path (PRT_RELOAD_PATH)
    float thr = 0.f;
    TravRay r;
    TravState ts;
    ts.done = true;
    for (;;)
    {
        // --- refill idle lanes ---------------------------------------------
        unsigned idle = __ballot_sync(FULL, !has);
        if (!exhausted && (__popc(idle) >= kRefillMin || idle == FULL))
        {
            int n = __popc(idle);
            int base = 0;
            if (lane == 0) base = atomicAdd(&a.fetch[depth], n);
            base = __shfl_sync(FULL, base, 0);
            if (base + n >= total) exhausted = true;
            int i = base + __popc(idle & ltMask);
            if (!has && i < total)
            {
                float3 org, dir;
                bool ok = true;
                if (kFirst)
                {
                    int pass = i / perPass;
                    int x, y;
                    if (!wave_item_pixel(i - pass * perPass, a.tilesX, W, H, x, y))
                    {
                        ok = false;
                    }
                    else
                    {
                        pixel = x + y * W;
                        rng = rng_seed(pass0 + pass, pixel);
                        camera_ray(a.cam, x, y, rng, org, dir);
                        thr = kAlbedo ? 1.0f : a.thrConst;
                    }
                }
                else if (PRT_RELOAD_PATH)
                {
                    // L2 only: the record is read again (pixel, RNG, direction) when
                    // the lane shades
                    const float4* p = reinterpret_cast<const float4*>(a.qin + i);
                    const float4 w0 = __ldcg(p), w1 = __ldcg(p + 1);
                    org = f3(w0.x, w0.y, w0.z);
                    dir = f3(w1.x, w1.y, w1.z);
                    qi = i;
                    thr = kAlbedo ? __ldcs(a.thrIn + i) : a.thrConst;
                }
                else
                {
                    PathRec pr = load_path(a.qin, i);
                    org = f3(pr.w0.x, pr.w0.y, pr.w0.z);
                    pixel = __float_as_int(pr.w0.w);
                    dir = f3(pr.w1.x, pr.w1.y, pr.w1.z);
                    rng = __float_as_uint(pr.w1.w);
                    thr = kAlbedo ? __ldcs(a.thrIn + i) : a.thrConst;
                }
                if (ok)
                {
                    has = true;
                    trav_setup(r, org, dir);
                    trav_init(ts, a.scene, FLT_MAX, st);
                }
            }
        }
        if (__ballot_sync(FULL, has) == 0)
        {
            if (exhausted) break;
            continue;
        }
        // --- traverse until the warp has enough idle lanes ------------------
        if (PRT_DEFER_TRIS && a.scene.deferTris)
        {
            // node visits queue their triangles; the warp tests them 32 at a
            // time, and every pending test is done before any lane shades
            constexpr bool kPair = kFirst ? PRT_PAIRED_FIRST : (PRT_RELOAD_PATH && PRT_PAIRED_LATER);
            warp_trav_deferred<kPair>(*tq, ts, a.scene, r, 0.0f, st, has, !exhausted, kRefillMin, lane,
                                      PRT_COUNTERS ? &cNodes : nullptr, PRT_COUNTERS ? &cTris : nullptr,
                                      PRT_COUNTERS ? &cSteps : nullptr, PRT_COUNTERS ? &cLaneSteps : nullptr,
                                      PRT_COUNTERS ? &cTriIters : nullptr);
        }
        else
        for (;;)
        {
            if (PRT_COUNTERS)
            {
                unsigned run0 = __ballot_sync(FULL, has && !ts.done);
                uint32_t tris = 0;
                if (has && !ts.done) trav_step<false>(ts, a.scene, r, 0.0f, st, &cNodes, &tris);
                cTris += tris;
                cLaneSteps += __popc(run0);
                cSteps += 1;
                cTriIters += __reduce_max_sync(FULL, tris);
            }
            else if (has && !ts.done)
            {
                trav_step<false>(ts, a.scene, r, 0.0f, st);
            }
            unsigned running = __ballot_sync(FULL, has && !ts.done);
            if (running == 0) break;
            if (!exhausted && 32 - __popc(running) >= kRefillMin) break;
        }
        // --- finish the lanes whose traversal is complete ---------------------
        // (the finished path's pixel, RNG state and rays are iteration-local, so
        // only what traversal needs is carried around the loop)
        const bool fin = has && ts.done;
        bool cont = false;
        float contrib = 0.f;
        int fpix = 0;
        uint32_t frng = 0;
        float3 forg = r.org, fdir = f3(0.f, 0.f, 0.f);
        if (fin)
        {
            if (!kFirst && PRT_RELOAD_PATH)
            {
                const float4* p = reinterpret_cast<const float4*>(a.qin + qi);
                const float4 w1 = __ldcs(p + 1);
                fpix = __float_as_int(__ldcs(reinterpret_cast<const float*>(p) + 3));
                fdir = f3(w1.x, w1.y, w1.z);
                frng = __float_as_uint(w1.w);
            }
            else
            {
                fpix = pixel;
                fdir = r.dir;
                frng = rng;
            }
            if (ts.triHit < 0)
            {
                contrib = __fmul_rn(thr, a.sky);
            }
            else if (!final)
            {
                if (kAlbedo) thr = __fmul_rn(thr, a.scene.albedo ? __ldg(a.scene.albedo + ts.primHit) : 0.8f);
                diffuse_bounce(a.scene.tris, ts.triHit, forg, fdir, ts.tHit, frng);
                cont = true;
            }
        }
        int o = warp_append(cont, &a.counts[depth + 1]);
        if (cont)
        {
            store_path(a.qout, o, forg, fpix, fdir, frng);
            if (kAlbedo) __stcs(a.thrOut + o, thr);
        }
        else if (fin)
        {
            red_add_v4(a.accum + fpix, contrib, contrib, contrib, 1.0f);
        }
        if (fin)
        {
            has = false;
            ++cRays;
        }
    }
    if (PRT_COUNTERS)
    {
        unsigned long long n = cNodes, t = cTris, ry = cRays;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            n += __shfl_down_sync(FULL, n, off);
            t += __shfl_down_sync(FULL, t, off);
            ry += __shfl_down_sync(FULL, ry, off);
        }
        if (lane == 0)
        {
            atomicAdd(&g_counters[0], n);
            atomicAdd(&g_counters[1], t);
            atomicAdd(&g_counters[2], ry);
            atomicAdd(&g_counters[3], cSteps);
            atomicAdd(&g_counters[4], cLaneSteps);
            atomicAdd(&g_counters[5], cTriIters);
        }
    }
}

// Primary rays as warp packets (trees with one-triangle leaves).  A warp takes
// 32 consecutive wave items, half of an 8x8 tile (an 8x4 pixel block of one
// pass), and traverses the tree once for all of them: every lane tests its own
// ray against the node all lanes are at (one broadcast load of the node), the
// node's child hits are OR-ed over the warp, and the children are visited in
// the order of one ray octant shared by the warp, from a stack in shared
// memory that the warp shares.  Each lane culls with its own closest hit and
// tests the triangles of the leaves its own ray hits, so its result is its
// closest hit, the same as per-lane traversal gives (exact ties go to the
// lower primitive id either way).  Camera rays of a small pixel block visit
// nearly the same nodes when pixels are fine, so the lanes stay busy together
// where the per-lane traversal of k_bounce runs 20 of 32 lanes per instruction
// at this depth; with coarse pixels the union of the rays' nodes grows and the
// packet loses (measured: +1.8% at 1920x1080, -26% at 480x272 on the terrain),
// so it is a launch option (LaunchCfg::packet) the autotuner chooses.
#ifndef PRT_PACKET_PRIMARY
#define PRT_PACKET_PRIMARY 1
#endif
constexpr int kPacketStack = 64;   // >= levels of the deepest tree the build accepts (32)

// The child test of a shared-origin packet split over 24 lanes, one axis of
// one child each, combined with shuffles: the same bounds with about half the
// instructions per node (terrain frame 3061 -> 3106 Mrays/s).
#ifndef PRT_PACKET_IA_SPLIT
#define PRT_PACKET_IA_SPLIT 1
#endif

// Interval traversal of a packet whose rays share one direction octant.  The
// warp tests the packet, not each ray, against a node: lane c (of 0..7) takes
// child c (with a shared origin, lanes c, c + 8 and c + 16 take its x, y and
// z axis, PRT_PACKET_IA_SPLIT) and bounds the entry and exit distances of
// every ray of the packet on each axis from the packet's origin and
// inverse-direction ranges (interval
// products of [plane - omax, plane - omin] and [imin, imax]); the child is
// entered if the largest entry bound does not pass the smallest exit bound,
// clipped to [0, the packet's farthest closest hit].  Child planes are widened
// by one quantization step on both sides (the per-ray test's decode error is
// 2^-9 of a step), so a child that any ray's own test would enter is entered:
// the packet visits a superset of the nodes its rays visit, every lane tests
// its ray against every triangle of the entered leaves with the exact test,
// and each lane's result is its own closest hit.  One child test per node
// instead of one per ray and child; packets of a pinhole camera share one
// origin and need half the interval products (the terrain frame 3015 -> 3060
// Mrays/s).  A launch option (LaunchCfg::packet 2) the autotuner chooses: it
// wins where a packet's rays stay close (fine pixels, short rays; the 1080p
// terrain frame: 3021 against 2982 Mrays/s with per-ray packet tests, before
// the shared-origin case) and loses where they spread apart over long, often
// missing rays (the packet culls with its farthest hit; the 10M-triangle
// field: 2286 against 2859).  Testing each lane's own ray against a leaf's box
// before its triangle (planes kept in shared memory) won back part of the
// field (2580) but cost the terrain as much (2979), and also culling children
// with the four side planes of a pinhole packet's frustum (built from the
// camera basis and the packet's pixel block) cost more than it saved (terrain
// 3063 -> 2921, field 2323 -> 2142), so neither is done.

__device__ __forceinline__ float warp_min_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_max_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Bounds of (plane - o) * inv over o in [omin, omax], inv in [imin, imax]
// (kPoint: one origin shared by the packet, omin == omax).
template <bool kPoint>
__device__ __forceinline__ float ia_min(float plane, float omin, float omax, float imin, float imax)
{
    if (kPoint)
    {
        const float d = plane - omin;
        return fminf(d * imin, d * imax);
    }
    const float d0 = plane - omax, d1 = plane - omin;
    return fminf(fminf(d0 * imin, d0 * imax), fminf(d1 * imin, d1 * imax));
}

template <bool kPoint>
__device__ __forceinline__ float ia_max(float plane, float omin, float omax, float imin, float imax)
{
    if (kPoint)
    {
        const float d = plane - omin;
        return fmaxf(d * imin, d * imax);
    }
    const float d0 = plane - omax, d1 = plane - omin;
    return fmaxf(fmaxf(d0 * imin, d0 * imax), fmaxf(d1 * imin, d1 * imax));
}

// The traversal loop of packet_closest_hit_ia over the packet's ranges.
template <bool kPoint>
__device__ __forceinline__ void packet_ia_loop(const SceneDev& sc, const TravRay& r, bool valid, uint32_t woct,
                                               uint2* stk, unsigned lane, float& tHit, int& primHit, int& triHit,
                                               float oxmin, float oxmax, float oymin, float oymax, float ozmin,
                                               float ozmax, float ixmin, float ixmax, float iymin, float iymax,
                                               float izmin, float izmax)
{
    const unsigned FULL = 0xffffffffu;
    const uint32_t oct = 7u - woct;   // bit k: negative direction on axis k
    const bool nx = (oct & 1u) != 0u, ny = (oct & 2u) != 0u, nz = (oct & 4u) != 0u;
    const int c = (int)(lane & 7u);
    const int cw = c >> 2, cb = c & 3;
    // the axis this lane bounds in the split child test (lanes 24..31 repeat z)
    const int ax = min((int)(lane >> 3), 2);
    const float oa = ax == 0 ? oxmin : (ax == 1 ? oymin : ozmin);
    const float ia0 = ax == 0 ? ixmin : (ax == 1 ? iymin : izmin), ia1 = ax == 0 ? ixmax : (ax == 1 ? iymax : izmax);
    const bool na = ax == 0 ? nx : (ax == 1 ? ny : nz);
    float tfarP = FLT_MAX;
    int sp = 0;
    uint2 ng = make_uint2(0u, 0x80000000u);   // the root: one internal child at base 0
    for (;;)
    {
        const uint32_t b = 31u - __clz(ng.y & 0xff000000u);
        ng.y &= ~(1u << b);
        const uint32_t slot = (b - 24u) ^ woct;
        const uint32_t nodeIdx = ng.x + __popc((ng.y & 0xffu) & ((1u << slot) - 1u));
        if ((ng.y & 0xff000000u) && sp < kPacketStack)
        {
            if (lane == 0) stk[sp] = ng;
            ++sp;
        }
        const uint4* qp = reinterpret_cast<const uint4*>(sc.nodes + nodeIdx);
        uint4 q[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) q[k] = __ldg(qp + k);
        // child c of the node against the packet; a relative slack of 2^-18 on
        // both bounds is far more than the rounding of either test at any
        // distance the planes' step margin does not cover
        bool enter;
        if constexpr (kPoint && PRT_PACKET_IA_SPLIT)
        {
            // lane (axis a, child c) bounds one axis; lanes c, c + 8, c + 16
            // hold the x, y, z bounds of child c and lane c combines them
            const uint32_t sh = 8u * (uint32_t)ax;
            const float sa = __uint_as_float(((q[0].w >> sh) & 0xffu) << 23);
            const float pa = __uint_as_float(ax == 0 ? q[0].x : (ax == 1 ? q[0].y : q[0].z));
            const uint32_t loW = ax == 0 ? (cw ? q[2].y : q[2].x)
                                          : (ax == 1 ? (cw ? q[2].w : q[2].z) : (cw ? q[3].y : q[3].x));
            const uint32_t hiW = ax == 0 ? (cw ? q[3].w : q[3].z)
                                          : (ax == 1 ? (cw ? q[4].y : q[4].x) : (cw ? q[4].w : q[4].z));
            const float lo = fmaf(byte_f(loW, cb) - 1.0f, sa, pa), hi = fmaf(byte_f(hiW, cb) + 1.0f, sa, pa);
            const float dn = (na ? hi : lo) - oa, df = (na ? lo : hi) - oa;
            const float tn = fminf(dn * ia0, dn * ia1), tf = fmaxf(df * ia0, df * ia1);
            const float tn1 = __shfl_sync(FULL, tn, c + 8), tn2 = __shfl_sync(FULL, tn, c + 16);
            const float tf1 = __shfl_sync(FULL, tf, c + 8), tf2 = __shfl_sync(FULL, tf, c + 16);
            const float t0 = fmaxf(fmax3(tn, tn1, tn2), 0.0f);
            const float t1 = fminf(fmin3(tf, tf1, tf2), tfarP * 1.0000004f);
            enter = t0 * 0.999996f <= t1 * 1.000004f;
        }
        else
        {
            const uint32_t e = q[0].w;
            const float sx = __uint_as_float((e & 0xffu) << 23), sy = __uint_as_float(((e >> 8) & 0xffu) << 23),
                        sz = __uint_as_float(((e >> 16) & 0xffu) << 23);
            const float px = __uint_as_float(q[0].x), py = __uint_as_float(q[0].y), pz = __uint_as_float(q[0].z);
            const float lx = fmaf(byte_f(cw ? q[2].y : q[2].x, cb) - 1.0f, sx, px);
            const float ly = fmaf(byte_f(cw ? q[2].w : q[2].z, cb) - 1.0f, sy, py);
            const float lz = fmaf(byte_f(cw ? q[3].y : q[3].x, cb) - 1.0f, sz, pz);
            const float hx = fmaf(byte_f(cw ? q[3].w : q[3].z, cb) + 1.0f, sx, px);
            const float hy = fmaf(byte_f(cw ? q[4].y : q[4].x, cb) + 1.0f, sy, py);
            const float hz = fmaf(byte_f(cw ? q[4].w : q[4].z, cb) + 1.0f, sz, pz);
            const float t0 = fmaxf(fmax3(ia_min<kPoint>(nx ? hx : lx, oxmin, oxmax, ixmin, ixmax),
                                         ia_min<kPoint>(ny ? hy : ly, oymin, oymax, iymin, iymax),
                                         ia_min<kPoint>(nz ? hz : lz, ozmin, ozmax, izmin, izmax)),
                                   0.0f);
            const float t1 = fminf(fmin3(ia_max<kPoint>(nx ? lx : hx, oxmin, oxmax, ixmin, ixmax),
                                         ia_max<kPoint>(ny ? ly : hy, oymin, oymax, iymin, iymax),
                                         ia_max<kPoint>(nz ? lz : hz, ozmin, ozmax, izmin, izmax)),
                                   tfarP * 1.0000004f);
            enter = t0 * 0.999996f <= t1 * 1.000004f;
        }
        uint32_t c8 = __ballot_sync(FULL, enter) & 0xffu;
        // non-empty slots (bit 5 of each meta byte), leaves and internal children
        const uint32_t ne = ((((q[1].z >> 5) & 0x01010101u) * 0x01020408u) >> 24) |
                            (((((q[1].w >> 5) & 0x01010101u) * 0x01020408u) >> 24) << 4);
        c8 &= ne;
        const uint32_t imask = q[0].w >> 24;
        const uint32_t leafMask = ne & ~imask;
        uint32_t lb = c8 & leafMask;
        if (lb)
        {
            do
            {
                const uint32_t bit = __ffs(lb) - 1u;
                lb &= lb - 1u;
                const int ti = (int)(q[1].y + __popc(leafMask & ((1u << bit) - 1u)));
                if (valid)
                {
                    const float4* tp = reinterpret_cast<const float4*>(sc.tris + ti);
                    const float4 v0 = __ldg(tp), v1 = __ldg(tp + 1), v2 = __ldg(tp + 2);
                    const int prim = __float_as_int(v0.w);
                    float t, u, v;
                    if (tri_test(r, f3(v0.x, v0.y, v0.z), f3(v1.x, v1.y, v1.z), f3(v2.x, v2.y, v2.z), 0.0f, tHit,
                                 prim, primHit, t, u, v))
                    {
                        tHit = t;
                        primHit = prim;
                        triHit = ti;
                    }
                }
            } while (lb);
            tfarP = __uint_as_float(__reduce_max_sync(FULL, valid ? __float_as_uint(tHit) : 0u));
        }
        // internal hits: bit slot -> bit slot ^ octinv, as node_hits1 orders them
        uint32_t in8 = c8 & imask;
        uint32_t sw = ((in8 & 0x55u) << 1) | ((in8 >> 1) & 0x55u);
        in8 = (woct & 1u) ? sw : in8;
        sw = ((in8 & 0x33u) << 2) | ((in8 >> 2) & 0x33u);
        in8 = (woct & 2u) ? sw : in8;
        sw = ((in8 & 0x0fu) << 4) | ((in8 >> 4) & 0x0fu);
        in8 = (woct & 4u) ? sw : in8;
        ng = make_uint2(q[1].x, (in8 << 24) | imask);
        if (!(ng.y & 0xff000000u))
        {
            if (sp == 0) break;
            __syncwarp();
            ng = stk[--sp];
            __syncwarp();
        }
    }
}

__device__ __forceinline__ void packet_closest_hit_ia(const SceneDev& sc, const TravRay& r, bool valid,
                                                      unsigned vmask, uint32_t woct, uint2* stk, unsigned lane,
                                                      float& tHit, int& primHit, int& triHit)
{
    const unsigned FULL = 0xffffffffu;
    // packet ranges (lanes without a ray take the first ray's values)
    const int lead = __ffs(vmask) - 1;
    const float lox = __shfl_sync(FULL, r.org.x, lead), loy = __shfl_sync(FULL, r.org.y, lead),
                loz = __shfl_sync(FULL, r.org.z, lead);
    const float lix = __shfl_sync(FULL, r.inv.x, lead), liy = __shfl_sync(FULL, r.inv.y, lead),
                liz = __shfl_sync(FULL, r.inv.z, lead);
    const float ox = valid ? r.org.x : lox, oy = valid ? r.org.y : loy, oz = valid ? r.org.z : loz;
    const float ix = valid ? r.inv.x : lix, iy = valid ? r.inv.y : liy, iz = valid ? r.inv.z : liz;
    const float oxmin = warp_min_f(ox), oxmax = warp_max_f(ox);
    const float oymin = warp_min_f(oy), oymax = warp_max_f(oy);
    const float ozmin = warp_min_f(oz), ozmax = warp_max_f(oz);
    const float ixmin = warp_min_f(ix), ixmax = warp_max_f(ix);
    const float iymin = warp_min_f(iy), iymax = warp_max_f(iy);
    const float izmin = warp_min_f(iz), izmax = warp_max_f(iz);
    // pinhole packets share one origin: half the interval products
    if (oxmin == oxmax && oymin == oymax && ozmin == ozmax)
        packet_ia_loop<true>(sc, r, valid, woct, stk, lane, tHit, primHit, triHit, oxmin, oxmax, oymin, oymax, ozmin,
                             ozmax, ixmin, ixmax, iymin, iymax, izmin, izmax);
    else
        packet_ia_loop<false>(sc, r, valid, woct, stk, lane, tHit, primHit, triHit, oxmin, oxmax, oymin, oymax, ozmin,
                              ozmax, ixmin, ixmax, iymin, iymax, izmin, izmax);
}

// Warp-collective closest-hit traversal of the warp's rays as one packet (one-
// triangle leaves; every lane of the warp calls it).  valid: this lane holds a
// ray; vmask: the ballot of valid; stk: the warp's kPacketStack entries of
// shared memory.  Returns this lane's closest hit (triHit -1: none).
template <bool kPair, bool kIA>
__device__ __forceinline__ void packet_closest_hit(const SceneDev& sc, const TravRay& r, bool valid, unsigned vmask,
                                                   uint2* stk, unsigned lane, float& tHit, int& primHit, int& triHit)
{
    const unsigned FULL = 0xffffffffu;
    const uint32_t woct = __shfl_sync(FULL, r.octinv, __ffs(vmask) - 1);
    tHit = FLT_MAX;
    primHit = 0x7fffffff;
    triHit = -1;
    if (!sc.hasRoot) return;
    if (kIA && __all_sync(FULL, !valid || r.octinv == woct))
    {
        packet_closest_hit_ia(sc, r, valid, vmask, woct, stk, lane, tHit, primHit, triHit);
        return;
    }
    int sp = 0;
    uint2 ng = make_uint2(0u, 0x80000000u);   // the root: one internal child at base 0
    for (;;)
    {
        const uint32_t b = 31u - __clz(ng.y & 0xff000000u);
        ng.y &= ~(1u << b);
        const uint32_t slot = (b - 24u) ^ woct;
        const uint32_t nodeIdx = ng.x + __popc((ng.y & 0xffu) & ((1u << slot) - 1u));
        if ((ng.y & 0xff000000u) && sp < kPacketStack)
        {
            if (lane == 0) stk[sp] = ng;
            ++sp;
        }
        const uint4* qp = reinterpret_cast<const uint4*>(sc.nodes + nodeIdx);
        uint4 q[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) q[k] = __ldg(qp + k);
        uint32_t leafMask = 0;
        const uint32_t hits = valid ? node_hits1<kPair>(r, q, 0.0f, tHit, leafMask, woct) : 0u;
        // this lane's leaf triangles (leaf slot j -> triBase + rank of j among the leaf slots)
        uint32_t lb = hits & 0xffu;
        while (lb)
        {
            const uint32_t bit = __ffs(lb) - 1u;
            lb &= lb - 1u;
            const int ti = (int)(q[1].y + __popc(leafMask & ((1u << bit) - 1u)));
            const float4* tp = reinterpret_cast<const float4*>(sc.tris + ti);
            const float4 v0 = __ldg(tp), v1 = __ldg(tp + 1), v2 = __ldg(tp + 2);
            const int prim = __float_as_int(v0.w);
            float t, u, v;
            if (tri_test(r, f3(v0.x, v0.y, v0.z), f3(v1.x, v1.y, v1.z), f3(v2.x, v2.y, v2.z), 0.0f, tHit, prim,
                         primHit, t, u, v))
            {
                tHit = t;
                primHit = prim;
                triHit = ti;
            }
        }
        ng = make_uint2(q[1].x, __reduce_or_sync(FULL, hits & 0xff000000u) | (q[0].w >> 24));
        if (!(ng.y & 0xff000000u))
        {
            if (sp == 0) break;
            __syncwarp();
            ng = stk[--sp];
            __syncwarp();
        }
    }
}

template <bool kAlbedo, bool kIA>
__global__ void __launch_bounds__(128, PRT_BOUNCE_MIN_BLOCKS) k_primary_packet(WaveArgs a)
{
    extern __shared__ uint2 s_packet[];
    uint2* stk = s_packet + (threadIdx.x >> 5) * kPacketStack;
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const int W = a.cam.width, H = a.cam.height;
    const int perPass = a.tilesX * a.tilesY * 64;
    const int total = a.passes * perPass;
    const int pass0 = *a.passBase + a.passOffset;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicAdd(a.rays, (unsigned long long)a.passes * (unsigned long long)W * (unsigned long long)H);
    const bool final = a.maxDepth == 0;
    for (;;)
    {
        int base = 0;
        if (lane == 0) base = atomicAdd(&a.fetch[0], 32);
        base = __shfl_sync(FULL, base, 0);
        if (base >= total) break;
        const int i = base + (int)lane;
        bool valid = false;
        int pixel = 0;
        uint32_t rng = 0;
        float3 org = f3(0.f, 0.f, 0.f), dir = f3(0.f, 0.f, 1.f);
        if (i < total)
        {
            const int pass = i / perPass;
            int x, y;
            if (wave_item_pixel(i - pass * perPass, a.tilesX, W, H, x, y))
            {
                valid = true;
                pixel = x + y * W;
                rng = rng_seed(pass0 + pass, pixel);
                camera_ray(a.cam, x, y, rng, org, dir);
            }
        }
        const unsigned vmask = __ballot_sync(FULL, valid);
        if (!vmask) continue;
        TravRay r;
        trav_setup(r, org, dir);
        float tHit;
        int primHit, triHit;
        packet_closest_hit<PRT_PAIRED_PACKET, kIA>(a.scene, r, valid, vmask, stk, lane, tHit, primHit, triHit);
        // shade / append / accumulate, as k_bounce does at depth 0
        bool cont = false;
        float contrib = 0.f;
        float thr = kAlbedo ? 1.0f : a.thrConst;
        if (valid)
        {
            if (triHit < 0)
            {
                contrib = __fmul_rn(thr, a.sky);
            }
            else if (!final)
            {
                if (kAlbedo) thr = __fmul_rn(thr, a.scene.albedo ? __ldg(a.scene.albedo + primHit) : 0.8f);
                diffuse_bounce(a.scene.tris, triHit, org, dir, tHit, rng);
                cont = true;
            }
        }
        const int o = warp_append(cont, &a.counts[1]);
        if (cont)
        {
            store_path(a.qout, o, org, pixel, dir, rng);
            if (kAlbedo) __stcs(a.thrOut + o, thr);
        }
        else if (valid)
        {
            red_add_v4(a.accum + pixel, contrib, contrib, contrib, 1.0f);
        }
    }
}

// Bounce kernel of the next-event-estimation integrator
// (render/diffuse2_integrator_single.h:41-90, render/diffuse2_renderer_cuda.cu:63-239).
// A lane takes a path's extension ray; at a hit before maxDepth it samples a
// shadow direction and an extension direction from the same frame, traces the
// shadow ray for any occluder in the same lane (+0.5 * throughput * sky if it
// escapes), then appends the extension ray with its gathered radiance.  An
// escaping extension ray adds throughput * sky weighted 1 from the camera and
// 0.5 after a bounce.  Shadow rays are counted as rays.
template <bool kFirst, bool kAlbedo>
__global__ void __launch_bounds__(128, PRT_BOUNCE_MIN_BLOCKS) k_bounce_nee(WaveArgs a, int depth)
{
    extern __shared__ uint2 s_stack[];
    TravStack st;
    st.sh = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    st.overflow = false;
    TriQueue* tq = reinterpret_cast<TriQueue*>(s_stack + kShared * blockDim.x) + (threadIdx.x >> 5);   // deferTris
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned ltMask = (1u << lane) - 1u;
    const int W = a.cam.width, H = a.cam.height;
    const int perPass = a.tilesX * a.tilesY * 64;
    int total;
    int pass0 = 0;
    if (kFirst)
    {
        total = a.passes * perPass;
        pass0 = *a.passBase + a.passOffset;
    }
    else
    {
        total = *(volatile int*)&a.counts[depth];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicAdd(a.rays, kFirst ? (unsigned long long)a.passes * (unsigned long long)W * (unsigned long long)H
                                 : (unsigned long long)total);
    const bool final = depth == a.maxDepth;
    const float missWeight = depth > 0 ? 0.5f : 1.0f;

    bool has = false, exhausted = false, shadow = false;
    int pixel = 0;
    uint32_t rng = 0;
    int qi = 0;               // input-queue index of this lane's path (PRT_RELOAD_PATH)
    int slot = 0;             // output-queue slot of the extension ray while its shadow ray is traced
    float thr = 0.f, L = 0.f;
    unsigned long long shadowRays = 0;
    TravRay r;
    TravState ts;
    ts.done = true;
    for (;;)
    {
        unsigned idle = __ballot_sync(FULL, !has);
        if (!exhausted && (__popc(idle) >= kRefillMin || idle == FULL))
        {
            int n = __popc(idle);
            int base = 0;
            if (lane == 0) base = atomicAdd(&a.fetch[depth], n);
            base = __shfl_sync(FULL, base, 0);
            if (base + n >= total) exhausted = true;
            int i = base + __popc(idle & ltMask);
            if (!has && i < total)
            {
                float3 org, dir;
                bool ok = true;
                if (kFirst)
                {
                    int pass = i / perPass;
                    int x, y;
                    if (!wave_item_pixel(i - pass * perPass, a.tilesX, W, H, x, y))
                    {
                        ok = false;
                    }
                    else
                    {
                        pixel = x + y * W;
                        rng = rng_seed(pass0 + pass, pixel);
                        camera_ray(a.cam, x, y, rng, org, dir);
                        thr = kAlbedo ? 1.0f : a.thrConst;
                        L = 0.0f;
                    }
                }
                else if (PRT_RELOAD_PATH)
                {
                    // pixel, RNG state and direction are read again when the lane shades
                    const float4* p = reinterpret_cast<const float4*>(a.qin + i);
                    const float4 w0 = __ldcg(p), w1 = __ldcg(p + 1);
                    org = f3(w0.x, w0.y, w0.z);
                    dir = f3(w1.x, w1.y, w1.z);
                    qi = i;
                    thr = kAlbedo ? __ldcs(a.thrIn + i) : a.thrConst;
                    L = __ldcs(a.Lin + i);
                }
                else
                {
                    PathRec pr = load_path(a.qin, i);
                    org = f3(pr.w0.x, pr.w0.y, pr.w0.z);
                    pixel = __float_as_int(pr.w0.w);
                    dir = f3(pr.w1.x, pr.w1.y, pr.w1.z);
                    rng = __float_as_uint(pr.w1.w);
                    thr = kAlbedo ? __ldcs(a.thrIn + i) : a.thrConst;
                    L = __ldcs(a.Lin + i);
                }
                if (ok)
                {
                    has = true;
                    shadow = false;
                    trav_setup(r, org, dir);
                    trav_init(ts, a.scene, FLT_MAX, st);
                }
            }
        }
        if (__ballot_sync(FULL, has) == 0)
        {
            if (exhausted) break;
            continue;
        }
        if (PRT_DEFER_NEE && a.scene.deferTris)
        {
            // extension rays (closest hit) and shadow rays (any hit) share the queue
            constexpr bool kPair = !kFirst && PRT_RELOAD_PATH && PRT_PAIRED_NEE;
            warp_trav_deferred<kPair>(*tq, ts, a.scene, r, 0.0f, st, has, true, kRefillMin, lane, nullptr, nullptr,
                                      nullptr, nullptr, nullptr, shadow);
        }
        else
        for (;;)
        {
            if (has && !ts.done) trav_step<false>(ts, a.scene, r, 0.0f, st, nullptr, nullptr, shadow);
            unsigned running = __ballot_sync(FULL, has && !ts.done);
            if (running == 0) break;
            if (32 - __popc(running) >= kRefillMin) break;
        }
        // Extension-ray lanes that hit sample their shadow and extension rays,
        // append the extension ray at once and keep only its queue slot while
        // the shadow ray is traced; the radiance gathered so far is written to
        // that slot when the shadow ray finishes.  Values of a finished path
        // are iteration-local, so nothing else is carried around the loop.
        const bool finExt = has && ts.done && !shadow;
        const bool finShadow = has && ts.done && shadow;
        bool spawn = false, end = false;
        int fpix = 0;
        uint32_t frng = 0;
        float3 so = f3(0.f, 0.f, 0.f), sd = f3(0.f, 0.f, 1.f), eo = so, ed = sd;
        if (finExt)
        {
            float3 fdir;
            if (!kFirst && PRT_RELOAD_PATH)
            {
                const float4* p = reinterpret_cast<const float4*>(a.qin + qi);
                const float4 w1 = __ldcs(p + 1);
                fpix = __float_as_int(__ldcs(reinterpret_cast<const float*>(p) + 3));
                fdir = f3(w1.x, w1.y, w1.z);
                frng = __float_as_uint(w1.w);
            }
            else
            {
                fpix = pixel;
                fdir = r.dir;
                frng = rng;
            }
            if (ts.triHit < 0)
            {
                L = __fadd_rn(L, __fmul_rn(__fmul_rn(thr, a.sky), missWeight));
                end = true;
            }
            else if (final)
            {
                end = true;
            }
            else
            {
                if (kAlbedo)
                    thr = __fmul_rn(thr, a.scene.albedo ? __ldg(a.scene.albedo + ts.primHit) : 0.8f);
                else
                    thr = __fmul_rn(thr, 0.8f);
                HitFrame hf = hit_frame(a.scene.tris, ts.triHit, r.org, fdir, ts.tHit);
                sample_bounce(hf, frng, so, sd);   // shadow ray
                sample_bounce(hf, frng, eo, ed);   // extension ray
                spawn = true;
            }
        }
        const int o = warp_append(spawn, &a.counts[depth + 1]);
        if (spawn)
        {
            store_path(a.qout, o, eo, fpix, ed, frng);
            if (kAlbedo) __stcs(a.thrOut + o, thr);
            slot = o;
            trav_setup(r, so, sd);
            trav_init(ts, a.scene, FLT_MAX, st);
            shadow = true;
            ++shadowRays;
        }
        else if (end)
        {
            red_add_v4(a.accum + fpix, L, L, L, 1.0f);
            has = false;
        }
        if (finShadow)
        {
            if (ts.triHit < 0) L = __fadd_rn(L, __fmul_rn(__fmul_rn(thr, a.sky), 0.5f));
            __stcs(a.Lout + slot, L);
            has = false;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) shadowRays += __shfl_down_sync(FULL, shadowRays, off);
    if (lane == 0 && shadowRays) atomicAdd(a.rays, shadowRays);
}

// The IntersectorStreamCuda seam (core/intersector_stream_cuda.h:32-33):
// closest or any hit for n ray records.  Persistent warps with the same
// dynamic per-lane refill as k_bounce: a lane whose query is complete writes
// its hit record, and once kRefillMin lanes of the warp are free they claim
// the next rays from the call's work counter, so incoherent queries of very
// different lengths keep the warp's lanes busy.
template <bool kAnyHit>
__global__ void __launch_bounds__(128, PRT_BOUNCE_MIN_BLOCKS) k_intersect(SceneDev sc, const RayRec* __restrict__ rays,
                                                                         HitRec* __restrict__ hits,
                                                                         float* __restrict__ anyOut, int n, int* fetch)
{
    extern __shared__ uint2 s_stack[];
    TravStack st;
    st.sh = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    st.overflow = false;
    TriQueue* tq = reinterpret_cast<TriQueue*>(s_stack + kShared * blockDim.x) + (threadIdx.x >> 5);   // deferTris
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned ltMask = (1u << lane) - 1u;
    bool has = false, exhausted = false;
    int idx = 0;
    float tnear = 0.f;
    TravRay r;
    TravState ts;
    ts.done = true;
    for (;;)
    {
        unsigned idle = __ballot_sync(FULL, !has);
        if (!exhausted && (__popc(idle) >= kRefillMin || idle == FULL))
        {
            int cnt = __popc(idle);
            int base = 0;
            if (lane == 0) base = atomicAdd(fetch, cnt);
            base = __shfl_sync(FULL, base, 0);
            if (base + cnt >= n) exhausted = true;
            int i = base + __popc(idle & ltMask);
            if (!has && i < n)
            {
                const float4* rp = reinterpret_cast<const float4*>(rays + i);
                float4 a = __ldcs(rp), b = __ldcs(rp + 1);
                trav_setup(r, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z));
                trav_init(ts, sc, b.w, st);
                tnear = a.w;
                idx = i;
                has = true;
            }
        }
        if (__ballot_sync(FULL, has) == 0)
        {
            if (exhausted) break;
            continue;
        }
        if (PRT_DEFER_ISECT && sc.deferTris)
        {
            constexpr bool kPair = kAnyHit && PRT_PAIRED_QUERY;
            warp_trav_deferred<kPair>(*tq, ts, sc, r, tnear, st, has, !exhausted, kRefillMin, lane, nullptr, nullptr,
                                      nullptr, nullptr, nullptr, kAnyHit);
        }
        else
        for (;;)
        {
            if (has && !ts.done) trav_step<kAnyHit>(ts, sc, r, tnear, st);
            unsigned running = __ballot_sync(FULL, has && !ts.done);
            if (running == 0) break;
            if (!exhausted && 32 - __popc(running) >= kRefillMin) break;
        }
        if (has && ts.done)
        {
            const bool hit = ts.triHit >= 0;
            if (kAnyHit)
                __stcs(anyOut + idx, hit ? ts.tHit : -1.0f);
            else
                __stcs(reinterpret_cast<float4*>(hits) + idx,
                       hit ? make_float4(ts.tHit, __int_as_float(ts.primHit), ts.uHit, ts.vHit)
                           : make_float4(-1.0f, __int_as_float(-1), 0.f, 0.f));
            has = false;
        }
    }
}

// Hit point and geometric normal of one query ray (Renderer::queryRay).
__global__ void k_query(SceneDev sc, const RayRec* ray, HitRec* hit, float* pNg)
{
    __shared__ uint2 s_stack[kShared];
    TravStack st;
    st.sh = s_stack;
    st.stride = 1;
    st.overflow = false;
    RayRec rr = *ray;
    TravRay r;
    trav_setup(r, f3(rr.ox, rr.oy, rr.oz), f3(rr.dx, rr.dy, rr.dz));
    float t, u, v;
    int prim;
    int ti = traverse<false>(sc, r, rr.tnear, rr.tfar, st, t, prim, u, v);
    if (ti < 0)
    {
        *hit = HitRec{-1.0f, -1, 0.f, 0.f};
        return;
    }
    *hit = HitRec{t, prim, u, v};
    float3 p = madd(r.org, t, r.dir);
    const TriRec tr = sc.tris[ti];
    float3 p0 = f3(tr.v0.x, tr.v0.y, tr.v0.z), p1 = f3(tr.v1.x, tr.v1.y, tr.v1.z), p2 = f3(tr.v2.x, tr.v2.y, tr.v2.z);
    float3 Ng = normalize(cross(sub(p1, p0), sub(p2, p0)));
    if (dot(Ng, r.dir) > 0.0f) Ng = f3(-Ng.x, -Ng.y, -Ng.z);
    pNg[0] = p.x; pNg[1] = p.y; pNg[2] = p.z;
    pNg[3] = Ng.x; pNg[4] = Ng.y; pNg[5] = Ng.z;
}

// Gamma-2.2 BGRA8 resolve (image/accum_buffer_cuda.cu:22-37; channel order of
// encodeBgr8, image/pixel.h:42-46).
__global__ void k_resolve_ldr(const float4* __restrict__ accum, uint32_t* __restrict__ out, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = accum[i];
    float w = a.w > 0.f ? 1.0f / a.w : 0.0f;
    const float g = 1.0f / 2.2f;
    int r = min(max((int)(powf(a.x * w, g) * 255.0f), 0), 255);
    int gg = min(max((int)(powf(a.y * w, g) * 255.0f), 0), 255);
    int b = min(max((int)(powf(a.z * w, g) * 255.0f), 0), 255);
    out[i] = (uint32_t)b | ((uint32_t)gg << 8) | ((uint32_t)r << 16);
}

__global__ void k_advance_pass(int* passBase, int spp) { *passBase += spp; }

constexpr int kReplayMaxDepth = 16;
constexpr int kAggSlots = 1024;   // block-private gradient slots of the adjoint

// Path-replay megakernel: each lane carries whole paths (pass, pixel), from
// the camera ray to escape or maxDepth.  The forward mode accumulates the
// path's radiance; the backward mode re-traces the same path from its seed
// and scatters dL/d(radiance) into the albedo of every triangle the path
// bounced off and into the sky radiance:
//   radiance = sky * prod_k albedo[prim_k]
//   d radiance / d albedo[prim_k] = radiance / albedo[prim_k]
//   d radiance / d sky            = prod_k albedo[prim_k]
// Paths are regenerated per lane (a lane whose path ends takes the next one
// once kRefillMin lanes of its warp are free), and traversal advances one node
// per step, as in k_bounce.  The bounce arithmetic is the same device code as
// the wavefront renderer's, so both compute bit-identical paths.
template <bool kBackward>
__global__ void __launch_bounds__(128, 8) k_replay(SceneDev sc, CameraDev cam, float4* accum, int pass0, int spp,
                                                   int maxDepth, float sky, const float* __restrict__ dL,
                                                   float* dAlbedo, float* dSky, unsigned long long* rays,
                                                   int* fetch)
{
    extern __shared__ uint2 s_stack[];
    // Block-private accumulation of albedo gradients: a few triangles (a
    // ground plane) receive most of the contributions, so per-path global
    // atomics would serialise on them.  Slot = prim mod kAggSlots; a slot
    // holds one triangle, collisions go straight to global memory.
    __shared__ int s_key[kBackward ? kAggSlots : 1];
    __shared__ float s_val[kBackward ? kAggSlots : 1];
    if (kBackward)
    {
        for (int i = threadIdx.x; i < kAggSlots; i += blockDim.x)
        {
            s_key[i] = -1;
            s_val[i] = 0.f;
        }
        __syncthreads();
    }
    TravStack st;
    st.sh = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    st.overflow = false;
    TriQueue* tq = reinterpret_cast<TriQueue*>(s_stack + kShared * blockDim.x) + (threadIdx.x >> 5);   // forward, deferTris
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned ltMask = (1u << lane) - 1u;
    const int W = cam.width, H = cam.height;
    const long long npix = (long long)W * H;
    const long long total = (long long)spp * npix;
    float skyGrad = 0.f;
    unsigned long long myRays = 0;

    bool has = false;
    bool exhausted = false;
    int pixel = 0, depth = 0, np = 0;
    uint32_t rng = 0;
    float thr = 1.f, g = 0.f;
    int prims[kBackward ? kReplayMaxDepth : 1];
    TravRay r;
    TravState ts;
    ts.done = true;
    for (;;)
    {
        unsigned idle = __ballot_sync(FULL, !has);
        if (!exhausted && (__popc(idle) >= kRefillMin || idle == FULL))
        {
            int n = __popc(idle);
            long long base = 0;
            if (lane == 0) base = (long long)atomicAdd(reinterpret_cast<unsigned long long*>(fetch), (unsigned long long)n);
            base = __shfl_sync(FULL, base, 0);
            if (base + n >= total) exhausted = true;
            long long gi = base + __popc(idle & ltMask);
            if (!has && gi < total)
            {
                int pass = (int)(gi / npix);
                pixel = (int)(gi - (long long)pass * npix);
                bool ok = true;
                if (kBackward)
                {
                    g = dL[3 * (size_t)pixel] + dL[3 * (size_t)pixel + 1] + dL[3 * (size_t)pixel + 2];
                    ok = g != 0.f;
                }
                if (ok)
                {
                    rng = rng_seed(pass0 + pass, pixel);
                    float3 org, dir;
                    camera_ray(cam, pixel % W, pixel / W, rng, org, dir);
                    trav_setup(r, org, dir);
                    trav_init(ts, sc, FLT_MAX, st);
                    thr = 1.0f;
                    depth = 0;
                    np = 0;
                    has = true;
                }
            }
        }
        if (__ballot_sync(FULL, has) == 0)
        {
            if (exhausted) break;
            continue;
        }
        if (PRT_DEFER_REPLAY && !kBackward && sc.deferTris)
        {
            warp_trav_deferred(*tq, ts, sc, r, 0.0f, st, has, true, kRefillMin, lane);
        }
        else
        for (;;)
        {
            if (has && !ts.done) trav_step<false>(ts, sc, r, 0.0f, st);
            unsigned running = __ballot_sync(FULL, has && !ts.done);
            if (running == 0) break;
            if (32 - __popc(running) >= kRefillMin) break;
        }
        if (has && ts.done)
        {
            ++myRays;
            bool escaped = ts.triHit < 0;
            if (!escaped && depth < maxDepth)
            {
                // continue the path in this lane
                thr = __fmul_rn(thr, sc.albedo ? __ldg(sc.albedo + ts.primHit) : 0.8f);
                if (kBackward) prims[np++] = ts.primHit;
                float3 org = r.org, dir = r.dir;
                diffuse_bounce(sc.tris, ts.triHit, org, dir, ts.tHit, rng);
                trav_setup(r, org, dir);
                trav_init(ts, sc, FLT_MAX, st);
                ++depth;
            }
            else
            {
                float c = escaped ? __fmul_rn(thr, sky) : 0.0f;
                if (!kBackward)
                {
                    red_add_v4(accum + pixel, c, c, c, 1.0f);
                }
                else if (escaped)
                {
                    skyGrad += g * thr;
                    float gc = g * c;
                    for (int k = 0; k < np; ++k)
                    {
                        const int pk = prims[k];
                        float al = sc.albedo ? __ldg(sc.albedo + pk) : 0.8f;
                        float v = gc / al;
                        const int slot = pk & (kAggSlots - 1);
                        int key = s_key[slot];
                        if (key == -1) key = atomicCAS(&s_key[slot], -1, pk);   // -1: claimed by us
                        if (key == -1 || key == pk) atomicAdd(&s_val[slot], v);
                        else atomicAdd(dAlbedo + pk, v);
                    }
                }
                has = false;
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        skyGrad += __shfl_down_sync(FULL, skyGrad, off);
        myRays += __shfl_down_sync(FULL, myRays, off);
    }
    if (lane == 0)
    {
        if (kBackward && skyGrad != 0.f) atomicAdd(dSky, skyGrad);
        if (rays) atomicAdd(rays, myRays);
    }
    if (kBackward)
    {
        __syncthreads();
        for (int i = threadIdx.x; i < kAggSlots; i += blockDim.x)
            if (s_key[i] >= 0) atomicAdd(dAlbedo + s_key[i], s_val[i]);
    }
}

// Batched bounce: the paths of many requests share one queue.  Item i of the
// first bounce is a global path index resolved to (request, pass, tile,
// Morton index) by a binary search over the requests' path ranges; later
// bounces carry (request << 24 | pixel) in the path record.  Lanes refill
// dynamically as in k_bounce.
template <bool kFirst>
__global__ void __launch_bounds__(128, 8) k_batch_bounce(BatchArgs a, int depth)
{
    extern __shared__ uint2 s_dyn[];
    uint2* s_stack = s_dyn;
    long long* s_begin = reinterpret_cast<long long*>(s_dyn + kShared * blockDim.x);
    TriQueue* tq = reinterpret_cast<TriQueue*>(s_begin + a.nreq) + (threadIdx.x >> 5);   // when a.leaf1
    for (int q = threadIdx.x; q < a.nreq; q += blockDim.x) s_begin[q] = a.reqs[q].pathBegin;
    __syncthreads();
    TravStack st;
    st.sh = s_stack + threadIdx.x;
    st.stride = blockDim.x;
    st.overflow = false;
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned ltMask = (1u << lane) - 1u;
    const long long total = kFirst ? (a.waveEnd - a.waveBegin) : (long long)*(volatile int*)&a.counts[depth];
    if (!kFirst && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(a.rays, (unsigned long long)total);
    unsigned long long myRays = 0;
    float thrDepth = 1.0f;
    for (int d = 0; d < depth; ++d) thrDepth = __fmul_rn(thrDepth, 0.8f);

    bool has = false;
    bool exhausted = false;
    int pixel = 0, req = 0;
    uint32_t rng = 0;
    int qi = 0;               // input-queue index of this lane's path (PRT_RELOAD_PATH)
    TravRay r;
    TravState ts;
    ts.done = true;
    for (;;)
    {
        unsigned idle = __ballot_sync(FULL, !has);
        if (!exhausted && (__popc(idle) >= kRefillMin || idle == FULL))
        {
            int n = __popc(idle);
            int base = 0;
            if (lane == 0) base = atomicAdd(&a.fetch[depth], n);
            base = __shfl_sync(FULL, base, 0);
            if (base + n >= total) exhausted = true;
            int i = base + __popc(idle & ltMask);
            if (!has && i < total)
            {
                float3 org, dir;
                bool ok = true;
                if (kFirst)
                {
                    long long gi = a.waveBegin + i;
                    int lo = 0, hi = a.nreq - 1;
                    while (lo < hi)
                    {
                        int mid = (lo + hi + 1) >> 1;
                        if (s_begin[mid] <= gi) lo = mid;
                        else hi = mid - 1;
                    }
                    req = lo;
                    const BatchReq& R = a.reqs[req];
                    long long local = gi - s_begin[req];
                    int perPass = R.tilesX * R.tilesY * 64;
                    int pass = (int)(local / perPass);
                    int x, y;
                    if (!wave_item_pixel((int)(local - (long long)pass * perPass), R.tilesX, R.cam.width,
                                         R.cam.height, x, y))
                    {
                        ok = false;
                    }
                    else
                    {
                        pixel = x + y * R.cam.width;
                        rng = rng_seed(pass, pixel);
                        camera_ray(R.cam, x, y, rng, org, dir);
                        ++myRays;
                    }
                }
                else if (PRT_RELOAD_PATH)
                {
                    // as in k_bounce: pixel, RNG and direction are read again when
                    // the lane shades; the request id stays (it selects the scene)
                    const float4* p = reinterpret_cast<const float4*>(a.qin + i);
                    const float4 w0 = __ldcg(p), w1 = __ldcg(p + 1);
                    org = f3(w0.x, w0.y, w0.z);
                    dir = f3(w1.x, w1.y, w1.z);
                    req = (int)((uint32_t)__float_as_int(w0.w) >> 24);
                    qi = i;
                }
                else
                {
                    PathRec pr = load_path(a.qin, i);
                    org = f3(pr.w0.x, pr.w0.y, pr.w0.z);
                    int tag = __float_as_int(pr.w0.w);
                    req = (int)((uint32_t)tag >> 24);
                    pixel = tag & 0xffffff;
                    dir = f3(pr.w1.x, pr.w1.y, pr.w1.z);
                    rng = __float_as_uint(pr.w1.w);
                }
                if (ok)
                {
                    has = true;
                    trav_setup(r, org, dir);
                    trav_init(ts, a.reqs[req].scene, FLT_MAX, st);
                }
            }
        }
        if (__ballot_sync(FULL, has) == 0)
        {
            if (exhausted) break;
            continue;
        }
        if (PRT_DEFER_TRIS && a.leaf1)
        {
            constexpr bool kPair = !kFirst && PRT_RELOAD_PATH && PRT_PAIRED_LATER;
            warp_trav_deferred<kPair>(*tq, ts, a.reqs[req].scene, r, 0.0f, st, has, !exhausted, kRefillMin, lane);
        }
        else
        for (;;)
        {
            if (has && !ts.done) trav_step<false>(ts, a.reqs[req].scene, r, 0.0f, st);
            unsigned running = __ballot_sync(FULL, has && !ts.done);
            if (running == 0) break;
            if (!exhausted && 32 - __popc(running) >= kRefillMin) break;
        }
        const bool fin = has && ts.done;
        bool cont = false;
        float contrib = 0.f;
        int fpix = 0;
        uint32_t frng = 0;
        float3 forg = r.org, fdir = f3(0.f, 0.f, 0.f);
        if (fin)
        {
            if (!kFirst && PRT_RELOAD_PATH)
            {
                const float4* p = reinterpret_cast<const float4*>(a.qin + qi);
                const float4 w1 = __ldcs(p + 1);
                fpix = __float_as_int(__ldcs(reinterpret_cast<const float*>(p) + 3)) & 0xffffff;
                fdir = f3(w1.x, w1.y, w1.z);
                frng = __float_as_uint(w1.w);
            }
            else
            {
                fpix = pixel;
                fdir = r.dir;
                frng = rng;
            }
            const BatchReq& R = a.reqs[req];
            if (ts.triHit < 0)
            {
                contrib = __fmul_rn(thrDepth, a.sky);
            }
            else if (depth < R.maxDepth)
            {
                diffuse_bounce(R.scene.tris, ts.triHit, forg, fdir, ts.tHit, frng);
                cont = true;
            }
        }
        int o = warp_append(cont, &a.counts[depth + 1]);
        if (cont) store_path(a.qout, o, forg, (req << 24) | fpix, fdir, frng);
        else if (fin) red_add_v4(a.reqs[req].accum + fpix, contrib, contrib, contrib, 1.0f);
        if (fin) has = false;
    }
    if (kFirst)
    {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) myRays += __shfl_down_sync(FULL, myRays, off);
        if (lane == 0 && myRays) atomicAdd(a.rays, myRays);
    }
}

// Depth 0 of the batched renderer as warp packets (k_primary_packet's
// traversal).  The 32 items a warp takes always belong to one request:
// requests own multiples of 64 paths, and the host uses this kernel only when
// waves start at multiples of 32 paths.
template <bool kIA>
__global__ void __launch_bounds__(128, 8) k_batch_primary_packet(BatchArgs a)
{
    extern __shared__ uint2 s_dyn[];
    long long* s_begin = reinterpret_cast<long long*>(s_dyn);
    uint2* stk = reinterpret_cast<uint2*>(s_begin + a.nreq) + (threadIdx.x >> 5) * kPacketStack;
    for (int q = threadIdx.x; q < a.nreq; q += blockDim.x) s_begin[q] = a.reqs[q].pathBegin;
    __syncthreads();
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const long long total = a.waveEnd - a.waveBegin;
    unsigned long long myRays = 0;
    for (;;)
    {
        int base = 0;
        if (lane == 0) base = atomicAdd(&a.fetch[0], 32);
        base = __shfl_sync(FULL, base, 0);
        if (base >= total) break;
        // the warp's request: the one whose path range holds its first item
        const long long g0 = a.waveBegin + base;
        int lo = 0, hi = a.nreq - 1;
        while (lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if (s_begin[mid] <= g0) lo = mid;
            else hi = mid - 1;
        }
        const int req = lo;
        const BatchReq& R = a.reqs[req];
        bool valid = false;
        int pixel = 0;
        uint32_t rng = 0;
        float3 org = f3(0.f, 0.f, 0.f), dir = f3(0.f, 0.f, 1.f);
        if (base + (long long)lane < total)
        {
            const long long local = g0 + lane - s_begin[req];
            const int perPass = R.tilesX * R.tilesY * 64;
            const int pass = (int)(local / perPass);
            int x, y;
            if (wave_item_pixel((int)(local - (long long)pass * perPass), R.tilesX, R.cam.width, R.cam.height, x, y))
            {
                valid = true;
                pixel = x + y * R.cam.width;
                rng = rng_seed(pass, pixel);
                camera_ray(R.cam, x, y, rng, org, dir);
                ++myRays;
            }
        }
        const unsigned vmask = __ballot_sync(FULL, valid);
        if (!vmask) continue;
        TravRay r;
        trav_setup(r, org, dir);
        float tHit;
        int primHit, triHit;
        packet_closest_hit<PRT_PAIRED_PACKET, kIA>(R.scene, r, valid, vmask, stk, lane, tHit, primHit, triHit);
        bool cont = false;
        float contrib = 0.f;
        if (valid)
        {
            if (triHit < 0)
            {
                contrib = a.sky;   // throughput 1 at depth 0
            }
            else if (R.maxDepth > 0)
            {
                diffuse_bounce(R.scene.tris, triHit, org, dir, tHit, rng);
                cont = true;
            }
        }
        const int o = warp_append(cont, &a.counts[1]);
        if (cont) store_path(a.qout, o, org, (req << 24) | pixel, dir, rng);
        else if (valid) red_add_v4(R.accum + pixel, contrib, contrib, contrib, 1.0f);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) myRays += __shfl_down_sync(FULL, myRays, off);
    if (lane == 0 && myRays) atomicAdd(a.rays, myRays);
}

template <class Kernel>
int grid_for(Kernel kernel, int block, size_t shmem, int numSMs, const LaunchCfg& cfg)
{
    int resident = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, block, shmem) != cudaSuccess || resident < 1)
        resident = 1;
    int perSM = cfg.blocksPerSM > 0 ? std::min(cfg.blocksPerSM, resident) : resident;
    return numSMs * perSM;
}

} // namespace

int launch_bounce(const WaveArgs& a, int depth, const LaunchCfg& cfg, int numSMs, cudaStream_t s)
{
    size_t shmem = sizeof(uint2) * kShared * cfg.block;
    if (a.scene.deferTris && (a.Lout ? PRT_DEFER_NEE : PRT_DEFER_TRIS))
        shmem += sizeof(TriQueue) * (cfg.block / 32);   // the bounce kernels' triangle queues
    bool albedo = a.thrIn != nullptr || a.thrOut != nullptr;
    auto go = [&](auto kernel) {
        int grid = grid_for(kernel, cfg.block, shmem, numSMs, cfg);
        kernel<<<grid, cfg.block, shmem, s>>>(a, depth);
    };
    if (a.Lout)
    {
        if (depth == 0)
        {
            if (albedo) go(k_bounce_nee<true, true>);
            else go(k_bounce_nee<true, false>);
        }
        else
        {
            if (albedo) go(k_bounce_nee<false, true>);
            else go(k_bounce_nee<false, false>);
        }
        return 1;
    }
    if (depth == 0 && PRT_PACKET_PRIMARY && cfg.packet && a.scene.leafTris == 1)
    {
        const size_t pshmem = sizeof(uint2) * kPacketStack * (cfg.block / 32);
        auto goPacket = [&](auto kernel) {
            int grid = grid_for(kernel, cfg.block, pshmem, numSMs, cfg);
            kernel<<<grid, cfg.block, pshmem, s>>>(a);
        };
        if (cfg.packet == 2)
        {
            if (albedo) goPacket(k_primary_packet<true, true>);
            else goPacket(k_primary_packet<false, true>);
        }
        else
        {
            if (albedo) goPacket(k_primary_packet<true, false>);
            else goPacket(k_primary_packet<false, false>);
        }
        return 1;
    }
    if (depth == 0)
    {
        if (albedo) go(k_bounce<true, true>);
        else go(k_bounce<true, false>);
    }
    else
    {
        if (albedo) go(k_bounce<false, true>);
        else go(k_bounce<false, false>);
    }
    return 1;
}

int launch_batch_bounce(const BatchArgs& a, int depth, const LaunchCfg& cfg, int numSMs, cudaStream_t s)
{
    size_t shmem = sizeof(uint2) * kShared * cfg.block + sizeof(long long) * a.nreq;
    if (PRT_DEFER_TRIS && a.leaf1) shmem += sizeof(TriQueue) * (cfg.block / 32);
    auto go = [&](auto kernel) {
        int grid = grid_for(kernel, cfg.block, shmem, numSMs, cfg);
        kernel<<<grid, cfg.block, shmem, s>>>(a, depth);
    };
    if (depth == 0 && PRT_PACKET_PRIMARY && cfg.packet && a.packet)
    {
        const size_t pshmem = sizeof(long long) * a.nreq + sizeof(uint2) * kPacketStack * (cfg.block / 32);
        auto goPacket = [&](auto kernel) {
            int grid = grid_for(kernel, cfg.block, pshmem, numSMs, cfg);
            kernel<<<grid, cfg.block, pshmem, s>>>(a);
        };
        if (cfg.packet == 2) goPacket(k_batch_primary_packet<true>);
        else goPacket(k_batch_primary_packet<false>);
        return 1;
    }
    if (depth == 0) go(k_batch_bounce<true>);
    else go(k_batch_bounce<false>);
    return 1;
}

int launch_intersect(const SceneDev& sc, const RayRec* rays, HitRec* hits, int n, bool anyHit, float* anyOut,
                     int* fetch, int numSMs, cudaStream_t s)
{
    if (n <= 0) return 0;
    const int block = 128;
    size_t shmem = sizeof(uint2) * kShared * block;
    if (PRT_DEFER_ISECT && sc.deferTris) shmem += sizeof(TriQueue) * (block / 32);
    LaunchCfg cfg;
    auto go = [&](auto kernel) {
        // no more warps than rays: 32 rays per warp
        int grid = std::min(grid_for(kernel, block, shmem, numSMs, cfg), (n + block - 1) / block);
        kernel<<<grid, block, shmem, s>>>(sc, rays, hits, anyOut, n, fetch);
    };
    if (anyHit) go(k_intersect<true>);
    else go(k_intersect<false>);
    return 1;
}

int launch_query(const SceneDev& sc, const RayRec* ray, HitRec* hit, float* pNg, cudaStream_t s)
{
    k_query<<<1, 1, 0, s>>>(sc, ray, hit, pNg);
    return 1;
}

int launch_resolve_ldr(const float4* accum, uint32_t* out, int n, cudaStream_t s)
{
    if (n <= 0) return 0;
    k_resolve_ldr<<<(n + 255) / 256, 256, 0, s>>>(accum, out, n);
    return 1;
}

namespace {

// The primary rays of one pass, written per pixel (row-major) as 32-byte ray
// records (org, tnear 0, dir, tfar FLT_MAX): the wave item -> pixel mapping,
// RNG seeding and camera_ray of the bounce kernels' first depth, exposed so
// the generated rays can be compared with a reference one by one.
__global__ void k_primary_rays(CameraDev cam, int tilesX, int tilesY, int pass, RayRec* out)
{
    const int perPass = tilesX * tilesY * 64;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < perPass; i += gridDim.x * blockDim.x)
    {
        int x, y;
        if (!wave_item_pixel(i, tilesX, cam.width, cam.height, x, y)) continue;
        const int pixel = x + y * cam.width;
        uint32_t rng = rng_seed(pass, pixel);
        float3 org, dir;
        camera_ray(cam, x, y, rng, org, dir);
        float4* o = reinterpret_cast<float4*>(out + pixel);
        o[0] = make_float4(org.x, org.y, org.z, 0.0f);
        o[1] = make_float4(dir.x, dir.y, dir.z, FLT_MAX);
    }
}

} // namespace

int launch_primary_rays(const CameraDev& cam, int pass, RayRec* out, cudaStream_t s)
{
    const int tilesX = (cam.width + 7) / 8, tilesY = (cam.height + 7) / 8;
    const int perPass = tilesX * tilesY * 64;
    if (perPass <= 0) return 0;
    k_primary_rays<<<std::min((perPass + 255) / 256, 4096), 256, 0, s>>>(cam, tilesX, tilesY, pass, out);
    return 1;
}

int launch_advance_pass(int* passBase, int spp, cudaStream_t s)
{
    k_advance_pass<<<1, 1, 0, s>>>(passBase, spp);
    return 1;
}

int launch_replay(const SceneDev& sc, const CameraDev& cam, float4* accum, int pass0, int spp, int maxDepth, float sky,
                  const float* dL, float* dAlbedo, float* dSky, unsigned long long* rays, int* fetch, bool backward,
                  int numSMs, cudaStream_t s)
{
    long long total = (long long)spp * cam.width * cam.height;
    if (total <= 0) return 0;
    const int block = 128;
    size_t shmem = sizeof(uint2) * kShared * block;
    // the backward kernel keeps in-lane triangle tests: with its gradient table
    // in shared memory the queues would cost it occupancy (measured 17% slower)
    if (PRT_DEFER_REPLAY && !backward && sc.deferTris) shmem += sizeof(TriQueue) * (block / 32);
    LaunchCfg cfg;
    auto go = [&](auto kernel) {
        int grid = grid_for(kernel, block, shmem, numSMs, cfg);
        kernel<<<grid, block, shmem, s>>>(sc, cam, accum, pass0, spp, maxDepth, sky, dL, dAlbedo, dSky, rays, fetch);
    };
    if (backward) go(k_replay<true>);
    else go(k_replay<false>);
    return 1;
}

int replay_max_depth() { return kReplayMaxDepth; }

int read_counters(unsigned long long* out, bool reset, cudaStream_t s)
{
    if (!PRT_COUNTERS) return -1;
    if (cudaMemcpyFromSymbolAsync(out, g_counters, sizeof(g_counters), 0, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return 1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return 1;
    if (reset)
    {
        static const unsigned long long zero[8] = {};
        if (cudaMemcpyToSymbolAsync(g_counters, zero, sizeof(zero), 0, cudaMemcpyHostToDevice, s) != cudaSuccess)
            return 1;
        if (cudaStreamSynchronize(s) != cudaSuccess) return 1;
    }
    return 0;
}

} // namespace prt_b200
