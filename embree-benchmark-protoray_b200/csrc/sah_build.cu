// Full SAH binary tree for the high-quality BVH build (build_bvh8 in
// bvh_build.cu groups and collapses it into 8-wide nodes).
//
// From the root (the triangles in Morton order), every task (a node and its
// contiguous range of triangles) with more than kSahLeaves triangles is split
// by binned SAH, its triangles are partitioned into the two halves of the
// range, and the halves become the next level's tasks, subtrees of
// 2..kSahLeaves triangles or leaves; each subtree is then built by one block
// with an exact sweep SAH.  Output: child / range / parent of the n - 1
// internal nodes (root 0; a child reference ~p is the triangle at position p
// of perm) and perm, the triangle order.
#include <algorithm>
#include <cfloat>
#include <vector>

#include "prt_device.cuh"
#include "prt_internal.h"

namespace prt_b200 {

// Task and split records of the top-down phase (declared in prt_internal.h).
struct TopTask
{
    int lo, hi, node, pad;
    float cmin[3], cmax[3];   // centroid bounds
};

struct TopSplit
{
    int axis;       // -1: no bin separates the centroids; split the range in the middle
    int bin;        // left: bins 0..bin
    int nl;         // triangles going left
    int pad;
    // centroid bounds of the two halves, as order-preserving bits (ford):
    // reduced with integer atomics by k_top_count
    uint32_t cmin[2][3], cmax[2][3];
};

namespace {

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

__device__ __forceinline__ float box_half_area_lh(const float* lo, const float* hi)
{
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
}

// --- subtrees of at most kSahLeaves triangles: exact sweep SAH, one block each -
//
// A subtree of 2..kSahLeaves triangles covers a contiguous range [a, b] of the
// triangle order; one block builds it top-down to single-triangle leaves, all
// nodes of a depth at once, permuting the triangles only inside [a, b].
// Splits: for each axis the range's triangles sorted by centroid, the split
// after position p costs area(left box) x |left| + area(right box) x |right|;
// the least cost wins (ties to the more balanced split, then the lower axis
// and position).
constexpr int kSahLeaves = 256;

struct SahShared
{
    float box[6][kSahLeaves];         // triangle boxes of the range (lo xyz, hi xyz)
    float cen[3][kSahLeaves];         // doubled centroids
    int list[2][3][kSahLeaves];       // per axis: elements in centroid order (double buffered)
    float scan[6][kSahLeaves];        // prefix / suffix boxes of one axis list
    float preArea[kSahLeaves];        // area of the prefix box ending at each position
    unsigned long long best[kSahLeaves];   // per segment: least split key
    int segStart[kSahLeaves], segEnd[kSahLeaves], segNode[kSahLeaves], segRight[kSahLeaves];
    int segOf[kSahLeaves];            // per position: its segment
    int rank[3][kSahLeaves];          // segmented scan of the left marks, per axis list
    int orig[kSahLeaves];             // triangle id of each element
    int pool[kSahLeaves];             // internal node indices of the subtree (root first)
    unsigned char mark[kSahLeaves];   // element goes left
    int nseg, poolNext, splitting, rootPos;   // rootPos: the first new node index
    int maxSeg, nextMaxSeg;   // largest segment of this depth / of the next
};

__device__ __forceinline__ float area6(float lx, float ly, float lz, float hx, float hy, float hz)
{
    const float dx = hx - lx, dy = hy - ly, dz = hz - lz;
    return dx * dy + dy * dz + dz * dx;
}

// One subtree per block: roots[i] is its root (an internal node whose range
// holds 2..kSahLeaves triangles); its other internal nodes take new indices
// from *nodeCounter.
__global__ void __launch_bounds__(kSahLeaves) k_sah_rebuild(int n, const int* __restrict__ roots,
                                                          const int* __restrict__ numRoots,
                                                          const float* __restrict__ triBox, uint32_t* vals,
                                                          int2* child, int2* range, int* parent, int* nodeCounter)
{
    __shared__ SahShared S;
    const int t = threadIdx.x;
    const int count = *numRoots;
    for (int ri = blockIdx.x; ri < count; ri += gridDim.x)
    {
        const int u = roots[ri];
        const int2 rg = range[u];
        const int a = rg.x, ns = rg.y - rg.x + 1;   // 2 <= ns <= kSahLeaves
        if (t == 0) S.rootPos = ns > 2 ? atomicAdd(nodeCounter, ns - 2) : 0;   // first new index
        // --- load the range ---------------------------------------------------
        if (t < ns)
        {
            const uint32_t tri = vals[a + t];
            S.orig[t] = (int)tri;
#pragma unroll
            for (int k = 0; k < 6; ++k) S.box[k][t] = triBox[6 * (size_t)tri + k];
#pragma unroll
            for (int k = 0; k < 3; ++k) S.cen[k][t] = S.box[k][t] + S.box[3 + k][t];
            S.segOf[t] = 0;
        }
        if (t == 0)
        {
            S.nseg = 1;
            S.segStart[0] = 0;
            S.segEnd[0] = ns - 1;
            S.poolNext = 1;
        }
        __syncthreads();
        if (t < ns - 1) S.pool[t] = t == 0 ? u : S.rootPos + t - 1;
        if (t == 0) S.segNode[0] = u;
        // --- per axis: elements sorted by centroid (bitonic, ties by element;
        //     the three axes side by side) ---------------------------------------
#pragma unroll
        for (int ax = 0; ax < 3; ++ax)
        {
            S.scan[ax][t] = t < ns ? S.cen[ax][t] : FLT_MAX;
            S.list[0][ax][t] = t < ns ? t : kSahLeaves + t;
        }
        __syncthreads();
        for (int size = 2; size <= kSahLeaves; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1)
            {
                const int o = t ^ stride;
                const bool up = (t & size) == 0;
                const bool lower = t < o;
                float ko[3];
                int io[3];
                bool take[3];
#pragma unroll
                for (int ax = 0; ax < 3; ++ax)
                {
                    ko[ax] = S.scan[ax][o];
                    io[ax] = S.list[0][ax][o];
                    const float km = S.scan[ax][t];
                    const int im = S.list[0][ax][t];
                    const bool mGreater = km > ko[ax] || (km == ko[ax] && im > io[ax]);
                    take[ax] = lower ? (up ? mGreater : !mGreater) : (up ? !mGreater : mGreater);
                }
                __syncthreads();
#pragma unroll
                for (int ax = 0; ax < 3; ++ax)
                    if (take[ax])
                    {
                        S.scan[ax][t] = ko[ax];
                        S.list[0][ax][t] = io[ax];
                    }
                __syncthreads();
            }
        int cur = 0;
        if (t == 0)
        {
            S.splitting = 0;
            S.maxSeg = ns;
        }
        __syncthreads();
        // --- one depth of the subtree per pass -------------------------------------
        for (int depth = 0; depth < kSahLeaves; ++depth)
        {
            if (t < S.nseg)
            {
                S.best[t] = ~0ull;
                if (S.segEnd[t] > S.segStart[t]) S.splitting = 1;
            }
            __syncthreads();
            if (!S.splitting) break;
            const int s = t < ns ? S.segOf[t] : 0;
            const int st0 = t < ns ? S.segStart[s] : 0, en0 = t < ns ? S.segEnd[s] : 0;
            const int span = S.maxSeg;   // scans within segments need log2(span) steps
            if (t == 0) S.nextMaxSeg = 1;
            for (int ax = 0; ax < 3; ++ax)
            {
                // prefix boxes along the axis list, within segments
                float v[6];
                if (t < ns)
                {
                    const int e = S.list[cur][ax][t];
#pragma unroll
                    for (int k = 0; k < 6; ++k) v[k] = S.box[k][e];
#pragma unroll
                    for (int k = 0; k < 6; ++k) S.scan[k][t] = v[k];
                }
                __syncthreads();
                for (int off = 1; off < span; off <<= 1)
                {
                    const bool take = t < ns && t - off >= st0;
                    float w[6];
                    if (take)
#pragma unroll
                        for (int k = 0; k < 6; ++k) w[k] = S.scan[k][t - off];
                    __syncthreads();
                    if (take)
                    {
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                        {
                            v[k] = fminf(v[k], w[k]);
                            v[3 + k] = fmaxf(v[3 + k], w[3 + k]);
                            S.scan[k][t] = v[k];
                            S.scan[3 + k][t] = v[3 + k];
                        }
                    }
                    __syncthreads();
                }
                if (t < ns) S.preArea[t] = area6(v[0], v[1], v[2], v[3], v[4], v[5]);
                // suffix boxes
                if (t < ns)
                {
                    const int e = S.list[cur][ax][t];
#pragma unroll
                    for (int k = 0; k < 6; ++k) v[k] = S.box[k][e];
                }
                __syncthreads();
                if (t < ns)
#pragma unroll
                    for (int k = 0; k < 6; ++k) S.scan[k][t] = v[k];
                __syncthreads();
                for (int off = 1; off < span; off <<= 1)
                {
                    const bool take = t < ns && t + off <= en0;
                    float w[6];
                    if (take)
#pragma unroll
                        for (int k = 0; k < 6; ++k) w[k] = S.scan[k][t + off];
                    __syncthreads();
                    if (take)
                    {
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                        {
                            v[k] = fminf(v[k], w[k]);
                            v[3 + k] = fmaxf(v[3 + k], w[3 + k]);
                            S.scan[k][t] = v[k];
                            S.scan[3 + k][t] = v[3 + k];
                        }
                    }
                    __syncthreads();
                }
                // cost of the split after position t (the suffix from t + 1)
                if (t < ns && t < en0)
                {
                    const float sa = area6(S.scan[0][t + 1], S.scan[1][t + 1], S.scan[2][t + 1], S.scan[3][t + 1],
                                           S.scan[4][t + 1], S.scan[5][t + 1]);
                    const int nl = t - st0 + 1, nr = en0 - t;
                    const float c = S.preArea[t] * (float)nl + sa * (float)nr;
                    const unsigned imbalance = (unsigned)abs(nl - nr);
                    const unsigned long long key = ((unsigned long long)__float_as_uint(fmaxf(c, 0.f)) << 32) |
                                                   ((unsigned long long)imbalance << 16) | ((unsigned)ax << 8) |
                                                   (unsigned)(t - st0);
                    atomicMin(&S.best[s], key);
                }
                __syncthreads();
            }
            // marks: the chosen axis list's prefix goes left
            if (t < ns && en0 > st0)
            {
                const unsigned long long b = S.best[s];
                const int ax = (int)((b >> 8) & 0xff), sp = st0 + (int)(b & 0xff);
                S.mark[S.list[cur][ax][t]] = t <= sp ? 1 : 0;
            }
            __syncthreads();
            // stable partition of the three lists within the splitting segments
            int m[3] = {0, 0, 0};
            if (t < ns && en0 > st0)
#pragma unroll
                for (int ax = 0; ax < 3; ++ax) m[ax] = S.mark[S.list[cur][ax][t]];
            int incl[3] = {m[0], m[1], m[2]};
            if (t < ns)
#pragma unroll
                for (int ax = 0; ax < 3; ++ax) S.rank[ax][t] = incl[ax];
            __syncthreads();
            for (int off = 1; off < span; off <<= 1)
            {
                const bool take = t < ns && t - off >= st0;
                int w[3] = {0, 0, 0};
                if (take)
#pragma unroll
                    for (int ax = 0; ax < 3; ++ax) w[ax] = S.rank[ax][t - off];
                __syncthreads();
                if (take)
#pragma unroll
                    for (int ax = 0; ax < 3; ++ax)
                    {
                        incl[ax] += w[ax];
                        S.rank[ax][t] = incl[ax];
                    }
                __syncthreads();
            }
            if (t < ns)
            {
                if (en0 > st0)
                {
                    const unsigned long long b = S.best[s];
                    const int nl = (int)(b & 0xff) + 1;
#pragma unroll
                    for (int ax = 0; ax < 3; ++ax)
                    {
                        const int before = incl[ax] - m[ax];   // left elements before t in the segment
                        const int np = m[ax] ? st0 + before : st0 + nl + (t - st0 - before);
                        S.list[cur ^ 1][ax][np] = S.list[cur][ax][t];
                    }
                }
                else
                {
#pragma unroll
                    for (int ax = 0; ax < 3; ++ax) S.list[cur ^ 1][ax][t] = S.list[cur][ax][t];
                }
            }
            __syncthreads();
            // nodes: each splitting segment is an internal node with two children
            const int nsegOld = S.nseg;
            __syncthreads();
            if (t < nsegOld && S.segEnd[t] > S.segStart[t])
            {
                const int st = S.segStart[t], en = S.segEnd[t], node = S.segNode[t];
                const int sp = st + (int)(S.best[t] & 0xff);
                int refs[2];
                const int cs[2] = {st, sp + 1}, ce[2] = {sp, en};
                const int right = atomicAdd(&S.nseg, 1);
#pragma unroll
                for (int c = 0; c < 2; ++c)
                {
                    const int segId = c == 0 ? t : right;
                    if (ce[c] == cs[c])
                    {
                        refs[c] = ~(a + cs[c]);
                        parent[(n - 1) + a + cs[c]] = node;
                        S.segNode[segId] = -1;
                    }
                    else
                    {
                        const int id = S.pool[atomicAdd(&S.poolNext, 1)];
                        refs[c] = id;
                        parent[id] = node;
                        range[id] = make_int2(a + cs[c], a + ce[c]);
                        S.segNode[segId] = id;
                    }
                }
                child[node] = make_int2(refs[0], refs[1]);
                atomicMax(&S.nextMaxSeg, max(sp - st + 1, en - sp));
                S.segRight[t] = right;
                S.segStart[right] = sp + 1;
                S.segEnd[right] = en;
                S.segEnd[t] = sp;
            }
            __syncthreads();
            if (t < ns && en0 > st0)
            {
                const unsigned long long b = S.best[s];
                const int sp = st0 + (int)(b & 0xff);
                if (t > sp) S.segOf[t] = S.segRight[s];
            }
            if (t == 0)
            {
                S.splitting = 0;
                S.maxSeg = S.nextMaxSeg;
            }
            cur ^= 1;
            __syncthreads();
        }
        // the triangles in their new order
        if (t < ns) vals[a + t] = (uint32_t)S.orig[S.list[cur][0][t]];
        __syncthreads();
    }
}

// --- above kSahLeaves triangles: top-down binned SAH ----------------------------
//
// The high-quality build makes a full SAH tree instead of the Morton
// hierarchy.  From the root (the triangles in Morton order), every task (a
// node and its contiguous range of triangles) with more than kSahLeaves
// triangles is split by the least SAH cost over
// kTopBins centroid bins per axis (bin boxes and counts gathered per chunk of
// the range in shared memory, then merged with atomics), its triangles are
// partitioned into the two halves of the range, and the halves become the
// next level's tasks, k_sah_rebuild's subtrees (2..kSahLeaves triangles) or
// leaves.  The halves' centroid bounds (the next level's bin ranges) are
// gathered by the counting pass over the split, not per bin.  One host
// read-back per level (the next tasks' count and ranges) sizes the next
// level's launches.
constexpr int kTopBins = 32;
constexpr int kTopChunk = 4096;        // triangles per block of the binning and partition passes
constexpr int kBinWords = 7;           // count, box lo, box hi (order-preserving float bits)

__device__ __forceinline__ uint32_t ford(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funord(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ int top_bin(float c, float cmin, float scale)
{
    return min(kTopBins - 1, max(0, (int)((c - cmin) * scale)));
}

__device__ __forceinline__ float top_scale(float cmin, float cmax)
{
    const float e = cmax - cmin;
    return e > 0.f ? (float)kTopBins * 0.99999f / e : 0.f;
}

__global__ void k_top_init_bins(uint32_t* bins, int words)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x)
    {
        const int w = i % kBinWords;
        // count 0; lo fields (1-3) start at the largest value, hi fields (4-6) at 0
        bins[i] = w == 0 ? 0u : (w <= 3 ? 0xffffffffu : 0u);
    }
}

// Chunk c: task chunks[c].x, triangles [chunks[c].y, chunks[c].z].
__global__ void __launch_bounds__(256) k_top_bin(const int4* __restrict__ chunks, const TopTask* __restrict__ tasks,
                                                 const uint32_t* __restrict__ perm, const float* __restrict__ triBox,
                                                 uint32_t* bins)
{
    __shared__ uint32_t sb[3 * kTopBins * kBinWords];
    const int4 ch = chunks[blockIdx.x];
    const TopTask tk = tasks[ch.x];
    for (int i = threadIdx.x; i < 3 * kTopBins * kBinWords; i += blockDim.x)
    {
        const int w = i % kBinWords;
        sb[i] = w == 0 ? 0u : (w <= 3 ? 0xffffffffu : 0u);
    }
    __syncthreads();
    float sc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) sc[k] = top_scale(tk.cmin[k], tk.cmax[k]);
    const unsigned lane = threadIdx.x & 31u;
    for (int i0 = ch.y; i0 <= ch.z; i0 += blockDim.x)
    {
        // the lanes of a warp that fall into one bin (neighbours in the
        // triangle order often do) merge their boxes with warp reductions and
        // one lane updates the bin
        const int i = i0 + threadIdx.x;
        const bool valid = i <= ch.z;
        uint32_t lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0, 0, 0};
        float c[3] = {0.f, 0.f, 0.f};
        if (valid)
        {
            const uint32_t tri = perm[i];
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                const float bl = triBox[6 * (size_t)tri + k], bh = triBox[6 * (size_t)tri + 3 + k];
                lo[k] = ford(bl);
                hi[k] = ford(bh);
                c[k] = 0.5f * (bl + bh);
            }
        }
#pragma unroll
        for (int ax = 0; ax < 3; ++ax)
        {
            const int bin = valid ? top_bin(c[ax], tk.cmin[ax], sc[ax]) : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, bin);
            uint32_t r[7];
            r[0] = __popc(peers);
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                r[1 + k] = __reduce_min_sync(peers, lo[k]);
                r[4 + k] = __reduce_max_sync(peers, hi[k]);
            }
            if (valid && lane == (unsigned)(__ffs(peers) - 1))
            {
                uint32_t* w = sb + (ax * kTopBins + bin) * kBinWords;
                atomicAdd(w, r[0]);
#pragma unroll
                for (int k = 0; k < 3; ++k)
                {
                    atomicMin(w + 1 + k, r[1 + k]);
                    atomicMax(w + 4 + k, r[4 + k]);
                }
            }
        }
    }
    __syncthreads();
    uint32_t* g = bins + (size_t)ch.x * 3 * kTopBins * kBinWords;
    for (int i = threadIdx.x; i < 3 * kTopBins * kBinWords; i += blockDim.x)
    {
        const int w = i % kBinWords;
        if (w == 0)
        {
            if (sb[i]) atomicAdd(g + i, sb[i]);
        }
        else if (w <= 3)
        {
            if (sb[i] != 0xffffffffu) atomicMin(g + i, sb[i]);
        }
        else if (sb[i])
        {
            atomicMax(g + i, sb[i]);
        }
    }
}

__device__ __forceinline__ float shfl_ud(float v, int off, bool down)
{
    return down ? __shfl_down_sync(0xffffffffu, v, off) : __shfl_up_sync(0xffffffffu, v, off);
}

// One warp per task, lane b = bin b: the least-cost split over the bins of
// the three axes (prefix and suffix boxes by warp scans; ties to the lower
// axis, then the lower bin).  The halves' centroid bounds start empty here
// and are gathered by k_top_count.
__global__ void k_top_split(const TopTask* __restrict__ tasks, int numTasks, const uint32_t* __restrict__ bins,
                            TopSplit* splits)
{
    static_assert(kTopBins == 32, "one lane per bin");
    const int ti = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (ti >= numTasks) return;   // warp-uniform
    const int lane = threadIdx.x & 31;
    const TopTask tk = tasks[ti];
    const uint32_t* g = bins + (size_t)ti * 3 * kTopBins * kBinWords;
    unsigned long long best = ~0ull;   // (cost bits << 32) | (axis * 32 + bin)
    for (int ax = 0; ax < 3; ++ax)
    {
        const uint32_t* w = g + (ax * kTopBins + lane) * kBinWords;
        const int cnt = (int)w[0];
        float lo[3], hi[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            lo[k] = cnt ? funord(w[1 + k]) : FLT_MAX;
            hi[k] = cnt ? funord(w[4 + k]) : -FLT_MAX;
        }
        // left: inclusive prefix over bins 0..lane; right: suffix over lane..31
        int lc = cnt, rc = cnt;
        float llo[3], lhi[3], rlo[3], rhi[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            llo[k] = rlo[k] = lo[k];
            lhi[k] = rhi[k] = hi[k];
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const int ulc = __shfl_up_sync(0xffffffffu, lc, off);
            const int drc = __shfl_down_sync(0xffffffffu, rc, off);
            float ul[3], uh[3], dl[3], dh[3];
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                ul[k] = shfl_ud(llo[k], off, false);
                uh[k] = shfl_ud(lhi[k], off, false);
                dl[k] = shfl_ud(rlo[k], off, true);
                dh[k] = shfl_ud(rhi[k], off, true);
            }
            if (lane >= off)
            {
                lc += ulc;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                {
                    llo[k] = fminf(llo[k], ul[k]);
                    lhi[k] = fmaxf(lhi[k], uh[k]);
                }
            }
            if (lane + off < 32)
            {
                rc += drc;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                {
                    rlo[k] = fminf(rlo[k], dl[k]);
                    rhi[k] = fmaxf(rhi[k], dh[k]);
                }
            }
        }
        // split after bin `lane`: the suffix from lane + 1
        const int nrc = __shfl_down_sync(0xffffffffu, rc, 1);
        float nlo[3], nhi[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            nlo[k] = __shfl_down_sync(0xffffffffu, rlo[k], 1);
            nhi[k] = __shfl_down_sync(0xffffffffu, rhi[k], 1);
        }
        if (lane < 31 && lc > 0 && nrc > 0)
        {
            const float c = box_half_area_lh(llo, lhi) * (float)lc + box_half_area_lh(nlo, nhi) * (float)nrc;
            const unsigned long long key = ((unsigned long long)__float_as_uint(fmaxf(c, 0.f)) << 32) |
                                           (unsigned)(ax * kTopBins + lane);
            best = key < best ? key : best;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, best, off);
        best = o < best ? o : best;
    }
    TopSplit sp;
    sp.pad = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            sp.cmin[h][k] = 0xffffffffu;
            sp.cmax[h][k] = 0u;
        }
    if (best == ~0ull)
    {
        sp.axis = -1;
        sp.bin = 0;
        sp.nl = (tk.hi - tk.lo + 1) / 2;
    }
    else
    {
        const int code = (int)(best & 0xffffffffu);
        sp.axis = code / kTopBins;
        sp.bin = code % kTopBins;
        const uint32_t* w = g + (sp.axis * kTopBins + lane) * kBinWords;
        const int cnt = (int)w[0];
        sp.nl = __reduce_add_sync(0xffffffffu, lane <= sp.bin ? cnt : 0);
    }
    if (lane == 0) splits[ti] = sp;
}

// One thread per task: the two halves become internal nodes (next-level tasks
// or rebuild subtrees) or leaves.
__global__ void k_top_children(const TopTask* __restrict__ tasks, int numTasks, const TopSplit* __restrict__ splits,
                               int n, TopTask* nextTasks, int* numNext,
                               int* small, int* numSmall, int* nodeCounter, int2* child, int2* range, int* parent)
{
    const int ti = blockIdx.x * blockDim.x + threadIdx.x;
    if (ti >= numTasks) return;
    const TopTask tk = tasks[ti];
    const TopSplit sp = splits[ti];
    const int lo[2] = {tk.lo, tk.lo + sp.nl}, hi[2] = {tk.lo + sp.nl - 1, tk.hi};
    int refs[2];
    for (int side = 0; side < 2; ++side)
    {
        const int size = hi[side] - lo[side] + 1;
        if (size == 1)
        {
            refs[side] = ~lo[side];
            parent[(n - 1) + lo[side]] = tk.node;
            continue;
        }
        const int id = atomicAdd(nodeCounter, 1);
        refs[side] = id;
        parent[id] = tk.node;
        range[id] = make_int2(lo[side], hi[side]);
        if (size <= kSahLeaves)
        {
            small[atomicAdd(numSmall, 1)] = id;
            continue;
        }
        TopTask c;
        c.lo = lo[side];
        c.hi = hi[side];
        c.node = id;
        c.pad = 0;
        for (int k = 0; k < 3; ++k)
        {
            c.cmin[k] = funord(sp.cmin[side][k]);
            c.cmax[k] = funord(sp.cmax[side][k]);
        }
        nextTasks[atomicAdd(numNext, 1)] = c;
    }
    child[tk.node] = make_int2(refs[0], refs[1]);
}

__device__ __forceinline__ int top_side(const TopTask& tk, const TopSplit& sp, float sc, int i, uint32_t tri,
                                        const float* __restrict__ triBox)
{
    if (sp.axis < 0) return i - tk.lo < sp.nl ? 0 : 1;
    const float c = 0.5f * (triBox[6 * (size_t)tri + sp.axis] + triBox[6 * (size_t)tri + 3 + sp.axis]);
    return top_bin(c, tk.cmin[sp.axis], sc) <= sp.bin ? 0 : 1;
}

// Triangles of each chunk that go left, and the centroid bounds of the two
// halves (merged into the task's split record with integer atomics on the
// order-preserving bits).
__global__ void __launch_bounds__(256) k_top_count(const int4* __restrict__ chunks, const TopTask* __restrict__ tasks,
                                                   TopSplit* splits, const uint32_t* __restrict__ perm,
                                                   const float* __restrict__ triBox, uint32_t* leftCount)
{
    __shared__ int warpCount[8];
    const int4 ch = chunks[blockIdx.x];
    const TopTask tk = tasks[ch.x];
    TopSplit sp;
    sp.axis = splits[ch.x].axis;
    sp.bin = splits[ch.x].bin;
    sp.nl = splits[ch.x].nl;
    const float sc = sp.axis >= 0 ? top_scale(tk.cmin[sp.axis], tk.cmax[sp.axis]) : 0.f;
    int mine = 0;
    uint32_t cmin[2][3], cmax[2][3];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            cmin[h][k] = 0xffffffffu;
            cmax[h][k] = 0u;
        }
    for (int i = ch.y + threadIdx.x; i <= ch.z; i += blockDim.x)
    {
        const uint32_t tri = perm[i];
        const int side = top_side(tk, sp, sc, i, tri, triBox);
        mine += side == 0;
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            const uint32_t c = ford(0.5f * (triBox[6 * (size_t)tri + k] + triBox[6 * (size_t)tri + 3 + k]));
            if (side == 0)
            {
                cmin[0][k] = min(cmin[0][k], c);
                cmax[0][k] = max(cmax[0][k], c);
            }
            else
            {
                cmin[1][k] = min(cmin[1][k], c);
                cmax[1][k] = max(cmax[1][k], c);
            }
        }
    }
    mine = __reduce_add_sync(0xffffffffu, mine);
    if ((threadIdx.x & 31) == 0) warpCount[threadIdx.x >> 5] = mine;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            const uint32_t lo = __reduce_min_sync(0xffffffffu, cmin[h][k]);
            const uint32_t hi = __reduce_max_sync(0xffffffffu, cmax[h][k]);
            if ((threadIdx.x & 31) == 0)
            {
                if (lo != 0xffffffffu) atomicMin(&splits[ch.x].cmin[h][k], lo);
                if (hi != 0u) atomicMax(&splits[ch.x].cmax[h][k], hi);
            }
        }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        int tot = 0;
        for (int w = 0; w < 8; ++w) tot += warpCount[w];
        leftCount[blockIdx.x] = (uint32_t)tot;
    }
}

// The triangles of each chunk to their half of the task's range (in tmp), in
// their order: leftBase = the chunk's left triangles before it in its task
// (exclusive scan of k_top_count's counts minus the scan at the task's first
// chunk, chunks[c].w).
__global__ void __launch_bounds__(256) k_top_partition(const int4* __restrict__ chunks,
                                                       const TopTask* __restrict__ tasks,
                                                       const TopSplit* __restrict__ splits,
                                                       const uint32_t* __restrict__ perm,
                                                       const float* __restrict__ triBox,
                                                       const uint32_t* __restrict__ leftScan, uint32_t* tmp)
{
    __shared__ int warpCount[2][8];
    const int4 ch = chunks[blockIdx.x];
    const TopTask tk = tasks[ch.x];
    const TopSplit sp = splits[ch.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float sc = sp.axis >= 0 ? top_scale(tk.cmin[sp.axis], tk.cmax[sp.axis]) : 0.f;
    int base[2];
    base[0] = (int)(leftScan[blockIdx.x] - leftScan[ch.w]);
    base[1] = (ch.y - tk.lo) - base[0];
    for (int i0 = ch.y; i0 <= ch.z; i0 += blockDim.x)
    {
        const int i = i0 + threadIdx.x;
        const bool valid = i <= ch.z;
        uint32_t tri = 0;
        int side = 0;
        if (valid)
        {
            tri = perm[i];
            side = top_side(tk, sp, sc, i, tri, triBox);
        }
        const unsigned left = __ballot_sync(0xffffffffu, valid && side == 0);
        const unsigned right = __ballot_sync(0xffffffffu, valid && side == 1);
        if (lane == 0)
        {
            warpCount[0][warp] = __popc(left);
            warpCount[1][warp] = __popc(right);
        }
        __syncthreads();
        if (valid)
        {
            int before = 0;
            for (int w = 0; w < warp; ++w) before += warpCount[side][w];
            const unsigned m = side == 0 ? left : right;
            const int r = base[side] + before + __popc(m & ((1u << lane) - 1u));
            const int dst = side == 0 ? tk.lo + r : tk.lo + sp.nl + r;
            if (dst <= tk.hi) tmp[dst] = tri;
        }
        int tl = 0, tr = 0;
        for (int w = 0; w < 8; ++w)
        {
            tl += warpCount[0][w];
            tr += warpCount[1][w];
        }
        base[0] += tl;
        base[1] += tr;
        __syncthreads();
    }
}

__global__ void k_top_copy(const int4* __restrict__ chunks, const uint32_t* __restrict__ tmp, uint32_t* perm)
{
    const int4 ch = chunks[blockIdx.x];
    for (int i = ch.y + threadIdx.x; i <= ch.z; i += blockDim.x) perm[i] = tmp[i];
}

// The root: node 0 over all n triangles, a task (n > kSahLeaves) or a rebuild
// subtree.  counters: [0] next-level tasks, [1] rebuild subtrees, [2] nodes.
__global__ void k_top_root(const float* __restrict__ cbounds, int n, TopTask* tasks, int* small, int* counters,
                           int2* range, int* parent)
{
    range[0] = make_int2(0, n - 1);
    parent[0] = -1;
    counters[0] = 0;
    counters[1] = 0;
    counters[2] = 1;
    if (n <= kSahLeaves)
    {
        small[0] = 0;
        counters[1] = 1;
        return;
    }
    TopTask t;
    t.lo = 0;
    t.hi = n - 1;
    t.node = 0;
    t.pad = 0;
    for (int k = 0; k < 3; ++k)
    {
        t.cmin[k] = cbounds[k];
        t.cmax[k] = cbounds[3 + k];
    }
    tasks[0] = t;
}

} // namespace

void sah_tree_carve(Carve& c, int n, SahTreeBuffers& B)
{
    B.maxTasks = n / (kSahLeaves + 1) + 2;
    B.maxChunks = n / kTopChunk + B.maxTasks + 2;
    B.task[0] = c.take<TopTask>(B.maxTasks);
    B.task[1] = c.take<TopTask>(B.maxTasks);
    B.splits = c.take<TopSplit>(B.maxTasks);
    B.bins = c.take<uint32_t>((size_t)B.maxTasks * 3 * kTopBins * kBinWords);
    B.leftCount = c.take<uint32_t>(B.maxChunks);
    B.scanSums = c.take<uint32_t>(scan_sums_entries(B.maxChunks));
    B.small = c.take<int>((size_t)n / 2 + 1);
    B.counters = c.take<int>(3);
    B.chunks = c.take<int4>(B.maxChunks);
}


// Top-down binned SAH from the root down to subtrees of kSahLeaves triangles,
// then k_sah_rebuild for those.  perm: the triangles (reordered in place).
cudaError_t sah_build_tree(int n, const float* triBox, const float* cbounds, uint32_t* perm, int2* child, int2* range,
                           int* parent, const SahTreeBuffers& B, int numSMs, cudaStream_t stream)
{
    k_top_root<<<1, 1, 0, stream>>>(cbounds, n, B.task[0], B.small, B.counters, range, parent);
    cudaError_t e = cudaGetLastError();
    int numTasks = n > kSahLeaves ? 1 : 0;
    int cur = 0;
    std::vector<TopTask> host(1);   // the tasks' ranges (the root's is known)
    host[0].lo = 0;
    host[0].hi = n - 1;
    std::vector<int4> chunks;
    while (e == cudaSuccess && numTasks > 0)
    {
        if (numTasks > B.maxTasks) return cudaErrorInvalidValue;
        chunks.clear();
        for (int ti = 0; ti < numTasks; ++ti)
        {
            const int first = (int)chunks.size();
            for (int s = host[ti].lo; s <= host[ti].hi; s += kTopChunk)
                chunks.push_back(make_int4(ti, s, std::min(host[ti].hi, s + kTopChunk - 1), first));
        }
        const int nch = (int)chunks.size();
        if (nch > B.maxChunks) return cudaErrorInvalidValue;
        e = cudaMemcpyAsync(B.chunks, chunks.data(), sizeof(int4) * nch, cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) break;
        const int words = numTasks * 3 * kTopBins * kBinWords;
        k_top_init_bins<<<std::min(div_up(words, 256), 4 * numSMs), 256, 0, stream>>>(B.bins, words);
        k_top_bin<<<nch, 256, 0, stream>>>(B.chunks, B.task[cur], perm, triBox, B.bins);
        k_top_split<<<div_up(numTasks, 4), 128, 0, stream>>>(B.task[cur], numTasks, B.bins, B.splits);
        k_top_count<<<nch, 256, 0, stream>>>(B.chunks, B.task[cur], B.splits, perm, triBox, B.leftCount);
        e = cudaMemsetAsync(B.counters, 0, sizeof(int), stream);
        if (e != cudaSuccess) break;
        k_top_children<<<div_up(numTasks, 128), 128, 0, stream>>>(B.task[cur], numTasks, B.splits, n,
                                                                   B.task[cur ^ 1], B.counters, B.small,
                                                                   B.counters + 1, B.counters + 2, child, range,
                                                                   parent);
        exclusive_scan_u32(B.leftCount, B.leftCount, B.scanSums, nch, stream);
        k_top_partition<<<nch, 256, 0, stream>>>(B.chunks, B.task[cur], B.splits, perm, triBox, B.leftCount, B.tmp);
        k_top_copy<<<nch, 256, 0, stream>>>(B.chunks, B.tmp, perm);
        e = cudaGetLastError();
        // one read-back per level: the count and the ranges of the next tasks
        // (at most two per task)
        const int cap = std::min(B.maxTasks, 2 * numTasks);
        host.resize(cap);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&numTasks, B.counters, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(host.data(), B.task[cur ^ 1], sizeof(TopTask) * cap, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        cur ^= 1;
    }
    if (e != cudaSuccess) return e;
    int perSM = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_sah_rebuild, kSahLeaves, 0);
    k_sah_rebuild<<<std::max(1, perSM) * numSMs, kSahLeaves, 0, stream>>>(n, B.small, B.counters + 1, triBox, perm,
                                                                       child, range, parent, B.counters + 2);
    return cudaGetLastError();
}


} // namespace prt_b200
