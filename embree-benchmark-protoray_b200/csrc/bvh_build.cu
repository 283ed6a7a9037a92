// GPU BVH build into the compressed 8-wide node layout of prt_device.cuh.
//
// Replaces the acceleration-structure build of the reference's GPU path
// (OptiX Prime model->setTriangles/update, accel/optix/optix_intersector_stream_cuda.cpp:49-59;
// Embree rtcCommitScene on the CPU, accel/embree/embree_intersector.cpp:65-85).
//
// Steps (all on the device):
//   1. triangle boxes + centroid bounds (block partials, one final reduce)
//   2. 30-bit Morton codes of the centroids (10 bits per axis)
//   3. stable LSD radix sort of (code, triangle) pairs, 8-bit digits
//   4. the binary tree: for the high-quality build (default) a full SAH tree
//      built top-down from that order (binned SAH above kSahLeaves triangles,
//      an exact sweep SAH per block below); otherwise the binary radix tree
//      over the sorted codes (Karras, HPG 2012; equal codes are ordered by
//      their position, so duplicates are handled)
//   5. bottom-up bounds refit (second child to arrive computes the union),
//      fused with the SAH-optimal grouping of the binary nodes into 8-wide
//      nodes (dynamic program of Ylitie et al. 2017 over the binary tree)
//   6. top-down collapse into 8-wide nodes, one tree level per launch (no
//      host round trip between levels), one 8-lane group per node:
//      children are the roots chosen by the dynamic program (or, for trees
//      the program makes deeper than the traversal stack, opened greedily by
//      largest surface area while fewer than 8 exist); child slots are
//      assigned so that slot s holds the child nearest the origin of rays in
//      direction octant s; child boxes are quantized to 8 bits per axis.
#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "prt_device.cuh"
#include "prt_internal.h"

namespace prt_b200 {

namespace {

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

struct Box6
{
    float lo[3], hi[3];
};

__device__ __forceinline__ uint32_t expand10(uint32_t v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// --- 1. triangle boxes and centroid bounds --------------------------------

__global__ void k_tri_boxes(const float* __restrict__ pos, const int* __restrict__ idx, int nt, float* __restrict__ triBox,
                            float* __restrict__ partial)
{
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nt; p += gridDim.x * blockDim.x)
    {
        int i0 = idx[3 * p], i1 = idx[3 * p + 1], i2 = idx[3 * p + 2];
        float lo[3], hi[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            float a = pos[3 * i0 + k], b = pos[3 * i1 + k], c = pos[3 * i2 + k];
            lo[k] = fminf(a, fminf(b, c));
            hi[k] = fmaxf(a, fmaxf(b, c));
            triBox[6 * (size_t)p + k] = lo[k];
            triBox[6 * (size_t)p + 3 + k] = hi[k];
            float cc = 0.5f * (lo[k] + hi[k]);
            clo[k] = fminf(clo[k], cc);
            chi[k] = fmaxf(chi[k], cc);
        }
    }
    __shared__ float s[6][256];
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        s[k][threadIdx.x] = clo[k];
        s[3 + k][threadIdx.x] = chi[k];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1)
    {
        if ((int)threadIdx.x < w)
        {
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                s[k][threadIdx.x] = fminf(s[k][threadIdx.x], s[k][threadIdx.x + w]);
                s[3 + k][threadIdx.x] = fmaxf(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < 6) partial[6 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

__global__ void k_reduce_bounds(const float* __restrict__ partial, int nblocks, float* __restrict__ out)
{
    __shared__ float s[6][256];
    float v[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        for (int k = 0; k < 3; ++k)
        {
            v[k] = fminf(v[k], partial[6 * b + k]);
            v[3 + k] = fmaxf(v[3 + k], partial[6 * b + 3 + k]);
        }
    for (int k = 0; k < 6; ++k) s[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1)
    {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < 3; ++k)
            {
                s[k][threadIdx.x] = fminf(s[k][threadIdx.x], s[k][threadIdx.x + w]);
                s[3 + k][threadIdx.x] = fmaxf(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) out[threadIdx.x] = s[threadIdx.x][0];
}

// --- 2. Morton codes -------------------------------------------------------

// Cells of the Morton grid: per-axis normalisation (0) stretches a flat scene's
// thin axis to the full 10 bits, so high tree levels split along it; cubic
// cells (1) normalise every axis by the largest extent.
#ifndef PRT_MORTON_CUBE
#define PRT_MORTON_CUBE 0
#endif

__global__ void k_morton(const float* __restrict__ triBox, int nt, const float* __restrict__ cb, uint32_t* __restrict__ keys,
                         uint32_t* __restrict__ vals)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nt) return;
    uint32_t code = 0;
    const float extMax = fmaxf(cb[3] - cb[0], fmaxf(cb[4] - cb[1], cb[5] - cb[2]));
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        float c = 0.5f * (triBox[6 * (size_t)p + k] + triBox[6 * (size_t)p + 3 + k]);
        float ext = PRT_MORTON_CUBE ? extMax : cb[3 + k] - cb[k];
        float u = ext > 0.f ? (c - cb[k]) / ext : 0.f;
        uint32_t q = (uint32_t)fminf(fmaxf(u * 1024.0f, 0.0f), 1023.0f);
        code |= expand10(q) << k;
    }
    keys[p] = code;
    vals[p] = (uint32_t)p;
}

// --- 3. radix sort: radix_sort_pairs (sort_scan.cu) -------------------------

// --- 4. Karras binary radix tree --------------------------------------------

__device__ __forceinline__ int delta(const uint32_t* __restrict__ keys, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    uint32_t a = keys[i], b = keys[j];
    if (a != b) return __clz(a ^ b);
    return 32 + __clz((uint32_t)i ^ (uint32_t)j);
}

// internal nodes 0..n-2; child encoding: >= 0 internal, < 0 leaf ~k
__global__ void k_karras(const uint32_t* __restrict__ keys, int n, int2* __restrict__ child, int2* __restrict__ range,
                         int* __restrict__ parent)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(keys, n, i, j);
    int s = 0;
    int t = l;
    do
    {
        t = (t + 1) >> 1;
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int gamma = i + s * d + min(d, 0);
    int lo = min(i, j), hi = max(i, j);
    int left = (lo == gamma) ? ~gamma : gamma;
    int right = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    child[i] = make_int2(left, right);
    range[i] = make_int2(lo, hi);
    // parents: internal nodes at [0, n-1), leaves at [n-1, 2n-1)
    parent[left >= 0 ? left : (n - 1) + ~left] = i;
    parent[right >= 0 ? right : (n - 1) + ~right] = i;
    if (i == 0) parent[0] = -1;
}

__device__ __forceinline__ float box_half_area_lh(const float* lo, const float* hi)
{
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
}

// --- 4b. exact sweep SAH for subtrees of at most kSahLeaves triangles ---------
//
// A subtree of 2..kSahLeaves triangles covers a contiguous range [a, b] of the
// triangle order; one block builds it top-down to single-triangle leaves, all
// nodes of a depth at once, permuting the triangles only inside [a, b].
// Splits: for each axis the range's triangles sorted by centroid, the split
// after position p costs area(left box) x |left| + area(right box) x |right|;
// the least cost wins (ties to the more balanced split, then the lower axis
// and position).
#ifndef PRT_SAH_BUILD
#define PRT_SAH_BUILD 1
#endif
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

// --- 4c. top-down binned SAH above kSahLeaves triangles ------------------------
//
// The high-quality build makes a full SAH tree instead of the Morton
// hierarchy.  From the root (the triangles in Morton order), every task (a
// node and its contiguous range of triangles) with more than kSahLeaves
// triangles is split by the least SAH cost over
// kTopBins centroid bins per axis (bin boxes and counts gathered per chunk of
// the range in shared memory, then merged with atomics), its triangles are
// partitioned into the two halves of the range, and the halves become the
// next level's tasks, k_sah_rebuild's subtrees (2..kSahLeaves triangles) or
// leaves.  One host read-back per level (the next tasks' count and ranges)
// sizes the next level's launches.
constexpr int kTopBins = 32;
constexpr int kTopChunk = 4096;        // triangles per block of the binning and partition passes
constexpr int kBinWords = 13;          // count, box lo/hi, centroid lo/hi (order-preserving float bits)

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
    float cmin[2][3], cmax[2][3];   // centroid bounds of the two halves
};

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
        // count 0; lo fields (1-3, 7-9) start at the largest value, hi fields at 0
        bins[i] = w == 0 ? 0u : (((w >= 1 && w <= 3) || (w >= 7 && w <= 9)) ? 0xffffffffu : 0u);
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
        sb[i] = w == 0 ? 0u : (((w >= 1 && w <= 3) || (w >= 7 && w <= 9)) ? 0xffffffffu : 0u);
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
        uint32_t cq[3] = {0, 0, 0};
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
                cq[k] = ford(c[k]);
            }
        }
#pragma unroll
        for (int ax = 0; ax < 3; ++ax)
        {
            const int bin = valid ? top_bin(c[ax], tk.cmin[ax], sc[ax]) : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, bin);
            uint32_t r[13];
            r[0] = __popc(peers);
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                r[1 + k] = __reduce_min_sync(peers, lo[k]);
                r[4 + k] = __reduce_max_sync(peers, hi[k]);
                r[7 + k] = __reduce_min_sync(peers, cq[k]);
                r[10 + k] = __reduce_max_sync(peers, cq[k]);
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
                    atomicMin(w + 7 + k, r[7 + k]);
                    atomicMax(w + 10 + k, r[10 + k]);
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
        else if ((w >= 1 && w <= 3) || (w >= 7 && w <= 9))
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
// axis, then the lower bin), and the centroid bounds of the two halves.
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
    if (best == ~0ull)
    {
        sp.axis = -1;
        sp.bin = 0;
        sp.nl = (tk.hi - tk.lo + 1) / 2;
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                sp.cmin[h][k] = tk.cmin[k];
                sp.cmax[h][k] = tk.cmax[k];
            }
    }
    else
    {
        const int code = (int)(best & 0xffffffffu);
        sp.axis = code / kTopBins;
        sp.bin = code % kTopBins;
        const uint32_t* w = g + (sp.axis * kTopBins + lane) * kBinWords;
        const int cnt = (int)w[0];
        const bool left = lane <= sp.bin;
        sp.nl = __reduce_add_sync(0xffffffffu, left ? cnt : 0);
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            const uint32_t cl = cnt ? w[7 + k] : 0xffffffffu, chh = cnt ? w[10 + k] : 0u;
            sp.cmin[0][k] = funord(__reduce_min_sync(0xffffffffu, left ? cl : 0xffffffffu));
            sp.cmax[0][k] = funord(__reduce_max_sync(0xffffffffu, left ? chh : 0u));
            sp.cmin[1][k] = funord(__reduce_min_sync(0xffffffffu, left ? 0xffffffffu : cl));
            sp.cmax[1][k] = funord(__reduce_max_sync(0xffffffffu, left ? 0u : chh));
        }
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
            c.cmin[k] = sp.cmin[side][k];
            c.cmax[k] = sp.cmax[side][k];
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

// Triangles of each chunk that go left.
__global__ void __launch_bounds__(256) k_top_count(const int4* __restrict__ chunks, const TopTask* __restrict__ tasks,
                                                   const TopSplit* __restrict__ splits,
                                                   const uint32_t* __restrict__ perm,
                                                   const float* __restrict__ triBox, uint32_t* leftCount)
{
    __shared__ int warpCount[8];
    const int4 ch = chunks[blockIdx.x];
    const TopTask tk = tasks[ch.x];
    const TopSplit sp = splits[ch.x];
    const float sc = sp.axis >= 0 ? top_scale(tk.cmin[sp.axis], tk.cmax[sp.axis]) : 0.f;
    int mine = 0;
    for (int i = ch.y + threadIdx.x; i <= ch.z; i += blockDim.x) mine += top_side(tk, sp, sc, i, perm[i], triBox) == 0;
    mine = __reduce_add_sync(0xffffffffu, mine);
    if ((threadIdx.x & 31) == 0) warpCount[threadIdx.x >> 5] = mine;
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

struct TopBuffers
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

// Top-down binned SAH from the root down to subtrees of kSahLeaves triangles,
// then k_sah_rebuild for those.  perm: the triangles (reordered in place).
cudaError_t sah_top_down(int n, const float* triBox, const float* cbounds, uint32_t* perm, int2* child, int2* range,
                         int* parent, const TopBuffers& B, int numSMs, cudaStream_t stream)
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
        e = cudaMemsetAsync(B.counters, 0, sizeof(int), stream);
        if (e != cudaSuccess) break;
        k_top_children<<<div_up(numTasks, 128), 128, 0, stream>>>(B.task[cur], numTasks, B.splits, n,
                                                                   B.task[cur ^ 1], B.counters, B.small,
                                                                   B.counters + 1, B.counters + 2, child, range,
                                                                   parent);
        k_top_count<<<nch, 256, 0, stream>>>(B.chunks, B.task[cur], B.splits, perm, triBox, B.leftCount);
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

// --- 5. bottom-up refit and SAH-optimal grouping into 8-wide nodes ----------
//
// One thread per triangle walks up the tree; the second thread to arrive at
// a node (atomic counter) computes it from its two finished children, so every
// node is computed once, after both children.
//
// The node box is the union of the children's boxes.  With kGroup the same
// pass runs the dynamic program of Ylitie, Karras and Laine (HPG 2017,
// sec. 4.1) over the binary tree: C(u, i), i = 1..8, is the least SAH cost of
// representing subtree u by at most i roots (children of the enclosing 8-wide
// node).  A leaf root costs area x cTri x triangles, an 8-wide node area x
// cNode plus the best split of its 8 slots between the binary children;
// C(u, i) = min(C(u, i - 1), best split of i slots).  Costs are relative to
// cNode = 1 and kept for internal nodes only (a single triangle costs its
// area x cTri for every i).  Byte i - 1 of dec[u] records the choice: for
// i = 1 whether u is best a leaf (1) or an 8-wide node (0); for i >= 2 the
// slots j given to the left child (low 7 bits), with 0x80 set when at most
// i - 1 roots are no worse.
#ifndef PRT_WIDE_DP
#define PRT_WIDE_DP 1
#endif
#ifndef PRT_SAH_CTRI
#define PRT_SAH_CTRI 0.7f
#endif

__device__ __forceinline__ float box_half_area(const float* b)
{
    float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    return dx * dy + dy * dz + dz * dx;
}

struct RefitArgs
{
    int n;
    const uint32_t* vals;   // sorted triangle ids
    const float* triBox;    // 6 floats per triangle, by triangle id
    const int2* child;
    const int2* range;
    const int* parent;
    float* box;             // 6 floats per node: internal [0, n-1), leaves [n-1, 2n-1)
    int* flag;              // arrivals per internal node, zeroed
    float4* cost;           // kGroup: 2 float4 (C(u, 1..8)) per internal node
    uint2* dec;             // kGroup: 8 decision bytes per internal node
    int leafMax;
};

// C(child, 1..8) of a binary child: loaded for an internal node, its area x
// cTri for a single triangle.
__device__ __forceinline__ void child_costs(const RefitArgs& a, int ref, const float* b, float* c)
{
    if (ref < 0)
    {
        const float leafCost = box_half_area(b) * PRT_SAH_CTRI;
#pragma unroll
        for (int i = 0; i < 8; ++i) c[i] = leafCost;
        return;
    }
    const float4 lo = __ldcg(a.cost + 2 * (size_t)ref), hi = __ldcg(a.cost + 2 * (size_t)ref + 1);
    c[0] = lo.x; c[1] = lo.y; c[2] = lo.z; c[3] = lo.w;
    c[4] = hi.x; c[5] = hi.y; c[6] = hi.z; c[7] = hi.w;
}

// Node `node` (children ch, triangle range rg) from its two finished
// children: box, and with kGroup its grouping costs and decisions.
template <bool kGroup>
__device__ __forceinline__ void refit_node(const RefitArgs& a, int node, int2 ch, int2 rg)
{
    const int n = a.n;
    const int ia = ch.x >= 0 ? ch.x : (n - 1) + ~ch.x;
    const int ib = ch.y >= 0 ? ch.y : (n - 1) + ~ch.y;
    float ba[6], bb[6], r[6];
#pragma unroll
    for (int c = 0; c < 6; ++c)
    {
        ba[c] = __ldcg(a.box + 6 * (size_t)ia + c);
        bb[c] = __ldcg(a.box + 6 * (size_t)ib + c);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        r[c] = fminf(ba[c], bb[c]);
        r[3 + c] = fmaxf(ba[3 + c], bb[3 + c]);
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) __stcg(a.box + 6 * (size_t)node + c, r[c]);
    if (kGroup)
    {
        float ca[8], cb[8];
        child_costs(a, ch.x, ba, ca);
        child_costs(a, ch.y, bb, cb);
        const float area = box_half_area(r);
        const int cnt = rg.y - rg.x + 1;
        float dist[8];
        uint8_t split[8];
        dist[0] = FLT_MAX;
        split[0] = 0;
#pragma unroll
        for (int i = 2; i <= 8; ++i)
        {
            float best = FLT_MAX;
            int bj = 1;
#pragma unroll
            for (int j = 1; j < i; ++j)
            {
                const float v = ca[j - 1] + cb[i - j - 1];
                if (v < best)
                {
                    best = v;
                    bj = j;
                }
            }
            dist[i - 1] = best;
            split[i - 1] = (uint8_t)bj;
        }
        const float leafOpt = cnt <= a.leafMax ? area * PRT_SAH_CTRI * (float)cnt : FLT_MAX;
        const float wideOpt = area + dist[7];
        float cs[8];
        float c = fminf(leafOpt, wideOpt);
        cs[0] = c;
        uint32_t d0 = leafOpt <= wideOpt ? 1u : 0u, d1 = 0;
#pragma unroll
        for (int i = 2; i <= 8; ++i)
        {
            uint32_t d = split[i - 1];
            if (c <= dist[i - 1]) d |= 0x80;
            else c = dist[i - 1];
            cs[i - 1] = c;
            if (i <= 4) d0 |= d << (8 * (i - 1));
            else d1 |= d << (8 * (i - 5));
        }
        __stcg(a.cost + 2 * (size_t)node, make_float4(cs[0], cs[1], cs[2], cs[3]));
        __stcg(a.cost + 2 * (size_t)node + 1, make_float4(cs[4], cs[5], cs[6], cs[7]));
        __stcg(a.dec + node, make_uint2(d0, d1));
    }
}

// Arrival at a node: the atomic increment releases this thread's writes (its
// child's box and costs) and, for the second arrival, acquires the sibling's.
__device__ __forceinline__ unsigned arrive(int* flag)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(flag) : "memory");
    return old;
}

// The bottom-up walk with lanes refilled: each warp owns a run of consecutive
// leaves; a lane whose walk ends (first arrival at a node, or the root) takes
// the warp's next leaf, so the warp's lanes stay busy while the walks that
// continue towards the root are short or long.
constexpr int kRefitBlock = 256;

template <bool kGroup>
__global__ void __launch_bounds__(kRefitBlock) k_refit(RefitArgs a, int leavesPerWarp)
{
    const int n = a.n;
    const int lane = threadIdx.x & 31;
    const long long warpId = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    long long next = warpId * leavesPerWarp;
    const long long end = min((long long)n, next + leavesPerWarp);
    int node = -1;   // the node this lane arrives at next; -1: none
    for (;;)
    {
        const unsigned idleMask = __ballot_sync(0xffffffffu, node < 0);
        if (node < 0)
        {
            const long long k = next + __popc(idleMask & ((1u << lane) - 1u));
            if (k < end)
            {
                // leaf box
                const uint32_t p = a.vals[k];
                float* lb = a.box + 6 * (size_t)((n - 1) + k);
#pragma unroll
                for (int c = 0; c < 6; ++c) lb[c] = a.triBox[6 * (size_t)p + c];
                node = a.parent[(n - 1) + k];
            }
        }
        next += __popc(idleMask);
        if (!__any_sync(0xffffffffu, node >= 0) && next >= end) break;
        if (node >= 0)
        {
            // the tree links are read-only here: fetch them before the arrival
            const int2 ch = a.child[node];
            const int2 rg = kGroup ? a.range[node] : make_int2(0, 0);
            const int up = a.parent[node];
            if (arrive(a.flag + node) == 0)
            {
                node = -1;   // the sibling finishes this node
            }
            else
            {
                refit_node<kGroup>(a, node, ch, rg);
                node = up;
            }
        }
    }
}

// --- 6. collapse into 8-wide nodes ------------------------------------------

struct CollapseArgs
{
    int n;
    const int2* child;
    const int2* range;
    const float* box;
    const uint32_t* vals;
    const float* pos;
    const int* idx;
    Bvh8Node* nodes;
    TriRec* tris;
    unsigned long long* alloc;   // 8-wide nodes allocated (high 32 bits), leaf triangles (low 32 bits)
    int nodeCapacity;
    int* error;
    int leafMax;          // subtrees of at most this many triangles (1..3) become leaves
    const uint2* dec;     // grouping decisions of k_refit<true>, or nullptr for the greedy grouping
    int* binRef;          // per 8-wide node: the binary reference it is built from
    int* marks;           // level l is nodes [marks[l], marks[l + 1]); kCollapseLevels + 2 entries
};

// Levels launched; a tree that needs more would overflow the traversal stack
// (two entries per level) and is rejected.
constexpr int kCollapseLevels = kStackMax / 2;
constexpr int kCollapseBlock = 128;
constexpr int kGroupsPerBlock = kCollapseBlock / 8;

__device__ __forceinline__ int ref_count(const CollapseArgs& a, int ref)
{
    if (ref < 0) return 1;
    int2 r = a.range[ref];
    return r.y - r.x + 1;
}

__device__ __forceinline__ const float* ref_box(const CollapseArgs& a, int ref)
{
    return a.box + 6 * (size_t)(ref >= 0 ? ref : (a.n - 1) + ~ref);
}

__device__ __forceinline__ float half_area(const float* b)
{
    float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ uint32_t dec_byte(uint2 d, int b)
{
    return ((b < 4 ? d.x : d.y) >> (8 * (b & 3))) & 0xffu;
}

// Per-group shared staging: the node being written (80 bytes), the children's
// slot records and the work list of the grouping walk.
struct __align__(16) CollapseGroup
{
    uint8_t node[80];
    uint32_t slotRec[8];   // per slot: bit 31 occupied, bit 30 internal, low bits triangle count
    int2 front[8];
};

// One 8-lane group builds 8-wide node nodeIdx from binary reference
// binRef[nodeIdx]: lane c holds child c of the node.  A binary reference of
// ~0 with n == 1 is the single-triangle scene.
__device__ void collapse_node(const CollapseArgs& a, int nodeIdx, int sub, unsigned gmask, CollapseGroup& g)
{
    const int bref = a.binRef[nodeIdx];

    // 1. children: the roots chosen by the grouping decisions (or greedily
    //    opened), left to right in tree order, child c in lane c
    int r = 0, nc;
    if (bref < 0)
    {
        r = bref;
        nc = 1;
    }
    else if (a.dec)
    {
        // expand the split list breadth-first: an entry (u, i) gives i slots
        // to subtree u; it is final for a triangle or i = 1, else the largest
        // i' <= i without the "no worse with fewer" bit splits it between the
        // binary children (i' = 1: u itself is the root)
        const int2 c = a.child[bref];
        const int j = (int)(dec_byte(__ldg(a.dec + bref), 7) & 0x7f);
        r = sub == 0 ? c.x : c.y;
        int ri = sub == 0 ? j : 8 - j;
        nc = 2;
        for (int round = 0; round < 8; ++round)
        {
            const bool valid = sub < nc;
            const bool expand = valid && r >= 0 && ri > 1;
            uint2 d = make_uint2(0, 0);
            int2 cc = make_int2(0, 0);
            if (expand)
            {
                d = __ldg(a.dec + r);
                cc = a.child[r];
            }
            int ii = ri;
            if (expand)
                while (ii > 1 && (dec_byte(d, ii - 1) & 0x80)) --ii;
            const bool split = expand && ii > 1;
            const unsigned splitMask = (__ballot_sync(gmask, split) & gmask) >> (__ffs(gmask) - 1);
            if (!splitMask) break;
            if (nc + __popc(splitMask) > 8)
            {
                // slot counts that do not add up to 8: inconsistent decisions
                if (sub == 0) atomicExch(a.error, 1);
                return;
            }
            const int at = min(sub, nc) + __popc(splitMask & ((1u << sub) - 1));
            if (split)
            {
                const int dj = (int)dec_byte(d, ii - 1);
                g.front[at] = make_int2(cc.x, dj);
                g.front[at + 1] = make_int2(cc.y, ii - dj);
            }
            else if (valid)
            {
                g.front[at] = make_int2(r, expand ? 1 : ri);
            }
            nc += __popc(splitMask);
            __syncwarp(gmask);
            if (sub < nc)
            {
                r = g.front[sub].x;
                ri = g.front[sub].y;
            }
            __syncwarp(gmask);
        }
    }
    else
    {
        // greedy: open the child of largest surface area while fewer than 8
        // (ties to the lower child); the opened child keeps its left half in
        // its lane and the right half goes to lane nc
        const int2 c = a.child[bref];
        r = sub == 0 ? c.x : c.y;
        nc = 2;
        bool stale = true;
        uint32_t key = 0;
        while (nc < 8)
        {
            if (stale)
            {
                key = 0;
                if (sub < nc && r >= 0 && ref_count(a, r) > a.leafMax)
                {
                    const float ar = half_area(ref_box(a, r));
                    if (ar >= 0.f) key = ((__float_as_uint(ar) | 0x80000000u) & ~7u) | (uint32_t)(7 - sub);
                }
                stale = false;
            }
            const uint32_t top = __reduce_max_sync(gmask, key);
            if (!top) break;
            const int best = 7 - (int)(top & 7u);
            int2 c2 = make_int2(0, 0);
            if (sub == best) c2 = a.child[r];
            const int right = __shfl_sync(gmask, c2.y, best, 8);
            if (sub == best)
            {
                r = c2.x;
                stale = true;
            }
            if (sub == nc)
            {
                r = right;
                stale = true;
            }
            ++nc;
        }
    }

    // 2. this lane's child: triangle count, leaf or 8-wide node, box
    const bool valid = sub < nc;
    int cnt = 0, first = 0;
    bool leaf = false;
    float b[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    if (valid)
    {
        if (r < 0)
        {
            cnt = 1;
            first = ~r;
            leaf = true;
        }
        else
        {
            const int2 rg = a.range[r];
            cnt = rg.y - rg.x + 1;
            first = rg.x;
            leaf = cnt <= a.leafMax && (a.dec ? dec_byte(__ldg(a.dec + r), 0) == 1 : true);
        }
        const float* rb = ref_box(a, r);
#pragma unroll
        for (int k = 0; k < 6; ++k) b[k] = rb[k];
    }

    // 3. node box: union over the group
    float nb[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) nb[k] = b[k];
#pragma unroll
    for (int off = 1; off < 8; off <<= 1)
    {
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            nb[k] = fminf(nb[k], __shfl_xor_sync(gmask, nb[k], off, 8));
            nb[3 + k] = fmaxf(nb[3 + k], __shfl_xor_sync(gmask, nb[3 + k], off, 8));
        }
    }

    // 4. slot assignment: greedy on cost(slot s, child c) = projection of the
    //    child centroid on the direction of octant s (smaller = nearer); each
    //    round places the least cost over free slots and unplaced children,
    //    ties to the lower slot, then the lower child
    float cost[8];
    {
        const float cx = 0.5f * (b[0] + b[3]), cy = 0.5f * (b[1] + b[4]), cz = 0.5f * (b[2] + b[5]);
#pragma unroll
        for (int s = 0; s < 8; ++s)
        {
            const float dx = (s & 1) ? -1.f : 1.f, dy = (s & 2) ? -1.f : 1.f, dz = (s & 4) ? -1.f : 1.f;
            cost[s] = cx * dx + cy * dy + cz * dz;
        }
    }
    int slot = -1;
    unsigned freeSlots = 0xffu;
    for (int it = 0; it < nc; ++it)
    {
        // key: cost (order-preserving bits, 6 low bits dropped), slot, lane;
        // least wins
        uint32_t key = 0xffffffffu;
        if (valid && slot < 0)
        {
            float bc = FLT_MAX;
            int bs = 8;
#pragma unroll
            for (int s = 0; s < 8; ++s)
                if (((freeSlots >> s) & 1u) && cost[s] < bc)
                {
                    bc = cost[s];
                    bs = s;
                }
            if (bs < 8)
            {
                const uint32_t u = __float_as_uint(bc);
                const uint32_t ord = u ^ ((uint32_t)((int)u >> 31) | 0x80000000u);
                key = (ord & ~63u) | ((uint32_t)bs << 3) | (uint32_t)sub;
            }
        }
        const uint32_t least = __reduce_min_sync(gmask, key);
        int bs, bl;
        if (least != 0xffffffffu)
        {
            bs = (int)((least >> 3) & 7u);
            bl = (int)(least & 7u);
        }
        else
        {
            // no finite cost left (degenerate boxes): lowest free slot to the
            // lowest unplaced child
            bs = __ffs(freeSlots) - 1;
            const unsigned unplaced = __ballot_sync(gmask, valid && slot < 0) & gmask;
            bl = __ffs(unplaced >> (__ffs(gmask) - 1)) - 1;
        }
        if (sub == bl) slot = bs;
        freeSlots &= ~(1u << bs);
    }

    // 5. per-slot records: internal children numbered and leaf triangles
    //    packed in slot order
    if (valid) g.slotRec[slot] = 0x80000000u | (leaf ? 0u : 0x40000000u) | (uint32_t)cnt;
    if ((freeSlots >> sub) & 1u) g.slotRec[sub] = 0;   // the empty slots
    __syncwarp(gmask);
    int nInternal = 0, nTris = 0, internalRank = 0, triOff = 0;
    uint32_t imask = 0;
#pragma unroll
    for (int s = 0; s < 8; ++s)
    {
        const uint32_t rec = g.slotRec[s];
        if (!(rec & 0x80000000u)) continue;
        if (rec & 0x40000000u)
        {
            if (s < slot) ++internalRank;
            ++nInternal;
            imask |= 1u << s;
        }
        else
        {
            const int c = (int)(rec & 0xffffu);
            if (s < slot) triOff += c;
            nTris += c;
        }
    }
    int childBase = 0, triBase = 0, bad = 0;
    if (sub == 0)
    {
        // one atomic for the child nodes and leaf triangles of all the groups
        // of this warp that are here together
        const unsigned m = __activemask();
        const int me = threadIdx.x & 31;
        const unsigned long long req = ((unsigned long long)nInternal << 32) | (unsigned)nTris;
        unsigned long long before = 0, total = 0;
        for (unsigned rest = m; rest; rest &= rest - 1)
        {
            const int l = __ffs(rest) - 1;
            const unsigned long long v = __shfl_sync(m, req, l);
            if (l < me) before += v;
            total += v;
        }
        const int first = __ffs(m) - 1;
        unsigned long long base = 0;
        if (me == first) base = atomicAdd(a.alloc, total);
        base = __shfl_sync(m, base, first) + before;
        childBase = (int)(base >> 32);
        triBase = (int)(base & 0xffffffffu);
        bad = childBase + nInternal > a.nodeCapacity || triBase + nTris > a.n;
        if (bad) atomicExch(a.error, 1);
    }
    const int leader = __ffs(gmask) - 1;
    if (__shfl_sync(gmask, bad, leader)) return;   // group-uniform
    childBase = __shfl_sync(gmask, childBase, leader);
    triBase = __shfl_sync(gmask, triBase, leader);

    // 6. header: per-axis power-of-two scale s with the node box spanning at
    //    most 253 steps, and origin one step below the box, so every quantized
    //    plane lies at least 2^-8 of a step outside the child box it bounds (the
    //    traversal's plane decode may move a plane inwards by up to 2^-9 step)
    uint32_t ebits[3];
    float scale[3];
    float origin[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        float ext = nb[3 + k] - nb[k];
        int e = -100;
        if (ext > 0.f)
        {
            e = (int)ceilf(log2f(ext / 253.0f));
            while (ldexpf(253.0f, e) < ext) ++e;
        }
        // a step of at least 16 ulps of the coordinates, so that thin or flat
        // boxes keep distinct planes below and above them
        float mag = fmaxf(fabsf(nb[k]), fabsf(nb[3 + k]));
        if (mag > 0.f)
        {
            int me;
            frexpf(mag, &me);
            e = max(e, me - 20);
        }
        e = max(e, -126);
        e = min(e, 100);   // the traversal adds 15 to the biased exponent
        ebits[k] = (uint32_t)(e + 127);
        scale[k] = ldexpf(1.0f, e);
        // round the origin down so that it stays at least one step below the box
        double o = (double)nb[k] - (double)scale[k];
        float of = (float)o;
        if ((double)of > o) of = nextafterf(of, -FLT_MAX);
        origin[k] = of;
    }

    // 7. this lane's slot: quantized planes and meta byte; the lane numbered
    //    by an empty slot fills in an empty box
    if ((freeSlots >> sub) & 1u)
    {
        g.node[24 + sub] = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            g.node[32 + 8 * k + sub] = 255;
            g.node[56 + 8 * k + sub] = 0;
        }
    }
    if (valid)
    {
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            // scale is a power of two: multiplying by its inverse is exact
            const double inv = __longlong_as_double((long long)(127 - (int)ebits[k] + 1023) << 52);
            double lo = floor(((double)b[k] - (double)origin[k]) * inv - 1.0 / 256.0);
            double hi = ceil(((double)b[3 + k] - (double)origin[k]) * inv + 1.0 / 256.0);
            g.node[32 + 8 * k + slot] = (uint8_t)fmax(0.0, fmin(255.0, lo));
            g.node[56 + 8 * k + slot] = (uint8_t)fmax(0.0, fmin(255.0, hi));
        }
        if (!leaf)
        {
            g.node[24 + slot] = (uint8_t)(0x20 | (24 + slot));
            a.binRef[childBase + internalRank] = r;
        }
        else
        {
            const uint32_t unary = (1u << cnt) - 1u;
            g.node[24 + slot] = (uint8_t)((unary << 5) | (uint32_t)triOff);
            // the triangles of the leaf (a contiguous sorted range)
            for (int k = 0; k < cnt; ++k)
            {
                const uint32_t prim = a.vals[first + k];
                const int i0 = a.idx[3 * prim], i1 = a.idx[3 * prim + 1], i2 = a.idx[3 * prim + 2];
                TriRec tr;
                tr.v0 = make_float4(a.pos[3 * i0], a.pos[3 * i0 + 1], a.pos[3 * i0 + 2], __int_as_float((int)prim));
                tr.v1 = make_float4(a.pos[3 * i1], a.pos[3 * i1 + 1], a.pos[3 * i1 + 2], 0.f);
                tr.v2 = make_float4(a.pos[3 * i2], a.pos[3 * i2 + 1], a.pos[3 * i2 + 2], 0.f);
                a.tris[triBase + triOff + k] = tr;
            }
        }
    }
    if (sub == 0)
    {
        uint32_t* w = reinterpret_cast<uint32_t*>(g.node);
        w[0] = __float_as_uint(origin[0]);
        w[1] = __float_as_uint(origin[1]);
        w[2] = __float_as_uint(origin[2]);
        w[3] = ebits[0] | (ebits[1] << 8) | (ebits[2] << 16) | (imask << 24);
        w[4] = (uint32_t)childBase;
        w[5] = (uint32_t)triBase;
    }
    __syncwarp(gmask);
    if (sub < 5) a.nodes[nodeIdx].q[sub] = reinterpret_cast<const uint4*>(g.node)[sub];
    __syncwarp(gmask);
}

// One tree level: nodes [marks[level], marks[level + 1]), one per 8-lane
// group, grid-strided.
__global__ void __launch_bounds__(kCollapseBlock) k_collapse(CollapseArgs a, int level)
{
    __shared__ CollapseGroup groups[kGroupsPerBlock];
    if (*(volatile int*)a.error) return;
    const int begin = *(volatile int*)(a.marks + level);
    const int end = *(volatile int*)(a.marks + level + 1);
    const int lane = threadIdx.x & 31;
    const int sub = lane & 7;
    const unsigned gmask = 0xffu << (lane & 24);
    CollapseGroup& g = groups[threadIdx.x >> 3];
    const int stride = gridDim.x * kGroupsPerBlock;
    for (int w = begin + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 3); w < end; w += stride)
        collapse_node(a, w, sub, gmask, g);
}

// After level l: the nodes allocated so far end level l + 1.
__global__ void k_collapse_mark(CollapseArgs a, int level)
{
    a.marks[level + 2] = (int)(*(volatile unsigned long long*)a.alloc >> 32);
}


// Runs the collapse from the root, one launch per level, without waiting for
// the host between levels: launches past the last level find no nodes and
// return.  The counters are read back after the first kCollapseBatch levels
// and, for a deeper tree, after the rest.  On success sets the node and
// triangle counts and the number of 8-wide levels (kCollapseLevels + 1 for a
// tree deeper than the launches).
constexpr int kCollapseBatch = 16;

int collapse_levels(const CollapseArgs& a, int n, int numSMs, cudaStream_t stream, int& nodeCount, int& triCount,
                    int& levels, std::string& err)
{
    const int root = n > 1 ? 0 : ~0;
    const unsigned long long alloc0 = 1ull << 32;   // the root
    const int marks0[2] = {0, 1};
    int hostErr = 0;
    unsigned long long hostAlloc = 0;
    int marks[kCollapseLevels + 2];
    cudaError_t e = cudaMemcpyAsync(a.binRef, &root, sizeof(int), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(a.alloc, &alloc0, sizeof(alloc0), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.error, 0, sizeof(int), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.marks, 0, sizeof(int) * (kCollapseLevels + 2), stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(a.marks, marks0, sizeof(marks0), cudaMemcpyHostToDevice, stream);
    int perSM = 1;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_collapse, kCollapseBlock, 0);
    const long long maxBlocks = (long long)std::max(1, numSMs) * std::max(1, perSM);
    long long bound = 1;   // level l holds at most 8^l nodes
    int l = 0;
    while (e == cudaSuccess && l < kCollapseLevels)
    {
        const int stop = std::min(kCollapseLevels, l + kCollapseBatch);
        for (; e == cudaSuccess && l < stop; ++l)
        {
            const int blocks = (int)std::min(maxBlocks, (bound + kGroupsPerBlock - 1) / kGroupsPerBlock);
            k_collapse<<<blocks, kCollapseBlock, 0, stream>>>(a, l);
            k_collapse_mark<<<1, 1, 0, stream>>>(a, l);
            e = cudaGetLastError();
            bound = std::min<long long>(bound * 8, 1ll << 32);
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&hostErr, a.error, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&hostAlloc, a.alloc, sizeof(hostAlloc), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(marks, a.marks, sizeof(marks), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e == cudaSuccess && (hostErr || marks[l + 1] == marks[l])) break;   // error, or no level l
    }
    if (e != cudaSuccess)
    {
        err = std::string("BVH8 collapse: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? PRT_ENOMEM : PRT_ECUDA;
    }
    if (hostErr)
    {
        err = "BVH8 collapse exceeded its node or triangle capacity";
        return PRT_EINTERNAL;
    }
    levels = 0;
    while (levels <= kCollapseLevels && marks[levels + 1] > marks[levels]) ++levels;
    nodeCount = (int)(hostAlloc >> 32);
    triCount = (int)(hostAlloc & 0xffffffffu);
    return PRT_OK;
}

} // namespace

#define BUILD_CHECK(x)                                                                                          \
    do                                                                                                         \
    {                                                                                                          \
        cudaError_t e_ = (x);                                                                                  \
        if (e_ != cudaSuccess)                                                                                 \
        {                                                                                                      \
            err = std::string(#x) + ": " + cudaGetErrorString(e_);                                              \
            status = e_ == cudaErrorMemoryAllocation ? PRT_ENOMEM : PRT_ECUDA;                                 \
            goto done;                                                                                         \
        }                                                                                                      \
    } while (0)

int build_bvh8(const float* dPos, int nv, const int* dIdx, int nt, Bvh8Device& out, cudaStream_t stream,
               std::string& err, BuildInfo* info, int leafMax, bool sahGrouping, DeviceScratch* scratch)
{
    (void)nv;
    int status = PRT_OK;
    out.release();
    if (nt <= 0) return PRT_OK;   // empty scene: no root

    const int n = nt;
    const int nInternal = n > 1 ? n - 1 : 0;
    const size_t histCount = radix_sort_hist_entries(n);
    const int boundBlocks = std::min(1024, div_up(n, 256));
    const int nodeCapacity = std::max(1, nInternal);
    const bool group = PRT_WIDE_DP && sahGrouping && nInternal > 0;
    const bool rebuild = PRT_SAH_BUILD && sahGrouping && nInternal > 0;
    int device = 0, numSMs = 148;
    if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device);

    char* block = nullptr;
    float *triBox, *partial, *cbounds, *box;
    uint32_t *keysA, *keysB, *valsA, *valsB, *hist;
    int2 *child, *range;
    int *parent, *flag, *collapseErr, *marks, *binRef;
    TopBuffers top{};
    unsigned long long* collapseAlloc;
    float4* dpCost;
    uint2* dpDec;
    auto carve = [&](char* base) {
        Carve c{base};
        triBox = c.take<float>(6 * (size_t)n);
        partial = c.take<float>(6 * (size_t)boundBlocks);
        cbounds = c.take<float>(6);
        keysA = c.take<uint32_t>(n);
        keysB = c.take<uint32_t>(n);
        valsA = c.take<uint32_t>(n);
        valsB = c.take<uint32_t>(n);
        hist = c.take<uint32_t>(histCount);
        child = c.take<int2>(nodeCapacity);
        range = c.take<int2>(nodeCapacity);
        parent = c.take<int>(2 * (size_t)n);
        flag = c.take<int>(nodeCapacity);
        box = c.take<float>(6 * (size_t)(2 * n));
        binRef = c.take<int>(nodeCapacity);
        if (rebuild)
        {
            top.maxTasks = n / (kSahLeaves + 1) + 2;
            top.maxChunks = n / kTopChunk + top.maxTasks + 2;
            top.task[0] = c.take<TopTask>(top.maxTasks);
            top.task[1] = c.take<TopTask>(top.maxTasks);
            top.splits = c.take<TopSplit>(top.maxTasks);
            top.bins = c.take<uint32_t>((size_t)top.maxTasks * 3 * kTopBins * kBinWords);
            top.leftCount = c.take<uint32_t>(top.maxChunks);
            top.scanSums = c.take<uint32_t>(scan_sums_entries(top.maxChunks));
            top.small = c.take<int>((size_t)n / 2 + 1);
            top.counters = c.take<int>(3);
            top.chunks = c.take<int4>(top.maxChunks);
        }
        collapseAlloc = c.take<unsigned long long>(1);
        collapseErr = c.take<int>(1);
        marks = c.take<int>(kCollapseLevels + 2);
        dpCost = group ? c.take<float4>(2 * (size_t)nodeCapacity) : nullptr;
        dpDec = group ? c.take<uint2>(nodeCapacity) : nullptr;
        return c.off;
    };
    const size_t scratchBytes = carve(nullptr);
    int levels = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    BUILD_CHECK(cudaEventCreate(&ev0));
    BUILD_CHECK(cudaEventCreate(&ev1));
    BUILD_CHECK(cudaEventRecord(ev0, stream));

    if (scratch)
    {
        BUILD_CHECK(scratch->reserve(scratchBytes));
        block = static_cast<char*>(scratch->p);
    }
    else
    {
        BUILD_CHECK(dev_malloc(&block, scratchBytes));
    }
    carve(block);
    {
        const size_t nodeBytes = (sizeof(Bvh8Node) * (size_t)nodeCapacity + 255) & ~(size_t)255;
        out.bytes = nodeBytes + sizeof(TriRec) * (size_t)n;
        char* blk = nullptr;
        BUILD_CHECK(dev_malloc(&blk, out.bytes));
        out.block = blk;
        out.nodes = reinterpret_cast<Bvh8Node*>(blk);
        out.tris = reinterpret_cast<TriRec*>(blk + nodeBytes);
    }

    k_tri_boxes<<<boundBlocks, 256, 0, stream>>>(dPos, dIdx, n, triBox, partial);
    k_reduce_bounds<<<1, 256, 0, stream>>>(partial, boundBlocks, cbounds);
    k_morton<<<div_up(n, 256), 256, 0, stream>>>(triBox, n, cbounds, keysA, valsA);
    radix_sort_pairs(keysA, valsA, keysB, valsB, hist, n, 30, stream);
    if (nInternal > 0)
    {
        if (rebuild)
        {
            top.tmp = keysB;   // free after the sort
            BUILD_CHECK(sah_top_down(n, triBox, cbounds, valsA, child, range, parent, top, numSMs, stream));
        }
        else
        {
            k_karras<<<div_up(nInternal, 256), 256, 0, stream>>>(keysA, n, child, range, parent);
        }
        BUILD_CHECK(cudaMemsetAsync(flag, 0, sizeof(int) * (size_t)nInternal, stream));
    }
    else
    {
        int minus1 = -1;
        BUILD_CHECK(cudaMemcpyAsync(parent, &minus1, sizeof(int), cudaMemcpyHostToDevice, stream));
    }
    {
        RefitArgs ra;
        ra.n = n;
        ra.vals = valsA;
        ra.triBox = triBox;
        ra.child = child;
        ra.range = range;
        ra.parent = parent;
        ra.box = box;
        ra.flag = flag;
        ra.cost = dpCost;
        ra.dec = dpDec;
        ra.leafMax = std::max(1, std::min(3, leafMax));
        int perSM = 1;
        if (group) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_refit<true>, kRefitBlock, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_refit<false>, kRefitBlock, 0);
        const int blocks = std::max(1, std::min(std::max(1, perSM) * numSMs, div_up(n, kRefitBlock)));
        const int leavesPerWarp = div_up(n, (long long)blocks * (kRefitBlock / 32));
        if (group) k_refit<true><<<blocks, kRefitBlock, 0, stream>>>(ra, leavesPerWarp);
        else k_refit<false><<<blocks, kRefitBlock, 0, stream>>>(ra, leavesPerWarp);
    }
    BUILD_CHECK(cudaGetLastError());

    {
        CollapseArgs a;
        a.n = n;
        a.child = child;
        a.range = range;
        a.box = box;
        a.vals = valsA;
        a.pos = dPos;
        a.idx = dIdx;
        a.nodes = out.nodes;
        a.tris = out.tris;
        a.alloc = collapseAlloc;
        a.nodeCapacity = nodeCapacity;
        a.error = collapseErr;
        a.leafMax = std::max(1, std::min(3, leafMax));
        a.dec = dpDec;
        a.binRef = binRef;
        a.marks = marks;
        int nodeCount = 0, triCount = 0;
        status = collapse_levels(a, n, numSMs, stream, nodeCount, triCount, levels, err);
        if (status == PRT_OK && a.dec && 2 * levels > kStackMax)
        {
            // the SAH grouping came out deeper than the traversal stack allows
            // (possible for degenerate inputs): group greedily instead
            a.dec = nullptr;
            status = collapse_levels(a, n, numSMs, stream, nodeCount, triCount, levels, err);
        }
        if (status != PRT_OK) goto done;
        out.nodeCount = nodeCount;
        out.triCount = triCount;
        out.leafMax = a.leafMax;
        out.levels = levels;
        if (2 * levels > kStackMax)
        {
            err = "BVH8 is deeper than the traversal stack";
            status = PRT_EINTERNAL;
            goto done;
        }
        if (out.triCount != n)
        {
            err = "BVH8 collapse lost triangles";
            status = PRT_EINTERNAL;
            goto done;
        }
    }
    BUILD_CHECK(cudaEventRecord(ev1, stream));
    BUILD_CHECK(cudaEventSynchronize(ev1));
    if (info)
    {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0, ev1);
        info->buildMs = ms;
        info->nodeCount = out.nodeCount;
        info->levels = levels;
    }

done:
    if (!scratch) cudaFree(block);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (status != PRT_OK) out.release();
    return status;
}

} // namespace prt_b200
