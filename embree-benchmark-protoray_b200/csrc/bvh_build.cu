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
//      built top-down from that order (sah_build.cu: binned SAH above 256
//      triangles, an exact sweep SAH per block below); otherwise the binary radix tree
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

namespace {

constexpr const char* kTooDeep = "BVH8 is deeper than the traversal stack";

// sahTree: the top-down SAH binary tree (else the Karras hierarchy over the
// Morton order); sahGrouping: the SAH-optimal grouping into 8-wide nodes
// (else greedy).
int build_bvh8_tree(const float* dPos, int nv, const int* dIdx, int nt, Bvh8Device& out, cudaStream_t stream,
                    std::string& err, BuildInfo* info, int leafMax, bool sahTree, bool sahGrouping,
                    DeviceScratch* scratch)
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
    const bool rebuild = sahTree && nInternal > 0;   // the SAH tree (sah_build.cu)
    int device = 0, numSMs = 148;
    if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device);

    char* block = nullptr;
    float *triBox, *partial, *cbounds, *box;
    uint32_t *keysA, *keysB, *valsA, *valsB, *hist;
    int2 *child, *range;
    int *parent, *flag, *collapseErr, *marks, *binRef;
    SahTreeBuffers top{};
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
        if (rebuild) sah_tree_carve(c, n, top);
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
            BUILD_CHECK(sah_build_tree(n, triBox, cbounds, valsA, child, range, parent, top, numSMs, stream));
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
            err = kTooDeep;
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

} // namespace

int build_bvh8(const float* dPos, int nv, const int* dIdx, int nt, Bvh8Device& out, cudaStream_t stream,
               std::string& err, BuildInfo* info, int leafMax, bool sahGrouping, DeviceScratch* scratch)
{
    int st = build_bvh8_tree(dPos, nv, dIdx, nt, out, stream, err, info, leafMax, sahGrouping, sahGrouping, scratch);
    if (st == PRT_EINTERNAL && sahGrouping && err == kTooDeep)
    {
        // The SAH tree has no depth limit: a chain-shaped input (triangle sizes
        // shrinking geometrically, each split peeling one off) can come out
        // deeper than the traversal stack even after greedy grouping.  The
        // Karras hierarchy over 30-bit Morton codes is at most about 30 + log2(n)
        // binary levels deep, so build that instead.
        err.clear();
        st = build_bvh8_tree(dPos, nv, dIdx, nt, out, stream, err, info, leafMax, false, true, scratch);
    }
    return st;
}

} // namespace prt_b200
