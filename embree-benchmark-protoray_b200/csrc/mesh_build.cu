// GPU mesh builder: triangle soup -> indexed mesh in Morton order.
//
// Replaces TriangleMeshBuilder (geometry/triangle_mesh_builder.cpp), which
// runs on one CPU thread: a chained hash map over whole vertices (:98-125)
// and a recursive median split of vertices and triangle centres (:143-201).
// Here every step is a data-parallel pass over the soup in HBM:
//   1. k_soup_scan     attribute flags (any normal / texcoord / matId != 0,
//                      :70-87) and position bounds, block partials + one reduce
//   2. k_soup_corners  one 32-byte record per corner {pos, normal, tex}; a zero
//                      normal becomes the triangle's cross product when the
//                      soup has normals (:92-96); triangle centroid Morton keys
//   3. k_dedup_insert  open-addressing hash set of corner records; equal
//                      records share one slot, which keeps the lowest corner
//                      index (atomicCAS to claim, atomicMin to lower)
//   4. k_dedup_resolve representative corner per corner, unique flags
//   5. exclusive scan of the flags -> compacted unique vertex list
//   6. 30-bit Morton keys of the unique vertices, stable radix sort: vertex
//      order = (Morton code, first occurrence in the soup)
//   7. k_vertex_emit   interleaved attributes in .mesh layout, old -> new ids
//   8. radix sort of the triangle keys, k_tri_emit: indices and material ids
// The result is deterministic.  It holds the same triangles (as vertex
// triples) and the same set of unique vertices as the reference builder's
// mesh; only the order differs (Morton instead of median split).
//
// Equality of vertices is bitwise, which matches the reference's float ==
// except for signed zeros (the reference hashes the bits and then compares
// with ==, so +0 and -0 merge only when their hashes share a bucket) and NaN
// (never equal in the reference; vertices with a NaN component are kept
// unique here as well).
#include <algorithm>
#include <chrono>
#include <cstring>

#include "prt_internal.h"

namespace prt_b200 {

namespace {

constexpr uint32_t kEmptySlot = 0xffffffffu;
constexpr int kSoupFloats = 25;   // prt_soup_triangle: 3 x 8 floats + matId
constexpr int kFlagNormals = 1, kFlagTexcoords = 2, kFlagMaterials = 4;

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

__device__ __forceinline__ uint32_t expand10(uint32_t v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t morton30(float x, float y, float z, const float* __restrict__ b)
{
    const float c[3] = {x, y, z};
    uint32_t code = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        const float ext = b[3 + k] - b[k];
        const float u = ext > 0.f ? (c[k] - b[k]) / ext : 0.f;
        const uint32_t q = (uint32_t)fminf(fmaxf(u * 1024.0f, 0.0f), 1023.0f);
        code |= expand10(q) << k;
    }
    return code;
}

// 1. flags and bounds ----------------------------------------------------------

__global__ void __launch_bounds__(256) k_soup_scan(const float* __restrict__ soup, int n, unsigned* __restrict__ flags,
                                                 float* __restrict__ partial)
{
    __shared__ float s[6][8];
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    unsigned f = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    {
        const float* r = soup + kSoupFloats * t;
#pragma unroll
        for (int v = 0; v < 3; ++v)
        {
            const float* q = r + 8 * v;
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                lo[k] = fminf(lo[k], q[k]);
                hi[k] = fmaxf(hi[k], q[k]);
            }
            // Vec3f != zero (math/vec3.h:285-288): any component compares unequal (NaN does)
            if (q[3] != 0.f || q[4] != 0.f || q[5] != 0.f) f |= kFlagNormals;
            if (q[6] != 0.f || q[7] != 0.f) f |= kFlagTexcoords;
        }
        if (__float_as_int(r[24]) != 0) f |= kFlagMaterials;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
        }
    }
    f = __reduce_or_sync(0xffffffffu, f);
    if (lane == 0)
    {
        for (int k = 0; k < 3; ++k)
        {
            s[k][warp] = lo[k];
            s[3 + k][warp] = hi[k];
        }
        if (f) atomicOr(flags, f);
    }
    __syncthreads();
    if (threadIdx.x < 6)
    {
        const int k = threadIdx.x;
        float v = s[k][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = k < 3 ? fminf(v, s[k][w]) : fmaxf(v, s[k][w]);
        partial[6 * blockIdx.x + k] = v;
    }
}

// One warp per bound component (6 warps): strided reads of the block partials, then a shuffle reduction.
__global__ void __launch_bounds__(192) k_bounds_final(const float* __restrict__ partial, int nblocks,
                                                      float* __restrict__ out)
{
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool isMin = k < 3;
    float v = isMin ? FLT_MAX : -FLT_MAX;
    for (int b = lane; b < nblocks; b += 32) v = isMin ? fminf(v, partial[6 * b + k]) : fmaxf(v, partial[6 * b + k]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        const float o = __shfl_xor_sync(0xffffffffu, v, off);
        v = isMin ? fminf(v, o) : fmaxf(v, o);
    }
    if (lane == 0) out[k] = v;
}

// 2. corner records and triangle keys --------------------------------------------

// cross(b - a, c - a) as the reference's compiled cross() evaluates it
// (math/vec3.h:401-406 with the first product of each component fused:
// fma(x1, y2, -(x2 * y1))).
__device__ __forceinline__ float cross_comp(float a1, float b2, float a2, float b1)
{
    return __fmaf_rn(a1, b2, -__fmul_rn(a2, b1));
}

__global__ void __launch_bounds__(256) k_soup_corners(const float* __restrict__ soup, int n,
                                                    const unsigned* __restrict__ flags, const float* __restrict__ bounds,
                                                    float4* __restrict__ corners, uint32_t* __restrict__ triKeys,
                                                    uint32_t* __restrict__ triVals)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float* r = soup + kSoupFloats * t;
    float v[24];
#pragma unroll
    for (int i = 0; i < 24; ++i) v[i] = r[i];
    if (*flags & kFlagNormals)
    {
        const float e1x = __fsub_rn(v[8], v[0]), e1y = __fsub_rn(v[9], v[1]), e1z = __fsub_rn(v[10], v[2]);
        const float e2x = __fsub_rn(v[16], v[0]), e2y = __fsub_rn(v[17], v[1]), e2z = __fsub_rn(v[18], v[2]);
        const float nx = cross_comp(e1y, e2z, e1z, e2y);
        const float ny = cross_comp(e1z, e2x, e1x, e2z);
        const float nz = cross_comp(e1x, e2y, e1y, e2x);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (v[8 * k + 3] == 0.f && v[8 * k + 4] == 0.f && v[8 * k + 5] == 0.f)
            {
                v[8 * k + 3] = nx;
                v[8 * k + 4] = ny;
                v[8 * k + 5] = nz;
            }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        corners[2 * (3 * t + k)] = make_float4(v[8 * k], v[8 * k + 1], v[8 * k + 2], v[8 * k + 3]);
        corners[2 * (3 * t + k) + 1] = make_float4(v[8 * k + 4], v[8 * k + 5], v[8 * k + 6], v[8 * k + 7]);
    }
    // centre as FatTriangle::getCenter (geometry/triangle.h:59-62)
    const float third = 1.0f / 3.0f;
    const float cx = __fmul_rn(__fadd_rn(__fadd_rn(v[0], v[8]), v[16]), third);
    const float cy = __fmul_rn(__fadd_rn(__fadd_rn(v[1], v[9]), v[17]), third);
    const float cz = __fmul_rn(__fadd_rn(__fadd_rn(v[2], v[10]), v[18]), third);
    triKeys[t] = morton30(cx, cy, cz, bounds);
    triVals[t] = (uint32_t)t;
}

// 3./4. de-duplication ---------------------------------------------------------------

__device__ __forceinline__ uint32_t mix32(uint32_t h, uint32_t w)
{
    h ^= w * 0xcc9e2d51u;
    h = (h << 15) | (h >> 17);
    return h * 0x1b873593u + 0xe6546b64u;
}

__device__ __forceinline__ bool has_nan(const float4& a, const float4& b)
{
    return isnan(a.x) || isnan(a.y) || isnan(a.z) || isnan(a.w) || isnan(b.x) || isnan(b.y) || isnan(b.z) ||
           isnan(b.w);
}

__device__ __forceinline__ bool same_bits(const float4& a, const float4& b)
{
    return __float_as_uint(a.x) == __float_as_uint(b.x) && __float_as_uint(a.y) == __float_as_uint(b.y) &&
           __float_as_uint(a.z) == __float_as_uint(b.z) && __float_as_uint(a.w) == __float_as_uint(b.w);
}

__global__ void __launch_bounds__(256) k_dedup_insert(const float4* __restrict__ corners, int nc,
                                                    uint32_t* __restrict__ table, uint32_t mask, int* __restrict__ slotOf,
                                                    int* __restrict__ error)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const float4 a = corners[2 * (size_t)c], b = corners[2 * (size_t)c + 1];
    if (has_nan(a, b))
    {
        slotOf[c] = -1;
        return;
    }
    uint32_t h = 0x2545f491u;
    h = mix32(h, __float_as_uint(a.x));
    h = mix32(h, __float_as_uint(a.y));
    h = mix32(h, __float_as_uint(a.z));
    h = mix32(h, __float_as_uint(a.w));
    h = mix32(h, __float_as_uint(b.x));
    h = mix32(h, __float_as_uint(b.y));
    h = mix32(h, __float_as_uint(b.z));
    h = mix32(h, __float_as_uint(b.w));
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    uint32_t slot = h & mask;
    // at most one full sweep of the table (it holds at least twice as many slots as corners)
    for (uint32_t probe = 0; probe <= mask; ++probe)
    {
        uint32_t s = *((volatile uint32_t*)&table[slot]);
        if (s == kEmptySlot)
        {
            const uint32_t prev = atomicCAS(&table[slot], kEmptySlot, (uint32_t)c);
            if (prev == kEmptySlot)
            {
                slotOf[c] = (int)slot;
                return;
            }
            s = prev;
        }
        // s only ever moves to lower corners with the same record
        if (same_bits(corners[2 * (size_t)s], a) && same_bits(corners[2 * (size_t)s + 1], b))
        {
            atomicMin(&table[slot], (uint32_t)c);
            slotOf[c] = (int)slot;
            return;
        }
        slot = (slot + 1) & mask;
    }
    atomicExch(error, 1);
    slotOf[c] = -1;
}

__global__ void __launch_bounds__(256) k_dedup_resolve(const int* __restrict__ slotOf, const uint32_t* __restrict__ table,
                                                     int nc, int* __restrict__ rep, uint32_t* __restrict__ unique)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int s = slotOf[c];
    const int r = s < 0 ? c : (int)table[s];
    rep[c] = r;
    unique[c] = r == c ? 1u : 0u;
}

// 6./7. vertices ---------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_vertex_keys(const uint32_t* __restrict__ unique, const uint32_t* __restrict__ pos,
                                                   const float4* __restrict__ corners, int nc,
                                                   const float* __restrict__ bounds, uint32_t* __restrict__ keys,
                                                   uint32_t* __restrict__ vals)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc || !unique[c]) return;
    const float4 a = corners[2 * (size_t)c];
    const uint32_t i = pos[c];
    keys[i] = morton30(a.x, a.y, a.z, bounds);
    vals[i] = (uint32_t)c;
}

__global__ void __launch_bounds__(256) k_vertex_emit(const uint32_t* __restrict__ order, int nv,
                                                   const float4* __restrict__ corners, const unsigned* __restrict__ flags,
                                                   float* __restrict__ attr, int* __restrict__ newId)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nv) return;
    const uint32_t c = order[j];
    newId[c] = j;
    const float4 a = corners[2 * (size_t)c], b = corners[2 * (size_t)c + 1];
    const unsigned f = *flags;
    const bool hn = f & kFlagNormals, ht = f & kFlagTexcoords;
    const int stride = 3 + (hn ? 3 : 0) + (ht ? 2 : 0);
    float* o = attr + (size_t)j * stride;
    o[0] = a.x;
    o[1] = a.y;
    o[2] = a.z;
    int k = 3;
    if (hn)
    {
        o[k++] = a.w;
        o[k++] = b.x;
        o[k++] = b.y;
    }
    if (ht)
    {
        o[k++] = b.z;
        o[k++] = b.w;
    }
}

// 8. triangles -----------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_tri_emit(const uint32_t* __restrict__ order, int n, const int* __restrict__ rep,
                                                const int* __restrict__ newId, const float* __restrict__ soup,
                                                const unsigned* __restrict__ flags, int* __restrict__ idx,
                                                int* __restrict__ mat)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const long long t = order[j];
#pragma unroll
    for (int k = 0; k < 3; ++k) idx[3 * (size_t)j + k] = newId[rep[3 * t + k]];
    mat[j] = (*flags & kFlagMaterials) ? __float_as_int(soup[kSoupFloats * t + 24]) : 0;
}

// 0. expansion of an indexed soup into 100-byte triangle records on the device

__global__ void __launch_bounds__(256) k_soup_expand(const float* __restrict__ v, const float* __restrict__ vt,
                                                   const float* __restrict__ vn, const int* __restrict__ corners,
                                                   int cornerInts, const int* __restrict__ mat, int n,
                                                   float* __restrict__ soup)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int* c = corners + 3 * cornerInts * t;
    float* o = soup + kSoupFloats * t;
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        const long long p = c[cornerInts * k];
        const int tx = cornerInts == 3 ? c[3 * k + 1] : -1, nr = cornerInts == 3 ? c[3 * k + 2] : -1;
        o[8 * k + 0] = v[3 * p];
        o[8 * k + 1] = v[3 * p + 1];
        o[8 * k + 2] = v[3 * p + 2];
        o[8 * k + 3] = nr >= 0 ? vn[3 * (long long)nr] : 0.f;
        o[8 * k + 4] = nr >= 0 ? vn[3 * (long long)nr + 1] : 0.f;
        o[8 * k + 5] = nr >= 0 ? vn[3 * (long long)nr + 2] : 0.f;
        o[8 * k + 6] = tx >= 0 ? vt[2 * (long long)tx] : 0.f;
        o[8 * k + 7] = tx >= 0 ? vt[2 * (long long)tx + 1] : 0.f;
    }
    o[24] = __int_as_float(mat[t]);
}

} // namespace

int build_mesh_gpu(const prt_soup_triangle* hostTris, int n, cudaStream_t stream, BuiltMesh& out, std::string& err,
                   double* buildMs, long long* launchesOut, bool soupOnDevice, DeviceScratch* scratch)
{
    out.reset();
    if (n < 0 || n > 0x7fffffff / 3)
    {
        err = "triangle count out of range";
        return PRT_EINVAL;
    }
    int status = PRT_OK;
    long long launches = 0;
    const int nc = 3 * n;
    const int scanBlocks = std::min(1024, std::max(1, div_up(n, 256)));
    uint32_t tableSize = 1024;
    while (tableSize < 2u * (uint32_t)std::max(nc, 1)) tableSize <<= 1;

    char* block = nullptr;        // the scratch buffers below
    float* soup = nullptr;
    float* partial = nullptr;
    float* bounds = nullptr;      // [6]
    unsigned* small = nullptr;    // [0] flags, [1] error
    float4* corners = nullptr;
    uint32_t *triKeys = nullptr, *triVals = nullptr, *keysTmp = nullptr, *valsTmp = nullptr, *hist = nullptr;
    uint32_t* table = nullptr;
    int *slotOf = nullptr, *rep = nullptr;
    uint32_t *unique = nullptr, *pos = nullptr, *sums = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    unsigned hostSmall[2] = {0, 0};
    uint32_t nv32 = 0;
    float hb[6];

#define MB_CHECK(x)                                                                                              \
    do                                                                                                           \
    {                                                                                                            \
        cudaError_t e_ = (x);                                                                                    \
        if (e_ != cudaSuccess)                                                                                   \
        {                                                                                                        \
            err = std::string(#x) + ": " + cudaGetErrorString(e_);                                              \
            status = e_ == cudaErrorMemoryAllocation ? PRT_ENOMEM : PRT_ECUDA;                                 \
            goto done;                                                                                           \
        }                                                                                                        \
    } while (0)

    MB_CHECK(cudaEventCreate(&ev0));
    MB_CHECK(cudaEventCreate(&ev1));
    {
        // every scratch buffer in one block
        const size_t hc = n > 0 ? radix_sort_hist_entries(std::max(n, nc)) : 0;
        auto carve = [&](char* base) {
            Carve c{base};
            small = c.take<unsigned>(2);
            bounds = c.take<float>(6);
            partial = c.take<float>(6 * (size_t)scanBlocks);
            if (n > 0)
            {
                if (!soupOnDevice) soup = c.take<float>(sizeof(prt_soup_triangle) / sizeof(float) * (size_t)n);
                corners = c.take<float4>(2 * (size_t)nc);
                triKeys = c.take<uint32_t>(n);
                triVals = c.take<uint32_t>(n);
                keysTmp = c.take<uint32_t>(nc);
                valsTmp = c.take<uint32_t>(nc);
                hist = c.take<uint32_t>(hc);
                table = c.take<uint32_t>(tableSize);
                slotOf = c.take<int>(nc);
                rep = c.take<int>(nc);
                unique = c.take<uint32_t>(nc);
                pos = c.take<uint32_t>(nc);
                sums = c.take<uint32_t>(scan_sums_entries(nc));
            }
            return c.off;
        };
        const size_t bytes = carve(nullptr);
        if (scratch)
        {
            MB_CHECK(scratch->reserve(bytes));
            block = static_cast<char*>(scratch->p);
        }
        else
        {
            MB_CHECK(dev_malloc(&block, bytes));
        }
        carve(block);
    }
    if (n > 0)
    {
        if (soupOnDevice) soup = const_cast<float*>(reinterpret_cast<const float*>(hostTris));
        if (!soupOnDevice)
            MB_CHECK(cudaMemcpyAsync(soup, hostTris, sizeof(prt_soup_triangle) * (size_t)n, cudaMemcpyDefault, stream));
    }
    MB_CHECK(cudaMemsetAsync(small, 0, sizeof(unsigned) * 2, stream));
    MB_CHECK(cudaEventRecord(ev0, stream));
    k_soup_scan<<<scanBlocks, 256, 0, stream>>>(soup, n, small, partial);
    k_bounds_final<<<1, 192, 0, stream>>>(partial, scanBlocks, bounds);
    launches += 2;
    if (n > 0)
    {
        k_soup_corners<<<div_up(n, 256), 256, 0, stream>>>(soup, n, small, bounds, corners, triKeys, triVals);
        MB_CHECK(cudaMemsetAsync(table, 0xff, sizeof(uint32_t) * (size_t)tableSize, stream));
        k_dedup_insert<<<div_up(nc, 256), 256, 0, stream>>>(corners, nc, table, tableSize - 1, slotOf, (int*)small + 1);
        k_dedup_resolve<<<div_up(nc, 256), 256, 0, stream>>>(slotOf, table, nc, rep, unique);
        launches += 3;
        launches += exclusive_scan_u32(unique, pos, sums, nc, stream);
        MB_CHECK(cudaGetLastError());
        MB_CHECK(cudaMemcpyAsync(&nv32, sums + scan_sums_entries(nc) - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 stream));
    }
    MB_CHECK(cudaMemcpyAsync(hostSmall, small, sizeof(hostSmall), cudaMemcpyDeviceToHost, stream));
    MB_CHECK(cudaMemcpyAsync(hb, bounds, sizeof(hb), cudaMemcpyDeviceToHost, stream));
    MB_CHECK(cudaStreamSynchronize(stream));
    if (hostSmall[1])
    {
        err = "mesh builder hash table overflow";
        status = PRT_EINTERNAL;
        goto done;
    }
    out.triCount = n;
    out.vertCount = (int)nv32;
    out.hasNormals = hostSmall[0] & kFlagNormals;
    out.hasTexcoords = hostSmall[0] & kFlagTexcoords;
    out.hasMaterials = hostSmall[0] & kFlagMaterials;
    out.stride = 3 + (out.hasNormals ? 3 : 0) + (out.hasTexcoords ? 2 : 0);
    std::memcpy(out.lo, hb, 12);
    std::memcpy(out.hi, hb + 3, 12);
    {
        // the outputs in one block
        auto carveOut = [&](char* base) {
            Carve c{base};
            out.idx = c.take<int>(3 * (size_t)std::max(n, 1));
            out.mat = c.take<int>((size_t)std::max(n, 1));
            out.attr = c.take<float>((size_t)out.stride * (size_t)std::max(out.vertCount, 1));
            return c.off;
        };
        const size_t bytes = carveOut(nullptr);
        if (out.blockBytes < bytes)
        {
            if (out.block) cudaFree(out.block);
            out.block = nullptr;
            out.blockBytes = 0;
            char* ob = nullptr;
            MB_CHECK(dev_malloc(&ob, bytes));
            out.block = ob;
            out.blockBytes = bytes;
        }
        carveOut(static_cast<char*>(out.block));
    }
    if (n > 0)
    {
        const int nv = out.vertCount;
        // storage no longer needed is reused: the hash table (>= 2 nc words) and
        // slotOf hold the unique vertex keys and values, pos becomes newId once
        // the keys are made
        uint32_t* vKeys = table;
        uint32_t* vVals = reinterpret_cast<uint32_t*>(slotOf);
        uint32_t* kt = keysTmp;
        uint32_t* vt = valsTmp;
        k_vertex_keys<<<div_up(nc, 256), 256, 0, stream>>>(unique, pos, corners, nc, bounds, vKeys, vVals);
        launches++;
        launches += radix_sort_pairs(vKeys, vVals, kt, vt, hist, nv, 30, stream);
        int* newId = reinterpret_cast<int*>(pos);
        k_vertex_emit<<<div_up(nv, 256), 256, 0, stream>>>(vVals, nv, corners, small, out.attr, newId);
        launches++;
        uint32_t* tk = triKeys;
        uint32_t* tv = triVals;
        kt = keysTmp;
        vt = valsTmp;
        launches += radix_sort_pairs(tk, tv, kt, vt, hist, n, 30, stream);
        k_tri_emit<<<div_up(n, 256), 256, 0, stream>>>(tv, n, rep, newId, soup, small, out.idx, out.mat);
        launches++;
        MB_CHECK(cudaGetLastError());
    }
    MB_CHECK(cudaEventRecord(ev1, stream));
    MB_CHECK(cudaStreamSynchronize(stream));
    if (buildMs)
    {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0, ev1);
        *buildMs = ms;
    }
    out.valid = true;

done:
#undef MB_CHECK
    if (!scratch) cudaFree(block);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (status != PRT_OK) out.release();
    if (launchesOut) *launchesOut += launches;
    return status;
}

int build_mesh_gpu_indexed(const SoupIndexed& s, cudaStream_t stream, BuiltMesh& out, std::string& err, double* buildMs,
                           long long* launchesOut, DeviceScratch* scratch, DeviceScratch* upload)
{
    out.reset();
    if (s.triCount < 0 || s.triCount > 0x7fffffff / 3)
    {
        err = "triangle count out of range";
        return PRT_EINVAL;
    }
    const int n = (int)s.triCount;
    if (n == 0) return build_mesh_gpu(nullptr, 0, stream, out, err, buildMs, launchesOut, false, scratch);
    int status = PRT_OK;
    float *dv = nullptr, *dvt = nullptr, *dvn = nullptr, *dsoup = nullptr;
    int *dcorners = nullptr, *dmat = nullptr;
    const size_t cornerInts = 3 * (size_t)s.cornerInts * (size_t)n;
    // the uploaded lists and the expanded records in one block
    auto carve = [&](char* base) {
        Carve c{base};
        dv = c.take<float>(3 * (size_t)std::max(1LL, s.nv));
        dvt = s.nvt ? c.take<float>(2 * (size_t)s.nvt) : nullptr;
        dvn = s.nvn ? c.take<float>(3 * (size_t)s.nvn) : nullptr;
        dcorners = c.take<int>(cornerInts);
        dmat = c.take<int>((size_t)n);
        dsoup = c.take<float>(sizeof(prt_soup_triangle) / sizeof(float) * (size_t)n);
        return c.off;
    };
    char* block = nullptr;
    cudaError_t e = cudaSuccess;
    if (upload)
    {
        e = upload->reserve(carve(nullptr));
        block = static_cast<char*>(upload->p);
    }
    else
    {
        e = dev_malloc(&block, carve(nullptr));
    }
    if (e == cudaSuccess) carve(block);
    if (e == cudaSuccess && s.nv) e = cudaMemcpyAsync(dv, s.v, sizeof(float) * 3 * (size_t)s.nv, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && s.nvt)
        e = cudaMemcpyAsync(dvt, s.vt, sizeof(float) * 2 * (size_t)s.nvt, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && s.nvn)
        e = cudaMemcpyAsync(dvn, s.vn, sizeof(float) * 3 * (size_t)s.nvn, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dcorners, s.corners, sizeof(int) * cornerInts, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dmat, s.mat, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
    {
        k_soup_expand<<<div_up(n, 256), 256, 0, stream>>>(dv, dvt, dvn, dcorners, s.cornerInts, dmat, n, dsoup);
        if (launchesOut) ++*launchesOut;
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
    {
        err = std::string("indexed soup upload: ") + cudaGetErrorString(e);
        status = e == cudaErrorMemoryAllocation ? PRT_ENOMEM : PRT_ECUDA;
    }
    else
    {
        status = build_mesh_gpu(reinterpret_cast<const prt_soup_triangle*>(dsoup), n, stream, out, err, buildMs,
                                launchesOut, true, scratch);
    }
    if (!upload) cudaFree(block);
    if (status != PRT_OK) out.release();
    return status;
}

} // namespace prt_b200
