// Device sort and scan primitives shared by the BVH build and the mesh
// builder: a stable LSD radix sort of (uint32 key, uint32 value) pairs with
// 4-bit digits, and an exclusive scan of uint32 values.
#include <algorithm>
#include <utility>

#include "prt_internal.h"

namespace prt_b200 {

namespace {

constexpr int kSortBlock = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortBlock * kSortItems;
constexpr int kRadixBits = 4;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kScanBlock = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanBlock * kScanItems;

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

__global__ void __launch_bounds__(kSortBlock) k_sort_hist(const uint32_t* __restrict__ keys, int n, int shift,
                                                        uint32_t* __restrict__ hist, int nblocks)
{
    __shared__ uint32_t h[kRadix];
    if (threadIdx.x < kRadix) h[threadIdx.x] = 0;
    __syncthreads();
    int base = blockIdx.x * kSortTile;
    for (int k = 0; k < kSortItems; ++k)
    {
        int i = base + k * kSortBlock + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kRadix) hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// exclusive scan of hist (kRadix * nblocks entries, digit-major) in one block
__global__ void __launch_bounds__(1024) k_sort_scan(uint32_t* __restrict__ hist, int count)
{
    __shared__ uint32_t part[1024];
    int per = (count + 1023) / 1024;
    int b0 = threadIdx.x * per, b1 = min(count, b0 + per);
    uint32_t sum = 0;
    for (int i = b0; i < b1; ++i) sum += hist[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1)
    {
        uint32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
    for (int i = b0; i < b1; ++i)
    {
        uint32_t v = hist[i];
        hist[i] = run;
        run += v;
    }
}

// Each thread owns kSortItems consecutive keys of the tile; per-thread digit
// counts are scanned block-wide in (digit, thread) order, which gives every
// key its stable rank within the tile.
__global__ void __launch_bounds__(kSortBlock) k_sort_scatter(const uint32_t* __restrict__ keysIn,
                                                           const uint32_t* __restrict__ valsIn, uint32_t* __restrict__ keysOut,
                                                           uint32_t* __restrict__ valsOut, int n, int shift,
                                                           const uint32_t* __restrict__ hist, int nblocks)
{
    __shared__ uint32_t cnt[kRadix * kSortBlock];   // [digit][thread]
    __shared__ uint32_t warpSum[kSortBlock / 32];
    __shared__ uint32_t digitStart[kRadix];
    const int t = threadIdx.x;
    const int base = blockIdx.x * kSortTile + t * kSortItems;
    uint32_t key[kSortItems], val[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k)
    {
        int i = base + k;
        key[k] = i < n ? keysIn[i] : 0xffffffffu;
        val[k] = i < n ? valsIn[i] : 0u;
    }
#pragma unroll
    for (int d = 0; d < kRadix; ++d) cnt[d * kSortBlock + t] = 0;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k)
        if (base + k < n) cnt[((key[k] >> shift) & (kRadix - 1)) * kSortBlock + t]++;
    __syncthreads();
    // block-wide exclusive scan over cnt[] (kRadix * kSortBlock entries):
    // thread t scans entries [t*kRadix, (t+1)*kRadix) sequentially
    uint32_t local[kRadix];
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < kRadix; ++j)
    {
        local[j] = cnt[t * kRadix + j];
        sum += local[j];
    }
    // scan of per-thread sums
    uint32_t x = sum;
    const int lane = t & 31, warp = t >> 5;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warpSum[warp] = x;
    __syncthreads();
    if (warp == 0)
    {
        uint32_t w = lane < kSortBlock / 32 ? warpSum[lane] : 0u;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        if (lane < kSortBlock / 32) warpSum[lane] = w;
    }
    __syncthreads();
    uint32_t excl = x - sum + (warp ? warpSum[warp - 1] : 0u);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kRadix; ++j)
    {
        cnt[t * kRadix + j] = excl;
        excl += local[j];
    }
    __syncthreads();
    if (t < kRadix) digitStart[t] = cnt[t * kSortBlock];
    __syncthreads();
    uint32_t seen[kRadix];
#pragma unroll
    for (int d = 0; d < kRadix; ++d) seen[d] = 0;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k)
    {
        if (base + k >= n) continue;
        uint32_t d = (key[k] >> shift) & (kRadix - 1);
        uint32_t rankInTile = cnt[d * kSortBlock + t] + seen[d];
#pragma unroll
        for (int dd = 0; dd < kRadix; ++dd)
            if (dd == (int)d) seen[dd]++;
        uint32_t dst = hist[d * nblocks + blockIdx.x] + (rankInTile - digitStart[d]);
        keysOut[dst] = key[k];
        valsOut[dst] = val[k];
    }
}

// --- exclusive scan ---------------------------------------------------------

// Block-exclusive scan of one kScanTile tile; the tile's sum goes to sums[block].
__global__ void __launch_bounds__(kScanBlock) k_scan_tiles(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                          int n, uint32_t* __restrict__ sums)
{
    __shared__ uint32_t warpSum[kScanBlock / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const long long base = (long long)blockIdx.x * kScanTile + (long long)t * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        v[k] = base + k < n ? in[base + k] : 0u;
        sum += v[k];
    }
    uint32_t x = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warpSum[warp] = x;
    __syncthreads();
    if (warp == 0)
    {
        uint32_t w = lane < kScanBlock / 32 ? warpSum[lane] : 0u;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        if (lane < kScanBlock / 32) warpSum[lane] = w;
    }
    __syncthreads();
    uint32_t run = x - sum + (warp ? warpSum[warp - 1] : 0u);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (t == kScanBlock - 1) sums[blockIdx.x] = run;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_add(uint32_t* __restrict__ out, int n,
                                                        const uint32_t* __restrict__ offsets)
{
    const uint32_t add = offsets[blockIdx.x];
    const long long base = (long long)blockIdx.x * kScanTile;
    for (int k = threadIdx.x; k < kScanTile; k += kScanBlock)
        if (base + k < n) out[base + k] += add;
}

} // namespace

size_t radix_sort_hist_entries(int n) { return (size_t)kRadix * (size_t)std::max(1, div_up(n, kSortTile)); }

int radix_sort_pairs(uint32_t*& keys, uint32_t*& vals, uint32_t*& keysTmp, uint32_t*& valsTmp, uint32_t* hist, int n,
                     int bits, cudaStream_t stream)
{
    if (n <= 0) return 0;
    const int blocks = div_up(n, kSortTile);
    const int histCount = kRadix * blocks;
    int launches = 0;
    for (int shift = 0; shift < bits; shift += kRadixBits)
    {
        k_sort_hist<<<blocks, kSortBlock, 0, stream>>>(keys, n, shift, hist, blocks);
        k_sort_scan<<<1, 1024, 0, stream>>>(hist, histCount);
        k_sort_scatter<<<blocks, kSortBlock, 0, stream>>>(keys, vals, keysTmp, valsTmp, n, shift, hist, blocks);
        std::swap(keys, keysTmp);
        std::swap(vals, valsTmp);
        launches += 3;
    }
    return launches;
}

size_t scan_sums_entries(int n) { return (size_t)std::max(1, div_up(n, kScanTile)) + 1; }

int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t* sums, int n, cudaStream_t stream)
{
    const int blocks = std::max(1, div_up(n, kScanTile));
    cudaMemsetAsync(sums + blocks, 0, sizeof(uint32_t), stream);
    k_scan_tiles<<<blocks, kScanBlock, 0, stream>>>(in, out, n, sums);
    k_sort_scan<<<1, 1024, 0, stream>>>(sums, blocks + 1);
    k_scan_add<<<blocks, kScanBlock, 0, stream>>>(out, n, sums);
    return 3;
}

} // namespace prt_b200
