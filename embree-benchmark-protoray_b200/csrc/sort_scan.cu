// Device sort and scan primitives shared by the BVH build and the mesh
// builder: a stable LSD radix sort of (uint32 key, uint32 value) pairs with
// 8-bit digits, and an exclusive scan of uint32 values.
//
// One sort pass over tiles of kSortTile pairs: k_sort_hist counts the digits
// of every tile (digit-major table, one column per tile), exclusive_scan_u32
// turns the table into the first output position of every (digit, tile), and
// k_sort_scatter ranks the tile's pairs stably by digit in shared memory and
// writes them out in rank order, so that runs of one digit go out as
// consecutive addresses.
#include <algorithm>
#include <utility>

#include "prt_internal.h"

namespace prt_b200 {

namespace {

constexpr int kSortBlock = 256;
constexpr int kSortWarps = kSortBlock / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortBlock * kSortItems;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kScanBlock = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanBlock * kScanItems;
static_assert(kRadix == kSortBlock, "one thread per digit in the tile scans");

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// Pair j of a tile is read by warp j / (32 kSortItems), item (j / 32) % kSortItems,
// lane j % 32: each item is one coalesced 128-byte row, and the (warp, item,
// lane) order is the input order, which keeps the ranking stable.
__device__ __forceinline__ int tile_index(int warp, int item, int lane)
{
    return warp * 32 * kSortItems + item * 32 + lane;
}

__global__ void __launch_bounds__(kSortBlock) k_sort_hist(const uint32_t* __restrict__ keys, int n, int shift,
                                                        uint32_t* __restrict__ hist, int nblocks)
{
    __shared__ uint32_t h[kSortWarps][kRadix];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = lane; d < kRadix; d += 32) h[warp][d] = 0;
    __syncwarp();
    const long long base = (long long)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int k = 0; k < kSortItems; ++k)
    {
        const long long i = base + tile_index(warp, k, lane);
        const bool valid = i < n;
        const uint32_t d = valid ? (__ldg(keys + i) >> shift) & (kRadix - 1) : kRadix;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (valid && lane == __ffs(peers) - 1) h[warp][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    uint32_t sum = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) sum += h[w][threadIdx.x];
    hist[(size_t)threadIdx.x * nblocks + blockIdx.x] = sum;
}

__global__ void __launch_bounds__(kSortBlock) k_sort_scatter(const uint32_t* __restrict__ keysIn,
                                                           const uint32_t* __restrict__ valsIn, uint32_t* __restrict__ keysOut,
                                                           uint32_t* __restrict__ valsOut, int n, int shift,
                                                           const uint32_t* __restrict__ offsets, int nblocks)
{
    __shared__ uint32_t warpCnt[kSortWarps][kRadix];   // per warp: digit counts, then offsets
    __shared__ uint32_t tileStart[kRadix];             // first tile rank of each digit
    __shared__ int gbase[kRadix];                      // output position of tile rank 0 of each digit
    __shared__ uint32_t warpSum[kSortWarps];
    __shared__ uint32_t sKeys[kSortTile];
    __shared__ uint32_t sVals[kSortTile];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const long long base = (long long)blockIdx.x * kSortTile;
    const int tileCount = (int)std::min<long long>(kSortTile, n - base);

    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k)
    {
        const long long i = base + tile_index(warp, k, lane);
        key[k] = i < n ? __ldg(keysIn + i) : 0u;
        val[k] = i < n ? __ldg(valsIn + i) : 0u;
    }
    for (int d = lane; d < kRadix; d += 32) warpCnt[warp][d] = 0;
    __syncwarp();
    // rank within the warp: earlier items, then lower lanes of this item
#pragma unroll
    for (int k = 0; k < kSortItems; ++k)
    {
        const bool valid = tile_index(warp, k, lane) < tileCount;
        const uint32_t d = valid ? (key[k] >> shift) & (kRadix - 1) : kRadix;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = valid ? warpCnt[warp][d] : 0u;
        rank[k] = before + __popc(peers & ((1u << lane) - 1u));
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) warpCnt[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // thread t = digit t: offsets of the warps within the digit, the digit's
    // tile total, and (block scan over digits) its first tile rank
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w)
    {
        const uint32_t c = warpCnt[w][t];
        warpCnt[w][t] = total;
        total += c;
    }
    uint32_t x = total;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warpSum[warp] = x;
    __syncthreads();
    uint32_t before = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w)
        if (w < warp) before += warpSum[w];
    const uint32_t start = before + x - total;
    tileStart[t] = start;
    gbase[t] = (int)offsets[(size_t)t * nblocks + blockIdx.x] - (int)start;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k)
    {
        if (tile_index(warp, k, lane) >= tileCount) continue;
        const uint32_t d = (key[k] >> shift) & (kRadix - 1);
        const uint32_t r = tileStart[d] + warpCnt[warp][d] + rank[k];
        sKeys[r] = key[k];
        sVals[r] = val[k];
    }
    __syncthreads();
    for (int r = t; r < tileCount; r += kSortBlock)
    {
        const uint32_t kk = sKeys[r];
        const int dst = gbase[(kk >> shift) & (kRadix - 1)] + r;
        keysOut[dst] = kk;
        valsOut[dst] = sVals[r];
    }
}

// exclusive scan of count entries in one block (the tile sums of the scan)
__global__ void __launch_bounds__(1024) k_scan_one_block(uint32_t* __restrict__ a, int count)
{
    __shared__ uint32_t part[1024];
    int per = (count + 1023) / 1024;
    int b0 = threadIdx.x * per, b1 = min(count, b0 + per);
    uint32_t sum = 0;
    for (int i = b0; i < b1; ++i) sum += a[i];
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
        uint32_t v = a[i];
        a[i] = run;
        run += v;
    }
}

// --- exclusive scan ---------------------------------------------------------

// Block-exclusive scan of one kScanTile tile; the tile's sum goes to sums[block].
// in and out may be the same array (each thread reads its items before it
// writes them).
__global__ void __launch_bounds__(kScanBlock) k_scan_tiles(const uint32_t* in, uint32_t* out,
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

size_t scan_sums_entries(int n);

size_t radix_sort_hist_entries(int n)
{
    const size_t table = (size_t)kRadix * (size_t)std::max(1, div_up(n, kSortTile));
    return table + scan_sums_entries((int)table);
}

int radix_sort_pairs(uint32_t*& keys, uint32_t*& vals, uint32_t*& keysTmp, uint32_t*& valsTmp, uint32_t* hist, int n,
                     int bits, cudaStream_t stream)
{
    if (n <= 0) return 0;
    const int blocks = div_up(n, kSortTile);
    const int table = kRadix * blocks;
    uint32_t* sums = hist + table;
    int launches = 0;
    for (int shift = 0; shift < bits; shift += kRadixBits)
    {
        k_sort_hist<<<blocks, kSortBlock, 0, stream>>>(keys, n, shift, hist, blocks);
        launches += 1 + exclusive_scan_u32(hist, hist, sums, table, stream);
        k_sort_scatter<<<blocks, kSortBlock, 0, stream>>>(keys, vals, keysTmp, valsTmp, n, shift, hist, blocks);
        std::swap(keys, keysTmp);
        std::swap(vals, valsTmp);
        launches += 1;
    }
    return launches;
}

size_t scan_sums_entries(int n) { return (size_t)std::max(1, div_up(n, kScanTile)) + 1; }

int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t* sums, int n, cudaStream_t stream)
{
    const int blocks = std::max(1, div_up(n, kScanTile));
    cudaMemsetAsync(sums + blocks, 0, sizeof(uint32_t), stream);
    k_scan_tiles<<<blocks, kScanBlock, 0, stream>>>(in, out, n, sums);
    k_scan_one_block<<<1, 1024, 0, stream>>>(sums, blocks + 1);
    k_scan_add<<<blocks, kScanBlock, 0, stream>>>(out, n, sums);
    return 3;
}

} // namespace prt_b200
