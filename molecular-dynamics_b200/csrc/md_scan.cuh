// Exclusive prefix sums on the device (cell starts, CSR offsets). Three passes: per-tile totals, one-block
// scan of the tile totals, per-tile scan plus the tile's offset. Integer sums, so the result does not depend
// on the launch shape.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace md {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one long long per thread; returns the thread's exclusive prefix and writes
// the block total to *total. Needs kScanThreads / 32 + 1 longs of shared memory.
__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* warp_tot, long long* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        long long w = lane < nw ? warp_tot[lane] : 0;
        long long winc = w;
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, winc, o);
            if (lane >= o) winc += u;
        }
        if (lane < nw) warp_tot[lane] = winc - w;
        if (lane == nw - 1) *total = winc;
    }
    __syncthreads();
    const long long r = warp_tot[warp] + inc - v;
    __syncthreads();
    return r;
}

template <typename TIn>
__global__ void k_scan_reduce(const TIn* __restrict__ in, long long n, long long* __restrict__ tile_sums) {
    __shared__ long long red[kScanThreads / 32];
    const long long base = static_cast<long long>(blockIdx.x) * kScanTile;
    long long s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const long long i = base + static_cast<long long>(k) * kScanThreads + threadIdx.x;
        if (i < n) s += static_cast<long long>(in[i]);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < kScanThreads / 32; ++w) t += red[w];
        tile_sums[blockIdx.x] = t;
    }
}

// One block of kScanThreads: exclusive scan of tile_sums[0..nt) in place; tile_sums[nt] = grand total.
__global__ void k_scan_tiles(long long* __restrict__ tile_sums, int nt) {
    __shared__ long long warp_tot[kScanThreads / 32 + 1];
    __shared__ long long total;
    const int per = (nt + kScanThreads - 1) / kScanThreads;
    const int b = threadIdx.x * per;
    long long s = 0;
    for (int k = 0; k < per; ++k)
        if (b + k < nt) s += tile_sums[b + k];
    const long long ex = block_exclusive_scan(s, warp_tot, &total);
    long long run = ex;
    for (int k = 0; k < per; ++k) {
        if (b + k < nt) {
            const long long v = tile_sums[b + k];
            tile_sums[b + k] = run;
            run += v;
        }
    }
    if (threadIdx.x == 0) tile_sums[nt] = total;
}

// out[i] = sum of in[0..i) for i in [0, n]; out has n + 1 entries
template <typename TIn, typename TOut>
__global__ void k_scan_down(const TIn* __restrict__ in, long long n, const long long* __restrict__ tile_off,
                            TOut* __restrict__ out) {
    __shared__ long long warp_tot[kScanThreads / 32 + 1];
    __shared__ long long total;
    const long long base = static_cast<long long>(blockIdx.x) * kScanTile + static_cast<long long>(threadIdx.x) * kScanItems;
    long long v[kScanItems];
    long long s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const long long i = base + k;
        v[k] = i < n ? static_cast<long long>(in[i]) : 0;
        s += v[k];
    }
    long long run = block_exclusive_scan(s, warp_tot, &total) + tile_off[blockIdx.x];
    for (int k = 0; k < kScanItems; ++k) {
        const long long i = base + k;
        if (i < n) out[i] = static_cast<TOut>(run);
        run += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = static_cast<TOut>(tile_off[gridDim.x]);
}

// Host launcher: tile_sums must hold ceil(n / kScanTile) + 1 entries.
template <typename TIn, typename TOut>
inline void exclusive_scan(const TIn* in, long long n, TOut* out, long long* tile_sums, cudaStream_t st) {
    const int nt = static_cast<int>((n + kScanTile - 1) / kScanTile);
    if (nt == 0) {
        cudaMemsetAsync(out, 0, sizeof(TOut), st);
        return;
    }
    k_scan_reduce<TIn><<<nt, kScanThreads, 0, st>>>(in, n, tile_sums);
    k_scan_tiles<<<1, kScanThreads, 0, st>>>(tile_sums, nt);
    k_scan_down<TIn, TOut><<<nt, kScanThreads, 0, st>>>(in, n, tile_sums, out);
}

inline long long scan_tiles_needed(long long n) { return (n + kScanTile - 1) / kScanTile + 1; }

}  // namespace md
