// sort.cu — distinct-pair counting by radix sort (the sort mode of the
// body-size deduplication).
//
// In sort mode the engine appends one 64-bit key per body grounding that
// reaches hO: [sort index of the plan | hS row | hO rank] (see emit_pair in
// kernels.cu).  This file sorts those keys with a least-significant-digit
// radix sort, 8 bits per pass over only the bits in use, and then counts
// each plan's distinct keys into its result slot.  The reference does the
// same job with Thrust: a comparison sort of int2 pairs followed by unique
// (GPU_03/gpu_rules_lib.cu:485-518, after an overflow-and-double retry loop);
// here both are written for this data, and the buffer is sized exactly from
// the append cursor when an estimate was short (see Staged in engine.hpp).
//
// Per pass (tile = 2,048 keys, 256 threads x 8 keys, read coalesced):
//   radix_hist_kernel     digit counts per tile, stored digit-major, and
//                         per-digit totals
//   radix_scan_kernel     one block per digit: the exclusive prefix of its
//                         counts over tiles, plus the digit's base
//   radix_scatter_kernel  stable rank of each key within its tile
//                         (__match_any_sync per warp, then a prefix over
//                         (key round, warp) per digit), keys reordered by
//                         digit in shared memory and written out in runs
// The key count lives on the device (the append cursor, clamped to the
// capacity), so every kernel reads it there and the whole sequence can be
// captured in a CUDA graph with grids sized for the capacity.
#include <cuda_runtime.h>

#include <cstdint>

namespace gr {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortPerThread = 8;
constexpr int kSortTile = kSortThreads * kSortPerThread;
constexpr int kRadix = 256;
constexpr int kSortWarps = kSortThreads / 32;

__device__ __forceinline__ long long keys_in(const unsigned long long* count, unsigned long long cap) {
    const unsigned long long n = *count;
    return (long long)(n < cap ? n : cap);
}

// hist[d * tilesCap + t]: keys of tile t with digit d; hist[kRadix * tilesCap + d]:
// keys with digit d (zeroed before the pass).
__global__ void __launch_bounds__(kSortThreads)
radix_hist_kernel(const unsigned long long* __restrict__ keys, const unsigned long long* count, unsigned long long cap,
                  int shift, uint32_t* hist, long long tilesCap) {
    __shared__ uint32_t h[kRadix];
    const long long n = keys_in(count, cap);
    const long long tiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* totals = hist + (size_t)kRadix * tilesCap;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
        h[threadIdx.x] = 0u;
        __syncthreads();
        const long long base = t * kSortTile;
        const unsigned lower = (1u << (threadIdx.x & 31)) - 1u;
#pragma unroll
        for (int k = 0; k < kSortPerThread; ++k) {
            const long long i = base + (long long)k * kSortThreads + threadIdx.x;
            const int d = i < n ? (int)((unsigned)(keys[i] >> shift) & (kRadix - 1)) : kRadix;
            // one shared atomic per distinct digit of the warp (the high
            // digits of small keys are mostly equal)
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            if (d < kRadix && (peers & lower) == 0) atomicAdd(&h[d], (uint32_t)__popc(peers));
        }
        __syncthreads();
        const uint32_t c = h[threadIdx.x];
        hist[(size_t)threadIdx.x * tilesCap + t] = c;
        if (c) atomicAdd(&totals[threadIdx.x], c);
        __syncthreads();
    }
}

// Block-wide inclusive scan of one value per thread (blockDim.x = 1024).
__device__ __forceinline__ uint32_t block_incl_scan(uint32_t v, uint32_t* warpSums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += y;
    }
    if (lane == 31) warpSums[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t w = lane < nw ? warpSums[lane] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w += y;
        }
        if (lane < nw) warpSums[lane] = w;
    }
    __syncthreads();
    return v + (warp > 0 ? warpSums[warp - 1] : 0u);
}

// One block per digit d: hist[d][t] becomes the output position of tile t's
// first key with digit d.
__global__ void __launch_bounds__(1024)
radix_scan_kernel(uint32_t* hist, const unsigned long long* count, unsigned long long cap, long long tilesCap) {
    __shared__ uint32_t warpSums[32];
    __shared__ uint32_t base;
    const int d = blockIdx.x;
    const long long n = keys_in(count, cap);
    const long long tiles = (n + kSortTile - 1) / kSortTile;
    const uint32_t* totals = hist + (size_t)kRadix * tilesCap;
    if (threadIdx.x < 32) {
        uint32_t b = 0;
        for (int e = (int)threadIdx.x; e < d; e += 32) b += totals[e];
#pragma unroll
        for (int o = 16; o; o >>= 1) b += __shfl_xor_sync(0xffffffffu, b, o);
        if (threadIdx.x == 0) base = b;
    }
    __syncthreads();
    uint32_t carry = base;
    uint32_t* row = hist + (size_t)d * tilesCap;
    for (long long c0 = 0; c0 < tiles; c0 += blockDim.x) {
        const long long i = c0 + threadIdx.x;
        const uint32_t v = i < tiles ? row[i] : 0u;
        const uint32_t incl = block_incl_scan(v, warpSums);
        if (i < tiles) row[i] = carry + incl - v;
        // every thread reads the chunk's total before the next chunk's scan
        // overwrites warpSums
        carry += warpSums[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kSortThreads)
radix_scatter_kernel(const unsigned long long* __restrict__ in, unsigned long long* __restrict__ out,
                     const unsigned long long* count, unsigned long long cap, int shift, const uint32_t* hist,
                     long long tilesCap) {
    // per (key round k, warp w, digit d): keys of that warp and round with
    // digit d, then their exclusive prefix in tile order; the same memory
    // later holds the tile reordered by digit
    __shared__ union {
        uint16_t cnt[kSortPerThread][kSortWarps][kRadix];
        unsigned long long tile[kSortTile];
    } sh;
    __shared__ uint32_t dStart[kRadix];   // tile-local first position of each digit
    __shared__ uint32_t dOut[kRadix];     // output position of the tile's first key of each digit
    __shared__ uint32_t warpSums[kSortWarps];
    const long long n = keys_in(count, cap);
    const long long tiles = (n + kSortTile - 1) / kSortTile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lower = (1u << lane) - 1u;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
        uint32_t* c32 = reinterpret_cast<uint32_t*>(&sh.cnt[0][0][0]);
        for (int i = tid; i < kSortPerThread * kSortWarps * kRadix / 2; i += kSortThreads) c32[i] = 0u;
        __syncthreads();
        const long long base = t * kSortTile;
        unsigned long long key[kSortPerThread];
        int dig[kSortPerThread];
        int below[kSortPerThread];
#pragma unroll
        for (int k = 0; k < kSortPerThread; ++k) {
            const long long i = base + (long long)k * kSortThreads + tid;
            key[k] = i < n ? in[i] : 0ull;
            dig[k] = i < n ? (int)((unsigned)(key[k] >> shift) & (kRadix - 1)) : kRadix;
            const unsigned peers = __match_any_sync(0xffffffffu, dig[k]);
            below[k] = __popc(peers & lower);
            if (dig[k] < kRadix && below[k] == 0) sh.cnt[k][warp][dig[k]] = (uint16_t)__popc(peers);
        }
        __syncthreads();
        // thread d: prefix of digit d over (round, warp), i.e. in tile order
        uint32_t run = 0;
        for (int k = 0; k < kSortPerThread; ++k)
            for (int w = 0; w < kSortWarps; ++w) {
                const uint32_t x = sh.cnt[k][w][tid];
                sh.cnt[k][w][tid] = (uint16_t)run;
                run += x;
            }
        dOut[tid] = hist[(size_t)tid * tilesCap + t];
        // exclusive scan of the per-digit tile counts over the 256 digits
        uint32_t v = run;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= d) v += y;
        }
        if (lane == 31) warpSums[warp] = v;
        __syncthreads();
        uint32_t before = 0;
        for (int w = 0; w < warp; ++w) before += warpSums[w];
        dStart[tid] = before + v - run;
        __syncthreads();
        uint32_t pos[kSortPerThread];
#pragma unroll
        for (int k = 0; k < kSortPerThread; ++k)
            pos[k] = dig[k] < kRadix ? dStart[dig[k]] + sh.cnt[k][warp][dig[k]] + (uint32_t)below[k] : 0xffffffffu;
        __syncthreads();   // the counters are read; the tile may overwrite them
#pragma unroll
        for (int k = 0; k < kSortPerThread; ++k)
            if (pos[k] != 0xffffffffu) sh.tile[pos[k]] = key[k];
        __syncthreads();
        const int m = (int)(n - base < kSortTile ? n - base : kSortTile);
        for (int j = tid; j < m; j += kSortThreads) {
            const unsigned long long x = sh.tile[j];
            const int d = (int)((unsigned)(x >> shift) & (kRadix - 1));
            out[(size_t)dOut[d] + (size_t)(j - (int)dStart[d])] = x;
        }
        __syncthreads();
    }
}

// Distinct keys of the sorted array, added per plan: the key's bits from
// slotShift up are the plan's sort index, slotOf maps it to a result slot.
// Each thread takes a run of consecutive keys and flushes its count when
// the plan changes.  A sort index outside [0, nSlots) is reported through
// status (bit 64) and skipped.
__global__ void __launch_bounds__(kSortThreads)
pairs_unique_kernel(const unsigned long long* __restrict__ keys, const unsigned long long* count,
                    unsigned long long cap, int slotShift, const int32_t* slotOf, int nSlots,
                    unsigned long long* results, int* status) {
    constexpr long long kRun = 16;
    const long long n = keys_in(count, cap);
    const long long stride = (long long)gridDim.x * blockDim.x * kRun;
    for (long long c0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kRun; c0 < n; c0 += stride) {
        const long long c1 = c0 + kRun < n ? c0 + kRun : n;
        unsigned long long prev = c0 > 0 ? keys[c0 - 1] : 0ull;
        int cur = -1;
        unsigned long long acc = 0;
        for (long long i = c0; i < c1; ++i) {
            const unsigned long long x = keys[i];
            if (i == 0 || x != prev) {
                const unsigned long long sx = x >> slotShift;
                const int s = sx < (unsigned long long)nSlots ? (int)sx : -1;
                if (s < 0) atomicOr(status, 64);
                if (s != cur) {
                    if (acc) atomicAdd(results + slotOf[cur], acc);
                    cur = s;
                    acc = 0;
                }
                if (s >= 0) ++acc;
            }
            prev = x;
        }
        if (acc) atomicAdd(results + slotOf[cur], acc);
    }
}

}  // namespace

size_t pairs_sort_hist_words(unsigned long long cap) {
    const unsigned long long tiles = (cap + kSortTile - 1) / kSortTile;
    return (size_t)kRadix * (size_t)(tiles > 0 ? tiles : 1) + kRadix;
}

unsigned long long* radix_sort_keys(unsigned long long* keys, unsigned long long* tmp, const unsigned long long* count,
                                    unsigned long long cap, int bits, uint32_t* hist, int grid, cudaStream_t stream,
                                    cudaError_t* err);

// Sorts the first min(*count, cap) keys by their low `bits` bits, ping-
// ponging between keys and tmp, then adds each plan's distinct keys to
// results[slotOf[key >> slotShift]] (nSlots sort indices; status as the
// engine's).  hist: pairs_sort_hist_words(cap) words.  grid: blocks of the
// per-tile kernels (they loop over tiles).
cudaError_t pairs_sort_count(unsigned long long* keys, unsigned long long* tmp, const unsigned long long* count,
                             unsigned long long cap, int bits, int slotShift, const int32_t* slotOf, int nSlots,
                             unsigned long long* results, int* status, uint32_t* hist, int grid,
                             cudaStream_t stream) {
    if (cap == 0) return cudaSuccess;
    if (bits < 1 || bits > 64 || slotShift < 0 || slotShift > 63 || cap > 0xffffffffull) return cudaErrorInvalidValue;
    const long long tilesCap = (long long)((cap + kSortTile - 1) / kSortTile);
    const int g = (int)(tilesCap < grid ? tilesCap : grid);
    cudaError_t e = cudaSuccess;
    unsigned long long* a = radix_sort_keys(keys, tmp, count, cap, bits, hist, grid, stream, &e);
    if (e != cudaSuccess) return e;
    pairs_unique_kernel<<<g, kSortThreads, 0, stream>>>(a, count, cap, slotShift, slotOf, nSlots, results, status);
    return cudaGetLastError();
}

unsigned long long* radix_sort_keys(unsigned long long* keys, unsigned long long* tmp, const unsigned long long* count,
                                    unsigned long long cap, int bits, uint32_t* hist, int grid, cudaStream_t stream,
                                    cudaError_t* err) {
    *err = cudaSuccess;
    if (cap == 0) return keys;
    if (bits < 1 || bits > 64 || cap > 0xffffffffull) {
        *err = cudaErrorInvalidValue;
        return keys;
    }
    const long long tilesCap = (long long)((cap + kSortTile - 1) / kSortTile);
    const int g = (int)(tilesCap < grid ? tilesCap : grid);
    unsigned long long* a = keys;
    unsigned long long* b = tmp;
    for (int shift = 0; shift < bits; shift += 8) {
        cudaError_t e = cudaMemsetAsync(hist + (size_t)kRadix * tilesCap, 0, kRadix * sizeof(uint32_t), stream);
        if (e != cudaSuccess) { *err = e; return a; }
        radix_hist_kernel<<<g, kSortThreads, 0, stream>>>(a, count, cap, shift, hist, tilesCap);
        radix_scan_kernel<<<kRadix, 1024, 0, stream>>>(hist, count, cap, tilesCap);
        radix_scatter_kernel<<<g, kSortThreads, 0, stream>>>(a, b, count, cap, shift, hist, tilesCap);
        unsigned long long* x = a;
        a = b;
        b = x;
    }
    *err = cudaGetLastError();
    return a;
}

}  // namespace gr
