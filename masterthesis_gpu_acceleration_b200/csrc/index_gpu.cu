// index_gpu.cu — the graph index of index.cpp, built on the device.
//
// The reference builds its CSR on the host, predicate by predicate, with a
// sort of each predicate's pairs and a dense row-pointer array
// (GPU_03/gpu_index.cuh:33-79; CPU_01_nonparallel/RdfIndexes.cpp:60-79).
// Here the triples are packed into 64-bit (predicate, key, value) keys once
// per direction and radix-sorted on the device (sort.cu), and every array of
// the index follows from the sorted keys with flag / prefix-sum passes:
//   unique triples           flag key != previous key, scan, compact
//   rows                     flag (predicate, key) change, scan: row ids,
//                            rowKey and rowBeg at the row starts
//   predRow / predEdge       binary search of each predicate's first key
//   srcRank / valRank        row id minus the predicate's first row; the
//                            value's row in the other direction (binary
//                            search among the predicate's keys there)
//   lookup table             one thread per row, linear probing by CAS
//   row signatures           per entity OR of sig_bit over its rows, read
//                            beside every edge's value, and per row the
//                            suffix OR
// and the arrays are copied back, because the planner and the task builder
// read the index on the host as well.  Hub bitmaps are then built on the
// host (build_hub_rows).  The result equals build_index's array for array,
// except for the order of colliding entries in the lookup table (lookups
// are the same); tests/test_index_gpu.py compares the two.
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.hpp"
#include "index.hpp"

namespace gr {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanPer = 16;
constexpr int kScanTile = kScanThreads * kScanPer;

// ---- exclusive prefix sums of int32 flags (n known on the host) ----

__device__ __forceinline__ int block_excl_scan_int(int v, int* warpSums, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        constexpr int kW = kScanThreads / 32;
        int w = lane < kW ? warpSums[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w += y;
        }
        if (lane < kW) warpSums[lane] = w;
    }
    __syncthreads();
    if (total) *total = warpSums[kScanThreads / 32 - 1];
    return x - v + (warp > 0 ? warpSums[warp - 1] : 0);
}

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums(const int* in, long long n, int* sums) {
    __shared__ int warpSums[kScanThreads / 32];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanPer;
    int v = 0;
    for (int k = 0; k < kScanPer; ++k)
        if (base + k < n) v += in[base + k];
    int total = 0;
    block_excl_scan_int(v, warpSums, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One block: exclusive scan of the tile sums in place.
__global__ void __launch_bounds__(kScanThreads) scan_sums(int* sums, int tiles) {
    __shared__ int warpSums[kScanThreads / 32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int c0 = 0; c0 < tiles; c0 += kScanThreads) {
        const int i = c0 + threadIdx.x;
        const int v = i < tiles ? sums[i] : 0;
        int total = 0;
        const int ex = block_excl_scan_int(v, warpSums, &total);
        if (i < tiles) sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_tiles(const int* in, int* out, long long n, const int* sums) {
    __shared__ int warpSums[kScanThreads / 32];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanPer;
    int v[kScanPer];
    int t = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        t += v[k];
    }
    int run = sums[blockIdx.x] + block_excl_scan_int(t, warpSums, nullptr);
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

// ---- index passes ----

__global__ void pack_kernel(const int32_t* spo, long long n, int E, unsigned long long* k0, unsigned long long* k1) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long s = (uint32_t)spo[3 * i], p = (uint32_t)spo[3 * i + 1], o = (uint32_t)spo[3 * i + 2];
        k0[i] = (p << (2 * E)) | (s << E) | o;
        k1[i] = (p << (2 * E)) | (o << E) | s;
    }
}

// flag[i] = 1 where key i differs from key i - 1 in the bits from `shift` up
__global__ void change_flags(const unsigned long long* k, long long n, int shift, int* flag) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || (k[i] >> shift) != (k[i - 1] >> shift)) ? 1 : 0;
}

__global__ void compact_kernel(const unsigned long long* k, long long n, const int* flag, const int* pos,
                               unsigned long long* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (flag[i]) out[pos[i]] = k[i];
}

// Edges of one direction from its sorted unique keys: values, keys, row ids,
// and rowKey / rowBeg at every row start.
__global__ void edges_kernel(const unsigned long long* u, long long m, int E, const int* rflag, const int* rpos,
                             int32_t* val, int32_t* src, int32_t* rowId, int32_t* rowKey, int32_t* rowBeg) {
    const unsigned long long mask = (1ull << E) - 1ull;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long x = u[i];
        val[i] = (int32_t)(x & mask);
        src[i] = (int32_t)((x >> E) & mask);
        const int r = rpos[i] + rflag[i] - 1;
        rowId[i] = r;
        if (rflag[i]) {
            rowKey[r] = src[i];
            rowBeg[r] = (int32_t)i;
        }
    }
}

// predEdge[p] = first edge of a predicate >= p; predRow[p] = rows before it.
__global__ void pred_kernel(const unsigned long long* u, long long m, int E, int nPred, const int* rpos, int rows,
                            int32_t* predEdge, int32_t* predRow) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > nPred) return;
    long long lo = 0, hi = m;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if ((long long)(u[mid] >> (2 * E)) < p) lo = mid + 1; else hi = mid;
    }
    predEdge[p] = (int32_t)lo;
    predRow[p] = lo < m ? rpos[lo] : rows;
}

__global__ void src_rank_kernel(const unsigned long long* u, long long m, int E, const int32_t* rowId,
                                const int32_t* predRow, int32_t* srcRank) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
        srcRank[i] = rowId[i] - predRow[(int)(u[i] >> (2 * E))];
}

// The value's row among its predicate's rows of the other direction.
__global__ void val_rank_kernel(const unsigned long long* u, long long m, int E, const int32_t* val,
                                const int32_t* otherRowKey, const int32_t* otherPredRow, int32_t* valRank) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(u[i] >> (2 * E));
        const int b = otherPredRow[p];
        int lo = b, hi = otherPredRow[p + 1];
        const int v = val[i];
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (otherRowKey[mid] < v) lo = mid + 1; else hi = mid;
        }
        valRank[i] = lo - b;
    }
}

__global__ void hash_init_kernel(HashSlot* h, long long cap) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cap; i += (long long)gridDim.x * blockDim.x)
        h[i] = HashSlot{kEmptyTag, 0u, 0u, 0u};
}

// Rows of one direction into the (predicate, direction, key) table, and
// their row-signature bits into the entities' signatures.
__global__ void rows_kernel(const unsigned long long* u, int E, int d, int rows, const int32_t* rowKey,
                            const int32_t* rowBeg, HashSlot* h, uint32_t mask, unsigned long long* entSig) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        const int beg = rowBeg[r], end = rowBeg[r + 1];
        const int p = (int)(u[beg] >> (2 * E));
        const uint32_t tag = (uint32_t)p * 2u + (uint32_t)d;
        const uint32_t key = (uint32_t)rowKey[r];
        uint32_t i = slot_hash(tag, key) & mask;
        for (uint32_t probe = 0; probe <= mask; ++probe) {   // the table has room for every row
            if (atomicCAS(&h[i].tag, kEmptyTag, tag) == kEmptyTag) {
                h[i].key = key;
                h[i].beg = (uint32_t)beg;
                h[i].end = (uint32_t)end;
                break;
            }
            i = (i + 1) & mask;
        }
        atomicOr(&entSig[key], 1ull << sig_bit(p, d));
    }
}

__global__ void val_sig_kernel(const int32_t* val, long long m, const unsigned long long* entSig, uint64_t* valSig) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
        valSig[i] = entSig[val[i]];
}

__global__ void suf_sig_kernel(const int32_t* rowBeg, int rows, const uint64_t* valSig, uint64_t* sufSig) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        uint64_t acc = 0;
        for (int e = rowBeg[r + 1] - 1; e >= rowBeg[r]; --e) sufSig[e] = acc |= valSig[e];
    }
}

int bits_of(int64_t n) {   // bits of the values 0 .. n - 1
    int b = 1;
    while (b < 63 && n > 1 && ((n - 1) >> b) != 0) ++b;
    return b;
}

// A device array of exactly `count` elements, freed with `keep`.
template <class T>
T* dalloc(std::vector<std::unique_ptr<DevBuf>>& keep, size_t count) {
    keep.emplace_back(new DevBuf());
    DevBuf& b = *keep.back();
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    ck(cudaMalloc(&b.p, bytes), "cudaMalloc(index build)");
    b.cap = bytes;
    return static_cast<T*>(b.p);
}

template <class T>
void down(std::vector<T>& v, const T* d, size_t count, cudaStream_t s) {
    v.resize(count);
    if (count) ck(cudaMemcpyAsync(v.data(), d, count * sizeof(T), cudaMemcpyDeviceToHost, s), "D2H index");
}

struct Scanner {
    int* sums = nullptr;
    size_t tilesCap = 0;
    cudaStream_t s;
    // out = exclusive prefix sums of in[0, n); returns the total
    int run(const int* in, int* out, long long n, int* hostTotal, const int* lastIn) {
        const int tiles = (int)((n + kScanTile - 1) / kScanTile);
        if (tiles <= 0) return 0;
        scan_tile_sums<<<tiles, kScanThreads, 0, s>>>(in, n, sums);
        scan_sums<<<1, kScanThreads, 0, s>>>(sums, tiles);
        scan_tiles<<<tiles, kScanThreads, 0, s>>>(in, out, n, sums);
        ck(cudaGetLastError(), "scan");
        int a = 0, b = 0;
        ck(cudaMemcpyAsync(&a, out + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H scan");
        ck(cudaMemcpyAsync(&b, lastIn, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H scan");
        ck(cudaStreamSynchronize(s), "scan");
        *hostTotal = a + b;
        return *hostTotal;
    }
};

}  // namespace

HostIndex build_index_device(const std::vector<int32_t>& spo, int32_t nEnt, int32_t nPred, int32_t hubMinDegree) {
    const long long n = (long long)(spo.size() / 3);
    const int E = bits_of(std::max<int64_t>(nEnt, 2));
    const int Pb = bits_of(std::max<int64_t>(nPred, 2));
    if (n == 0 || 2 * E + Pb > 64 || n > 0x7fffffffLL) return build_index(spo, nEnt, nPred, hubMinDegree);
    const int bits = 2 * E + Pb;
    HostIndex ix;
    ix.nEnt = nEnt;
    ix.nPred = nPred;
    int dev = 0, sms = 1;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    cudaStream_t s = nullptr;
    ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
    } guard{s};
    std::vector<std::unique_ptr<DevBuf>> keep;
    const int grid = sms * 8, threads = 256;

    int32_t* dSpo = dalloc<int32_t>(keep, 3 * (size_t)n);
    ck(cudaMemcpyAsync(dSpo, spo.data(), 3 * (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, s), "H2D triples");
    unsigned long long* key[2] = {dalloc<unsigned long long>(keep, n), dalloc<unsigned long long>(keep, n)};
    unsigned long long* tmp = dalloc<unsigned long long>(keep, n);
    uint32_t* hist = dalloc<uint32_t>(keep, pairs_sort_hist_words((unsigned long long)n));
    unsigned long long* count = dalloc<unsigned long long>(keep, 1);
    const unsigned long long nn = (unsigned long long)n;
    ck(cudaMemcpyAsync(count, &nn, sizeof(nn), cudaMemcpyHostToDevice, s), "H2D count");
    pack_kernel<<<grid, threads, 0, s>>>(dSpo, n, E, key[0], key[1]);
    ck(cudaGetLastError(), "pack");

    Scanner sc;
    sc.s = s;
    sc.sums = dalloc<int>(keep, (size_t)(n + kScanTile - 1) / kScanTile + 1);
    int* flag = dalloc<int>(keep, n);
    int* pos = dalloc<int>(keep, n);
    // per direction: sorted unique keys, their row flags / positions and row ids
    unsigned long long* uniq[2];
    int* rflag[2];
    int* rpos[2];
    int32_t* rowId[2];
    int32_t *dVal[2], *dSrc[2], *dSrcRank[2], *dValRank[2], *dRowKey[2], *dRowBeg[2], *dPredRow[2], *dPredEdge[2];
    int rows[2] = {0, 0};
    int m = 0;
    for (int d = 0; d < 2; ++d) {
        cudaError_t e = cudaSuccess;
        unsigned long long* sorted = radix_sort_keys(key[d], tmp, count, nn, bits, hist, grid, s, &e);
        ck(e, "radix sort");
        change_flags<<<grid, threads, 0, s>>>(sorted, n, 0, flag);
        int md = 0;
        sc.run(flag, pos, n, &md, flag + n - 1);
        if (d == 1 && md != m) throw CudaError("device index: the two directions hold different triples");
        m = md;
        uniq[d] = dalloc<unsigned long long>(keep, m);
        compact_kernel<<<grid, threads, 0, s>>>(sorted, n, flag, pos, uniq[d]);
        rflag[d] = dalloc<int>(keep, m);
        rpos[d] = dalloc<int>(keep, m);
        change_flags<<<grid, threads, 0, s>>>(uniq[d], m, E, rflag[d]);
        sc.run(rflag[d], rpos[d], m, &rows[d], rflag[d] + m - 1);
        dVal[d] = dalloc<int32_t>(keep, m);
        dSrc[d] = dalloc<int32_t>(keep, m);
        rowId[d] = dalloc<int32_t>(keep, m);
        dRowKey[d] = dalloc<int32_t>(keep, rows[d]);
        dRowBeg[d] = dalloc<int32_t>(keep, (size_t)rows[d] + 1);
        edges_kernel<<<grid, threads, 0, s>>>(uniq[d], m, E, rflag[d], rpos[d], dVal[d], dSrc[d], rowId[d], dRowKey[d],
                                               dRowBeg[d]);
        const int32_t mm = m;
        ck(cudaMemcpyAsync(dRowBeg[d] + rows[d], &mm, sizeof(mm), cudaMemcpyHostToDevice, s), "H2D row end");
        dPredRow[d] = dalloc<int32_t>(keep, (size_t)nPred + 1);
        dPredEdge[d] = dalloc<int32_t>(keep, (size_t)nPred + 1);
        pred_kernel<<<(nPred + 1 + 255) / 256, 256, 0, s>>>(uniq[d], m, E, nPred, rpos[d], rows[d], dPredEdge[d],
                                                            dPredRow[d]);
        dSrcRank[d] = dalloc<int32_t>(keep, m);
        src_rank_kernel<<<grid, threads, 0, s>>>(uniq[d], m, E, rowId[d], dPredRow[d], dSrcRank[d]);
        ck(cudaGetLastError(), "index rows");
        ck(cudaStreamSynchronize(s), "index rows");   // `m` and the row count of this direction are on the host
    }
    ix.nTriples = m;
    for (int d = 0; d < 2; ++d) {
        dValRank[d] = dalloc<int32_t>(keep, m);
        val_rank_kernel<<<grid, threads, 0, s>>>(uniq[d], m, E, dVal[d], dRowKey[1 - d], dPredRow[1 - d], dValRank[d]);
    }
    // lookup table at load factor <= 1/2, and row signatures
    size_t cap = 1024;
    while (cap < 2 * ((size_t)rows[0] + (size_t)rows[1])) cap <<= 1;
    ix.hashMask = (uint32_t)(cap - 1);
    HashSlot* dHash = dalloc<HashSlot>(keep, cap);
    hash_init_kernel<<<grid, threads, 0, s>>>(dHash, (long long)cap);
    unsigned long long* entSig = dalloc<unsigned long long>(keep, (size_t)std::max(nEnt, 1));
    ck(cudaMemsetAsync(entSig, 0, (size_t)std::max(nEnt, 1) * 8, s), "memset signatures");
    for (int d = 0; d < 2; ++d)
        rows_kernel<<<grid, threads, 0, s>>>(uniq[d], E, d, rows[d], dRowKey[d], dRowBeg[d], dHash, ix.hashMask, entSig);
    uint64_t* dValSig[2];
    uint64_t* dSufSig[2];
    for (int d = 0; d < 2; ++d) {
        dValSig[d] = dalloc<uint64_t>(keep, m);
        dSufSig[d] = dalloc<uint64_t>(keep, m);
        val_sig_kernel<<<grid, threads, 0, s>>>(dVal[d], m, entSig, dValSig[d]);
        suf_sig_kernel<<<grid, threads, 0, s>>>(dRowBeg[d], rows[d], dValSig[d], dSufSig[d]);
    }
    ck(cudaGetLastError(), "index tables");
    for (int d = 0; d < 2; ++d) {
        down(ix.val[d], dVal[d], m, s);
        down(ix.valRank[d], dValRank[d], m, s);
        down(ix.src[d], dSrc[d], m, s);
        down(ix.srcRank[d], dSrcRank[d], m, s);
        down(ix.rowKey[d], dRowKey[d], rows[d], s);
        down(ix.rowBeg[d], dRowBeg[d], (size_t)rows[d] + 1, s);
        down(ix.predRow[d], dPredRow[d], (size_t)nPred + 1, s);
        down(ix.predEdge[d], dPredEdge[d], (size_t)nPred + 1, s);
        down(ix.valSig[d], dValSig[d], m, s);
        down(ix.sufSig[d], dSufSig[d], m, s);
    }
    down(ix.hash, dHash, cap, s);
    ck(cudaStreamSynchronize(s), "device index");
    build_hub_rows(ix, hubMinDegree);
    return ix;
}

}  // namespace gr
