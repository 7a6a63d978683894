// kernels.cu — the rule-evaluation engine for sm_100a.
//
// One persistent kernel serves both phases of every rule.  Blocks pull
// tasks (a plan and a range of roots) from a device queue.  A task is
// evaluated as a depth-first search over *chunks*: the block keeps, for each
// plan level, a bounded frontier of partial bindings in shared memory and
// always extends the deepest level that still has work.  Each frontier item
// carries the neighbour segment of its next step (looked up once, when the
// item is created).  Extending a level lays the segments of up to B items end
// to end (a block-wide prefix sum) and hands the resulting candidates to
// threads one per slot, so a hub with 50,000 neighbours is spread over the
// whole block instead of serialising one thread.  Frontier memory is bounded
// by construction (each round produces at most `cap` items), so any fan-out
// fits.
//
// Outputs:
//  * kExist: roots with at least one complete grounding (a bit per root);
//    support counts head triples, body size with hS == hO counts hS values.
//  * kPairs: distinct (root, hO) pairs for the body size; each root is one
//    hS value, the hO value is replaced by its rank in the value domain of
//    the atom that binds it, and the pairs go into a per-task bitmap in
//    shared memory (or a per-plan bitmap in global memory for very large
//    domains).  Counting is done on insertion (atomicOr returns the old
//    word), so there is no separate popcount pass, and shared bitmaps never
//    touch HBM.  A partial binding whose (root, hO) pair is already present
//    is dropped, which is the reference's early prune
//    (CPU_01_nonparallel/SupportCounting.cpp:284-290).
//
// Block sizes 128, 256 and 512 are instantiated; shared memory scales with
// the block (16 ints of frontier and 32 bitmap words per thread), so 8, 4 or
// 2 blocks stay resident per SM.
//
// The reference's kernels (GPU_03/gpu_kernels.cuh:34-443) run one thread
// per head triple or per first-atom triple with template-unrolled
// recursion; this engine replaces them as a whole.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>

#include "common.hpp"

namespace gr {

namespace cg = cooperative_groups;

// Counts the global-memory bytes the algorithm requests (the roofline's
// algorithmic bytes).  Compiled out of the timed kernel.
template <bool kOn>
struct Meter {
    unsigned long long bytes = 0;
    __device__ __forceinline__ void add(unsigned long long n) {
        if constexpr (kOn) bytes += n;
    }
};

template <int B>
struct BlockState {
    static constexpr int kWarps = B / 32;
    int task;
    int stop;                       // the block's deadline passed: abandon the task
    unsigned long long deadline;    // global-timer ns (0: none)
    int curItem[kMaxBody + 1];      // a level's position, saved when the search descends below it
    long long curOff[kMaxBody + 1];
    int count[kMaxBody + 1];
    int firstFail;                  // first candidate of a wide round that found the next level full
    unsigned safeLevels;            // bit l: level l takes capacity-sized rounds until exhausted
    int levelOff[kMaxBody + 1];
    long long warpSum[kWarps];
    unsigned long long red[kWarps];
    int exRank[kWarps][kMaxVars];   // per warp: hO-domain ranks of the bound values of a hub item
};

template <int B>
struct Smem {
    DevPlan plan;
    BlockState<B> st;
    int wBeg[B];
    long long wLen[B];
    long long wLoc[B];   // inclusive prefix of wLen within the item's warp
    int pool[Geom::pool_for(B)];   // frontier levels, then the dedup bitmap at plan.bitmapOff
};

template <bool kC>
__device__ __forceinline__ int2 row_lookup(const DevIndex& ix, int pred, int dir, int key, Meter<kC>& mt) {
    if (key < 0) return make_int2(0, 0);
    const uint32_t tag = (uint32_t)pred * 2u + (uint32_t)dir;
    uint32_t i = slot_hash(tag, (uint32_t)key) & ix.hashMask;
    for (uint32_t probe = 0; probe <= ix.hashMask; ++probe) {
        const uint4 s = __ldg(reinterpret_cast<const uint4*>(ix.hash) + i);
        mt.add(16);
        if (s.x == kEmptyTag) break;
        if (s.x == tag && s.y == (uint32_t)key) return make_int2((int)s.z, (int)s.w);
        i = (i + 1) & ix.hashMask;
    }
    return make_int2(0, 0);
}

template <bool kC>
__device__ __forceinline__ bool has_edge(const DevIndex& ix, int pred, int dir, int key, int target, Meter<kC>& mt) {
    const int2 r = row_lookup(ix, pred, dir, key, mt);
    int lo = r.x, hi = r.y;
    const int* v = ix.val[dir];
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        mt.add(4);
        if (__ldg(v + mid) < target) lo = mid + 1; else hi = mid;
    }
    if (lo < r.y) mt.add(4);
    return lo < r.y && __ldg(v + lo) == target;
}

// Whether value x occurs in the sorted values v[beg, beg + len).
template <bool kC>
__device__ __forceinline__ bool seg_has(const int* v, int beg, int len, int x, Meter<kC>& mt) {
    int lo = beg, hi = beg + len;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        mt.add(4);
        if (__ldg(v + mid) < x) lo = mid + 1; else hi = mid;
    }
    return lo < beg + len && __ldg(v + lo) == x;
}

template <bool kC, class Val>
__device__ __forceinline__ bool pass_filters(const DevPlan& P, const DevIndex& ix, int lvl, Meter<kC>& mt, Val val) {
    const int cb = P.chkBeg[lvl], cn = P.chkN[lvl];
    for (int c = 0; c < cn; ++c) {
        const DevCheck& C = P.checks[cb + c];
        const int s = val(C.s), o = val(C.o);
        if (!has_edge(ix, C.pred, C.dir, C.dir == 0 ? s : o, C.dir == 0 ? o : s, mt)) return false;
    }
    const int ub = P.usedBeg[lvl], un = P.usedN[lvl];
    for (int u = 0; u < un; ++u) {
        const DevUsed& U = P.used[ub + u];
        if (val(U.sA) == val(U.sB) && val(U.oA) == val(U.oB)) return false;
    }
    return true;
}

// Edge range of step `s` (0-based) for a binding resolved by `val`.
template <bool kC, class Val>
__device__ __forceinline__ int2 step_segment(const DevPlan& P, const DevIndex& ix, int s, Meter<kC>& mt, Val val) {
    const DevStep& st = P.steps[s];
    if (st.kind == kExpand) return row_lookup(ix, st.pred, st.dir, val(st.keyRef), mt);
    mt.add(8);
    return make_int2(__ldg(ix.predEdge[0] + st.pred), __ldg(ix.predEdge[0] + st.pred + 1));
}

template <int B>
struct Smem;

// Publishes a window's prefix sums with one barrier: every thread stores
// the inclusive sum of x over its warp's threads up to itself (wLoc) and
// every warp its total (warpSum), so item i's block-wide prefix is the
// totals of the warps before i's warp plus wLoc[i] (WinCursor reads it
// that way).  The barrier also ORs `flag` over the block.
template <int B>
__device__ __forceinline__ bool publish_window(long long x, bool flag, Smem<B>& sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    sm.wLoc[threadIdx.x] = x;
    if (lane == 31) sm.st.warpSum[warp] = x;
    return __syncthreads_or(flag) != 0;
}

// The window's candidate total: the warps' totals summed by shuffles.
// (Up to 256 threads the eight totals are added directly; the two forms
// differ only in the registers the kernel needs around them.)
template <int B>
__device__ __forceinline__ long long window_total(const Smem<B>& sm) {
    if constexpr (B <= 256) {
        long long v = 0;
#pragma unroll
        for (int w = 0; w < B / 32; ++w) v += sm.st.warpSum[w];
        return v;
    } else {
        const int lane = threadIdx.x & 31;
        long long v = lane < B / 32 ? sm.st.warpSum[lane] : 0;
#pragma unroll
        for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        return v;
    }
}

// The window item that holds candidate j, for j that never decreases:
// whole warps are stepped over by their totals, then the item is searched
// among its warp's 32 prefixes, starting after the previous item (a hub's
// long segment costs one probe per candidate).
template <int B>
struct WinCursor {
    int item = 0, warp = 0;
    long long base = 0;   // candidates of the warps before `warp`
    __device__ __forceinline__ void seek(const Smem<B>& sm, int nw, long long j) {
        if (base + sm.wLoc[item] > j) return;
        long long end = base + sm.st.warpSum[warp];
        while (end <= j) {
            base = end;
            ++warp;
            end = base + sm.st.warpSum[warp];
        }
        int lo = max(item + 1, warp * 32), hi = min(nw, warp * 32 + 32) - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (base + sm.wLoc[mid] > j) hi = mid; else lo = mid + 1;
        }
        item = lo;
    }
    // index of the item's first candidate
    __device__ __forceinline__ long long first(const Smem<B>& sm) const { return base + sm.wLoc[item] - sm.wLen[item]; }
};

template <int B>
__device__ __forceinline__ unsigned long long block_sum(unsigned long long x, BlockState<B>& st) {
    constexpr int kWarps = B / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 16; d; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
    if (lane == 0) st.red[warp] = x;
    __syncthreads();
    unsigned long long t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kWarps; ++w) t += st.red[w];
    return t;  // valid in thread 0
}

// List capacity of a three-step memo item's exceptions (plus one slot for
// the root's own rank) in the warp's kMaxVars-int buffer.
constexpr int kMemo3List = kMaxVars - 1;

// Three-step suffix memos, for body-size plans hS -> x -> v2 -> v3 -> hO
// (memoSteps == 3) at an item (a, x) whose x is a memoised hub row.  The
// memo of x holds S1 = {h : C(h) > 0} and C(h), the number of paths
// x -> v2 -> v3 -> h with x, v2, v3, h distinct, as a byte that saturates
// at 255.  The item's pairs are the h != a with a path that also avoids a,
// i.e. with C(h) > C_a(h), C_a(h) the paths through a:
//   a = v2 (when a is a neighbour of x): v3 in N2(a) \ {x, a, h}, h in N3(v3);
//   a = v3: v2 in N1(x) with a in N2(v2), v2 not in {x, a, h}, and h in N3(a).
// Only h reached that way (listed, at most kMemo3List by the check in
// classify_item) can have C_a(h) > 0; every other bit of S1 stands.  The
// same check bounds C_a(h) by kMemo3List + 64 < 255 (at most one path per
// v3 in N2(a), and per v2 in a's reverse row), so a saturated count still
// compares exactly.
// memo3_exceptions lists the ranks to clear from S1 and memo_item applies
// them.  Its parts are small leaf functions called one after the other, so
// that few of the caller's registers need to be free for them.
//
// memo3_count (whole warp): 2 * K + [a in N1(x)], K = #{v2 in N1(x) : a in
// N2(v2), v2 not in {x, a}} (lanes split a's reverse row under step 2).
template <bool kC>
__device__ __noinline__ int memo3_count(const DevPlan& P, const DevIndex& ix, const int* par, int lenK, int lane,
                                        Meter<kC>& mt) {
    const int p2 = P.steps[2].pred, d2 = P.steps[2].dir;
    const int* v1 = ix.val[P.steps[1].dir];
    const int a = par[kTupleHead], x = par[kTupleHead + 1];
    const int segBeg = par[lenK], segLen = par[lenK + 1];   // x's row under step 1
    const int2 rInv = row_lookup(ix, p2, 1 - d2, a, mt);
    int k = 0;
    for (int e = rInv.x + lane; e < rInv.y; e += 32) {
        const int u = __ldg(ix.val[1 - d2] + e);
        mt.add(4);
        if (u != x && u != a && seg_has(v1, segBeg, segLen, u, mt)) ++k;
    }
    return 2 * __reduce_add_sync(0xffffffffu, k) + (seg_has(v1, segBeg, segLen, a, mt) ? 1 : 0);
}

// memo3_list (one lane): the ranks of the h a path through a reaches, into
// ex[0..n) (repeats allowed), and a's own rank (h != a) into ex[n] (-1 when
// a is outside hO's domain); returns n.
template <bool kC>
__device__ __noinline__ int memo3_list(const DevPlan& P, const DevIndex& ix, const int* par, int kv, int* ex,
                                       Meter<kC>& mt) {
    const int p2 = P.steps[2].pred, d2 = P.steps[2].dir;
    const int p3 = P.steps[3].pred, d3 = P.steps[3].dir;
    const int a = par[kTupleHead], x = par[kTupleHead + 1];
    int n = 0;
    if (kv & 1) {
        const int2 r2a = row_lookup(ix, p2, d2, a, mt);
        for (int e2 = r2a.x; e2 < r2a.y; ++e2) {
            const int v3 = __ldg(ix.val[d2] + e2);
            if (v3 == x || v3 == a) continue;
            const int2 r3 = row_lookup(ix, p3, d3, v3, mt);
            for (int e3 = r3.x; e3 < r3.y && n < kMemo3List; ++e3) {
                const int h = __ldg(ix.val[d3] + e3);
                if (h != x && h != a && h != v3) ex[n++] = __ldg(ix.valRank[d3] + e3);
            }
        }
    }
    const int2 r3a = row_lookup(ix, p3, d3, a, mt);
    for (int e3 = r3a.x; e3 < r3a.y && n < kMemo3List; ++e3) {
        const int h = __ldg(ix.val[d3] + e3);
        if (h != x && h != a) ex[n++] = __ldg(ix.valRank[d3] + e3);
    }
    const int2 ra = row_lookup(ix, p3, 1 - d3, a, mt);
    ex[n] = ra.y > ra.x ? __ldg(ix.srcRank[1 - d3] + ra.x) : -1;
    return n;
}

// memo3_keep (one lane per listed rank r): whether a path avoiding a still
// reaches r's value h, i.e. C(h) > C_a(h).
template <bool kC>
__device__ __noinline__ bool memo3_keep(const DevPlan& P, const DevIndex& ix, const int* par, int lenK, int r,
                                        int kv, const uint32_t* C, Meter<kC>& mt) {
    const unsigned c = (__ldg(C + (r >> 2)) >> ((r & 3) * 8)) & 0xffu;   // saturates at 255
    mt.add(4);
    const int p3 = P.steps[3].pred, d3 = P.steps[3].dir;
    const int a = par[kTupleHead];
    const int h = __ldg(ix.rowKey[1 - d3] + __ldg(ix.predRow[1 - d3] + p3) + r);
    unsigned ca = 0;
    if (has_edge(ix, p3, d3, a, h, mt)) {   // paths with v3 = a
        const int p2 = P.steps[2].pred, d2 = P.steps[2].dir;
        const bool hIsV2 = has_edge(ix, p2, 1 - d2, a, h, mt) &&
                           seg_has(ix.val[P.steps[1].dir], par[lenK], par[lenK + 1], h, mt);
        ca = (unsigned)((kv >> 1) - (hIsV2 ? 1 : 0));
    }
    if (kv & 1) {   // paths with v2 = a
        const int p2 = P.steps[2].pred, d2 = P.steps[2].dir;
        const int x = par[kTupleHead + 1];
        const int2 r2a = row_lookup(ix, p2, d2, a, mt);
        for (int e2 = r2a.x; e2 < r2a.y && ca < c; ++e2) {
            const int v3 = __ldg(ix.val[d2] + e2);
            if (v3 != x && v3 != a && v3 != h && has_edge(ix, p3, d3, v3, h, mt)) ++ca;
        }
    }
    return c > ca;
}

// The exceptions of an item (whole warp): ex[0..n] holds the ranks to clear
// from S1 of memo slot `slot` (-1: none); returns n + 1.
template <bool kC>
__device__ __forceinline__ int memo3_exceptions(const DevPlan& P, const DevIndex& ix, const int* par, int lenK,
                                                int slot, int words, int* ex, int lane, Meter<kC>& mt) {
    const int kv = memo3_count(P, ix, par, lenK, lane, mt);
    int n = 0;
    if (lane == 0) n = memo3_list(P, ix, par, kv, ex, mt);
    n = __shfl_sync(0xffffffffu, n, 0);
    __syncwarp();
    if (lane < n) {
        const uint32_t* C = P.memoBits + (long long)slot * ((long long)words + ((P.wo + 3) >> 2)) + words;
        if (memo3_keep(P, ix, par, lenK, ex[lane], kv, C, mt)) ex[lane] = -1;   // still reached: keep its bit
    }
    __syncwarp();
    return n + 1;
}

// One level-k item whose first suffix step expands a hub row x with a memo:
// for the plan suffix x -[stA]-> y -[stB]-> hO, the memo holds, over hO's
// rank domain, S1 = {h : at least one y in N1(x) with h in N2(y), h != y}
// and S2 = {h : at least two such y}.  The item's valid hO are S1 minus the
// ranks of its bound values (injectivity on hO) minus, when one bound value
// y0 lies in N1(x) (injectivity on y), the h in N2(y0) that have no witness
// but y0 (those outside S2).  Ranks within a row ascend with the values, so
// each lane merges its own run of words with N2(y0)'s sorted ranks.  The
// whole warp calls this; new pair bits are counted on insertion and
// returned (per lane).  Steps come by value and counts go back as the
// result, so that the caller's loop state never needs an address.
template <bool kC>
__device__ __noinline__ unsigned long long memo_item(const DevPlan& P, const DevIndex& ix, const DevStep stA,
                                                     const DevStep stB, const int* par, int lenK, int slot,
                                                     uint32_t* dst, int words, int* ex, int lane, Meter<kC>& mt,
                                                     bool sharedDst, int nEx3) {
    unsigned long long myNew = 0;
    const bool three = nEx3 > 0;
    const uint32_t* S1 = P.memoBits + (long long)slot * (three ? (long long)words + ((P.wo + 3) >> 2) : 2LL * words);
    int nEx = lenK - kTupleHead;
    unsigned wmask = 0;
    if (three) {
        nEx = nEx3;
    } else {
        const int exDir = 1 - stB.dir;
        const int segBeg = par[lenK], segLen = par[lenK + 1];
        bool isW = false;
        if (lane < nEx) {
            const int u = par[kTupleHead + lane];
            const int2 r = row_lookup(ix, stB.pred, exDir, u, mt);
            ex[lane] = r.y > r.x ? __ldg(ix.srcRank[exDir] + r.x) : -1;
            isW = seg_has(ix.val[stA.dir], segBeg, segLen, u, mt);
        }
        wmask = __ballot_sync(0xffffffffu, isW);
        __syncwarp();
    }
    int e0 = 0, e1 = 0;
    if (wmask) {
        const int2 r = row_lookup(ix, stB.pred, stB.dir, par[kTupleHead + __ffs(wmask) - 1], mt);
        e0 = r.x;
        e1 = r.y;
    }
    const uint32_t* S2 = S1 + words;
    const int* rk = ix.valRank[stB.dir];
    const int per = (words + 31) >> 5;
    const int wb = min(words, lane * per), we = min(words, wb + per);
    int e = e0;
    if (e1 > e0 && wb < we) {
        int lo = e0, hi = e1;
        const int key = wb << 5;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            mt.add(4);
            if (__ldg(rk + mid) < key) lo = mid + 1; else hi = mid;
        }
        e = lo;
    }
    for (int w = wb; w < we; ++w) {
        uint32_t m = __ldg(S1 + w);
        mt.add(4);
        for (int q = 0; q < nEx; ++q)
            if (ex[q] >= 0 && (ex[q] >> 5) == w) m &= ~(1u << (ex[q] & 31));
        if (e < e1) {
            const int lim = (w + 1) << 5;
            uint32_t s2 = 0u;
            bool s2Loaded = false;
            while (e < e1) {
                const int r = __ldg(rk + e);
                if (r >= lim) break;
                if (!s2Loaded) { s2 = __ldg(S2 + w); s2Loaded = true; mt.add(4); }
                if (!((s2 >> (r & 31)) & 1u)) m &= ~(1u << (r & 31));
                ++e;
                mt.add(4);
            }
        }
        if (m) {
            const uint32_t old = atomicOr(dst + w, m);
            if (!sharedDst) mt.add(8);
            myNew += (unsigned long long)__popc(m & ~old);
        }
    }
    __syncwarp();
    return myNew;
}

// kExist counterpart of memo_item: the item's last step expands a hub row x
// with a memo and its only remaining test is the check (h, y) for a bound
// variable h.  A valid y exists iff h has a witness y in N1(x) other than
// the bound values: with no bound value among h's witnesses that is the S1
// bit of h, with one the S2 bit; with more the item is left to enumeration.
// Returns 1 (a grounding exists), 0 (none) or -1 (undecided).
template <bool kC>
__device__ __noinline__ int memo_exists(const DevPlan& P, const DevIndex& ix, const DevStep stA, const int* it,
                                        int lenK, int segBeg, int segLen, int slot, Meter<kC>& mt) {
    const int h = it[P.memoH];
    const int dDom = 1 - P.memoD2;
    const int2 hr = row_lookup(ix, P.memoP2, dDom, h, mt);
    if (hr.y <= hr.x) return 0;   // no y reaches h at all
    const int rank = __ldg(ix.srcRank[dDom] + hr.x);
    int nRem = 0;
    for (int q = kTupleHead; q < lenK; ++q) {
        const int u = it[q];
        if (u == h || !seg_has(ix.val[stA.dir], segBeg, segLen, u, mt)) continue;
        if (!has_edge(ix, P.memoP2, P.memoD2, u, h, mt)) continue;
        if (++nRem >= 2) return -1;
    }
    const uint32_t* S = P.memoBits + ((long long)slot * 2 + nRem) * P.memoWords;
    mt.add(4);
    return (int)((__ldg(S + (rank >> 5)) >> (rank & 31)) & 1u);
}

// Whether an item (a, x) of a three-step memo plan is answered by its memo:
// the paths through a must reach at most kMemo3List values (the warp's
// list) and a's reverse row under the second step must be short.
template <bool kC>
__device__ __forceinline__ bool memo3_fits(const DevPlan& P, const DevIndex& ix, int a, Meter<kC>& mt) {
    const DevStep s2 = P.steps[2], s3 = P.steps[3];
    const int2 rInv = row_lookup(ix, s2.pred, 1 - s2.dir, a, mt);
    if (rInv.y - rInv.x > 64) return false;
    const int2 r2 = row_lookup(ix, s2.pred, s2.dir, a, mt);
    if (r2.y - r2.x > kMemo3List) return false;
    const int2 r3a = row_lookup(ix, s3.pred, s3.dir, a, mt);
    int reach = r3a.y - r3a.x;
    for (int e2 = r2.x; e2 < r2.y && reach <= kMemo3List; ++e2) {
        const int2 r3 = row_lookup(ix, s3.pred, s3.dir, __ldg(ix.val[s2.dir] + e2), mt);
        reach += r3.y - r3.x;
    }
    return reach <= kMemo3List;
}

// Items of a round that may skip enumeration, kept out of line so that the
// main loop's registers stay free.  kind 1: a leaf item whose segment is a
// whole hub row (returns the hub index); 2: an item at the memo level whose
// segment is a memoised hub row with at most one bound value among its
// neighbours (returns the memo slot); 3: a kExist leaf item decided by the
// existence memo (returns -3, its found bit set; -4 when the bit is new and
// the task counts on insertion).  -1: enumerate as usual.
template <bool kC>
__device__ __noinline__ int classify_item(const DevPlan& P, const DevIndex& ix, const DevStep stp, const int* it,
                                          int lenK, int kind, int segBeg, int segLen, uint32_t* fb, bool heavy,
                                          Meter<kC>& mt) {
    const int row = __ldg(ix.predRow[stp.dir] + stp.pred) + __ldg(ix.srcRank[stp.dir] + segBeg);
    const int h = __ldg(ix.hubOf[stp.dir] + row);
    mt.add(12);
    if (h < 0 || __ldg(ix.rowBeg[stp.dir] + row) != segBeg || __ldg(ix.rowBeg[stp.dir] + row + 1) - segBeg != segLen)
        return -1;
    if (kind == 1) return h;
    const int slot = __ldg(P.memoTab + h);
    if (slot < 0) return -1;
    if (kind == 2) {
        if (P.memoSteps == 3) return memo3_fits(P, ix, it[kTupleHead], mt) ? slot : -1;
        // bound values that are also first-step neighbours are witnesses the
        // memo must not count; one is corrected exactly, more enumerate
        int nR = 0;
        for (int q = kTupleHead; q < lenK && nR < 2; ++q)
            nR += seg_has(ix.val[stp.dir], segBeg, segLen, it[q], mt) ? 1 : 0;
        return nR <= 1 ? slot : -1;
    }
    const int res = memo_exists(P, ix, stp, it, lenK, segBeg, segLen, slot, mt);
    if (res < 0) return -1;
    if (res == 1) {
        const int root = it[0];
        const uint32_t mask = 1u << (root & 31);
        const uint32_t old = atomicOr(&fb[root >> 5], mask);
        if (heavy) {
            mt.add(8);
            if (!(old & mask)) return -4;
        }
    }
    return -3;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Sort mode: appends the pair key of (row, rank) to the plan's key buffer.
// The threads that emit together take consecutive slots with one atomic; the
// cursor keeps counting past the capacity, so the host learns the exact
// number of keys when they did not fit (and runs again with that size).
__device__ __forceinline__ void emit_pair(const DevPlan& P, long long row, int rank) {
    const unsigned long long key = P.keyBase | ((unsigned long long)row << P.rankBits) | (unsigned)rank;
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(P.keyCursor, (unsigned long long)g.size());
    base = g.shfl(base, 0);
    const unsigned long long slot = base + g.thread_rank();
    if (slot < P.keyCap) P.pairKeys[slot] = key;
}

// Claims a leaf hub item of (root, hub) with middle value `mid` in the
// task's table (see kHubSeen); false when two other middle values are
// claimed already.
__device__ __forceinline__ bool hub_claim(unsigned long long* seen, int root, int hub, int mid) {
    const unsigned long long key = ((unsigned long long)root << 20) | (unsigned long long)hub;   // 30 bits
    unsigned long long* w = seen + (((uint32_t)key * 0x9E3779B1u) >> (32 - kHubSeenBits));
    const unsigned long long m = (uint32_t)mid;
    unsigned long long old = __ldcg(w);
    for (int t = 0; t < 8; ++t) {
        unsigned long long want;
        const unsigned state = (unsigned)(old >> 32) & 3u;
        if ((old >> 34) == key && state != 0u) {
            if (state >= 2u) return false;
            if ((old & 0xffffffffull) == m) return true;   // the first value again
            want = (old & ~(3ull << 32)) | (2ull << 32);
        } else {
            want = (key << 34) | (1ull << 32) | m;   // displaces another pair: it may repeat items, never lose one
        }
        const unsigned long long prev = atomicCAS(w, old, want);
        if (prev == old) return true;
        old = prev;
    }
    return true;
}

// The claims of a round's leaf hub items [0, cut) (items at `items`,
// `stride` ints apart): items that add nothing get wBeg -1.  Out of line,
// so that the caller's loop keeps its registers.
__device__ __noinline__ void hub_claims(unsigned long long* seen, const int* items, int stride, int cut, int midAt,
                                        int* wBeg, int nThreads) {
    for (int i = threadIdx.x; i < cut; i += nThreads) {
        const int wb = wBeg[i];
        if (wb <= -2) {
            const int* it = items + i * stride;
            if (!hub_claim(seen, it[0], -2 - wb, it[midAt])) wBeg[i] = -1;
        }
    }
}

// Fused support (plans with supN > 0): the head triples (hS, supPred[j],
// b), b != hS, of rule j whose pair (hS, b) is set in the plan's row of
// root i (rows at bm + i * rowWords for the roots rootBeg + i, i < G).
// Warps take the roots, lanes a root's head triples; returns this lane's
// count.  Out of line and small: it runs once per task, after the search.
// `part` of `nParts` takes every nParts-th group of 32 head triples.
template <bool kC>
__device__ __noinline__ unsigned long long fused_support(const DevPlan& P, const DevIndex& ix, int j, int rootBeg,
                                                         int G, const uint32_t* bm, int warp, int nWarps, int lane,
                                                         int part, int nParts, Meter<kC>& mt) {
    unsigned long long n = 0;
    const int hp = P.supPred[j], dp = P.supDomPred, dd = P.supDomDir;
    for (int i = warp; i < G; i += nWarps) {
        const int a = __ldg(ix.rowKey[P.rootDir] + rootBeg + i);
        mt.add(4);
        const int2 hr = row_lookup(ix, hp, 0, a, mt);
        const uint32_t* row = bm + (long long)i * P.rowWords;
        for (int e = hr.x + 32 * part + lane; e < hr.y; e += 32 * nParts) {
            const int b = __ldg(ix.val[0] + e);
            mt.add(4);
            if (b == a) continue;
            const int2 br = row_lookup(ix, dp, dd, b, mt);
            if (br.y <= br.x) continue;   // b never binds hO
            const int rank = __ldg(ix.srcRank[dd] + br.x);
            mt.add(8);
            if ((row[rank >> 5] >> (rank & 31)) & 1u) ++n;
        }
    }
    return n;
}

template <int B, bool kC, bool kD>
__device__ __forceinline__ void run_task(Smem<B>& sm, const DevIndex& ix, const DevTask& task,
                                         unsigned long long* results, int* status, Meter<kC>& mt) {
    constexpr int kLeafChunk = 16 * B;
    // candidates of a non-leaf round whose next step has a signature test
    // (most candidates die on it): more than the next level's capacity, so
    // a round may find that level full (see `wide` below)
    constexpr int kWideChunk = 8 * B;
    // candidates per thread per group (1, 2 and 4 measured on c3: 44.96,
    // 45.22 and 46.92 ms per launch; 8 makes compilation impractical)
    constexpr int kU = 1;
    const DevPlan& P = sm.plan;
    BlockState<B>& S = sm.st;
    const int tid = threadIdx.x;
    const int G = task.end - task.beg;
    const bool pairs = P.mode == kPairs;
    // Dedup targets.  A split heavy root (one root, G == 1) uses its global
    // row for both the pair bits and the found bit; counting happens on
    // insertion so that the slices of one root count each result once.
    const bool heavy = task.gRow >= 0;
    // Sort mode appends pair keys instead of setting bits (no bitmap at
    // all); block rows keep the task's rows in the block's own region of a
    // global buffer instead of one row per root of the phase.
    const bool sortMode = pairs && P.pairKeys != nullptr;
    const bool blockRows = pairs && !heavy && !sortMode && P.gBlockWords > 0;
    const bool shared = !heavy && !(pairs && (P.gBitmap || sortMode));
    uint32_t* sbits = reinterpret_cast<uint32_t*>(sm.pool + P.bitmapOff);
    int* const items = sm.pool;
    uint32_t* bm = heavy ? (P.gHeavy ? P.gHeavy + (long long)task.gRow * P.rowWords : nullptr)
                         : (shared ? sbits : (blockRows ? P.gBitmap + (long long)blockIdx.x * P.gBlockWords : P.gBitmap));
    uint32_t* fb = heavy ? bm : sbits;   // kExist found bits
    const long long rowBase = (heavy || shared || blockRows) ? 0 : (long long)task.beg - P.gRowBase;
    const long long keyRow0 = (long long)task.beg - P.gRowBase;   // sort mode: key row of the task's root 0

    // clear the task's shared dedup bits
    // pair rows are word-aligned: row r occupies words [r * rowWords, (r + 1) * rowWords)
    const long long rowBits = (long long)P.rowWords << 5;
    const int nWords = heavy ? 0 : (shared ? (int)(pairs ? (long long)G * P.rowWords : ((G + 31) >> 5))
                                           : (pairs ? 0 : ((G + 31) >> 5)));
    for (int i = tid; i < nWords; i += B) sbits[i] = 0u;
    if (blockRows && (long long)G * P.rowWords > P.gBlockWords) {   // the task builder keeps tasks this small
        if (tid == 0) atomicOr(status, 32);
        return;
    }
    if (blockRows) {
        // the region is 16-byte aligned and a whole number of uint4 long
        uint4* b4 = reinterpret_cast<uint4*>(bm);
        const long long n4 = ((long long)G * P.rowWords + 3) >> 2;
        for (long long i = tid; i < n4; i += B) b4[i] = make_uint4(0u, 0u, 0u, 0u);
        if (tid == 0) mt.add(16 * (unsigned long long)n4);
    }
    // leaf hub items: the task's claim table (roots and hubs must fit its fields)
    const bool claims = P.hubSeen && G <= 1024 && ix.nHub <= (1 << 20);
    if (claims)
        for (int i = tid; i < kHubSeen; i += B) P.hubSeen[(long long)blockIdx.x * kHubSeen + i] = 0ull;
    if (tid == 0) {
        S.firstFail = INT_MAX;
        S.safeLevels = 0;
        int off = 0;
        for (int l = 0; l <= kMaxBody; ++l) {
            S.curItem[l] = 0;
            S.curOff[l] = 0;
            S.count[l] = 0;
            S.levelOff[l] = off;
            if (l < P.m) off += P.cap * (P.tupleLen[l] + 2);
            else if (P.m == 0 && l == 0) off += P.cap * P.tupleLen[0];
        }
    }
    __syncthreads();

    // ---- level 0: roots (tuple, then the segment of step 1) ----
    {
        const int len0 = P.tupleLen[0];
        const int stride0 = P.m > 0 ? len0 + 2 : len0;
        // as for deeper items: a root whose segment has no value able to
        // take step 2 (keyed on that value) is not stored
        const bool lookTest0 = P.m >= 2 && P.steps[0].kind == kExpand && P.steps[1].kind == kExpand &&
                               P.steps[1].keyRef == len0;
        const int lookBit0 = lookTest0 ? sig_bit(P.steps[1].pred, P.steps[1].dir) : 0;
        const uint32_t* lookWords0 =
            reinterpret_cast<const uint32_t*>(ix.sufSig[lookTest0 ? P.steps[0].dir : 0]) + (lookBit0 >> 5);
        for (int i = tid; i < G; i += B) {
            const int r = task.beg + i;
            int tv[kTupleHead + 2];
            tv[0] = i;
            tv[1] = 0;
            int nv = kTupleHead;
            bool ok = true;
            if (P.rootKind == kRootRows) {
                tv[nv++] = __ldg(ix.rowKey[P.rootDir] + r);
                mt.add(4);
            } else {
                mt.add(8);
                const int key = __ldg(ix.src[P.rootDir] + r);
                const int v = __ldg(ix.val[P.rootDir] + r);
                if (P.rootKeyEqVal && key != v) ok = false;
                if (P.rootKeyNeVal && key == v) ok = false;
                if (P.rootValConst < 0 && v != P.consts[-1 - P.rootValConst]) ok = false;
                if (P.rootAppendKey) tv[nv++] = key;
                if (P.rootAppendVal) tv[nv++] = v;
            }
            if (ok && nv != len0) { ok = false; atomicOr(status, 2); }
            auto val0 = [&](TermRef ref) -> int { return ref < 0 ? P.consts[-1 - ref] : tv[ref < nv ? ref : 0]; };
            if (ok) ok = pass_filters(P, ix, 0, mt, val0);
            int2 seg = make_int2(0, 0);
            if (ok && P.m > 0) {
                seg = step_segment(P, ix, 0, mt, val0);
                if (heavy) {
                    const int b0 = seg.x;
                    seg.x = min(seg.y, b0 + task.sub0);
                    seg.y = min(seg.y, b0 + task.sub1);
                }
                ok = seg.y > seg.x;
                if (ok && lookTest0) {
                    mt.add(4);
                    ok = (__ldg(lookWords0 + 2 * (long long)seg.x) >> (lookBit0 & 31)) & 1u;
                }
            }
            if (ok) {
                const int slot = atomicAdd(&S.count[0], 1);
                if (slot < P.cap) {
                    int* dst = items + S.levelOff[0] + slot * stride0;
                    for (int q = 0; q < len0; ++q) dst[q] = tv[q];
                    if (P.m > 0) { dst[len0] = seg.x; dst[len0 + 1] = seg.y - seg.x; }
                } else {
                    atomicOr(status, 4);
                }
            }
        }
    }
    __syncthreads();

    unsigned long long myNew = 0;
    if (P.m == 0) {
        for (int i = tid; i < S.count[0] && i < P.cap; i += B) {
            const int root = items[S.levelOff[0] + i * P.tupleLen[0]];
            const uint32_t old = atomicOr(&fb[root >> 5], 1u << (root & 31));
            if (heavy && !(old & (1u << (root & 31)))) myNew++;
        }
    } else {
        // The search position (level k, first window item w0, candidates of
        // that item consumed already) is kept alike in every thread's
        // registers; a level's position goes to shared memory only when the
        // search descends below it.  A round takes two barriers: one
        // publishes the window's prefix sums, one closes the round.  Reads
        // of the shared counters that a later step may reset can only see
        // the reset when the decision they feed is the same either way.
        int k = 0, w0 = 0;
        long long off = 0;
        for (;;) {
            const int cnt = min(S.count[k], P.cap);
            if (w0 >= cnt) {
                if (k == 0) break;
                // nobody reads level k's bit again before it is re-entered
                if (tid == 0) S.safeLevels &= ~(1u << k);
                --k;
                w0 = S.curItem[k];
                off = S.curOff[k];
                continue;
            }
            const int nw = min(B, cnt - w0);
            const int lenK = P.tupleLen[k];
            const int strideK = lenK + 2;
            const int* baseK = items + S.levelOff[k];
            const DevStep stp = P.steps[k];   // uniform for the round: keep it in registers
            const bool leaf = (k + 1 == P.m);
            const bool hasFilters = (P.chkN[k + 1] | P.usedN[k + 1]) != 0;
            const bool itemHasRank = pairs && P.hoLevel >= 1 && k >= P.hoLevel;
            // Hub path: when the leaf binds hO and tests nothing but
            // injectivity, an item whose segment is a whole hub row is
            // counted by OR-ing the row's rank bitmap into its pair row (32
            // candidates per word) instead of candidate by candidate.
            const bool hubPath = leaf && pairs && !sortMode && stp.hoWhich != 0 && stp.kind == kExpand &&
                                 stp.nNew == 1 && !hasFilters && ix.nHub > 0 && !(heavy && k == 0);
            // Memo path: the plan ends in two expand steps x -> y -> hO with
            // nothing but injectivity to test; an item whose first segment
            // is a hub row with a suffix memo is counted from the memo's
            // "one witness y" / "two witnesses y" bitmaps (see below).
            const bool memoPath = !leaf && pairs && !sortMode && P.memoTab != nullptr && k + 1 == P.memoLevel;
            const bool existMemo = leaf && !pairs && P.memoTab != nullptr && k + 1 == P.memoLevel &&
                                   !(heavy && k == 0);
            bool isHub = false;   // item marked for the hub or memo pass

            // window: the stored neighbour segment of each item
            int myBeg = 0;
            long long myLen = 0;
            if (tid < nw) {
                const int* it = baseK + (w0 + tid) * strideK;
                bool pruned = false;
                if (!pairs) {
                    pruned = (fb[it[0] >> 5] >> (it[0] & 31)) & 1u;
                    if (heavy) mt.add(4);
                } else if (itemHasRank && !sortMode) {
                    const long long bit = (rowBase + it[0]) * rowBits + it[1];
                    pruned = (bm[bit >> 5] >> (bit & 31)) & 1u;
                    if (!shared) mt.add(4);
                }
                if (!pruned) {
                    myBeg = it[lenK];
                    myLen = it[lenK + 1];
                    const int pathKind = hubPath ? 1 : (memoPath ? 2 : (existMemo ? 3 : 0));
                    if (pathKind && myLen > 0 && !(tid == 0 && off != 0)) {
                        int code = classify_item(P, ix, stp, it, lenK, pathKind, myBeg, (int)myLen, fb, heavy, mt);
                        if (code == -4) {
                            myNew += 1;          // a new found bit of a split root
                            code = -3;
                        }
                        if (code >= 0) {
                            isHub = true;
                            myBeg = -2 - code;   // marks the item for the hub or memo pass; no candidates
                            myLen = 0;
                        } else if (code == -3) {
                            myLen = 0;           // decided by the existence memo
                        }
                    }
                    if (tid == 0 && !isHub) {
                        myBeg += (int)off;
                        myLen = myLen > off ? myLen - off : 0;
                    }
                }
            }
            sm.wBeg[tid] = myBeg;
            sm.wLen[tid] = myLen;
            if (tid == 0 && !leaf) S.count[k + 1] = 0;
            const bool anyHub = publish_window<B>(myLen, isHub, sm) && (hubPath || memoPath);
            const long long total = window_total<B>(sm);
            // When the next step expands from the value this step binds,
            // that value's row signature (stored beside it) drops most
            // candidates whose next row is absent before any lookup.
            const bool sigTest = !leaf && stp.kind == kExpand && P.steps[k + 1].kind == kExpand &&
                                 P.steps[k + 1].keyRef == lenK;
            // Wide round: up to kWideChunk candidates although each survivor
            // takes a slot of the next level.  A survivor that finds it full
            // records its candidate index, and the level resumes from the
            // first such candidate; items made from later candidates are made
            // again then, which changes no count (every dedup structure is a
            // set counted on insertion).  A level that overflowed takes
            // capacity-sized rounds, which cannot overflow, until it is
            // exhausted, so the search always advances.  Sort mode keeps
            // capacity-sized rounds: its key count must not depend on how
            // the threads raced (a launch is staged again with that count).
            const bool wide = sigTest && !sortMode && !((S.safeLevels >> k) & 1u);
            const long long take = min(total, (long long)(leaf ? kLeafChunk : (wide ? kWideChunk : P.cap)));
            const int lenN = leaf ? 0 : P.tupleLen[k + 1];
            const int strideN = lenN + 2;
            int* baseN = leaf ? nullptr : items + S.levelOff[k + 1];

            // A new item of level k + 1 whose segment holds no value with a
            // row under step k + 2 (keyed on that value) is not stored.
            const bool lookTest = k + 2 < P.m && P.steps[k + 1].kind == kExpand && P.steps[k + 2].kind == kExpand &&
                                  P.steps[k + 2].keyRef == P.tupleLen[k + 1];
            const int lookBit = lookTest ? sig_bit(P.steps[k + 2].pred, P.steps[k + 2].dir) : 0;
            const uint32_t* lookWords =
                reinterpret_cast<const uint32_t*>(ix.sufSig[lookTest ? P.steps[k + 1].dir : 0]) + (lookBit >> 5);

            // One candidate: its parent item `lo`, edge `e`, new value(s)
            // n0/n1 and (when this step binds hO) the loaded rank.
            auto eval = [&](int lo, int e, int n0, int n1, int rankLoaded, int j) {
                const int* par = baseK + (w0 + lo) * strideK;
                const int root = par[0];
                if (!pairs && ((fb[root >> 5] >> (root & 31)) & 1u)) return;
                if (stp.kind == kScan && (stp.sameVar ? (n0 != n1) : (n0 == n1))) return;
                for (int q = kTupleHead; q < lenK; ++q) {
                    const int x = par[q];
                    if (x == n0 || (stp.nNew == 2 && x == n1)) return;
                }
                auto valN = [&](TermRef ref) -> int {
                    if (ref < 0) return P.consts[-1 - ref];
                    if (ref < lenK) return par[ref];
                    return ref == lenK ? n0 : n1;
                };
                if (hasFilters && !pass_filters(P, ix, k + 1, mt, valN)) return;
                int rank = par[1];
                if (pairs && stp.hoWhich) {
                    rank = rankLoaded;
                    if (!leaf && !sortMode) {
                        const long long bit = (rowBase + root) * rowBits + rank;
                        if (!shared) mt.add(4);
                        if ((bm[bit >> 5] >> (bit & 31)) & 1u) return;
                    }
                }
                if (leaf) {
                    if (!pairs) {
                        const uint32_t mask = 1u << (root & 31);
                        const uint32_t old = atomicOr(&fb[root >> 5], mask);
                        if (heavy) { mt.add(8); myNew += (old & mask) ? 0ull : 1ull; }
                    } else if (sortMode) {
                        emit_pair(P, keyRow0 + root, rank);
                        mt.add(8);
                    } else {
                        const long long bit = (rowBase + root) * rowBits + rank;
                        const uint32_t mask = 1u << (bit & 31);
                        const uint32_t old = atomicOr(&bm[bit >> 5], mask);
                        if (!shared) mt.add(8);
                        myNew += (old & mask) ? 0ull : 1ull;
                    }
                } else {
                    const int2 seg = step_segment(P, ix, k + 1, mt, valN);
                    if (seg.y <= seg.x) return;
                    if (lookTest) {
                        mt.add(4);
                        if (!((__ldg(lookWords + 2 * (long long)seg.x) >> (lookBit & 31)) & 1u)) return;
                    }
                    const int slot = atomicAdd(&S.count[k + 1], 1);
                    if (slot >= P.cap) {
                        if (wide) atomicMin(&S.firstFail, j);
                        else atomicOr(status, 8);   // a capacity-sized round cannot fill the level
                        return;
                    }
                    int* dst = baseN + slot * strideN;
                    dst[0] = root;
                    dst[1] = rank;
                    for (int q = kTupleHead; q < lenK; ++q) dst[q] = par[q];
                    dst[lenK] = n0;
                    if (stp.nNew == 2) dst[lenK + 1] = n1;
                    dst[lenN] = seg.x;
                    dst[lenN + 1] = seg.y - seg.x;
                }
            };

            // Candidates j = tid, tid + B, ... in groups of kU per thread: all
            // group members are located first, then their loads are issued
            // together, then they are evaluated.
            const int* vbase = stp.kind == kExpand ? ix.val[stp.dir] : ix.src[0];
            const int* rbase = stp.kind == kExpand ? ix.valRank[stp.dir]
                                                   : (stp.hoWhich == 1 ? ix.srcRank[0] : ix.valRank[0]);
            const bool wantRank = pairs && stp.hoWhich;
            const int sigBit = sig_bit(P.steps[k + 1 < P.m ? k + 1 : k].pred, P.steps[k + 1 < P.m ? k + 1 : k].dir);
            const uint32_t* sigWords = reinterpret_cast<const uint32_t*>(ix.valSig[stp.dir]) + (sigBit >> 5);
            WinCursor<B> cur;
            for (long long jb = tid; jb < take; jb += (long long)B * kU) {
                int lo_[kU], e_[kU], n0_[kU], n1_[kU], rk_[kU];
                uint32_t sw_[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const long long j = jb + (long long)u * B;
                    lo_[u] = -1;
                    e_[u] = 0;
                    if (j < take) {
                        cur.seek(sm, nw, j);
                        lo_[u] = cur.item;
                        e_[u] = sm.wBeg[cur.item] + (int)(j - cur.first(sm));
                    }
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    n0_[u] = n1_[u] = rk_[u] = 0;
                    sw_[u] = ~0u;
                    if (lo_[u] < 0) continue;
                    if (sigTest) { sw_[u] = __ldg(sigWords + 2 * (long long)e_[u]); mt.add(4); }
                    n0_[u] = __ldg(vbase + e_[u]);
                    if (stp.kind == kScan) { n1_[u] = __ldg(ix.val[0] + e_[u]); mt.add(8); } else mt.add(4);
                    if (wantRank) { rk_[u] = __ldg(rbase + e_[u]); mt.add(4); }
                }
#pragma unroll
                for (int u = 0; u < kU; ++u)
                    if (lo_[u] >= 0 && ((sw_[u] >> (sigBit & 31)) & 1u))
                        eval(lo_[u], e_[u], n0_[u], n1_[u], rk_[u], (int)(jb + (long long)u * B));
            }
            // where the next round at this level starts: the item holding
            // candidate `take` (items before it are consumed), and how much
            // of it is (computed here, not before the candidates, so that it
            // holds no registers across them)
            int cut = nw;
            long long cutOff = 0;
            {
                if (take < window_total<B>(sm)) {
                    WinCursor<B> c;
                    c.seek(sm, nw, take);
                    cut = c.item;
                    cutOff = take - c.first(sm) + (c.item == 0 ? off : 0);
                }
            }
            if (anyHub && leaf && claims) {
                // leaf hub items of a (root, hub) after two middle values add nothing
                hub_claims(P.hubSeen + (long long)blockIdx.x * kHubSeen, baseK + w0 * strideK, strideK, cut,
                           stp.keyRef == kTupleHead + 1 ? kTupleHead + 2 : kTupleHead + 1, sm.wBeg, B);
                __syncthreads();
            }
            if (anyHub) {
                // hub items of the consumed part of the window: [0, cut)
                const int lane = tid & 31, warp = tid >> 5;
                constexpr int kWarps = B / 32;
                const int words = P.rowWords;
                // memo items and domains up to 1,024 words: one warp per item
                // (a round's hub items in parallel); larger rows: the whole
                // block on each item in turn
                const bool perWarp = !leaf || words <= 1024;
                const int nEx = lenK - kTupleHead;
                const int exDir = 1 - stp.dir;
                int ordinal = 0;
                for (int base = 0; base < cut; base += 32) {
                    const int i = base + lane;
                    unsigned bal = __ballot_sync(0xffffffffu, i < cut && sm.wBeg[i] <= -2);
                    while (bal) {
                        const int item = base + __ffs(bal) - 1;
                        bal &= bal - 1;
                        const int mine = ordinal++;
                        if (perWarp && mine % kWarps != warp) continue;
                        const int* par = baseK + (w0 + item) * strideK;
                        if (!leaf) {
                            const int slot = -2 - sm.wBeg[item];
                            const int nEx3 = P.memoSteps == 3
                                ? memo3_exceptions(P, ix, par, lenK, slot, words, S.exRank[warp], lane, mt) : 0;
                            myNew += memo_item(P, ix, stp, P.steps[k + 1], par, lenK, slot,
                                               bm + (rowBase + par[0]) * (long long)words, words, S.exRank[warp],
                                               lane, mt, shared, nEx3);
                            continue;
                        }
                        // hO must differ from every bound value: their ranks in hO's domain
                        int* ex = S.exRank[warp];
                        if (lane < nEx) {
                            const int2 r = row_lookup(ix, stp.pred, exDir, par[kTupleHead + lane], mt);
                            ex[lane] = r.y > r.x ? __ldg(ix.srcRank[exDir] + r.x) : -1;
                        }
                        __syncwarp();
                        const int h = -2 - sm.wBeg[item];
                        const uint32_t* hb = ix.hubBits + __ldg(ix.hubOff + h);
                        uint32_t* dst = bm + (rowBase + par[0]) * (long long)words;
                        const int w0b = perWarp ? lane : tid;
                        const int step = perWarp ? 32 : B;
                        for (int w = w0b; w < words; w += step) {
                            uint32_t m = __ldg(hb + w);
                            for (int q = 0; q < nEx; ++q)
                                if ((ex[q] >> 5) == w && ex[q] >= 0) m &= ~(1u << (ex[q] & 31));
                            mt.add(4);
                            if (m) {
                                const uint32_t old = atomicOr(dst + w, m);
                                if (!shared) mt.add(8);
                                myNew += (unsigned long long)__popc(m & ~old);
                            }
                        }
                        __syncwarp();
                    }
                }
            }
            if constexpr (kD) {
                if (tid == 0 && global_ns() > S.deadline) S.stop = 1;
            }
            __syncthreads();
            if constexpr (kD) {
                if (S.stop) break;   // set before the barrier, read by every thread after it: all leave together
            }
            if (wide) {
                const int ff = S.firstFail;   // final after the barrier
                if (ff < take) {
                    WinCursor<B> c;
                    c.seek(sm, nw, ff);
                    cut = c.item;
                    cutOff = ff - c.first(sm) + (c.item == 0 ? off : 0);
                    if (tid == 0) S.safeLevels |= 1u << k;
                    // every thread has read the window and firstFail: the
                    // next round may rewrite them
                    __syncthreads();
                    if (tid == 0) S.firstFail = INT_MAX;
                }
            }
            const int nextItem = w0 + cut;
            if (!leaf && S.count[k + 1] > 0) {
                if (tid == 0) {
                    S.curItem[k] = nextItem;
                    S.curOff[k] = cutOff;
                }
                ++k;
                w0 = 0;
                off = 0;
            } else {
                w0 = nextItem;
                off = cutOff;
            }
        }
    }
    __syncthreads();

    // ---- fused support: every pair row of the task is complete here (a
    // split heavy root's row only after the launch: support_rows_kernel) ----
    if (P.supN > 0 && !heavy) {
        const int lane = tid & 31;
        for (int j = 0; j < P.supN; ++j) {
            unsigned long long n = fused_support(P, ix, j, task.beg, G, bm, tid >> 5, B / 32, lane, 0, 1, mt);
#pragma unroll
            for (int d = 16; d; d >>= 1) n += __shfl_down_sync(0xffffffffu, n, d);
            if (lane == 0 && n) atomicAdd(results + P.supSlot[j], n);
        }
    }

    // ---- result ----
    unsigned long long mine = 0;
    if (!pairs && !heavy) {
        for (int i = tid; i < ((G + 31) >> 5); i += B) mine += __popc(sbits[i]);
    } else {
        mine = myNew;
    }
    const unsigned long long tot = block_sum<B>(mine, S);
    if (tid == 0 && tot) atomicAdd(results + P.resultSlot, tot);
    if (tid == 0) mt.add(8);
}

// kI: 0 plain; 1 records each task's start and end time; 2 also counts
// the algorithmic bytes; 3 records task times under a deadline (served
// launches: past prof.budgetNs from the block's start the block abandons
// its task at the end of a frontier round, skips the rest, and marks the
// plans that lost a task in prof.incomplete).
template <int B, int kI>
__global__ void __launch_bounds__(B, 1024 / B)
engine_kernel(const __grid_constant__ DevIndex ix, const DevPlan* __restrict__ plans, const DevTask* __restrict__ tasks,
              int nTasks, int* taskCounter, unsigned long long* results, int* status, EngineProfile prof) {
    constexpr bool kC = kI == 2;
    constexpr bool kD = kI == 3;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<B>& sm = *reinterpret_cast<Smem<B>*>(smem_raw);
    Meter<kC> mt;
    if (prof.span && threadIdx.x == 0) atomicMax(prof.span, ~global_ns());
    if constexpr (kD) {
        if (threadIdx.x == 0) sm.st.deadline = global_ns() + prof.budgetNs;
    }
    for (;;) {
        if (threadIdx.x == 0) {
            sm.st.task = atomicAdd(taskCounter, 1);
            if constexpr (kD) sm.st.stop = global_ns() > sm.st.deadline ? 1 : 0;
        }
        __syncthreads();
        const int t = sm.st.task;
        if (t >= nTasks) break;
        const DevTask task = tasks[t];
        if constexpr (kD) {
            if (sm.st.stop) {   // past the deadline: the task is skipped and its plan marked
                if (threadIdx.x == 0) atomicOr(prof.incomplete + task.plan, 1);
                __syncthreads();
                continue;
            }
        }
        unsigned long long t0 = 0;
        if constexpr (kI >= 1) {
            if (threadIdx.x == 0) {
                mt.add(sizeof(DevTask) + sizeof(DevPlan) + 8);
                t0 = global_ns();
            }
        }
        const int* src = reinterpret_cast<const int*>(plans + task.plan);
        int* dst = reinterpret_cast<int*>(&sm.plan);
        for (int i = threadIdx.x; i < (int)(sizeof(DevPlan) / 4); i += B) dst[i] = src[i];
        __syncthreads();
        run_task<B, kC, kD>(sm, ix, task, results, status, mt);
        __syncthreads();
        if constexpr (kD) {
            if (threadIdx.x == 0 && sm.st.stop) atomicOr(prof.incomplete + task.plan, 1);
        }
        if constexpr (kI >= 1) {
            if (threadIdx.x == 0 && prof.taskNs) {
                prof.taskNs[2 * t] = t0;
                prof.taskNs[2 * t + 1] = global_ns();
            }
        }
    }
    if constexpr (kC) {
        unsigned long long b = mt.bytes;
        for (int d = 16; d; d >>= 1) b += __shfl_down_sync(0xffffffffu, b, d);
        if ((threadIdx.x & 31) == 0 && b && prof.bytes) atomicAdd(prof.bytes, b);
    }
    if (prof.span && threadIdx.x == 0) atomicMax(prof.span + 1, global_ns());
}

template <int B>
static cudaError_t configure_b() {
    const int smem = (int)sizeof(Smem<B>);
    cudaError_t e = cudaFuncSetAttribute(engine_kernel<B, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(engine_kernel<B, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(engine_kernel<B, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(engine_kernel<B, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    return e;
}

size_t engine_smem_bytes(int block) {
    switch (block) {
        case 128: return sizeof(Smem<128>);
        case 256: return sizeof(Smem<256>);
        default: return sizeof(Smem<512>);
    }
}

cudaError_t engine_configure() {
    cudaError_t e = configure_b<128>();
    if (e == cudaSuccess) e = configure_b<256>();
    if (e == cudaSuccess) e = configure_b<512>();
    return e;
}

template <int B>
static void launch_b(const DevIndex& ix, const DevPlan* plans, const DevTask* tasks, int nTasks, int* taskCounter,
                     unsigned long long* results, int* status, int grid, cudaStream_t stream,
                     const EngineProfile* prof) {
    const size_t smem = sizeof(Smem<B>);
    const EngineProfile p = prof ? *prof : EngineProfile{};
    if (p.bytes)
        engine_kernel<B, 2><<<grid, B, smem, stream>>>(ix, plans, tasks, nTasks, taskCounter, results, status, p);
    else if (p.budgetNs && p.incomplete && p.taskNs)
        engine_kernel<B, 3><<<grid, B, smem, stream>>>(ix, plans, tasks, nTasks, taskCounter, results, status, p);
    else if (p.taskNs)
        engine_kernel<B, 1><<<grid, B, smem, stream>>>(ix, plans, tasks, nTasks, taskCounter, results, status, p);
    else
        engine_kernel<B, 0><<<grid, B, smem, stream>>>(ix, plans, tasks, nTasks, taskCounter, results, status, p);
}

// Suffix memos (see memo_item): one block per job (a hub row x of one
// transition); warps take the y in N1(x), lanes the h in N2(y).  The first
// witness of h sets its S1 bit, any later one its S2 bit (atomicOr returns
// the old word).
// Adds one path ending at `rank` to a three-step memo's counts: a 32-bit
// shared counter, or the saturating byte in global memory.
__device__ __forceinline__ void memo3_count_path(uint32_t* smemCnt, uint32_t* cnt, uint32_t* S1, int rank) {
    if (smemCnt) {
        atomicAdd(smemCnt + rank, 1u);
        return;
    }
    uint32_t* cw = cnt + (rank >> 2);
    const int sh = (rank & 3) * 8;
    uint32_t old = *cw;
    while (((old >> sh) & 0xffu) != 0xffu) {
        const uint32_t seen = atomicCAS(cw, old, old + (1u << sh));
        if (seen == old) break;
        old = seen;
    }
    atomicOr(S1 + (rank >> 5), 1u << (rank & 31));
}

__global__ void memo_build_kernel(DevIndex ix, const MemoJob* jobs, int nJobs) {
    extern __shared__ uint32_t memoSmem[];
    if ((int)blockIdx.x >= nJobs) return;
    const MemoJob job = jobs[blockIdx.x];
    uint32_t* S1 = job.bits;
    uint32_t* S2 = S1 + job.words;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5;
    const int rb = ix.rowBeg[job.d1][job.row], re = ix.rowBeg[job.d1][job.row + 1];
    const int b = rb + job.b0, e = job.b1 < 0 ? re : rb + job.b1;
    Meter<false> mt;
    if (job.p3 >= 0) {
        // three steps: warps take the v2 of the slice, lanes the v3 in
        // N2(v2) and their N3 rows (a long one by the whole warp); every
        // path x -> v2 -> v3 -> h with x, v2, v3, h distinct counts once for
        // h, in shared counters added into the memo's bytes at the end
        const int x = ix.rowKey[job.d1][job.row];
        uint32_t* cnt = S1 + job.words;
        uint32_t* sc = job.wo <= kMemoSmemRanks ? memoSmem : nullptr;
        if (sc) {
            for (int r = threadIdx.x; r < job.wo; r += blockDim.x) sc[r] = 0u;
            __syncthreads();
        }
        for (int i = b + warp; i < e; i += nWarps) {
            const int v2 = __ldg(ix.val[job.d1] + i);
            if (v2 == x) continue;
            const int2 r2 = row_lookup(ix, job.p2, job.d2, v2, mt);
            for (int j0 = r2.x; j0 < r2.y; j0 += 32) {
                const int j = j0 + lane;
                int v3 = -1;
                int2 r3 = make_int2(0, 0);
                if (j < r2.y) {
                    v3 = __ldg(ix.val[job.d2] + j);
                    if (v3 != x && v3 != v2) r3 = row_lookup(ix, job.p3, job.d3, v3, mt);
                }
                const bool longRow = r3.y - r3.x >= 32;
                if (!longRow)
                    for (int t = r3.x; t < r3.y; ++t) {
                        const int h = __ldg(ix.val[job.d3] + t);
                        if (h == x || h == v2 || h == v3) continue;
                        const int rank = __ldg(ix.valRank[job.d3] + t);
                        if (rank >= 0 && rank < job.wo) memo3_count_path(sc, cnt, S1, rank);
                    }
                unsigned big = __ballot_sync(0xffffffffu, longRow);
                while (big) {   // long N3 rows: the whole warp walks each
                    const int src = __ffs(big) - 1;
                    big &= big - 1;
                    const int w3 = __shfl_sync(0xffffffffu, v3, src);
                    const int t0 = __shfl_sync(0xffffffffu, r3.x, src), t1 = __shfl_sync(0xffffffffu, r3.y, src);
                    for (int t = t0 + lane; t < t1; t += 32) {
                        const int h = __ldg(ix.val[job.d3] + t);
                        if (h == x || h == v2 || h == w3) continue;
                        const int rank = __ldg(ix.valRank[job.d3] + t);
                        if (rank >= 0 && rank < job.wo) memo3_count_path(sc, cnt, S1, rank);
                    }
                }
            }
        }
        if (sc) {
            __syncthreads();
            for (int r = threadIdx.x; r < job.wo; r += blockDim.x) {
                const uint32_t add = min(sc[r], 255u);
                if (!add) continue;
                uint32_t* cw = cnt + (r >> 2);
                const int sh = (r & 3) * 8;
                uint32_t old = *cw;
                for (;;) {
                    const uint32_t cur = (old >> sh) & 0xffu;
                    const uint32_t nv = min(cur + add, 255u);
                    if (nv == cur) break;
                    const uint32_t seen = atomicCAS(cw, old, (old & ~(0xffu << sh)) | (nv << sh));
                    if (seen == old) break;
                    old = seen;
                }
                atomicOr(S1 + (r >> 5), 1u << (r & 31));
            }
        }
        return;
    }
    for (int i = b + warp; i < e; i += nWarps) {
        const int y = __ldg(ix.val[job.d1] + i);
        const int2 r = row_lookup(ix, job.p2, job.d2, y, mt);
        for (int j = r.x + lane; j < r.y; j += 32) {
            if (__ldg(ix.val[job.d2] + j) == y) continue;
            const int rank = __ldg(ix.valRank[job.d2] + j);
            if (rank < 0 || rank >= (job.words << 5)) continue;
            const uint32_t bit = 1u << (rank & 31);
            const uint32_t old = atomicOr(S1 + (rank >> 5), bit);
            if (old & bit) atomicOr(S2 + (rank >> 5), bit);
        }
    }
}

// Fused support of split heavy roots: one block per job, its warps share the
// head triples of the job's root, counted against its completed global row.
__global__ void support_rows_kernel(const __grid_constant__ DevIndex ix, const DevPlan* plans, const SupJob* jobs,
                                    int nJobs, unsigned long long* results) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5;
    if ((int)blockIdx.x >= nJobs) return;
    const SupJob jb = jobs[blockIdx.x];
    const DevPlan& P = plans[jb.plan];
    if (!P.gHeavy) return;
    const uint32_t* row = P.gHeavy + (long long)jb.gRow * P.rowWords;
    Meter<false> mt;
    for (int j = 0; j < P.supN; ++j) {
        unsigned long long n = fused_support(P, ix, j, jb.root, 1, row, 0, 1, lane, warp, nWarps, mt);
        for (int d = 16; d; d >>= 1) n += __shfl_down_sync(0xffffffffu, n, d);
        if (lane == 0 && n) atomicAdd(results + P.supSlot[j], n);
    }
}

cudaError_t support_rows(const DevIndex& ix, const DevPlan* plans, const SupJob* jobs, int nJobs,
                         unsigned long long* results, cudaStream_t stream) {
    if (nJobs <= 0) return cudaSuccess;
    support_rows_kernel<<<nJobs, 256, 0, stream>>>(ix, plans, jobs, nJobs, results);
    return cudaGetLastError();
}

cudaError_t memo_build(const DevIndex& ix, const MemoJob* jobs, int nJobs, int maxWo, cudaStream_t stream) {
    if (nJobs <= 0) return cudaSuccess;
    const size_t smem = (size_t)std::min(maxWo, kMemoSmemRanks) * 4;
    if (smem > 48 * 1024) {
        const cudaError_t e =
            cudaFuncSetAttribute(memo_build_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    memo_build_kernel<<<nJobs, 256, smem, stream>>>(ix, jobs, nJobs);
    return cudaGetLastError();
}

// prof (optional): task times when prof->taskNs is set, also byte counts
// when prof->bytes is set (instrumented variants); a launch span when
// prof->span is set (any variant).
cudaError_t engine_launch(const DevIndex& ix, const DevPlan* plans, const DevTask* tasks, int nTasks,
                          int* taskCounter, unsigned long long* results, int* status, int grid, int block,
                          cudaStream_t stream, const EngineProfile* prof) {
    if (nTasks <= 0) return cudaSuccess;
    switch (block) {
        case 128: launch_b<128>(ix, plans, tasks, nTasks, taskCounter, results, status, grid, stream, prof); break;
        case 256: launch_b<256>(ix, plans, tasks, nTasks, taskCounter, results, status, grid, stream, prof); break;
        case 512: launch_b<512>(ix, plans, tasks, nTasks, taskCounter, results, status, grid, stream, prof); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace gr
