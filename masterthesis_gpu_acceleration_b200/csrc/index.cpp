// index.cpp — builds the per-direction, per-predicate CSR and its lookup table.
//
// The reference keeps a dense rowPtr[N+1] per predicate and direction on the
// device (GPU_03/gpu_index.cuh:24-99), which costs P x N x 8 bytes (480 MB
// for 600 predicates over 100k entities) and scatters row lookups across it.
// Here rows are key-compressed (only keys that occur, as in
// CPU_01_nonparallel/RdfIndexes.cpp:91-138) and found through one
// open-addressing table keyed by (predicate, direction, key), so the whole
// lookup structure of a DBpedia-sized graph stays inside L2.
#include "index.hpp"
#include "parallel.hpp"

#include <algorithm>
#include <numeric>

namespace gr {
namespace {

struct T3 { int32_t p, k, v; };

inline bool t3_less(const T3& a, const T3& b) {
    if (a.p != b.p) return a.p < b.p;
    if (a.k != b.k) return a.k < b.k;
    return a.v < b.v;
}

void build_dir(HostIndex& ix, int d, std::vector<T3>& t) {
    if (!std::is_sorted(t.begin(), t.end(), t3_less)) parallel_sort(t, t3_less);
    size_t n = t.size();
    auto& val = ix.val[d];
    auto& src = ix.src[d];
    auto& rowKey = ix.rowKey[d];
    auto& rowBeg = ix.rowBeg[d];
    auto& predRow = ix.predRow[d];
    auto& predEdge = ix.predEdge[d];
    auto& srcRank = ix.srcRank[d];
    val.resize(n); src.resize(n); srcRank.resize(n);
    rowKey.clear(); rowBeg.clear();
    predRow.assign(ix.nPred + 1, 0);
    predEdge.assign(ix.nPred + 1, 0);
    int32_t curP = -1, curK = 0;
    size_t pi = 0;
    for (size_t i = 0; i < n; ++i) {
        const T3& x = t[i];
        while ((int32_t)pi <= x.p) {  // open predicates up to x.p
            predRow[pi] = (int32_t)rowKey.size();
            predEdge[pi] = (int32_t)i;
            ++pi;
        }
        if (x.p != curP || x.k != curK) {
            rowKey.push_back(x.k);
            rowBeg.push_back((int32_t)i);
            curP = x.p; curK = x.k;
        }
        val[i] = x.v;
        src[i] = x.k;
        srcRank[i] = (int32_t)rowKey.size() - 1 - predRow[x.p];
    }
    while ((int32_t)pi <= ix.nPred) {
        predRow[pi] = (int32_t)rowKey.size();
        predEdge[pi] = (int32_t)n;
        ++pi;
    }
    rowBeg.push_back((int32_t)n);
}

// Rank of `key` among the keys of predicate p in direction d.
int32_t key_rank(const HostIndex& ix, int d, int32_t p, int32_t key) {
    const int32_t* b = ix.rowKey[d].data() + ix.predRow[d][p];
    const int32_t* e = ix.rowKey[d].data() + ix.predRow[d][p + 1];
    return (int32_t)(std::lower_bound(b, e, key) - b);
}

// Rows whose expansion is cheaper as a bitmap OR than edge by edge: at
// least minDegree edges and a value domain (the predicate's rows in the
// other direction) of at most 8 words per edge.  Heaviest rows first, up to
// kHubBudgetWords of bitmap in total.
constexpr int64_t kHubBudgetWords = int64_t(1) << 28;   // 1 GiB

void build_hubs(HostIndex& ix, int32_t minDegree) {
    struct Cand { int32_t d, row, deg; int64_t words; };
    std::vector<Cand> c;
    for (int d = 0; d < 2; ++d) {
        ix.hubOf[d].assign(ix.rowKey[d].size(), -1);
        for (int32_t p = 0; p < ix.nPred; ++p) {
            const int64_t words = (ix.pred_rows(p, 1 - d) + 31) / 32;
            for (int32_t r = ix.predRow[d][p]; r < ix.predRow[d][p + 1]; ++r) {
                const int32_t deg = ix.rowBeg[d][r + 1] - ix.rowBeg[d][r];
                if (minDegree > 0 && deg >= minDegree && words <= 8LL * deg) c.push_back({d, r, deg, words});
            }
        }
    }
    std::sort(c.begin(), c.end(), [](const Cand& a, const Cand& b) { return a.deg > b.deg; });
    int64_t used = 0;
    ix.hubOff.clear();
    ix.hubBits.clear();
    for (const Cand& h : c) {
        if (used + h.words > kHubBudgetWords) continue;
        ix.hubOf[h.d][h.row] = (int32_t)ix.hubOff.size();
        ix.hubOff.push_back(used);
        used += h.words;
    }
    ix.hubBits.assign((size_t)used, 0u);
    for (int d = 0; d < 2; ++d)
        for (size_t r = 0; r < ix.hubOf[d].size(); ++r) {
            const int32_t h = ix.hubOf[d][r];
            if (h < 0) continue;
            uint32_t* bits = ix.hubBits.data() + ix.hubOff[h];
            for (int32_t e = ix.rowBeg[d][r]; e < ix.rowBeg[d][r + 1]; ++e) {
                const int32_t k = ix.valRank[d][e];
                bits[k >> 5] |= 1u << (k & 31);
            }
        }
}

}  // namespace

void build_hub_rows(HostIndex& ix, int32_t minDegree) { build_hubs(ix, minDegree); }

std::pair<int32_t, int32_t> HostIndex::row_range(int32_t p, int d, int32_t key) const {
    if (p < 0 || p >= nPred || key < 0 || hash.empty()) return {0, 0};
    uint32_t tag = (uint32_t)p * 2u + (uint32_t)d;
    uint32_t i = slot_hash(tag, (uint32_t)key) & hashMask;
    for (uint32_t probe = 0; probe <= hashMask; ++probe) {
        const HashSlot& s = hash[i];
        if (s.tag == kEmptyTag) return {0, 0};
        if (s.tag == tag && s.key == (uint32_t)key) return {(int32_t)s.beg, (int32_t)s.end};
        i = (i + 1) & hashMask;
    }
    return {0, 0};
}

bool HostIndex::has_triple(int32_t p, int32_t s, int32_t o) const {
    auto r = row_range(p, 0, s);
    const int32_t* b = val[0].data() + r.first;
    const int32_t* e = val[0].data() + r.second;
    return std::binary_search(b, e, o);
}

HostIndex build_index(const std::vector<int32_t>& spo, int32_t nEnt, int32_t nPred, int32_t hubMinDegree) {
    HostIndex ix;
    ix.nEnt = nEnt;
    ix.nPred = nPred;
    size_t n = spo.size() / 3;
    std::vector<T3> t(n);
    for (size_t i = 0; i < n; ++i) t[i] = {spo[3 * i + 1], spo[3 * i], spo[3 * i + 2]};
    parallel_sort(t, t3_less);
    t.erase(std::unique(t.begin(), t.end(), [](const T3& a, const T3& b) {
                return a.p == b.p && a.k == b.k && a.v == b.v;
            }), t.end());
    ix.nTriples = (int64_t)t.size();
    std::vector<T3> rev(t.size());
    for (size_t i = 0; i < t.size(); ++i) rev[i] = {t[i].p, t[i].v, t[i].k};
    build_dir(ix, 0, t);
    build_dir(ix, 1, rev);
    // value ranks: the value's row in the other direction
    for (int d = 0; d < 2; ++d) {
        auto& vr = ix.valRank[d];
        vr.resize(ix.val[d].size());
        parallel_for((size_t)nPred, [&](size_t p) {
            for (int32_t e = ix.predEdge[d][p]; e < ix.predEdge[d][p + 1]; ++e)
                vr[e] = key_rank(ix, 1 - d, (int32_t)p, ix.val[d][e]);
        }, 1);
    }
    // (pred, dir, key) table at load factor <= 1/2
    size_t rows = ix.rowKey[0].size() + ix.rowKey[1].size();
    size_t cap = 1024;
    while (cap < 2 * rows) cap <<= 1;
    ix.hash.assign(cap, HashSlot{kEmptyTag, 0, 0, 0});
    ix.hashMask = (uint32_t)(cap - 1);
    // rows are distinct, so threads only need to claim empty slots (the
    // slot order may differ between runs; lookups do not depend on it)
    for (int d = 0; d < 2; ++d) {
        parallel_for((size_t)nPred, [&](size_t p) {
            const uint32_t tag = (uint32_t)p * 2u + (uint32_t)d;
            for (int32_t r = ix.predRow[d][p]; r < ix.predRow[d][p + 1]; ++r) {
                const uint32_t key = (uint32_t)ix.rowKey[d][r];
                uint32_t i = slot_hash(tag, key) & ix.hashMask;
                for (;;) {
                    uint32_t expect = kEmptyTag;
                    if (__atomic_compare_exchange_n(&ix.hash[i].tag, &expect, tag, false, __ATOMIC_RELAXED,
                                                    __ATOMIC_RELAXED))
                        break;
                    i = (i + 1) & ix.hashMask;
                }
                ix.hash[i].key = key;
                ix.hash[i].beg = (uint32_t)ix.rowBeg[d][r];
                ix.hash[i].end = (uint32_t)ix.rowBeg[d][r + 1];
            }
        }, 1);
    }
    // row signatures: per entity, then copied beside every edge's value
    std::vector<uint64_t> entSig((size_t)std::max(nEnt, 1), 0);
    for (int d = 0; d < 2; ++d)
        parallel_for((size_t)nPred, [&](size_t p) {
            const uint64_t bit = 1ull << sig_bit((int32_t)p, d);
            for (int32_t r = ix.predRow[d][p]; r < ix.predRow[d][p + 1]; ++r)
                __atomic_fetch_or(&entSig[(size_t)ix.rowKey[d][r]], bit, __ATOMIC_RELAXED);
        }, 1);
    for (int d = 0; d < 2; ++d) {
        const size_t nE = ix.val[d].size();
        ix.valSig[d].resize(nE);
        parallel_for((nE + 65535) / 65536, [&](size_t c) {
            const size_t e1 = std::min(nE, (c + 1) * 65536);
            for (size_t e = c * 65536; e < e1; ++e) ix.valSig[d][e] = entSig[(size_t)ix.val[d][e]];
        }, 1);
        ix.sufSig[d].resize(nE);
        parallel_for((size_t)nPred, [&](size_t p) {
            for (int32_t r = ix.predRow[d][p]; r < ix.predRow[d][p + 1]; ++r) {
                uint64_t acc = 0;
                for (int32_t e = ix.rowBeg[d][r + 1] - 1; e >= ix.rowBeg[d][r]; --e)
                    ix.sufSig[d][(size_t)e] = acc |= ix.valSig[d][(size_t)e];
            }
        }, 1);
    }
    build_hubs(ix, hubMinDegree);
    return ix;
}

}  // namespace gr
