// index.hpp — host-side graph index (the device copy mirrors it).
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

#include "common.hpp"

namespace gr {

struct HostIndex {
    int32_t nPred = 0, nEnt = 0;
    int64_t nTriples = 0;
    std::vector<int32_t> val[2], valRank[2], src[2], srcRank[2];
    std::vector<int32_t> rowKey[2], rowBeg[2];
    std::vector<int32_t> predRow[2], predEdge[2];
    std::vector<HashSlot> hash;
    uint32_t hashMask = 0;
    // Hub rows: rows with many edges get a bitmap of their values' ranks
    // (bit valRank of every edge), so that a body-size expansion through
    // them can OR 32 candidates at a time.  hubOf[d][row] = hub index or -1;
    // hub h's bitmap is hubBits[hubOff[h] .. hubOff[h] + words of its domain).
    std::vector<int32_t> hubOf[2];
    std::vector<int64_t> hubOff;
    std::vector<uint32_t> hubBits;
    // Per direction, per edge: the row signature (sig_bit) of the edge's
    // value, read beside the value so that an expansion can drop a
    // candidate whose next row does not exist without looking it up.
    std::vector<uint64_t> valSig[2];
    // Per direction, per edge: the union of valSig from the edge to the end
    // of its row, so that an item whose whole segment cannot continue is
    // never stored.
    std::vector<uint64_t> sufSig[2];

    int64_t pred_size(int32_t p) const {
        return (p < 0 || p >= nPred) ? 0 : predEdge[0][p + 1] - predEdge[0][p];
    }
    int64_t pred_rows(int32_t p, int d) const {
        return (p < 0 || p >= nPred) ? 0 : predRow[d][p + 1] - predRow[d][p];
    }
    // Edge range [beg, end) of row (p, d, key); (0, 0) if absent.
    std::pair<int32_t, int32_t> row_range(int32_t p, int d, int32_t key) const;
    bool has_triple(int32_t p, int32_t s, int32_t o) const;
    double avg_degree(int32_t p, int d) const {
        int64_t r = pred_rows(p, d);
        return r ? (double)pred_size(p) / (double)r : 0.0;
    }
};

// Rows with at least this many edges may become hub rows (0 = none).
constexpr int32_t kHubMinDegree = 128;

// Builds the index from (s, p, o) triples (duplicates removed).
// hubMinDegree: see kHubMinDegree.
HostIndex build_index(const std::vector<int32_t>& spo, int32_t nEnt, int32_t nPred,
                      int32_t hubMinDegree = kHubMinDegree);

// The same index with the sorts, rows, ranks, lookup table and signatures
// built on the current CUDA device and copied back (index_gpu.cu); only the
// hub bitmaps are built on the host.  Throws on a CUDA error.  A graph whose
// packed (predicate, key, value) keys need more than 64 bits is built on the
// host.
HostIndex build_index_device(const std::vector<int32_t>& spo, int32_t nEnt, int32_t nPred,
                             int32_t hubMinDegree = kHubMinDegree);

// Hub rows and their bitmaps of an index whose other arrays are complete.
void build_hub_rows(HostIndex& ix, int32_t minDegree);

}  // namespace gr
