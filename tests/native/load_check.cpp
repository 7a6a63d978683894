// Native check of the graph load path (built and run by tests/test_load_cpu.py):
//   1. the multi-threaded Turtle read gives the same dictionaries and triples,
//      in the same order, as one reader over the whole text;
//   2. in the index built on several threads every row is found through the
//      lookup table at its own edge range, every triple is found, and every
//      value rank is the value's row in the other direction;
//   3. row signatures have no false negatives: every edge's value signature
//      holds the bit of every (pred, dir) under which the value keys a row,
//      and every suffix signature is the union of the value signatures from
//      its edge to the end of its row;
//   4. every hub row's bitmap has exactly the bits of its edges' value
//      ranks, within its predicate's domain;
//   5. the graph written to a binary file reads back identical, and a
//      truncated copy, or a copy with any one byte changed, is refused.
// Usage: load_check FILE.ttl MIN_CHUNK_BYTES [SCRATCH_FILE]
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../masterthesis_gpu_acceleration_b200/csrc/index.hpp"
#include "../../masterthesis_gpu_acceleration_b200/csrc/index_io.hpp"
#include "../../masterthesis_gpu_acceleration_b200/csrc/turtle.hpp"

using namespace gr;

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    std::string text, err;
    if (!read_file(argv[1], text, &err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 2; }
    TermDict e1, p1, e2, p2;
    std::vector<int32_t> s1, s2;
    parse_turtle_text(text, e1, p1, s1);
    parse_turtle_text_parallel(text, e2, p2, s2, (size_t)std::atol(argv[2]));
    if (e1.names != e2.names || p1.names != p2.names || s1 != s2) {
        std::printf("parallel read differs\n");
        return 1;
    }
    HostIndex ix = build_index(s2, (int32_t)e2.size(), (int32_t)p2.size(), 1);
    long bad = 0;
    for (int d = 0; d < 2; ++d)
        for (int32_t p = 0; p < ix.nPred; ++p)
            for (int32_t r = ix.predRow[d][p]; r < ix.predRow[d][p + 1]; ++r) {
                auto rr = ix.row_range(p, d, ix.rowKey[d][r]);
                if (rr.first != ix.rowBeg[d][r] || rr.second != ix.rowBeg[d][r + 1]) ++bad;
                for (int32_t e = ix.rowBeg[d][r]; e < ix.rowBeg[d][r + 1]; ++e) {
                    auto back = ix.row_range(p, 1 - d, ix.val[d][e]);
                    const int32_t row = ix.predRow[1 - d][p] + ix.valRank[d][e];
                    if (back.first != ix.rowBeg[1 - d][row]) ++bad;
                }
            }
    for (size_t i = 0; i + 2 < s2.size(); i += 3)
        if (!ix.has_triple(s2[i + 1], s2[i], s2[i + 2])) ++bad;
    // the signature each entity must carry, rebuilt here row by row
    std::vector<uint64_t> want((size_t)ix.nEnt, 0);
    for (int d = 0; d < 2; ++d)
        for (int32_t p = 0; p < ix.nPred; ++p)
            for (int32_t r = ix.predRow[d][p]; r < ix.predRow[d][p + 1]; ++r)
                want[(size_t)ix.rowKey[d][r]] |= 1ull << sig_bit(p, d);
    long badSig = 0;
    for (int d = 0; d < 2; ++d) {
        if (ix.valSig[d].size() != ix.val[d].size() || ix.sufSig[d].size() != ix.val[d].size()) { ++badSig; continue; }
        for (int32_t p = 0; p < ix.nPred; ++p)
            for (int32_t r = ix.predRow[d][p]; r < ix.predRow[d][p + 1]; ++r) {
                uint64_t acc = 0;
                for (int32_t e = ix.rowBeg[d][r + 1] - 1; e >= ix.rowBeg[d][r]; --e) {
                    if (ix.valSig[d][e] != want[(size_t)ix.val[d][e]]) ++badSig;
                    acc |= ix.valSig[d][e];
                    if (ix.sufSig[d][e] != acc) ++badSig;
                }
            }
    }
    bad += badSig;
    long badHub = 0;
    for (int d = 0; d < 2; ++d)
        for (int32_t p = 0; p < ix.nPred; ++p) {
            const int64_t words = (ix.pred_rows(p, 1 - d) + 31) / 32;
            for (int32_t r = ix.predRow[d][p]; r < ix.predRow[d][p + 1]; ++r) {
                const int32_t h = ix.hubOf[d][r];
                if (h < 0) continue;
                std::vector<uint32_t> want((size_t)words, 0u);
                for (int32_t e = ix.rowBeg[d][r]; e < ix.rowBeg[d][r + 1]; ++e)
                    want[(size_t)(ix.valRank[d][e] >> 5)] |= 1u << (ix.valRank[d][e] & 31);
                if (ix.hubOff[h] + words > (int64_t)ix.hubBits.size() ||
                    !std::equal(want.begin(), want.end(), ix.hubBits.begin() + ix.hubOff[h]))
                    ++badHub;
            }
        }
    bad += badHub;
    long badFile = 0;
    if (argc >= 4) {
        const std::string file = argv[3];
        const Prefixes pf = scan_rule_prefixes_text(text);
        std::string e;
        if (!save_graph_file(file, e2, p2, pf, ix, &e)) { std::printf("save: %s\n", e.c_str()); ++badFile; }
        TermDict e3, p3;
        Prefixes pf3;
        HostIndex ix3;
        if (!load_graph_file(file, e3, p3, pf3, ix3, &e)) { std::printf("load: %s\n", e.c_str()); ++badFile; }
        if (e3.names != e2.names || p3.names != p2.names || pf3 != pf) ++badFile;
        for (size_t i = 0; i < e3.names.size(); ++i)
            if (e3.find(e3.names[i]) != (int32_t)i) { ++badFile; break; }
        if (ix3.nPred != ix.nPred || ix3.nEnt != ix.nEnt || ix3.nTriples != ix.nTriples || ix3.hashMask != ix.hashMask) ++badFile;
        for (int d = 0; d < 2; ++d)
            if (ix3.val[d] != ix.val[d] || ix3.valRank[d] != ix.valRank[d] || ix3.src[d] != ix.src[d] ||
                ix3.srcRank[d] != ix.srcRank[d] || ix3.rowKey[d] != ix.rowKey[d] || ix3.rowBeg[d] != ix.rowBeg[d] ||
                ix3.predRow[d] != ix.predRow[d] || ix3.predEdge[d] != ix.predEdge[d] || ix3.hubOf[d] != ix.hubOf[d] ||
                ix3.valSig[d] != ix.valSig[d] || ix3.sufSig[d] != ix.sufSig[d])
                ++badFile;
        if (ix3.hubOff != ix.hubOff || ix3.hubBits != ix.hubBits || ix3.hash.size() != ix.hash.size() ||
            std::memcmp(ix3.hash.data(), ix.hash.data(), ix.hash.size() * sizeof(HashSlot)) != 0)
            ++badFile;
        // a truncated copy must be refused
        std::string all;
        read_file(file, all, &e);
        const std::string cut = file + ".cut";
        if (FILE* f = std::fopen(cut.c_str(), "wb")) {
            std::fwrite(all.data(), 1, all.size() / 2, f);
            std::fclose(f);
        }
        TermDict e4, p4;
        Prefixes pf4;
        HostIndex ix4;
        if (load_graph_file(cut, e4, p4, pf4, ix4, &e)) ++badFile;
        // single changed bytes at seeded positions
        uint64_t x = 0x9E3779B97F4A7C15ull;
        for (int k = 0; k < 24 && !all.empty(); ++k) {
            x = x * 6364136223846793005ull + 1442695040888963407ull;
            std::string bent = all;
            bent[(size_t)((x >> 17) % all.size())] ^= (char)(1 + (x >> 61));
            if (FILE* f = std::fopen(cut.c_str(), "wb")) {
                std::fwrite(bent.data(), 1, bent.size(), f);
                std::fclose(f);
            }
            TermDict e5, p5;
            Prefixes pf5;
            HostIndex ix5;
            if (load_graph_file(cut, e5, p5, pf5, ix5, &e)) ++badFile;
        }
        std::remove(cut.c_str());
    }
    bad += badFile;
    std::printf("triples %zu rows %zu hubs %zu mismatches %ld (signatures %ld, hub bitmaps %ld, graph file %ld)\n",
                s2.size() / 3, ix.rowKey[0].size() + ix.rowKey[1].size(), ix.hubOff.size(), bad, badSig, badHub,
                badFile);
    return bad == 0 ? 0 : 1;
}
