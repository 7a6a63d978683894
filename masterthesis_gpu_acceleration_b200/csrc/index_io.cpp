// index_io.cpp — binary graph files (see index_io.hpp).
#include "index_io.hpp"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

namespace gr {
namespace {

constexpr char kMagic[8] = {'G', 'R', 'G', 'R', 'A', 'P', 'H', '1'};
constexpr char kEnd[8] = {'G', 'R', 'E', 'N', 'D', '0', '0', '2'};
constexpr uint32_t kVersion = 2;

// Running 64-bit checksum of everything written before it.  Each call's
// bytes go into four independent multiply-xorshift lanes, 32 bytes a round
// (so that the lanes' multiplies overlap), then its trailing words and
// bytes into the first lane; the lanes fold into one word at every call.
struct Checksum {
    uint64_t h = 0x6A09E667F3BCC909ull;
    static uint64_t mix(uint64_t x, uint64_t w) {
        x = (x ^ w) * 0x9E3779B97F4A7C15ull;
        return x ^ (x >> 31);
    }
    void add(const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        uint64_t l[4] = {h, h ^ 0xBB67AE8584CAA73Bull, h ^ 0x3C6EF372FE94F82Bull, h ^ 0xA54FF53A5F1D36F1ull};
        size_t i = 0;
        for (; i + 32 <= n; i += 32) {
            uint64_t w[4];
            std::memcpy(w, b + i, 32);
            for (int k = 0; k < 4; ++k) l[k] = mix(l[k], w[k]);
        }
        for (; i + 8 <= n; i += 8) {
            uint64_t w;
            std::memcpy(&w, b + i, 8);
            l[0] = mix(l[0], w);
        }
        for (; i < n; ++i) l[0] = (l[0] ^ b[i]) * 0x100000001B3ull;
        h = mix(mix(mix(l[0], l[1]), l[2]), l[3] ^ (uint64_t)n);
    }
};
constexpr uint32_t kByteOrder = 0x01020304u;

struct Header {
    char magic[8];
    uint32_t version, byteOrder;
    int32_t nPred, nEnt;
    int64_t nTriples;
    uint32_t hashMask, pad;
};

struct FileCloser {
    void operator()(FILE* f) const { if (f) std::fclose(f); }
};
using File = std::unique_ptr<FILE, FileCloser>;

struct Writer {
    FILE* f;
    bool ok = true;
    Checksum sum;
    void bytes(const void* p, size_t n) {
        if (ok && n && std::fwrite(p, 1, n, f) != n) ok = false;
        sum.add(p, n);
    }
    template <class T> void pod(const T& v) { bytes(&v, sizeof(T)); }
    template <class T> void vec(const std::vector<T>& v) {
        pod<uint64_t>(v.size());
        bytes(v.data(), v.size() * sizeof(T));
    }
    void str(const std::string& s) {
        pod<uint32_t>((uint32_t)s.size());
        bytes(s.data(), s.size());
    }
};

struct Reader {
    FILE* f;
    uint64_t left;   // bytes not yet read: no count may claim more
    bool ok = true;
    Checksum sum;
    void bytes(void* p, size_t n) {
        if (!ok || n > left || (n && std::fread(p, 1, n, f) != n)) { ok = false; return; }
        left -= n;
        sum.add(p, n);
    }
    template <class T> void pod(T& v) { bytes(&v, sizeof(T)); }
    template <class T> void vec(std::vector<T>& v) {
        uint64_t n = 0;
        pod(n);
        if (!ok || n > left / sizeof(T)) { ok = false; return; }
        v.resize((size_t)n);
        bytes(v.data(), (size_t)n * sizeof(T));
    }
    void str(std::string& s) {
        uint32_t n = 0;
        pod(n);
        if (!ok || n > left) { ok = false; return; }
        s.resize(n);
        bytes(&s[0], n);
    }
};

void names_out(Writer& w, const TermDict& d) {
    w.pod<uint64_t>(d.names.size());
    for (const auto& s : d.names) w.str(s);
}

bool names_in(Reader& r, TermDict& d) {
    uint64_t n = 0;
    r.pod(n);
    if (!r.ok || n > r.left / 4) return false;
    d.names.resize((size_t)n);
    d.map.clear();
    d.map.reserve((size_t)n);
    for (uint64_t i = 0; i < n && r.ok; ++i) {
        r.str(d.names[(size_t)i]);
        if (r.ok && !d.map.emplace(d.names[(size_t)i], (int32_t)i).second) return false;   // names are distinct
    }
    return r.ok;
}

// Every array of the index in file order (dir 0 then dir 1 for the
// per-direction ones).
template <class F>
void each_array(HostIndex& ix, F f) {
    for (int d = 0; d < 2; ++d) {
        f(ix.val[d]); f(ix.valRank[d]); f(ix.src[d]); f(ix.srcRank[d]);
        f(ix.rowKey[d]); f(ix.rowBeg[d]); f(ix.predRow[d]); f(ix.predEdge[d]);
    }
    f(ix.hash);
    f(ix.hubOf[0]); f(ix.hubOf[1]);
    f(ix.hubOff);
    f(ix.hubBits);
    f(ix.valSig[0]); f(ix.valSig[1]);
    f(ix.sufSig[0]); f(ix.sufSig[1]);
}

bool monotone(const std::vector<int32_t>& v, int64_t lo, int64_t hi) {
    if (v.empty() || v.front() != lo || v.back() != hi) return false;
    for (size_t i = 1; i < v.size(); ++i)
        if (v[i] < v[i - 1]) return false;
    return true;
}

// Every size, range and offset the kernels and the host code index by, so
// that a damaged file is refused rather than read out of bounds.
bool consistent(const HostIndex& ix, size_t nEntNames, size_t nPredNames, std::string* why) {
    auto fail = [&](const char* m) { if (why) *why = m; return false; };
    const int32_t P = ix.nPred, N = ix.nEnt;
    if (P < 0 || N < 0 || (size_t)P != nPredNames || (size_t)N != nEntNames) return fail("dictionary sizes");
    const int64_t E = ix.nTriples;
    if (E < 0 || E > INT32_MAX) return fail("triple count");
    for (int d = 0; d < 2; ++d) {
        const size_t rows = ix.rowKey[d].size();
        if (ix.val[d].size() != (size_t)E || ix.valRank[d].size() != (size_t)E || ix.src[d].size() != (size_t)E ||
            ix.srcRank[d].size() != (size_t)E || ix.valSig[d].size() != (size_t)E || ix.sufSig[d].size() != (size_t)E)
            return fail("edge arrays");
        if (ix.rowBeg[d].size() != rows + 1 || ix.hubOf[d].size() != rows || rows > (size_t)INT32_MAX)
            return fail("row arrays");
        if (ix.predRow[d].size() != (size_t)P + 1 || ix.predEdge[d].size() != (size_t)P + 1) return fail("predicate arrays");
        if (!monotone(ix.predRow[d], 0, (int64_t)rows) || !monotone(ix.predEdge[d], 0, E) ||
            !monotone(ix.rowBeg[d], 0, E))
            return fail("offsets");
        for (size_t e = 0; e < (size_t)E; ++e)
            if (ix.val[d][e] < 0 || ix.val[d][e] >= N || ix.src[d][e] < 0 || ix.src[d][e] >= N) return fail("entity ids");
        for (size_t r = 0; r < rows; ++r)
            if (ix.rowKey[d][r] < 0 || ix.rowKey[d][r] >= N) return fail("row keys");
    }
    for (int d = 0; d < 2; ++d)
        for (int32_t p = 0; p < P; ++p) {
            if (ix.predRow[d][p + 1] > ix.predRow[d][p] &&
                (ix.rowBeg[d][ix.predRow[d][p]] != ix.predEdge[d][p] || ix.rowBeg[d][ix.predRow[d][p + 1]] != ix.predEdge[d][p + 1]))
                return fail("rows and predicates disagree");
            const int64_t own = ix.pred_rows(p, d), other = ix.pred_rows(p, 1 - d);
            for (int32_t e = ix.predEdge[d][p]; e < ix.predEdge[d][p + 1]; ++e)
                if (ix.srcRank[d][e] < 0 || ix.srcRank[d][e] >= own || ix.valRank[d][e] < 0 || ix.valRank[d][e] >= other)
                    return fail("ranks");
        }
    const size_t slots = ix.hash.size();
    if (slots == 0 || (slots & (slots - 1)) != 0 || ix.hashMask != slots - 1) return fail("lookup table size");
    for (const HashSlot& s : ix.hash)
        if (s.tag != kEmptyTag && (s.tag >= 2u * (uint32_t)P || s.beg > s.end || s.end > (uint64_t)E))
            return fail("lookup table entries");
    const int64_t hubs = (int64_t)ix.hubOff.size();
    for (int d = 0; d < 2; ++d)
        for (int32_t p = 0; p < P; ++p) {
            const int64_t words = (ix.pred_rows(p, 1 - d) + 31) / 32;
            for (int32_t r = ix.predRow[d][p]; r < ix.predRow[d][p + 1]; ++r) {
                const int32_t h = ix.hubOf[d][r];
                if (h < -1 || h >= hubs) return fail("hub ids");
                if (h >= 0 && (ix.hubOff[h] < 0 || ix.hubOff[h] + words > (int64_t)ix.hubBits.size()))
                    return fail("hub bitmaps");
            }
        }
    return true;
}

}  // namespace

bool save_graph_file(const std::string& path, const TermDict& ents, const TermDict& preds, const Prefixes& prefixes,
                     const HostIndex& ix, std::string* err) {
    File f(std::fopen(path.c_str(), "wb"));
    if (!f) { if (err) *err = "cannot open " + path + " for writing"; return false; }
    std::vector<char> buf(1 << 22);
    std::setvbuf(f.get(), buf.data(), _IOFBF, buf.size());
    Writer w{f.get()};
    Header h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.byteOrder = kByteOrder;
    h.nPred = ix.nPred;
    h.nEnt = ix.nEnt;
    h.nTriples = ix.nTriples;
    h.hashMask = ix.hashMask;
    w.pod(h);
    names_out(w, ents);
    names_out(w, preds);
    std::vector<std::pair<std::string, std::string>> pf(prefixes.begin(), prefixes.end());
    std::sort(pf.begin(), pf.end());
    w.pod<uint64_t>(pf.size());
    for (const auto& kv : pf) { w.str(kv.first); w.str(kv.second); }
    each_array(const_cast<HostIndex&>(ix), [&](auto& v) { w.vec(v); });
    const uint64_t sum = w.sum.h;
    w.pod(sum);
    w.bytes(kEnd, 8);
    const bool flushed = std::fflush(f.get()) == 0;
    if (!w.ok || !flushed) { if (err) *err = "write failed: " + path; return false; }
    return true;
}

bool load_graph_file(const std::string& path, TermDict& ents, TermDict& preds, Prefixes& prefixes, HostIndex& ix,
                     std::string* err) {
    auto fail = [&](const std::string& m) { if (err) *err = m + ": " + path; return false; };
    File f(std::fopen(path.c_str(), "rb"));
    if (!f) return fail("cannot open graph file");
    std::vector<char> buf(1 << 22);
    std::setvbuf(f.get(), buf.data(), _IOFBF, buf.size());
    if (std::fseek(f.get(), 0, SEEK_END) != 0) return fail("cannot size graph file");
    const long size = std::ftell(f.get());
    if (size < 0 || std::fseek(f.get(), 0, SEEK_SET) != 0) return fail("cannot size graph file");
    Reader r{f.get(), (uint64_t)size};
    Header h{};
    r.pod(h);
    if (!r.ok || std::memcmp(h.magic, kMagic, 8) != 0) return fail("not a graph file");
    if (h.version != kVersion || h.byteOrder != kByteOrder) return fail("graph file of another version or byte order");
    ix = HostIndex{};
    ix.nPred = h.nPred;
    ix.nEnt = h.nEnt;
    ix.nTriples = h.nTriples;
    ix.hashMask = h.hashMask;
    if (!names_in(r, ents) || !names_in(r, preds)) return fail("damaged dictionaries in graph file");
    uint64_t np = 0;
    r.pod(np);
    if (!r.ok || np > r.left / 8) return fail("damaged prefixes in graph file");
    prefixes.clear();
    for (uint64_t i = 0; i < np && r.ok; ++i) {
        std::string k, v;
        r.str(k);
        r.str(v);
        prefixes.emplace(std::move(k), std::move(v));
    }
    each_array(ix, [&](auto& v) { r.vec(v); });
    const uint64_t want = r.sum.h;
    uint64_t sum = 0;
    r.pod(sum);
    char end[8] = {};
    r.bytes(end, 8);
    if (!r.ok || std::memcmp(end, kEnd, 8) != 0 || r.left != 0) return fail("truncated or damaged graph file");
    if (sum != want) return fail("graph file checksum mismatch");
    std::string why;
    if (!consistent(ix, ents.names.size(), preds.names.size(), &why)) return fail("inconsistent graph file (" + why + ")");
    return true;
}

}  // namespace gr
