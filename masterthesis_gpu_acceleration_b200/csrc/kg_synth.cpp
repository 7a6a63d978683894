// kg_synth.cpp — seeded synthetic knowledge graphs and closed chain rules.
//
// The reference benchmarks on Turtle graphs and rule files that are not
// distributed with it (README.md:103-108).  These generators stand in for
// them: each configuration reproduces the stated shape (entity count,
// predicate count, triple count, degree distributions, rule lengths), is fully
// determined by its seed, and writes
//
//   triples.bin  int32 [T][3] (subject, predicate, object), entities 0..N-1,
//                predicates 0..P-1, duplicates removed
//   graph.ttl    the same triples as Turtle: <http://e/i> <http://p/k> <http://e/j> .
//   rules.txt    one rule per line in the reference's text rule syntax
//                (RuleParser.cpp:199-270), e.g.
//                (?a <http://p/3> ?v1) ^ (?v1 <http://p/7> ?b) => (?a <http://p/1> ?b)
//   rules.ir     int32 stream per rule: nb, head(p,sK,sV,oK,oV), body(p,sK,sV,oK,oV)*nb
//                with K = 0 for a variable (V = dense id in first-seen order,
//                body atoms first, then the head, as RuleParser.cpp:229-238 does)
//                and K = 1 for a constant entity id
//   meta.txt     key=value summary
//
// Random numbers come from splitmix64; integers in [0,n) use the 128-bit
// multiply-shift reduction.  Zipf(s) samples ranks 1..n with P(k) ~ k^-s by
// binary search in the cumulative weights, then maps the rank through a
// per-predicate random permutation of the entities.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_set>
#include <vector>

namespace {

struct Rng {
    uint64_t x;
    explicit Rng(uint64_t seed) : x(seed * 0x9E3779B97F4A7C15ull + 0xD1B54A32D192ED03ull) {}
    uint64_t next() {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    uint64_t below(uint64_t n) { return (uint64_t)(((__uint128_t)next() * n) >> 64); }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Zipf {
    std::vector<double> cdf;
    Zipf(int n, double s) : cdf(n) {
        double acc = 0.0;
        for (int k = 1; k <= n; ++k) { acc += std::pow((double)k, -s); cdf[k - 1] = acc; }
    }
    int sample(Rng& r) const {  // rank 0..n-1
        double u = r.unit() * cdf.back();
        int i = (int)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        return i < (int)cdf.size() ? i : (int)cdf.size() - 1;
    }
};

struct Triple { int32_t s, p, o; };

struct Graph {
    int N = 0, P = 0;
    std::vector<Triple> t;
    std::vector<int64_t> predCount;
};

static inline uint64_t pack(int s, int p, int o) {
    return ((uint64_t)(uint32_t)p << 42) | ((uint64_t)(uint32_t)s << 21) | (uint64_t)(uint32_t)o;
}

static std::vector<int> permutation(int n, Rng& r) {
    std::vector<int> v(n);
    for (int i = 0; i < n; ++i) v[i] = i;
    for (int i = n - 1; i > 0; --i) std::swap(v[i], v[r.below((uint64_t)i + 1)]);
    return v;
}

// Splits T triples over P predicates with weights w (at least one triple each).
static std::vector<int64_t> split_counts(int64_t T, const std::vector<double>& w) {
    int P = (int)w.size();
    double tot = 0.0;
    for (double x : w) tot += x;
    std::vector<int64_t> c(P);
    int64_t sum = 0;
    for (int k = 0; k < P; ++k) {
        c[k] = std::max<int64_t>(1, (int64_t)std::llround((double)T * w[k] / tot));
        sum += c[k];
    }
    // fix the rounding on the largest predicate
    int big = (int)(std::max_element(c.begin(), c.end()) - c.begin());
    c[big] += T - sum;
    return c;
}

enum class Dist { Uniform, Zipf };

struct PredSpec {
    Dist sd = Dist::Uniform, od = Dist::Uniform;
    double ss = 0.0, os = 0.0;
};

// Fills `count` distinct (s,o) pairs of predicate p.
static void fill_pred(Graph& g, std::unordered_set<uint64_t>& seen, int p, int64_t count,
                      const PredSpec& ps, const Zipf* zs, const Zipf* zo, Rng& r,
                      const std::vector<std::pair<int,int>>& forced = {}) {
    std::vector<int> permS, permO;
    if (ps.sd == Dist::Zipf) permS = permutation(g.N, r);
    if (ps.od == Dist::Zipf) permO = permutation(g.N, r);
    int64_t made = 0;
    for (auto& f : forced) {
        if (made >= count) break;
        if (seen.insert(pack(f.first, p, f.second)).second) {
            g.t.push_back({f.first, p, f.second});
            ++made;
        }
    }
    int64_t attempts = 0, limit = count * 200 + 1000;
    while (made < count && attempts < limit) {
        ++attempts;
        int s = ps.sd == Dist::Zipf ? permS[zs->sample(r)] : (int)r.below(g.N);
        int o = ps.od == Dist::Zipf ? permO[zo->sample(r)] : (int)r.below(g.N);
        if (seen.insert(pack(s, p, o)).second) {
            g.t.push_back({s, p, o});
            ++made;
        }
    }
    g.predCount[p] = made;
}

struct RuleIR {
    // atom = (p, sK, sV, oK, oV); head first in `atoms`, then body
    std::vector<std::vector<int>> body;
    std::vector<int> head;
};

static int pick_weighted(const std::vector<double>& cum, Rng& r) {
    double u = r.unit() * cum.back();
    int i = (int)(std::upper_bound(cum.begin(), cum.end(), u) - cum.begin());
    return std::min(i, (int)cum.size() - 1);
}

// A closed chain rule: head (?a ph ?b); body links ?a -> ?v1 -> ... -> ?b.
// Variable ids follow the reference parser's first-seen numbering.
static RuleIR chain_rule(int L, int ph, const std::vector<int>& preds, const std::vector<int>& dirs) {
    // chain variables by position: 0 = ?a, L = ?b, 1..L-1 = fresh
    std::vector<int> id(L + 1, -1);
    int next = 0;
    RuleIR r;
    for (int i = 0; i < L; ++i) {
        int x = i, y = i + 1;
        int subj = dirs[i] ? y : x, obj = dirs[i] ? x : y;
        if (id[subj] < 0) id[subj] = next++;
        if (id[obj] < 0) id[obj] = next++;
        r.body.push_back({preds[i], 0, id[subj], 0, id[obj]});
    }
    if (id[0] < 0) id[0] = next++;
    if (id[L] < 0) id[L] = next++;
    r.head = {ph, 0, id[0], 0, id[L]};
    return r;
}

static std::string var_name(int chainPos, int L) {
    if (chainPos == 0) return "?a";
    if (chainPos == L) return "?b";
    return "?v" + std::to_string(chainPos);
}

static std::string chain_text(int L, int ph, const std::vector<int>& preds, const std::vector<int>& dirs) {
    std::string out;
    for (int i = 0; i < L; ++i) {
        int x = i, y = i + 1;
        int subj = dirs[i] ? y : x, obj = dirs[i] ? x : y;
        if (i) out += " ^ ";
        out += "(" + var_name(subj, L) + " <http://p/" + std::to_string(preds[i]) + "> " + var_name(obj, L) + ")";
    }
    out += " => (?a <http://p/" + std::to_string(ph) + "> ?b)";
    return out;
}

// Bumped whenever a configuration's output changes (cached datasets with an
// older version are regenerated).
constexpr int kGenVersion = 2;

struct RuleSpec {
    int n = 10;
    std::vector<double> lenWeights;  // index = L-1
    bool predByFreq = false;
    int hubRules = 0;                // first hubRules rules include a hub predicate
    int nHubPreds = 0;
};

// Shape of the biomedical-style configurations: entities, triples, hub
// in-degree (two hubs on each of 5 hub predicates).
struct BioShape {
    int N;
    int64_t T;
    int hubDegree;
};

static bool write_all(const std::string& dir, const Graph& g, const std::vector<RuleIR>& rules,
                      const std::vector<std::string>& texts, const std::string& cfg, uint64_t seed,
                      uint64_t ruleSeed = ~0ull) {
    {
        FILE* f = std::fopen((dir + "/triples.bin").c_str(), "wb");
        if (!f) return false;
        std::fwrite(g.t.data(), sizeof(Triple), g.t.size(), f);
        std::fclose(f);
    }
    {
        FILE* f = std::fopen((dir + "/graph.ttl").c_str(), "wb");
        if (!f) return false;
        std::vector<char> buf(1 << 20);
        std::setvbuf(f, buf.data(), _IOFBF, buf.size());
        for (auto& x : g.t) std::fprintf(f, "<http://e/%d> <http://p/%d> <http://e/%d> .\n", x.s, x.p, x.o);
        std::fclose(f);
    }
    {
        FILE* f = std::fopen((dir + "/rules.txt").c_str(), "wb");
        if (!f) return false;
        for (auto& s : texts) std::fprintf(f, "%s\n", s.c_str());
        std::fclose(f);
    }
    {
        FILE* f = std::fopen((dir + "/rules.ir").c_str(), "wb");
        if (!f) return false;
        for (auto& r : rules) {
            int32_t nb = (int32_t)r.body.size();
            std::fwrite(&nb, 4, 1, f);
            std::fwrite(r.head.data(), 4, 5, f);
            for (auto& a : r.body) std::fwrite(a.data(), 4, 5, f);
        }
        std::fclose(f);
    }
    {
        FILE* f = std::fopen((dir + "/meta.txt").c_str(), "wb");
        if (!f) return false;
        std::fprintf(f, "config=%s\nseed=%llu\nentities=%d\npredicates=%d\ntriples=%zu\nrules=%zu\ngen=%d\n",
                     cfg.c_str(), (unsigned long long)seed, g.N, g.P, g.t.size(), rules.size(), kGenVersion);
        if (ruleSeed != ~0ull) std::fprintf(f, "rule_seed=%llu\n", (unsigned long long)ruleSeed);
        std::fclose(f);
    }
    return true;
}

static void make_rules(const Graph& g, const RuleSpec& rs, Rng& r,
                       std::vector<RuleIR>& rules, std::vector<std::string>& texts) {
    std::vector<double> predCum(g.P), lenCum(rs.lenWeights.size());
    double acc = 0.0;
    for (int p = 0; p < g.P; ++p) { acc += rs.predByFreq ? (double)g.predCount[p] : 1.0; predCum[p] = acc; }
    acc = 0.0;
    for (size_t i = 0; i < rs.lenWeights.size(); ++i) { acc += rs.lenWeights[i]; lenCum[i] = acc; }
    for (int i = 0; i < rs.n; ++i) {
        int L = pick_weighted(lenCum, r) + 1;
        int ph = pick_weighted(predCum, r);
        std::vector<int> preds(L), dirs(L);
        for (int k = 0; k < L; ++k) {
            preds[k] = pick_weighted(predCum, r);
            dirs[k] = (int)r.below(2);
        }
        if (i < rs.hubRules && rs.nHubPreds > 0) {
            const int hp = (int)r.below(rs.nHubPreds);
            if (i % 2 == 0 && L >= 2) {
                // through a hub from both sides: (?x hp ?v) ^ (?y hp ?v)
                const int k = (int)r.below(L - 1);
                preds[k] = preds[k + 1] = hp;
                dirs[k] = 0;
                dirs[k + 1] = 1;
            } else {
                preds[r.below(L)] = hp;
            }
        }
        rules.push_back(chain_rule(L, ph, preds, dirs));
        texts.push_back(chain_text(L, ph, preds, dirs));
    }
}

}  // namespace

extern "C" {

// Writes configuration `cfg` (c1, c2, c2s, c3, c4, c4s) for graph seed `seed`
// into `outDir`; the rules continue the graph's random stream, or, when
// ruleSeed != ~0, come from their own stream seeded with ruleSeed (the graph
// is the same either way).  nRules < 0 keeps the configuration's rule count.
// Returns the triple count, or -1 on an unknown configuration or I/O error.
long long kg_synth_write2(const char* cfg, unsigned long long seed, unsigned long long ruleSeed, int nRules,
                          const char* outDir) {
    std::string c(cfg);
    Rng r(seed);
    Graph g;
    RuleSpec rs;
    std::unordered_set<uint64_t> seen;
    if (c == "c1" || c == "c2" || c == "c2s") {
        bool c1 = c == "c1";
        g.N = c1 ? 10000 : 2000;
        g.P = c1 ? 20 : 10;
        int64_t T = 100000;
        g.predCount.assign(g.P, 0);
        seen.reserve((size_t)T * 2);
        std::vector<double> w(g.P, 1.0);
        auto cnt = split_counts(T, w);
        PredSpec ps;
        Zipf zs(g.N, 1.3);
        if (c == "c2s") { ps.sd = Dist::Zipf; ps.ss = 1.3; }
        for (int p = 0; p < g.P; ++p) fill_pred(g, seen, p, cnt[p], ps, &zs, nullptr, r);
        rs.n = 10;
        rs.lenWeights = c1 ? std::vector<double>{1, 1} : std::vector<double>{0, 1, 1};
    } else if (c == "c3") {
        g.N = 100000; g.P = 600;
        int64_t T = 206000;
        g.predCount.assign(g.P, 0);
        seen.reserve((size_t)T * 2);
        std::vector<double> w(g.P);
        for (int k = 0; k < g.P; ++k) w[k] = std::pow((double)(k + 1), -1.1);
        auto cnt = split_counts(T, w);
        PredSpec ps; ps.sd = Dist::Zipf; ps.ss = 1.5; ps.od = Dist::Zipf; ps.os = 1.3;
        Zipf zs(g.N, 1.5), zo(g.N, 1.3);
        for (int p = 0; p < g.P; ++p) fill_pred(g, seen, p, cnt[p], ps, &zs, &zo, r);
        rs.n = 10000;
        rs.lenWeights = {0.2, 0.4, 0.3, 0.1};
        rs.predByFreq = true;
    } else if (c == "c4" || c == "c4s") {
        // c4s: the same construction at a tenth of the size
        const BioShape sh = c == "c4" ? BioShape{300000, 6800000, 50000} : BioShape{30000, 680000, 5000};
        g.N = sh.N; g.P = 50;
        const int64_t T = sh.T;
        g.predCount.assign(g.P, 0);
        seen.reserve((size_t)T * 2);
        const int hubPreds = 5;
        const double hubShare = (double)T * 400000.0 / 6800000.0;
        std::vector<double> w(g.P);
        for (int k = 0; k < g.P; ++k) w[k] = k < hubPreds ? hubShare : ((double)T - hubPreds * hubShare) / (g.P - hubPreds);
        auto cnt = split_counts(T, w);
        PredSpec ps; ps.od = Dist::Zipf; ps.os = 1.2;
        Zipf zo(g.N, 1.2);
        for (int p = 0; p < g.P; ++p) {
            std::vector<std::pair<int,int>> forced;
            if (p < hubPreds) {
                // two hub objects with in-degree sh.hubDegree each
                for (int h = 0; h < 2; ++h) {
                    int hub = (int)r.below(g.N);
                    std::vector<int> subj = permutation(g.N, r);
                    for (int k = 0; k < sh.hubDegree; ++k) forced.push_back({subj[k], hub});
                }
            }
            fill_pred(g, seen, p, cnt[p], ps, nullptr, &zo, r, forced);
        }
        rs.n = 50;
        rs.lenWeights = {0, 1, 1, 1, 1};
        rs.predByFreq = true;
        rs.hubRules = 10;
        rs.nHubPreds = hubPreds;
    } else {
        return -1;
    }
    if (nRules >= 0) rs.n = nRules;
    if (ruleSeed != ~0ull) r = Rng(ruleSeed ^ 0xA5A5A5A5DEADBEEFull);
    std::vector<RuleIR> rules;
    std::vector<std::string> texts;
    make_rules(g, rs, r, rules, texts);
    if (!write_all(outDir, g, rules, texts, c, seed, ruleSeed)) return -1;
    return (long long)g.t.size();
}

long long kg_synth_write(const char* cfg, unsigned long long seed, int nRules, const char* outDir) {
    return kg_synth_write2(cfg, seed, ~0ull, nRules, outDir);
}

// Request stream for the serving configuration: n closed chain rules over a
// graph with the given per-predicate triple counts; body length is
// geometric(p) truncated to 1..maxLen, predicates are drawn by frequency.
// Writes rules.txt / rules.ir into outDir.  Returns n, or -1 on I/O error.
int kg_synth_rule_stream(const long long* predCount, int P, int n, double p, int maxLen,
                         unsigned long long seed, const char* outDir) {
    Rng r(seed ^ 0x5E5E5E5Eull);
    Graph g;
    g.P = P;
    g.predCount.assign(predCount, predCount + P);
    RuleSpec rs;
    rs.n = n;
    rs.predByFreq = true;
    rs.lenWeights.resize(maxLen);
    for (int L = 1; L <= maxLen; ++L) rs.lenWeights[L - 1] = std::pow(1.0 - p, L - 1) * p;
    std::vector<RuleIR> rules;
    std::vector<std::string> texts;
    make_rules(g, rs, r, rules, texts);
    std::string dir(outDir);
    FILE* f = std::fopen((dir + "/rules.txt").c_str(), "wb");
    if (!f) return -1;
    for (auto& s : texts) std::fprintf(f, "%s\n", s.c_str());
    std::fclose(f);
    f = std::fopen((dir + "/rules.ir").c_str(), "wb");
    if (!f) return -1;
    for (auto& rr : rules) {
        int32_t nb = (int32_t)rr.body.size();
        std::fwrite(&nb, 4, 1, f);
        std::fwrite(rr.head.data(), 4, 5, f);
        for (auto& a : rr.body) std::fwrite(a.data(), 4, 5, f);
    }
    std::fclose(f);
    return n;
}

}  // extern "C"
