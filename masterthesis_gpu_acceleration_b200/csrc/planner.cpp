// planner.cpp — turns a parsed rule into device plans.
//
// Semantics (CPU_01_nonparallel/SupportCounting.cpp):
//  * support (474-552): head triples that match the head pattern injectively
//    (9-34) and admit a body grounding; the head triple counts as used.
//  * body size (563-631): distinct (hS, hO) over body groundings, with the
//    keys of the smallest body atom containing hS as hS candidates; hS == hO,
//    or hO absent from the body, counts candidates with a grounding.
//  * injective bindings: a newly bound variable differs from every bound
//    variable (SupportCounting.hpp:43-48); constants take no part.
//  * used triples: no ground triple appears twice in one grounding
//    (SupportCounting.hpp:50-55).  With injective variables two atoms can
//    only ground to the same triple if they have the same predicate and no
//    position holds two different variables.  Atoms that are identical term
//    for term always collide (the count is 0); atoms that might collide
//    because a constant meets a variable get a runtime comparison.
//
// Plan shape: the bound variables form a tuple [root, hO rank, v0, v1, ...]
// in binding order.  Atoms are grounded greedily: every atom whose terms are
// all bound becomes a membership check as soon as possible; otherwise the
// atom with one bound term and the smallest average fan-out is expanded from
// that term; otherwise the smallest predicate is scanned.  The order only
// affects speed: every complete grounding satisfies the same constraints
// whichever order finds it (the reference's greedy choice in
// SupportCounting.cpp:38-79 is likewise a speed heuristic).
#include "planner.hpp"

#include <algorithm>
#include <cstring>
#include <limits>

namespace gr {
namespace {

enum Rel { kEq, kNe, kMaybe };

Rel rel(const Term& a, const Term& b) {
    if (a.isVar == b.isVar) return a.id == b.id ? kEq : kNe;
    return kMaybe;
}

bool has_unknown(const Atom& a) {
    return a.pred < 0 || (!a.s.isVar && a.s.id < 0) || (!a.o.isVar && a.o.id < 0);
}

struct Builder {
    const HostIndex& ix;
    DevPlan& P;
    int32_t pos[kMaxVars];
    int32_t tupleLen = kTupleHead;
    int32_t nConsts = 0;
    bool ok = true;

    Builder(const HostIndex& x, DevPlan& p) : ix(x), P(p) {
        for (int i = 0; i < kMaxVars; ++i) pos[i] = -1;
    }
    bool bound(const Term& t) const { return !t.isVar || pos[t.id] >= 0; }
    void bind(int32_t var) {
        if (pos[var] < 0) pos[var] = tupleLen++;
    }
    TermRef ref(const Term& t) {
        if (t.isVar) return (TermRef)pos[t.id];
        for (int k = 0; k < nConsts; ++k)
            if (P.consts[k] == t.id) return (TermRef)(-1 - k);
        if (nConsts >= kMaxConsts) { ok = false; return 0; }
        P.consts[nConsts] = t.id;
        return (TermRef)(-1 - nConsts++);
    }
};

int check_dir(const HostIndex& ix, int32_t p) {
    return ix.avg_degree(p, 0) <= ix.avg_degree(p, 1) ? 0 : 1;
}

// Grounding order for `body` given the variables already bound in `b`.
// `head` (support phase) is the used head triple, or null.  Returns false
// when two atoms always ground to the same triple.
bool build_steps(Builder& b, const std::vector<Atom>& body, const Atom* head, int32_t hO, bool pairs) {
    DevPlan& P = b.P;
    const HostIndex& ix = b.ix;
    const int nb = (int)body.size();   // at most kMaxBody (plan_rule checks)
    // fixed-size bookkeeping (no allocation per plan): levels and order of
    // the atoms, and the checks in the order they were found
    int level[kMaxBody], order[kMaxBody], nOrder = 0;
    for (int i = 0; i < nb; ++i) level[i] = -1;
    struct LevelCheck { int lvl; DevCheck c; };
    LevelCheck found[kMaxBody];
    int nFound = 0;
    auto add_checks = [&](int lvl) {
        for (int i = 0; i < nb; ++i) {
            if (level[i] >= 0 || !b.bound(body[i].s) || !b.bound(body[i].o)) continue;
            level[i] = lvl;
            order[nOrder++] = i;
            DevCheck c{};
            c.pred = body[i].pred;
            c.s = b.ref(body[i].s);
            c.o = b.ref(body[i].o);
            c.dir = (int8_t)check_dir(ix, body[i].pred);
            found[nFound++] = LevelCheck{lvl, c};
        }
    };
    P.tupleLen[0] = b.tupleLen;
    add_checks(0);
    int lvl = 0;
    while (nOrder < nb) {
        int best = -1, bestDir = 0;
        double bestFan = std::numeric_limits<double>::infinity();
        for (int i = 0; i < nb; ++i) {
            if (level[i] >= 0) continue;
            bool sB = b.bound(body[i].s), oB = b.bound(body[i].o);
            if (sB == oB) continue;
            int d = sB ? 0 : 1;
            double fan = ix.avg_degree(body[i].pred, d);
            if (fan < bestFan) { bestFan = fan; best = i; bestDir = d; }
        }
        ++lvl;
        DevStep& st = P.steps[lvl - 1];
        st = DevStep{};
        if (best >= 0) {
            const Atom& a = body[best];
            st.kind = kExpand;
            st.pred = a.pred;
            st.dir = (int8_t)bestDir;
            st.keyRef = b.ref(bestDir == 0 ? a.s : a.o);
            const Term& nv = bestDir == 0 ? a.o : a.s;
            b.bind(nv.id);
            st.nNew = 1;
            st.hoWhich = (pairs && nv.id == hO) ? 1 : 0;
        } else {
            int64_t bestSize = std::numeric_limits<int64_t>::max();
            for (int i = 0; i < nb; ++i) {
                if (level[i] >= 0) continue;
                int64_t sz = ix.pred_size(body[i].pred);
                if (sz < bestSize) { bestSize = sz; best = i; }
            }
            const Atom& a = body[best];
            st.kind = kScan;
            st.pred = a.pred;
            st.dir = 0;
            if (a.s.id == a.o.id) {
                st.sameVar = 1;
                st.nNew = 1;
                b.bind(a.s.id);
                st.hoWhich = (pairs && a.s.id == hO) ? 1 : 0;
            } else {
                st.nNew = 2;
                b.bind(a.s.id);
                b.bind(a.o.id);
                st.hoWhich = !pairs ? 0 : (a.s.id == hO ? 1 : (a.o.id == hO ? 2 : 0));
            }
        }
        level[best] = lvl;
        order[nOrder++] = best;
        P.tupleLen[lvl] = b.tupleLen;
        add_checks(lvl);
    }
    P.m = lvl;

    // used-triple comparisons, attached where the later atom is grounded
    const Atom* seq[kMaxBody + 1];
    int seqLevel[kMaxBody + 1], nSeq = 0;
    if (head) { seq[nSeq] = head; seqLevel[nSeq++] = 0; }
    for (int k = 0; k < nOrder; ++k) { seq[nSeq] = &body[order[k]]; seqLevel[nSeq++] = level[order[k]]; }
    struct LevelUsed { int lvl; DevUsed u; };
    LevelUsed pairs_[(kMaxBody + 1) * kMaxBody / 2];
    int nPairs = 0;
    for (int j = 0; j < nSeq; ++j) {
        for (int i = 0; i < j; ++i) {
            const Atom& A = *seq[i];
            const Atom& B = *seq[j];
            if (A.pred != B.pred) continue;
            Rel rs = rel(A.s, B.s), ro = rel(A.o, B.o);
            if (rs == kNe || ro == kNe) continue;
            if (rs == kEq && ro == kEq) return false;
            pairs_[nPairs++] = LevelUsed{seqLevel[j], DevUsed{b.ref(A.s), b.ref(A.o), b.ref(B.s), b.ref(B.o)}};
        }
    }
    // per level, in the order found
    int nc = 0, nu = 0;
    for (int l = 0; l <= kMaxBody; ++l) {
        P.chkBeg[l] = (int8_t)nc;
        int cnt = 0;
        for (int k = 0; k < nFound; ++k) {
            if (found[k].lvl != l) continue;
            ++cnt;
            if (nc >= kMaxChecks) { b.ok = false; continue; }
            P.checks[nc++] = found[k].c;
        }
        P.chkN[l] = (int8_t)cnt;
        P.usedBeg[l] = (int8_t)nu;
        cnt = 0;
        for (int k = 0; k < nPairs; ++k) {
            if (pairs_[k].lvl != l) continue;
            ++cnt;
            if (nu >= kMaxUsed) { b.ok = false; continue; }
            P.used[nu++] = pairs_[k].u;
        }
        P.usedN[l] = (int8_t)cnt;
    }
    return true;
}

// Splits the block's shared pool between the frontier (levels 0..m-1, each
// `cap` items of tuple + stored segment) and the dedup bitmap: kExist keeps
// one bit per root of the task (at most 1024 roots); kPairs gives its bitmap
// rows up to half the pool (ceil(wo / 32) words per root), or none when one
// row does not fit next to a minimal frontier (the plan then deduplicates in
// a global bitmap).  Returns false in that last case.
// kExist plans whose last step expands x -> y (y new) and whose only test
// after it is one membership check between y and a bound value or
// constant h: whether some valid y exists is one bit of the suffix memo of
// (last step) -> (the check seen from y), see memo_exists in kernels.cu.
void exist_memo_eligibility(DevPlan& P) {
    if (P.mode != kExist || P.m < 1) return;
    const int k = P.m - 1;
    const DevStep& a = P.steps[k];
    if (a.kind != kExpand || a.nNew != 1 || P.usedN[k + 1] != 0 || P.chkN[k + 1] != 1) return;
    const DevCheck& c = P.checks[P.chkBeg[k + 1]];
    const TermRef y = (TermRef)P.tupleLen[k];
    TermRef hRef;
    int d2;
    if (c.s == y && c.o != y) { hRef = c.o; d2 = 0; }        // (y p h): h among y's objects
    else if (c.o == y && c.s != y) { hRef = c.s; d2 = 1; }   // (h p y): h among y's subjects
    else return;
    // h must be a variable: the memo never lets y equal h, which injectivity
    // forbids only between variables
    if (hRef < kTupleHead || hRef >= y) return;
    P.memoLevel = k + 1;
    P.memoP2 = c.pred;
    P.memoD2 = d2;
    P.memoH = hRef;
}

bool finish_capacity(DevPlan& P, const Geom& geom) {
    int sum = 0;
    if (P.m == 0) sum = P.tupleLen[0];
    for (int l = 0; l < P.m; ++l) sum += P.tupleLen[l] + 2;
    sum = std::max(sum, 1);
    const int pool = geom.poolInts();
    bool local = true;
    int bitmapInts = 0, groupMax = 0;
    if (P.mode == kPairs) {
        const int rowWords = std::max(1, (P.wo + 31) / 32);
        if ((int64_t)rowWords + 32LL * sum > pool) {
            local = false;
            groupMax = 512;
        } else {
            int g = std::max(1, std::min(1024, (pool / 2) / rowWords));
            while (g > 1 && pool - g * rowWords < 32 * sum) --g;
            bitmapInts = g * rowWords;
            groupMax = g;
        }
    } else {
        bitmapInts = 32;  // 1024 found bits
        groupMax = 1024;
    }
    P.cap = std::max(((pool - bitmapInts) / sum) & ~31, 32);
    P.bitmapOff = pool - bitmapInts;
    P.groupMax = std::min(groupMax, P.cap);
    P.rowWords = P.mode == kPairs ? std::max(1, (P.wo + 31) / 32) : 1;
    return local;
}

}  // namespace

RulePlan plan_rule(const Rule& rule, const HostIndex& ix, const Geom& geom) {
    RulePlan rp;
    const Atom& h = rule.head;
    int nb = (int)rule.body.size();
    // head measures (SupportCounting.cpp:482-503)
    if (h.pred >= 0 && h.pred < ix.nPred) {
        rp.headSize = ix.pred_size(h.pred);
        bool sC = !h.s.isVar, oC = !h.o.isVar;
        if (!sC && !oC) rp.headSupport = rp.headSize;
        else if (sC && !oC) { auto r = ix.row_range(h.pred, 0, h.s.id); rp.headSupport = r.second - r.first; }
        else if (!sC && oC) { auto r = ix.row_range(h.pred, 1, h.o.id); rp.headSupport = r.second - r.first; }
        else rp.headSupport = (h.s.id >= 0 && h.o.id >= 0 && ix.has_triple(h.pred, h.s.id, h.o.id)) ? 1 : 0;
    }
    if (nb > kMaxBody || rule.nVars > kMaxVars) {
        rp.status = kRuleUnsupported;
        rp.headSupport = rp.headSize;   // GPU_03/gpu_rules_lib.cu:345-357
        return rp;
    }
    bool bodyUnknown = false;
    for (const auto& a : rule.body) bodyUnknown |= has_unknown(a);
    bool bodyDup = false;   // two identical body atoms: no grounding at all
    for (int i = 0; i < nb; ++i)
        for (int j = i + 1; j < nb; ++j)
            if (rule.body[i].pred == rule.body[j].pred && rel(rule.body[i].s, rule.body[j].s) == kEq &&
                rel(rule.body[i].o, rule.body[j].o) == kEq)
                bodyDup = true;

    // ---- support ----
    PhasePlan& S = rp.support;
    S.how = kStatic;
    S.value = 0;
    if (h.pred >= 0 && rp.headSupport > 0 && !bodyUnknown && !bodyDup) {
        if (nb == 0) {
            // every matching head triple counts (bodyExists of an empty body)
            if (h.s.isVar && h.o.isVar) {
                int64_t n = 0;
                for (int32_t e = ix.predEdge[0][h.pred]; e < ix.predEdge[0][h.pred + 1]; ++e) {
                    bool eq = ix.src[0][e] == ix.val[0][e];
                    n += (h.s.id == h.o.id) ? eq : !eq;
                }
                S.value = n;
            } else {
                S.value = rp.headSupport;
            }
        } else {
            DevPlan& P = S.plan;
            std::memset(&P, 0, sizeof(P));
            Builder b(ix, P);
            P.mode = kExist;
            P.rootKind = kRootEdges;
            P.rootPred = h.pred;
            std::pair<int32_t, int32_t> range{ix.predEdge[0][h.pred], ix.predEdge[0][h.pred + 1]};
            if (h.s.isVar && h.o.isVar) {
                P.rootDir = 0;
                P.rootAppendKey = 1;
                b.bind(h.s.id);
                if (h.s.id == h.o.id) P.rootKeyEqVal = 1;
                else { P.rootAppendVal = 1; P.rootKeyNeVal = 1; b.bind(h.o.id); }
            } else if (!h.s.isVar && h.o.isVar) {
                P.rootDir = 0;
                range = ix.row_range(h.pred, 0, h.s.id);
                P.rootAppendVal = 1;
                b.bind(h.o.id);
            } else if (h.s.isVar && !h.o.isVar) {
                P.rootDir = 1;
                range = ix.row_range(h.pred, 1, h.o.id);
                P.rootAppendVal = 1;
                b.bind(h.s.id);
            } else {
                P.rootDir = 0;
                range = ix.row_range(h.pred, 0, h.s.id);
                P.rootValConst = b.ref(h.o);
            }
            if (build_steps(b, rule.body, &h, -1, false) && b.ok) {
                finish_capacity(P, geom);
                exist_memo_eligibility(P);
                S.how = kDevice;
                S.rootBeg = range.first;
                S.rootEnd = range.second;
                S.estCost = (double)(range.second - range.first);
            } else if (!b.ok) {
                rp.status = kRuleUnsupported;
            }
        }
    }

    // ---- body size ----
    PhasePlan& B = rp.body;
    B.how = kStatic;
    B.value = 0;
    if (nb > 0 && h.s.isVar && h.o.isVar && !bodyUnknown && !bodyDup) {
        int32_t hS = h.s.id, hO = h.o.id;
        int seedPred = -1, seedDir = 0;
        int64_t bestSize = std::numeric_limits<int32_t>::max();
        for (const auto& a : rule.body) {
            int64_t sz = ix.pred_size(a.pred);
            if (a.s.isVar && a.s.id == hS && sz < bestSize) { seedPred = a.pred; seedDir = 0; bestSize = sz; }
            if (a.o.isVar && a.o.id == hS && sz < bestSize) { seedPred = a.pred; seedDir = 1; bestSize = sz; }
        }
        bool hoInBody = false;
        for (const auto& a : rule.body)
            hoInBody |= (a.s.isVar && a.s.id == hO) || (a.o.isVar && a.o.id == hO);
        if (seedPred >= 0) {
            DevPlan& P = B.plan;
            std::memset(&P, 0, sizeof(P));
            Builder b(ix, P);
            bool pairs = hS != hO && hoInBody;
            P.mode = pairs ? kPairs : kExist;
            P.rootKind = kRootRows;
            P.rootDir = seedDir;
            P.rootPred = seedPred;
            b.bind(hS);
            if (build_steps(b, rule.body, nullptr, hO, pairs) && b.ok) {
                if (pairs) {
                    for (int l = 0; l < P.m; ++l) {
                        const DevStep& st = P.steps[l];
                        if (!st.hoWhich) continue;
                        P.hoLevel = l + 1;
                        if (st.kind == kExpand) P.wo = (int32_t)ix.pred_rows(st.pred, 1 - st.dir);
                        else P.wo = (int32_t)ix.pred_rows(st.pred, st.hoWhich == 1 ? 0 : 1);
                    }
                }
                const bool local = finish_capacity(P, geom);
                // suffix memo eligibility: the last two steps expand x -> y -> hO
                // (y bound by the first, keying the second) with no test at
                // either level but injectivity
                if (pairs && P.m >= 2) {
                    const int k = P.m - 2;
                    const DevStep& a = P.steps[k];
                    const DevStep& c = P.steps[k + 1];
                    if (a.kind == kExpand && a.nNew == 1 && a.hoWhich == 0 && c.kind == kExpand && c.nNew == 1 &&
                        c.hoWhich != 0 && c.keyRef == P.tupleLen[k] && P.chkN[k + 1] == 0 && P.usedN[k + 1] == 0 &&
                        P.chkN[k + 2] == 0 && P.usedN[k + 2] == 0) {
                        P.memoLevel = k + 1;
                        P.memoP2 = c.pred;
                        P.memoD2 = c.dir;
                    }
                }
                // three-step suffix memo: hS -> x, then x -> v2 -> v3 -> hO,
                // each step keyed by the value the one before bound, and no
                // test after x but injectivity; items (hS, x) whose x is a
                // memoised hub row are answered by memo3_item (kernels.cu)
                if (pairs && P.m == 4 && P.tupleLen[0] == kTupleHead + 1) {
                    bool ok = true;
                    for (int l = 0; l < 4 && ok; ++l) {
                        const DevStep& st = P.steps[l];
                        ok = st.kind == kExpand && st.nNew == 1 && st.keyRef == P.tupleLen[l] - 1 &&
                             (st.hoWhich != 0) == (l == 3);
                    }
                    for (int l = 2; l <= 4 && ok; ++l) ok = P.chkN[l] == 0 && P.usedN[l] == 0;
                    if (ok) {
                        P.memoLevel = 2;
                        P.memoP2 = P.steps[2].pred;
                        P.memoD2 = P.steps[2].dir;
                        P.memoSteps = 3;
                    }
                }
                B.how = kDevice;
                B.rootBeg = ix.predRow[seedDir][seedPred];
                B.rootEnd = ix.predRow[seedDir][seedPred + 1];
                B.needsGlobalBitmap = pairs && !local;
                B.estCost = (double)(ix.predEdge[seedDir][seedPred + 1] - ix.predEdge[seedDir][seedPred]);
            } else if (!b.ok) {
                rp.status = kRuleUnsupported;
            }
        }
    }
    if (rp.status != kRuleOk) {
        rp.support = PhasePlan{};
        rp.body = PhasePlan{};
        rp.headSupport = rp.headSize;
    } else if (S.how == kDevice && B.how == kDevice && h.s.isVar && h.o.isVar && h.s.id != h.o.id &&
               B.plan.mode == kPairs && B.plan.rootKind == kRootRows && B.plan.hoLevel >= 1) {
        // support from the body-size pairs: the support plan is the body
        // grounded from a head triple (a, b) with a != b, and with no
        // used-triple test the head triple never constrains it, so a head
        // triple has a grounding exactly when (a, b) is a body pair
        bool used = false;
        for (int l = 0; l <= kMaxBody; ++l) used |= S.plan.usedN[l] != 0;
        if (!used) rp.supFuse = h.pred;
    }
    return rp;
}

std::pair<int32_t, int32_t> ho_domain(const DevPlan& P) {
    const DevStep& st = P.steps[P.hoLevel - 1];
    if (st.kind == kExpand) return {st.pred, 1 - st.dir};
    return {st.pred, st.hoWhich == 1 ? 0 : 1};
}

}  // namespace gr
