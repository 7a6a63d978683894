/* rules_oracle.c — CPU restatement of the reference's rule-counting semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine:
 * only the tests, the smoke check and the CPU-baseline leg of the benchmark
 * load it.  The engine never calls it and has no CPU fallback.
 *
 * It restates, in plain C, the semantics of the reference's optimised CPU
 * implementation (CPU_01_nonparallel), which is the primary oracle:
 *
 *   index      per predicate: sorted, de-duplicated (s,o) pairs plus a
 *              key-compressed CSR in both directions
 *              (CPU_01_nonparallel/RdfIndexes.cpp:91-168, PredIndex)
 *   Env        variable bindings v[16] (0 = unbound, id+1 = bound) and the
 *              list of ground triples already used by the current grounding
 *              (CPU_01_nonparallel/SupportCounting.hpp:29-58)
 *   head match injective head binding (SupportCounting.cpp:9-34)
 *   scoring    greedy choice of the atom with the fewest live candidates
 *              (SupportCounting.cpp:38-79)
 *   dfsExists  existence search (SupportCounting.cpp:83-247)
 *   dfsEnum    enumeration with the early prune on known (hS,hO) pairs
 *              (SupportCounting.cpp:272-445)
 *   support    SupportCounting.cpp:474-552
 *   bodySize   SupportCounting.cpp:563-631 (always computed, as CPU_01 does)
 *
 * Counts are kept in 64 bits; the reference stores them in `int`.
 *
 * Rule input ("rule IR", int32 stream per rule):
 *   nb, head(p,sK,sV,oK,oV), body(p,sK,sV,oK,oV) * nb
 * K = 0: variable with dense id V (< 16); K = 1: constant entity id V.
 * A predicate outside [0, nPred) or a negative constant matches nothing,
 * which is what an interned-but-absent term does in the reference
 * (RuleParser.cpp:240-242, RdfIndexes.cpp:186-189).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_MAX_VARS 16   /* SupportCounting.hpp:21 */
#define OR_MAX_USED 9    /* SupportCounting.hpp:22 */
#define OR_MAX_BODY 8

typedef struct { int32_t a, b; } Pair;

typedef struct {
    int32_t* keys; int32_t* off; int32_t* vals; int nkeys;
} Csr;

typedef struct {
    Pair* spo; int n;     /* sorted unique (s,o) */
    Csr fwd;              /* subject -> objects */
    Csr rev;              /* object  -> subjects */
} PredIdx;

typedef struct {
    int nPred;
    PredIdx* preds;
} OracleGraph;

typedef struct { int p, sK, sV, oK, oV; } OAtom;

typedef struct { int s, p, o; } Used;

typedef struct {
    int v[OR_MAX_VARS];
    Used used[OR_MAX_USED + 1];
    int usedCount;
} Env;

/* ── index build (RdfIndexes.cpp:91-138) ─────────────────────────────── */

static int cmp_pair(const void* x, const void* y) {
    const Pair* a = (const Pair*)x; const Pair* b = (const Pair*)y;
    if (a->a != b->a) return a->a < b->a ? -1 : 1;
    if (a->b != b->b) return a->b < b->b ? -1 : 1;
    return 0;
}

static int sort_unique(Pair* p, int n) {
    if (n == 0) return 0;
    qsort(p, (size_t)n, sizeof(Pair), cmp_pair);
    int w = 1;
    for (int i = 1; i < n; ++i)
        if (p[i].a != p[w - 1].a || p[i].b != p[w - 1].b) p[w++] = p[i];
    return w;
}

static void build_csr(const Pair* sorted, int n, Csr* c) {
    c->keys = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    c->off = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 2));
    c->vals = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    int k = 0, i = 0;
    while (i < n) {
        int key = sorted[i].a;
        c->keys[k] = key;
        c->off[k] = i;
        ++k;
        while (i < n && sorted[i].a == key) { c->vals[i] = sorted[i].b; ++i; }
    }
    c->off[k] = n;
    c->nkeys = k;
}

OracleGraph* oracle_graph_build(const int32_t* spo, int64_t nTriples, int nPred) {
    OracleGraph* g = (OracleGraph*)calloc(1, sizeof(OracleGraph));
    g->nPred = nPred;
    g->preds = (PredIdx*)calloc((size_t)(nPred > 0 ? nPred : 1), sizeof(PredIdx));
    int* cnt = (int*)calloc((size_t)(nPred > 0 ? nPred : 1), sizeof(int));
    for (int64_t i = 0; i < nTriples; ++i) {
        int p = spo[3 * i + 1];
        if (p >= 0 && p < nPred) cnt[p]++;
    }
    for (int p = 0; p < nPred; ++p) {
        g->preds[p].spo = (Pair*)malloc(sizeof(Pair) * (size_t)(cnt[p] + 1));
        g->preds[p].n = 0;
    }
    for (int64_t i = 0; i < nTriples; ++i) {
        int p = spo[3 * i + 1];
        if (p < 0 || p >= nPred) continue;
        PredIdx* pi = &g->preds[p];
        pi->spo[pi->n].a = spo[3 * i];
        pi->spo[pi->n].b = spo[3 * i + 2];
        pi->n++;
    }
    for (int p = 0; p < nPred; ++p) {
        PredIdx* pi = &g->preds[p];
        pi->n = sort_unique(pi->spo, pi->n);
        build_csr(pi->spo, pi->n, &pi->fwd);
        Pair* r = (Pair*)malloc(sizeof(Pair) * (size_t)(pi->n + 1));
        for (int i = 0; i < pi->n; ++i) { r[i].a = pi->spo[i].b; r[i].b = pi->spo[i].a; }
        int m = sort_unique(r, pi->n);
        build_csr(r, m, &pi->rev);
        free(r);
    }
    free(cnt);
    return g;
}

void oracle_graph_free(OracleGraph* g) {
    if (!g) return;
    for (int p = 0; p < g->nPred; ++p) {
        PredIdx* pi = &g->preds[p];
        free(pi->spo);
        free(pi->fwd.keys); free(pi->fwd.off); free(pi->fwd.vals);
        free(pi->rev.keys); free(pi->rev.off); free(pi->rev.vals);
    }
    free(g->preds);
    free(g);
}

static const PredIdx* get_pred(const OracleGraph* g, int p) {
    if (p < 0 || p >= g->nPred) return NULL;
    return &g->preds[p];
}

/* spoRange / posRange (RdfIndexes.cpp:140-160): binary search on the keys */
static const int32_t* csr_range(const Csr* c, int key, int* count) {
    int lo = 0, hi = c->nkeys;
    while (lo < hi) {
        int m = (lo + hi) >> 1;
        if (c->keys[m] < key) lo = m + 1; else hi = m;
    }
    if (lo == c->nkeys || c->keys[lo] != key) { *count = 0; return NULL; }
    *count = c->off[lo + 1] - c->off[lo];
    return c->vals + c->off[lo];
}

/* hasTriple (RdfIndexes.cpp:162-168) */
static int has_triple(const PredIdx* pi, int s, int o) {
    int cnt = 0;
    const int32_t* objs = csr_range(&pi->fwd, s, &cnt);
    if (!objs) return 0;
    int lo = 0, hi = cnt;
    while (lo < hi) {
        int m = (lo + hi) >> 1;
        if (objs[m] < o) lo = m + 1; else hi = m;
    }
    return lo < cnt && objs[lo] == o;
}

/* ── Env (SupportCounting.hpp:29-58) ─────────────────────────────────── */

static inline int env_bound(const Env* e, int var) { return e->v[var] != 0; }
static inline int env_resolve(const Env* e, int var) { return e->v[var] - 1; }
static inline void env_bind(Env* e, int var, int c) { e->v[var] = c + 1; }
static inline int env_contains_value(const Env* e, int c) {
    int enc = c + 1;
    for (int i = 0; i < OR_MAX_VARS; ++i) if (e->v[i] == enc) return 1;
    return 0;
}
static inline int env_contains_atom(const Env* e, int s, int p, int o) {
    for (int i = 0; i < e->usedCount; ++i)
        if (e->used[i].s == s && e->used[i].p == p && e->used[i].o == o) return 1;
    return 0;
}
static inline void env_push(Env* e, int s, int p, int o) {
    e->used[e->usedCount].s = s; e->used[e->usedCount].p = p; e->used[e->usedCount].o = o;
    e->usedCount++;
}

static inline int term_bound(const Env* e, int k, int v) { return k == 1 || env_bound(e, v); }
static inline int term_value(const Env* e, int k, int v) { return k == 1 ? v : env_resolve(e, v); }

/* matchHeadAtom (SupportCounting.cpp:9-34) */
static int match_head(const OAtom* h, int s, int o, Env* e) {
    if (h->sK == 0 && h->oK == 0 && h->sV != h->oV && s == o) return 0;
    if (h->sK == 1) { if (h->sV != s) return 0; }
    else env_bind(e, h->sV, s);
    if (h->oK == 1) { if (h->oV != o) return 0; }
    else {
        if (env_bound(e, h->oV)) { if (env_resolve(e, h->oV) != o) return 0; }
        else { if (env_contains_value(e, o)) return 0; env_bind(e, h->oV, o); }
    }
    return 1;
}

/* scoreAtom / chooseBestAtom (SupportCounting.cpp:38-79) */
static int score_atom(const OracleGraph* g, const OAtom* a, const Env* e) {
    int sB = term_bound(e, a->sK, a->sV), oB = term_bound(e, a->oK, a->oV);
    const PredIdx* pi = get_pred(g, a->p);
    if (!pi) return 0;
    if (sB && oB) return has_triple(pi, term_value(e, a->sK, a->sV), term_value(e, a->oK, a->oV));
    int cnt = 0;
    if (sB) { csr_range(&pi->fwd, term_value(e, a->sK, a->sV), &cnt); return cnt; }
    if (oB) { csr_range(&pi->rev, term_value(e, a->oK, a->oV), &cnt); return cnt; }
    return pi->n;
}

static int choose_best(const OracleGraph* g, const OAtom* body, int n, unsigned remaining, const Env* e) {
    int best = -1, bestScore = 0;
    for (int i = 0; i < n; ++i) {
        if (!(remaining & (1u << i))) continue;
        int sc = score_atom(g, &body[i], e);
        if (best < 0 || sc < bestScore) { best = i; bestScore = sc; }
    }
    return best;
}

/* ── per-headS set of headO values (PairSet in SupportCounting.hpp:11-18,
 *    restricted to one headS as countBodySize uses it) ─────────────────── */

typedef struct {
    int32_t* key; uint32_t* gen; uint32_t cap, size, cur;
} IntSet;

static void set_init(IntSet* s) {
    s->cap = 1024; s->size = 0; s->cur = 1;
    s->key = (int32_t*)malloc(sizeof(int32_t) * s->cap);
    s->gen = (uint32_t*)calloc(s->cap, sizeof(uint32_t));
}
static void set_free(IntSet* s) { free(s->key); free(s->gen); }
static void set_clear(IntSet* s) {
    s->size = 0;
    if (++s->cur == 0) { memset(s->gen, 0, sizeof(uint32_t) * s->cap); s->cur = 1; }
}
static inline uint32_t set_hash(int32_t k) { uint32_t x = (uint32_t)k * 0x9E3779B1u; return x ^ (x >> 15); }
static int set_has(const IntSet* s, int32_t k) {
    uint32_t m = s->cap - 1, i = set_hash(k) & m;
    while (s->gen[i] == s->cur) { if (s->key[i] == k) return 1; i = (i + 1) & m; }
    return 0;
}
static void set_grow(IntSet* s);
static int set_insert(IntSet* s, int32_t k) {
    if ((s->size + 1) * 2 > s->cap) set_grow(s);
    uint32_t m = s->cap - 1, i = set_hash(k) & m;
    while (s->gen[i] == s->cur) { if (s->key[i] == k) return 0; i = (i + 1) & m; }
    s->gen[i] = s->cur; s->key[i] = k; s->size++;
    return 1;
}
static void set_grow(IntSet* s) {
    uint32_t oc = s->cap, ocur = s->cur;
    int32_t* ok = s->key; uint32_t* og = s->gen;
    s->cap = oc * 2; s->size = 0; s->cur = 1;
    s->key = (int32_t*)malloc(sizeof(int32_t) * s->cap);
    s->gen = (uint32_t*)calloc(s->cap, sizeof(uint32_t));
    for (uint32_t i = 0; i < oc; ++i) if (og[i] == ocur) set_insert(s, ok[i]);
    free(ok); free(og);
}

/* ── DFS (SupportCounting.cpp:83-247 and 272-445) ─────────────────────
 * One routine serves both searches.  In existence mode it returns 1 on
 * the first complete grounding.  In enumeration mode it inserts the
 * resolved headO value of every complete grounding into `set` (headS is
 * fixed by the caller) and skips a subtree once headO is bound to a value
 * already in the set (SupportCounting.cpp:284-290). */

typedef struct {
    const OracleGraph* g;
    const OAtom* body;
    int n;
    int enumerate;
    int hO;
    IntSet* set;
} Dfs;

static int dfs(const Dfs* d, unsigned remaining, Env* e, int matched);

/* Tries binding (s,o) for `a`; recurses; restores.  Returns the recursion's
 * result (0 when the candidate is rejected). */
static int try_ground(const Dfs* d, const OAtom* a, unsigned nextRem, Env* e, int matched,
                      int s, int o) {
    int sVar = -1, oVar = -1, savedS = 0, savedO = 0;
    if (a->sK == 0) {
        if (env_bound(e, a->sV)) { if (env_resolve(e, a->sV) != s) return 0; }
        else {
            if (env_contains_value(e, s)) return 0;
            sVar = a->sV; savedS = e->v[sVar]; env_bind(e, sVar, s);
        }
    }
    if (a->oK == 0) {
        if (env_bound(e, a->oV)) {
            if (env_resolve(e, a->oV) != o) { if (sVar >= 0) e->v[sVar] = savedS; return 0; }
        } else {
            if (env_contains_value(e, o)) { if (sVar >= 0) e->v[sVar] = savedS; return 0; }
            oVar = a->oV; savedO = e->v[oVar]; env_bind(e, oVar, o);
        }
    }
    if (env_contains_atom(e, s, a->p, o)) {
        if (oVar >= 0) e->v[oVar] = savedO;
        if (sVar >= 0) e->v[sVar] = savedS;
        return 0;
    }
    env_push(e, s, a->p, o);
    int r = dfs(d, nextRem, e, matched + 1);
    e->usedCount--;
    if (oVar >= 0) e->v[oVar] = savedO;
    if (sVar >= 0) e->v[sVar] = savedS;
    return r;
}

static int dfs(const Dfs* d, unsigned remaining, Env* e, int matched) {
    if (matched == d->n) {
        if (d->enumerate) { set_insert(d->set, env_resolve(e, d->hO)); return 0; }
        return 1;
    }
    if (d->enumerate && env_bound(e, d->hO) && set_has(d->set, env_resolve(e, d->hO))) return 0;

    int best = choose_best(d->g, d->body, d->n, remaining, e);
    if (best < 0) return 0;
    const OAtom* a = &d->body[best];
    unsigned nextRem = remaining & ~(1u << best);
    const PredIdx* pi = get_pred(d->g, a->p);
    if (!pi) return 0;
    int sB = term_bound(e, a->sK, a->sV), oB = term_bound(e, a->oK, a->oV);

    if (sB && oB) {   /* Case 1 */
        int s = term_value(e, a->sK, a->sV), o = term_value(e, a->oK, a->oV);
        if (!has_triple(pi, s, o)) return 0;
        if (env_contains_atom(e, s, a->p, o)) return 0;
        env_push(e, s, a->p, o);
        int r = dfs(d, nextRem, e, matched + 1);
        e->usedCount--;
        return r;
    }
    if (sB) {         /* Case 2 */
        int s = term_value(e, a->sK, a->sV), cnt = 0;
        const int32_t* objs = csr_range(&pi->fwd, s, &cnt);
        for (int i = 0; i < cnt; ++i)
            if (try_ground(d, a, nextRem, e, matched, s, objs[i]) && !d->enumerate) return 1;
        return 0;
    }
    if (oB) {         /* Case 3 */
        int o = term_value(e, a->oK, a->oV), cnt = 0;
        const int32_t* subjs = csr_range(&pi->rev, o, &cnt);
        for (int i = 0; i < cnt; ++i)
            if (try_ground(d, a, nextRem, e, matched, subjs[i], o) && !d->enumerate) return 1;
        return 0;
    }
    /* Case 4: neither bound — scan every pair of the predicate */
    for (int i = 0; i < pi->n; ++i) {
        int s = pi->spo[i].a, o = pi->spo[i].b;
        if (a->sK == 0 && a->oK == 0 && a->sV != a->oV && s == o) continue;
        if (try_ground(d, a, nextRem, e, matched, s, o) && !d->enumerate) return 1;
    }
    return 0;
}

static int body_exists(const OracleGraph* g, const OAtom* body, int n, Env* e) {
    if (n == 0) return 1;
    Dfs d = { g, body, n, 0, 0, NULL };
    return dfs(&d, (1u << n) - 1u, e, 0);
}

static void env_init(Env* e) { memset(e, 0, sizeof(*e)); }

/* countSupport (SupportCounting.cpp:474-552) */
static int64_t count_support(const OracleGraph* g, const OAtom* head, const OAtom* body, int nb,
                             int64_t* headSize, int64_t* headSupport) {
    const PredIdx* pi = get_pred(g, head->p);
    if (!pi) { *headSize = 0; *headSupport = 0; return 0; }
    *headSize = pi->n;
    int sB = head->sK == 1, oB = head->oK == 1, cnt = 0;
    int64_t hsup;
    if (!sB && !oB) hsup = pi->n;
    else if (sB && !oB) { csr_range(&pi->fwd, head->sV, &cnt); hsup = cnt; }
    else if (!sB && oB) { csr_range(&pi->rev, head->oV, &cnt); hsup = cnt; }
    else hsup = has_triple(pi, head->sV, head->oV);
    *headSupport = hsup;
    if (hsup == 0) return 0;

    int64_t support = 0;
    Env e;
#define OR_PROCESS(S, O) do { env_init(&e); \
        if (match_head(head, (S), (O), &e)) { env_push(&e, (S), head->p, (O)); \
            if (body_exists(g, body, nb, &e)) ++support; } } while (0)
    if (sB && oB) {
        if (has_triple(pi, head->sV, head->oV)) OR_PROCESS(head->sV, head->oV);
    } else if (sB) {
        const int32_t* objs = csr_range(&pi->fwd, head->sV, &cnt);
        for (int i = 0; i < cnt; ++i) OR_PROCESS(head->sV, objs[i]);
    } else if (oB) {
        const int32_t* subjs = csr_range(&pi->rev, head->oV, &cnt);
        for (int i = 0; i < cnt; ++i) OR_PROCESS(subjs[i], head->oV);
    } else {
        for (int i = 0; i < pi->n; ++i) OR_PROCESS(pi->spo[i].a, pi->spo[i].b);
    }
#undef OR_PROCESS
    return support;
}

/* countBodySize (SupportCounting.cpp:563-631) */
static int64_t count_body_size(const OracleGraph* g, const OAtom* head, const OAtom* body, int nb) {
    if (nb == 0 || head->sK == 1 || head->oK == 1) return 0;
    int hS = head->sV, hO = head->oV;
    const PredIdx* seed = NULL;
    int seedIsSubj = 1;
    int bestSize = 0x7fffffff;
    for (int i = 0; i < nb; ++i) {
        const PredIdx* pi = get_pred(g, body[i].p);
        if (!pi) continue;
        if (body[i].sK == 0 && body[i].sV == hS && pi->n < bestSize) { seed = pi; seedIsSubj = 1; bestSize = pi->n; }
        if (body[i].oK == 0 && body[i].oV == hS && pi->n < bestSize) { seed = pi; seedIsSubj = 0; bestSize = pi->n; }
    }
    if (!seed) return 0;
    const Csr* cand = seedIsSubj ? &seed->fwd : &seed->rev;
    int64_t total = 0;
    IntSet set;
    set_init(&set);
    Dfs d = { g, body, nb, 1, hO, &set };
    for (int k = 0; k < cand->nkeys; ++k) {
        Env e;
        env_init(&e);
        env_bind(&e, hS, cand->keys[k]);
        if (hS == hO) {
            if (body_exists(g, body, nb, &e)) total++;
        } else {
            set_clear(&set);
            dfs(&d, (1u << nb) - 1u, &e, 0);
            total += set.size;
        }
    }
    set_free(&set);
    return total;
}

/* Evaluates nRules rules from the IR stream.  Rules with more than 8 body
 * atoms or a variable id >= 16 are reported as unsupported (status 1) with
 * zero measures, which is what the reference library returns for them
 * (GPU_03/gpu_rules_lib.cu:352-357).  out4 receives per rule:
 * support, headSize, headSupport, bodySize.  Returns 0, or -1 on a
 * malformed stream. */
int oracle_eval_rules(const OracleGraph* g, const int32_t* ir, int64_t irLen, int nRules,
                      int64_t* out4, int32_t* status) {
    int64_t pos = 0;
    for (int r = 0; r < nRules; ++r) {
        if (pos + 6 > irLen) return -1;
        int nb = ir[pos];
        if (nb < 0 || pos + 6 + 5LL * nb > irLen) return -1;
        OAtom head, body[OR_MAX_BODY];
        const int32_t* h = ir + pos + 1;
        head.p = h[0]; head.sK = h[1]; head.sV = h[2]; head.oK = h[3]; head.oV = h[4];
        int ok = nb <= OR_MAX_BODY;
        int maxVar = -1;
#define OR_TRACK(K, V) do { if ((K) == 0) { if ((V) < 0) ok = 0; if ((V) > maxVar) maxVar = (V); } } while (0)
        OR_TRACK(head.sK, head.sV); OR_TRACK(head.oK, head.oV);
        for (int i = 0; ok && i < nb; ++i) {
            const int32_t* a = ir + pos + 6 + 5 * i;
            body[i].p = a[0]; body[i].sK = a[1]; body[i].sV = a[2]; body[i].oK = a[3]; body[i].oV = a[4];
            OR_TRACK(body[i].sK, body[i].sV); OR_TRACK(body[i].oK, body[i].oV);
        }
#undef OR_TRACK
        if (maxVar >= OR_MAX_VARS) ok = 0;
        int64_t* o = out4 + 4 * (int64_t)r;
        if (!ok) {
            const PredIdx* pi = get_pred(g, head.p);
            o[0] = 0; o[1] = pi ? pi->n : 0; o[2] = o[1]; o[3] = 0;
            status[r] = 1;
        } else {
            int64_t hsz = 0, hsup = 0;
            o[0] = count_support(g, &head, body, nb, &hsz, &hsup);
            o[1] = hsz; o[2] = hsup;
            o[3] = count_body_size(g, &head, body, nb);
            status[r] = 0;
        }
        pos += 6 + 5LL * nb;
    }
    return 0;
}
