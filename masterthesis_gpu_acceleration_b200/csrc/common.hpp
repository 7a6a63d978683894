// common.hpp — types shared by the host planner and the device engine.
//
// Limits follow the reference (GPU_03/gpu_common.cuh:25-27): at most 16
// distinct variables and 8 body atoms per rule.
#pragma once
#include <cstdint>
#ifndef __CUDACC__
#define __host__
#define __device__
#endif

namespace gr {

constexpr int kMaxVars = 16;
constexpr int kMaxBody = 8;
constexpr int kMaxConsts = 20;
constexpr int kTupleHead = 2;                  // [root index, hO rank]
constexpr int kMaxTuple = kTupleHead + kMaxVars;
constexpr int kMaxChecks = 16;
constexpr int kMaxUsed = 40;
constexpr int kMaxSupFused = 4;   // rules whose support one body-size plan counts

// One slot of the (predicate, direction, key) -> edge range table.
// tag = pred * 2 + dir; tag 0xffffffff marks an empty slot.
struct alignas(16) HashSlot {
    uint32_t tag, key, beg, end;
};
constexpr uint32_t kEmptyTag = 0xffffffffu;

__host__ __device__ inline uint32_t slot_hash(uint32_t tag, uint32_t key) {
    uint64_t x = ((uint64_t)tag << 32) | key;
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return (uint32_t)x;
}

// Bit of (pred, dir) in an entity's row signature: the signature of an
// entity has the bits of every (pred, dir) under which it keys a row, so a
// clear bit proves that the row is absent (a set bit may be a collision).
__host__ __device__ inline int sig_bit(int32_t pred, int dir) {
    return (int)(((uint32_t)pred * 2u + (uint32_t)dir) * 0x9E3779B1u >> 26);
}

// Device-resident graph index.  Triples are stored once per direction:
// dir 0 (SPO) keys edges by subject and stores objects as values, dir 1
// (POS) keys them by object and stores subjects.  Within a direction edges
// are sorted by (predicate, key, value), so each (predicate, key) row is a
// contiguous, sorted run of values.
struct DevIndex {
    // per direction, per edge
    const int32_t* val[2];       // neighbour value
    const int32_t* valRank[2];   // rank of the value among the predicate's distinct values
                                 // in that position (= its row index in the other direction)
    const int32_t* src[2];       // the edge's key
    const int32_t* srcRank[2];   // rank of the key among the predicate's keys in this direction
    // per direction, per row
    const int32_t* rowKey[2];
    const int32_t* rowBeg[2];    // rows + 1 entries (edge offsets)
    // per direction, per predicate
    const int32_t* predRow[2];   // P + 1 entries
    const int32_t* predEdge[2];  // P + 1 entries
    // (predicate, direction, key) -> edge range, open addressing
    const struct HashSlot* hash;
    // hub rows (rows whose values also exist as a rank bitmap)
    const int32_t* hubOf[2];     // per row: hub index or -1
    const int64_t* hubOff;       // per hub: first word in hubBits
    const uint32_t* hubBits;
    // per direction, per edge: the row signature of the edge's value, and
    // the union of those signatures from the edge to the end of its row
    const uint64_t* valSig[2];
    const uint64_t* sufSig[2];
    int32_t nHub;
    uint32_t hashMask;
    int32_t nPred;
    int32_t nEnt;
    int64_t nTriples;
};

// Term reference inside a plan: r >= 0 is a tuple position; r < 0 is
// constant number (-1 - r).
using TermRef = int16_t;

struct DevCheck {        // membership filter: the triple (s, pred, o) must exist
    int32_t pred;
    TermRef s, o;
    int8_t dir;          // direction probed (0: key = s, 1: key = o)
    int8_t pad[3];
};

struct DevUsed {         // used-triple rule: reject when the two triples are equal
    TermRef sA, oA, sB, oB;
};

enum StepKind : int8_t { kExpand = 0, kScan = 1 };

struct DevStep {
    int32_t pred;
    int8_t dir;          // EXPAND: direction of the lookup; SCAN: always 0
    int8_t kind;
    int8_t sameVar;      // SCAN with one variable in both positions
    int8_t nNew;         // values appended to the tuple (1 or 2)
    TermRef keyRef;      // EXPAND: the bound key
    int8_t hoWhich;      // 0: hO not bound here; 1/2: hO is the first/second new value
    int8_t pad;
};

enum PlanMode : int32_t { kExist = 0, kPairs = 1 };
enum RootKind : int32_t { kRootEdges = 0, kRootRows = 1 };

// One phase (support or body size) of one rule.
// Every byte of a plan belongs to a field (explicit pads, no implicit
// padding), so that equal plans compare and hash equal after any copy.
struct DevPlan {
    int32_t mode;            // kExist: count roots with a grounding; kPairs: count distinct (root, hO)
    int32_t m;               // binding steps
    int32_t resultSlot;      // index into the u64 result array
    int32_t rootKind;        // kRootEdges: edges of rootDir in [task.beg, task.end)
                             // kRootRows: rows of rootDir in [task.beg, task.end), hS = row key
    int32_t rootDir;
    int32_t rootPred;
    int8_t rootAppendKey;    // edges: append the edge key to the tuple
    int8_t rootAppendVal;    // edges: append the edge value
    int8_t rootKeyEqVal;     // edges: require key == value
    int8_t rootKeyNeVal;     // edges: require key != value
    TermRef rootValConst;    // edges: require value == constant (-1 - k), or 0 for none
    int16_t pad0;
    // filters per level (level 0 = roots, level l = after step l)
    int8_t chkBeg[kMaxBody + 1], chkN[kMaxBody + 1];
    int8_t usedBeg[kMaxBody + 1], usedN[kMaxBody + 1];
    int32_t wo;              // kPairs: bitmap row width (size of hO's value domain)
    int32_t bitmapOff;       // where the dedup bitmap starts in the block's shared pool (ints)
    int32_t hoLevel;         // kPairs: level whose step binds hO (1..m)
    int32_t cap;             // frontier capacity per level (items)
    int32_t groupMax;        // max roots per task
    int32_t tupleLen[kMaxBody + 1];
    int32_t consts[kMaxConsts];
    DevStep steps[kMaxBody];
    DevCheck checks[kMaxChecks];
    DevUsed used[kMaxUsed];
    int32_t pad1;                 // explicit: plans are compared and hashed byte by byte
    uint32_t* gBitmap;            // kPairs with a global bitmap (null: shared memory)
    int64_t gRowBase;             // first root of the plan, for global bitmap rows
    uint32_t* gHeavy;             // global dedup rows of split heavy roots
    int32_t rowWords;             // words per heavy row (kPairs: ceil(wo / 32); kExist: 1)
    int32_t memoLevel;            // level + 1 whose items may use a suffix memo (0: none): kPairs
                                  // plans ending in two expand steps x -> y -> hO (memo_item),
                                  // kExist plans ending in x -> y and the check (h, y) (memo_exists)
    int32_t memoP2, memoD2;       // the memo's second relation: y -> h through (memoP2, memoD2) rows
    TermRef memoH;                // kExist: tuple ref of h
    int8_t memoSteps;             // kPairs: 3 for a three-step suffix memo x -> v2 -> v3 -> hO (memo3_item),
                                  // otherwise the two-step one
    int8_t pad2;
    int32_t memoWords;            // words per memo bitmap (the rows of (memoP2, 1 - memoD2))
    const int32_t* memoTab;       // per hub row: memo slot or -1 (null: no memo)
    const uint32_t* memoBits;     // per slot: S1 then S2, memoWords words each
    // kPairs deduplication outside the shared pool (per launch; see DedupMode):
    int64_t gBlockWords;          // > 0: block rows, each block owns gBitmap + blockIdx.x * gBlockWords
                                  // words for its current task's rows (cleared at task start)
    unsigned long long* pairKeys;   // non-null: sort mode, keys keyBase | row << rankBits | rank appended
    unsigned long long* keyCursor;  // sort mode: append cursor (keeps counting past keyCap)
    unsigned long long keyCap;      // sort mode: capacity of pairKeys
    unsigned long long keyBase;     // sort mode: the plan's key prefix (its sort index, shifted)
    int32_t rankBits;               // sort mode: bits of the hO rank field
    int32_t pad3;
    // Fused support (kPairs plans with rows in shared memory or block rows):
    // for j < supN, results[supSlot[j]] gains the number of head triples
    // (hS, supPred[j], b), b != hS, whose pair (hS, b) the plan's rows hold;
    // b's rank is that of its row in (supDomPred, supDomDir), hO's domain.
    int32_t supN;
    int32_t supDomPred, supDomDir;
    int32_t supPred[kMaxSupFused];
    int32_t supSlot[kMaxSupFused];
    int32_t pad4;
    // Hub items of the leaf (see kHubSeen): per resident block kHubSeen
    // claim entries at hubSeen + blockIdx.x * kHubSeen (null: every hub item
    // is OR-ed).  Set for plans whose leaf items are (hS, u, w) expanding
    // from u or w with nothing to test but injectivity.
    unsigned long long* hubSeen;
};

// Leaf hub items of one root and one hub row differ only in the one bound
// value that is neither the root nor the row key (the middle value), and
// each excludes only its own bound values from the row: two items with
// different middle values already cover every value any further one would
// add.  A task claims its (root, hub) pairs in a direct-mapped table of
// kHubSeen 64-bit entries [root 10 bits | hub 20 | state 2 | first middle
// value 32] (state 1: one middle value seen, 2: two) and skips the items
// that come after two different middle values.  The same item may come
// twice (a wide round makes some items again); it never counts as a second
// value, and a displaced entry only costs repeats.
constexpr int kHubSeenBits = 8;
constexpr int kHubSeen = 1 << kHubSeenBits;

// A split heavy root of a plan with fused support: its global row gRow is
// complete only after the launch, when support_rows_kernel counts it.
struct SupJob {
    int32_t plan, root, gRow, pad;
};

// How a kPairs phase deduplicates its (hS row, hO rank) pairs.
enum DedupMode : int32_t {
    kDedupShared = 0,     // bitmap rows in the block's shared pool (the task's roots)
    kDedupRows = 1,       // one global bitmap row per root of the phase, cleared before the launch
    kDedupBlockRows = 2,  // global rows per resident block for its current task, cleared by the block
    kDedupSort = 3,       // 64-bit pair keys appended, radix-sorted and counted once each
};

// A unit of device work: the roots [beg, end) of one plan.  A heavy root is
// split over several tasks (gRow >= 0, end == beg + 1): each takes the slice
// [sub0, sub1) of the root's first neighbour segment and deduplicates into
// the plan's global row gRow, so the slices together count each pair (or
// the root) once.
struct DevTask {
    int32_t plan;
    int32_t beg, end;        // root range
    int32_t sub0, sub1;      // heavy root: slice of the first segment
    int32_t gRow;            // heavy root: global dedup row, else -1
};

// Engine launch geometry: block size B (128, 256 or 512 threads) with a
// shared-memory pool of 48 ints per thread that each plan splits between
// its frontier levels and its dedup bitmap, so 1024 / B blocks stay
// resident per SM.
struct Geom {
    int block = 256;
    static constexpr int pool_for(int b) { return 48 * b; }
    int poolInts() const { return pool_for(block); }
};

// Profiling outputs of the instrumented kernel variant (null members are
// skipped): requested global-memory bytes, and per task its start and end
// time (globaltimer ns).
// One suffix memo to build for hub row `row` of (p1, d1), or the part that
// starts from the row's values [b0, b1) (b1 < 0: all of them; the parts of
// one memo add into the same bits).  Two steps (p3 < 0): through (p2, d2),
// bitmaps S1 then S2 of `words` words at `bits`.  Three steps: through
// (p2, d2) then (p3, d3), the bitmap S1 (`words` words) then one path count
// per rank of the domain (`wo` ranks), a byte each (four to a word) that
// saturates at 255.
struct MemoJob {
    int32_t p1, d1, p2, d2, row, words;
    int32_t p3, d3, wo, b0, b1, pad;
    uint32_t* bits;
};
// Three-step memo parts count paths in shared memory (one 32-bit counter
// per rank) when the domain has at most this many ranks.
constexpr int kMemoSmemRanks = 16384;

struct EngineProfile {
    unsigned long long* bytes = nullptr;
    unsigned long long* taskNs = nullptr;
    // Launch span (any variant): span[0] = max of ~start over blocks (so a
    // zeroed word works as the initial value), span[1] = max block end,
    // both in device global-timer ns.
    unsigned long long* span = nullptr;
    // Served launches: a device-time budget in ns from each block's start
    // (0: none), after which blocks abandon the task they run and skip the
    // rest; incomplete[plan] is set for every plan that lost a task.
    unsigned long long budgetNs = 0;
    int* incomplete = nullptr;
};

}  // namespace gr
