/* gpu_rules_api.h — C ABI of libgpu_rules.so (B200 engine).
 *
 * Drop-in replacement for the reference library's interface
 * (GPU_03/gpu_rules_api.h): the five reference entry points keep their
 * names, argument meaning, return codes and the result struct layout, so
 * the existing Scala/JNA binding (GPU_03/GpuRulesLib.scala:23-58) loads this
 * library unchanged.  The remaining entry points are additive.
 *
 * Counting semantics are those of the reference's CPU implementation
 * (CPU_01_nonparallel/SupportCounting.cpp): injective variable bindings, no
 * ground triple used twice in one grounding (the head triple included for
 * support), and the body size always computed.
 */
#ifndef GPU_RULES_API_H
#define GPU_RULES_API_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Result of one rule.  Same fields, order and natural alignment as the
 * reference (GPU_03/gpu_rules_api.h:21-30): 56 bytes on x86-64 with offsets
 * 0, 4, 8, 16, 24, 32, 40, 48.  Counts above INT_MAX saturate at INT_MAX. */
typedef struct {
    int    support;       /* head triples whose body has a grounding          */
    int    headSize;      /* triples of the head predicate                     */
    int    headSupport;   /* head triples matching the head's constants        */
    double headCoverage;  /* support / headSize (0 when headSize is 0)         */
    int    bodySize;      /* distinct (hS, hO) pairs with a body grounding     */
    double confidence;    /* support / bodySize (0 when bodySize is 0)         */
    double supportMs;     /* device time of the support phase (ms); 0 when the */
                          /* body-size launch counted the support too          */
    double confidenceMs;  /* device time of the body-size phase (ms)           */
} GpuRuleResult;

/* Replaces gpu_load_graph (GPU_03/gpu_rules_api.h:43).
 * Parses the Turtle file, builds the index and keeps it resident on the
 * current CUDA device.  Returns an opaque context, or NULL on a parse,
 * memory or CUDA error (the process is never terminated). */
void* gpu_load_graph(const char* ttlPath);

/* Replaces gpu_evaluate_rule (GPU_03/gpu_rules_api.h:59).
 * Evaluates one rule in the text syntax, e.g.
 *   "(?a <http://ex/livesIn> ?b) => (?a <http://ex/bornIn> ?b)"
 * One device launch per phase.  Returns 0 on success (also for rules the
 * engine does not support: more than 8 body atoms or 16 variables, which
 * yield zero measures except headSize/headSupport, as in the reference),
 * -1 on null arguments, a malformed rule or a CUDA error.
 * Not thread-safe within one context; distinct contexts are independent. */
int gpu_evaluate_rule(void* ctx, const char* ruleText, GpuRuleResult* out);

/* Replaces gpu_evaluate_rule_json (GPU_03/gpu_rules_api.h:72).
 * Same as gpu_evaluate_rule for one rule in the RDFRules JSON export format. */
int gpu_evaluate_rule_json(void* ctx, const char* ruleJson, GpuRuleResult* out);

/* Replaces gpu_free_graph (GPU_03/gpu_rules_api.h:79).  NULL is ignored. */
void gpu_free_graph(void* ctx);

/* Replaces gpu_query_vram (GPU_03/gpu_rules_api.h:87).
 * Free and total memory of the current device; 0 on success, -1 without a
 * CUDA device. */
int gpu_query_vram(size_t* freeBytesOut, size_t* totalBytesOut);

/* ---- additive entry points (no counterpart in the reference) ---- */

/* Evaluates n rules (text, or JSON when isJson != 0) in one persistent
 * device launch that covers both phases of every rule.  out[i] receives
 * rule i's result; status[i] (optional) receives 0 on success or -1 when
 * rule i does not parse (its result is then zero).  deviceMs (optional)
 * receives the device time of the whole batch.  Per-rule supportMs and
 * confidenceMs are 0 in this mode.  Returns 0, or -1 on null arguments or a
 * CUDA error (then every out[i] is zero and every status[i] is -1). */
int gpu_evaluate_rules_batch(void* ctx, const char* const* rules, int n, int isJson,
                             GpuRuleResult* out, int* status, double* deviceMs);

/* Prepared batches: parse, plan and upload n rules once, then run the
 * device work any number of times as one CUDA-graph launch (the batched
 * persistent form with its inputs resident in device memory).  Returns a
 * batch handle, or NULL on null arguments or a CUDA error; rules that do not
 * parse are reported by gpu_batch_run's status array.  A batch belongs to
 * the context it was prepared on and must be freed before it. */
void* gpu_batch_prepare(void* ctx, const char* const* rules, int n, int isJson);

/* Runs a prepared batch.  flushBytes > 0 first overwrites a scratch buffer
 * of that size (outside the timed span) so that the run starts with a cold
 * L2.  out/status (optional, n entries) receive the results; deviceMs
 * (optional) the device time between two events around the graph launch.
 * Returns 0, or -1 on a CUDA error. */
int gpu_batch_run(void* batch, long long flushBytes, GpuRuleResult* out, int* status, double* deviceMs);

/* The last run's counts in 64 bits (GpuRuleResult's int fields saturate at
 * INT_MAX): counts[4 * i + 0..3] = support, headSize, headSupport, bodySize
 * of rule i; status (optional) as gpu_batch_run.  No counterpart in the
 * reference (its counts are int).  Returns 0, or -1 on null arguments. */
int gpu_batch_counts(void* batch, long long* counts, int* status);

/* One rule split over nShards workers (one per GPU): evaluates only slice
 * `shard` of each device phase's roots — head triples for support, rows of
 * the seed atom keyed by the head subject for body size — cut so that the
 * slices carry about equal estimated work.  Body pairs of different head
 * subjects are distinct, so summing counts[0] (support) and counts[3]
 * (bodySize) over all shards gives the whole rule's counts (one int64 sum
 * all-reduce across GPUs); counts[1..2] (headSize, headSupport) are the
 * whole rule's in every shard.  No counterpart in the reference.  Returns
 * 0, or -1 on bad arguments, a malformed rule or a CUDA error. */
int gpu_evaluate_rule_shard(void* ctx, const char* ruleText, int shard, int nShards, long long* counts);

/* Device plans, tasks, bytes copied host->device at preparation and bytes
 * copied device->host per run. */
int gpu_batch_info(void* batch, long long* plans, long long* tasks, long long* h2dBytes, long long* d2hBytes);

/* Kernels one gpu_batch_run launches on the device (the engine, the fused
 * support of split heavy roots, the pair sort when staged), or -1 for a
 * null batch.  No counterpart in the reference (its batch is one kernel
 * launch per rule phase). */
int gpu_batch_kernels(void* batch);

/* Runs the batch once with the byte-counting variant of the kernel and
 * returns the global-memory bytes the algorithm requested (the roofline's
 * algorithmic bytes).  Not timed. */
int gpu_batch_count_bytes(void* batch, unsigned long long* bytes);

/* Runs the batch once with the instrumented kernel variant.  bytes
 * (optional) receives the algorithmic bytes as gpu_batch_count_bytes does;
 * for the first maxTasks device tasks, taskNs (optional, 2 per task)
 * receives the start and end time (device global timer, ns) and taskInfo
 * (optional, 3 per task) the owner (rule * 2 + phase, phase 0 = support,
 * 1 = body size) and the root range.  Not timed. */
int gpu_batch_profile(void* batch, unsigned long long* bytes, unsigned long long* taskNs, int* taskInfo,
                      long long maxTasks);

/* Feedback-directed task balancing: runs the instrumented kernel `rounds`
 * times; after each run the context's task builder learns, per plan
 * signature, the device time per unit of estimated work, marks the phases
 * whose slowest task held up the launch for an exact per-root measurement,
 * and the batch's tasks are rebuilt and re-uploaded.  What is learnt stays
 * with the context and also balances later batches and per-rule calls with
 * the same plans.  Returns 0, or -1 on a CUDA error. */
int gpu_batch_autotune(void* batch, int rounds);

/* Frees a prepared batch (NULL is ignored). */
void gpu_batch_free(void* batch);

/* How each rule's body size deduplicates its (hS, hO) pairs in the batch's
 * current staging (no counterpart in the reference, which picks a bitmap or
 * a pair buffer with sort + unique from one N^2 size test,
 * GPU_03/gpu_rules_lib.cu:296-316): modes[i] (n entries) = 0 bitmap rows in
 * shared memory, 1 one global bitmap row per head subject, 2 global rows per
 * resident block (memory bounded by the launch, not the rows), 3 pair keys
 * radix-sorted and counted once each; -1 when rule i's body size needs no
 * pair deduplication on the device.  sortKeys (optional): pair keys the last
 * run appended.  Returns 0, or -1 on null arguments. */
int gpu_batch_dedup(void* batch, int* modes, long long* sortKeys);

/* No counterpart in the reference.  Same as gpu_evaluate_rule, for callers
 * that cannot allocate device memory while they evaluate: a host framework
 * that owns a fixed device-memory budget and forbids allocation per request,
 * or a serving loop that must not call cudaMalloc/cudaFree because they can
 * synchronise the whole device.  The per-call device buffers (plan, tasks,
 * counters, status and, for very large hO domains, the pair bitmap) come from
 * one 8 MiB array built into the library (held on every GPU that loads it
 * until the process exits); a rule that needs more returns -1 with the size
 * in gpu_last_error().  The first call on a device looks up the array's
 * device address (make it before any stream capture).  Calls share the array:
 * calls that overlap on the same GPU race and must be serialised. */
int gpu_evaluate_rule_noalloc(void* ctx, const char* ruleText, GpuRuleResult* out);

/* Engine option for later calls on this context.  "block": threads per
 * block of the engine kernel, 128, 256 or 512 (default 256; the environment
 * variable GPU_RULES_BLOCK sets it at load).  "task_target": fixed work per
 * task in candidate bindings (0 = automatic balancing).  "walk_threshold":
 * estimated work above which a phase's roots are measured one by one before
 * splitting (default 200000).  "rule_block": block size the plain per-rule
 * calls launch on (default 512; 0, or a size not above "block", = "block");
 * their plans keep the layout of "block", so they reuse what batches learnt.
 * "rule_walk_budget": per-root measurement allowed per per-rule call.
 * "batch_chunks": pipelined chunks of gpu_evaluate_rules_batch (0 =
 * automatic).  "batch_phases": which phases batches prepared afterwards run
 * on the device, 1 support, 2 body size, 3 both (default); a phase left out
 * reads 0 (for timing one phase's launches alone).  Servers started afterwards: "serve_lanes"
 * (1: keep a heavy lane, default; 0: all slots alike), "serve_heavy_share"
 * (the heavy lane launches on 1/share of the blocks, default 2) and
 * "serve_heavy_us" (expected device time in microseconds above which a
 * request is heavy, default 5000), "serve_deadline_us" (device time a
 * served launch may take, from each block's start; past it the blocks
 * abandon their work at the end of a frontier round and the requests that
 * lost work complete with status -4; 0, the default: none) and
 * "serve_max_us" (requests whose expected device time exceeds it are
 * refused at admission with status -4; 0, the default: none).  "dedup_budget": device bytes that one
 * launch's global pair bitmaps may take (default 8 GiB); beyond it each
 * body-size phase whose pairs do not fit shared memory uses either bitmap
 * rows per resident block or pair keys sorted on the device, whichever
 * moves fewer bytes (see gpu_batch_dedup).  "dedup_mode": 0 automatic, or
 * force 1, 2 or 3 of gpu_batch_dedup's modes on every pair-counting phase
 * (for tests).  Returns 0, or -1 for an unknown name or value. */
int gpu_set_option(void* ctx, const char* name, long long value);

/* ---- serving: continuous batching on a resident graph ---- */

/* One completed request.  status: 0 ok, -1 the rule does not parse, -2 the
 * rule's device-memory estimate exceeds the server's whole budget, -3 a CUDA
 * or engine error, -4 over the server's time limits (its expected device
 * time exceeds "serve_max_us", or its launch reached "serve_deadline_us"
 * before the rule was counted; see gpu_set_option); the result is then
 * zero.  latencyMs: from gpu_serve_submit to completion. */
typedef struct {
    long long     requestId;
    int           status;
    GpuRuleResult result;
    double        latencyMs;
} GpuServeResult;

/* Starts a request loop on a loaded graph: a worker thread with `slots`
 * launch slots (streams, 1..16), at most maxBatch rules per launch, and at
 * most memBudgetBytes of estimated device memory (plans, tasks, dedup
 * buffers) held by launches in flight.  The worker plans requests as they
 * arrive.  Whenever a slot is free, the waiting requests are admitted in
 * arrival order while their memory fits and are launched together without
 * waiting for the other slots, so requests that arrive while others run are
 * batched onto the GPU as slots and memory free up.  With two or more slots
 * the last one serves requests whose expected device time is long (heavy
 * lane), launched on half of the SMs so that they never hold the whole
 * GPU; when heavy work piles up and no light request waits, the other
 * slots take heavy requests too.  Every launch records its task times, from
 * which the context learns each plan shape's cost (later launches, and
 * later batches on the same context, split slow shapes finer).  While a
 * server runs, its context must not be used by other calls.
 * Returns a server handle or NULL. */
void* gpu_serve_start(void* ctx, int slots, int maxBatch, long long memBudgetBytes);

/* Queues one rule (text syntax).  Thread-safe.  Returns 0, or -1 when the
 * server is stopping or an argument is null. */
int gpu_serve_submit(void* server, long long requestId, const char* ruleText);

/* Copies up to max completed results into out, waiting up to waitMs for the
 * first one.  Thread-safe.  Returns the number copied, or -1. */
int gpu_serve_poll(void* server, GpuServeResult* out, int max, int waitMs);

/* Requests submitted and completed, launches issued, device memory
 * currently held by launches in flight, the summed device span of the
 * completed launches and the worker's summed host preparation time. */
int gpu_serve_stats(void* server, long long* submitted, long long* completed, long long* launches,
                    long long* memInUse, double* deviceMs, double* hostMs);

/* Finishes every queued request, stops the worker and frees the server
 * (uncollected results are dropped).  NULL is ignored. */
void gpu_serve_stop(void* server);

/* Number of entities, predicates and distinct triples of a loaded graph. */
int gpu_graph_stats(void* ctx, long long* entities, long long* predicates, long long* triples);

/* Predicate `index` (0 .. predicates - 1): its IRI into name (at most
 * capacity - 1 bytes and a terminating 0; name may be NULL to ask for the
 * length) and its distinct triples into *triples (optional).  Returns the
 * IRI's length, or -1 for a bad index.  No counterpart in the reference (a
 * rule miner enumerates head and body predicates with it). */
int gpu_graph_predicate(void* ctx, long long index, char* name, int capacity, long long* triples);

/* Writes the loaded graph (dictionaries, rule prefixes and the whole host
 * index) to one binary file; 0, or -1 with gpu_last_error() set.  No
 * counterpart in the reference, which parses and indexes the Turtle file on
 * every load (gpu_index.cuh:33-79). */
int gpu_save_index(void* ctx, const char* path);

/* Loads a graph from a file written by gpu_save_index, skipping the Turtle
 * parse and the index build; otherwise like gpu_load_graph (NULL with
 * gpu_last_error() set on failure, including a file of another format
 * version, one whose checksum does not match, or one whose sizes or offsets
 * do not agree). */
void* gpu_load_index(const char* path);

/* Last error message of the calling thread ("" if none). */
const char* gpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GPU_RULES_API_H */
