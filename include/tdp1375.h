/*
 * tdp1375_b200 — C ABI of the B200 transposition-sequence search and permutation filter.
 *
 * The library replaces the native side of the reference's GPUSortingSearch
 * (src/main/java/br/unb/cic/tdp/base/GPUSortingSearch.java:30-45).  Every entry point
 * below names the reference function it replaces.  Plain pointers and sizes only:
 * a JNI, ctypes, cgo or N-API binding can call it directly.
 *
 * Threading: tdp_search / tdp_search_batch block the calling thread; different slots
 * may be used concurrently from different threads (one stream per slot), exactly like
 * the reference's slot pool.  tdp_cancel may be called from any thread.
 */
#ifndef TDP1375_H
#define TDP1375_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- outcomes (>= 0) and errors (< 0) ----------------------------------------- */
#define TDP_NOT_FOUND 0        /* no sequence within the ratio/depth (reference: empty array) */
#define TDP_FOUND 1            /* a sequence was found */
#define TDP_CANCELLED 2        /* "GPU sorting search cancelled" (sorting_search.cu:841-843) */
#define TDP_OVERFLOW 3         /* "GPU sorting search queue overflow" (sorting_search.cu:844-846);
                                  never produced: this engine has no bounded node queue */
#define TDP_ERR_ARGUMENT (-1)  /* invalid argument (message via tdp_last_error) */
#define TDP_ERR_SLOT (-2)      /* "invalid slot" */
#define TDP_ERR_CUDA (-3)      /* CUDA runtime error */
#define TDP_ERR_OUT_OF_MEMORY (-4)
#define TDP_ERR_DEVICE (-5)    /* device-side guard tripped (spin limit or deadline) */
#define TDP_ERR_NOT_INITIALISED (-6)

#define TDP_MAX_N 63     /* MAX_N, core/common.cuh:33-35 */
#define TDP_MAX_DEPTH 15 /* MAX_DEPTH, core/common.cuh:29-31 */

/* Message of the last failing call on this thread (the text the reference's JNI layer
 * puts into RuntimeException, jni_sorter.cu:16-23). */
const char *tdp_last_error(void);

/* Replaces initGpuSortSlots (slot_manager.cu:62-98), JNI initSlots (jni_sorter.cu:25-34).
 * Destroys previous slots, then creates total_slots slots; slot s lives on device
 * s % devices_count.  queue_bytes_budget (bytes) bounds the work-donation mailboxes; dedup_table_size
 * is the transposition-table capacity in entries (rounded up to a power of two). */
int tdp_init_slots(int total_slots, int devices_count, int64_t queue_bytes_budget, int dedup_table_size);

/* Replaces destroyGpuSortSlots (slot_manager.cu:22-60), JNI destroySlots (jni_sorter.cu:36-43).
 * Idempotent. */
int tdp_destroy_slots(void);

/* Replaces performGpuSortingSearch (sorting_search.cu:701-856) and JNI searchForSortingSeq
 * (jni_sorter.cu:45-104).  pi/spi are n bytes (read unsigned).  On TDP_FOUND, out_depth
 * receives d and out_positions 3*d ints: the (i,j,k) positions of each move on the pi array
 * as it stands before that move (the array GPUSortingSearch.java:65-74 replays).  On
 * TDP_NOT_FOUND out_depth is 0.  Errors: n > 63, max_moves outside [1,15], spi/pi not
 * permutations of 0..n-1, bad slot. */
int tdp_search(int slot, const uint8_t *pi, const uint8_t *spi, int n, int initial_even_cycles, float min_rate,
               int max_moves, int full_sorting, int32_t *out_positions, int32_t *out_depth);

/* Replaces cancelGpuSort (slot_manager.cu:100-125), JNI cancelSort (jni_sorter.cu:106-109). */
int tdp_cancel(int slot);

/* Replaces performGpuPiFilter (pi_filter.cu:157-260), JNI filterPiPermutations
 * (jni_sorter.cu:111-150).  Visits every pi with pi[0]=0 over n symbols and keeps those where
 * oriented_triple is in cyclic order, cycle is oriented and (unless skip_2move_check) cycle
 * admits no 2-move.  Writes at most max_rows rows of n bytes to out, in lexicographic order
 * (the reference's order is arbitrary), and returns the total number of hits (< 0: error). */
int64_t tdp_pi_filter(const uint8_t *cycle, int cycle_len, const uint8_t *oriented_triple, int triple_len, int n,
                      int skip_2move_check, uint8_t *out, int64_t max_rows);
/* Device time in ms (CUDA events around its kernels) of this thread's last tdp_pi_filter call. */
double tdp_pi_filter_last_kernel_ms(void);

/* ---- batched search (no counterpart in the reference; one persistent launch over many
 *      instances with device-side admission) ---------------------------------------- */
typedef struct tdp_instance {
    uint8_t n;
    uint8_t max_depth;
    uint8_t full_sorting;
    uint8_t reserved;
    int32_t initial_even_cycles;
    uint8_t pi[64];
    uint8_t spi[64];
} tdp_instance; /* 136 bytes */

typedef struct tdp_result {
    int32_t status;        /* TDP_FOUND / TDP_NOT_FOUND / TDP_CANCELLED / error */
    int32_t depth;
    uint64_t nodes;        /* expanded nodes */
    uint64_t children;     /* children evaluated */
    int32_t positions[45]; /* 3*depth positions, as tdp_search */
    int32_t reserved;
} tdp_result; /* 208 bytes */

int tdp_search_batch(int slot, const tdp_instance *instances, int count, float min_rate, tdp_result *results);

/* Device-resident batch: upload once, run many times, read results. */
int tdp_batch_prepare(int slot, const tdp_instance *instances, int count, float min_rate);
int tdp_batch_run(int slot);
int tdp_batch_results(int slot, tdp_result *results);

/* ---- engine statistics and tuning ---------------------------------------------- */
typedef struct tdp_stats {
    uint64_t nodes;
    uint64_t children;
    uint64_t dedup_probes;
    uint64_t dedup_pruned;
    uint64_t dedup_inserts;
    uint64_t dedup_full;
    uint64_t donations;
    uint64_t task_pops;
    double kernel_ms;
    int32_t error;
    int32_t launches;
    uint64_t busy_warp_cycles; /* SM cycles warps spent holding a task, summed over warps */
    uint64_t warp_cycles;      /* SM cycles from each warp's start to its exit, summed */
    uint64_t dedup_replaced;   /* inserts that overwrote a live entry of a full probe window */
    uint64_t table_atomics;    /* table atomics issued: entry claims and best-depth updates */
    uint64_t commute_skips;    /* children skipped by the partial-order reduction (commute) */
} tdp_stats;

/* Statistics of the last search/batch run on the slot. */
int tdp_last_stats(int slot, tdp_stats *out);

typedef struct tdp_engine_config {
    int32_t blocks_per_sm;   /* 0 = occupancy maximum */
    int32_t poll_interval;   /* chunks between flag polls / donation checks (default 64) */
    int32_t tight_bound;     /* 1 = verdict-preserving strengthened prune, 0 = reference prune only */
    int32_t task_capacity;   /* read-only: warp mailboxes for work donation (sized from the queue budget) */
    double time_limit_s;     /* device deadline per launch */
    int32_t sparse_enumeration; /* 0 = every (i,j,k); 1 = same-cycle pairs where -2 children are useless;
                                   2 (default) = also same-cycle triples where only +2 children are useful */
    int32_t use_cuda_graph;     /* 1 = tdp_batch_run replays one captured CUDA graph per prepared batch */
    int32_t warps_per_instance; /* 0 = admit instances while any warp is free; w > 0 = at most
                                   (grid warps / w) instances in flight, the other warps join them
                                   through work donation (bounds the live transposition-table load) */
    int32_t table_replacement;  /* what a full 8-entry probe window does with a new state:
                                   0 = admit it without recording, as sorting_search.cu:291-297;
                                   1 = overwrite the deepest entry if it is at least as deep;
                                   2 = overwrite the oldest entry; 3 = overwrite the deepest
                                   entry, the oldest among equally deep ones.  Under 2 and 3 an
                                   entry that prunes a state counts as new again.  Verdicts are
                                   the same under every policy; the default is 2 (on a table far
                                   smaller than a search's states, recency keeps the duplicates
                                   that nearby subtrees produce). */
    int32_t commute;            /* 1 (default) = partial-order reduction: a child move on symbols
                                   disjoint from the move that reached the node is skipped when the
                                   two moves could also be made in the other order and the child's
                                   smallest symbol is the smaller (that order reaches the same state
                                   at the same depth); 0 = every child.  Verdicts are the same. */
    int32_t probe_leaves;       /* 0 (default) = a child whose own children can only be tested for
                                   success (nothing two levels down is admitted for expansion) is
                                   admitted without a table probe: expanding it again costs less
                                   than the lookup; 1 = probe every admitted child, as the
                                   reference does.  Verdicts are the same. */
} tdp_engine_config;

int tdp_get_engine_config(int slot, tdp_engine_config *cfg);
int tdp_set_engine_config(int slot, const tdp_engine_config *cfg);

int tdp_device_count(void);

/* ---- batched canonical form (replaces Configuration.getCanonical / hashCode,
 * Configuration.java:147-195, 241-245, 290-303, for many configurations at once) --------
 * Row r is spi over n[r] symbols (2 <= n[r] <= 63) as a 64-byte successor array
 * (spi[x] = the symbol after x in its cycle; every symbol in a cycle of length >= 2), with
 * pi = (0 1 ... n-1).  For each row: the canonical signature (64 floats, the first n[r]
 * used: cycle label, plus index/100 on oriented cycles), its hash code (CRC32 of the
 * big-endian float bytes as a signed int, equal to Configuration.hashCode) and the variant
 * that produced it (2r: pi started at symbol r; 2r+1: its mirror).  tdp_canonical takes
 * host buffers and validates the rows (TDP_ERR_ARGUMENT on a bad row); the _device form
 * takes device buffers on `stream` and does not validate. */
int tdp_canonical(const uint8_t *spi, const uint8_t *n, int count, float *signature, int32_t *hash_code,
                  int32_t *variant);
int tdp_canonical_device(const uint8_t *spi, const uint8_t *n, int count, float *signature, int32_t *hash_code,
                         int32_t *variant, void *stream);

/* ---- batched extension filter (no counterpart in the reference) -----------------------
 * Applies the permutation-filter predicates of tdp_pi_filter to every extension of `count`
 * base configurations (spi/pi rows of 64 bytes, n symbols each, 3 <= n <= 60) that adds one
 * 3-cycle: 2*C(n,3) extensions on existing symbols (spi o (a b c) and spi o (a c b)) followed
 * by 2*C(n+3,3) on three new symbols n, n+1, n+2 inserted into pi before positions
 * g1 <= g2 <= g3 (as (x y z) and (x z y)).  An extension is kept (keep byte 1) when its added
 * cycle is in cyclic order in pi', some cycle is oriented and no oriented cycle admits a
 * 2-move.  keep has count * tdp_extension_count(n) bytes; returns the number kept. */
int tdp_extension_count(int n);
int64_t tdp_extension_filter(const uint8_t *spi, const uint8_t *pi, int n, int count, uint8_t *keep);
/* Same on device buffers, on `stream`; returns 0 (the caller counts keep bytes). */
int tdp_extension_filter_device(const uint8_t *spi, const uint8_t *pi, int n, int count, uint8_t *keep,
                                void *stream);

/* ---- extend step: one-3-cycle insertions (Extensions.java:95-141, Type 1 and Type 2) ----
 * For `count` configurations (spi rows of 64 bytes over n[r] <= 60 symbols, pi = identity),
 * slot e of configuration r (tdp_insertion_extension_slots(max_n) slots each, the multisets
 * a <= b <= c over [0, max_n) in lexicographic order) inserts a new unoriented 3-cycle before
 * old positions a, b, c.  flags[r * slots + e] = 1 for a Type 1 extension (the configuration
 * has open gates and one of a, b, c is one), 2 for a Type 2 extension (no open gate), 0
 * otherwise; the extended spi (n + 3 symbols) goes to out[(r * slots + e) * 64].  gates[r]
 * receives the open-gate mask (CommonOperations.getOpenGates).  Device buffers, on `stream`. */
int64_t tdp_insertion_extension_slots(int max_n);
int tdp_insertion_extensions_device(const uint8_t *spi, const uint8_t *n, int count, int max_n, uint64_t *gates,
                                    uint8_t *flags, uint8_t *out, void *stream);
const char *tdp_insertion_extensions_error(void);

/* ---- learned move ordering (no counterpart in the reference) ------------------------
 * A 1088 -> 256 -> 256 -> 256 -> 4960 BF16 MLP (fp32 accumulation on the tcgen05 tensor
 * cores) scores the (i,j,k) triples of a configuration with n <= 32; the batched search then
 * expands each instance's root children (and, with two levels, the first level's best
 * children) in descending score order.  Ordering only permutes children: verdicts are
 * unchanged.  The entry points below take DEVICE pointers and a
 * cudaStream_t (as void*); they are the building blocks of inference and training. */
#define TDP_MLP_FEATURES 1088
#define TDP_MLP_HIDDEN 256
#define TDP_MLP_TRIPLES 4960
#define TDP_MLP_TRIPLES_PADDED 5120

/* C[m x n] = A[m x k] * B[n x k]^T (+bias[n]) (ReLU if relu); A, B bf16 row-major, k % 8 == 0,
 * 16-byte aligned; out bf16 (out_fp32 = 0) or fp32 with row stride ldo. */
int tdp_mlp_gemm(const void *a, const void *b, int m, int n, int k, const float *bias, int relu, void *out,
                 int out_fp32, int ldo, void *stream);
/* Features of count states (spi/pi rows of 64 bytes, n[count]) into x [count x 1088] bf16. */
int tdp_mlp_features(const uint8_t *spi, const uint8_t *pi, const uint8_t *n, int count, void *x, void *stream);
int tdp_mlp_softmax_xent(const float *logits, int ld, const uint8_t *n, const int32_t *target, int rows,
                         void *dlogits, float *loss, void *stream);
int tdp_mlp_transpose(const void *in, int rows, int cols, void *out, void *stream);
int tdp_mlp_relu_backward(void *grad, const void *act, int64_t count, void *stream);
int tdp_mlp_column_sums(const void *grad, int rows, int cols, float *out, void *stream);
int tdp_mlp_adam(float *master, void *weight, const float *grad, float *m, float *v, int64_t count, float lr,
                 float beta1, float beta2, float eps, int step, void *stream);
int tdp_mlp_order(const float *scores, int ld, const uint8_t *n, int count, uint16_t *order, int order_stride,
                  void *stream);
/* 0 when no tensor-core wait has timed out since the last call (the flag is then cleared). */
int tdp_mlp_error(void);

/* Installs the ordering model on a slot (host arrays: bf16 weights as uint16 bits in the
 * torch.nn.Linear [out, in] layout, fp32 biases; w4 has 4960 rows).  tdp_enable_order_model
 * sets how many levels it orders: 0 keeps the weights but searches in plain order; 1 orders
 * each root's children; 2 also scores the states after each root's 16 best children and
 * expands each one's 32 best-scoring children first (then all of its children in plain
 * order, so the search stays exhaustive). */
int tdp_set_order_model(int slot, const uint16_t *w1, const float *b1, const uint16_t *w2, const float *b2,
                        const uint16_t *w3, const float *b3, const uint16_t *w4, const float *b4);
int tdp_enable_order_model(int slot, int enable);

/* ---- allocation-free permutation filter (no counterpart in the reference) ------------
 * The same filter as tdp_pi_filter for hosts that must not call cudaMalloc: a JVM or
 * database process whose own pool allocator already owns the device heap (a second
 * allocator would fragment it or fail), and real-time services that allocate everything at
 * start-up and may not allocate, nor take the allocator's locks, once they serve requests.
 * It calls no cudaMalloc, cudaFree or allocating library routine.  Its scratch is a static
 * 156 KB device array inside this library, which every GPU that loads the library holds
 * until the process exits; the caller passes the inputs in host memory and out_device, a
 * DEVICE buffer of max_rows * n bytes that it owns.  Limit: n <= 12, i.e. (n-1)! <= 11!
 * candidates; a larger n returns TDP_ERR_ARGUMENT.  The work runs on `stream` (a
 * cudaStream_t, may be null) and the call returns when it is done, with the total number
 * of hits (rows beyond max_rows are counted but not written).  The first call on a device
 * (and the first after that device's context was reset) looks up the array's device
 * address with cudaGetSymbolAddress.  All calls share the one array and it keeps the last
 * call's contents, so calls that overlap on the GPU (other streams or threads at the same
 * time) race: serialise them. */
int64_t tdp_pi_filter_noalloc(const uint8_t *cycle, int cycle_len, const uint8_t *oriented_triple, int triple_len,
                              int n, int skip_2move_check, uint8_t *out_device, int64_t max_rows, void *stream);

/* ---- measurement helper (no counterpart in the reference) ---------------------------
 * Throughput of returning 32-bit atomics (atomicCAS if use_cas, else atomicAdd) at random
 * 32-byte entries of a fresh device buffer of `entries` entries (a power of two), on the
 * current device: with entries * 32 bytes below the L2 size this is the L2 atomic roof that
 * bounds transposition-table claims.  Allocates and frees its buffer. */
int tdp_measure_atomics(int64_t entries, int use_cas, int iters, double *atomics_per_s);
const char *tdp_measure_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* TDP1375_H */
