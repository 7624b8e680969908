/* fk.h -- C ABI of libfk, the B200 sieve + strong-probable-prime engine for
 * the three prime-constellation hunts of jhg023/first-knowns:
 *
 *   FK_EULER    Euler-form runs      x^2 + x + p          (line variable p)
 *   FK_DICKSON  Dickson ladders      m*k^2 + 1, k = W*j   (line variable j)
 *   FK_AP       primorial-step APs   p + i*d              (line variable p)
 *
 * The reference engines are Python classes (no FFI of their own); each
 * entry point below replaces one device-side step of them and is what the
 * ctypes layer in first-knowns_b200/fk_abi.py binds.  Plain pointers and
 * sizes only.  Line values are unsigned 128-bit integers passed as two
 * little-endian uint64 limbs.  Results are owned by the engine (or batch)
 * and stay valid until its next call.  Every call is single-threaded per
 * handle, as the reference engines are (one host thread per engine).
 */
#ifndef FK_H
#define FK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t fk_status;
#define FK_OK 0
#define FK_ERR_DOMAIN 1   /* ValueError in the reference: bad range/params */
#define FK_ERR_OVERFLOW 2 /* RuntimeError: a queue or buffer overflowed   */
#define FK_ERR_DEVICE 3   /* CUDA error                                    */
#define FK_ERR_TIMEOUT 4  /* a bounded device wait gave up                 */
#define FK_ERR_ARG 5      /* null pointer / invalid handle                 */

#define FK_EULER 0
#define FK_DICKSON 1
#define FK_AP 2

typedef struct fk_engine fk_engine;
typedef struct fk_batch fk_batch;

/* Engine construction parameters.
 *   Euler:   GpuEngine(n, wheel_primes)  euler-prime-runs/euler_gpu.py:1010
 *   Dickson: GpuEngine(n, q2, ...)       dickson-ladders/ladder_gpu.py:424
 *   AP:      GpuEngine(n, q2, launch_u)  primorial-ap/ap_gpu.py:401      */
typedef struct fk_params {
  uint32_t kind;      /* FK_EULER / FK_DICKSON / FK_AP                       */
  uint32_t n;         /* filter: values x^2+x+p for x < n; m = 1..n; AP n     */
  uint32_t q2;        /* sieve depth: primes below q2 (0: 65536)              */
  uint32_t p0;        /* first pattern-sieve prime index: 6, 7, 9 or 11       *
                       * (all sieve primes below it are folded into the       *
                       * wheel); 0 picks a default for the kind               */
  uint64_t d_lo, d_hi;/* AP difference (0, 0: the n-th primorial)             */
  uint32_t two_pass;  /* Dickson: launcher's two-pass sprp_run depth          */
  uint32_t sieve;     /* 0 auto (cost model + lane length), 1 compaction      *
                       * rounds only, 2 marking sieve for every item          */
} fk_params;

/* Read-only description of an engine, for the Python mirrors. */
typedef struct fk_info {
  uint64_t M;          /* wheel period of the device line                     */
  uint64_t W;          /* Dickson k = W*j                                     */
  uint32_t L;          /* wheel lanes                                         */
  uint32_t NP;         /* sieve primes                                        */
  uint32_t first_prime;/* smallest sieve prime not folded into the wheel      */
  uint32_t nrounds;    /* compaction rounds                                   */
  uint64_t device_bytes; /* bytes this engine holds on the device             */
  uint32_t use_mark;   /* long lanes use the marking sieve (cost model)      */
  uint32_t marked_primes; /* primes the marking sieve covers                 */
  double survival;     /* expected pre-primality survivors per unit of the   *
                        * line (product of 1 - f_q/q over the wheel and     *
                        * sieve primes, f_q forbidden residues of q)        */
} fk_info;

/* One ordered result: x = base + offset[i]; depth[i] is the chain depth
 * (0 for pre-primality streams). */
typedef struct fk_result {
  uint64_t count;
  const uint64_t* offset;
  const uint8_t* depth;
} fk_result;

/* One interval of a batch. */
typedef struct fk_item {
  uint32_t engine;     /* index into the batch's engine list                  */
  uint32_t mode;       /* 0 sieve stream, 1 hunt (classified), 2 dense        */
  uint32_t threshold;  /* keep depth >= threshold (hunt / dense)              */
  uint32_t cap;        /* chain cap                                           */
  uint64_t lo[2];      /* [lo, hi) in the engine's line variable              */
  uint64_t hi[2];
} fk_item;

/* Batch result: per item, its slice of the concatenated ordered stream. */
typedef struct fk_batch_result {
  uint64_t nitems;
  const uint64_t* item_start;  /* [nitems + 1] slice boundaries               */
  const uint64_t* offset;      /* x - item.lo                                 */
  const uint8_t* depth;
} fk_batch_result;

/* ---- engines ---------------------------------------------------------- */
/* Builds the wheel, pattern tables, per-prime kill tests and compaction
 * rounds, and uploads them; they stay device-resident until destroy.    */
fk_status fk_engine_create(const fk_params* params, fk_engine** out);
void fk_engine_destroy(fk_engine* e);
fk_status fk_engine_info(const fk_engine* e, fk_info* out);

/* Pre-primality survivor stream of [lo, hi), ascending.
 * Replaces survivors_pre_mr   euler-prime-runs/euler_gpu.py:1335-1456,
 *          survivors_j        dickson-ladders/ladder_gpu.py:757-781,
 *          survivors          primorial-ap/ap_gpu.py:555-635.           */
fk_status fk_sieve(fk_engine* e, const uint64_t lo[2], const uint64_t hi[2],
                   fk_result* out);

/* Survivors of [lo, hi) classified on the device; those whose depth
 * reaches `threshold`, ascending, with depths.
 * Replaces hunt               euler-prime-runs/euler_gpu.py:1458-1464,
 *                             dickson-ladders/ladder_gpu.py:819-829,
 *                             primorial-ap/ap_gpu.py:661-670,
 * and the host classification pools that follow them in the launchers
 * (euler-prime-runs/launch.py:664-667, dickson-ladders/launch.py:310-402,
 * primorial-ap/launch.py:195-234).                                      */
fk_status fk_hunt(fk_engine* e, const uint64_t lo[2], const uint64_t hi[2],
                  uint32_t threshold, uint32_t cap, fk_result* out);

/* Every x in [lo, hi) classified directly, no sieve (the launchers' low
 * passes below the engine floors: euler-prime-runs/launch.py:410-420,
 * dickson-ladders/launch.py:653-669, where x is k itself).              */
fk_status fk_dense(fk_engine* e, const uint64_t lo[2], const uint64_t hi[2],
                   uint32_t threshold, uint32_t cap, fk_result* out);

/* Chain depth of explicit line values (count values, two limbs each).
 * Replaces chain_depth  primorial-ap/ap_gpu.py:651-659 and run_length
 * dickson-ladders/ladder_gpu.py:813-817 for caller-supplied values.     */
fk_status fk_depths(fk_engine* e, const uint64_t* x_limbs, uint64_t count,
                    uint32_t cap, uint8_t* depth_out);

/* ---- batches: many intervals, one persistent launch per run ---------- */
fk_status fk_batch_create(fk_engine* const* engines, uint32_t nengines,
                          fk_batch** out);
void fk_batch_destroy(fk_batch* b);
/* Appends engines to a batch (item.engine indexes them after the existing
 * ones).  The batch keeps its device and pinned buffers, so a caller that
 * meets new engine configurations while it serves does not rebuild (and
 * regrow) them.  No counterpart in the reference: batching is new here. */
fk_status fk_batch_add_engines(fk_batch* b, fk_engine* const* engines,
                               uint32_t nengines);
/* Runs all items; use_graph != 0 replays a captured CUDA graph. */
fk_status fk_batch_run(fk_batch* b, const fk_item* items, uint64_t nitems,
                       int use_graph, fk_batch_result* out);
/* Asynchronous form for the serving loop: submit, then wait. */
fk_status fk_batch_submit(fk_batch* b, const fk_item* items, uint64_t nitems,
                          int use_graph);
fk_status fk_batch_wait(fk_batch* b, fk_batch_result* out);
/* Non-blocking: *ready = 1 once a submitted run has finished on the
 * device (fk_batch_wait then returns without waiting on the GPU). */
fk_status fk_batch_ready(fk_batch* b, int* ready);
/* Device time (ms) of the last run's kernels, from CUDA events. */
fk_status fk_batch_last_ms(const fk_batch* b, float* sieve_ms,
                           float* classify_ms, float* total_ms);

/* Kernel shape of a batch (or of an engine's plain calls).  None of these
 * changes a result; they only move time.  fk_tune.py searches them.
 * Zero in any field keeps that field's current value.                   */
typedef struct fk_tuning {
  uint32_t sieve_ctas_per_sm;    /* k_sieve persistent grid: CTAs per SM (1-3)  */
  uint32_t mark_ctas_per_sm;     /* k_mark persistent grid: CTAs per SM (1-3)   */
  uint32_t chains_per_sm;        /* lanes are cut into chains until about this *
                                  * many chains per SM exist (64-65536)        */
  uint32_t warp_queue;           /* compaction: a warp's queue shorter than    *
                                  * this runs one candidate per warp over all  *
                                  * later primes (1-513; 513: always)         */
  uint32_t seg_per_task;         /* marking: segments per task (1-64)          */
  uint32_t classify_ctas_per_sm; /* k_classify grid: CTAs per SM (1-32)        */
  uint32_t mark_limit;           /* sieve-prime bound of the marking sieve:    *
                                  * primes below it are marked, the rest are   *
                                  * tested per candidate (2^16 = all marked)   */
  float mark_bias;               /* an item is marked when the modelled cost   *
                                  * of marking is below mark_bias times that   *
                                  * of the compaction rounds                   */
  uint32_t warp_lane_words;      /* lanes of at least this many 64-period      *
                                  * words are swept one warp per lane (>= 32)  */
  float capacity_scale;          /* first candidate / output buffer size as a  *
                                  * multiple of the survival model's estimate *
                                  * (0.0001-1000): too small only costs a     *
                                  * grow-and-rerun (fk_stats.reruns)           */
  float round_cut;               /* a compaction round ends once survival     *
                                  * within it falls below this (0.05-0.95)    */
  uint32_t group_lane_words;     /* lanes of at least this many words (and    *
                                  * fewer than warp_lane_words) are swept by  *
                                  * eight threads per lane (>= 8)             */
  uint32_t mark_segment;         /* marking: periods per shared-memory        *
                                  * segment, one byte each (16384, 32768 or   *
                                  * 65536: a kernel variant)                  */
  uint32_t pattern_primes;       /* pattern sieve + compaction rounds: sieve  *
                                  * primes each CTA stages as shared-memory   *
                                  * pattern tables (24, 32 or 40: a kernel    *
                                  * variant); the rest are tested per         *
                                  * candidate                                 */
  uint32_t mark_pattern_primes;  /* the same for the marking sieve (24, 32 or *
                                  * 40); the primes past them are marked      */
  uint32_t warp_tasks;           /* pattern sieve + rounds: blocks of 32      *
                                  * threads' chains per CTA task (8, 16 or    *
                                  * 32), claimed by the CTA's warps one at a  *
                                  * time; the CTA waits for its slowest warp  *
                                  * once per task                             */
} fk_tuning;
fk_status fk_batch_set_tuning(fk_batch* b, const fk_tuning* t);
fk_status fk_batch_get_tuning(const fk_batch* b, fk_tuning* out);
/* The same for the engine's plain calls (fk_sieve / fk_hunt / fk_dense). */
fk_status fk_engine_set_tuning(fk_engine* e, const fk_tuning* t);

/* Counters of the last run (device-side work accounting). */
typedef struct fk_stats {
  uint64_t launches;     /* kernels launched by the run                      */
  uint64_t items;        /* device items (launch-sized sub-ranges)          */
  uint64_t candidates;   /* pre-primality survivors (or dense values)       */
  uint64_t outputs;      /* ordered entries returned                        */
  uint64_t s1_words;     /* 64-candidate words the pattern sieve processed  */
  uint64_t s2_tests;     /* per-candidate prime tests in the rounds         */
  uint64_t imad_alg;     /* algorithmic 32-bit multiply-adds of the SPRP    *
                          * stage: (bits(N)-1)*(4l^2+2l) per strong base,   *
                          * l = ceil(bits(N)/32)                            */
  uint64_t sprp_values;  /* values strong-tested                            */
  uint64_t marks;        /* byte marks of the marking sieve                 */
  uint64_t h2d_bytes;    /* host-to-device bytes the run copied             */
  uint64_t d2h_bytes;    /* device-to-host bytes the run copied             */
  float sieve_ms, classify_ms, total_ms;
  float mark_ms;         /* device time of the marking-sieve launches       */
  float rounds_ms;       /* device time of the pattern + rounds launches    */
  uint32_t reruns;       /* pipeline reruns after a buffer overflow grew    *
                          * the buffers (the result is the rerun's)         */
} fk_stats;
fk_status fk_batch_stats(const fk_batch* b, fk_stats* out);
/* The same counters for an engine's last plain call. */
fk_status fk_engine_stats(const fk_engine* e, fk_stats* out);

/* ---- allocation-free sieve ---------------------------------------------
 * No counterpart in the reference (its engines allocate through CuPy).
 * For callers that cannot allocate device memory while they sweep (a fixed
 * memory budget, an allocator they own, or no implicit synchronisation
 * allowed): the pre-primality survivors of [lo, hi), as ascending offsets
 * x - lo, written into the caller's device buffer d_offsets (capacity
 * entries) with their number in *d_count (a device uint64).  It allocates
 * nothing: all scratch lives in one fixed device array of about 5.3 MiB
 * that every GPU loading the library holds until exit.  Limits: at most
 * 65536 sieve primes and periods * M below 2^55, on top of fk_sieve's own
 * domain checks (else FK_ERR_DOMAIN), and at most 262144 survivors per
 * call.  The engine's device must be current (else FK_ERR_DEVICE, before
 * any launch).  At run time *d_count receives the survivor count, or
 *   UINT64_MAX      more than 262144 survivors, or more than capacity:
 *                   split the interval and call again;
 *   UINT64_MAX - 1  a bounded device wait gave up (pattern staging): a
 *                   device fault or stall, which splitting does not cure.
 * Asynchronous on `stream` (a cudaStream_t, NULL for the default stream):
 * synchronise before reading the outputs.  Calls share the array, so calls
 * that overlap on the GPU race; serialise them.  The first call on a
 * device (with that device current) looks the array up; make it before
 * any stream capture.                                                     */
fk_status fk_sieve_noalloc(fk_engine* e, const uint64_t lo[2],
                           const uint64_t hi[2], uint64_t* d_offsets,
                           uint64_t capacity, uint64_t* d_count,
                           void* stream);

/* ---- misc -------------------------------------------------------------- */
/* Last error message on this thread. */
const char* fk_last_error(void);
/* Device SPRP verdicts for explicit values (three limbs each):
 * huntlib/primes.py mr_is_prime (base2_only = 0) / sprp_base2 (1).      */
fk_status fk_sprp(const uint64_t* v_limbs, uint64_t count, int base2_only,
                  uint8_t* out);
/* Library version string. */
const char* fk_version(void);
/* Select the CUDA device for this host thread's later libfk calls (libfk
 * carries its own runtime state; a caller's runtime does not set it). */
fk_status fk_set_device(int device);
/* Measured device peaks for the rooflines: which = 0 gives 32-bit integer
 * multiply-adds per second (IMAD, lo and hi halves alternating), which = 1
 * shared-memory load bytes per second (64-bit, bank-conflict free),
 * which = 2 shared-memory byte stores per second (bank-conflict free),
 * 3 mad.lo.u32 alone and 4 mad.hi.u32 alone per second, 5 mul.hi.u64
 * (high half of a 64 x 64-bit product) per second, 6 shared-memory bit
 * marks (red.shared.or.b32, bank-conflict free) per second.            */
fk_status fk_peak(int which, double* per_second);

#ifdef __cplusplus
}
#endif
#endif /* FK_H */
