/*
 * dr_engine.h -- C ABI of the B200 Deleglise-Rivat Mertens engine (libdrb200.so).
 *
 * Everything below is plain C: integers, doubles, pointers and sizes.  No
 * exceptions cross this boundary; every entry point returns an int status
 * (DR_OK = 0, negative on error) and dr_last_error() describes the last
 * failure on the calling thread.  Device memory is owned by an opaque
 * dr_ctx (one CUDA stream per context).  A context is not thread-safe;
 * separate contexts are.
 *
 * Reference interfaces replaced (ecreeth/deleglise-rivat):
 *   dr_mertens()            <- DelégliseRivatEngine::compute_mertens(int64 X, int threads)
 *                              mertens_dr.hpp:968, and ::compute_compressed(int64, int)
 *                              mertens_dr.hpp:1442 (policy DR_POLICY_REFERENCE picks the
 *                              same dense/streamed parameters); also
 *                              CudaDelégliseRivatEngine::compute_mertens(int64, int,
 *                              TimingStats*) mertens_cuda.cuh:441 (timings in dr_stats).
 *   dr_default_params()     <- choose_cx :914, choose_sieve_limit :931,
 *                              choose_compressed_limit :1401, dense target and mu limit
 *                              :1033-1038, :1451-1461, use_compressed_default :1421,
 *                              use_chmt_env :1430 (MERTENS_* environment overrides).
 *   dr_table_build() / dr_table_read() / dr_table_checksums()
 *                           <- CompressedMertensTable(u_total, u_dense, threads, max_mu)
 *                              mertens_dr.hpp:689, get_M :707, get_mu :714 and the raw
 *                              members dense_M/mu/chunks/checkpoints :681-687 (SieveTable
 *                              :376-457 when u_dense == u_total).
 *   dr_mertens_batch()      <- no counterpart (the reference evaluates one X per call);
 *                              it is the batched mode of compute_mertens.  A batch
 *                              repeated with identical inputs replays a captured
 *                              CUDA graph of its whole pipeline.
 */
#ifndef DR_ENGINE_H
#define DR_ENGINE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DR_OK 0
#define DR_ERR_ARG -1     /* invalid argument                              */
#define DR_ERR_PARAMS -2  /* parameters fail the endpoint-coverage check   */
#define DR_ERR_NOMEM -3   /* device or host allocation failed / over budget */
#define DR_ERR_CUDA -4    /* CUDA runtime error                            */
#define DR_ERR_DEVICE -5  /* device-side check failed (error flag set)     */

/* Parameter policies for dr_default_params(). */
#define DR_POLICY_REFERENCE 0 /* exactly the reference CPU engine's choice  */
#define DR_POLICY_DENSE 1     /* reference dense path (MERTENS_USE_CHMT=0)  */
#define DR_POLICY_COMPRESSED 2 /* reference streamed path (compute_compressed) */
#define DR_POLICY_GPU 3       /* B200 defaults: larger u, compressed tier   */
#define DR_POLICY_REFERENCE_GPU 4 /* the reference GPU engine's choice, default
                                     host thread count (dr_reference_gpu_params) */

typedef struct dr_ctx dr_ctx;

typedef struct {
    int64_t u_total;     /* sieve / table limit u                               */
    int64_t u_dense;     /* dense int16 prefix covers 0..u_dense (<= u_total)   */
    double cx;           /* S1/S2 split, A = floor(cx*sqrt(y)) (parameter only) */
    int64_t mu_limit;    /* Mobius values kept for 1..mu_limit                  */
    int32_t segment_log2;/* sieve segment = 2^segment_log2 values (0: default)  */
    int32_t block_threads;/* threads per sieve CTA (0: default)                 */
    int32_t chunk_log2;  /* S1/S2 work item = 2^chunk_log2 ops (0: default)    */
    int32_t s1_window_log2; /* windowed S1 of a single query: windows of 2^k
                               table values, k in 12..16 (0 or negative: off) */
} dr_params;

typedef struct {
    int64_t M;               /* M(X)                                           */
    uint64_t C, S1, S2;      /* checksums: M = C - S1 - S2 (mod 2^64)           */
    int64_t terms, evals;    /* outer terms, single/comb2 evaluations           */
    uint64_t s1_ops, s2_ops; /* S1 lookups, S2 wheel positions (2 j each)       */
    double table_ms;         /* device time: sieve + prefix + compressed tier   */
    double plan_ms;          /* device time: term list, op counts, scan         */
    double sums_ms;          /* device time: persistent S1/S2 kernel            */
    double total_ms;         /* host wall time of the call                      */
    double h2d_ms, d2h_ms;   /* copies (batched inputs / results)              */
    int32_t sieve_launches, sums_launches, kernel_launches;
    int32_t reserved;
    uint64_t h2d_bytes, d2h_bytes; /* host<->device bytes copied by the call   */
    uint64_t s1_comp_ops;    /* S1 lookups in the compressed tier (q > u_dense) */
    double band_table_ms;    /* streamed table (both within sums_ms): device time of the */
    double band_sums_ms;     /* bands' sieve + scan + fix-up, and of their S1 passes      */
    int64_t bands;           /* bands streamed by the call (0: the table was held whole) */
} dr_stats;

typedef struct {
    uint64_t dense_sum, dense_wsum, mu_wsum, nz_wsum, neg_wsum, ckpt_wsum;
} dr_table_sums;

/* Context -------------------------------------------------------------- */
int dr_ctx_create(int device, void *cuda_stream /* NULL: own stream */, dr_ctx **out);
int dr_ctx_destroy(dr_ctx *ctx);
const char *dr_last_error(void);
/* Cap on device bytes the context may hold (0: 92% of the free memory plus what the
 * context holds).  Buffers grow to the largest call served and are kept; a call that
 * would exceed the cap first releases them (after the work in flight) and runs once
 * more, so only a call that does not fit on its own fails with DR_ERR_NOMEM. */
int dr_ctx_set_hbm_budget(dr_ctx *ctx, uint64_t bytes);
/* Streamed table for tables larger than device memory (the idea of the reference's
 * windowed engine, mertens_dr_windowed.hpp:218-374, which streams M windows over
 * [1, u] instead of storing them).  A single query (dr_mertens) whose u_total
 * exceeds u_resident keeps only M up to u_res (u_resident rounded down to a sieve
 * segment of the compressed tier, at least one segment above u_dense) in memory; the
 * compressed tier above is sieved band by band, band_values values at a time (0: as
 * many as the resident compressed tier holds), and after each band the S1 lookups
 * whose quotient falls in it are summed.  M(X) and the C/S1/S2 checksums are those
 * of the whole table.  Needs X > u_total and mu_limit <= u_res; batches never
 * stream.  u_resident = 0 (the default) holds every table whole.  The bands'
 * build and lookups count in dr_stats.sums_ms (split out in band_table_ms and
 * band_sums_ms). */
int dr_ctx_set_resident_limit(dr_ctx *ctx, int64_t u_resident, int64_t band_values);
int dr_device_info(int device, int *sm_count, uint64_t *hbm_bytes);

/* Parameters ------------------------------------------------------------- */
int dr_default_params(int64_t X, int policy, dr_params *out);
/* The parameters the reference GPU engine picks for X (mertens_cuda.cuh:421-436
 * choose_gpu_sieve_limit, :473 cx, :492 mu limit): one dense table of u values,
 * u capped at 6e8 for host_threads in {1, 2} and 1.4e9 otherwise (host_threads
 * <= 0: OMP_NUM_THREADS, else the hardware thread count, as omp_get_max_threads()
 * would give); at X <= 5e7 the reference CPU engine's dense parameters (that
 * engine hands such X to compute_mertens, :458-460). */
int dr_reference_gpu_params(int64_t X, int host_threads, dr_params *out);
/* Endpoint-coverage and budget check (0 = usable). */
int dr_check_params(int64_t X, const dr_params *p, uint64_t hbm_budget);
/* Device bytes a table with these limits needs. */
uint64_t dr_table_bytes(int64_t u_total, int64_t u_dense, int64_t mu_limit);
/* Device bytes one query needs: the table plus its reciprocal tables and
 * work arrays (what dr_check_params compares with the budget). */
uint64_t dr_query_bytes(int64_t X, const dr_params *p);

/* Single query (reference: compute_mertens / compute_compressed) ------------- */
int dr_mertens(dr_ctx *ctx, int64_t X, const dr_params *p /* NULL: reference policy */,
               int64_t *out, dr_stats *stats /* nullable */);

/* Batched queries: one shared table, one persistent launch for all S1/S2 work.
 * p: one params struct per query (NULL: reference policy per X) -- the table is
 * built to cover the largest u_total/u_dense/mu_limit among them. */
int dr_mertens_batch(dr_ctx *ctx, const int64_t *X, int64_t count, const dr_params *p,
                     int64_t *out, dr_stats *stats);
/* Per-query checksums of the last batch (count x {C, S1, S2}). */
int dr_batch_checksums(dr_ctx *ctx, uint64_t *out3, int64_t count);
/* Batch autotuner -- no counterpart in the reference.  Times the given batch
 * on the device for up to max_trials configurations (coordinate descent over
 * the shared table size, cx, sieve segment length and block shape, and the
 * S1/S2 work-item size) and writes the best one as count dr_params (all
 * sharing one table) plus its device time.  Every configuration gives the
 * same exact M(X). */
int dr_autotune_batch(dr_ctx *ctx, const int64_t *X, int64_t count, int max_trials, dr_params *out,
                      double *best_ms);

/* Learned tuner -- no counterpart in the reference (whose parameters come from
 * the fixed heuristics choose_cx / choose_compressed_limit, mertens_dr.hpp:914,
 * :1401).  A 4-64-64-4 FP32 MLP on the device with hand-written forward,
 * backward and Adam kernels.  Inputs: log10 X, log2 HBM budget, SM count,
 * log2 batch size; outputs: cx, log2 fx, log2 u_cap, log2 segment length with
 * u = min(fx (X / ln ln X)^(2/3), u_cap); both normalised by fixed affine
 * maps (dr_tuner_features), inputs clamped to the training domain (log10 X in
 * [10, 16], budget 8..160 GiB).  4740 parameters in the order W1[64][4] b1[64]
 * W2[64][64] b2[64] W3[4][64] b3[4]. */
typedef struct dr_mlp dr_mlp;
int dr_mlp_create(dr_ctx *ctx, uint64_t seed, dr_mlp **out);
int dr_mlp_destroy(dr_mlp *mlp);
int64_t dr_mlp_num_params(void);
int dr_mlp_set_weights(dr_mlp *mlp, const float *w, int64_t count);
int dr_mlp_get_weights(dr_mlp *mlp, float *w, int64_t count);
/* Forward pass on B normalised feature rows (B x 4 -> B x 4, host arrays). */
int dr_mlp_forward(dr_mlp *mlp, const float *x, int64_t B, float *y);
/* Gradient of the mean squared error over B examples (no update). */
int dr_mlp_grad(dr_mlp *mlp, const float *x, const float *t, int64_t B, float *grad, float *loss);
/* `steps` full-batch Adam updates (each one replay of a captured CUDA graph). */
int dr_mlp_train(dr_mlp *mlp, const float *x, const float *t, int64_t B, int steps, float lr,
                 float *final_loss);
int dr_tuner_features(int64_t X, uint64_t hbm_budget, int sm_count, int batch, float *out4);
int dr_tuner_params(int64_t X, const float *y_normalised, dr_params *out);
/* Proposal for X: inference on the device, mapped to parameters, then the
 * endpoint-coverage and budget check; a failing proposal is replaced by the
 * reference's default heuristic and *fallback is set to 1. */
int dr_tuner_propose(dr_mlp *mlp, int64_t X, uint64_t hbm_budget, int sm_count, int batch,
                     dr_params *out, int *fallback);

/* Tables (reference: CompressedMertensTable / SieveTable) -------------------- */
int dr_table_build(dr_ctx *ctx, int64_t u_total, int64_t u_dense, int64_t mu_limit,
                   const dr_params *tuning /* nullable: segment / block shape */,
                   dr_stats *stats);
/* M(n) and mu(n) for n in [first, first+count), any pointer may be NULL. */
int dr_table_read(dr_ctx *ctx, int64_t first, int64_t count, int32_t *M, int8_t *mu);
int dr_table_checksums(dr_ctx *ctx, dr_table_sums *out);
/* Mobius values as held in the mod-6 wheel that S2 and the term list read
 * (0 for n sharing a factor with 6 or n > mu_limit); test support. */
int dr_table_read_wheel(dr_ctx *ctx, int64_t first, int64_t count, int8_t *mu);

/* Test support: the device's exact quotient floor(y[i]/d[i]) and S2 summand
 * piece[i](q[i]) (pieces 1..8 combined, 9..12 single) on host arrays.  The
 * reference has no counterpart (its quotients are fast_div, mertens_dr.hpp:80,
 * and its summands Piece1..SinglePiece4, :470-482).  dr_debug_udiv_rcp runs the
 * reciprocal-estimate quotient of the S1/S2 loops; it writes UINT64_MAX where
 * d >= 2^32 or y/d >= 2^50 (outside that routine's domain). */
int dr_debug_udiv(dr_ctx *ctx, const uint64_t *y, const uint64_t *d, int64_t n, uint64_t *q);
int dr_debug_udiv_rcp(dr_ctx *ctx, const uint64_t *y, const uint64_t *d, int64_t n, uint64_t *q);
int dr_debug_piece(dr_ctx *ctx, const int32_t *piece, const uint64_t *q, int64_t n, int64_t *out);
/* The 32-bit routes of the S1/S2 fast paths: dr_debug_udiv32 writes UINT64_MAX
 * where d >= 2^31, y/d >= 2^31 or y < d, dr_debug_piece32 writes INT64_MIN where
 * q >= 2^31 (outside their domains).  No counterpart in the reference. */
int dr_debug_udiv32(dr_ctx *ctx, const uint64_t *y, const uint64_t *d, int64_t n, uint64_t *q);
int dr_debug_piece32(dr_ctx *ctx, const int32_t *piece, const uint64_t *q, int64_t n, int64_t *out);
/* Test support (no counterpart in the reference): the sieve launches a table build
 * makes, as {first segment, end segment, odd mode} triples in stream order, for
 * 2^segment_log2-value segments and a first wave of first_wave segments (one per
 * full-mode CTA).  Writes at most cap triples; returns their number, or a negative
 * DR_ERR_* code.  Needs no GPU. */
int64_t dr_debug_sieve_plan(int64_t u_total, int64_t u_dense, int32_t segment_log2, int64_t first_wave,
                            int64_t *out, int64_t cap);
/* The bands a streamed table (dr_ctx_set_resident_limit) of these limits would use --
 * test support, no counterpart in the reference: *u_res = the resident part's end
 * (u_total when nothing streams), then per band {vlo, vhi, odd}: its values (vlo, vhi]
 * and whether it is sieved in odd mode.  Writes at most cap triples; returns the band
 * count (0: nothing streams) or a negative DR_ERR_* code.  Needs no GPU. */
int64_t dr_debug_stream_plan(int64_t u_total, int64_t u_dense, int32_t segment_log2, int64_t u_resident,
                             int64_t band_values, int64_t *u_res, int64_t *out, int64_t cap);

/* Measured throughput ceilings of the units this engine's kernels are bound by
 * (measurement support for bench.py; no counterpart in the reference).  Each is
 * the best of three timed launches of a synthetic kernel on `device`, in
 * operations per second over the whole GPU: 32-bit shared-memory atomicAdd with
 * the 32 lanes of an instruction on distinct banks (the sieve's marks), the same
 * with the sieve's own address pattern (lane l at byte j + l*m, m odd), 32-bit
 * integer multiply-add, and FP64 fused multiply-add.  Allocates a few KB of
 * device memory and synchronises its own stream; takes ~0.1 s. */
typedef struct dr_peaks {
    double smem_atomic_per_s;
    double smem_atomic_stride_per_s;
    double imad_per_s;
    double dfma_per_s;
} dr_peaks;
int dr_measure_peaks(int device, dr_peaks *out);

/* Table build that allocates nothing.  It has no counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc/cudaFree: code whose device memory
 * belongs to its own allocator (a framework's caching allocator, a pool
 * reserved at start-up) or that must not allocate once it is serving.  The
 * caller passes the four table buffers it allocated itself.  The build's
 * scratch -- per-segment Mobius sums and their offsets, the sieving primes,
 * the periodic stencil, per-prime reciprocals and marking work items -- is one
 * fixed 796,848-byte __device__ array inside libdrb200.so, which every GPU that
 * loads the library holds until the process exits.
 *
 *   u_total in [1, DR_NOALLOC_MAX_U = 2^33]; larger sizes are rejected with
 *   DR_ERR_ARG and a message in dr_last_error().  0 <= u_dense <= u_total
 *   (and <= 7.6e9), 0 <= mu_limit <= u_total.  Buffers, with W =
 *   ceil((u_total - u_dense) / 64):
 *     dM     int16[u_dense], dM[i] = M(i + 1)          16-byte aligned
 *     planes 16*W bytes: per 64 values {nonzero, negative} bit words
 *     ckpt   int32[W]: M just before each 64-value word
 *     wheel  16*(mu_limit/192 + 2) bytes, zeroed by the call, 16-byte aligned
 * The result equals dr_table_build()'s table.  Work is queued on `stream` (a
 * cudaStream_t; NULL is the default stream) and the call returns without
 * waiting: the table is ready when the stream is.  The first call on a device
 * sets up the scratch for that device (it looks up the array's device address
 * and copies the primes and the stencil into it, synchronously); make that
 * first call before any stream capture (on a capturing stream it returns
 * DR_ERR_ARG and leaves the stream untouched).  A set-up that failed is retried
 * by the next call, and a call in a new CUDA context of the device (after
 * cudaDeviceReset) sets up again, synchronously.  All calls share the one scratch
 * array, which keeps the last call's contents, so calls whose work overlaps on
 * the GPU (other streams, other threads) race on it: serialise them. */
#define DR_NOALLOC_MAX_U 8589934592LL
int dr_table_build_noalloc(int device, void *stream, int64_t u_total, int64_t u_dense,
                           int64_t mu_limit, int16_t *dM, void *planes, int32_t *ckpt,
                           void *wheel);

#ifdef __cplusplus
}
#endif
#endif /* DR_ENGINE_H */
