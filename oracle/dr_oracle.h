/*
 * dr_oracle.h -- CPU oracle for the Deleglise-Rivat Mertens path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * engine's algorithm (ecreeth/deleglise-rivat, mertens_dr.hpp) used as the
 * checker for the CUDA engine.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product path never calls it.
 *
 * Pinning: the oracle is checked against the reference's known-answer values
 * (test_dr.cpp:26-47, test_cuda.cu:38-60, README.md:188) and against the
 * reference engine itself compiled from its own sources into oracle/_ref
 * (tables, S2 intervals, S1/S2 checksums, M(X)); see tests/test_oracle.py.
 *
 * Checksum convention shared by the oracle, the reference harness and the
 * CUDA engine (all sums wrap modulo 2^64):
 *   for every outer term k (k coprime to 6, mu(k) != 0, k <= N = X/u) and each
 *   of its evaluations e (sign s_e = +1 for the first, -1 for the second):
 *     C  += mu(k) * s_e * C_e     C_e  = 1 + kappa*M(A)          (single)
 *                                       kappa_y*M(A) - kappa_y2*M(B) (comb2)
 *     S1 += mu(k) * s_e * S1_e
 *     S2 += mu(k) * s_e * S2_e
 *   M(X) = C - S1 - S2.
 */
#ifndef DR_ORACLE_H
#define DR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Parameters of one M(X) evaluation (the reference derives them at
 * mertens_dr.hpp:1033-1038 for the dense path, :1451-1461 for the streamed). */
typedef struct {
    int64_t X;
    int64_t u_total;   /* sieve / table limit u                          */
    int64_t u_dense;   /* dense int16 prefix limit (== u_total: dense)   */
    double  cx;        /* S1/S2 split: A = floor(cx * sqrt(y))           */
    int64_t mu_limit;  /* mu table kept for 1..mu_limit                  */
} dro_params;

typedef struct {
    int64_t  M;         /* M(X)                                          */
    uint64_t C, S1, S2; /* checksums defined above                       */
    int64_t  terms;     /* number of outer terms                         */
    int64_t  evals;     /* number of single / comb2 evaluations          */
    uint64_t s1_lookups, s2_candidates; /* work counts                  */
} dro_result;

/* Table: dense int16 prefix for 0..u_dense, compressed words above it. */
typedef struct {
    int64_t  u_total, u_dense, mu_limit;
    int64_t  num_words;  /* 64-value words in the compressed tier        */
    int16_t *dense_M;    /* [u_dense + 1]                                */
    int8_t  *mu;         /* [mu_limit + 1]                               */
    uint64_t *nz, *neg;  /* [num_words] bit planes                       */
    int32_t *ckpt;       /* [num_words] M just before each word          */
} dro_table;

typedef struct {
    uint64_t dense_sum;     /* sum of dense_M[n]                          */
    uint64_t dense_wsum;    /* sum of dense_M[n] * (2n+1)                 */
    uint64_t mu_wsum;       /* sum of mu[n] * (2n+1)                      */
    uint64_t nz_wsum;       /* sum of nz[w] * (2w+1)                      */
    uint64_t neg_wsum;      /* sum of neg[w] * (2w+1)                     */
    uint64_t ckpt_wsum;     /* sum of ckpt[w] * (2w+1)                    */
} dro_table_sums;

/* ---- parameter policy (restated from mertens_dr.hpp:914-962, 1390-1461) */
int64_t dro_isqrt(int64_t n);
double  dro_choose_cx(int64_t X);
int64_t dro_choose_sieve_limit(int64_t X);
int64_t dro_choose_compressed_limit(int64_t X);
int     dro_use_compressed(int64_t X);              /* env + default rule */
void    dro_default_params(int64_t X, int compressed, dro_params *out);

/* ---- table build (mertens_dr.hpp:755-901) */
int  dro_table_build(dro_table *t, int64_t u_total, int64_t u_dense,
                     int64_t mu_limit, int threads);
void dro_table_free(dro_table *t);
int32_t dro_table_M(const dro_table *t, int64_t q);  /* get_M :707-712 */
int8_t  dro_table_mu(const dro_table *t, int64_t j); /* get_mu :714-716 */
void dro_table_checksums(const dro_table *t, dro_table_sums *out);

/* ---- S2 pieces and intervals (mertens_dr.hpp:462-660) */
int64_t dro_piece(int piece, uint64_t q);  /* 1..8 combined, 9..12 single */
int64_t dro_s2_interval(int piece, int64_t j_first, int64_t j_last,
                        uint64_t y, const int8_t *mu);
int64_t dro_s2_single(uint64_t y, int64_t A, const int8_t *mu);
int64_t dro_s2_combined(uint64_t y, int64_t A, int64_t B, const int8_t *mu);

/* ---- byte-log finalisation rule (mertens_dr.hpp:145-171), one byte */
int8_t dro_finalize_byte(uint8_t acc, uint64_t n);

/* ---- full evaluation with explicit parameters (mertens_dr.hpp:1442-1635) */
int dro_mertens_params(const dro_params *p, int threads, dro_result *out);
/* Reference policy end to end (compute_mertens :968-1383) */
int64_t dro_mertens(int64_t X, int threads);

/* Direct Mobius prefix for small X (independent check; O(X) memory). */
int64_t dro_mertens_direct(int64_t X);

/* Independent cross-check (dirichlet_dp.c): M(x) from sum_{d<=x} M(x/d) = 1 over
 * a sieved Mobius prefix up to x^(2/3); no part of the Deleglise-Rivat path.
 * INT64_MIN if memory runs out. */
int64_t dro_mertens_dirichlet(int64_t x);

#ifdef __cplusplus
}
#endif
#endif
