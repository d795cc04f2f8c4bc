/*
 * dr_oracle.c -- CPU oracle (plain C11 + OpenMP) for the Deleglise-Rivat path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine.  It restates the
 * reference's algorithm (ecreeth/deleglise-rivat, mertens_dr.hpp); every
 * function names the reference lines it follows.  Quotients are exact C
 * integer divisions (the reference's double/SSE2 quotient path is exact, so
 * results coincide).  S2 summands are written from their inclusion-exclusion
 * definitions rather than from the reference's lookup tables; the tests check
 * both against each other.
 */
#include "dr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define DRO_BLOCK 131072 /* values per sieve block (mertens_dr.hpp:764) */
#define DRO_STENCIL 13860 /* lcm(2,3,5,7,11,4,9) (mertens_dr.hpp:784-793) */

static int bit_width_u64(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }
static int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }
static int64_t max64(int64_t a, int64_t b) { return a > b ? a : b; }

static int default_threads(int threads) {
    if (threads > 0) return threads;
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Parameter policy                                                         */
/* ------------------------------------------------------------------------ */

/* Exact floor square root (mertens_dr.hpp:65-74). */
int64_t dro_isqrt(int64_t n) {
    if (n <= 0) return 0;
    const uint64_t target = (uint64_t)n;
    uint64_t s = (uint64_t)sqrt((double)n);
    while ((s + 1) * (s + 1) <= target) ++s;
    while (s * s > target) --s;
    return (int64_t)s;
}

/* choose_cx (mertens_dr.hpp:914-923), MERTENS_CX override in (0.1, 5.0). */
double dro_choose_cx(int64_t X) {
    const char *e = getenv("MERTENS_CX");
    if (e) {
        double v = atof(e);
        if (v > 0.1 && v < 5.0) return v;
    }
    if (X >= 1000000000000000LL) return 1.35;
    if (X >= 10000000000000LL) return 1.15;
    if (X >= 100000000000LL) return 0.95;
    return 0.70;
}

/* choose_sieve_limit (mertens_dr.hpp:931-962): dense-table cutoff. */
int64_t dro_choose_sieve_limit(int64_t X) {
    if (X <= 50000000LL) return X;
    double loglogX = log(fmax(2.0, log((double)X)));
    double fx = 0.32;
    const char *e = getenv("MERTENS_FX");
    if (e) {
        double v = atof(e);
        if (v >= 0.1 && v <= 3.0) fx = v;
    }
    int64_t u = (int64_t)(fx * pow((double)X / loglogX, 2.0 / 3.0));
    int64_t S = dro_isqrt(X);
    if (u < 3 * S) u = 3 * S;
    int64_t cap = 1500000000LL;
    e = getenv("MERTENS_U_CAP");
    if (e) {
        int64_t v = (int64_t)atoll(e);
        if (v >= 100000000LL && v <= 4000000000LL) cap = v;
    }
    return min64(u, cap);
}

/* choose_compressed_limit (mertens_dr.hpp:1401-1419). */
int64_t dro_choose_compressed_limit(int64_t X) {
    if (X < 50000000LL) return X;
    double loglogX = log(fmax(2.0, log((double)X)));
    double fx = 0.95;
    if (X >= 1000000000000000LL) fx = 1.25;
    if (X >= 10000000000000000LL) fx = 1.50;
    int64_t u = (int64_t)(fx * pow((double)X / loglogX, 2.0 / 3.0));
    int64_t S = dro_isqrt(X);
    if (u < 3 * S) u = 3 * S;
    u = ((u + 255) / 256) * 256;
    int64_t cap = 8000000000LL;
    const char *e = getenv("MERTENS_CHMT_U_CAP");
    if (e) {
        int64_t v = (int64_t)atoll(e);
        if (v >= 100000000LL && v <= 10000000000LL) cap = v;
    }
    int64_t endpoints = (int64_t)(dro_choose_cx(X) * sqrt((double)X)) + 1000;
    cap = max64(cap, max64(S + 1000, endpoints));
    return min64(u, cap);
}

/* Strategy switch (mertens_dr.hpp:1027-1029, 1421-1435; x86-64 defaults). */
int dro_use_compressed(int64_t X) {
    const char *e = getenv("MERTENS_USE_CHMT");
    int on;
    if (e) {
        on = (e[0] == '1' || e[0] == 'y' || e[0] == 'Y' || e[0] == 't' || e[0] == 'T');
    } else {
        on = X >= 100000000000LL && !getenv("MERTENS_FX") && !getenv("MERTENS_U_CAP");
    }
    return X >= 100000000000LL && on;
}

/* Parameters exactly as compute_mertens (:1033-1041) or compute_compressed
 * (:1451-1463) derive them, with the table constructors' clamps applied
 * (SieveTable :396, CompressedMertensTable :691, :701). */
void dro_default_params(int64_t X, int compressed, dro_params *out) {
    memset(out, 0, sizeof(*out));
    out->X = X;
    const double cx = dro_choose_cx(X);
    out->cx = cx;
    if (X < 1) return;
    if (!compressed) {
        int64_t u = dro_choose_sieve_limit(X);
        int64_t N = X / u;
        int64_t A_max = (int64_t)(cx * sqrt((double)X)) + 1000;
        int64_t mu_limit = max64(A_max, N + 1000);
        out->u_total = u;
        out->u_dense = u;
        out->mu_limit = (X <= u) ? u : min64(mu_limit, u);
        return;
    }
    int64_t u_total = dro_choose_compressed_limit(X);
    int64_t endpoint = (int64_t)(cx * sqrt((double)X)) + 1000;
    endpoint = (endpoint + 255) & ~255LL;
    int64_t dense_target = min64(128000000LL, ((u_total / 4 + 255) & ~255LL));
    int64_t u_dense = min64(u_total, max64(dense_target, endpoint));
    int64_t N = X / u_total;
    int64_t A_max = (int64_t)(cx * sqrt((double)X)) + 1000;
    int64_t mu_limit = max64(A_max, N + 1000);
    out->u_total = u_total;
    out->u_dense = u_dense;
    out->mu_limit = min64(u_total, mu_limit);
}

/* ------------------------------------------------------------------------ */
/* Byte-log Mobius sieve and tables                                         */
/* ------------------------------------------------------------------------ */

/* Weight of a sieved prime: ceil(log2 p) forced odd (mertens_dr.hpp:781). */
static uint8_t prime_weight(uint64_t p) { return (uint8_t)(bit_width_u64(p - 1) | 1u); }

/* One byte of the finalisation rule (mertens_dr.hpp:145-171): a square flag
 * gives 0; otherwise the parity of the weight sum gives the sign of the
 * sieved part, and a weight sum at or below floor(log2 n) reveals one
 * unsieved prime factor above sqrt(u), which flips the sign. */
int8_t dro_finalize_byte(uint8_t acc, uint64_t n) {
    const unsigned bits = (unsigned)bit_width_u64(n);
    const int sign = (acc & 1) ? -1 : 1;
    if (acc & 0x80) return 0;
    return (int8_t)(acc > bits - 1 ? sign : -sign);
}

static uint8_t g_stencil[DRO_STENCIL];
static int g_stencil_ready = 0;

/* Periodic pre-marking of 2,3,5,7,11 weights and 4,9 square flags
 * (mertens_dr.hpp:785-793); entry i describes n = i + 1. */
static void build_stencil(void) {
    if (g_stencil_ready) return;
    static const unsigned small[5] = {2, 3, 5, 7, 11};
    for (int n = 1; n <= DRO_STENCIL; ++n) {
        unsigned a = 0;
        for (int k = 0; k < 5; ++k)
            if (n % small[k] == 0) a += prime_weight(small[k]);
        if (n % 4 == 0 || n % 9 == 0) a |= 0x80;
        g_stencil[n - 1] = (uint8_t)a;
    }
    g_stencil_ready = 1;
}

typedef struct {
    int64_t *p;
    int64_t count;
} prime_list;

static prime_list primes_upto(int64_t root) {
    prime_list pl = {0, 0};
    if (root < 2) return pl;
    uint8_t *flag = (uint8_t *)malloc((size_t)root + 1);
    memset(flag, 1, (size_t)root + 1);
    int64_t cap = 64;
    pl.p = (int64_t *)malloc(sizeof(int64_t) * cap);
    for (int64_t p = 2; p <= root; ++p) {
        if (!flag[p]) continue;
        if (pl.count == cap) {
            cap *= 2;
            pl.p = (int64_t *)realloc(pl.p, sizeof(int64_t) * cap);
        }
        pl.p[pl.count++] = p;
        for (int64_t m = p * p; m <= root; m += p) flag[m] = 0;
    }
    free(flag);
    return pl;
}

/* Sieve mu(n) for n in [low, low+len) into out[] (one block of the streamed
 * builder, mertens_dr.hpp:813-839). */
static void sieve_block(int64_t low, int64_t len, const prime_list *pl, uint8_t *buf) {
    int64_t done = 0;
    while (done < len) {
        int64_t phase = (low - 1 + done) % DRO_STENCIL;
        int64_t count = min64(len - done, DRO_STENCIL - phase);
        memcpy(buf + done, g_stencil + phase, (size_t)count);
        done += count;
    }
    const int64_t end = low + len - 1;
    for (int64_t i = 0; i < pl->count; ++i) {
        const int64_t p = pl->p[i];
        if (p < 5) continue;
        const int64_t sq = p * p;
        if (sq > end) break;
        for (int64_t j = ((low + sq - 1) / sq) * sq - low; j < len; j += sq) buf[j] |= 0x80;
    }
    for (int64_t i = 0; i < pl->count; ++i) {
        const int64_t p = pl->p[i];
        if (p < 13) continue;
        const uint8_t w = prime_weight((uint64_t)p);
        for (int64_t j = ((low + p - 1) / p) * p - low; j < len; j += p) buf[j] += w;
    }
    for (int64_t j = 0; j < len; ++j) buf[j] = (uint8_t)dro_finalize_byte(buf[j], (uint64_t)(low + j));
    if (low == 1 && len >= 1) buf[0] = 1;            /* n = 1 (:838) */
    if (low <= 2 && low + len - 1 >= 2) buf[2 - low] = (uint8_t)(-1); /* n = 2 (:839) */
}

/* Streamed dense + compressed table (mertens_dr.hpp:689-705, 755-901). */
int dro_table_build(dro_table *t, int64_t u_total, int64_t u_dense, int64_t mu_limit, int threads) {
    memset(t, 0, sizeof(*t));
    if (u_total < 0) return -1;
    threads = default_threads(threads);
    build_stencil();
    u_dense = min64(u_total, u_dense);
    mu_limit = min64(u_total, mu_limit > 0 ? mu_limit : u_dense);
    t->u_total = u_total;
    t->u_dense = u_dense;
    t->mu_limit = mu_limit;
    const int64_t comp = max64(0, u_total - u_dense);
    t->num_words = (comp + 63) / 64;
    t->dense_M = (int16_t *)calloc((size_t)u_dense + 1, sizeof(int16_t));
    t->mu = (int8_t *)calloc((size_t)mu_limit + 1, 1);
    if (t->num_words) {
        t->nz = (uint64_t *)calloc((size_t)t->num_words, 8);
        t->neg = (uint64_t *)calloc((size_t)t->num_words, 8);
        t->ckpt = (int32_t *)calloc((size_t)t->num_words, 4);
    }
    if (!t->dense_M || !t->mu || (t->num_words && (!t->nz || !t->neg || !t->ckpt))) {
        dro_table_free(t);
        return -2;
    }
    prime_list pl = primes_upto(dro_isqrt(u_total));
    const int64_t dense_blocks = (u_dense + DRO_BLOCK - 1) / DRO_BLOCK;
    const int64_t comp_blocks = (comp + DRO_BLOCK - 1) / DRO_BLOCK;
    const int64_t nblocks = dense_blocks + comp_blocks;
    int32_t *block_sum = (int32_t *)calloc((size_t)nblocks + 1, 4);

#pragma omp parallel num_threads(threads)
    {
        uint8_t *buf = (uint8_t *)malloc(DRO_BLOCK);
#pragma omp for schedule(dynamic, 1)
        for (int64_t b = 0; b < nblocks; ++b) {
            const int dense = b < dense_blocks;
            const int64_t base = dense ? b * DRO_BLOCK : u_dense + (b - dense_blocks) * DRO_BLOCK;
            const int64_t end = min64(base + DRO_BLOCK, dense ? u_dense : u_total);
            const int64_t len = end - base, low = base + 1;
            sieve_block(low, len, &pl, buf);
            const int8_t *v = (const int8_t *)buf;
            if (base < mu_limit) memcpy(t->mu + low, v, (size_t)(min64(end, mu_limit) - base));
            int32_t s = 0;
            if (dense) {
                for (int64_t j = 0; j < len; ++j) {
                    s += v[j];
                    t->dense_M[low + j] = (int16_t)s;
                }
            } else {
                const int64_t w0 = (base - u_dense) / 64; /* blocks are word aligned */
                for (int64_t j = 0; j < len; ++j) {
                    const int64_t w = w0 + j / 64;
                    if ((j & 63) == 0) t->ckpt[w] = s;
                    if (v[j] != 0) t->nz[w] |= 1ULL << (j & 63);
                    if (v[j] < 0) t->neg[w] |= 1ULL << (j & 63);
                    s += v[j];
                }
            }
            block_sum[b + 1] = s;
        }
        free(buf);
    }
    for (int64_t b = 1; b <= nblocks; ++b) block_sum[b] += block_sum[b - 1];
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int64_t b = 0; b < nblocks; ++b) {
        const int32_t off = block_sum[b];
        if (b < dense_blocks) {
            const int64_t base = b * DRO_BLOCK, end = min64(base + DRO_BLOCK, u_dense);
            for (int64_t n = base + 1; n <= end; ++n) t->dense_M[n] = (int16_t)(t->dense_M[n] + off);
        } else {
            const int64_t w0 = (b - dense_blocks) * (DRO_BLOCK / 64);
            const int64_t w1 = min64(w0 + DRO_BLOCK / 64, t->num_words);
            for (int64_t w = w0; w < w1; ++w) t->ckpt[w] += off;
        }
    }
    free(block_sum);
    free(pl.p);
    return 0;
}

void dro_table_free(dro_table *t) {
    free(t->dense_M);
    free(t->mu);
    free(t->nz);
    free(t->neg);
    free(t->ckpt);
    memset(t, 0, sizeof(*t));
}

/* Two-popcount reconstruction (mertens_dr.hpp:741-752). */
static int32_t reconstruct(const dro_table *t, int64_t q) {
    const int64_t off = q - t->u_dense - 1;
    const int64_t w = off >> 6;
    const uint64_t mask = ~0ULL >> (63 - (off & 63));
    return t->ckpt[w] + __builtin_popcountll(t->nz[w] & mask) - 2 * __builtin_popcountll(t->neg[w] & mask);
}

int32_t dro_table_M(const dro_table *t, int64_t q) {
    return q <= t->u_dense ? (int32_t)t->dense_M[q] : reconstruct(t, q);
}

int8_t dro_table_mu(const dro_table *t, int64_t j) { return j <= t->mu_limit ? t->mu[j] : 0; }

void dro_table_checksums(const dro_table *t, dro_table_sums *o) {
    memset(o, 0, sizeof(*o));
    for (int64_t n = 0; n <= t->u_dense; ++n) {
        o->dense_sum += (uint64_t)(int64_t)t->dense_M[n];
        o->dense_wsum += (uint64_t)(int64_t)t->dense_M[n] * (uint64_t)(2 * n + 1);
    }
    for (int64_t n = 0; n <= t->mu_limit; ++n) o->mu_wsum += (uint64_t)(int64_t)t->mu[n] * (uint64_t)(2 * n + 1);
    for (int64_t w = 0; w < t->num_words; ++w) {
        const uint64_t k = (uint64_t)(2 * w + 1);
        o->nz_wsum += t->nz[w] * k;
        o->neg_wsum += t->neg[w] * k;
        o->ckpt_wsum += (uint64_t)(int64_t)t->ckpt[w] * k;
    }
}

/* ------------------------------------------------------------------------ */
/* S2: mod-6 piecewise sums (mertens_dr.hpp:462-660)                        */
/* ------------------------------------------------------------------------ */

/* Summand of j (coprime to 6, q = floor(y/j)) in each piece.  Combined pieces
 * 1..8 give f_A(q) - f_B(floor(q/2)) for S2(y) - S2(y/2) and single pieces
 * 9..12 give f_A(q) for S2(y), where f_L(q) = q - [2j<=L]q/2 - [3j<=L]q/3 +
 * [6j<=L]q/6 accounts for j, 2j, 3j, 6j.  Cut points of the combined pieces:
 * B/6, A/6, B/3, A/3, B/2, A/2, B, A; of the single: A/6, A/3, A/2, A. */
int64_t dro_piece(int piece, uint64_t q) {
    const int64_t h = (int64_t)(q / 2), t = (int64_t)(q / 3), f = (int64_t)(q / 4);
    const int64_t s = (int64_t)(q / 6), d = (int64_t)(q / 12), Q = (int64_t)q;
    switch (piece) {
    case 1: return (Q - h - t + s) - (h - f - s + d);
    case 2: return (Q - h - t + s) - (h - f - s);
    case 3: return (Q - h - t) - (h - f - s);
    case 4: return (Q - h - t) - (h - f);
    case 5: return (Q - h) - (h - f);
    case 6: return (Q - h) - h;
    case 7: return Q - h;
    case 8: return Q;
    case 9: return Q - h - t + s;
    case 10: return Q - h - t;
    case 11: return Q - h;
    case 12: return Q;
    }
    return 0;
}

/* run_s2_fast (mertens_dr.hpp:490-617) over j in [j_first, j_last]. */
int64_t dro_s2_interval(int piece, int64_t j_first, int64_t j_last, uint64_t y, const int8_t *mu) {
    if (j_first > j_last) return 0;
    uint64_t sum = 0;
    int64_t j = j_first < 1 ? 1 : j_first;
    while (j <= j_last && (j % 2 == 0 || j % 3 == 0)) ++j;
    while (j <= j_last) {
        const int8_t m = mu[j];
        if (m) sum += (uint64_t)((int64_t)m * dro_piece(piece, y / (uint64_t)j));
        j += (j % 6 == 1) ? 4 : 2;
    }
    return (int64_t)sum;
}

/* eval_s2_single (mertens_dr.hpp:647-660). */
int64_t dro_s2_single(uint64_t y, int64_t A, const int8_t *mu) {
    uint64_t s = 0;
    s += (uint64_t)dro_s2_interval(9, 1, A / 6, y, mu);
    s += (uint64_t)dro_s2_interval(10, A / 6 + 1, A / 3, y, mu);
    s += (uint64_t)dro_s2_interval(11, A / 3 + 1, A / 2, y, mu);
    s += (uint64_t)dro_s2_interval(12, A / 2 + 1, A, y, mu);
    return (int64_t)s;
}

/* eval_s2_combined (mertens_dr.hpp:622-642). */
int64_t dro_s2_combined(uint64_t y, int64_t A, int64_t B, const int8_t *mu) {
    uint64_t s = 0;
    s += (uint64_t)dro_s2_interval(1, 1, B / 6, y, mu);
    s += (uint64_t)dro_s2_interval(2, B / 6 + 1, A / 6, y, mu);
    s += (uint64_t)dro_s2_interval(3, A / 6 + 1, B / 3, y, mu);
    s += (uint64_t)dro_s2_interval(4, B / 3 + 1, A / 3, y, mu);
    s += (uint64_t)dro_s2_interval(5, A / 3 + 1, B / 2, y, mu);
    s += (uint64_t)dro_s2_interval(6, B / 2 + 1, A / 2, y, mu);
    s += (uint64_t)dro_s2_interval(7, A / 2 + 1, B, y, mu);
    s += (uint64_t)dro_s2_interval(8, B + 1, A, y, mu);
    return (int64_t)s;
}

/* ------------------------------------------------------------------------ */
/* S1 and the evaluations (mertens_dr.hpp:1490-1614)                         */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint64_t C, S1, S2, s1n, s2n;
} eval_out;

static int64_t split_point(double cx, int64_t y) {
    int64_t A = (int64_t)(cx * sqrt((double)y));
    if (A >= y) A = y - 1;
    if (A < 1) A = 1;
    return A;
}

/* sum of M(floor(y/n)) for n = first, first+stride, ..., <= last */
static uint64_t s1_range(const dro_table *t, uint64_t y, int64_t first, int64_t last, int stride, uint64_t *cnt) {
    uint64_t s = 0;
    for (int64_t n = first; n <= last; n += stride) {
        s += (uint64_t)(int64_t)dro_table_M(t, (int64_t)(y / (uint64_t)n));
        ++*cnt;
    }
    return s;
}

/* F(y) = 1 - S1 + kappa*M(A) - S2 (eval_single_S, :1490-1525 / :1081-1151) */
static void eval_single(const dro_table *t, double cx, uint64_t y, eval_out *o) {
    const int64_t A = split_point(cx, (int64_t)y);
    const int64_t kappa = (int64_t)(y / (uint64_t)(A + 1));
    const int64_t start = (int64_t)(y / (uint64_t)t->u_total) + 1;
    uint64_t cnt = 0;
    o->S1 = s1_range(t, y, start, kappa, 1, &cnt);
    o->s1n = cnt;
    o->S2 = (uint64_t)dro_s2_single(y, A, t->mu);
    o->s2n = (uint64_t)(A / 3 + 1);
    o->C = (uint64_t)(1 + kappa * (int64_t)dro_table_M(t, A));
}

/* F(y) - F(y/2) with parity-cancelled S1 (eval_comb2, :1527-1614 / :1158-1354) */
static void eval_comb2(const dro_table *t, double cx, uint64_t y, uint64_t y2, eval_out *o) {
    const int64_t A = split_point(cx, (int64_t)y);
    const int64_t B = split_point(cx, (int64_t)y2);
    const int64_t ky = (int64_t)(y / (uint64_t)(A + 1));
    const int64_t ky2 = (int64_t)(y2 / (uint64_t)(B + 1));
    const int64_t two_ky2 = 2 * ky2;
    int64_t start = (int64_t)(y / (uint64_t)t->u_total) + 1;
    if (start % 2 == 0) ++start;
    uint64_t cnt = 0, s1 = 0;
    s1 += s1_range(t, y, start, ky, 2, &cnt); /* odd n */
    if (two_ky2 > ky) {
        int64_t e = ky + 1;
        if (e % 2) ++e;
        s1 -= s1_range(t, y, e, two_ky2, 2, &cnt);
    } else if (two_ky2 < ky) {
        int64_t e = two_ky2 + 1;
        if (e % 2) ++e;
        s1 += s1_range(t, y, e, ky, 2, &cnt);
    }
    o->S1 = s1;
    o->s1n = cnt;
    o->S2 = (uint64_t)dro_s2_combined(y, A, B, t->mu);
    o->s2n = (uint64_t)(A / 3 + 1);
    o->C = (uint64_t)(ky * (int64_t)dro_table_M(t, A) - ky2 * (int64_t)dro_table_M(t, B));
}

int dro_mertens_params(const dro_params *p, int threads, dro_result *out) {
    memset(out, 0, sizeof(*out));
    const int64_t X = p->X;
    if (X < 1) return 0;
    threads = default_threads(threads);
    dro_table t;
    int rc = dro_table_build(&t, p->u_total, p->u_dense, p->mu_limit, threads);
    if (rc) return rc;
    if (X <= t.u_total) {
        out->M = dro_table_M(&t, X);
        dro_table_free(&t);
        return 0;
    }
    const int64_t N = X / t.u_total;
    if (N > t.mu_limit) {
        dro_table_free(&t);
        return -3;
    }
    const int64_t n6 = N / 6, n3 = N / 3, n2 = N / 2;
    uint64_t C = 0, S1 = 0, S2 = 0, s1n = 0, s2n = 0;
    int64_t terms = 0, evals = 0;
    const double cx = p->cx;
#pragma omp parallel for schedule(dynamic, 8) num_threads(threads) reduction(+ : C, S1, S2, s1n, s2n, terms, evals)
    for (int64_t k = 1; k <= N; ++k) {
        if (k % 2 == 0 || k % 3 == 0) continue;
        const int8_t mk = t.mu[k];
        if (!mk) continue;
        const uint64_t y = (uint64_t)(X / k);
        const uint64_t m = (uint64_t)(int64_t)mk;
        eval_out a, b;
        memset(&b, 0, sizeof(b));
        int two = 1;
        if (k <= n6) {
            eval_comb2(&t, cx, y, y / 2, &a);
            eval_comb2(&t, cx, y / 3, y / 6, &b);
        } else if (k <= n3) {
            eval_comb2(&t, cx, y, y / 2, &a);
            eval_single(&t, cx, y / 3, &b);
        } else if (k <= n2) {
            eval_comb2(&t, cx, y, y / 2, &a);
            two = 0;
        } else {
            eval_single(&t, cx, y, &a);
            two = 0;
        }
        C += m * (a.C - b.C);
        S1 += m * (a.S1 - b.S1);
        S2 += m * (a.S2 - b.S2);
        s1n += a.s1n + b.s1n;
        s2n += a.s2n + b.s2n;
        terms += 1;
        evals += 1 + two;
    }
    out->C = C;
    out->S1 = S1;
    out->S2 = S2;
    out->M = (int64_t)(C - S1 - S2);
    out->terms = terms;
    out->evals = evals;
    out->s1_lookups = s1n;
    out->s2_candidates = s2n;
    dro_table_free(&t);
    return 0;
}

int64_t dro_mertens(int64_t X, int threads) {
    if (X < 1) return 0;
    dro_params p;
    dro_default_params(X, dro_use_compressed(X), &p);
    dro_result r;
    if (dro_mertens_params(&p, threads, &r)) return INT64_MIN;
    return r.M;
}

/* Independent Eratosthenes Mobius prefix (the style of test_sieve.cpp:12-31). */
int64_t dro_mertens_direct(int64_t X) {
    if (X < 1) return 0;
    int8_t *mu = (int8_t *)malloc((size_t)X + 1);
    uint8_t *comp = (uint8_t *)calloc((size_t)X + 1, 1);
    for (int64_t n = 0; n <= X; ++n) mu[n] = 1;
    for (int64_t p = 2; p <= X; ++p) {
        if (comp[p]) continue;
        for (int64_t n = p; n <= X; n += p) {
            comp[n] = 1;
            mu[n] = (int8_t)-mu[n];
        }
        if (p <= X / p)
            for (int64_t n = p * p; n <= X; n += p * p) mu[n] = 0;
    }
    int64_t s = 0;
    for (int64_t n = 1; n <= X; ++n) s += mu[n];
    free(mu);
    free(comp);
    return s;
}
