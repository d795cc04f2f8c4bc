/*
 * dirichlet_dp.c -- an independent M(x) engine for cross-checking.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  The reference's
 * unit test cross-validates its Deleglise-Rivat engine against a "Dirichlet
 * hyperbola DP engine" (test_dr.cpp:8-11, 69-89) that is not part of the
 * reference project.  This file is that kind of second method, written from
 * the mathematics and sharing nothing with the Deleglise-Rivat decomposition
 * (no S1/S2 split, no mod-6 wheel, no byte-log sieve):
 *
 *   sum_{d <= x} M(floor(x/d)) = 1       (Dirichlet convolution of mu and 1)
 *
 * so M(x) = 1 - sum_{d=2..x} M(floor(x/d)).  Every argument that occurs is
 * floor(x/m) for some m; values v <= L come from a Mobius prefix sieved up to L
 * (a plain sieve of smallest prime factors), the others are computed bottom-up
 * in increasing v (decreasing m), each summing its distinct quotient blocks
 * (about 2 sqrt(v) of them).  With L ~ x^(2/3) the cost is O(x^(2/3)).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "dr_oracle.h"

static int64_t isqrt64(int64_t n) {
    if (n <= 0) return 0;
    int64_t s = (int64_t)sqrt((double)n);
    while ((s + 1) * (s + 1) <= n) ++s;
    while (s * s > n) --s;
    return s;
}

/* Mertens prefix M[0..L] from a smallest-prime-factor sieve. */
static int32_t *mertens_prefix(int64_t L) {
    int32_t *M = (int32_t *)malloc(((size_t)L + 1) * sizeof(int32_t));
    uint32_t *spf = (uint32_t *)calloc((size_t)L + 1, sizeof(uint32_t));
    int8_t *mu = (int8_t *)malloc((size_t)L + 1);
    if (!M || !spf || !mu) {
        free(M);
        free(spf);
        free(mu);
        return NULL;
    }
    mu[0] = 0;
    if (L >= 1) mu[1] = 1;
    for (int64_t n = 2; n <= L; ++n) {
        if (spf[n] == 0) { /* n is prime */
            for (int64_t m = n; m <= L; m += n)
                if (spf[m] == 0) spf[m] = (uint32_t)n;
        }
        const int64_t p = spf[n], r = n / p;
        mu[n] = (r % p == 0) ? 0 : (int8_t)-mu[r];
    }
    M[0] = 0;
    for (int64_t n = 1; n <= L; ++n) M[n] = M[n - 1] + mu[n];
    free(spf);
    free(mu);
    return M;
}

int64_t dro_mertens_dirichlet(int64_t x) {
    if (x < 1) return 0;
    int64_t L = (int64_t)pow((double)x, 2.0 / 3.0);
    if (L < 1000) L = x < 1000 ? x : 1000;
    if (L > x) L = x;
    int32_t *small = mertens_prefix(L);
    if (!small) return INT64_MIN;
    if (x <= L) {
        const int64_t r = small[x];
        free(small);
        return r;
    }
    /* big[m] = M(floor(x/m)) for the m with floor(x/m) > L, i.e. m < x/L */
    const int64_t mmax = x / (L + 1);
    int64_t *big = (int64_t *)malloc(((size_t)mmax + 2) * sizeof(int64_t));
    if (!big) {
        free(small);
        return INT64_MIN;
    }
    for (int64_t m = mmax; m >= 1; --m) {
        const int64_t v = x / m;
        /* M(v) = 1 - sum_{d=2..v} M(floor(v/d)); floor(v/d) = floor(x/(m d)) */
        int64_t acc = 1;
        const int64_t r = isqrt64(v);
        /* d <= v/r: each term on its own (the argument may be a big value) */
        const int64_t dlim = v / r;
        for (int64_t d = 2; d <= dlim; ++d) {
            const int64_t w = v / d;
            acc -= (w <= L) ? small[w] : big[m * d];
        }
        /* d > v/r: floor(v/d) = q < r, the block of d in (v/(q+1), v/q] */
        int64_t hi = v;  /* v / q at q = 1 */
        for (int64_t q = 1; q < r; ++q) {
            const int64_t next = v / (q + 1);
            const int64_t lo = (next + 1 > dlim + 1) ? next + 1 : dlim + 1;
            if (hi >= lo) acc -= (hi - lo + 1) * (int64_t)small[q];
            hi = next;
        }
        big[m] = acc;
    }
    const int64_t res = big[1];
    free(big);
    free(small);
    return res;
}
