// dr_params.hpp -- parameter policy of the engine (host C++).
//
// DR_POLICY_REFERENCE / _DENSE / _COMPRESSED restate the reference CPU
// engine's heuristics exactly (ecreeth/deleglise-rivat mertens_dr.hpp), so a
// drop-in caller gets the same u, u_dense, cx and mu limit -- and therefore the
// same intermediate S1/S2 checksums -- as the reference for the same X and
// environment.  DR_POLICY_REFERENCE_GPU restates the reference GPU engine's
// choice (mertens_cuda.cuh).  DR_POLICY_GPU is this engine's own default for B200.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <thread>

#include "../../include/dr_engine.h"

namespace drb {

// Exact floor square root (mertens_dr.hpp:65-74).
inline int64_t isqrt_i64(int64_t n) {
    if (n <= 0) return 0;
    const uint64_t target = (uint64_t)n;
    uint64_t s = (uint64_t)std::sqrt((double)n);
    while ((s + 1) * (s + 1) <= target) ++s;
    while (s * s > target) --s;
    return (int64_t)s;
}

// choose_cx (mertens_dr.hpp:914-923); MERTENS_CX in (0.1, 5.0) overrides.
inline double ref_choose_cx(int64_t X) {
    if (const char* e = std::getenv("MERTENS_CX")) {
        const double v = std::atof(e);
        if (v > 0.1 && v < 5.0) return v;
    }
    if (X >= 1000000000000000LL) return 1.35;
    if (X >= 10000000000000LL) return 1.15;
    if (X >= 100000000000LL) return 0.95;
    return 0.70;
}

// choose_sieve_limit (mertens_dr.hpp:931-962); MERTENS_FX, MERTENS_U_CAP.
inline int64_t ref_choose_sieve_limit(int64_t X) {
    if (X <= 50000000LL) return X;
    const double loglogX = std::log(std::max(2.0, std::log((double)X)));
    double fx = 0.32;
    if (const char* e = std::getenv("MERTENS_FX")) {
        const double v = std::atof(e);
        if (v >= 0.1 && v <= 3.0) fx = v;
    }
    int64_t u = (int64_t)(fx * std::pow((double)X / loglogX, 2.0 / 3.0));
    const int64_t S = isqrt_i64(X);
    if (u < 3 * S) u = 3 * S;
    int64_t cap = 1500000000LL;
    if (const char* e = std::getenv("MERTENS_U_CAP")) {
        const int64_t v = (int64_t)std::atoll(e);
        if (v >= 100000000LL && v <= 4000000000LL) cap = v;
    }
    return std::min(u, cap);
}

// choose_compressed_limit (mertens_dr.hpp:1401-1419); MERTENS_CHMT_U_CAP.
inline int64_t ref_choose_compressed_limit(int64_t X) {
    if (X < 50000000LL) return X;
    const double loglogX = std::log(std::max(2.0, std::log((double)X)));
    double fx = 0.95;
    if (X >= 1000000000000000LL) fx = 1.25;
    if (X >= 10000000000000000LL) fx = 1.50;
    int64_t u = (int64_t)(fx * std::pow((double)X / loglogX, 2.0 / 3.0));
    const int64_t S = isqrt_i64(X);
    if (u < 3 * S) u = 3 * S;
    u = ((u + 255) / 256) * 256;
    int64_t cap = 8000000000LL;
    if (const char* e = std::getenv("MERTENS_CHMT_U_CAP")) {
        const int64_t v = (int64_t)std::atoll(e);
        if (v >= 100000000LL && v <= 10000000000LL) cap = v;
    }
    const int64_t endpoints = (int64_t)(ref_choose_cx(X) * std::sqrt((double)X)) + 1000;
    cap = std::max(cap, std::max(S + 1000, endpoints));
    return std::min(u, cap);
}

// Strategy switch (mertens_dr.hpp:1027-1029, 1421-1435; x86-64 default rule).
inline bool ref_use_compressed(int64_t X) {
    bool on;
    if (const char* e = std::getenv("MERTENS_USE_CHMT")) {
        on = (e[0] == '1' || e[0] == 'y' || e[0] == 'Y' || e[0] == 't' || e[0] == 'T');
    } else {
        on = X >= 100000000000LL && !std::getenv("MERTENS_FX") && !std::getenv("MERTENS_U_CAP");
    }
    return X >= 100000000000LL && on;
}

inline void params_clear(dr_params* p) {
    p->u_total = p->u_dense = p->mu_limit = 0;
    p->cx = 0.0;
    p->segment_log2 = p->block_threads = p->chunk_log2 = p->s1_window_log2 = 0;
}

// Dense path parameters (mertens_dr.hpp:1033-1041 with SieveTable's clamp :396).
inline void ref_dense_params(int64_t X, dr_params* p) {
    params_clear(p);
    const double cx = ref_choose_cx(X);
    const int64_t u = ref_choose_sieve_limit(X);
    const int64_t N = X / u;
    const int64_t A_max = (int64_t)(cx * std::sqrt((double)X)) + 1000;
    const int64_t mu_limit = std::max(A_max, N + 1000);
    p->u_total = u;
    p->u_dense = u;
    p->cx = cx;
    p->mu_limit = (X <= u) ? u : std::min(mu_limit, u);
}

// Streamed path parameters (mertens_dr.hpp:1451-1463 with the table clamps :691, :701).
inline void ref_compressed_params(int64_t X, dr_params* p) {
    params_clear(p);
    const double cx = ref_choose_cx(X);
    const int64_t u_total = ref_choose_compressed_limit(X);
    int64_t endpoint = (int64_t)(cx * std::sqrt((double)X)) + 1000;
    endpoint = (endpoint + 255) & ~255LL;
    const int64_t dense_target = std::min<int64_t>(128000000LL, ((u_total / 4 + 255) & ~255LL));
    const int64_t u_dense = std::min(u_total, std::max(dense_target, endpoint));
    const int64_t N = X / u_total;
    const int64_t A_max = (int64_t)(cx * std::sqrt((double)X)) + 1000;
    const int64_t mu_limit = std::max(A_max, N + 1000);
    p->u_total = u_total;
    p->u_dense = u_dense;
    p->cx = cx;
    p->mu_limit = std::min(u_total, mu_limit);
}

// The thread count an OpenMP program uses by default (omp_get_max_threads() with
// no other setting): the first entry of OMP_NUM_THREADS if set, else the number of
// hardware threads.
inline int default_host_threads() {
    if (const char* e = std::getenv("OMP_NUM_THREADS")) {
        const int v = std::atoi(e);
        if (v > 0) return v;
    }
    const unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

// The reference GPU engine's parameters (mertens_cuda.cuh): u from
// choose_gpu_sieve_limit (:421-436) -- fx 1.10 / 1.45 / 2.20 at X below 10^15 /
// from 10^15 / from 10^16, at least 3 sqrt(X), capped at 6e8 for 1 or 2 host
// threads and 1.4e9 otherwise -- one dense table over [0, u] (SieveTable, :465),
// cx from choose_cx (:473), mu limit min(u, max(N, cx sqrt X) + 65536) (:492).
// At X <= 5e7 that engine calls the CPU engine (:458-460), whose dense parameters
// are returned instead.  threads <= 0 stands for the host's default thread count.
inline int64_t ref_gpu_sieve_limit(int64_t X, int threads) {
    if (X <= 50000000LL) return X;
    const double loglogX = std::log(std::max(2.0, std::log((double)X)));
    double fx = 1.10;
    if (X >= 1000000000000000LL) fx = 1.45;
    if (X >= 10000000000000000LL) fx = 2.20;
    int64_t u = (int64_t)(fx * std::pow((double)X / loglogX, 2.0 / 3.0));
    const int64_t S = isqrt_i64(X);
    if (u < 3 * S) u = 3 * S;
    if (threads <= 0) threads = default_host_threads();
    const int64_t cap = (threads > 0 && threads <= 2) ? 600000000LL : 1400000000LL;
    return std::min(u, cap);
}

inline void ref_gpu_params(int64_t X, int threads, dr_params* p) {
    if (X <= 50000000LL) {
        ref_dense_params(X, p);
        return;
    }
    params_clear(p);
    const int64_t u = ref_gpu_sieve_limit(X, threads);
    const double cx = ref_choose_cx(X);
    const int64_t N = X / u;
    const int64_t A = (int64_t)(cx * std::sqrt((double)X));
    p->u_total = u;
    p->u_dense = u;
    p->cx = cx;
    p->mu_limit = std::min<int64_t>(u, std::max(N, A) + 65536);
}

// B200 policy (DR_POLICY_GPU), fitted to sweeps of measured device times over
// X = 10^14 .. 10^18 (table build ~1.0 ms per 10^9 values with the odd-value sieve,
// S1 ~1.1 ms per 10^9 lookups, S2 ~1.9 ms per 10^9 wheel positions): the table is far
// cheaper to build on the GPU than on the CPU, so u is raised to
// 1.15 (X / ln ln X)^(2/3) -- the reference's u formula without its 8e9 cap -- and
// cx = 1.25.  The optimum is flat: at X = 10^16 every (cx, fx) in [1.2, 1.3] x
// [1.1, 1.35] is within 1% of the best, at 10^17 every cx in [1.2, 1.3] with
// fx = 1.1 .. 1.3.  u is capped at 2.5e11 values (~80 GB of compressed tier) and
// never below the endpoints; the dense tier holds max(1.28e8, u/16) values (<= 4e9).
inline void gpu_params(int64_t X, dr_params* p) {
    params_clear(p);
    const double cx = 1.25;
    const double loglogX = std::log(std::max(2.0, std::log((double)X)));
    int64_t u = (int64_t)(1.15 * std::pow((double)X / loglogX, 2.0 / 3.0));
    const int64_t S = isqrt_i64(X);
    u = std::max(u, 3 * S);
    u = std::min<int64_t>(u, 250000000000LL);
    u = ((u + 255) / 256) * 256;
    int64_t endpoint = (int64_t)(cx * std::sqrt((double)X)) + 1000;
    u = std::max(u, std::max(S + 1000, endpoint));
    endpoint = (endpoint + 255) & ~255LL;
    // dense int16 tier: at least the reference's 1.28e8 and u/16 (at most 4e9); S1 lookups
    // below it take one 2-byte gather instead of a plane word and a checkpoint
    const int64_t dense_target = std::min<int64_t>(4000000000LL, std::max<int64_t>(128000000LL, u / 16));
    const int64_t u_dense = std::min<int64_t>(u, std::max<int64_t>(endpoint, (dense_target + 255) & ~255LL));
    const int64_t N = X / u;
    const int64_t A_max = (int64_t)(cx * std::sqrt((double)X)) + 1000;
    p->u_total = u;
    p->u_dense = u_dense;
    p->cx = cx;
    p->mu_limit = std::min(u, std::max(A_max, N + 1000));
}

}  // namespace drb
