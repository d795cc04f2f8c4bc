// mertens_dr.hpp -- drop-in for the reference's CPU engine header.
//
// Keeps the entry signatures of ecreeth/deleglise-rivat mertens_dr.hpp
// (namespace mertens_dr, DelégliseRivatEngine::compute_mertens :968,
// ::compute_compressed :1442, choose_cx :914, choose_sieve_limit :931,
// choose_compressed_limit :1401) and forwards every call to the B200 engine
// through the C ABI in dr_engine.h.  Link with -ldrb200.  There is no CPU
// fallback: without a usable sm_100 device the calls throw.
//
// Behaviour kept from the reference: values in, values out; X < 1 gives 0;
// MERTENS_CX / MERTENS_FX / MERTENS_U_CAP / MERTENS_USE_CHMT /
// MERTENS_CHMT_U_CAP are read on every call and select the same parameters;
// errors surface as exceptions (std::runtime_error here, std::bad_alloc in
// the reference's CPU path).  The thread count arguments are accepted and
// ignored: the work runs on the GPU.
#ifndef MERTENS_DR_B200_SHIM_HPP
#define MERTENS_DR_B200_SHIM_HPP

#include <cstdlib>
#include <stdexcept>
#include <string>

#include "dr_engine.h"

namespace mertens_dr {

using int64 = long long;
using uint64 = unsigned long long;

namespace b200 {

// One engine context per host thread (a dr_ctx is not thread-safe), on the
// device named by DR_DEVICE (default 0).
inline dr_ctx* context() {
    struct Holder {
        dr_ctx* ctx = nullptr;
        ~Holder() {
            if (ctx) dr_ctx_destroy(ctx);
        }
    };
    thread_local Holder h;
    if (!h.ctx) {
        const char* d = std::getenv("DR_DEVICE");
        const int dev = d ? std::atoi(d) : 0;
        if (dr_ctx_create(dev, nullptr, &h.ctx) != DR_OK)
            throw std::runtime_error(std::string("B200 engine unavailable: ") + dr_last_error());
    }
    return h.ctx;
}

inline void check(int rc) {
    if (rc != DR_OK) throw std::runtime_error(std::string("B200 engine: ") + dr_last_error());
}

inline dr_params params(int64 X, int policy) {
    dr_params p;
    check(dr_default_params(X, policy, &p));
    return p;
}

}  // namespace b200

inline int64 isqrt(int64 n) noexcept {
    if (n <= 0) return 0;
    uint64 s = 0;
    for (int b = 31; b >= 0; --b) {
        const uint64 t = s | (1ULL << b);
        if (t * t <= (uint64)n) s = t;
    }
    return (int64)s;
}

class DelégliseRivatEngine {
public:
    static constexpr int64 COMPRESSED_THRESHOLD = 100000000000LL;
    static constexpr int64 DENSE_LIMIT = 128000000LL;

    static double choose_cx(int64 X) { return b200::params(X, DR_POLICY_DENSE).cx; }

    static int64 choose_sieve_limit(int64 X, int threads) {
        (void)threads;
        return X <= 0 ? X : b200::params(X, DR_POLICY_DENSE).u_total;
    }

    static int64 choose_compressed_limit(int64 X) {
        return X <= 100000LL ? X : b200::params(X, DR_POLICY_COMPRESSED).u_total;
    }

    // M(X) with the reference's own parameter choice (dense or streamed table).
    static int64 compute_mertens(int64 X, int num_threads = 0) {
        (void)num_threads;
        if (X < 1) return 0;
        int64_t out = 0;
        b200::check(dr_mertens(b200::context(), X, nullptr, &out, nullptr));
        return (int64)out;
    }

    // M(X) with the streamed-table parameters.
    static int64 compute_compressed(int64 X, int threads) {
        (void)threads;
        if (X < 1) return 0;
        const dr_params p = b200::params(X, DR_POLICY_COMPRESSED);
        int64_t out = 0;
        b200::check(dr_mertens(b200::context(), X, &p, &out, nullptr));
        return (int64)out;
    }
};

}  // namespace mertens_dr

#endif
