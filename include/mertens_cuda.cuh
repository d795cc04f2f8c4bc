// mertens_cuda.cuh -- drop-in for the reference's GPU engine header.
//
// Keeps the entry signature of ecreeth/deleglise-rivat mertens_cuda.cuh
// (namespace mertens_cuda, CudaDelégliseRivatEngine::compute_mertens(int64 X,
// int host_threads, TimingStats*) :441 and its TimingStats :410-416) and
// forwards to the B200 engine through the C ABI.  Unlike the reference, the
// Mobius sieve and both Mertens tables are built on the GPU, so
// host_sieve_time reports the device time of the table build; kernel_time is
// the planning + S1/S2 device time.  Errors throw std::runtime_error, as the
// reference's CUDA_CHECK does (mertens_cuda.cuh:20-28).
#ifndef MERTENS_CUDA_B200_SHIM_CUH
#define MERTENS_CUDA_B200_SHIM_CUH

#include "mertens_dr.hpp"

namespace mertens_cuda {

using int64 = long long;
using uint64 = unsigned long long;

class CudaDelégliseRivatEngine {
public:
    struct TimingStats {
        double host_sieve_time = 0.0;  // device time of the table build (seconds)
        double h2d_copy_time = 0.0;
        double kernel_time = 0.0;      // planning + S1/S2 (seconds)
        double d2h_copy_time = 0.0;
        double total_time = 0.0;       // wall time of the call (seconds)
    };

    // choose_gpu_sieve_limit :421-436: the reference GPU engine's u for X and its
    // host thread count (it caps u lower for 1 or 2 threads)
    static inline int64 choose_gpu_sieve_limit(int64 X, int threads) {
        dr_params p;
        mertens_dr::b200::check(dr_reference_gpu_params(X, threads > 0 ? threads : 0, &p));
        return X <= 50000000LL ? X : (int64)p.u_total;
    }

    // The parameters are the reference GPU engine's for (X, host_threads):
    // dr_reference_gpu_params restates them, so M(X) and the intermediate sums are
    // those of the same decomposition.
    static int64 compute_mertens(int64 X, int host_threads = 0, TimingStats* stats = nullptr) {
        if (X < 1) return 0;
        dr_stats st;
        dr_params p;
        int64_t out = 0;
        mertens_dr::b200::check(dr_reference_gpu_params(X, host_threads, &p));
        mertens_dr::b200::check(dr_mertens(mertens_dr::b200::context(), X, &p, &out, &st));
        if (stats) {
            stats->host_sieve_time = st.table_ms / 1e3;
            stats->h2d_copy_time = st.h2d_ms / 1e3;
            stats->kernel_time = (st.plan_ms + st.sums_ms) / 1e3;
            stats->d2h_copy_time = st.d2h_ms / 1e3;
            stats->total_time = st.total_ms / 1e3;
        }
        return (int64)out;
    }
};

}  // namespace mertens_cuda

#endif
