// ref_gpu_params.cu -- C ABI over the reference GPU engine's parameter heuristic
// (TEST INFRASTRUCTURE ONLY: the checker of dr_reference_gpu_params).
//
// Compiled from the reference's own header mertens_cuda.cuh (where it lies) by
// `make ref`; exposes CudaDelégliseRivatEngine::choose_gpu_sieve_limit
// (mertens_cuda.cuh:421-436) and the cx / mu limit that compute_mertens derives
// from it (:473, :492).  Nothing here launches a kernel.
#include "mertens_cuda.cuh"

extern "C" long long ref_gpu_sieve_limit(long long X, int threads) {
    return mertens_cuda::CudaDelégliseRivatEngine::choose_gpu_sieve_limit(X, threads);
}

extern "C" double ref_gpu_cx(long long X) { return mertens_dr::DelégliseRivatEngine::choose_cx(X); }

// mu limit of compute_mertens for (X, u) (mertens_cuda.cuh:474, :492)
extern "C" long long ref_gpu_mu_limit(long long X, long long u) {
    const double cx = mertens_dr::DelégliseRivatEngine::choose_cx(X);
    const long long N = X / u;
    return std::min(u, std::max(N, static_cast<long long>(cx * std::sqrt(static_cast<double>(X)))) + 65536LL);
}
