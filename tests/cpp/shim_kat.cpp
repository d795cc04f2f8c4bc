// Drop-in check: the reference's own call pattern (test_dr.cpp:52-67,
// test_cuda.cu:65-99) compiled against the B200 shims include/mertens_dr.hpp
// and include/mertens_cuda.cuh, linked with libdrb200.so.  Exit code 0/1 like
// the reference's test executables.
#include <cstdio>
#include <vector>

#include "mertens_cuda.cuh"
#include "mertens_dr.hpp"

int main() {
    using mertens_dr::int64;
    struct Case { int64 X, M; };
    const std::vector<Case> cases = {
        {1, 1}, {2, 0}, {3, -1}, {4, -1}, {5, -2}, {10, -1}, {100, 1}, {1000, 2}, {10000, -23},
        {100000, -48}, {1000000, 212}, {10000000, 1037}, {100000000, 1928}, {1000000000, -222},
        {10000000000LL, -33722}, {100000000000LL, -87856}, {1000000000000LL, 62366},
        {10000000000000LL, 599582}, {100000000000000LL, -875575}, {1000000000000000LL, -3216373},
        {10000000000000000LL, -3195437}};
    int failed = 0;
    for (const Case& c : cases) {
        const int64 a = mertens_dr::DelégliseRivatEngine::compute_mertens(c.X);
        mertens_cuda::CudaDelégliseRivatEngine::TimingStats st;
        const int64 b = mertens_cuda::CudaDelégliseRivatEngine::compute_mertens(c.X, 0, &st);
        const int64 d = c.X >= 100000 ? mertens_dr::DelégliseRivatEngine::compute_compressed(c.X, 0) : c.M;
        const bool ok = a == c.M && b == c.M && d == c.M;
        if (!ok) ++failed;
        std::printf("%s M(%lld) = %lld / %lld / %lld  (table %.4f s, kernels %.4f s)\n", ok ? "[PASS]" : "[FAIL]",
                    c.X, a, b, d, st.host_sieve_time, st.kernel_time);
    }
    if (mertens_dr::DelégliseRivatEngine::compute_mertens(0) != 0) ++failed;
    if (mertens_dr::DelégliseRivatEngine::compute_compressed(0, 0) != 0) ++failed;
    std::printf("%d failed\n", failed);
    return failed ? 1 : 0;
}
