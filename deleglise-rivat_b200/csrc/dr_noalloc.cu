// dr_noalloc.cu -- a table build that allocates no memory at all.
//
// Who needs it: code that owns device memory through its own allocator and is
// not allowed to call cudaMalloc/cudaFree behind that allocator's back -- a
// framework's caching allocator, a memory pool reserved up front, a service
// that must not allocate once it is serving.  Such a caller hands in the table
// buffers it allocated itself; everything else the build needs (per-segment
// Mobius sums and their offsets, the sieving primes, the periodic stencil)
// lives in one file-scope __device__ array of fixed size.
//
// It runs the same kernels as dr_table_build() (sieve_kernel, seg_scan_kernel,
// fixup_kernel) and produces the same table, bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/dr_engine.h"
#include "dr_kernels.cuh"

using namespace drb;

namespace {

constexpr int kNoAllocSegLog2 = 17;
constexpr int kNoAllocSeg = 1 << kNoAllocSegLog2;          // values per sieve segment
constexpr int64_t kNoAllocMaxSegs = DR_NOALLOC_MAX_U / kNoAllocSeg + 2;  // dense + compressed runs
constexpr int kNoAllocMaxRoot = 92681;                       // isqrt(DR_NOALLOC_MAX_U)
constexpr int kNoAllocMaxPrimes = 9216;                      // pi(92681) = 8952
constexpr int kMaxDevices = 64;

// scratch layout, in 32-bit words
constexpr size_t kOffStencil = 0;
constexpr size_t kOffSegSum = kOffStencil + (size_t)4 * kStencilWords;
constexpr size_t kOffSegOff = kOffSegSum + (size_t)kNoAllocMaxSegs;
constexpr size_t kOffPrimes = kOffSegOff + (size_t)kNoAllocMaxSegs;
constexpr size_t kOffPinv = kOffPrimes + (size_t)kNoAllocMaxPrimes;     // u64 reciprocals of p
constexpr size_t kOffSqinv = kOffPinv + 2 * (size_t)kNoAllocMaxPrimes;  // u64 reciprocals of p^2
constexpr size_t kOffItems = kOffSqinv + 2 * (size_t)kNoAllocMaxPrimes;   // uint4 sieve work items
constexpr size_t kScratchWords = kOffItems + 4 * (size_t)kMaxSieveItems;  // 796,848 bytes
static_assert(kOffPinv % 2 == 0 && kOffSqinv % 2 == 0, "u64 tables need 8-byte alignment");
static_assert(kOffItems % 4 == 0, "uint4 items need 16-byte alignment");

// The scratch.  In host code this name is only a host-side stand-in for the
// symbol, never a device address: the device address comes from
// cudaGetSymbolAddress() below, on every call, with the device current.
static __device__ __align__(256) uint32_t g_table_scratch[kScratchWords];

// Host-side constant inputs, filled once per process (static storage, no heap).
uint32_t g_host_primes[kNoAllocMaxPrimes];
uint64_t g_host_pinv[kNoAllocMaxPrimes];
uint64_t g_host_sqinv[kNoAllocMaxPrimes];
int g_host_prime_count = 0;
uint32_t g_host_stencil[4 * kStencilWords];
uint4 g_host_items[kMaxSieveItems];
int g_host_item_count = 0;
std::once_flag g_host_once;

void fill_host_constants() {
    static uint8_t composite[kNoAllocMaxRoot + 1];
    for (int64_t p = 2; p <= kNoAllocMaxRoot; ++p) {
        if (composite[p]) continue;
        g_host_pinv[g_host_prime_count] = ~0ull / (uint64_t)p;
        g_host_sqinv[g_host_prime_count] = ~0ull / (uint64_t)(p * p);
        g_host_primes[g_host_prime_count++] = (uint32_t)p;
        for (int64_t m = p * p; m <= kNoAllocMaxRoot; m += p) composite[m] = 1;
    }
    // a negative count means the items did not fit (set-up then fails)
    g_host_item_count = build_sieve_items(g_host_primes, g_host_prime_count, kNoAllocSeg, g_host_items, kMaxSieveItems);
    // periodic stencil, 4 copies shifted by 0..3 bytes; byte i describes n = i + 1
    auto stencil_byte = [](int i) -> uint32_t {
        const int n = (i % kStencilPeriod) + 1;
        uint32_t a = 0;
        const int small[5] = {2, 3, 5, 7, 11};
        for (int p : small)
            if (n % p == 0) a += (uint32_t)((32 - __builtin_clz((unsigned)(p - 1))) | 1);
        if (n % 4 == 0 || n % 9 == 0) a |= 0x80u;
        return a;
    };
    for (int s = 0; s < 4; ++s)
        for (int w = 0; w < kStencilWords; ++w) {
            uint32_t v = 0;
            for (int b = 0; b < 4; ++b) v |= stencil_byte(4 * w + s + b) << (8 * b);
            g_host_stencil[(size_t)s * kStencilWords + (size_t)w] = v;
        }
}

// Per-device set-up state.  `done` is set only after a set-up that succeeded, so
// a failed set-up is retried by the next call.  `ctx_id` is the unique id of the
// CUDA context the set-up ran in: a device reset (cudaDeviceReset, or any other
// replacement of the primary context) reloads the module, which loses the
// scratch's contents and may move it, so a call in another context runs the
// set-up again.
struct DeviceSetup {
    std::mutex mu;
    bool done = false;
    unsigned long long ctx_id = 0;
    uint32_t* scratch = nullptr;  // device address of g_table_scratch on this device
    int sieve_per_sm = 1;
    int sm_count = 1;
};
DeviceSetup g_dev[kMaxDevices];

// Unique id of the current CUDA context (cuCtxGetId through the runtime's driver
// entry points, so that the library needs no link against libcuda).
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
std::once_flag g_entry_once;

void load_entry_points() {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_get_current = (CtxGetCurrentFn)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_get_id = (CtxGetIdFn)f;
    cudaGetLastError();
}

// 0 where the id cannot be read (set-up then keys on the scratch address alone)
unsigned long long current_ctx_id() {
    std::call_once(g_entry_once, load_entry_points);
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!g_ctx_get_current || !g_ctx_get_id || g_ctx_get_current(&ctx) != 0 || !ctx) return 0;
    if (g_ctx_get_id(ctx, &id) != 0) return 0;
    return id;
}

int noalloc_fail(int code, const char* msg, cudaError_t e = cudaSuccess) {
    char buf[256];
    if (e != cudaSuccess) snprintf(buf, sizeof(buf), "dr_table_build_noalloc: %s: %s", msg, cudaGetErrorString(e));
    else snprintf(buf, sizeof(buf), "dr_table_build_noalloc: %s", msg);
    return record_error(code, buf);
}

// With the device current and d.mu held: fill the scratch's constant parts
// (stencil, primes, reciprocals, work items) at device address ptr.  Returns
// DR_OK and marks the set-up done only when every step succeeded.
int setup_device(int device, DeviceSetup& d, uint32_t* ptr, unsigned long long ctx_id) {
    std::call_once(g_host_once, fill_host_constants);
    d.done = false;
    if (g_host_item_count < 0) return noalloc_fail(DR_ERR_ARG, "sieve work items exceed their fixed capacity");
    cudaError_t e = cudaMemcpy(ptr + kOffStencil, g_host_stencil, sizeof(g_host_stencil), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(ptr + kOffPrimes, g_host_primes, sizeof(uint32_t) * (size_t)g_host_prime_count,
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(ptr + kOffPinv, g_host_pinv, sizeof(uint64_t) * (size_t)g_host_prime_count,
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(ptr + kOffSqinv, g_host_sqinv, sizeof(uint64_t) * (size_t)g_host_prime_count,
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(ptr + kOffItems, g_host_items, sizeof(uint4) * (size_t)g_host_item_count,
                       cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return noalloc_fail(DR_ERR_CUDA, "filling the table scratch failed", e);
    e = cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return noalloc_fail(DR_ERR_CUDA, "cudaDeviceGetAttribute failed", e);
    int per_sm = 0;
    sieve_kernel_attrs(sieve_smem_bytes(kNoAllocSeg, false), false, 1024, &per_sm);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(DR_ERR_CUDA, "sieve kernel attributes failed", e);
    d.sieve_per_sm = std::max(per_sm, 1);
    d.scratch = ptr;
    d.ctx_id = ctx_id;
    d.done = true;
    return DR_OK;
}

int count_primes_upto(int64_t x) {  // over the static host list
    int lo = 0, hi = g_host_prime_count;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if ((int64_t)g_host_primes[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

int64_t isqrt_exact(int64_t n) {
    if (n <= 0) return 0;
    uint64_t s = (uint64_t)std::sqrt((double)n);
    while ((s + 1) * (s + 1) <= (uint64_t)n) ++s;
    while (s * s > (uint64_t)n) --s;
    return (int64_t)s;
}

}  // namespace

extern "C" int dr_table_build_noalloc(int device, void* stream, int64_t u_total, int64_t u_dense, int64_t mu_limit,
                                      int16_t* dM, void* planes, int32_t* ckpt, void* wheel) {
    if (device < 0 || device >= kMaxDevices) return noalloc_fail(DR_ERR_ARG, "device index out of range");
    if (u_total < 1 || u_total > DR_NOALLOC_MAX_U)
        return noalloc_fail(DR_ERR_ARG, "u_total must be in [1, DR_NOALLOC_MAX_U = 2^33]");
    if (u_dense < 0 || u_dense > u_total) return noalloc_fail(DR_ERR_ARG, "u_dense must be in [0, u_total]");
    if (u_dense > 7600000000LL) return noalloc_fail(DR_ERR_ARG, "u_dense exceeds the int16 prefix range (7.6e9)");
    if (mu_limit < 0 || mu_limit > u_total) return noalloc_fail(DR_ERR_ARG, "mu_limit must be in [0, u_total]");
    const int64_t comp = u_total - u_dense;
    const int64_t nwords = (comp + 63) / 64;
    if ((u_dense > 0 && !dM) || (nwords > 0 && (!planes || !ckpt)) || !wheel)
        return noalloc_fail(DR_ERR_ARG, "a table buffer is NULL");
    if (((uintptr_t)dM & 15) || ((uintptr_t)planes & 15) || ((uintptr_t)wheel & 15) || ((uintptr_t)ckpt & 3))
        return noalloc_fail(DR_ERR_ARG, "dM, planes and wheel must be 16-byte aligned, ckpt 4-byte aligned");

    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return noalloc_fail(DR_ERR_CUDA, "cudaGetDevice failed", e);
    if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess)
        return noalloc_fail(DR_ERR_CUDA, "cudaSetDevice failed", e);
    DeviceSetup& d = g_dev[device];
    int rc = DR_OK;
    {
        // The scratch's device address, looked up on every call (cheap): a device
        // reset reloads the module, and the set-up reruns when the address or the
        // context changed.  A set-up copies synchronously, which is illegal under
        // stream capture, so it refuses a capturing stream before touching it.
        std::lock_guard<std::mutex> lock(d.mu);
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_table_scratch);
        if (e != cudaSuccess || !ptr) {
            rc = noalloc_fail(DR_ERR_CUDA, "cudaGetSymbolAddress(g_table_scratch) failed", e);
        } else {
            const unsigned long long id = current_ctx_id();
            if (!d.done || d.scratch != (uint32_t*)ptr || d.ctx_id != id) {
                cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
                e = cudaStreamIsCapturing((cudaStream_t)stream, &cs);
                if (e != cudaSuccess) rc = noalloc_fail(DR_ERR_CUDA, "cudaStreamIsCapturing failed", e);
                else if (cs != cudaStreamCaptureStatusNone)
                    rc = noalloc_fail(DR_ERR_ARG, "the first call on a device (or after a device reset) sets up the "
                                                  "scratch synchronously and must not run under stream capture");
                else rc = setup_device(device, d, (uint32_t*)ptr, id);
            }
        }
    }
    if (rc == DR_OK) {
        cudaStream_t s = (cudaStream_t)stream;
        const int S = kNoAllocSeg;
        const int64_t dense_segs = (u_dense + S - 1) / S;
        const int64_t nseg = dense_segs + (comp + S - 1) / S;
        const int64_t root = isqrt_exact(u_total);
        SieveArgs a;
        a.u_total = u_total;
        a.u_dense = u_dense;
        a.mu_limit = mu_limit;
        a.dense_segs = dense_segs;
        a.nseg = nseg;
        a.seg_begin = 0;  // every segment in full mode: no scratch for the dense tier's planes
        a.seg_end = nseg;
        a.dplanes = nullptr;
        a.stencil_odd4 = nullptr;
        a.S = S;
        a.S_sub = S;
        a.n_primes = count_primes_upto(root);
        a.sq_first = std::min(a.n_primes, count_primes_upto(4));
        a.w_first = std::min(a.n_primes, count_primes_upto(12));
        a.tierB_first = std::max(a.w_first, std::min(a.n_primes, count_primes_upto(S / kItemDiv - 1)));
        a.sqB_first = std::max(a.sq_first, std::min(a.n_primes, count_primes_upto(isqrt_exact(S / kItemDiv - 1))));
        a.n_items = sieve_items_prefix(g_host_items, g_host_item_count, a.n_primes);
        a.items = (const uint4*)(d.scratch + kOffItems);
        a.primes = d.scratch + kOffPrimes;
        a.pinv = (const u64*)(d.scratch + kOffPinv);
        a.sqinv = (const u64*)(d.scratch + kOffSqinv);
        a.prcp = nullptr;  // offsets from the 64-bit reciprocals, squares without a bucket
        a.sqC_first = a.n_primes;
        a.sq_off = nullptr;
        a.sq_seg0 = 0;
        a.sq_pos = nullptr;
        a.stencil4 = d.scratch + kOffStencil;
        a.dM = dM;
        a.planes = (ulonglong2*)planes;
        a.ckpt = ckpt;
        a.cword0 = 0;
        a.hplanes = (const ulonglong2*)planes;
        a.wheel = (uint4*)wheel;
        a.seg_sum = (int32_t*)(d.scratch + kOffSegSum);
        int32_t* seg_off = (int32_t*)(d.scratch + kOffSegOff);
        const int64_t wheel_groups = mu_limit / 192 + 2;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(nseg, (int64_t)d.sm_count * d.sieve_per_sm));
        // the wheel is OR-ed into, so it must start at zero; everything in the
        // scratch that this call reads it also writes first
        e = cudaMemsetAsync(wheel, 0, (size_t)wheel_groups * 16, s);
        if (e == cudaSuccess) {
            launch_sieve(a, false, grid, 1024, sieve_smem_bytes(S, false), s);
            launch_seg_scan(a.seg_sum, seg_off, nseg, s);
            launch_fixup(dM, u_dense, S, seg_off, ckpt, nwords, dense_segs, d.sm_count, s);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) rc = noalloc_fail(DR_ERR_CUDA, "table build launch failed", e);
    }
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    return rc;
}
