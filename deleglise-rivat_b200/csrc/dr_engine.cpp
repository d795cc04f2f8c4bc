// dr_engine.cpp -- host side (C++20) of the B200 Deleglise-Rivat engine and its C ABI.
//
// One dr_ctx owns a CUDA stream and grow-only device buffers.  A query runs as
//   table build : sieve_kernel -> seg_scan_kernel -> fixup_kernel
//   planning    : plan_kernel (op counts, constant parts) -> u64 scan
//   sums        : sums_kernel (persistent warps, device work queue)
// followed by one device->host copy of the per-query {C, S1, S2} sums.
// Nothing runs on the CPU except the parameter policy and the list of sieving
// primes up to sqrt(u); there is no CPU fallback.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dr_engine.h"
#include "dr_kernels.cuh"
#include "dr_params.hpp"

using namespace drb;

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

#define CU(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(DR_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                  \
    } while (0)

constexpr int64_t kDenseInt16Limit = 7600000000LL;  // |M(n)| < 32768 for n <= 7.6e9

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int drb::record_error(int code, const char* msg) { return fail(code, "%s", msg); }

struct dr_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint64_t budget = 0;
    uint64_t held = 0;
    // table buffers
    DevBuf dM, planes, ckpt, wheel, seg_sum, seg_off, primes, pinv, items, stencil, prcp;
    DevBuf items_odd, stencil_odd, dplanes;  // odd-mode sieve: items, stencil, dense-tier plane words
    DevBuf sq_cnt, sq_off, sq_cur, sq_pos, sq_tmp;  // bucketed square hits per segment
    // streamed table (dr_ctx_set_resident_limit): above u_resident the compressed tier
    // is built and consumed band by band in these two buffers, never held whole
    DevBuf bplanes, bckpt;
    int64_t u_resident = 0, band_values = 0;
    std::vector<cudaEvent_t> bev;  // band timing: start, then per band after its build and after its sums
    int64_t last_bands = 0;        // bands the enqueued call streams
    // query buffers
    DevBuf queries, ops, prefix, scan_tmp, acc, counts, ticket, misc, inv, invw, wdesc, witems, slots;
    // table state
    bool table_valid = false;
    int64_t t_u_total = 0, t_u_dense = 0, t_mu_limit = 0, t_nwords = 0;
    int t_S = 0;
    // host
    std::vector<uint32_t> host_primes;
    std::vector<uint64_t> host_pinv;  // per prime: floor((2^64-1)/p), then floor((2^64-1)/p^2)
    std::vector<double> host_prcp;    // per prime: RN(1/p)
    int64_t host_primes_root = -1;
    uint64_t* pinned = nullptr;  // 3 * pinned_q u64 + counts
    size_t pinned_cap = 0;
    std::vector<uint64_t> last_sums;
    cudaEvent_t ev[8] = {};
    // side stream of the table build: the segment scan and fix-up of each finished
    // sieve launch run there, beside the next sieve launch (fork/join by events)
    cudaStream_t side = nullptr;
    static constexpr int kForks = 40;
    cudaEvent_t fork[kForks] = {};
    cudaEvent_t join = nullptr;
    bool sieve_attr_set = false;
    // pinned staging for every host->device source of a call (a captured graph
    // owns its own staging, so replays never read memory a later call reuses)
    uint8_t* stage = nullptr;
    size_t stage_cap = 0, stage_used = 0;
    // pinned copy of the windowed-S1 work items (single queries only, never captured)
    S1WinItem* wstage = nullptr;
    size_t wstage_cap = 0, wstage_used = 0;
    bool capturing = false;
    struct Graph {
        std::vector<int64_t> X;
        std::vector<dr_params> P;
        dr_params tune;
        cudaGraphExec_t exec = nullptr;
        uint8_t* stage = nullptr;
        int launches = 0;
    };
    std::vector<Graph> graphs;  // replayable batch pipelines, most recent last
    bool graphs_enabled = true;
};

namespace {

void drop_graphs(dr_ctx* c) {
    for (auto& g : c->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.stage) cudaFreeHost(g.stage);
    }
    c->graphs.clear();
}

int ensure(dr_ctx* c, DevBuf& b, size_t bytes) {
    bytes = std::max<size_t>(bytes, 16);
    if (bytes <= b.cap) return DR_OK;
    if (c->capturing) return fail(DR_ERR_ARG, "internal: buffer growth during graph capture");
    drop_graphs(c);  // captured pipelines hold the old addresses
    const size_t rounded = (bytes + 255) & ~size_t(255);
    if (b.p) {
        cudaStreamSynchronize(c->stream);
        cudaFree(b.p);
        c->held -= b.cap;
        b.p = nullptr;
        b.cap = 0;
    }
    if (c->budget && c->held + rounded > c->budget)
        return fail(DR_ERR_NOMEM, "device budget exceeded: need %zu more bytes, hold %llu of %llu", rounded,
                    (unsigned long long)c->held, (unsigned long long)c->budget);
    cudaError_t e = cudaMalloc(&b.p, rounded);
    if (e != cudaSuccess) {
        b.p = nullptr;
        cudaGetLastError();
        return fail(DR_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", rounded, cudaGetErrorString(e));
    }
    b.cap = rounded;
    c->held += rounded;
    return DR_OK;
}

void release(dr_ctx* c, DevBuf& b) {
    if (b.p) {
        cudaFree(b.p);
        c->held -= b.cap;
    }
    b.p = nullptr;
    b.cap = 0;
}

// Every device buffer but the constant stencils is scratch of one call (each call
// rebuilds its table), but buffers only grow, so a context that served a call with
// other shapes can hold more than the next call leaves room for.  After the work in
// flight has finished, release them all; returns whether anything was released.
bool release_scratch(dr_ctx* c) {
    cudaStreamSynchronize(c->stream);
    cudaStreamSynchronize(c->side);
    cudaGetLastError();
    drop_graphs(c);
    DevBuf* bufs[] = {&c->dM, &c->planes, &c->ckpt, &c->wheel, &c->seg_sum, &c->seg_off, &c->primes, &c->pinv,
                      &c->items, &c->queries, &c->ops, &c->prefix, &c->scan_tmp, &c->acc, &c->counts, &c->ticket,
                      &c->misc, &c->inv, &c->invw, &c->wdesc, &c->witems, &c->slots, &c->prcp, &c->sq_cnt,
                      &c->sq_off, &c->sq_cur, &c->sq_pos, &c->sq_tmp, &c->items_odd, &c->dplanes, &c->bplanes,
                      &c->bckpt};
    bool any = false;
    for (DevBuf* b : bufs) {
        any = any || b->p;
        release(c, *b);
    }
    c->table_valid = false;
    return any;
}

// Timing events: under stream capture an event record must be an explicit
// graph node (cudaEventRecordExternal); a plain record there is only a
// dependency marker and the event would never complete.
cudaError_t record_event(dr_ctx* c, int i) {
    if (c->capturing) return cudaEventRecordWithFlags(c->ev[i], c->stream, cudaEventRecordExternal);
    return cudaEventRecord(c->ev[i], c->stream);
}

float elapsed_ms(dr_ctx* c, int a, int b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->ev[a], c->ev[b]) != cudaSuccess) {
        cudaGetLastError();  // timing is informational: never leave a sticky error behind
        ms = 0.f;
    }
    return ms;
}

int stage_reserve(dr_ctx* c, size_t bytes) {
    c->stage_used = 0;
    if (bytes <= c->stage_cap) return DR_OK;
    if (c->capturing) return fail(DR_ERR_ARG, "internal: staging growth during graph capture");
    if (c->stage) {
        cudaStreamSynchronize(c->stream);
        cudaFreeHost(c->stage);
    }
    c->stage = nullptr;
    c->stage_cap = 0;
    const size_t cap = (bytes + 4095) & ~size_t(4095);
    if (cudaMallocHost((void**)&c->stage, cap) != cudaSuccess) {
        cudaGetLastError();
        return fail(DR_ERR_NOMEM, "pinned staging allocation of %zu bytes failed", cap);
    }
    c->stage_cap = cap;
    return DR_OK;
}

// Copy `bytes` into the pinned staging area and return the pinned copy.
const void* stage_put(dr_ctx* c, const void* src, size_t bytes) {
    const size_t at = (c->stage_used + 15) & ~size_t(15);
    if (at + bytes > c->stage_cap) return nullptr;
    std::memcpy(c->stage + at, src, bytes);
    c->stage_used = at + bytes;
    return c->stage + at;
}

size_t stage_bytes_for(size_t n_primes, int64_t nq) {
    return n_primes * 28 + (size_t)kMaxSieveItems * 16 + (size_t)nq * sizeof(QueryDev) + 256;
}

// Sieving primes up to root, cached per context.
const std::vector<uint32_t>& primes_upto(dr_ctx* c, int64_t root) {
    if (c->host_primes_root == root) return c->host_primes;
    c->host_primes.clear();
    if (root >= 2) {
        std::vector<uint8_t> flag((size_t)root + 1, 1);
        for (int64_t p = 2; p <= root; ++p) {
            if (!flag[(size_t)p]) continue;
            c->host_primes.push_back((uint32_t)p);
            for (int64_t m = p * p; m <= root; m += p) flag[(size_t)m] = 0;
        }
    }
    c->host_primes_root = root;
    const size_t np = c->host_primes.size();
    c->host_pinv.assign(2 * np, 0);
    for (size_t i = 0; i < np; ++i) {
        const uint64_t p = c->host_primes[i];
        c->host_pinv[i] = ~0ull / p;
        c->host_pinv[np + i] = ~0ull / (p * p);
    }
    return c->host_primes;
}

int64_t num_candidates(int64_t N) {  // k <= N with gcd(k, 6) = 1
    if (N <= 0) return 0;
    const int64_t r = N % 6;
    return 2 * (N / 6) + (r >= 1) + (r >= 5);
}

int64_t split_point_host(double cx, int64_t y) {
    int64_t A = (int64_t)(cx * std::sqrt((double)y));
    if (A >= y) A = y - 1;
    if (A < 1) A = 1;
    return A;
}

int pick_segment(const dr_params* p) {
    int lg = (p && p->segment_log2) ? p->segment_log2 : 18;
    lg = std::max(12, std::min(lg, 18));
    return 1 << lg;
}

TableView view_of(dr_ctx* c) {
    TableView T;
    T.dM = (const int16_t*)c->dM.p;
    T.planes = (const ulonglong2*)c->planes.p;
    T.ckpt = (const int32_t*)c->ckpt.p;
    T.wheel = (const uint4*)c->wheel.p;
    T.u_dense = c->t_u_dense;
    T.u_total = c->t_u_total;
    T.mu_limit = c->t_mu_limit;
    T.cbase = 0;
    return T;
}

int check_table_limits(int64_t u_total, int64_t u_dense, int64_t mu_limit) {
    if (u_total < 1) return fail(DR_ERR_PARAMS, "u_total must be >= 1 (got %lld)", (long long)u_total);
    if (u_dense < 0 || u_dense > u_total)
        return fail(DR_ERR_PARAMS, "u_dense must be in [0, u_total] (got %lld)", (long long)u_dense);
    if (u_dense > kDenseInt16Limit)
        return fail(DR_ERR_PARAMS, "u_dense %lld exceeds the int16 prefix range (7.6e9)", (long long)u_dense);
    if (mu_limit < 0 || mu_limit > u_total)
        return fail(DR_ERR_PARAMS, "mu_limit must be in [0, u_total] (got %lld)", (long long)mu_limit);
    if (u_total > (int64_t)4000000000000LL) return fail(DR_ERR_PARAMS, "u_total above 4e12 is not supported");
    return DR_OK;
}

// The sieve's moduli for B sieved bytes per segment (S in full mode, S/2 in odd mode):
// warp items for the moduli below B/kItemDiv (uploaded into buf), one thread per prime
// above.  m.w_first and m.sq_first must be set.
int set_sieve_moduli(dr_ctx* c, const std::vector<uint32_t>& pr, int B, SieveArgs& m, DevBuf& buf) {
    m.tierB_first = std::max(m.w_first, (int)(std::lower_bound(pr.begin(), pr.end(),
                                                                (uint32_t)std::max(13, B / kItemDiv)) - pr.begin()));
    int k = m.sq_first;  // first prime whose square reaches B/kItemDiv
    while (k < (int)pr.size() && (uint64_t)pr[k] * pr[k] < (uint64_t)(B / kItemDiv)) ++k;
    m.sqB_first = k;
    std::vector<uint4> items(kMaxSieveItems);
    m.n_items = build_sieve_items(pr.data(), (int)pr.size(), B, items.data(), kMaxSieveItems);
    if (m.n_items < 0) return fail(DR_ERR_PARAMS, "sieve work items exceed %d for %d bytes per segment", kMaxSieveItems, B);
    int e = ensure(c, buf, (size_t)std::max(m.n_items, 1) * 16);
    if (e) return e;
    if (m.n_items) {
        const void* si = stage_put(c, items.data(), (size_t)m.n_items * 16);
        if (!si) return fail(DR_ERR_NOMEM, "internal: staging area too small");
        if (cudaMemcpyAsync(buf.p, si, (size_t)m.n_items * 16, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
            return fail(DR_ERR_CUDA, "sieve items upload failed");
    }
    m.items = (const uint4*)buf.p;
    return DR_OK;
}

int build_table(dr_ctx* c, int64_t u_total, int64_t u_dense, int64_t mu_limit, const dr_params* tuning,
                dr_stats* st) {
    int rc = check_table_limits(u_total, u_dense, mu_limit);
    if (rc) return rc;
    // From here on the old table is gone or being overwritten (a buffer may be
    // freed and regrown, or a launch fail partway): the table is valid again only
    // once every launch of this build has been enqueued.
    c->table_valid = false;
    const int S = pick_segment(tuning);
    const int block = (tuning && tuning->block_threads) ? tuning->block_threads : 1024;
    if (block < 128 || block > 1024 || (block & 31))
        return fail(DR_ERR_PARAMS, "block_threads must be a multiple of 32 in [128, 1024]");
    const int64_t comp = u_total - u_dense;
    const int64_t dense_segs = (u_dense + S - 1) / S;
    const int64_t comp_segs = (comp + S - 1) / S;
    const int64_t nseg = dense_segs + comp_segs;
    const int64_t nwords = (comp + 63) / 64;
    const int64_t wheel_groups = mu_limit / 192 + 2;
    if ((rc = ensure(c, c->dM, (size_t)u_dense * 2 + 64))) return rc;
    if ((rc = ensure(c, c->planes, (size_t)nwords * 16))) return rc;
    if ((rc = ensure(c, c->ckpt, (size_t)nwords * 4))) return rc;
    if ((rc = ensure(c, c->wheel, (size_t)wheel_groups * 16))) return rc;
    if ((rc = ensure(c, c->seg_sum, (size_t)nseg * 4))) return rc;
    if ((rc = ensure(c, c->seg_off, (size_t)(nseg + 1) * 4))) return rc;
    const std::vector<uint32_t>& pr = primes_upto(c, isqrt_i64(u_total));
    if ((rc = ensure(c, c->primes, pr.size() * 4))) return rc;
    if ((rc = ensure(c, c->pinv, pr.size() * 16))) return rc;
    if ((rc = ensure(c, c->prcp, pr.size() * 8))) return rc;
    if (c->host_prcp.size() != pr.size()) {
        c->host_prcp.resize(pr.size());
        for (size_t i = 0; i < pr.size(); ++i) c->host_prcp[i] = 1.0 / (double)pr[i];  // IEEE: RN(1/p)
    }
    if (!pr.empty()) {
        const void* sp = stage_put(c, pr.data(), pr.size() * 4);
        const void* sv = stage_put(c, c->host_pinv.data(), pr.size() * 16);
        const void* sr = stage_put(c, c->host_prcp.data(), pr.size() * 8);
        if (!sp || !sv || !sr) return fail(DR_ERR_NOMEM, "internal: staging area too small");
        CU(cudaMemcpyAsync(c->primes.p, sp, pr.size() * 4, cudaMemcpyHostToDevice, c->stream));
        CU(cudaMemcpyAsync(c->pinv.p, sv, pr.size() * 16, cudaMemcpyHostToDevice, c->stream));
        CU(cudaMemcpyAsync(c->prcp.p, sr, pr.size() * 8, cudaMemcpyHostToDevice, c->stream));
    }

    SieveArgs a;
    a.u_total = u_total;
    a.u_dense = u_dense;
    a.mu_limit = mu_limit;
    a.dense_segs = dense_segs;
    a.nseg = nseg;
    a.S = S;
    a.S_sub = std::min(S, kSieveFullPass);
    a.n_primes = (int)pr.size();
    auto first_at_least = [&](uint32_t v) {
        return (int)(std::lower_bound(pr.begin(), pr.end(), v) - pr.begin());
    };
    a.sq_first = first_at_least(5);
    a.w_first = first_at_least(13);
    auto set_moduli = [&](SieveArgs& m, int B, DevBuf& buf) { return set_sieve_moduli(c, pr, B, m, buf); };
    if ((rc = set_moduli(a, a.S_sub, c->items))) return rc;
    a.primes = (const uint32_t*)c->primes.p;
    a.pinv = (const u64*)c->pinv.p;
    a.sqinv = (const u64*)c->pinv.p + pr.size();
    a.prcp = (const double*)c->prcp.p;
    // squares above S hit a segment at most once: bucket their hits per segment
    // (sizes known here exactly: sum of floor(u_total / p^2) over those primes)
    int lgS = 0;
    while ((1 << lgS) < S) ++lgS;
    a.sqC_first = a.sqB_first;
    while (a.sqC_first < (int)pr.size() && (uint64_t)pr[a.sqC_first] * pr[a.sqC_first] <= (uint64_t)S) ++a.sqC_first;
    uint64_t sq_hits = 0;
    for (size_t i = (size_t)a.sqC_first; i < pr.size(); ++i) sq_hits += (uint64_t)u_total / ((uint64_t)pr[i] * pr[i]);
    a.sq_off = nullptr;
    a.sq_seg0 = 0;
    a.sq_pos = nullptr;
    if (sq_hits > 0) {
        if ((rc = ensure(c, c->sq_cnt, (size_t)nseg * 8))) return rc;
        if ((rc = ensure(c, c->sq_cur, (size_t)nseg * 8))) return rc;
        if ((rc = ensure(c, c->sq_off, (size_t)(nseg + 1) * 8))) return rc;
        if ((rc = ensure(c, c->sq_tmp, scan_u64_tmp_elems((u64)nseg) * 8))) return rc;
        if ((rc = ensure(c, c->sq_pos, (size_t)sq_hits * 4))) return rc;
        a.sq_off = (const u64*)c->sq_off.p;
        a.sq_pos = (const uint32_t*)c->sq_pos.p;
    }
    a.stencil4 = (const uint32_t*)c->stencil.p;
    a.stencil_odd4 = (const uint32_t*)c->stencil_odd.p;
    a.dM = (int16_t*)c->dM.p;
    a.planes = (ulonglong2*)c->planes.p;
    a.ckpt = (int32_t*)c->ckpt.p;
    a.cword0 = 0;
    a.hplanes = a.planes;
    a.wheel = (uint4*)c->wheel.p;
    a.seg_sum = (int32_t*)c->seg_sum.p;
    a.dplanes = nullptr;

    // Launch plan: the first wave of segments in full mode, the rest in odd mode,
    // in launches [b0, b1) whose halves lie below b0 (ranges roughly doubling).
    const size_t smem_f = sieve_smem_bytes(S, false), smem_o = sieve_smem_bytes(S, true);
    int per_f = 0, per_o = 0;
    sieve_kernel_attrs(smem_f, false, block, &per_f);
    sieve_kernel_attrs(smem_o, true, block, &per_o);
    const int64_t grid_f = (int64_t)c->sm_count * std::max(per_f, 1);
    const int64_t grid_o = (int64_t)c->sm_count * std::max(per_o, 1);
    const std::vector<SieveLaunch> plan = sieve_launch_plan(u_total, u_dense, S, grid_f);
    bool odd = false;
    for (const SieveLaunch& l : plan) odd = odd || l.odd;
    SieveArgs ao = a;
    if (odd) {
        if ((rc = ensure(c, c->dplanes, (size_t)(u_dense / 64 + 1) * 16))) return rc;
        a.dplanes = (ulonglong2*)c->dplanes.p;
        ao = a;
        if ((rc = set_moduli(ao, S / 2, c->items_odd))) return rc;
    }

    CU(record_event(c, 0));
    CU(cudaMemsetAsync(c->wheel.p, 0, (size_t)wheel_groups * 16, c->stream));
    int launches = 3;
    if (a.sq_off) {
        CU(cudaMemsetAsync(c->sq_cnt.p, 0, (size_t)nseg * 8, c->stream));
        CU(cudaMemsetAsync(c->sq_cur.p, 0, (size_t)nseg * 8, c->stream));
        launch_sq_bucket_count((const uint32_t*)c->primes.p, a.sqC_first, (int)pr.size(), 0, u_total, u_dense,
                               dense_segs, lgS, 0, (u64*)c->sq_cnt.p, c->stream);
        launch_scan_u64((const u64*)c->sq_cnt.p, (u64*)c->sq_off.p, (u64)nseg, (u64*)c->sq_tmp.p,
                        scan_u64_tmp_elems((u64)nseg), c->stream);
        launch_sq_bucket_fill((const uint32_t*)c->primes.p, a.sqC_first, (int)pr.size(), 0, u_total, u_dense,
                              dense_segs, lgS, 0, (const u64*)c->sq_off.p, (u64*)c->sq_cur.p, (uint32_t*)c->sq_pos.p,
                              c->stream);
        CU(cudaGetLastError());
        launches += 5;
    }
    // Each sieve launch covers the segments [begin, end) in order.  Once it is done, the
    // side stream scans their Mobius sums (continuing from the segments before) and
    // adds the offsets to their dense prefix values and checkpoints, while the main
    // stream sieves the next range: the fix-up, a pure memory pass, runs beside the
    // integer-bound sieve.  Nothing the sieve reads (plane words) is written by it.
    // More launches than fork events (never expected): the rest fix up at the end.
    int forks = 0;
    int64_t fixed = 0;  // segments below it are scanned and fixed up on the side stream
    for (size_t li = 0; li < plan.size(); ++li) {
        const SieveLaunch& l = plan[li];
        SieveArgs& m = l.odd ? ao : a;
        m.seg_begin = l.begin;
        m.seg_end = l.end;
        launch_sieve(m, l.odd, (int)std::max<int64_t>(1, std::min<int64_t>(l.end - l.begin, l.odd ? grid_o : grid_f)),
                     block, l.odd ? smem_o : smem_f, c->stream);
        CU(cudaGetLastError());
        if (forks < dr_ctx::kForks - 1 || li + 1 == plan.size()) {
            CU(cudaEventRecord(c->fork[forks], c->stream));
            CU(cudaStreamWaitEvent(c->side, c->fork[forks], 0));
            // beside a sieve launch the scan and fix-up stay small (one sieve CTA fills an
            // SM's shared memory, not its threads); after the last one they are the tail
            // of the build and take the whole GPU
            const bool last = li + 1 == plan.size();
            launch_seg_scan_range((const int32_t*)c->seg_sum.p, (int32_t*)c->seg_off.p, fixed, l.end,
                                  last ? 1024 : 256, c->side);
            launch_fixup_range((int16_t*)c->dM.p, u_dense, S, (const int32_t*)c->seg_off.p, (int32_t*)c->ckpt.p,
                               nwords, dense_segs, fixed, l.end, c->sm_count * (last ? 16 : 2), c->side);
            CU(cudaGetLastError());
            fixed = l.end;
            ++forks;
            launches += 2;
        }
    }
    CU(cudaEventRecord(c->join, c->side));
    CU(cudaStreamWaitEvent(c->stream, c->join, 0));
    launches += (int)plan.size() - 3;
    CU(record_event(c, 1));

    c->table_valid = true;
    c->t_u_total = u_total;
    c->t_u_dense = u_dense;
    c->t_mu_limit = mu_limit;
    c->t_nwords = nwords;
    c->t_S = S;
    if (st) st->kernel_launches += launches;
    return DR_OK;
}

// Endpoint-coverage check of one query against table limits.
int check_query(int64_t X, const dr_params& p, int64_t t_u_total, int64_t t_mu_limit) {
    if (X < 1) return DR_OK;
    if (!(p.cx > 0.0) || !(p.cx < 64.0)) return fail(DR_ERR_PARAMS, "cx must be in (0, 64)");
    if (p.u_total < 1 || p.u_total > t_u_total) return fail(DR_ERR_PARAMS, "query u exceeds table u_total");
    if (X <= t_u_total) return DR_OK;  // answered from the table
    const int64_t N = X / p.u_total;
    if (N > t_mu_limit)
        return fail(DR_ERR_PARAMS, "N = X/u = %lld exceeds mu_limit %lld", (long long)N, (long long)t_mu_limit);
    const int64_t A = split_point_host(p.cx, X);
    if (A > t_mu_limit)
        return fail(DR_ERR_PARAMS, "endpoint A = %lld exceeds mu_limit %lld", (long long)A, (long long)t_mu_limit);
    if (A > t_u_total) return fail(DR_ERR_PARAMS, "endpoint A exceeds u_total");
    return DR_OK;
}

int resolve_params(int64_t X, const dr_params* in, dr_params* out) {
    if (in) {
        *out = *in;
        return DR_OK;
    }
    return dr_default_params(X, DR_POLICY_REFERENCE, out);
}

// Work items of the windowed S1 for one query (s1win_kernel): every window of W
// values of the M table that some evaluation's windowed S1 lookups can reach, cut
// into candidate ranges of about 2^21 lookups each.  Evaluation y takes window w iff
// w < s1_win_count(y, stride) -- y >= DRB_WIN_MIN*W*(w+1)^2 at stride 1 -- and its S1
// quotients start at cx*sqrt(y/2) - 1 or above, so the candidates whose y lies in
// [DRB_WIN_MIN*W*(w+1)^2, 2*((w+1)*W + 4)^2/cx^2 + 16] cover the window (a superset:
// the kernel finds each evaluation's exact divisor range).  A candidate's work in the
// window is estimated from the overlap of its divisor range (n <= sqrt(2y)/cx or
// sqrt(y)/cx) with (y/((w+1)W), y/(wW)], sampled at geometric points of the
// candidate range and integrated; the cuts follow that estimate.
namespace {

double s1win_est(double y, int stride, uint64_t w, double W, double cx) {
    const double wc = std::floor(std::sqrt(y * W / ((double)DRB_WIN_MIN * stride)) / W);
    if ((double)w >= wc) return 0.0;
    const double nmax = (stride == 2 ? std::sqrt(2.0 * y) : std::sqrt(y)) / cx;
    const double hi = w ? std::min(y / ((double)w * W), nmax) : nmax;
    const double lo = y / ((double)(w + 1) * W);
    return hi > lo ? (hi - lo) / stride : 0.0;
}

// estimated windowed lookups of candidate c (both evaluations) in window w
double s1win_cand_est(int64_t c, uint64_t w, double W, const QueryDev& q) {
    const int64_t k = 3 * c + 1 + (c & 1);
    if (k > q.N) return 0.0;
    const int64_t N = q.N;
    const int range = k <= N / 6 ? 1 : k <= N / 3 ? 2 : k <= N / 2 ? 3 : 4;
    const double y = (double)q.X / (double)k;
    double t = s1win_est(y, range <= 3 ? 2 : 1, w, W, q.cx);
    if (range == 1) t += s1win_est(y / 3.0, 2, w, W, q.cx);
    else if (range == 2) t += s1win_est(y / 3.0, 1, w, W, q.cx);
    return t;
}

}  // namespace

std::vector<S1WinItem> s1win_items(const QueryDev& q, int qi) {
    std::vector<S1WinItem> out;
    if (q.win == 0 || q.nc <= 0) return out;
    const double W = (double)q.win, X = (double)q.X;
    const double target = 2097152.0;
    constexpr int kSamples = 32;
    std::vector<int64_t> edge;
    std::vector<double> cum;
    for (uint64_t w = 0; w < q.win_max; ++w) {
        const double ylo = (double)DRB_WIN_MIN * W * (double)(w + 1) * (double)(w + 1) * (1.0 - 1e-9) - 1.0;
        const double yhi = 2.0 * std::pow(((double)(w + 1) * W + 4.0) / q.cx, 2.0) + 16.0;
        if (ylo > X) break;  // larger windows need larger y still
        const double klo = std::max(1.0, X / (3.0 * (yhi + 1.0)) - 1.0);
        const double khi = std::min((double)q.N, X / ylo + 1.0);
        if (klo > khi) continue;
        const int64_t c0 = std::max<int64_t>(0, (int64_t)((klo - 2.0) / 3.0));
        const int64_t c1 = std::min<int64_t>(q.nc, (int64_t)(khi / 3.0) + 1);
        if (c0 >= c1) continue;
        // geometric sample edges c0 .. c1 and the integrated estimate up to each
        edge.assign(1, c0);
        for (int j = 1; j <= kSamples; ++j) {
            const int64_t e = j == kSamples ? c1
                                            : c0 + (int64_t)std::llround(std::pow((double)(c1 - c0), (double)j / kSamples)) - 1;
            if (e > edge.back() && e <= c1) edge.push_back(e);
        }
        if (edge.back() != c1) edge.push_back(c1);
        cum.assign(1, 0.0);
        for (size_t j = 1; j < edge.size(); ++j) {
            const double ga = s1win_cand_est(edge[j - 1], w, W, q), gb = s1win_cand_est(edge[j] - 1, w, W, q);
            cum.push_back(cum.back() + 0.5 * (ga + gb) * (double)(edge[j] - edge[j - 1]));
        }
        const double total = cum.back();
        // a window whose estimate is 0 may still hold a few lookups: one item
        const int64_t pieces = std::max<int64_t>(1, (int64_t)std::ceil(total / target));
        int64_t a = c0;
        size_t j = 1;
        for (int64_t i = 1; i <= pieces; ++i) {
            int64_t b = c1;
            if (i < pieces) {
                const double t = total * (double)i / (double)pieces;
                while (j + 1 < cum.size() && cum[j] < t) ++j;
                const double span = cum[j] - cum[j - 1];
                const double f = span > 0.0 ? (t - cum[j - 1]) / span : 1.0;
                b = std::min(c1, std::max(a, edge[j - 1] + (int64_t)(f * (double)(edge[j] - edge[j - 1]))));
            }
            while (a < b) {  // at most 2^15 candidates per item
                const int64_t e = std::min<int64_t>(b, a + 32768);
                out.push_back(S1WinItem{(uint32_t)w, (uint32_t)a, (uint32_t)e, (uint32_t)qi});
                a = e;
            }
        }
    }
    return out;
}

// Enqueue planning and sums for a batch of queries on the current table.
// Only stream operations: it can run under graph capture.
// A single query whose table (u_total values) exceeds the context's resident limit:
// the table holds [1, u_res] (the dense tier and the first compressed segments); the
// compressed segments above are sieved band by band, band_segs segments at a time, into
// bplanes / bckpt, and after each band a planning pass and a sums pass take the S1
// lookups whose quotient lies in that band (the idea of mertens_dr_windowed.hpp:218-374,
// which streams M windows instead of storing M up to u).  The layout of the segments
// and words is that of the whole table, so the segment scan continues across bands.
struct StreamPlan {
    int64_t u_total = 0, u_dense = 0, mu_limit = 0, u_res = 0;
    int S = 0, block = 0;
    int64_t dense_segs = 0, nseg = 0, nseg_res = 0, band_segs = 0, nbands = 0;
    std::vector<uint64_t> band_sq;  // bucketed square hits of each band
    int sqC_first = 0;
};

int64_t band_first_seg(const StreamPlan& sp, int64_t b) { return sp.nseg_res + b * sp.band_segs; }

// Values (vlo, vhi] of band b.
void band_values_of(const StreamPlan& sp, int64_t b, int64_t* vlo, int64_t* vhi) {
    const int64_t c0 = band_first_seg(sp, b), c1 = std::min(sp.nseg, c0 + sp.band_segs);
    *vlo = sp.u_dense + (c0 - sp.dense_segs) * sp.S;
    *vhi = std::min(sp.u_total, sp.u_dense + (c1 - sp.dense_segs) * sp.S);
}

// The bands of a table of ut values (dense tier ud, S-value segments) under a resident
// limit: the resident part ends on a segment boundary of the whole table's layout, at
// least one compressed segment above u_dense; sp->nbands == 0: nothing streams.
void stream_geometry(int64_t ut, int64_t ud, int S, int64_t u_resident, int64_t band_values, StreamPlan* sp) {
    *sp = StreamPlan{};
    if (u_resident <= 0 || ut <= u_resident) return;
    const int64_t res_segs = std::max<int64_t>(1, (u_resident - ud) / S);
    if (ud + res_segs * S >= ut) return;
    sp->S = S;
    sp->u_total = ut;
    sp->u_dense = ud;
    sp->u_res = ud + res_segs * S;
    sp->dense_segs = (ud + S - 1) / S;
    sp->nseg = sp->dense_segs + (ut - ud + S - 1) / S;
    sp->nseg_res = sp->dense_segs + res_segs;
    sp->band_segs = band_values > 0 ? std::max<int64_t>(1, band_values / S) : res_segs;
    sp->band_segs = std::min(sp->band_segs, sp->nseg - sp->nseg_res);
    sp->nbands = (sp->nseg - sp->nseg_res + sp->band_segs - 1) / sp->band_segs;
}

// A band whose halves n/2 all lie in the resident compressed tier (vlo >= 2 u_dense, vhi
// well below 2 u_res) can be sieved in odd mode, its even values' mu read from the
// resident plane words (odd mode needs u_dense on a 64-value word).
bool band_odd(const StreamPlan& sp, int64_t vlo, int64_t vhi) {
    return sp.u_dense % 64 == 0 && vlo >= 2 * sp.u_dense && vhi + 2 * (int64_t)sp.S <= 2 * sp.u_res;
}

// Decide whether the query streams, and reserve every buffer the bands use before the
// resident build (nothing may grow once launches are queued: the segment offsets of the
// resident table carry into the first band).  *sp.nbands == 0: no streaming.
int plan_stream(dr_ctx* c, int64_t X, int64_t ut, int64_t ud, int64_t ml, const dr_params& tune, StreamPlan* sp) {
    stream_geometry(ut, ud, pick_segment(&tune), c->u_resident, c->band_values, sp);
    if (sp->nbands == 0) return DR_OK;
    if (X <= ut) {
        *sp = StreamPlan{};
        return fail(DR_ERR_PARAMS, "a streamed table needs X > u_total (X = %lld, u_total = %lld)", (long long)X,
                    (long long)ut);
    }
    const int64_t S = sp->S;
    sp->block = tune.block_threads ? tune.block_threads : 1024;
    sp->mu_limit = ml;
    if (ml > sp->u_res) {
        *sp = StreamPlan{};
        return fail(DR_ERR_PARAMS, "mu_limit %lld above the resident table", (long long)ml);
    }
    const std::vector<uint32_t>& pr = primes_upto(c, isqrt_i64(ut));
    // squares above S go to per-band buckets (the resident build buckets its own)
    int k = 0;
    while (k < (int)pr.size() && (uint64_t)pr[k] * pr[k] <= (uint64_t)S) ++k;
    sp->sqC_first = k;
    sp->band_sq.assign((size_t)sp->nbands, 0);
    uint64_t max_sq = 0;
    for (int64_t b = 0; b < sp->nbands; ++b) {
        int64_t vlo, vhi;
        band_values_of(*sp, b, &vlo, &vhi);
        uint64_t h = 0;
        for (size_t i = (size_t)k; i < pr.size(); ++i) {
            const uint64_t q = (uint64_t)pr[i] * pr[i];
            h += (uint64_t)vhi / q - (uint64_t)vlo / q;
        }
        sp->band_sq[(size_t)b] = h;
        max_sq = std::max(max_sq, h);
    }
    const size_t bwords = (size_t)sp->band_segs * (size_t)(S / 64);
    const size_t np = pr.size();
    const size_t bsegs = (size_t)std::max(sp->band_segs, sp->nseg_res);
    int rc;
    if ((rc = ensure(c, c->seg_sum, (size_t)sp->nseg * 4))) return rc;
    if ((rc = ensure(c, c->seg_off, (size_t)(sp->nseg + 1) * 4))) return rc;
    if ((rc = ensure(c, c->primes, np * 4))) return rc;
    if ((rc = ensure(c, c->pinv, np * 16))) return rc;
    if ((rc = ensure(c, c->prcp, np * 8))) return rc;
    if ((rc = ensure(c, c->items, (size_t)kMaxSieveItems * 16))) return rc;
    if ((rc = ensure(c, c->items_odd, (size_t)kMaxSieveItems * 16))) return rc;
    if ((rc = ensure(c, c->bplanes, bwords * 16))) return rc;
    if ((rc = ensure(c, c->bckpt, bwords * 4))) return rc;
    if (max_sq > 0) {
        if ((rc = ensure(c, c->sq_cnt, bsegs * 8))) return rc;
        if ((rc = ensure(c, c->sq_cur, bsegs * 8))) return rc;
        if ((rc = ensure(c, c->sq_off, (bsegs + 1) * 8))) return rc;
        if ((rc = ensure(c, c->sq_tmp, scan_u64_tmp_elems((u64)bsegs) * 8))) return rc;
        if ((rc = ensure(c, c->sq_pos, (size_t)max_sq * 4))) return rc;
    }
    return DR_OK;
}

// The band passes of a streamed table, after the resident sums pass on the same stream:
// per band the square buckets, one full-mode sieve launch over its segments, the segment
// scan (continuing from the segments before) and fix-up, then planning (S1 lookups with q
// in the band only) and the sums kernel on the band's view of the table.
int stream_bands(dr_ctx* c, const StreamPlan& sp, const SumsArgs& base, int grid, int* launches) {
    const std::vector<uint32_t>& pr = primes_upto(c, isqrt_i64(sp.u_total));
    const size_t np = pr.size();
    std::vector<double> prcp(np);
    for (size_t i = 0; i < np; ++i) prcp[i] = 1.0 / (double)pr[i];  // IEEE: RN(1/p)
    const void* sp_ = stage_put(c, pr.data(), np * 4);
    const void* sv = stage_put(c, c->host_pinv.data(), np * 16);
    const void* sr = stage_put(c, prcp.data(), np * 8);
    if (!sp_ || !sv || !sr) return fail(DR_ERR_NOMEM, "internal: staging area too small");
    CU(cudaMemcpyAsync(c->primes.p, sp_, np * 4, cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemcpyAsync(c->pinv.p, sv, np * 16, cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemcpyAsync(c->prcp.p, sr, np * 8, cudaMemcpyHostToDevice, c->stream));
    const int S = sp.S;
    int lgS = 0;
    while ((1 << lgS) < S) ++lgS;
    SieveArgs a;  // full-mode arguments (ao: odd mode)
    a.u_total = sp.u_total;
    a.u_dense = sp.u_dense;
    a.mu_limit = sp.mu_limit;
    a.dense_segs = sp.dense_segs;
    a.nseg = sp.nseg;
    a.S = S;
    a.S_sub = std::min(S, kSieveFullPass);
    a.n_primes = (int)np;
    a.sq_first = (int)(std::lower_bound(pr.begin(), pr.end(), 5u) - pr.begin());
    a.w_first = (int)(std::lower_bound(pr.begin(), pr.end(), 13u) - pr.begin());
    int rc = set_sieve_moduli(c, pr, a.S_sub, a, c->items);
    if (rc) return rc;
    a.primes = (const uint32_t*)c->primes.p;
    a.pinv = (const u64*)c->pinv.p;
    a.sqinv = (const u64*)c->pinv.p + np;
    a.prcp = (const double*)c->prcp.p;
    const int sqC = std::max(sp.sqC_first, a.sqB_first);  // squares above S: bucketed per band
    a.sq_off = nullptr;
    a.sq_seg0 = 0;
    a.sq_pos = nullptr;
    a.stencil4 = (const uint32_t*)c->stencil.p;
    a.stencil_odd4 = (const uint32_t*)c->stencil_odd.p;
    a.dplanes = nullptr;
    a.dM = (int16_t*)c->dM.p;
    a.planes = (ulonglong2*)c->bplanes.p;
    a.ckpt = (int32_t*)c->bckpt.p;
    a.hplanes = (const ulonglong2*)c->planes.p;  // the resident compressed tier
    a.wheel = (uint4*)c->wheel.p;
    a.seg_sum = (int32_t*)c->seg_sum.p;
    const size_t smem = sieve_smem_bytes(S, false), smem_o = sieve_smem_bytes(S, true);
    int per = 0, per_o = 0;
    sieve_kernel_attrs(smem, false, sp.block, &per);
    sieve_kernel_attrs(smem_o, true, sp.block, &per_o);
    const int64_t sgrid = (int64_t)c->sm_count * std::max(per, 1);
    const int64_t sgrid_o = (int64_t)c->sm_count * std::max(per_o, 1);
    // odd-mode arguments for the bands whose halves are resident (band_odd)
    SieveArgs ao = a;
    const bool odd_ok = sp.u_dense % 64 == 0;
    if (odd_ok && (rc = set_sieve_moduli(c, pr, S / 2, ao, c->items_odd))) return rc;
    const int64_t nwords_all = (sp.u_total - sp.u_dense + 63) / 64;
    while ((int64_t)c->bev.size() < 2 * sp.nbands + 1) {
        cudaEvent_t e;
        CU(cudaEventCreate(&e));
        c->bev.push_back(e);
    }
    CU(cudaEventRecord(c->bev[0], c->stream));
    c->last_bands = sp.nbands;
    for (int64_t b = 0; b < sp.nbands; ++b) {
        const int64_t c0 = band_first_seg(sp, b), c1 = std::min(sp.nseg, c0 + sp.band_segs);
        int64_t vlo, vhi;
        band_values_of(sp, b, &vlo, &vhi);
        const int64_t cword0 = (c0 - sp.dense_segs) * (S / 64);
        const bool odd = band_odd(sp, vlo, vhi);
        SieveArgs& m = odd ? ao : a;
        m.seg_begin = c0;
        m.seg_end = c1;
        m.cword0 = cword0;
        m.sq_off = nullptr;
        m.sq_pos = nullptr;
        m.sq_seg0 = c0;
        m.sqC_first = sqC;
        if (sp.band_sq[(size_t)b] > 0 && sqC < (int)np) {
            const u64 nb = (u64)(c1 - c0);
            CU(cudaMemsetAsync(c->sq_cnt.p, 0, nb * 8, c->stream));
            CU(cudaMemsetAsync(c->sq_cur.p, 0, nb * 8, c->stream));
            launch_sq_bucket_count(m.primes, m.sqC_first, (int)np, vlo, vhi, sp.u_dense, sp.dense_segs, lgS, c0,
                                   (u64*)c->sq_cnt.p, c->stream);
            launch_scan_u64((const u64*)c->sq_cnt.p, (u64*)c->sq_off.p, nb, (u64*)c->sq_tmp.p,
                            scan_u64_tmp_elems(nb), c->stream);
            launch_sq_bucket_fill(m.primes, m.sqC_first, (int)np, vlo, vhi, sp.u_dense, sp.dense_segs, lgS, c0,
                                  (const u64*)c->sq_off.p, (u64*)c->sq_cur.p, (uint32_t*)c->sq_pos.p, c->stream);
            m.sq_off = (const u64*)c->sq_off.p;
            m.sq_pos = (const uint32_t*)c->sq_pos.p;
            *launches += 5;
        } else {
            m.sqC_first = (int)np;  // no bucketed hit in this band: squares thread-per-prime
        }
        launch_sieve(m, odd, (int)std::max<int64_t>(1, std::min<int64_t>(c1 - c0, odd ? sgrid_o : sgrid)), sp.block,
                     odd ? smem_o : smem, c->stream);
        launch_seg_scan_range((const int32_t*)c->seg_sum.p, (int32_t*)c->seg_off.p, c0, c1, 1024, c->stream);
        launch_fixup_range((int16_t*)c->dM.p, sp.u_dense, S, (const int32_t*)c->seg_off.p, (int32_t*)c->bckpt.p,
                           nwords_all, sp.dense_segs, c0, c1, c->sm_count * 16, c->stream, cword0);
        CU(cudaGetLastError());
        CU(cudaEventRecord(c->bev[(size_t)(2 * b + 1)], c->stream));
        SumsArgs sa = base;
        sa.T.planes = (const ulonglong2*)c->bplanes.p;
        sa.T.ckpt = (const int32_t*)c->bckpt.p;
        sa.T.cbase = cword0;
        CU(cudaMemsetAsync(c->ticket.p, 0, 8, c->stream));  // the work-queue counter (not the error flag)
        launch_plan(sa.queries, sa.nq, sa.T, sa.n_slots, (u64*)c->ops.p, sa.acc, (i64*)c->counts.p, nullptr,
                    (SlotDesc*)c->slots.p, c->sm_count, c->stream, S1Band{(u64)vlo + 1, (u64)vhi, 1});
        launch_scan_u64((const u64*)c->ops.p, (u64*)c->prefix.p, sa.n_slots, (u64*)c->scan_tmp.p,
                        scan_u64_tmp_elems(sa.n_slots), c->stream);
        launch_sums(sa, grid, 256, c->stream);
        CU(cudaGetLastError());
        CU(cudaEventRecord(c->bev[(size_t)(2 * b + 2)], c->stream));
        *launches += 9;
    }
    return DR_OK;
}

int enqueue_queries(dr_ctx* c, const int64_t* X, const dr_params* P, int64_t nq, const dr_params* tuning,
                    int* launches_out, const StreamPlan* sp = nullptr) {
    int rc;
    std::vector<QueryDev> qs((size_t)nq);
    u64 slots = 0;
    int64_t inv_limit = 0;  // largest S1 divisor n worth tabulating
    for (int64_t i = 0; i < nq; ++i) {
        QueryDev& q = qs[(size_t)i];
        q.X = (u64)std::max<int64_t>(X[i], 0);
        q.u = P[i].u_total;
        q.cx = P[i].cx;
        q.N = (X[i] <= c->t_u_total) ? 0 : X[i] / P[i].u_total;
        q.nc = num_candidates(q.N);
        q.slot_base = slots;
        slots += 2 * (u64)q.nc;
        if (q.N > 0) {
            // S1 divisors stay below kappa_y ~ sqrt(y)/cx and the even correction's
            // 2*kappa_{y/2} ~ sqrt(2y)/cx; larger n (never expected) fall back to udiv
            const double b = 1.4143 * std::sqrt((double)X[i]) / P[i].cx + 64.0;
            inv_limit = std::max<int64_t>(inv_limit, (int64_t)std::min(b, 4.0e9));
        }
    }
    // windowed S1: single queries (a batch keeps every lookup in the sums kernel)
    std::vector<S1WinItem> witems;
    for (int64_t i = 0; i < nq; ++i) {
        QueryDev& q = qs[(size_t)i];
        q.inv_limit = (u64)inv_limit;
        q.win = q.win_max = 0;
        // opt-in: since the S1 terms that cancel between a candidate's two evaluations
        // are left out, the direct S1 is faster at every X measured (10^15 .. 10^18)
        if (P[i].s1_window_log2 <= 0 || sp) continue;
        const int wl = P[i].s1_window_log2;
        if (nq != 1 || q.N <= 0 || wl < 12 || wl > 16) continue;
        const int64_t W = int64_t(1) << wl;
        q.win_max = (u64)(std::min<int64_t>(c->t_u_dense, (int64_t(1) << 31) - 1) / W);
        if (q.win_max < 2) continue;
        q.win = (u64)W;
        witems = s1win_items(q, (int)i);
        if (witems.empty()) q.win = q.win_max = 0;
    }
    const int64_t invw_count = c->t_mu_limit / 6 + 1;  // every S2 j <= A <= mu_limit
    if ((rc = ensure(c, c->queries, (size_t)nq * sizeof(QueryDev)))) return rc;
    if ((rc = ensure(c, c->acc, (size_t)nq * 3 * 8))) return rc;
    if ((rc = ensure(c, c->counts, (size_t)nq * kCountsPerQuery * 8))) return rc;
    if ((rc = ensure(c, c->ops, (size_t)std::max<u64>(slots, 1) * 8))) return rc;
    if ((rc = ensure(c, c->prefix, (size_t)(slots + 1) * 8))) return rc;
    if ((rc = ensure(c, c->slots, (size_t)std::max<u64>(slots, 1) * sizeof(SlotDesc)))) return rc;
    if ((rc = ensure(c, c->scan_tmp, scan_u64_tmp_elems(slots) * 8))) return rc;
    if ((rc = ensure(c, c->ticket, 32))) return rc;
    if (!witems.empty()) {
        if ((rc = ensure(c, c->wdesc, (size_t)std::max<u64>(slots, 1) * sizeof(S1WinDesc)))) return rc;
        if ((rc = ensure(c, c->witems, witems.size() * sizeof(S1WinItem)))) return rc;
    }
    if ((rc = ensure(c, c->inv, (size_t)(inv_limit + 1) * 8))) return rc;
    if ((rc = ensure(c, c->invw, (size_t)invw_count * 16))) return rc;
    const size_t need_pinned = (size_t)nq * (3 + kCountsPerQuery) + 2;
    if (c->pinned_cap < need_pinned) {
        if (c->capturing) return fail(DR_ERR_ARG, "internal: result buffer growth during graph capture");
        drop_graphs(c);
        if (c->pinned) cudaFreeHost(c->pinned);
        c->pinned = nullptr;
        CU(cudaMallocHost((void**)&c->pinned, need_pinned * 8));
        c->pinned_cap = need_pinned;
    }
    const void* sq = stage_put(c, qs.data(), (size_t)nq * sizeof(QueryDev));
    if (!sq) return fail(DR_ERR_NOMEM, "internal: staging area too small");
    const void* sw = nullptr;
    c->wstage_used = 0;
    c->last_bands = 0;
    if (!witems.empty()) {
        if (c->capturing) return fail(DR_ERR_ARG, "internal: windowed S1 under graph capture");
        if (c->wstage_cap < witems.size()) {  // the previous call's copy has completed (it synchronised)
            if (c->wstage) cudaFreeHost(c->wstage);
            c->wstage = nullptr;
            c->wstage_cap = 0;
            const size_t cap = witems.size() + witems.size() / 4 + 1024;
            CU(cudaMallocHost((void**)&c->wstage, cap * sizeof(S1WinItem)));
            c->wstage_cap = cap;
        }
        std::memcpy(c->wstage, witems.data(), witems.size() * sizeof(S1WinItem));
        c->wstage_used = witems.size() * sizeof(S1WinItem);
        sw = c->wstage;
    }
    const TableView T = view_of(c);
    const int qn = (int)nq;
    CU(record_event(c, 2));
    CU(cudaMemcpyAsync(c->queries.p, sq, (size_t)nq * sizeof(QueryDev), cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemsetAsync(c->acc.p, 0, (size_t)nq * 3 * 8, c->stream));
    CU(cudaMemsetAsync(c->counts.p, 0, (size_t)nq * kCountsPerQuery * 8, c->stream));
    CU(cudaMemsetAsync(c->ticket.p, 0, 32, c->stream));
    if (sw)
        CU(cudaMemcpyAsync(c->witems.p, sw, witems.size() * sizeof(S1WinItem), cudaMemcpyHostToDevice, c->stream));
    launch_direct((const QueryDev*)c->queries.p, qn, T, (u64*)c->acc.p, c->stream);
    int launches = 1;
    if (slots > 0) {
        launch_inverse((double*)c->inv.p, inv_limit, (double2*)c->invw.p, invw_count, T.wheel, c->sm_count,
                       c->stream);
        // a streamed table: this pass takes the S1 lookups with q <= u_res, the bands the rest
        launch_plan((const QueryDev*)c->queries.p, qn, T, slots, (u64*)c->ops.p, (u64*)c->acc.p, (i64*)c->counts.p,
                    sw ? (S1WinDesc*)c->wdesc.p : nullptr, (SlotDesc*)c->slots.p, c->sm_count, c->stream,
                    S1Band{0, sp ? (u64)sp->u_res : ~0ull, 0});
        launch_scan_u64((const u64*)c->ops.p, (u64*)c->prefix.p, slots, (u64*)c->scan_tmp.p,
                        scan_u64_tmp_elems(slots), c->stream);
        launches += 5;
    }
    CU(cudaGetLastError());
    CU(record_event(c, 3));
    if (slots > 0 && sw) {
        S1WinArgs wa;
        wa.items = (const S1WinItem*)c->witems.p;
        wa.n_items = witems.size();
        wa.desc = (const S1WinDesc*)c->wdesc.p;
        wa.queries = (const QueryDev*)c->queries.p;
        wa.T = T;
        wa.rcp = (const double*)c->inv.p;
        wa.ticket = (u64*)c->ticket.p + 2;
        wa.acc = (u64*)c->acc.p;
        launch_s1win(wa, qs[0].win, c->sm_count, c->stream);
        CU(cudaGetLastError());
        launches += 1;
    }
    if (slots > 0) {
        SumsArgs sa;
        sa.queries = (const QueryDev*)c->queries.p;
        sa.nq = qn;
        sa.T = T;
        sa.n_slots = slots;
        sa.prefix = (const u64*)c->prefix.p;
        sa.slots = (const SlotDesc*)c->slots.p;
        sa.ticket = (u64*)c->ticket.p;
        sa.acc = (u64*)c->acc.p;
        sa.chunk_log2 = tuning ? tuning->chunk_log2 : 0;
        sa.rcp = (const double*)c->inv.p;
        sa.inv_limit = inv_limit;
        sa.invw = (const double2*)c->invw.p;
        sa.invw_count = invw_count;
        int per_sm = 0;
        sums_kernel_occupancy(256, &per_sm);
        const int grid = c->sm_count * std::max(1, per_sm);
        launch_sums(sa, grid, 256, c->stream);
        CU(cudaGetLastError());
        launches += 1;
        if (sp && sp->nbands > 0) {
            rc = stream_bands(c, *sp, sa, grid, &launches);
            if (rc) return rc;
        }
    }
    CU(record_event(c, 4));
    CU(cudaMemcpyAsync(c->pinned, c->acc.p, (size_t)nq * 3 * 8, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaMemcpyAsync(c->pinned + (size_t)nq * 3, c->counts.p, (size_t)nq * kCountsPerQuery * 8, cudaMemcpyDeviceToHost,
                       c->stream));
    CU(cudaMemcpyAsync(c->pinned + (size_t)nq * (3 + kCountsPerQuery), c->ticket.p, 16, cudaMemcpyDeviceToHost,
                       c->stream));
    CU(record_event(c, 5));
    *launches_out = launches;
    return DR_OK;
}

// Wait for the enqueued work and turn the per-query sums into results.
int finish_queries(dr_ctx* c, const int64_t* X, int64_t nq, int launches, size_t h2d_bytes, int64_t* out,
                   dr_stats* st) {
    CU(cudaStreamSynchronize(c->stream));
    CU(cudaGetLastError());
    if (c->pinned[(size_t)nq * (3 + kCountsPerQuery) + 1])
        return fail(DR_ERR_DEVICE, "sums kernel: op count of an evaluation disagreed with its plan");
    for (int64_t i = 0; i < nq; ++i) {
        uint64_t* a = c->pinned + 3 * i;
        out[i] = X[i] < 1 ? 0 : (int64_t)(a[0] - a[1] - a[2]);
        // X <= u is answered from the table alone: no terms, so no checksums
        // (the reference returns get_M(X) there, mertens_dr.hpp:1465-1467)
        if (X[i] <= c->t_u_total) a[0] = a[1] = a[2] = 0;
    }
    c->last_sums.assign(c->pinned, c->pinned + (size_t)nq * 3);
    if (st) {
        st->table_ms += elapsed_ms(c, 0, 1);
        st->plan_ms += elapsed_ms(c, 2, 3);
        st->sums_ms += elapsed_ms(c, 3, 4);
        st->d2h_ms += elapsed_ms(c, 4, 5);
        for (int64_t b = 0; b < c->last_bands; ++b) {
            float t = 0.f, u = 0.f;
            if (cudaEventElapsedTime(&t, c->bev[(size_t)(2 * b)], c->bev[(size_t)(2 * b + 1)]) != cudaSuccess ||
                cudaEventElapsedTime(&u, c->bev[(size_t)(2 * b + 1)], c->bev[(size_t)(2 * b + 2)]) != cudaSuccess) {
                cudaGetLastError();  // timing is informational
                t = u = 0.f;
            }
            st->band_table_ms += t;
            st->band_sums_ms += u;
        }
        st->bands += c->last_bands;
        st->kernel_launches += launches;
        st->sieve_launches += 1;
        st->sums_launches += launches > 1 ? 1 : 0;
        st->h2d_bytes += (uint64_t)h2d_bytes;
        st->d2h_bytes += (uint64_t)nq * (3 + kCountsPerQuery) * 8 + 16;
        const uint64_t* cnt = c->pinned + (size_t)nq * 3;
        for (int64_t i = 0; i < nq; ++i) {
            const uint64_t* ci = cnt + (size_t)kCountsPerQuery * i;
            st->terms += (int64_t)ci[0];
            st->evals += (int64_t)ci[1];
            st->s1_ops += ci[2];
            st->s2_ops += ci[3];
            st->s1_comp_ops += ci[4];
        }
        if (nq == 1) {
            st->C = c->pinned[0];
            st->S1 = c->pinned[1];
            st->S2 = c->pinned[2];
            st->M = out[0];
        }
    }
    return DR_OK;
}

// Capture the whole batch pipeline (table build, planning, sums, result copy)
// into a CUDA graph for replay by the next identical call.  Runs right after an
// eager run of the same batch, so no buffer grows during capture.  Failing to
// capture is not an error: the batch simply keeps running eagerly.
void capture_graph(dr_ctx* c, const int64_t* X, const dr_params* P, int64_t nq, const dr_params& tune, int64_t ut,
                   int64_t ud, int64_t ml, size_t n_primes) {
    if (c->graphs.size() >= 4) {
        if (c->graphs.front().exec) cudaGraphExecDestroy(c->graphs.front().exec);
        if (c->graphs.front().stage) cudaFreeHost(c->graphs.front().stage);
        c->graphs.erase(c->graphs.begin());
    }
    dr_ctx::Graph g;
    g.X.assign(X, X + nq);
    g.P.assign(P, P + nq);
    g.tune = tune;
    const size_t need = stage_bytes_for(n_primes, nq);
    if (cudaMallocHost((void**)&g.stage, need) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    uint8_t* saved = c->stage;
    const size_t saved_cap = c->stage_cap, saved_used = c->stage_used;
    c->stage = g.stage;
    c->stage_cap = need;
    c->stage_used = 0;
    c->capturing = true;
    int rc = DR_ERR_CUDA;
    int launches = 0;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
        rc = build_table(c, ut, ud, ml, &tune, nullptr);
        if (rc == DR_OK) rc = enqueue_queries(c, X, P, nq, &tune, &launches);
        if (cudaStreamEndCapture(c->stream, &graph) != cudaSuccess) rc = DR_ERR_CUDA;
    }
    c->capturing = false;
    c->stage = saved;
    c->stage_cap = saved_cap;
    c->stage_used = saved_used;
    if (rc == DR_OK && graph && cudaGraphInstantiate(&g.exec, graph, 0) == cudaSuccess) {
        g.launches = launches + 3;
        c->graphs.push_back(std::move(g));
    } else {
        if (g.stage) cudaFreeHost(g.stage);
    }
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
}

bool same_batch(const dr_ctx::Graph& g, const int64_t* X, const dr_params* P, int64_t nq, const dr_params& tune) {
    if ((int64_t)g.X.size() != nq) return false;
    if (std::memcmp(g.X.data(), X, (size_t)nq * 8) != 0) return false;
    if (std::memcmp(g.P.data(), P, (size_t)nq * sizeof(dr_params)) != 0) return false;
    return std::memcmp(&g.tune, &tune, sizeof(dr_params)) == 0;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* dr_last_error(void) { return g_err; }

int dr_device_info(int device, int* sm_count, uint64_t* hbm_bytes) {
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    if (sm_count) *sm_count = prop.multiProcessorCount;
    if (hbm_bytes) *hbm_bytes = prop.totalGlobalMem;
    return DR_OK;
}

int dr_ctx_create(int device, void* cuda_stream, dr_ctx** out) {
    if (!out) return fail(DR_ERR_ARG, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    CU(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(DR_ERR_ARG, "device %d out of range (%d devices)", device, ndev);
    CU(cudaSetDevice(device));
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return fail(DR_ERR_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a", device, prop.major,
                    prop.minor);
    dr_ctx* c = new dr_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    if (cuda_stream) {
        c->stream = (cudaStream_t)cuda_stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return fail(DR_ERR_CUDA, "cudaStreamCreate failed");
        }
        c->own_stream = true;
    }
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    c->budget = (uint64_t)((double)free_b * 0.92);
    for (auto& e : c->ev) cudaEventCreate(&e);
    for (auto& e : c->fork) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming);
    if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess) {
        c->side = nullptr;
        dr_ctx_destroy(c);
        return fail(DR_ERR_CUDA, "cudaStreamCreate (side stream) failed");
    }
    init_piece_constants();
    std::vector<uint32_t> st = make_stencil4();
    std::vector<uint32_t> sto = make_stencil_odd4();
    int rc = ensure(c, c->stencil, st.size() * 4);
    if (!rc) rc = ensure(c, c->stencil_odd, sto.size() * 4);
    if (rc) {
        dr_ctx_destroy(c);
        return rc;
    }
    cudaMemcpy(c->stencil.p, st.data(), st.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(c->stencil_odd.p, sto.data(), sto.size() * 4, cudaMemcpyHostToDevice);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        dr_ctx_destroy(c);
        return fail(DR_ERR_CUDA, "context init failed: %s", cudaGetErrorString(e));
    }
    *out = c;
    return DR_OK;
}

int dr_ctx_destroy(dr_ctx* c) {
    if (!c) return DR_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    DevBuf* bufs[] = {&c->dM, &c->planes, &c->ckpt, &c->wheel, &c->seg_sum, &c->seg_off, &c->primes, &c->pinv, &c->items, &c->stencil,
                      &c->queries, &c->ops, &c->prefix, &c->scan_tmp, &c->acc, &c->counts, &c->ticket, &c->misc,
                      &c->inv, &c->invw, &c->wdesc, &c->witems, &c->slots, &c->prcp, &c->sq_cnt, &c->sq_off, &c->sq_cur,
                      &c->sq_pos, &c->sq_tmp, &c->items_odd, &c->stencil_odd, &c->dplanes, &c->bplanes, &c->bckpt};
    for (DevBuf* b : bufs) release(c, *b);
    drop_graphs(c);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->stage) cudaFreeHost(c->stage);
    if (c->wstage) cudaFreeHost(c->wstage);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->bev) cudaEventDestroy(e);
    if (c->side) {
        cudaStreamSynchronize(c->side);
        cudaStreamDestroy(c->side);
    }
    for (auto& e : c->fork)
        if (e) cudaEventDestroy(e);
    if (c->join) cudaEventDestroy(c->join);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return DR_OK;
}

int dr_ctx_set_resident_limit(dr_ctx* c, int64_t u_resident, int64_t band_values) {
    if (!c) return fail(DR_ERR_ARG, "ctx is NULL");
    if (u_resident < 0 || band_values < 0) return fail(DR_ERR_ARG, "u_resident and band_values must be >= 0");
    c->u_resident = u_resident;
    c->band_values = band_values;
    return DR_OK;
}

int dr_ctx_set_hbm_budget(dr_ctx* c, uint64_t bytes) {
    if (!c) return fail(DR_ERR_ARG, "ctx is NULL");
    if (bytes == 0) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        bytes = (uint64_t)((double)(free_b + c->held) * 0.92);
    }
    c->budget = bytes;
    return DR_OK;
}

int dr_default_params(int64_t X, int policy, dr_params* out) {
    if (!out) return fail(DR_ERR_ARG, "out is NULL");
    params_clear(out);
    if (X < 1) {
        out->cx = ref_choose_cx(X);
        return DR_OK;
    }
    switch (policy) {
    case DR_POLICY_REFERENCE:
        if (ref_use_compressed(X)) ref_compressed_params(X, out);
        else ref_dense_params(X, out);
        return DR_OK;
    case DR_POLICY_DENSE: ref_dense_params(X, out); return DR_OK;
    case DR_POLICY_COMPRESSED:
        if (X <= 100000LL) ref_dense_params(X, out);
        else ref_compressed_params(X, out);
        return DR_OK;
    case DR_POLICY_GPU:
        if (X <= 100000LL) ref_dense_params(X, out);
        else gpu_params(X, out);
        return DR_OK;
    case DR_POLICY_REFERENCE_GPU: ref_gpu_params(X, 0, out); return DR_OK;
    }
    return fail(DR_ERR_ARG, "unknown policy %d", policy);
}

int dr_reference_gpu_params(int64_t X, int host_threads, dr_params* out) {
    if (!out) return fail(DR_ERR_ARG, "out is NULL");
    params_clear(out);
    if (X < 1) {
        out->cx = ref_choose_cx(X);
        return DR_OK;
    }
    ref_gpu_params(X, host_threads, out);
    return DR_OK;
}

uint64_t dr_table_bytes(int64_t u_total, int64_t u_dense, int64_t mu_limit) {
    const int64_t comp = std::max<int64_t>(0, u_total - u_dense);
    const int64_t nwords = (comp + 63) / 64;
    const int64_t nseg = (u_total + 4095) / 4096 + 2;
    // + bucketed square hits: u * sum over primes p^2 > S of 1/p^2 < u / (sqrt(S) ln sqrt(S)),
    // 4 bytes each, for the default S = 2^17 (at most 0.0019 u bytes)
    // + the dense tier's plane words (16 bytes per 64 values) that the odd-mode sieve reads
    return (uint64_t)u_dense * 2 + (uint64_t)(u_dense / 64 + 1) * 16 + (uint64_t)nwords * 20 +
           (uint64_t)(mu_limit / 192 + 2) * 16 + (uint64_t)nseg * 32 + (uint64_t)u_total / 500;
}

uint64_t dr_query_bytes(int64_t X, const dr_params* p) {
    if (!p || X < 1) return 0;
    uint64_t b = dr_table_bytes(p->u_total, p->u_dense, p->mu_limit);
    if (X > p->u_total && p->cx > 0.0) {
        const double inv = 1.4143 * std::sqrt((double)X) / p->cx + 65.0;  // S1 reciprocals
        const int64_t slots = 2 * num_candidates(X / p->u_total);        // ops + prefix
        b += (uint64_t)(8.0 * inv) + (uint64_t)(p->mu_limit / 6 + 1) * 16 + (uint64_t)slots * (16 + sizeof(SlotDesc)) +
             scan_u64_tmp_elems((u64)slots) * 8;
    }
    return b;
}

int dr_check_params(int64_t X, const dr_params* p, uint64_t hbm_budget) {
    if (!p) return fail(DR_ERR_ARG, "params is NULL");
    if (X < 1) return DR_OK;
    int rc = check_table_limits(p->u_total, p->u_dense, p->mu_limit);
    if (rc) return rc;
    if ((rc = check_query(X, *p, p->u_total, p->mu_limit))) return rc;
    if (hbm_budget && dr_query_bytes(X, p) > hbm_budget)
        return fail(DR_ERR_NOMEM, "query needs %llu device bytes, budget %llu",
                    (unsigned long long)dr_query_bytes(X, p), (unsigned long long)hbm_budget);
    return DR_OK;
}

int dr_table_build(dr_ctx* c, int64_t u_total, int64_t u_dense, int64_t mu_limit, const dr_params* tuning,
                   dr_stats* st) {
    if (!c) return fail(DR_ERR_ARG, "ctx is NULL");
    CU(cudaSetDevice(c->device));
    const double t0 = now_ms();
    const size_t stage = stage_bytes_for(primes_upto(c, isqrt_i64(std::max<int64_t>(u_total, 0))).size(), 0);
    int rc = stage_reserve(c, stage);
    if (rc) return rc;
    rc = build_table(c, u_total, u_dense, mu_limit, tuning, st);
    if (rc == DR_ERR_NOMEM && release_scratch(c)) {  // retry once without the buffers of earlier calls
        if (st) std::memset(st, 0, sizeof(*st));
        rc = stage_reserve(c, stage);
        if (!rc) rc = build_table(c, u_total, u_dense, mu_limit, tuning, st);
    }
    if (rc) return rc;
    CU(cudaStreamSynchronize(c->stream));
    if (st) {
        st->table_ms += elapsed_ms(c, 0, 1);
        st->total_ms += now_ms() - t0;
    }
    return DR_OK;
}

int dr_mertens(dr_ctx* c, int64_t X, const dr_params* p, int64_t* out, dr_stats* st) {
    return dr_mertens_batch(c, &X, 1, p, out, st);
}

int dr_mertens_batch(dr_ctx* c, const int64_t* X, int64_t count, const dr_params* p, int64_t* out, dr_stats* st) {
    if (!c || !X || !out) return fail(DR_ERR_ARG, "NULL argument");
    if (count < 1 || count > (1 << 20)) return fail(DR_ERR_ARG, "count must be in [1, 2^20]");
    CU(cudaSetDevice(c->device));
    const double t0 = now_ms();
    if (st) std::memset(st, 0, sizeof(*st));
    std::vector<dr_params> P((size_t)count);
    int64_t ut = 1, ud = 0, ml = 0;
    bool any = false;
    for (int64_t i = 0; i < count; ++i) {
        int rc = resolve_params(X[i], p ? p + i : nullptr, &P[(size_t)i]);
        if (rc) return rc;
        if (X[i] < 1) continue;
        any = true;
        rc = check_table_limits(P[i].u_total, P[i].u_dense, P[i].mu_limit);
        if (rc) return rc;
        ut = std::max(ut, P[i].u_total);
        ud = std::max(ud, P[i].u_dense);
        ml = std::max(ml, P[i].mu_limit);
    }
    if (!any) {
        for (int64_t i = 0; i < count; ++i) out[i] = 0;
        return DR_OK;
    }
    for (int64_t i = 0; i < count; ++i) {
        if (X[i] < 1) continue;
        int rc = check_query(X[i], P[(size_t)i], ut, ml);
        if (rc) return rc;
    }
    // tuning knobs (segment length, block shape, work-item size) come from p[0]
    dr_params tune;
    params_clear(&tune);
    if (p) {
        tune.segment_log2 = p[0].segment_log2;
        tune.block_threads = p[0].block_threads;
        tune.chunk_log2 = p[0].chunk_log2;
    }
    // a batch seen before replays its captured CUDA graph: one graph launch
    // rebuilds the table and recomputes every query
    if (count > 1) {
        for (auto& g : c->graphs) {
            if (!same_batch(g, X, P.data(), count, tune)) continue;
            c->table_valid = false;  // the graph rebuilds the table in place
            CU(cudaGraphLaunch(g.exec, c->stream));
            c->table_valid = true;
            c->t_u_total = ut;
            c->t_u_dense = ud;
            c->t_mu_limit = ml;
            c->t_nwords = (ut - ud + 63) / 64;
            int rc = finish_queries(c, X, count, g.launches, stage_bytes_for(c->host_primes.size(), count), out, st);
            if (rc) return rc;
            if (st) st->total_ms = now_ms() - t0;
            return DR_OK;
        }
    }
    const size_t n_primes = primes_upto(c, isqrt_i64(ut)).size();
    int launches = 0;
    int rc = DR_OK;
    for (int attempt = 0; attempt < 2; ++attempt) {
        // a second attempt only after a budget or allocation failure that released
        // the buffers kept from earlier, larger calls
        if (attempt == 1 && !(rc == DR_ERR_NOMEM && release_scratch(c))) break;
        if (st) std::memset(st, 0, sizeof(*st));
        launches = 0;
        // a single query above the resident limit streams its table (plan_stream
        // reserves the bands' buffers first; the resident build then covers [1, u_res])
        StreamPlan sp;
        rc = count == 1 ? plan_stream(c, X[0], ut, ud, ml, tune, &sp) : DR_OK;
        const bool streamed = sp.nbands > 0;
        const size_t n_res = streamed ? primes_upto(c, isqrt_i64(sp.u_res)).size() : 0;
        if (!rc) rc = stage_reserve(c, stage_bytes_for(n_primes + n_res, count) + (streamed ? kMaxSieveItems * 16 : 0));
        if (!rc) rc = build_table(c, streamed ? sp.u_res : ut, ud, ml, &tune, st);
        if (!rc) rc = enqueue_queries(c, X, P.data(), count, &tune, &launches, streamed ? &sp : nullptr);
        if (!rc) break;
    }
    if (rc) return rc;
    rc = finish_queries(c, X, count, launches, c->stage_used + c->wstage_used, out, st);
    if (rc) return rc;
    if (st) st->total_ms = now_ms() - t0;
    if (count > 1 && c->graphs_enabled) capture_graph(c, X, P.data(), count, tune, ut, ud, ml, n_primes);
    return DR_OK;
}

// One candidate of the batch autotuner: every query shares a table of
// u = m * (B200-policy u of the largest X) values and uses all of it.
static int batch_candidate(const int64_t* X, int64_t n, double m, double cx, int seg, int block, int chunk,
                           std::vector<dr_params>& P) {
    int64_t xmax = 1;
    for (int64_t i = 0; i < n; ++i) xmax = std::max(xmax, X[i]);
    dr_params base;
    dr_default_params(xmax, DR_POLICY_GPU, &base);
    int64_t ut = (int64_t)((double)base.u_total * m);
    ut = std::min<int64_t>(std::max<int64_t>(ut, 64), 250000000000LL);
    ut = ((ut + 255) / 256) * 256;
    int64_t amax = 0, nmax = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (X[i] < 1) continue;
        amax = std::max<int64_t>(amax, (int64_t)(cx * std::sqrt((double)X[i])) + 1000);
        nmax = std::max<int64_t>(nmax, X[i] / ut + 1000);
    }
    const int64_t ud = std::min<int64_t>(ut, std::max<int64_t>((amax + 255) & ~255LL, std::min<int64_t>(128000000LL, ((ut / 4 + 255) & ~255LL))));
    const int64_t ml = std::min(ut, std::max(amax, nmax));
    P.assign((size_t)n, dr_params{});
    for (int64_t i = 0; i < n; ++i) {
        dr_params& q = P[(size_t)i];
        params_clear(&q);
        q.u_total = ut;
        q.u_dense = ud;
        q.cx = cx;
        q.mu_limit = ml;
        q.segment_log2 = seg;
        q.block_threads = block;
        q.chunk_log2 = chunk;
        if (X[i] >= 1 && check_query(X[i], q, ut, ml) != DR_OK) return DR_ERR_PARAMS;
    }
    return DR_OK;
}

int dr_autotune_batch(dr_ctx* c, const int64_t* X, int64_t count, int max_trials, dr_params* out, double* best_ms) {
    if (!c || !X || !out || count < 1) return fail(DR_ERR_ARG, "bad argument");
    const bool saved_graphs = c->graphs_enabled;
    c->graphs_enabled = false;  // trials run eagerly; only the winner is worth a graph
    std::vector<int64_t> res((size_t)count);
    struct State { double m, cx; int seg, block, chunk; } cur{1.0, 1.2, 18, 1024, 0}, best_state = cur;
    double best = 1e300;
    int trials = 0;
    if (max_trials <= 0) max_trials = 24;
    auto eval = [&](const State& st_) -> double {
        std::vector<dr_params> P;
        if (batch_candidate(X, count, st_.m, st_.cx, st_.seg, st_.block, st_.chunk, P) != DR_OK) return 1e300;
        if (dr_check_params(1, &P[0], c->budget / 2) != DR_OK) return 1e300;
        if (dr_table_bytes(P[0].u_total, P[0].u_dense, P[0].mu_limit) > c->budget / 2) return 1e300;
        double t = 1e300;
        for (int rep = 0; rep < 2; ++rep) {
            dr_stats st;
            if (dr_mertens_batch(c, X, count, P.data(), res.data(), &st) != DR_OK) return 1e300;
            t = std::min(t, st.table_ms + st.plan_ms + st.sums_ms);
        }
        ++trials;
        return t;
    };
    best = eval(cur);
    best_state = cur;
    const double ms[] = {0.25, 0.5, 2.0, 4.0, 8.0, 16.0};
    const double cxs[] = {0.9, 1.05, 1.4, 1.7};
    const int segs[] = {16, 17};
    const int blocks[] = {512};
    const int chunks[] = {12, 14, 16};
    for (int pass = 0; pass < 2 && trials < max_trials; ++pass) {
        for (double v : ms) {
            if (trials >= max_trials) break;
            State t = best_state;
            t.m = v;
            if (t.m == best_state.m) continue;
            const double r = eval(t);
            if (r < best) best = r, best_state = t;
        }
        for (double v : cxs) {
            if (trials >= max_trials) break;
            State t = best_state;
            t.cx = v;
            const double r = eval(t);
            if (r < best) best = r, best_state = t;
        }
        for (int v : segs) {
            if (trials >= max_trials) break;
            State t = best_state;
            t.seg = v;
            const double r = eval(t);
            if (r < best) best = r, best_state = t;
        }
        for (int v : blocks) {
            if (trials >= max_trials) break;
            State t = best_state;
            t.block = v;
            const double r = eval(t);
            if (r < best) best = r, best_state = t;
        }
        for (int v : chunks) {
            if (trials >= max_trials) break;
            State t = best_state;
            t.chunk = v;
            const double r = eval(t);
            if (r < best) best = r, best_state = t;
        }
    }
    c->graphs_enabled = saved_graphs;
    std::vector<dr_params> P;
    if (best >= 1e299 || batch_candidate(X, count, best_state.m, best_state.cx, best_state.seg, best_state.block,
                                         best_state.chunk, P) != DR_OK)
        return fail(DR_ERR_PARAMS, "autotune found no valid configuration");
    std::memcpy(out, P.data(), (size_t)count * sizeof(dr_params));
    if (best_ms) *best_ms = best;
    return DR_OK;
}

int dr_batch_checksums(dr_ctx* c, uint64_t* out3, int64_t count) {
    if (!c || !out3) return fail(DR_ERR_ARG, "NULL argument");
    if ((size_t)count * 3 > c->last_sums.size()) return fail(DR_ERR_ARG, "count exceeds the last batch");
    std::memcpy(out3, c->last_sums.data(), (size_t)count * 3 * 8);
    return DR_OK;
}

int dr_table_read(dr_ctx* c, int64_t first, int64_t count, int32_t* M, int8_t* mu) {
    if (!c) return fail(DR_ERR_ARG, "ctx is NULL");
    if (!c->table_valid) return fail(DR_ERR_ARG, "no table built");
    if (count < 0) return fail(DR_ERR_ARG, "negative count");
    if (count == 0) return DR_OK;
    CU(cudaSetDevice(c->device));
    int rc = ensure(c, c->misc, (size_t)count * 6);
    if (rc) return rc;
    int32_t* dM = (int32_t*)c->misc.p;
    int8_t* dmu = (int8_t*)((char*)c->misc.p + (size_t)count * 4);
    launch_table_read(view_of(c), first, count, M ? dM : nullptr, mu ? dmu : nullptr, nullptr, c->stream);
    CU(cudaGetLastError());
    if (M) CU(cudaMemcpyAsync(M, dM, (size_t)count * 4, cudaMemcpyDeviceToHost, c->stream));
    if (mu) CU(cudaMemcpyAsync(mu, dmu, (size_t)count, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return DR_OK;
}

// Mobius values as stored in the wheel (0 for n sharing a factor with 6).
int dr_table_read_wheel(dr_ctx* c, int64_t first, int64_t count, int8_t* mu) {
    if (!c || !mu) return fail(DR_ERR_ARG, "NULL argument");
    if (!c->table_valid) return fail(DR_ERR_ARG, "no table built");
    if (count <= 0) return DR_OK;
    CU(cudaSetDevice(c->device));
    int rc = ensure(c, c->misc, (size_t)count);
    if (rc) return rc;
    launch_table_read(view_of(c), first, count, nullptr, nullptr, (int8_t*)c->misc.p, c->stream);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(mu, c->misc.p, (size_t)count, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return DR_OK;
}

int dr_table_checksums(dr_ctx* c, dr_table_sums* out) {
    if (!c || !out) return fail(DR_ERR_ARG, "NULL argument");
    if (!c->table_valid) return fail(DR_ERR_ARG, "no table built");
    CU(cudaSetDevice(c->device));
    int rc = ensure(c, c->misc, 64);
    if (rc) return rc;
    CU(cudaMemsetAsync(c->misc.p, 0, 48, c->stream));
    launch_table_sums(view_of(c), c->t_nwords, (u64*)c->misc.p, c->sm_count, c->stream);
    CU(cudaGetLastError());
    uint64_t h[6];
    CU(cudaMemcpyAsync(h, c->misc.p, 48, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    out->dense_sum = h[0];
    out->dense_wsum = h[1];
    out->mu_wsum = h[2];
    out->nz_wsum = h[3];
    out->neg_wsum = h[4];
    out->ckpt_wsum = h[5];
    return DR_OK;
}

static int debug_udiv(dr_ctx* c, const uint64_t* y, const uint64_t* d, int64_t n, uint64_t* q, int rcp) {
    if (!c || !y || !d || !q || n < 0) return fail(DR_ERR_ARG, "bad argument");
    if (n == 0) return DR_OK;
    CU(cudaSetDevice(c->device));
    int rc = ensure(c, c->misc, (size_t)n * 24);
    if (rc) return rc;
    u64* dy = (u64*)c->misc.p;
    u64* dd = dy + n;
    u64* dq = dd + n;
    CU(cudaMemcpyAsync(dy, y, (size_t)n * 8, cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemcpyAsync(dd, d, (size_t)n * 8, cudaMemcpyHostToDevice, c->stream));
    launch_debug_udiv(dy, dd, dq, n, rcp, c->stream);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(q, dq, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return DR_OK;
}

int dr_debug_udiv(dr_ctx* c, const uint64_t* y, const uint64_t* d, int64_t n, uint64_t* q) {
    return debug_udiv(c, y, d, n, q, 0);
}

int dr_debug_udiv_rcp(dr_ctx* c, const uint64_t* y, const uint64_t* d, int64_t n, uint64_t* q) {
    return debug_udiv(c, y, d, n, q, 1);
}

int dr_debug_udiv32(dr_ctx* c, const uint64_t* y, const uint64_t* d, int64_t n, uint64_t* q) {
    return debug_udiv(c, y, d, n, q, 2);
}

static int debug_piece(dr_ctx* c, const int32_t* piece, const uint64_t* q, int64_t n, int64_t* out, int fast) {
    if (!c || !piece || !q || !out || n < 0) return fail(DR_ERR_ARG, "bad argument");
    if (n == 0) return DR_OK;
    CU(cudaSetDevice(c->device));
    int rc = ensure(c, c->misc, (size_t)n * 20);
    if (rc) return rc;
    u64* dq = (u64*)c->misc.p;
    i64* dout = (i64*)(dq + n);
    int32_t* dp = (int32_t*)(dout + n);
    CU(cudaMemcpyAsync(dq, q, (size_t)n * 8, cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemcpyAsync(dp, piece, (size_t)n * 4, cudaMemcpyHostToDevice, c->stream));
    launch_debug_piece(dp, dq, dout, n, fast, c->stream);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(out, dout, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return DR_OK;
}

int dr_debug_piece(dr_ctx* c, const int32_t* piece, const uint64_t* q, int64_t n, int64_t* out) {
    return debug_piece(c, piece, q, n, out, 0);
}

int dr_debug_piece32(dr_ctx* c, const int32_t* piece, const uint64_t* q, int64_t n, int64_t* out) {
    return debug_piece(c, piece, q, n, out, 1);
}

int64_t dr_debug_stream_plan(int64_t u_total, int64_t u_dense, int32_t segment_log2, int64_t u_resident,
                             int64_t band_values, int64_t* u_res, int64_t* out, int64_t cap) {
    if (!u_res || (cap > 0 && !out) || segment_log2 < 12 || segment_log2 > 18 || u_dense < 0 || u_dense > u_total)
        return DR_ERR_ARG;
    StreamPlan sp;
    stream_geometry(u_total, u_dense, 1 << segment_log2, u_resident, band_values, &sp);
    *u_res = sp.nbands ? sp.u_res : u_total;
    for (int64_t b = 0; b < sp.nbands && b < cap; ++b) {
        band_values_of(sp, b, out + 3 * b, out + 3 * b + 1);
        out[3 * b + 2] = band_odd(sp, out[3 * b], out[3 * b + 1]) ? 1 : 0;
    }
    return sp.nbands;
}

int64_t dr_debug_sieve_plan(int64_t u_total, int64_t u_dense, int32_t segment_log2, int64_t first_wave,
                            int64_t* out, int64_t cap) {
    if (u_total < 1 || u_dense < 0 || u_dense > u_total || segment_log2 < 12 || segment_log2 > 18 || first_wave < 1 ||
        cap < 0 || (cap > 0 && !out))
        return fail(DR_ERR_ARG, "dr_debug_sieve_plan: bad arguments");
    const std::vector<SieveLaunch> plan = sieve_launch_plan(u_total, u_dense, 1 << segment_log2, first_wave);
    for (size_t i = 0; i < plan.size() && (int64_t)i < cap; ++i) {
        out[3 * i] = plan[i].begin;
        out[3 * i + 1] = plan[i].end;
        out[3 * i + 2] = plan[i].odd ? 1 : 0;
    }
    return (int64_t)plan.size();
}

}  // extern "C"
