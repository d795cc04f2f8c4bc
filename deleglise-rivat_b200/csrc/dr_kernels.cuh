// dr_kernels.cuh -- kernel argument blocks and launch wrappers (host side).
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "dr_device.cuh"

namespace drb {

constexpr int kStencilPeriod = 13860;                       // lcm(4, 9, 5, 7, 11)
constexpr int kStencilWords = (kStencilPeriod + 3 + 3) / 4;  // words per shifted copy
// Odd-value stencil: entry k describes the odd n = 2k + 1 (mod 2 * 3465): weights of
// 3, 5, 7, 11 and the square flag of 9 (lcm(9, 5, 7, 11) = 3465 odd values).
constexpr int kStencilOddPeriod = 3465;
// Values per full-mode pass: the full-mode shared buffer holds one byte per value.
constexpr int kSieveFullPass = 1 << 17;
constexpr int kStencilOddWords = (kStencilOddPeriod + 3 + 3) / 4;

// The sieve runs in two modes over the same segments of S values.  Full mode
// sieves every value of a segment.  Odd mode sieves its odd values only (half the
// marks, stencil and finalisation) and takes each even value from the Mobius bits
// of its half, mu(2m) = -mu(m) for odd m and 0 for even m, read from the 64-value
// plane words of the values <= u_total / 2 that earlier launches wrote: the
// compressed planes above u_dense and the scratch planes `dplanes` below it.  A
// launch covers segments [seg_begin, seg_end); odd-mode launches are ordered so that
// every half they read lies in segments of earlier launches.
struct SieveArgs {
    i64 u_total, u_dense, mu_limit;
    i64 dense_segs, nseg;
    i64 seg_begin, seg_end;  // segments of this launch
    int S;              // values per segment (multiple of 4096)
    int S_sub;          // values per full-mode pass: min(S, kSieveFullPass)
    int n_primes;       // primes <= isqrt(u_total), ascending
    int sq_first;       // first prime >= 5 (square flags)
    int w_first;        // first prime >= 13 (weights)
    int tierB_first;    // first prime whose weights are marked thread-per-prime (p >= B/kItemDiv)
    int sqB_first;      // first prime whose square is marked thread-per-prime (p^2 >= B/kItemDiv)
    int n_items;        // warp work items for the smaller moduli (see build_sieve_items)
    const uint4* items; // {modulus, start offset, weight or 0x80, prime index | square bit 31}
    const uint32_t* primes;
    const u64* pinv;           // floor((2^64-1)/p) per prime: segment offsets without division
    const u64* sqinv;          // floor((2^64-1)/p^2) per prime
    const double* prcp;        // RN(1/p) per prime (32-bit offset route; NULL: umod_inv only)
    int sqC_first;             // first prime whose square is bucketed (p^2 > S); n_primes: none
    const u64* sq_off;         // bucketed square hits of each segment from sq_seg0 on (NULL: no bucket)
    i64 sq_seg0;               // segment of sq_off[0] (0, or a streamed band's first segment)
    const uint32_t* sq_pos;    // their positions within the segment
    const uint32_t* stencil4;  // 4 copies shifted by 0..3 bytes, kStencilWords each (full mode)
    const uint32_t* stencil_odd4;  // the same for the odd-value stencil, kStencilOddWords each
    ulonglong2* dplanes;       // {nonzero, negative} plane words of the values <= u_dense
                               // (64 per word; NULL: not written, odd mode unavailable)
    int16_t* dM;
    ulonglong2* planes;
    int32_t* ckpt;
    i64 cword0;                // compressed-tier word held in planes[0] / ckpt[0] (0, or a
                               // streamed band's first word)
    const ulonglong2* hplanes; // the compressed tier's plane words from word 0, where odd mode
                               // reads the halves (planes itself, or the resident table's
                               // planes for a streamed band whose halves are resident)
    uint4* wheel;
    int32_t* seg_sum;
};

// One evaluation as seen by s1win_kernel (written by plan_kernel): its S1 segments
// (divisors s1_n_at(n0, |sg|, i), i < cnt) with sign sg/|sg| (mu(k) times the
// segment's sign), and the windows [w0, wc) in which each segment has windowed lookups.
struct S1WinDesc {
    u64 y;
    uint32_t n0[kS1Seg];   // first divisor (first wheel index for S1_WHEEL segments)
    uint32_t cnt[kS1Seg];
    uint32_t w0[kS1Seg];   // first window holding a lookup: floor(y / n_last) / W
    uint32_t wc[kS1Seg];
    int32_t sg[kS1Seg];    // +-stride code (1, 2, 6 or S1_WHEEL); 0: no S1 segment
};

// Work item of s1win_kernel: window w of query q, evaluation candidates [c0, c1).
struct S1WinItem {
    uint32_t w, c0, c1, q;
};

struct S1WinArgs {
    const S1WinItem* items;
    u64 n_items;
    const S1WinDesc* desc;  // per evaluation slot
    const QueryDev* queries;
    TableView T;
    const double* rcp;      // RN(1/n), n <= inv_limit
    u64* ticket;            // work-queue counter, zeroed before launch
    u64* acc;               // [3 * nq]: C, S1, S2
};

struct SumsArgs {
    const QueryDev* queries;
    int nq;
    TableView T;
    u64 n_slots;
    const u64* prefix;  // [n_slots + 1] exclusive op prefix
    const SlotDesc* slots;  // [n_slots] each slot's evaluation, written by plan_kernel
    u64* ticket;        // [0]: work-queue counter, [1]: error flag; zeroed before launch
    u64* acc;           // [3 * nq]: C, S1, S2
    int chunk_log2;     // 0: chosen on the device from the total
    const double* rcp;       // rcp[n] = RN(1/n), 1 <= n <= inv_limit (< 2^32)
    i64 inv_limit;
    const double2* invw;     // invw[m] = {rcp(6m+1), rcp(6m+5)} with mu(j) in the low bits, m < invw_count
    i64 invw_count;
};

void launch_sieve(const SieveArgs& a, bool odd, int grid, int block, size_t smem, cudaStream_t s);
// Bucketed squares: the multiples m*p^2 in (vlo, vhi] of the primes p = primes[first..n)
// (p^2 > S: at most one per segment), counted per segment, then written per segment
// in the order of off = exclusive scan of the counts (cur: zeroed cursors); bucket
// arrays indexed by segment - seg0 (the whole table: vlo = seg0 = 0, vhi = u_total).
void launch_sq_bucket_count(const uint32_t* primes, int first, int n, i64 vlo, i64 vhi, i64 u_dense, i64 dense_segs,
                            int lgS, i64 seg0, u64* counts, cudaStream_t s);
void launch_sq_bucket_fill(const uint32_t* primes, int first, int n, i64 vlo, i64 vhi, i64 u_dense, i64 dense_segs,
                           int lgS, i64 seg0, const u64* off, u64* cur, uint32_t* pos, cudaStream_t s);

// Moduli with at least kItemDiv hits in the B bytes a segment sieves (m < B/kItemDiv)
// are marked by warp work items, larger ones one prime per thread (at most kItemDiv
// hits each).  64 measured best: the M(10^16) table takes 20.36 ms against 20.68 ms
// with 32 and 21.10 ms with 24 (48: 20.36 ms).
constexpr int kItemDiv = 64;
// Hits per warp item: 2048 measured best (the M(10^16) table: 20.04 ms against 20.41 with
// 1024, 20.56 with 512, 20.30 with 4096, 20.46 with 8192).
constexpr int kItemHits = 2048;

// Warp work items for the sieve's smaller moduli: the multiples of every prime
// 13 <= p < S/kItemDiv (log weights) and of every square p^2 < S/kItemDiv, p >= 5 (flags),
// cut into pieces of at most kItemHits hits (32 lanes x 64 strides), so that the
// warps of a CTA get equal shares of the marking instead of one warp holding
// p = 13.  Items are ordered by prime index: the items valid for the first n
// primes are a prefix.  Returns the count written (<= cap), or -1 if the items
// do not fit in cap (none is ever dropped silently: a missing item would leave
// marks out and the Mobius values wrong).  For the sieved bytes per segment used
// here (at most 2^17) there are fewer than 700 items.
constexpr int kMaxSieveItems = 2048;
int build_sieve_items(const uint32_t* primes, int n_primes, int S, uint4* out, int cap);
// Number of leading items whose prime index is below n_primes.
int sieve_items_prefix(const uint4* items, int n_items, int n_primes);
size_t sieve_smem_bytes(int S, bool odd);
// Segment offsets out[i] = sum of in[j < i] for i <= n (out holds n + 1 entries).
void launch_seg_scan(const int32_t* in, int32_t* out, i64 n, cudaStream_t s);
// The same for the segments [b0, b1) given out[b0] (written by the range before,
// 0 for b0 = 0); also writes out[b1].  One CTA of `threads` (32 .. 1024, a multiple of 32).
void launch_seg_scan_range(const int32_t* in, int32_t* out, i64 b0, i64 b1, int threads, cudaStream_t s);
// Offsets added to the dense prefix and the checkpoints of the segments [b0, b1).
// cword0: the compressed-tier word held in ckpt[0] (0 for a whole table, a band's
// first word for a streamed band)
void launch_fixup_range(int16_t* dM, i64 u_dense, int S, const int32_t* seg_off, int32_t* ckpt, i64 nwords,
                        i64 dense_segs, i64 b0, i64 b1, int blocks, cudaStream_t s, i64 cword0 = 0);
void launch_fixup(int16_t* dM, i64 u_dense, int S, const int32_t* seg_off, int32_t* ckpt, i64 nwords,
                  i64 dense_segs, int sm_count, cudaStream_t s);
// Per-query counters written by plan_kernel: counts[kCountsPerQuery*q + 0..4] =
// outer terms, evaluations, S1 lookups, S2 wheel positions, and the S1 lookups
// whose quotient lies in the compressed tier (q > u_dense).
constexpr int kCountsPerQuery = 5;
// A band pass of a streamed table: evaluations with at most this many S1 lookups in the
// band are summed by the planning thread itself (ops 0 for the sums kernel).
constexpr int kBandInThread = 64;
void launch_plan(const QueryDev* q, int nq, const TableView& T, u64 n_slots, u64* ops, u64* acc,
                 i64* counts, S1WinDesc* wdesc, SlotDesc* slots, int sm_count, cudaStream_t s,
                 const S1Band& band = S1Band{0, ~0ull, 0});
// Windowed S1 (window length win: a power of two, 2^12 .. 2^16).
void launch_s1win(const S1WinArgs& a, u64 win, int sm_count, cudaStream_t s);
void launch_scan_u64(const u64* in, u64* out, u64 n, u64* tmp, size_t tmp_elems, cudaStream_t s);
size_t scan_u64_tmp_elems(u64 n);
void launch_sums(const SumsArgs& a, int grid, int block, cudaStream_t s);
// Reciprocal tables shared by every evaluation of a launch.
void launch_inverse(double* rcp, i64 inv_limit, double2* invw, i64 invw_count, const uint4* wheel, int sm_count,
                    cudaStream_t s);
void launch_direct(const QueryDev* q, int nq, const TableView& T, u64* acc, cudaStream_t s);
void launch_table_read(const TableView& T, i64 first, i64 count, int32_t* M, int8_t* mu, int8_t* wheel_mu,
                       cudaStream_t s);
void launch_table_sums(const TableView& T, i64 nwords, u64* out6, int sm_count, cudaStream_t s);
void init_piece_constants();
// Record a message for dr_last_error() (fixed thread-local buffer) and return code.
int record_error(int code, const char* msg);
// Opt the sieve kernel into `smem` bytes of dynamic shared memory and report
// how many CTAs of `block` threads fit on one SM.
void sieve_kernel_attrs(size_t smem, bool odd, int block, int* per_sm);
// Segments [a, b) of an odd-mode launch that may follow launches covering [0, a):
// the largest b such that the halves of every value of [a, b) lie below segment a.
i64 sieve_odd_range_end(i64 a, i64 nseg, i64 dense_segs, i64 u_dense, i64 u_total, int S);
// Whether odd mode applies: value words aligned at u_dense and enough segments.
bool sieve_odd_ok(i64 u_dense, i64 nseg, i64 first_odd);
// The sieve launches of a table build, in stream order: the first wave of
// first_wave segments in full mode, then odd-mode ranges from sieve_odd_range_end
// (or everything in full mode where odd mode does not apply).
struct SieveLaunch {
    i64 begin, end;
    bool odd;
};
std::vector<SieveLaunch> sieve_launch_plan(i64 u_total, i64 u_dense, int S, i64 first_wave);
std::vector<uint32_t> make_stencil4();
std::vector<uint32_t> make_stencil_odd4();
void sums_kernel_occupancy(int block, int* per_sm);
void launch_debug_udiv(const u64* y, const u64* d, u64* q, i64 n, int rcp, cudaStream_t s);
void launch_debug_piece(const int32_t* piece, const u64* q, i64* out, i64 n, int fast, cudaStream_t s);

}  // namespace drb
