// dr_device.cuh -- device helpers shared by the B200 Deleglise-Rivat kernels.
//
// Exact integer quotients, the mod-6 S2 summands, table lookups (dense int16
// prefix, compressed bit planes, Mobius wheel) and the decoding of one outer
// evaluation into its S1 / S2 index ranges.  Reference lines are cited as
// mertens_dr.hpp:<line> (ecreeth/deleglise-rivat).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace drb {

typedef unsigned long long u64;
typedef long long i64;

// ---------------------------------------------------------------------------
// Exact floor(y / d) without floating point in the result.
//
// The reference divides in IEEE double when y <= 2^53 and in int64 above
// (fast_div, mertens_dr.hpp:80-86).  Here every quotient is integer-exact:
// an FP32 reciprocal *estimate* that never exceeds 1/d proposes a partial
// quotient t <= floor(r/d); the integer remainder r -= t*d is then exact and
// stays non-negative, and the loop repeats on the remainder (about 17 new
// quotient bits per step) until r < d.  Floating point only proposes; the
// integer arithmetic decides.
// ---------------------------------------------------------------------------

#ifdef __CUDACC__
// 1/d rounded down with margin: RU conversion makes fd >= d, rcp.approx is
// within a few ulp of 1/fd, and the (1 - 2^-17) factor absorbs that error.
__device__ __forceinline__ float rcp_floor_estimate(uint32_t d) {
    const float fd = __uint2float_ru(d);
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(fd));
    return r * 0.999992370605468750f;
}

// y < 2^64, 1 <= d < 2^32, inv = rcp_floor_estimate(d).
__device__ __forceinline__ u64 udiv_u64_u32(u64 y, uint32_t d, float inv) {
    u64 q = 0;
    while (y >= d) {
        u64 t = __float2ull_rz(__fmul_rz(__ull2float_rz(y), inv));
        t = t ? t : 1ull;
        q += t;
        y -= t * (u64)d;
    }
    return q;
}

// floor(y / n) from a tabulated double reciprocal r = RN(1/n), for n < 2^32 and
// y / n < 2^50, with yd = RN(y).  p = RN(yd * r) is within (y/n) * 3 * 2^-53 < 3/8
// of y/n, so trunc(p) is floor(y/n) or a neighbour of it; the exact remainder
// y - trunc(p) * n, which lies in [-n, 2n), selects the right one.  trunc(p) is
// the low mantissa of RZ(p + 2^52) (0 <= p < 2^52, where that sum has ulp 1).
__device__ __forceinline__ u64 udiv_rcp(u64 y, double yd, uint32_t n, double r) {
    const double p = __dmul_rn(yd, r);
    const u64 qe = (u64)__double_as_longlong(__dadd_rz(p, 4503599627370496.0)) & 0xFFFFFFFFFFFFFull;
    const u64 prod = (u64)(uint32_t)qe * n + ((u64)((uint32_t)(qe >> 32) * n) << 32);  // qe * n < 2^64
    const i64 rem = (i64)(y - prod);
    return qe + (u64)(i64)((int)(rem >= (i64)n) - (int)(rem < 0));
}

#endif  // __CUDACC__

// 32-bit quotients of the S1 / S2 fast paths (n < 2^31 and floor(y/n) < 2^31).
// qest: ceil(yd*r - 1/2) read from the low mantissa word of RU(yd*r + 2^52 - 1/2)
// (one FMA; for y >= n the sum lies in [2^52, 2^53), where the spacing is 1).  yd*r
// is within (y/n) * 2^-52 < 1/2 of y/n, so the estimate qp is floor(y/n) or
// floor(y/n) + 1.  Callers divide only y >= n (every S1/S2 quotient is >= 1).
// qfix: y - qp*n lies in [-n, n), so its low 32 bits, read as a signed integer,
// say which one (n < 2^31); one IMAD and a sign bit replace the 64-bit remainder.
constexpr double kQBias = 4503599627370495.5;  // 2^52 - 1/2

#ifdef __CUDACC__
__device__ __forceinline__ uint32_t qest(double yd, double r) {
    return (uint32_t)__double2loint(__fma_ru(yd, r, kQBias));
}

__device__ __forceinline__ uint32_t qfix(uint32_t qp, uint32_t ylo, uint32_t n) {
    const uint32_t d = ylo - qp * n;  // y - qp*n mod 2^32
    return qp - (d >> 31);
}

__device__ __forceinline__ u64 udiv(u64 y, u64 d) {
    if (d >> 32) return y / d;  // divisor above 32 bits: rare, exact library path
    if ((y >> 32) == 0) return (uint32_t)y / (uint32_t)d;
    return udiv_u64_u32(y, (uint32_t)d, rcp_floor_estimate((uint32_t)d));
}

#endif  // __CUDACC__

// ---------------------------------------------------------------------------
// S2 summands (mertens_dr.hpp:462-482 tabulates them; here they come from
// their definitions).  For j coprime to 6 and q = floor(y/j), the terms of
// j, 2j, 3j, 6j in S2(L) = sum_{m<=L} mu(m) floor(y/m) give
//   f_L(q) = q - [2j<=L] q/2 - [3j<=L] q/3 + [6j<=L] q/6.
// Combined pieces 1..8 are f_A(q) - f_B(floor(q/2)) (S2(y) - S2(y/2), cut at
// B/6 A/6 B/3 A/3 B/2 A/2 B A); single pieces 9..12 are f_A(q) (cut at A/6
// A/3 A/2 A).  Each is additive over q = 12k + r:
//   piece(q) = piece(12) * k + piece(r),
// so the device evaluates a*k + T[r] with T packed as 5-bit fields (+16);
// T[r] ranges over [-1, 11] (piece(q) = q has T[r] = r).
// ---------------------------------------------------------------------------
__host__ __device__ constexpr i64 piece_formula(int piece, i64 q) {
    const i64 h = q / 2, t = q / 3, f = q / 4, s = q / 6, d = q / 12;
    switch (piece) {
    case 1: return (q - h - t + s) - (h - f - s + d);
    case 2: return (q - h - t + s) - (h - f - s);
    case 3: return (q - h - t) - (h - f - s);
    case 4: return (q - h - t) - (h - f);
    case 5: return (q - h) - (h - f);
    case 6: return (q - h) - h;
    case 7: return q - h;
    case 8: return q;
    case 9: return q - h - t + s;
    case 10: return q - h - t;
    case 11: return q - h;
    case 12: return q;
    default: return 0;
    }
}

struct PieceCoef {
    i64 a;       // piece(12)
    u64 packed;  // bits 5r..5r+4 hold piece(r) + 16, r = 0..11
};

__host__ __device__ constexpr PieceCoef make_piece_coef(int piece) {
    PieceCoef c{piece_formula(piece, 12), 0};
    for (int r = 0; r < 12; ++r) c.packed |= (u64)(piece_formula(piece, r) + 16) << (5 * r);
    return c;
}

#ifdef __CUDACC__
__device__ __forceinline__ i64 piece_eval(const PieceCoef& c, u64 q) {
    u64 k;
    uint32_t r;
    if ((q >> 32) == 0) {  // most S2 quotients: 32-bit division by the constant 12
        const uint32_t q32 = (uint32_t)q, k32 = q32 / 12u;
        k = k32;
        r = q32 - k32 * 12u;
    } else {
        k = q / 12u;
        r = (uint32_t)(q - k * 12u);
    }
    const int t = (int)((c.packed >> (5 * r)) & 31u) - 16;
    return c.a * (i64)k + t;
}

#endif  // __CUDACC__

// ---------------------------------------------------------------------------
// Tables in HBM.
//   dM[i]      = M(i + 1) as int16, 0 <= i < u_dense   (dense prefix)
//   planes[w]  = {nonzero, negative} bits of mu over n = u_dense+1+64w .. +63
//   ckpt[w]    = M(u_dense + 64w)                       (int32 checkpoint)
//   wheel[g]   = mu(j) for j = 6m+1 (x: nonzero, y: negative) and j = 6m+5
//                (z, w) with m = 32g + bit, j <= mu_limit
// The compressed tier is the reference's format (mertens_dr.hpp:662-752:
// two 32-byte planes + four int32 checkpoints per 256 values) with each
// word's two plane words stored side by side, so one lookup reads one 16-byte
// sector of planes plus one checkpoint.
// ---------------------------------------------------------------------------
struct TableView {
    const int16_t* dM;
    const ulonglong2* planes;
    const int32_t* ckpt;
    const uint4* wheel;
    i64 u_dense, u_total, mu_limit;
    i64 cbase;  // compressed-tier word held in planes[0] / ckpt[0]: 0, or a streamed band's first word
};

#ifdef __CUDACC__
__device__ __forceinline__ int32_t table_M(const TableView& t, u64 q) {
    if (q <= (u64)t.u_dense) return q ? (int32_t)__ldg(t.dM + (q - 1)) : 0;
    const u64 off = q - (u64)t.u_dense - 1;
    const u64 w = (off >> 6) - (u64)t.cbase;
    const ulonglong2 p = __ldg(t.planes + w);
    const int32_t c = __ldg(t.ckpt + w);
    const u64 mask = ~0ull >> (63 - (off & 63));
    return c + __popcll(p.x & mask) - 2 * __popcll(p.y & mask);
}

// mu(j) for j coprime to 6, j <= mu_limit
__device__ __forceinline__ int wheel_mu(const uint4* wheel, u64 j) {
    const u64 m = j / 6u;
    const bool five = (j - m * 6u) == 5u;
    const uint4 w = __ldg(wheel + (m >> 5));
    const uint32_t b = (uint32_t)(m & 31u);
    const uint32_t nz = five ? w.z : w.x, ng = five ? w.w : w.y;
    return ((nz >> b) & 1u) ? (((ng >> b) & 1u) ? -1 : 1) : 0;
}

#endif  // __CUDACC__

// ---------------------------------------------------------------------------
// One query of a (possibly batched) launch.
// ---------------------------------------------------------------------------
struct QueryDev {
    u64 X;
    i64 u;          // this query's S1 lower cut: n > y/u (u <= table u_total)
    double cx;      // split parameter
    i64 N;          // X / u
    i64 nc;         // candidates k <= N coprime to 6
    u64 slot_base;  // first global evaluation slot of this query
    u64 win;        // S1 window length W (a power of two; 0: no windowed S1)
    u64 win_max;    // windows w < win_max lie in the dense tier ((w+1)*W <= u_dense < 2^31)
    u64 inv_limit;  // largest tabulated S1 reciprocal 1/n
};

#ifndef DRB_WIN_MIN
#define DRB_WIN_MIN 64  // lookups of a segment in its last window (a power of two)
#endif

#ifdef __CUDACC__
// Windowed S1 (s1win_kernel): the S1 lookups M(q) of an S1 segment with q below a
// cut are summed window by window (q in [w*W, (w+1)*W), the window of the M table in
// shared memory), the ones above it by the sums kernel.  The cut, a multiple of W,
// sits where one window still holds about 64 of the segment's lookups
// (y*W / (stride*Q^2) = 64), capped by the dense tier; it is returned as the
// number of windowed windows.  IEEE operations only, so every kernel computes the
// same cut.
__device__ __forceinline__ u64 s1_win_count(u64 y, int stride, u64 W, u64 win_max) {
    if (W == 0) return 0;
    const double v = __dmul_rn(__ull2double_rn(y), (double)W / ((double)DRB_WIN_MIN * (double)stride));  // exact
    const u64 wc = __double2ull_rz(__dmul_rn(__dsqrt_rn(v), 1.0 / (double)W));
    return wc < win_max ? wc : win_max;
}

// Split point A = floor(cx * sqrt(y)) clamped to [1, y-1] (mertens_dr.hpp:1491-1493,
// 1528-1533).  It is a parameter, not part of any sum: every A in range gives the
// same M(X).  It is computed with the reference's IEEE double operations (correctly
// rounded sqrt and product, truncation) so that intermediate S1/S2 checksums can be
// compared with the reference at identical parameters.
__device__ __forceinline__ i64 split_point(double cx, i64 y) {
    i64 A = __double2ll_rz(__dmul_rn(cx, __dsqrt_rn(__ll2double_rn(y))));
    if (A >= y) A = y - 1;
    if (A < 1) A = 1;
    return A;
}

// Outer candidate c -> k: 1, 5, 7, 11, ... (k coprime to 6).
__device__ __forceinline__ i64 candidate_k(i64 c) { return 3 * c + 1 + (c & 1); }

#endif  // __CUDACC__

enum { EVAL_NONE = 0, EVAL_SINGLE = 1, EVAL_COMB2 = 2 };

// S1 segments: arithmetic progressions n = n0 + stride*i (stride 1, 2 or 6), or,
// with stride code S1_WHEEL, the divisors coprime to 6 n = candidate_k(n0 + i)
// (n0 then indexes the wheel).  Four segments per evaluation (kS1Seg).
constexpr int kS1Seg = 4;
enum { S1_WHEEL = 3 };

#ifdef __CUDACC__
__device__ __forceinline__ u64 s1_n_at(i64 n0, int st, u64 i) {
    return st == S1_WHEEL ? (u64)candidate_k(n0 + (i64)i) : (u64)n0 + (u64)st * i;
}

// smallest wheel index c with candidate_k(c) >= n, largest with candidate_k(c) <= n (n >= 1)
__device__ __forceinline__ i64 wheel_lower(i64 n) {
    const i64 c = (n - 1) / 3;
    return c + (candidate_k(c) < n ? 1 : 0);
}
__device__ __forceinline__ i64 wheel_upper(i64 n) {
    const i64 c = (n - 1) / 3;
    return c - (candidate_k(c) > n ? 1 : 0);
}

#endif  // __CUDACC__

// The S1 lookups one planning pass keeps: those with qlo <= floor(y/n) <= qhi.  A table
// streamed in bands (the compressed tier above u_resident never held whole) is summed
// in passes: the resident pass keeps q <= u_resident with S2 and the constant parts,
// each band pass the q of its band and nothing else (s1_only).  Every lookup falls in
// exactly one pass, so the S1 total is the same sum of the same terms.
struct S1Band {
    u64 qlo, qhi;  // whole table: 0, ~0
    int s1_only;
};

// Index ranges of one evaluation in op order: S1 segments first, then S2 pieces.
struct EvalDesc {
    u64 y;
    i64 coef;       // mu(k) * (+1 first eval / -1 second eval)
    int kind;
    int npieces;    // 4 (single) or 8 (comb2)
    int piece0;     // 9 (single) or 1 (comb2)
    int nseg;       // 2 + npieces
    i64 A, B, ky, ky2;
    i64 s1_n0[kS1Seg];
    i64 s1_cnt[kS1Seg];   // lookups of each S1 segment left to the sums kernel
    i64 s1_full[kS1Seg];  // all lookups of each S1 segment
    u64 s1_wc[kS1Seg];    // windows of each S1 segment summed by s1win_kernel
    int s1_stride[kS1Seg];
    int s1_sign[kS1Seg];
    i64 jlo[8], jhi[8];
    i64 mcnt[8];
    u64 total;
};

// One evaluation slot as the planner leaves it for the sums kernel (96 bytes): y, the
// split points, the S1 segments and, in `bits`, the kind (bits 0-1), the sign of the
// coefficient (bit 2), per S1 segment g a stride code and sign (bits 3+3g ..) and
// kSlotS1Only (a band pass of a streamed table: S1 lookups only, no S2 pieces).
struct __align__(16) SlotDesc {
    u64 y;
    i64 A, B;
    i64 n0[kS1Seg];
    i64 cnt[kS1Seg];
    u64 bits;
};
static_assert(sizeof(SlotDesc) == 96, "SlotDesc is six 16-byte words");
constexpr u64 kSlotS1Only = 1ull << 15;

#ifdef __CUDACC__
__device__ __forceinline__ i64 piece_mcount(i64 lo, i64 hi) {
    return lo > hi ? 0 : hi / 6 - lo / 6 + 1;
}

// The main S1 range of F(Y) (single) or of the odd-n sum of F(Y) - F(Y/2) (comb2):
// n in [s, kap], s = floor(Y/u) + 1 (rounded up to odd for comb2), kap = kappa_Y.
__device__ __forceinline__ void s1_main(const QueryDev& Q, u64 Y, bool comb2, i64* s, i64* kap) {
    const i64 A = split_point(Q.cx, (i64)Y);
    *kap = (i64)udiv(Y, (u64)(A + 1));
    i64 st = (i64)udiv(Y, (u64)Q.u) + 1;
    if (comb2 && (st & 1) == 0) ++st;
    *s = st;
}

__device__ __forceinline__ void s1_set(EvalDesc& d, int g, i64 n0, int stride, i64 last, int sign) {
    d.s1_n0[g] = n0;
    d.s1_stride[g] = stride;
    d.s1_sign[g] = sign;
    if (stride == S1_WHEEL) d.s1_cnt[g] = last >= 0 && last >= n0 ? last - n0 + 1 : 0;  // n0, last: wheel indices
    else d.s1_cnt[g] = last >= n0 ? (last - n0) / stride + 1 : 0;
}

// The S2 pieces of an evaluation from its kind and split points (A; B = the split
// point of y/2 for comb2): single pieces 9..12 over j in [1, A/6], (A/6, A/3],
// (A/3, A/2], (A/2, A]; combined pieces 1..8 cut at B/6 A/6 B/3 A/3 B/2 A/2 B A
// (eval_s2_single / eval_s2_combined, mertens_dr.hpp:622-660).
__device__ __forceinline__ void eval_pieces(EvalDesc& d) {
    const i64 A = d.A, B = d.B;
    if (d.kind == EVAL_SINGLE) {
        d.npieces = 4; d.piece0 = 9;
        const i64 a6 = A / 6, a3 = A / 3, a2 = A / 2;
        d.jlo[0] = 1;      d.jhi[0] = a6;
        d.jlo[1] = a6 + 1; d.jhi[1] = a3;
        d.jlo[2] = a3 + 1; d.jhi[2] = a2;
        d.jlo[3] = a2 + 1; d.jhi[3] = A;
    } else {
        d.npieces = 8; d.piece0 = 1;
        const i64 b6 = B / 6, a6 = A / 6, b3 = B / 3, a3 = A / 3, b2 = B / 2, a2 = A / 2;
        d.jlo[0] = 1;      d.jhi[0] = b6;
        d.jlo[1] = b6 + 1; d.jhi[1] = a6;
        d.jlo[2] = a6 + 1; d.jhi[2] = b3;
        d.jlo[3] = b3 + 1; d.jhi[3] = a3;
        d.jlo[4] = a3 + 1; d.jhi[4] = b2;
        d.jlo[5] = b2 + 1; d.jhi[5] = a2;
        d.jlo[6] = a2 + 1; d.jhi[6] = B;
        d.jlo[7] = B + 1;  d.jhi[7] = A;
    }
    d.nseg = kS1Seg + d.npieces;
}

// Wheel positions of every piece and the evaluation's op count (S1 lookups left to
// the sums kernel + S2 wheel positions).
__device__ __forceinline__ void eval_total(EvalDesc& d) {
    u64 tot = 0;
    for (int g = 0; g < kS1Seg; ++g) tot += (u64)d.s1_cnt[g];
    for (int p = 0; p < d.npieces; ++p) {
        d.mcnt[p] = piece_mcount(d.jlo[p], d.jhi[p]);
        tot += (u64)d.mcnt[p];
    }
    d.total = tot;
}

// Decode evaluation e (0/1) of candidate c of query Q.  Follows the outer
// reduction of mertens_dr.hpp:1470-1485, 1616-1632 and the ranges of
// eval_single_S (:1490-1525) and eval_comb2 (:1527-1614).
//
// S1 terms that cancel between the two evaluations of a candidate are left out:
// for k <= N/3 the second evaluation works on y/3 with the opposite sign, and its
// term M(floor(floor(y/3)/n')) = M(floor(y/(3n'))) at odd n' equals the first
// evaluation's term at n = 3n'.  Wherever both exist -- odd n' in [clo, chi] with
// 3*clo >= s0, 3*chi <= kappa_y -- both are dropped: the first evaluation keeps its
// odd n coprime to 3 (the wheel) and the multiples of 3 outside [3clo, 3chi], the
// second its divisors outside [clo, chi].  The S1 total is unchanged term for term.
__device__ __forceinline__ void s1_band_cut(EvalDesc& d, const S1Band& band) {
    const u64 y = d.y;
    // n >= nlo <=> q <= qhi;  n <= nhi <=> q >= qlo (and n <= y: q >= 1)
    const i64 nlo = band.qhi >= y ? 1 : (i64)udiv(y, band.qhi + 1) + 1;
    const i64 nhi = band.qlo <= 1 ? (i64)y : (i64)udiv(y, band.qlo);
    for (int g = 0; g < kS1Seg; ++g) {
        const i64 cnt = d.s1_cnt[g], n0 = d.s1_n0[g];
        if (cnt <= 0) continue;
        const int st = d.s1_stride[g];
        if (st == S1_WHEEL) {  // n0: wheel index
            const i64 first = max(n0, wheel_lower(nlo));
            const i64 last = min(n0 + cnt - 1, wheel_upper(nhi));
            d.s1_n0[g] = first;
            d.s1_cnt[g] = last >= first ? last - first + 1 : 0;
        } else {
            const i64 ia = nlo > n0 ? (nlo - n0 + st - 1) / st : 0;
            const i64 ib = nhi >= n0 ? min(cnt - 1, (nhi - n0) / st) : -1;
            d.s1_n0[g] = n0 + st * ia;
            d.s1_cnt[g] = ib >= ia ? ib - ia + 1 : 0;
        }
    }
    if (band.s1_only) {
        d.npieces = 0;
        d.nseg = kS1Seg;
    }
}

__device__ inline void decode_eval(const QueryDev& Q, const TableView& T, i64 c, int e, EvalDesc& d,
                                   const S1Band band = S1Band{0, ~0ull, 0}) {
    d.kind = EVAL_NONE;
    d.total = 0;
    d.nseg = 0;
    const i64 k = candidate_k(c);
    if (k > Q.N) return;
    const int muk = wheel_mu(T.wheel, (u64)k);
    if (muk == 0) return;
    const i64 N = Q.N;
    int range;
    if (k <= N / 6) range = 1;
    else if (k <= N / 3) range = 2;
    else if (k <= N / 2) range = 3;
    else range = 4;
    const u64 yk = udiv(Q.X, (u64)k);
    u64 y, y2 = 0;
    if (e == 0) {
        d.coef = muk;
        if (range <= 3) { d.kind = EVAL_COMB2; y = yk; y2 = yk / 2; }
        else { d.kind = EVAL_SINGLE; y = yk; }
    } else {
        d.coef = -muk;
        if (range == 1) { d.kind = EVAL_COMB2; y = yk / 3; y2 = yk / 6; }
        else if (range == 2) { d.kind = EVAL_SINGLE; y = yk / 3; }
        else return;
    }
    d.y = y;
    for (int g = 0; g < kS1Seg; ++g) s1_set(d, g, 0, 2, -1, 1);
    // cancelled odd n' in [clo, chi] of y/3 (ranges 1, 2)
    i64 s0 = 0, kap0 = 0, s1 = 0, kap1 = 0, clo = 1, chi = -1;
    if (range <= 2) {
        s1_main(Q, yk, true, &s0, &kap0);
        s1_main(Q, yk / 3, range == 1, &s1, &kap1);
        i64 lo = max(s1, (s0 + 2) / 3);
        if ((lo & 1) == 0) ++lo;
        i64 hi = min(kap1, kap0 / 3);
        if ((hi & 1) == 0) --hi;
        clo = lo;
        chi = hi;
    }
    const bool cancel = clo <= chi;
    if (d.kind == EVAL_SINGLE) {
        const i64 A = split_point(Q.cx, (i64)y);
        const i64 ky = (i64)udiv(y, (u64)(A + 1));
        const i64 start = (i64)udiv(y, (u64)Q.u) + 1;
        d.A = A; d.B = 0; d.ky = ky; d.ky2 = 0;
        if (e == 1 && cancel) {  // range 2: all n' of [start, ky] but the odd ones in [clo, chi]
            const i64 so = start | 1;
            s1_set(d, 0, so, 2, clo - 2, 1);
            s1_set(d, 1, chi + 2, 2, ky, 1);
            s1_set(d, 2, (start + 1) & ~1ll, 2, ky, 1);
        } else {
            s1_set(d, 0, start, 1, ky, 1);
        }
        eval_pieces(d);
    } else {
        const i64 A = split_point(Q.cx, (i64)y);
        const i64 B = split_point(Q.cx, (i64)y2);
        const i64 ky = (i64)udiv(y, (u64)(A + 1));
        const i64 ky2 = (i64)udiv(y2, (u64)(B + 1));
        const i64 two = 2 * ky2;
        i64 start = (i64)udiv(y, (u64)Q.u) + 1;
        if ((start & 1) == 0) ++start;
        d.A = A; d.B = B; d.ky = ky; d.ky2 = ky2;
        if (e == 0 && cancel) {  // odd n of [start, ky]: the wheel + multiples of 3 outside [3clo, 3chi]
            s1_set(d, 0, wheel_lower(start), S1_WHEEL, wheel_upper(ky), 1);
            i64 m3 = start;  // first odd multiple of 3 >= start
            while (m3 % 3) m3 += 2;
            s1_set(d, 1, m3, 6, 3 * clo - 6, 1);
            s1_set(d, 2, 3 * chi + 6, 6, ky, 1);
        } else if (e == 1 && cancel) {  // range 1: odd n' of [start, ky] outside [clo, chi]
            s1_set(d, 0, start, 2, clo - 2, 1);
            s1_set(d, 1, chi + 2, 2, ky, 1);
        } else {
            s1_set(d, 0, start, 2, ky, 1);
        }
        // even-n correction between kappa_y and 2*kappa_{y/2} (:1568-1610)
        i64 e0 = 0, last = -1;
        int sg = 1;
        if (two > ky) { e0 = ky + 1; last = two; sg = -1; }
        else if (two < ky) { e0 = two + 1; last = ky; sg = 1; }
        if (e0 & 1) ++e0;
        s1_set(d, 3, e0, 2, last, sg);
        eval_pieces(d);
    }
    if (band.qlo > 1 || band.qhi < (u64)Q.u || band.s1_only) s1_band_cut(d, band);
    // windowed S1: the lookups with q < wc*W, i.e. n > y/(wc*W), go to s1win_kernel
    for (int g = 0; g < kS1Seg; ++g) {
        d.s1_full[g] = d.s1_cnt[g];
        d.s1_wc[g] = 0;
        const i64 cnt = d.s1_cnt[g];
        if (cnt <= 0 || Q.win == 0) continue;
        const int st = d.s1_stride[g];
        const i64 nlast = (i64)s1_n_at(d.s1_n0[g], st, (u64)(cnt - 1));
        // the windowed kernel divides on the 32-bit route with tabulated reciprocals
        if (nlast >= (1ll << 31) || (u64)nlast > Q.inv_limit) continue;
        const u64 wc = s1_win_count(y, st, Q.win, Q.win_max);  // the wheel's density is that of stride 3
        if (wc == 0) continue;
        const i64 ncut = (i64)udiv(y, wc * Q.win) + 1;  // n >= ncut <=> q < wc*W
        d.s1_wc[g] = wc;
        if (st == S1_WHEEL) d.s1_cnt[g] = min(cnt, max(0ll, wheel_upper(ncut - 1) - d.s1_n0[g] + 1));
        else d.s1_cnt[g] = ncut <= d.s1_n0[g] ? 0 : min(cnt, (ncut - 1 - d.s1_n0[g]) / st + 1);
    }
    eval_total(d);
}

// Stride codes of SlotDesc: 1, 2, 6 and the wheel (S1_WHEEL) in two bits.
__device__ __forceinline__ u64 stride_code(int st) { return st == 1 ? 0u : st == 2 ? 1u : st == 6 ? 2u : 3u; }
__device__ __forceinline__ int stride_of_code(u64 c) { return c == 0 ? 1 : c == 1 ? 2 : c == 2 ? 6 : S1_WHEEL; }

// An evaluation as the sums kernel needs it, written once by the planner.
__device__ __forceinline__ void pack_slot(const EvalDesc& d, SlotDesc* out) {
    SlotDesc s;
    if (d.kind == EVAL_NONE) {  // no terms: the sums kernel never reads it
        s.y = 0;
        s.A = s.B = 0;
        for (int g = 0; g < kS1Seg; ++g) s.n0[g] = s.cnt[g] = 0;
        s.bits = 0;
        *out = s;
        return;
    }
    s.y = d.y;
    s.A = d.A;
    s.B = d.kind == EVAL_COMB2 ? d.B : 0;
    u64 bits = (u64)d.kind | (d.coef < 0 ? 4ull : 0ull) | (d.npieces == 0 ? kSlotS1Only : 0ull);
    for (int g = 0; g < kS1Seg; ++g) {
        s.n0[g] = d.s1_n0[g];
        s.cnt[g] = d.s1_cnt[g];
        bits |= (stride_code(d.s1_stride[g]) | (d.s1_sign[g] < 0 ? 4ull : 0ull)) << (3 + 3 * g);
    }
    s.bits = bits;
    *out = s;
}

// The planner's evaluation back from its SlotDesc: S1 segments as stored, S2
// pieces and op count recomputed from the split points.
__device__ __forceinline__ void unpack_slot(const SlotDesc& s, EvalDesc& d) {
    d.y = s.y;
    d.kind = (int)(s.bits & 3u);
    d.coef = (s.bits & 4u) ? -1 : 1;
    d.A = s.A;
    d.B = s.B;
    for (int g = 0; g < kS1Seg; ++g) {
        const u64 c = s.bits >> (3 + 3 * g);
        d.s1_n0[g] = s.n0[g];
        d.s1_cnt[g] = s.cnt[g];
        d.s1_stride[g] = stride_of_code(c & 3u);
        d.s1_sign[g] = (c & 4u) ? -1 : 1;
    }
    if (d.kind == EVAL_NONE) {
        d.nseg = 0;
        d.total = 0;
        return;
    }
    eval_pieces(d);
    if (s.bits & kSlotS1Only) {
        d.npieces = 0;
        d.nseg = kS1Seg;
    }
    eval_total(d);
}

// Constant part of an evaluation: 1 + kappa*M(A) (single) or
// kappa_y*M(A) - kappa_y2*M(B) (comb2), mertens_dr.hpp:1524, 1613.
__device__ __forceinline__ i64 eval_constant(const EvalDesc& d, const TableView& T) {
    if (d.kind == EVAL_SINGLE) return 1 + d.ky * (i64)table_M(T, (u64)d.A);
    if (d.kind == EVAL_COMB2)
        return d.ky * (i64)table_M(T, (u64)d.A) - d.ky2 * (i64)table_M(T, (u64)d.B);
    return 0;
}

__device__ __forceinline__ u64 warp_sum_u64(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

#endif  // __CUDACC__

}  // namespace drb
