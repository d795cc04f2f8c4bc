// dr_kernels.cu -- sm_100a kernels of the Deleglise-Rivat Mertens engine.
//
//  sieve_kernel      segmented byte-log Mobius sieve in shared memory and the
//                    three table outputs of each segment: dense int16 prefix,
//                    compressed bit planes + checkpoints, Mobius wheel bits
//                    (mertens_dr.hpp:755-883 for the streamed builder,
//                    :180-296 / :300-368 for the dense one); full mode sieves
//                    every value, odd mode the odd values only and derives the
//                    even ones from the planes of their halves
//  sq_bucket_*       per-segment hit lists of the squares p^2 > S
//  seg_scan_kernel   exclusive scan of per-segment Mobius sums
//  fixup_kernel      global offsets into the dense prefix and checkpoints
//                    (mertens_dr.hpp:884-900)
//  plan_kernel       one thread per outer evaluation slot: op counts and the
//                    constant part kappa*M(A) ... (mertens_dr.hpp:1470-1485)
//  scan_u64 kernels  op-count prefix (the flattened work space)
//  sums_kernel       persistent warps pull fixed-size chunks of the flattened
//                    S1/S2 index space from a device work queue
//                    (mertens_dr.hpp:1490-1632)
#include "dr_kernels.cuh"

#include <algorithm>

namespace drb {

__constant__ PieceCoef c_piece[13];

void init_piece_constants() {
    PieceCoef h[13];
    for (int p = 0; p < 13; ++p) h[p] = make_piece_coef(p);
    cudaMemcpyToSymbol(c_piece, h, sizeof(h));
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t umod_u64_u32(u64 y, uint32_t d) {
    if ((y >> 32) == 0) return (uint32_t)y % d;
    const u64 q = udiv_u64_u32(y, d, rcp_floor_estimate(d));
    return (uint32_t)(y - q * d);
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive scan of a[0..n) in shared memory; returns the total.  wtot holds
// 33 ints of scratch.  Every thread of the block must call it.
__device__ int block_excl_scan(int32_t* a, int n, int32_t* wtot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int ntiles = (n + 31) >> 5;
    const int tpw = (ntiles + nwarps - 1) / nwarps;
    const int t0 = warp * tpw, t1 = min(ntiles, t0 + tpw);
    int carry = 0;
    for (int t = t0; t < t1; ++t) {
        const int idx = (t << 5) + lane;
        const int v = idx < n ? a[idx] : 0;
        const int x = warp_incl_scan(v, lane);
        if (idx < n) a[idx] = carry + x - v;
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) wtot[warp] = carry;
    __syncthreads();
    if (warp == 0) {
        const int v = lane < nwarps ? wtot[lane] : 0;
        const int x = warp_incl_scan(v, lane);
        wtot[lane] = x - v;
        if (lane == 31) wtot[32] = x;
    }
    __syncthreads();
    const int off = wtot[warp];
    for (int t = t0; t < t1; ++t) {
        const int idx = (t << 5) + lane;
        if (idx < n) a[idx] += off;
    }
    const int total = wtot[32];
    __syncthreads();
    return total;
}

// y mod d from a tabulated reciprocal inv = floor((2^64-1)/d): umulhi(y, inv)
// undershoots floor(y/d) by at most one, so one subtraction corrects the remainder
__device__ __forceinline__ u64 umod_inv(u64 y, u64 d, u64 inv) {
    const u64 r = y - __umul64hi(y, inv) * d;
    return r >= d ? r - d : r;
}

// Byte-log rule (mertens_dr.hpp:145-171) for value n with accumulator acc.
__device__ __forceinline__ uint32_t finalize_byte(uint32_t acc, u64 n) {
    if (n <= 2) return n == 1 ? 1u : (n == 2 ? 0xFFu : 0u);  // explicit 1 and 2 (:838-839)
    if (acc & 0x80u) return 0u;
    const uint32_t bits = 64u - __clzll(n);
    const bool sieved_all = acc > bits - 1;
    const bool odd = acc & 1u;
    // sign = (-1)^acc when every factor was sieved, else the opposite sign
    return (odd == sieved_all) ? 0xFFu : 1u;
}

// Shared memory of a sieve CTA.  Full mode: a pass of min(S, 2^17) bytes and its
// 16-value group sums.  Odd mode: S/2 bytes (the odd values), 64-value word sums and
// plane words.
size_t sieve_smem_bytes(int S, bool odd) {
    const int B = odd ? S : std::min(S, kSieveFullPass);
    return odd ? (size_t)B / 2 + (size_t)(B / 64) * 4 + (size_t)(B / 64) * 16 + 64
               : (size_t)B + (size_t)(B / 16) * 4 + 64;
}

// {nonzero, negative} plane words of 64 consecutive mu bytes src[16w .. 16w+16)
// (words at or past nw16 read as 0), one 64-value word per thread.  A mu byte is 0,
// 1 or 0xFF, so bit 0 is its nonzero bit and bit 7 its negative bit; per shared word
// both are moved to bits 0 and 4 of each byte and gathered into two nibbles (bits
// 24..27: nonzero, 28..31: negative) by one multiply, whose partial products land on
// distinct bits.  Lane l reads its 16 words starting at word l/2, which puts the 32
// lanes of a warp on 32 distinct banks; the planes are rotated back by 4*(l/2) bits.
__device__ __forceinline__ void planes_of_bytes(const uint32_t* buf32, int w, int nw16, int lane, u64* nz,
                                                u64* neg) {
    const uint32_t rot = (uint32_t)(lane >> 1);
    const uint32_t* src = buf32 + 16 * w;
    const bool full = 16 * w + 16 <= nw16;
    uint32_t zl = 0, zh = 0, gl = 0, gh = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const uint32_t kk = ((uint32_t)k + rot) & 15u;
        const uint32_t v = (full || 16 * w + (int)kk < nw16) ? src[kk] : 0u;
        const uint32_t x = (v & 0x01010101u) | ((v >> 3) & 0x10101010u);
        const uint32_t pr = x * 0x01020408u;
        const uint32_t z = (pr >> 24) & 0xFu, g = pr >> 28;
        if (k < 8) {
            zl |= z << (4 * k);
            gl |= g << (4 * k);
        } else {
            zh |= z << (4 * (k - 8));
            gh |= g << (4 * (k - 8));
        }
    }
    if (rot >= 8u) {
        uint32_t t = zl;
        zl = zh;
        zh = t;
        t = gl;
        gl = gh;
        gh = t;
    }
    const uint32_t sh = (4u * rot) & 31u;
    *nz = ((u64)__funnelshift_l(zl, zh, sh) << 32) | __funnelshift_l(zh, zl, sh);
    *neg = ((u64)__funnelshift_l(gl, gh, sh) << 32) | __funnelshift_l(gh, gl, sh);
}

// bit k of x -> bit 2k of the result (k < 32)
__device__ __forceinline__ uint32_t spread16(uint32_t x) {
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    return (x | (x << 1)) & 0x55555555u;
}
__device__ __forceinline__ u64 spread32(uint32_t x) {
    return ((u64)spread16(x >> 16) << 32) | spread16(x & 0xFFFFu);
}

// Plane words of 64-value word w of an odd-mode segment (values base+1+64w+b, b <
// 64).  Odd values (even b) from the mu bytes buf8[32w + b/2], i.e. the 8 shared
// words 8w.., lane l starting at word (l/4) & 7 (conflict-free for a warp of
// consecutive w): per word the nonzero and negative bits of its 4 bytes land on bits
// 0, 2, 4, 6 of a byte by one multiply each (partial products on distinct bits).
// Even values 2m (odd b = 2k+1, m = base/2 + 32w + k + 1) from the plane bits of m:
// mu(2m) = -mu(m) for odd m (k even), 0 for even m; the 32 values m are one aligned
// half of a plane word (base/2 + 32w is a multiple of 32).
//
// Fused finalisation (fz.on): the shared words still hold the sieve's accumulator
// bytes, and the byte-log rule of step 4 is applied here, word by word, instead of in
// a pass of its own: a byte is nonzero iff its square flag (bit 7) is clear, negative
// iff also bit 7 of a + k (k below or above the power-of-two edge) equals its parity
// bit.  Word fz.skip (the one straddling the edge, if any) was finalised by step 4;
// bytes at or past nb read as 0.
struct FusedFinal {
    bool on;
    int skip;            // word index already finalised, or -1
    int nb;              // sieved bytes
    i64 edge;            // first byte whose value reaches the next power of two
    uint32_t kbelow, kabove;
};

__device__ __forceinline__ void planes_odd_mode(const SieveArgs& a, const uint32_t* buf32, int w, int nw16,
                                                int lane, i64 base, const FusedFinal& fz, u64* nz, u64* neg) {
    const uint32_t rot = (uint32_t)(lane >> 2) & 7u;
    const uint32_t* src = buf32 + 8 * w;
    const bool full = 8 * w + 8 <= nw16;
    // nearly every word: all 32 bytes sieved, none at or across the power-of-two edge,
    // so one constant k serves the whole word and no byte needs a mask
    const i64 b0 = 32 * (i64)w;
    const bool simple = fz.on && full && b0 + 32 <= fz.nb && (b0 + 32 <= fz.edge || b0 >= fz.edge);
    const uint32_t kw = b0 + 32 <= fz.edge ? fz.kbelow : fz.kabove;
    uint32_t zl = 0, zh = 0, gl = 0, gh = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const uint32_t tt = ((uint32_t)t + rot) & 7u;
        const int idx = 8 * w + (int)tt;
        const uint32_t v = (full || idx < nw16) ? src[tt] : 0u;
        uint32_t nzb, ngb;
        if (simple) {
            const uint32_t x = ((((v & 0x7F7F7F7Fu) + kw) >> 7) ^ v) & 0x01010101u;
            nzb = ~(v >> 7) & 0x01010101u;
            ngb = nzb & ~x;
        } else if (fz.on && idx != fz.skip) {
            const i64 j0 = 4 * (i64)idx;
            const uint32_t s = (v & 0x7F7F7F7Fu) + (j0 < fz.edge ? fz.kbelow : fz.kabove);
            const uint32_t x = ((s >> 7) ^ v) & 0x01010101u;  // 1: mu = +1 (if not flagged)
            nzb = ~(v >> 7) & 0x01010101u;
            ngb = nzb & ~x;
            const int rem = fz.nb - 4 * idx;
            if (rem < 4) {
                const uint32_t m = rem <= 0 ? 0u : (0x01010101u & ((1u << (8 * rem)) - 1u));
                nzb &= m;
                ngb &= m;
            }
        } else {
            nzb = v & 0x01010101u;
            ngb = (v >> 7) & 0x01010101u;
        }
        const uint32_t z = (nzb * 0x01041040u) >> 24;  // bits 0, 2, 4, 6
        const uint32_t g = (ngb * 0x01041040u) >> 24;
        if (t < 4) {
            zl |= z << (8 * t);
            gl |= g << (8 * t);
        } else {
            zh |= z << (8 * (t - 4));
            gh |= g << (8 * (t - 4));
        }
    }
    if (rot >= 4u) {
        uint32_t t = zl;
        zl = zh;
        zh = t;
        t = gl;
        gl = gh;
        gh = t;
    }
    const uint32_t sh = (8u * rot) & 31u;
    u64 z = ((u64)__funnelshift_l(zl, zh, sh) << 32) | __funnelshift_l(zh, zl, sh);
    u64 g = ((u64)__funnelshift_l(gl, gh, sh) << 32) | __funnelshift_l(gh, gl, sh);
    const i64 q0 = (base >> 1) + 32 * (i64)w;  // 0-based bit index of m = q0 + 1
    const i64 G = q0 >> 6;
    const ulonglong2 P = G < (a.u_dense >> 6) ? __ldg(a.dplanes + G) : __ldg(a.hplanes + (G - (a.u_dense >> 6)));
    const uint32_t hz = (uint32_t)(((q0 >> 5) & 1) ? P.x >> 32 : P.x);
    const uint32_t hg = (uint32_t)(((q0 >> 5) & 1) ? P.y >> 32 : P.y);
    z |= spread32(hz & 0x55555555u) << 1;
    g |= spread32(hz & ~hg & 0x55555555u) << 1;
    *nz = z;
    *neg = g;
}

// Marks of one warp item I from its first hit at byte j0 (lane l takes j0 + l*m, then
// every 32nd multiple, up to the item's kItemHits hits or the end of the sieved bytes).
// A lane's strides are 32*m bytes, a multiple of 4: its byte position within the
// 32-bit word, and so the shifted mark, stays the same, and the word advances by 8*m.
__device__ __forceinline__ void mark_item_from(uint32_t* buf32, const uint4 I, uint32_t j0, int nb, int lane) {
    const uint32_t m = I.x;
    const uint32_t j = j0 + (uint32_t)lane * m;
    const uint32_t jend = min((uint32_t)nb, I.y + (uint32_t)kItemHits * m);
    const uint32_t ph = j & 3u;
    // byte 4*(p - buf32) + ph < jend  <=>  p - buf32 < (jend - ph + 3) / 4
    const uint32_t wend = jend + 3u >= ph ? (jend + 3u - ph) >> 2 : 0u;
    uint32_t* p = buf32 + (j >> 2);
    uint32_t* const pend = buf32 + wend;
    if (I.w >> 31) {
        const uint32_t v = 0x80u << (8u * ph);
        for (; p < pend; p += 8u * m) atomicOr(p, v);
    } else {
        const uint32_t v = I.z << (8u * ph);
        for (; p < pend; p += 8u * m) atomicAdd(p, v);
    }
}


// Weight w at bytes j, j + p, j + 2p, ... below nb (one thread, p odd).  Four
// consecutive hits span 4p bytes = p words, so their byte positions within the word
// repeat every four hits: the four shifted weights and word offsets are set up once
// and each group of four hits is four atomics and one pointer step.
__device__ __forceinline__ void mark_prime(uint32_t* buf32, uint32_t j, uint32_t p, uint32_t w, uint32_t nb) {
    if (j + 4u * p <= nb) {  // at least four hits: the unrolled loop
        const uint32_t j1 = j + p, j2 = j1 + p, j3 = j2 + p;
        const uint32_t v0 = w << ((j & 3u) * 8u), v1 = w << ((j1 & 3u) * 8u);
        const uint32_t v2 = w << ((j2 & 3u) * 8u), v3 = w << ((j3 & 3u) * 8u);
        const uint32_t o1 = (j1 >> 2) - (j >> 2), o2 = (j2 >> 2) - (j >> 2), o3 = (j3 >> 2) - (j >> 2);
        uint32_t* q = buf32 + (j >> 2);
        for (; j + 3u * p < nb; j += 4u * p, q += p) {
            atomicAdd(q, v0);
            atomicAdd(q + o1, v1);
            atomicAdd(q + o2, v2);
            atomicAdd(q + o3, v3);
        }
    }
    for (; j < nb; j += p) atomicAdd(&buf32[j >> 2], w << ((j & 3) * 8));
}

// Marks of one warp item I = {modulus m, first byte, weight or 0x80, prime index |
// square bit 31}: lanes stride the multiples of m at or after byte I.y (ODD: the odd
// multiples, m bytes apart), kItemHits/32 strides each, with the 64-bit reciprocal inv of m.
template <bool ODD>
__device__ __forceinline__ void mark_item(uint32_t* buf32, const uint4 I, const u64 inv, i64 low, int nb,
                                          int lane) {
    const uint32_t m = I.x;
    const u64 v0 = (u64)low + (ODD ? 2ull * I.y : (u64)I.y);  // value of byte I.y
    const uint32_t r = (uint32_t)umod_inv(v0, m, inv);
    uint32_t d = r ? m - r : 0u;  // first multiple: v0 + d
    if (ODD && (d & 1u)) d += m;  // v0 is odd: the first odd multiple
    mark_item_from(buf32, I, I.y + (ODD ? d >> 1 : d), nb, lane);
}

// ---------------------------------------------------------------------------
// Segmented byte-log Mobius sieve + table outputs (ODD: odd values only).
// ---------------------------------------------------------------------------
template <bool ODD>
__global__ void __launch_bounds__(1024) sieve_kernel(const SieveArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint8_t* buf = smem;
    uint32_t* buf32 = reinterpret_cast<uint32_t*>(smem);
    int32_t* gs = reinterpret_cast<int32_t*>(smem + (ODD ? a.S / 2 : a.S_sub));
    ulonglong2* wpl = reinterpret_cast<ulonglong2*>(smem + a.S / 2 + (a.S / 64) * 4);  // ODD only
    __shared__ int32_t wtot[33];

    const int T = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = T >> 5;

    // Each warp keeps its marking items -- items warp + nwarps*k, k < 32, one per lane,
    // with the modulus reciprocal -- in registers for every segment and reads them by
    // shuffles, instead of two dependent loads per item and segment (more items: the
    // loop from memory below).
    //
    // Odd mode carries each item's first hit from one segment of the CTA to its next
    // one instead of recomputing it: consecutive segments of a CTA in the same tier lie
    // D = gridDim.x * S values apart, the odd multiples of m are m bytes apart, so the
    // first hit at or after byte I.y moves from b to (b - D/2) mod m.  myC holds
    // (D/2) mod m; the first segment of the CTA and the first one after the dense /
    // compressed boundary (where the bases stop being D apart) compute b afresh.
    uint4 myI = make_uint4(0u, 0xFFFFFFFFu, 0u, 0u);
    u64 myInv = 0;
    uint32_t myB = 0, myC = 0;
    const bool ireg = a.n_items <= 32 * nwarps;
    // lane k of warp w holds item nwarps*k + w (k even) or nwarps*k + nwarps-1-w (k odd):
    // items are sorted by modulus, so the heavy ones of each round of nwarps items
    // alternate between the first and the last warps
    const int my_it = nwarps * lane + ((lane & 1) ? nwarps - 1 - warp : warp);
    const bool my_valid = ireg && my_it < a.n_items;
    if (my_valid) {
        myI = __ldg(a.items + my_it);
        if (ODD) {
            myC = (uint32_t)(((u64)gridDim.x * (u64)(a.S / 2)) % (u64)myI.x);
        } else {
            const uint32_t pidx = myI.w & 0x7fffffffu;
            myInv = (myI.w >> 31) ? __ldg(a.sqinv + pidx) : __ldg(a.pinv + pidx);
        }
    }
    const int my_cnt = __popc(__ballot_sync(0xffffffffu, my_valid));  // valid items are a prefix of the lanes
    i64 prev_seg = -1;
    for (i64 seg = a.seg_begin + blockIdx.x; seg < a.seg_end; seg += gridDim.x) {
        const bool dense = seg < a.dense_segs;
        const i64 seg_base = dense ? seg * (i64)a.S : a.u_dense + (seg - a.dense_segs) * (i64)a.S;
        if (ODD && my_valid) {
            const uint32_t m = myI.x;
            if (prev_seg >= 0 && (prev_seg < a.dense_segs) == dense) {
                myB = myB >= myC ? myB - myC : myB + m - myC;
            } else {
                const uint32_t pidx = myI.w & 0x7fffffffu;
                const u64 inv = (myI.w >> 31) ? __ldg(a.sqinv + pidx) : __ldg(a.pinv + pidx);
                const u64 v0 = (u64)seg_base + 1 + 2ull * myI.y;  // the odd value of byte I.y
                const uint32_t r = (uint32_t)umod_inv(v0, m, inv);
                uint32_t d = r ? m - r : 0u;
                if (d & 1u) d += m;
                myB = d >> 1;
            }
        }
        prev_seg = seg;
        const i64 seg_end = min(seg_base + (i64)a.S, dense ? a.u_dense : a.u_total);
        // Full mode sieves a segment in passes of S_sub values (the shared buffer holds
        // S_sub bytes), carrying the Mobius sum of the earlier passes into the outputs.
        const i64 pass_len = ODD ? (i64)a.S : (i64)a.S_sub;
        int carry = 0;
      for (i64 base = seg_base; base < seg_end; base += pass_len) {
        const i64 end = min(base + pass_len, seg_end);
        const int len = (int)(end - base);
        const i64 low = base + 1;
        // sieved bytes: value low + j (full) or the odd value low + 2j (ODD; low is odd)
        const int nb = ODD ? (len + 1) >> 1 : len;
        const int ng = (nb + 15) >> 4;  // 16-byte groups
        const int nw16 = ng * 4;        // words covering the groups

        // 1. periodic stencil: weights of 2,3,5,7,11 and flags of 4, 9 (:818-823);
        //    ODD: weights of 3,5,7,11 and the flag of 9 on the odd values.  The
        //    phase of word i, (p0 + 4i) mod the period, is stepped by 4T.
        {
            const uint32_t P = ODD ? (uint32_t)kStencilOddPeriod : (uint32_t)kStencilPeriod;
            const uint32_t* st = ODD ? a.stencil_odd4 : a.stencil4;
            const uint32_t W = ODD ? (uint32_t)kStencilOddWords : (uint32_t)kStencilWords;
            const i64 p0 = ODD ? base >> 1 : base;
            uint32_t ph = (uint32_t)((p0 + 4 * (i64)tid) % P);
            const uint32_t step = (4u * (uint32_t)T) % P;
            for (int i = tid; i < nw16; i += T) {
                buf32[i] = __ldg(st + (ph & 3u) * W + (ph >> 2));
                ph += step;
                if (ph >= P) ph -= P;
            }
        }
        __syncthreads();

        // 2-3. square flags for p >= 5 (:824-829) and log weights for p >= 13
        //    (:830-835).  Flags are idempotent ORs; weight bytes stay below 0x80,
        //    so a 32-bit add of w << 8*(j&3) never carries into a neighbour and
        //    the order of the marks does not matter.  ODD: the odd multiples only,
        //    consecutive ones 2m apart in value, m apart in bytes.
        //    Smaller moduli: balanced warp items (lanes stride the multiples).
        for (int k = 0; k < (ireg ? my_cnt : 0); ++k) {
            uint4 I;
            I.x = __shfl_sync(0xffffffffu, myI.x, k);
            I.y = __shfl_sync(0xffffffffu, myI.y, k);
            I.z = __shfl_sync(0xffffffffu, myI.z, k);
            I.w = __shfl_sync(0xffffffffu, myI.w, k);
            if (ODD) {
                const uint32_t b = __shfl_sync(0xffffffffu, myB, k);
                if (I.y < (uint32_t)nb) mark_item_from(buf32, I, I.y + b, nb, lane);
            } else {
                if (I.y < (uint32_t)nb) mark_item<ODD>(buf32, I, __shfl_sync(0xffffffffu, myInv, k), low, nb, lane);
            }
        }
        for (int it = warp; it < (ireg ? 0 : a.n_items); it += nwarps) {
            const uint4 I = __ldg(a.items + it);
            if (I.y >= (uint32_t)nb) continue;
            const uint32_t pidx = I.w & 0x7fffffffu;
            mark_item<ODD>(buf32, I, (I.w >> 31) ? __ldg(a.sqinv + pidx) : __ldg(a.pinv + pidx), low, nb, lane);
        }
        //    Larger moduli (at most kItemDiv hits per segment): one prime per thread.
        //    Squares above S hit a segment at most once: their hits come from
        //    the per-segment bucket (sq_off / sq_pos: value offsets) when there is one.
        const int sq_end = a.sq_off ? a.sqC_first : a.n_primes;
        for (int i = a.sqB_first + tid; i < sq_end; i += T) {
            const u64 p = a.primes[i];
            const u64 sq = p * p;
            if (sq > (u64)end) break;
            const u64 r = umod_inv((u64)low, sq, a.sqinv[i]);
            u64 d = r ? sq - r : 0;
            if (ODD && (d & 1)) d += sq;
            for (u64 j = ODD ? d >> 1 : d; j < (u64)nb; j += sq)
                atomicOr(&buf32[j >> 2], 0x80u << ((j & 3) * 8));
        }
        if (a.sq_off) {
            const u64 h1 = __ldg(a.sq_off + (seg - a.sq_seg0) + 1);
            const uint32_t off = (uint32_t)(base - seg_base);  // this pass's first offset
            for (u64 h = __ldg(a.sq_off + (seg - a.sq_seg0)) + tid; h < h1; h += T) {
                uint32_t j = __ldg(a.sq_pos + h);  // offset in the segment
                if (j < off || j - off >= (uint32_t)len) continue;
                j -= off;
                if (ODD) {
                    if (j & 1u) continue;  // even value
                    j >>= 1;
                }
                atomicOr(&buf32[j >> 2], 0x80u << ((j & 3) * 8));
            }
        }
        //    Offsets low mod p: on the 32-bit quotient route (qest/qfix) while
        //    p <= low and low/p < 2^31, else from the 64-bit reciprocal.  Round k
        //    gives thread t the prime T*k + t (k even) or T*k + T-1-t (k odd): the
        //    small primes of each round (the most hits) alternate between the
        //    first and the last warps, which evens out the warps' marking before
        //    the barrier.
        const double lowd = __ull2double_rn((u64)low);
        uint32_t p_n = 0;
        double rc_n = 0.0;
        if (a.tierB_first + tid < a.n_primes) {
            p_n = __ldg(a.primes + a.tierB_first + tid);
            if (a.prcp) rc_n = __ldg(a.prcp + a.tierB_first + tid);
        }
        for (int k = 0, i = a.tierB_first + tid; i < a.n_primes; ++k) {
            const uint32_t p = p_n;  // loaded one iteration ahead
            const double rc = rc_n;
            const int inext = a.tierB_first + T * (k + 1) + ((k & 1) ? tid : T - 1 - tid);
            if (inext < a.n_primes) {
                p_n = __ldg(a.primes + inext);
                if (a.prcp) rc_n = __ldg(a.prcp + inext);
            }
            const uint32_t w = (32u - __clz(p - 1)) | 1u;
            uint32_t r;
            if (a.prcp && (u64)low >= p && ((u64)low >> 31) < p)
                r = (uint32_t)low - qfix(qest(lowd, rc), (uint32_t)low, p) * p;
            else
                r = (uint32_t)umod_inv((u64)low, p, a.pinv[i]);
            uint32_t d = r ? p - r : 0;
            if (ODD && (d & 1u)) d += p;
            mark_prime(buf32, ODD ? d >> 1 : d, p, w, (uint32_t)nb);
            i = inext;
        }
        __syncthreads();

        // 4. finalize to mu bytes in place, four at a time with byte-parallel
        //    arithmetic.  With bits = bit_width(n), a byte a without the square
        //    flag has every factor sieved iff a > bits - 1, i.e. iff bit 7 of
        //    a + (0x7F - (bits - 1)) is set (no byte carries into the next); mu is
        //    -1 where that bit equals a's parity bit, else 1.  A segment holds at
        //    most one power of two above its start once low >= len (bits steps
        //    there); the word straddling it, the words holding n <= 2 and the
        //    first segments take the per-byte rule.  Bytes past nb become 0.
        //    Odd-mode segments that write no wheel bits leave this to the plane
        //    assembly (FusedFinal) but for the word straddling the power-of-two edge.
        FusedFinal fz;
        {
            const int bw_low = 64 - __clzll((u64)low);
            const u64 pow2 = 1ull << bw_low;  // first n above low with a larger bit width
            const uint32_t kbelow = (uint32_t)(0x7F - (bw_low - 1)) * 0x01010101u;
            const uint32_t kabove = (uint32_t)(0x7F - bw_low) * 0x01010101u;
            const bool simple = (u64)low >= 3 && (u64)low >= (u64)len;
            // first byte whose value reaches pow2
            const i64 edge = ODD ? (i64)((pow2 - (u64)low + 1) >> 1) : (i64)(pow2 - (u64)low);
            fz.on = ODD && simple && low > a.mu_limit;
            fz.skip = ((edge & 3) && edge < 4 * (i64)nw16) ? (int)(edge >> 2) : -1;
            fz.nb = nb;
            fz.edge = edge;
            fz.kbelow = kbelow;
            fz.kabove = kabove;
            const int i_first = fz.on ? (tid == 0 && fz.skip >= 0 ? fz.skip : nw16) : tid;
            const int i_end = fz.on ? min(nw16, fz.skip + 1) : nw16;
            for (int i = i_first; i < i_end; i += T) {
                const uint32_t v = buf32[i];
                const i64 j0 = 4 * (i64)i;
                uint32_t o;
                if (simple && (j0 + 3 < edge || j0 >= edge)) {
                    const uint32_t t = (v & 0x7F7F7F7Fu) + (j0 < edge ? kbelow : kabove);
                    const uint32_t x = ((t >> 7) ^ v) & 0x01010101u;         // 1: mu = +1, 0: mu = -1
                    const uint32_t f = ((v >> 7) & 0x01010101u) * 0xFFu;   // square flag bytes
                    o = ~f & (~(x * 0xFFu) | 0x01010101u);
                } else {
                    const u64 n0 = (u64)(low + (ODD ? 2 * j0 : j0));
                    o = 0;
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        o |= finalize_byte((v >> (8 * b)) & 0xFFu, n0 + (ODD ? 2 * b : b)) << (8 * b);
                }
                const int rem = nb - 4 * i;
                if (rem < 4) o = rem <= 0 ? 0u : (o & ((1u << (8 * rem)) - 1u));
                buf32[i] = o;
            }
        }
        __syncthreads();

        // Mobius wheel bits for j <= mu_limit coprime to 6; groups of 32 m
        // may straddle segments, hence atomicOr into the zeroed wheel.
        if (low <= a.mu_limit) {
            const i64 hi = min(end, a.mu_limit);
            const i64 g0 = (low - 1) / 192, g1 = (hi - 1) / 192;
            for (i64 g = g0 + warp; g <= g1; g += nwarps) {
                const i64 m = 32 * g + lane;
                const i64 j1 = 6 * m + 1, j5 = 6 * m + 5;
                const int v1 = (j1 >= low && j1 <= hi) ? (int)(int8_t)buf[ODD ? (j1 - low) >> 1 : j1 - low] : 0;
                const int v5 = (j5 >= low && j5 <= hi) ? (int)(int8_t)buf[ODD ? (j5 - low) >> 1 : j5 - low] : 0;
                const uint32_t a1 = __ballot_sync(0xffffffffu, v1 != 0);
                const uint32_t b1 = __ballot_sync(0xffffffffu, v1 < 0);
                const uint32_t a5 = __ballot_sync(0xffffffffu, v5 != 0);
                const uint32_t b5 = __ballot_sync(0xffffffffu, v5 < 0);
                if (lane == 0) {
                    uint32_t* wp = reinterpret_cast<uint32_t*>(a.wheel + g);
                    if (a1) atomicOr(wp + 0, a1);
                    if (b1) atomicOr(wp + 1, b1);
                    if (a5) atomicOr(wp + 2, a5);
                    if (b5) atomicOr(wp + 3, b5);
                }
            }
        }

        const int nwords = (len + 63) >> 6;  // 64-value words
        int total;
        if (ODD) {
            // 5. plane words of the segment (odd values sieved, even ones from their
            //    halves), their Mobius sums and exclusive scan
            const u64 lastmask = (len & 63) ? (1ull << (len & 63)) - 1 : ~0ull;
            for (int w = tid; w < nwords; w += T) {
                u64 nz, neg;
                planes_odd_mode(a, buf32, w, nw16, lane, base, fz, &nz, &neg);
                if (w == nwords - 1) {
                    nz &= lastmask;
                    neg &= lastmask;
                }
                gs[w] = __popcll(nz) - 2 * __popcll(neg);
                wpl[w] = make_ulonglong2(nz, neg);
                if (dense) a.dplanes[(base >> 6) + w] = make_ulonglong2(nz, neg);
                else a.planes[((base - a.u_dense) >> 6) - a.cword0 + w] = make_ulonglong2(nz, neg);
            }
            __syncthreads();
            total = block_excl_scan(gs, nwords, wtot);
            if (dense) {
                // 6. dM[i] = M(i+1) local to the segment, 16 values per thread
                int16_t* out = a.dM + base;
                for (int g = tid; g < 4 * nwords; g += T) {
                    const int w = g >> 2, sub = g & 3;
                    const ulonglong2 P = wpl[w];
                    const u64 below = sub ? (1ull << (16 * sub)) - 1 : 0ull;
                    int run = carry + gs[w] + __popcll(P.x & below) - 2 * __popcll(P.y & below);
                    const uint32_t z = (uint32_t)(P.x >> (16 * sub)) & 0xFFFFu;
                    const uint32_t n = (uint32_t)(P.y >> (16 * sub)) & 0xFFFFu;
                    uint32_t pk[8];
#pragma unroll
                    for (int b = 0; b < 16; b += 2) {
                        run += (int)((z >> b) & 1u) - 2 * (int)((n >> b) & 1u);
                        const uint32_t lo = (uint32_t)(run & 0xFFFF);
                        run += (int)((z >> (b + 1)) & 1u) - 2 * (int)((n >> (b + 1)) & 1u);
                        pk[b >> 1] = lo | ((uint32_t)(run & 0xFFFF) << 16);
                    }
                    if (16 * g + 16 <= len) {
                        uint4* dst = reinterpret_cast<uint4*>(out + 16 * g);
                        dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                        dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                    } else {
                        const int rem = len - 16 * g;  // fewer than 16 values left: constant indices
#pragma unroll
                        for (int b = 0; b < 16; ++b)
                            if (b < rem) out[16 * g + b] = (int16_t)((pk[b >> 1] >> (16 * (b & 1))) & 0xFFFFu);
                    }
                }
            } else {
                int32_t* ck = a.ckpt + (((base - a.u_dense) >> 6) - a.cword0);
                for (int w = tid; w < nwords; w += T) ck[w] = carry + gs[w];
            }
        } else {
            // 5. 16-value group sums and their exclusive scan
            for (int g = tid; g < ng; g += T) {
                const uint4 v = reinterpret_cast<const uint4*>(buf)[g];
                int s = __dp4a((int)v.x, 0x01010101, 0);
                s = __dp4a((int)v.y, 0x01010101, s);
                s = __dp4a((int)v.z, 0x01010101, s);
                s = __dp4a((int)v.w, 0x01010101, s);
                gs[g] = s;
            }
            __syncthreads();
            total = block_excl_scan(gs, ng, wtot);

            // 6. outputs
            if (dense) {
                // dM[i] = M(i+1) local to the segment; offsets added by fixup_kernel
                int16_t* out = a.dM + base;
                for (int g = tid; g < ng; g += T) {
                    const uint4 v = reinterpret_cast<const uint4*>(buf)[g];
                    int run = carry + gs[g];
                    uint32_t pk[8];
                    const uint32_t words[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int b = 0; b < 16; b += 2) {
                        run += (int)(int8_t)((words[b >> 2] >> (8 * (b & 3))) & 0xFFu);
                        const uint32_t lo = (uint32_t)(run & 0xFFFF);
                        run += (int)(int8_t)((words[(b + 1) >> 2] >> (8 * ((b + 1) & 3))) & 0xFFu);
                        pk[b >> 1] = lo | ((uint32_t)(run & 0xFFFF) << 16);
                    }
                    if (16 * g + 16 <= len) {
                        uint4* dst = reinterpret_cast<uint4*>(out + 16 * g);
                        dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                        dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                    } else {
                        const int rem = len - 16 * g;  // fewer than 16 values left: constant indices
#pragma unroll
                        for (int b = 0; b < 16; ++b)
                            if (b < rem) out[16 * g + b] = (int16_t)((pk[b >> 1] >> (16 * (b & 1))) & 0xFFFFu);
                    }
                }
            }
            if (!dense || a.dplanes) {
                // 64-value plane words (compressed tier, or the dense scratch planes
                // that odd-mode segments read) and the local checkpoints
                for (int w = tid; w < nwords; w += T) {
                    u64 nz, neg;
                    planes_of_bytes(buf32, w, nw16, lane, &nz, &neg);
                    if (dense) {
                        a.dplanes[(base >> 6) + w] = make_ulonglong2(nz, neg);
                    } else {
                        const i64 wbase = ((base - a.u_dense) >> 6) - a.cword0;
                        a.planes[wbase + w] = make_ulonglong2(nz, neg);
                        a.ckpt[wbase + w] = carry + gs[4 * w];
                    }
                }
            }
        }
        carry += total;
        __syncthreads();  // the next pass reuses the shared buffer
      }
        if (tid == 0) a.seg_sum[seg] = carry;
    }
}

int build_sieve_items(const uint32_t* primes, int n_primes, int S, uint4* out, int cap) {
    const uint32_t lim = (uint32_t)(S / kItemDiv);
    int n = 0;
    for (int i = 0; i < n_primes; ++i) {
        const uint32_t p = primes[i];
        if (p >= 13 && p < lim) {
            const uint32_t w = (32u - (uint32_t)__builtin_clz(p - 1)) | 1u;
            for (uint32_t st = 0; st < (uint32_t)S; st += (uint32_t)kItemHits * p) {
                if (n >= cap) return -1;  // an item would be dropped: its marks would be missing
                out[n++] = make_uint4(p, st, w, (uint32_t)i);
            }
        }
        if (p >= 5 && p * p < lim) {
            const uint32_t q = p * p;
            for (uint32_t st = 0; st < (uint32_t)S; st += (uint32_t)kItemHits * q) {
                if (n >= cap) return -1;
                out[n++] = make_uint4(q, st, 0x80u, (uint32_t)i | 0x80000000u);
            }
        }
    }
    return n;
}

int sieve_items_prefix(const uint4* items, int n_items, int n_primes) {
    int k = 0;
    while (k < n_items && (int)(items[k].w & 0x7fffffffu) < n_primes) ++k;
    return k;
}

void sieve_kernel_attrs(size_t smem, bool odd, int block, int* per_sm) {
    *per_sm = 0;
    if (odd) {
        cudaFuncSetAttribute(sieve_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, sieve_kernel<true>, block, smem);
    } else {
        cudaFuncSetAttribute(sieve_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, sieve_kernel<false>, block, smem);
    }
}

void launch_sieve(const SieveArgs& a, bool odd, int grid, int block, size_t smem, cudaStream_t s) {
    if (a.seg_end <= a.seg_begin) return;
    if (odd) sieve_kernel<true><<<grid, block, smem, s>>>(a);
    else sieve_kernel<false><<<grid, block, smem, s>>>(a);
}

namespace {
// segment holding value v (1 <= v <= u_total)
i64 segment_of_value(i64 v, i64 dense_segs, i64 u_dense, int S) {
    return v <= u_dense ? (v - 1) / S : dense_segs + (v - 1 - u_dense) / S;
}
}  // namespace

i64 sieve_odd_range_end(i64 a, i64 nseg, i64 dense_segs, i64 u_dense, i64 u_total, int S) {
    // the halves of segment s reach value floor(end_s / 2); that bound grows with s
    i64 b = a;
    while (b < nseg) {
        const bool dense = b < dense_segs;
        const i64 base = dense ? b * (i64)S : u_dense + (b - dense_segs) * (i64)S;
        const i64 end = std::min(base + (i64)S, dense ? u_dense : u_total);
        if (segment_of_value(end / 2, dense_segs, u_dense, S) >= a) break;
        ++b;
    }
    return b;
}

bool sieve_odd_ok(i64 u_dense, i64 nseg, i64 first_odd) { return (u_dense % 64) == 0 && nseg > first_odd; }

std::vector<SieveLaunch> sieve_launch_plan(i64 u_total, i64 u_dense, int S, i64 first_wave) {
    const i64 dense_segs = (u_dense + S - 1) / S;
    const i64 nseg = dense_segs + (u_total - u_dense + S - 1) / S;
    const i64 first_odd = std::min<i64>(nseg, std::max<i64>(first_wave, 1));
    std::vector<SieveLaunch> plan;
    if (!sieve_odd_ok(u_dense, nseg, first_odd)) {
        plan.push_back({0, nseg, false});
        return plan;
    }
    plan.push_back({0, first_odd, false});
    for (i64 b0 = first_odd; b0 < nseg;) {
        const i64 b1 = sieve_odd_range_end(b0, nseg, dense_segs, u_dense, u_total, S);
        if (b1 <= b0) {  // never expected: the rest in full mode
            plan.push_back({b0, nseg, false});
            break;
        }
        plan.push_back({b0, b1, true});
        b0 = b1;
    }
    return plan;
}

// 4 copies of the periodic stencil shifted by 0..3 bytes (entry i describes
// n = i + 1: weights of 2,3,5,7,11 and square flags of 4 and 9).
std::vector<uint32_t> make_stencil4() {
    std::vector<uint8_t> st(kStencilPeriod + 8);
    const unsigned small[5] = {2, 3, 5, 7, 11};
    for (int i = 0; i < kStencilPeriod + 8; ++i) {
        const int n = (i % kStencilPeriod) + 1;
        unsigned a = 0;
        for (unsigned p : small)
            if (n % (int)p == 0) a += (unsigned)((32 - __builtin_clz(p - 1)) | 1);
        if (n % 4 == 0 || n % 9 == 0) a |= 0x80u;
        st[(size_t)i] = (uint8_t)a;
    }
    std::vector<uint32_t> out((size_t)4 * kStencilWords);
    for (int s = 0; s < 4; ++s)
        for (int w = 0; w < kStencilWords; ++w) {
            uint32_t v = 0;
            for (int b = 0; b < 4; ++b) {
                const size_t idx = (size_t)(4 * w + s + b);
                v |= (uint32_t)(idx < st.size() ? st[idx] : 0) << (8 * b);
            }
            out[(size_t)s * kStencilWords + (size_t)w] = v;
        }
    return out;
}

// The same for the odd values: entry k describes n = 2k + 1 (mod 2 * 3465).
std::vector<uint32_t> make_stencil_odd4() {
    std::vector<uint8_t> st(kStencilOddPeriod + 8);
    const unsigned small[4] = {3, 5, 7, 11};
    for (int k = 0; k < kStencilOddPeriod + 8; ++k) {
        const int n = 2 * (k % kStencilOddPeriod) + 1;
        unsigned a = 0;
        for (unsigned p : small)
            if (n % (int)p == 0) a += (unsigned)((32 - __builtin_clz(p - 1)) | 1);
        if (n % 9 == 0) a |= 0x80u;
        st[(size_t)k] = (uint8_t)a;
    }
    std::vector<uint32_t> out((size_t)4 * kStencilOddWords);
    for (int s = 0; s < 4; ++s)
        for (int w = 0; w < kStencilOddWords; ++w) {
            uint32_t v = 0;
            for (int b = 0; b < 4; ++b) {
                const size_t idx = (size_t)(4 * w + s + b);
                v |= (uint32_t)(idx < st.size() ? st[idx] : 0) << (8 * b);
            }
            out[(size_t)s * kStencilOddWords + (size_t)w] = v;
        }
    return out;
}

// segment of value n (1 <= n <= u_total) and its position there (dense segments
// cover [seg*S + 1, ...], compressed ones [u_dense + (seg - dense_segs)*S + 1, ...])
__device__ __forceinline__ void segment_of(u64 n, i64 u_dense, i64 dense_segs, int lgS, u64* seg, uint32_t* j) {
    const u64 o = n <= (u64)u_dense ? n - 1 : n - 1 - (u64)u_dense;
    const u64 k = o >> lgS;
    *seg = n <= (u64)u_dense ? k : (u64)dense_segs + k;
    *j = (uint32_t)(o - (k << lgS));
}

// one CTA per prime, threads over the multiples m*p^2
// The multiples of p^2 in (vlo, vhi]; bucket arrays indexed by segment - seg0 (a
// streamed band buckets only its own segments: vlo, seg0 = its first value - 1 and
// segment; the whole table: vlo = seg0 = 0, vhi = u_total).
__global__ void sq_bucket_count_kernel(const uint32_t* primes, int first, i64 vlo, i64 vhi, i64 u_dense,
                                       i64 dense_segs, int lgS, i64 seg0, u64* counts) {
    const u64 p = primes[first + blockIdx.x], sq = p * p;
    for (u64 n = sq * ((u64)vlo / sq + 1 + threadIdx.x); n <= (u64)vhi; n += sq * blockDim.x) {
        u64 seg;
        uint32_t j;
        segment_of(n, u_dense, dense_segs, lgS, &seg, &j);
        atomicAdd(counts + (seg - (u64)seg0), 1ull);
    }
}

__global__ void sq_bucket_fill_kernel(const uint32_t* primes, int first, i64 vlo, i64 vhi, i64 u_dense,
                                      i64 dense_segs, int lgS, i64 seg0, const u64* off, u64* cur, uint32_t* pos) {
    const u64 p = primes[first + blockIdx.x], sq = p * p;
    for (u64 n = sq * ((u64)vlo / sq + 1 + threadIdx.x); n <= (u64)vhi; n += sq * blockDim.x) {
        u64 seg;
        uint32_t j;
        segment_of(n, u_dense, dense_segs, lgS, &seg, &j);
        const u64 b = seg - (u64)seg0;
        pos[off[b] + atomicAdd(cur + b, 1ull)] = j;
    }
}

void launch_sq_bucket_count(const uint32_t* primes, int first, int n, i64 vlo, i64 vhi, i64 u_dense, i64 dense_segs,
                            int lgS, i64 seg0, u64* counts, cudaStream_t s) {
    if (n > first)
        sq_bucket_count_kernel<<<n - first, 128, 0, s>>>(primes, first, vlo, vhi, u_dense, dense_segs, lgS, seg0,
                                                         counts);
}

void launch_sq_bucket_fill(const uint32_t* primes, int first, int n, i64 vlo, i64 vhi, i64 u_dense, i64 dense_segs,
                           int lgS, i64 seg0, const u64* off, u64* cur, uint32_t* pos, cudaStream_t s) {
    if (n > first)
        sq_bucket_fill_kernel<<<n - first, 128, 0, s>>>(primes, first, vlo, vhi, u_dense, dense_segs, lgS, seg0, off,
                                                        cur, pos);
}

// ---------------------------------------------------------------------------
// Segment offsets (single block) and the fix-up pass.
// ---------------------------------------------------------------------------
// out[i] = sum of in[j] for j < i, for i in [b0, b1], given out[b0] (0 for b0 = 0):
// the segment offsets of the segments [b0, b1) plus the running total at b1, so that
// the scan of the next range [b1, ...) can start there.
__global__ void __launch_bounds__(1024) seg_scan_kernel(const int32_t* in, int32_t* out, i64 b0, i64 b1) {
    __shared__ int32_t tile[1024];
    __shared__ int32_t wtot[33];
    int carry = b0 == 0 ? 0 : out[b0];
    for (i64 b = b0; b < b1; b += blockDim.x) {
        const i64 i = b + threadIdx.x;
        tile[threadIdx.x] = i < b1 ? in[i] : 0;
        __syncthreads();
        const int tot = block_excl_scan(tile, (int)blockDim.x, wtot);
        if (i < b1) out[i] = carry + tile[threadIdx.x];
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[b1] = carry;
}

void launch_seg_scan(const int32_t* in, int32_t* out, i64 n, cudaStream_t s) {
    seg_scan_kernel<<<1, 1024, 0, s>>>(in, out, 0, n);
}

void launch_seg_scan_range(const int32_t* in, int32_t* out, i64 b0, i64 b1, int threads, cudaStream_t s) {
    if (b1 > b0) seg_scan_kernel<<<1, threads, 0, s>>>(in, out, b0, b1);
}

// Adds the segment offsets to the dense prefix values of the 8-value groups [g0, g1)
// and to the checkpoints [w0, w1) (int16 wrap-around on the dense tier, as the
// reference's int16 conversion).
__global__ void fixup_kernel(int16_t* dM, i64 u_dense, int lgS, const int32_t* seg_off, int32_t* ckpt, i64 g0,
                             i64 g1, i64 w0, i64 w1, i64 dense_segs, i64 cword0) {
    const i64 stride = (i64)gridDim.x * blockDim.x;
    const i64 t0 = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    for (i64 i = g0 + t0; i < g1; i += stride) {
        const int32_t off = seg_off[(8 * i) >> lgS];
        if (8 * i + 8 <= u_dense) {
            uint4* p = reinterpret_cast<uint4*>(dM) + i;
            uint4 v = *p;
            const uint32_t o2 = ((uint32_t)off & 0xFFFFu) * 0x10001u;
            v.x = __vadd2(v.x, o2);
            v.y = __vadd2(v.y, o2);
            v.z = __vadd2(v.z, o2);
            v.w = __vadd2(v.w, o2);
            *p = v;
        } else {
            for (i64 k = 8 * i; k < u_dense; ++k) dM[k] = (int16_t)(dM[k] + off);
        }
    }
    for (i64 w = w0 + t0; w < w1; w += stride) ckpt[w - cword0] += seg_off[dense_segs + ((64 * w) >> lgS)];
}

// The fix-up of segments [b0, b1): their dense groups and their checkpoint words.
void launch_fixup_range(int16_t* dM, i64 u_dense, int S, const int32_t* seg_off, int32_t* ckpt, i64 nwords,
                        i64 dense_segs, i64 b0, i64 b1, int blocks, cudaStream_t s, i64 cword0) {
    int lgS = 0;  // S is a power of two (2^12 .. 2^18)
    while ((1 << lgS) < S) ++lgS;
    const i64 n8 = (u_dense + 7) / 8;
    const i64 g0 = std::min(n8, (b0 * (i64)S) / 8), g1 = std::min(n8, (std::min(b1, dense_segs) * (i64)S) / 8);
    const i64 c0 = std::max(b0, dense_segs) - dense_segs, c1 = std::max(b1, dense_segs) - dense_segs;
    const i64 w0 = std::min(nwords, c0 * (i64)(S / 64)), w1 = std::min(nwords, c1 * (i64)(S / 64));
    // the last dense segment may end inside a group: its tail group belongs to it
    const i64 g1x = (b1 >= dense_segs) ? n8 : g1;
    const i64 work = std::max(g1x - g0, w1 - w0);
    if (work <= 0) return;
    const int grid = (int)std::max<i64>(1, std::min<i64>((work + 255) / 256, (i64)blocks));
    fixup_kernel<<<grid, 256, 0, s>>>(dM, u_dense, lgS, seg_off, ckpt, g0, g1x, w0, w1, dense_segs, cword0);
}

void launch_fixup(int16_t* dM, i64 u_dense, int S, const int32_t* seg_off, int32_t* ckpt, i64 nwords,
                  i64 dense_segs, int sm_count, cudaStream_t s) {
    const i64 nseg_all = dense_segs + (nwords * 64 + S - 1) / S;
    launch_fixup_range(dM, u_dense, S, seg_off, ckpt, nwords, dense_segs, 0, std::max<i64>(nseg_all, dense_segs),
                       sm_count * 8, s, 0);
}

// ---------------------------------------------------------------------------
// Planning: op counts and constant parts per evaluation slot.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int query_of_slot(const QueryDev* q, int nq, u64 s) {
    int lo = 0, hi = nq - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (q[mid].slot_base <= s) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// S1 lookups of an evaluation whose quotient y/n lies in the compressed tier
// (q > u_dense, i.e. n <= y/(u_dense+1)): a prefix of each S1 segment's divisors.
__device__ __forceinline__ u64 s1_compressed_lookups(const EvalDesc& d, const TableView& T) {
    const i64 nc = (i64)udiv(d.y, (u64)T.u_dense + 1);  // largest n with y/n > u_dense
    u64 tot = 0;
    for (int g = 0; g < kS1Seg; ++g) {
        const i64 cnt = d.s1_full[g], n0 = d.s1_n0[g];
        if (cnt <= 0) continue;
        const int st = d.s1_stride[g];
        i64 k;
        if (st == S1_WHEEL) k = nc >= 1 ? wheel_upper(nc) - n0 + 1 : 0;
        else k = nc >= n0 ? (nc - n0) / st + 1 : 0;
        tot += (u64)max(0ll, min(k, cnt));
    }
    return tot;
}

// counts[kCountsPerQuery*q + 0..4]: terms, evaluations, S1 lookups, S2 wheel
// positions, compressed-tier S1 lookups -- summed over the warp before the atomics
// (a band pass of a streamed table, band.s1_only, counts only its S1 lookups and adds
// no constant part: those belong to the resident pass)
__global__ void plan_kernel(const QueryDev* __restrict__ qs, int nq, const TableView T, u64 n_slots,
                            u64* __restrict__ ops, u64* __restrict__ acc, i64* __restrict__ counts,
                            S1WinDesc* __restrict__ wdesc, SlotDesc* __restrict__ slots, const S1Band band) {
    // whole warps step together (the stride is a multiple of 32), so the counters
    // can be summed over the warp with every lane taking part
    const u64 stride = (u64)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (u64 s0 = (u64)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); s0 < n_slots; s0 += stride) {
        const u64 s = s0 + (u64)lane;
        const bool valid = s < n_slots;
        const int qi = query_of_slot(qs, nq, valid ? s : n_slots - 1);
        u64 v[7] = {0, 0, 0, 0, 0, 0, 0};  // C, terms, evaluations, S1, S2, compressed S1, S1 sum
        if (valid) {
            const QueryDev Q = qs[qi];
            const u64 local = s - Q.slot_base;
            EvalDesc d;
            decode_eval(Q, T, (i64)(local >> 1), (int)(local & 1), d, band);
            if (band.s1_only && d.kind != EVAL_NONE && d.total <= kBandInThread) {
                // a band pass: nearly every evaluation has a handful of lookups in the band;
                // this thread sums them (exact quotients, the band's view of the table), so
                // the sums kernel only walks the few evaluations with more
                i64 part = 0;
                for (int g = 0; g < kS1Seg; ++g) {
                    i64 pg = 0;
                    for (i64 i = 0; i < d.s1_cnt[g]; ++i)
                        pg += table_M(T, udiv(d.y, s1_n_at(d.s1_n0[g], d.s1_stride[g], (u64)i)));
                    part += d.coef * d.s1_sign[g] > 0 ? pg : -pg;
                }
                v[6] = (u64)part;
                for (int g = 0; g < kS1Seg; ++g) d.s1_cnt[g] = 0;
                d.total = 0;
            }
            ops[s] = d.total;
            pack_slot(d, slots + s);
            if (wdesc && Q.win) {
                S1WinDesc w;
                w.y = d.y;
                for (int g = 0; g < kS1Seg; ++g) {
                    const bool on = d.kind != EVAL_NONE && d.s1_full[g] > 0 && d.s1_wc[g] > 0;
                    w.n0[g] = on ? (uint32_t)d.s1_n0[g] : 0u;
                    w.cnt[g] = on ? (uint32_t)d.s1_full[g] : 0u;
                    w.wc[g] = on ? (uint32_t)d.s1_wc[g] : 0u;
                    w.w0[g] = on ? (uint32_t)(udiv(d.y, s1_n_at(d.s1_n0[g], d.s1_stride[g], (u64)(d.s1_full[g] - 1))) /
                                              Q.win)
                                 : 0u;
                    w.sg[g] = on ? (int32_t)(d.coef * d.s1_sign[g]) * d.s1_stride[g] : 0;
                }
                wdesc[s] = w;
            }
            if (d.kind != EVAL_NONE) {
                if (!band.s1_only) {
                    v[0] = (u64)(d.coef * eval_constant(d, T));
                    v[1] = (local & 1) == 0 ? 1 : 0;
                    v[2] = 1;
                }
                u64 s1d = 0, s1f = 0;  // lookups left to the sums kernel, all lookups
                for (int g = 0; g < kS1Seg; ++g) {
                    s1d += (u64)d.s1_cnt[g];
                    s1f += (u64)d.s1_full[g];
                }
                v[3] = s1f;
                v[4] = d.total - s1d;
                v[5] = s1_compressed_lookups(d, T);
            }
        }
        // one atomic per counter and warp where all its slots belong to one query
        const int q0 = __shfl_sync(0xffffffffu, qi, 0);
        if (__all_sync(0xffffffffu, qi == q0)) {
#pragma unroll
            for (int i = 0; i < 7; ++i) v[i] = warp_sum_u64(v[i]);
            if (lane == 0) {
                atomicAdd(acc + 3 * qi, v[0]);
                if (v[6]) atomicAdd(acc + 3 * qi + 1, v[6]);
                unsigned long long* cq = reinterpret_cast<unsigned long long*>(counts + kCountsPerQuery * qi);
                for (int i = 0; i < 5; ++i)
                    if (v[i + 1]) atomicAdd(cq + i, v[i + 1]);
            }
        } else if (valid) {
            if (v[0]) atomicAdd(acc + 3 * qi, v[0]);
            if (v[6]) atomicAdd(acc + 3 * qi + 1, v[6]);
            unsigned long long* cq = reinterpret_cast<unsigned long long*>(counts + kCountsPerQuery * qi);
            for (int i = 0; i < 5; ++i)
                if (v[i + 1]) atomicAdd(cq + i, v[i + 1]);
        }
    }
}

void launch_plan(const QueryDev* q, int nq, const TableView& T, u64 n_slots, u64* ops, u64* acc, i64* counts,
                 S1WinDesc* wdesc, SlotDesc* slots, int sm_count, cudaStream_t s, const S1Band& band) {
    if (n_slots == 0) return;
    const int grid = (int)std::min<u64>((n_slots + 127) / 128, (u64)sm_count * 16);
    plan_kernel<<<grid, 128, 0, s>>>(q, nq, T, n_slots, ops, acc, counts, wdesc, slots, band);
}

// Direct answers for queries with X <= table u_total (get_M, :1465-1467).
__global__ void direct_kernel(const QueryDev* qs, int nq, const TableView T, u64* acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nq && qs[i].N == 0) acc[3 * i] = (u64)(i64)table_M(T, qs[i].X);
}

void launch_direct(const QueryDev* q, int nq, const TableView& T, u64* acc, cudaStream_t s) {
    direct_kernel<<<(nq + 127) / 128, 128, 0, s>>>(q, nq, T, acc);
}

// ---------------------------------------------------------------------------
// u64 exclusive scan: out[0..n] with out[n] = total (three passes).
// ---------------------------------------------------------------------------
constexpr int kScanBlock = 1024;
constexpr int kScanItems = 8;
constexpr u64 kScanTile = (u64)kScanBlock * kScanItems;

__device__ u64 block_excl_scan_u64(u64 v, u64* wtot, u64* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    u64 x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u64 t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) wtot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const u64 w = lane < nwarps ? wtot[lane] : 0;
        u64 y = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u64 t = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += t;
        }
        wtot[lane] = y - w;
        if (lane == 31) wtot[32] = y;
    }
    __syncthreads();
    const u64 r = wtot[warp] + x - v;
    *total = wtot[32];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanBlock) scan_tile_sums(const u64* in, u64 n, u64* tile_sums) {
    __shared__ u64 wtot[33];
    const u64 base = (u64)blockIdx.x * kScanTile + (u64)threadIdx.x * kScanItems;
    u64 s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += in[base + k];
    u64 total;
    block_excl_scan_u64(s, wtot, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) scan_tile_offsets(u64* tile_sums, u64 ntiles) {
    __shared__ u64 wtot[33];
    u64 carry = 0;
    for (u64 b = 0; b < ntiles; b += kScanBlock) {
        const u64 i = b + threadIdx.x;
        const u64 v = i < ntiles ? tile_sums[i] : 0;
        u64 total;
        const u64 e = block_excl_scan_u64(v, wtot, &total);
        if (i < ntiles) tile_sums[i] = carry + e;
        carry += total;
    }
    if (threadIdx.x == 0) tile_sums[ntiles] = carry;
}

__global__ void __launch_bounds__(kScanBlock) scan_tile_apply(const u64* in, u64 n, const u64* tile_off, u64* out,
                                                              u64 ntiles) {
    __shared__ u64 wtot[33];
    const u64 base = (u64)blockIdx.x * kScanTile + (u64)threadIdx.x * kScanItems;
    u64 v[kScanItems];
    u64 s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    u64 total;
    u64 run = tile_off[blockIdx.x] + block_excl_scan_u64(s, wtot, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tile_off[ntiles];
}

size_t scan_u64_tmp_elems(u64 n) { return (size_t)((n + kScanTile - 1) / kScanTile) + 1; }

void launch_scan_u64(const u64* in, u64* out, u64 n, u64* tmp, size_t, cudaStream_t s) {
    const u64 ntiles = (n + kScanTile - 1) / kScanTile;
    if (ntiles == 0) {
        cudaMemsetAsync(out, 0, sizeof(u64), s);
        return;
    }
    scan_tile_sums<<<(unsigned)ntiles, kScanBlock, 0, s>>>(in, n, tmp);
    scan_tile_offsets<<<1, kScanBlock, 0, s>>>(tmp, ntiles);
    scan_tile_apply<<<(unsigned)ntiles, kScanBlock, 0, s>>>(in, n, tmp, out, ntiles);
}

// ---------------------------------------------------------------------------
// Persistent S1 / S2 kernel over the flattened op space.
// ---------------------------------------------------------------------------

// Code-shape knobs of the sums kernel (chosen by measurement on B200: 80
// registers, 3 CTAs of 256 threads per SM -- with the S1 software pipeline the
// extra registers beat the fourth CTA: sums phase 49.3 against 50.2 ms at M(10^16)).
#ifndef DRB_SUMS_MINB
#define DRB_SUMS_MINB 3
#endif
#ifndef DRB_S1_UNROLL
#define DRB_S1_UNROLL 8
#endif

constexpr int kS1Unroll = DRB_S1_UNROLL;  // independent gathers in flight per lane

// Exact double of a 32-bit integer on the FP64 pipe (the conversion
// instructions run on the narrow XU pipe): the low mantissa word of 2^52 + v.
__device__ __forceinline__ double u32_to_double(uint32_t v) {
    return __hiloint2double(0x43300000, (int)v) - 4503599627370496.0;
}

// 1/n for the kS1Unroll divisors n = nfirst + nstep*k of a lane's group
// (nfirst + nstep*(kS1Unroll-1) < 2^31), given r0 = 1/nfirst as tabulated.  From
// nfirst >= 256*nstep on, only r0 is read; the others start from the first-order Taylor value r0*(1 -
// k*nstep*r0), relative error (k*nstep/nfirst)^2 <= (7/256)^2 = 2^-10.4, and two Newton steps
// r += r*(1 - n*r) square that error twice (to below 2^-41, on the FP64 pipe,
// which the loop leaves idle) -- far inside what the 32-bit dense route needs
// (q < 2^32).  Below that every reciprocal is loaded.  This cuts the
// L2 traffic of the reciprocal table by a factor kS1Unroll where the loop is
// bound by it.
__device__ __forceinline__ void rcp_group(const double* rcp, uint32_t nfirst, uint32_t nstep, double nstep_d,
                                          const double r0, double* rv) {
    if (nfirst >= 512u * nstep) {
        // Second-order Taylor value r0*(1 - k*t + k^2*t^2), t = nstep*r0: relative error
        // (k*t)^3 <= (7/512)^3 = 2^-18.5; one Newton step squares it to below 2^-37,
        // still far inside the 32-bit route's need (q < 2^32: error below 2^-5)
        const double xr = nstep_d * r0 * r0;  // t * r0
        const double x2 = xr * (nstep_d * r0);  // t^2 * r0
        const double nd = u32_to_double(nfirst);
        rv[0] = r0;
#pragma unroll
        for (int k = 1; k < kS1Unroll; ++k) {
            const double nk = __fma_rn((double)k, nstep_d, nd);  // exact
            double r = __fma_rn((double)(k * k), x2, __fma_rn(-(double)k, xr, r0));
            r = __fma_rn(r, __fma_rn(-nk, r, 1.0), r);
            rv[k] = r;
        }
    } else if (nfirst >= 256u * nstep) {
        const double xr = nstep_d * r0 * r0;
        const double nd = u32_to_double(nfirst);
        rv[0] = r0;
#pragma unroll
        for (int k = 1; k < kS1Unroll; ++k) {
            const double nk = __fma_rn((double)k, nstep_d, nd);  // exact
            double r = __fma_rn(-(double)k, xr, r0);
#pragma unroll
            for (int it = 0; it < 2; ++it) r = __fma_rn(r, __fma_rn(-nk, r, 1.0), r);
            rv[k] = r;
        }
    } else {
        const double* p = rcp + nfirst;
        rv[0] = r0;
#pragma unroll
        for (int k = 1; k < kS1Unroll; ++k) rv[k] = __ldg(p + nstep * (uint32_t)k);
    }
}

// sum of M(floor(y/n)) over n = n0 + stride*i, i in [i0, i1), lanes interleaved.
// Each lane walks groups of kS1Unroll of its divisors (n, n + 32*stride, ...)
// whose reciprocal loads, quotients and table gathers issue back to back, software
// pipelined over the groups: a group's first reciprocal is loaded one group ahead,
// and the gathers of a group on the dense route are summed one group later,
// so a warp's reciprocal and table latencies overlap its own arithmetic instead of
// adding up group after group.  A group
// whose divisors are tabulated and below 2^31 and whose first (largest) quotient
// is in the dense tier and below 2^32 - 1 -- q falls as n grows, so then every quotient is -- runs on
// 32-bit quotients (qest/qfix); the rest use the 64-bit routine (every q here is
// at most u_total < 2^42, inside udiv_rcp's domain) or udiv above the tables.
__device__ __forceinline__ i64 s1_part(const SumsArgs& a, u64 y, i64 n0, int stride, u64 i0, u64 i1, int lane) {
    i64 acc = 0;
    const u64 lim = (u64)a.inv_limit;
    const u64 lim31 = min(lim, (u64)0x7FFFFFFF);
    // a lane's divisors form an arithmetic progression: i -> i + 32 adds 32*stride,
    // or 96 on the wheel (candidate_k keeps its parity pattern every 32 steps)
    const uint32_t nstep = stride == S1_WHEEL ? 96u : 32u * (uint32_t)stride;
    const double nstep_d = u32_to_double(nstep);
    const double yd = __ull2double_rn(y);
    const uint32_t ylo = (uint32_t)y;
    // 2^52 + the largest quotient of the 32-bit dense route: q <= u_dense and q < 2^32 - 1
    // (the dense tier may reach 7.6e9 values; larger quotients take the 64-bit route)
    const double dense_t = 4503599627370496.0 + (double)min(a.T.u_dense, (i64)0xFFFFFFFEll);
    const int16_t* dMm1 = a.T.dM - 1;                                  // dMm1[q] = M(q)
    const u64 il = i0 + (u64)lane;
    // this lane's full groups: il + 32*kS1Unroll*g + 32*(kS1Unroll-1) < i1
    const u64 span = 32ull * (kS1Unroll - 1);
    const uint32_t groups = il + span < i1 ? (uint32_t)((i1 - il - span - 1) / (32ull * kS1Unroll) + 1) : 0u;
    const u64 gstep = (u64)nstep * kS1Unroll;
    const u64 nl = s1_n_at(n0, stride, il);  // this lane's first divisor
    u64 nfirst = nl;
    int32_t pv[kS1Unroll];  // the previous dense group's gathered M values, not yet summed
#pragma unroll
    for (int k = 0; k < kS1Unroll; ++k) pv[k] = 0;
    double r0 = groups && nl <= lim ? __ldg(a.rcp + nl) : 0.0;  // 1/nfirst of the coming group
    for (uint32_t g = 0; g < groups; ++g, nfirst += gstep) {
        const u64 nlast = nfirst + (u64)nstep * (kS1Unroll - 1);
        const double r0g = r0;
        r0 = g + 1 < groups && nfirst + gstep <= lim ? __ldg(a.rcp + nfirst + gstep) : 0.0;
        if (nlast <= lim31) {
            const uint32_t nf = (uint32_t)nfirst;
            double rv[kS1Unroll];
            rcp_group(a.rcp, nf, nstep, nstep_d, r0g, rv);
            // t0 = 2^52 + qest of the first divisor: qest <= u_dense bounds q
            const double t0 = __fma_ru(yd, rv[0], kQBias);
            if (t0 <= dense_t) {
                uint32_t qq[kS1Unroll];
#pragma unroll
                for (int k = 0; k < kS1Unroll; ++k) {
                    const uint32_t qp = k == 0 ? (uint32_t)__double2loint(t0) : qest(yd, rv[k]);
                    qq[k] = qfix(qp, ylo, nf + nstep * (uint32_t)k);
                }
                int32_t part = 0;
#pragma unroll
                for (int k = 0; k < kS1Unroll; ++k) {
                    part += pv[k];
                    pv[k] = __ldg(dMm1 + qq[k]);
                }
                acc += part;
            } else {  // compressed tier or q >= 2^32 - 1 (rare): exact tabulated reciprocals, udiv_rcp
#pragma unroll
                for (int k = 0; k < kS1Unroll; ++k) {
                    const uint32_t n = nf + nstep * (uint32_t)k;
                    acc += table_M(a.T, udiv_rcp(y, yd, n, __ldg(a.rcp + n)));
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < kS1Unroll; ++k) {
                const u64 n = nfirst + (u64)nstep * k;
                acc += table_M(a.T, n <= lim ? udiv_rcp(y, yd, (uint32_t)n, __ldg(a.rcp + n)) : udiv(y, n));
            }
        }
    }
    {
        int32_t part = 0;
#pragma unroll
        for (int k = 0; k < kS1Unroll; ++k) part += pv[k];
        acc += part;
    }
    u64 n = nl + gstep * groups;
    for (u64 i = il + 32ull * kS1Unroll * groups; i < i1; i += 32, n += nstep)
        acc += table_M(a.T, n <= lim ? udiv_rcp(y, yd, (uint32_t)n, __ldg(a.rcp + n)) : udiv(y, n));
    return acc;
}

// Summand kinds: most positions fall in pieces whose summand needs no
// division by 12 (the split of f_A(q) - f_B(q/2) and f_A(q) of dr_device.cuh):
//   kind 1: q            (pieces 8, 12)
//   kind 2: (q + 1) >> 1 (pieces 7, 11)
//   kind 3: q & 1        (piece 6)
//   kind 4: (q >> 2) + (q & 1)  (piece 5)
//   kind 0: a * (q / 12) + T[q mod 12]  (pieces 1-4, 9, 10)
__host__ __device__ constexpr int piece_kind(int piece) {
    return piece == 8 || piece == 12 ? 1 : piece == 7 || piece == 11 ? 2 : piece == 6 ? 3 : piece == 5 ? 4 : 0;
}

template <int KIND>
__device__ __forceinline__ i64 piece_value(const PieceCoef& pc, u64 q) {
    if (KIND == 1) return (i64)q;
    if (KIND == 2) return (i64)((q + 1) >> 1);
    if (KIND == 3) return (i64)(q & 1);
    if (KIND == 4) return (i64)((q >> 2) + (q & 1));
    return piece_eval(pc, q);
}

// mu(j) * piece(floor(y/j)) for one wheel position m (j = 6m+1, 6m+5); only the
// first and last position of a piece can have a j outside [jlo, jhi].
template <int KIND, bool RCP>
__device__ __forceinline__ u64 s2_position(u64 y, double yd, const PieceCoef& pc, i64 jlo, i64 jhi, u64 m,
                                           bool edge, const uint4 w, const double2 iv) {
    const uint32_t b = (uint32_t)(m & 31u);
    bool t1 = (w.x >> b) & 1u, t5 = (w.z >> b) & 1u;
    if (edge) {
        const i64 j1 = (i64)(6 * m + 1), j5 = (i64)(6 * m + 5);
        t1 = t1 && j1 >= jlo && j1 <= jhi;
        t5 = t5 && j5 >= jlo && j5 <= jhi;
    }
    u64 acc = 0;
    if (t1) {
        const u64 q = RCP ? udiv_rcp(y, yd, (uint32_t)(6 * m + 1), iv.x) : udiv(y, 6 * m + 1);
        const u64 v = (u64)piece_value<KIND>(pc, q);
        const u64 sg = 0ull - (u64)((w.y >> b) & 1u);  // all ones when mu = -1
        acc += (v ^ sg) - sg;
    }
    if (t5) {
        const u64 q = RCP ? udiv_rcp(y, yd, (uint32_t)(6 * m + 5), iv.y) : udiv(y, 6 * m + 5);
        const u64 v = (u64)piece_value<KIND>(pc, q);
        const u64 sg = 0ull - (u64)((w.w >> b) & 1u);
        acc += (v ^ sg) - sg;
    }
    return acc;
}

// sum of mu(j) * piece(floor(y/j)) for j in {6m+1, 6m+5} within [jlo, jhi],
// m = jlo/6 + i, i in [i0, i1) of the piece's mcnt positions (64-bit quotients).
// RCP: every j of the range is below 2^32 and every y/j below 2^48 (udiv_rcp
// applies to invw's reciprocals).
template <int KIND, bool RCP>
__device__ __forceinline__ u64 s2_part(const SumsArgs& a, u64 y, const PieceCoef pc, i64 jlo, i64 jhi, u64 mcnt,
                                       u64 i0, u64 i1, int lane) {
    u64 acc = 0;
    const double yd = __ull2double_rn(y);
    const u64 m0 = (u64)(jlo / 6);
    const u64 last = mcnt - 1;
    for (u64 i = i0 + lane; i < i1; i += 32) {
        const u64 m = m0 + i;
        acc += s2_position<KIND, RCP>(y, yd, pc, jlo, jhi, m, i == 0 || i == last, __ldg(a.T.wheel + (m >> 5)),
                                      __ldg(a.invw + m));
    }
    return acc;
}

// The summand on q < 2^31 in 32-bit arithmetic; sT[r] = piece(r), r < 12.
template <int KIND>
__device__ __forceinline__ int32_t piece32(int32_t a12, const int32_t* sT, uint32_t q) {
    if (KIND == 1) return (int32_t)q;
    if (KIND == 2) return (int32_t)((q + 1) >> 1);
    if (KIND == 3) return (int32_t)(q & 1);
    if (KIND == 4) return (int32_t)((q >> 2) + (q & 1));
    const uint32_t k = q / 12u;
    return a12 * (int32_t)k + sT[q - 12u * k];
}

// mu(j) from the low mantissa bits of invw's reciprocal (inverse_kernel)
__device__ __forceinline__ int32_t mu_code(double r) {
    return (int32_t)((uint32_t)__double2loint(r) << 30) >> 30;
}

__device__ __forceinline__ i64 mad_wide(int32_t a, int32_t b, i64 c) {
    i64 r;
    asm("mad.wide.s32 %0, %1, %2, %3;" : "=l"(r) : "r"(a), "r"(b), "l"(c));
    return r;
}

// mu(j) * piece(floor(y/j)) for the two j of a position, j1 = 6m+1 and j1 + 4,
// on the 32-bit route; take1/take5 clear j outside the piece (edge positions)
template <int KIND>
__device__ __forceinline__ i64 s2_pair32(i64 acc, double yd, uint32_t ylo, int32_t a12, const int32_t* sT,
                                         uint32_t j1, double2 iv, bool take1 = true, bool take5 = true) {
    const int32_t mu1 = take1 ? mu_code(iv.x) : 0, mu5 = take5 ? mu_code(iv.y) : 0;
    acc = mad_wide(mu1, piece32<KIND>(a12, sT, qfix(qest(yd, iv.x), ylo, j1)), acc);
    return mad_wide(mu5, piece32<KIND>(a12, sT, qfix(qest(yd, iv.y), ylo, j1 + 4u)), acc);
}

// The same sum when every j of the range is below 2^31 and every y/j below 2^31:
// 32-bit quotients (qest/qfix) and summands, mu(j) from invw as a multiplier in
// {-1, 0, 1} (both j of a position are evaluated, whatever their mu).  The
// piece's first and last positions -- the only ones that can hold a j outside
// [jlo, jhi] -- are peeled off to lanes 0 and 1.
template <int KIND>
__device__ __forceinline__ u64 s2_fast(const SumsArgs& a, u64 y, int32_t a12, const int32_t* sT, i64 jlo, i64 jhi,
                                       u64 mcnt, u64 i0, u64 i1, int lane) {
    const double yd = __ull2double_rn(y);
    const uint32_t ylo = (uint32_t)y;
    const u64 m0 = (u64)(jlo / 6);
    const u64 last = mcnt - 1;
    i64 acc = 0;
    const u64 b0 = max(i0, (u64)1), b1 = min(i1, last);  // interior positions [b0, b1)
    const u64 i = b0 + (u64)lane;
    if (i < b1) {
        const uint32_t cnt = (uint32_t)((b1 - i + 31) >> 5);
        const double2* p = a.invw + (m0 + i);
        const uint32_t j1 = (uint32_t)(6 * (m0 + i) + 1);
        for (uint32_t t = 0; t < cnt; ++t)
            acc = s2_pair32<KIND>(acc, yd, ylo, a12, sT, j1 + 192u * t, __ldg(p + 32u * t));
    }
    if (lane < 2) {
        const u64 e = lane == 0 ? 0 : last;
        if (e >= i0 && e < i1 && (lane == 0 || last != 0)) {
            const u64 m = m0 + e;
            const i64 j1 = (i64)(6 * m + 1), j5 = j1 + 4;
            acc = s2_pair32<KIND>(acc, yd, ylo, a12, sT, (uint32_t)j1, __ldg(a.invw + m), j1 >= jlo && j1 <= jhi,
                                  j5 >= jlo && j5 <= jhi);
        }
    }
    return (u64)acc;
}

// sT: the residue table of every piece in shared memory (sT[12*piece + r]).
__device__ __forceinline__ u64 s2_dispatch(const SumsArgs& a, const int32_t* sT, u64 y, int piece, i64 jlo,
                                           i64 jhi, u64 mcnt, u64 i0, u64 i1, int lane) {
    const PieceCoef pc = c_piece[piece];
    const u64 m0 = (u64)(jlo / 6);
    const u64 jmin = 6 * (m0 + i0) + 1, jmax = 6 * (m0 + i1) + 5;  // bounds every j of [i0, i1)
    if (jmax < 0x7FFFFFFFull && (y >> 31) < jmin) {
        const int32_t* T = sT + 12 * piece;
        const int32_t a12 = (int32_t)pc.a;
        switch (piece_kind(piece)) {
        case 1: return s2_fast<1>(a, y, a12, T, jlo, jhi, mcnt, i0, i1, lane);
        case 2: return s2_fast<2>(a, y, a12, T, jlo, jhi, mcnt, i0, i1, lane);
        case 3: return s2_fast<3>(a, y, a12, T, jlo, jhi, mcnt, i0, i1, lane);
        case 4: return s2_fast<4>(a, y, a12, T, jlo, jhi, mcnt, i0, i1, lane);
        default: return s2_fast<0>(a, y, a12, T, jlo, jhi, mcnt, i0, i1, lane);
        }
    }
    // invw's reciprocals carry mu in their two low bits (up to 3.5 ulp from 1/j):
    // udiv_rcp's +-1 correction then covers y/j < 2^48, not its full 2^50
    if (jmax >> 32 || (y >> 48) >= jmin) return s2_part<0, false>(a, y, pc, jlo, jhi, mcnt, i0, i1, lane);
    switch (piece_kind(piece)) {
    case 1: return s2_part<1, true>(a, y, pc, jlo, jhi, mcnt, i0, i1, lane);
    case 2: return s2_part<2, true>(a, y, pc, jlo, jhi, mcnt, i0, i1, lane);
    case 3: return s2_part<3, true>(a, y, pc, jlo, jhi, mcnt, i0, i1, lane);
    case 4: return s2_part<4, true>(a, y, pc, jlo, jhi, mcnt, i0, i1, lane);
    default: return s2_part<0, true>(a, y, pc, jlo, jhi, mcnt, i0, i1, lane);
    }
}

__device__ __forceinline__ u64 upper_slot(const u64* prefix, u64 n_slots, u64 o) {
    // largest s in [0, n_slots) with prefix[s] <= o
    u64 lo = 0, hi = n_slots - 1;
    while (lo < hi) {
        const u64 mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= o) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(256, DRB_SUMS_MINB) sums_kernel(const SumsArgs a) {
    __shared__ EvalDesc sdesc[8];  // one decoded evaluation per warp
    __shared__ int32_t sT[13 * 12];  // piece(r) for r < 12, every piece
    for (int t = threadIdx.x; t < 13 * 12; t += blockDim.x) {
        const PieceCoef pc = c_piece[t / 12];
        sT[t] = (int32_t)((pc.packed >> (5 * (t % 12))) & 31u) - 16;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    EvalDesc& d = sdesc[threadIdx.x >> 5];
    const u64 total = a.prefix[a.n_slots];
    int lg = a.chunk_log2;
    if (lg <= 0) {
        const u64 warps = (u64)gridDim.x * (blockDim.x >> 5);
        const u64 want = total / (warps * 16) + 1;
        lg = 64 - __clzll(want);
        lg = max(11, min(lg, 16));
    }
    const u64 W = 1ull << lg;
    int cur_q = -1;
    u64 s1 = 0, s2 = 0;
    for (;;) {
        u64 chunk = 0;
        if (lane == 0) chunk = atomicAdd(a.ticket, 1ull);
        chunk = __shfl_sync(0xffffffffu, chunk, 0);
        u64 o = chunk * W;
        if (o >= total) break;
        const u64 o_end = min(o + W, total);
        u64 s = upper_slot(a.prefix, a.n_slots, o);
        while (o < o_end) {
            // the next slot with ops: a few steps over slots without, then a search (a
            // band pass of a streamed table leaves long runs of such slots)
            for (int k = 0; k < 4 && a.prefix[s + 1] <= o; ++k) ++s;
            if (a.prefix[s + 1] <= o) s = upper_slot(a.prefix, a.n_slots, o);
            const u64 sbase = a.prefix[s];
            const int qi = a.nq == 1 ? 0 : query_of_slot(a.queries, a.nq, s);
            __syncwarp();
            if (lane == 0) unpack_slot(a.slots[s], d);  // the planner's decoded evaluation
            __syncwarp();
            if (qi != cur_q) {
                if (cur_q >= 0) {
                    const u64 t1 = warp_sum_u64(s1), t2 = warp_sum_u64(s2);
                    if (lane == 0) {
                        atomicAdd(a.acc + 3 * cur_q + 1, t1);
                        atomicAdd(a.acc + 3 * cur_q + 2, t2);
                    }
                }
                s1 = s2 = 0;
                cur_q = qi;
            }
            const u64 lo = o - sbase;
            const u64 hi = min(o_end - sbase, d.total);
            if (hi <= lo) {
                // planning and decoding disagree on this slot's op count: flag
                // it and abandon the chunk instead of spinning without progress
                if (lane == 0) atomicOr(a.ticket + 1, 1ull);
                break;
            }
            const u64 y = d.y;
            const i64 coef = d.coef;
            const int nseg = d.nseg;
            u64 segstart = 0;
            for (int g = 0; g < nseg && segstart < hi; ++g) {
                const u64 cnt = g < kS1Seg ? (u64)d.s1_cnt[g] : (u64)d.mcnt[g - kS1Seg];
                const u64 sb = segstart;
                segstart += cnt;
                const u64 a0 = max(lo, sb), a1 = min(hi, segstart);
                if (a0 >= a1) continue;
                if (g < kS1Seg) {
                    const i64 part = s1_part(a, y, d.s1_n0[g], d.s1_stride[g], a0 - sb, a1 - sb, lane);
                    const i64 sg = coef * d.s1_sign[g];
                    s1 += sg > 0 ? (u64)part : (u64)(-part);
                } else {
                    const int p = g - kS1Seg;
                    const u64 part = s2_dispatch(a, sT, y, d.piece0 + p, d.jlo[p], d.jhi[p], (u64)d.mcnt[p], a0 - sb,
                                                 a1 - sb, lane);
                    s2 += coef > 0 ? part : (u64)(0 - part);
                }
            }
            o = sbase + hi;
            ++s;
        }
    }
    if (cur_q >= 0) {
        const u64 t1 = warp_sum_u64(s1), t2 = warp_sum_u64(s2);
        if (lane == 0) {
            atomicAdd(a.acc + 3 * cur_q + 1, t1);
            atomicAdd(a.acc + 3 * cur_q + 2, t2);
        }
    }
}

// ---------------------------------------------------------------------------
// Windowed S1.  Each work item is one window of the M table, q in [w*W, (w+1)*W),
// and a range of evaluation candidates: the CTA stages M(w*W - 7 .. (w+1)*W), i.e.
// dM[w*W - 8 .. (w+1)*W - 1], in shared memory (16-byte loads; window 0 element by
// element, M(0) = 0), and its warps sum, candidate by candidate, every
// windowed S1 lookup M(floor(y/n)) whose quotient falls in the window: for each
// S1 segment the divisors n in (y/((w+1)W), y/(wW)] -- two exact quotients per
// evaluation and window -- with lanes on consecutive n.  Each lookup is one
// reciprocal load, the 32-bit quotient route and one shared-memory read, so the M
// gathers no longer cross L2.  The lookups with q above a segment's windows are
// the sums kernel's (decode_eval); together they are every S1 lookup exactly once.
// ---------------------------------------------------------------------------
constexpr int kWinThreads = 512;

// sum of M(q) over a segment's divisors in the window [qbase, qbase + W) (qbase a
// multiple of W, so q - qbase = q & (W - 1)): lanes take consecutive divisors, so a
// lane's divisors are nl, nl + nstep, ... (nstep = 32*stride, 96 on the wheel), cntl
// of them.  The reciprocal loads mostly hit L1 (neighbouring windows reuse them).
__device__ __forceinline__ int32_t s1win_range(const int16_t* win, uint32_t wmask, const double* rcp, double yd,
                                               uint32_t ylo, uint32_t nl, uint32_t nstep, uint32_t cntl) {
    int32_t part = 0;
    const int16_t* w7 = win + 7;
    uint32_t t = 0;
    for (; t + 3 < cntl; t += 4) {
        uint32_t n[4];
        double r[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            n[k] = nl + nstep * (t + k);
            r[k] = __ldg(rcp + n[k]);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) part += w7[qfix(qest(yd, r[k]), ylo, n[k]) & wmask];
    }
    for (; t < cntl; ++t) {
        const uint32_t nn = nl + nstep * t;
        part += w7[qfix(qest(yd, __ldg(rcp + nn)), ylo, nn) & wmask];
    }
    return part;
}

__global__ void __launch_bounds__(kWinThreads, 2) s1win_kernel(const S1WinArgs a, uint32_t W) {
    extern __shared__ __align__(16) int16_t win[];  // win[7 + i] = M(w*W + i), i < W
    __shared__ S1WinItem it;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t wmask = W - 1u;
    uint32_t cur = 0xFFFFFFFFu;
    int cur_q = -1;
    i64 acc = 0;
    for (;;) {
        __syncthreads();  // the previous item's readers are done with `it` and the window
        if (threadIdx.x == 0) {
            const u64 t = atomicAdd(a.ticket, 1ull);
            it = t < a.n_items ? a.items[t] : S1WinItem{0xFFFFFFFFu, 0u, 0u, 0u};
        }
        __syncthreads();
        const S1WinItem I = it;
        if (I.w == 0xFFFFFFFFu) break;
        if ((int)I.q != cur_q) {
            if (cur_q >= 0) {
                const u64 t = warp_sum_u64((u64)acc);
                if (lane == 0) atomicAdd(a.acc + 3 * cur_q + 1, t);
            }
            acc = 0;
            cur_q = (int)I.q;
            cur = 0xFFFFFFFFu;
        }
        if (I.w != cur) {  // stage the window: win[t] = M(w*W - 7 + t) = dM[w*W - 8 + t], t < W + 8
            if (I.w > 0) {
                const uint4* src = reinterpret_cast<const uint4*>(a.T.dM + ((u64)I.w * W - 8));
                uint4* dst = reinterpret_cast<uint4*>(win);
                for (uint32_t t = threadIdx.x; t < (W + 8u) / 8u; t += blockDim.x) dst[t] = __ldg(src + t);
            } else {
                for (uint32_t t = threadIdx.x; t < W + 8u; t += blockDim.x)
                    win[t] = t >= 8u ? __ldg(a.T.dM + (t - 8u)) : (int16_t)0;
            }
            cur = I.w;
            __syncthreads();
        }
        const QueryDev Q = a.queries[I.q];
        const u64 qlo = (u64)I.w * W, qhi = qlo + W;  // window: q in [qlo, qhi)
        const double rlo = qlo ? __drcp_rn((double)qlo) : 0.0, rhi = __drcp_rn((double)qhi);
        for (uint32_t c = I.c0 + (uint32_t)warp; c < I.c1; c += (uint32_t)nwarps) {
#pragma unroll 1
            for (int e = 0; e < 2; ++e) {
                const S1WinDesc D = a.desc[Q.slot_base + 2ull * c + (u64)e];
                bool any = false;
#pragma unroll
                for (int g = 0; g < kS1Seg; ++g) any |= D.cnt[g] && D.w0[g] <= I.w && I.w < D.wc[g];
                if (!any) continue;
                const double yd = __ull2double_rn(D.y);
                // n in (y/qhi, y/qlo]  <=>  floor(y/n) in [qlo, qhi);
                // exact quotients: udiv_rcp while y/q < 2^50 (q < 2^31 here), else udiv
                const u64 nlo = ((D.y >> 50) < qhi ? udiv_rcp(D.y, yd, (uint32_t)qhi, rhi) : udiv(D.y, qhi)) + 1;
                const u64 nhi = qlo == 0 ? ~0ull
                                         : (D.y >> 50) < qlo ? udiv_rcp(D.y, yd, (uint32_t)qlo, rlo) : udiv(D.y, qlo);
#pragma unroll 1
                for (int g = 0; g < kS1Seg; ++g) {
                    if (!(D.cnt[g] && D.w0[g] <= I.w && I.w < D.wc[g])) continue;
                    const int st = D.sg[g] < 0 ? -D.sg[g] : D.sg[g];
                    // index range [ia, ib] of the segment's divisors in [nlo, nhi]
                    i64 ia, ib;
                    if (st == S1_WHEEL) {
                        ia = max((i64)0, wheel_lower((i64)nlo) - (i64)D.n0[g]);
                        ib = min((i64)D.cnt[g] - 1, nhi > 0x7FFFFFFFull ? (i64)D.cnt[g] - 1
                                                                     : wheel_upper((i64)nhi) - (i64)D.n0[g]);
                    } else {
                        ia = nlo <= D.n0[g] ? 0 : (i64)((nlo - D.n0[g] + st - 1) / st);
                        ib = nhi < D.n0[g] ? -1
                             : nhi > 0x7FFFFFFFull ? (i64)D.cnt[g] - 1  // window 0: no upper bound
                                                   : min((i64)D.cnt[g] - 1, (i64)((nhi - D.n0[g]) / st));
                    }
                    if (ia > ib) continue;
                    const u64 cnt = (u64)(ib - ia + 1);
                    const uint32_t cntl = cnt > (u64)lane ? (uint32_t)((cnt - lane + 31) >> 5) : 0u;
                    const uint32_t nstep = st == S1_WHEEL ? 96u : 32u * (uint32_t)st;
                    const uint32_t nl = (uint32_t)s1_n_at(D.n0[g], st, (u64)(ia + lane));
                    const int32_t part = s1win_range(win, wmask, a.rcp, yd, (uint32_t)D.y, nl, nstep, cntl);
                    acc += D.sg[g] > 0 ? (i64)part : -(i64)part;
                }
            }
        }
    }
    if (cur_q >= 0) {
        const u64 t = warp_sum_u64((u64)acc);
        if (lane == 0) atomicAdd(a.acc + 3 * cur_q + 1, t);
    }
}

void launch_s1win(const S1WinArgs& a, u64 win, int sm_count, cudaStream_t s) {
    if (a.n_items == 0) return;
    const size_t smem = (size_t)(win + 8) * 2;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(s1win_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(((1u << 16) + 8) * 2));
        attr = true;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, s1win_kernel, kWinThreads, smem);
    const int grid = sm_count * std::max(1, per_sm);
    s1win_kernel<<<grid, kWinThreads, smem, s>>>(a, (uint32_t)win);
}

// rcp[n] = RN(1/n) for 1 <= n <= inv_limit.  invw[m] = {rcp(6m+1), rcp(6m+5)} with
// mu(j) in the two low mantissa bits (mu & 3: 0, 1, or 3 for -1), so the S2 loops
// read j's reciprocal and its Mobius value with one load; the three ulp this may
// move 1/j are far inside what the S2 quotient routes tolerate (mu_code, s2_part).
__device__ __forceinline__ double rcp_with_mu(u64 j, const uint4* wheel) {
    const u64 m = j / 6u;
    const uint4 w = __ldg(wheel + (m >> 5));
    const uint32_t b = (uint32_t)(m & 31u);
    const bool five = (j - 6u * m) == 5u;
    const uint32_t nz = ((five ? w.z : w.x) >> b) & 1u, ng = ((five ? w.w : w.y) >> b) & 1u;
    const u64 bits = (u64)__double_as_longlong(__drcp_rn((double)j));
    return __longlong_as_double((long long)((bits & ~3ull) | (u64)(nz | (ng << 1))));
}

__global__ void inverse_kernel(double* rcp, i64 inv_limit, double2* invw, i64 invw_count, const uint4* wheel) {
    const i64 stride = (i64)gridDim.x * blockDim.x;
    const i64 t0 = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    for (i64 n = t0; n <= inv_limit; n += stride) rcp[n] = n ? __drcp_rn((double)n) : 0.0;
    for (i64 m = t0; m < invw_count; m += stride)
        invw[m] = make_double2(rcp_with_mu((u64)(6 * m + 1), wheel), rcp_with_mu((u64)(6 * m + 5), wheel));
}

void launch_inverse(double* rcp, i64 inv_limit, double2* invw, i64 invw_count, const uint4* wheel, int sm_count,
                    cudaStream_t s) {
    const i64 work = std::max<i64>(inv_limit + 1, invw_count);
    const int grid = (int)std::min<i64>((work + 255) / 256, (i64)sm_count * 16);
    inverse_kernel<<<std::max(grid, 1), 256, 0, s>>>(rcp, inv_limit, invw, invw_count, wheel);
}

void sums_kernel_occupancy(int block, int* per_sm) {
    *per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, sums_kernel, block, 0);
}

void launch_sums(const SumsArgs& a, int grid, int block, cudaStream_t s) {
    sums_kernel<<<grid, block, 0, s>>>(a);
}

// ---------------------------------------------------------------------------
// Table read-back and checksums (test support, reference get_M / get_mu).
// ---------------------------------------------------------------------------
__global__ void table_read_kernel(const TableView T, i64 first, i64 count, int32_t* M, int8_t* mu, int8_t* wmu) {
    const i64 stride = (i64)gridDim.x * blockDim.x;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const i64 n = first + i;
        const bool in = n >= 0 && n <= T.u_total;
        const int32_t m = in ? table_M(T, (u64)n) : 0;
        if (M) M[i] = m;
        if (mu) mu[i] = (int8_t)((in && n >= 1 && n <= T.mu_limit) ? m - table_M(T, (u64)(n - 1)) : 0);
        if (wmu) {
            int v = 0;
            if (n >= 1 && n <= T.mu_limit && (n % 2) && (n % 3)) v = wheel_mu(T.wheel, (u64)n);
            wmu[i] = (int8_t)v;
        }
    }
}

void launch_table_read(const TableView& T, i64 first, i64 count, int32_t* M, int8_t* mu, int8_t* wmu, cudaStream_t s) {
    if (count <= 0) return;
    const int grid = (int)std::min<i64>((count + 255) / 256, 4096);
    table_read_kernel<<<grid, 256, 0, s>>>(T, first, count, M, mu, wmu);
}

__global__ void table_sums_kernel(const TableView T, i64 nwords, u64* out) {
    const i64 stride = (i64)gridDim.x * blockDim.x;
    const i64 t0 = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    u64 ds = 0, dw = 0, mw = 0, nzw = 0, ngw = 0, cw = 0;
    for (i64 n = 1 + t0; n <= T.u_dense; n += stride) {
        const i64 v = T.dM[n - 1];
        ds += (u64)v;
        dw += (u64)v * (u64)(2 * n + 1);
    }
    for (i64 n = 1 + t0; n <= T.mu_limit; n += stride) {
        const i64 m = (i64)table_M(T, (u64)n) - (i64)table_M(T, (u64)(n - 1));
        mw += (u64)m * (u64)(2 * n + 1);
    }
    for (i64 w = t0; w < nwords; w += stride) {
        const u64 k = (u64)(2 * w + 1);
        const ulonglong2 p = T.planes[w];
        nzw += p.x * k;
        ngw += p.y * k;
        cw += (u64)(i64)T.ckpt[w] * k;
    }
    ds = warp_sum_u64(ds);
    dw = warp_sum_u64(dw);
    mw = warp_sum_u64(mw);
    nzw = warp_sum_u64(nzw);
    ngw = warp_sum_u64(ngw);
    cw = warp_sum_u64(cw);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out + 0, ds);
        atomicAdd(out + 1, dw);
        atomicAdd(out + 2, mw);
        atomicAdd(out + 3, nzw);
        atomicAdd(out + 4, ngw);
        atomicAdd(out + 5, cw);
    }
}

void launch_table_sums(const TableView& T, i64 nwords, u64* out6, int sm_count, cudaStream_t s) {
    table_sums_kernel<<<sm_count * 8, 256, 0, s>>>(T, nwords, out6);
}

// ---------------------------------------------------------------------------
// Test support: the device quotient and S2 summand on caller-chosen inputs.
// ---------------------------------------------------------------------------
// rcp = 0: udiv; rcp = 1: udiv_rcp with a device-computed reciprocal, ~0 where
// (y, d) is outside its domain (d >= 2^32 or y/d >= 2^50); rcp = 2: the 32-bit
// route of the S1/S2 fast paths (qest + qfix), ~0 where d >= 2^31, y/d >= 2^31 or
// y < d (the fast paths only divide y by d <= y)
__global__ void debug_udiv_kernel(const u64* y, const u64* d, u64* q, i64 n, int rcp) {
    const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u64 yy = y[i], dd = d[i];
    if (rcp == 0) q[i] = dd ? udiv(yy, dd) : 0;
    else if (rcp == 1) {
        if (dd == 0 || (dd >> 32) || (yy >> 50) >= dd) q[i] = ~0ull;
        else q[i] = udiv_rcp(yy, __ull2double_rn(yy), (uint32_t)dd, __drcp_rn((double)dd));
    } else {
        if (dd == 0 || (dd >> 31) || (yy >> 31) >= dd || yy < dd) q[i] = ~0ull;
        else q[i] = qfix(qest(__ull2double_rn(yy), __drcp_rn((double)dd)), (uint32_t)yy, (uint32_t)dd);
    }
}

// wide = 0: piece_eval (64-bit); wide = 1: piece32 of the S2 fast path on q < 2^31
// (INT64_MIN for larger q)
__global__ void debug_piece_kernel(const int32_t* piece, const u64* q, i64* out, i64 n, int fast) {
    const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = piece[i];
    if (p < 1 || p > 12) {
        out[i] = 0;
    } else if (!fast) {
        out[i] = piece_eval(c_piece[p], q[i]);
    } else if (q[i] >> 31) {
        out[i] = INT64_MIN;
    } else {
        const PieceCoef pc = c_piece[p];
        int32_t T[12];
        for (int r = 0; r < 12; ++r) T[r] = (int32_t)((pc.packed >> (5 * r)) & 31u) - 16;
        const uint32_t v = (uint32_t)q[i];
        const int32_t a12 = (int32_t)pc.a;
        switch (piece_kind(p)) {
        case 1: out[i] = piece32<1>(a12, T, v); break;
        case 2: out[i] = piece32<2>(a12, T, v); break;
        case 3: out[i] = piece32<3>(a12, T, v); break;
        case 4: out[i] = piece32<4>(a12, T, v); break;
        default: out[i] = piece32<0>(a12, T, v); break;
        }
    }
}

void launch_debug_udiv(const u64* y, const u64* d, u64* q, i64 n, int rcp, cudaStream_t s) {
    if (n > 0) debug_udiv_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(y, d, q, n, rcp);
}

void launch_debug_piece(const int32_t* piece, const u64* q, i64* out, i64 n, int fast, cudaStream_t s) {
    if (n > 0) debug_piece_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(piece, q, out, n, fast);
}

}  // namespace drb
