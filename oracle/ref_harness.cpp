// ref_harness.cpp -- C ABI over the reference engine, compiled from the
// reference's own header (mertens_dr.hpp, included from its source tree by
// oracle/Makefile).  TEST INFRASTRUCTURE ONLY: it pins the oracle and makes
// the golden fixtures; nothing in the product links it.
//
// The reference's S1 loops are lambdas inside compute_mertens/compute_compressed
// (mertens_dr.hpp:1081-1354, :1490-1614) and cannot be called, so
// ref_dr_checksums() re-walks the same outer terms and S1 ranges over the
// reference's own table (CompressedMertensTable::reconstruct_compressed,
// sum_dense_quotients) and S2 functions (eval_s2_single / eval_s2_combined),
// and returns the C/S1/S2 checksums defined in dr_oracle.h.  Its M(X) is
// asserted equal to compute_compressed()/compute_mertens() by the tests.
#include "mertens_dr.hpp"

#include <cstdint>
#include <cstring>
#include <memory>

using namespace mertens_dr;

namespace {

int64 split_point(double cx, int64 y) {
    int64 A = static_cast<int64>(cx * std::sqrt(static_cast<double>(y)));
    if (A >= y) A = y - 1;
    if (A < 1) A = 1;
    return A;
}

struct Sums {
    uint64_t C = 0, S1 = 0, S2 = 0;
};

}  // namespace

extern "C" {

int64_t ref_compute_mertens(int64_t X, int threads) {
    return DelégliseRivatEngine::compute_mertens(X, threads);
}

int64_t ref_compute_compressed(int64_t X, int threads) {
    return DelégliseRivatEngine::compute_compressed(X, threads);
}

double ref_choose_cx(int64_t X) { return DelégliseRivatEngine::choose_cx(X); }
int64_t ref_choose_sieve_limit(int64_t X) { return DelégliseRivatEngine::choose_sieve_limit(X, 0); }
int64_t ref_choose_compressed_limit(int64_t X) { return DelégliseRivatEngine::choose_compressed_limit(X); }
int64_t ref_isqrt(int64_t n) { return isqrt(n); }

// ---- tables --------------------------------------------------------------

void* ref_table_new(int64_t u_total, int64_t u_dense, int64_t mu_limit, int threads) {
    return new CompressedMertensTable(u_total, u_dense, threads, mu_limit);
}

void ref_table_free(void* h) { delete static_cast<CompressedMertensTable*>(h); }

void ref_table_info(void* h, int64_t* out4) {
    auto* t = static_cast<CompressedMertensTable*>(h);
    out4[0] = t->u_total;
    out4[1] = t->u_dense;
    out4[2] = t->mu_limit;
    out4[3] = t->num_chunks;
}

// M(n) and mu(n) for n in [first, first+count) through get_M / get_mu.
void ref_table_get(void* h, int64_t first, int64_t count, int32_t* M, int8_t* mu) {
    auto* t = static_cast<CompressedMertensTable*>(h);
    for (int64_t i = 0; i < count; ++i) {
        if (M) M[i] = t->get_M(first + i);
        if (mu) mu[i] = t->get_mu(first + i);
    }
}

// Checksums over the raw members (layout of dr_oracle.h dro_table_sums).
void ref_table_checksums(void* h, uint64_t* out6) {
    auto* t = static_cast<CompressedMertensTable*>(h);
    std::memset(out6, 0, 6 * sizeof(uint64_t));
    for (size_t n = 0; n < t->dense_M.size(); ++n) {
        out6[0] += static_cast<uint64_t>(static_cast<int64_t>(t->dense_M[n]));
        out6[1] += static_cast<uint64_t>(static_cast<int64_t>(t->dense_M[n])) * (2 * n + 1);
    }
    for (size_t n = 0; n < t->mu.size(); ++n)
        out6[2] += static_cast<uint64_t>(static_cast<int64_t>(t->mu[n])) * (2 * n + 1);
    const int64_t words = (t->compressed_size + 63) / 64;
    for (int64_t w = 0; w < words; ++w) {
        const BitChunk& c = t->chunks[static_cast<size_t>(w >> 2)];
        uint64_t nz, neg;
        std::memcpy(&nz, c.nonzero + (w & 3) * 8, 8);
        std::memcpy(&neg, c.sign + (w & 3) * 8, 8);
        const uint64_t k = static_cast<uint64_t>(2 * w + 1);
        out6[3] += nz * k;
        out6[4] += neg * k;
        out6[5] += static_cast<uint64_t>(static_cast<int64_t>(t->checkpoints[static_cast<size_t>(w)])) * k;
    }
}

// Dense odd-sieve table (SieveTable, :376-457) for the dense path.
void* ref_sieve_new(int64_t u, int64_t mu_limit, int threads) {
    return new SieveTable(u, threads, mu_limit);
}
void ref_sieve_free(void* h) { delete static_cast<SieveTable*>(h); }
void ref_sieve_get(void* h, int64_t first, int64_t count, int32_t* M, int8_t* mu) {
    auto* t = static_cast<SieveTable*>(h);
    for (int64_t i = 0; i < count; ++i) {
        if (M) M[i] = t->get_M(first + i);
        if (mu) mu[i] = t->get_mu(first + i);
    }
}

// ---- S2 helpers over a caller-provided mu array ----------------------------

int64_t ref_s2_single(int64_t y, int64_t A, const int8_t* mu) { return eval_s2_single(y, A, mu); }
int64_t ref_s2_combined(int64_t y, int64_t A, int64_t B, const int8_t* mu) {
    return eval_s2_combined(y, A, B, mu);
}

// piece 1..8 -> Piece1..8, 9..12 -> SinglePiece1..4 (:470-482), over [first,last]
int64_t ref_s2_interval(int piece, int64_t first, int64_t last, int64_t y, const int8_t* mu) {
    const double dy = static_cast<double>(y);
    switch (piece) {
    case 1: return run_s2_fast<Piece1>(first, last, y, dy, mu);
    case 2: return run_s2_fast<Piece2>(first, last, y, dy, mu);
    case 3: return run_s2_fast<Piece3>(first, last, y, dy, mu);
    case 4: return run_s2_fast<Piece4>(first, last, y, dy, mu);
    case 5: return run_s2_fast<Piece5>(first, last, y, dy, mu);
    case 6: return run_s2_fast<Piece6>(first, last, y, dy, mu);
    case 7: return run_s2_fast<Piece7>(first, last, y, dy, mu);
    case 8: return run_s2_fast<Piece8>(first, last, y, dy, mu);
    case 9: return run_s2_fast<SinglePiece1>(first, last, y, dy, mu);
    case 10: return run_s2_fast<SinglePiece2>(first, last, y, dy, mu);
    case 11: return run_s2_fast<SinglePiece3>(first, last, y, dy, mu);
    case 12: return run_s2_fast<SinglePiece4>(first, last, y, dy, mu);
    }
    return 0;
}

int64_t ref_piece(int piece, int64_t q) {
    switch (piece) {
    case 1: return Piece1::eval(q);
    case 2: return Piece2::eval(q);
    case 3: return Piece3::eval(q);
    case 4: return Piece4::eval(q);
    case 5: return Piece5::eval(q);
    case 6: return Piece6::eval(q);
    case 7: return Piece7::eval(q);
    case 8: return Piece8::eval(q);
    case 9: return SinglePiece1::eval(q);
    case 10: return SinglePiece2::eval(q);
    case 11: return SinglePiece3::eval(q);
    case 12: return SinglePiece4::eval(q);
    }
    return 0;
}

void ref_finalize_bytes(uint8_t* values, int64_t len, int64_t first, int stride) {
    if (stride == 2) finalize_mobius_bytes<2>(values, len, first);
    else finalize_mobius_bytes<1>(values, len, first);
}

// ---- full walk with checksums ---------------------------------------------
// out: [0]=M, [1]=C, [2]=S1, [3]=S2 (uint64 bit patterns), [4]=terms
int ref_dr_checksums(int64_t X, int64_t u_total, int64_t u_dense, double cx, int64_t mu_limit,
                     int threads, int64_t* out) {
    std::memset(out, 0, 5 * sizeof(int64_t));
    if (X < 1) return 0;
    if (threads <= 0) threads = omp_get_max_threads();
    CompressedMertensTable table(u_total, u_dense, threads, mu_limit);
    if (X <= table.u_total) {
        out[0] = table.get_M(X);
        return 0;
    }
    const int64 N = X / table.u_total;
    const int64 n6 = N / 6, n3 = N / 3, n2 = N / 2;
    const int16_t* M_dense = table.dense_data();
    const int8_t* mu = table.mu.data();
    const int64 ut = table.u_total, ud = table.u_dense;

    auto single = [&](int64 y) {
        Sums s;
        const int64 A = split_point(cx, y);
        const int64 kappa = y / (A + 1);
        const int64 start = y / ut + 1;
        const int64 split = std::min(kappa, y / (ud + 1));
        int64 S1 = 0;
        for (int64 n = start; n <= split; ++n) S1 += table.reconstruct_compressed(y / n);
        const int64 n = std::max(start, split + 1);
        S1 += sum_dense_quotients<1>(y, n, kappa, M_dense);
        s.S1 = static_cast<uint64_t>(S1);
        s.S2 = static_cast<uint64_t>(eval_s2_single(y, A, mu));
        s.C = static_cast<uint64_t>(1 + kappa * static_cast<int64>(M_dense[A]));
        return s;
    };
    auto comb2 = [&](int64 y, int64 y2) {
        Sums s;
        const int64 A = split_point(cx, y), B = split_point(cx, y2);
        const int64 ky = y / (A + 1), ky2 = y2 / (B + 1), two = 2 * ky2;
        int64 start = y / ut + 1;
        if (start % 2 == 0) ++start;
        const int64 split = std::min(ky, y / (ud + 1));
        int64 S1 = 0, n = start;
        for (; n <= split; n += 2) S1 += table.reconstruct_compressed(y / n);
        S1 += sum_dense_quotients<2>(y, n, ky, M_dense);
        if (two > ky) {
            int64 e = ky + 1;
            if (e % 2) ++e;
            S1 -= sum_dense_quotients<2>(y, e, two, M_dense);
        } else if (two < ky) {
            int64 e = two + 1;
            if (e % 2) ++e;
            S1 += sum_dense_quotients<2>(y, e, ky, M_dense);
        }
        s.S1 = static_cast<uint64_t>(S1);
        s.S2 = static_cast<uint64_t>(eval_s2_combined(y, A, B, mu));
        s.C = static_cast<uint64_t>(ky * static_cast<int64>(M_dense[A]) - ky2 * static_cast<int64>(M_dense[B]));
        return s;
    };

    uint64_t C = 0, S1 = 0, S2 = 0;
    int64_t terms = 0;
#pragma omp parallel for schedule(dynamic, 8) num_threads(threads) reduction(+ : C, S1, S2, terms)
    for (int64 k = 1; k <= N; ++k) {
        if (k % 2 == 0 || k % 3 == 0) continue;
        const int8_t mk = table.get_mu(k);
        if (!mk) continue;
        const int64 y = X / k;
        Sums a, b;
        if (k <= n6) {
            a = comb2(y, y / 2);
            b = comb2(y / 3, y / 6);
        } else if (k <= n3) {
            a = comb2(y, y / 2);
            b = single(y / 3);
        } else if (k <= n2) {
            a = comb2(y, y / 2);
        } else {
            a = single(y);
        }
        const uint64_t m = static_cast<uint64_t>(static_cast<int64_t>(mk));
        C += m * (a.C - b.C);
        S1 += m * (a.S1 - b.S1);
        S2 += m * (a.S2 - b.S2);
        terms += 1;
    }
    out[0] = static_cast<int64_t>(C - S1 - S2);
    out[1] = static_cast<int64_t>(C);
    out[2] = static_cast<int64_t>(S1);
    out[3] = static_cast<int64_t>(S2);
    out[4] = terms;
    return 0;
}

}  // extern "C"
