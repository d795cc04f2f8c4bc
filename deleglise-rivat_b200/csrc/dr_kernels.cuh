// dr_kernels.cuh -- kernel argument blocks and launch wrappers (host side).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dr_device.cuh"

namespace drb {

constexpr int kStencilPeriod = 13860;                       // lcm(4, 9, 5, 7, 11)
constexpr int kStencilWords = (kStencilPeriod + 3 + 3) / 4;  // words per shifted copy

struct SieveArgs {
    i64 u_total, u_dense, mu_limit;
    i64 dense_segs, nseg;
    int S;              // values per segment (multiple of 4096)
    int n_primes;       // primes <= isqrt(u_total), ascending
    int sq_first;       // first prime >= 5 (square flags)
    int w_first;        // first prime >= 13 (weights)
    int tierB_first;    // first prime sieved thread-per-prime
    const uint32_t* primes;
    const uint32_t* stencil4;  // 4 copies shifted by 0..3 bytes, kStencilWords each
    int16_t* dM;
    ulonglong2* planes;
    int32_t* ckpt;
    uint4* wheel;
    int32_t* seg_sum;
};

struct SumsArgs {
    const QueryDev* queries;
    int nq;
    TableView T;
    u64 n_slots;
    const u64* prefix;  // [n_slots + 1] exclusive op prefix
    u64* ticket;        // [0]: work-queue counter, [1]: error flag; zeroed before launch
    u64* acc;           // [3 * nq]: C, S1, S2
    int chunk_log2;     // 0: chosen on the device from the total
};

void launch_sieve(const SieveArgs& a, int grid, int block, size_t smem, cudaStream_t s);
size_t sieve_smem_bytes(int S);
void launch_seg_scan(const int32_t* in, int32_t* out, i64 n, cudaStream_t s);
void launch_fixup(int16_t* dM, i64 u_dense, int S, const int32_t* seg_off, int32_t* ckpt, i64 nwords,
                  i64 dense_segs, int sm_count, cudaStream_t s);
void launch_plan(const QueryDev* q, int nq, const TableView& T, u64 n_slots, u64* ops, u64* acc,
                 i64* counts, int sm_count, cudaStream_t s);
void launch_scan_u64(const u64* in, u64* out, u64 n, u64* tmp, size_t tmp_elems, cudaStream_t s);
size_t scan_u64_tmp_elems(u64 n);
void launch_sums(const SumsArgs& a, int grid, int block, cudaStream_t s);
void launch_direct(const QueryDev* q, int nq, const TableView& T, u64* acc, cudaStream_t s);
void launch_table_read(const TableView& T, i64 first, i64 count, int32_t* M, int8_t* mu, int8_t* wheel_mu,
                       cudaStream_t s);
void launch_table_sums(const TableView& T, i64 nwords, u64* out6, int sm_count, cudaStream_t s);
void init_piece_constants();
// Record a message for dr_last_error() (fixed thread-local buffer) and return code.
int record_error(int code, const char* msg);
// Opt the sieve kernel into `smem` bytes of dynamic shared memory and report
// how many CTAs of `block` threads fit on one SM.
void sieve_kernel_attrs(size_t smem, int block, int* per_sm);
void sums_kernel_occupancy(int block, int* per_sm);
void launch_debug_udiv(const u64* y, const u64* d, u64* q, i64 n, cudaStream_t s);
void launch_debug_piece(const int32_t* piece, const u64* q, i64* out, i64 n, cudaStream_t s);

}  // namespace drb
