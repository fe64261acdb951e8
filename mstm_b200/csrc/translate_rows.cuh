// translate_rows.cuh -- the FP32 pair translation pass of monodisperse
// clusters with operator rows broadcast from shared memory, and the FP32
// "row" operator record it streams.
#pragma once
#include "translate_tiled.cuh"

// Row record of one pair (floats), every row 16-byte aligned so a lane reads
// it four floats at a time, and laid out so that consecutive floats pair up
// as the operands of the packed FP32x2 FMA:
//   [0, rr_hdr(L))         e^{i m phi}, m = 0..L (complex), 0-padded
//   rotation, degree n = 1..L: rows k = 0..n of rr_rw(n) floats,
//       [E_n(k,0), 0, E_n(k,1), O_n(k,1), ..., E_n(k,n), O_n(k,n), 0...]
//       (O_n(0, .) = 0)
//   axial, m = 0: rows n = 1..L of rr_zw0(L) floats, Z_0(n, l) complex for l = 1..L (0-padded)
//   axial, m = 1..L: rows n = m..L of 4 rr_zq(L - m + 1) floats,
//       [Z_m^0(n, l), Z_m^1(n, l)] for l = m..L (the two modes' blocks interleaved, 0-padded)
//   (the axial rows hold an even number of 16-byte units, so that two lanes
//   split every row without a bounds test)
//   padding to row_record_units(L) = 4 (mod 32) floats, so that the records of
//   consecutive pairs fall on different shared-memory banks.
__host__ __device__ constexpr int rr_hdr(int L) { return (2 * (L + 1) + 3) & ~3; }
__host__ __device__ constexpr int rr_rw(int n) { return (2 * n + 2 + 3) & ~3; }
__host__ __device__ constexpr int rr_rot_off(int n, int L)
{
    int s = rr_hdr(L);
    for (int q = 1; q < n; q++) s += (q + 1) * rr_rw(q);
    return s;
}
__host__ __device__ constexpr int rr_zq(int dim) { return (dim + 1) & ~1; }   // 16-byte units of an m > 0 row
__host__ __device__ constexpr int rr_zw0(int L) { return 4 * rr_zq((L + 1) / 2); }   // floats of an m = 0 row
__host__ __device__ constexpr int rr_z_off(int m, int L)
{
    int s = rr_rot_off(L + 1, L);
    if (m > 0) s += L * rr_zw0(L);
    for (int q = 1; q < m; q++) s += 4 * (L - q + 1) * rr_zq(L - q + 1);
    return s;
}
__host__ __device__ constexpr int row_record_units(int L)
{
    const int u = rr_z_off(L + 1, L);
    return u + (((4 - u) % 32) + 32) % 32;
}

// The row pass covers every FP32 pass of the tiled path: L = 3..10 and
// 1, 2 or 4 columns per chunk.
bool rows_supported(int L, int nrhs);
int launch_translate_rows(const TiledArgs<float>& a, int L, int nsm, cudaStream_t st);
