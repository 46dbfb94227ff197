// Operand layout of the CH4-CO2 tensor-core dipole kernel (hh_ch4co2_tc.cuh), shared
// by the kernel and by the host code that builds the coefficient images
// (hh_ch4co2_host.cpp).
#pragma once
#include <stddef.h>

#ifdef __CUDACC__
#define HH_TC_HD __host__ __device__
#else
#define HH_TC_HD
#endif

namespace hh {

constexpr int CH4TC_M = 128;                      // records per task (= MMA M, TMEM lanes)
constexpr int CH4TC_NY1 = 196;                    // Y1 functions (columns used per component)
constexpr int CH4TC_N = 208;                      // columns per component accumulator (N % 16 == 0)
constexpr int CH4TC_K = 368;                      // 4 powers x 91 Y2 = 364, padded to a multiple of 16
constexpr int CH4TC_KC = 16;                      // K per chunk (two MMAs of K = 8)
constexpr int CH4TC_NCHUNK = CH4TC_K / CH4TC_KC;  // 23
// B image bytes per chunk (rows x KC x 4 B), hi and lo each
constexpr int CH4TC_IMG0 = 2 * CH4TC_N * CH4TC_KC * 4;  // pass 0 (components 0, 1): 26,624
constexpr int CH4TC_IMG1 = CH4TC_N * CH4TC_KC * 4;      // pass 1 (component 2): 13,312
constexpr size_t CH4TC_PIECE_BYTES = (size_t)CH4TC_NCHUNK * 2 * (CH4TC_IMG0 + CH4TC_IMG1);

// float offset of element (row, kk) of a K-chunk image, kk < 16: the core matrix
// (row / 8, kk / 4) of 8 rows x 16 bytes sits at (row / 8) * 512 B + (kk / 4) * 128 B,
// its rows 16 B apart (no-swizzle K-major canonical layout: LBO 128 B, SBO 512 B)
HH_TC_HD constexpr int ch4tc_img_off(int row, int kk) {
  return (row >> 3) * 128 + (kk >> 2) * 32 + (row & 7) * 4 + (kk & 3);
}

// K order of the A and B images: column group i (columns 4 i .. 4 i + 3 of a chunk,
// the powers x^0..x^3) of chunk c holds Y2 index CH4TC_QLEN i + c, so the four quarters
// of the Y2 sequence sit side by side and a thread that writes group i walks only its
// quarter, one value per chunk; -1 past the sequence's end (a zero group)
constexpr int CH4TC_QLEN = 23;  // Y2 values per quarter: 23 x 4 >= 91, and 23 chunks
HH_TC_HD constexpr int ch4tc_k_of(int c, int i) {
  return (c < CH4TC_QLEN && CH4TC_QLEN * i + c < 91) ? CH4TC_QLEN * i + c : -1;
}

// byte offset of the (hi, lo) image pair of piece p, pass q, chunk c in the blob
HH_TC_HD constexpr size_t ch4tc_blob_off(int p, int q, int c) {
  return (size_t)p * CH4TC_PIECE_BYTES + (q == 0 ? (size_t)c * 2 * CH4TC_IMG0
                                                 : (size_t)CH4TC_NCHUNK * 2 * CH4TC_IMG0 + (size_t)c * 2 * CH4TC_IMG1);
}

// column of Y1 (l1, m1, cos = 0 / sin = 1) in an accumulator: m-major, l = m..13,
// cos then sin (sin only for m > 0)
HH_TC_HD constexpr int ch4tc_y1_col(int l1, int m1, int cs, int l1max) {
  int c = 0;
  for (int m = 0; m < m1; ++m) c += (m == 0 ? 1 : 2) * (l1max + 1 - m);
  return c + (m1 == 0 ? l1 : 2 * (l1 - m1) + cs);
}

}  // namespace hh
