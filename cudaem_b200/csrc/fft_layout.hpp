// Per-size thread layout of the FFT passes (shared by host and device code).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace msb {

// Per-size layout of the passes.
//   G: threads per transform; E = N/G points per thread.
//   ROWS: transforms per block in the row pass (one team each, inside a warp).
//   TC: columns per block in the column pass (teams span warps).
template <int N>
struct FftCfg;
template <>
struct FftCfg<128> {
    static constexpr int G = 8, ROWS = 16, TC = 16;
};
template <>
struct FftCfg<256> {
    static constexpr int G = 16, ROWS = 16, TC = 16;
};
template <>
struct FftCfg<512> {
    static constexpr int G = 16, ROWS = 16, TC = 16;
};
template <>
struct FftCfg<1024> {
    static constexpr int G = 32, ROWS = 8, TC = 8;
};
template <>
struct FftCfg<2048> {
    static constexpr int G = 32, ROWS = 4, TC = 8;
};

template <int N>
struct FftLayout {
    static constexpr int G = FftCfg<N>::G;
    static constexpr int E = N / G;
    static constexpr int ROWS = FftCfg<N>::ROWS;
    static constexpr int TC = FftCfg<N>::TC;
    static constexpr int ROW_THREADS = ROWS * G;
    static constexpr int COL_THREADS = TC * G;
    static constexpr int COL_MINB = (N == 2048) ? 1 : 2;   // resident column blocks per SM (register cap)
    static constexpr bool COL_TW_GLOBAL = false;            // twiddles staged in shared memory
    static constexpr int ROW_MINB = (N == 2048) ? 1 : 2;   // resident row blocks per SM (register cap)
    // transpose scratch of one transform: E rows of G+1 slots, plus padding so that
    // consecutive transforms start on banks that keep a half-warp conflict-free
    static constexpr int SCR_BASE = E * (G + 1);
    static constexpr int SCR_STRIDE_ROW = SCR_BASE + 1;
    static constexpr int SCR_STRIDE_COL =
        (TC == 16) ? (SCR_BASE + ((1 - SCR_BASE % 16) + 16) % 16) : (SCR_BASE + ((2 - SCR_BASE % 16) + 16) % 16);
    // transpose scratch, twiddles (high and low parts), and the 1024-entry exp(i phi) table
    static constexpr size_t ROW_SMEM = sizeof(float2) * ((size_t)ROWS * SCR_STRIDE_ROW + 2 * N + 1024);
    static constexpr size_t COL_SMEM = sizeof(float2) * ((size_t)TC * SCR_STRIDE_COL + (COL_TW_GLOBAL ? 0 : 2 * N));
};

}  // namespace msb
