// Per-size thread layout of the FFT passes (shared by host and device code).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace msb {

// Dithered tables of the operators that every slice repeats.  The inter-level FFT twiddles
// (kTwSets sets) and the propagator P(k) (kPropSets tables) are each rounded to float in several
// versions, and slice s uses version s mod K.  The versions follow sigma-delta rounding: version t
// is the float nearest to (t + 1) w minus the sum of versions 0..t-1, so the running sum over
// consecutive slices stays within half an ulp of the exact multiple of w.  A single rounded table
// would repeat the same rounding error at every slice; its effect on the wave adds up coherently
// over a thick specimen (at 240 slices the propagator's rounding alone costs about 5e-6 relative).
constexpr int kTwSets = 8;
constexpr int kPropSets = 8;

#ifdef __CUDACC__
#define MS_FL_HD __host__ __device__
#else
#define MS_FL_HD
#endif
// Versions t = 0..K-1 of the complex value (re, im), written to out[t * stride].
template <class F2>
MS_FL_HD inline void dither_sets(double re, double im, int K, F2* out, size_t stride)
{
    double sr = 0.0, si = 0.0;
    for (int t = 0; t < K; t++) {
        const float vr = (float)((t + 1) * re - sr), vi = (float)((t + 1) * im - si);
        sr += (double)vr;
        si += (double)vi;
        out[(size_t)t * stride].x = vr;
        out[(size_t)t * stride].y = vi;
    }
}

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

// Narrow tiles for batches too small to fill the GPU (one 512^2 HRTEM wave has 32 wide row
// blocks for 148 SMs): one warp of rows per row block, four columns per column block (32-byte
// row segments, one sector each; two columns, the narrowest 16-byte tensor-map box, measured
// slower).  The twiddles are then read from global memory (L1) instead of being staged per block.
template <int N>
struct NarrowCfg {
    static constexpr int G = FftCfg<N>::G;
    static constexpr int ROWS = G >= 32 ? 1 : 32 / G;
    static constexpr int TC = N < 256 ? 32 / G : 4;
};

template <int N, int ROWS_ = FftCfg<N>::ROWS, int TC_ = FftCfg<N>::TC>
struct FftLayoutT {
    static constexpr int G = FftCfg<N>::G;
    static constexpr int E = N / G;
    static constexpr int ROWS = ROWS_;
    static constexpr int TC = TC_;
    static constexpr int ROW_THREADS = ROWS * G;
    static constexpr int COL_THREADS = TC * G;
    static constexpr bool NARROW = ROWS_ != FftCfg<N>::ROWS || TC_ != FftCfg<N>::TC;
    // resident blocks per SM that the register cap allows (__launch_bounds__)
    static constexpr int COL_MINB = NARROW ? (N == 2048 ? 2 : 4) : ((N == 2048) ? 1 : 2);
    static constexpr bool COL_TW_GLOBAL = false;            // twiddles staged in shared memory
    static constexpr int ROW_MINB = NARROW ? (N == 2048 ? 4 : 8) : ((N == 2048) ? 1 : 2);
    // transpose scratch of one transform: E rows of G+1 slots, plus padding so that
    // consecutive transforms start on banks that keep a half-warp conflict-free
    static constexpr int SCR_BASE = E * (G + 1);
    static constexpr int SCR_STRIDE_ROW = SCR_BASE + 1;
    static constexpr int SCR_STRIDE_COL =
        (TC == 16) ? (SCR_BASE + ((1 - SCR_BASE % 16) + 16) % 16) : (SCR_BASE + ((2 - SCR_BASE % 16) + 16) % 16);
    // transpose scratch, one set of twiddles, and the 1024-entry exp(i phi) table
    static constexpr size_t ROW_SMEM = sizeof(float2) * ((size_t)ROWS * SCR_STRIDE_ROW + N + 1024);
    static constexpr size_t COL_SMEM = sizeof(float2) * ((size_t)TC * SCR_STRIDE_COL + (COL_TW_GLOBAL ? 0 : N));
};
template <int N>
using FftLayout = FftLayoutT<N>;
template <int N>
using NarrowLayout = FftLayoutT<N, NarrowCfg<N>::ROWS, NarrowCfg<N>::TC>;

// Tile shape of the hot slice passes (PassArgs.tile): a narrow row step and a narrow column step
// are chosen independently; TILE_WARP_COLS (1024-point columns) takes one warp per column
enum TileShape { TILE_WIDE = 0, TILE_NARROW_ROWS = 1, TILE_NARROW_COLS = 2, TILE_NARROW = 3, TILE_WARP_COLS = 4 };

}  // namespace msb
