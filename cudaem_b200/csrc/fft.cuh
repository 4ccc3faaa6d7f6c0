// FP32 complex FFT building blocks for the fused slice passes.
//
// An N-point transform is computed by a "team" of G threads, each holding
// E = N/G points in registers, as a two-level Cooley-Tukey factorisation
// N = E x G:
//   1. each thread g takes x[g + G j] (j < E) and runs an E-point DFT in
//      registers (radix-4 decimation in frequency, constant twiddles from
//      __constant__ memory, fully unrolled);
//   2. the E outputs are multiplied by the inter-level twiddles W_N^(g k1)
//      (a shared-memory table laid out [k1][g] so a team reads it without
//      bank conflicts);
//   3. one transpose through shared memory (padded rows) hands every thread
//      the G values of E/G columns k1, and a G-point register DFT finishes
//      each.
// The result is X[g + G j'] in thread g, i.e. the same distribution as the
// input, so an inverse transform, a pointwise multiply and a forward
// transform chain in registers with no data movement.  Forward transforms
// use exp(-2 pi i jk/N) and are unnormalised, like CUFFT_FORWARD.
#pragma once
#include <cuda_runtime.h>

#include "fft_layout.hpp"

namespace msb {

// W_64^m = exp(-2 pi i m / 64) as an unevaluated sum hi + lo of two floats: hi is the double
// value rounded to float, lo the rounded remainder.  The values are computed at compile time
// (tw64::cos_m / sin_m: the octant by an exact rotation, the remainder angle below pi/4 by its
// Taylor series in double), so every translation unit's copy of the table is initialised in its
// module image and nothing is uploaded at run time.
namespace tw64 {
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kRsqrt2 = 0.70710678118654752440084436210484903928;
// sin a and cos a for 0 <= a <= pi/4 (terms to a^41: truncation far below double rounding)
constexpr double sin_series(double a)
{
    double t = a, s = a;
    for (int k = 1; k <= 20; k++) {
        t *= -a * a / ((2.0 * k) * (2.0 * k + 1.0));
        s += t;
    }
    return s;
}
constexpr double cos_series(double a)
{
    double t = 1.0, s = 1.0;
    for (int k = 1; k <= 20; k++) {
        t *= -a * a / ((2.0 * k - 1.0) * (2.0 * k));
        s += t;
    }
    return s;
}
// cos and sin of 2 pi m / 64 = q pi/4 + r pi/32 with q = m / 8, r = m % 8
constexpr double cq_of(int q) { return q == 0 ? 1.0 : q == 1 ? kRsqrt2 : q == 2 ? 0.0 : q == 3 ? -kRsqrt2 : q == 4 ? -1.0 : q == 5 ? -kRsqrt2 : q == 6 ? 0.0 : kRsqrt2; }
constexpr double sq_of(int q) { return q == 0 ? 0.0 : q == 1 ? kRsqrt2 : q == 2 ? 1.0 : q == 3 ? kRsqrt2 : q == 4 ? 0.0 : q == 5 ? -kRsqrt2 : q == 6 ? -1.0 : -kRsqrt2; }
constexpr double cos_m(int m)
{
    const double a = kPi * (m % 8) / 32.0;
    return cq_of(m / 8) * cos_series(a) - sq_of(m / 8) * sin_series(a);
}
constexpr double sin_m(int m)
{
    const double a = kPi * (m % 8) / 32.0;
    return sq_of(m / 8) * cos_series(a) + cq_of(m / 8) * sin_series(a);
}
}  // namespace tw64

// entry m of the forward twiddle exp(-i 2 pi m / 64) = (cos, -sin)
#define MS_TW_HI(m) float2{(float)tw64::cos_m(m), (float)(-tw64::sin_m(m))}
#define MS_TW_LO(m) float2{(float)(tw64::cos_m(m) - (double)(float)tw64::cos_m(m)), \
                           (float)(-tw64::sin_m(m) - (double)(float)(-tw64::sin_m(m)))}
static __constant__ float2 c_tw64[64] = {
    MS_TW_HI(0), MS_TW_HI(1), MS_TW_HI(2), MS_TW_HI(3), MS_TW_HI(4), MS_TW_HI(5), MS_TW_HI(6), MS_TW_HI(7),
    MS_TW_HI(8), MS_TW_HI(9), MS_TW_HI(10), MS_TW_HI(11), MS_TW_HI(12), MS_TW_HI(13), MS_TW_HI(14), MS_TW_HI(15),
    MS_TW_HI(16), MS_TW_HI(17), MS_TW_HI(18), MS_TW_HI(19), MS_TW_HI(20), MS_TW_HI(21), MS_TW_HI(22), MS_TW_HI(23),
    MS_TW_HI(24), MS_TW_HI(25), MS_TW_HI(26), MS_TW_HI(27), MS_TW_HI(28), MS_TW_HI(29), MS_TW_HI(30), MS_TW_HI(31),
    MS_TW_HI(32), MS_TW_HI(33), MS_TW_HI(34), MS_TW_HI(35), MS_TW_HI(36), MS_TW_HI(37), MS_TW_HI(38), MS_TW_HI(39),
    MS_TW_HI(40), MS_TW_HI(41), MS_TW_HI(42), MS_TW_HI(43), MS_TW_HI(44), MS_TW_HI(45), MS_TW_HI(46), MS_TW_HI(47),
    MS_TW_HI(48), MS_TW_HI(49), MS_TW_HI(50), MS_TW_HI(51), MS_TW_HI(52), MS_TW_HI(53), MS_TW_HI(54), MS_TW_HI(55),
    MS_TW_HI(56), MS_TW_HI(57), MS_TW_HI(58), MS_TW_HI(59), MS_TW_HI(60), MS_TW_HI(61), MS_TW_HI(62), MS_TW_HI(63)
};
static __constant__ float2 c_tw64_lo[64] = {
    MS_TW_LO(0), MS_TW_LO(1), MS_TW_LO(2), MS_TW_LO(3), MS_TW_LO(4), MS_TW_LO(5), MS_TW_LO(6), MS_TW_LO(7),
    MS_TW_LO(8), MS_TW_LO(9), MS_TW_LO(10), MS_TW_LO(11), MS_TW_LO(12), MS_TW_LO(13), MS_TW_LO(14), MS_TW_LO(15),
    MS_TW_LO(16), MS_TW_LO(17), MS_TW_LO(18), MS_TW_LO(19), MS_TW_LO(20), MS_TW_LO(21), MS_TW_LO(22), MS_TW_LO(23),
    MS_TW_LO(24), MS_TW_LO(25), MS_TW_LO(26), MS_TW_LO(27), MS_TW_LO(28), MS_TW_LO(29), MS_TW_LO(30), MS_TW_LO(31),
    MS_TW_LO(32), MS_TW_LO(33), MS_TW_LO(34), MS_TW_LO(35), MS_TW_LO(36), MS_TW_LO(37), MS_TW_LO(38), MS_TW_LO(39),
    MS_TW_LO(40), MS_TW_LO(41), MS_TW_LO(42), MS_TW_LO(43), MS_TW_LO(44), MS_TW_LO(45), MS_TW_LO(46), MS_TW_LO(47),
    MS_TW_LO(48), MS_TW_LO(49), MS_TW_LO(50), MS_TW_LO(51), MS_TW_LO(52), MS_TW_LO(53), MS_TW_LO(54), MS_TW_LO(55),
    MS_TW_LO(56), MS_TW_LO(57), MS_TW_LO(58), MS_TW_LO(59), MS_TW_LO(60), MS_TW_LO(61), MS_TW_LO(62), MS_TW_LO(63)
};
#undef MS_TW_HI
#undef MS_TW_LO

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b)
{
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// Twiddle multiply d * (hi + lo) with the twiddle carried to about 48 bits.  Rounding a
// twiddle to one float is a fixed error of the transform operator; applied the same way at
// every slice of a crystal it adds up coherently (about 6e-5 relative after 240 slices at
// 1024^2, against 5e-6 with the split).  The low part enters through an FMA chain:
// re = vx hx - vy hy + (vx lx - vy ly), im = vx hy + vy hx + (vx ly + vy lx).
__device__ __forceinline__ float2 cmul_split(float2 d, float2 hi, float2 lo)
{
    const float cre = fmaf(d.x, lo.x, -(d.y * lo.y));
    const float cim = fmaf(d.x, lo.y, d.y * lo.x);
    return make_float2(fmaf(d.x, hi.x, fmaf(-d.y, hi.y, cre)), fmaf(d.x, hi.y, fmaf(d.y, hi.x, cim)));
}
__device__ __forceinline__ float2 cmulc_split(float2 d, float2 hi, float2 lo)
{
    return cmul_split(d, make_float2(hi.x, -hi.y), make_float2(lo.x, -lo.y));
}

// Multiply by W_64^m (DIR < 0) or its conjugate (DIR > 0); m is a compile-time
// constant once the callers are unrolled.
template <int DIR>
__device__ __forceinline__ float2 tw_apply(float2 d, int m)
{
    if (m == 0) return d;
    if (m == 16) return DIR < 0 ? make_float2(d.y, -d.x) : make_float2(-d.y, d.x);
    if (m == 8 || m == 24) {
        // W_64^8 = (1 - i)/sqrt2 and W_64^24 = (-1 - i)/sqrt2 (their conjugates for DIR > 0): a sum
        // and a difference of the two parts, each scaled by 1/sqrt2 carried as hi + lo
        const float hs = c_tw64[8].x, ls = c_tw64_lo[8].x;
        float re, im;
        if (DIR < 0) {
            re = (m == 8) ? d.x + d.y : d.y - d.x;
            im = (m == 8) ? d.y - d.x : -(d.x + d.y);
        } else {
            re = (m == 8) ? d.x - d.y : -(d.x + d.y);
            im = (m == 8) ? d.x + d.y : d.x - d.y;
        }
        return make_float2(fmaf(re, hs, re * ls), fmaf(im, hs, im * ls));
    }
    return DIR < 0 ? cmul_split(d, c_tw64[m], c_tw64_lo[m]) : cmulc_split(d, c_tw64[m], c_tw64_lo[m]);
}

template <int E>
__host__ __device__ constexpr int brev(int k)
{
    int r = 0;
    for (int b = 1; b < E; b <<= 1) {
        r = (r << 1) | (k & 1);
        k >>= 1;
    }
    return r;
}

// multiply by -i (DIR < 0) or +i (DIR > 0)
template <int DIR>
__device__ __forceinline__ float2 mul_mi(float2 d)
{
    return DIR < 0 ? make_float2(d.y, -d.x) : make_float2(-d.y, d.x);
}

// In-register E-point DFT, E a power of two <= 64, by radix-4 decimation in frequency (a final
// radix-2 stage when log2 E is odd).  A radix-4 step is two radix-2 stages with their twiddles
// combined (W^(j+len/4) = -i W^j and W^j W^2j = W^3j), so it needs three twiddle products per four points
// instead of four, and most of its twiddles are trivial or eighth-turn.  Output in bit-reversed
// order, as the radix-2 form: after the call a[brev<E>(k)] holds X[k].
template <int E, int DIR>
__device__ __forceinline__ void dft_reg(float2 (&a)[E])
{
    // radix-4 steps, each equal to two radix-2 decimation-in-frequency stages (same output order):
    // x0..x3 at j, j+q, j+2q, j+3q become (x0+x2)+(x1+x3), ((x0+x2)-(x1+x3)) W^2j,
    // ((x0-x2) -+ i (x1-x3)) W^j, ((x0-x2) +- i (x1-x3)) W^3j with W = W_len (forward: -i first)
#pragma unroll
    for (int len = E; len >= 4; len >>= 2) {
        const int q = len >> 2;
#pragma unroll
        for (int base = 0; base < E; base += len) {
#pragma unroll
            for (int j = 0; j < q; j++) {
                const float2 x0 = a[base + j], x1 = a[base + j + q], x2 = a[base + j + 2 * q], x3 = a[base + j + 3 * q];
                const float2 t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = mul_mi<DIR>(csub(x1, x3));
                const int m = j * (64 / len);
                a[base + j] = cadd(t0, t2);
                a[base + j + q] = tw_apply<DIR>(csub(t0, t2), (2 * m) & 63);
                a[base + j + 2 * q] = tw_apply<DIR>(cadd(t1, t3), m);
                a[base + j + 3 * q] = tw_apply<DIR>(csub(t1, t3), (3 * m) & 63);
            }
        }
    }
    // a remaining radix-2 stage when log2(E) is odd
    constexpr int LOG = (E >= 64) ? 6 : (E >= 32) ? 5 : (E >= 16) ? 4 : (E >= 8) ? 3 : (E >= 4) ? 2 : 1;
    if constexpr (LOG % 2 == 1) {
#pragma unroll
        for (int base = 0; base < E; base += 2) {
            const float2 u = a[base], v = a[base + 1];
            a[base] = cadd(u, v);
            a[base + 1] = csub(u, v);
        }
    }
}

// Team transform.  On entry v[j] = x[g + G j]; on exit v[j] = X[g + G j].
// `tw` is the shared table W_N^(g k1) at tw[k1 * G + g] (one of the dithered sets: the
// engine's slices take the sets in turn, see kTwSets).  `scr(k1, g)` returns
// the shared-memory slot for the transpose; `sync()` orders the team's shared
// accesses (a warp barrier when the team is inside one warp, a block barrier
// otherwise).
template <int N, int G, int DIR, class Scr, class Sync>
__device__ __forceinline__ void team_fft(float2 (&v)[N / G], int g, const float2* __restrict__ tw, Scr scr,
                                         Sync sync)
{
    constexpr int E = N / G;
    static_assert(E >= G && E % G == 0, "team layout needs E >= G");
    dft_reg<E, DIR>(v);
#pragma unroll
    for (int k1 = 1; k1 < E; k1++) {
        const float2 w = tw[k1 * G + g];
        v[brev<E>(k1)] = DIR < 0 ? cmul(v[brev<E>(k1)], w) : cmulc(v[brev<E>(k1)], w);
    }
    sync();
#pragma unroll
    for (int k1 = 0; k1 < E; k1++) *scr(k1, g) = v[brev<E>(k1)];
    sync();
    constexpr int M = E / G;
#pragma unroll
    for (int m = 0; m < M; m++) {
        float2 u[G];
#pragma unroll
        for (int q = 0; q < G; q++) u[q] = *scr(g + G * m, q);
        dft_reg<G, DIR>(u);
#pragma unroll
        for (int k2 = 0; k2 < G; k2++) v[m + M * k2] = u[brev<G>(k2)];
    }
}

}  // namespace msb
