// Device helpers and launch bookkeeping shared by the kernel translation units (kernels.cu and
// the per-size pass files passes_<N>.cu).
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "kernels.cuh"

namespace msb {

// one more launch of this library's kernels (ms_last_launch_count)
void count_launch();
// a launch error of the kernel just launched becomes an MsError naming `what`
void check_launch(const char* what);
// raises a kernel's dynamic shared-memory limit to `bytes` when a launch needs more than the limit
// already set on this device
void smem_attr_raw(const void* kernel, size_t bytes);
template <class F>
inline void smem_attr(F* kernel, size_t bytes)
{
    smem_attr_raw((const void*)kernel, bytes);
}
int num_sms();

// ---------------------------------------------------------------------------
// lens phase (coherent_phase_shift, basic_functions_dev.cuh:215-234) in FP64
// ---------------------------------------------------------------------------
__device__ __forceinline__ double chi_d(const LensDev& L, double cc10, double gx, double gy)
{
    double g2 = gx * gx + gy * gy, g4 = g2 * g2, g6 = g4 * g2;
    double chi = cc10 * g2 + L.cc30 * g4 + L.cc50 * g6;
    if (L.phi_req) {
        double g = sqrt(g2), g3 = g2 * g, g5 = g4 * g;
        double ph = atan2(gy, gx);
        if (fabs(ph) > 1e-5) chi += L.m * ph;
        chi += L.cc12 * g2 * sin(2 * (ph - L.p12));
        chi += L.cc21 * g3 * sin(ph - L.p21) + L.cc23 * g3 * sin(3 * (ph - L.p23));
        chi += L.cc32 * g4 * sin(2 * (ph - L.p32)) + L.cc34 * g4 * sin(4 * (ph - L.p34));
        chi += L.cc41 * g5 * sin(ph - L.p41) + L.cc43 * g5 * sin(3 * (ph - L.p43)) + L.cc45 * g5 * sin(5 * (ph - L.p45));
        chi += L.cc52 * g6 * sin(2 * (ph - L.p52)) + L.cc54 * g6 * sin(4 * (ph - L.p54)) + L.cc56 * g6 * sin(6 * (ph - L.p56));
    }
    return chi;
}

// exp(i ph) for a phase formed in FP64: reduced modulo 2 pi in FP64, then FP32 sincos.
__device__ __forceinline__ float2 expi_d(double ph)
{
    const double two_pi = 6.283185307179586476925286766559;
    double r = ph - two_pi * rint(ph * (1.0 / two_pi));
    float s, c;
    sincosf((float)r, &s, &c);
    return make_float2(c, s);
}

__device__ __forceinline__ double freq_d(int i, int n, double dg) { return (double)((i < n / 2) ? i : i - n) * dg; }

// exp(i phi) for the transmission: phi = k h + d with h = 2 pi / 1024 (Cody-Waite split, exact
// product for |k| < 4096), exp(i k h) from a table rounded from FP64, and exp(i d) for
// |d| <= pi/1024 from its Taylor series to d^4 / d^5 (truncation below 3e-15).  The result
// carries about one ulp of error, like sincosf, at a third of its instructions.
constexpr int kExpTab = 1024;
__device__ __forceinline__ float2 expi_tab(float phi, const float2* __restrict__ tab)
{
    const float kf = rintf(phi * 162.97466172610083f);
    float d = fmaf(-kf, 0.006134033203125f, phi);
    d = fmaf(-kf, 1.8899484075518558e-06f, d);
    const float2 T = tab[(int)kf & (kExpTab - 1)];
    const float d2 = d * d;
    const float c = fmaf(d2, fmaf(d2, 0.041666666666666664f, -0.5f), 1.0f);
    const float s = d * fmaf(d2, -0.16666666666666666f, 1.0f);
    return make_float2(T.x * c - T.y * s, T.x * s + T.y * c);
}

// Hides a pointer's provenance from the optimiser (no instruction is emitted).
template <class T>
__device__ __forceinline__ T* opaque(T* p)
{
    asm volatile("" : "+l"(p));
    return p;
}

template <int E>
__device__ __forceinline__ void conj_all(float2 (&v)[E])
{
#pragma unroll
    for (int j = 0; j < E; j++) v[j].y = -v[j].y;
}

// ---------------------------------------------------------------------------
// row pass

}  // namespace msb
