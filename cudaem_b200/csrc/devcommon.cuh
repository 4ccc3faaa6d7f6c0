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
// A 2-D tensor map over a wave batch seen as rows x (2 nx) floats (rows = waves x ny), with boxes of
// box_cols floats x box_rows rows; false when the driver cannot encode it.
bool encode_wave_tile_map(void* map, const void* psi, int nx, int64_t rows, int box_cols, int box_rows,
                          bool swizzle64 = false);

// ---------------------------------------------------------------------------
// L2 eviction policies for the slice passes (createpolicy over the whole access) and loads /
// stores that carry them
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t l2_policy_evict_last()
{
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first()
{
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_normal()
{
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// read-only data of the whole launch (tables, the transmission store)
__device__ __forceinline__ float2 ld_nc_l2hint(const float2* ptr, uint64_t pol)
{
    float2 v;
    asm("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(ptr), "l"(pol));
    return v;
}
// the wave (written by the previous pass)
__device__ __forceinline__ float2 ld_l2hint(const float2* ptr, uint64_t pol)
{
    float2 v;
    asm volatile("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(ptr), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_l2hint(float2* ptr, float2 v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(ptr), "f"(v.x), "f"(v.y), "l"(pol)
                 : "memory");
}
// Policy of the wave batch's stores and of the transmission loads of one pass (PassArgs.l2_mode):
// L2_WAVES_RESIDENT keeps the batch's waves in L2 between the passes and streams the transmission;
// L2_SHARED_T keeps the transmission (read by every wave of the batch) and streams the waves.
__device__ __forceinline__ uint64_t l2_policy_wave(int mode)
{
    return mode == L2_WAVES_RESIDENT ? l2_policy_evict_last()
                                     : (mode == L2_SHARED_T ? l2_policy_evict_first() : l2_policy_evict_normal());
}
__device__ __forceinline__ uint64_t l2_policy_trans(int mode)
{
    return mode == L2_WAVES_RESIDENT ? l2_policy_evict_first()
                                     : (mode == L2_SHARED_T ? l2_policy_evict_last() : l2_policy_evict_normal());
}

// ---------------------------------------------------------------------------
// Tensor-memory-access (TMA) tile loads into shared memory, completed on an mbarrier
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// Waits for phase `phase` of the barrier for at most `limit` clock cycles; false when the wait ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned phase, long long limit)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, phase))
        if (clock64() - t0 > limit) return false;
    return true;
}
// One 2-D box of the tensor map into shared memory at dst (128-byte aligned); x is the inner
// coordinate in elements (its byte offset a multiple of 16), y the row.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* map, int x, int y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
// One 2-D box from shared memory at src (aligned as the map's swizzle needs) to the tensor map's
// (x, y), in the thread's bulk async-group; the caller commits the group and waits for it before
// the shared memory is reused or the block exits.
__device__ __forceinline__ void tma_store_2d(const void* map, int x, int y, const void* src)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
                 ::"l"(map), "r"(x), "r"(y), "r"(smem_u32(src))
                 : "memory");
}
// the same with an L2 eviction priority (createpolicy) for the written lines
__device__ __forceinline__ void tma_store_2d_hint(const void* map, int x, int y, const void* src, uint64_t pol)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group.L2::cache_hint [%0, {%1, %2}], [%3], %4;"
                 ::"l"(map), "r"(x), "r"(y), "r"(smem_u32(src)), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void tma_store_commit_and_wait()
{
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
// default limit of a device-side wait: about one second at the B200's clock
constexpr long long kWaitCycles = 2000000000LL;

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
