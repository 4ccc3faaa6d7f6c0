// The fused slice passes: row and column FFT kernels with the per-slice operators folded in.
//
// Per slice the wave batch makes two passes through memory:
//   row pass    : inverse row FFT -> transmission t_s = exp(i sigma V_s) -> forward row FFT
//   column pass : forward column FFT -> Fresnel propagator P(k) -> inverse column FFT
// which together equal the reference's transmit (forward cuFFT with the
// exp(iV) load callback, transmission_function.cuh:107-119) and propagate
// (inverse cuFFT with the P load callback, propagation_function.cuh:41-48).
// The probe is generated inside the first column pass and the CTF inside the
// HRTEM column pass.  Every transform length is compiled in its own translation
// unit (passes_<N>.cu), which instantiates row_dispatch<N> and col_dispatch<N>.
#pragma once
#include <cuda.h>

#include <algorithm>
#include <cstdint>

#include "detmath.cuh"
#include "devcommon.cuh"
#include "fft.cuh"
#include "kernels.cuh"

namespace msb {

// The twiddle set of this launch's slice (kTwSets dithered sets of N entries at a.tw).
template <int N>
__device__ __forceinline__ const float2* tw_set(const PassArgs& a)
{
    return a.tw + (size_t)((unsigned)a.slice % (unsigned)kTwSets) * N;
}
// The propagator table of this launch's slice: kPropSets dithered tables of nx*ny entries.
__device__ __forceinline__ const float2* prop_set(const float2* base, const PassArgs& a)
{
    return base + (size_t)((unsigned)a.slice % (unsigned)kPropSets) * ((size_t)a.grid.nx * a.grid.ny);
}

// ---------------------------------------------------------------------------
template <int N, int OP>
__global__ void __launch_bounds__(FftLayout<N>::ROW_THREADS, FftLayout<N>::ROW_MINB) k_row(PassArgs a)
{
    using L = FftLayout<N>;
    constexpr int G = L::G, E = L::E;
    extern __shared__ float2 smem[];
    const int ny = a.grid.ny;
    const int blocks_per_wave = ny / L::ROWS;
    const int b = blockIdx.x / blocks_per_wave;
    const int team = threadIdx.x / G, g = threadIdx.x % G;
    const int r = (blockIdx.x % blocks_per_wave) * L::ROWS + team;
    const WaveInfo wi = a.waves[b];
    const bool beyond = a.slice >= wi.n_slices;
    constexpr bool kT = OP == ROW_T_FWD || OP == ROW_INV_T_FWD || OP == ROW_INV_T_FWD_X || OP == ROW_INV_TT_FWD ||
                        OP == ROW_TT_FWD;
    constexpr bool kTT = OP == ROW_INV_TT_FWD || OP == ROW_TT_FWD;
    if (kT && beyond && !(a.flags & PF_VACUUM_BEYOND)) return;

    const size_t row_off = ((size_t)b * ny + r) * N;
    float2 v[E];
    // the wave's loads go out first, so their latency overlaps the table staging below
    if (OP == ROW_INV_T_FWD || OP == ROW_INV_T_FWD_X || OP == ROW_INV_TT_FWD || OP == ROW_ADJ) {
#pragma unroll
        for (int j = 0; j < E; j++) v[j] = a.psi[row_off + g + G * j];
    }
    float2* tw = smem + L::ROWS * L::SCR_STRIDE_ROW;
    float2* etab = tw + N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_set<N>(a)[i];
    if ((kT && !kTT) || OP == ROW_ADJ)
        for (int i = threadIdx.x; i < kExpTab; i += blockDim.x) etab[i] = a.exptab[i];
    __syncthreads();
    float2* scr_base = smem + team * L::SCR_STRIDE_ROW;
    auto scr = [scr_base](int k1, int q) { return scr_base + k1 * (G + 1) + q; };
    auto sync = []() { __syncwarp(); };

    if (kT || OP == ROW_ADJ) {
        const size_t voff = ((size_t)(a.slice - a.sV_slice_base) * ny + r) * N;
        const float* vr = kTT ? nullptr : (wi.sV ? wi.sV : a.sV + (size_t)wi.conf_slot * a.sV_slot_stride) + voff;
        const float2* tr = kTT ? a.tt + (size_t)wi.conf_slot * a.sV_slot_stride + voff : nullptr;
        if (OP == ROW_T_FWD || OP == ROW_TT_FWD) {
            if (a.flags & PF_TILT_INCIDENT) {
                // apply_beam_tilt / exp_r_factor_2d (incident_wave.cuh:72-78, device_kernels.cuh:519-533):
                // the plane wave exp(2 pi i (g0x Rx + g0y Ry)), R measured from the box centre, phase in FP64
                const double ry = (double)r * (a.grid.ly / ny) - 0.5 * a.grid.ly;
#pragma unroll
                for (int j = 0; j < E; j++) {
                    const double rx = (double)(g + G * j) * (a.grid.lx / N) - 0.5 * a.grid.lx;
                    v[j] = expi_d(6.283185307179586476925 * (a.grid.g0x * rx + a.grid.g0y * ry));
                }
            } else {
#pragma unroll
                for (int j = 0; j < E; j++) v[j] = make_float2(1.0f, 0.0f);
            }
        }
        // pass 0: inverse row FFT as conj(FFT(conj(x))), then the transmission;
        // pass 1: forward row FFT.  One copy of the transform code serves both.
        // ROW_ADJ is the adjoint of the same operator: with xbar the inverse row transform of the
        // adjoint wave and x = t psi the stored forward wave, dL/dV += Re(i x conj(xbar)) and the
        // adjoint continues as conj(t) xbar (or_stem_backward's chain, restated per row).
#pragma unroll 1
        for (int pass = (OP == ROW_T_FWD || OP == ROW_TT_FWD) ? 1 : 0; pass < 2; pass++) {
            if (pass == 0) conj_all(v);
            else if (OP == ROW_ADJ) {
                // each wave's dL/dV contribution goes to its own plane of a.dV ([B][ny][nx]); the planes
                // are summed in a fixed order afterwards, so the gradient is reproducible bit for bit
                const float2* xr = a.xs + row_off;
                float* gr = a.dV + row_off;
#pragma unroll
                for (int j = 0; j < E; j++) {
                    const float2 x = __ldg(xr + g + G * j);
                    gr[g + G * j] = x.x * v[j].y - x.y * v[j].x;
                    v[j] = cmulc(v[j], expi_tab(__ldg(vr + g + G * j), etab));
                }
            } else if (!beyond) {
                if constexpr (kTT) {
#pragma unroll
                    for (int j = 0; j < E; j++) v[j] = cmul(v[j], __ldg(tr + g + G * j));
                } else {
#pragma unroll
                    for (int j = 0; j < E; j++) v[j] = cmul(v[j], expi_tab(__ldg(vr + g + G * j), etab));
                }
                if constexpr (OP == ROW_INV_T_FWD_X) {
#pragma unroll
                    for (int j = 0; j < E; j++) a.xs[row_off + g + G * j] = v[j];
                }
            }
            team_fft<N, G, -1>(v, g, tw, scr, sync);
            if (pass == 0) conj_all(v);
        }
#pragma unroll
        for (int j = 0; j < E; j++) a.psi[row_off + g + G * j] = v[j];
        return;
    } else {
        const float2* src = (OP == ROW_INV_ABS2 && (a.flags & PF_FILTER_AUX)) ? a.aux : a.psi;
#pragma unroll
        for (int j = 0; j < E; j++) v[j] = src[row_off + g + G * j];
        team_fft<N, G, +1>(v, g, tw, scr, sync);
    }
    if (OP == ROW_INV_ABS2) {
        float* o = a.out_real + ((a.flags & PF_FILTER_AUX) ? (size_t)r * N : row_off);
        const float w = wi.weight;
#pragma unroll
        for (int j = 0; j < E; j++) {
            float i2 = w * (v[j].x * v[j].x + v[j].y * v[j].y);
            if (a.flags & PF_ACCUMULATE) o[g + G * j] += i2;
            else o[g + G * j] = i2;
        }
    } else if (OP == ROW_INV_STORE) {
#pragma unroll
        for (int j = 0; j < E; j++) a.aux[row_off + g + G * j] = v[j];
    }
}

// Row pass on a transmission store (ROW_INV_TT_FWD), the hot pass of the CBED, HRTEM, STEM and
// thickness loops: inverse row FFT, times t, forward row FFT, one row per warp.  A lean copy of
// k_row's path: only the wave's slice count and configuration slot are read from its descriptor,
// and the addresses are formed where they are used, so nothing stays live across the transforms
// but the row's values (k_row's general form spills here).  Loads and stores carry the L2
// eviction priorities of PassArgs.l2_mode, a template argument MODE (a policy chosen at run time
// costs the registers that make the kernel spill).
// L is the tile layout: FftLayout<N> (wide, the default) or NarrowLayout<N> (one warp of rows per
// block, twiddles read from global memory).  SV: the slice is a σV store (the wave's own, WaveInfo.sV,
// or the configuration's slot of PassArgs.sV) and t = exp(iσV) is formed here from the exp table
// (read through L1), as k_row's ROW_INV_T_FWD does: the same values as a transmission store.
// XS (with SV): the transmitted real-space wave t·ψ is also written to PassArgs.xs, as
// ROW_INV_T_FWD_X does for the adjoint's checkpoints.
template <int N, int MODE, class L = FftLayout<N>, bool SV = false, bool XS = false>
__global__ void __launch_bounds__(L::ROW_THREADS, L::ROW_MINB) k_row_tt(PassArgs a)
{
    constexpr int G = L::G, E = L::E;
    extern __shared__ float2 smem[];
    const int ny = a.grid.ny;
    const int blocks_per_wave = ny / L::ROWS;
    const int b = blockIdx.x / blocks_per_wave;
    const int team = threadIdx.x / G, g = threadIdx.x % G;
    const int r = (blockIdx.x % blocks_per_wave) * L::ROWS + team;
    const bool beyond = a.slice >= a.waves[b].n_slices;
    if (beyond && !(a.flags & PF_VACUUM_BEYOND)) return;
    float2 v[E];
    {
        const float2* src = a.psi + ((size_t)b * ny + r) * N + g;
#pragma unroll
        for (int j = 0; j < E; j++) v[j] = src[G * j];
    }
    const float2* tw;
    if constexpr (L::NARROW) {
        tw = tw_set<N>(a);
    } else {
        float2* tws = smem + L::ROWS * L::SCR_STRIDE_ROW;
        for (int i = threadIdx.x; i < N; i += blockDim.x) tws[i] = tw_set<N>(a)[i];
        __syncthreads();
        tw = tws;
    }
    float2* scr_base = smem + team * L::SCR_STRIDE_ROW;
    auto scr = [scr_base](int k1, int q) { return scr_base + k1 * (G + 1) + q; };
    auto sync = []() { __syncwarp(); };
    // inverse row FFT as conj(FFT(conj(x)))
    conj_all(v);
    team_fft<N, G, -1>(v, g, tw, scr, sync);
    conj_all(v);
    if (!beyond) {
        const WaveInfo* wi = opaque(a.waves + b);
        const size_t voff = ((size_t)(a.slice - a.sV_slice_base) * ny + r) * N + g;
        if constexpr (SV) {
            const float* vr = (wi->sV ? wi->sV : opaque(a.sV) + (size_t)wi->conf_slot * a.sV_slot_stride) + voff;
#pragma unroll
            for (int j = 0; j < E; j++) v[j] = cmul(v[j], expi_tab(__ldg(vr + G * j), a.exptab));
            if constexpr (XS) {
                float2* xr = opaque(a.xs) + ((size_t)b * ny + r) * N + g;
#pragma unroll
                for (int j = 0; j < E; j++) xr[G * j] = v[j];
            }
        } else {
            const float2* tr = opaque(a.tt) + (size_t)wi->conf_slot * a.sV_slot_stride + voff;
            const uint64_t pol = l2_policy_trans(MODE);
#pragma unroll
            for (int j = 0; j < E; j++) v[j] = cmul(v[j], ld_nc_l2hint(tr + G * j, pol));
        }
    }
    team_fft<N, G, -1>(v, g, tw, scr, sync);
    float2* dst = opaque(a.psi) + ((size_t)b * ny + r) * N + g;
    const uint64_t pol = l2_policy_wave(MODE);
#pragma unroll
    for (int j = 0; j < E; j++) st_l2hint(dst + G * j, v[j], pol);
}

// ---------------------------------------------------------------------------
// column pass
// ---------------------------------------------------------------------------
template <int N, int OP>
__global__ void __launch_bounds__(FftLayout<N>::COL_THREADS, FftLayout<N>::COL_MINB) k_col(PassArgs a)
{
    using L = FftLayout<N>;
    constexpr int G = L::G, E = L::E, TC = L::TC;
    extern __shared__ float2 smem[];
    const int nx = a.grid.nx;
    const int tiles = nx / TC;
    const int b = blockIdx.x / tiles;
    const int col0 = (blockIdx.x % tiles) * TC;
    const int c = threadIdx.x % TC, g = threadIdx.x / TC;
    const int col = col0 + c;
    const WaveInfo wi = a.waves[b];
    bool final_step = false;
    if (OP == COL_STEP || OP == COL_STEP_SEP) {
        if (a.slice >= wi.n_slices && !(a.flags & PF_VACUUM_BEYOND)) return;
        final_step = (a.slice == wi.n_slices - 1) && !(a.flags & PF_PROP_ALWAYS);
    }

    float2* base = a.psi + (size_t)b * N * nx;
    // element (g + G j, col) of the wave sits at cp[j * cs]; the pointer is made opaque before each
    // later use so the compiler recomputes the E addresses (one IMAD each) instead of keeping E
    // 64-bit addresses live across the transforms
    float2* cp = base + (size_t)g * nx + col;
    const size_t cs = (size_t)G * nx;
    float2 v[E];
    // the wave's loads go out first, so their latency overlaps the table staging below
    if constexpr (OP != COL_PROBE_INV) {
#pragma unroll
        for (int j = 0; j < E; j++) v[j] = cp[j * cs];
    }
    const float2* tw;
    if constexpr (L::COL_TW_GLOBAL) {
        tw = a.tw;   // read through L1: shared memory is kept for the transposes of three blocks per SM
    } else {
        float2* tws = smem + TC * L::SCR_STRIDE_COL;
        for (int i = threadIdx.x; i < N; i += blockDim.x) tws[i] = tw_set<N>(a)[i];
        __syncthreads();
        tw = tws;
    }
    float2* scr_base = smem + c * L::SCR_STRIDE_COL;
    auto scr = [scr_base](int k1, int q) { return scr_base + k1 * (G + 1) + q; };
    auto sync = []() { __syncthreads(); };
    if constexpr (OP == COL_PROBE_INV) {
        // Generate_probe / Generate_multi_probe (device_kernels.cuh:363-444): aperture mask on the
        // float frequency, phase chi + x gx + y gy formed in FP64.
        const double gx = freq_d(col, nx, a.grid.dgx);
        const double xf = -6.283185307179586476925 * wi.px, yf = -6.283185307179586476925 * wi.py;
#pragma unroll
        for (int j = 0; j < E; j++) {
            const int k = g + G * j;
            float g2 = det_g2(col, k, nx, N, a.grid.dgx_f, a.grid.dgy_f);
            if (a.lens.g2min <= g2 && g2 < a.lens.g2max) {
                double gy = freq_d(k, N, a.grid.dgy);
                v[j] = expi_d(chi_d(a.lens, wi.cc10, gx, gy) + xf * gx + yf * gy);
            } else {
                v[j] = make_float2(0.0f, 0.0f);
            }
        }
        team_fft<N, G, +1>(v, g, tw, scr, sync);
        cp = opaque(cp);
#pragma unroll
        for (int j = 0; j < E; j++) cp[j * cs] = v[j];
        return;
    } else {
    if constexpr (OP == COL_STEP || OP == COL_STEP_SEP) {
        // pass 0: forward column FFT, then P (or stop: the exit wave of the wave's last slice);
        // pass 1: inverse column FFT as conj(FFT(conj(x))).  One copy of the transform code.
#pragma unroll 1
        for (int pass = 0; pass < 2; pass++) {
            team_fft<N, G, -1>(v, g, tw, scr, sync);
            if (pass == 1) {
                conj_all(v);
                break;
            }
            if (final_step) break;
            if (OP == COL_STEP) {
                // P(k) = (1/N) bwl(g^2) exp(i w |g - g0|^2) (gen_propagator_kernel, device_kernels.cuh:215-234),
                // tabulated once per grid in FP64 and rounded to FP32; shared by every wave, so it stays in L2.
                // The barrier keeps the table loads after the transform, so they do not hold registers
                // across it.
                // The slice's dithered table, read through L2 with the evict-last policy: every wave of
                // the launch reads it.
                const float2* pp = opaque(prop_set(wi.prop ? wi.prop : a.prop, a) + (size_t)g * nx + col);
                const uint64_t pl = l2_policy_evict_last();
                if (a.flags & PF_CONJ_PROP) {
#pragma unroll
                    for (int j = 0; j < E; j++) v[j] = cmulc(v[j], ld_nc_l2hint(pp + j * cs, pl));
                } else {
#pragma unroll
                    for (int j = 0; j < E; j++) v[j] = cmul(v[j], ld_nc_l2hint(pp + j * cs, pl));
                }
            } else {
                // P formed per element from the separable FP64-rounded phase factors and the band limit
                // (where no table may be stored)
                const float2 px = __ldg(a.prop_x + col);
#pragma unroll
                for (int j = 0; j < E; j++) {
                    const int k = g + G * j;
                    float amp = a.grid.inv_n;
                    float g2 = det_g2(col, k, nx, N, a.grid.dgx_f, a.grid.dgy_f);
                    if (a.grid.bwl) amp = amp / (1.0f + expf(a.grid.alpha_f * (g2 - a.grid.gl2_f)));
                    const float2 P = cscale(cmul(px, __ldg(a.prop_y + k)), amp);
                    v[j] = (a.flags & PF_CONJ_PROP) ? cmulc(v[j], P) : cmul(v[j], P);
                }
            }
            if (a.flags & PF_FILTER_AUX) {
                float2* ab = opaque(a.aux + (size_t)b * N * nx + (size_t)g * nx + col);
#pragma unroll
                for (int j = 0; j < E; j++) {
                    const int k = g + G * j;
                    float g2 = det_g2(col, k, nx, N, a.grid.dgx_f, a.grid.dgy_f);
                    bool in = (a.filt_g2in <= g2 && g2 <= a.filt_g2out);
                    ab[j * cs] = in ? v[j] : make_float2(0.0f, 0.0f);
                }
            }
            conj_all(v);
        }
    } else if constexpr (OP == COL_CTF_INV) {
        // apply_CTF_kernel (device_kernels.cuh:445-468) with the source-point shift (gxu, gyu) and
        // amplitude of a TCC quadrature point, or apply_PCTF_kernel (:505-518) with the partially
        // coherent envelope (incoherent_phase_shift, basic_functions_dev.cuh:235-268)
        const double gx = freq_d(col, nx, a.grid.dgx) + a.lens.gxu;
        const float gxu = (float)a.lens.gxu, gyu = (float)a.lens.gyu;
        // a defocus series (apply_CTF_kernel_batch, device_kernels.cuh:469-503) gives every wave its
        // own defocus term; the other coefficients are the lens's
        const double cc10 = (a.flags & PF_WAVE_DEFOCUS) ? wi.cc10 : a.lens.cc10;
#pragma unroll
        for (int j = 0; j < E; j++) {
            const int k = g + G * j;
            float g2 = det_g2_shift(col, k, nx, N, a.grid.dgx_f, a.grid.dgy_f, gxu, gyu);
            if (a.lens.g2min <= g2 && g2 < a.lens.g2max) {
                double gy = freq_d(k, N, a.grid.dgy) + a.lens.gyu;
                double amp = a.lens.amp;
                if (a.lens.pctf) {
                    const double gg = gx * gx + gy * gy;
                    const double u = 1.0 + 2.0 * a.lens.pe_a * a.lens.pe_a * gg;
                    const double ct = a.lens.pe_b * gg;
                    const double cs = a.lens.pe_c * (a.lens.pe_d * gg - a.lens.pe_e);
                    amp *= exp(-(cs * cs * gg + 0.5 * ct * ct) / u) / sqrt(u);
                }
                v[j] = cmul(v[j], cscale(expi_d(chi_d(a.lens, cc10, gx, gy)), (float)amp));
            } else {
                v[j] = make_float2(0.0f, 0.0f);
            }
        }
        team_fft<N, G, +1>(v, g, tw, scr, sync);
    } else if constexpr (OP == COL_INV) {
        team_fft<N, G, +1>(v, g, tw, scr, sync);
    } else if constexpr (OP == COL_SEED) {
        // lambda(k) = sum_d 4 (I_d - T_d) Psi(k) [g^2 in annulus d], then the inverse column FFT
        // (the first adjoint step of or_stem_backward: mu = D^H lambda, here its column half)
        const double* rs = a.resid + (size_t)b * a.ndet;
#pragma unroll
        for (int j = 0; j < E; j++) {
            const int k = g + G * j;
            const float g2 = det_g2(col, k, nx, N, a.grid.dgx_f, a.grid.dgy_f);
            double f = 0.0;
            for (int d = 0; d < a.ndet; d++)
                if (a.det_thr[d] <= g2 && g2 <= a.det_thr[a.ndet + d]) f += rs[d];
            v[j] = cscale(v[j], (float)f);
        }
        team_fft<N, G, +1>(v, g, tw, scr, sync);
    } else if constexpr (OP == COL_GRAD_PROBE) {
        // Psi0bar = forward column FFT of the row-transformed adjoint; q = Re(i Psi0 conj(Psi0bar))
        // with Psi0 regenerated exactly as COL_PROBE_INV does; sums of g^2 q and g^4 q give
        // dL/dC10 and dL/dC30 (or_stem_backward's lens-phase gradient).
        team_fft<N, G, -1>(v, g, tw, scr, sync);
        const double gx = freq_d(col, nx, a.grid.dgx);
        const double xf = -6.283185307179586476925 * wi.px, yf = -6.283185307179586476925 * wi.py;
        double s2 = 0.0, s4 = 0.0;
#pragma unroll
        for (int j = 0; j < E; j++) {
            const int k = g + G * j;
            const float g2 = det_g2(col, k, nx, N, a.grid.dgx_f, a.grid.dgy_f);
            if (a.lens.g2min <= g2 && g2 < a.lens.g2max) {
                const double gy = freq_d(k, N, a.grid.dgy);
                const float2 w0 = expi_d(chi_d(a.lens, wi.cc10, gx, gy) + xf * gx + yf * gy);
                const double q = (double)w0.x * v[j].y - (double)w0.y * v[j].x;
                const double gg = gx * gx + gy * gy;
                s2 += gg * q;
                s4 += gg * gg * q;
            }
        }
        __shared__ double red[2][32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s2 += __shfl_down_sync(0xffffffffu, s2, o);
            s4 += __shfl_down_sync(0xffffffffu, s4, o);
        }
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) {
            red[0][wid] = s2;
            red[1][wid] = s4;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double t2 = 0.0, t4 = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
                t2 += red[0][w];
                t4 += red[1][w];
            }
            double* o = a.chi_part + ((size_t)b * tiles + (size_t)(col0 / TC)) * 2;
            o[0] = t2;
            o[1] = t4;
        }
        return;
    }
    cp = opaque(cp);
    if constexpr (OP == COL_STEP) {
        // the propagated wave goes on to the next row pass
        const uint64_t pol = l2_policy_wave(a.l2_mode);
#pragma unroll
        for (int j = 0; j < E; j++) st_l2hint(cp + j * cs, v[j], pol);
    } else {
#pragma unroll
        for (int j = 0; j < E; j++) cp[j * cs] = v[j];
    }
    }
}

// Column step (COL_STEP) with the wave tile brought in by the tensor memory accelerator: one
// thread issues the 2-D box loads of the block's N x TC tile into shared memory (N / 256 boxes of
// TC columns), the block stages its twiddles meanwhile, and every thread then reads its column
// elements from shared memory (a warp reads whole row segments: no bank conflicts).  The tile
// region is the transposition scratch of the transforms that follow, so the block needs no more
// shared memory than the classic kernel.  Compared with one 8-byte load per element and thread,
// the copy engine moves the tile in large requests and leaves the load/store unit free.  The wait
// for the tile is bounded (PassArgs.wait_cycles): when it runs out the block records the failure
// in PassArgs.err and returns.  The arithmetic is k_col's COL_STEP.
template <int N, class L = FftLayout<N>>
__global__ void __launch_bounds__(L::COL_THREADS, L::COL_MINB)
    k_col_step_tma(PassArgs a, const __grid_constant__ CUtensorMap tmap)
{
    constexpr int G = L::G, E = L::E, TC = L::TC;
    constexpr int BOX = N < 256 ? N : 256;
    constexpr unsigned TILE_BYTES = (unsigned)(N * TC * sizeof(float2));
    static_assert((size_t)TILE_BYTES <= TC * L::SCR_STRIDE_COL * sizeof(float2), "the tile lives in the scratch");
    __shared__ __align__(8) uint64_t bar;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // 128-byte aligned base (the launch adds 128 bytes of slack)
    float2* smem = reinterpret_cast<float2*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
    const int nx = a.grid.nx;
    const int tiles = nx / TC;
    const int b = blockIdx.x / tiles;
    const int col0 = (blockIdx.x % tiles) * TC;
    const int c = threadIdx.x % TC, g = threadIdx.x / TC;
    const int col = col0 + c;
    const WaveInfo& wi = a.waves[b];
    if (a.slice >= wi.n_slices && !(a.flags & PF_VACUUM_BEYOND)) return;
    const bool final_step = (a.slice == wi.n_slices - 1) && !(a.flags & PF_PROP_ALWAYS);
    float2* tile = smem;
    float2* tws = smem + TC * L::SCR_STRIDE_COL;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_expect_tx(&bar, TILE_BYTES + ((a.flags & PF_TEST_WAIT) ? 16u : 0u));
#pragma unroll
        for (int q = 0; q < N / BOX; q++) tma_load_2d(tile + q * BOX * TC, &tmap, 2 * col0, b * N + q * BOX, &bar);
    }
    if constexpr (!L::NARROW)
        for (int i = threadIdx.x; i < N; i += blockDim.x) tws[i] = tw_set<N>(a)[i];
    const float2* twp = L::NARROW ? tw_set<N>(a) : tws;
    __syncthreads();
    const long long limit = (a.flags & PF_TEST_WAIT) ? 2000000LL : (a.wait_cycles > 0 ? a.wait_cycles : kWaitCycles);
    const bool late = !mbar_wait_bounded(&bar, 0, limit);
    if (__syncthreads_or(late)) {
        if (threadIdx.x == 0 && a.err) atomicOr(a.err, 1);
        return;
    }
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; j++) v[j] = tile[(g + G * j) * TC + c];
    __syncthreads();   // every thread holds its values: the tile region becomes the scratch
    float2* scr_base = smem + c * L::SCR_STRIDE_COL;
    auto scr = [scr_base](int k1, int q) { return scr_base + k1 * (G + 1) + q; };
    auto sync = []() { __syncthreads(); };
    const size_t cs = (size_t)G * nx;
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
        team_fft<N, G, -1>(v, g, twp, scr, sync);
        if (pass == 1) {
            conj_all(v);
            break;
        }
        if (final_step) break;
        const float2* pp = opaque(prop_set(wi.prop ? wi.prop : a.prop, a) + (size_t)g * nx + col);
        const uint64_t pl = l2_policy_evict_last();
        if (a.flags & PF_CONJ_PROP) {
#pragma unroll
            for (int j = 0; j < E; j++) v[j] = cmulc(v[j], ld_nc_l2hint(pp + j * cs, pl));
        } else {
#pragma unroll
            for (int j = 0; j < E; j++) v[j] = cmul(v[j], ld_nc_l2hint(pp + j * cs, pl));
        }
        conj_all(v);
    }
    float2* cp = opaque(a.psi + (size_t)b * N * nx + (size_t)g * nx + col);
    const uint64_t pol = l2_policy_wave(a.l2_mode);
#pragma unroll
    for (int j = 0; j < E; j++) st_l2hint(cp + j * cs, v[j], pol);
}

// Column step with one warp per column (TILE_WARP_COLS, 1024-point columns: a team of G = 32
// threads is one warp, so the transforms synchronise within the warp only).  The block's 8
// columns arrive by TMA through a tensor map with the 64-byte swizzle: in a 64-byte row of the
// tile, the 16-byte chunk c/2 of column c sits at chunk (c/2) XOR (row/2 mod 4), so a warp reading
// one column down 32 rows touches 8 bank pairs per half-warp (a 2-way conflict) instead of 2.  The
// propagator comes from the transposed tables (PassArgs.propT, [kx][ky]), read along the column
// with whole-warp coalesced loads.  The results go back into the swizzled tile and out by TMA
// stores carrying the L2 mode's priority.  The arithmetic is k_col_step_tma's (the same transforms, twiddles and products), so
// the outputs are identical.
template <int N>
__global__ void __launch_bounds__(256, 2) k_col_step_warp(PassArgs a, const __grid_constant__ CUtensorMap tmap)
{
    using L = FftLayout<N>;
    constexpr int G = L::G, E = L::E, TC = 8, BOX = 256;
    static_assert(G == 32, "one team per warp");
    constexpr int SCR = E * (G + 1) + 1;                      // one team's transposition scratch (float2)
    constexpr unsigned TILE_BYTES = (unsigned)(N * TC * sizeof(float2));
    static_assert((size_t)TILE_BYTES <= (size_t)TC * SCR * sizeof(float2), "the tile lives in the scratch");
    __shared__ __align__(8) uint64_t bar;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // 1024-byte aligned base (the launch adds 1024 bytes of slack): the swizzle acts on address bits
    unsigned char* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const int nx = a.grid.nx;
    const int tiles = nx / TC;
    const int b = blockIdx.x / tiles;
    const int col0 = (blockIdx.x % tiles) * TC;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const WaveInfo& wi = a.waves[b];
    if (a.slice >= wi.n_slices && !(a.flags & PF_VACUUM_BEYOND)) return;
    const bool final_step = (a.slice == wi.n_slices - 1) && !(a.flags & PF_PROP_ALWAYS);
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_expect_tx(&bar, TILE_BYTES + ((a.flags & PF_TEST_WAIT) ? 16u : 0u));
#pragma unroll
        for (int q = 0; q < N / BOX; q++) tma_load_2d(base + q * BOX * 64, &tmap, 2 * col0, b * N + q * BOX, &bar);
    }
    __syncthreads();
    const long long limit = (a.flags & PF_TEST_WAIT) ? 2000000LL : (a.wait_cycles > 0 ? a.wait_cycles : kWaitCycles);
    const bool late = !mbar_wait_bounded(&bar, 0, limit);
    if (__syncthreads_or(late)) {
        if (threadIdx.x == 0 && a.err) atomicOr(a.err, 1);
        return;
    }
    // element (row r, column c) of the swizzled tile
    auto at = [base](int r, int c) {
        return reinterpret_cast<float2*>(base + r * 64 + ((((c >> 1) ^ ((r >> 1) & 3)) << 4) | ((c & 1) << 3)));
    };
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; j++) v[j] = *at(lane + G * j, w);
    __syncthreads();   // every warp holds its column: the tile region becomes the scratch
    float2* scr_base = reinterpret_cast<float2*>(base) + w * SCR;
    auto scr = [scr_base](int k1, int q) { return scr_base + k1 * (G + 1) + q; };
    auto sync = []() { __syncwarp(); };
    const float2* tw = tw_set<N>(a);   // through L1
    const int col = col0 + w;
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
        team_fft<N, G, -1>(v, lane, tw, scr, sync);
        if (pass == 1) {
            conj_all(v);
            break;
        }
        if (final_step) break;
        const float2* pp = opaque(prop_set(a.propT, a) + (size_t)col * N + lane);
        const uint64_t pl = l2_policy_evict_last();
        if (a.flags & PF_CONJ_PROP) {
#pragma unroll
            for (int j = 0; j < E; j++) v[j] = cmulc(v[j], ld_nc_l2hint(pp + G * j, pl));
        } else {
#pragma unroll
            for (int j = 0; j < E; j++) v[j] = cmul(v[j], ld_nc_l2hint(pp + G * j, pl));
        }
        conj_all(v);
    }
    __syncthreads();   // every warp is done with its scratch: the region takes the result tile
#pragma unroll
    for (int j = 0; j < E; j++) *at(lane + G * j, w) = v[j];
    // the tile's ordinary stores before the tensor-memory-accelerator reads of it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        // the wave's lines keep the L2 mode's priority (evict-last while the batch fits in L2)
        const uint64_t pw = l2_policy_wave(a.l2_mode);
#pragma unroll
        for (int q = 0; q < N / BOX; q++)
            tma_store_2d_hint(&tmap, 2 * col0, b * N + q * BOX, base + q * BOX * 64, pw);
        tma_store_commit_and_wait();
    }
}

template <int N>
static bool col_step_warp(const PassArgs& a, int nwaves, int nx, cudaStream_t st)
{
    if constexpr (N != 1024) {
        return false;
    } else {
        using L = FftLayout<N>;
        if (!a.propT || nx % 8 != 0 || ((uintptr_t)a.psi & 15) != 0) return false;
        CUtensorMap map;
        if (!encode_wave_tile_map(&map, a.psi, nx, (int64_t)nwaves * N, 16, 256, true)) return false;
        constexpr size_t sm = sizeof(float2) * 8 * (L::E * (L::G + 1) + 1) + 1024;
        smem_attr(k_col_step_warp<N>, sm);
        k_col_step_warp<N><<<(unsigned)(nwaves * (nx / 8)), 256, sm, st>>>(a, map);
        return true;
    }
}

template <int N, class L = FftLayout<N>>
static bool col_step_tma(const PassArgs& a, int nwaves, int nx, cudaStream_t st)
{
    if constexpr (N < 256) {
        return false;
    } else {
        if (((uintptr_t)a.psi & 15) != 0) return false;
        CUtensorMap map;
        if (!encode_wave_tile_map(&map, a.psi, nx, (int64_t)nwaves * N, 2 * L::TC, N < 256 ? N : 256)) return false;
        const size_t sm = L::COL_SMEM + 128;
        smem_attr(k_col_step_tma<N, L>, sm);
        k_col_step_tma<N, L><<<(unsigned)(nwaves * (nx / L::TC)), L::COL_THREADS, sm, st>>>(a, map);
        return true;
    }
}

// ---------------------------------------------------------------------------
// Persistent, software-pipelined forms of the two slice passes (ROW_INV_T_FWD and
// COL_STEP with the propagator table).  One block of 256 threads per SM stays resident
// and walks the pass's work items with a grid stride; the twiddle and exp tables are
// staged into shared memory once per block instead of once per item.  While an item is
// transformed, the next item's wave values are already in flight into registers (the
// block has the whole register file: 255 per thread), the row pass issues the item's
// potential loads before its first transform, and the column pass brings the next item's
// propagator tile into shared memory with cp.async.  The arithmetic is the classic
// kernels' (the compiler may contract a few products differently, so the two forms agree
// to about one rounding per operation rather than bit for bit).
// ---------------------------------------------------------------------------
constexpr int kPipeThreads = 256;

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <int N>
__global__ void __launch_bounds__(kPipeThreads, 1) k_row_p(PassArgs a, int nwaves)
{
    using L = FftLayout<N>;
    constexpr int G = L::G, E = L::E;
    constexpr int R = 32 / G;                       // rows per warp item (one per team)
    constexpr int WARPS = kPipeThreads / 32;
    constexpr int VROW = R * N;                     // potential floats of one item
    // cp.async destinations must sit on 16-byte boundaries
    static_assert(((WARPS * R * L::SCR_STRIDE_ROW + N + kExpTab) * sizeof(float2)) % 16 == 0, "vbuf alignment");
    static_assert((VROW * sizeof(float)) % 16 == 0, "vbuf alignment");
    extern __shared__ float2 smem[];
    float2* tw = smem + WARPS * R * L::SCR_STRIDE_ROW;
    float2* etab = tw + N;
    float* vbuf_all = reinterpret_cast<float*>(etab + kExpTab);   // [WARPS][2][VROW]
    for (int i = threadIdx.x; i < N; i += kPipeThreads) tw[i] = tw_set<N>(a)[i];
    for (int i = threadIdx.x; i < kExpTab; i += kPipeThreads) etab[i] = a.exptab[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tm = lane / G, g = lane % G;
    float2* scr_base = smem + (warp * R + tm) * L::SCR_STRIDE_ROW;
    auto scr = [scr_base](int k1, int q) { return scr_base + k1 * (G + 1) + q; };
    auto sync = []() { __syncwarp(); };
    float* vbuf = vbuf_all + warp * 2 * VROW;
    const int ny = a.grid.ny;
    const int64_t n_items = (int64_t)nwaves * ny / R;
    const int64_t stride = (int64_t)gridDim.x * WARPS;
    const bool vac = (a.flags & PF_VACUUM_BEYOND) != 0;
    // items whose wave has no slice here are skipped whole (the classic kernel's early return)
    auto next_live = [&](int64_t it) {
        while (it < n_items && !vac && a.slice >= a.waves[(int)((it * R) / ny)].n_slices) it += stride;
        return it;
    };
    // the item's R potential rows (contiguous: the rows of one wave) into vbuf[buf], 16 bytes a piece
    auto fetch_pot = [&](int64_t it, int buf) {
        const int64_t row0 = it * R;
        const int b = (int)(row0 / ny), r0 = (int)(row0 % ny);
        const WaveInfo& wi = a.waves[b];
        if (a.slice < wi.n_slices) {
            const float* vr = (wi.sV ? wi.sV : a.sV + (size_t)wi.conf_slot * a.sV_slot_stride) +
                              ((size_t)(a.slice - a.sV_slice_base) * ny + r0) * N;
            for (int q = lane; q < VROW / 4; q += 32) cp_async16(vbuf + buf * VROW + 4 * q, vr + 4 * q);
        }
        cp_async_commit();
    };
    int64_t it = next_live((int64_t)blockIdx.x * WARPS + warp);
    float2 vn[E];
    if (it < n_items) {
        const float2* src = a.psi + (it * R + tm) * N;
#pragma unroll
        for (int j = 0; j < E; j++) vn[j] = src[g + G * j];
        fetch_pot(it, 0);
    }
    int buf = 0;
    while (it < n_items) {
        const int64_t row = it * R + tm;
        const int b = (int)(row / ny);
        float2 v[E];
#pragma unroll
        for (int j = 0; j < E; j++) v[j] = vn[j];
        const int64_t nxt = next_live(it + stride);
        if (nxt < n_items) {
            const float2* src = a.psi + (nxt * R + tm) * N;
#pragma unroll
            for (int j = 0; j < E; j++) vn[j] = src[g + G * j];
            fetch_pot(nxt, buf ^ 1);
        } else {
            cp_async_commit();
        }
        const bool beyond = a.slice >= a.waves[b].n_slices;
        const float* vv = vbuf + buf * VROW + tm * N;
#pragma unroll 1
        for (int pass = 0; pass < 2; pass++) {
            if (pass == 0) conj_all(v);
            else if (!beyond) {
                asm volatile("cp.async.wait_group 1;\n" ::: "memory");
                __syncwarp();
#pragma unroll
                for (int j = 0; j < E; j++) v[j] = cmul(v[j], expi_tab(vv[g + G * j], etab));
            }
            team_fft<N, G, -1>(v, g, tw, scr, sync);
            if (pass == 0) conj_all(v);
        }
        float2* dst = a.psi + row * N;
#pragma unroll
        for (int j = 0; j < E; j++) dst[g + G * j] = v[j];
        buf ^= 1;
        it = nxt;
    }
    cp_async_wait_all();
}

// Row pass on a transmission store (ROW_INV_TT_FWD), 12 warps per SM.  One persistent block of
// 384 threads per SM; each warp walks its rows with a grid stride and double-buffers them in
// shared memory: while a row is transformed, the next one arrives by cp.async (no registers, no
// wait until it is needed), and the buffer a row arrived in serves as its transposition scratch
// (XOR-swizzled so that the N points fill exactly N slots without bank conflicts).  The row's
// transmission values are loaded into registers before the inverse transform and consumed after
// it.  The arithmetic is the classic kernel's.
constexpr int kQWarps = 12;

template <int N>
__global__ void __launch_bounds__(kQWarps * 32, 1) k_row_q(PassArgs a, int nwaves)
{
    using L = FftLayout<N>;
    constexpr int G = L::G, E = L::E;
    constexpr int R = 32 / G;        // rows per warp item (one per team)
    constexpr int ITEM = R * N;      // float2 of one item
    extern __shared__ float2 smem[];
    float2* tw = smem;
    for (int i = threadIdx.x; i < N; i += kQWarps * 32) tw[i] = tw_set<N>(a)[i];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tm = lane / G, g = lane % G;
    float2* wbuf = smem + N + (size_t)warp * 2 * ITEM;
    __syncthreads();
    const int ny = a.grid.ny;
    const int64_t n_items = (int64_t)nwaves * ny / R;
    const int64_t stride = (int64_t)gridDim.x * kQWarps;
    const bool vac = (a.flags & PF_VACUUM_BEYOND) != 0;
    auto next_live = [&](int64_t it) {
        while (it < n_items && !vac && a.slice >= a.waves[(int)((it * R) / ny)].n_slices) it += stride;
        return it;
    };
    auto t_item = [&](int64_t it) -> const float2* {
        const int64_t row0 = it * R;
        const WaveInfo& wi = a.waves[(int)(row0 / ny)];
        if (a.slice >= wi.n_slices) return nullptr;
        return a.tt + (size_t)wi.conf_slot * a.sV_slot_stride +
               ((size_t)(a.slice - a.sV_slice_base) * ny + (int)(row0 % ny)) * N;
    };
    // the item's wave rows into dst by cp.async; its transmission rows towards L2 (they are read
    // after the first transform, so a register copy would only raise the register count)
    auto fetch = [&](int64_t it, float2* dst) {
        const float2* src = a.psi + it * ITEM;
        for (int q = lane; q < ITEM / 2; q += 32) cp_async16(dst + 2 * q, src + 2 * q);
        cp_async_commit();
        if (const float2* tr = t_item(it))
            for (int q = lane; q < ITEM / 16; q += 32)
                asm volatile("prefetch.global.L2 [%0];\n" ::"l"(tr + 16 * q));
    };
    int64_t it = next_live((int64_t)blockIdx.x * kQWarps + warp);
    int cur = 0;
    if (it < n_items) fetch(it, wbuf);
    while (it < n_items) {
        cp_async_wait_all();
        __syncwarp();
        float2* B = wbuf + cur * ITEM;
        float2 v[E];
#pragma unroll
        for (int j = 0; j < E; j++) v[j] = B[tm * N + g + G * j];
        const int64_t nxt = next_live(it + stride);
        // the other buffer was the previous item's scratch; every lane is past its last use
        if (nxt < n_items) fetch(nxt, wbuf + (cur ^ 1) * ITEM);
        const int64_t row = it * R + tm;
        const float2* tr = t_item(it);
        if (tr) tr += (size_t)tm * N;
        float2* scr_base = B + tm * N;
        auto scr = [scr_base](int k1, int q) { return scr_base + k1 * G + (q ^ (k1 & (G - 1))); };
        auto sync = []() { __syncwarp(); };
#pragma unroll 1
        for (int pass = 0; pass < 2; pass++) {
            if (pass == 0) conj_all(v);
            else if (tr) {
#pragma unroll
                for (int j = 0; j < E; j++) v[j] = cmul(v[j], __ldg(tr + g + G * j));
            }
            team_fft<N, G, -1>(v, g, tw, scr, sync);
            if (pass == 0) conj_all(v);
        }
        float2* dst = a.psi + row * N;
#pragma unroll
        for (int j = 0; j < E; j++) dst[g + G * j] = v[j];
        __syncwarp();
        cur ^= 1;
        it = nxt;
    }
    cp_async_wait_all();
}

template <int N>
static bool row_q(const PassArgs& a, int nwaves, int ny, cudaStream_t st)
{
    if constexpr (N != 512 && N != 1024) {
        return false;
    } else {
        using L = FftLayout<N>;
        constexpr int R = 32 / L::G;
        const int64_t items = (int64_t)nwaves * ny / R;
        const int64_t blocks = std::min<int64_t>((items + kQWarps - 1) / kQWarps, num_sms());
        const size_t sm = sizeof(float2) * ((size_t)N + (size_t)kQWarps * 2 * R * N);
        smem_attr(k_row_q<N>, sm);
        k_row_q<N><<<(unsigned)blocks, kQWarps * 32, sm, st>>>(a, nwaves);
        return true;
    }
}

template <int N>
__global__ void __launch_bounds__(kPipeThreads, 1) k_col_p(PassArgs a, int nwaves)
{
    using L = FftLayout<N>;
    constexpr int G = L::G, E = L::E, TC = L::TC;
    static_assert(TC * G == kPipeThreads, "the column tile must occupy the whole block");
    extern __shared__ float2 smem[];
    float2* tw = smem + TC * L::SCR_STRIDE_COL;
    float2* ptile = tw + N;                         // propagator tile [N][TC]
    static_assert(((TC * L::SCR_STRIDE_COL + N) * sizeof(float2)) % 16 == 0, "ptile alignment");
    static_assert(TC % 2 == 0, "16-byte propagator pieces");
    for (int i = threadIdx.x; i < N; i += kPipeThreads) tw[i] = tw_set<N>(a)[i];
    const int nx = a.grid.nx;
    const int tiles = nx / TC;
    const int64_t n_items = (int64_t)nwaves * tiles;
    const bool vac = (a.flags & PF_VACUUM_BEYOND) != 0;
    auto next_live = [&](int64_t it) {
        while (it < n_items && !vac && a.slice >= a.waves[(int)(it / tiles)].n_slices) it += gridDim.x;
        return it;
    };
    const int tid = threadIdx.x;
    const int c = tid % TC, g = tid / TC;
    float2* scr_base = smem + c * L::SCR_STRIDE_COL;
    auto scr = [scr_base](int k1, int q) { return scr_base + k1 * (G + 1) + q; };
    auto sync = []() { __syncthreads(); };
    const size_t cs = (size_t)G * nx;
    // the propagator tile of item `it`: N rows of TC float2, in 16-byte pieces
    auto fetch_prop = [&](int64_t it) {
        const int col0 = (int)(it % tiles) * TC;
        const float2* P = prop_set(a.waves[(int)(it / tiles)].prop ? a.waves[(int)(it / tiles)].prop : a.prop, a) + col0;
        constexpr int PIECES = N * TC / 2;
        for (int q = tid; q < PIECES; q += kPipeThreads) {
            const int row = q / (TC / 2), part = q % (TC / 2);
            cp_async16(ptile + row * TC + 2 * part, P + (size_t)row * nx + 2 * part);
        }
        cp_async_commit();
    };
    int64_t it = next_live(blockIdx.x);
    float2 vn[E];
    if (it < n_items) {
        const float2* cp = a.psi + (size_t)(it / tiles) * N * nx + (size_t)g * nx + (it % tiles) * TC + c;
#pragma unroll
        for (int j = 0; j < E; j++) vn[j] = cp[j * cs];
        fetch_prop(it);
    }
    __syncthreads();
    while (it < n_items) {
        const int b = (int)(it / tiles);
        const int col = (int)(it % tiles) * TC + c;
        float2 v[E];
#pragma unroll
        for (int j = 0; j < E; j++) v[j] = vn[j];
        const int64_t nxt = next_live(it + gridDim.x);
        if (nxt < n_items) {
            const float2* cp = a.psi + (size_t)(nxt / tiles) * N * nx + (size_t)g * nx + (nxt % tiles) * TC + c;
#pragma unroll
            for (int j = 0; j < E; j++) vn[j] = cp[j * cs];
        }
        const WaveInfo& wi = a.waves[b];
        const bool final_step = (a.slice == wi.n_slices - 1) && !(a.flags & PF_PROP_ALWAYS);
        // forward column FFT, then P (or stop: the exit wave of the wave's last slice), then the
        // inverse column FFT as conj(FFT(conj(x)))
#pragma unroll 1
        for (int pass = 0; pass < 2; pass++) {
            team_fft<N, G, -1>(v, g, tw, scr, sync);
            if (pass == 1) {
                conj_all(v);
                break;
            }
            if (final_step) break;
            cp_async_wait_all();
            __syncthreads();
            const float2* pp = ptile + g * TC + c;
            if (a.flags & PF_CONJ_PROP) {
#pragma unroll
                for (int j = 0; j < E; j++) v[j] = cmulc(v[j], pp[j * G * TC]);
            } else {
#pragma unroll
                for (int j = 0; j < E; j++) v[j] = cmul(v[j], pp[j * G * TC]);
            }
            conj_all(v);
        }
        // every thread is past its reads of the tile: bring in the next item's
        cp_async_wait_all();
        __syncthreads();
        if (nxt < n_items) fetch_prop(nxt);
        float2* cp = a.psi + (size_t)b * N * nx + (size_t)g * nx + col;
#pragma unroll
        for (int j = 0; j < E; j++) cp[j * cs] = v[j];
        it = nxt;
    }
    cp_async_wait_all();
}

// Grids of 128..1024 points for the row pass; the column pass needs a full 256-thread tile
// (TC x G = 256: 256..1024 points).  2048-point passes use the classic kernels.
template <int N>
struct PipeSupported {
    static constexpr bool value = (N >= 128 && N <= 1024);
};
template <int N>
struct ColPipeSupported {
    static constexpr bool value = (N >= 256 && N <= 1024 && FftLayout<N>::TC * FftLayout<N>::G == kPipeThreads);
};


template <int N>
static bool row_pipe(const PassArgs& a, int nwaves, int ny, cudaStream_t st)
{
    if constexpr (!PipeSupported<N>::value) {
        return false;
    } else {
        using L = FftLayout<N>;
        constexpr int R = 32 / L::G;
        const int64_t items = (int64_t)nwaves * ny / R;
        const int64_t blocks = std::min<int64_t>((items + 7) / 8, num_sms());
        const size_t sm = sizeof(float2) * ((size_t)(kPipeThreads / 32) * R * L::SCR_STRIDE_ROW + N + kExpTab) +
                          sizeof(float) * (size_t)(kPipeThreads / 32) * 2 * R * N;
        smem_attr(k_row_p<N>, sm);
        k_row_p<N><<<(unsigned)blocks, kPipeThreads, sm, st>>>(a, nwaves);
        return true;
    }
}

template <int N>
static bool col_pipe(const PassArgs& a, int nwaves, int nx, cudaStream_t st)
{
    if constexpr (!ColPipeSupported<N>::value) {
        return false;
    } else {
        using L = FftLayout<N>;
        const int64_t items = (int64_t)nwaves * (nx / L::TC);
        const int64_t blocks = std::min<int64_t>(items, num_sms());
        const size_t sm = sizeof(float2) * ((size_t)L::TC * L::SCR_STRIDE_COL + N + (size_t)N * L::TC);
        smem_attr(k_col_p<N>, sm);
        k_col_p<N><<<(unsigned)blocks, kPipeThreads, sm, st>>>(a, nwaves);
        return true;
    }
}

template <int N>
void row_dispatch(int op, const PassArgs& a, int nwaves, int ny, cudaStream_t st)
{
    using L = FftLayout<N>;
    // the pipelined form copies potential rows with 16-byte cp.async: it needs an aligned store
    if (op == ROW_INV_T_FWD && a.variant == PASS_PIPELINED && !(a.flags & PF_STORE_X) && !a.tt && a.sV &&
        ((uintptr_t)a.sV & 15) == 0 && row_pipe<N>(a, nwaves, ny, st))
        return;
    dim3 grid((unsigned)(nwaves * (ny / L::ROWS))), block(L::ROW_THREADS);
    size_t sm = L::ROW_SMEM;
    if (op == ROW_INV_T_FWD && (a.flags & PF_STORE_X) && !a.tt) {
        // the adjoint's forward step that keeps t psi: the lean kernel with the extra store
        if (a.tile & TILE_NARROW_ROWS) {
            using NL = NarrowLayout<N>;
            const size_t nsm = sizeof(float2) * (size_t)NL::ROWS * NL::SCR_STRIDE_ROW;
            smem_attr(k_row_tt<N, L2_DEFAULT, NL, true, true>, nsm);
            k_row_tt<N, L2_DEFAULT, NL, true, true>
                <<<(unsigned)(nwaves * (ny / NL::ROWS)), NL::ROW_THREADS, nsm, st>>>(a);
        } else {
            smem_attr(k_row_tt<N, L2_DEFAULT, L, true, true>, sm);
            k_row_tt<N, L2_DEFAULT, L, true, true><<<grid, block, sm, st>>>(a);
        }
        return;
    }
    if (op == ROW_INV_T_FWD && (a.flags & PF_STORE_X)) op = ROW_INV_T_FWD_X;
    else if (a.tt && op == ROW_INV_T_FWD) op = ROW_INV_TT_FWD;
    else if (a.tt && op == ROW_T_FWD) op = ROW_TT_FWD;
    // the 12-warp form copies wave rows with 16-byte cp.async: it needs an aligned wave
    if (op == ROW_INV_TT_FWD && a.variant == PASS_PIPELINED && ((uintptr_t)a.psi & 15) == 0 &&
        row_q<N>(a, nwaves, ny, st))
        return;
    if (op == ROW_INV_TT_FWD && (a.tile & TILE_NARROW_ROWS)) {
        // one warp of rows per block; only the transpose scratch lives in shared memory
        using NL = NarrowLayout<N>;
        auto kern = a.l2_mode == L2_WAVES_RESIDENT ? k_row_tt<N, L2_WAVES_RESIDENT, NL>
                    : a.l2_mode == L2_SHARED_T     ? k_row_tt<N, L2_SHARED_T, NL>
                                                   : k_row_tt<N, L2_DEFAULT, NL>;
        const size_t nsm = sizeof(float2) * (size_t)NL::ROWS * NL::SCR_STRIDE_ROW;
        smem_attr(kern, nsm);
        kern<<<(unsigned)(nwaves * (ny / NL::ROWS)), NL::ROW_THREADS, nsm, st>>>(a);
        return;
    }
    if (op == ROW_INV_T_FWD) {
        // the row step on a σV store in the lean kernel (wide or narrow tiles; the wave stores keep
        // the L2 mode's priority)
        if (a.tile & TILE_NARROW_ROWS) {
            using NL = NarrowLayout<N>;
            auto kern = a.l2_mode == L2_WAVES_RESIDENT ? k_row_tt<N, L2_WAVES_RESIDENT, NL, true>
                        : a.l2_mode == L2_SHARED_T     ? k_row_tt<N, L2_SHARED_T, NL, true>
                                                       : k_row_tt<N, L2_DEFAULT, NL, true>;
            const size_t nsm = sizeof(float2) * (size_t)NL::ROWS * NL::SCR_STRIDE_ROW;
            smem_attr(kern, nsm);
            kern<<<(unsigned)(nwaves * (ny / NL::ROWS)), NL::ROW_THREADS, nsm, st>>>(a);
        } else {
            auto kern = a.l2_mode == L2_WAVES_RESIDENT ? k_row_tt<N, L2_WAVES_RESIDENT, L, true>
                        : a.l2_mode == L2_SHARED_T     ? k_row_tt<N, L2_SHARED_T, L, true>
                                                       : k_row_tt<N, L2_DEFAULT, L, true>;
            smem_attr(kern, sm);
            kern<<<grid, block, sm, st>>>(a);
        }
        return;
    }
    switch (op) {
    case ROW_T_FWD:
        smem_attr(k_row<N, ROW_T_FWD>, sm);
        k_row<N, ROW_T_FWD><<<grid, block, sm, st>>>(a);
        break;
    case ROW_INV_T_FWD:
        smem_attr(k_row<N, ROW_INV_T_FWD>, sm);
        k_row<N, ROW_INV_T_FWD><<<grid, block, sm, st>>>(a);
        break;
    case ROW_INV_ABS2:
        smem_attr(k_row<N, ROW_INV_ABS2>, sm);
        k_row<N, ROW_INV_ABS2><<<grid, block, sm, st>>>(a);
        break;
    case ROW_INV_STORE:
        smem_attr(k_row<N, ROW_INV_STORE>, sm);
        k_row<N, ROW_INV_STORE><<<grid, block, sm, st>>>(a);
        break;
    case ROW_ADJ:
        smem_attr(k_row<N, ROW_ADJ>, sm);
        k_row<N, ROW_ADJ><<<grid, block, sm, st>>>(a);
        break;
    case ROW_INV_T_FWD_X:
        smem_attr(k_row<N, ROW_INV_T_FWD_X>, sm);
        k_row<N, ROW_INV_T_FWD_X><<<grid, block, sm, st>>>(a);
        break;
    case ROW_INV_TT_FWD: {
        auto kern = a.l2_mode == L2_WAVES_RESIDENT ? k_row_tt<N, L2_WAVES_RESIDENT>
                                                   : (a.l2_mode == L2_SHARED_T ? k_row_tt<N, L2_SHARED_T>
                                                                               : k_row_tt<N, L2_DEFAULT>);
        smem_attr(kern, sm);
        kern<<<grid, block, sm, st>>>(a);
    } break;
    case ROW_TT_FWD:
        smem_attr(k_row<N, ROW_TT_FWD>, sm);
        k_row<N, ROW_TT_FWD><<<grid, block, sm, st>>>(a);
        break;
    default: throw MsError(MS_ERR_INTERNAL, "unknown row pass");
    }
}

template <int N>
void col_dispatch(int op, const PassArgs& a, int nwaves, int nx, cudaStream_t st)
{
    using L = FftLayout<N>;
    if (op == COL_STEP && a.variant == PASS_PIPELINED && !(a.flags & PF_FILTER_AUX) && ((uintptr_t)a.prop & 15) == 0 &&
        col_pipe<N>(a, nwaves, nx, st))
        return;
    // the hot column step reads its tile through the tensor memory accelerator
    if (op == COL_STEP && a.variant != PASS_PIPELINED && !(a.flags & PF_FILTER_AUX)) {
        if ((a.tile & TILE_WARP_COLS) && col_step_warp<N>(a, nwaves, nx, st)) return;
        if ((a.tile & TILE_NARROW_COLS) && col_step_tma<N, NarrowLayout<N>>(a, nwaves, nx, st)) return;
        if (col_step_tma<N>(a, nwaves, nx, st)) return;
    }
    dim3 grid((unsigned)(nwaves * (nx / L::TC))), block(L::COL_THREADS);
    size_t sm = L::COL_SMEM;
    switch (op) {
    case COL_PROBE_INV:
        smem_attr(k_col<N, COL_PROBE_INV>, sm);
        k_col<N, COL_PROBE_INV><<<grid, block, sm, st>>>(a);
        break;
    case COL_STEP:
        smem_attr(k_col<N, COL_STEP>, sm);
        k_col<N, COL_STEP><<<grid, block, sm, st>>>(a);
        break;
    case COL_INV:
        smem_attr(k_col<N, COL_INV>, sm);
        k_col<N, COL_INV><<<grid, block, sm, st>>>(a);
        break;
    case COL_CTF_INV:
        smem_attr(k_col<N, COL_CTF_INV>, sm);
        k_col<N, COL_CTF_INV><<<grid, block, sm, st>>>(a);
        break;
    case COL_STEP_SEP:
        smem_attr(k_col<N, COL_STEP_SEP>, sm);
        k_col<N, COL_STEP_SEP><<<grid, block, sm, st>>>(a);
        break;
    case COL_SEED:
        smem_attr(k_col<N, COL_SEED>, sm);
        k_col<N, COL_SEED><<<grid, block, sm, st>>>(a);
        break;
    case COL_GRAD_PROBE:
        smem_attr(k_col<N, COL_GRAD_PROBE>, sm);
        k_col<N, COL_GRAD_PROBE><<<grid, block, sm, st>>>(a);
        break;
    default: throw MsError(MS_ERR_INTERNAL, "unknown column pass");
    }
}

}  // namespace msb

#include "slice_engine.cuh"

namespace msb {

template <int N>
bool engine_dispatch(int rowop, const PassArgs& a, const EngineArgs& e, int nwaves, cudaStream_t st)
{
    using L = FftLayout<N>;
    using EL = EngineLayout<N>;
    if (((uintptr_t)a.psi & 15) != 0 || e.n_items <= 0) return false;
    CUtensorMap map;
    if (!encode_wave_tile_map(&map, a.psi, N, (int64_t)nwaves * N, 2 * L::TC, N < 256 ? N : 256)) return false;
    auto kern = rowop != ROW_INV_TT_FWD          ? k_slice_engine<N, ROW_INV_T_FWD, L2_DEFAULT>
                : a.l2_mode == L2_WAVES_RESIDENT ? k_slice_engine<N, ROW_INV_TT_FWD, L2_WAVES_RESIDENT>
                : a.l2_mode == L2_SHARED_T       ? k_slice_engine<N, ROW_INV_TT_FWD, L2_SHARED_T>
                                                 : k_slice_engine<N, ROW_INV_TT_FWD, L2_DEFAULT>;
    smem_attr(kern, EL::SMEM);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, EL::THREADS, EL::SMEM);
    const int64_t blocks = std::min<int64_t>(e.n_items, (int64_t)num_sms() * std::max(1, per_sm));
    kern<<<(unsigned)blocks, EL::THREADS, EL::SMEM, st>>>(a, e, map);
    return true;
}

}  // namespace msb
