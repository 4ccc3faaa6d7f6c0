/*
 * ref_kernels.cu -- TEST INFRASTRUCTURE ONLY (reference-kernel shim).
 *
 * A C-ABI wrapper that runs cudaEM's own device kernels, compiled unchanged from the
 * reference tree (device_kernels.cuh and the headers it includes) with the constants
 * of host_basic_def.hpp in this directory, so that the oracle's restatement of each
 * operator can be checked against the reference's code on the same inputs:
 *   gen_propagator_kernel  (device_kernels.cuh:215-234)  Fresnel propagator P(k)
 *   Generate_probe         (device_kernels.cuh:363-388)  convergent probe in k-space
 *   apply_CTF_kernel       (device_kernels.cuh:445-468)  objective-lens CTF
 *   apply_PCTF_kernel      (device_kernels.cuh:505-518)  partially coherent CTF
 *   sum_square_over_Det    (device_kernels.cuh:535-579)  annular detector sum
 *   gen_slice_potential_kernel (device_kernels.cuh:28-47) spline potential of a slice
 * Everything runs in float, as the reference's T = float build.  Built by
 * oracle/Makefile (target `ref`) into oracle/_ref/ where the reference tree is present;
 * nothing in the engine links or loads it.
 */
#include <cmath>
#include <cstdio>
#include <vector>

#include "device_kernels.cuh"

using namespace cudaEM;

namespace {

int ck(cudaError_t e)
{
    if (e != cudaSuccess) {
        std::fprintf(stderr, "ref shim: %s\n", cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

Grid_2d_Dev<float> make_grid(int nx, int ny, double lx, double ly, double dz, int bwl)
{
    Grid_2d_Dev<float> g;
    g.set_input_data(nx, ny, (float)lx, (float)ly, (float)dz, bwl != 0);
    return g;
}

// Lens_Dev with the round-symmetric aberrations C10, C30, C50 (lens_dev.cuh:40-57: c_c_10 =
// -pi C10 lambda, c_c_30 = -pi C30 lambda^3 / 2, c_c_50 = -pi C50 lambda^5 / 3), the aperture
// as squared frequencies, and the spreads of the partially coherent model (dsf_iehwgd =
// sqrt(2) dsf_sigma, lens_dev.cuh:138-142).
Lens_Dev<float> make_lens(double lambda, double c10, double c30, double c50, float g2min, float g2max,
                          double dsf_sigma, double ssf_beta)
{
    Lens_Dev<float> L;
    L.m = 0;
    L.c_10 = (float)c10;
    L.c_30 = (float)c30;
    L.lambda = (float)lambda;
    L.lambda_squared = (float)(lambda * lambda);
    L.c_c_10 = (float)(-c_Pi * c10 * lambda);
    L.c_c_12 = L.c_c_21 = L.c_c_23 = 0.f;
    L.c_c_30 = (float)(-c_Pi * c30 * lambda * lambda * lambda / 2.0);
    L.c_c_32 = L.c_c_34 = L.c_c_41 = L.c_c_43 = L.c_c_45 = 0.f;
    L.c_c_50 = (float)(-c_Pi * c50 * std::pow(lambda, 5) / 3.0);
    L.c_c_52 = L.c_c_54 = L.c_c_56 = 0.f;
    L.phi_12 = L.phi_21 = L.phi_23 = L.phi_32 = L.phi_34 = L.phi_41 = L.phi_43 = L.phi_45 = 0.f;
    L.phi_52 = L.phi_54 = L.phi_56 = 0.f;
    L.g2_min = g2min;
    L.g2_max = g2max;
    L.dsf_sigma = (float)dsf_sigma;
    L.dsf_iehwgd = (float)(c_2i2 * dsf_sigma);
    L.ssf_beta = (float)ssf_beta;
    return L;
}

dim3 blocks2d(int nx, int ny) { return dim3((nx + c_thrnxny - 1) / c_thrnxny, (ny + c_thrnxny - 1) / c_thrnxny); }

}  // namespace

extern "C" {

// P(k) of one slice: update_prop_function(0, 0, dz) with propagator_factor = -pi lambda
// (propagation_function.cuh:31, :49-57).  out: nx*ny interleaved re, im.
int ref_propagator(int nx, int ny, double lx, double ly, double dz, int bwl, double lambda, float* out)
{
    Grid_2d_Dev<float> g = make_grid(nx, ny, lx, ly, dz, bwl);
    T_complex<float>* d = nullptr;
    if (ck(cudaMalloc(&d, sizeof(T_complex<float>) * nx * ny))) return 1;
    gen_propagator_kernel<float><<<blocks2d(nx, ny), dim3(c_thrnxny, c_thrnxny)>>>(
        g, (float)(dz * (-c_Pi * lambda)), 0.f, 0.f, d);
    int r = ck(cudaMemcpy(out, d, sizeof(T_complex<float>) * nx * ny, cudaMemcpyDeviceToHost));
    cudaFree(d);
    return r;
}

// Probe in reciprocal space before its inverse FFT (generate_incident_beam, incident_wave.cuh:
// 29-46) at x = -2 pi px, y = -2 pi py (exp_factor_x_pos with x_b - L/2 = px, grid_dev.cuh:104-111).
int ref_probe(int nx, int ny, double lx, double ly, double lambda, double c10, double c30, float g2min,
              float g2max, double px, double py, float* out)
{
    Grid_2d_Dev<float> g = make_grid(nx, ny, lx, ly, 1.0, 0);
    Lens_Dev<float> L = make_lens(lambda, c10, c30, 0.0, g2min, g2max, 0.0, 0.0);
    T_complex<float>* d = nullptr;
    if (ck(cudaMalloc(&d, sizeof(T_complex<float>) * nx * ny))) return 1;
    Generate_probe<float><<<blocks2d(nx, ny), dim3(c_thrnxny, c_thrnxny)>>>(
        g, L, (float)(-c_2Pi * px), (float)(-c_2Pi * py), 0.f, 0.f, d);
    int r = ck(cudaMemcpy(out, d, sizeof(T_complex<float>) * nx * ny, cudaMemcpyDeviceToHost));
    cudaFree(d);
    return r;
}

// Objective lens on a reciprocal-space wave: pctf = 0 apply_CTF_kernel with the frequency
// shift (gxu, gyu); pctf = 1 apply_PCTF_kernel with the spreads.  in/out: interleaved re, im.
int ref_ctf(int nx, int ny, double lx, double ly, double lambda, double c10, double c30, float g2min, float g2max,
            int pctf, double dsf_sigma, double ssf_beta, double gxu, double gyu, const float* in, float* out)
{
    Grid_2d_Dev<float> g = make_grid(nx, ny, lx, ly, 1.0, 0);
    Lens_Dev<float> L = make_lens(lambda, c10, c30, 0.0, g2min, g2max, dsf_sigma, ssf_beta);
    T_complex<float> *di = nullptr, *dout = nullptr;
    const size_t b = sizeof(T_complex<float>) * nx * ny;
    if (ck(cudaMalloc(&di, b)) || ck(cudaMalloc(&dout, b))) return 1;
    if (ck(cudaMemcpy(di, in, b, cudaMemcpyHostToDevice))) return 1;
    if (pctf)
        apply_PCTF_kernel<float><<<blocks2d(nx, ny), dim3(c_thrnxny, c_thrnxny)>>>(g, L, di, dout);
    else
        apply_CTF_kernel<float><<<blocks2d(nx, ny), dim3(c_thrnxny, c_thrnxny)>>>(g, L, (float)gxu, (float)gyu, di,
                                                                                  dout);
    int r = ck(cudaMemcpy(out, dout, b, cudaMemcpyDeviceToHost));
    cudaFree(di);
    cudaFree(dout);
    return r;
}

// Annular detector sum over g2min <= g^2 <= g2max: the block partial sums of
// sum_square_over_Det added on the host (integrated_intensity, wave_function.cuh:135-146).
int ref_detector(int nx, int ny, double lx, double ly, float g2min, float g2max, const float* in, double* sum)
{
    Grid_2d_Dev<float> g = make_grid(nx, ny, lx, ly, 1.0, 0);
    T_complex<float>* di = nullptr;
    float* dp = nullptr;
    const size_t b = sizeof(T_complex<float>) * nx * ny;
    const dim3 grid(4, 4);
    if (ck(cudaMalloc(&di, b)) || ck(cudaMalloc(&dp, sizeof(float) * 16))) return 1;
    if (ck(cudaMemcpy(di, in, b, cudaMemcpyHostToDevice))) return 1;
    sum_square_over_Det<float><<<grid, dim3(c_thrnxny, c_thrnxny)>>>(g, g2min, g2max, di, dp);
    float part[16];
    int r = ck(cudaMemcpy(part, dp, sizeof(part), cudaMemcpyDeviceToHost));
    double s = 0.0;
    for (float v : part) s += v;
    *sum = s;
    cudaFree(di);
    cudaFree(dp);
    return r;
}

// Projected potential of one slice from per-atom cubic splines (c_nR nodes each, the same
// table for every atom): gen_slice_potential_kernel with coeff = sigma_factor.
int ref_potential(int nx, int ny, double lx, double ly, int n_atoms, const float* x, const float* y,
                  const float* occ, const float* R2, const float* c0, const float* c1, const float* c2,
                  const float* c3, double rmax, double coeff, float* V)
{
    Grid_2d_Dev<float> g = make_grid(nx, ny, lx, ly, 1.0, 0);
    float *dR2, *dc0, *dc1, *dc2, *dc3, *dV;
    const size_t tb = sizeof(float) * c_nR;
    if (ck(cudaMalloc(&dR2, tb)) || ck(cudaMalloc(&dc0, tb)) || ck(cudaMalloc(&dc1, tb)) ||
        ck(cudaMalloc(&dc2, tb)) || ck(cudaMalloc(&dc3, tb)) || ck(cudaMalloc(&dV, sizeof(float) * nx * ny)))
        return 1;
    cudaMemcpy(dR2, R2, tb, cudaMemcpyHostToDevice);
    cudaMemcpy(dc0, c0, tb, cudaMemcpyHostToDevice);
    cudaMemcpy(dc1, c1, tb, cudaMemcpyHostToDevice);
    cudaMemcpy(dc2, c2, tb, cudaMemcpyHostToDevice);
    cudaMemcpy(dc3, c3, tb, cudaMemcpyHostToDevice);
    cudaMemset(dV, 0, sizeof(float) * nx * ny);
    std::vector<Combined_Element_Coeff_Ptrs<float>> at((size_t)n_atoms);
    for (int i = 0; i < n_atoms; i++) {
        at[i].x = x[i];
        at[i].y = y[i];
        at[i].occ = occ[i];
        at[i].z_middle = 0.f;
        at[i].R_tap_squared = 0.f;
        at[i].tap_cf = 0.f;
        at[i].R_min_squared = R2[0];
        at[i].R_max_squared = (float)(rmax * rmax);
        at[i].R2_dev = dR2;
        at[i].c0_dev = dc0;
        at[i].c1_dev = dc1;
        at[i].c2_dev = dc2;
        at[i].c3_dev = dc3;
        at[i].cl_dev = nullptr;
        at[i].cnl_dev = nullptr;
    }
    Combined_Element_Coeff_Ptrs<float>* dat = nullptr;
    if (ck(cudaMalloc(&dat, sizeof(Combined_Element_Coeff_Ptrs<float>) * (n_atoms > 0 ? n_atoms : 1)))) return 1;
    cudaMemcpy(dat, at.data(), sizeof(Combined_Element_Coeff_Ptrs<float>) * n_atoms, cudaMemcpyHostToDevice);
    gen_slice_potential_kernel<float><<<blocks2d(nx, ny), dim3(c_thrnxny, c_thrnxny)>>>(g, dat, dV, n_atoms,
                                                                                        (float)coeff);
    int r = ck(cudaMemcpy(V, dV, sizeof(float) * nx * ny, cudaMemcpyDeviceToHost));
    cudaFree(dR2);
    cudaFree(dc0);
    cudaFree(dc1);
    cudaFree(dc2);
    cudaFree(dc3);
    cudaFree(dV);
    cudaFree(dat);
    return r;
}

}  // extern "C"
