/*
 * ref_loop.cu -- TEST INFRASTRUCTURE ONLY (reference-kernel shim).
 *
 * The reference's composed slice loop, driven through its own cuFFT wrapper and load
 * callbacks, compiled unchanged from the reference tree:
 *   FFT_Dev               (fft_dev.cuh:69-190)     2-D cuFFT plans, single and batched
 *   CB_ComplexValLD_R/RB  (fftcallbacks.cuh:36-64) load callback psi * exp(i V)
 *   CB_ComplexValLD_C/CB  (fftcallbacks.cuh:11-35) load callback Psi * P
 * in the order of Wave_Function::wave_modulation / wave_modulation_batch
 * (wave_function.cuh:60-87): for every slice but the last, a forward FFT whose load
 * callback applies the transmission of that slice (Transmission_Function::transmit /
 * transmit_batch, transmission_function.cuh:100-119) and an inverse FFT whose load
 * callback applies the propagator (Propagator::propagate / propagate_batch,
 * propagation_function.cuh:41-48); the last slice only transmits, leaving the exit wave in
 * reciprocal space.  The transmission and the propagator have plans of their own
 * (fft_trans_dev and fft_prop_dev, multislice_params_dev.cuh:74-75, :197-198).  Everything is
 * float, as the reference's T = float build; the callbacks need the static cuFFT library
 * and relocatable device code (oracle/Makefile, target `ref`).
 *
 * The batched callbacks broadcast the potential and the propagator with the compile-time
 * PROBE_DIM * PROBE_DIM (fftcallbacks.cuh:28, :55), so the batched entry point requires the
 * grid to be PROBE_DIM x PROBE_DIM.
 */
#include <cufft.h>
#include <cufftXt.h>

#include <cstdio>
#include <iostream>   // fft_dev.cuh prints with std::cout and relies on a missing header for it

#define PROBE_DIM 256   // the batched callbacks' pixel count per wave (a missing host header's constant)

#include "host_basic_def.hpp"
#include "device_basic_def.cuh"
#include "fft_dev.cuh"
#include "fftcallbacks.cuh"

using namespace cudaEM;

namespace {

int ck(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        std::fprintf(stderr, "ref loop: %s: %s\n", what, cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

template <class P>
int callback_of(P* host_ptr, const P& dev_symbol)
{
    return ck(cudaMemcpyFromSymbol(host_ptr, dev_symbol, sizeof(P)), "callback pointer");
}

}  // namespace

extern "C" {

// n x n grid, S slices of phase V [S][n][n] (rad), B waves psi0 [B][n][n] (interleaved re, im),
// the propagator P [n][n] (interleaved); out [B][n][n] gets the exit waves in reciprocal space.
// B == 1 runs wave_modulation on the single plans, B > 1 wave_modulation_batch on the batched
// plans (n must then equal PROBE_DIM).  Returns 0 on success.
int ref_slice_loop(int n, int S, const float* V, int B, const float* psi0, const float* P, float* out)
{
    if (n <= 0 || S <= 0 || B <= 0 || (B > 1 && n != PROBE_DIM)) return 2;
    const size_t N = (size_t)n * n;
    float* dV = nullptr;          // all slices (the batched path's stored potentials)
    float* dV0 = nullptr;         // the single path's one-slice buffer V_0_ptr
    T_complex<float>* dP = nullptr;
    T_complex<float>* dw = nullptr;
    int rc = 0;
    rc |= ck(cudaMalloc(&dV, sizeof(float) * N * S), "malloc");
    rc |= ck(cudaMalloc(&dV0, sizeof(float) * N), "malloc");
    rc |= ck(cudaMalloc(&dP, sizeof(T_complex<float>) * N), "malloc");
    rc |= ck(cudaMalloc(&dw, sizeof(T_complex<float>) * N * B), "malloc");
    if (rc) return 1;
    rc |= ck(cudaMemcpy(dV, V, sizeof(float) * N * S, cudaMemcpyHostToDevice), "copy");
    rc |= ck(cudaMemcpy(dP, P, sizeof(T_complex<float>) * N, cudaMemcpyHostToDevice), "copy");
    rc |= ck(cudaMemcpy(dw, psi0, sizeof(T_complex<float>) * N * B, cudaMemcpyHostToDevice), "copy");
    {
        FFT_Dev<float> trans, prop;
        trans.create_plan_2d_many(n, n, B);
        prop.create_plan_2d_many(n, n, B);
        const cufftXtCallbackType_t type = get_callback_type<float>();
        T_Callback<float> cb_r, cb_rb, cb_c, cb_cb;
        rc |= callback_of(&cb_r, d_loadCBCPtr_R);
        rc |= callback_of(&cb_rb, d_loadCBCPtr_RB);
        rc |= callback_of(&cb_c, d_loadCBCPtr_C);
        rc |= callback_of(&cb_cb, d_loadCBCPtr_CB);
        if (B == 1) {
            // Propagator::attach_callback and Transmission_Function::attach_callback
            prop.attach_callback((void**)&cb_c, type, (void**)&dP);
            trans.attach_callback((void**)&cb_r, type, (void**)&dV0);
            int i = 0;
            for (; i < S - 1; i++) {
                rc |= ck(cudaMemcpy(dV0, dV + (size_t)i * N, sizeof(float) * N, cudaMemcpyDeviceToDevice), "slice");
                trans.forward(dw);
                prop.inverse(dw);
            }
            rc |= ck(cudaMemcpy(dV0, dV + (size_t)i * N, sizeof(float) * N, cudaMemcpyDeviceToDevice), "slice");
            trans.forward(dw);
            trans.deattach_callback(type);
            prop.deattach_callback(type);
        } else {
            prop.attach_callback_batch((void**)&cb_cb, type, (void**)&dP);
            int i = 0;
            for (; i < S; i++) {
                float* potent = dV + (size_t)i * N;
                trans.attach_callback_batch((void**)&cb_rb, type, (void**)&potent);
                trans.forward_batch(dw);
                trans.deattach_callback_batch(type);
                if (i < S - 1) prop.inverse_batch(dw);
            }
            prop.deattach_callback_batch(type);
        }
        rc |= ck(cudaDeviceSynchronize(), "loop");
    }
    rc |= ck(cudaMemcpy(out, dw, sizeof(T_complex<float>) * N * B, cudaMemcpyDeviceToHost), "copy");
    cudaFree(dV);
    cudaFree(dV0);
    cudaFree(dP);
    cudaFree(dw);
    return rc;
}

}  // extern "C"
