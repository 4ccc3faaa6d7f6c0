/*
 * ms_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of cudaEM's multislice operators.  It exists to
 * check the CUDA engine; nothing in the shipped library links, loads or
 * calls it.  Only tests/, __graft_entry__.smoke() and the cpu_baseline leg
 * of bench.py use it.
 *
 * Parity status: the reference publishes no golden vectors and its source
 * cannot be built as shipped (eleven headers are missing).  Its device
 * kernels do compile from their own files with the small constants header
 * in oracle/ref_shim/, so each per-pixel operator below (propagator, probe,
 * CTF and PCTF, detector sum, spline potential) is pinned against the
 * reference's own kernels on the same inputs (or_op_* entry points); the
 * host-side pieces whose sources are missing (slicing driver, phonon RNG,
 * quadrature tables, element tables) and the composed simulations rest on
 * the file:line restatement plus physics invariants.
 */
#ifndef MS_ORACLE_H
#define MS_ORACLE_H
#include <stdint.h>
#include "../include/cudaem_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* physics */
void or_physics(double E0_kV, double* lambda, double* sigma, double* gamma);

/* deterministic Gaussian pair keyed by (seed, conf, atom, stream) */
double or_det_log(double s);
void or_gauss_pair(uint64_t seed, int conf, int64_t atom, int stream, double* g0, double* g1);
void or_displace(const ms_params* p, const ms_atoms* a, int conf, float* x, float* y, float* z);

/* slicing on float z: returns the number of slices, fills bounds (n+1) and atom_slice */
int or_slices(const ms_params* p, const float* z, int64_t n, float* bounds, int cap, int* atom_slice);

/* radial spline of one element (FP64): R2, c0..c3 with MS_NR entries each */
int or_spline(const ms_params* p, int Z, double* R2, double* c0, double* c1, double* c2, double* c3,
              double* rmax);
/* projected potential V_z(R) and dV_z/dR^2 of one element (before tapering) */
int or_projected(const ms_params* p, int Z, double R, double* Vz, double* dVz_dR2);

/* sigma-scaled projected potentials of configuration conf: V[n_slices][ny][nx] (rad) */
int or_potential(const ms_params* p, const ms_atoms* a, int conf, double* V, int64_t cap,
                 int* n_slices, double* z_init);

/* unnormalised 2-D FFT, sign -1 forward, +1 inverse; data interleaved re,im */
void or_fft2(double* data, int nx, int ny, int sign);

/* simulators: outputs in double, same layouts as ms_output */
int or_simulate_tem(const ms_params* p, const ms_atoms* a, double* img, double* re, double* im);
int or_simulate_cbed(const ms_params* p, const ms_atoms* a, double* img, double* re, double* im);
int or_simulate_stem(const ms_params* p, const ms_atoms* a, double* stem);
int or_simulate_thickness(const ms_params* p, const ms_atoms* a, double* frames, int64_t cap,
                          int* n_frames);

/* CBED with the wave, FFTs, transmission and propagator in FP32 (the CPU baseline's FP32 figure) */
int or_simulate_cbed_f32(const ms_params* p, const ms_atoms* a, double* img);

/* HRTEM defocus series: images at objective C10 + df[i], [nd][ny][nx] */
int or_simulate_tem_series(const ms_params* p, const ms_atoms* a, int nd, const double* df, double* img, double* re,
                           double* im);

/* the slice loop alone (wave_modulation) on caller phases V[S][ny][nx] and incident waves psi0
   [B][ny][nx] (interleaved complex): the exit waves in reciprocal space into out */
int or_slice_loop(const ms_params* p, const float* V, int S, int B, const double* psi0, double* out);

/* raw STEM forward / adjoint on caller phase arrays V[n_slices][ny][nx] */
int or_stem_forward_potential(const ms_params* p, const float* V, int n_slices, double z_init,
                              const double* probe_xy, int n_probe, double* I);
int or_stem_backward(const ms_params* p, const float* V, int n_slices, double z_init,
                     const double* probe_xy, int n_probe, const float* target, double* loss,
                     double* dL_dV, double* dL_dC10, double* dL_dC30);
/* central differences of the same loss L = sum (I - target)^2 of the FP64 forward: with respect to
   single potential pixels (flat index idx[j] into V, step h[j]) and to the condenser C10 and C30
   (steps h10, h30); fd_pix[j] = (L(V + h e_j) - L(V - h e_j)) / (2 h[j]) */
int or_stem_loss_fd(const ms_params* p, const float* V, int n_slices, double z_init, const double* probe_xy,
                    int n_probe, const float* target, int n_pix, const int64_t* idx, const double* h,
                    double h10, double h30, double* fd_pix, double* fd_c10, double* fd_c30);

/* operator-level entry points, checked against the reference's own kernels (ref_shim/):
   propagator table, k-space probe, CTF / PCTF (no inverse FFT), detector sums, and the slice
   potential of atoms of one element; complex arrays interleaved re, im */
int or_op_propagator(const ms_params* p, double* P);
int or_op_probe(const ms_params* p, double px, double py, double z_init, double* W);
int or_op_ctf(const ms_params* p, int pctf, double c10_shift, double gxu, double gyu, const double* in, double* out);
int or_op_detect(const ms_params* p, const double* W, double* Iout);
int or_op_slice_potential(const ms_params* p, int Z, int64_t n, const float* x, const float* y, const float* occ,
                          double* V);

/* fine slicing: Gauss-Legendre quadrature on [-1/2, 1/2] (weights sum to 1) and the spline of
   one atom's potential integrated over a slice of thickness dzs whose middle lies a above it */
void or_gauss_legendre_half(int n, double* x, double* w);
int or_fine_spline_table(const ms_params* p, int Z, double a, double dzs, double* R2, double* c0, double* c1,
                         double* c2, double* c3);

/* Gauss-Hermite quadrature for exp(-x^2), weights normalised to sum 1 */
void or_gauss_hermite(int n, double* x, double* w);

/* number of OpenMP threads the oracle uses (0 = runtime default) */
void or_set_threads(int n);
int or_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
