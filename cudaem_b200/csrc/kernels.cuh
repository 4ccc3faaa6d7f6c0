// Device data structures and launchers of the engine's kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "engine.hpp"

namespace msb {

// One wave of a batch.
struct WaveInfo {
    double px = 0.0, py = 0.0;   // probe position, Angstrom
    double cc10 = 0.0;           // -pi (C10 + z_init) lambda of the probe, gated like Lens_Dev
    int conf_slot = 0;           // which potential slot (configuration) the wave reads
    int n_slices = 0;            // slices of the wave's specimen
    float weight = 1.0f;         // configuration weight
    int pos = 0;                 // output index (scan position) of the wave
    const float* sV = nullptr;      // if set: this wave's own potential store [slice][ny][nx] (uneven batches)
    const float2* prop = nullptr;   // if set: this wave's own propagator table [2][ny][nx] (hi, lo planes)
};

struct GridDev {
    int nx, ny;
    float dgx_f, dgy_f;
    double dgx, dgy;
    float gl2_f, alpha_f;
    int bwl;
    float inv_n;
    double lx, ly;     // box, Angstrom
    double g0x, g0y;   // beam tilt as a spatial frequency (gx_0, gy_0: multislice_params_dev.cuh:201-208)
};

struct LensDev {
    int m, phi_req;
    double cc10, cc12, cc21, cc23, cc30, cc32, cc34, cc41, cc43, cc45, cc50, cc52, cc54, cc56;
    double p12, p21, p23, p32, p34, p41, p43, p45, p52, p54, p56;
    float g2min, g2max;
    // image-forming lens only (COL_CTF_INV): frequency shift of a source point, amplitude
    // factor, and the partially coherent envelope (pctf = 1) with
    // pe_a = pi beta D, pe_b = pi D lambda, pe_c = pi beta, pe_d = C30 lambda^2, pe_e = C10
    double gxu, gyu, amp;
    int pctf;
    double pe_a, pe_b, pe_c, pe_d, pe_e;
};

enum RowOp {
    ROW_T_FWD = 0,
    ROW_INV_T_FWD = 1,
    ROW_INV_ABS2 = 2,
    ROW_INV_STORE = 3,
    ROW_ADJ = 4,
    ROW_INV_T_FWD_X = 5,  // ROW_INV_T_FWD that also keeps t psi in xs (selected by PF_STORE_X)
    ROW_INV_TT_FWD = 6,   // ROW_INV_T_FWD with t = exp(i V) read from a transmission store (selected by tt)
    ROW_TT_FWD = 7        // ROW_T_FWD likewise
};
enum ColOp {
    COL_PROBE_INV = 0,
    COL_STEP = 1,
    COL_INV = 2,
    COL_CTF_INV = 3,
    COL_STEP_SEP = 4,
    COL_SEED = 5,        // adjoint seed: annulus-weighted residuals times Psi, then inverse column FFT
    COL_GRAD_PROBE = 6   // adjoint end: forward column FFT, then the lens-phase gradient sums
};

enum PassFlags {
    PF_VACUUM_BEYOND = 1,  // slices past a wave's own count are empty (t = 1) instead of skipped
    PF_ACCUMULATE = 2,     // ROW_INV_ABS2 adds into its output
    PF_FILTER_AUX = 4,     // COL_STEP also writes the annulus-filtered spectrum to aux
    PF_PROP_ALWAYS = 8,    // COL_STEP propagates even after the wave's last slice
    PF_STORE_X = 16,       // ROW_INV_T_FWD also writes the transmitted real-space wave to xs
    PF_CONJ_PROP = 32,     // COL_STEP multiplies by conj(P) (the adjoint step)
    PF_WAVE_DEFOCUS = 64,  // COL_CTF_INV takes each wave's own defocus term (WaveInfo.cc10) instead of the lens's
    PF_TILT_INCIDENT = 128, // ROW_T_FWD / ROW_TT_FWD start from the tilted plane wave exp(2 pi i g0.(r - L/2))
    PF_TEST_WAIT = 256      // fault injection: the TMA column pass waits for bytes that never come
};

struct PassArgs {
    float2* psi;            // [B][ny][nx]
    float2* aux;            // [B][ny][nx] (filtered branch, complex outputs)
    float* out_real;        // [B][ny][nx] or a frame
    const WaveInfo* waves;  // [B]
    int slice;
    int flags;
    const float* sV;          // potential store, [slot][slice][ny][nx], rad
    const float2* tt;         // or, if set, the transmission store exp(i sV) with the same layout
    int64_t sV_slot_stride;   // elements per slot
    int sV_slice_base;        // slice index held at the store's slice 0
    const float2* tw;         // inter-level twiddles for this pass's length
    const float2* prop_x;     // [nx] exp(i w (gx - g0x)^2)
    const float2* prop_y;     // [ny] exp(i w (gy - g0y)^2)
    const float2* prop;       // [kPropSets][ny][nx] full propagator P(k) including 1/N and the band limit (dithered)
    const float2* propT;      // the same tables transposed, [kPropSets][nx][ny] (the warp-column step), or null
    const float2* exptab;     // [1024] exp(2 pi i k / 1024) for the transmission
    GridDev grid;
    LensDev lens;
    float filt_g2in, filt_g2out;
    // adjoint
    float2* xs;               // [B][ny][nx] transmitted real-space waves t_s psi_s of one slice
    float* dV;                // [B][ny][nx] each wave's dL/dV contribution of one slice
    const double* resid;      // [B][ndet] 4 (I - target) per wave and detector
    const float* det_thr;     // [2][ndet] inner, outer g^2 thresholds
    int ndet;
    double* chi_part;         // [B][nx / TC][2] partial sums of g^2 q and g^4 q
    int variant;              // PassVariant of the row / column pass kernels (host side only)
    int tile;                 // TileShape of the classic hot passes (host side only)
    int l2_mode;              // L2Mode: eviction priorities of the wave and transmission accesses
    int* err;                 // device word set to a nonzero code when a bounded device-side wait runs out
    long long wait_cycles;    // limit of such a wait in clock cycles (0: about one second)
};

// L2 eviction priorities of the slice passes' wave stores and transmission loads.
enum L2Mode {
    L2_DEFAULT = 0,         // no priority
    L2_WAVES_RESIDENT = 1,  // the batch's waves fit in L2: waves evict-last, transmission evict-first
    L2_SHARED_T = 2         // one transmission slice serves every wave: transmission evict-last, waves evict-first
};

// The persistent slice engine's bookkeeping (slice_engine.cuh).  The ticket, the per-wave item
// counters and the completion times live in device memory and start at zero.
struct EngineState {
    unsigned ticket;
    unsigned pad[31];
};
struct EngineArgs {
    EngineState* state;
    const int* phase_start;        // [2 S_max + 1]: first ticket of (slice slice0 + j, phase), k = 2 j + (column)
    int n_items, S_max;            // S_max: slices in the launch (slice0 .. slice0 + S_max - 1)
    int slice0;                    // first slice of the launch (earlier slices are done)
    int sub;                       // row blocks / column tiles per work item (a power of two <= 8)
    unsigned* rows_done;           // [nwaves] row items done (all slices)
    unsigned* cols_done;           // [nwaves] column items done
    unsigned long long* done_ns;   // [nwaves] device clock when the wave's last slice was done (may be null)
    long long wait_cycles;         // limit of a dependency wait (0: about one second)
};

// Kernel form of ROW_INV_T_FWD and COL_STEP.  PASS_CLASSIC (the default) launches the classic
// one-block-per-tile kernels slice by slice for CBED / TEM / STEM (measured fastest there) and runs
// an uneven batch's grid groups in the persistent slice engine (measured 1.35x faster there, with
// half the completion latency); PASS_PIPELINED the persistent pipelined kernels (grids of
// 128..1024 points); PASS_ENGINE the slice engine everywhere; PASS_PER_SLICE the classic kernels
// everywhere.  All compute the same operations.
enum PassVariant { PASS_CLASSIC = 0, PASS_PIPELINED = 1, PASS_ENGINE = 2, PASS_PER_SLICE = 3 };

// Spatial cells of the atom binning: a ncx x ncy grid of square cells of side 1/inv_cell.
struct CellGrid {
    int ncx, ncy;
    float inv_cell;
    float lx, ly;
    int wrap;
};

// Sorted atoms of a group of configurations.
struct PotArgs {
    const float* ax;
    const float* ay;
    const float* aw;            // Vr_factor * occupancy
    const int* ae;              // element index | (wrap count x + 8) << 8 | (wrap count y + 8) << 12
    const unsigned* seg;        // [n_conf][S_cap + 1][ncx*ncy] + 1 start offsets of each (conf, slice, cell)
    const int* ns;              // slices per configuration
    int S_cap;                  // slice slots per configuration
    int slice0, nslice;         // slices computed by this launch
    float* V;                   // [n_conf][S_cap][ny][nx] (or [n_conf][nslice][...] with slice0 offset)
    int64_t V_conf_stride;      // floats per configuration in V
    int V_slice_base;           // slice index stored at V's slice 0
    int nx, ny;
    float dx, dy, lx, ly;
    float dx_hi, dx_lo, dy_hi, dy_lo;  // sampling split in two floats: ix*dx - x is formed to float accuracy
    int wrap;
    int ncx, ncy;
    float inv_cell;
    float rmax_all;             // largest cut-off radius of the elements
    const ElemTable* elems;
    int n_elem;
    const float4* pair_coef;    // fine slicing: spline coefficients of every sorted (atom, slice) pair
    float2* T;                  // if set: write the transmission exp(i V) here instead of V
    const float2* exptab;       // [1024] exp(2 pi i k / 1024) for the transmission
};

struct ElemCoefDev;

// slice passes of one transform length (passes_<N>.cu)
template <int N>
void row_dispatch(int op, const PassArgs& a, int nwaves, int ny, cudaStream_t st);
// the persistent slice engine over nwaves square N x N waves (rowop ROW_INV_TT_FWD or
// ROW_INV_T_FWD); false when it cannot run here (the tensor map could not be made)
template <int N>
bool engine_dispatch(int rowop, const PassArgs& a, const EngineArgs& e, int nwaves, cudaStream_t st);
template <int N>
void col_dispatch(int op, const PassArgs& a, int nwaves, int nx, cudaStream_t st);

// launchers (kernels.cu); all asynchronous on `st`
void launch_row(int N, int op, const PassArgs& a, int nwaves, int ny, cudaStream_t st);
void launch_stamp(unsigned long long* dst, cudaStream_t st);   // *dst = the device clock (ns)
bool launch_slice_engine(int N, int rowop, const PassArgs& a, const EngineArgs& e, int nwaves, cudaStream_t st);
// rows of one engine row item and columns of one column item at transform length N
int engine_rows(int N);
int num_sms();   // streaming multiprocessors of the current device
bool tensor_maps_available();   // the driver offers tensor-map encoding (TMA tile loads)
int engine_cols(int N);
void launch_col(int N, int op, const PassArgs& a, int nwaves, int nx, cudaStream_t st);
size_t row_smem(int N);
size_t col_smem(int N);
void launch_potential(const PotArgs& a, int n_conf, cudaStream_t st);
void launch_prop_table(int nx, int ny, double dgx, double dgy, double g0x, double g0y, double w, double alpha,
                       double gl2, int bwl, float2* P, cudaStream_t st, float2* PT = nullptr);

// specimen on the device
void launch_displace(const float* x, const float* y, const float* z, const float* sig, int64_t n, const int* confs,
                     int nconf, uint64_t seed, int dx, int dy, int dzf, float* xd, float* yd, float* zd,
                     cudaStream_t st);
void launch_zrange(const float* zd, int64_t n, int nconf, unsigned* zmin_bits, unsigned* zmax_bits, cudaStream_t st);
void launch_assign(const float* xd, const float* yd, const float* zd, int64_t n, int nconf, const float* bounds,
                   int bstride, const int* nv, const float* vmax, int S_cap, const CellGrid& cg, unsigned* keys,
                   int* vals, unsigned* counts, cudaStream_t st);
void launch_gather(const unsigned* keys, const int* vals, int64_t total, int64_t n, int S_cap, const CellGrid& cg,
                   const float* xd, const float* yd, const float* occ, const int* elem, float vr_factor, float* ax,
                   float* ay, float* aw, int* ae, cudaStream_t st);
// fine slicing: (atom, slice) pairs, maxper slots per atom (unused slots carry the key nkeys),
// their gather (with the atom's z), and the slice-integrated spline of every pair
void launch_fine_assign(const float* xd, const float* yd, const float* zd, int64_t n, int nconf, const float* bounds,
                        int bstride, const int* nv, const float* zmax, int S_cap, const CellGrid& cg, float rint,
                        int maxper, unsigned nkeys, unsigned* keys, int* vals, unsigned* counts, cudaStream_t st);
void launch_fine_gather(const unsigned* keys, const int* vals, int64_t total, int64_t n, int S_cap, const CellGrid& cg,
                        unsigned nkeys, const float* xd, const float* yd, const float* zd, const float* occ,
                        const int* elem, float vr_factor, float* ax, float* ay, float* aw, int* ae, float* az,
                        cudaStream_t st);
void launch_fine_tables(const unsigned* keys, const float* az, const int* ae, const unsigned* seg, unsigned nkeys,
                        int64_t total, const float* bounds, int bstride, int S_cap, const CellGrid& cg,
                        const ElemCoefDev* coefs, double rmin, double rmax, const double* qz, float4* out,
                        cudaStream_t st);

// post-processing
void launch_detect(const float2* psi, int nwaves, int nx, int ny, float dgx, float dgy, const float* g2in,
                   const float* g2out, int ndet, double* partial, int nblk, cudaStream_t st);
void launch_det_finalize(const double* partial, int nwaves, int nblk, int ndet, const WaveInfo* waves,
                         double* I_wave, double* image, int npos, int accumulate, cudaStream_t st);
void launch_acc_abs2(const float2* psi, int nwaves, const WaveInfo* waves, int64_t N, double* acc, int first,
                     cudaStream_t st);
void launch_acc_cplx(const float2* psi, int nwaves, const WaveInfo* waves, int64_t N, double* re, double* im,
                     int first, cudaStream_t st);
void launch_acc_real(const float* in, int nwaves, int64_t N, double* acc, int first, cudaStream_t st);
void launch_emit(const double* acc, int nx, int ny, int shift, float* out, cudaStream_t st);
void launch_d2f(const double* in, int64_t n, float* out, cudaStream_t st);
void launch_scan_counts(const unsigned* counts, int n, int64_t* seg, cudaStream_t st);
void launch_fill_c(float2* p, int64_t n, float2 v, cudaStream_t st);

// adjoint helpers
void launch_resid(const double* I, const float* target, int n, double* resid, double* sq, cudaStream_t st);
void launch_chi_finalize(const double* part, int nwaves, int nparts, double* acc, cudaStream_t st);
// out[p] += sum over b = 0..nwaves-1, in that order, of in[b N + p]
void launch_sum_waves(const float* in, int nwaves, int64_t N, float* out, cudaStream_t st);
int col_tiles(int N, int nx);

int64_t kernel_launches();     // running count of this library's launches
void reset_kernel_launches();
void add_kernel_launches(int64_t n);   // launches replayed through (or captured into) a CUDA graph

}  // namespace msb
