// Kernels of the multislice engine other than the slice passes (passes.cuh): the propagator
// table, the projected potential, the specimen pipeline (displacement, slicing, sort, gather),
// fine slicing, detectors, accumulation and output, and the adjoint's helpers.
#include <cub/device/device_radix_sort.cuh>
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <utility>
#include <cfloat>

#include "detmath.cuh"
#include "devcommon.cuh"
#include "fft_layout.hpp"
#include "kernels.cuh"
#include "vr.cuh"

namespace msb {

static std::atomic<int64_t> g_launches{0};
int64_t kernel_launches() { return g_launches.load(); }
void reset_kernel_launches() { g_launches.store(0); }
void add_kernel_launches(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// Raises a kernel's dynamic shared-memory limit only when a launch needs more than the limit
// already set on this device (the attribute stays set for the process), instead of before every
// launch: the slice loop launches thousands of kernels per call and the host must keep ahead of
// them.  The limit is only ever raised: setting it lowers it too, below sizes launched before.
static std::mutex g_attr_mtx;
static std::map<std::pair<int, const void*>, size_t> g_attr_max;

void smem_attr_raw(const void* kernel, size_t bytes)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_pair(dev, kernel);
    std::lock_guard<std::mutex> lk(g_attr_mtx);
    auto it = g_attr_max.find(key);
    if (it != g_attr_max.end() && it->second >= bytes) return;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    g_attr_max[key] = bytes;
}

// cuTensorMapEncodeTiled, looked up once through the runtime's driver entry points (the library
// does not link the driver library).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = (PFN_cuTensorMapEncodeTiled_v12000)f;
        cudaGetLastError();
    });
    return encode;
}

bool tensor_maps_available() { return tensor_map_encoder() != nullptr; }

bool encode_wave_tile_map(void* map, const void* psi, int nx, int64_t rows, int box_cols, int box_rows,
                          bool swizzle64)
{
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)2 * nx, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)2 * nx * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return encode((CUtensorMap*)map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(psi), dims, strides, box,
                  estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  swizzle64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void check_launch(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw MsError(MS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int num_sms()
{
    static int n[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (!n[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        n[dev] = v > 0 ? v : 148;
    }
    return n[dev];
}

// Full propagator table in FP64 (gen_propagator_kernel, device_kernels.cuh:215-234), rounded to
// kPropSets dithered FP32 tables (fft_layout.hpp): P holds kPropSets * nx * ny entries, table t
// used by the slices s with s mod kPropSets = t.
__global__ void k_prop_table(int nx, int ny, double dgx, double dgy, double g0x, double g0y, double w, double alpha,
                             double gl2, int bwl, double inv_n, float2* P, float2* PT)
{
    int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y;
    if (ix >= nx) return;
    double gx = freq_d(ix, nx, dgx), gy = freq_d(iy, ny, dgy);
    double amp = inv_n;
    if (bwl) amp = amp / (1.0 + exp(alpha * (gx * gx + gy * gy - gl2)));
    double th = w * ((gx - g0x) * (gx - g0x) + (gy - g0y) * (gy - g0y));
    double s, c;
    sincos(th, &s, &c);
    dither_sets(amp * c, amp * s, kPropSets, P + (size_t)iy * nx + ix, (size_t)nx * ny);
    // the same tables transposed ([set][kx][ky]) for the warp-column step
    if (PT) dither_sets(amp * c, amp * s, kPropSets, PT + (size_t)ix * ny + iy, (size_t)nx * ny);
}

void launch_prop_table(int nx, int ny, double dgx, double dgy, double g0x, double g0y, double w, double alpha,
                       double gl2, int bwl, float2* P, cudaStream_t st, float2* PT)
{
    k_prop_table<<<dim3((nx + 127) / 128, ny), 128, 0, st>>>(nx, ny, dgx, dgy, g0x, g0y, w, alpha, gl2, bwl,
                                                             1.0 / ((double)nx * ny), P, PT);
    count_launch();
    check_launch("propagator table");
}

void launch_row(int N, int op, const PassArgs& a, int nwaves, int ny, cudaStream_t st)
{
    if (nwaves <= 0) return;
    switch (N) {
    case 128: row_dispatch<128>(op, a, nwaves, ny, st); break;
    case 256: row_dispatch<256>(op, a, nwaves, ny, st); break;
    case 512: row_dispatch<512>(op, a, nwaves, ny, st); break;
    case 1024: row_dispatch<1024>(op, a, nwaves, ny, st); break;
    case 2048: row_dispatch<2048>(op, a, nwaves, ny, st); break;
    default: throw MsError(MS_ERR_UNSUPPORTED, "unsupported row length");
    }
    count_launch();
    check_launch("row pass");
}

void launch_col(int N, int op, const PassArgs& a, int nwaves, int nx, cudaStream_t st)
{
    if (nwaves <= 0) return;
    switch (N) {
    case 128: col_dispatch<128>(op, a, nwaves, nx, st); break;
    case 256: col_dispatch<256>(op, a, nwaves, nx, st); break;
    case 512: col_dispatch<512>(op, a, nwaves, nx, st); break;
    case 1024: col_dispatch<1024>(op, a, nwaves, nx, st); break;
    case 2048: col_dispatch<2048>(op, a, nwaves, nx, st); break;
    default: throw MsError(MS_ERR_UNSUPPORTED, "unsupported column length");
    }
    count_launch();
    check_launch("column pass");
}

__global__ void k_stamp(unsigned long long* dst)
{
    unsigned long long ns;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(ns));
    *dst = ns;
}

void launch_stamp(unsigned long long* dst, cudaStream_t st)
{
    k_stamp<<<1, 1, 0, st>>>(dst);
    count_launch();
    check_launch("stamp");
}

bool launch_slice_engine(int N, int rowop, const PassArgs& a, const EngineArgs& e, int nwaves, cudaStream_t st)
{
    bool ok = false;
    switch (N) {
    case 128: ok = engine_dispatch<128>(rowop, a, e, nwaves, st); break;
    case 256: ok = engine_dispatch<256>(rowop, a, e, nwaves, st); break;
    case 512: ok = engine_dispatch<512>(rowop, a, e, nwaves, st); break;
    case 1024: ok = engine_dispatch<1024>(rowop, a, e, nwaves, st); break;
    case 2048: ok = engine_dispatch<2048>(rowop, a, e, nwaves, st); break;
    default: throw MsError(MS_ERR_UNSUPPORTED, "unsupported transform length");
    }
    if (ok) {
        count_launch();
        check_launch("slice engine");
    }
    return ok;
}

// the thread layout of the engine (slice_engine.cuh): threads = max(row, column threads)
template <int N>
static int engine_rows_n()
{
    using L = FftLayout<N>;
    return (L::ROW_THREADS > L::COL_THREADS ? L::ROW_THREADS : L::COL_THREADS) / L::G;
}
int engine_rows(int N)
{
    switch (N) {
    case 128: return engine_rows_n<128>();
    case 256: return engine_rows_n<256>();
    case 512: return engine_rows_n<512>();
    case 1024: return engine_rows_n<1024>();
    case 2048: return engine_rows_n<2048>();
    }
    throw MsError(MS_ERR_UNSUPPORTED, "unsupported transform length");
}
int engine_cols(int N) { return col_tiles(N, N) > 0 ? N / col_tiles(N, N) : 0; }

int col_tiles(int N, int nx)
{
    switch (N) {
    case 128: return nx / FftLayout<128>::TC;
    case 256: return nx / FftLayout<256>::TC;
    case 512: return nx / FftLayout<512>::TC;
    case 1024: return nx / FftLayout<1024>::TC;
    case 2048: return nx / FftLayout<2048>::TC;
    }
    throw MsError(MS_ERR_UNSUPPORTED, "unsupported column length");
}

// Residuals of the detector loss: resid = 4 (I - target), sq = (I - target)^2.
__global__ void k_resid(const double* I, const float* target, int n, double* resid, double* sq)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double r = I[i] - (double)target[i];
    resid[i] = 4.0 * r;
    sq[i] = r * r;
}

void launch_resid(const double* I, const float* target, int n, double* resid, double* sq, cudaStream_t st)
{
    k_resid<<<(n + 127) / 128, 128, 0, st>>>(I, target, n, resid, sq);
    count_launch();
    check_launch("loss residuals");
}

// Adds the per-wave planes of one slice's dL/dV into the gradient, wave by wave in a fixed order.
__global__ void k_sum_waves(const float* in, int nwaves, int64_t N, float* out)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    float s = out[p];
    for (int b = 0; b < nwaves; b++) s += in[(int64_t)b * N + p];
    out[p] = s;
}

void launch_sum_waves(const float* in, int nwaves, int64_t N, float* out, cudaStream_t st)
{
    k_sum_waves<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(in, nwaves, N, out);
    count_launch();
    check_launch("dL/dV sum over waves");
}

// Sums the lens-phase gradient partials of every wave in a fixed order into acc[0..1].
__global__ void k_chi_finalize(const double* part, int n, double* acc)
{
    __shared__ double red[2][256];
    double s2 = 0.0, s4 = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        s2 += part[2 * i];
        s4 += part[2 * i + 1];
    }
    red[0][threadIdx.x] = s2;
    red[1][threadIdx.x] = s4;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t2 = 0.0, t4 = 0.0;
        for (int k = 0; k < (int)blockDim.x; k++) {
            t2 += red[0][k];
            t4 += red[1][k];
        }
        acc[0] += t2;
        acc[1] += t4;
    }
}

void launch_chi_finalize(const double* part, int nwaves, int nparts, double* acc, cudaStream_t st)
{
    k_chi_finalize<<<1, 256, 0, st>>>(part, nwaves * nparts, acc);
    count_launch();
    check_launch("lens gradient sum");
}

size_t row_smem(int N)
{
    switch (N) {
    case 128: return FftLayout<128>::ROW_SMEM;
    case 256: return FftLayout<256>::ROW_SMEM;
    case 512: return FftLayout<512>::ROW_SMEM;
    case 1024: return FftLayout<1024>::ROW_SMEM;
    case 2048: return FftLayout<2048>::ROW_SMEM;
    }
    return 0;
}
size_t col_smem(int N)
{
    switch (N) {
    case 128: return FftLayout<128>::COL_SMEM;
    case 256: return FftLayout<256>::COL_SMEM;
    case 512: return FftLayout<512>::COL_SMEM;
    case 1024: return FftLayout<1024>::COL_SMEM;
    case 2048: return FftLayout<2048>::COL_SMEM;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// projected potential: gen_slice_potential_kernel (device_kernels.cuh:28-47)
// restructured as atom-culled 64x16 pixel tiles with float4 stores
// ---------------------------------------------------------------------------
constexpr int kPotTX = 64, kPotTY = 32, kPotThreads = 256;
constexpr int kPotRowsPerThread = kPotTY / (kPotThreads / (kPotTX / 4));   // 2 rows of 4 pixels

__device__ __forceinline__ float spline_eval(const ElemTable& T, float r2)
{
    // index of unrolledBinarySearch_c_nR (basic_functions_dev.cuh:47-67): the largest node
    // i <= nR-2 with R2[i] <= r2 (or 0).  The nodes are log-spaced, so the index is the floor of
    // log2(r2) on the node scale; a guess off by one (r2 within the log2 rounding, ~1e-6, of a
    // node) evaluates the neighbouring cubic a hair outside its interval, which the Hermite
    // spline's continuity of value and slope makes equal to 1e-12.
    // log2(r2) for r2 = 0 is -inf, which the floor conversion and the clamp turn into node 0
    int i = __float2int_rd(fmaf(__log2f(r2), T.inv_dl, T.l0s));
    i = min(max(i, 0), MS_NR - 2);
    float d = r2 - T.R2[i];
    const ElemCoef4 c = T.c[i];
    return ((c.c3 * d + c.c2) * d + c.c1) * d + c.c0;  // get_value_Cubic_Spline
}


// the same with the cubic coefficients read from a per-pair table (fine slicing)
__device__ __forceinline__ float spline_eval_c(const ElemTable& T, const float4* __restrict__ coef, float r2)
{
    int i = __float2int_rd(fmaf(__log2f(r2), T.inv_dl, T.l0s));
    i = min(max(i, 0), MS_NR - 2);
    float d = r2 - T.R2[i];
    const float4 c = __ldg(coef + i);
    return ((c.w * d + c.z) * d + c.y) * d + c.x;
}

constexpr int kPotMaxRanges = 64;

// Cells of one axis that hold the atoms of the interval [lo, hi]: with periodic wrapping, one piece
// per periodic image k that the interval reaches (at most three: a tile spans at most half the box
// and the cut-off stays below half the box), each the interval shifted by -k L,
// clipped to the box and turned into a cell range; without wrapping, one piece of cells clamped to
// the grid (atoms outside the box sit in the edge cells).  Atoms are binned by
// floor((x - k L) / cell) on the wrapped coordinate, so a range taken per image is exact even when
// L is not a multiple of the cell size.  Returns the number of pieces; b/e are the first and last
// cell, o the image.  Unrolled with constant indices, so the pieces stay in registers.
__device__ __forceinline__ int cell_pieces(float lo, float hi, float L, int nc, float inv_cell, bool wrap, int (&b)[3],
                                           int (&e)[3], int (&o)[3])
{
    int n = 0;
    if (!wrap) {
        b[0] = max((int)floorf(lo * inv_cell), 0);
        e[0] = min((int)floorf(hi * inv_cell), nc - 1);
        o[0] = 0;
        return b[0] <= e[0] ? 1 : 0;
    }
    const int k0 = (int)floorf(lo / L), k1 = (int)floorf(hi / L);
#pragma unroll
    for (int piece = 0; piece < 3; piece++) {
        const int k = k0 + piece;
        const int c0 = max((int)floorf(fmaxf(lo - (float)k * L, 0.f) * inv_cell), 0);
        const int c1 = min((int)floorf(fminf(hi - (float)k * L, L) * inv_cell), nc - 1);
        if (k <= k1 && c0 <= c1) {
            // n only grows, so pieces land at their own index or below (constant indices after unrolling)
            if (n == 0) { b[0] = c0; e[0] = c1; o[0] = k; }
            else if (n == 1) { b[1] = c0; e[1] = c1; o[1] = k; }
            else { b[2] = c0; e[2] = c1; o[2] = k; }
            n++;
        }
    }
    return n;
}

// WRAP is the periodic wrap of the specimen (a.wrap), a template argument so that the
// non-periodic kernel carries none of the per-image lookup code
template <bool FINE, bool WRAP>
__global__ void __launch_bounds__(kPotThreads, 8) k_potential(PotArgs a)
{
    extern __shared__ __align__(16) unsigned char psm[];
    ElemTable* el = reinterpret_cast<ElemTable*>(psm);
    float4* cand = reinterpret_cast<float4*>(psm + sizeof(ElemTable) * a.n_elem);
    unsigned* candp = reinterpret_cast<unsigned*>(cand + kPotThreads);   // fine slicing: pair index
    __shared__ int wsum[kPotThreads / 32];
    __shared__ int total_s;
    // per warp: the candidates whose disc reaches the warp's 16 x 16 pixel block (indices into cand)
    __shared__ unsigned short whit[kPotThreads / 32][kPotThreads];
    __shared__ unsigned r_beg[kPotMaxRanges], r_pre[kPotMaxRanges + 1];
    __shared__ int r_img[kPotMaxRanges];
    __shared__ int n_ranges;

    const int conf = blockIdx.z;
    const int sl = a.slice0 + blockIdx.y;
    const int tiles_x = a.nx / kPotTX;
    const int tx0 = (blockIdx.x % tiles_x) * kPotTX, ty0 = (blockIdx.x / tiles_x) * kPotTY;
    // Each warp owns a compact 16x16-pixel block of the 64x32 tile (4 x 2 blocks), each lane 4 pixels
    // in x on 2 rows, so a candidate atom far from a warp's block is skipped by the whole warp.
    const int t = threadIdx.x, wblk = t >> 5, ln = t & 31;
    const int px = (wblk % 4) * 4 + (ln % 4);          // in units of 4 pixels across the tile
    const int py = (wblk / 4) * 16 + (ln / 4);         // first row of the lane inside the tile
    constexpr int RY = kPotRowsPerThread, ROW_STEP = 8;
    float acc[RY][4];
#pragma unroll
    for (int r = 0; r < RY; r++)
#pragma unroll
        for (int k = 0; k < 4; k++) acc[r][k] = 0.f;

    if (sl < a.ns[conf]) {
        {
            const float4* src = reinterpret_cast<const float4*>(a.elems);
            float4* dst = reinterpret_cast<float4*>(el);
            int nv4 = (int)(sizeof(ElemTable) * a.n_elem / 16);
            for (int i = t; i < nv4; i += kPotThreads) dst[i] = src[i];
        }
        const float X0 = (float)tx0 * a.dx, X1 = (float)(tx0 + kPotTX - 1) * a.dx;
        const float Y0 = (float)ty0 * a.dy, Y1 = (float)(ty0 + kPotTY - 1) * a.dy;
        // this warp's block: pixels tx0 + [16 (wblk % 4), +16), ty0 + [16 (wblk / 4), +16), with a
        // margin of one pixel for the float rounding of the block corners
        const float WX0 = (float)(tx0 + (wblk % 4) * 16 - 1) * a.dx, WX1 = (float)(tx0 + (wblk % 4) * 16 + 16) * a.dx;
        const float WY0 = (float)(ty0 + (wblk / 4) * 16 - 1) * a.dy, WY1 = (float)(ty0 + (wblk / 4) * 16 + 16) * a.dy;
        if (t < 32) {
            // Atoms are sorted by (configuration, slice, cell) with cells of a.cell A in a
            // ncx x ncy grid over the box.  The tile needs the cells its rectangle, grown by the
            // largest cut-off, touches: one contiguous key range per cell row and periodic image.
            // Warp 0 looks the ranges up in parallel (one (row, image) item per lane) and keeps the
            // non-empty ones in item order, with their running atom counts.
            const int lane = t;
            const float R = a.rmax_all * 1.0001f + 1e-4f;
            const int64_t key_base = ((int64_t)conf * (a.S_cap + 1) + sl) * a.ncx * a.ncy;
            int xs_b[3] = {0, 0, 0}, xs_e[3] = {0, 0, 0}, xs_o[3] = {0, 0, 0};
            int ys_b[3] = {0, 0, 0}, ys_e[3] = {0, 0, 0}, ys_o[3] = {0, 0, 0};
            const int nxs = cell_pieces(X0 - R, X1 + R, a.lx, a.ncx, a.inv_cell, WRAP, xs_b, xs_e, xs_o);
            const int nys = cell_pieces(Y0 - R, Y1 + R, a.ly, a.ncy, a.inv_cell, WRAP, ys_b, ys_e, ys_o);
            const int ny0 = nys > 0 ? ys_e[0] - ys_b[0] + 1 : 0, ny1 = nys > 1 ? ys_e[1] - ys_b[1] + 1 : 0;
            const int ny2 = nys > 2 ? ys_e[2] - ys_b[2] + 1 : 0;
            // items: (cell row of a y piece, x piece), rows in image order, then x pieces in image order
            const int n_items = (ny0 + ny1 + ny2) * nxs;
            int nr = 0;
            unsigned run = 0;
            for (int base = 0; base < n_items && nr < kPotMaxRanges; base += 32) {
                const int it = base + lane;
                unsigned b0 = 0, b1 = 0;
                int img = 0;
                if (it < n_items) {
                    const int rr = it / nxs, xi = it % nxs;
                    int cyw, oy;
                    if (rr < ny0) {
                        cyw = ys_b[0] + rr;
                        oy = ys_o[0];
                    } else if (rr < ny0 + ny1) {
                        cyw = ys_b[1] + (rr - ny0);
                        oy = ys_o[1];
                    } else {
                        cyw = ys_b[2] + (rr - ny0 - ny1);
                        oy = ys_o[2];
                    }
                    const int pb = xi == 0 ? xs_b[0] : (xi == 1 ? xs_b[1] : xs_b[2]);
                    const int pe = xi == 0 ? xs_e[0] : (xi == 1 ? xs_e[1] : xs_e[2]);
                    const int po = xi == 0 ? xs_o[0] : (xi == 1 ? xs_o[1] : xs_o[2]);
                    const int64_t k0 = key_base + (int64_t)cyw * a.ncx + pb;
                    b0 = a.seg[k0];
                    b1 = a.seg[k0 + (pe - pb) + 1];
                    img = (po + 8) | ((oy + 8) << 8);
                }
                const bool ok = b1 > b0;
                const unsigned mask = __ballot_sync(0xffffffffu, ok);
                const int pos = nr + __popc(mask & ((1u << lane) - 1u));
                unsigned incl = ok ? b1 - b0 : 0u;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                if (ok && pos < kPotMaxRanges) {
                    r_beg[pos] = b0;
                    r_img[pos] = img;
                    r_pre[pos + 1] = run + incl;
                }
                nr = min(nr + __popc(mask), kPotMaxRanges);
                run += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) {
                r_pre[0] = 0;
                n_ranges = nr;
            }
        }
        __syncthreads();
        const int nr = n_ranges;
        const unsigned n_atoms = r_pre[nr];
        const int lane = t & 31, wid = t >> 5;
        for (unsigned vbase = 0; vbase < n_atoms; vbase += kPotThreads) {
            const unsigned v = vbase + t;
            float4 cv = make_float4(0.f, 0.f, 0.f, 0.f);
            unsigned cpi = 0;
            int cnt = 0;
            if (v < n_atoms) {
                int r = 0;
                while (r + 1 < nr && r_pre[r + 1] <= v) r++;
                const unsigned i = r_beg[r] + (v - r_pre[r]);
                const float xa = a.ax[i], ya = a.ay[i], w = a.aw[i];
                const int pk = a.ae[i];
                const int e = pk & 0xFF;
                // image of the atom seen through this range: the range's image of the atom's
                // wrapped cell, minus the atom's own wrap count
                const int ox = (r_img[r] & 0xFF) - 8 - (((pk >> 8) & 15) - 8);
                const int oy = ((r_img[r] >> 8) & 0xFF) - 8 - (((pk >> 12) & 15) - 8);
                const float rm = el[e].rmax * 1.0001f + 1e-4f;
                const float xs = xa + (float)ox * a.lx, ys = ya + (float)oy * a.ly;  // culling only
                const float dxr = fmaxf(0.f, fmaxf(X0 - xs, xs - X1));
                const float dyr = fmaxf(0.f, fmaxf(Y0 - ys, ys - Y1));
                if (dxr * dxr + dyr * dyr < rm * rm) {
                    cv = make_float4(xa, ya, w, __int_as_float(e | ((ox + 4) << 8) | ((oy + 4) << 12)));
                    cpi = i;
                    cnt = 1;
                }
            }
            // ordered compaction (deterministic: cell order, then atom order)
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane == 31) wsum[wid] = incl;
            __syncthreads();
            if (t == 0) {
                int run = 0;
                for (int w = 0; w < kPotThreads / 32; w++) {
                    int vv = wsum[w];
                    wsum[w] = run;
                    run += vv;
                }
                total_s = run;
            }
            __syncthreads();
            const int off = wsum[wid] + incl - cnt;
            if (cnt > 0) {
                cand[off] = cv;
                if (FINE) candp[off] = cpi;
            }
            __syncthreads();
            const int total = total_s;
            // The warp's own list, one candidate per lane: an atom whose disc misses the warp's 16 x 16
            // pixel block is dropped here (its spline evaluations would all be masked off, yet a
            // divergent warp still issues them), so the loop below runs over hits only.
            int nh = 0;
            for (int base = 0; base < total; base += 32) {
                const int q = base + lane;
                bool hit = false;
                if (q < total) {
                    const float4 cd = cand[q];
                    const int bits = __float_as_int(cd.w);
                    const float rmax2 = el[bits & 0xFF].rmax2;
                    const int ox = ((bits >> 8) & 15) - 4, oy = ((bits >> 12) & 15) - 4;
                    const float xs = cd.x + (float)ox * a.lx, ys = cd.y + (float)oy * a.ly;
                    const float dxr = fmaxf(0.f, fmaxf(WX0 - xs, xs - WX1));
                    const float dyr = fmaxf(0.f, fmaxf(WY0 - ys, ys - WY1));
                    hit = dxr * dxr + dyr * dyr < rmax2 * 1.0002f + 1e-4f;
                }
                const unsigned m = __ballot_sync(0xffffffffu, hit);
                if (hit) whit[wid][nh + __popc(m & ((1u << lane) - 1u))] = (unsigned short)q;
                nh += __popc(m);
            }
            __syncwarp();
            for (int h = 0; h < nh; h++) {
                const int q = whit[wid][h];
                const float4 cd = cand[q];
                const int bits = __float_as_int(cd.w);
                const ElemTable& T = el[bits & 0xFF];
                const float rmax2 = T.rmax2;
                const int ox = ((bits >> 8) & 15) - 4, oy = ((bits >> 12) & 15) - 4;
                // distance to the image (ox, oy) of the atom: pixel index shifted by -ox*nx, and
                // i*dx - x formed with dx split in two floats, so the offset is accurate to its own
                // rounding (the pixel coordinate i*dx alone would carry ~1e-6 A of error)
                const float fx0 = (float)(tx0 + 4 * px - ox * a.nx), fy0 = (float)(ty0 + py - oy * a.ny);
                float dx2[4], dy2[RY];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const float fx = fx0 + (float)k;
                    const float d = fmaf(fx, a.dx_lo, fmaf(fx, a.dx_hi, -cd.x));
                    dx2[k] = d * d;
                }
#pragma unroll
                for (int r = 0; r < RY; r++) {
                    const float fy = fy0 + (float)(r * ROW_STEP);
                    const float d = fmaf(fy, a.dy_lo, fmaf(fy, a.dy_hi, -cd.y));
                    dy2[r] = d * d;
                }
#pragma unroll
                for (int r = 0; r < RY; r++) {
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const float r2 = dx2[k] + dy2[r];
                        if (r2 < rmax2) {
                            if (FINE) acc[r][k] += cd.z * spline_eval_c(T, a.pair_coef + (size_t)candp[q] * MS_NR, r2);
                            else acc[r][k] += cd.z * spline_eval(T, r2);
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int r = 0; r < RY; r++) {
        const int64_t o = (int64_t)conf * a.V_conf_stride + (int64_t)(sl - a.V_slice_base) * a.nx * a.ny +
                          (int64_t)(ty0 + py + r * ROW_STEP) * a.nx + tx0 + 4 * px;
        if (a.T) {
            // the transmission function t = exp(i V) of the four pixels, as the row pass would form it
            // (transmission_function.cuh:107-119), so the slice passes read t instead of V
            float2 t[4];
#pragma unroll
            for (int k = 0; k < 4; k++) t[k] = expi_tab(acc[r][k], a.exptab);
            float4* out = reinterpret_cast<float4*>(a.T + o);
            out[0] = make_float4(t[0].x, t[0].y, t[1].x, t[1].y);
            out[1] = make_float4(t[2].x, t[2].y, t[3].x, t[3].y);
        } else {
            *reinterpret_cast<float4*>(a.V + o) = make_float4(acc[r][0], acc[r][1], acc[r][2], acc[r][3]);
        }
    }
}

void launch_potential(const PotArgs& a, int n_conf, cudaStream_t st)
{
    if (a.nslice <= 0 || n_conf <= 0) return;
    dim3 grid((unsigned)((a.nx / kPotTX) * (a.ny / kPotTY)), (unsigned)a.nslice, (unsigned)n_conf);
    size_t sm = sizeof(ElemTable) * a.n_elem + sizeof(float4) * kPotThreads;
    if (a.pair_coef) sm += sizeof(unsigned) * kPotThreads;
    auto go = [&](auto kern) {
        smem_attr(kern, sm);
        kern<<<grid, kPotThreads, sm, st>>>(a);
    };
    if (a.pair_coef) {
        if (a.wrap) go(k_potential<true, true>);
        else go(k_potential<true, false>);
    } else {
        if (a.wrap) go(k_potential<false, true>);
        else go(k_potential<false, false>);
    }
    count_launch();
    check_launch("potential");
}

// ---------------------------------------------------------------------------
// specimen on the device: displacement, z range, slice assignment, gather
// ---------------------------------------------------------------------------
__global__ void k_displace(const float* x, const float* y, const float* z, const float* sig, int64_t n,
                           const int* confs, uint64_t seed, int dx, int dy, int dzf, float* xd, float* yd, float* zd)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int ci = blockIdx.y;
    float xi = x[i], yi = y[i], zi = z[i];
    det_displace(seed, confs[ci], i, sig[i], dx, dy, dzf, &xi, &yi, &zi);
    int64_t o = (int64_t)ci * n + i;
    xd[o] = xi;
    yd[o] = yi;
    zd[o] = zi;
}

void launch_displace(const float* x, const float* y, const float* z, const float* sig, int64_t n, const int* confs,
                     int nconf, uint64_t seed, int dx, int dy, int dzf, float* xd, float* yd, float* zd,
                     cudaStream_t st)
{
    dim3 grid((unsigned)((n + 255) / 256), (unsigned)nconf);
    k_displace<<<grid, 256, 0, st>>>(x, y, z, sig, n, confs, seed, dx, dy, dzf, xd, yd, zd);
    count_launch();
    check_launch("displace");
}

__device__ __forceinline__ unsigned f2ord(float f)
{
    unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__global__ void k_zrange(const float* zd, int64_t n, unsigned* zmin, unsigned* zmax)
{
    int ci = blockIdx.y;
    unsigned lo = 0xFFFFFFFFu, hi = 0u;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        unsigned k = f2ord(zd[(int64_t)ci * n + i]);
        lo = min(lo, k);
        hi = max(hi, k);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(zmin + ci, lo);
        atomicMax(zmax + ci, hi);
    }
}

void launch_zrange(const float* zd, int64_t n, int nconf, unsigned* zmin_bits, unsigned* zmax_bits, cudaStream_t st)
{
    cudaMemsetAsync(zmin_bits, 0xFF, sizeof(unsigned) * nconf, st);
    cudaMemsetAsync(zmax_bits, 0x00, sizeof(unsigned) * nconf, st);
    int blocks = (int)std::min<int64_t>(1184, (n + 255) / 256);
    k_zrange<<<dim3(blocks, nconf), 256, 0, st>>>(zd, n, zmin_bits, zmax_bits);
    count_launch();
    check_launch("z range");
}

// Periodic wrap count of a coordinate (0 without wrapping), clamped to the 4 bits it is packed in.
__device__ __forceinline__ int wrap_count(float x, float L, int wrap)
{
    if (!wrap) return 0;
    int k = (int)floorf(x / L);
    return min(max(k, -8), 7);
}

__device__ __forceinline__ int cell_of(float x, float L, const CellGrid& cg, int nc)
{
    const int k = wrap_count(x, L, cg.wrap);
    const int c = (int)floorf((x - (float)k * L) * cg.inv_cell);
    return min(max(c, 0), nc - 1);
}

// Key of an atom: (configuration, slice, cell) with the atoms outside every slice in slice slot
// S_cap; one stable radix sort then groups atoms by slice and, inside a slice, by cell.
__global__ void k_assign(const float* xd, const float* yd, const float* zd, int64_t n, const float* bounds,
                         int bstride, const int* nv, const float* vmax, int S_cap, CellGrid cg, unsigned* keys,
                         int* vals, unsigned* counts)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int ci = blockIdx.y;
    const int64_t o = (int64_t)ci * n + i;
    int s = det_slice_of(zd[o], bounds + (int64_t)ci * bstride, nv[ci], vmax[ci]);
    const int nc = cg.ncx * cg.ncy;
    const int cell = (s >= 0) ? cell_of(yd[o], cg.ly, cg, cg.ncy) * cg.ncx + cell_of(xd[o], cg.lx, cg, cg.ncx) : 0;
    unsigned key = ((unsigned)ci * (unsigned)(S_cap + 1) + (unsigned)(s >= 0 ? s : S_cap)) * (unsigned)nc + cell;
    keys[o] = key;
    vals[o] = (int)i;
    atomicAdd(counts + key, 1u);
}

void launch_assign(const float* xd, const float* yd, const float* zd, int64_t n, int nconf, const float* bounds,
                   int bstride, const int* nv, const float* vmax, int S_cap, const CellGrid& cg, unsigned* keys,
                   int* vals, unsigned* counts, cudaStream_t st)
{
    dim3 grid((unsigned)((n + 255) / 256), (unsigned)nconf);
    k_assign<<<grid, 256, 0, st>>>(xd, yd, zd, n, bounds, bstride, nv, vmax, S_cap, cg, keys, vals, counts);
    count_launch();
    check_launch("slice assignment");
}

__global__ void k_gather(const unsigned* keys, const int* vals, int64_t total, int64_t n, int S_cap, CellGrid cg,
                         const float* xd, const float* yd, const float* occ, const int* elem, float vr, float* ax,
                         float* ay, float* aw, int* ae)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    unsigned key = keys[i];
    int64_t ci = key / ((unsigned)(S_cap + 1) * (unsigned)(cg.ncx * cg.ncy));
    int64_t at = vals[i];
    const float x = xd[ci * n + at], y = yd[ci * n + at];
    ax[i] = x;
    ay[i] = y;
    aw[i] = vr * occ[at];
    // element index and the atom's own periodic wrap counts, packed for the potential kernel
    ae[i] = elem[at] | ((wrap_count(x, cg.lx, cg.wrap) + 8) << 8) | ((wrap_count(y, cg.ly, cg.wrap) + 8) << 12);
}

void launch_gather(const unsigned* keys, const int* vals, int64_t total, int64_t n, int S_cap, const CellGrid& cg,
                   const float* xd, const float* yd, const float* occ, const int* elem, float vr_factor, float* ax,
                   float* ay, float* aw, int* ae, cudaStream_t st)
{
    k_gather<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(keys, vals, total, n, S_cap, cg, xd, yd, occ, elem,
                                                              vr_factor, ax, ay, aw, ae);
    count_launch();
    check_launch("gather");
}

// ---------------------------------------------------------------------------
// fine slicing: (atom, slice) pairs and their slice-integrated splines
// (generate_potential_by_height with enable_fine_slicing, projected_potential.cuh:94-133;
// gen_sa_coeff_kernel and fill_spl_coeff_kernel, device_kernels.cuh:48-105)
// ---------------------------------------------------------------------------
__global__ void k_fine_assign(const float* xd, const float* yd, const float* zd, int64_t n, const float* bounds,
                              int bstride, const int* nv, const float* zmax, int S_cap, CellGrid cg, float rint,
                              int maxper, unsigned nkeys, unsigned* keys, int* vals, unsigned* counts)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int ci = blockIdx.y;
    const int64_t o = (int64_t)ci * n + i;
    const float z = zd[o];
    const float* b = bounds + (int64_t)ci * bstride;
    const int ns = nv[ci] - 1;
    const int ncell = cg.ncx * cg.ncy;
    const int cell = cell_of(yd[o], cg.ly, cg, cg.ncy) * cg.ncx + cell_of(xd[o], cg.lx, cg, cg.ncx);
    // candidate slices: every slice whose middle lies within rint + one slice of z (the membership
    // test below decides exactly)
    const float dz = b[1] - b[0];
    int s0 = (int)floorf((z - rint - b[0]) / dz) - 2, s1 = (int)ceilf((z + rint - b[0]) / dz) + 2;
    s0 = max(s0, 0);
    s1 = min(s1, ns - 1);
    int k = 0;
    for (int s = s0; s <= s1 && k < maxper; s++) {
        if (!det_fine_member(z, b[s], b[s + 1], rint, zmax[ci])) continue;
        const unsigned key = ((unsigned)ci * (unsigned)(S_cap + 1) + (unsigned)s) * (unsigned)ncell + (unsigned)cell;
        keys[o * maxper + k] = key;
        vals[o * maxper + k] = (int)i;
        atomicAdd(counts + key, 1u);
        k++;
    }
    for (; k < maxper; k++) {
        keys[o * maxper + k] = nkeys;
        vals[o * maxper + k] = (int)i;
    }
}

void launch_fine_assign(const float* xd, const float* yd, const float* zd, int64_t n, int nconf, const float* bounds,
                        int bstride, const int* nv, const float* zmax, int S_cap, const CellGrid& cg, float rint,
                        int maxper, unsigned nkeys, unsigned* keys, int* vals, unsigned* counts, cudaStream_t st)
{
    dim3 grid((unsigned)((n + 255) / 256), (unsigned)nconf);
    k_fine_assign<<<grid, 256, 0, st>>>(xd, yd, zd, n, bounds, bstride, nv, zmax, S_cap, cg, rint, maxper, nkeys,
                                        keys, vals, counts);
    count_launch();
    check_launch("fine slicing assignment");
}

__global__ void k_fine_gather(const unsigned* keys, const int* vals, int64_t total, int64_t n, int S_cap, CellGrid cg,
                              unsigned nkeys, const float* xd, const float* yd, const float* zd, const float* occ,
                              const int* elem, float vr, float* ax, float* ay, float* aw, int* ae, float* az)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const unsigned key = keys[i];
    if (key >= nkeys) return;   // unused slot (sorted past every pair)
    const int64_t ci = key / ((unsigned)(S_cap + 1) * (unsigned)(cg.ncx * cg.ncy));
    const int64_t at = vals[i];
    const float x = xd[ci * n + at], y = yd[ci * n + at];
    ax[i] = x;
    ay[i] = y;
    az[i] = zd[ci * n + at];
    aw[i] = vr * occ[at];
    ae[i] = elem[at] | ((wrap_count(x, cg.lx, cg.wrap) + 8) << 8) | ((wrap_count(y, cg.ly, cg.wrap) + 8) << 12);
}

void launch_fine_gather(const unsigned* keys, const int* vals, int64_t total, int64_t n, int S_cap, const CellGrid& cg,
                        unsigned nkeys, const float* xd, const float* yd, const float* zd, const float* occ,
                        const int* elem, float vr_factor, float* ax, float* ay, float* aw, int* ae, float* az,
                        cudaStream_t st)
{
    k_fine_gather<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(keys, vals, total, n, S_cap, cg, nkeys, xd, yd, zd,
                                                                   occ, elem, vr_factor, ax, ay, aw, ae, az);
    count_launch();
    check_launch("fine slicing gather");
}

// One block per pair, one thread per spline node: the atom's potential integrated over the
// slice by the kNqz-point z quadrature in FP64 (V and dV/dR^2), the cosine taper in R^2 from
// 0.85 R_max, then the Hermite cubic coefficients of each node interval.
__global__ void __launch_bounds__(MS_NR) k_fine_tables(const unsigned* keys, const float* az, const int* ae,
                                                       const unsigned* seg, unsigned nkeys, const float* bounds,
                                                       int bstride, int S_cap, int ncell, const ElemCoefDev* coefs,
                                                       double rmin, double rmax, const double* qz, float4* out)
{
    const int64_t p = blockIdx.x;
    if (p >= (int64_t)seg[nkeys]) return;
    __shared__ double sR2[MS_NR], sV[MS_NR], sdV[MS_NR];
    const int i = threadIdx.x;
    const unsigned key = keys[p];
    const int ci = (int)(key / ((unsigned)(S_cap + 1) * (unsigned)ncell));
    const int s = (int)((key / (unsigned)ncell) % (unsigned)(S_cap + 1));
    const float zs = bounds[(int64_t)ci * bstride + s], ze = bounds[(int64_t)ci * bstride + s + 1];
    const float zm = MSF_MUL(0.5f, MSF_ADD(zs, ze));
    const double amid = (double)MSF_SUB(zm, az[p]), dzs = (double)MSF_SUB(ze, zs);
    const ElemCoefDev& c = coefs[ae[p] & 0xFF];
    const double R = (i == MS_NR - 1) ? rmax : rmin * pow(rmax / rmin, (double)i / (double)(MS_NR - 1));
    const double R2 = R * R;
    double v = 0.0, d = 0.0;
    for (int k = 0; k < kNqz; k++) {
        const double z = dzs * qz[k] + amid;
        const double r = sqrt(z * z + R2);
        double Vr, dVr;
        vr_eval(c, r, &Vr, &dVr);
        v += qz[kNqz + k] * dzs * Vr;
        d += qz[kNqz + k] * dzs * dVr / r;
    }
    d *= 0.5;
    const double R2tap = (0.85 * rmax) * (0.85 * rmax);
    const double tap_cf = 3.14159265358979323846264338327950288 / (2.0 * (rmax * rmax - R2tap));
    if (R2tap < R2) {
        const double tap = cos(tap_cf * (R2 - R2tap)), dtap = sin(tap_cf * (R2 - R2tap));
        d = d * tap - tap_cf * v * dtap;
        v = v * tap;
    }
    sR2[i] = R2;
    sV[i] = v;
    sdV[i] = d;
    __syncthreads();
    double c2 = 0.0, c3 = 0.0;
    if (i < MS_NR - 1) {
        const double idR = 1.0 / (sR2[i + 1] - R2);
        const double m = (sV[i + 1] - v) * idR;
        const double nn = d + sdV[i + 1];
        c2 = (3.0 * m - nn - d) * idR;
        c3 = (nn - 2.0 * m) * idR * idR;
    }
    out[p * MS_NR + i] = make_float4((float)v, (float)d, (float)c2, (float)c3);
}

void launch_fine_tables(const unsigned* keys, const float* az, const int* ae, const unsigned* seg, unsigned nkeys,
                        int64_t total, const float* bounds, int bstride, int S_cap, const CellGrid& cg,
                        const ElemCoefDev* coefs, double rmin, double rmax, const double* qz, float4* out,
                        cudaStream_t st)
{
    if (total <= 0) return;
    k_fine_tables<<<(unsigned)total, MS_NR, 0, st>>>(keys, az, ae, seg, nkeys, bounds, bstride, S_cap,
                                                     cg.ncx * cg.ncy, coefs, rmin, rmax, qz, out);
    count_launch();
    check_launch("fine slicing splines");
}

// ---------------------------------------------------------------------------
// post-processing
// ---------------------------------------------------------------------------
constexpr int kDetThreads = 256;

// sum_square_over_Det_batch (device_kernels.cuh:625-671): annular sums of |Psi|^2 per wave,
// accumulated in FP64 per thread and reduced in a fixed order.
__global__ void __launch_bounds__(kDetThreads) k_detect(const float2* psi, int nx, int ny, float dgx, float dgy,
                                                        const float* g2in, const float* g2out, int ndet,
                                                        double* partial)
{
    __shared__ double red[MS_MAX_DET][kDetThreads / 32];
    const int b = blockIdx.y;
    const int64_t N = (int64_t)nx * ny;
    const int64_t per = (N + gridDim.x - 1) / gridDim.x;
    const int64_t p0 = per * blockIdx.x, p1 = min(N, p0 + per);
    float gi[MS_MAX_DET], go[MS_MAX_DET];
    double acc[MS_MAX_DET];
#pragma unroll
    for (int d = 0; d < MS_MAX_DET; d++) {
        gi[d] = d < ndet ? g2in[d] : 1.f;
        go[d] = d < ndet ? g2out[d] : 0.f;
        acc[d] = 0.0;
    }
    const float2* w = psi + (int64_t)b * N;
    for (int64_t p = p0 + threadIdx.x; p < p1; p += kDetThreads) {
        int ix = (int)(p % nx), iy = (int)(p / nx);
        float g2 = det_g2(ix, iy, nx, ny, dgx, dgy);
        float2 v = w[p];
        double a2 = (double)v.x * v.x + (double)v.y * v.y;
#pragma unroll
        for (int d = 0; d < MS_MAX_DET; d++)
            if (gi[d] <= g2 && g2 <= go[d]) acc[d] += a2;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < MS_MAX_DET; d++) {
        double v = acc[d];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[d][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < ndet) {
        double s = 0.0;
        for (int k = 0; k < kDetThreads / 32; k++) s += red[threadIdx.x][k];
        partial[((int64_t)b * gridDim.x + blockIdx.x) * ndet + threadIdx.x] = s;
    }
}

void launch_detect(const float2* psi, int nwaves, int nx, int ny, float dgx, float dgy, const float* g2in,
                   const float* g2out, int ndet, double* partial, int nblk, cudaStream_t st)
{
    k_detect<<<dim3(nblk, nwaves), kDetThreads, 0, st>>>(psi, nx, ny, dgx, dgy, g2in, g2out, ndet, partial);
    count_launch();
    check_launch("detector");
}

__global__ void k_det_finalize(const double* partial, int nwaves, int nblk, int ndet, const WaveInfo* waves,
                               double* I_wave, double* image, int npos, int accumulate)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nwaves * ndet) return;
    int b = i / ndet, d = i % ndet;
    double s = 0.0;
    for (int k = 0; k < nblk; k++) s += partial[((int64_t)b * nblk + k) * ndet + d];
    if (I_wave) I_wave[i] = s;
    if (image) {
        double v = (double)waves[b].weight * s;
        int64_t o = (int64_t)d * npos + waves[b].pos;
        image[o] = accumulate ? image[o] + v : v;
    }
}

void launch_det_finalize(const double* partial, int nwaves, int nblk, int ndet, const WaveInfo* waves,
                         double* I_wave, double* image, int npos, int accumulate, cudaStream_t st)
{
    int n = nwaves * ndet;
    k_det_finalize<<<(n + 127) / 128, 128, 0, st>>>(partial, nwaves, nblk, ndet, waves, I_wave, image, npos,
                                                     accumulate);
    count_launch();
    check_launch("detector finalize");
}

// add_scale_square / add_scale_components / add_weighted_scale over configurations
// (device_kernels.cuh:296-329), accumulated in FP64 in wave order.
__global__ void k_acc_abs2(const float2* psi, int nwaves, const WaveInfo* waves, int64_t N, double* acc, int first)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    double s = first ? 0.0 : acc[p];
    for (int b = 0; b < nwaves; b++) {
        float2 v = psi[(int64_t)b * N + p];
        s += (double)waves[b].weight * ((double)v.x * v.x + (double)v.y * v.y);
    }
    acc[p] = s;
}

void launch_acc_abs2(const float2* psi, int nwaves, const WaveInfo* waves, int64_t N, double* acc, int first,
                     cudaStream_t st)
{
    k_acc_abs2<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(psi, nwaves, waves, N, acc, first);
    count_launch();
    check_launch("accumulate |psi|^2");
}

__global__ void k_acc_cplx(const float2* psi, int nwaves, const WaveInfo* waves, int64_t N, double* re, double* im,
                           int first)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    double sr = first ? 0.0 : re[p], si = first ? 0.0 : im[p];
    for (int b = 0; b < nwaves; b++) {
        float2 v = psi[(int64_t)b * N + p];
        sr += (double)waves[b].weight * v.x;
        si += (double)waves[b].weight * v.y;
    }
    re[p] = sr;
    im[p] = si;
}

void launch_acc_cplx(const float2* psi, int nwaves, const WaveInfo* waves, int64_t N, double* re, double* im,
                     int first, cudaStream_t st)
{
    k_acc_cplx<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(psi, nwaves, waves, N, re, im, first);
    count_launch();
    check_launch("accumulate wave");
}

__global__ void k_acc_real(const float* in, int nwaves, int64_t N, double* acc, int first)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    double s = first ? 0.0 : acc[p];
    for (int b = 0; b < nwaves; b++) s += (double)in[(int64_t)b * N + p];
    acc[p] = s;
}

void launch_acc_real(const float* in, int nwaves, int64_t N, double* acc, int first, cudaStream_t st)
{
    k_acc_real<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(in, nwaves, N, acc, first);
    count_launch();
    check_launch("accumulate image");
}

// FP64 accumulator -> float output, optionally quadrant-swapped (fft_shift, device_kernels.cuh:342-362)
__global__ void k_emit(const double* acc, int nx, int ny, int shift, float* out)
{
    int64_t N = (int64_t)nx * ny;
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    int ix = (int)(p % nx), iy = (int)(p / nx);
    int64_t q = shift ? (int64_t)((iy + ny / 2) % ny) * nx + (ix + nx / 2) % nx : p;
    out[q] = (float)acc[p];
}

void launch_emit(const double* acc, int nx, int ny, int shift, float* out, cudaStream_t st)
{
    int64_t N = (int64_t)nx * ny;
    k_emit<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(acc, nx, ny, shift, out);
    count_launch();
    check_launch("emit");
}

__global__ void k_d2f(const double* in, int64_t n, float* out)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) out[p] = (float)in[p];
}

void launch_d2f(const double* in, int64_t n, float* out, cudaStream_t st)
{
    if (n <= 0) return;
    k_d2f<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, n, out);
    count_launch();
    check_launch("convert");
}

// seg[0] = 0, seg[i+1] = seg[i] + counts[i]: one block, chunked sequential sums
__global__ void k_scan_counts(const unsigned* counts, int n, int64_t* seg)
{
    __shared__ int64_t part[1024];
    const int t = threadIdx.x, T = blockDim.x;
    const int per = (n + T - 1) / T;
    const int i0 = min(n, t * per), i1 = min(n, i0 + per);
    int64_t s = 0;
    for (int i = i0; i < i1; i++) s += counts[i];
    part[t] = s;
    __syncthreads();
    if (t == 0) {
        int64_t run = 0;
        for (int k = 0; k < T; k++) {
            int64_t v = part[k];
            part[k] = run;
            run += v;
        }
    }
    __syncthreads();
    int64_t run = part[t];
    if (t == 0) seg[0] = 0;
    for (int i = i0; i < i1; i++) {
        run += counts[i];
        seg[i + 1] = run;
    }
}

void launch_scan_counts(const unsigned* counts, int n, int64_t* seg, cudaStream_t st)
{
    k_scan_counts<<<1, 1024, 0, st>>>(counts, n, seg);
    count_launch();
    check_launch("scan");
}

__global__ void k_fill_c(float2* p, int64_t n, float2 v)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

void launch_fill_c(float2* p, int64_t n, float2 v, cudaStream_t st)
{
    if (n <= 0) return;
    k_fill_c<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, n, v);
    count_launch();
    check_launch("fill");
}

}  // namespace msb
