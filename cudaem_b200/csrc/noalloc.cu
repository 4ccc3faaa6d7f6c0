// STEM forward pass on caller potentials that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: a host application whose
// memory manager owns every device allocation (a framework plugin that must
// stay inside its pool), a real-time acquisition loop that forbids the
// implicit synchronisation cudaMalloc/cudaFree bring, or a process that has
// already handed nearly all device memory to a pre-sized arena.  For them
// this file runs the same fused slice passes as ms_stem_forward_potential,
// but every scratch buffer it needs -- the probe-batch wave, the FFT
// twiddles, the propagator factors, the wave table and the detector partial
// sums -- lives in one file-scope __device__ array of fixed size.  The
// caller provides the potentials and the output in its own device memory.
//
// The array is created when the library's module for this file is loaded on
// a device and stays until the process exits (about 34 MiB per GPU).  Its
// device address is looked up on the first call made with that device
// current (and again whenever the device's CUDA context has changed, e.g.
// after cudaDeviceReset); that first call should therefore come before any
// stream capture.  Every call synchronises the stream after each probe batch,
// so it returns only when its results are in the caller's output.  Every call
// shares the one array, so calls that overlap on the GPU (different streams,
// or host threads) race on it and must be serialised by the caller.  Nothing
// in the array needs to start at zero: each call writes every value before
// reading it.  The FFT and propagator tables of the last grid stay in the
// array and are not uploaded again while the grid, beam and slice thickness
// are unchanged.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "engine.hpp"
#include "fft_layout.hpp"
#include "kernels.cuh"

namespace msb {

namespace {
constexpr size_t kWaveBytes = size_t(32) << 20;       // probe-batch waves: nx*ny*8*batch <= 32 MiB
constexpr int kMaxBatch = 256;
constexpr int kMaxN = 2048;
constexpr int kMaxBlk = 64;
constexpr int kExpN = 1024;
// tw_x and tw_y (kTwSets dithered sets each), prop_x, prop_y, exp table
constexpr size_t kTableBytes = sizeof(float2) * (2 * (size_t)kTwSets * kMaxN + 2 * kMaxN + kExpN);
constexpr size_t kWaveInfoBytes = sizeof(WaveInfo) * kMaxBatch;
constexpr size_t kThrBytes = 256;                                                     // 2 * MS_MAX_DET floats
constexpr size_t kIwaveBytes = sizeof(double) * kMaxBatch * MS_MAX_DET;
constexpr size_t kPartialBytes = sizeof(double) * kMaxBatch * kMaxBlk * MS_MAX_DET;
constexpr size_t kOffTables = 0;
constexpr size_t kOffWaveInfo = kOffTables + kTableBytes;
constexpr size_t kOffThr = kOffWaveInfo + kWaveInfoBytes;
constexpr size_t kOffIwave = kOffThr + kThrBytes;
constexpr size_t kOffPartial = kOffIwave + kIwaveBytes;
constexpr size_t kOffWave = (kOffPartial + kPartialBytes + 255) / 256 * 256;
constexpr size_t kScratchBytes = kOffWave + kWaveBytes;
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {
std::mutex g_mtx;

// What the array holds on one device: the CUDA context it was set up in, its device address, and
// the key of the FFT / propagator tables it currently holds.
struct TableKey {
    int nx, ny;
    double dgx, dgy, g0x, g0y, prop_w;
};
struct DevState {
    unsigned long long ctx_id = 0;
    unsigned char* addr = nullptr;
    bool have_tables = false;
    TableKey key{};
};
DevState g_state[128];

// Identifier of the calling thread's current CUDA context (cuCtxGetId through the runtime's
// driver entry points; no link against the driver library).  0 when no context is current yet
// or the driver does not provide the call, which makes every call set up again.
unsigned long long current_context_id()
{
    static PFN_cuCtxGetCurrent_v4000 get_cur = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_cur = (PFN_cuCtxGetCurrent_v4000)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (PFN_cuCtxGetId_v12000)f;
        cudaGetLastError();
        looked_up = true;
    }
    if (!get_cur || !get_id) return 0;
    CUcontext cx = nullptr;
    unsigned long long id = 0;
    if (get_cur(&cx) != CUDA_SUCCESS || !cx || get_id(cx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Set-up on the current device: the device address of the scratch array (cudaGetSymbolAddress;
// the array's name is only a host-side stand-in).  Done on the first call with this device current
// and again whenever the current context differs from the one the set-up was made in (a reset
// device reloads the modules, and the array may move; the tables it held are gone).  The caller
// holds g_mtx.
DevState& setup_current_device()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) throw MsError(MS_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    MS_REQUIRE(dev >= 0 && dev < 128, MS_ERR_NO_DEVICE, "device ordinal out of range");
    DevState& s = g_state[dev];
    unsigned long long id = current_context_id();
    if (id != 0 && id == s.ctx_id && s.addr) return s;
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
        throw MsError(MS_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array: ") + cudaGetErrorString(e));
    s.addr = (unsigned char*)p;
    s.ctx_id = current_context_id();   // the look-up above made the device's context current
    s.have_tables = false;
    return s;
}

int team_size_of(int N)
{
    switch (N) {
    case 128: return FftCfg<128>::G;
    case 256: return FftCfg<256>::G;
    case 512: return FftCfg<512>::G;
    case 1024: return FftCfg<1024>::G;
    case 2048: return FftCfg<2048>::G;
    }
    throw MsError(MS_ERR_UNSUPPORTED, "unsupported transform length");
}

// the kTwSets dithered sets of the inter-level twiddles, set t at out[t * N]
void twiddle_table(int N, float2* out)
{
    const double pi = 3.14159265358979323846264338327950288;
    int G = team_size_of(N), E = N / G;
    for (int k1 = 0; k1 < E; k1++)
        for (int g = 0; g < G; g++) {
            double a = -2.0 * pi * (double)((int64_t)g * k1 % N) / (double)N;
            dither_sets(std::cos(a), std::sin(a), kTwSets, out + (size_t)k1 * G + g, (size_t)N);
        }
}

void ck(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw MsError(MS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace

size_t noalloc_scratch_bytes() { return kScratchBytes; }

void stem_forward_noalloc(cudaStream_t st, const ms_params& p, const float* V, int S, double z_init, const double* xy,
                          int np, float* I)
{
    validate_params(p);
    MS_REQUIRE(V && xy && I, MS_ERR_INVALID_ARG, "V, probe_xy and I must not be NULL");
    MS_REQUIRE(S >= 1 && np >= 1, MS_ERR_INVALID_ARG, "need at least one slice and one probe");
    MS_REQUIRE(p.n_det >= 1 && p.n_det <= MS_MAX_DET, MS_ERR_INVALID_ARG, "need 1..8 detectors");
    const int64_t N = (int64_t)p.nx * p.ny;
    // validate_params already caps each axis at 2048 points, which is exactly this limit; the check
    // keeps the array's size and the accepted grids tied together if either changes
    MS_REQUIRE((size_t)N * sizeof(float2) <= kWaveBytes, MS_ERR_UNSUPPORTED,
               "grid too large for the fixed scratch array: nx*ny*8 bytes must not exceed 32 MiB");
    Physics ph = physics_of(p.E0, p.theta);
    GridConst gc = grid_of(p, ph);
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mtx);
        DevState& ds = setup_current_device();
        base = ds.addr;
        float2* tw_x = (float2*)(base + kOffTables);
        float2* tw_y = tw_x + (size_t)kTwSets * kMaxN;
        float2* prop_x = tw_y + (size_t)kTwSets * kMaxN;
        float2* prop_y = prop_x + kMaxN;
        float2* exptab = prop_y + kMaxN;
        const TableKey key{p.nx, p.ny, gc.dgx, gc.dgy, gc.g0x, gc.g0y, gc.prop_w};
        if (!ds.have_tables) {
            // the exp(i phi) table depends on nothing; it is uploaded once per set-up
            std::vector<float2> et(kExpN);
            for (int k = 0; k < kExpN; k++) {
                double e = 2.0 * 3.14159265358979323846264338327950288 * k / (double)kExpN;
                et[k] = make_float2((float)std::cos(e), (float)std::sin(e));
            }
            ck(cudaMemcpyAsync(exptab, et.data(), sizeof(float2) * kExpN, cudaMemcpyHostToDevice, st), "table upload");
        }
        if (!ds.have_tables || std::memcmp(&key, &ds.key, sizeof(key)) != 0) {
            // only the entries this grid uses: kTwSets (nx + ny) twiddles, nx + ny propagator factors
            ds.have_tables = false;
            std::vector<float2> tab((size_t)(kTwSets + 1) * (p.nx + p.ny));
            float2* tx = tab.data();
            float2* ty = tx + (size_t)kTwSets * p.nx;
            float2* px = ty + (size_t)kTwSets * p.ny;
            float2* py = px + p.nx;
            twiddle_table(p.nx, tx);
            twiddle_table(p.ny, ty);
            for (int i = 0; i < p.nx; i++) {
                double g = (double)((i < p.nx / 2) ? i : i - p.nx) * gc.dgx - gc.g0x;
                double th = gc.prop_w * g * g;
                px[i] = make_float2((float)std::cos(th), (float)std::sin(th));
            }
            for (int i = 0; i < p.ny; i++) {
                double g = (double)((i < p.ny / 2) ? i : i - p.ny) * gc.dgy - gc.g0y;
                double th = gc.prop_w * g * g;
                py[i] = make_float2((float)std::cos(th), (float)std::sin(th));
            }
            ck(cudaMemcpyAsync(tw_x, tx, sizeof(float2) * kTwSets * p.nx, cudaMemcpyHostToDevice, st), "table upload");
            ck(cudaMemcpyAsync(tw_y, ty, sizeof(float2) * kTwSets * p.ny, cudaMemcpyHostToDevice, st), "table upload");
            ck(cudaMemcpyAsync(prop_x, px, sizeof(float2) * p.nx, cudaMemcpyHostToDevice, st), "table upload");
            ck(cudaMemcpyAsync(prop_y, py, sizeof(float2) * p.ny, cudaMemcpyHostToDevice, st), "table upload");
            ds.key = key;
            ds.have_tables = true;
        }
    }
    float2* tw_x = (float2*)(base + kOffTables);
    float2* tw_y = tw_x + (size_t)kTwSets * kMaxN;
    float2* prop_x = tw_y + (size_t)kTwSets * kMaxN;
    float2* prop_y = prop_x + kMaxN;
    float2* exptab = prop_y + kMaxN;
    WaveInfo* dwv = (WaveInfo*)(base + kOffWaveInfo);
    float* thr = (float*)(base + kOffThr);
    double* Iw = (double*)(base + kOffIwave);
    double* partial = (double*)(base + kOffPartial);
    float2* psi = (float2*)(base + kOffWave);
    const int ndet = p.n_det;
    float th_h[2 * MS_MAX_DET];
    for (int d = 0; d < ndet; d++) {
        th_h[d] = g2_threshold(p.det_inner[d], ph.lambda);
        th_h[ndet + d] = g2_threshold(p.det_outer[d], ph.lambda);
    }
    ck(cudaMemcpyAsync(thr, th_h, sizeof(float) * 2 * ndet, cudaMemcpyHostToDevice, st), "threshold upload");

    GridDev gd;
    gd.nx = p.nx;
    gd.ny = p.ny;
    gd.dgx_f = gc.dgx_f;
    gd.dgy_f = gc.dgy_f;
    gd.dgx = gc.dgx;
    gd.dgy = gc.dgy;
    gd.gl2_f = (float)gc.gl2;
    gd.alpha_f = (float)gc.alpha;
    gd.bwl = p.bwl ? 1 : 0;
    gd.inv_n = 1.0f / (float)N;
    gd.lx = p.lx;
    gd.ly = p.ly;
    gd.g0x = gc.g0x;
    gd.g0y = gc.g0y;
    LensCoef lc = lens_coef(p.cond_lens, ph.lambda, 0.0);
    LensDev lens;
    std::memset(&lens, 0, sizeof(lens));
    lens.m = lc.m; lens.phi_req = lc.phi_req;
    lens.cc10 = lc.cc10; lens.cc12 = lc.cc12; lens.cc21 = lc.cc21; lens.cc23 = lc.cc23; lens.cc30 = lc.cc30;
    lens.cc32 = lc.cc32; lens.cc34 = lc.cc34; lens.cc41 = lc.cc41; lens.cc43 = lc.cc43; lens.cc45 = lc.cc45;
    lens.cc50 = lc.cc50; lens.cc52 = lc.cc52; lens.cc54 = lc.cc54; lens.cc56 = lc.cc56;
    lens.p12 = lc.p12; lens.p21 = lc.p21; lens.p23 = lc.p23; lens.p32 = lc.p32; lens.p34 = lc.p34;
    lens.p41 = lc.p41; lens.p43 = lc.p43; lens.p45 = lc.p45; lens.p52 = lc.p52; lens.p54 = lc.p54;
    lens.p56 = lc.p56;
    lens.g2min = lc.g2min;
    lens.g2max = lc.g2max;

    const int B = (int)std::min<int64_t>(std::min<int64_t>(kMaxBatch, np), (int64_t)(kWaveBytes / (N * 8)));
    const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>(kMaxBlk, N / 4096));
    const double cc10 = gate_coef(-3.14159265358979323846 * (p.cond_lens.c10 + z_init) * ph.lambda);
    std::vector<WaveInfo> wv((size_t)B);
    for (int start = 0; start < np; start += B) {
        const int nb = std::min(B, np - start);
        for (int i = 0; i < nb; i++) {
            wv[i].px = xy[2 * (start + i)];
            wv[i].py = xy[2 * (start + i) + 1];
            wv[i].cc10 = cc10;
            wv[i].conf_slot = 0;
            wv[i].n_slices = S;
            wv[i].weight = 1.0f;
            wv[i].pos = start + i;
        }
        ck(cudaMemcpyAsync(dwv, wv.data(), sizeof(WaveInfo) * nb, cudaMemcpyHostToDevice, st), "wave table upload");
        PassArgs a;
        std::memset(&a, 0, sizeof(a));
        a.psi = psi;
        a.waves = dwv;
        a.sV = V;
        a.sV_slot_stride = (int64_t)S * N;
        a.prop_x = prop_x;
        a.prop_y = prop_y;
        a.exptab = exptab;
        a.grid = gd;
        a.lens = lens;
        a.tw = tw_y;
        launch_col(p.ny, COL_PROBE_INV, a, nb, p.nx, st);
        for (int sl = 0; sl < S; sl++) {
            a.slice = sl;
            a.tw = tw_x;
            launch_row(p.nx, ROW_INV_T_FWD, a, nb, p.ny, st);
            a.tw = tw_y;
            launch_col(p.ny, COL_STEP_SEP, a, nb, p.nx, st);
        }
        launch_detect(psi, nb, p.nx, p.ny, gd.dgx_f, gd.dgy_f, thr, thr + ndet, ndet, partial, nblk, st);
        launch_det_finalize(partial, nb, nblk, ndet, dwv, Iw, nullptr, 0, 0, st);
        launch_d2f(Iw, (int64_t)nb * ndet, I + (int64_t)start * ndet, st);
        // the host wave table is rewritten for the next batch
        ck(cudaStreamSynchronize(st), "stream synchronize");
    }
}

}  // namespace msb
