// Mode drivers of the engine: the specimen pipeline on the device and the
// HRTEM/ED, CBED, STEM and thickness loops over the fused slice passes.
//
// Call structure (one blocking C-ABI call):
//   upload atoms -> displace every configuration of a group (device) ->
//   z range (one small device-to-host read) -> slicing planes (host, bit-exact
//   with the device) -> slice assignment + stable radix sort + gather (device)
//   -> projected potentials of all slices of the group (device) ->
//   probe / plane wave -> per slice: row pass, column pass -> post passes ->
//   FP64 accumulation over configurations -> output.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "ctx.hpp"
#include "detmath.cuh"
#include "fft_layout.hpp"
#include "kernels.cuh"
#include "vr.cuh"

#define CK(x)                                                                                              \
    do {                                                                                                   \
        cudaError_t e_ = (x);                                                                              \
        if (e_ != cudaSuccess)                                                                             \
            throw ::msb::MsError(e_ == cudaErrorMemoryAllocation ? MS_ERR_OUT_OF_MEMORY : MS_ERR_CUDA,     \
                                 std::string(#x) + ": " + cudaGetErrorString(e_));                         \
    } while (0)

size_t ms_ctx::free_mem()
{
    if (!free_known) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        free_seen = fr;
        free_known = true;
    }
    return free_seen;
}

void* ms_ctx::buf(const std::string& name, size_t bytes)
{
    Buf& b = bufs[name];
    if (b.p && b.bytes >= bytes) return b.p;
    forget_free_mem();
    if (b.p) {
        cudaStreamSynchronize(stream);
        drop_graph();   // a captured graph may hold the old address
        cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
    }
    size_t want = std::max<size_t>(bytes, 256);
    void* p = nullptr;
    cudaError_t e = inject == MS_INJECT_ALLOC_FAIL ? cudaErrorMemoryAllocation : cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw msb::MsError(MS_ERR_OUT_OF_MEMORY,
                           "device allocation of " + std::to_string(want) + " bytes for '" + name + "' failed");
    }
    b.p = p;
    b.bytes = want;
    return p;
}

void ms_ctx::drop_graph()
{
    for (auto& kv : graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    graphs.clear();
}

void ms_ctx::release_all()
{
    forget_free_mem();
    if (stream) cudaStreamSynchronize(stream);
    drop_graph();
    for (auto& kv : bufs)
        if (kv.second.p) cudaFree(kv.second.p);
    bufs.clear();
    for (auto& kv : twiddles) cudaFree(kv.second);
    twiddles.clear();
    if (exptab) cudaFree(exptab);
    exptab = nullptr;
    if (d_err) cudaFree(d_err);
    d_err = nullptr;
    prop_key.clear();
}

cudaEvent_t ms_ctx::prof_event()
{
    if (ev_used == ev_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) throw msb::MsError(MS_ERR_CUDA, "event creation failed");
        ev_pool.push_back(e);
    }
    return ev_pool[ev_used++];
}

void ms_ctx::prof_resolve()
{
    for (auto& pe : ev_pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ev_pool[pe.second], ev_pool[pe.second + 1]) == cudaSuccess) {
            auto& a = prof[pe.first];
            a.first += 1;
            a.second += ms;
        }
    }
    ev_pending.clear();
    ev_used = 0;
}

namespace msb {

namespace {
// Launch wrappers: with profiling on, each launch sits between two events on the context stream.
template <class F>
void timed(ms_ctx* c, const char* cls, F&& launch)
{
    if (!c->profile) {
        launch();
        return;
    }
    size_t i0 = c->ev_used;
    cudaEvent_t a = c->prof_event();
    cudaEvent_t b = c->prof_event();
    cudaEventRecord(a, c->stream);
    launch();
    cudaEventRecord(b, c->stream);
    c->ev_pending.emplace_back(cls, i0);
}

// Kernel classes of the per-launch timing: the forward passes are "row" and "col"; the
// adjoint's own launches get classes of their own.
void run_row(ms_ctx* c, int N, int op, const PassArgs& a, int nw, int ny, cudaStream_t st)
{
    const char* cls = op == ROW_ADJ ? "row_adj" : ((a.flags & PF_STORE_X) ? "row_store" : "row");
    timed(c, cls, [&] { launch_row(N, op, a, nw, ny, st); });
}

void run_col(ms_ctx* c, int N, int op, const PassArgs& a, int nw, int nx, cudaStream_t st)
{
    const char* cls = op == COL_PROBE_INV       ? "probe"
                      : op == COL_SEED          ? "seed"
                      : op == COL_GRAD_PROBE    ? "grad_probe"
                      : (a.flags & PF_CONJ_PROP) ? "col_adj"
                                                 : "col";
    timed(c, cls, [&] { launch_col(N, op, a, nw, nx, st); });
}

void run_potential(ms_ctx* c, const PotArgs& a, int n_conf, cudaStream_t st)
{
    timed(c, "potential", [&] { launch_potential(a, n_conf, st); });
}
}  // namespace

namespace {
constexpr double kPi = 3.14159265358979323846264338327950288;

int team_size(int N)
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

// Inter-level twiddles W_N^(g k1) at [k1 * G + g], in kTwSets dithered sets of N entries (set t
// used by the slices s with s mod kTwSets = t), from FP64 values.
const float2* twiddles(ms_ctx* c, int N)
{
    auto it = c->twiddles.find(N);
    if (it != c->twiddles.end()) return (const float2*)it->second;
    int G = team_size(N), E = N / G;
    std::vector<float2> t((size_t)kTwSets * N);
    for (int k1 = 0; k1 < E; k1++)
        for (int g = 0; g < G; g++) {
            double a = -2.0 * kPi * (double)((int64_t)g * k1 % N) / (double)N;
            dither_sets(std::cos(a), std::sin(a), kTwSets, t.data() + (size_t)k1 * G + g, (size_t)N);
        }
    void* p = nullptr;
    CK(cudaMalloc(&p, sizeof(float2) * t.size()));
    c->forget_free_mem();
    CK(cudaMemcpy(p, t.data(), sizeof(float2) * t.size(), cudaMemcpyHostToDevice));
    c->twiddles[N] = p;
    return (const float2*)p;
}

LensDev lens_dev(const LensCoef& L)
{
    LensDev d;
    std::memset(&d, 0, sizeof(d));
    d.m = L.m;
    d.phi_req = L.phi_req;
    d.cc10 = L.cc10; d.cc12 = L.cc12; d.cc21 = L.cc21; d.cc23 = L.cc23; d.cc30 = L.cc30; d.cc32 = L.cc32;
    d.cc34 = L.cc34; d.cc41 = L.cc41; d.cc43 = L.cc43; d.cc45 = L.cc45; d.cc50 = L.cc50; d.cc52 = L.cc52;
    d.cc54 = L.cc54; d.cc56 = L.cc56;
    d.p12 = L.p12; d.p21 = L.p21; d.p23 = L.p23; d.p32 = L.p32; d.p34 = L.p34; d.p41 = L.p41; d.p43 = L.p43;
    d.p45 = L.p45; d.p52 = L.p52; d.p54 = L.p54; d.p56 = L.p56;
    d.g2min = L.g2min;
    d.g2max = L.g2max;
    d.amp = 1.0;
    return d;
}

// Gauss-Hermite nodes and weights for exp(-x^2), weights normalised to sum 1: the Newton
// iteration on the orthonormal Hermite recurrence with the usual asymptotic starting points
// (the reference's quadrature tables come from the missing multislice_params.hpp).
void gauss_hermite(int n, std::vector<double>* x, std::vector<double>* w)
{
    x->assign(n, 0.0);
    w->assign(n, 1.0);
    if (n == 1) return;
    const double pim4 = 0.7511255444649425;
    double z = 0.0, pp = 0.0;
    const int m = (n + 1) / 2;
    for (int i = 0; i < m; i++) {
        if (i == 0) z = std::sqrt(2.0 * n + 1.0) - 1.85575 * std::pow(2.0 * n + 1.0, -0.16667);
        else if (i == 1) z -= 1.14 * std::pow((double)n, 0.426) / z;
        else if (i == 2) z = 1.86 * z - 0.86 * (*x)[0];
        else if (i == 3) z = 1.91 * z - 0.91 * (*x)[1];
        else z = 2.0 * z - (*x)[i - 2];
        for (int it = 0; it < 100; it++) {
            double p1 = pim4, p2 = 0.0;
            for (int j = 1; j <= n; j++) {
                const double p3 = p2;
                p2 = p1;
                p1 = z * std::sqrt(2.0 / j) * p2 - std::sqrt((double)(j - 1) / j) * p3;
            }
            pp = std::sqrt(2.0 * n) * p2;
            const double z1 = z;
            z = z1 - p1 / pp;
            if (std::fabs(z - z1) <= 1e-15 * (1.0 + std::fabs(z))) break;
        }
        (*x)[i] = z;
        (*x)[n - 1 - i] = -z;
        (*w)[i] = (*w)[n - 1 - i] = 2.0 / (pp * pp);
    }
    if (n % 2 == 1) (*x)[m - 1] = 0.0;
    double sw = 0.0;
    for (double v : *w) sw += v;
    for (double& v : *w) v /= sw;
}

// Partially coherent envelope constants of the objective lens (PCTF_TEM, lens_modulation.cuh:
// 91-110): temporal-only drops the source divergence, spatial-only the defocus spread;
// dsf_iehwgd = sqrt(2) dsf_sigma (lens_dev.cuh:138-142).
void set_pctf(LensDev* d, const ms_params& p, double lambda)
{
    const ms_lens& L = p.obj_lens;
    const int tsi = p.temporal_spatial_incoh ? p.temporal_spatial_incoh : MS_TSI_TEMPORAL_SPATIAL;
    const double beta = tsi == MS_TSI_TEMPORAL ? 0.0 : L.ssf_beta;
    const double D = tsi == MS_TSI_SPATIAL ? 0.0 : std::sqrt(2.0) * L.dsf_sigma;
    d->pctf = 1;
    d->pe_a = kPi * beta * D;
    d->pe_b = kPi * D * lambda;
    d->pe_c = kPi * beta;
    d->pe_d = L.c30 * lambda * lambda;
    d->pe_e = L.c10;
}

struct Setup {
    Physics ph;
    GridConst gc;
    GridDev gd;
    const float2* tw_x;
    const float2* tw_y;
    const float2* prop_x;
    const float2* prop_y;
    const float2* prop;
    const float2* propT = nullptr;   // transposed propagator tables (1024-point columns), or null
    const float2* exptab;
    int64_t N;
    int variant = PASS_CLASSIC;
    int* err = nullptr;        // the context's device wait-error word
};

Setup make_setup(ms_ctx* c, const ms_params& p)
{
    Setup s;
    s.variant = c->pass_variant;
    s.err = c->d_err;
    s.ph = physics_of(p.E0, p.theta);
    s.gc = grid_of(p, s.ph);
    s.N = (int64_t)p.nx * p.ny;
    s.gd.nx = p.nx;
    s.gd.ny = p.ny;
    s.gd.dgx_f = s.gc.dgx_f;
    s.gd.dgy_f = s.gc.dgy_f;
    s.gd.dgx = s.gc.dgx;
    s.gd.dgy = s.gc.dgy;
    s.gd.gl2_f = (float)s.gc.gl2;
    s.gd.alpha_f = (float)s.gc.alpha;
    s.gd.bwl = p.bwl ? 1 : 0;
    s.gd.inv_n = 1.0f / (float)s.N;
    s.gd.lx = p.lx;
    s.gd.ly = p.ly;
    s.gd.g0x = s.gc.g0x;
    s.gd.g0y = s.gc.g0y;
    s.tw_x = twiddles(c, p.nx);
    s.tw_y = twiddles(c, p.ny);
    // separable propagator phase exp(i w (g - g0)^2) per axis, formed in FP64 (device_kernels.cuh:215-234)
    std::vector<float2> px(p.nx), py(p.ny);
    for (int i = 0; i < p.nx; i++) {
        double g = (double)((i < p.nx / 2) ? i : i - p.nx) * s.gc.dgx - s.gc.g0x;
        double th = s.gc.prop_w * g * g;
        px[i] = make_float2((float)std::cos(th), (float)std::sin(th));
    }
    for (int i = 0; i < p.ny; i++) {
        double g = (double)((i < p.ny / 2) ? i : i - p.ny) * s.gc.dgy - s.gc.g0y;
        double th = s.gc.prop_w * g * g;
        py[i] = make_float2((float)std::cos(th), (float)std::sin(th));
    }
    float2* dpx = (float2*)c->buf("prop_x", sizeof(float2) * p.nx);
    float2* dpy = (float2*)c->buf("prop_y", sizeof(float2) * p.ny);
    CK(cudaMemcpyAsync(dpx, px.data(), sizeof(float2) * p.nx, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dpy, py.data(), sizeof(float2) * p.ny, cudaMemcpyHostToDevice, c->stream));
    s.prop_x = dpx;
    s.prop_y = dpy;
    // full table P(k), rebuilt only when the grid, wavelength, slice thickness or tilt change
    char key[256];
    std::snprintf(key, sizeof(key), "%d,%d,%.17g,%.17g,%.17g,%.17g,%.17g,%d", p.nx, p.ny, p.lx, p.ly, s.gc.prop_w,
                  s.gc.g0x, s.gc.g0y, p.bwl);
    float2* P = (float2*)c->buf("prop", sizeof(float2) * kPropSets * s.N);   // dithered tables
    // transposed copy for the warp-column step (1024-point columns)
    float2* PT = p.ny == 1024 ? (float2*)c->buf("propT", sizeof(float2) * kPropSets * s.N) : nullptr;
    if (c->prop_key != key || (PT && !c->propT_built)) {
        launch_prop_table(p.nx, p.ny, s.gc.dgx, s.gc.dgy, s.gc.g0x, s.gc.g0y, s.gc.prop_w, s.gc.alpha, s.gc.gl2,
                          p.bwl ? 1 : 0, P, c->stream, PT);
        c->prop_key = key;
        c->propT_built = PT != nullptr;
    }
    s.prop = P;
    s.propT = PT;
    if (!c->exptab) {
        std::vector<float2> e(1024);
        for (int k = 0; k < 1024; k++) {
            double a = 2.0 * kPi * k / 1024.0;
            e[k] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        CK(cudaMalloc(&c->exptab, sizeof(float2) * 1024));
        c->forget_free_mem();
        CK(cudaMemcpy(c->exptab, e.data(), sizeof(float2) * 1024, cudaMemcpyHostToDevice));
    }
    s.exptab = (const float2*)c->exptab;
    return s;
}

// Atoms on the device plus one radial spline table per distinct element.
struct AtomsDev {
    int64_t n;
    const float *x, *y, *z, *sig, *occ;
    const int* elem;
    const ElemTable* tables;
    const ElemCoefDev* coefs;   // V(r) coefficients per element (fine slicing)
    int n_elem;
    float rmax_all;   // largest cut-off radius over the elements
};

std::string elem_key(const ms_params& p, int Z)
{
    std::string k = std::to_string(Z) + "|" + std::to_string(p.potential_type) + "|" + std::to_string(p.pot_rmin) +
                    "|" + std::to_string(p.pot_rmax);
    for (int i = 0; i < p.n_element_coefs; i++)
        if (p.element_coefs[i].Z == Z) {
            k += "|" + std::to_string(p.element_coefs[i].form);
            for (int j = 0; j < MS_MAX_COEF; j++)
                k += "," + std::to_string(p.element_coefs[i].cl[j]) + "," + std::to_string(p.element_coefs[i].cnl[j]);
        }
    return k;
}

AtomsDev upload_atoms(ms_ctx* c, const ms_params& p, const ms_atoms& a)
{
    AtomsDev d;
    d.n = a.n;
    // distinct atomic numbers in ascending order, and each atom's index among them, in O(n)
    // (Z is validated to 1..103)
    int zmap[128];
    std::fill(zmap, zmap + 128, -1);
    for (int64_t i = 0; i < a.n; i++) zmap[a.Z[i] & 127] = 0;
    std::vector<int> zs;
    for (int z = 0; z < 128; z++)
        if (zmap[z] >= 0) {
            zmap[z] = (int)zs.size();
            zs.push_back(z);
        }
    MS_REQUIRE(zs.size() <= 16, MS_ERR_UNSUPPORTED, "at most 16 distinct elements per specimen");
    std::vector<ElemTable> tabs(zs.size());
    for (size_t i = 0; i < zs.size(); i++) {
        std::string k = elem_key(p, zs[i]);
        auto it = c->elem_cache.find(k);
        if (it == c->elem_cache.end()) {
            ElemTable t;
            build_elem_table(p, zs[i], &t);
            it = c->elem_cache.emplace(k, t).first;
        }
        tabs[i] = it->second;
    }
    std::vector<int> el(a.n);
    for (int64_t i = 0; i < a.n; i++) el[i] = zmap[a.Z[i] & 127];
    size_t fb = sizeof(float) * (size_t)a.n;
    float* x = (float*)c->buf("at_x", fb);
    float* y = (float*)c->buf("at_y", fb);
    float* z = (float*)c->buf("at_z", fb);
    float* sg = (float*)c->buf("at_s", fb);
    float* oc = (float*)c->buf("at_o", fb);
    int* e = (int*)c->buf("at_e", sizeof(int) * (size_t)a.n);
    ElemTable* t = (ElemTable*)c->buf("at_tab", sizeof(ElemTable) * tabs.size());
    CK(cudaMemcpyAsync(x, a.x, fb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(y, a.y, fb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(z, a.z, fb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(sg, a.sigma, fb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(oc, a.occ, fb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(e, el.data(), sizeof(int) * (size_t)a.n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(t, tabs.data(), sizeof(ElemTable) * tabs.size(), cudaMemcpyHostToDevice, c->stream));
    std::vector<ElemCoefDev> cf(zs.size());
    for (size_t i = 0; i < zs.size(); i++) cf[i] = elem_coef_dev(p, zs[i]);
    ElemCoefDev* dcf = (ElemCoefDev*)c->buf("at_coef", sizeof(ElemCoefDev) * cf.size());
    CK(cudaMemcpyAsync(dcf, cf.data(), sizeof(ElemCoefDev) * cf.size(), cudaMemcpyHostToDevice, c->stream));
    d.coefs = dcf;
    d.x = x; d.y = y; d.z = z; d.sig = sg; d.occ = oc; d.elem = e; d.tables = t;
    d.n_elem = (int)tabs.size();
    d.rmax_all = 0.f;
    for (auto& tb : tabs) d.rmax_all = std::max(d.rmax_all, tb.rmax);
    return d;
}

// Displaced, sliced and slice-sorted atoms of a group of configurations.
struct SpecGroup {
    int nconf = 0;
    std::vector<int> confs;
    std::vector<int> ns;
    std::vector<double> z_init;
    int S_cap = 0;
    const float *ax = nullptr, *ay = nullptr, *aw = nullptr;
    const int* ae = nullptr;
    const unsigned* seg = nullptr;
    const int* ns_d = nullptr;
    const float4* pair_coef = nullptr;   // fine slicing: per-pair spline coefficients
    CellGrid cg;
};

inline float ord2f(unsigned k)
{
    unsigned b = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

SpecGroup build_specimen(ms_ctx* c, const ms_params& p, const AtomsDev& A, const std::vector<int>& confs,
                         const Physics& ph)
{
    SpecGroup g;
    g.confs = confs;
    g.nconf = (int)confs.size();
    const int64_t n = A.n, nc = g.nconf;
    cudaStream_t st = c->stream;
    int* dconf = (int*)c->buf("sp_conf", sizeof(int) * nc);
    CK(cudaMemcpyAsync(dconf, confs.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st));
    size_t fb = sizeof(float) * (size_t)(n * nc);
    float* xd = (float*)c->buf("sp_xd", fb);
    float* yd = (float*)c->buf("sp_yd", fb);
    float* zd = (float*)c->buf("sp_zd", fb);
    launch_displace(A.x, A.y, A.z, A.sig, n, dconf, (int)nc, p.pn_seed, p.pn_dim_x, p.pn_dim_y, p.pn_dim_z, xd, yd,
                    zd, st);
    unsigned* zr = (unsigned*)c->buf("sp_zr", sizeof(unsigned) * 2 * nc);
    launch_zrange(zd, n, (int)nc, zr, zr + nc, st);
    std::vector<unsigned> zh(2 * nc);
    CK(cudaMemcpyAsync(zh.data(), zr, sizeof(unsigned) * 2 * nc, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // slicing planes on the host, bit-identical with the device arithmetic
    const float dz = (float)p.dz;
    const int border = border_of(p);
    std::vector<int> nv(nc);
    std::vector<float> vmax(nc);
    g.ns.resize(nc);
    g.z_init.resize(nc);
    int S_cap = 1;
    const bool fine = p.enable_fine_slicing != 0;
    const float rint = fine ? fine_radius(p) : 0.0f;
    // the planes' range: the atoms' z range, grown by the integration radius under fine slicing
    auto plane_lo = [&](float lo) { return fine ? MSF_SUB(lo, rint) : lo; };
    auto plane_hi = [&](float hi) { return fine ? MSF_ADD(hi, rint) : hi; };
    for (int i = 0; i < nc; i++) {
        float lo = ord2f(zh[i]), hi = ord2f(zh[nc + i]);
        nv[i] = det_nplanes(plane_lo(lo), plane_hi(hi), dz);
        vmax[i] = hi;
        g.ns[i] = nv[i] - 1;
        S_cap = std::max(S_cap, g.ns[i]);
    }
    MS_REQUIRE(S_cap <= 100000, MS_ERR_INVALID_ARG, "more than 100000 slices");
    const int bstride = S_cap + 1;
    std::vector<float> bounds((size_t)nc * bstride, 0.0f);
    for (int i = 0; i < nc; i++) {
        float lo = ord2f(zh[i]), hi = ord2f(zh[nc + i]);
        for (int k = 0; k < nv[i]; k++)
            bounds[(size_t)i * bstride + k] = det_plane(k, nv[i], plane_lo(lo), plane_hi(hi), dz, border);
        float sum = bounds[(size_t)i * bstride] + bounds[(size_t)i * bstride + 1];
        g.z_init[i] = (double)(float)(0.5 * (double)sum);  // Slice::z_m (slice.hpp:19-22)
    }
    g.S_cap = S_cap;
    float* db = (float*)c->buf("sp_bounds", sizeof(float) * bounds.size());
    int* dnv = (int*)c->buf("sp_nv", sizeof(int) * nc);
    float* dvmax = (float*)c->buf("sp_vmax", sizeof(float) * nc);
    int* dns = (int*)c->buf("sp_ns", sizeof(int) * nc);
    CK(cudaMemcpyAsync(db, bounds.data(), sizeof(float) * bounds.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dnv, nv.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dvmax, vmax.data(), sizeof(float) * nc, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dns, g.ns.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st));
    // spatial cells: at least the largest cut-off and a quarter of a potential tile (64 x 32 pixels),
    // so a tile touches at most 7 x 5 cells
    const double cell = std::max({(double)A.rmax_all, 16.0 * p.lx / p.nx, 16.0 * p.ly / p.ny, 0.25});
    g.cg.ncx = std::max(1, (int)std::ceil(p.lx / cell));
    g.cg.ncy = std::max(1, (int)std::ceil(p.ly / cell));
    g.cg.inv_cell = (float)(1.0 / cell);
    g.cg.lx = (float)p.lx;
    g.cg.ly = (float)p.ly;
    g.cg.wrap = p.pot_wrap ? 1 : 0;
    const int64_t nkeys64 = nc * (S_cap + 1) * (int64_t)g.cg.ncx * g.cg.ncy;
    MS_REQUIRE(nkeys64 < (1LL << 31), MS_ERR_UNSUPPORTED, "too many (configuration, slice, cell) bins");
    const int nkeys = (int)nkeys64;
    // fine slicing: up to maxper (atom, slice) pairs per atom, unused slots keyed past every bin
    const int maxper = fine ? (int)std::ceil(2.0 * rint / dz) + 4 : 1;
    const int64_t total = n * nc * maxper;
    MS_REQUIRE(total < (1LL << 31), MS_ERR_UNSUPPORTED, "atoms x configurations must stay below 2^31 per group");
    unsigned* keys = (unsigned*)c->buf("sp_keys", sizeof(unsigned) * total);
    unsigned* keys2 = (unsigned*)c->buf("sp_keys2", sizeof(unsigned) * total);
    int* vals = (int*)c->buf("sp_vals", sizeof(int) * total);
    int* vals2 = (int*)c->buf("sp_vals2", sizeof(int) * total);
    unsigned* counts = (unsigned*)c->buf("sp_counts", sizeof(unsigned) * (nkeys + 1));
    CK(cudaMemsetAsync(counts, 0, sizeof(unsigned) * (nkeys + 1), st));
    if (fine)
        launch_fine_assign(xd, yd, zd, n, (int)nc, db, bstride, dnv, dvmax, S_cap, g.cg, rint, maxper,
                           (unsigned)nkeys, keys, vals, counts, st);
    else
        launch_assign(xd, yd, zd, n, (int)nc, db, bstride, dnv, dvmax, S_cap, g.cg, keys, vals, counts, st);
    int end_bit = 1;
    while ((1LL << end_bit) <= nkeys) end_bit++;
    size_t tmp_bytes = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, vals, vals2, (int)total, 0, end_bit, st));
    void* tmp = c->buf("sp_sorttmp", tmp_bytes);
    CK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, vals, vals2, (int)total, 0, end_bit, st));
    unsigned* seg = (unsigned*)c->buf("sp_seg", sizeof(unsigned) * (nkeys + 1));
    size_t scan_bytes = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts, seg, nkeys + 1, st));
    void* scan_tmp = c->buf("sp_scantmp", scan_bytes);
    CK(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, counts, seg, nkeys + 1, st));
    float* ax = (float*)c->buf("sp_ax", sizeof(float) * total);
    float* ay = (float*)c->buf("sp_ay", sizeof(float) * total);
    float* aw = (float*)c->buf("sp_aw", sizeof(float) * total);
    int* ae = (int*)c->buf("sp_ae", sizeof(int) * total);
    if (fine) {
        float* az = (float*)c->buf("sp_az", sizeof(float) * total);
        launch_fine_gather(keys2, vals2, total, n, S_cap, g.cg, (unsigned)nkeys, xd, yd, zd, A.occ, A.elem,
                           (float)ph.vr_factor, ax, ay, aw, ae, az, st);
        // the z quadrature on [-1/2, 1/2] (nodes, then weights)
        double* qz = (double*)c->buf("fine_qz", sizeof(double) * 2 * kNqz);
        std::vector<double> q(2 * kNqz);
        gauss_legendre_half(kNqz, q.data(), q.data() + kNqz);
        CK(cudaMemcpyAsync(qz, q.data(), sizeof(double) * 2 * kNqz, cudaMemcpyHostToDevice, st));
        float4* tab = (float4*)c->buf("sp_fine_tab", sizeof(float4) * MS_NR * total);
        launch_fine_tables(keys2, az, ae, seg, (unsigned)nkeys, total, db, bstride, S_cap, g.cg, A.coefs,
                           p.pot_rmin > 0 ? p.pot_rmin : 0.01, p.pot_rmax > 0 ? p.pot_rmax : 3.0, qz, tab, st);
        g.pair_coef = tab;
    } else {
        launch_gather(keys2, vals2, total, n, S_cap, g.cg, xd, yd, A.occ, A.elem, (float)ph.vr_factor, ax, ay, aw,
                      ae, st);
    }
    g.ax = ax; g.ay = ay; g.aw = aw; g.ae = ae; g.seg = seg; g.ns_d = dns;
    return g;
}

PotArgs pot_args(const ms_params& p, const Setup& s, const AtomsDev& A, const SpecGroup& g, float* V,
                 int64_t conf_stride, int slice0, int nslice, int base)
{
    PotArgs a;
    std::memset(&a, 0, sizeof(a));
    a.ax = g.ax; a.ay = g.ay; a.aw = g.aw; a.ae = g.ae; a.seg = g.seg; a.ns = g.ns_d;
    a.S_cap = g.S_cap;
    a.slice0 = slice0;
    a.nslice = nslice;
    a.V = V;
    a.V_conf_stride = conf_stride;
    a.V_slice_base = base;
    a.nx = p.nx;
    a.ny = p.ny;
    a.dx = (float)s.gc.dx;
    a.dy = (float)s.gc.dy;
    a.lx = (float)p.lx;
    a.ly = (float)p.ly;
    a.ncx = g.cg.ncx;
    a.ncy = g.cg.ncy;
    a.inv_cell = g.cg.inv_cell;
    a.rmax_all = A.rmax_all;
    a.dx_hi = (float)s.gc.dx;
    a.dx_lo = (float)(s.gc.dx - (double)a.dx_hi);
    a.dy_hi = (float)s.gc.dy;
    a.dy_lo = (float)(s.gc.dy - (double)a.dy_hi);
    a.wrap = p.pot_wrap ? 1 : 0;
    a.elems = A.tables;
    a.n_elem = A.n_elem;
    a.pair_coef = g.pair_coef;
    return a;
}

// Potential chunks computed on a side stream when the context's potential overlap is on (see
// sim_tem_like); otherwise all slices in one launch before the slice loop.
constexpr int kPotChunk = 16;
struct PotChunks {
    std::vector<cudaEvent_t> ev;   // ev[k]: slices [k kPotChunk, (k+1) kPotChunk) are written
    void wait(ms_ctx* c, int slice) const
    {
        if (slice % kPotChunk == 0 && slice > 0 && (size_t)(slice / kPotChunk) < ev.size() && ev[slice / kPotChunk])
            CK(cudaStreamWaitEvent(c->stream, ev[slice / kPotChunk], 0));
    }
};

cudaStream_t pot_stream(ms_ctx* c)
{
    if (!c->pot_stream) CK(cudaStreamCreateWithFlags(&c->pot_stream, cudaStreamNonBlocking));
    return c->pot_stream;
}

cudaEvent_t chunk_event(ms_ctx* c, size_t k)
{
    while (c->chunk_ev.size() <= k) {
        cudaEvent_t e = nullptr;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->chunk_ev.push_back(e);
    }
    return c->chunk_ev[k];
}

PotChunks launch_potential_chunks(ms_ctx* c, PotArgs a, int n_conf, int S)
{
    PotChunks pc;
    const int nchunk = (S + kPotChunk - 1) / kPotChunk;
    if (c->profile || nchunk <= 1 || !c->pot_overlap) {
        run_potential(c, a, n_conf, c->stream);
        return pc;
    }
    pc.ev.assign((size_t)nchunk, nullptr);
    // the side stream starts once the specimen (sorted atoms) is ready on the context stream
    cudaEvent_t ready = chunk_event(c, 0);
    CK(cudaEventRecord(ready, c->stream));
    cudaStream_t side = pot_stream(c);
    CK(cudaStreamWaitEvent(side, ready, 0));
    PotArgs a0 = a;
    a0.slice0 = 0;
    a0.nslice = std::min(kPotChunk, S);
    launch_potential(a0, n_conf, c->stream);
    for (int k = 1; k < nchunk; k++) {
        PotArgs ak = a;
        ak.slice0 = k * kPotChunk;
        ak.nslice = std::min(kPotChunk, S - k * kPotChunk);
        launch_potential(ak, n_conf, side);
        pc.ev[k] = chunk_event(c, (size_t)k);
        CK(cudaEventRecord(pc.ev[k], side));
    }
    return pc;
}

// The potential kernel writing the transmission function t = exp(i V) (complex) instead of V:
// the slice passes then read t, and the exponential is formed once per pixel and slice in the
// potential kernel, instead of once per wave in the latency-bound row pass.
PotArgs with_transmission(PotArgs a, float2* T, const Setup& s)
{
    a.T = T;
    a.exptab = s.exptab;
    return a;
}

PassArgs pass_args(const Setup& s, float2* psi, const WaveInfo* waves, const float* sV, int64_t slot_stride,
                   const LensDev& lens)
{
    PassArgs a;
    std::memset(&a, 0, sizeof(a));
    a.psi = psi;
    a.waves = waves;
    a.sV = sV;
    a.sV_slot_stride = slot_stride;
    a.sV_slice_base = 0;
    a.prop_x = s.prop_x;
    a.prop_y = s.prop_y;
    a.prop = s.prop;
    a.propT = s.propT;
    a.exptab = s.exptab;
    a.grid = s.gd;
    a.lens = lens;
    a.variant = s.variant;
    a.err = s.err;
    return a;
}

// The waves of a batch stay in L2 between the passes (evict-last) when they take at most 72 MiB of
// the 126 MB L2 next to the 16 MiB propagator table; the transmission slices then stream through.
int l2_mode_for_waves(int nwaves, int64_t N)
{
    return (double)nwaves * (double)N * sizeof(float2) <= 72.0 * 1024 * 1024 ? L2_WAVES_RESIDENT : L2_DEFAULT;
}

// Tile shape of the hot passes (row step on the transmission store, column step) for a batch of
// nw waves on an nx x ny grid: forced by ms_set_tile_shape, else the fastest of the four
// combinations of wide and narrow row and column tiles, timed on the call's own transmission store
// (slices 0..nslices-1), wave descriptors and wave buffer, before the wave is set up.  Each timing covers enough slice
// steps for about 2 ms of work (at least two), so that a single small wave is timed above the
// event resolution; a shape's time is the best of two timed rounds after one untimed round.  The
// choice is kept per device, grid and batch size in the context and in the JSON cache file when
// one is set.  Under a profiler the timings are distorted: a cache file written by a plain run
// keeps the choice of a profiled run the same.
int choose_tile(ms_ctx* c, PassArgs pa, int nx, int ny, int nw, int nslices, cudaStream_t st)
{
    if (c->tile_shape >= 0) return c->tile_shape;
    if ((!pa.tt && !pa.sV) || pa.variant == PASS_PIPELINED || nslices <= 0) return TILE_WIDE;
    char key[64];
    std::snprintf(key, sizeof(key), "%d,%d,%d", nx, ny, nw);
    auto it = c->tile_choice.find(key);
    if (it != c->tile_choice.end()) return it->second;
    if (c->profile) return TILE_WIDE;   // per-launch events would time the events
    // the steps run on the call's own wave buffer (pa.psi), before the probe or the plane wave
    // is written into it: every caller fills the buffer completely before its slice loop reads it
    pa.flags = 0;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // the warp-column step joins the candidates on 1024-point columns with transposed tables
    const bool warp_cols = ny == 1024 && pa.propT != nullptr;
    constexpr int kShapes[6] = {TILE_WIDE, TILE_NARROW_ROWS, TILE_NARROW_COLS, TILE_NARROW, TILE_WARP_COLS,
                                TILE_WARP_COLS | TILE_NARROW_ROWS};
    const int nshape = warp_cols ? 6 : 4;
    float t_best[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int steps = 2;
    auto launch_steps = [&](int shape) {
        pa.tile = shape;
        for (int sl = 0; sl < steps; sl++) {
            pa.slice = sl % nslices;
            pa.tw = twiddles(c, nx);
            launch_row(nx, ROW_INV_T_FWD, pa, nw, ny, st);
            pa.tw = twiddles(c, ny);
            launch_col(ny, COL_STEP, pa, nw, nx, st);
        }
    };
    // The slice loops these shapes serve replay from CUDA graphs, so the timed steps replay from
    // graphs too when the stream allows a capture: timed as direct launches, a small wave's steps
    // are bound by the host's launch rate and every shape looks the same.
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const bool graphs = c->use_graphs && st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread &&
                        cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone;
    cudaGraphExec_t ge[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    struct GeFree {
        cudaGraphExec_t* g;
        ~GeFree()
        {
            for (int i = 0; i < 6; i++)
                if (g[i]) cudaGraphExecDestroy(g[i]);
        }
    } ge_free{ge};
    // the first pass over the shapes warms them up (the first launch of a kernel also loads it);
    // the step count of the two timed passes comes from two more steps of the wide shape
    for (int rep = 0; rep < 3; rep++) {
        if (rep == 1) {
            CK(cudaEventRecord(e0, st));
            launch_steps(TILE_WIDE);
            CK(cudaEventRecord(e1, st));
            CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            steps = std::max(2, std::min(64, (int)(2.0 * steps / std::max(ms, 1e-3f))));
        }
        for (int si = 0; si < nshape; si++) {
            if (graphs && rep == 1 && !ge[si]) {
                const int64_t l0 = kernel_launches();
                CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                try {
                    launch_steps(kShapes[si]);
                } catch (...) {
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(st, &g);
                    if (g) cudaGraphDestroy(g);
                    cudaGetLastError();
                    throw;
                }
                cudaGraph_t g = nullptr;
                CK(cudaStreamEndCapture(st, &g));
                const cudaError_t e = cudaGraphInstantiate(&ge[si], g, 0);
                cudaGraphDestroy(g);
                CK(e);
                add_kernel_launches(-(kernel_launches() - l0));   // captured, not run
            }
            CK(cudaEventRecord(e0, st));
            if (ge[si]) CK(cudaGraphLaunch(ge[si], st));
            else launch_steps(kShapes[si]);
            CK(cudaEventRecord(e1, st));
            CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (rep == 1 || (rep == 2 && ms < t_best[si])) t_best[si] = ms;
        }
    }
    int best = TILE_WIDE;
    for (int si = 1; si < nshape; si++)
        if (t_best[si] < t_best[best]) best = si;
    best = kShapes[best];
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->tile_choice[key] = best;
    tune_save(c);
    return best;
}

// The whole slice loop of a wave batch in one persistent launch (slice_engine.cuh), from slice
// `slice0` to each wave's last.  ns[w] is wave w's slice count; the items of slice s cover the
// waves up to the last one with more than s slices (waves inside that prefix whose slices are
// done skip their items).  engine_plan uploads the item table and clears the counters on the
// stream; the launch that follows it (engine_launch, possibly captured in a graph) consumes them.
EngineArgs engine_plan(ms_ctx* c, const std::vector<int>& ns, int slice0, int N, cudaStream_t st,
                       unsigned long long* done_ns, const std::string& tag = std::string())
{
    const int nw = (int)ns.size();
    int S_end = 0;
    for (int v : ns) S_end = std::max(S_end, v);
    const int S = std::max(0, S_end - slice0);
    // row blocks / column tiles per work item: as many as keep the items of one slice phase at
    // least four times the resident blocks (fewer, larger items mean fewer dependency checks and
    // completion counts per slice)
    int sub = 1;
    const int64_t resident = 2LL * num_sms();
    while (sub < 8 && (int64_t)nw * (N / engine_rows(N)) / (2 * sub) >= 4 * resident) sub *= 2;
    const int RB = N / engine_rows(N) / sub, CT = N / engine_cols(N) / sub;
    std::vector<int> start(2 * (size_t)S + 1);
    int t = 0;
    for (int j = 0; j < S; j++) {
        int nact = nw;
        while (nact > 0 && ns[nact - 1] <= slice0 + j) nact--;
        start[2 * j] = t;
        t += nact * RB;
        start[2 * j + 1] = t;
        t += nact * CT;
    }
    start[2 * (size_t)S] = t;
    EngineArgs e;
    std::memset(&e, 0, sizeof(e));
    e.state = (EngineState*)c->buf("eng_state" + tag, sizeof(EngineState));
    int* dstart = (int*)c->buf("eng_start" + tag, sizeof(int) * start.size());
    unsigned* cnt = (unsigned*)c->buf("eng_cnt" + tag, sizeof(unsigned) * 2 * nw);
    CK(cudaMemsetAsync(e.state, 0, sizeof(EngineState), st));
    CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned) * 2 * nw, st));
    // pageable source: the copy has read the table when the call returns
    CK(cudaMemcpyAsync(dstart, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice, st));
    e.phase_start = dstart;
    e.n_items = t;
    e.S_max = S;
    e.slice0 = slice0;
    e.sub = sub;
    e.rows_done = cnt;
    e.cols_done = cnt + nw;
    e.done_ns = done_ns;
    return e;
}

// Whether the engine runs a batch: selected (everywhere, or by default for an uneven batch's grid
// groups), a square grid (one layout serves rows and columns), the plain slice step (no stored
// inputs, filters or vacuum continuation), and tensor-map encoding (its column items' tile loads);
// otherwise the batch runs slice by slice.
bool engine_fits(const ms_ctx* c, int nx, int ny, int flags, bool uneven = false)
{
    const bool wanted = c->pass_variant == PASS_ENGINE || (uneven && c->pass_variant == PASS_CLASSIC);
    return wanted && nx == ny && tensor_maps_available() &&
           !(flags & (PF_STORE_X | PF_FILTER_AUX | PF_VACUUM_BEYOND | PF_PROP_ALWAYS | PF_TILT_INCIDENT));
}

void engine_launch(const PassArgs& pa, const EngineArgs& e, int N, int nwaves, cudaStream_t st)
{
    if (e.n_items <= 0) return;
    EngineArgs ee = e;
    ee.wait_cycles = pa.wait_cycles;
    if (!launch_slice_engine(N, pa.tt ? ROW_INV_TT_FWD : ROW_INV_T_FWD, pa, ee, nwaves, st))
        throw MsError(MS_ERR_INTERNAL, "the slice engine could not be launched (wave alignment or tensor map)");
}

// Device time and launches of one call; the context's wait-error word is cleared at the start and
// read at the end (a kernel whose bounded wait ran out has set it).
struct Timer {
    ms_ctx* c;
    int64_t l0;
    explicit Timer(ms_ctx* cc) : c(cc), l0(kernel_launches())
    {
        CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
        CK(cudaEventRecord(c->ev0, c->stream));
    }
    void stop()
    {
        CK(cudaEventRecord(c->ev1, c->stream));
        CK(cudaEventSynchronize(c->ev1));
        int e = 0;
        CK(cudaMemcpy(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e & 1) throw MsError(MS_ERR_TIMEOUT, "a device-side wait for a shared-memory tile ran out");
        if (e) throw MsError(MS_ERR_TIMEOUT, "a device-side wait for another block's slice work ran out");
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        c->last_ms = ms;
        c->last_launches = kernel_launches() - l0;
        if (c->profile) c->prof_resolve();
    }
};

// free device memory budget for the potential store
size_t free_budget(ms_ctx* c)
{
    return (size_t)(c->free_mem() * 0.6);
}

void copy_out(ms_ctx* c, float* dst, const float* src, int64_t n, int on_dev)
{
    CK(cudaMemcpyAsync(dst, src, sizeof(float) * n, on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       c->stream));
}

int estimate_slices(const ms_params& p, const ms_atoms& a)
{
    float lo = a.z[0], hi = a.z[0], smax = 0.f;
    for (int64_t i = 0; i < a.n; i++) {
        lo = std::min(lo, a.z[i]);
        hi = std::max(hi, a.z[i]);
        smax = std::max(smax, a.sigma[i]);
    }
    const float grow = p.enable_fine_slicing ? 2.0f * fine_radius(p) : 0.0f;
    return (int)((hi - lo + 12.0f * smax + grow) / (float)p.dz) + 3;
}

// device bytes per configuration of the fine-slicing pair tables and sort buffers
size_t fine_bytes_per_conf(const ms_params& p, const ms_atoms& a)
{
    if (!p.enable_fine_slicing) return 0;
    const int maxper = (int)std::ceil(2.0 * fine_radius(p) / (float)p.dz) + 4;
    return (size_t)a.n * maxper * (sizeof(float) * 4 * MS_NR + 48);
}

}  // namespace

void ctx_activate(ms_ctx* c)
{
    CK(cudaSetDevice(c->device));
    if (!c->d_err) {
        CK(cudaMalloc(&c->d_err, sizeof(int)));
        c->forget_free_mem();
        CK(cudaMemset(c->d_err, 0, sizeof(int)));
    }
}

// ---------------------------------------------------------------------------
// HRTEM / ED (ED_HRTEM, single_simulator.cuh:11-126) and CBED (CBED_CBEI, :128-206)
// ---------------------------------------------------------------------------
namespace {
// Launch arguments that a captured batch graph bakes in, as a byte string.
std::string graph_key_of(const PassArgs& pa, int nb, int S, int nblk, int ndet, const void* partial,
                         const void* Iw, const void* img, const void* thr, int npos)
{
    std::string k((const char*)&pa, sizeof(PassArgs));
    const int ints[5] = {nb, S, nblk, ndet, npos};
    const void* ptrs[4] = {partial, Iw, img, thr};
    k.append((const char*)ints, sizeof(ints));
    k.append((const char*)ptrs, sizeof(ptrs));
    return k;
}

// Runs `body` (launches only) on the context stream through a cached CUDA graph: captured on
// first use or when `key` changes, replayed otherwise.  Falls back to direct launches while
// profiling (per-launch events), on the legacy default stream, or when the stream is already
// being captured by the caller.
template <class F>
void run_graphed(ms_ctx* c, const std::string& key, F&& body)
{
    cudaStream_t st = c->stream;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    bool ok = c->use_graphs && !c->profile && st != nullptr && st != cudaStreamLegacy &&
              st != cudaStreamPerThread && cudaStreamIsCapturing(st, &cs) == cudaSuccess &&
              cs == cudaStreamCaptureStatusNone;
    if (!ok) {
        body();
        return;
    }
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) {
        if (c->graphs.size() >= 4) c->drop_graph();   // full batches, the last partial batch, ...
        const int64_t l0 = kernel_launches();
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            body();
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
        cudaGraph_t g = nullptr;
        CK(cudaStreamEndCapture(st, &g));
        cudaGraphExec_t ge = nullptr;
        cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        CK(e);
        ms_ctx::Graph gr;
        gr.exec = ge;
        gr.launches = kernel_launches() - l0;
        add_kernel_launches(-gr.launches);   // captured, not run
        it = c->graphs.emplace(key, gr).first;
    }
    CK(cudaGraphLaunch(it->second.exec, st));
    add_kernel_launches(it->second.launches);
}
}  // namespace

void sim_tem_like(ms_ctx* c, const ms_params& p, const ms_atoms& a, ms_output* out, bool force_cbed,
                  const DefocusSeries* series)
{
    validate_params(p);
    validate_atoms(p, &a);
    MS_REQUIRE(out != nullptr, MS_ERR_INVALID_ARG, "output is NULL");
    const bool kspace = force_cbed || p.simulation_type != MS_SIM_HRTEM;
    const bool full = p.data_record == MS_RECORD_WAVE;
    const int nser = series ? series->n : 0;
    if (series) {
        MS_REQUIRE(!kspace, MS_ERR_INVALID_ARG, "a defocus series needs simulation_type HRTEM");
        MS_REQUIRE(nser >= 1 && series->df != nullptr, MS_ERR_INVALID_ARG, "need at least one defocus value");
        MS_REQUIRE(p.illumination_model == 0 || p.illumination_model == MS_ILLUM_COHERENT, MS_ERR_UNSUPPORTED,
                   "a defocus series images with the coherent CTF (apply_CTF_kernel_batch)");
        for (int i = 0; i < nser; i++)
            MS_REQUIRE(std::isfinite(series->df[i]), MS_ERR_INVALID_ARG, "defocus values must be finite");
    }
    const int nimg = std::max(1, nser);
    MS_REQUIRE(full ? (out->image_real && out->image_imag) : (out->image_intensity != nullptr), MS_ERR_INVALID_ARG,
               "output buffers for the requested data_record are NULL");
    ctx_activate(c);
    cudaStream_t st = c->stream;
    Timer tm(c);
    Setup s = make_setup(c, p);
    const int64_t N = s.N;
    AtomsDev A = upload_atoms(c, p, a);
    ConfSet cs = conf_set(p);
    const int iw = force_cbed ? (p.iw_type > 0 ? p.iw_type : MS_IW_CONVERGENT) : iw_of(p);
    LensDev cond = lens_dev(lens_coef(p.cond_lens, s.ph.lambda, 0.0));
    LensDev obj = lens_dev(lens_coef(p.obj_lens, s.ph.lambda, 0.0));

    // configurations per group: potential store + waves must fit the memory budget
    int S_est = estimate_slices(p, a);
    size_t per_conf = (size_t)S_est * N * 8 + (size_t)N * 8 * 2 + (size_t)N * 4 + (size_t)a.n * 40 +
                      fine_bytes_per_conf(p, a);
    int gsize = (int)std::max<size_t>(1, std::min<size_t>(cs.confs.size(), free_budget(c) / per_conf));

    double* acc = (double*)c->buf("acc0", sizeof(double) * N * nimg);
    double* acc_im = full ? (double*)c->buf("acc1", sizeof(double) * N * nimg) : nullptr;
    bool first = true;
    int ns_first = 0;
    for (size_t g0 = 0; g0 < cs.confs.size(); g0 += gsize) {
        std::vector<int> confs(cs.confs.begin() + g0, cs.confs.begin() + std::min(cs.confs.size(), g0 + gsize));
        SpecGroup g = build_specimen(c, p, A, confs, s.ph);
        if (g0 == 0) ns_first = g.ns[0];
        const int nw = g.nconf;
        const int64_t slot = (int64_t)g.S_cap * N;
        // the slices as a transmission store t = exp(iσV) (8 bytes per pixel, formed once per pixel in
        // the potential kernel) or as a σV store (4 bytes, t formed in the row step)
        float2* sT = c->trans_store ? (float2*)c->buf("sT", sizeof(float2) * slot * nw) : nullptr;
        float* sVs = c->trans_store ? nullptr : (float*)c->buf("sVs", sizeof(float) * slot * nw);
        // Potentials of every slice before the loop (default), or, with the overlap switched on, in
        // chunks of kPotChunk slices: the first on the context stream, the rest on a side stream while
        // the slice passes of earlier slices run; the row pass of the first slice of each chunk then
        // waits for that chunk's event.  With per-launch profiling on, all run in order.
        const PotArgs pa0 = pot_args(p, s, A, g, sVs, slot, 0, g.S_cap, 0);
        PotChunks pc = launch_potential_chunks(c, sT ? with_transmission(pa0, sT, s) : pa0, nw, g.S_cap);
        std::vector<WaveInfo> wv(nw);
        for (int i = 0; i < nw; i++) {
            wv[i].px = p.iw_x;
            wv[i].py = p.iw_y;
            wv[i].cc10 = gate_coef(-kPi * (p.cond_lens.c10 + g.z_init[i]) * s.ph.lambda);
            wv[i].conf_slot = i;
            wv[i].n_slices = g.ns[i];
            wv[i].weight = (float)cs.weight;
            wv[i].pos = 0;
        }
        WaveInfo* dwv = (WaveInfo*)c->buf("waves", sizeof(WaveInfo) * nw);
        CK(cudaMemcpyAsync(dwv, wv.data(), sizeof(WaveInfo) * nw, cudaMemcpyHostToDevice, st));
        float2* psi = (float2*)c->buf("psi", sizeof(float2) * N * nw);
        PassArgs pa = pass_args(s, psi, dwv, sVs, slot, cond);
        pa.l2_mode = l2_mode_for_waves(nw, N);
        pa.tt = sT;
        pa.tile = choose_tile(c, pa, p.nx, p.ny, nw, g.S_cap, st);
        c->last_tile = pa.tile;
        if (iw == MS_IW_CONVERGENT) {
            pa.tw = s.tw_y;
            run_col(c, p.ny, COL_PROBE_INV, pa, nw, p.nx, st);
        }
        const int S_max = *std::max_element(g.ns.begin(), g.ns.end());
        const bool plane = iw == MS_IW_PLANE || iw == MS_IW_PLANE_TILTED;
        // with the persistent engine, a plane wave's first slice (no inverse row transform, the
        // tilt) runs as separate passes and the engine takes the slices after it
        const bool eng = engine_fits(c, p.nx, p.ny, pa.flags);
        const int sl_end = eng ? (plane ? std::min(1, S_max) : 0) : S_max;
        auto slices = [&] {
            PassArgs q = pa;
            for (int sl = 0; sl < sl_end; sl++) {
                pc.wait(c, sl);
                q.slice = sl;
                q.tw = s.tw_x;
                PassArgs pr = q;
                if (sl == 0 && iw == MS_IW_PLANE_TILTED) pr.flags |= PF_TILT_INCIDENT;
                run_row(c, p.nx, (sl == 0 && plane) ? ROW_T_FWD : ROW_INV_T_FWD, pr, nw, p.ny, st);
                q.tw = s.tw_y;
                PassArgs pq = q;
                if (c->inject == MS_INJECT_WAIT_TIMEOUT) pq.flags |= PF_TEST_WAIT;
                run_col(c, p.ny, COL_STEP, pq, nw, p.nx, st);
            }
        };
        if (pc.ev.size() <= 1 && sl_end > 1) {
            // the slice loop replays from a captured graph (no potential chunks to wait for)
            std::string key = graph_key_of(pa, nw, sl_end, iw, c->inject, nullptr, nullptr, nullptr, nullptr, -1);
            run_graphed(c, key, slices);
        } else {
            slices();
        }
        if (eng) {
            for (int sl = sl_end; sl < S_max; sl++) pc.wait(c, sl);
            PassArgs pe = pa;
            pe.tw = s.tw_x;
            if (c->inject == MS_INJECT_WAIT_TIMEOUT) pe.flags |= PF_TEST_WAIT;
            const EngineArgs e = engine_plan(c, g.ns, sl_end, p.nx, st, nullptr);
            timed(c, "engine", [&] { engine_launch(pe, e, p.nx, nw, st); });
        }
        const int illum = p.illumination_model ? p.illumination_model : MS_ILLUM_COHERENT;
        const int tsi = p.temporal_spatial_incoh ? p.temporal_spatial_incoh : MS_TSI_TEMPORAL_SPATIAL;
        if (!kspace && illum == MS_ILLUM_TCC && tsi != MS_TSI_COHERENT) {
            // TCC_TEM (lens_modulation.cuh:130-176): every (source point, defocus node) pair images a
            // copy of the exit wave; intensities (or complex fields) add with the quadrature weights
            const ms_lens& OL = p.obj_lens;
            std::vector<double> xt, wt, xs, ws;
            gauss_hermite(tsi == MS_TSI_SPATIAL ? 1 : OL.dsf_npoints, &xt, &wt);
            gauss_hermite(tsi == MS_TSI_TEMPORAL ? 1 : OL.ssf_npoints, &xs, &ws);
            const double df_hw = std::sqrt(2.0) * OL.dsf_sigma;        // dsf_iehwgd
            const double sf_hw = std::sin(OL.ssf_beta) / s.ph.lambda;  // ssf_iehwgd (lens_dev.cuh:143-148)
            float2* q = (float2*)c->buf("tcc_q", sizeof(float2) * N * nw);
            float2* aux = full ? (float2*)c->buf("aux", sizeof(float2) * N * nw) : nullptr;
            float* img = full ? nullptr : (float*)c->buf("img_w", sizeof(float) * N * nw);
            bool firstq = true;
            for (size_t iy = 0; iy < xs.size(); iy++)
                for (size_t ix = 0; ix < xs.size(); ix++)
                    for (size_t j = 0; j < xt.size(); j++) {
                        const double wq = ws[ix] * ws[iy] * wt[j];
                        LensDev Lq = lens_dev(lens_coef(OL, s.ph.lambda, df_hw * xt[j]));
                        Lq.gxu = sf_hw * xs[ix];
                        Lq.gyu = sf_hw * xs[iy];
                        Lq.amp = full ? wq : std::sqrt(wq);
                        CK(cudaMemcpyAsync(q, psi, sizeof(float2) * N * nw, cudaMemcpyDeviceToDevice, st));
                        PassArgs pq = pa;
                        pq.psi = q;
                        pq.lens = Lq;
                        pq.tw = s.tw_y;
                        run_col(c, p.ny, COL_CTF_INV, pq, nw, p.nx, st);
                        pq.tw = s.tw_x;
                        if (full) {
                            pq.aux = aux;
                            run_row(c, p.nx, ROW_INV_STORE, pq, nw, p.ny, st);
                            launch_acc_cplx(aux, nw, dwv, N, acc, acc_im, first && firstq, st);
                        } else {
                            pq.out_real = img;
                            pq.flags = firstq ? 0 : PF_ACCUMULATE;
                            run_row(c, p.nx, ROW_INV_ABS2, pq, nw, p.ny, st);
                        }
                        firstq = false;
                    }
            if (!full) launch_acc_real(img, nw, N, acc, first, st);
        } else if (!kspace && nser > 0) {
            // defocus series (apply_CTF_kernel_batch, device_kernels.cuh:469-503): the exit waves of the
            // group are copied once per defocus value into one batch whose wave descriptors carry
            // chi's defocus term -pi (C10 + df_i) lambda; one CTF column pass and one |.|^2 row pass
            // cover the chunk, then each defocus value's images are summed over configurations
            const int per = std::max(1, (int)std::min<int64_t>(nser, (int64_t)(free_budget(c) / 4 / ((size_t)N * 8 * nw))));
            float2* q = (float2*)c->buf("ser_q", sizeof(float2) * N * nw * per);
            float2* aux = full ? (float2*)c->buf("ser_aux", sizeof(float2) * N * nw * per) : nullptr;
            float* img = full ? nullptr : (float*)c->buf("ser_img", sizeof(float) * N * nw * per);
            WaveInfo* dwq = (WaveInfo*)c->buf("ser_waves", sizeof(WaveInfo) * nw * per);
            std::vector<WaveInfo> wq((size_t)nw * per);
            for (int d0 = 0; d0 < nser; d0 += per) {
                const int nd = std::min(per, nser - d0);
                for (int i = 0; i < nd; i++) {
                    const double cc = gate_coef(-kPi * (p.obj_lens.c10 + series->df[d0 + i]) * s.ph.lambda);
                    for (int w = 0; w < nw; w++) {
                        wq[(size_t)i * nw + w] = wv[w];
                        wq[(size_t)i * nw + w].cc10 = cc;
                    }
                    CK(cudaMemcpyAsync(q + (size_t)i * nw * N, psi, sizeof(float2) * N * nw, cudaMemcpyDeviceToDevice,
                                       st));
                }
                CK(cudaMemcpyAsync(dwq, wq.data(), sizeof(WaveInfo) * nw * nd, cudaMemcpyHostToDevice, st));
                PassArgs pq = pa;
                pq.psi = q;
                pq.waves = dwq;
                pq.lens = obj;
                pq.flags = PF_WAVE_DEFOCUS;
                pq.tw = s.tw_y;
                run_col(c, p.ny, COL_CTF_INV, pq, nw * nd, p.nx, st);
                pq.flags = 0;
                pq.tw = s.tw_x;
                if (full) {
                    pq.aux = aux;
                    run_row(c, p.nx, ROW_INV_STORE, pq, nw * nd, p.ny, st);
                } else {
                    pq.out_real = img;
                    run_row(c, p.nx, ROW_INV_ABS2, pq, nw * nd, p.ny, st);
                }
                for (int i = 0; i < nd; i++) {
                    double* ai = acc + (size_t)(d0 + i) * N;
                    if (full)
                        launch_acc_cplx(aux + (size_t)i * nw * N, nw, dwq + (size_t)i * nw, N, ai,
                                        acc_im + (size_t)(d0 + i) * N, first, st);
                    else
                        launch_acc_real(img + (size_t)i * nw * N, nw, N, ai, first, st);
                }
                // the host wave table is rewritten for the next chunk
                CK(cudaStreamSynchronize(st));
            }
        } else if (!kspace) {
            // OL_modulation -> CTF_TEM (wave_function.cuh:96-110, lens_modulation.cuh:78-89), or
            // PCTF_TEM (:91-110) with the partially coherent envelope
            pa.lens = obj;
            if (illum == MS_ILLUM_PARTIAL) set_pctf(&pa.lens, p, s.ph.lambda);
            pa.tw = s.tw_y;
            run_col(c, p.ny, COL_CTF_INV, pa, nw, p.nx, st);
            pa.tw = s.tw_x;
            if (full) {
                float2* aux = (float2*)c->buf("aux", sizeof(float2) * N * nw);
                pa.aux = aux;
                run_row(c, p.nx, ROW_INV_STORE, pa, nw, p.ny, st);
                launch_acc_cplx(aux, nw, dwv, N, acc, acc_im, first, st);
            } else {
                float* img = (float*)c->buf("img_w", sizeof(float) * N * nw);
                pa.out_real = img;
                run_row(c, p.nx, ROW_INV_ABS2, pa, nw, p.ny, st);
                launch_acc_real(img, nw, N, acc, first, st);
            }
        } else {
            if (full) launch_acc_cplx(psi, nw, dwv, N, acc, acc_im, first, st);
            else launch_acc_abs2(psi, nw, dwv, N, acc, first, st);
        }
        first = false;
        CK(cudaStreamSynchronize(st));  // host wave table reused by the next group
    }
    float* o0 = (float*)c->buf("out0", sizeof(float) * N * nimg);
    for (int i = 0; i < nimg; i++) launch_emit(acc + (size_t)i * N, p.nx, p.ny, kspace ? 1 : 0, o0 + (size_t)i * N, st);
    if (full) {
        copy_out(c, out->image_real, o0, N * nimg, out->on_device);
        float* o1 = (float*)c->buf("out1", sizeof(float) * N * nimg);
        for (int i = 0; i < nimg; i++)
            launch_emit(acc_im + (size_t)i * N, p.nx, p.ny, kspace ? 1 : 0, o1 + (size_t)i * N, st);
        copy_out(c, out->image_imag, o1, N * nimg, out->on_device);
    } else {
        copy_out(c, out->image_intensity, o0, N * nimg, out->on_device);
    }
    tm.stop();
    out->row = p.ny;
    out->col = p.nx;
    out->n_slices = ns_first;
    out->interval_x = p.lx / p.nx;
    out->interval_y = p.ly / p.ny;
    out->total_intensity = 0.0;
}

// ---------------------------------------------------------------------------
// STEM (run_STEM_tile_simu, scan_simulator.cuh:11-113; plain form run_STEM_general_simu, :115-183)
// ---------------------------------------------------------------------------
namespace {
// Largest probe batch the memory budget allows (the waves take at most a quarter of free memory).
int batch_cap(ms_ctx* c, int64_t N)
{
    const size_t fr = c->free_mem();
    int64_t cap = (int64_t)(fr * 0.25 / (double)(N * 8));
    return (int)std::min<int64_t>(256, std::max<int64_t>(1, cap));
}

// Probe-batch autotuner: times one probe generation and two slice steps (row + column pass)
// for each candidate batch size on the call's own grid and potentials, and keeps the size
// with the highest probe*slice rate.  The choice is cached in the context per grid, slice
// count and cap.  Candidates are powers of two from 32 to 256 within the memory cap.
int autotune_batch(ms_ctx* c, const ms_params& p, const Setup& s, const PassArgs& base, const WaveInfo& w0, int S,
                   int npos, int cap)
{
    const int hi = std::min(cap, npos);
    std::vector<int> cand;
    for (int b = 32; b <= 256; b *= 2)
        if (b <= hi) cand.push_back(b);
    if (cand.empty()) return std::max(1, hi);
    if (cand.size() == 1 || c->profile) return cand.back();
    char key[96];
    std::snprintf(key, sizeof(key), "%d,%d,%d,%d", p.nx, p.ny, std::min(S, 2), hi);
    auto it = c->batch_choice.find(key);
    if (it != c->batch_choice.end()) return std::max(1, std::min(it->second, hi));
    cudaStream_t st = c->stream;
    const int bmax = cand.back();
    std::vector<WaveInfo> wv((size_t)bmax, w0);
    WaveInfo* dwv = (WaveInfo*)c->buf("waves_tune", sizeof(WaveInfo) * bmax);
    CK(cudaMemcpyAsync(dwv, wv.data(), sizeof(WaveInfo) * bmax, cudaMemcpyHostToDevice, st));
    float2* psi = (float2*)c->buf("psi", sizeof(float2) * s.N * bmax);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int best = cand.back();
    double best_rate = -1.0;
    PassArgs pa = base;
    pa.psi = psi;
    pa.waves = dwv;
    for (int rep = 0; rep < 2; rep++) {   // the first round warms up every candidate
        for (int b : cand) {
            CK(cudaEventRecord(e0, st));
            pa.tw = s.tw_y;
            launch_col(p.ny, COL_PROBE_INV, pa, b, p.nx, st);
            for (int sl = 0; sl < 2; sl++) {
                pa.slice = std::min(sl, S - 1);
                pa.tw = s.tw_x;
                launch_row(p.nx, ROW_INV_T_FWD, pa, b, p.ny, st);
                pa.tw = s.tw_y;
                launch_col(p.ny, COL_STEP, pa, b, p.nx, st);
            }
            CK(cudaEventRecord(e1, st));
            CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            // a batch does one probe generation per S slice steps
            const double rate = (double)b * 2.0 / (ms * (1.0 + 0.5 / std::max(S, 1)));
            if (rep == 1 && rate > best_rate) {
                best_rate = rate;
                best = b;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->batch_choice[key] = best;
    tune_save(c);
    return best;
}

}  // namespace

// General scan (run_STEM_general_simu, scan_simulator.cuh:115-183): for every phonon configuration
// and probe position, the grid box is a window of lx x ly centred on the probe; the displaced atoms
// inside it +- 2 A are cropped and shifted into the window (remove_atoms_outside_xy_range,
// shift_atoms, :146-157), and the window is simulated with the probe at its centre.  A window
// without atoms records the unscattered probe's detector intensity (the blank intensity, :159-166):
// N^2 times the aperture pixels inside the detector.  The reference assigns each configuration's
// weighted intensity over the previous one; here the configurations are summed with their weights.
// Coordinates are cropped and shifted in float, as the reference's T = float code does.
void sim_stem_general(ms_ctx* c, const ms_params& p, const ms_atoms& a, ms_output* out)
{
    validate_params(p);
    validate_atoms(p, &a);
    MS_REQUIRE(p.simulation_type == MS_SIM_STEM, MS_ERR_INVALID_ARG, "simulation_type must be STEM");
    MS_REQUIRE(out != nullptr && out->stem_intensity != nullptr, MS_ERR_INVALID_ARG, "stem_intensity is NULL");
    ctx_activate(c);
    cudaStream_t st = c->stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    struct Ev {
        cudaEvent_t a, b;
        ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } ev{e0, e1};
    CK(cudaEventRecord(e0, st));
    const int64_t l0 = kernel_launches();
    const int npos = p.scan_nx * p.scan_ny, ndet = p.n_det;
    const int64_t N = (int64_t)p.nx * p.ny;
    const Physics ph = physics_of(p.E0, p.theta);
    // blank intensity per detector: N^2 per aperture pixel inside the detector's annulus
    std::vector<double> blank((size_t)ndet, 0.0);
    {
        const GridConst gc = grid_of(p, ph);
        const LensCoef L = lens_coef(p.cond_lens, ph.lambda, 0.0);
        for (int d = 0; d < ndet; d++) {
            const float gi = g2_threshold(p.det_inner[d], ph.lambda), go = g2_threshold(p.det_outer[d], ph.lambda);
            double cnt = 0.0;
            for (int iy = 0; iy < p.ny; iy++)
                for (int ix = 0; ix < p.nx; ix++) {
                    const float g2 = det_g2(ix, iy, p.nx, p.ny, gc.dgx_f, gc.dgy_f);
                    if (L.g2min <= g2 && g2 < L.g2max && gi <= g2 && g2 <= go) cnt += 1.0;
                }
            blank[d] = cnt * (double)N * (double)N;
        }
    }
    ConfSet cs = conf_set(p);
    std::vector<double> img((size_t)ndet * npos, 0.0);
    std::vector<float> xd(a.n), yd(a.n), zd(a.n);
    std::vector<int> cz;
    std::vector<float> cx, cy, czz, csig, cocc;
    ms_params q = p;
    q.phonon_model = MS_PHONON_STILL;   // the cropped atoms are already displaced
    q.pn_nconf = 1;
    q.exec_mode = MS_EXEC_BATCHED;
    q.scan_nx = q.scan_ny = 1;
    q.scan_x0 = 0.5 * p.lx;
    q.scan_y0 = 0.5 * p.ly;
    q.scan_dx = q.scan_dy = 0.0;
    q.probe_batch = 1;
    std::vector<float> Iw((size_t)ndet);
    for (int conf : cs.confs) {
        host_displace(p, a, conf, xd.data(), yd.data(), zd.data());
        for (int ip = 0; ip < npos; ip++) {
            const int ix = ip % p.scan_nx, iy = ip / p.scan_nx;
            const double px = p.scan_x0 + ix * p.scan_dx, py = p.scan_y0 + iy * p.scan_dy;
            const float xs = (float)(px - 0.5 * p.lx), ys = (float)(py - 0.5 * p.ly);
            const float xlo = xs - 2.0f, xhi = (xs + (float)p.lx) + 2.0f;
            const float ylo = ys - 2.0f, yhi = (ys + (float)p.ly) + 2.0f;
            cz.clear(); cx.clear(); cy.clear(); czz.clear(); csig.clear(); cocc.clear();
            for (int64_t k = 0; k < a.n; k++) {
                if (xd[k] < xlo || xd[k] > xhi || yd[k] < ylo || yd[k] > yhi) continue;
                cz.push_back(a.Z[k]);
                cx.push_back(xd[k] - xs);
                cy.push_back(yd[k] - ys);
                czz.push_back(zd[k]);
                csig.push_back(a.sigma ? a.sigma[k] : 0.0f);
                cocc.push_back(a.occ ? a.occ[k] : 1.0f);
            }
            if (cz.empty()) {
                for (int d = 0; d < ndet; d++) img[(size_t)d * npos + ip] += cs.weight * blank[d];
                continue;
            }
            ms_atoms w;
            w.n = (int64_t)cz.size();
            w.Z = cz.data();
            w.x = cx.data();
            w.y = cy.data();
            w.z = czz.data();
            w.sigma = csig.data();
            w.occ = cocc.data();
            ms_output o;
            std::memset(&o, 0, sizeof(o));
            o.stem_intensity = Iw.data();
            sim_stem(c, q, w, &o);
            for (int d = 0; d < ndet; d++) img[(size_t)d * npos + ip] += cs.weight * (double)Iw[d];
        }
    }
    std::vector<float> res(img.size());
    for (size_t k = 0; k < img.size(); k++) res[k] = (float)img[k];
    CK(cudaMemcpyAsync(out->stem_intensity, res.data(), sizeof(float) * res.size(),
                       out->on_device ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost, st));
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    c->last_ms = ms;
    c->last_launches = kernel_launches() - l0;
    c->last_batch = 1;
    out->row = p.scan_ny;
    out->col = p.scan_nx;
    out->interval_x = p.scan_dx;
    out->interval_y = p.scan_dy;
    out->n_slices = 0;
    double tot = 0.0;
    {
        const GridConst gc = grid_of(p, ph);
        const LensCoef L = lens_coef(p.cond_lens, ph.lambda, 0.0);
        for (int iy = 0; iy < p.ny; iy++)
            for (int ix = 0; ix < p.nx; ix++) {
                const float g2 = det_g2(ix, iy, p.nx, p.ny, gc.dgx_f, gc.dgy_f);
                if (L.g2min <= g2 && g2 < L.g2max) tot += 1.0;
            }
    }
    out->total_intensity = tot * (double)N * (double)N;
}

void sim_stem(ms_ctx* c, const ms_params& p, const ms_atoms& a, ms_output* out)
{
    if (p.exec_mode == MS_EXEC_GENERAL) {
        sim_stem_general(c, p, a, out);
        return;
    }
    validate_params(p);
    validate_atoms(p, &a);
    MS_REQUIRE(p.simulation_type == MS_SIM_STEM, MS_ERR_INVALID_ARG, "simulation_type must be STEM");
    MS_REQUIRE(out != nullptr && out->stem_intensity != nullptr, MS_ERR_INVALID_ARG, "stem_intensity is NULL");
    ctx_activate(c);
    cudaStream_t st = c->stream;
    Timer tm(c);
    Setup s = make_setup(c, p);
    const int64_t N = s.N;
    AtomsDev A = upload_atoms(c, p, a);
    ConfSet cs = conf_set(p);
    LensDev cond = lens_dev(lens_coef(p.cond_lens, s.ph.lambda, 0.0));
    const int npos = p.scan_nx * p.scan_ny, ndet = p.n_det;
    const bool plain = p.exec_mode == MS_EXEC_PLAIN;
    std::vector<float> thr(2 * ndet);
    for (int d = 0; d < ndet; d++) {
        thr[d] = g2_threshold(p.det_inner[d], s.ph.lambda);
        thr[ndet + d] = g2_threshold(p.det_outer[d], s.ph.lambda);
    }
    float* dthr = (float*)c->buf("det_thr", sizeof(float) * 2 * ndet);
    CK(cudaMemcpyAsync(dthr, thr.data(), sizeof(float) * 2 * ndet, cudaMemcpyHostToDevice, st));
    double* img = (double*)c->buf("stem_acc", sizeof(double) * ndet * npos);
    CK(cudaMemsetAsync(img, 0, sizeof(double) * ndet * npos, st));
    const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>(64, N / 4096));
    const int cap = plain ? 1 : (p.probe_batch > 0 ? std::min(p.probe_batch, npos) : batch_cap(c, N));
    int B = plain ? 1 : std::min(cap, npos);
    bool tuned = plain || p.probe_batch > 0;
    std::vector<WaveInfo> wv((size_t)npos);
    std::vector<double> Ih((size_t)ndet);
    for (int conf : cs.confs) {
        SpecGroup g = build_specimen(c, p, A, std::vector<int>{conf}, s.ph);
        const int S = g.ns[0];
        const double cc10 = gate_coef(-kPi * (p.cond_lens.c10 + g.z_init[0]) * s.ph.lambda);
        float2* sT;
        float* sVs = nullptr;   // σV store instead of the transmission store (ms_set_transmission_store)
        int64_t slot = (int64_t)S * N;
        if (!plain && !c->trans_store) {
            sT = nullptr;
            sVs = (float*)c->buf("sVs", sizeof(float) * slot);
            run_potential(c, pot_args(p, s, A, g, sVs, slot, 0, S, 0), 1, st);
        } else if (!plain) {
            sT = (float2*)c->buf("sT", sizeof(float2) * slot);
            run_potential(c, with_transmission(pot_args(p, s, A, g, nullptr, slot, 0, S, 0), sT, s), 1, st);
        } else {
            sT = (float2*)c->buf("sT1", sizeof(float2) * N);
        }
        // every scan position of this configuration, uploaded once (run_STEM_tile_simu's tile loop,
        // scan_simulator.cuh:57-104, without a host round trip per batch)
        for (int ip = 0; ip < npos; ip++) {
            const int ix = ip % p.scan_nx, iy = ip / p.scan_nx;
            wv[ip].px = p.scan_x0 + ix * p.scan_dx;
            wv[ip].py = p.scan_y0 + iy * p.scan_dy;
            wv[ip].cc10 = cc10;
            wv[ip].conf_slot = 0;
            wv[ip].n_slices = S;
            wv[ip].weight = (float)cs.weight;
            wv[ip].pos = ip;
        }
        WaveInfo* dwv_all = (WaveInfo*)c->buf("waves_all", sizeof(WaveInfo) * npos);
        CK(cudaMemcpyAsync(dwv_all, wv.data(), sizeof(WaveInfo) * npos, cudaMemcpyHostToDevice, st));
        if (!tuned) {
            PassArgs base = pass_args(s, nullptr, nullptr, nullptr, slot, cond);
            base.tt = sT;
            B = autotune_batch(c, p, s, base, wv[0], S, npos, cap);
            tuned = true;
        }
        WaveInfo* dwv = (WaveInfo*)c->buf("waves", sizeof(WaveInfo) * B);
        float2* psi = (float2*)c->buf("psi", sizeof(float2) * N * B);
        double* partial = (double*)c->buf("det_part", sizeof(double) * B * nblk * ndet);
        double* Iw = (double*)c->buf("det_I", sizeof(double) * B * ndet);
        for (int start = 0; start < npos; start += B) {
            const int nb = std::min(B, npos - start);
            CK(cudaMemcpyAsync(dwv, dwv_all + start, sizeof(WaveInfo) * nb, cudaMemcpyDeviceToDevice, st));
            PassArgs pa = pass_args(s, psi, dwv, sVs, plain ? 0 : slot, cond);
            pa.l2_mode = plain ? L2_DEFAULT : L2_SHARED_T;   // one transmission slice serves the whole batch
            pa.tt = sT;
            if (!plain) {
                pa.tile = choose_tile(c, pa, p.nx, p.ny, nb, S, st);
                c->last_tile = pa.tile;
            }
            if (!plain) {
                const bool eng = engine_fits(c, p.nx, p.ny, pa.flags);
                EngineArgs e;
                if (eng) e = engine_plan(c, std::vector<int>((size_t)nb, S), 0, p.nx, st, nullptr);
                auto body = [&] {
                    PassArgs q = pa;
                    q.tw = s.tw_y;
                    run_col(c, p.ny, COL_PROBE_INV, q, nb, p.nx, st);
                    if (eng) {
                        q.tw = s.tw_x;
                        timed(c, "engine", [&] { engine_launch(q, e, p.nx, nb, st); });
                    }
                    for (int sl = 0; sl < (eng ? 0 : S); sl++) {
                        q.slice = sl;
                        q.tw = s.tw_x;
                        run_row(c, p.nx, ROW_INV_T_FWD, q, nb, p.ny, st);
                        q.tw = s.tw_y;
                        run_col(c, p.ny, COL_STEP, q, nb, p.nx, st);
                    }
                    launch_detect(psi, nb, p.nx, p.ny, s.gd.dgx_f, s.gd.dgy_f, dthr, dthr + ndet, ndet, partial, nblk,
                                  st);
                    launch_det_finalize(partial, nb, nblk, ndet, dwv, Iw, img, npos, 1, st);
                };
                run_graphed(c, graph_key_of(pa, nb, S, nblk, ndet, partial, Iw, img, dthr, npos), body);
                continue;
            }
            // plain form (run_STEM_general_simu): one probe per launch, the slice potential
            // regenerated for every probe and slice (transmit -> generate_potential_single_slice,
            // transmission_function.cuh:107-111), a blocking read of the probe's detector sums
            // (integrated_intensity, wave_function.cuh:135-146)
            pa.tw = s.tw_y;
            run_col(c, p.ny, COL_PROBE_INV, pa, nb, p.nx, st);
            for (int sl = 0; sl < S; sl++) {
                pa.slice = sl;
                run_potential(c, with_transmission(pot_args(p, s, A, g, nullptr, 0, sl, 1, sl), sT, s), 1, st);
                pa.sV_slice_base = sl;
                pa.tw = s.tw_x;
                run_row(c, p.nx, ROW_INV_T_FWD, pa, nb, p.ny, st);
                pa.tw = s.tw_y;
                run_col(c, p.ny, COL_STEP, pa, nb, p.nx, st);
            }
            launch_detect(psi, nb, p.nx, p.ny, s.gd.dgx_f, s.gd.dgy_f, dthr, dthr + ndet, ndet, partial, nblk, st);
            launch_det_finalize(partial, nb, nblk, ndet, dwv, Iw, img, npos, 1, st);
            CK(cudaMemcpyAsync(Ih.data(), Iw, sizeof(double) * nb * ndet, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
    }
    c->last_batch = B;
    float* o = (float*)c->buf("stem_out", sizeof(float) * ndet * npos);
    launch_d2f(img, (int64_t)ndet * npos, o, st);
    copy_out(c, out->stem_intensity, o, (int64_t)ndet * npos, out->on_device);
    tm.stop();
    out->row = p.scan_ny;
    out->col = p.scan_nx;
    out->interval_x = p.scan_dx;
    out->interval_y = p.scan_dy;
    out->n_slices = 0;
    // total_intensity: vacuum exit intensity sum_k N^2 A(k) (the reference's blank intensity
    // table, scan_simulator.cuh:34); probes have |Psi0(k)| in {0,1}
    {
        LensCoef L = lens_coef(p.cond_lens, s.ph.lambda, 0.0);
        double tot = 0.0;
        for (int iy = 0; iy < p.ny; iy++)
            for (int ix = 0; ix < p.nx; ix++) {
                float g2 = det_g2(ix, iy, p.nx, p.ny, s.gd.dgx_f, s.gd.dgy_f);
                if (L.g2min <= g2 && g2 < L.g2max) tot += 1.0;
            }
        out->total_intensity = tot * (double)N * (double)N;
    }
}

// ---------------------------------------------------------------------------
// thickness series (run_thickness_simu, thickness_simulator.cuh:11-85)
// ---------------------------------------------------------------------------
void sim_thickness(ms_ctx* c, const ms_params& p, const ms_atoms& a, ms_output* out)
{
    validate_params(p);
    validate_atoms(p, &a);
    MS_REQUIRE(out != nullptr && out->thickness_frames != nullptr, MS_ERR_INVALID_ARG, "thickness_frames is NULL");
    MS_REQUIRE(p.thick_det >= 0 && p.thick_det < p.n_det, MS_ERR_INVALID_ARG, "thick_det must name a detector");
    ctx_activate(c);
    cudaStream_t st = c->stream;
    Timer tm(c);
    Setup s = make_setup(c, p);
    const int64_t N = s.N;
    AtomsDev A = upload_atoms(c, p, a);
    ConfSet cs = conf_set(p);
    LensDev cond = lens_dev(lens_coef(p.cond_lens, s.ph.lambda, 0.0));
    const int iw = iw_of(p);
    // frames follow the static specimen's slices (thickness_simulator.cuh:22-25)
    std::vector<int> sl0(a.n);
    int nf = host_slices(p, a.z, a.n, nullptr, nullptr);
    MS_REQUIRE((int64_t)nf * N <= out->thickness_capacity, MS_ERR_INVALID_ARG,
               "thickness_frames holds fewer than n_slices*ny*nx floats");
    float* frames = (float*)c->buf("frames", sizeof(float) * N * nf);
    CK(cudaMemsetAsync(frames, 0, sizeof(float) * N * nf, st));
    const float g2in = g2_threshold(p.det_inner[p.thick_det], s.ph.lambda);
    const float g2out = g2_threshold(p.det_outer[p.thick_det], s.ph.lambda);
    for (int conf : cs.confs) {
        SpecGroup g = build_specimen(c, p, A, std::vector<int>{conf}, s.ph);
        const int S = g.ns[0];
        const int64_t slot = (int64_t)S * N;
        float2* sT = (float2*)c->buf("sT", sizeof(float2) * slot);
        run_potential(c, with_transmission(pot_args(p, s, A, g, nullptr, slot, 0, S, 0), sT, s), 1, st);
        WaveInfo wv;
        wv.px = p.iw_x;
        wv.py = p.iw_y;
        wv.cc10 = gate_coef(-kPi * (p.cond_lens.c10 + g.z_init[0]) * s.ph.lambda);
        wv.conf_slot = 0;
        wv.n_slices = S;
        wv.weight = (float)cs.weight;
        wv.pos = 0;
        WaveInfo* dwv = (WaveInfo*)c->buf("waves", sizeof(WaveInfo));
        CK(cudaMemcpyAsync(dwv, &wv, sizeof(WaveInfo), cudaMemcpyHostToDevice, st));
        float2* psi = (float2*)c->buf("psi", sizeof(float2) * N);
        float2* aux = (float2*)c->buf("aux", sizeof(float2) * N);
        PassArgs pa = pass_args(s, psi, dwv, nullptr, slot, cond);
        pa.l2_mode = l2_mode_for_waves(1, N);
        pa.tt = sT;
        pa.aux = aux;
        pa.filt_g2in = g2in;
        pa.filt_g2out = g2out;
        if (iw == MS_IW_CONVERGENT) {
            pa.tw = s.tw_y;
            run_col(c, p.ny, COL_PROBE_INV, pa, 1, p.nx, st);
        }
        for (int sl = 0; sl < nf; sl++) {
            pa.slice = sl;
            pa.flags = PF_VACUUM_BEYOND;
            pa.tw = s.tw_x;
            if (sl == 0 && iw == MS_IW_PLANE_TILTED) pa.flags |= PF_TILT_INCIDENT;
            run_row(c, p.nx, (sl == 0 && iw != MS_IW_CONVERGENT) ? ROW_T_FWD : ROW_INV_T_FWD, pa, 1, p.ny, st);
            pa.flags = PF_VACUUM_BEYOND | PF_PROP_ALWAYS | PF_FILTER_AUX;
            pa.tw = s.tw_y;
            run_col(c, p.ny, COL_STEP, pa, 1, p.nx, st);
            // filtered branch: IFFT2 of the annulus-masked spectrum, |.|^2 into frame sl (Filter_wave,
            // device_kernels.cuh:389-410, wave_filter, wave_function.cuh:163-174)
            PassArgs pb = pa;
            pb.psi = aux;
            pb.aux = aux;
            pb.flags = 0;
            run_col(c, p.ny, COL_INV, pb, 1, p.nx, st);
            pb.flags = PF_FILTER_AUX | PF_ACCUMULATE;
            pb.out_real = frames + (int64_t)sl * N;
            pb.tw = s.tw_x;
            run_row(c, p.nx, ROW_INV_ABS2, pb, 1, p.ny, st);
        }
        CK(cudaStreamSynchronize(st));
    }
    copy_out(c, out->thickness_frames, frames, (int64_t)nf * N, out->on_device);
    tm.stop();
    out->row = p.ny;
    out->col = p.nx;
    out->n_slices = nf;
    out->interval_x = p.lx / p.nx;
    out->interval_y = p.ly / p.ny;
}

// ---------------------------------------------------------------------------
// projected potentials of one configuration
// ---------------------------------------------------------------------------
void sim_potential(ms_ctx* c, const ms_params& p, const ms_atoms& a, int conf, float* V, int64_t cap, int on_dev,
                   int* n_slices)
{
    validate_params(p);
    validate_atoms(p, &a);
    MS_REQUIRE(conf >= 0, MS_ERR_INVALID_ARG, "conf must be >= 0");
    ctx_activate(c);
    cudaStream_t st = c->stream;
    Timer tm(c);
    Setup s = make_setup(c, p);
    AtomsDev A = upload_atoms(c, p, a);
    SpecGroup g = build_specimen(c, p, A, std::vector<int>{conf}, s.ph);
    const int S = g.ns[0];
    if (n_slices) *n_slices = S;
    if (V) {
        MS_REQUIRE((int64_t)S * s.N <= cap, MS_ERR_INVALID_ARG, "V_out holds fewer than n_slices*ny*nx floats");
        int64_t slot = (int64_t)S * s.N;
        float* sV = (float*)c->buf("sV", sizeof(float) * slot);
        run_potential(c, pot_args(p, s, A, g, sV, slot, 0, S, 0), 1, st);
        copy_out(c, V, sV, slot, on_dev);
    }
    tm.stop();
}

// ---------------------------------------------------------------------------
// STEM on caller potentials (wave_modulation_batch, wave_function.cuh:74-87)
// ---------------------------------------------------------------------------
void sim_stem_forward_potential(ms_ctx* c, const ms_params& p, const float* V, int S, int on_dev, double z_init,
                                const double* xy, int np, float* I)
{
    validate_params(p);
    MS_REQUIRE(V && xy && I && S >= 1 && np >= 1 && p.n_det >= 1, MS_ERR_INVALID_ARG, "bad arguments");
    ctx_activate(c);
    cudaStream_t st = c->stream;
    Timer tm(c);
    Setup s = make_setup(c, p);
    const int64_t N = s.N, slot = (int64_t)S * N;
    LensDev cond = lens_dev(lens_coef(p.cond_lens, s.ph.lambda, 0.0));
    const float* sV = V;
    if (!on_dev) {
        float* d = (float*)c->buf("sV", sizeof(float) * slot);
        CK(cudaMemcpyAsync(d, V, sizeof(float) * slot, cudaMemcpyHostToDevice, st));
        sV = d;
    }
    const int ndet = p.n_det;
    std::vector<float> thr(2 * ndet);
    for (int d = 0; d < ndet; d++) {
        thr[d] = g2_threshold(p.det_inner[d], s.ph.lambda);
        thr[ndet + d] = g2_threshold(p.det_outer[d], s.ph.lambda);
    }
    float* dthr = (float*)c->buf("det_thr", sizeof(float) * 2 * ndet);
    CK(cudaMemcpyAsync(dthr, thr.data(), sizeof(float) * 2 * ndet, cudaMemcpyHostToDevice, st));
    const int B = std::min(np, p.probe_batch > 0 ? p.probe_batch : 256);
    const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>(64, N / 4096));
    double* partial = (double*)c->buf("det_part", sizeof(double) * B * nblk * ndet);
    double* Iw = (double*)c->buf("det_I_all", sizeof(double) * np * ndet);
    const double cc10 = gate_coef(-kPi * (p.cond_lens.c10 + z_init) * s.ph.lambda);
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
        WaveInfo* dwv = (WaveInfo*)c->buf("waves", sizeof(WaveInfo) * B);
        CK(cudaMemcpyAsync(dwv, wv.data(), sizeof(WaveInfo) * nb, cudaMemcpyHostToDevice, st));
        float2* psi = (float2*)c->buf("psi", sizeof(float2) * N * B);
        PassArgs pa = pass_args(s, psi, dwv, sV, slot, cond);
        pa.tw = s.tw_y;
        run_col(c, p.ny, COL_PROBE_INV, pa, nb, p.nx, st);
        for (int sl = 0; sl < S; sl++) {
            pa.slice = sl;
            pa.tw = s.tw_x;
            run_row(c, p.nx, ROW_INV_T_FWD, pa, nb, p.ny, st);
            pa.tw = s.tw_y;
            run_col(c, p.ny, COL_STEP, pa, nb, p.nx, st);
        }
        launch_detect(psi, nb, p.nx, p.ny, s.gd.dgx_f, s.gd.dgy_f, dthr, dthr + ndet, ndet, partial, nblk, st);
        launch_det_finalize(partial, nb, nblk, ndet, dwv, Iw + (int64_t)start * ndet, nullptr, 0, 0, st);
        CK(cudaStreamSynchronize(st));
    }
    float* o = (float*)c->buf("stem_out", sizeof(float) * np * ndet);
    launch_d2f(Iw, (int64_t)np * ndet, o, st);
    CK(cudaMemcpyAsync(I, o, sizeof(float) * np * ndet, cudaMemcpyDeviceToHost, st));
    tm.stop();
}

// ---------------------------------------------------------------------------
// Adjoint of the STEM forward on caller potentials (or_stem_backward restated on the fused
// passes).  Per probe batch:
//   forward sweep, storing the wave every k slices (and, for the last segment, the
//   transmitted real-space waves x_s = t_s psi_s directly) -> detector sums -> residuals ->
//   seed lambda = sum_d 4 (I_d - T_d) Psi [annulus d] and its inverse column transform ->
//   per segment, last to first: recompute x_s from the segment's checkpoint, then sweep the
//   adjoint back through the segment (row adjoint with the dL/dV update, conj(P) column step)
//   -> at slice 0 the lens-phase gradient sums.
// ---------------------------------------------------------------------------
void sim_stem_backward(ms_ctx* c, const ms_params& p, const float* V, int S, int on_dev, double z_init,
                       const double* xy, int np, const float* target, double* loss, float* dV, double* dC10,
                       double* dC30)
{
    validate_params(p);
    MS_REQUIRE(V && xy && target && S >= 1 && np >= 1 && p.n_det >= 1, MS_ERR_INVALID_ARG, "bad arguments");
    MS_REQUIRE(p.ckpt_interval >= 1, MS_ERR_INVALID_ARG, "ckpt_interval must be >= 1");
    ctx_activate(c);
    cudaStream_t st = c->stream;
    Timer tm(c);
    Setup s = make_setup(c, p);
    const int64_t N = s.N, slot = (int64_t)S * N;
    LensDev cond = lens_dev(lens_coef(p.cond_lens, s.ph.lambda, 0.0));
    const float* sV = V;
    if (!on_dev) {
        float* d = (float*)c->buf("sV", sizeof(float) * slot);
        CK(cudaMemcpyAsync(d, V, sizeof(float) * slot, cudaMemcpyHostToDevice, st));
        sV = d;
    }
    const int ndet = p.n_det;
    std::vector<float> thr(2 * ndet);
    for (int d = 0; d < ndet; d++) {
        thr[d] = g2_threshold(p.det_inner[d], s.ph.lambda);
        thr[ndet + d] = g2_threshold(p.det_outer[d], s.ph.lambda);
    }
    float* dthr = (float*)c->buf("det_thr", sizeof(float) * 2 * ndet);
    CK(cudaMemcpyAsync(dthr, thr.data(), sizeof(float) * 2 * ndet, cudaMemcpyHostToDevice, st));
    float* dtgt = (float*)c->buf("adj_target", sizeof(float) * np * ndet);
    CK(cudaMemcpyAsync(dtgt, target, sizeof(float) * np * ndet, cudaMemcpyHostToDevice, st));

    const int k = p.ckpt_interval;
    const int nseg = (S + k - 1) / k;
    // probes per batch: adjoint wave, forward wave, one segment of transmitted waves and the
    // checkpoints must fit the memory budget
    const size_t per_wave = (size_t)N * 8 * (2 + 2 * (size_t)k + (size_t)(nseg - 1)) + (size_t)N * 4;
    int B = p.probe_batch > 0 ? p.probe_batch : 256;
    B = (int)std::max<size_t>(1, std::min<size_t>((size_t)B, free_budget(c) / per_wave));
    B = std::min(B, np);
    const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>(64, N / 4096));
    const int tiles = col_tiles(p.ny, p.nx);
    float2* adj = (float2*)c->buf("adj_psi", sizeof(float2) * N * B);
    // transmitted waves of two segments: the one being swept back and the one being recomputed
    float2* xseg = (float2*)c->buf("adj_xseg", sizeof(float2) * N * B * k * 2);
    float2* ckpt = nseg > 1 ? (float2*)c->buf("adj_ckpt", sizeof(float2) * N * B * (nseg - 1)) : nullptr;
    float* gV = on_dev ? dV : (float*)c->buf("adj_dV", sizeof(float) * slot);
    float* gVw = (float*)c->buf("adj_dVw", sizeof(float) * N * B);   // per-wave planes of one slice
    double* partial = (double*)c->buf("det_part", sizeof(double) * B * nblk * ndet);
    double* Iw = (double*)c->buf("det_I", sizeof(double) * B * ndet);
    double* resid = (double*)c->buf("adj_resid", sizeof(double) * B * ndet);
    double* sq = (double*)c->buf("adj_sq", sizeof(double) * np * ndet);
    double* chi_part = (double*)c->buf("adj_chi_part", sizeof(double) * B * tiles * 2);
    double* chi_acc = (double*)c->buf("adj_chi", sizeof(double) * 2);
    CK(cudaMemsetAsync(gV, 0, sizeof(float) * slot, st));
    CK(cudaMemsetAsync(chi_acc, 0, sizeof(double) * 2, st));
    const double cc10 = gate_coef(-kPi * (p.cond_lens.c10 + z_init) * s.ph.lambda);
    std::vector<WaveInfo> wv((size_t)B);
    for (int start = 0; start < np; start += B) {
        const int nb = std::min(B, np - start);
        const int64_t wstride = (int64_t)nb * N;   // one slice of the batch in xseg / ckpt
        for (int i = 0; i < nb; i++) {
            wv[i].px = xy[2 * (start + i)];
            wv[i].py = xy[2 * (start + i) + 1];
            wv[i].cc10 = cc10;
            wv[i].conf_slot = 0;
            wv[i].n_slices = S;
            wv[i].weight = 1.0f;
            wv[i].pos = start + i;
        }
        WaveInfo* dwv = (WaveInfo*)c->buf("waves", sizeof(WaveInfo) * B);
        CK(cudaMemcpyAsync(dwv, wv.data(), sizeof(WaveInfo) * nb, cudaMemcpyHostToDevice, st));
        PassArgs pa = pass_args(s, adj, dwv, sV, slot, cond);
        pa.det_thr = dthr;
        pa.ndet = ndet;
        pa.resid = resid;
        pa.chi_part = chi_part;
        // forward sweep with checkpoints
        pa.tw = s.tw_y;
        run_col(c, p.ny, COL_PROBE_INV, pa, nb, p.nx, st);
        const int last0 = (nseg - 1) * k;
        auto xbuf = [&](int seg) { return xseg + (int64_t)(seg % 2) * k * wstride; };
        for (int sl = 0; sl < S; sl++) {
            if (sl < last0 && sl % k == 0)
                CK(cudaMemcpyAsync(ckpt + (int64_t)(sl / k) * wstride, adj, sizeof(float2) * wstride,
                                   cudaMemcpyDeviceToDevice, st));
            pa.slice = sl;
            pa.flags = sl >= last0 ? PF_STORE_X : 0;
            pa.xs = xbuf(nseg - 1) + (int64_t)(sl - last0) * wstride;
            pa.tw = s.tw_x;
            run_row(c, p.nx, ROW_INV_T_FWD, pa, nb, p.ny, st);
            pa.flags = 0;
            pa.tw = s.tw_y;
            run_col(c, p.ny, COL_STEP, pa, nb, p.nx, st);
        }
        launch_detect(adj, nb, p.nx, p.ny, s.gd.dgx_f, s.gd.dgy_f, dthr, dthr + ndet, ndet, partial, nblk, st);
        launch_det_finalize(partial, nb, nblk, ndet, dwv, Iw, nullptr, 0, 0, st);
        launch_resid(Iw, dtgt + (int64_t)start * ndet, nb * ndet, resid, sq + (int64_t)start * ndet, st);
        pa.tw = s.tw_y;
        run_col(c, p.ny, COL_SEED, pa, nb, p.nx, st);
        // Segments are recomputed on a second stream one segment ahead of the backward sweep,
        // into the other half of the transmitted-wave buffer; events order each recompute after
        // the sweep that last read its half, and each sweep after its recompute.  With
        // per-launch profiling on, everything runs in order on the context stream.
        const bool two = !c->profile && nseg > 1;
        cudaStream_t rs = two ? pot_stream(c) : st;
        auto recompute = [&](int seg) {
            const int c0 = seg * k, c1 = std::min(S, c0 + k);
            PassArgs pr = pa;
            pr.psi = ckpt + (int64_t)seg * wstride;   // in place on the segment's checkpoint
            for (int sl = c0; sl < c1; sl++) {
                pr.slice = sl;
                pr.flags = PF_STORE_X;
                pr.xs = xbuf(seg) + (int64_t)(sl - c0) * wstride;
                pr.tw = s.tw_x;
                run_row(c, p.nx, ROW_INV_T_FWD, pr, nb, p.ny, rs);
                if (sl < c1 - 1) {
                    pr.flags = 0;
                    pr.tw = s.tw_y;
                    run_col(c, p.ny, COL_STEP, pr, nb, p.nx, rs);
                }
            }
        };
        auto ev_rec = [&](int seg) { return chunk_event(c, (size_t)(2 * seg)); };
        auto ev_back = [&](int seg) { return chunk_event(c, (size_t)(2 * seg + 1)); };
        if (two) {
            cudaEvent_t fwd_done = chunk_event(c, (size_t)(2 * nseg));
            CK(cudaEventRecord(fwd_done, st));
            CK(cudaStreamWaitEvent(rs, fwd_done, 0));
            recompute(nseg - 2);
            CK(cudaEventRecord(ev_rec(nseg - 2), rs));
        }
        for (int seg = nseg - 1; seg >= 0; seg--) {
            const int c0 = seg * k, c1 = std::min(S, c0 + k);
            if (seg != nseg - 1) {
                if (two) CK(cudaStreamWaitEvent(st, ev_rec(seg), 0));
                else recompute(seg);
            }
            for (int i = c1 - 1; i >= c0; i--) {
                pa.slice = i;
                pa.flags = 0;
                pa.xs = xbuf(seg) + (int64_t)(i - c0) * wstride;
                pa.dV = gVw;
                pa.tw = s.tw_x;
                run_row(c, p.nx, ROW_ADJ, pa, nb, p.ny, st);
                launch_sum_waves(gVw, nb, N, gV + (int64_t)i * N, st);
                pa.tw = s.tw_y;
                if (i > 0) {
                    pa.slice = i - 1;
                    pa.flags = PF_CONJ_PROP | PF_PROP_ALWAYS;
                    run_col(c, p.ny, COL_STEP, pa, nb, p.nx, st);
                } else {
                    run_col(c, p.ny, COL_GRAD_PROBE, pa, nb, p.nx, st);
                    launch_chi_finalize(chi_part, nb, tiles, chi_acc, st);
                }
            }
            if (two && seg - 2 >= 0) {
                // the segment two below reuses this segment's half of the buffer
                CK(cudaEventRecord(ev_back(seg), st));
                CK(cudaStreamWaitEvent(rs, ev_back(seg), 0));
                recompute(seg - 2);
                CK(cudaEventRecord(ev_rec(seg - 2), rs));
            }
        }
        CK(cudaStreamSynchronize(st));  // the host wave table is refilled by the next batch
    }
    if (!on_dev) CK(cudaMemcpyAsync(dV, gV, sizeof(float) * slot, cudaMemcpyDeviceToHost, st));
    std::vector<double> hsq((size_t)np * ndet);
    double hchi[2];
    CK(cudaMemcpyAsync(hsq.data(), sq, sizeof(double) * np * ndet, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hchi, chi_acc, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
    tm.stop();
    double L = 0.0;
    for (double v : hsq) L += v;
    if (loss) *loss = L;
    const double lam = s.ph.lambda;
    if (dC10) *dC10 = -kPi * lam * hchi[0];
    if (dC30) *dC30 = -kPi * lam * lam * lam / 2.0 * hchi[1];
}

// ---------------------------------------------------------------------------
// Uneven batch: n independent CBED simulations of mixed grid sizes, slice counts, beam
// energies and probes in one call.  Instances with the same grid share every pass launch:
// one row pass and one column pass per slice cover the waves of all instances of that
// grid that still have slices left, each wave reading its own instance's potential store
// and propagator table through its wave descriptor.  Grid groups run on their own streams
// and interleave slice by slice; an instance's pattern is accumulated and written as soon
// as its last slice is done, and an event records that completion.
// ---------------------------------------------------------------------------
namespace {
cudaStream_t side_stream(ms_ctx* c, size_t i)
{
    while (c->side.size() <= i) {
        cudaStream_t s = nullptr;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        c->side.push_back(s);
    }
    return c->side[i];
}
}  // namespace

void sim_many(ms_ctx* c, int n, const ms_params* ps, const ms_atoms* as, ms_output* outs, double* lat)
{
    for (int i = 0; i < n; i++) {
        validate_params(ps[i]);
        validate_atoms(ps[i], &as[i]);
        MS_REQUIRE(ps[i].simulation_type == MS_SIM_CBED, MS_ERR_UNSUPPORTED,
                   "uneven batches run CBED simulations (simulation_type = MS_SIM_CBED)");
        MS_REQUIRE(ps[i].data_record == MS_RECORD_INTENSITY, MS_ERR_UNSUPPORTED,
                   "uneven batches record intensities");
        MS_REQUIRE(outs[i].image_intensity != nullptr, MS_ERR_INVALID_ARG, "image_intensity is NULL");
    }
    ctx_activate(c);
    cudaStream_t st = c->stream;
    const bool prof = c->profile;
    c->profile = false;   // per-launch events live on the context stream; groups run on side streams
    struct Restore {
        ms_ctx* c;
        bool v;
        ~Restore() { c->profile = v; }
    } restore{c, prof};
    Timer tm(c);
    std::vector<cudaEvent_t> done((size_t)n, nullptr);
    struct EvFree {
        std::vector<cudaEvent_t>* v;
        ~EvFree()
        {
            for (auto e : *v)
                if (e) cudaEventDestroy(e);
        }
    } evfree{&done};
    for (int i = 0; i < n; i++) CK(cudaEventCreate(&done[i]));
    // instances that run in the persistent engine report the device clock at which their waves
    // were done, against this stamp of the call's start
    unsigned long long* t0_ns = (unsigned long long*)c->buf("many_t0", sizeof(unsigned long long));
    launch_stamp(t0_ns, st);
    std::vector<unsigned long long> inst_done_ns((size_t)n, 0ull);

    // per instance: physics, propagator table, potential store
    struct Inst {
        int nconf = 0;
        std::vector<WaveInfo> waves;
        int S_max = 0;
        GridDev gd;
        LensDev cond;
        float* sV = nullptr;
        float2* prop = nullptr;
        float* out = nullptr;
    };
    std::vector<Inst> in((size_t)n);
    // memory plan: instances whose stores do not fit together run in successive rounds
    std::vector<size_t> need((size_t)n);
    for (int i = 0; i < n; i++) {
        const int64_t N = (int64_t)ps[i].nx * ps[i].ny;
        const ConfSet cs = conf_set(ps[i]);
        need[i] = (size_t)N * (4 * (size_t)estimate_slices(ps[i], as[i]) * cs.confs.size() + 8 + 4 + 8 * cs.confs.size());
    }
    int r0 = 0;
    while (r0 < n) {
        size_t budget = free_budget(c), used = 0;
        int r1 = r0;
        while (r1 < n && (r1 == r0 || used + need[r1] <= budget)) used += need[r1++];
        // one arena, cached in the context like every other buffer, holds the round's per-instance
        // potential stores, propagator tables and patterns (bump allocation, 256-byte aligned);
        // an instance whose store outgrows its estimate gets a buffer of its own
        unsigned char* arena = (unsigned char*)c->buf("many_arena", used);
        size_t arena_off = 0;
        auto take = [&](const std::string& name, size_t bytes) -> void* {
            bytes = (bytes + 255) / 256 * 256;
            if (arena_off + bytes <= used) {
                void* p = arena + arena_off;
                arena_off += bytes;
                return p;
            }
            return c->buf(name, bytes);
        };
        // ---- phase 1 (context stream): specimens, potentials, propagators
        for (int i = r0; i < r1; i++) {
            const ms_params& p = ps[i];
            Inst& I = in[i];
            const Physics ph = physics_of(p.E0, p.theta);
            const GridConst gc = grid_of(p, ph);
            const int64_t N = (int64_t)p.nx * p.ny;
            Setup s0;
            s0.ph = ph;
            s0.gc = gc;
            s0.N = N;
            s0.gd.nx = p.nx;
            s0.gd.ny = p.ny;
            s0.gd.dgx_f = gc.dgx_f;
            s0.gd.dgy_f = gc.dgy_f;
            s0.gd.dgx = gc.dgx;
            s0.gd.dgy = gc.dgy;
            s0.gd.gl2_f = (float)gc.gl2;
            s0.gd.alpha_f = (float)gc.alpha;
            s0.gd.bwl = p.bwl ? 1 : 0;
            s0.gd.inv_n = 1.0f / (float)N;
            s0.gd.lx = p.lx;
            s0.gd.ly = p.ly;
            s0.gd.g0x = gc.g0x;
            s0.gd.g0y = gc.g0y;
            I.gd = s0.gd;
            I.cond = lens_dev(lens_coef(p.cond_lens, ph.lambda, 0.0));
            AtomsDev A = upload_atoms(c, p, as[i]);
            ConfSet cs = conf_set(p);
            SpecGroup g = build_specimen(c, p, A, cs.confs, ph);
            I.nconf = g.nconf;
            const int64_t slot = (int64_t)g.S_cap * N;
            I.sV = (float*)take("many_sV_" + std::to_string(i), sizeof(float) * slot * g.nconf);
            run_potential(c, pot_args(p, s0, A, g, I.sV, slot, 0, g.S_cap, 0), g.nconf, st);
            I.prop = (float2*)take("many_prop_" + std::to_string(i), sizeof(float2) * kPropSets * N);
            launch_prop_table(p.nx, p.ny, gc.dgx, gc.dgy, gc.g0x, gc.g0y, gc.prop_w, gc.alpha, gc.gl2, p.bwl ? 1 : 0,
                              I.prop, st);
            I.out = (float*)take("many_out_" + std::to_string(i), sizeof(float) * N);
            I.waves.assign((size_t)g.nconf, WaveInfo());
            I.S_max = 0;
            for (int k = 0; k < g.nconf; k++) {
                WaveInfo& w = I.waves[k];
                w.px = p.iw_x;
                w.py = p.iw_y;
                w.cc10 = gate_coef(-kPi * (p.cond_lens.c10 + g.z_init[k]) * ph.lambda);
                w.conf_slot = 0;
                w.n_slices = g.ns[k];
                w.weight = (float)cs.weight;
                w.pos = i;
                w.sV = I.sV + (int64_t)k * slot;
                w.prop = I.prop;
                I.S_max = std::max(I.S_max, g.ns[k]);
            }
        }
        // ---- phase 2: grid groups on side streams, interleaved slice by slice
        struct Group {
            int nx, ny;
            std::vector<int> inst;      // instances, longest first
            std::vector<int> off;       // first wave of each instance
            std::vector<WaveInfo> waves;
            WaveInfo* dwv = nullptr;
            float2* psi = nullptr;
            double* acc = nullptr;
            cudaStream_t s = nullptr;
            int S_max = 0;
            size_t done_off = 0;        // first entry of the group's waves in the completion clocks
            bool engine = false;        // the group runs in the persistent slice engine
        };
        std::vector<Group> groups;
        for (int i = r0; i < r1; i++) {
            size_t gi = 0;
            while (gi < groups.size() && !(groups[gi].nx == ps[i].nx && groups[gi].ny == ps[i].ny)) gi++;
            if (gi == groups.size()) {
                groups.emplace_back();
                groups.back().nx = ps[i].nx;
                groups.back().ny = ps[i].ny;
            }
            groups[gi].inst.push_back(i);
        }
        // tables every group reads, made before the groups fork off the context stream
        if (!c->exptab) make_setup(c, ps[r0]);
        const float2* ex = (const float2*)c->exptab;
        size_t nwaves_all = 0;
        for (Group& G : groups) {
            twiddles(c, G.nx);
            twiddles(c, G.ny);
            G.done_off = nwaves_all;
            for (int i : G.inst) nwaves_all += in[i].waves.size();
            G.engine = engine_fits(c, G.nx, G.ny, 0, true);
        }
        unsigned long long* dns = (unsigned long long*)c->buf("many_done_ns", sizeof(unsigned long long) * nwaves_all);
        CK(cudaMemsetAsync(dns, 0, sizeof(unsigned long long) * nwaves_all, st));
        cudaEvent_t fork = chunk_event(c, 0);
        CK(cudaEventRecord(fork, st));
        for (size_t gi = 0; gi < groups.size(); gi++) {
            Group& G = groups[gi];
            std::stable_sort(G.inst.begin(), G.inst.end(), [&](int a, int b) { return in[a].S_max > in[b].S_max; });
            for (int i : G.inst) {
                G.off.push_back((int)G.waves.size());
                G.waves.insert(G.waves.end(), in[i].waves.begin(), in[i].waves.end());
            }
            G.S_max = in[G.inst.front()].S_max;
            const int64_t N = (int64_t)G.nx * G.ny;
            const std::string tag = std::to_string(G.nx) + "x" + std::to_string(G.ny);
            G.dwv = (WaveInfo*)c->buf("many_waves_" + tag, sizeof(WaveInfo) * G.waves.size());
            G.psi = (float2*)c->buf("many_psi_" + tag, sizeof(float2) * N * G.waves.size());
            G.acc = (double*)c->buf("many_acc_" + tag, sizeof(double) * N);
            G.s = side_stream(c, gi);
            CK(cudaStreamWaitEvent(G.s, fork, 0));
            CK(cudaMemcpyAsync(G.dwv, G.waves.data(), sizeof(WaveInfo) * G.waves.size(), cudaMemcpyHostToDevice, G.s));
        }
        // probes, per instance (each has its own lens, grid and wavelength)
        for (Group& G : groups) {
            for (size_t k = 0; k < G.inst.size(); k++) {
                const Inst& I = in[G.inst[k]];
                PassArgs pa;
                std::memset(&pa, 0, sizeof(pa));
                pa.psi = G.psi + (int64_t)G.off[k] * G.nx * G.ny;
                pa.waves = G.dwv + G.off[k];
                pa.grid = I.gd;
                pa.lens = I.cond;
                pa.tw = twiddles(c, G.ny);
                launch_col(G.ny, COL_PROBE_INV, pa, I.nconf, G.nx, G.s);
            }
        }
        // groups in the engine: every slice of every instance in one launch, then the patterns
        for (size_t gi = 0; gi < groups.size(); gi++) {
            Group& G = groups[gi];
            if (!G.engine) continue;
            std::vector<int> ns;
            for (const WaveInfo& w : G.waves) ns.push_back(w.n_slices);
            const EngineArgs e = engine_plan(c, ns, 0, G.nx, G.s, dns + G.done_off, "_many" + std::to_string(gi));
            PassArgs pa;
            std::memset(&pa, 0, sizeof(pa));
            pa.psi = G.psi;
            pa.waves = G.dwv;
            pa.exptab = ex;
            pa.grid = in[G.inst.front()].gd;
            pa.err = c->d_err;
            pa.tw = twiddles(c, G.nx);
            engine_launch(pa, e, G.nx, (int)G.waves.size(), G.s);
            const int64_t N = (int64_t)G.nx * G.ny;
            for (size_t kk = 0; kk < G.inst.size(); kk++) {
                const int i = G.inst[kk];
                launch_acc_abs2(G.psi + (int64_t)G.off[kk] * N, in[i].nconf, G.dwv + G.off[kk], N, G.acc, 1, G.s);
                launch_emit(G.acc, G.nx, G.ny, 1, in[i].out, G.s);
                CK(cudaEventRecord(done[i], G.s));
            }
        }
        int S_all = 0;
        for (Group& G : groups) S_all = std::max(S_all, G.S_max);
        std::vector<size_t> next((size_t)groups.size(), 0);   // next instance (in S order) to finish, per group
        for (int sl = 0; sl < S_all; sl++) {
            for (size_t gi = 0; gi < groups.size(); gi++) {
                Group& G = groups[gi];
                if (G.engine || sl >= G.S_max) continue;
                // active waves: instances with slices left form a prefix
                size_t ki = 0;
                while (ki < G.inst.size() && in[G.inst[ki]].S_max > sl) ki++;
                const int nact = ki < G.inst.size() ? G.off[ki] : (int)G.waves.size();
                PassArgs pa;
                std::memset(&pa, 0, sizeof(pa));
                pa.psi = G.psi;
                pa.waves = G.dwv;
                pa.slice = sl;
                pa.exptab = ex;
                pa.grid = in[G.inst.front()].gd;
                pa.err = c->d_err;
                pa.tw = twiddles(c, G.nx);
                launch_row(G.nx, ROW_INV_T_FWD, pa, nact, G.ny, G.s);
                pa.tw = twiddles(c, G.ny);
                launch_col(G.ny, COL_STEP, pa, nact, G.nx, G.s);
                // instances whose last slice this was: pattern out, completion event
                while (next[gi] < G.inst.size() && in[G.inst[G.inst.size() - 1 - next[gi]]].S_max == sl + 1) {
                    const size_t kk = G.inst.size() - 1 - next[gi];
                    const int i = G.inst[kk];
                    const int64_t N = (int64_t)G.nx * G.ny;
                    launch_acc_abs2(G.psi + (int64_t)G.off[kk] * N, in[i].nconf, G.dwv + G.off[kk], N, G.acc, 1, G.s);
                    launch_emit(G.acc, G.nx, G.ny, 1, in[i].out, G.s);
                    CK(cudaEventRecord(done[i], G.s));
                    next[gi]++;
                }
            }
        }
        for (size_t gi = 0; gi < groups.size(); gi++) {
            cudaEvent_t j = chunk_event(c, 1 + gi);
            CK(cudaEventRecord(j, groups[gi].s));
            CK(cudaStreamWaitEvent(st, j, 0));
        }
        for (int i = r0; i < r1; i++) copy_out(c, outs[i].image_intensity, in[i].out, (int64_t)ps[i].nx * ps[i].ny,
                                               outs[i].on_device);
        CK(cudaStreamSynchronize(st));
        if (lat) {
            std::vector<unsigned long long> h(nwaves_all);
            CK(cudaMemcpy(h.data(), dns, sizeof(unsigned long long) * nwaves_all, cudaMemcpyDeviceToHost));
            for (const Group& G : groups) {
                if (!G.engine) continue;
                for (size_t kk = 0; kk < G.inst.size(); kk++)
                    for (int k = 0; k < in[G.inst[kk]].nconf; k++)
                        inst_done_ns[G.inst[kk]] = std::max(inst_done_ns[G.inst[kk]], h[G.done_off + G.off[kk] + k]);
            }
        }
        // buffers of instances that outgrew the arena are this call's alone
        for (int i = r0; i < r1; i++) {
            for (const char* nm : {"many_sV_", "many_prop_", "many_out_"}) {
                auto it = c->bufs.find(nm + std::to_string(i));
                if (it != c->bufs.end()) {
                    cudaFree(it->second.p);
                    c->bufs.erase(it);
                    c->forget_free_mem();
                }
            }
        }
        r0 = r1;
    }
    tm.stop();
    for (int i = 0; i < n; i++) {
        outs[i].row = ps[i].ny;
        outs[i].col = ps[i].nx;
        outs[i].n_slices = in[i].S_max;
        outs[i].interval_x = ps[i].lx / ps[i].nx;
        outs[i].interval_y = ps[i].ly / ps[i].ny;
        outs[i].total_intensity = 0.0;
        if (lat) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, c->ev0, done[i]));
            lat[i] = ms;
            if (inst_done_ns[i]) {
                // engine instances: the device clock when the instance's last wave was done
                unsigned long long t0 = 0;
                CK(cudaMemcpy(&t0, t0_ns, sizeof(t0), cudaMemcpyDeviceToHost));
                if (inst_done_ns[i] > t0) lat[i] = (double)(inst_done_ns[i] - t0) * 1e-6;
            }
        }
    }
}

}  // namespace msb
