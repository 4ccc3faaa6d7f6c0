// Host side of the engine: beam physics, lens coefficients, radial spline
// tables, the host specimen surface (displacement, slicing, crystal slabs)
// and parameter validation.  Compiled with -ffp-contract=off so that the
// float arithmetic of the slicing planes matches the device bit for bit.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>

#include "detmath.cuh"
#include "vr.cuh"
#include "engine.hpp"

namespace msb {

namespace {
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kH = 6.62607015e-34;     // Planck constant, J s (CODATA 2018)
constexpr double kMe = 9.1093837015e-31;  // electron rest mass, kg
constexpr double kQe = 1.602176634e-19;   // elementary charge, C
constexpr double kC = 299792458.0;        // speed of light, m/s
}  // namespace

Physics physics_of(double E0_kV, double theta)
{
    Physics ph;
    double E = E0_kV * 1e3;
    ph.gamma = 1.0 + kQe * E / (kMe * kC * kC);
    double lam = kH / std::sqrt(2.0 * kMe * kQe * E * (1.0 + kQe * E / (2.0 * kMe * kC * kC)));
    ph.lambda = lam * 1e10;
    ph.sigma = 2.0 * kPi * ph.gamma * kMe * kQe * lam / (kH * kH) * 1e-10;
    ph.vr_factor = ph.sigma / std::cos(theta);
    return ph;
}

GridConst grid_of(const ms_params& p, const Physics& ph)
{
    GridConst g;
    g.nx = p.nx;
    g.ny = p.ny;
    g.lx = p.lx;
    g.ly = p.ly;
    g.dx = p.lx / p.nx;
    g.dy = p.ly / p.ny;
    g.dgx = 1.0 / p.lx;
    g.dgy = 1.0 / p.ly;
    g.dx_f = (float)g.dx;
    g.dy_f = (float)g.dy;
    g.dgx_f = 1.0f / (float)p.lx;
    g.dgy_f = 1.0f / (float)p.ly;
    double gmax = std::fmin((p.nx / 2) * g.dgx, (p.ny / 2) * g.dgy);
    double gl = 2.0 * gmax / 3.0;
    g.gl2 = gl * gl;
    g.alpha = std::log(1.0 / 1e-2 - 1.0) / ((gl + 0.25) * (gl + 0.25) - g.gl2);
    g.bwl = p.bwl;
    g.g0x = std::sin(p.theta) * std::cos(p.phi) / ph.lambda;
    g.g0y = std::sin(p.theta) * std::sin(p.phi) / ph.lambda;
    g.prop_w = -kPi * ph.lambda * p.dz;
    return g;
}

double gate_coef(double v) { return std::fabs(v) > 1e-5 ? v : 0.0; }

float fine_radius(const ms_params& p) { return (float)(p.pot_rmax > 0 ? p.pot_rmax : 3.0); }

float g2_threshold(double angle, double lambda)
{
    float g = (float)(std::sin(angle) / lambda);
    return g * g;
}

LensCoef lens_coef(const ms_lens& L, double lambda, double c10_shift)
{
    LensCoef o;
    double l = lambda, l2 = l * l, l3 = l2 * l, l4 = l3 * l, l5 = l4 * l;
    o.m = L.m;
    o.cc10 = gate_coef(-kPi * (L.c10 + c10_shift) * l);
    o.cc12 = gate_coef(-kPi * L.c12 * l);
    o.cc21 = gate_coef(-2.0 * kPi * L.c21 * l2 / 3.0);
    o.cc23 = gate_coef(-2.0 * kPi * L.c23 * l2 / 3.0);
    o.cc30 = gate_coef(-kPi * L.c30 * l3 / 2.0);
    o.cc32 = gate_coef(-kPi * L.c32 * l3 / 2.0);
    o.cc34 = gate_coef(-kPi * L.c34 * l3 / 2.0);
    o.cc41 = gate_coef(-2.0 * kPi * L.c41 * l4 / 5.0);
    o.cc43 = gate_coef(-2.0 * kPi * L.c43 * l4 / 5.0);
    o.cc45 = gate_coef(-2.0 * kPi * L.c45 * l4 / 5.0);
    o.cc50 = gate_coef(-kPi * L.c50 * l5 / 3.0);
    o.cc52 = gate_coef(-kPi * L.c52 * l5 / 3.0);
    o.cc54 = gate_coef(-kPi * L.c54 * l5 / 3.0);
    o.cc56 = gate_coef(-kPi * L.c56 * l5 / 3.0);
    o.p12 = L.phi12; o.p21 = L.phi21; o.p23 = L.phi23; o.p32 = L.phi32; o.p34 = L.phi34;
    o.p41 = L.phi41; o.p43 = L.phi43; o.p45 = L.phi45; o.p52 = L.phi52; o.p54 = L.phi54;
    o.p56 = L.phi56;
    o.g2min = L.inner_aper_ang > 0 ? g2_threshold(L.inner_aper_ang, lambda) : 0.0f;
    o.g2max = L.outer_aper_ang > 0 ? g2_threshold(L.outer_aper_ang, lambda) : FLT_MAX;
    o.phi_req = (o.m != 0) || o.cc12 != 0 || o.cc21 != 0 || o.cc23 != 0 || o.cc32 != 0 || o.cc34 != 0 ||
                o.cc41 != 0 || o.cc43 != 0 || o.cc45 != 0 || o.cc52 != 0 || o.cc54 != 0 || o.cc56 != 0;
    return o;
}

// ---------------------------------------------------------------------------
// Element potentials.  V(r) and V'(r) follow the reference's functional forms
// (Vr_dVrir_*_dev, basic_functions_dev.cuh:102-186).  The built-in table is
// Moliere's approximation to the Thomas-Fermi screening function,
// phi(x) = 0.35 e^-0.3x + 0.55 e^-1.2x + 0.10 e^-6x, x = r / a_TF with
// a_TF = 0.88534 a0 Z^(-1/3); V(r) = (e^2 / 4 pi eps0) (Z/r) phi(r/a_TF) is then
// three Yukawa terms of the Kirkland form.
// ---------------------------------------------------------------------------
namespace {
struct Coef {
    int form;
    double cl[MS_MAX_COEF], cnl[MS_MAX_COEF];
};

Coef moliere(int Z)
{
    const double a0 = 0.529177210903;
    const double ke = 14.399645478425668;
    const double tf = 0.88534138;
    double aTF = tf * a0 * std::pow((double)Z, -1.0 / 3.0);
    const double al[3] = {0.35, 0.55, 0.10}, be[3] = {0.3, 1.2, 6.0};
    Coef c;
    std::memset(&c, 0, sizeof(c));
    c.form = MS_POT_KIRKLAND_0_12;
    for (int i = 0; i < 3; i++) {
        c.cl[i] = ke * Z * al[i];
        c.cnl[i] = be[i] / aTF;
    }
    for (int i = 3; i < 6; i++) {
        c.cl[i] = 0.0;
        c.cnl[i] = 1.0;
    }
    return c;
}

Coef coef_for(const ms_params& p, int Z)
{
    for (int i = 0; i < p.n_element_coefs; i++) {
        const ms_element_coef& e = p.element_coefs[i];
        if (e.Z == Z) {
            Coef c;
            c.form = e.form;
            for (int k = 0; k < MS_MAX_COEF; k++) {
                c.cl[k] = e.cl[k];
                c.cnl[k] = e.cnl[k];
            }
            return c;
        }
    }
    return moliere(Z);
}

void Vr(const Coef& c, double r, double* V, double* dV)
{
    ElemCoefDev e;
    e.form = c.form;
    e.pad = 0;
    for (int k = 0; k < MS_MAX_COEF; k++) {
        e.cl[k] = c.cl[k];
        e.cnl[k] = c.cnl[k];
    }
    vr_eval(e, r, V, dV);
}

// Projection along z with the substitution z = R sinh(u):
//   V_z(R) = 2 int_0^inf V(R cosh u) R cosh u du,  dV_z/dR^2 = int_0^inf V'(R cosh u) du,
// evaluated with the trapezoid rule in u, which converges exponentially here.
void project(const Coef& c, double R, double* Vz, double* dVz)
{
    const double h = 0.02;
    double V, dV;
    Vr(c, R, &V, &dV);
    double sv = 0.5 * V * R, sd = 0.5 * dV;
    for (int k = 1; k < 4000; k++) {
        double r = R * std::cosh(k * h);
        Vr(c, r, &V, &dV);
        double tv = V * r, td = dV;
        sv += tv;
        sd += td;
        if (std::fabs(tv) < 1e-18 * std::fabs(sv) && std::fabs(td) < 1e-18 * std::fabs(sd) && k > 10) break;
    }
    *Vz = 2.0 * h * sv;
    *dVz = h * sd;
}
}  // namespace

ElemCoefDev elem_coef_dev(const ms_params& p, int Z)
{
    Coef c = coef_for(p, Z);
    ElemCoefDev e;
    e.form = c.form;
    e.pad = 0;
    for (int k = 0; k < MS_MAX_COEF; k++) {
        e.cl[k] = c.cl[k];
        e.cnl[k] = c.cnl[k];
    }
    return e;
}

void gauss_legendre_half(int n, double* x, double* w)
{
    const int m = (n + 1) / 2;
    for (int i = 0; i < m; i++) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5)), pp = 1.0;
        for (int it = 0; it < 100; it++) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; j++) {
                const double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            const double z1 = z;
            z = z1 - p1 / pp;
            if (std::fabs(z - z1) <= 1e-15) break;
        }
        x[i] = -0.5 * z;
        x[n - 1 - i] = 0.5 * z;
        w[i] = w[n - 1 - i] = 1.0 / ((1.0 - z * z) * pp * pp);
    }
}

void projected_potential_fp64(const ms_params& p, int Z, double R, double* Vz, double* dVz_dR2)
{
    project(coef_for(p, Z), R, Vz, dVz_dR2);
}

void build_elem_table(const ms_params& p, int Z, ElemTable* t)
{
    Coef c = coef_for(p, Z);
    double rmn = p.pot_rmin > 0 ? p.pot_rmin : 0.01;
    double rmx = p.pot_rmax > 0 ? p.pot_rmax : 3.0;
    double R2tap = (0.85 * rmx) * (0.85 * rmx);
    double tap_cf = kPi / (2.0 * (rmx * rmx - R2tap));
    double R2[MS_NR], c0[MS_NR], c1[MS_NR];
    for (int i = 0; i < MS_NR; i++) {
        double R = rmn * std::pow(rmx / rmn, (double)i / (double)(MS_NR - 1));
        if (i == MS_NR - 1) R = rmx;
        double Vz, dVz;
        project(c, R, &Vz, &dVz);
        R2[i] = R * R;
        if (R2tap < R2[i]) {  // apply_tapering_dev (basic_functions_dev.cuh:90-101), in R^2
            double tap = std::cos(tap_cf * (R2[i] - R2tap));
            double dtap = std::sin(tap_cf * (R2[i] - R2tap));
            dVz = dVz * tap - tap_cf * Vz * dtap;
            Vz = Vz * tap;
        }
        c0[i] = Vz;
        c1[i] = dVz;
    }
    std::memset(t, 0, sizeof(*t));
    for (int i = 0; i < MS_NR; i++) {
        t->R2[i] = (float)R2[i];
        t->c[i].c0 = (float)c0[i];
        t->c[i].c1 = (float)c1[i];
    }
    for (int i = 0; i < MS_NR - 1; i++) {  // get_cubic_poly_coef (basic_functions_dev.cuh:76-89)
        double idR = 1.0 / (R2[i + 1] - R2[i]);
        double m = (c0[i + 1] - c0[i]) * idR;
        double n = c1[i] + c1[i + 1];
        t->c[i].c2 = (float)((3.0 * m - n - c1[i]) * idR);
        t->c[i].c3 = (float)((n - 2.0 * m) * idR * idR);
    }
    t->rmax = (float)rmx;
    t->rmax2 = (float)(rmx * rmx);
    t->l0 = (float)std::log2(R2[0]);
    t->inv_dl = (float)((MS_NR - 1) / std::log2(R2[MS_NR - 1] / R2[0]));
    t->l0s = -t->l0 * t->inv_dl;
    t->Z = Z;
}

// ---------------------------------------------------------------------------
// Specimen
// ---------------------------------------------------------------------------
int border_of(const ms_params& p)
{
    if (p.slice_border >= 0) return p.slice_border;
    return p.simulation_type == MS_SIM_HRTEM ? MS_BORDER_MAX : MS_BORDER_MIN;  // specimen.cuh:24-35
}

int iw_of(const ms_params& p)
{
    if (p.iw_type > 0) return p.iw_type;
    return (p.simulation_type == MS_SIM_HRTEM || p.simulation_type == MS_SIM_ED) ? MS_IW_PLANE : MS_IW_CONVERGENT;
}

void host_displace(const ms_params& p, const ms_atoms& a, int conf, float* x, float* y, float* z)
{
    int64_t n = a.n;
    auto work = [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; i++) {
            float xi = a.x[i], yi = a.y[i], zi = a.z[i];
            det_displace(p.pn_seed, conf, i, a.sigma[i], p.pn_dim_x, p.pn_dim_y, p.pn_dim_z, &xi, &yi, &zi);
            x[i] = xi;
            y[i] = yi;
            z[i] = zi;
        }
    };
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < 20000 || conf <= 0) {
        work(0, n);
        return;
    }
    std::vector<std::thread> th;
    int64_t chunk = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        int64_t i0 = t * chunk, i1 = std::min<int64_t>(n, i0 + chunk);
        if (i0 < i1) th.emplace_back(work, i0, i1);
    }
    for (auto& t : th) t.join();
}

int host_slices(const ms_params& p, const float* z, int64_t n, std::vector<float>* bounds, int* atom_slice)
{
    if (n <= 0) {
        if (bounds) bounds->clear();
        return 0;
    }
    float vmin = z[0], vmax = z[0];
    for (int64_t i = 1; i < n; i++) {
        vmin = std::min(vmin, z[i]);
        vmax = std::max(vmax, z[i]);
    }
    float dz = (float)p.dz;
    const float zmax_atoms = vmax;
    if (p.enable_fine_slicing) {
        // planes over the z range grown by the integration radius (slice_generator.hpp:56-76)
        vmin = MSF_SUB(vmin, fine_radius(p));
        vmax = MSF_ADD(vmax, fine_radius(p));
    }
    int nv = det_nplanes(vmin, vmax, dz);
    int border = border_of(p);
    std::vector<float> b(nv);
    for (int i = 0; i < nv; i++) b[i] = det_plane(i, nv, vmin, vmax, dz, border);
    if (atom_slice)
        for (int64_t k = 0; k < n; k++) atom_slice[k] = det_slice_of(z[k], b.data(), nv, zmax_atoms);
    if (bounds) *bounds = b;
    return nv - 1;
}

ConfSet conf_set(const ms_params& p)
{
    ConfSet c;
    if (p.phonon_model == MS_PHONON_FROZEN && p.pn_nconf > 0) {
        for (int i = 1; i <= p.pn_nconf; i++) c.confs.push_back(i);
        c.weight = 1.0 / (double)p.pn_nconf;
    } else {
        c.confs.push_back(0);
        c.weight = 1.0;
    }
    return c;
}

static bool pow2_in_range(int n) { return n >= 128 && n <= 2048 && (n & (n - 1)) == 0; }

void validate_params(const ms_params& p)
{
    MS_REQUIRE(p.simulation_type >= MS_SIM_HRTEM && p.simulation_type <= MS_SIM_STEM, MS_ERR_INVALID_ARG,
               "simulation_type must be HRTEM, ED, CBED or STEM");
    MS_REQUIRE(pow2_in_range(p.nx) && pow2_in_range(p.ny), MS_ERR_UNSUPPORTED,
               "nx and ny must be powers of two between 128 and 2048");
    MS_REQUIRE(p.lx > 0 && p.ly > 0 && std::isfinite(p.lx) && std::isfinite(p.ly), MS_ERR_INVALID_ARG,
               "lx and ly must be positive");
    MS_REQUIRE(p.dz > 0 && std::isfinite(p.dz), MS_ERR_INVALID_ARG, "dz must be positive");
    MS_REQUIRE(p.E0 > 0 && p.E0 < 10000, MS_ERR_INVALID_ARG, "E0 must be in (0, 10000) kV");
    MS_REQUIRE(std::fabs(p.theta) < 1.0, MS_ERR_INVALID_ARG, "beam tilt theta out of range");
    MS_REQUIRE(p.iw_type <= 0 || (p.iw_type >= MS_IW_PLANE && p.iw_type <= MS_IW_PLANE_TILTED), MS_ERR_INVALID_ARG,
               "iw_type must be plane, convergent or tilted plane (or <= 0 for the mode's default)");
    MS_REQUIRE(p.exec_mode >= MS_EXEC_BATCHED && p.exec_mode <= MS_EXEC_GENERAL, MS_ERR_INVALID_ARG,
               "exec_mode must be batched, plain or general");
    MS_REQUIRE(p.enable_fine_slicing == 0 || p.enable_fine_slicing == 1, MS_ERR_INVALID_ARG,
               "enable_fine_slicing must be 0 or 1");
    MS_REQUIRE(p.illumination_model == 0 || (p.illumination_model >= MS_ILLUM_COHERENT && p.illumination_model <= MS_ILLUM_TCC),
               MS_ERR_INVALID_ARG, "illumination_model must be coherent, partial or TCC");
    MS_REQUIRE(p.temporal_spatial_incoh >= 0 && p.temporal_spatial_incoh <= MS_TSI_COHERENT, MS_ERR_INVALID_ARG,
               "temporal_spatial_incoh must be 1..4 (0 selects 1)");
    MS_REQUIRE(p.obj_lens.dsf_sigma >= 0 && p.obj_lens.ssf_beta >= 0 && p.obj_lens.ssf_beta < 0.5, MS_ERR_INVALID_ARG,
               "defocus spread and source divergence must be non-negative");
    MS_REQUIRE(p.illumination_model != MS_ILLUM_TCC ||
                   (p.obj_lens.dsf_npoints >= 1 && p.obj_lens.dsf_npoints <= 64 && p.obj_lens.ssf_npoints >= 1 &&
                    p.obj_lens.ssf_npoints <= 16),
               MS_ERR_INVALID_ARG, "TCC needs 1..64 defocus and 1..16 source quadrature points per axis");
    MS_REQUIRE(p.gpu_num <= 1, MS_ERR_UNSUPPORTED, "one GPU per context: gpu_num must be 1");
    MS_REQUIRE(p.phonon_model == MS_PHONON_STILL || p.phonon_model == MS_PHONON_FROZEN, MS_ERR_INVALID_ARG,
               "phonon_model must be still or frozen");
    MS_REQUIRE(p.phonon_model != MS_PHONON_FROZEN || (p.pn_nconf >= 1 && p.pn_nconf <= 100000), MS_ERR_INVALID_ARG,
               "frozen phonons need pn_nconf >= 1");
    double rmn = p.pot_rmin > 0 ? p.pot_rmin : 0.01, rmx = p.pot_rmax > 0 ? p.pot_rmax : 3.0;
    MS_REQUIRE(rmn < rmx, MS_ERR_INVALID_ARG, "pot_rmin must be below pot_rmax");
    MS_REQUIRE(!p.pot_wrap || (2 * rmx < p.lx && 2 * rmx < p.ly), MS_ERR_INVALID_ARG,
               "periodic potentials need pot_rmax below half the box");
    MS_REQUIRE(p.n_det >= 0 && p.n_det <= MS_MAX_DET, MS_ERR_INVALID_ARG, "n_det out of range");
    for (int d = 0; d < p.n_det; d++)
        MS_REQUIRE(p.det_inner[d] >= 0 && p.det_outer[d] >= p.det_inner[d], MS_ERR_INVALID_ARG,
                   "detector angles must satisfy 0 <= inner <= outer");
    MS_REQUIRE(p.n_element_coefs >= 0 && (p.n_element_coefs == 0 || p.element_coefs != nullptr), MS_ERR_INVALID_ARG,
               "element_coefs is NULL");
    for (int i = 0; i < p.n_element_coefs; i++)
        MS_REQUIRE(p.element_coefs[i].form >= MS_POT_DOYLE_0_4 && p.element_coefs[i].form <= MS_POT_MOLIERE,
                   MS_ERR_INVALID_ARG, "unknown potential form in element_coefs");
    if (p.simulation_type == MS_SIM_STEM) {
        MS_REQUIRE(p.scan_nx >= 1 && p.scan_ny >= 1, MS_ERR_INVALID_ARG, "STEM needs a scan of at least 1x1");
        MS_REQUIRE((int64_t)p.scan_nx * p.scan_ny <= (1LL << 26), MS_ERR_INVALID_ARG, "scan too large");
        MS_REQUIRE(p.n_det >= 1, MS_ERR_INVALID_ARG, "STEM needs at least one detector");
    }
    MS_REQUIRE(p.probe_batch >= 0 && p.probe_batch <= 4096, MS_ERR_INVALID_ARG, "probe_batch out of range");
}

void validate_atoms(const ms_params& p, const ms_atoms* a)
{
    (void)p;
    MS_REQUIRE(a != nullptr, MS_ERR_INVALID_ARG, "atoms is NULL");
    MS_REQUIRE(a->n >= 1, MS_ERR_INVALID_ARG, "the specimen has no atoms");
    MS_REQUIRE(a->n <= (1LL << 31) - 1, MS_ERR_INVALID_ARG, "too many atoms");
    MS_REQUIRE(a->Z && a->x && a->y && a->z && a->sigma && a->occ, MS_ERR_INVALID_ARG, "atom arrays must not be NULL");
    for (int64_t i = 0; i < a->n; i++) {
        MS_REQUIRE(a->Z[i] >= 1 && a->Z[i] <= 103, MS_ERR_INVALID_ARG, "atomic number out of range");
        MS_REQUIRE(std::isfinite(a->x[i]) && std::isfinite(a->y[i]) && std::isfinite(a->z[i]) &&
                       std::isfinite(a->sigma[i]) && std::isfinite(a->occ[i]),
                   MS_ERR_INVALID_ARG, "atom coordinates must be finite");
    }
}

}  // namespace msb
