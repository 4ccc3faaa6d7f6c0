/*
 * ms_oracle.c -- TEST INFRASTRUCTURE ONLY (see ms_oracle.h).
 *
 * An FP64 restatement of cudaEM's multislice operators, written from the
 * reference's source.  Each function cites the reference lines it follows.
 * The arithmetic that must agree bit-for-bit with the CUDA engine (the
 * phonon random numbers, the slicing planes, the aperture and detector
 * masks) is done here in the same IEEE operations the engine uses, with
 * floating-point contraction disabled at compile time.  Everything else is
 * computed in double precision.
 *
 * Compile with -ffp-contract=off (oracle/Makefile does).
 */
#include "ms_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_PI 3.14159265358979323846264338327950288
#define MS_NQZ 64 /* z quadrature points of fine slicing (c_nqz) */
typedef double complex cplx;

static int g_threads = 0;
void or_set_threads(int n) { g_threads = n; }
int or_get_threads(void)
{
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* physics: relativistic wavelength, interaction constant.  The reference's   */
/* get_Vr_factor lives in a missing header (transmission_function.cuh:60-61); */
/* these are the textbook expressions with CODATA 2018 constants.             */
/* ------------------------------------------------------------------------ */
static const double C_H = 6.62607015e-34;     /* J s */
static const double C_ME = 9.1093837015e-31;  /* kg */
static const double C_QE = 1.602176634e-19;   /* C */
static const double C_C = 299792458.0;        /* m/s */

void or_physics(double E0_kV, double* lambda, double* sigma, double* gamma)
{
    double E = E0_kV * 1e3;
    double g = 1.0 + C_QE * E / (C_ME * C_C * C_C);
    double lam = C_H / sqrt(2.0 * C_ME * C_QE * E * (1.0 + C_QE * E / (2.0 * C_ME * C_C * C_C)));
    if (lambda) *lambda = lam * 1e10;
    if (sigma) *sigma = 2.0 * OR_PI * g * C_ME * C_QE * lam / (C_H * C_H) * 1e-10;
    if (gamma) *gamma = g;
}

/* ------------------------------------------------------------------------ */
/* frozen-phonon random numbers.  The reference's vibrate_atom_positions and  */
/* random_lib.hpp are missing (single_simulator.cuh:65-74); this is the       */
/* engine's own counter-based generator: SplitMix64 mixing of                 */
/* (seed, conf, atom, stream), Marsaglia's polar method, and a logarithm      */
/* built only from IEEE-exact operations so that host and device agree bit    */
/* for bit.                                                                   */
/* ------------------------------------------------------------------------ */
static uint64_t or_mix(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double or_det_log(double s)
{
    /* s = m 2^e with m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(t), t = (m-1)/(m+1),
       summed as the Maclaurin series of atanh to t^27 (|t| <= 0.1716). */
    int e;
    double m = frexp(s, &e);
    if (m < 0.70710678118654752440) {
        m = m * 2.0;
        e = e - 1;
    }
    double t = (m - 1.0) / (m + 1.0);
    double t2 = t * t;
    double q = 1.0 / 27.0;
    q = q * t2 + 1.0 / 25.0;
    q = q * t2 + 1.0 / 23.0;
    q = q * t2 + 1.0 / 21.0;
    q = q * t2 + 1.0 / 19.0;
    q = q * t2 + 1.0 / 17.0;
    q = q * t2 + 1.0 / 15.0;
    q = q * t2 + 1.0 / 13.0;
    q = q * t2 + 1.0 / 11.0;
    q = q * t2 + 1.0 / 9.0;
    q = q * t2 + 1.0 / 7.0;
    q = q * t2 + 1.0 / 5.0;
    q = q * t2 + 1.0 / 3.0;
    q = q * t2 + 1.0;
    double lm = 2.0 * t * q;
    return (double)e * 0.69314718055994530942 + lm;
}

void or_gauss_pair(uint64_t seed, int conf, int64_t atom, int stream, double* g0, double* g1)
{
    uint64_t key = or_mix(or_mix(or_mix(seed) ^ (uint64_t)(int64_t)conf) ^
                          (((uint64_t)atom << 2) | (uint64_t)stream));
    for (int it = 0; it < 64; it++) {
        uint64_t r0 = or_mix(key + (uint64_t)(2 * it));
        uint64_t r1 = or_mix(key + (uint64_t)(2 * it + 1));
        double u = ((double)(r0 >> 11) + 0.5) * 0x1.0p-53;
        double v = ((double)(r1 >> 11) + 0.5) * 0x1.0p-53;
        u = 2.0 * u - 1.0;
        v = 2.0 * v - 1.0;
        double s = u * u + v * v;
        if (s < 1.0 && s > 0.0) {
            double f = sqrt(-2.0 * or_det_log(s) / s);
            *g0 = u * f;
            *g1 = v * f;
            return;
        }
    }
    *g0 = 0.0;
    *g1 = 0.0;
}

/* Displacement of configuration conf >= 1; conf 0 is the static specimen. */
void or_displace(const ms_params* p, const ms_atoms* a, int conf, float* x, float* y, float* z)
{
    for (int64_t i = 0; i < a->n; i++) {
        float xi = a->x[i], yi = a->y[i], zi = a->z[i];
        if (conf > 0) {
            double g0, g1, g2, g3;
            or_gauss_pair(p->pn_seed, conf, i, 0, &g0, &g1);
            or_gauss_pair(p->pn_seed, conf, i, 1, &g2, &g3);
            double s = (double)a->sigma[i];
            if (p->pn_dim_x) xi = xi + (float)(s * g0);
            if (p->pn_dim_y) yi = yi + (float)(s * g1);
            if (p->pn_dim_z) zi = zi + (float)(s * g2);
        }
        x[i] = xi;
        y[i] = yi;
        z[i] = zi;
    }
}

/* ------------------------------------------------------------------------ */
/* slicing: Slice_Generator::gene_bounds / get_slicing / fd_by_z             */
/* (slice_generator.hpp:56-168), in float like the reference's T = float.     */
/* z_eps is epsilon_rel<float>() of the missing host header, taken as 1e-4    */
/* (the relative epsilon of the reference's float compare, misc_dev.cuh:17-23)*/
/* ------------------------------------------------------------------------ */
static double or_rmin(const ms_params* p) { return p->pot_rmin > 0 ? p->pot_rmin : 0.01; }
static double or_rmax(const ms_params* p) { return p->pot_rmax > 0 ? p->pot_rmax : 3.0; }

static int or_border(const ms_params* p)
{
    if (p->slice_border >= 0) return p->slice_border;
    return p->simulation_type == MS_SIM_HRTEM ? MS_BORDER_MAX : MS_BORDER_MIN; /* specimen.cuh:24-35 */
}

int or_slices(const ms_params* p, const float* z, int64_t n, float* bounds, int cap, int* atom_slice)
{
    const float z_eps = 1e-4f;
    const float dz = (float)p->dz;
    if (n <= 0) return 0;
    float vmin = z[0], vmax = z[0];
    for (int64_t i = 1; i < n; i++) {
        if (z[i] < vmin) vmin = z[i];
        if (z[i] > vmax) vmax = z[i];
    }
    float zmax_atoms = vmax;
    if (p->enable_fine_slicing) {
        /* fine slicing: planes over the atoms' z range grown by the integration radius
           (get_slice_boundary with atoms.z_int_min/max, slice_generator.hpp:56-76) */
        const float R_int = (float)or_rmax(p);
        vmin = vmin - R_int;
        vmax = vmax + R_int;
    }
    float s_v = vmax - vmin;
    int nv = (int)floorf((s_v + z_eps) / dz) + 2;
    float* b = (float*)malloc(sizeof(float) * (size_t)nv);
    int border = or_border(p);
    if (border == MS_BORDER_MIN) {
        float zb = vmin - 2 * z_eps;
        for (int i = 0; i < nv; i++) b[i] = zb + (float)i * dz;
    } else if (border == MS_BORDER_MAX) {
        float zt = vmax + 2 * z_eps;
        for (int i = 0; i < nv; i++) b[nv - 1 - i] = zt - (float)i * dz;
    } else {
        float zb = 0.5f * (vmin + vmax - (float)(nv - 1) * dz);
        for (int i = 0; i < nv; i++) b[i] = zb + (float)i * dz;
    }
    int ns = nv - 1;
    if (bounds)
        for (int i = 0; i < nv && i < cap; i++) bounds[i] = b[i];
    if (atom_slice) {
        /* slice i holds bound[i] <= z < bound[i+1]; the top atom equal to the last plane
           belongs to the last slice (fd_by_z, slice_generator.hpp:109-129). */
        for (int64_t k = 0; k < n; k++) {
            float zk = z[k];
            int s = -1;
            if (zk >= b[0] && zk < b[nv - 1]) {
                int lo = 0, hi = nv - 1; /* largest i with b[i] <= zk */
                while (hi - lo > 1) {
                    int mid = (lo + hi) / 2;
                    if (b[mid] <= zk) lo = mid; else hi = mid;
                }
                s = lo;
            } else if (zk == b[nv - 1] && zk == zmax_atoms) {
                s = ns - 1;
            }
            atom_slice[k] = s;
        }
    }
    free(b);
    return ns;
}

/* ------------------------------------------------------------------------ */
/* element potentials.  V(r) and V'(r) in the reference's functional forms   */
/* (basic_functions_dev.cuh:102-186); the default table is Moliere's          */
/* Thomas-Fermi screening approximation written in the Kirkland form (three   */
/* Yukawa terms): V(r) = (e^2/4 pi eps0) Z/r sum a_i exp(-b_i r/a_TF),         */
/* a_i = (0.35, 0.55, 0.10), b_i = (0.3, 1.2, 6.0), a_TF = 0.88534 a0 Z^-1/3.   */
/* ------------------------------------------------------------------------ */
typedef struct {
    int form;
    int n;
    double cl[MS_MAX_COEF], cnl[MS_MAX_COEF];
} or_coef;

static void or_moliere(int Z, or_coef* c)
{
    const double a0 = 0.529177210903;                    /* Bohr radius, A */
    const double ke = 14.399645478425668;                /* e^2/(4 pi eps0), eV A */
    const double tf = 0.88534138;                        /* (9 pi^2 / 128)^(1/3) */
    double aTF = tf * a0 * pow((double)Z, -1.0 / 3.0);
    const double al[3] = {0.35, 0.55, 0.10}, be[3] = {0.3, 1.2, 6.0};
    memset(c, 0, sizeof(*c));
    c->form = MS_POT_KIRKLAND_0_12;
    c->n = 6;
    for (int i = 0; i < 3; i++) {
        c->cl[i] = ke * Z * al[i];
        c->cnl[i] = be[i] / aTF;
    }
    for (int i = 3; i < 6; i++) {
        c->cl[i] = 0.0;
        c->cnl[i] = 1.0;
    }
}

static void or_coef_for(const ms_params* p, int Z, or_coef* c)
{
    for (int i = 0; i < p->n_element_coefs; i++) {
        const ms_element_coef* e = &p->element_coefs[i];
        if (e->Z == Z) {
            memset(c, 0, sizeof(*c));
            c->form = e->form;
            c->n = (e->form == MS_POT_DOYLE_0_4) ? 4 : (e->form == MS_POT_PENG_0_4 || e->form == MS_POT_PENG_0_12 ||
                                                      e->form == MS_POT_LOBATO_0_12) ? 5 : 6;
            for (int k = 0; k < MS_MAX_COEF; k++) {
                c->cl[k] = e->cl[k];
                c->cnl[k] = e->cnl[k];
            }
            return;
        }
    }
    or_moliere(Z, c);
}

/* V(r) and V'(r) (note: the reference returns dVrir = V'(r)/r) */
static void or_Vr(const or_coef* c, double r, double* V, double* dV)
{
    double v = 0.0, d = 0.0;
    switch (c->form) {
    case MS_POT_DOYLE_0_4:
    case MS_POT_PENG_0_4:
    case MS_POT_PENG_0_12: {
        int n = (c->form == MS_POT_DOYLE_0_4) ? 4 : 5;
        for (int i = 0; i < n; i++) {
            double e = c->cl[i] * exp(-c->cnl[i] * r * r);
            v += e;
            d += -2.0 * c->cnl[i] * r * e;
        }
    } break;
    case MS_POT_KIRKLAND_0_12:
    case MS_POT_MOLIERE: {
        for (int i = 0; i < 3; i++) {
            double e = c->cl[i] * exp(-c->cnl[i] * r) / r;
            v += e;
            d += -e * (c->cnl[i] + 1.0 / r);
        }
        for (int i = 3; i < 6; i++) {
            double e = c->cl[i] * exp(-c->cnl[i] * r * r);
            v += e;
            d += -2.0 * c->cnl[i] * r * e;
        }
    } break;
    case MS_POT_WEICKENMEIER_0_12: {
        double s = 0.0, sd = 0.0;
        for (int i = 0; i < 6; i++) {
            s += c->cl[i] * erfc(c->cnl[i] * r);
            sd += c->cl[i] * c->cnl[i] * exp(-c->cnl[i] * c->cnl[i] * r * r);
        }
        v = s / r;
        d = -(2.0 * sd / 1.772453850905516027298) / r - s / (r * r);
    } break;
    case MS_POT_LOBATO_0_12: {
        for (int i = 0; i < 5; i++) {
            double br = c->cnl[i] * r;
            double e = c->cl[i] * exp(-br);
            v += e * (2.0 / br + 1.0);
            d += -e * (2.0 / (br * r) + 2.0 / r + c->cnl[i]);
        }
    } break;
    default:
        break;
    }
    *V = v;
    *dV = d;
}

/* V_z(R) = 2 int_0^inf V(R cosh u) R cosh u du ; dV_z/dR^2 = int_0^inf V'(R cosh u) du.
   Trapezoid rule in u (exponentially convergent for these integrands). */
static void or_project(const or_coef* c, double R, double* Vz, double* dVz)
{
    const double h = 0.02;
    double sv = 0.0, sd = 0.0;
    double V, dV;
    or_Vr(c, R, &V, &dV);
    sv = 0.5 * V * R;
    sd = 0.5 * dV;
    for (int k = 1; k < 4000; k++) {
        double ch = cosh(k * h);
        double r = R * ch;
        or_Vr(c, r, &V, &dV);
        double tv = V * r, td = dV;
        sv += tv;
        sd += td;
        if (fabs(tv) < 1e-18 * fabs(sv) && fabs(td) < 1e-18 * fabs(sd) && k > 10) break;
    }
    *Vz = 2.0 * h * sv;
    *dVz = h * sd;
}

int or_projected(const ms_params* p, int Z, double R, double* Vz, double* dVz_dR2)
{
    or_coef c;
    or_coef_for(p, Z, &c);
    or_project(&c, R, Vz, dVz_dR2);
    return 0;
}


/* Radial spline table (the VR_Cubic coefficients of Element_Coeffs,
   device_containers.cuh:243-249): log-spaced nodes in R, values and
   derivatives in R^2, a cosine taper in R^2 from R_tap = 0.85 R_max
   (apply_tapering_dev, basic_functions_dev.cuh:90-101) and Hermite cubic
   coefficients (get_cubic_poly_coef, basic_functions_dev.cuh:76-89). */
/* R of spline node i: log-spaced from R_min to R_max */
static double or_node_R(const ms_params* p, int i)
{
    double rmn = or_rmin(p), rmx = or_rmax(p);
    double R = rmn * pow(rmx / rmn, (double)i / (double)(MS_NR - 1));
    return i == MS_NR - 1 ? rmx : R;
}

/* Gauss-Legendre nodes and weights on [-1/2, 1/2] with weights summing to 1: the z
   quadrature qz of fine slicing (gen_sa_coeff_kernel, device_kernels.cuh:48-86; the
   reference's table comes from the missing multislice_params.hpp).  Newton iteration on the
   Legendre recurrence from the usual cosine starting points. */
void or_gauss_legendre_half(int n, double* x, double* w)
{
    int m = (n + 1) / 2;
    for (int i = 0; i < m; i++) {
        double z = cos(OR_PI * (i + 0.75) / (n + 0.5)), z1, pp = 1.0;
        for (int it = 0; it < 100; it++) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; j++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) <= 1e-15) break;
        }
        x[i] = -0.5 * z;
        x[n - 1 - i] = 0.5 * z;
        w[i] = w[n - 1 - i] = 1.0 / ((1.0 - z * z) * pp * pp);
    }
}

/* Slice-integrated potential of one atom at node R (fine slicing, gen_sa_coeff_kernel,
   device_kernels.cuh:48-86): V = sum_k w_k dz V(r_k), dV/dR^2 = 1/2 sum_k w_k dz V'(r_k)/r_k,
   r_k = sqrt(z_k^2 + R^2), z_k = dz x_k + a, a = slice middle - atom z. */
static void or_fine_node(const or_coef* c, double R, double a, double dzs, double* V, double* dV)
{
    double xq[MS_NQZ], wq[MS_NQZ];
    or_gauss_legendre_half(MS_NQZ, xq, wq);
    double v = 0.0, d = 0.0;
    for (int k = 0; k < MS_NQZ; k++) {
        double z = dzs * xq[k] + a;
        double r = sqrt(z * z + R * R);
        double Vr, dVr;
        or_Vr(c, r, &Vr, &dVr);
        v += wq[k] * dzs * Vr;
        d += wq[k] * dzs * dVr / r;
    }
    *V = v;
    *dV = 0.5 * d;
}

/* taper (apply_tapering_dev, basic_functions_dev.cuh:90-101) and Hermite coefficients
   (get_cubic_poly_coef, basic_functions_dev.cuh:76-89) of node values c0 and slopes c1 */
static void or_spline_finish(const ms_params* p, const double* R2, double* c0, double* c1, double* c2, double* c3)
{
    double rmx = or_rmax(p);
    double R2tap = (0.85 * rmx) * (0.85 * rmx);
    double tap_cf = OR_PI / (2.0 * (rmx * rmx - R2tap));
    for (int i = 0; i < MS_NR; i++)
        if (R2tap < R2[i]) {
            double tap = cos(tap_cf * (R2[i] - R2tap));
            double dtap = sin(tap_cf * (R2[i] - R2tap));
            c1[i] = c1[i] * tap - tap_cf * c0[i] * dtap;
            c0[i] = c0[i] * tap;
        }
    for (int i = 0; i < MS_NR - 1; i++) {
        double idR = 1.0 / (R2[i + 1] - R2[i]);
        double m = (c0[i + 1] - c0[i]) * idR;
        double n = c1[i] + c1[i + 1];
        c2[i] = (3.0 * m - n - c1[i]) * idR;
        c3[i] = (n - 2.0 * m) * idR * idR;
    }
    c2[MS_NR - 1] = 0.0;
    c3[MS_NR - 1] = 0.0;
}

/* spline of one (atom, slice) pair under fine slicing */
static void or_fine_spline(const ms_params* p, int Z, double a, double dzs, double* R2, double* c0, double* c1,
                           double* c2, double* c3)
{
    or_coef c;
    or_coef_for(p, Z, &c);
    for (int i = 0; i < MS_NR; i++) {
        double R = or_node_R(p, i);
        R2[i] = R * R;
        or_fine_node(&c, R, a, dzs, &c0[i], &c1[i]);
    }
    or_spline_finish(p, R2, c0, c1, c2, c3);
}

int or_fine_spline_table(const ms_params* p, int Z, double a, double dzs, double* R2, double* c0, double* c1,
                         double* c2, double* c3)
{
    or_fine_spline(p, Z, a, dzs, R2, c0, c1, c2, c3);
    return 0;
}

int or_spline(const ms_params* p, int Z, double* R2, double* c0, double* c1, double* c2, double* c3, double* rmax)
{
    or_coef c;
    or_coef_for(p, Z, &c);
    double rmn = or_rmin(p), rmx = or_rmax(p);
    double R2tap = (0.85 * rmx) * (0.85 * rmx);
    double tap_cf = OR_PI / (2.0 * (rmx * rmx - R2tap));
    (void)rmn;
    for (int i = 0; i < MS_NR; i++) {
        double R = or_node_R(p, i);
        double Vz, dVz;
        or_project(&c, R, &Vz, &dVz);
        R2[i] = R * R;
        if (R2tap < R2[i]) {
            double tap = cos(tap_cf * (R2[i] - R2tap));
            double dtap = sin(tap_cf * (R2[i] - R2tap));
            dVz = dVz * tap - tap_cf * Vz * dtap;
            Vz = Vz * tap;
        }
        c0[i] = Vz;
        c1[i] = dVz;
    }
    for (int i = 0; i < MS_NR - 1; i++) {
        double idR = 1.0 / (R2[i + 1] - R2[i]);
        double V = c0[i], Vn = c0[i + 1], dV = c1[i], dVn = c1[i + 1];
        double m = (Vn - V) * idR;
        double n = dV + dVn;
        c2[i] = (3.0 * m - n - dV) * idR;
        c3[i] = (n - 2.0 * m) * idR * idR;
    }
    c2[MS_NR - 1] = 0.0;
    c3[MS_NR - 1] = 0.0;
    if (rmax) *rmax = rmx;
    return 0;
}

/* unrolledBinarySearch_c_nR + get_value_Cubic_Spline (basic_functions_dev.cuh:47-75) */
static double or_spline_eval(const double* R2, const double* c0, const double* c1, const double* c2,
                             const double* c3, double x)
{
    int i0 = 0, ie = MS_NR - 1;
    for (int k = 0; k < 7; k++) {
        int im = (i0 + ie) >> 1;
        if (x < R2[im]) ie = im; else i0 = im;
    }
    double d = x - R2[i0];
    return ((c3[i0] * d + c2[i0]) * d + c1[i0]) * d + c0[i0];
}

/* ------------------------------------------------------------------------ */
/* common simulation context                                                 */
/* ------------------------------------------------------------------------ */
typedef struct {
    double lambda, sigma, gamma, vr_factor;
    int nx, ny;
    long N;
    double lx, ly, dx, dy;
    float dgx_f, dgy_f;
    double dgx, dgy;
    double gl2, alpha;
    double g0x, g0y;
    double prop_w;
} or_sim;

static void or_sim_init(const ms_params* p, or_sim* s)
{
    or_physics(p->E0, &s->lambda, &s->sigma, &s->gamma);
    s->vr_factor = s->sigma / cos(p->theta); /* get_Vr_factor(lambda, gamma, theta) */
    s->nx = p->nx;
    s->ny = p->ny;
    s->N = (long)p->nx * p->ny;
    s->lx = p->lx;
    s->ly = p->ly;
    s->dx = p->lx / p->nx;
    s->dy = p->ly / p->ny;
    s->dgx = 1.0 / p->lx;
    s->dgy = 1.0 / p->ly;
    s->dgx_f = 1.0f / (float)p->lx;
    s->dgy_f = 1.0f / (float)p->ly;
    /* Grid_2d_Dev::set_input_data (grid_dev.cuh:307-325) */
    double gmax = fmin((p->nx / 2) * s->dgx, (p->ny / 2) * s->dgy);
    double gl = 2.0 * gmax / 3.0;
    s->gl2 = gl * gl;
    s->alpha = log(1.0 / 1e-2 - 1.0) / ((gl + 0.25) * (gl + 0.25) - s->gl2);
    /* gx_0 / gy_0 (multislice_params_dev.cuh:201-208) */
    s->g0x = sin(p->theta) * cos(p->phi) / s->lambda;
    s->g0y = sin(p->theta) * sin(p->phi) / s->lambda;
    s->prop_w = -OR_PI * s->lambda * p->dz; /* propagator_factor * z (propagation_function.cuh:31, :49-57) */
}

static inline int or_fshift(int i, int n) { return i < n / 2 ? i : i - n; }

/* float frequency squared, exactly as the engine computes it for masks */
static inline float or_g2f(const or_sim* s, int ix, int iy)
{
    float gx = (float)or_fshift(ix, s->nx) * s->dgx_f;
    float gy = (float)or_fshift(iy, s->ny) * s->dgy_f;
    return gx * gx + gy * gy;
}

static float or_g2_thr(double ang, double lambda)
{
    float g = (float)(sin(ang) / lambda);
    return g * g;
}

/* Lens_Dev coefficients (lens_dev.cuh:40-57); a term is dropped when its
   coefficient is zero within the reference's float tolerance (nonZero_dev,
   misc_dev.cuh:17-23, 1e-5 absolute). */
typedef struct {
    int m;
    double cc10, cc12, cc21, cc23, cc30, cc32, cc34, cc41, cc43, cc45, cc50, cc52, cc54, cc56;
    double p12, p21, p23, p32, p34, p41, p43, p45, p52, p54, p56;
    float g2min, g2max;
    int phi_req;
} or_lens;

static double or_gate(double v) { return fabs(v) > 1e-5 ? v : 0.0; }

static void or_lens_init(const ms_lens* L, double lambda, double c10_shift, or_lens* o)
{
    double l = lambda, l2 = l * l, l3 = l2 * l, l4 = l3 * l, l5 = l4 * l;
    o->m = L->m;
    o->cc10 = or_gate(-OR_PI * (L->c10 + c10_shift) * l);
    o->cc12 = or_gate(-OR_PI * L->c12 * l);
    o->cc21 = or_gate(-2.0 * OR_PI * L->c21 * l2 / 3.0);
    o->cc23 = or_gate(-2.0 * OR_PI * L->c23 * l2 / 3.0);
    o->cc30 = or_gate(-OR_PI * L->c30 * l3 / 2.0);
    o->cc32 = or_gate(-OR_PI * L->c32 * l3 / 2.0);
    o->cc34 = or_gate(-OR_PI * L->c34 * l3 / 2.0);
    o->cc41 = or_gate(-2.0 * OR_PI * L->c41 * l4 / 5.0);
    o->cc43 = or_gate(-2.0 * OR_PI * L->c43 * l4 / 5.0);
    o->cc45 = or_gate(-2.0 * OR_PI * L->c45 * l4 / 5.0);
    o->cc50 = or_gate(-OR_PI * L->c50 * l5 / 3.0);
    o->cc52 = or_gate(-OR_PI * L->c52 * l5 / 3.0);
    o->cc54 = or_gate(-OR_PI * L->c54 * l5 / 3.0);
    o->cc56 = or_gate(-OR_PI * L->c56 * l5 / 3.0);
    o->p12 = L->phi12; o->p21 = L->phi21; o->p23 = L->phi23; o->p32 = L->phi32; o->p34 = L->phi34;
    o->p41 = L->phi41; o->p43 = L->phi43; o->p45 = L->phi45; o->p52 = L->phi52; o->p54 = L->phi54;
    o->p56 = L->phi56;
    o->g2min = L->inner_aper_ang > 0 ? or_g2_thr(L->inner_aper_ang, lambda) : 0.0f;
    o->g2max = L->outer_aper_ang > 0 ? or_g2_thr(L->outer_aper_ang, lambda) : FLT_MAX;
    o->phi_req = (o->m != 0) || o->cc12 != 0 || o->cc21 != 0 || o->cc23 != 0 || o->cc32 != 0 ||
                 o->cc34 != 0 || o->cc41 != 0 || o->cc43 != 0 || o->cc45 != 0 || o->cc52 != 0 ||
                 o->cc54 != 0 || o->cc56 != 0;
}

/* coherent_phase_shift (basic_functions_dev.cuh:215-234) */
static double or_chi(const or_lens* o, double gx, double gy)
{
    double g2 = gx * gx + gy * gy, g4 = g2 * g2, g6 = g4 * g2;
    double chi = o->cc10 * g2 + o->cc30 * g4 + o->cc50 * g6;
    if (o->phi_req) {
        double g = sqrt(g2), g3 = g2 * g, g5 = g4 * g;
        double ph = atan2(gy, gx);
        if (fabs(ph) > 1e-5) chi += o->m * ph;
        chi += o->cc12 * g2 * sin(2 * (ph - o->p12));
        chi += o->cc21 * g3 * sin(ph - o->p21) + o->cc23 * g3 * sin(3 * (ph - o->p23));
        chi += o->cc32 * g4 * sin(2 * (ph - o->p32)) + o->cc34 * g4 * sin(4 * (ph - o->p34));
        chi += o->cc41 * g5 * sin(ph - o->p41) + o->cc43 * g5 * sin(3 * (ph - o->p43)) +
               o->cc45 * g5 * sin(5 * (ph - o->p45));
        chi += o->cc52 * g6 * sin(2 * (ph - o->p52)) + o->cc54 * g6 * sin(4 * (ph - o->p54)) +
               o->cc56 * g6 * sin(6 * (ph - o->p56));
    }
    return chi;
}

/* ------------------------------------------------------------------------ */
/* FFT: iterative radix-2, unnormalised, sign -1 forward (CUFFT_FORWARD)      */
/* ------------------------------------------------------------------------ */
static void or_fft1(cplx* a, int n, int sign, const cplx* tw /* n/2 entries exp(-2 pi i k/n) */)
{
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            cplx t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int step = n / len;
        for (int i = 0; i < n; i += len) {
            for (int k = 0; k < len / 2; k++) {
                cplx w = tw[k * step];
                if (sign > 0) w = conj(w);
                cplx u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
        }
    }
}

static cplx* or_twiddles(int n)
{
    cplx* t = (cplx*)malloc(sizeof(cplx) * (size_t)(n / 2 > 0 ? n / 2 : 1));
    for (int k = 0; k < n / 2; k++) {
        double a = -2.0 * OR_PI * (double)k / (double)n;
        t[k] = cos(a) + I * sin(a);
    }
    return t;
}

static void or_fft2c(cplx* d, int nx, int ny, int sign)
{
    cplx* twx = or_twiddles(nx);
    cplx* twy = or_twiddles(ny);
    int inpar = 0;
#ifdef _OPENMP
    inpar = omp_in_parallel();
#endif
    int nth = inpar ? 1 : or_get_threads();
#pragma omp parallel for num_threads(nth) schedule(static)
    for (int r = 0; r < ny; r++) or_fft1(d + (size_t)r * nx, nx, sign, twx);
#pragma omp parallel num_threads(nth)
    {
        cplx* col = (cplx*)malloc(sizeof(cplx) * (size_t)ny);
#pragma omp for schedule(static)
        for (int c = 0; c < nx; c++) {
            for (int r = 0; r < ny; r++) col[r] = d[(size_t)r * nx + c];
            or_fft1(col, ny, sign, twy);
            for (int r = 0; r < ny; r++) d[(size_t)r * nx + c] = col[r];
        }
        free(col);
    }
    free(twx);
    free(twy);
}

void or_fft2(double* data, int nx, int ny, int sign) { or_fft2c((cplx*)data, nx, ny, sign); }

/* ------------------------------------------------------------------------ */
/* specimen of one configuration: displaced, sliced, grouped by slice        */
/* ------------------------------------------------------------------------ */
typedef struct {
    int ns;
    float* bounds;
    int64_t n;
    float *x, *y, *z;
    int* slice;
    int64_t* order;    /* atom indices sorted by slice */
    int64_t* start;    /* ns+1 offsets into order */
    double z_init;     /* slice_middle_z(0) */
} or_spec;

static int or_spec_build(const ms_params* p, const ms_atoms* a, int conf, or_spec* sp)
{
    memset(sp, 0, sizeof(*sp));
    sp->n = a->n;
    sp->x = (float*)malloc(sizeof(float) * (size_t)(a->n + 1));
    sp->y = (float*)malloc(sizeof(float) * (size_t)(a->n + 1));
    sp->z = (float*)malloc(sizeof(float) * (size_t)(a->n + 1));
    sp->slice = (int*)malloc(sizeof(int) * (size_t)(a->n + 1));
    or_displace(p, a, conf, sp->x, sp->y, sp->z);
    int ns = or_slices(p, sp->z, a->n, NULL, 0, NULL);
    sp->ns = ns;
    sp->bounds = (float*)malloc(sizeof(float) * (size_t)(ns + 1));
    or_slices(p, sp->z, a->n, sp->bounds, ns + 1, sp->slice);
    sp->start = (int64_t*)calloc((size_t)ns + 2, sizeof(int64_t));
    if (p->enable_fine_slicing) {
        /* fine slicing: slice i takes every atom with z in its integration range
           [min(z_m - R, z_start), max(z_m + R, z_end)] grown by z_eps (get_slicing and fd_by_z with
           Inc_Borders, slice_generator.hpp:78-129): z >= lower and (z < upper, or the highest atom
           lies at or below upper) */
        const float z_eps = 1e-4f, R_int = (float)or_rmax(p);
        float zmax = a->n > 0 ? sp->z[0] : 0.f;
        for (int64_t i = 1; i < a->n; i++)
            if (sp->z[i] > zmax) zmax = sp->z[i];
        int64_t cap = 16, cnt = 0;
        int64_t* ord = (int64_t*)malloc(sizeof(int64_t) * (size_t)cap);
        for (int s = 0; s < ns; s++) {
            float zs = sp->bounds[s], ze = sp->bounds[s + 1];
            float zm = 0.5f * (zs + ze);
            float lo = fminf(zm - R_int, zs) - z_eps, hi = fmaxf(zm + R_int, ze) + z_eps;
            for (int64_t i = 0; i < a->n; i++) {
                float z = sp->z[i];
                if (z >= lo && (z < hi || zmax <= hi)) {
                    if (cnt == cap) {
                        cap *= 2;
                        ord = (int64_t*)realloc(ord, sizeof(int64_t) * (size_t)cap);
                    }
                    ord[cnt++] = i;
                }
            }
            sp->start[s + 1] = cnt;
        }
        sp->order = ord;
        sp->z_init = ns > 0 ? (double)(float)(0.5 * (double)(sp->bounds[1] + sp->bounds[0])) : 0.0;
        return ns;
    }
    sp->order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(a->n + 1));
    for (int64_t i = 0; i < a->n; i++)
        if (sp->slice[i] >= 0) sp->start[sp->slice[i] + 1]++;
    for (int s = 0; s < ns; s++) sp->start[s + 1] += sp->start[s];
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(ns + 1));
    for (int s = 0; s <= ns; s++) fill[s] = sp->start[s];
    for (int64_t i = 0; i < a->n; i++)
        if (sp->slice[i] >= 0) sp->order[fill[sp->slice[i]]++] = i;
    free(fill);
    /* Slice::z_m (slice.hpp:19-22) */
    sp->z_init = ns > 0 ? (double)(float)(0.5 * (double)(sp->bounds[1] + sp->bounds[0])) : 0.0;
    return ns;
}

static void or_spec_free(or_spec* sp)
{
    free(sp->bounds);
    free(sp->x);
    free(sp->y);
    free(sp->z);
    free(sp->slice);
    free(sp->order);
    free(sp->start);
}

/* element spline cache */
typedef struct {
    int Z;
    double R2[MS_NR], c0[MS_NR], c1[MS_NR], c2[MS_NR], c3[MS_NR];
    double rmax;
} or_elem;

typedef struct {
    int n;
    or_elem e[128];
} or_elems;

static or_elem* or_elem_get(const ms_params* p, or_elems* es, int Z)
{
    for (int i = 0; i < es->n; i++)
        if (es->e[i].Z == Z) return &es->e[i];
    or_elem* e = &es->e[es->n++];
    e->Z = Z;
    or_spline(p, Z, e->R2, e->c0, e->c1, e->c2, e->c3, &e->rmax);
    return e;
}

/* generate_potential_single_slice: gen_slice_potential_kernel
   (device_kernels.cuh:28-47) with coeff = Vr_factor; each atom adds
   occ * spline(R^2) to every pixel with R^2 < R_max^2. */
static void or_slice_potential(const ms_params* p, const ms_atoms* a, const or_sim* s, const or_spec* sp,
                               or_elems* es, int islice, double* V)
{
    memset(V, 0, sizeof(double) * (size_t)s->N);
    if (islice < 0 || islice >= sp->ns) return;
    or_elem fe;
    for (int64_t k = sp->start[islice]; k < sp->start[islice + 1]; k++) {
        int64_t ia = sp->order[k];
        or_elem* e = or_elem_get(p, es, a->Z[ia]);
        if (p->enable_fine_slicing) {
            /* the atom's potential integrated over this slice (generate_potential_by_height with
               z_middle = slice middle - atom z, projected_potential.cuh:94-133) */
            float zs = sp->bounds[islice], ze = sp->bounds[islice + 1];
            float zm = 0.5f * (ze + zs);
            double a_mid = (double)(zm - sp->z[ia]);
            or_fine_spline(p, a->Z[ia], a_mid, (double)(ze - zs), fe.R2, fe.c0, fe.c1, fe.c2, fe.c3);
            fe.rmax = e->rmax;
            fe.Z = e->Z;
            e = &fe;
        }
        double xa = sp->x[ia], ya = sp->y[ia];
        double rmax2 = e->rmax * e->rmax;
        double coeff = s->vr_factor * (double)a->occ[ia];
        int ix0 = (int)floor((xa - e->rmax) / s->dx) - 1, ix1 = (int)ceil((xa + e->rmax) / s->dx) + 1;
        int iy0 = (int)floor((ya - e->rmax) / s->dy) - 1, iy1 = (int)ceil((ya + e->rmax) / s->dy) + 1;
        for (int iy = iy0; iy <= iy1; iy++) {
            int ry;
            if (p->pot_wrap) ry = ((iy % s->ny) + s->ny) % s->ny;
            else {
                if (iy < 0 || iy >= s->ny) continue;
                ry = iy;
            }
            double dyp = iy * s->dy - ya;
            for (int ix = ix0; ix <= ix1; ix++) {
                int rx;
                if (p->pot_wrap) rx = ((ix % s->nx) + s->nx) % s->nx;
                else {
                    if (ix < 0 || ix >= s->nx) continue;
                    rx = ix;
                }
                double dxp = ix * s->dx - xa;
                double R2 = dxp * dxp + dyp * dyp;
                if (R2 < rmax2) V[(size_t)ry * s->nx + rx] += coeff * or_spline_eval(e->R2, e->c0, e->c1, e->c2, e->c3, R2);
            }
        }
    }
}

int or_potential(const ms_params* p, const ms_atoms* a, int conf, double* V, int64_t cap, int* n_slices,
                 double* z_init)
{
    or_sim s;
    or_sim_init(p, &s);
    or_spec sp;
    or_spec_build(p, a, conf, &sp);
    or_elems* es = (or_elems*)calloc(1, sizeof(or_elems));
    if (n_slices) *n_slices = sp.ns;
    if (z_init) *z_init = sp.z_init;
    int rc = 0;
    if (V) {
        if ((int64_t)sp.ns * s.N > cap) rc = 1;
        else
            for (int i = 0; i < sp.ns; i++) or_slice_potential(p, a, &s, &sp, es, i, V + (size_t)i * s.N);
    }
    free(es);
    or_spec_free(&sp);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* operators on a wave                                                       */
/* ------------------------------------------------------------------------ */
/* Propagator table P(k) (gen_propagator_kernel, device_kernels.cuh:215-234) */
static void or_propagator(const ms_params* p, const or_sim* s, cplx* P)
{
    for (int iy = 0; iy < s->ny; iy++)
        for (int ix = 0; ix < s->nx; ix++) {
            size_t k = (size_t)iy * s->nx + ix;
            if (p->dz == 0.0) {
                P[k] = 1.0;
                continue;
            }
            double gx = or_fshift(ix, s->nx) * s->dgx, gy = or_fshift(iy, s->ny) * s->dgy;
            double amp = 1.0 / (double)s->N;
            if (p->bwl) amp *= 1.0 / (1.0 + exp(s->alpha * (gx * gx + gy * gy - s->gl2)));
            double th = s->prop_w * ((gx - s->g0x) * (gx - s->g0x) + (gy - s->g0y) * (gy - s->g0y));
            P[k] = amp * (cos(th) + I * sin(th));
        }
}

/* k-space probe (Generate_probe, device_kernels.cuh:363-388) */
static void or_probe_k(const or_sim* s, const or_lens* L, double px, double py, cplx* W)
{
    double xf = -2.0 * OR_PI * px, yf = -2.0 * OR_PI * py; /* exp_factor_*_pos with x_b - L/2 = position */
    for (int iy = 0; iy < s->ny; iy++)
        for (int ix = 0; ix < s->nx; ix++) {
            size_t k = (size_t)iy * s->nx + ix;
            float g2 = or_g2f(s, ix, iy);
            if (L->g2min <= g2 && g2 < L->g2max) {
                double gx = or_fshift(ix, s->nx) * s->dgx, gy = or_fshift(iy, s->ny) * s->dgy;
                double ph = or_chi(L, gx, gy) + xf * gx + yf * gy;
                W[k] = cos(ph) + I * sin(ph);
            } else
                W[k] = 0.0;
        }
}

/* incident wave (Incident_Wave::generate_incident_beam, incident_wave.cuh:29-46) */
static void or_incident(const ms_params* p, const or_sim* s, double px, double py, double z_init, cplx* w)
{
    int iw = p->iw_type;
    if (iw < 0) iw = (p->simulation_type == MS_SIM_HRTEM || p->simulation_type == MS_SIM_ED) ? MS_IW_PLANE : MS_IW_CONVERGENT;
    if (iw == MS_IW_CONVERGENT) {
        or_lens L;
        or_lens_init(&p->cond_lens, s->lambda, z_init, &L);
        or_probe_k(s, &L, px, py, w);
        or_fft2c(w, s->nx, s->ny, +1);
    } else if (iw == MS_IW_PLANE_TILTED) {
        /* Incident_Wave::apply_beam_tilt (incident_wave.cuh:72-78) on the plane wave: exp_r_factor_2d
           (device_kernels.cuh:519-533) with (2 pi gx_0, 2 pi gy_0), R = (i dx - lx/2, j dy - ly/2) */
        for (int iy = 0; iy < s->ny; iy++)
            for (int ix = 0; ix < s->nx; ix++) {
                double rx = ix * s->dx - 0.5 * s->lx, ry = iy * s->dy - 0.5 * s->ly;
                double ph = 2.0 * OR_PI * (s->g0x * rx + s->g0y * ry);
                w[(size_t)iy * s->nx + ix] = cos(ph) + I * sin(ph);
            }
    } else {
        for (long k = 0; k < s->N; k++) w[k] = 1.0;
    }
}

/* wave_modulation (wave_function.cuh:60-73): for every slice but the last,
   transmit (forward FFT of t*psi, fftcallbacks.cuh:36-49) then propagate
   (inverse FFT of P*Psi, fftcallbacks.cuh:11-22); the last slice only
   transmits, leaving the exit wave in reciprocal space. */
static void or_transmit(cplx* w, const double* V, long N)
{
    for (long k = 0; k < N; k++) w[k] *= cos(V[k]) + I * sin(V[k]);
}

static void or_multislice(const or_sim* s, cplx* w, const double* Vall, int ns, const cplx* P,
                          const ms_params* p, const ms_atoms* a, const or_spec* sp, or_elems* es, double* Vtmp)
{
    for (int i = 0; i < ns; i++) {
        const double* V = Vall ? Vall + (size_t)i * s->N : NULL;
        if (!V) {
            or_slice_potential(p, a, s, sp, es, i, Vtmp);
            V = Vtmp;
        }
        or_transmit(w, V, s->N);
        or_fft2c(w, s->nx, s->ny, -1);
        if (i < ns - 1) {
            for (long k = 0; k < s->N; k++) w[k] *= P[k];
            or_fft2c(w, s->nx, s->ny, +1);
        }
    }
}

/* fft_shift (device_kernels.cuh:342-362) on a real image */
static void or_fftshift(double* img, int nx, int ny)
{
    double* t = (double*)malloc(sizeof(double) * (size_t)nx * ny);
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++)
            t[(size_t)((iy + ny / 2) % ny) * nx + (ix + nx / 2) % nx] = img[(size_t)iy * nx + ix];
    memcpy(img, t, sizeof(double) * (size_t)nx * ny);
    free(t);
}

static void or_confs(const ms_params* p, int* c0, int* c1, double* w)
{
    if (p->phonon_model == MS_PHONON_FROZEN && p->pn_nconf > 0) {
        *c0 = 1;
        *c1 = p->pn_nconf;
        *w = 1.0 / (double)p->pn_nconf; /* get_weight (multislice_params_dev.cuh:209-216) */
    } else {
        *c0 = 0;
        *c1 = 0;
        *w = 1.0;
    }
}

/* ------------------------------------------------------------------------ */
/* partial coherence of the objective lens                                   */
/* ------------------------------------------------------------------------ */
/* Gauss-Hermite nodes and weights for the weight exp(-x^2), n points, weights normalised to
   sum 1.  The reference's quadrature tables (output_qt / output_qs of the missing
   multislice_params.hpp) are not shipped; this is the standard Newton iteration on the
   orthonormal Hermite recurrence (Golub and Welsch give the same nodes), with the usual
   asymptotic starting points. */
void or_gauss_hermite(int n, double* x, double* w)
{
    const double pim4 = 0.7511255444649425; /* pi^(-1/4) */
    double z = 0.0, pp = 0.0;
    int m = (n + 1) / 2;
    for (int i = 0; i < m; i++) {
        if (i == 0) z = sqrt(2.0 * n + 1.0) - 1.85575 * pow(2.0 * n + 1.0, -0.16667);
        else if (i == 1) z -= 1.14 * pow((double)n, 0.426) / z;
        else if (i == 2) z = 1.86 * z - 0.86 * x[0];
        else if (i == 3) z = 1.91 * z - 0.91 * x[1];
        else z = 2.0 * z - x[i - 2];
        for (int it = 0; it < 100; it++) {
            double p1 = pim4, p2 = 0.0;
            for (int j = 1; j <= n; j++) {
                double p3 = p2;
                p2 = p1;
                p1 = z * sqrt(2.0 / j) * p2 - sqrt((double)(j - 1) / j) * p3;
            }
            pp = sqrt(2.0 * n) * p2;
            double z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) <= 1e-15 * (1.0 + fabs(z))) break;
        }
        x[i] = z;
        x[n - 1 - i] = -z;
        w[i] = 2.0 / (pp * pp);
        w[n - 1 - i] = w[i];
    }
    if (n % 2 == 1) x[m - 1] = 0.0;
    double sw = 0.0;
    for (int i = 0; i < n; i++) sw += w[i];
    for (int i = 0; i < n; i++) w[i] /= sw;
}

/* partially coherent envelope (incoherent_phase_shift, basic_functions_dev.cuh:235-268),
   dsf_iehwgd = sqrt(2) dsf_sigma (lens_dev.cuh:138-142); temporal-only zeroes the source
   divergence, spatial-only the defocus spread (PCTF_TEM, lens_modulation.cuh:91-110) */
static double or_pctf_env(const ms_params* p, double lambda, double g2)
{
    const ms_lens* L = &p->obj_lens;
    int tsi = p->temporal_spatial_incoh ? p->temporal_spatial_incoh : MS_TSI_TEMPORAL_SPATIAL;
    double beta = (tsi == MS_TSI_TEMPORAL) ? 0.0 : L->ssf_beta;
    double df = (tsi == MS_TSI_SPATIAL) ? 0.0 : sqrt(2.0) * L->dsf_sigma;
    double c = OR_PI * beta * df;
    double u = 1.0 + 2.0 * c * c * g2;
    c = OR_PI * df * lambda * g2;
    double temp_inc = 0.5 * c * c;
    c = OR_PI * beta * (L->c30 * lambda * lambda * g2 - L->c10);
    double spa_inc = c * c * g2;
    return exp(-(spa_inc + temp_inc) / u) / sqrt(u);
}

/* the image-forming lens on an exit wave in reciprocal space: apply_CTF_kernel (device_kernels.cuh:
   445-468) with the frequency shift (gxu, gyu), the optional envelope, and an amplitude factor;
   then the inverse FFT.  out may be W itself (the update is element by element). */
static void or_ctf_apply(const ms_params* p, const or_sim* s, const or_lens* L, double gxu, double gyu, int pctf,
                         double amp, const cplx* W, cplx* out)
{
    float gxuf = (float)gxu, gyuf = (float)gyu;
    for (int iy = 0; iy < s->ny; iy++)
        for (int ix = 0; ix < s->nx; ix++) {
            size_t k = (size_t)iy * s->nx + ix;
            float gxf = (float)or_fshift(ix, s->nx) * s->dgx_f + gxuf;
            float gyf = (float)or_fshift(iy, s->ny) * s->dgy_f + gyuf;
            float g2 = gxf * gxf + gyf * gyf;
            if (L->g2min <= g2 && g2 < L->g2max) {
                double gx = or_fshift(ix, s->nx) * s->dgx + gxu, gy = or_fshift(iy, s->ny) * s->dgy + gyu;
                double ch = or_chi(L, gx, gy);
                double a = amp;
                if (pctf) a *= or_pctf_env(p, s->lambda, gx * gx + gy * gy);
                out[k] = W[k] * a * (cos(ch) + I * sin(ch));
            } else
                out[k] = 0.0;
        }
}

static void or_ctf_image(const ms_params* p, const or_sim* s, const or_lens* L, double gxu, double gyu, int pctf,
                         double amp, const cplx* W, cplx* out)
{
    or_ctf_apply(p, s, L, gxu, gyu, pctf, amp, W, out);
    or_fft2c(out, s->nx, s->ny, +1);
}

/* ED_HRTEM (single_simulator.cuh:11-126) and CBED_CBEI (:128-206) */
static int or_tem_like(const ms_params* p, const ms_atoms* a, double* img, double* re, double* im, int kspace)
{
    or_sim s;
    or_sim_init(p, &s);
    int c0, c1;
    double w;
    or_confs(p, &c0, &c1, &w);
    int full = p->data_record == MS_RECORD_WAVE;
    if (img) memset(img, 0, sizeof(double) * (size_t)s.N);
    if (re) memset(re, 0, sizeof(double) * (size_t)s.N);
    if (im) memset(im, 0, sizeof(double) * (size_t)s.N);
    cplx* wv = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
    cplx* P = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
    double* Vt = (double*)malloc(sizeof(double) * (size_t)s.N);
    or_propagator(p, &s, P);
    or_elems* es = (or_elems*)calloc(1, sizeof(or_elems));
    for (int c = c0; c <= c1; c++) {
        or_spec sp;
        or_spec_build(p, a, c, &sp);
        or_incident(p, &s, p->iw_x, p->iw_y, sp.z_init, wv);
        or_multislice(&s, wv, NULL, sp.ns, P, p, a, &sp, es, Vt);
        int tsi = p->temporal_spatial_incoh ? p->temporal_spatial_incoh : MS_TSI_TEMPORAL_SPATIAL;
        if (!kspace && p->illumination_model == MS_ILLUM_TCC && tsi != MS_TSI_COHERENT) {
            /* TCC_TEM (lens_modulation.cuh:130-176): incoherent sum over the defocus quadrature
               (c10 + dsf_iehwgd x_j) and the source quadrature (frequency shift qs_i) */
            const ms_lens* OL = &p->obj_lens;
            int nt = (tsi == MS_TSI_SPATIAL) ? 1 : OL->dsf_npoints;
            int ns1 = (tsi == MS_TSI_TEMPORAL) ? 1 : OL->ssf_npoints;
            double xt[64], wt[64], xs[16], ws[16];
            if (nt == 1) { xt[0] = 0.0; wt[0] = 1.0; } else or_gauss_hermite(nt, xt, wt);
            if (ns1 == 1) { xs[0] = 0.0; ws[0] = 1.0; } else or_gauss_hermite(ns1, xs, ws);
            double df_hw = sqrt(2.0) * OL->dsf_sigma;               /* dsf_iehwgd */
            double sf_hw = sin(OL->ssf_beta) / s.lambda;            /* ssf_iehwgd (lens_dev.cuh:143-148) */
            cplx* tmp = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
            for (int iy_s = 0; iy_s < ns1; iy_s++)
                for (int ix_s = 0; ix_s < ns1; ix_s++)
                    for (int j = 0; j < nt; j++) {
                        double wq = ws[ix_s] * ws[iy_s] * wt[j];
                        or_lens L;
                        or_lens_init(OL, s.lambda, df_hw * xt[j], &L);
                        or_ctf_image(p, &s, &L, sf_hw * xs[ix_s], sf_hw * xs[iy_s], 0, 1.0, wv, tmp);
                        for (long k = 0; k < s.N; k++) {
                            if (full) {
                                re[k] += w * wq * creal(tmp[k]);
                                im[k] += w * wq * cimag(tmp[k]);
                            } else
                                img[k] += w * wq * (creal(tmp[k]) * creal(tmp[k]) + cimag(tmp[k]) * cimag(tmp[k]));
                        }
                    }
            free(tmp);
            or_spec_free(&sp);
            continue;
        }
        if (!kspace) {
            /* OL_modulation -> CTF_TEM (lens_modulation.cuh:78-89) or PCTF_TEM (:91-110):
               apply_CTF_kernel / apply_PCTF_kernel, inverse FFT */
            or_lens L;
            or_lens_init(&p->obj_lens, s.lambda, 0.0, &L);
            or_ctf_image(p, &s, &L, 0.0, 0.0, p->illumination_model == MS_ILLUM_PARTIAL, 1.0, wv, wv);
        }
        for (long k = 0; k < s.N; k++) {
            if (full) {
                re[k] += w * creal(wv[k]);
                im[k] += w * cimag(wv[k]);
            } else
                img[k] += w * (creal(wv[k]) * creal(wv[k]) + cimag(wv[k]) * cimag(wv[k]));
        }
        or_spec_free(&sp);
    }
    if (kspace) {
        if (full) {
            or_fftshift(re, s.nx, s.ny);
            or_fftshift(im, s.nx, s.ny);
        } else
            or_fftshift(img, s.nx, s.ny);
    }
    free(es);
    free(wv);
    free(P);
    free(Vt);
    return 0;
}

/* Defocus series (apply_CTF_kernel_batch, device_kernels.cuh:469-503): every exit wave imaged
   through the coherent objective lens with chi + defocus-term(df_i) g^2, i.e. the lens at
   C10 + df[i]; images (or complex fields) summed over configurations, [nd][ny][nx]. */
int or_simulate_tem_series(const ms_params* p, const ms_atoms* a, int nd, const double* df, double* img, double* re,
                           double* im)
{
    or_sim s;
    or_sim_init(p, &s);
    int c0, c1;
    double w;
    or_confs(p, &c0, &c1, &w);
    int full = p->data_record == MS_RECORD_WAVE;
    size_t NN = (size_t)s.N * nd;
    if (img) memset(img, 0, sizeof(double) * NN);
    if (re) memset(re, 0, sizeof(double) * NN);
    if (im) memset(im, 0, sizeof(double) * NN);
    cplx* wv = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
    cplx* tmp = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
    cplx* P = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
    double* Vt = (double*)malloc(sizeof(double) * (size_t)s.N);
    or_propagator(p, &s, P);
    or_elems* es = (or_elems*)calloc(1, sizeof(or_elems));
    for (int c = c0; c <= c1; c++) {
        or_spec sp;
        or_spec_build(p, a, c, &sp);
        or_incident(p, &s, p->iw_x, p->iw_y, sp.z_init, wv);
        or_multislice(&s, wv, NULL, sp.ns, P, p, a, &sp, es, Vt);
        for (int i = 0; i < nd; i++) {
            or_lens L;
            or_lens_init(&p->obj_lens, s.lambda, df[i], &L);
            or_ctf_image(p, &s, &L, 0.0, 0.0, 0, 1.0, wv, tmp);
            size_t o = (size_t)i * s.N;
            for (long k = 0; k < s.N; k++) {
                if (full) {
                    re[o + k] += w * creal(tmp[k]);
                    im[o + k] += w * cimag(tmp[k]);
                } else
                    img[o + k] += w * (creal(tmp[k]) * creal(tmp[k]) + cimag(tmp[k]) * cimag(tmp[k]));
            }
        }
        or_spec_free(&sp);
    }
    free(es);
    free(wv);
    free(tmp);
    free(P);
    free(Vt);
    return 0;
}

int or_simulate_tem(const ms_params* p, const ms_atoms* a, double* img, double* re, double* im)
{
    return or_tem_like(p, a, img, re, im, p->simulation_type != MS_SIM_HRTEM);
}

int or_simulate_cbed(const ms_params* p, const ms_atoms* a, double* img, double* re, double* im)
{
    return or_tem_like(p, a, img, re, im, 1);
}

/* detector sums (sum_square_over_Det, device_kernels.cuh:534-579) */
static void or_detect(const ms_params* p, const or_sim* s, const cplx* W, double* out)
{
    float g2i[MS_MAX_DET], g2o[MS_MAX_DET];
    for (int d = 0; d < p->n_det; d++) {
        g2i[d] = or_g2_thr(p->det_inner[d], s->lambda);
        g2o[d] = or_g2_thr(p->det_outer[d], s->lambda);
        out[d] = 0.0;
    }
    for (int iy = 0; iy < s->ny; iy++)
        for (int ix = 0; ix < s->nx; ix++) {
            size_t k = (size_t)iy * s->nx + ix;
            float g2 = or_g2f(s, ix, iy);
            double a2 = creal(W[k]) * creal(W[k]) + cimag(W[k]) * cimag(W[k]);
            for (int d = 0; d < p->n_det; d++)
                if (g2i[d] <= g2 && g2 <= g2o[d]) out[d] += a2;
        }
}

/* run_STEM_general_simu (scan_simulator.cuh:115-183): per configuration and probe position, the
   displaced atoms inside the probe-centred window (lx x ly) +- 2 A are cropped and shifted into it
   (remove_atoms_outside_xy_range / shift_atoms, :146-157, in float as the reference's T = float),
   and the window is simulated with the probe at its centre; an empty window records the blank
   intensity N^2 x (aperture pixels inside the detector).  Configurations are summed with their
   weights (the reference assigns each over the previous one). */
static int or_simulate_stem_general(const ms_params* p, const ms_atoms* a, double* stem)
{
    or_sim s;
    or_sim_init(p, &s);
    int c0, c1;
    double w;
    or_confs(p, &c0, &c1, &w);
    int npos = p->scan_nx * p->scan_ny;
    memset(stem, 0, sizeof(double) * (size_t)p->n_det * npos);
    double blank[MS_MAX_DET];
    {
        or_lens L;
        or_lens_init(&p->cond_lens, s.lambda, 0.0, &L);
        for (int d = 0; d < p->n_det; d++) {
            float gi = or_g2_thr(p->det_inner[d], s.lambda), go = or_g2_thr(p->det_outer[d], s.lambda);
            double cnt = 0.0;
            for (int iy = 0; iy < s.ny; iy++)
                for (int ix = 0; ix < s.nx; ix++) {
                    float g2 = or_g2f(&s, ix, iy);
                    if (L.g2min <= g2 && g2 < L.g2max && gi <= g2 && g2 <= go) cnt += 1.0;
                }
            blank[d] = cnt * (double)s.N * (double)s.N;
        }
    }
    int64_t n = a->n;
    float* xd = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* yd = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* zd = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    int* cZ = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    float* cx = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* cy = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* cz = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* cs = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* co = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    ms_params q = *p;
    q.phonon_model = MS_PHONON_STILL;
    q.pn_nconf = 1;
    q.exec_mode = MS_EXEC_BATCHED;
    q.scan_nx = q.scan_ny = 1;
    q.scan_x0 = 0.5 * p->lx;
    q.scan_y0 = 0.5 * p->ly;
    q.scan_dx = q.scan_dy = 0.0;
    double Id[MS_MAX_DET];
    for (int c = c0; c <= c1; c++) {
        or_displace(p, a, c, xd, yd, zd);
        for (int ip = 0; ip < npos; ip++) {
            int ix = ip % p->scan_nx, iy = ip / p->scan_nx;
            double px = p->scan_x0 + ix * p->scan_dx, py = p->scan_y0 + iy * p->scan_dy;
            float xs = (float)(px - 0.5 * p->lx), ys = (float)(py - 0.5 * p->ly);
            float xlo = xs - 2.0f, xhi = (xs + (float)p->lx) + 2.0f;
            float ylo = ys - 2.0f, yhi = (ys + (float)p->ly) + 2.0f;
            int64_t m = 0;
            for (int64_t k = 0; k < n; k++) {
                if (xd[k] < xlo || xd[k] > xhi || yd[k] < ylo || yd[k] > yhi) continue;
                cZ[m] = a->Z[k];
                cx[m] = xd[k] - xs;
                cy[m] = yd[k] - ys;
                cz[m] = zd[k];
                cs[m] = a->sigma ? a->sigma[k] : 0.0f;
                co[m] = a->occ ? a->occ[k] : 1.0f;
                m++;
            }
            if (m == 0) {
                for (int d = 0; d < p->n_det; d++) stem[(size_t)d * npos + ip] += w * blank[d];
                continue;
            }
            ms_atoms wa;
            wa.n = m;
            wa.Z = cZ;
            wa.x = cx;
            wa.y = cy;
            wa.z = cz;
            wa.sigma = cs;
            wa.occ = co;
            or_simulate_stem(&q, &wa, Id);
            for (int d = 0; d < p->n_det; d++) stem[(size_t)d * npos + ip] += w * Id[d];
        }
    }
    free(xd); free(yd); free(zd); free(cZ); free(cx); free(cy); free(cz); free(cs); free(co);
    return 0;
}

/* run_STEM_tile_simu (scan_simulator.cuh:11-113) for a grid that covers the
   specimen: per configuration, store all slice potentials, then run every
   probe position and integrate each detector. */
int or_simulate_stem(const ms_params* p, const ms_atoms* a, double* stem)
{
    if (p->exec_mode == MS_EXEC_GENERAL) return or_simulate_stem_general(p, a, stem);
    or_sim s;
    or_sim_init(p, &s);
    int c0, c1;
    double w;
    or_confs(p, &c0, &c1, &w);
    int npos = p->scan_nx * p->scan_ny;
    memset(stem, 0, sizeof(double) * (size_t)p->n_det * npos);
    cplx* P = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
    or_propagator(p, &s, P);
    or_elems* es = (or_elems*)calloc(1, sizeof(or_elems));
    for (int c = c0; c <= c1; c++) {
        or_spec sp;
        or_spec_build(p, a, c, &sp);
        double* V = (double*)malloc(sizeof(double) * (size_t)s.N * (sp.ns > 0 ? sp.ns : 1));
        for (int i = 0; i < sp.ns; i++) or_slice_potential(p, a, &s, &sp, es, i, V + (size_t)i * s.N);
        int nth = or_get_threads();
#pragma omp parallel num_threads(nth)
        {
            cplx* wv = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
            double Id[MS_MAX_DET];
#pragma omp for schedule(dynamic, 1)
            for (int ip = 0; ip < npos; ip++) {
                int ix = ip % p->scan_nx, iy = ip / p->scan_nx;
                double px = p->scan_x0 + ix * p->scan_dx, py = p->scan_y0 + iy * p->scan_dy;
                or_incident(p, &s, px, py, sp.z_init, wv);
                or_multislice(&s, wv, V, sp.ns, P, p, a, &sp, es, NULL);
                or_detect(p, &s, wv, Id);
                for (int d = 0; d < p->n_det; d++) stem[(size_t)d * npos + ip] += w * Id[d];
            }
            free(wv);
        }
        free(V);
        or_spec_free(&sp);
    }
    free(es);
    free(P);
    return 0;
}

/* run_thickness_simu (thickness_simulator.cuh:11-85), with the transmission
   the reference forgets to attach in this path applied: after each slice
   (transmit + propagate) the wave is filtered by the annulus of detector
   `thick_det` (Filter_wave, device_kernels.cuh:389-410) and its intensity
   recorded.  Frames follow the static specimen's slice count; a phonon
   configuration with fewer slices continues through empty slices. */
int or_simulate_thickness(const ms_params* p, const ms_atoms* a, double* frames, int64_t cap, int* n_frames)
{
    or_sim s;
    or_sim_init(p, &s);
    int c0, c1;
    double w;
    or_confs(p, &c0, &c1, &w);
    or_spec sp0;
    or_spec_build(p, a, 0, &sp0);
    int nf = sp0.ns;
    or_spec_free(&sp0);
    if (n_frames) *n_frames = nf;
    if (!frames) return 0;
    if ((int64_t)nf * s.N > cap) return 1;
    memset(frames, 0, sizeof(double) * (size_t)nf * s.N);
    cplx* P = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
    or_propagator(p, &s, P);
    cplx* wv = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
    cplx* tmp = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
    double* V = (double*)malloc(sizeof(double) * (size_t)s.N);
    or_elems* es = (or_elems*)calloc(1, sizeof(or_elems));
    int d = p->thick_det;
    float g2i = or_g2_thr(p->det_inner[d], s.lambda), g2o = or_g2_thr(p->det_outer[d], s.lambda);
    for (int c = c0; c <= c1; c++) {
        or_spec sp;
        or_spec_build(p, a, c, &sp);
        or_incident(p, &s, p->iw_x, p->iw_y, sp.z_init, wv);
        for (int i = 0; i < nf; i++) {
            or_slice_potential(p, a, &s, &sp, es, i, V);
            or_transmit(wv, V, s.N);
            or_fft2c(wv, s.nx, s.ny, -1);
            for (long k = 0; k < s.N; k++) wv[k] *= P[k];
            or_fft2c(wv, s.nx, s.ny, +1);
            memcpy(tmp, wv, sizeof(cplx) * (size_t)s.N);
            or_fft2c(tmp, s.nx, s.ny, -1);
            for (int iy = 0; iy < s.ny; iy++)
                for (int ix = 0; ix < s.nx; ix++) {
                    size_t k = (size_t)iy * s.nx + ix;
                    float g2 = or_g2f(&s, ix, iy);
                    if (g2i <= g2 && g2 <= g2o) tmp[k] *= 1.0 / (double)s.N;
                    else tmp[k] = 0.0;
                }
            or_fft2c(tmp, s.nx, s.ny, +1);
            double* f = frames + (size_t)i * s.N;
            for (long k = 0; k < s.N; k++) f[k] += w * (creal(tmp[k]) * creal(tmp[k]) + cimag(tmp[k]) * cimag(tmp[k]));
        }
        or_spec_free(&sp);
    }
    free(es);
    free(V);
    free(tmp);
    free(wv);
    free(P);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* raw STEM forward and its adjoint on caller phase arrays                   */
/* ------------------------------------------------------------------------ */
static void or_exp_phase(const float* V, long N, cplx* t)
{
    for (long k = 0; k < N; k++) t[k] = cos((double)V[k]) + I * sin((double)V[k]);
}

int or_stem_forward_potential(const ms_params* p, const float* V, int n_slices, double z_init,
                              const double* probe_xy, int n_probe, double* Iout)
{
    or_sim s;
    or_sim_init(p, &s);
    cplx* P = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
    or_propagator(p, &s, P);
    int nth = or_get_threads();
#pragma omp parallel num_threads(nth)
    {
        cplx* wv = (cplx*)malloc(sizeof(cplx) * (size_t)s.N);
        double* Vd = (double*)malloc(sizeof(double) * (size_t)s.N);
#pragma omp for schedule(dynamic, 1)
        for (int ip = 0; ip < n_probe; ip++) {
            ms_params q = *p;
            q.iw_type = MS_IW_CONVERGENT;
            or_incident(&q, &s, probe_xy[2 * ip], probe_xy[2 * ip + 1], z_init, wv);
            for (int i = 0; i < n_slices; i++) {
                for (long k = 0; k < s.N; k++) Vd[k] = V[(size_t)i * s.N + k];
                or_transmit(wv, Vd, s.N);
                or_fft2c(wv, s.nx, s.ny, -1);
                if (i < n_slices - 1) {
                    for (long k = 0; k < s.N; k++) wv[k] *= P[k];
                    or_fft2c(wv, s.nx, s.ny, +1);
                }
            }
            or_detect(p, &s, wv, Iout + (size_t)ip * p->n_det);
        }
        free(wv);
        free(Vd);
    }
    free(P);
    return 0;
}

/* Adjoint: with D the unnormalised forward DFT, the forward chain is
   psi_0 = D^H Psi0, x_s = t_s psi_s, psi_{s+1} = D^H (P . D x_s), Psi = D x_{S-1}.
   For L = sum_d (I_d - T_d)^2 the backward chain is
   lambda = sum_d 4 (I_d - T_d) Psi [k in d],   mu = D^H lambda,
   dL/dV_s = Re(i t_s psi_s conj(xbar_s)),      nu_s = conj(t_s) xbar_s,
   xbar_{s} = D^H (conj(P) . D nu_{s+1}),       Psi0bar = D nu_0,
   dL/dC = sum chi_C Re(i Psi0 conj(Psi0bar)). */
int or_stem_backward(const ms_params* p, const float* V, int n_slices, double z_init, const double* probe_xy,
                     int n_probe, const float* target, double* loss, double* dL_dV, double* dL_dC10,
                     double* dL_dC30)
{
    or_sim s;
    or_sim_init(p, &s);
    long N = s.N;
    int S = n_slices;
    cplx* P = (cplx*)malloc(sizeof(cplx) * (size_t)N);
    or_propagator(p, &s, P);
    cplx* T = (cplx*)malloc(sizeof(cplx) * (size_t)N * S);
    for (int i = 0; i < S; i++) or_exp_phase(V + (size_t)i * N, N, T + (size_t)i * N);
    memset(dL_dV, 0, sizeof(double) * (size_t)N * S);
    double Ltot = 0.0, g10 = 0.0, g30 = 0.0;
    or_lens L;
    or_lens_init(&p->cond_lens, s.lambda, z_init, &L);
    float g2i[MS_MAX_DET], g2o[MS_MAX_DET];
    for (int d = 0; d < p->n_det; d++) {
        g2i[d] = or_g2_thr(p->det_inner[d], s.lambda);
        g2o[d] = or_g2_thr(p->det_outer[d], s.lambda);
    }
    int nth = or_get_threads();
    double* gV_all = (double*)calloc((size_t)nth * N * S, sizeof(double));
    double Lp[1024] = {0}, a10p[1024] = {0}, a30p[1024] = {0};
    if (nth > 1024) nth = 1024;
#pragma omp parallel num_threads(nth)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double* gV = gV_all + (size_t)tid * N * S;
        cplx* psi = (cplx*)malloc(sizeof(cplx) * (size_t)N * S);
        cplx* W0 = (cplx*)malloc(sizeof(cplx) * (size_t)N);
        cplx* w = (cplx*)malloc(sizeof(cplx) * (size_t)N);
#pragma omp for schedule(dynamic, 1)
        for (int ip = 0; ip < n_probe; ip++) {
            or_probe_k(&s, &L, probe_xy[2 * ip], probe_xy[2 * ip + 1], W0);
            memcpy(w, W0, sizeof(cplx) * (size_t)N);
            or_fft2c(w, s.nx, s.ny, +1);
            for (int i = 0; i < S; i++) {
                memcpy(psi + (size_t)i * N, w, sizeof(cplx) * (size_t)N);
                const cplx* t = T + (size_t)i * N;
                for (long k = 0; k < N; k++) w[k] *= t[k];
                or_fft2c(w, s.nx, s.ny, -1);
                if (i < S - 1) {
                    for (long k = 0; k < N; k++) w[k] *= P[k];
                    or_fft2c(w, s.nx, s.ny, +1);
                }
            }
            double Id[MS_MAX_DET];
            or_detect(p, &s, w, Id);
            double r[MS_MAX_DET];
            for (int d = 0; d < p->n_det; d++) {
                r[d] = Id[d] - (double)target[(size_t)ip * p->n_det + d];
                Lp[tid] += r[d] * r[d];
            }
            for (int iy = 0; iy < s.ny; iy++)
                for (int ix = 0; ix < s.nx; ix++) {
                    size_t k = (size_t)iy * s.nx + ix;
                    float g2 = or_g2f(&s, ix, iy);
                    double f = 0.0;
                    for (int d = 0; d < p->n_det; d++)
                        if (g2i[d] <= g2 && g2 <= g2o[d]) f += 4.0 * r[d];
                    w[k] *= f;
                }
            or_fft2c(w, s.nx, s.ny, +1); /* mu = xbar_{S-1} */
            for (int i = S - 1; i >= 0; i--) {
                if (i < S - 1) {
                    or_fft2c(w, s.nx, s.ny, -1);
                    for (long k = 0; k < N; k++) w[k] *= conj(P[k]);
                    or_fft2c(w, s.nx, s.ny, +1);
                }
                const cplx* t = T + (size_t)i * N;
                const cplx* ps = psi + (size_t)i * N;
                double* g = gV + (size_t)i * N;
                for (long k = 0; k < N; k++) {
                    g[k] += creal(I * t[k] * ps[k] * conj(w[k]));
                    w[k] *= conj(t[k]);
                }
            }
            or_fft2c(w, s.nx, s.ny, -1); /* Psi0bar */
            for (int iy = 0; iy < s.ny; iy++)
                for (int ix = 0; ix < s.nx; ix++) {
                    size_t k = (size_t)iy * s.nx + ix;
                    if (W0[k] == 0.0) continue;
                    double gx = or_fshift(ix, s.nx) * s.dgx, gy = or_fshift(iy, s.ny) * s.dgy;
                    double g2 = gx * gx + gy * gy;
                    double q = creal(I * W0[k] * conj(w[k]));
                    a10p[tid] += -OR_PI * s.lambda * g2 * q;
                    a30p[tid] += -OR_PI * s.lambda * s.lambda * s.lambda * g2 * g2 / 2.0 * q;
                }
        }
        free(psi);
        free(W0);
        free(w);
    }
    for (int t = 0; t < nth; t++) {
        Ltot += Lp[t];
        g10 += a10p[t];
        g30 += a30p[t];
        const double* gV = gV_all + (size_t)t * N * S;
        for (long k = 0; k < N * S; k++) dL_dV[k] += gV[k];
    }
    free(gV_all);
    *loss = Ltot;
    *dL_dC10 = g10;
    *dL_dC30 = g30;
    free(T);
    free(P);
    return 0;
}

/* Central finite differences of the loss of or_stem_forward_potential.  Every task (one pixel
   and one sign, or one lens coefficient and one sign) runs single-threaded on its own wave;
   a pixel task restarts each probe from the unperturbed wave stored every FD_CK slices before
   the perturbed slice, so only the slices from that store on are recomputed. */
#define FD_CK 8
static double or_fd_loss_from(const ms_params* p, const or_sim* s, const cplx* T, const cplx* P, int S, int s0,
                              int sp, long kp, double dv, const cplx* w0, const float* target, int ip, cplx* w)
{
    long N = s->N;
    memcpy(w, w0, sizeof(cplx) * (size_t)N);
    for (int i = s0; i < S; i++) {
        const cplx* t = T + (size_t)i * N;
        for (long k = 0; k < N; k++) w[k] *= t[k];
        if (i == sp) w[kp] *= cos(dv) + I * sin(dv); /* exp(i (V + dv)) = exp(i V) exp(i dv) */
        or_fft2c(w, s->nx, s->ny, -1);
        if (i < S - 1) {
            for (long k = 0; k < N; k++) w[k] *= P[k];
            or_fft2c(w, s->nx, s->ny, +1);
        }
    }
    double Id[MS_MAX_DET], L = 0.0;
    or_detect(p, s, w, Id);
    for (int d = 0; d < p->n_det; d++) {
        double r = Id[d] - (double)target[(size_t)ip * p->n_det + d];
        L += r * r;
    }
    return L;
}

int or_stem_loss_fd(const ms_params* p, const float* V, int n_slices, double z_init, const double* probe_xy,
                    int n_probe, const float* target, int n_pix, const int64_t* idx, const double* h,
                    double h10, double h30, double* fd_pix, double* fd_c10, double* fd_c30)
{
    or_sim s;
    or_sim_init(p, &s);
    long N = s.N;
    int S = n_slices;
    int nck = (S + FD_CK - 1) / FD_CK;
    cplx* P = (cplx*)malloc(sizeof(cplx) * (size_t)N);
    or_propagator(p, &s, P);
    cplx* T = (cplx*)malloc(sizeof(cplx) * (size_t)N * S);
    for (int i = 0; i < S; i++) or_exp_phase(V + (size_t)i * N, N, T + (size_t)i * N);
    /* unperturbed waves in front of slices 0, FD_CK, 2 FD_CK, ... per probe */
    cplx* ck = (cplx*)malloc(sizeof(cplx) * (size_t)N * nck * n_probe);
    int nth = or_get_threads();
#pragma omp parallel for num_threads(nth) schedule(dynamic, 1)
    for (int ip = 0; ip < n_probe; ip++) {
        ms_params q = *p;
        q.iw_type = MS_IW_CONVERGENT;
        cplx* w = ck + (size_t)ip * nck * N;
        or_incident(&q, &s, probe_xy[2 * ip], probe_xy[2 * ip + 1], z_init, w);
        for (int c = 1; c < nck; c++) {
            cplx* nx = w + (size_t)c * N;
            memcpy(nx, w + (size_t)(c - 1) * N, sizeof(cplx) * (size_t)N);
            for (int i = (c - 1) * FD_CK; i < c * FD_CK; i++) {
                const cplx* t = T + (size_t)i * N;
                for (long k = 0; k < N; k++) nx[k] *= t[k];
                or_fft2c(nx, s.nx, s.ny, -1);
                for (long k = 0; k < N; k++) nx[k] *= P[k];
                or_fft2c(nx, s.nx, s.ny, +1);
            }
        }
    }
    int ntask = 2 * n_pix + 4;
    double* Ls = (double*)calloc((size_t)ntask, sizeof(double));
#pragma omp parallel num_threads(nth)
    {
        cplx* w = (cplx*)malloc(sizeof(cplx) * (size_t)N);
        cplx* w0 = (cplx*)malloc(sizeof(cplx) * (size_t)N);
#pragma omp for schedule(dynamic, 1)
        for (int task = 0; task < ntask; task++) {
            double L = 0.0;
            if (task < 2 * n_pix) {
                int j = task / 2;
                double dv = (task % 2 == 0) ? h[j] : -h[j];
                int sp = (int)(idx[j] / N);
                long kp = (long)(idx[j] % N);
                int c = sp / FD_CK;
                for (int ip = 0; ip < n_probe; ip++)
                    L += or_fd_loss_from(p, &s, T, P, S, c * FD_CK, sp, kp, dv, ck + ((size_t)ip * nck + c) * N,
                                         target, ip, w);
            } else {
                int lt = task - 2 * n_pix;
                ms_params q = *p;
                q.iw_type = MS_IW_CONVERGENT;
                double sg = (lt % 2 == 0) ? 1.0 : -1.0;
                if (lt < 2) q.cond_lens.c10 += sg * h10;
                else q.cond_lens.c30 += sg * h30;
                for (int ip = 0; ip < n_probe; ip++) {
                    or_incident(&q, &s, probe_xy[2 * ip], probe_xy[2 * ip + 1], z_init, w0);
                    L += or_fd_loss_from(p, &s, T, P, S, 0, -1, 0, 0.0, w0, target, ip, w);
                }
            }
            Ls[task] = L;
        }
        free(w);
        free(w0);
    }
    for (int j = 0; j < n_pix; j++) fd_pix[j] = (Ls[2 * j] - Ls[2 * j + 1]) / (2.0 * h[j]);
    *fd_c10 = (Ls[2 * n_pix] - Ls[2 * n_pix + 1]) / (2.0 * h10);
    *fd_c30 = (Ls[2 * n_pix + 2] - Ls[2 * n_pix + 3]) / (2.0 * h30);
    free(Ls);
    free(ck);
    free(T);
    free(P);
    return 0;
}

/* wave_modulation / wave_modulation_batch (wave_function.cuh:60-87) on caller phases and incident
   waves: for every slice but the last, transmit then FFT, then P then inverse FFT; the last
   slice transmits and FFTs, leaving the exit waves in reciprocal space.  V [S][ny][nx] float,
   psi0 and out [B][ny][nx] complex (interleaved). */
int or_slice_loop(const ms_params* p, const float* V, int S, int B, const double* psi0, double* out)
{
    or_sim s;
    or_sim_init(p, &s);
    long N = s.N;
    cplx* P = (cplx*)malloc(sizeof(cplx) * (size_t)N);
    double* Vd = (double*)malloc(sizeof(double) * (size_t)N * S);
    or_propagator(p, &s, P);
    for (long k = 0; k < N * S; k++) Vd[k] = (double)V[k];
    cplx* w = (cplx*)out;
    memcpy(w, psi0, sizeof(cplx) * (size_t)N * B);
    for (int b = 0; b < B; b++) or_multislice(&s, w + (size_t)b * N, Vd, S, P, p, NULL, NULL, NULL, NULL);
    free(Vd);
    free(P);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* FP32 host multislice (CPU baseline only): the CBED loop of or_tem_like with */
/* the wave, its FFTs, the transmission and the propagator in single          */
/* precision; potentials, probe and pattern sums as in the FP64 path.         */
/* ------------------------------------------------------------------------ */
typedef float complex fcplx;

static void or_fft1f(fcplx* a, int n, int sign, const fcplx* tw)
{
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            fcplx t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int step = n / len;
        for (int i = 0; i < n; i += len) {
            for (int k = 0; k < len / 2; k++) {
                fcplx w = tw[k * step];
                if (sign > 0) w = conjf(w);
                fcplx u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
        }
    }
}

static fcplx* or_twiddlesf(int n)
{
    fcplx* t = (fcplx*)malloc(sizeof(fcplx) * (size_t)(n / 2 > 0 ? n / 2 : 1));
    for (int k = 0; k < n / 2; k++) {
        double a = -2.0 * OR_PI * (double)k / (double)n;
        t[k] = (float)cos(a) + I * (float)sin(a);
    }
    return t;
}

static void or_fft2cf(fcplx* d, int nx, int ny, int sign, const fcplx* twx, const fcplx* twy)
{
    int nth = or_get_threads();
#pragma omp parallel for num_threads(nth) schedule(static)
    for (int r = 0; r < ny; r++) or_fft1f(d + (size_t)r * nx, nx, sign, twx);
#pragma omp parallel num_threads(nth)
    {
        fcplx* col = (fcplx*)malloc(sizeof(fcplx) * (size_t)ny);
#pragma omp for schedule(static)
        for (int c = 0; c < nx; c++) {
            for (int r = 0; r < ny; r++) col[r] = d[(size_t)r * nx + c];
            or_fft1f(col, ny, sign, twy);
            for (int r = 0; r < ny; r++) d[(size_t)r * nx + c] = col[r];
        }
        free(col);
    }
}

int or_simulate_cbed_f32(const ms_params* p, const ms_atoms* a, double* img)
{
    or_sim s;
    or_sim_init(p, &s);
    int c0, c1;
    double w;
    or_confs(p, &c0, &c1, &w);
    long N = s.N;
    memset(img, 0, sizeof(double) * (size_t)N);
    cplx* wd = (cplx*)malloc(sizeof(cplx) * (size_t)N);
    cplx* Pd = (cplx*)malloc(sizeof(cplx) * (size_t)N);
    fcplx* wv = (fcplx*)malloc(sizeof(fcplx) * (size_t)N);
    fcplx* P = (fcplx*)malloc(sizeof(fcplx) * (size_t)N);
    double* V = (double*)malloc(sizeof(double) * (size_t)N);
    fcplx* twx = or_twiddlesf(s.nx);
    fcplx* twy = or_twiddlesf(s.ny);
    or_propagator(p, &s, Pd);
    for (long k = 0; k < N; k++) P[k] = (float)creal(Pd[k]) + I * (float)cimag(Pd[k]);
    or_elems* es = (or_elems*)calloc(1, sizeof(or_elems));
    ms_params q = *p;
    if (q.iw_type < 0) q.iw_type = MS_IW_CONVERGENT;
    for (int c = c0; c <= c1; c++) {
        or_spec sp;
        or_spec_build(p, a, c, &sp);
        or_incident(&q, &s, p->iw_x, p->iw_y, sp.z_init, wd);
        for (long k = 0; k < N; k++) wv[k] = (float)creal(wd[k]) + I * (float)cimag(wd[k]);
        for (int i = 0; i < sp.ns; i++) {
            or_slice_potential(p, a, &s, &sp, es, i, V);
            for (long k = 0; k < N; k++) {
                float v = (float)V[k];
                wv[k] *= cosf(v) + I * sinf(v);
            }
            or_fft2cf(wv, s.nx, s.ny, -1, twx, twy);
            if (i < sp.ns - 1) {
                for (long k = 0; k < N; k++) wv[k] *= P[k];
                or_fft2cf(wv, s.nx, s.ny, +1, twx, twy);
            }
        }
        for (long k = 0; k < N; k++) {
            double re = crealf(wv[k]), im = cimagf(wv[k]);
            img[k] += w * (re * re + im * im);
        }
        or_spec_free(&sp);
    }
    or_fftshift(img, s.nx, s.ny);
    free(es);
    free(twx);
    free(twy);
    free(V);
    free(P);
    free(wv);
    free(Pd);
    free(wd);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* operator-level entry points, checked against the reference's own kernels  */
/* (oracle/ref_shim) on the same inputs                                      */
/* ------------------------------------------------------------------------ */
int or_op_propagator(const ms_params* p, double* P)
{
    or_sim s;
    or_sim_init(p, &s);
    or_propagator(p, &s, (cplx*)P);
    return 0;
}

int or_op_probe(const ms_params* p, double px, double py, double z_init, double* W)
{
    or_sim s;
    or_sim_init(p, &s);
    or_lens L;
    or_lens_init(&p->cond_lens, s.lambda, z_init, &L);
    or_probe_k(&s, &L, px, py, (cplx*)W);
    return 0;
}

int or_op_ctf(const ms_params* p, int pctf, double c10_shift, double gxu, double gyu, const double* in, double* out)
{
    or_sim s;
    or_sim_init(p, &s);
    or_lens L;
    or_lens_init(&p->obj_lens, s.lambda, c10_shift, &L);
    or_ctf_apply(p, &s, &L, gxu, gyu, pctf, 1.0, (const cplx*)in, (cplx*)out);
    return 0;
}

int or_op_detect(const ms_params* p, const double* W, double* Iout)
{
    or_sim s;
    or_sim_init(p, &s);
    or_detect(p, &s, (const cplx*)W, Iout);
    return 0;
}

int or_op_slice_potential(const ms_params* p, int Z, int64_t n, const float* x, const float* y, const float* occ,
                          double* V)
{
    or_sim s;
    or_sim_init(p, &s);
    or_elems* es = (or_elems*)calloc(1, sizeof(or_elems));
    or_spec sp;
    memset(&sp, 0, sizeof(sp));
    int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    int64_t start[2] = {0, n};
    int* Zs = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) {
        order[i] = i;
        Zs[i] = Z;
    }
    float* xx = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* yy = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    memcpy(xx, x, sizeof(float) * (size_t)n);
    memcpy(yy, y, sizeof(float) * (size_t)n);
    ms_atoms a;
    memset(&a, 0, sizeof(a));
    a.n = n;
    a.Z = Zs;
    a.x = x;
    a.y = y;
    a.occ = occ;
    sp.ns = 1;
    sp.start = start;
    sp.order = order;
    sp.x = xx;
    sp.y = yy;
    or_slice_potential(p, &a, &s, &sp, es, 0, V);
    free(order);
    free(Zs);
    free(xx);
    free(yy);
    free(es);
    return 0;
}
