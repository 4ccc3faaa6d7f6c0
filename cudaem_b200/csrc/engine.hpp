// Internal declarations shared by the host code, the kernels and the C ABI.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cudaem_b200.h"

namespace msb {

struct MsError : std::runtime_error {
    ms_status st;
    MsError(ms_status s, const std::string& m) : std::runtime_error(m), st(s) {}
};

#define MS_REQUIRE(cond, status, msg)                  \
    do {                                               \
        if (!(cond)) throw ::msb::MsError(status, msg); \
    } while (0)

// Beam physics: relativistic wavelength (A), interaction constant (rad/(V A)), gamma,
// and the transmission factor Vr_factor = sigma / cos(theta) (transmission_function.cuh:60-61).
struct Physics {
    double lambda, sigma, gamma, vr_factor;
};
Physics physics_of(double E0_kV, double theta);

// Grid constants (Grid_2d_Dev::set_input_data, grid_dev.cuh:307-325) in double and in the
// float forms the device masks use.
struct GridConst {
    int nx, ny;
    double lx, ly, dx, dy, dgx, dgy;
    float dx_f, dy_f, dgx_f, dgy_f;
    double gl2, alpha;
    int bwl;
    double g0x, g0y;   // beam tilt in reciprocal space (multislice_params_dev.cuh:201-208)
    double prop_w;     // -pi * lambda * dz (propagation_function.cuh:31)
};
GridConst grid_of(const ms_params& p, const Physics& ph);

// Lens_Dev coefficients (lens_dev.cuh:40-57), each dropped to zero when it is zero within
// the reference's float tolerance (nonZero_dev, misc_dev.cuh:17-23).  The aperture limits
// are float squares of float frequencies, exactly as the masks compare them.
struct LensCoef {
    int m, phi_req;
    double cc10, cc12, cc21, cc23, cc30, cc32, cc34, cc41, cc43, cc45, cc50, cc52, cc54, cc56;
    double p12, p21, p23, p32, p34, p41, p43, p45, p52, p54, p56;
    float g2min, g2max;
};
LensCoef lens_coef(const ms_lens& L, double lambda, double c10_shift);
double gate_coef(double v);
float g2_threshold(double angle, double lambda);

// Radial spline of one element in the device layout (VR_Cubic coefficients of
// Element_Coeffs_Dev, device_containers.cuh:243-249).
struct ElemCoef4 {
    float c0, c1, c2, c3;
};
struct ElemTable {
    float R2[MS_NR];
    ElemCoef4 c[MS_NR];   // cubic coefficients of node i, packed for one 16-byte load
    float rmax, rmax2;
    float l0, inv_dl;   // log2(R2[0]) and nodes per log2 unit, for the direct index guess
    float l0s;          // -l0 * inv_dl: the index guess is floor(log2(r2) * inv_dl + l0s)
    int Z;
    int pad[2];
};
void build_elem_table(const ms_params& p, int Z, ElemTable* t);
// Projected potential V_z(R) and dV_z/dR^2 of an element, before tapering (FP64).
void projected_potential_fp64(const ms_params& p, int Z, double R, double* Vz, double* dVz_dR2);

// Host specimen: Specimen::update_atom + Slice_Generator::calculate.
int border_of(const ms_params& p);
int iw_of(const ms_params& p);
void host_displace(const ms_params& p, const ms_atoms& a, int conf, float* x, float* y, float* z);
int host_slices(const ms_params& p, const float* z, int64_t n, std::vector<float>* bounds, int* atom_slice);

// Fine slicing: the integration radius (the largest cut-off radius, atoms.R_int_max),
// each element's coefficients for the device, and the z quadrature on [-1/2, 1/2].
float fine_radius(const ms_params& p);
struct ElemCoefDev;
ElemCoefDev elem_coef_dev(const ms_params& p, int Z);
void gauss_legendre_half(int n, double* x, double* w);
constexpr int kNqz = 64;   // z quadrature points per slice (c_nqz)

void validate_params(const ms_params& p);
void validate_atoms(const ms_params& p, const ms_atoms* a);

// Configurations run by one call: conf indices (1-based for frozen phonons, 0 for the
// static specimen) and their weight (get_weight, multislice_params_dev.cuh:209-216).
struct ConfSet {
    std::vector<int> confs;
    double weight;
};
ConfSet conf_set(const ms_params& p);

}  // namespace msb
