// Deterministic arithmetic shared by host and device code.
//
// The frozen-phonon displacements and the slicing planes decide which slice
// an atom lands in, so the host implementation (specimen API) and the device
// implementation (the simulate path) must produce the same bits.  Every
// operation here is an IEEE-754 correctly rounded add, multiply, divide or
// square root, written through macros that map to the explicit
// round-to-nearest intrinsics on the device (which never contract into FMA)
// and to plain operators on the host (compiled with -ffp-contract=off).
//
// The Gaussian generator keys SplitMix64 on (seed, configuration, atom,
// stream) and applies Marsaglia's polar method; the logarithm it needs is
// evaluated from frexp and the Maclaurin series of atanh, so no libm or
// CUDA math-library routine enters the result.  The reference's own
// generator lives in headers it does not ship (random_lib.hpp,
// atom_coor_data.hpp; called at single_simulator.cuh:65-74).
#pragma once
#include <cstdint>
#include <cmath>
#include <cstring>

#ifdef __CUDA_ARCH__
#define MSD_ADD(a, b) __dadd_rn((a), (b))
#define MSD_SUB(a, b) __dadd_rn((a), -(b))
#define MSD_MUL(a, b) __dmul_rn((a), (b))
#define MSD_DIV(a, b) __ddiv_rn((a), (b))
#define MSD_SQRT(a) __dsqrt_rn(a)
#define MSF_ADD(a, b) __fadd_rn((a), (b))
#define MSF_SUB(a, b) __fsub_rn((a), (b))
#define MSF_MUL(a, b) __fmul_rn((a), (b))
#define MSF_DIV(a, b) __fdiv_rn((a), (b))
#else
#define MSD_ADD(a, b) ((a) + (b))
#define MSD_SUB(a, b) ((a) - (b))
#define MSD_MUL(a, b) ((a) * (b))
#define MSD_DIV(a, b) ((a) / (b))
#define MSD_SQRT(a) std::sqrt(a)
#define MSF_ADD(a, b) ((a) + (b))
#define MSF_SUB(a, b) ((a) - (b))
#define MSF_MUL(a, b) ((a) * (b))
#define MSF_DIV(a, b) ((a) / (b))
#endif

#if defined(__CUDACC__)
#define MS_HD __host__ __device__ __forceinline__
#else
#define MS_HD inline
#endif

namespace msb {

MS_HD uint64_t det_mix(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// frexp for finite positive normal doubles, by bit manipulation (exact).
MS_HD double det_frexp(double s, int* e)
{
    uint64_t b;
#ifdef __CUDA_ARCH__
    b = (uint64_t)__double_as_longlong(s);
#else
    std::memcpy(&b, &s, 8);
#endif
    int ex = (int)((b >> 52) & 0x7FF);
    *e = ex - 1022;
    b = (b & 0x800FFFFFFFFFFFFFULL) | (0x3FEULL << 52);
    double m;
#ifdef __CUDA_ARCH__
    m = __longlong_as_double((long long)b);
#else
    std::memcpy(&m, &b, 8);
#endif
    return m;
}

// log(s) for s in (0, 1), from IEEE-exact operations only.
MS_HD double det_log(double s)
{
    int e;
    double m = det_frexp(s, &e);
    if (m < 0.70710678118654752440) {
        m = MSD_MUL(m, 2.0);
        e = e - 1;
    }
    double t = MSD_DIV(MSD_SUB(m, 1.0), MSD_ADD(m, 1.0));
    double t2 = MSD_MUL(t, t);
    const double inv[14] = {1.0 / 27.0, 1.0 / 25.0, 1.0 / 23.0, 1.0 / 21.0, 1.0 / 19.0, 1.0 / 17.0, 1.0 / 15.0,
                            1.0 / 13.0, 1.0 / 11.0, 1.0 / 9.0,  1.0 / 7.0,  1.0 / 5.0,  1.0 / 3.0,  1.0};
    double q = inv[0];
#pragma unroll
    for (int k = 1; k < 14; k++) q = MSD_ADD(MSD_MUL(q, t2), inv[k]);
    double lm = MSD_MUL(MSD_MUL(2.0, t), q);
    return MSD_ADD(MSD_MUL((double)e, 0.69314718055994530942), lm);
}

MS_HD void det_gauss_pair(uint64_t seed, int conf, int64_t atom, int stream, double* g0, double* g1)
{
    uint64_t key = det_mix(det_mix(det_mix(seed) ^ (uint64_t)(int64_t)conf) ^
                           (((uint64_t)atom << 2) | (uint64_t)stream));
    for (int it = 0; it < 64; it++) {
        uint64_t r0 = det_mix(key + (uint64_t)(2 * it));
        uint64_t r1 = det_mix(key + (uint64_t)(2 * it + 1));
        double u = MSD_MUL(MSD_ADD((double)(r0 >> 11), 0.5), 1.1102230246251565404e-16);
        double v = MSD_MUL(MSD_ADD((double)(r1 >> 11), 0.5), 1.1102230246251565404e-16);
        u = MSD_SUB(MSD_MUL(2.0, u), 1.0);
        v = MSD_SUB(MSD_MUL(2.0, v), 1.0);
        double s = MSD_ADD(MSD_MUL(u, u), MSD_MUL(v, v));
        if (s < 1.0 && s > 0.0) {
            double f = MSD_SQRT(MSD_DIV(MSD_MUL(-2.0, det_log(s)), s));
            *g0 = MSD_MUL(u, f);
            *g1 = MSD_MUL(v, f);
            return;
        }
    }
    *g0 = 0.0;
    *g1 = 0.0;
}

// Displaced position of one atom in configuration conf (>= 1); conf 0 leaves it in place.
MS_HD void det_displace(uint64_t seed, int conf, int64_t atom, float sigma, int dx, int dy, int dzf, float* x,
                        float* y, float* z)
{
    if (conf <= 0) return;
    double g0, g1, g2, g3;
    det_gauss_pair(seed, conf, atom, 0, &g0, &g1);
    det_gauss_pair(seed, conf, atom, 1, &g2, &g3);
    double s = (double)sigma;
    if (dx) *x = MSF_ADD(*x, (float)MSD_MUL(s, g0));
    if (dy) *y = MSF_ADD(*y, (float)MSD_MUL(s, g1));
    if (dzf) *z = MSF_ADD(*z, (float)MSD_MUL(s, g2));
}

// Slice planes of Slice_Generator::gene_bounds (slice_generator.hpp:130-168) in float.
// z_eps stands for epsilon_rel<float>() of the reference's missing host header.
constexpr float kSliceEps = 1e-4f;

MS_HD int det_nplanes(float vmin, float vmax, float dz)
{
    float s_v = MSF_SUB(vmax, vmin);
    return (int)floorf(MSF_DIV(MSF_ADD(s_v, kSliceEps), dz)) + 2;
}

MS_HD float det_plane(int i, int nv, float vmin, float vmax, float dz, int border)
{
    if (border == 0) {  // eMB_Min
        float zb = MSF_SUB(vmin, MSF_MUL(2.0f, kSliceEps));
        return MSF_ADD(zb, MSF_MUL((float)i, dz));
    } else if (border == 1) {  // eMB_Max: plane nv-1-k = z_top - k dz
        float zt = MSF_ADD(vmax, MSF_MUL(2.0f, kSliceEps));
        int k = nv - 1 - i;
        return MSF_SUB(zt, MSF_MUL((float)k, dz));
    } else {  // eMB_Middle
        float zb = MSF_MUL(0.5f, MSF_SUB(MSF_ADD(vmin, vmax), MSF_MUL((float)(nv - 1), dz)));
        return MSF_ADD(zb, MSF_MUL((float)i, dz));
    }
}

// Slice of an atom at height zk: the i with b[i] <= zk < b[i+1]; the topmost atom sitting
// exactly on the last plane belongs to the last slice (fd_by_z, slice_generator.hpp:109-129).
MS_HD int det_slice_of(float zk, const float* b, int nv, float vmax)
{
    if (zk >= b[0] && zk < b[nv - 1]) {
        int lo = 0, hi = nv - 1;
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (b[mid] <= zk) lo = mid; else hi = mid;
        }
        return lo;
    }
    if (zk == b[nv - 1] && zk == vmax) return nv - 2;
    return -1;
}

// Fine slicing: does slice [zs, ze) integrate the atom at height z?  Its integration range is
// [min(z_m - R, zs), max(z_m + R, ze)] grown by the slicing epsilon, with z_m the slice middle
// (get_slicing and fd_by_z with Inc_Borders, slice_generator.hpp:78-129): z >= lower and
// (z < upper, or the highest atom lies at or below upper).
MS_HD bool det_fine_member(float z, float zs, float ze, float rint, float zmax)
{
    const float zm = MSF_MUL(0.5f, MSF_ADD(zs, ze));
    const float lo = MSF_SUB(fminf(MSF_SUB(zm, rint), zs), kSliceEps);
    const float hi = MSF_ADD(fmaxf(MSF_ADD(zm, rint), ze), kSliceEps);
    return z >= lo && (z < hi || zmax <= hi);
}

// Frequency of FFT index i on an n-point axis, as float (grid_dev.cuh:429-444).
MS_HD float det_gfreq(int i, int n, float dg)
{
    int k = (i < n / 2) ? i : i - n;
    return MSF_MUL((float)k, dg);
}

MS_HD float det_g2(int ix, int iy, int nx, int ny, float dgx, float dgy)
{
    float gx = det_gfreq(ix, nx, dgx), gy = det_gfreq(iy, ny, dgy);
    return MSF_ADD(MSF_MUL(gx, gx), MSF_MUL(gy, gy));
}

// The same with the frequencies shifted by (gxu, gyu) (apply_CTF_kernel's source-point shift,
// device_kernels.cuh:454-456); a zero shift gives det_g2's value exactly.
MS_HD float det_g2_shift(int ix, int iy, int nx, int ny, float dgx, float dgy, float gxu, float gyu)
{
    float gx = MSF_ADD(det_gfreq(ix, nx, dgx), gxu), gy = MSF_ADD(det_gfreq(iy, ny, dgy), gyu);
    return MSF_ADD(MSF_MUL(gx, gx), MSF_MUL(gy, gy));
}

}  // namespace msb
