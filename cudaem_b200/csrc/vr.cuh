// Radial atomic potential V(r) and dV/dr in the reference's functional forms
// (Vr_dVrir_*_dev, basic_functions_dev.cuh:102-186), shared by the host spline builder
// (projected splines) and the device fine-slicing kernel (slice-integrated splines).
// Double precision throughout.
#pragma once
#include <cmath>

#include "../../include/cudaem_b200.h"

#ifdef __CUDACC__
#define MS_VR_HD __host__ __device__ __forceinline__
#else
#define MS_VR_HD inline
#endif

namespace msb {

// One element's coefficients in an MS_POT_* form (cl, cnl of Element_Coeffs).
struct ElemCoefDev {
    int form;
    int pad;
    double cl[MS_MAX_COEF], cnl[MS_MAX_COEF];
};

MS_VR_HD void vr_eval(const ElemCoefDev& c, double r, double* V, double* dV)
{
    double v = 0.0, d = 0.0;
    switch (c.form) {
    case MS_POT_DOYLE_0_4:
    case MS_POT_PENG_0_4:
    case MS_POT_PENG_0_12: {
        const int n = (c.form == MS_POT_DOYLE_0_4) ? 4 : 5;
        for (int i = 0; i < n; i++) {
            const double e = c.cl[i] * exp(-c.cnl[i] * r * r);
            v += e;
            d += -2.0 * c.cnl[i] * r * e;
        }
    } break;
    case MS_POT_KIRKLAND_0_12:
    case MS_POT_MOLIERE: {
        for (int i = 0; i < 3; i++) {
            const double e = c.cl[i] * exp(-c.cnl[i] * r) / r;
            v += e;
            d += -e * (c.cnl[i] + 1.0 / r);
        }
        for (int i = 3; i < 6; i++) {
            const double e = c.cl[i] * exp(-c.cnl[i] * r * r);
            v += e;
            d += -2.0 * c.cnl[i] * r * e;
        }
    } break;
    case MS_POT_WEICKENMEIER_0_12: {
        double s = 0.0, sd = 0.0;
        for (int i = 0; i < 6; i++) {
            s += c.cl[i] * erfc(c.cnl[i] * r);
            sd += c.cl[i] * c.cnl[i] * exp(-c.cnl[i] * c.cnl[i] * r * r);
        }
        v = s / r;
        d = -(2.0 * sd / 1.772453850905516027298) / r - s / (r * r);
    } break;
    case MS_POT_LOBATO_0_12: {
        for (int i = 0; i < 5; i++) {
            const double br = c.cnl[i] * r;
            const double e = c.cl[i] * exp(-br);
            v += e * (2.0 / br + 1.0);
            d += -e * (2.0 / (br * r) + 2.0 / r + c.cnl[i]);
        }
    } break;
    default:
        break;
    }
    *V = v;
    *dV = d;
}

}  // namespace msb
