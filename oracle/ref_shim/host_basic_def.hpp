/*
 * host_basic_def.hpp -- TEST INFRASTRUCTURE ONLY (reference-kernel shim).
 *
 * cudaEM's device headers (device_kernels.cuh, basic_functions_dev.cuh, grid_dev.cuh,
 * lens_dev.cuh, misc_dev.cuh, device_basic_def.cuh, device_containers.cuh) include a
 * host_basic_def.hpp that the reference does not ship.  This file supplies only the
 * constants and enums those headers name, so that the reference's own kernels can be
 * compiled unchanged from their location in the reference tree and run beside the
 * oracle.  Values are the ones the reference's code fixes: c_nR = 128 is forced by the
 * seven-step unrolled search (basic_functions_dev.cuh:51-65); the others are this
 * project's choices, shared with the oracle.
 */
#ifndef MSB_REF_SHIM_HOST_BASIC_DEF_HPP
#define MSB_REF_SHIM_HOST_BASIC_DEF_HPP
#include <cmath>
#include <vector>

namespace cudaEM
{
    const int c_nR = 128;          // radial spline nodes
    const int c_nqz = 64;          // z quadrature points of fine slicing
    const int c_thrnxny = 16;      // 2-D thread block edge
    const double c_Pi = 3.141592653589793238463;
    const double c_2Pi = 6.283185307179586476925;
    const double c_2i2 = 1.414213562373095048802;   // sqrt(2)

    // host zero test and guarded division, as the device helpers of misc_dev.cuh:5-59
    // (absolute 1e-5 / relative 1e-4 for float, 1e-13 / 1e-8 for double)
    template <class T>
    inline bool isZero(const T& x)
    {
        return std::fabs((double)x) <= (sizeof(T) == sizeof(float) ? 1e-5 : 1e-13);
    }
    template <class T, class U>
    inline T Div(const T& a, const U& b)
    {
        return isZero(b) ? T(0) : T(a / T(b));
    }

    enum ePotential_Type
    {
        ePT_Doyle_0_4 = 1, ePT_Peng_0_4 = 2, ePT_Peng_0_12 = 3, ePT_Kirkland_0_12 = 4,
        ePT_Weickenmeier_0_12 = 5, ePT_Lobato_0_12 = 6, ePT_none = 0
    };
}
#endif
