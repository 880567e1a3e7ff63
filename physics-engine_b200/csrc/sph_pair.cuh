// Per-pair f64 helpers shared by the SPH passes (cubic spline with the exact
// division by h, and the boundary half-space filter). Compiled with
// --fmad=false like every f64 pass.
#pragma once

#include "pe_math.cuh"
#include "wcsph_device.cuh"

namespace pe {

// a / h, correctly rounded, in one multiply and two fused multiply-adds.
// Markstein's theorem: with y = RN(1/h) and q0 = RN(a y) (within one ulp of
// a/h), the remainder r = a - q0 h is exact in an fma and RN(q0 + r y) =
// RN(a/h), for results in the normal range. The rare non-finite or tiny
// operands take the IEEE division.
__device__ __forceinline__ double div_h(double a, const StepConst& k) {
    if (!(fabs(a) < 1e300) || fabs(a) < 1e-290) return a / k.h;
    const double q0 = a * k.inv_h;
    const double r = fma(-q0, k.h, a);
    return fma(r, k.inv_h, q0);
}

// kernels.rs:86 cubic_spline_w with q = r / h by div_h (same bits)
__device__ __forceinline__ double kern_w(double r, const StepConst& k) {
    if (r < 0.0) return 0.0;
    const double q = div_h(r, k);
    if (q >= 2.0) return 0.0;
    if (q < 1.0) return k.alpha * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
    const double t = 2.0 - q;
    return k.alpha * 0.25 * t * t * t;
}

// kernels.rs:102 cubic_spline_dwdr with both divisions by h by div_h
__device__ __forceinline__ double kern_dwdr(double r, const StepConst& k) {
    const double q = div_h(r, k);
    if (q >= 2.0 || q <= 0.0) return 0.0;
    double dwdq;
    if (q < 1.0) {
        dwdq = k.alpha * (-3.0 * q + 2.25 * q * q);
    } else {
        const double t = 2.0 - q;
        dwdq = k.alpha * (-0.75 * t * t);
    }
    return div_h(dwdq, k);
}

// particles.rs:126 boundary_sees_fluid
__device__ __forceinline__ bool sees_fluid(const StepConst& k, double4 xb, double4 nb,
                                           double xfx, double xfy, double xfz) {
    double n2 = nb.x * nb.x + nb.y * nb.y + nb.z * nb.z;
    if (n2 <= 0.0) return true;
    double eps = k.boundary_eps_h * sqrt(fmax(n2, 0.0));
    double d = (xfx - xb.x) * nb.x + (xfy - xb.y) * nb.y + (xfz - xb.z) * nb.z;
    return d > -eps;
}

}  // namespace pe
