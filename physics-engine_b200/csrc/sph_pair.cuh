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
__device__ __forceinline__ double kern_w_cubic(double r, const StepConst& k) {
    if (r < 0.0) return 0.0;
    const double q = div_h(r, k);
    if (q >= 2.0) return 0.0;
    if (q < 1.0) return k.alpha * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
    const double t = 2.0 - q;
    return k.alpha * 0.25 * t * t * t;
}

// kernels.rs:102 cubic_spline_dwdr with both divisions by h by div_h
__device__ __forceinline__ double kern_dwdr_cubic(double r, const StepConst& k) {
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

// kernels.rs:40 w for k.kernel (Wendland C2 kernels.rs:129, poly6 :169,
// spiky :196; the cubic spline above)
__device__ __forceinline__ double kern_w(double r, const StepConst& k) {
    if (k.kernel == 0) return kern_w_cubic(r, k);
    if (r < 0.0) return 0.0;
    const double a = k.alpha;
    switch (k.kernel) {
        case 1: {
            const double q = div_h(r, k);
            if (q >= 2.0) return 0.0;
            const double t = 1.0 - 0.5 * q;
            return a * t * t * t * t * (2.0 * q + 1.0);
        }
        case 2: {
            if (r >= k.h) return 0.0;
            const double t = k.h * k.h - r * r;
            return a * t * t * t;
        }
        default: {
            if (r >= k.h) return 0.0;
            const double t = k.h - r;
            return a * t * t * t;
        }
    }
}

// dW/dr for k.kernel (kernels.rs:139, 178, 205; the cubic spline above)
__device__ __forceinline__ double kern_dwdr(double r, const StepConst& k) {
    if (k.kernel == 0) return kern_dwdr_cubic(r, k);
    const double a = k.alpha;
    switch (k.kernel) {
        case 1: {
            const double q = div_h(r, k);
            if (q >= 2.0 || q <= 0.0) return 0.0;
            const double t = 1.0 - 0.5 * q;
            const double dwdq = a * (-5.0 * q) * t * t * t;
            return div_h(dwdq, k);
        }
        case 2: {
            if (r >= k.h || r <= 0.0) return 0.0;
            const double t = k.h * k.h - r * r;
            return a * (-6.0 * r * t * t);
        }
        default: {
            if (r >= k.h || r <= 0.0) return 0.0;
            const double t = k.h - r;
            return a * (-3.0 * t * t);
        }
    }
}

// The passes' kernel: the cubic spline alone (the hot path) or any kind.
template <bool CUBIC>
__device__ __forceinline__ double kw(double r, const StepConst& k) {
    return CUBIC ? kern_w_cubic(r, k) : kern_w(r, k);
}
template <bool CUBIC>
__device__ __forceinline__ double kdwdr(double r, const StepConst& k) {
    return CUBIC ? kern_dwdr_cubic(r, k) : kern_dwdr(r, k);
}

// r inside the kernel's support (kernels.rs:32)
__device__ __forceinline__ bool in_support(double r, const StepConst& k) {
    return k.kernel <= 1 ? div_h(r, k) < 2.0 : r < k.h;
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
