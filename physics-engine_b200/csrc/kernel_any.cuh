// The four SPH kernels of crates/pe-fluid/src/kernels.rs (cubic spline,
// Wendland C2, poly6, spiky) for the PBF and DFSPH steps, with the
// reference's operand order. Divisions by h go through the exact division
// (RN(1/h) and one Markstein correction, returns RN(a/h)); the pow
// normalisations of poly6 and spiky are computed once on the host by the
// correctly rounded integer power. Compiled with --fmad=false like every f64
// pass.
#pragma once

#include <cmath>

#include "pe_math.cuh"

namespace pe {

enum KernelKind : int { kCubic = 0, kWendland = 1, kPoly6 = 2, kSpiky = 3 };  // kernels.rs:19

struct KernelFn {
    int kind;
    double h, inv_h;  // inv_h = RN(1 / h)
    double alpha;     // the kind's normalisation for (h, dim)
};

// kernels.rs:32 support_radius
inline double kernel_support(int kind, double h) { return (kind == kCubic || kind == kWendland) ? 2.0 * h : h; }

// Normalisations (kernels.rs:79, 121, 153, 181), host side.
inline double kernel_alpha(int kind, double h, int dim) {
    const double pi = 3.14159265358979311599796346854;  // f64::consts::PI
    switch (kind) {
        case kCubic: return dim == 2 ? 10.0 / (7.0 * pi * h * h) : 1.0 / (pi * h * h * h);
        case kWendland: return dim == 2 ? 7.0 / (4.0 * pi * h * h) : 21.0 / (16.0 * pi * h * h * h);
        case kPoly6: return dim == 2 ? 4.0 / (pi * pow_int_dd(h, 8)) : 315.0 / (64.0 * pi * pow_int_dd(h, 9));
        default: return dim == 2 ? 10.0 / (pi * pow_int_dd(h, 5)) : 15.0 / (pi * pow_int_dd(h, 6));
    }
}

inline KernelFn make_kernel_fn(int kind, double h, int dim) {
    return KernelFn{kind, h, 1.0 / h, kernel_alpha(kind, h, dim)};
}

// RN(a / h): on the device by one multiply and a Markstein correction, on the
// host by the IEEE division (the same value)
PE_HD double kdiv_h(double a, const KernelFn& k) {
#ifdef __CUDA_ARCH__
    if (!(fabs(a) < 1e300) || fabs(a) < 1e-290) return a / k.h;
    const double q0 = a * k.inv_h;
    const double r = fma(-q0, k.h, a);
    return fma(r, k.inv_h, q0);
#else
    return a / k.h;
#endif
}

// kernels.rs:40 w
PE_HD double kfn_w(const KernelFn& k, double r) {
    if (k.h <= 0.0 || r < 0.0) return 0.0;
    const double a = k.alpha;
    switch (k.kind) {
        case kCubic: {
            const double q = kdiv_h(r, k);
            if (q >= 2.0) return 0.0;
            if (q < 1.0) return a * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
            const double t = 2.0 - q;
            return a * 0.25 * t * t * t;
        }
        case kWendland: {
            const double q = kdiv_h(r, k);
            if (q >= 2.0) return 0.0;
            const double t = 1.0 - 0.5 * q;
            return a * t * t * t * t * (2.0 * q + 1.0);
        }
        case kPoly6: {
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

// dW/dr of each kind (kernels.rs:102, 139, 169, 197)
PE_HD double kfn_dwdr(const KernelFn& k, double r) {
    const double a = k.alpha;
    switch (k.kind) {
        case kCubic: {
            const double q = kdiv_h(r, k);
            if (q >= 2.0 || q <= 0.0) return 0.0;
            double dwdq;
            if (q < 1.0) {
                dwdq = a * (-3.0 * q + 2.25 * q * q);
            } else {
                const double t = 2.0 - q;
                dwdq = a * (-0.75 * t * t);
            }
            return kdiv_h(dwdq, k);
        }
        case kWendland: {
            const double q = kdiv_h(r, k);
            if (q >= 2.0 || q <= 0.0) return 0.0;
            const double t = 1.0 - 0.5 * q;
            const double dwdq = a * (-5.0 * q) * t * t * t;
            return kdiv_h(dwdq, k);
        }
        case kPoly6: {
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

// kernels.rs:56 grad_w at rij = rj - ri (returns grad_i W)
PE_HD void kfn_grad(const KernelFn& k, double rx, double ry, double rz, double* gx,
                                         double* gy, double* gz) {
    if (k.h <= 0.0) {
        *gx = *gy = *gz = 0.0;
        return;
    }
    const double r = sqrt(rx * rx + ry * ry + rz * rz);
    const double dwdr = kfn_dwdr(k, r);
    if (r < 1e-30) {
        *gx = *gy = *gz = 0.0;
        return;
    }
    const double s = -dwdr / r;
    *gx = rx * s;
    *gy = ry * s;
    *gz = rz * s;
}

}  // namespace pe
