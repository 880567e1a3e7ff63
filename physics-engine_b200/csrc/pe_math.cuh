// Scalar math shared by host and device code of the WCSPH step.
//
// Every routine keeps the operand order and association of the reference
// (`crates/pe-fluid/src/kernels.rs`, `eos.rs`, `grid.rs`) so that, compiled
// without FMA contraction (`--fmad=false`), results are bit-identical to the
// reference's f64 arithmetic.
#pragma once

#include <cstdint>
#include <cmath>

#if defined(__CUDACC__)
#define PE_HD __host__ __device__ __forceinline__
#else
#define PE_HD inline
#endif

namespace pe {

// f64::consts::PI (0x400921FB54442D18).
constexpr double kPi = 3.14159265358979311599796346854;

// kernels.rs:79 cubic_alpha. 3-D: 1 / (pi h^3); 2-D: 10 / (7 pi h^2).
PE_HD double cubic_alpha(double h, int dim) {
    return dim == 2 ? 10.0 / (7.0 * kPi * h * h) : 1.0 / (kPi * h * h * h);
}

// kernels.rs:40 w + kernels.rs:86 cubic_spline_w, with alpha hoisted (it is a
// pure function of h and dim, so hoisting does not change any bit).
PE_HD double cubic_w(double r, double h, double alpha) {
    if (h <= 0.0 || r < 0.0) return 0.0;
    double q = r / h;
    if (q >= 2.0) return 0.0;
    if (q < 1.0) return alpha * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
    double t = 2.0 - q;
    return alpha * 0.25 * t * t * t;
}

// kernels.rs:102 cubic_spline_dwdr.
PE_HD double cubic_dwdr(double r, double h, double alpha) {
    double q = r / h;
    if (q >= 2.0 || q <= 0.0) return 0.0;
    double dwdq;
    if (q < 1.0) {
        dwdq = alpha * (-3.0 * q + 2.25 * q * q);
    } else {
        double t = 2.0 - q;
        dwdq = alpha * (-0.75 * t * t);
    }
    return dwdq / h;
}

// grid.rs:144 floor_i32: floor toward -inf, non-finite -> 0, clamped to the
// open i32 range.
PE_HD int32_t floor_i32(double x) {
    if (!(x - x == 0.0)) return 0;  // NaN or +-inf
    const double lo = -2147483647.0, hi = 2147483646.0;
    double c = x < lo ? lo : (x > hi ? hi : x);
    int32_t t = (int32_t)c;
    if ((double)t > c) return t - 1;
    return t;
}

// ---------------------------------------------------------------------------
// Tait power (ratio^gamma, eos.rs:68).
//
// For an integer exponent the power is evaluated by binary exponentiation in
// double-double arithmetic (Dekker 1971 products; error-free product via an
// explicit fma, which is exact and unaffected by --fmad=false) and rounded
// once, which gives the correctly rounded double except when the exact value
// lies within ~2^-100 (relative) of a rounding midpoint. Host and device use
// this same routine, so the GPU path and the host bookkeeping agree bitwise.
// ---------------------------------------------------------------------------
struct DD {
    double hi, lo;
};

PE_HD DD dd_mul(DD a, DD b) {
    double p = a.hi * b.hi;
    double e = fma(a.hi, b.hi, -p);  // exact: a.hi*b.hi - p
    e += a.hi * b.lo + a.lo * b.hi;
    double s = p + e;                 // renormalise (fast two-sum, |p| >= |e|)
    return DD{s, e - (s - p)};
}

PE_HD double pow_int_dd(double x, int n) {
    unsigned e = n < 0 ? (unsigned)(-n) : (unsigned)n;
    DD r{1.0, 0.0};
    DD b{x, 0.0};
    while (e) {
        if (e & 1u) r = dd_mul(r, b);
        e >>= 1;
        if (e) b = dd_mul(b, b);
    }
    if (!(r.hi - r.hi == 0.0)) return r.hi;  // overflow to inf / NaN input
    if (n < 0) {
        // 1 / (hi + lo) to double-double accuracy, then round.
        double q = 1.0 / r.hi;
        double rem = fma(-q, r.hi, 1.0) - q * r.lo;
        return q + rem / r.hi;
    }
    return r.hi + r.lo;
}

// Returns the exponent as an int if gamma is an integer in [-64, 64], else 0
// with *is_int = false.
PE_HD int integer_exponent(double gamma, bool* is_int) {
    if (gamma == gamma && gamma >= -64.0 && gamma <= 64.0 && (double)(int)gamma == gamma) {
        *is_int = true;
        return (int)gamma;
    }
    *is_int = false;
    return 0;
}

}  // namespace pe
