// Divergence-free SPH (crates/pe-fluid/src/dfsph.rs) on the cell-sorted state
// of a World whose grid cell is the kernel's support radius.
//
// Slot state: pos = (x, psi), vel = (v, rho), acc = (v*, warm-start kappa of
// the density solver), nout = (n_out, warm-start kappa of the divergence
// solver), bf = boundary reaction, p = the density solver's kappa (the
// reference's pressure diagnostic). All of it moves with the re-sort.
//
// Lists: a fluid slot's visit list holds its fluid neighbours in support and
// every boundary candidate of the 27 (9) neighbour cells, as the reference's
// lists do: the reaction weights (dfsph.rs:498-518) range over every boundary
// candidate, in or out of the support. Fluid candidates out of the support add
// +-0 and are left out; the solver's neighbour count (dfsph.rs:281-296), which
// counts every candidate, takes them from the union size the list build records.
//
// Boundary reactions: the reference scatters, for fluid i in ascending index,
// F_b(i) wt_ij / sum_j wt_ij onto each boundary candidate j. The neighbour
// relation of the cell grid is symmetric, so a boundary slot gathers the same
// terms from its fluid candidates in ascending original index (its "lower"
// list), which is the reference's order of additions.
//
// The solvers' average errors are sequential sums in original index order
// (dfsph.rs:552-569, 604-616) of non-negative terms, and only their comparison
// with the tolerance is used. Any summation order of n non-negative terms lies
// within gamma_(n-1) = (n-1)u / (1 - (n-1)u) (relative) of the exact sum, so a
// parallel sum S brackets the sequential one in S (1 +- 2 gamma / (1 - gamma)).
// When the whole bracket, divided by the fluid count, falls on one side of the
// tolerance, that is the reference's decision; otherwise the terms (scattered
// to original order) are summed sequentially by one thread. Either way the
// convergence decision is the reference's bit for bit. Compiled with
// --fmad=false.
#include <algorithm>
#include <cmath>
#include <limits>

#include "dfsph.cuh"
#include "list_iter.cuh"

namespace pe {

namespace {

constexpr uint32_t kDfThreads = 128;

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

__device__ __forceinline__ bool is_boundary(const StateBufs& s, uint32_t i) { return s.flags[i] & kFlagBoundary; }

// particles.rs:126 boundary_sees_fluid (un-oriented samples see everything)
__device__ __forceinline__ bool sees(const DfsphConst& k, const double4& xb, const double4& nb, bool oriented,
                                     const double4& xf) {
    if (!oriented) return true;
    const double n2 = nb.x * nb.x + nb.y * nb.y + nb.z * nb.z;
    if (n2 <= 0.0) return true;
    const double eps = k.eps_h * sqrt(fmax(n2, 0.0));
    const double d = (xf.x - xb.x) * nb.x + (xf.y - xb.y) * nb.y + (xf.z - xb.z) * nb.z;
    return d > -eps;
}

// A candidate beyond the kernel's support adds an exact +-0 to the gradient
// and kernel sums (W and grad W vanish there); those sums skip it. The margin
// on far2 keeps the test conservative under rounding.
__device__ __forceinline__ bool far_pair(const DfsphConst& k, const double4& xi, const double4& xj) {
    const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    return dx * dx + dy * dy + dz * dz > k.far2;
}

// dfsph.rs:309-323 neighbour_mass_for
__device__ __forceinline__ double nmass(const DfsphConst& k, const StateBufs& s, uint32_t e, const double4& xj,
                                        const double4& xi) {
    if (!(e & kEntryBoundary)) return k.mass;
    const uint32_t j = e & kEntrySlotMask;
    const bool oriented = e & kEntryOriented;
    return sees(k, xj, oriented ? s.nout[j] : make_double4(0, 0, 0, 0), oriented, xi) ? k.rho0 * xj.w : 0.0;
}

// dfsph.rs:718-735: boundary forces cleared, v* = v + g dt (2-D: z = 0)
__global__ void k_df_begin(uint32_t n, DfsphConst k, double dt, StateBufs s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 f = s.bf[i];
    f.x = 0.0;
    f.y = 0.0;
    f.z = 0.0;
    s.bf[i] = f;
    const double4 v = s.vel[i];
    double4 a = s.acc[i];
    if (is_boundary(s, i)) {
        a.x = v.x;
        a.y = v.y;
        a.z = v.z;
    } else {
        const double gx = k.gx * dt, gy = k.gy * dt, gz = k.gz * dt;
        a.x = v.x + gx;
        a.y = v.y + gy;
        a.z = k.dim == 2 ? 0.0 : v.z + gz;
    }
    s.acc[i] = a;
}

// dfsph.rs:382-416 XSPH on v* (fluid neighbours)
__global__ void __launch_bounds__(kDfThreads) k_df_xsph(uint32_t n, DfsphConst k, StateBufs s, ListBufs l,
                                                       double4* __restrict__ dv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (is_boundary(s, i)) {
        dv[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        return;
    }
    const double4 xi = s.pos[i], vi = s.acc[i];
    const double rho_i = s.vel[i].w;
    double cx = 0.0, cy = 0.0, cz = 0.0;
    for_each_entry(list_ref(l, i, kListVisit), [&](uint32_t e) {
        if (e & kEntryBoundary) return;
        const uint32_t j = e & kEntrySlotMask;
        const double4 xj = s.pos[j];
        if (far_pair(k, xi, xj)) return;
        const double4 vj = s.acc[j];
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double wij = kfn_w(k.kf, sqrt(dx * dx + dy * dy + dz * dz));
        const double rho_bar = 0.5 * (rho_i + s.vel[j].w);
        const double f = k.mass / fmax(rho_bar, 1e-12) * wij;
        cx = cx + (vj.x - vi.x) * f;
        cy = cy + (vj.y - vi.y) * f;
        cz = cz + (vj.z - vi.z) * f;
    });
    dv[i] = make_double4(cx * k.xsph_eps, cy * k.xsph_eps, cz * k.xsph_eps, 0.0);
}

__global__ void k_df_xsph_apply(uint32_t n, StateBufs s, const double4* __restrict__ dv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || is_boundary(s, i)) return;
    double4 a = s.acc[i];
    const double4 d = dv[i];
    a.x = a.x + d.x;
    a.y = a.y + d.y;
    a.z = a.z + d.z;
    s.acc[i] = a;
}

// kappa = the warm-start accumulator (which 0: density, acc.w; 1: divergence, nout.w)
__global__ void k_df_warm_load(uint32_t n, DfsphConst k, int which, StateBufs s, double* __restrict__ kappa,
                               double* __restrict__ kr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double kap = which ? s.nout[i].w : s.acc[i].w;
    kappa[i] = kap;
    kr[i] = is_boundary(s, i) ? 0.0 / k.rho0 : kap / fmax(s.vel[i].w, 1e-12);
}

__global__ void k_df_warm_zero(uint32_t n, int which, StateBufs s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (which) s.nout[i].w = 0.0;
    else s.acc[i].w = 0.0;
}

// dfsph.rs:326-351 density_derivative with v*
__device__ __forceinline__ double density_rate(const DfsphConst& k, const StateBufs& s, const ListBufs& l,
                                               uint32_t i) {
    const double4 xi = s.pos[i], vi = s.acc[i];
    double drho = 0.0;
    for_each_loaded(
        list_ref(l, i, kListVisit), [&](uint32_t e) { return s.pos[e & kEntrySlotMask]; },
        [&](uint32_t e, const double4& xj) {
            if (far_pair(k, xi, xj)) return;
            const double mj = nmass(k, s, e, xj, xi);
            if (mj == 0.0) return;
            const uint32_t j = e & kEntrySlotMask;
            double gx, gy, gz;
            kfn_grad(k.kf, xj.x - xi.x, xj.y - xi.y, xj.z - xi.z, &gx, &gy, &gz);
            const double4 vj = (e & kEntryBoundary) ? s.vel[j] : s.acc[j];
            const double wx = vi.x - vj.x, wy = vi.y - vj.y, wz = vi.z - vj.z;
            drho += mj * (wx * gx + wy * gy + wz * gz);
        });
    return drho;
}

// One error pass of a solver (dfsph.rs:552-569 density, 604-616 divergence):
// kappa, the warm-start accumulation, the pressure diagnostic and the error
// term of each particle in original order.
__global__ void __launch_bounds__(kDfThreads) k_df_error(uint32_t n, DfsphConst k, int divergence, double dt,
                                                        double dt2, StateBufs s, ListBufs l,
                                                        const double* __restrict__ alpha, double* __restrict__ kappa,
                                                        double* __restrict__ kr, double* __restrict__ err_orig) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t o = s.orig[i];
    if (is_boundary(s, i)) {
        kappa[i] = 0.0;
        kr[i] = 0.0 / k.rho0;  // dfsph.rs:462-469: kj = 0, rho_j = rho0
        err_orig[o] = 0.0;
        return;
    }
    const double drho = density_rate(k, s, l, i);
    double kap, e;
    if (!divergence) {
        const double rho_star = s.vel[i].w + dt * drho;
        const double err = fmax(rho_star - k.rho0, 0.0);
        e = err / k.rho0;
        kap = k.omega * err / dt2 * alpha[i];
        s.p[i] = kap;  // dfsph.rs:761 p = kappa after the step
        if (k.warm_start) s.acc[i].w = s.acc[i].w + kap;
    } else {
        const double d = fmax(drho, 0.0);
        e = d / k.rho0;
        kap = k.omega * (1.0 / dt) * d * alpha[i];
        if (k.warm_start) s.nout[i].w = s.nout[i].w + kap;
    }
    kappa[i] = kap;
    // dfsph.rs:436, 470: kappa / max(rho, 1e-12), the same quotient the
    // reference forms for every pair, formed once
    kr[i] = kap / fmax(s.vel[i].w, 1e-12);
    err_orig[o] = e;
}

// Partial sums of v (any order: only bounds are taken from them).
constexpr uint32_t kSumBlocks = 148, kSumThreads = 256;

__global__ void __launch_bounds__(kSumThreads) k_df_partial_sums(uint32_t n, const double* __restrict__ v,
                                                                double* __restrict__ part) {
    __shared__ double red[kSumThreads];
    double s = 0.0;
    for (uint32_t i = blockIdx.x * kSumThreads + threadIdx.x; i < n; i += kSumBlocks * kSumThreads) s += v[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (uint32_t o = kSumThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(kSumThreads) k_df_final_sum(const double* __restrict__ part,
                                                             double* __restrict__ out) {
    __shared__ double red[kSumThreads];
    red[threadIdx.x] = threadIdx.x < kSumBlocks ? part[threadIdx.x] : 0.0;
    __syncthreads();
    for (uint32_t o = kSumThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// Sequential sum in original index order (the reference's accumulation order).
__global__ void k_df_serial_sum(uint32_t n, const double* __restrict__ v, double* __restrict__ out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double s = 0.0;
    for (uint32_t i = 0; i < n; ++i) s += v[i];
    *out = s;
}

// dfsph.rs:422-530, fluid side: dv from kappa, the cap, the reaction total and
// weight sum, v* += dv.
__global__ void __launch_bounds__(kDfThreads) k_df_pressure_fluid(uint32_t n, DfsphConst k, double dt,
                                                                 double inv_dt, StateBufs s, ListBufs l,
                                                                 const double* __restrict__ kr,
                                                                 double4* __restrict__ react) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (is_boundary(s, i)) return;
    const double4 xi = s.pos[i];
    const double kri = kr[i];  // ki / rho_i
    double dx = 0.0, dy = 0.0, dz = 0.0, bx = 0.0, by = 0.0, bz = 0.0;
    const ListRef lr = list_ref(l, i, kListVisit);
    for_each_loaded(
        lr, [&](uint32_t e) { return s.pos[e & kEntrySlotMask]; },
        [&](uint32_t e, const double4& xj) {
            if (far_pair(k, xi, xj)) return;
            const double mj = nmass(k, s, e, xj, xi);
            if (mj == 0.0) return;
            const uint32_t j = e & kEntrySlotMask;
            double gx, gy, gz;
            kfn_grad(k.kf, xj.x - xi.x, xj.y - xi.y, xj.z - xi.z, &gx, &gy, &gz);
            const bool bnd = e & kEntryBoundary;
            const double coeff = mj * (kri + kr[j]);  // mj (ki / rho_i + kj / rho_j)
            const double tx = gx * coeff, ty = gy * coeff, tz = gz * coeff;
            dx = dx + tx;
            dy = dy + ty;
            dz = dz + tz;
            if (bnd) {
                bx = bx + tx;
                by = by + ty;
                bz = bz + tz;
            }
        });
    dx = dx * (-dt);
    dy = dy * (-dt);
    dz = dz * (-dt);
    bx = bx * (-dt);
    by = by * (-dt);
    bz = bz * (-dt);
    double scale = 1.0;
    if (k.dv_cap > 0.0) {
        const double s2 = dx * dx + dy * dy + dz * dz;
        if (s2 > k.dv_cap * k.dv_cap) {
            scale = k.dv_cap / sqrt(s2);
            dx = dx * scale;
            dy = dy * scale;
            dz = dz * scale;
        }
    }
    bx = bx * scale;
    by = by * scale;
    bz = bz * scale;
    double4 rec = make_double4(0.0, 0.0, 0.0, 0.0);
    if (bx * bx + by * by + bz * bz > 0.0) {
        double wsum = 0.0;
        for_each_entry(lr, [&](uint32_t e) {
            if (!(e & kEntryBoundary)) return;
            const uint32_t j = e & kEntrySlotMask;
            const double4 xj = s.pos[j];
            const bool oriented = e & kEntryOriented;
            if (!sees(k, xj, oriented ? s.nout[j] : make_double4(0, 0, 0, 0), oriented, xi)) return;
            const double rx = xj.x - xi.x, ry = xj.y - xi.y, rz = xj.z - xi.z;
            const double r = sqrt(rx * rx + ry * ry + rz * rz);
            wsum += fmin(1.0 / fmax(r, 1e-9), 1e6);
        });
        if (wsum > 0.0) {
            const double m = -k.mass * inv_dt;
            rec = make_double4(bx * m, by * m, bz * m, wsum);
        }
    }
    react[i] = rec;
    double4 a = s.acc[i];
    a.x = a.x + dx;
    a.y = a.y + dy;
    a.z = k.dim == 2 ? 0.0 : a.z + dz;
    s.acc[i] = a;
}

// dfsph.rs:508-517, boundary side: the reaction shares of the fluid
// candidates, in ascending original index.
__global__ void __launch_bounds__(kDfThreads) k_df_pressure_boundary(uint32_t n, DfsphConst k, StateBufs s,
                                                                    ListBufs l, const double4* __restrict__ react) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || !is_boundary(s, j)) return;
    const double4 xj = s.pos[j];
    const bool oriented = s.flags[j] & kFlagOriented;
    const double4 nj = oriented ? s.nout[j] : make_double4(0, 0, 0, 0);
    double4 f = s.bf[j];
    for_each_entry(list_ref(l, j, kListLower), [&](uint32_t e) {
        const uint32_t i = e & kEntrySlotMask;
        const double4 rec = react[i];
        if (!(rec.w > 0.0)) return;
        const double4 xi = s.pos[i];
        if (!sees(k, xj, nj, oriented, xi)) return;
        const double rx = xj.x - xi.x, ry = xj.y - xi.y, rz = xj.z - xi.z;
        const double r = sqrt(rx * rx + ry * ry + rz * rz);
        const double wt = fmin(1.0 / fmax(r, 1e-9), 1e6);
        const double sh = wt / rec.w;
        f.x = f.x + rec.x * sh;
        f.y = f.y + rec.y * sh;
        f.z = f.z + rec.z * sh;
    });
    s.bf[j] = f;
}

// dfsph.rs:742-748 x += v* dt (fluid; 2-D: z = 0)
__global__ void k_df_advect(uint32_t n, int dim, double dt, StateBufs s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || is_boundary(s, i)) return;
    double4 p = s.pos[i];
    const double4 a = s.acc[i];
    p.x = p.x + a.x * dt;
    p.y = p.y + a.y * dt;
    p.z = dim == 2 ? 0.0 : p.z + a.z * dt;
    s.pos[i] = p;
}

// dfsph.rs:668-715
__global__ void k_df_free_slip(uint32_t n, DfsphConst k, StateBufs s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || is_boundary(s, i)) return;
    double4 x = s.pos[i], v = s.acc[i];
    if (k.has_slip[0] && x.x < k.slip[0]) {
        x.x = k.slip[0];
        if (v.x < 0.0) v.x = 0.0;
    }
    if (k.has_slip[1] && x.y < k.slip[1]) {
        x.y = k.slip[1];
        if (v.y < 0.0) v.y = 0.0;
    }
    if (k.has_slip[2] && x.x > k.slip[2]) {
        x.x = k.slip[2];
        if (v.x > 0.0) v.x = 0.0;
    }
    if (k.has_slip[3] && x.y > k.slip[3]) {
        x.y = k.slip[3];
        if (v.y > 0.0) v.y = 0.0;
    }
    s.pos[i] = x;
    s.acc[i] = v;
}

// dfsph.rs:214-244 density with the oriented-boundary filter
__global__ void __launch_bounds__(kDfThreads) k_df_density(uint32_t n, DfsphConst k, StateBufs s, ListBufs l) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (is_boundary(s, i)) {
        s.vel[i].w = k.rho0;
        return;
    }
    const double4 xi = s.pos[i];
    double rho = k.rho_self;
    for_each_loaded(
        list_ref(l, i, kListVisit), [&](uint32_t e) { return s.pos[e & kEntrySlotMask]; },
        [&](uint32_t e, const double4& xj) {
            if (far_pair(k, xi, xj)) return;
            const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            const double wij = kfn_w(k.kf, sqrt(dx * dx + dy * dy + dz * dz));
            if (!(e & kEntryBoundary)) {
                rho += k.mass * wij;
            } else {
                const uint32_t j = e & kEntrySlotMask;
                const bool oriented = e & kEntryOriented;
                if (sees(k, xj, oriented ? s.nout[j] : make_double4(0, 0, 0, 0), oriented, xi))
                    rho += k.rho0 * xj.w * wij;
            }
        });
    s.vel[i].w = fmax(rho, 1e-12);
}

// dfsph.rs:252-307 alpha = rho / max(|sum m grad W|^2 + sum |m grad W|^2, floor)
__global__ void __launch_bounds__(kDfThreads) k_df_alpha(uint32_t n, DfsphConst k, StateBufs s, ListBufs l,
                                                        double* __restrict__ alpha) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (is_boundary(s, i)) {
        alpha[i] = 0.0;
        return;
    }
    const double4 xi = s.pos[i];
    double sx = 0.0, sy = 0.0, sz = 0.0, sq = 0.0;
    uint32_t nb_all = 0, nb_kept = 0;
    for_each_loaded(
        list_ref(l, i, kListVisit), [&](uint32_t e) { return s.pos[e & kEntrySlotMask]; },
        [&](uint32_t e, const double4& xj) {
            const double mj = nmass(k, s, e, xj, xi);
            if (e & kEntryBoundary) {
                ++nb_all;
                if (mj == 0.0) return;
                ++nb_kept;
            }
            if (far_pair(k, xi, xj)) return;
            double gx, gy, gz;
            kfn_grad(k.kf, xj.x - xi.x, xj.y - xi.y, xj.z - xi.z, &gx, &gy, &gz);
            const double ax = gx * mj, ay = gy * mj, az = gz * mj;
            sx = sx + ax;
            sy = sy + ay;
            sz = sz + az;
            sq += ax * ax + ay * ay + az * az;
        });
    // every fluid candidate but i itself, and the boundary ones of non-zero mass
    const uint32_t nn = (l.ncand[i] - 1u - nb_all) + nb_kept;
    if (nn < 2) {
        alpha[i] = 0.0;
        return;
    }
    const double denom = fmax(sx * sx + sy * sy + sz * sz + sq, k.denom_floor);
    alpha[i] = s.vel[i].w / denom;
}

// dfsph.rs:755-765 v = v* (2-D: z = 0)
__global__ void k_df_finish(uint32_t n, int dim, StateBufs s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || is_boundary(s, i)) return;
    double4 v = s.vel[i];
    const double4 a = s.acc[i];
    v.x = a.x;
    v.y = a.y;
    v.z = dim == 2 ? 0.0 : a.z;
    s.vel[i] = v;
}

__global__ void k_df_export_orig(uint32_t n, const uint32_t* __restrict__ orig, const double* __restrict__ src,
                                 double* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[orig[i]] = src[i];
}

}  // namespace

DfsphSolver::DfsphSolver(const DfsphParams& prm, const WorldConfig& cfg, int dim, double rest_density, double mass,
                         double h, uint64_t n, const double* x, const double* v, const uint8_t* kind,
                         const double* psi, const double* n_out)
    : prm_(prm) {
    // dfsph.rs:139-152: diameter defaults to h; 2-D particles are planar
    if (prm_.particle_diameter <= 0.0) prm_.particle_diameter = h;
    std::vector<double> xs(x, x + 3 * n), vs;
    if (v) vs.assign(v, v + 3 * n);
    else vs.assign(3 * n, 0.0);
    if (dim == 2)
        for (uint64_t i = 0; i < n; ++i) {
            xs[3 * i + 2] = 0.0;
            vs[3 * i + 2] = 0.0;
        }
    for (uint64_t i = 0; i < n; ++i) n_fluid_ += kind[i] == 0;
    WorldParams wp{};
    wp.kernel = 0;
    wp.eos_rest_density = rest_density;
    wp.eos_sound_speed = 1.0;
    wp.eos_gamma = 7.0;
    for (int a = 0; a < 3; ++a) wp.gravity[a] = prm.gravity[a];
    WorldConfig wc = cfg;
    wc.precision = 0;
    wc.use_graph = 0;
    w_.reset(new World(wp, wc, dim, rest_density, mass, h, n, xs.data(), vs.data(), kind, psi, n_out, nullptr, 1,
                       kernel_support(prm.kernel, h)));
    w_->list_keep_boundary_ = true;
    w_->refresh_step_const();
    const size_t N = std::max<uint64_t>(n, 1);
    alpha_ = w_->alloc<double>(N);
    kappa_ = w_->alloc<double>(N);
    kr_ = w_->alloc<double>(N);
    dv_ = w_->alloc<double4>(N);
    react_ = w_->alloc<double4>(N);
    err_orig_ = w_->alloc<double>(N);
    sum_ = w_->alloc<double>(1);
    part_ = w_->alloc<double>(kSumBlocks);
    w_->check(cudaMallocHost(&sum_host_, sizeof(double)), "pinned");
    refresh_const();
    // dfsph.rs:177-179
    rebuild();
    density_and_alpha();
    w_->check(cudaStreamSynchronize(w_->st_), "dfsph init");
}

DfsphSolver::~DfsphSolver() {
    if (sum_host_) cudaFreeHost(sum_host_);
}

void DfsphSolver::rebuild_neighbours() { rebuild(); }

void DfsphSolver::compute_density() {
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    if (!n) return;
    k_df_density<<<blocks_for(n, kDfThreads), kDfThreads, 0, w.st_>>>(n, kc_, w.cur_, w.lists_);
    w.launches_ += 1;
}

void DfsphSolver::compute_alpha() {
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    if (!n) return;
    k_df_alpha<<<blocks_for(n, kDfThreads), kDfThreads, 0, w.st_>>>(n, kc_, w.cur_, w.lists_, alpha_);
    w.launches_ += 1;
}

double DfsphSolver::mean_density_error() {
    World& w = *w_;
    const uint64_t n = w.n_;
    std::vector<double> rho(n);
    std::vector<uint8_t> kind(n);
    if (n) {
        w.get_scalar(0, rho.data());
        w.get_kind(kind.data());
    }
    double s = 0.0;
    uint64_t c = 0;
    for (uint64_t i = 0; i < n; ++i)
        if (kind[i] == 0) {
            s += std::fabs(rho[i] - w.rho0_) / w.rho0_;
            c += 1;
        }
    return c == 0 ? 0.0 : s / (double)c;
}

double DfsphSolver::v_max() {
    World& w = *w_;
    const uint64_t n = w.n_;
    std::vector<double> v(3 * n);
    std::vector<uint8_t> kind(n);
    if (n) {
        w.get_vec(1, v.data());
        w.get_kind(kind.data());
    }
    double m = 0.0;
    for (uint64_t i = 0; i < n; ++i)
        if (kind[i] == 0) m = std::fmax(m, v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
    return std::sqrt(m);
}

void DfsphSolver::set_params(const DfsphParams& p) {
    if (kernel_support(p.kernel, w_->h_) != kernel_support(prm_.kernel, w_->h_))
        throw std::invalid_argument("the support radius is fixed at creation");
    prm_ = p;
    if (prm_.particle_diameter <= 0.0) prm_.particle_diameter = w_->h_;
    refresh_const();
}

void DfsphSolver::refresh_const() {
    DfsphConst& k = kc_;
    const World& w = *w_;
    k.dim = w.dim_;
    k.kf = make_kernel_fn(prm_.kernel, w.h_, w.dim_);
    k.mass = w.mass_;
    k.rho0 = w.rho0_;
    // dfsph.rs:225 rho = mass * w(kern, 0.0, h, dim)
    double w0;
    switch (prm_.kernel) {
        case kCubic: w0 = k.kf.alpha * (1.0 - 1.5 * 0.0 * 0.0 + 0.75 * 0.0 * 0.0 * 0.0); break;
        case kWendland: w0 = k.kf.alpha * 1.0 * 1.0 * 1.0 * 1.0 * (2.0 * 0.0 + 1.0); break;
        case kPoly6: {
            const double t = w.h_ * w.h_ - 0.0 * 0.0;
            w0 = k.kf.alpha * t * t * t;
            break;
        }
        default: {
            const double t = w.h_ - 0.0;
            w0 = k.kf.alpha * t * t * t;
            break;
        }
    }
    k.rho_self = k.mass * w0;
    k.eps_h = 0.15 * w.h_;
    // dfsph.rs:260-267
    const double h_safe = std::fmax(w.h_, 1e-12);
    const double char_grad = w.dim_ == 2 ? k.mass / (h_safe * h_safe * h_safe)
                                         : k.mass / (h_safe * h_safe * h_safe * h_safe);
    k.denom_floor = std::fmax(1e-6 * char_grad * char_grad, 1e-12);
    k.xsph_eps = prm_.xsph_epsilon;
    k.gx = prm_.gravity[0];
    k.gy = prm_.gravity[1];
    k.gz = prm_.gravity[2];
    k.omega = prm_.solver_omega;
    k.dv_cap = prm_.max_velocity_correction;
    k.warm_start = prm_.warm_start;
    {
        const double far = kernel_support(prm_.kernel, w.h_) * (1.0 + 1e-9);
        k.far2 = far * far;
    }
    for (int a = 0; a < 4; ++a) {
        k.has_slip[a] = prm_.has_slip[a];
        k.slip[a] = prm_.slip[a];
    }
}

void DfsphSolver::rebuild() {
    World& w = *w_;
    w.build_grid(nullptr, nullptr);
    w.ensure_lists(false);  // visit lists (fluid) and ascending fluid lists (boundary)
}

void DfsphSolver::density_and_alpha() {
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    if (!n) return;
    const uint32_t nb = blocks_for(n, kDfThreads);
    k_df_density<<<nb, kDfThreads, 0, w.st_>>>(n, kc_, w.cur_, w.lists_);
    k_df_alpha<<<nb, kDfThreads, 0, w.st_>>>(n, kc_, w.cur_, w.lists_, alpha_);
    w.launches_ += 2;
}

void DfsphSolver::pressure_update(double dt, bool /*divergence*/) {
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    const uint32_t nb = blocks_for(n, kDfThreads);
    const double inv_dt = 1.0 / std::fmax(dt, 1e-12);
    k_df_pressure_fluid<<<nb, kDfThreads, 0, w.st_>>>(n, kc_, dt, inv_dt, w.cur_, w.lists_, kr_, react_);
    k_df_pressure_boundary<<<nb, kDfThreads, 0, w.st_>>>(n, kc_, w.cur_, w.lists_, react_);
    w.launches_ += 2;
}

double DfsphSolver::solve_error(double dt, bool divergence) {
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    const uint32_t nb = blocks_for(n, kDfThreads);
    k_df_error<<<nb, kDfThreads, 0, w.st_>>>(n, kc_, divergence ? 1 : 0, dt, dt * dt, w.cur_, w.lists_, alpha_,
                                             kappa_, kr_, err_orig_);
    k_df_partial_sums<<<kSumBlocks, kSumThreads, 0, w.st_>>>(n, err_orig_, part_);
    k_df_final_sum<<<1, kSumThreads, 0, w.st_>>>(part_, sum_);
    w.launches_ += 3;
    // the sequential sum's terms are kept until the decision is known: the
    // pressure update does not touch them
    pressure_update(dt, divergence);
    w.check(cudaMemcpyAsync(sum_host_, sum_, sizeof(double), cudaMemcpyDeviceToHost, w.st_), "dfsph error");
    w.check(cudaStreamSynchronize(w.st_), "dfsph error");
    const double tol = divergence ? prm_.divergence_error_tol : prm_.density_error_tol;
    const double cnt = n_fluid_ > 0 ? (double)n_fluid_ : 1.0;
    const double S = *sum_host_;
    const double u = std::ldexp(1.0, -53);
    const double nm1 = n > 1 ? (double)(n - 1) : 0.0;
    const double gam = nm1 * u / (1.0 - nm1 * u);
    // generous outward margin for the bracket's own roundings
    const double delta = (2.0 * gam / (1.0 - gam)) * S * (1.0 + 1e-6) + 4.0 * std::numeric_limits<double>::denorm_min();
    const double hi = (S + delta) / cnt, lo = std::fmax(S - delta, 0.0) / cnt;
    if (std::isfinite(S) && hi <= tol) return S / cnt;            // the sequential average is <= tol too
    if (std::isfinite(S) && lo > tol && lo == lo) return S / cnt;  // and > tol here
    // within the bracket's width of the tolerance (or non-finite): the sequential sum decides
    k_df_serial_sum<<<1, 32, 0, w.st_>>>(n, err_orig_, sum_);
    w.launches_ += 1;
    w.check(cudaMemcpyAsync(sum_host_, sum_, sizeof(double), cudaMemcpyDeviceToHost, w.st_), "dfsph error");
    w.check(cudaStreamSynchronize(w.st_), "dfsph error");
    ++serial_sums_;
    double avg = *sum_host_;
    if (n_fluid_ > 0) avg /= (double)n_fluid_;
    return avg;
}

uint64_t DfsphSolver::correct_density_error(double dt) {
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    const uint32_t nb = blocks_for(n, kDfThreads);
    if (prm_.warm_start) {
        k_df_warm_load<<<nb, kDfThreads, 0, w.st_>>>(n, kc_, 0, w.cur_, kappa_, kr_);
        w.launches_ += 1;
        pressure_update(dt, false);
    }
    k_df_warm_zero<<<nb, kDfThreads, 0, w.st_>>>(n, 0, w.cur_);
    w.launches_ += 1;
    uint64_t iters = 0;
    for (;;) {
        const double avg = solve_error(dt, false);
        iters += 1;
        err_density_ = avg;
        if ((avg <= prm_.density_error_tol && iters >= 2) || iters >= prm_.max_density_iters) break;
    }
    return iters;
}

uint64_t DfsphSolver::correct_divergence_error(double dt) {
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    const uint32_t nb = blocks_for(n, kDfThreads);
    if (prm_.warm_start) {
        k_df_warm_load<<<nb, kDfThreads, 0, w.st_>>>(n, kc_, 1, w.cur_, kappa_, kr_);
        w.launches_ += 1;
        pressure_update(dt, true);
    }
    k_df_warm_zero<<<nb, kDfThreads, 0, w.st_>>>(n, 1, w.cur_);
    w.launches_ += 1;
    uint64_t iters = 0;
    for (;;) {
        const double avg = solve_error(dt, true);
        iters += 1;
        err_divergence_ = avg;
        if ((avg <= prm_.divergence_error_tol && iters >= 1) || iters >= prm_.max_divergence_iters) break;
    }
    return iters;
}

void DfsphSolver::free_slip() {
    if (!prm_.has_slip[0] && !prm_.has_slip[1] && !prm_.has_slip[2] && !prm_.has_slip[3]) return;
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    k_df_free_slip<<<blocks_for(n, kDfThreads), kDfThreads, 0, w.st_>>>(n, kc_, w.cur_);
    w.launches_ += 1;
}

void DfsphSolver::step(double dt_in) {
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    const double dt = std::fmax(dt_in, 1e-12);
    last_dt_ = dt;
    if (n == 0) {
        w.t_ += dt;
        return;
    }
    const uint32_t nb = blocks_for(n, kDfThreads);
    cudaStream_t st = w.st_;
    k_df_begin<<<nb, kDfThreads, 0, st>>>(n, kc_, dt, w.cur_);
    w.launches_ += 1;
    if (prm_.xsph_epsilon != 0.0) {
        k_df_xsph<<<nb, kDfThreads, 0, st>>>(n, kc_, w.cur_, w.lists_, dv_);
        k_df_xsph_apply<<<nb, kDfThreads, 0, st>>>(n, w.cur_, dv_);
        w.launches_ += 2;
    }
    it_density_ = correct_density_error(dt);
    k_df_advect<<<nb, kDfThreads, 0, st>>>(n, w.dim_, dt, w.cur_);
    w.launches_ += 1;
    free_slip();
    rebuild();
    density_and_alpha();
    it_divergence_ = correct_divergence_error(dt);
    free_slip();
    k_df_finish<<<nb, kDfThreads, 0, st>>>(n, w.dim_, w.cur_);
    w.launches_ += 1;
    w.check(cudaGetLastError(), "dfsph step");
    w.t_ += dt;
    a_adv_set_ = true;
}

double DfsphSolver::suggest_dt() {
    World& w = *w_;
    const uint64_t n = w.n_;
    std::vector<double> v(3 * n);
    std::vector<uint8_t> kind(n);
    if (n) {
        w.get_vec(1, v.data());
        w.get_kind(kind.data());
    }
    const double g2 = prm_.gravity[0] * prm_.gravity[0] + prm_.gravity[1] * prm_.gravity[1] +
                      prm_.gravity[2] * prm_.gravity[2];
    double vmax = 0.0, amax = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
        if (kind[i] != 0) continue;
        vmax = std::fmax(vmax, v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
        amax = std::fmax(amax, a_adv_set_ ? g2 : 0.0);
    }
    vmax = std::sqrt(vmax);
    amax = std::sqrt(amax);
    const double d = std::fmax(prm_.particle_diameter, 1e-12);
    const double dt_v = prm_.cfl_lambda * d / std::fmax(vmax, 1e-6);
    // cfl.rs:36 suggested_dt(h, 0, vmax, max(amax, 1e-6), {cfl_lambda, 0.25})
    const double am = std::fmax(amax, 1e-6);
    const double dv2 = prm_.cfl_lambda * w.h_ / std::fmax(0.0 + vmax, 1e-12);
    const double df2 = am > 1e-12 ? 0.25 * std::sqrt(w.h_ / am) : std::numeric_limits<double>::infinity();
    const double dt_f = std::fmin(dv2, df2);
    const double r = std::fmin(dt_v, dt_f);
    return r < 1e-6 ? 1e-6 : (r > 1e-2 ? 1e-2 : r);
}

double DfsphSolver::step_adaptive() {
    a_adv_set_ = true;  // dfsph.rs:774 compute_nonpressure_accel
    const double dt = prm_.adaptive_dt ? suggest_dt() : std::fmax(last_dt_, 1e-4);
    step(dt);
    return dt;
}

void DfsphSolver::run(double dt, uint64_t steps) {
    for (uint64_t s = 0; s < steps; ++s) {
        step(dt);
        if ((s + 1) % 16 == 0) w_->status();
    }
}

void DfsphSolver::get_alpha(double* out) {
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    if (!n) return;
    k_df_export_orig<<<blocks_for(n, 256), 256, 0, w.st_>>>(n, w.cur_.orig, alpha_, err_orig_);
    w.check(cudaMemcpyAsync(out, err_orig_, sizeof(double) * n, cudaMemcpyDeviceToHost, w.st_), "alpha");
    w.check(cudaStreamSynchronize(w.st_), "alpha");
}

}  // namespace pe
