// Position Based Fluids (crates/pe-fluid/src/pbf.rs) on the cell-sorted state
// of a World whose grid cell is the PBF support radius.
//
// Slot state during a step: pos = predicted position (the grid is built on
// it, pbf.rs:146-156), acc = the position at the start of the step (kept
// through the re-sort so v = (pred - x) / dt can be formed, pbf.rs:413-421),
// vel = (v, rho). Every pass is a gather over the slot's visit list in the
// reference's visiting order, so each per-particle sum is the reference's
// sequence of additions; candidates outside the support add +-0 and are left
// out of the lists. Compiled with --fmad=false.
#include <algorithm>
#include <cmath>

#include "list_iter.cuh"
#include "pbf.cuh"

namespace pe {

namespace {

constexpr uint32_t kPbfThreads = 128;
constexpr size_t kKeepBytes = (size_t)kKeepChunk * kPbfThreads * sizeof(uint32_t);  // for_each_kept buffer

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

struct D3 {
    double x, y, z;
};

__device__ __forceinline__ double4 load_pos(const StateBufs& s, uint32_t e) {
    return s.pos[e & kEntrySlotMask];
}

// A candidate beyond both kernels' support contributes an exact +-0 to every
// sum (W and grad W vanish there), which leaves the sums unchanged: it is
// skipped. The margin on far2 keeps the test conservative under rounding.
__device__ __forceinline__ bool far_pair(const PbfConst& k, const double4& xi, const double4& xj) {
    const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    return dx * dx + dy * dy + dz * dz > k.far2;
}

// pbf.rs:387-399: fluid v += g dt, pred = x + v dt (2-D: z = 0); the start
// position goes to acc, the prediction to pred (the grid build's next positions).
__global__ void k_pbf_predict(uint32_t n, PbfConst k, double dt, StateBufs s, double4* __restrict__ pred) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = s.pos[i];
    if (s.flags[i] & kFlagBoundary) {
        pred[i] = p;
        return;
    }
    const double4 v0 = s.vel[i];
    const double gx = k.gx * dt, gy = k.gy * dt, gz = k.gz * dt;
    double vx = v0.x + gx, vy = v0.y + gy, vz = v0.z + gz;
    double px = p.x + vx * dt, py = p.y + vy * dt, pz = p.z + vz * dt;
    if (k.dim == 2) {
        pz = 0.0;
        vz = 0.0;
    }
    s.vel[i] = make_double4(vx, vy, vz, v0.w);
    s.acc[i] = make_double4(p.x, p.y, p.z, 0.0);
    pred[i] = make_double4(px, py, pz, p.w);
}

// pbf.rs:159-187 density at the predicted positions into vel.w
__global__ void __launch_bounds__(kPbfThreads) k_pbf_density(uint32_t n, PbfConst k, StateBufs s, ListBufs l) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.flags[i] & kFlagBoundary) {
        s.vel[i].w = k.rho0;
        return;
    }
    extern __shared__ uint32_t s_keep[];
    const double4 xi = s.pos[i];
    double rho = k.rho_self;
    for_each_kept(
        list_ref(l, i, kListVisit), s_keep, [&](uint32_t e) { return load_pos(s, e); },
        [&](uint32_t, const double4& xj) { return !far_pair(k, xi, xj); },
        [&](uint32_t e, const double4& xj) {
            const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const double wij = kfn_w(k.dk, r);
            if (e & kEntryBoundary) rho += k.rho0 * xj.w * wij;
            else rho += k.mass * wij;
        });
    s.vel[i].w = fmax(rho, 1e-12);
}

// pbf.rs:189-227 lambda_i = -C_i / (sum |grad C|^2 + eps)
__global__ void __launch_bounds__(kPbfThreads) k_pbf_lambda(uint32_t n, PbfConst k, StateBufs s, ListBufs l,
                                                           double* __restrict__ lambda,
                                                           double* __restrict__ lambda_orig) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.flags[i] & kFlagBoundary) {
        lambda[i] = 0.0;
        lambda_orig[s.orig[i]] = 0.0;
        return;
    }
    const double4 xi = s.pos[i];
    const double ci = s.vel[i].w / k.rho0 - 1.0;
    double sum_grad_sq = 0.0;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    extern __shared__ uint32_t s_keep[];
    for_each_kept(
        list_ref(l, i, kListVisit), s_keep, [&](uint32_t e) { return load_pos(s, e); },
        [&](uint32_t, const double4& xj) { return !far_pair(k, xi, xj); },
        [&](uint32_t e, const double4& xj) {
            double wx, wy, wz;
            kfn_grad(k.gk, xj.x - xi.x, xj.y - xi.y, xj.z - xi.z, &wx, &wy, &wz);
            const bool fluid = !(e & kEntryBoundary);
            const double scale = fluid ? k.mass_over_rho0 : xj.w;
            const double cx = wx * scale, cy = wy * scale, cz = wz * scale;
            gx = gx + cx;
            gy = gy + cy;
            gz = gz + cz;
            if (fluid) sum_grad_sq += cx * cx + cy * cy + cz * cz;
        });
    sum_grad_sq += gx * gx + gy * gy + gz * gz;
    const double li = -ci / (sum_grad_sq + k.eps_lambda);
    lambda[i] = li;
    lambda_orig[s.orig[i]] = li;
}

// pbf.rs:229-235
__device__ __forceinline__ double art_pressure(const PbfConst& k, double wij) {
    if (k.w_dq <= 1e-30 || k.art_k == 0.0) return 0.0;
    const double ratio = fmin(wij / k.w_dq, 1.0);
    const double pw = k.art_n_is_int ? pow_int_dd(ratio, k.art_n_int) : pow(ratio, k.art_n);
    return -k.art_k * pw;
}

// pbf.rs:237-286 position correction, clamped to 0.4 h
__global__ void __launch_bounds__(kPbfThreads) k_pbf_delta_p(uint32_t n, PbfConst k, StateBufs s, ListBufs l,
                                                            const double* __restrict__ lambda,
                                                            double4* __restrict__ dp) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.flags[i] & kFlagBoundary) {
        dp[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        return;
    }
    const double4 xi = s.pos[i];
    const double li = lambda[i];
    double cx = 0.0, cy = 0.0, cz = 0.0;
    extern __shared__ uint32_t s_keep[];
    for_each_kept(
        list_ref(l, i, kListVisit), s_keep, [&](uint32_t e) { return load_pos(s, e); },
        [&](uint32_t, const double4& xj) { return !far_pair(k, xi, xj); },
        [&](uint32_t e, const double4& xj) {
            const double rx = xj.x - xi.x, ry = xj.y - xi.y, rz = xj.z - xi.z;
            const double r = sqrt(rx * rx + ry * ry + rz * rz);
            const double wij = kfn_w(k.dk, r);
            double wx, wy, wz;
            kfn_grad(k.gk, rx, ry, rz, &wx, &wy, &wz);
            const double s_corr = art_pressure(k, wij);
            double f;
            if (e & kEntryBoundary) {
                const double coeff = li + s_corr;
                f = xj.w * coeff;
            } else {
                const double coeff = li + lambda[e & kEntrySlotMask] + s_corr;
                f = k.mass_over_rho0 * coeff;
            }
            cx = cx + wx * f;
            cy = cy + wy * f;
            cz = cz + wz * f;
        });
    const double mag = sqrt(cx * cx + cy * cy + cz * cz);
    if (mag > k.max_corr && mag > 0.0) {
        const double sc = k.max_corr / mag;
        cx = cx * sc;
        cy = cy * sc;
        cz = cz * sc;
    }
    dp[i] = make_double4(cx, cy, cz, 0.0);
}

// pbf.rs:403-409 pred += dp (fluid; 2-D: z = 0)
__global__ void k_pbf_apply_dp(uint32_t n, int dim, StateBufs s, const double4* __restrict__ dp) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (s.flags[i] & kFlagBoundary)) return;
    double4 p = s.pos[i];
    const double4 d = dp[i];
    p.x = p.x + d.x;
    p.y = p.y + d.y;
    p.z = dim == 2 ? 0.0 : p.z + d.z;
    s.pos[i] = p;
}

// pbf.rs:413-421 v = (pred - x) * (1 / dt) when dt > 0; x = pred (pos already is)
__global__ void k_pbf_finalize(uint32_t n, double dt, StateBufs s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (s.flags[i] & kFlagBoundary) || !(dt > 0.0)) return;
    const double4 p = s.pos[i], x0 = s.acc[i];
    const double inv = 1.0 / dt;
    double4 v = s.vel[i];
    v.x = (p.x - x0.x) * inv;
    v.y = (p.y - x0.y) * inv;
    v.z = (p.z - x0.z) * inv;
    s.vel[i] = v;
}

// pbf.rs:298-317 XSPH-style viscosity: dv_i = eps * sum_j (v_j - v_i) m / rho_bar W
__global__ void __launch_bounds__(kPbfThreads) k_pbf_viscosity(uint32_t n, PbfConst k, StateBufs s, ListBufs l,
                                                              double4* __restrict__ dv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.flags[i] & kFlagBoundary) {
        dv[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        return;
    }
    const double4 xi = s.pos[i], vi = s.vel[i];
    double cx = 0.0, cy = 0.0, cz = 0.0;
    for_each_entry(list_ref(l, i, kListVisit), [&](uint32_t e) {
        if (e & kEntryBoundary) return;
        const uint32_t j = e & kEntrySlotMask;
        const double4 xj = s.pos[j];
        if (far_pair(k, xi, xj)) return;
        const double4 vj = s.vel[j];
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double wij = kfn_w(k.dk, r);
        const double rho_bar = 0.5 * (vi.w + vj.w);
        const double f = k.mass / fmax(rho_bar, 1e-12) * wij;
        cx = cx + (vj.x - vi.x) * f;
        cy = cy + (vj.y - vi.y) * f;
        cz = cz + (vj.z - vi.z) * f;
    });
    dv[i] = make_double4(cx * k.visc_eps, cy * k.visc_eps, cz * k.visc_eps, 0.0);
}

// pbf.rs:318-320 v += dv for every particle
__global__ void k_pbf_add_dv(uint32_t n, StateBufs s, const double4* __restrict__ dv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 v = s.vel[i];
    const double4 d = dv[i];
    v.x = v.x + d.x;
    v.y = v.y + d.y;
    v.z = v.z + d.z;
    s.vel[i] = v;
}

// vec3.rs:87-93
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {
    return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// pbf.rs:330-349 vorticity omega_i = sum_j (v_j - v_i) x grad W m / rho_bar
__global__ void __launch_bounds__(kPbfThreads) k_pbf_omega(uint32_t n, PbfConst k, StateBufs s, ListBufs l,
                                                          double4* __restrict__ omega) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.flags[i] & kFlagBoundary) {
        omega[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        return;
    }
    const double4 xi = s.pos[i], vi = s.vel[i];
    D3 w{0.0, 0.0, 0.0};
    for_each_entry(list_ref(l, i, kListVisit), [&](uint32_t e) {
        if (e & kEntryBoundary) return;
        const uint32_t j = e & kEntrySlotMask;
        const double4 xj = s.pos[j];
        if (far_pair(k, xi, xj)) return;
        const double4 vj = s.vel[j];
        D3 g;
        kfn_grad(k.gk, xj.x - xi.x, xj.y - xi.y, xj.z - xi.z, &g.x, &g.y, &g.z);
        const double rho_bar = 0.5 * (vi.w + vj.w);
        const D3 c = cross3(D3{vj.x - vi.x, vj.y - vi.y, vj.z - vi.z}, g);
        const double f = k.mass / fmax(rho_bar, 1e-12);
        w = D3{w.x + c.x * f, w.y + c.y * f, w.z + c.z * f};
    });
    omega[i] = make_double4(w.x, w.y, w.z, 0.0);
}

// pbf.rs:350-379 confinement: v += (n_hat x omega_i) eps dt, n_hat = eta / |eta|
__global__ void __launch_bounds__(kPbfThreads) k_pbf_confine(uint32_t n, PbfConst k, double dt, StateBufs s,
                                                            ListBufs l, const double4* __restrict__ omega) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (s.flags[i] & kFlagBoundary)) return;
    const double4 xi = s.pos[i];
    const double rho_i = s.vel[i].w;
    const double4 oi = omega[i];
    const double om_i = sqrt(oi.x * oi.x + oi.y * oi.y + oi.z * oi.z);
    D3 eta{0.0, 0.0, 0.0};
    for_each_entry(list_ref(l, i, kListVisit), [&](uint32_t e) {
        if (e & kEntryBoundary) return;
        const uint32_t j = e & kEntrySlotMask;
        const double4 xj = s.pos[j];
        if (far_pair(k, xi, xj)) return;
        const double4 oj = omega[j];
        D3 g;
        kfn_grad(k.gk, xj.x - xi.x, xj.y - xi.y, xj.z - xi.z, &g.x, &g.y, &g.z);
        const double rho_bar = 0.5 * (rho_i + s.vel[j].w);
        const double f = k.mass / fmax(rho_bar, 1e-12) * (sqrt(oj.x * oj.x + oj.y * oj.y + oj.z * oj.z) - om_i);
        eta = D3{eta.x + g.x * f, eta.y + g.y * f, eta.z + g.z * f};
    });
    const double nrm = sqrt(eta.x * eta.x + eta.y * eta.y + eta.z * eta.z);
    if (nrm > 1e-12) {
        const D3 nh{eta.x / nrm, eta.y / nrm, eta.z / nrm};
        const D3 c = cross3(nh, D3{oi.x, oi.y, oi.z});
        const D3 f{c.x * k.vort_eps, c.y * k.vort_eps, c.z * k.vort_eps};
        double4 v = s.vel[i];
        v.x = v.x + f.x * dt;
        v.y = v.y + f.y * dt;
        v.z = v.z + f.z * dt;
        s.vel[i] = v;
    }
}

}  // namespace

PbfSolver::PbfSolver(const PbfParams& prm, const WorldConfig& cfg, int dim, double rest_density, double mass,
                     double h, uint64_t n, const double* x, const double* v, const uint8_t* kind,
                     const double* psi, const double* n_out)
    : prm_(prm) {
    WorldParams wp{};
    wp.kernel = 0;
    wp.eos_rest_density = rest_density;
    wp.eos_sound_speed = 1.0;
    wp.eos_gamma = 7.0;
    for (int a = 0; a < 3; ++a) wp.gravity[a] = prm.gravity[a];
    const double support = std::fmax(kernel_support(prm.density_kernel, h), kernel_support(prm.grad_kernel, h));
    WorldConfig wc = cfg;
    wc.precision = 0;
    wc.use_graph = 0;
    w_.reset(new World(wp, wc, dim, rest_density, mass, h, n, x, v, kind, psi, n_out, nullptr, 1, support));
    const size_t N = std::max<uint64_t>(n, 1);
    lambda_ = w_->alloc<double>(N);
    lambda_orig_ = w_->alloc<double>(N);
    dp_ = w_->alloc<double4>(N);
    omega_ = w_->alloc<double4>(N);
    refresh_const();
}

PbfSolver::~PbfSolver() = default;

void PbfSolver::set_params(const PbfParams& p) {
    const double h = w_->h_;
    const double s_old = std::fmax(kernel_support(prm_.density_kernel, h), kernel_support(prm_.grad_kernel, h));
    const double s_new = std::fmax(kernel_support(p.density_kernel, h), kernel_support(p.grad_kernel, h));
    if (s_old != s_new) throw std::invalid_argument("the support radius is fixed at creation");
    prm_ = p;
    refresh_const();
}

void PbfSolver::refresh_const() {
    PbfConst& k = kc_;
    const World& w = *w_;
    k.dim = w.dim_;
    k.dk = make_kernel_fn(prm_.density_kernel, w.h_, w.dim_);
    k.gk = make_kernel_fn(prm_.grad_kernel, w.h_, w.dim_);
    k.mass = w.mass_;
    k.rho0 = w.rho0_;
    // pbf.rs:171 rho = mass * w(kern, 0.0, h, dim): host evaluation of W(0)
    double w0;
    switch (prm_.density_kernel) {
        case kCubic: w0 = k.dk.alpha * (1.0 - 1.5 * 0.0 * 0.0 + 0.75 * 0.0 * 0.0 * 0.0); break;
        case kWendland: w0 = k.dk.alpha * 1.0 * 1.0 * 1.0 * 1.0 * (2.0 * 0.0 + 1.0); break;
        case kPoly6: {
            const double t = w.h_ * w.h_ - 0.0 * 0.0;
            w0 = k.dk.alpha * t * t * t;
            break;
        }
        default: {
            const double t = w.h_ - 0.0;
            w0 = k.dk.alpha * t * t * t;
            break;
        }
    }
    k.rho_self = k.mass * w0;
    k.mass_over_rho0 = k.mass / k.rho0;
    k.eps_lambda = prm_.epsilon_lambda;
    k.art_k = prm_.art_pressure_k;
    k.art_n = prm_.art_pressure_n;
    bool is_int = false;
    k.art_n_int = integer_exponent(prm_.art_pressure_n, &is_int);
    k.art_n_is_int = is_int ? 1 : 0;
    // pbf.rs:245-246 w_dq = w(dkern, dq_over_h * h): evaluated once on the device path's formula
    {
        const double dq = prm_.art_pressure_dq_over_h * w.h_;
        const double a = k.dk.alpha, h = w.h_;
        double wd = 0.0;
        if (!(h <= 0.0 || dq < 0.0)) {
            switch (prm_.density_kernel) {
                case kCubic: {
                    const double q = dq / h;
                    if (q < 2.0) {
                        if (q < 1.0) wd = a * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
                        else {
                            const double t = 2.0 - q;
                            wd = a * 0.25 * t * t * t;
                        }
                    }
                    break;
                }
                case kWendland: {
                    const double q = dq / h;
                    if (q < 2.0) {
                        const double t = 1.0 - 0.5 * q;
                        wd = a * t * t * t * t * (2.0 * q + 1.0);
                    }
                    break;
                }
                case kPoly6:
                    if (dq < h) {
                        const double t = h * h - dq * dq;
                        wd = a * t * t * t;
                    }
                    break;
                default:
                    if (dq < h) {
                        const double t = h - dq;
                        wd = a * t * t * t;
                    }
                    break;
            }
        }
        k.w_dq = wd;
    }
    k.max_corr = 0.4 * w.h_;
    {
        const double sup = std::fmax(kernel_support(prm_.density_kernel, w.h_), kernel_support(prm_.grad_kernel, w.h_));
        const double far = sup * (1.0 + 1e-9);
        k.far2 = far * far;
    }
    k.visc_eps = prm_.viscosity_eps;
    k.vort_eps = prm_.vorticity_eps;
    k.gx = prm_.gravity[0];
    k.gy = prm_.gravity[1];
    k.gz = prm_.gravity[2];
}

void PbfSolver::lists(bool all_candidates) {
    World& w = *w_;
    if (w.list_all_candidates_ != all_candidates) {
        w.list_all_candidates_ = all_candidates;
        w.refresh_step_const();
        w.lists_valid_ = false;
    }
    w.ensure_lists(true);
}

void PbfSolver::step(double dt) {
    World& w = *w_;
    const uint32_t n = (uint32_t)w.n_;
    if (n == 0) {
        w.t_ += dt;
        return;
    }
    cudaStream_t st = w.st_;
    const uint32_t nb = blocks_for(n, kPbfThreads);
    // pbf.rs:387-401: predict, grid and lists on the predictions
    k_pbf_predict<<<nb, kPbfThreads, 0, st>>>(n, kc_, dt, w.cur_, w.pos_nx_);
    w.launches_ += 1;
    w.build_grid(w.pos_nx_, nullptr);
    // pbf.rs:146-156: lists the constraint iterations reuse while the
    // predictions move hold every candidate of the neighbour cells, as the
    // reference's; lists used only at the positions they were built for keep
    // the candidates in support (the others add +-0)
    const bool reused = prm_.reuse_neighbours && prm_.iterations > 1;
    lists(reused);
    // pbf.rs:403-411: constraint iterations
    for (uint64_t it = 0; it < prm_.iterations; ++it) {
        k_pbf_density<<<nb, kPbfThreads, kKeepBytes, st>>>(n, kc_, w.cur_, w.lists_);
        k_pbf_lambda<<<nb, kPbfThreads, kKeepBytes, st>>>(n, kc_, w.cur_, w.lists_, lambda_, lambda_orig_);
        k_pbf_delta_p<<<nb, kPbfThreads, kKeepBytes, st>>>(n, kc_, w.cur_, w.lists_, lambda_, dp_);
        k_pbf_apply_dp<<<nb, kPbfThreads, 0, st>>>(n, w.dim_, w.cur_, dp_);
        w.launches_ += 4;
        if (!prm_.reuse_neighbours) {
            w.build_grid(nullptr, nullptr);
            lists(false);
        }
    }
    // pbf.rs:413-426: velocities from the displacement, x = pred, grid and
    // lists on the final positions, density there
    k_pbf_finalize<<<nb, kPbfThreads, 0, st>>>(n, dt, w.cur_);
    w.launches_ += 1;
    w.build_grid(nullptr, nullptr);
    lists(false);
    k_pbf_density<<<nb, kPbfThreads, kKeepBytes, st>>>(n, kc_, w.cur_, w.lists_);
    w.launches_ += 1;
    // pbf.rs:288-381: the grid on x equals the one just built
    if (prm_.viscosity_eps != 0.0) {
        k_pbf_viscosity<<<nb, kPbfThreads, 0, st>>>(n, kc_, w.cur_, w.lists_, dp_);
        k_pbf_add_dv<<<nb, kPbfThreads, 0, st>>>(n, w.cur_, dp_);
        w.launches_ += 2;
    }
    if (prm_.vorticity_eps != 0.0 && dt != 0.0) {
        k_pbf_omega<<<nb, kPbfThreads, 0, st>>>(n, kc_, w.cur_, w.lists_, omega_);
        k_pbf_confine<<<nb, kPbfThreads, 0, st>>>(n, kc_, dt, w.cur_, w.lists_, omega_);
        w.launches_ += 2;
    }
    w.check(cudaGetLastError(), "pbf step");
    w.t_ += dt;
    w.grid_current_ = true;
    w.rho_current_ = false;
}

void PbfSolver::run(double dt, uint64_t steps) {
    for (uint64_t s = 0; s < steps; ++s) {
        step(dt);
        if ((s + 1) % 16 == 0) w_->status();
    }
}

void PbfSolver::get_lambda(double* out) {
    World& w = *w_;
    if (!w.n_) return;
    w.check(cudaMemcpyAsync(out, lambda_orig_, sizeof(double) * w.n_, cudaMemcpyDeviceToHost, w.st_), "lambda");
    w.check(cudaStreamSynchronize(w.st_), "lambda");
}

double PbfSolver::mean_density_error() {
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
            s += std::fabs(rho[i] / w.rho0_ - 1.0);
            c += 1;
        }
    return c == 0 ? 0.0 : s / (double)c;
}

double PbfSolver::v_max() {
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

}  // namespace pe
