// The f64 SPH passes of the WCSPH step, one thread per cell-sorted slot.
//
// Each pass walks the slot's neighbour list and reproduces the reference's
// floating-point sequence exactly (compiled with --fmad=false):
//   density   — wcsph.rs:117-154 (visiting order)
//   pressure  — wcsph.rs:157-178, eos.rs:59-80, viscosity.rs:89
//   forces    — wcsph.rs:181-259 + the kick/drift of wcsph.rs:332-342
//   xsph      — wcsph.rs:283-323
//
// Force-order argument. The reference accumulates a[i] by a symmetric
// scatter: for each fluid i in ascending index, for each neighbour j in
// visiting order, a fluid j > i adds f to a[i] and subtracts it from a[j].
// Hence the final a[k] is the sequence
//     0  -  f(i1,k) - f(i2,k) - ...      (fluid i < k, ascending i)
//        +  f(k,j) ...                   (fluid j > k and boundary j, visiting order)
//        +  g.
// Every factor of f(i,k) is symmetric in (i,k) bit for bit (sums commute,
// (-a)(-b) = ab exactly) except grad W, which flips sign exactly, so
// f(i,k) = -f(k,i) bitwise and x - f(i,k) = x + f(k,i). A gather that adds
// f(k,i) over the "lower" list (ascending original index) and then f(k,j)
// over the visiting-order list, skipping entries flagged lower, therefore
// yields the reference's bits. Pairs outside the support contribute +-0,
// which leaves a sum that started at +0 unchanged, so the lists may omit them.
#include "pe_math.cuh"
#include "wcsph_device.cuh"
#include "sph_pair.cuh"
#include "list_iter.cuh"

namespace pe {

namespace {

constexpr int kThreads = 128;
// Visit entries compacted per chunk in the force pass. 64 rather than 32: the
// warp's pair loop runs to the fullest lane of each chunk, and the spread of
// the kept counts shrinks relative to their mean as the chunk grows (forces
// 3.32 -> 3.17 ms at 1M). 64 x 4 bytes per thread is 32 KB per 128-thread
// CTA, which still leaves the pass register-limited (five CTAs per SM).
constexpr uint32_t kCompact = 64;

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

struct PosVel {
    double4 x, v;
};

__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

template <bool CUBIC>
__global__ void __launch_bounds__(kMaxPassThreads) k_density(uint32_t n, StepConst k, StateBufs s,
                                                      ListBufs l) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.flags[i] & kFlagBoundary) {
        s.vel[i].w = k.rho0;  // wcsph.rs:127
        return;
    }
    const double4 xi = s.pos[i];
    double rho = k.rho_self;  // 0.0 + mass * W(0)
    const ListRef vr = list_ref(l, i, kListVisit);
    // W of entry t kept at the entry's pool index for the XSPH pass, two
    // entries per 16-byte store (a whole sector over a group's four entries);
    // wrow walks the slot's rows of 16-byte groups
    bool keep_w = false;
    if (l.wpair) {
        keep_w = w_fits(l, vr);
        if (!keep_w) atomicOr(l.w_short, 1u);
    }
    double* wrow = keep_w ? l.wpair + (vr.p - l.pool) : nullptr;
    double wprev = 0.0;
    for_each_loaded2_t(
        vr, [&](uint32_t, uint32_t e) { return s.pos[e & kEntrySlotMask]; },
        [&](uint32_t t, uint32_t e, const double4& xj) {
        const uint32_t j = e & kEntrySlotMask;
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double wij = kw<CUBIC>(r, k);
        if (keep_w) {
            if (t & 1u) {
                *reinterpret_cast<double2*>(wrow + (t & 2u)) = make_double2(wprev, wij);
                if (t & 2u) wrow += vr.step;
            } else {
                wprev = wij;
            }
        }
        if ((e & kEntryOriented) && !sees_fluid(k, xj, s.nout[j], xi.x, xi.y, xi.z)) return;
        // fluid: mass * W; boundary: (rho0 * psi_j) * W (wcsph.rs:143-148)
        const double f = (e & kEntryBoundary) ? k.rho0 * xj.w : k.mass;
        rho += f * wij;
    });
    if (keep_w && (vr.n & 1u))  // the last entry's W, unpaired
        *reinterpret_cast<double2*>(wrow + ((vr.n - 1u) & 2u)) = make_double2(wprev, 0.0);
    rho = fmax(rho, 1e-12);  // wcsph.rs:152 (f64::max)
    s.vel[i].w = rho;
    // keep the cached p / rho^2 consistent with the new rho (the reference
    // divides the stored p by the current rho in every force pair)
    s.pos[i].w = s.p[i] / (rho * rho);
}

// max |v|^2 of each tank's fluid (viscosity.rs:89-100), as u64 bits: a warp
// whose lanes all belong to one tank reduces first, a warp across a tank
// boundary lets each lane add its own value.
__global__ void k_vmax(uint32_t n, Tanks tk, StateBufs s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    uint32_t t = 0xffffffffu;
    if (i < n) {
        t = tk.slot_tank[i];
        if (!(s.flags[i] & kFlagBoundary)) {
            double4 v = s.vel[i];
            double q = v.x * v.x + v.y * v.y + v.z * v.z;
            if (q > m) m = q;  // viscosity.rs:91-96 (NaN never exceeds m)
        }
    }
    unsigned long long b = __double_as_longlong(m);
    const uint32_t t0 = __shfl_sync(0xffffffffu, t, 0);
    if (i >= n) t = t0;  // idle lanes carry lane 0's tank and a zero
    if (__all_sync(0xffffffffu, t == t0)) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
            b = x > b ? x : b;
        }
        // Non-negative doubles order like their bit patterns.
        if ((threadIdx.x & 31u) == 0 && b != 0ull && t0 != 0xffffffffu) atomicMax(&tk.vmax2[t0], b);
    } else if (b != 0ull && i < n) {
        atomicMax(&tk.vmax2[t], b);
    }
}

__global__ void k_pressure(uint32_t n, StepConst k, Tanks tk, StateBufs s) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // compute_pressure (wcsph.rs:158-169): c = max(c, 10 * v_max), persisted
    // per tank. Every thread of a tank derives the same c; re-reading an
    // already-updated c gives the same value (the update is idempotent), so
    // the write by the tank's first slot is race-free in effect.
    const uint32_t t = tk.slot_tank[i];
    double c = tk.c[t];
    if (k.adapt_sound_speed) {
        double vmax = sqrt(__longlong_as_double((long long)tk.vmax2[t]));
        double min_c = 10.0 * fmax(vmax, 0.0);
        c = c < min_c ? min_c : c;
    }
    if (i == tk.desc[t].slot_begin) tk.c[t] = c;
    if (s.flags[i] & kFlagBoundary) {
        s.p[i] = 0.0;
        return;
    }
    double rho = s.vel[i].w;
    double ratio = rho / k.eos_rho0;
    double b = k.eos_rho0 * c * c / k.eos_gamma;
    double pw = k.gamma_is_int ? pow_int_dd(ratio, k.gamma_int) : pow(ratio, k.eos_gamma);
    double p = b * (pw - 1.0);
    s.p[i] = p;
    s.pos[i].w = p / (rho * rho);  // p_i / (rho_i * rho_i), used by every pair of i
}

// Pressure + Monaghan viscosity force of fluid pair (k, j), seen from k:
// rx = x_j - x_k (wcsph.rs:219), pi_ij(x_k, x_j, v_k, v_j, rho_k, rho_j).
template <bool CUBIC, bool BETA0>
__device__ __forceinline__ void fluid_pair(const StepConst& kc, double nac, double4 xk, double4 vk,
                                           double4 xj, double4 vj, double& ax, double& ay,
                                           double& az) {
    const double rx = xj.x - xk.x, ry = xj.y - xk.y, rz = xj.z - xk.z;
    const double r2 = rx * rx + ry * ry + rz * rz;
    const double r = sqrt(r2);
    if (r < 1e-30) return;
    const double dwdr = kdwdr<CUBIC>(r, kc);
    const double sc = -dwdr / r;
    const double gx = rx * sc, gy = ry * sc, gz = rz * sc;
    const double press = xk.w + xj.w;  // p_k/rho_k^2 + p_j/rho_j^2
    const double mp = -kc.mass * press;
    // viscosity.rs:51-73 with r_ij = x_k - x_j, v_ij = v_k - v_j. Evaluated for
    // every pair and selected, so that approaching and receding pairs do not
    // split the warp; a receding pair's value is discarded (pi = 0 exactly).
    // x_k - x_j is exactly -(x_j - x_k) (round to nearest is symmetric), so
    // |x_k - x_j|^2 is r2 bit for bit and v_ij . (x_k - x_j) is -(v_ij . r)
    // up to the sign of a zero, which only ever selects pi = 0.
    const double wx = vk.x - vj.x, wy = vk.y - vj.y, wz = vk.z - vj.z;
    const double vr = -(wx * rx + wy * ry + wz * rz);
    const double mu = kc.h * vr / (r2 + kc.eps_h2);
    const double rho_bar = 0.5 * (vk.w + vj.w);
    // With beta = 0 the beta mu^2 term is a signed zero, which leaves the
    // nonzero nac * mu of an approaching pair (mu < 0) unchanged.
    const double num = BETA0 ? nac * mu : nac * mu + kc.visc_beta * mu * mu;
    const double pic = num / rho_bar;
    const double pi = vr >= 0.0 ? 0.0 : pic;
    const double mv = -kc.mass * pi;
    ax += gx * mp + gx * mv;
    ay += gy * mp + gy * mv;
    az += gz * mp + gz * mv;
}

// Akinci boundary pressure of fluid k against boundary sample j (wcsph.rs:244-255).
template <bool CUBIC>
__device__ __forceinline__ void boundary_pair(const StepConst& kc, double4 xk, double4 xj,
                                              bool oriented, const double4* nout, uint32_t j,
                                              double& ax, double& ay, double& az) {
    double rx = xj.x - xk.x, ry = xj.y - xk.y, rz = xj.z - xk.z;
    double r2 = rx * rx + ry * ry + rz * rz;
    double r = sqrt(r2);
    if (r < 1e-30) return;
    if (oriented && !sees_fluid(kc, xj, nout[j], xk.x, xk.y, xk.z)) return;
    double dwdr = kdwdr<CUBIC>(r, kc);
    double sc = -dwdr / r;
    double gx = rx * sc, gy = ry * sc, gz = rz * sc;
    double m = -(kc.rho0 * xj.w) * xk.w;  // -(rho0 psi_j) * p_k/rho_k^2
    ax += gx * m;
    ay += gy * m;
    az += gz * m;
}

template <bool INTEGRATE, int DIM, bool CUBIC, bool BETA0>
__global__ void __launch_bounds__(kMaxPassThreads) k_forces(uint32_t n, StepConst kc, Tanks tk,
                                                            StateBufs s, ListBufs l, double dt,
                                                            double4* __restrict__ pos_next,
                                                            double4* __restrict__ vel_next,
                                                            const double4* __restrict__ st_a) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (s.flags[k] & kFlagBoundary) return;
    const double c0 = tk.c[tk.slot_tank[k]];
    const double nac = -kc.visc_alpha * c0;  // (-alpha) * c_bar, viscosity.rs:72
    const double4 xk = s.pos[k];
    const double4 vk = s.vel[k];
    double ax = 0.0, ay = 0.0, az = 0.0;
    // neighbour state gathered one entry ahead (boundary samples need no velocity)
    auto load = [&](uint32_t e) {
        PosVel d;
        const uint32_t j = e & kEntrySlotMask;
        d.x = s.pos[j];
        d.v = (e & kEntryBoundary) ? make_double4(0.0, 0.0, 0.0, 0.0) : s.vel[j];
        return d;
    };
    // fluid i < k, ascending original index
    for_each_loaded(list_ref(l, k, kListLower), load, [&](uint32_t, const PosVel& d) {
        fluid_pair<CUBIC, BETA0>(kc, nac, xk, vk, d.x, d.v, ax, ay, az);
    });
    // fluid j > k and boundary j, visiting order: the visit list without the
    // entries flagged lower (those came from the lower list, in index order).
    // The list is taken in chunks of kCompact entries whose kept entries are
    // first compacted into this thread's column of shared memory, so the pair
    // loop of a warp runs over kept entries only (the flagged ones are about
    // half and fall at different positions in each thread's list). Chunks stay
    // in step across the warp: a per-lane stream that refilled each lane's
    // buffer when it ran empty made the warp wait on every lane's list loads
    // in turn (forces 3.47 -> 4.75 ms at 1M, 19 of 32 lanes active).
    // The chunks are aligned to the list's end (the first one is the short
    // one): the kept entries cluster at the end of the visiting order (the
    // neighbour cells after the particle's own), so there every lane's chunk
    // is full and none waits on a fuller one.
    extern __shared__ uint32_t s_keep[];  // kCompact x blockDim.x, column per thread
    const uint32_t tid = threadIdx.x, bd = blockDim.x;
    const ListRef vr = list_ref(l, k, kListVisit);
    const uint32_t nv4 = (vr.n + 3u) & ~3u;  // chunk ends stay on 16-byte groups
    uint32_t t1 = nv4 ? nv4 - (nv4 - 1u) / kCompact * kCompact : 0u;
    for (uint32_t t0 = 0; t0 < vr.n; t0 = t1, t1 += kCompact) {
        const uint32_t te = min(vr.n, t1);
        uint32_t c = 0;
        for (uint32_t t = t0; t < te; t += 4) {
            const uint4 g4 = __ldg(reinterpret_cast<const uint4*>(vr.p + (size_t)(t >> 2) * vr.step));
            const uint32_t ge[4] = {g4.x, g4.y, g4.z, g4.w};
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q)
                if (t + q < te && !(ge[q] & kEntryLower)) s_keep[(c++) * bd + tid] = ge[q];
        }
        if (c == 0) continue;
        uint32_t e = s_keep[tid];
        PosVel d = load(e);
        for (uint32_t u = 0; u < c; ++u) {
            const uint32_t ec = e;
            const PosVel dc = d;
            if (u + 1 < c) {
                e = s_keep[(u + 1) * bd + tid];
                d = load(e);
            }
            if (ec & kEntryBoundary) {
                boundary_pair<CUBIC>(kc, xk, dc.x, (ec & kEntryOriented) != 0u, s.nout, ec & kEntrySlotMask, ax, ay, az);
            } else {
                fluid_pair<CUBIC, BETA0>(kc, nac, xk, vk, dc.x, dc.v, ax, ay, az);
            }
        }
    }
    ax += kc.gx;
    ay += kc.gy;
    az += kc.gz;
    if (st_a) {  // wcsph.rs:273-277 a += surface-tension acceleration
        const double4 t = st_a[k];
        ax += t.x;
        ay += t.y;
        az += t.z;
    }
    s.acc[k] = make_double4(ax, ay, az, 0.0);
    if (INTEGRATE) {
        // wcsph.rs:336-341 symplectic Euler
        double vx = vk.x + ax * dt, vy = vk.y + ay * dt, vz = vk.z + az * dt;
        double px = xk.x + vx * dt, py = xk.y + vy * dt, pz = xk.z + vz * dt;
        if (DIM == 2) {
            pz = 0.0;
            vz = 0.0;
        }
        pos_next[k] = make_double4(px, py, pz, xk.w);
        vel_next[k] = make_double4(vx, vy, vz, vk.w);
    }
}

// boundary_force[j] (wcsph.rs:254): sum over fluid i in ascending index of
// f(i,j) * (-m) with f = gradW(x_j - x_i) * (-(rho0 psi_j) * p_i/rho_i^2).
template <bool CUBIC>
__global__ void __launch_bounds__(kThreads) k_boundary_force(uint32_t n, StepConst kc, StateBufs s,
                                                             ListBufs l) {
    uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    if (!(s.flags[b] & kFlagBoundary)) return;
    const double4 xb = s.pos[b];
    const bool oriented = (s.flags[b] & kFlagOriented) != 0;
    const double4 nb = oriented ? s.nout[b] : make_double4(0, 0, 0, 0);
    const double mpsi = -(kc.rho0 * xb.w);
    const double mneg = -kc.mass;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for_each_entry(list_ref(l, b, kListLower), [&](uint32_t i) {
        double4 xi = s.pos[i];
        double rx = xb.x - xi.x, ry = xb.y - xi.y, rz = xb.z - xi.z;
        double r2 = rx * rx + ry * ry + rz * rz;
        double r = sqrt(r2);
        if (r < 1e-30) return;
        if (oriented && !sees_fluid(kc, xb, nb, xi.x, xi.y, xi.z)) return;
        double dwdr = kdwdr<CUBIC>(r, kc);
        double sc = -dwdr / r;
        double m = mpsi * xi.w;
        double ffx = (rx * sc) * m, ffy = (ry * sc) * m, ffz = (rz * sc) * m;
        fx += ffx * mneg;
        fy += ffy * mneg;
        fz += ffz * mneg;
    });
    s.bf[b] = make_double4(fx, fy, fz, 0.0);
}

// The XSPH sum of fluid slot i with velocity vi, each pair's W recomputed
// from the neighbour's position.
template <bool CUBIC>
__device__ __forceinline__ double3 xsph_dv(uint32_t i, const StepConst& kc, const StateBufs& s,
                                           const ListBufs& l, double4 vi) {
    const double4 xi = s.pos[i];
    double dvx = 0.0, dvy = 0.0, dvz = 0.0;
    for_each_loaded2(
        list_ref(l, i, kListVisit),
        [&](uint32_t e) {
            PosVel d{};
            if (!(e & kEntryBoundary)) {
                d.x = s.pos[e & kEntrySlotMask];
                d.v = s.vel[e & kEntrySlotMask];
            }
            return d;
        },
        [&](uint32_t e, const PosVel& d) {
        if (e & kEntryBoundary) return;
        const double4 xj = d.x;
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double wij = kw<CUBIC>(r, kc);
        const double4 vj = d.v;
        const double rho_bar = 0.5 * (vi.w + vj.w);
        const double f = kc.mass / rho_bar * wij;
        dvx += (vj.x - vi.x) * f;
        dvy += (vj.y - vi.y) * f;
        dvz += (vj.z - vi.z) * f;
    });
    return make_double3(dvx, dvy, dvz);
}

// short_only: run only if the density pass met a list beyond the pair-weight
// buffer (the launch that follows k_xsph_w, which then did nothing).
template <bool CUBIC>
__global__ void __launch_bounds__(kMaxPassThreads) k_xsph(uint32_t n, StepConst kc, StateBufs s,
                                                   ListBufs l, double4* __restrict__ vel_out,
                                                   bool short_only) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (short_only && !__ldg(l.w_short)) return;
    const double4 vi = s.vel[i];
    if (s.flags[i] & kFlagBoundary) {
        vel_out[i] = vi;
        return;
    }
    const double3 dv = xsph_dv<CUBIC>(i, kc, s, l, vi);
    vel_out[i] = make_double4(vi.x + dv.x * kc.xsph_eps, vi.y + dv.y * kc.xsph_eps,
                              vi.z + dv.z * kc.xsph_eps, vi.w);
}

// k_xsph with each pair's W(r) read from the density pass of the same lists
// and positions (the bits the pair would compute) instead of recomputed from
// the neighbour's position: per fluid pair one 8-byte read of a stream in
// place of a 32-byte gather, a square root and the kernel polynomial
// (XSPH 2.04 -> 1.44 ms at 1M, density 1.16 -> 1.43 ms for the stores).
// When the density pass met a list beyond the buffer, it does nothing and
// the k_xsph launch after it recomputes W for every particle (a separate
// kernel, so that this one keeps its own, smaller register count).
__global__ void __launch_bounds__(kMaxPassThreads) k_xsph_w(uint32_t n, StepConst kc, StateBufs s,
                                                     ListBufs l, double4* __restrict__ vel_out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (__ldg(l.w_short)) return;
    const double4 vi = s.vel[i];
    if (s.flags[i] & kFlagBoundary) {
        vel_out[i] = vi;
        return;
    }
    double dvx = 0.0, dvy = 0.0, dvz = 0.0;
    const ListRef vr = list_ref(l, i, kListVisit);
    const double* wrow = l.wpair + (vr.p - l.pool);  // walks the rows as the loads advance
    // Both streams (entries, weights) come from DRAM; their rows four ahead
    // are prefetched into L1 (within the slot's own rows): 1.44 -> 1.40 ms at 1M.
    constexpr uint32_t kPfRows = 4;
    const uint32_t nrows = (vr.n + 3u) >> 2;
    struct VelW {
        double4 v;
        double w;
    };
    for_each_loaded2_t(
        vr,
        [&](uint32_t t, uint32_t e) {  // called for t = 0, 1, 2, ... in order
            if ((t & 3u) == 0u && (t >> 2) + kPfRows < nrows) {
                prefetch_l1(vr.p + (size_t)((t >> 2) + kPfRows) * vr.step);
                prefetch_l1(wrow + (size_t)kPfRows * vr.step);
            }
            VelW d{};
            if (!(e & kEntryBoundary)) {
                d.v = s.vel[e & kEntrySlotMask];
                d.w = __ldg(wrow + (t & 3u));
            }
            if ((t & 3u) == 3u) wrow += vr.step;
            return d;
        },
        [&](uint32_t, uint32_t e, const VelW& d) {
        if (e & kEntryBoundary) return;
        const double4 vj = d.v;
        const double rho_bar = 0.5 * (vi.w + vj.w);
        const double f = kc.mass / rho_bar * d.w;
        dvx += (vj.x - vi.x) * f;
        dvy += (vj.y - vi.y) * f;
        dvz += (vj.z - vi.z) * f;
    });
    vel_out[i] = make_double4(vi.x + dvx * kc.xsph_eps, vi.y + dvy * kc.xsph_eps,
                              vi.z + dvz * kc.xsph_eps, vi.w);
}

__global__ void k_in_support(uint32_t n, StepConst kc, StateBufs s, ListBufs l, uint32_t* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.flags[i] & kFlagBoundary) {
        out[i] = 0;
        return;
    }
    const double4 xi = s.pos[i];
    uint32_t c = 0;
    for_each_entry(list_ref(l, i, kListVisit), [&](uint32_t e) {
        const double4 xj = s.pos[e & kEntrySlotMask];
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        c += in_support(r, kc);
    });
    out[i] = c;
}

template <bool I, int D, bool C, bool B>
void allow_compact_smem() {
    cudaFuncSetAttribute(k_forces<I, D, C, B>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kCompact * kMaxPassThreads * sizeof(uint32_t)));
}

template <bool I, int D>
void allow_compact_smem_all() {
    allow_compact_smem<I, D, true, true>();
    allow_compact_smem<I, D, true, false>();
    allow_compact_smem<I, D, false, true>();
    allow_compact_smem<I, D, false, false>();
}

}  // namespace

// The force pass's compaction buffer exceeds the 48 KB a launch gets without
// opting in once a CTA has more than 192 threads.
void forces_prepare() {
    allow_compact_smem_all<true, 3>();
    allow_compact_smem_all<false, 3>();
    allow_compact_smem_all<true, 2>();
    allow_compact_smem_all<false, 2>();
}

void launch_density(uint32_t n, uint32_t threads, const StepConst& k, const StateBufs& s,
                    const ListBufs& l, cudaStream_t st) {
    if (!n) return;
    if (k.kernel == 0) k_density<true><<<blocks_for(n, threads), threads, 0, st>>>(n, k, s, l);
    else k_density<false><<<blocks_for(n, threads), threads, 0, st>>>(n, k, s, l);
}

void launch_vmax(uint32_t n, const Tanks& tk, const StateBufs& s, cudaStream_t st) {
    if (n) k_vmax<<<blocks_for(n, 256), 256, 0, st>>>(n, tk, s);
}

void launch_pressure(uint32_t n, const StepConst& k, const Tanks& tk, const StateBufs& s,
                     cudaStream_t st) {
    if (n) k_pressure<<<blocks_for(n, 256), 256, 0, st>>>(n, k, tk, s);
}

void launch_forces(uint32_t n, uint32_t threads, const StepConst& k, const Tanks& tk,
                   const StateBufs& s, const ListBufs& l, bool integrate, double dt,
                   double4* pos_next, double4* vel_next, const double4* st_a, cudaStream_t st) {
    if (!n) return;
    const uint32_t b = blocks_for(n, threads);
    const size_t sm = (size_t)kCompact * threads * sizeof(uint32_t);
    const bool cubic = k.kernel == 0;
#define PE_FORCES(I, D, C, B) \
    k_forces<I, D, C, B><<<b, threads, sm, st>>>(n, k, tk, s, l, dt, pos_next, vel_next, st_a)
#define PE_FORCES_B(I, D, C)              \
    do {                                  \
        if (beta0) PE_FORCES(I, D, C, true); \
        else PE_FORCES(I, D, C, false);   \
    } while (0)
    const bool beta0 = k.visc_beta == 0.0;
    if (k.dim == 3) {
        if (cubic) {
            if (integrate) PE_FORCES_B(true, 3, true);
            else PE_FORCES_B(false, 3, true);
        } else {
            if (integrate) PE_FORCES_B(true, 3, false);
            else PE_FORCES_B(false, 3, false);
        }
    } else {
        if (cubic) {
            if (integrate) PE_FORCES_B(true, 2, true);
            else PE_FORCES_B(false, 2, true);
        } else {
            if (integrate) PE_FORCES_B(true, 2, false);
            else PE_FORCES_B(false, 2, false);
        }
    }
#undef PE_FORCES_B
#undef PE_FORCES
}

void launch_boundary_force(uint32_t n, const StepConst& k, const StateBufs& s, const ListBufs& l,
                           cudaStream_t st) {
    if (!n) return;
    if (k.kernel == 0) k_boundary_force<true><<<blocks_for(n, kThreads), kThreads, 0, st>>>(n, k, s, l);
    else k_boundary_force<false><<<blocks_for(n, kThreads), kThreads, 0, st>>>(n, k, s, l);
}

void launch_xsph(uint32_t n, uint32_t threads, const StepConst& k, const StateBufs& s,
                 const ListBufs& l, double4* vel_out, cudaStream_t st, bool use_w) {
    if (!n) return;
    const bool w = use_w && l.wpair;
    if (w) k_xsph_w<<<blocks_for(n, threads), threads, 0, st>>>(n, k, s, l, vel_out);
    if (k.kernel == 0) k_xsph<true><<<blocks_for(n, threads), threads, 0, st>>>(n, k, s, l, vel_out, w);
    else k_xsph<false><<<blocks_for(n, threads), threads, 0, st>>>(n, k, s, l, vel_out, w);
}

void launch_in_support_counts(uint32_t n, const StepConst& k, const StateBufs& s,
                              const ListBufs& l, uint32_t* out, cudaStream_t st) {
    if (n) k_in_support<<<blocks_for(n, 256), 256, 0, st>>>(n, k, s, l, out);
}

}  // namespace pe
