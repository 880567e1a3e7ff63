// Single-precision form of the SPH passes.
//
// The neighbour-loop state is float4: cell-local positions (offset from the
// corner of the particle's own grid cell, w = p/rho^2 for fluid or psi for
// boundary samples) and velocities (w = rho). The vector between two
// particles is (key_j - key_i) * cell + (local_j - local_i), so positions keep
// ~1e-9 m resolution at any distance from the origin. Pair arithmetic is
// single precision with fast reciprocals; the density, force and XSPH sums are
// Kahan-compensated. The grid, its sort and the global v_max reduction stay
// f64 (the f64 position of a particle is key * cell + local, exact in f64, and
// re-expressed against the new cell after each sort). This form does not
// reproduce the reference's bits; `bench.py --form f32` reports its error
// against the f64 path.
#include "list_iter.cuh"
#include "pe_math.cuh"
#include "wcsph_device.cuh"

namespace pe {

namespace {


inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

struct Kahan {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float x) {
        const float y = x - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

__device__ __forceinline__ float w_f32(float r, const F32Const& k) {
    const float q = r * k.inv_h;
    if (q >= 2.f) return 0.f;
    if (q < 1.f) return k.alpha * (1.f - 1.5f * q * q + 0.75f * q * q * q);
    const float t = 2.f - q;
    return k.alpha * 0.25f * t * t * t;
}

// dW/dr / r, the scale of grad W (0 outside the support and at r = 0)
__device__ __forceinline__ float dwdr_over_r_f32(float r, float inv_r, const F32Const& k) {
    const float q = r * k.inv_h;
    if (q >= 2.f || q <= 0.f) return 0.f;
    float dwdq;
    if (q < 1.f) {
        dwdq = k.alpha * (-3.f * q + 2.25f * q * q);
    } else {
        const float t = 2.f - q;
        dwdq = k.alpha * (-0.75f * t * t);
    }
    return dwdq * k.inv_h * inv_r;
}

// The pair vector x_j - x_i of two particles in the same or adjacent cells:
// their keys differ by -1, 0 or 1 per axis, which the keys mod 4 (cm, two
// bits per axis) determine, so a neighbour's full key need not be read.
__device__ __forceinline__ float3 rel(uint32_t ci, const float4& pi, uint32_t cj, const float4& pj,
                                      float cell) {
    const int dx = (int)(((cj & 3u) - (ci & 3u) + 1u) & 3u) - 1;
    const int dy = (int)((((cj >> 2) & 3u) - ((ci >> 2) & 3u) + 1u) & 3u) - 1;
    const int dz = (int)((((cj >> 4) & 3u) - ((ci >> 4) & 3u) + 1u) & 3u) - 1;
    return make_float3((float)dx * cell + (pj.x - pi.x), (float)dy * cell + (pj.y - pi.y),
                       (float)dz * cell + (pj.z - pi.z));
}

// particles.rs:126 boundary_sees_fluid for an oriented sample b seen from a
// fluid particle at d = x_b - x_f
__device__ __forceinline__ bool sees_fluid_f32(const F32Const& k, const double4& nb, float3 d) {
    const float nx = (float)nb.x, ny = (float)nb.y, nz = (float)nb.z;
    const float n2 = nx * nx + ny * ny + nz * nz;
    if (n2 <= 0.f) return true;
    const float eps = k.boundary_eps_h * sqrtf(n2);
    return -(d.x * nx + d.y * ny + d.z * nz) > -eps;
}

// A neighbour's loop state, gathered one entry ahead of its use.
struct Nb32 {
    float4 p;
    uint32_t km;  // cell key mod 4 (F32Bufs.kmod)
    float4 v;
};

__global__ void __launch_bounds__(kMaxPassThreads) k_density_f32(uint32_t n, F32Const k, StateBufs s,
                                                          F32Bufs f, ListBufs l) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.flags[i] & kFlagBoundary) {
        f.vel[i].w = k.rho0;
        return;
    }
    const float4 pi = f.pos[i];
    const uint32_t ci = f.kmod[i];
    Kahan rho;
    rho.add(k.rho_self);
    const ListRef vr = list_ref(l, i, kListVisit);
    // W of each entry kept for the XSPH pass, one 16-byte store per group of
    // four entries at the group's pool index (wrow walks the slot's rows)
    bool keep_w = false;
    if (l.wpair32) {
        keep_w = w_fits(l, vr);
        if (!keep_w) atomicOr(l.w_short, 1u);
    }
    float* wrow = keep_w ? l.wpair32 + (vr.p - l.pool) : nullptr;
    float w0 = 0.f, w1 = 0.f, w2 = 0.f;
    for_each_loaded_t(
        vr,
        [&](uint32_t, uint32_t e) {
            Nb32 b;
            b.p = f.pos[e & kEntrySlotMask];
            b.km = f.kmod[e & kEntrySlotMask];
            return b;
        },
        [&](uint32_t t, uint32_t e, const Nb32& b) {
            const float4 pj = b.p;
            const float3 d = rel(ci, pi, b.km, pj, k.cell);
            const float r = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
            const float w = w_f32(r, k);
            if (keep_w) {
                switch (t & 3u) {
                    case 0: w0 = w; break;
                    case 1: w1 = w; break;
                    case 2: w2 = w; break;
                    default:
                        *reinterpret_cast<float4*>(wrow) = make_float4(w0, w1, w2, w);
                        wrow += vr.step;
                }
            }
            if ((e & kEntryOriented) && !sees_fluid_f32(k, s.nout[e & kEntrySlotMask], d)) return;
            rho.add(((e & kEntryBoundary) ? k.rho0 * pj.w : k.mass) * w);
        });
    if (keep_w && (vr.n & 3u)) *reinterpret_cast<float4*>(wrow) = make_float4(w0, w1, w2, 0.f);
    const float r = fmaxf(rho.s, 1e-12f);
    f.vel[i].w = r;
    s.vel[i].w = (double)r;
}

__global__ void k_vmax_f32(uint32_t n, Tanks tk, StateBufs s, F32Bufs f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    uint32_t t = 0xffffffffu;
    if (i < n) {
        t = tk.slot_tank[i];
        if (!(s.flags[i] & kFlagBoundary)) {
            const float4 v = f.vel[i];
            const double q = (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z;
            if (q > m) m = q;
        }
    }
    unsigned long long b = __double_as_longlong(m);
    const uint32_t t0 = __shfl_sync(0xffffffffu, t, 0);
    if (i >= n) t = t0;
    if (__all_sync(0xffffffffu, t == t0)) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
            b = x > b ? x : b;
        }
        if ((threadIdx.x & 31u) == 0 && b != 0ull && t0 != 0xffffffffu) atomicMax(&tk.vmax2[t0], b);
    } else if (b != 0ull && i < n) {
        atomicMax(&tk.vmax2[t], b);
    }
}

__global__ void k_pressure_f32(uint32_t n, F32Const k, Tanks tk, StateBufs s, F32Bufs f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // f64 control of each tank's sound speed (wcsph.rs:158-169)
    const uint32_t t = tk.slot_tank[i];
    double c = tk.c[t];
    if (k.adapt_sound_speed) {
        const double vmax = sqrt(__longlong_as_double((long long)tk.vmax2[t]));
        const double min_c = 10.0 * fmax(vmax, 0.0);
        c = c < min_c ? min_c : c;
    }
    if (i == tk.desc[t].slot_begin) tk.c[t] = c;
    if (s.flags[i] & kFlagBoundary) {
        s.p[i] = 0.0;
        return;
    }
    const float rho = f.vel[i].w;
    const float x = rho * k.inv_eos_rho0;
    float pw;
    if (k.gamma7) {
        const float x2 = x * x, x4 = x2 * x2;
        pw = x4 * x2 * x;
    } else {
        pw = powf(x, k.eos_gamma);
    }
    const float b = (float)(k.eos_rho0 * c * c / k.eos_gamma_d);
    const float p = b * (pw - 1.f);
    s.p[i] = (double)p;
    f.pos[i].w = p / (rho * rho);
}

template <int DIM>
__global__ void __launch_bounds__(kMaxPassThreads) k_forces_f32(uint32_t n, F32Const k, Tanks tk,
                                                                StateBufs s, F32Bufs f, ListBufs l,
                                                                float dt, double4* __restrict__ pos_next,
                                                                double4* __restrict__ vel_next,
                                                                float* __restrict__ bf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (s.flags[i] & kFlagBoundary)) return;
    const float c0 = (float)tk.c[tk.slot_tank[i]];
    const float nac = -k.visc_alpha * c0;
    const float4 pi = f.pos[i];
    const float4 vi = f.vel[i];
    const int4 ki = s.key[i];
    const uint32_t ci = f.kmod[i];
    Kahan ax, ay, az;
    auto load = [&](uint32_t e) {
        Nb32 b;
        b.p = f.pos[e & kEntrySlotMask];
        b.km = f.kmod[e & kEntrySlotMask];
        b.v = f.vel[e & kEntrySlotMask];
        return b;
    };
    for_each_loaded(list_ref(l, i, kListVisit), load, [&](uint32_t e, const Nb32& b) {
        const uint32_t j = e & kEntrySlotMask;
        const float4 pj = b.p;
        const float3 d = rel(ci, pi, b.km, pj, k.cell);  // x_j - x_i
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        if (r2 < 1e-30f) return;
        const float inv_r = rsqrtf(r2);
        const float r = r2 * inv_r;
        const float sc_ = -dwdr_over_r_f32(r, inv_r, k);  // grad_i W = d * sc_
        if (e & kEntryBoundary) {
            if ((e & kEntryOriented) && !sees_fluid_f32(k, s.nout[j], d)) return;
            const float m = -(k.rho0 * pj.w) * pi.w;
            const float fx = d.x * sc_ * m, fy = d.y * sc_ * m, fz = d.z * sc_ * m;
            ax.add(fx);
            ay.add(fy);
            az.add(fz);
            if (bf) {
                atomicAdd(&bf[4 * (size_t)j], fx * -k.mass);
                atomicAdd(&bf[4 * (size_t)j + 1], fy * -k.mass);
                atomicAdd(&bf[4 * (size_t)j + 2], fz * -k.mass);
            }
            return;
        }
        const float4 vj = b.v;
        const float press = pi.w + pj.w;
        const float vr = (vi.x - vj.x) * -d.x + (vi.y - vj.y) * -d.y + (vi.z - vj.z) * -d.z;
        float pic = 0.f;
        if (vr < 0.f) {
            const float mu = k.h * vr / (r2 + k.eps_h2);
            pic = (nac * mu + k.visc_beta * mu * mu) * (2.f / (vi.w + vj.w));
        }
        const float s_ = sc_ * -k.mass * (press + pic);
        ax.add(d.x * s_);
        ay.add(d.y * s_);
        az.add(d.z * s_);
    });
    const float a_x = ax.s + k.gx, a_y = ay.s + k.gy, a_z = az.s + k.gz;
    s.acc[i] = make_double4(a_x, a_y, a_z, 0.0);
    // symplectic Euler in cell-local single precision
    float vx = vi.x + a_x * dt, vy = vi.y + a_y * dt, vz = vi.z + a_z * dt;
    float lx = pi.x + vx * dt, ly = pi.y + vy * dt, lz = pi.z + vz * dt;
    if (DIM == 2) {
        lz = 0.f;
        vz = 0.f;
    }
    // f64 position for the grid: key * cell + local, one f64 rounding
    pos_next[i] = make_double4((double)ki.x * k.cell_d + (double)lx, (double)ki.y * k.cell_d + (double)ly,
                               DIM == 2 ? 0.0 : (double)ki.z * k.cell_d + (double)lz, s.pos[i].w);
    vel_next[i] = make_double4(vx, vy, vz, vi.w);
}

// short_only: run only if the density pass met a list beyond the pair-weight
// buffer (the launch that follows k_xsph_f32_w, which then did nothing).
__global__ void __launch_bounds__(kMaxPassThreads) k_xsph_f32(uint32_t n, F32Const k, StateBufs s, F32Bufs f,
                                                       ListBufs l, float4* __restrict__ vel_out,
                                                       bool short_only) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (short_only && !__ldg(l.w_short)) return;
    const float4 vi = f.vel[i];
    if (s.flags[i] & kFlagBoundary) {
        vel_out[i] = vi;
        return;
    }
    const float4 pi = f.pos[i];
    const uint32_t ci = f.kmod[i];
    Kahan dx, dy, dz;
    auto load = [&](uint32_t e) {
        Nb32 b{};
        if (!(e & kEntryBoundary)) {
            b.p = f.pos[e & kEntrySlotMask];
            b.km = f.kmod[e & kEntrySlotMask];
            b.v = f.vel[e & kEntrySlotMask];
        }
        return b;
    };
    for_each_loaded(list_ref(l, i, kListVisit), load, [&](uint32_t e, const Nb32& b) {
        if (e & kEntryBoundary) return;
        const float4 pj = b.p;
        const float3 d = rel(ci, pi, b.km, pj, k.cell);
        const float r = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        const float w = w_f32(r, k);
        const float4 vj = b.v;
        const float g = k.mass * 2.f / (vi.w + vj.w) * w;
        dx.add((vj.x - vi.x) * g);
        dy.add((vj.y - vi.y) * g);
        dz.add((vj.z - vi.z) * g);
    });
    const float4 vn = make_float4(vi.x + dx.s * k.xsph_eps, vi.y + dy.s * k.xsph_eps,
                                  vi.z + dz.s * k.xsph_eps, vi.w);
    vel_out[i] = vn;
    s.vel[i] = make_double4(vn.x, vn.y, vn.z, vn.w);
}

// k_xsph_f32 with each pair's W read from the density pass of the same lists
// and positions instead of recomputed: the neighbour's velocity is the only
// gather (16 bytes in place of 48).
__global__ void __launch_bounds__(kMaxPassThreads) k_xsph_f32_w(uint32_t n, F32Const k, StateBufs s, F32Bufs f,
                                                         ListBufs l, float4* __restrict__ vel_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (__ldg(l.w_short)) return;  // k_xsph_f32 runs instead
    const float4 vi = f.vel[i];
    if (s.flags[i] & kFlagBoundary) {
        vel_out[i] = vi;
        return;
    }
    Kahan dx, dy, dz;
    const ListRef vr = list_ref(l, i, kListVisit);
    const float* wrow = l.wpair32 + (vr.p - l.pool);
    struct VelW {
        float4 v;
        float w;
    };
    auto load = [&](uint32_t t, uint32_t e) {  // t = 0, 1, 2, ... in order
        VelW b{};
        if (!(e & kEntryBoundary)) {
            b.v = f.vel[e & kEntrySlotMask];
            b.w = __ldg(wrow + (t & 3u));
        }
        if ((t & 3u) == 3u) wrow += vr.step;
        return b;
    };
    for_each_loaded_t(vr, load, [&](uint32_t, uint32_t e, const VelW& b) {
        if (e & kEntryBoundary) return;
        const float4 vj = b.v;
        const float g = k.mass * 2.f / (vi.w + vj.w) * b.w;
        dx.add((vj.x - vi.x) * g);
        dy.add((vj.y - vi.y) * g);
        dz.add((vj.z - vi.z) * g);
    });
    const float4 vn = make_float4(vi.x + dx.s * k.xsph_eps, vi.y + dy.s * k.xsph_eps,
                                  vi.z + dz.s * k.xsph_eps, vi.w);
    vel_out[i] = vn;
    s.vel[i] = make_double4(vn.x, vn.y, vn.z, vn.w);
}

// Cell-local single-precision state from the (sorted) f64 state.
__global__ void k_f32_from_f64(uint32_t n, double cell, StateBufs s, F32Bufs f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = s.pos[i];
    const int4 kk = s.key[i];
    const bool fluid = !(s.flags[i] & kFlagBoundary);
    f.pos[i] = make_float4((float)(p.x - (double)kk.x * cell), (float)(p.y - (double)kk.y * cell),
                           (float)(p.z - (double)kk.z * cell), fluid ? 0.f : (float)p.w);
    f.kmod[i] = (uint8_t)(((uint32_t)kk.x & 3u) | (((uint32_t)kk.y & 3u) << 2) | (((uint32_t)kk.z & 3u) << 4));
    const double4 v = s.vel[i];
    f.vel[i] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
}

__global__ void k_bf_to_f64(uint32_t n, const float* __restrict__ bf, StateBufs s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    s.bf[i] = make_double4(bf[4 * (size_t)i], bf[4 * (size_t)i + 1], bf[4 * (size_t)i + 2], 0.0);
}

}  // namespace

void launch_f32_from_f64(uint32_t n, double cell, const StateBufs& s, const F32Bufs& f,
                         cudaStream_t st) {
    if (n) k_f32_from_f64<<<blocks_for(n, 256), 256, 0, st>>>(n, cell, s, f);
}

void launch_density_f32(uint32_t n, uint32_t threads, const F32Const& k, const StateBufs& s,
                        const F32Bufs& f, const ListBufs& l, cudaStream_t st) {
    if (n) k_density_f32<<<blocks_for(n, threads), threads, 0, st>>>(n, k, s, f, l);
}

void launch_pressure_f32(uint32_t n, const F32Const& k, const Tanks& tk, const StateBufs& s,
                         const F32Bufs& f, cudaStream_t st) {
    if (!n) return;
    if (k.adapt_sound_speed) k_vmax_f32<<<blocks_for(n, 256), 256, 0, st>>>(n, tk, s, f);
    k_pressure_f32<<<blocks_for(n, 256), 256, 0, st>>>(n, k, tk, s, f);
}

void launch_forces_f32(uint32_t n, uint32_t threads, const F32Const& k, const Tanks& tk,
                       const StateBufs& s, const F32Bufs& f, const ListBufs& l, float dt,
                       double4* pos_next, double4* vel_next, float* bf, cudaStream_t st) {
    if (!n) return;
    if (bf) cudaMemsetAsync(bf, 0, sizeof(float) * 4 * (size_t)n, st);
    const uint32_t b = blocks_for(n, threads);
    if (k.dim == 3)
        k_forces_f32<3><<<b, threads, 0, st>>>(n, k, tk, s, f, l, dt, pos_next, vel_next, bf);
    else
        k_forces_f32<2><<<b, threads, 0, st>>>(n, k, tk, s, f, l, dt, pos_next, vel_next, bf);
    if (bf) k_bf_to_f64<<<blocks_for(n, 256), 256, 0, st>>>(n, bf, s);
}

void launch_xsph_f32(uint32_t n, uint32_t threads, const F32Const& k, const StateBufs& s,
                     const F32Bufs& f, const ListBufs& l, float4* vel_out, cudaStream_t st,
                     bool use_w) {
    if (!n) return;
    const bool w = use_w && l.wpair32;
    if (w) k_xsph_f32_w<<<blocks_for(n, threads), threads, 0, st>>>(n, k, s, f, l, vel_out);
    k_xsph_f32<<<blocks_for(n, threads), threads, 0, st>>>(n, k, s, f, l, vel_out, w);
}

}  // namespace pe
