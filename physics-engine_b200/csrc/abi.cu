// extern "C" boundary of the B200 WCSPH step (declared in
// include/pe_fluid_wcsph.h). Every entry point catches C++ exceptions and
// maps them to pe-ffi's integer codes (crates/pe-ffi/src/lib.rs:68-80,
// crates/pe-ffi/src/error.rs:4-16); nothing unwinds across the boundary.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <stdexcept>
#include <vector>

#include "../../include/pe_fluid_wcsph.h"
#include "pe_math.cuh"
#include "handles.cuh"
#include "kernel_any.cuh"
#include "coupling.cuh"
#include "world.cuh"

using namespace peabi;

namespace {

void push(PeParticles* p, const double* x, const double* v, uint8_t kind, double psi,
          const double* n) {
    p->x.insert(p->x.end(), x, x + 3);
    const double z3[3] = {0.0, 0.0, 0.0};
    p->v.insert(p->v.end(), v ? v : z3, (v ? v : z3) + 3);
    p->kind.push_back(kind);
    p->psi.push_back(psi);
    p->n_out.insert(p->n_out.end(), n ? n : z3, (n ? n : z3) + 3);
}

// xoshiro256** with SplitMix64 seeding (Blackman & Vigna; pe-math rng.rs:14-72)
struct Xoshiro256ss {
    uint64_t s[4];
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    explicit Xoshiro256ss(uint64_t seed) {
        uint64_t sm = seed;
        for (int i = 0; i < 4; ++i) {
            sm += 0x9e3779b97f4a7c15ULL;
            uint64_t z = sm;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
            s[i] = z ^ (z >> 31);
        }
        if (!(s[0] | s[1] | s[2] | s[3])) s[0] = 0x9e3779b97f4a7c15ULL;
    }
    uint64_t next() {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform(double lo, double hi) {
        double u = (double)(next() >> 11) * (1.0 / (double)(1ULL << 53));
        return lo + (hi - lo) * u;
    }
};

pe::WorldParams to_world(const PeWcsphParams& p) {
    pe::WorldParams w{};
    w.kernel = p.density_kernel;
    w.eos_rest_density = p.eos_rest_density;
    w.eos_sound_speed = p.eos_sound_speed;
    w.eos_gamma = p.eos_gamma;
    w.visc_alpha = p.visc_alpha;
    w.visc_beta = p.visc_beta;
    w.visc_eps = p.visc_eps;
    w.xsph_epsilon = p.xsph_epsilon;
    for (int i = 0; i < 3; ++i) w.gravity[i] = p.gravity[i];
    w.adapt_sound_speed = p.adapt_sound_speed;
    w.surface_tension_sigma = p.surface_tension_sigma;
    w.surface_tension_model = p.surface_tension_model;
    w.surface_tension_colour_gamma = p.surface_tension_colour_gamma;
    return w;
}

PeWcsphParams from_world(const pe::WorldParams& w) {
    PeWcsphParams p{};
    p.density_kernel = w.kernel;
    p.eos_rest_density = w.eos_rest_density;
    p.eos_sound_speed = w.eos_sound_speed;
    p.eos_gamma = w.eos_gamma;
    p.visc_alpha = w.visc_alpha;
    p.visc_beta = w.visc_beta;
    p.visc_eps = w.visc_eps;
    p.xsph_epsilon = w.xsph_epsilon;
    for (int i = 0; i < 3; ++i) p.gravity[i] = w.gravity[i];
    p.adapt_sound_speed = w.adapt_sound_speed;
    p.surface_tension_sigma = w.surface_tension_sigma;
    p.surface_tension_model = w.surface_tension_model;
    p.surface_tension_colour_gamma = w.surface_tension_colour_gamma;
    return p;
}

int check_params(const PeWcsphParams* p) {
    if (!p) return PE_ERR_NULL;
    if (p->density_kernel < PE_KERNEL_CUBIC_SPLINE || p->density_kernel > PE_KERNEL_SPIKY) return PE_ERR_ARG;
    if (!std::isfinite(p->surface_tension_sigma) || !std::isfinite(p->surface_tension_colour_gamma))
        return PE_ERR_ARG;
    if (p->surface_tension_model < PE_SURFACE_TENSION_NONE || p->surface_tension_model > PE_SURFACE_TENSION_COLOUR_FIELD)
        return PE_ERR_ARG;
    const double v[] = {p->eos_rest_density, p->eos_sound_speed, p->eos_gamma, p->visc_alpha,
                        p->visc_beta,        p->visc_eps,        p->xsph_epsilon};
    for (double d : v)
        if (!std::isfinite(d)) return PE_ERR_ARG;
    if (!finite3(p->gravity)) return PE_ERR_ARG;
    if (!(p->eos_rest_density > 0.0) || !(p->eos_gamma != 0.0)) return PE_ERR_ARG;
    return PE_OK;
}



}  // namespace

extern "C" {

// ---------------------------------------------------------------- particles
PeParticles* pe_fluid_particles_new(int32_t dim, double rest_density, double mass, double h) {
    if (!valid_dim(dim) || !std::isfinite(rest_density) || !std::isfinite(mass) || !std::isfinite(h))
        return nullptr;
    try {
        PeParticles* p = new PeParticles();
        p->dim = dim;
        p->rest_density = rest_density;
        p->mass = mass;
        p->h = h;
        return p;
    } catch (...) {
        return nullptr;
    }
}

void pe_fluid_particles_free(PeParticles* p) { delete p; }

int pe_fluid_particles_len(const PeParticles* p, uint64_t* out_len) {
    if (!p || !out_len) return PE_ERR_NULL;
    *out_len = p->len();
    return PE_OK;
}

int pe_fluid_particles_push_fluid(PeParticles* p, const double x[3], const double v[3]) {
    if (!p || !x) return PE_ERR_NULL;
    if (!finite3(x) || (v && !finite3(v))) return PE_ERR_ARG;
    return guard([&] {
        push(p, x, v, PE_PARTICLE_FLUID, 0.0, nullptr);
        return PE_OK;
    });
}

int pe_fluid_particles_push_boundary(PeParticles* p, const double x[3], double psi) {
    return pe_fluid_particles_push_boundary_oriented(p, x, psi, nullptr);
}

int pe_fluid_particles_push_boundary_oriented(PeParticles* p, const double x[3], double psi,
                                              const double n_out[3]) {
    if (!p || !x) return PE_ERR_NULL;
    if (!finite3(x) || !std::isfinite(psi) || (n_out && !finite3(n_out))) return PE_ERR_ARG;
    return guard([&] {
        push(p, x, nullptr, PE_PARTICLE_BOUNDARY, psi, n_out);
        return PE_OK;
    });
}

// particles.rs:220 fill_box: iz -> iy -> ix, position origin + i * dx.
int pe_fluid_fill_box(PeParticles* p, const double origin[3], uint64_t nx, uint64_t ny, uint64_t nz,
                      double dx, const double v0[3]) {
    if (!p || !origin) return PE_ERR_NULL;
    if (!finite3(origin) || !std::isfinite(dx) || (v0 && !finite3(v0))) return PE_ERR_ARG;
    if (p->dim == PE_DIM_2) nz = 1;
    if ((double)nx * (double)ny * (double)nz + (double)p->len() > (double)pe::kMaxParticles)
        return PE_ERR_BOUNDS;
    return guard([&] {
        for (uint64_t iz = 0; iz < nz; ++iz)
            for (uint64_t iy = 0; iy < ny; ++iy)
                for (uint64_t ix = 0; ix < nx; ++ix) {
                    const double x[3] = {origin[0] + (double)ix * dx, origin[1] + (double)iy * dx,
                                         origin[2] + (double)iz * dx};
                    push(p, x, v0, PE_PARTICLE_FLUID, 0.0, nullptr);
                }
        return PE_OK;
    });
}

// particles.rs:286 fill_box_boundary: six faces (four in 2-D) at spacing dx,
// provisional psi = dx^d; f64::round rounds half away from zero like std::round.
int pe_fluid_fill_box_boundary(PeParticles* p, const double mn[3], const double mx[3], double dx,
                               uint64_t layers) {
    if (!p || !mn || !mx) return PE_ERR_NULL;
    if (!finite3(mn) || !finite3(mx) || !std::isfinite(dx)) return PE_ERR_ARG;
    return guard([&] {
        const double psi = p->dim == PE_DIM_2 ? dx * dx : dx * dx * dx;
        if (layers < 1) layers = 1;
        auto pb = [&](double x, double y, double z) {
            const double q[3] = {x, y, z};
            push(p, q, nullptr, PE_PARTICLE_BOUNDARY, psi, nullptr);
        };
        const uint64_t nx = (uint64_t)std::round((mx[0] - mn[0]) / dx) + 1;
        const uint64_t ny = (uint64_t)std::round((mx[1] - mn[1]) / dx) + 1;
        if (p->dim == PE_DIM_2) {
            for (uint64_t layer = 0; layer < layers; ++layer) {
                const double off = (double)layer * dx;
                for (uint64_t i = 0; i < nx; ++i) {
                    const double x = mn[0] + (double)i * dx;
                    pb(x, mn[1] - off, 0.0);
                    pb(x, mx[1] + off, 0.0);
                }
                for (uint64_t j = 1; j + 1 < ny; ++j) {
                    const double y = mn[1] + (double)j * dx;
                    pb(mn[0] - off, y, 0.0);
                    pb(mx[0] + off, y, 0.0);
                }
            }
            return PE_OK;
        }
        const uint64_t nz = (uint64_t)std::round((mx[2] - mn[2]) / dx) + 1;
        for (uint64_t layer = 0; layer < layers; ++layer) {
            const double off = (double)layer * dx;
            for (uint64_t i = 0; i < nx; ++i)
                for (uint64_t j = 0; j < ny; ++j) {
                    const double x = mn[0] + (double)i * dx, y = mn[1] + (double)j * dx;
                    pb(x, y, mn[2] - off);
                    pb(x, y, mx[2] + off);
                }
            for (uint64_t i = 0; i < nx; ++i)
                for (uint64_t k = 1; k + 1 < nz; ++k) {
                    const double x = mn[0] + (double)i * dx, z = mn[2] + (double)k * dx;
                    pb(x, mn[1] - off, z);
                    pb(x, mx[1] + off, z);
                }
            for (uint64_t j = 1; j + 1 < ny; ++j)
                for (uint64_t k = 1; k + 1 < nz; ++k) {
                    const double y = mn[1] + (double)j * dx, z = mn[2] + (double)k * dx;
                    pb(mn[0] - off, y, z);
                    pb(mx[0] + off, y, z);
                }
        }
        if (p->len() > pe::kMaxParticles) throw std::length_error("too many particles");
        return PE_OK;
    });
}

// particles.rs:252: psi_b = 1 / (W(0) + sum over other boundary samples within
// support, in ascending index). Candidates come from a key-sorted grid of the
// boundary samples, then are sorted by index, which keeps the reference's
// summation order at O(N_b * neighbours) cost instead of O(N_b^2).
int pe_fluid_recomputed_akinci_psi(PeParticles* p, int32_t kernel) {
    if (!p) return PE_ERR_NULL;
    if (kernel != PE_KERNEL_CUBIC_SPLINE) return PE_ERR_UNSUPPORTED;
    return guard([&] {
        const double h = p->h;
        const double support = 2.0 * h;
        const double alpha = pe::cubic_alpha(h, p->dim);
        const double w0 = pe::cubic_w(0.0, h, alpha);
        std::vector<uint64_t> bound;
        for (uint64_t i = 0; i < p->len(); ++i)
            if (p->kind[i] == PE_PARTICLE_BOUNDARY) bound.push_back(i);
        // cells slightly larger than the support, so rounding of x / cell can
        // never push an in-support pair two cells apart
        const double inv = 1.0 / (support * (1.0 + 1e-6));
        struct Key {
            int64_t x, y, z;
            uint64_t idx;
        };
        std::vector<Key> keys(bound.size());
        for (size_t a = 0; a < bound.size(); ++a) {
            const double* q = &p->x[3 * bound[a]];
            keys[a] = Key{(int64_t)std::floor(q[0] * inv), (int64_t)std::floor(q[1] * inv),
                          (int64_t)std::floor(q[2] * inv), bound[a]};
        }
        std::vector<Key> sorted = keys;
        auto lt = [](const Key& a, const Key& b) {
            if (a.x != b.x) return a.x < b.x;
            if (a.y != b.y) return a.y < b.y;
            if (a.z != b.z) return a.z < b.z;
            return a.idx < b.idx;
        };
        std::sort(sorted.begin(), sorted.end(), lt);
        std::vector<double> psi_new(bound.size());
        std::vector<uint64_t> cand;
        for (size_t a = 0; a < bound.size(); ++a) {
            const Key& k = keys[a];
            cand.clear();
            for (int64_t dx = -1; dx <= 1; ++dx)
                for (int64_t dy = -1; dy <= 1; ++dy)
                    for (int64_t dz = -1; dz <= 1; ++dz) {
                        Key lo{k.x + dx, k.y + dy, k.z + dz, 0};
                        auto it = std::lower_bound(sorted.begin(), sorted.end(), lo, lt);
                        for (; it != sorted.end() && it->x == lo.x && it->y == lo.y && it->z == lo.z; ++it)
                            if (it->idx != k.idx) cand.push_back(it->idx);
                    }
            std::sort(cand.begin(), cand.end());
            const double* xb = &p->x[3 * k.idx];
            double delta = w0;
            for (uint64_t j : cand) {
                const double* xj = &p->x[3 * j];
                double dx = xj[0] - xb[0], dy = xj[1] - xb[1], dz = xj[2] - xb[2];
                double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                if (r < support) delta += pe::cubic_w(r, h, alpha);
            }
            psi_new[a] = delta > 1e-30 ? 1.0 / delta : 0.0;
        }
        for (size_t a = 0; a < bound.size(); ++a) p->psi[bound[a]] = psi_new[a];
        return PE_OK;
    });
}

int pe_fluid_particles_jitter_fluid(PeParticles* p, uint64_t seed, double amplitude) {
    if (!p) return PE_ERR_NULL;
    if (!std::isfinite(amplitude)) return PE_ERR_ARG;
    Xoshiro256ss r(seed);
    for (uint64_t i = 0; i < p->len(); ++i) {
        if (p->kind[i] != PE_PARTICLE_FLUID) continue;
        double jx = r.uniform(-amplitude, amplitude);
        double jy = r.uniform(-amplitude, amplitude);
        double jz = p->dim == PE_DIM_3 ? r.uniform(-amplitude, amplitude) : 0.0;
        p->x[3 * i] = p->x[3 * i] + jx;
        p->x[3 * i + 1] = p->x[3 * i + 1] + jy;
        p->x[3 * i + 2] = p->x[3 * i + 2] + jz;
    }
    return PE_OK;
}

int pe_fluid_rng_uniform(uint64_t seed, double lo, double hi, uint64_t count, double* out) {
    if (count && !out) return PE_ERR_NULL;
    if (!(std::isfinite(lo) && std::isfinite(hi))) return PE_ERR_ARG;
    Xoshiro256ss r(seed);
    for (uint64_t i = 0; i < count; ++i) out[i] = r.uniform(lo, hi);
    return PE_OK;
}

int pe_fluid_particles_export(const PeParticles* p, double* x, double* v, uint8_t* kind, double* psi,
                              double* n_out, uint64_t n) {
    if (!p) return PE_ERR_NULL;
    if (n != p->len()) return PE_ERR_BOUNDS;
    if (n == 0) return PE_OK;
    if (x) std::memcpy(x, p->x.data(), sizeof(double) * 3 * n);
    if (v) std::memcpy(v, p->v.data(), sizeof(double) * 3 * n);
    if (kind) std::memcpy(kind, p->kind.data(), n);
    if (psi) std::memcpy(psi, p->psi.data(), sizeof(double) * n);
    if (n_out) std::memcpy(n_out, p->n_out.data(), sizeof(double) * 3 * n);
    return PE_OK;
}

double pe_fluid_mass_from_spacing(double rest_density, double dx, int32_t dim) {
    return dim == PE_DIM_2 ? rest_density * dx * dx : rest_density * dx * dx * dx;
}

// particles.rs:178 mass_calibrated_to_rest (cubic spline)
double pe_fluid_mass_calibrated_to_rest(double rest_density, double dx, double h, int32_t dim,
                                        int32_t kernel) {
    if (kernel != PE_KERNEL_CUBIC_SPLINE || !valid_dim(dim)) return NAN;
    const double support = 2.0 * h;
    const double alpha = pe::cubic_alpha(h, dim);
    const int n = (int)std::ceil(support / dx) + 1;
    double sum_w = pe::cubic_w(0.0, h, alpha);
    for (int ix = -n; ix <= n; ++ix)
        for (int iy = -n; iy <= n; ++iy) {
            const int z0 = dim == PE_DIM_2 ? 0 : -n, z1 = dim == PE_DIM_2 ? 0 : n;
            for (int iz = z0; iz <= z1; ++iz) {
                if (ix == 0 && iy == 0 && iz == 0) continue;
                const double r = std::sqrt(((double)ix * dx) * ((double)ix * dx) +
                                           ((double)iy * dx) * ((double)iy * dx) +
                                           ((double)iz * dx) * ((double)iz * dx));
                if (r < support) sum_w += pe::cubic_w(r, h, alpha);
            }
        }
    return sum_w < 1e-30 ? pe_fluid_mass_from_spacing(rest_density, dx, dim) : rest_density / sum_w;
}

// ---------------------------------------------------------------- world
int pe_fluid_wcsph_params_water(double rest_density, double sound_speed, const double gravity[3],
                                PeWcsphParams* out) {
    if (!out || !gravity) return PE_ERR_NULL;
    PeWcsphParams p{};
    p.density_kernel = PE_KERNEL_CUBIC_SPLINE;
    p.eos_rest_density = rest_density;
    p.eos_sound_speed = sound_speed;
    p.eos_gamma = 7.0;                 // eos.rs:25 TAIT_GAMMA_WATER
    p.visc_alpha = 0.01;               // viscosity.rs:39-45
    p.visc_beta = 0.0;
    p.visc_eps = 0.01;
    p.xsph_epsilon = 0.25;             // viscosity.rs:82-86
    for (int i = 0; i < 3; ++i) p.gravity[i] = gravity[i];
    p.adapt_sound_speed = 1;           // wcsph.rs:50
    p.surface_tension_sigma = 0.0;     // wcsph.rs:51 SurfaceTensionParams::disabled()
    p.surface_tension_model = PE_SURFACE_TENSION_NONE;
    p.surface_tension_colour_gamma = 0.0;
    *out = p;
    return PE_OK;
}

int pe_fluid_wcsph_create_from_arrays(const PeWcsphParams* params, int32_t dim, double rest_density,
                                      double mass, double h, uint64_t n, const double* x,
                                      const double* v, const uint8_t* kind, const double* psi,
                                      const double* n_out, const PeWcsphConfig* cfg, PeWcsph** out) {
    return pe_fluid_wcsph_create_batch(params, dim, rest_density, mass, h, n, x, v, kind, psi, n_out,
                                       1, nullptr, cfg, out);
}

int pe_fluid_wcsph_create_batch(const PeWcsphParams* params, int32_t dim, double rest_density,
                                double mass, double h, uint64_t n, const double* x, const double* v,
                                const uint8_t* kind, const double* psi, const double* n_out,
                                uint32_t n_tanks, const uint64_t* tank_offsets,
                                const PeWcsphConfig* cfg, PeWcsph** out) {
    if (!out) return PE_ERR_NULL;
    *out = nullptr;
    if (n_tanks == 0) return PE_ERR_ARG;
    if (n_tanks > 65535u) return PE_ERR_BOUNDS;
    if (n_tanks > 1 && !tank_offsets) return PE_ERR_NULL;
    if (tank_offsets) {
        if (tank_offsets[0] != 0 || tank_offsets[n_tanks] != n) return PE_ERR_ARG;
        for (uint32_t t = 0; t < n_tanks; ++t)
            if (tank_offsets[t + 1] <= tank_offsets[t]) return PE_ERR_ARG;
    }
    *out = nullptr;
    int rc = check_params(params);
    if (rc != PE_OK) return rc;
    if (cfg && cfg->precision == PE_PRECISION_F32 &&
        (params->surface_tension_sigma != 0.0 || params->density_kernel != PE_KERNEL_CUBIC_SPLINE))
        return PE_ERR_UNSUPPORTED;  // the single-precision form: cubic spline, no surface tension
    if (!valid_dim(dim)) return PE_ERR_ARG;
    if (!(std::isfinite(rest_density) && rest_density > 0.0 && std::isfinite(mass) && mass > 0.0 &&
          std::isfinite(h) && h > 0.0))
        return PE_ERR_ARG;
    if (n > pe::kMaxParticles) return PE_ERR_BOUNDS;
    if (n && (!x || !kind)) return PE_ERR_NULL;
    for (uint64_t i = 0; i < n; ++i) {
        if (!finite3(x + 3 * i) || (v && !finite3(v + 3 * i))) return PE_ERR_ARG;
        if (kind[i] > 1) return PE_ERR_ARG;
        if (psi && !std::isfinite(psi[i])) return PE_ERR_ARG;
        if (n_out && !finite3(n_out + 3 * i)) return PE_ERR_ARG;
    }
    return guard([&] {
        std::vector<double> zero;
        const double* ps = psi;
        if (!ps) {
            zero.assign(n ? n : 1, 0.0);
            ps = zero.data();
        }
        pe::WorldConfig wc = to_config(cfg);
        wc.pair_weights = 1;
        auto* w = new pe::World(to_world(*params), wc, dim, rest_density, mass, h, n, x, v, kind, ps,
                                n_out, tank_offsets, n_tanks);
        *out = new PeWcsph{w};
        return PE_OK;
    });
}

int pe_fluid_wcsph_create(const PeParticles* particles, const PeWcsphParams* params,
                          const PeWcsphConfig* cfg, PeWcsph** out) {
    if (!particles) return PE_ERR_NULL;
    const PeParticles& p = *particles;
    return pe_fluid_wcsph_create_from_arrays(params, p.dim, p.rest_density, p.mass, p.h, p.len(),
                                             p.x.data(), p.v.data(), p.kind.data(), p.psi.data(),
                                             p.n_out.data(), cfg, out);
}

void pe_fluid_wcsph_destroy(PeWcsph* w) {
    if (!w) return;
    try {
        delete w->world;
    } catch (...) {
    }
    delete w;
}

int pe_fluid_wcsph_step(PeWcsph* w, double dt) {
    if (!w) return PE_ERR_NULL;
    if (!(std::isfinite(dt) && dt > 0.0)) return PE_ERR_ARG;
    return guard([&] {
        w->world->step(dt);
        return status_code(w->world->status());
    });
}

int pe_fluid_wcsph_run(PeWcsph* w, double dt, uint64_t steps) {
    if (!w) return PE_ERR_NULL;
    if (!(std::isfinite(dt) && dt > 0.0)) return PE_ERR_ARG;
    return guard([&] {
        w->world->run(dt, steps);
        return status_code(w->world->status());
    });
}

#define PE_PHASE(name)                             \
    int pe_fluid_wcsph_##name(PeWcsph* w) {        \
        if (!w) return PE_ERR_NULL;                \
        return guard([&] {                         \
            w->world->name();                      \
            w->world->synchronize();               \
            return status_code(w->world->status()); \
        });                                        \
    }
PE_PHASE(rebuild_grid)
PE_PHASE(compute_density)
PE_PHASE(compute_pressure)
PE_PHASE(compute_forces)
PE_PHASE(apply_xsph)
#undef PE_PHASE

int pe_fluid_wcsph_len(const PeWcsph* w, uint64_t* out_len) {
    if (!w || !out_len) return PE_ERR_NULL;
    *out_len = w->world->len();
    return PE_OK;
}

int pe_fluid_wcsph_get_time(const PeWcsph* w, double* t) {
    if (!w || !t) return PE_ERR_NULL;
    *t = w->world->time();
    return PE_OK;
}

int pe_fluid_wcsph_set_time(PeWcsph* w, double t) {
    if (!w) return PE_ERR_NULL;
    if (!std::isfinite(t)) return PE_ERR_ARG;
    w->world->set_time(t);
    return PE_OK;
}

int pe_fluid_wcsph_get_sound_speed(PeWcsph* w, double* c) {
    if (!w || !c) return PE_ERR_NULL;
    return guard([&] {
        *c = w->world->sound_speed();
        return PE_OK;
    });
}

int pe_fluid_wcsph_tanks(PeWcsph* w, uint32_t* n_tanks) {
    if (!w || !n_tanks) return PE_ERR_NULL;
    *n_tanks = w->world->tanks();
    return PE_OK;
}

int pe_fluid_wcsph_get_sound_speeds(PeWcsph* w, double* out, uint32_t n_tanks) {
    if (!w || !out) return PE_ERR_NULL;
    if (n_tanks != w->world->tanks()) return PE_ERR_BOUNDS;
    return guard([&] {
        w->world->get_sound_speeds(out);
        return PE_OK;
    });
}

int pe_fluid_wcsph_autotune(PeWcsph* w, uint32_t out[4]) {
    if (!w) return PE_ERR_NULL;
    return guard([&] {
        const pe::World::Shapes r = w->world->autotune();
        if (out) {
            out[0] = r.density;
            out[1] = r.forces;
            out[2] = r.xsph;
            out[3] = r.list_ctas_per_sm;
        }
        return status_code(w->world->status());
    });
}

int pe_fluid_wcsph_shapes(PeWcsph* w, uint32_t out[4]) {
    if (!w || !out) return PE_ERR_NULL;
    const pe::World::Shapes r = w->world->shapes();
    out[0] = r.density;
    out[1] = r.forces;
    out[2] = r.xsph;
    out[3] = r.list_ctas_per_sm;
    return PE_OK;
}

int pe_fluid_wcsph_list_chunk(PeWcsph* w, uint32_t* out) {
    if (!w || !out) return PE_ERR_NULL;
    *out = w->world->shapes().list_chunk;
    return PE_OK;
}

int pe_fluid_wcsph_set_pair_weights(PeWcsph* w, int32_t on) {
    if (!w) return PE_ERR_NULL;
    return guard([&] {
        w->world->set_pair_weights(on != 0);
        return PE_OK;
    });
}

int pe_fluid_wcsph_pair_weights(PeWcsph* w, int32_t* out) {
    if (!w || !out) return PE_ERR_NULL;
    *out = w->world->pair_weights() ? 1 : 0;
    return PE_OK;
}

int pe_fluid_wcsph_pair_weight_info(PeWcsph* w, uint64_t out[3]) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        w->world->pair_weight_info(out);
        return PE_OK;
    });
}

int pe_fluid_wcsph_get_params(PeWcsph* w, PeWcsphParams* out) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        w->world->sound_speed();  // refresh the persisted c
        *out = from_world(w->world->params());
        return PE_OK;
    });
}

int pe_fluid_wcsph_set_params(PeWcsph* w, const PeWcsphParams* params) {
    if (!w) return PE_ERR_NULL;
    int rc = check_params(params);
    if (rc != PE_OK) return rc;
    if (w->world->single_precision() &&
        (params->surface_tension_sigma != 0.0 || params->density_kernel != PE_KERNEL_CUBIC_SPLINE))
        return PE_ERR_UNSUPPORTED;
    return guard([&] {
        w->world->set_params(to_world(*params));
        return PE_OK;
    });
}

#define PE_GET_VEC(name, which)                                       \
    int pe_fluid_wcsph_##name(PeWcsph* w, double* out, uint64_t n) { \
        if (!w || !out) return PE_ERR_NULL;                          \
        if (n != w->world->len()) return PE_ERR_BOUNDS;              \
        return guard([&] {                                           \
            w->world->get_vec(which, out);                           \
            return PE_OK;                                            \
        });                                                          \
    }
PE_GET_VEC(get_positions, 0)
PE_GET_VEC(get_velocities, 1)
PE_GET_VEC(get_accelerations, 2)
PE_GET_VEC(get_boundary_forces, 3)
#undef PE_GET_VEC

int pe_fluid_wcsph_get_densities(PeWcsph* w, double* out, uint64_t n) {
    if (!w || !out) return PE_ERR_NULL;
    if (n != w->world->len()) return PE_ERR_BOUNDS;
    return guard([&] {
        w->world->get_scalar(0, out);
        return PE_OK;
    });
}

int pe_fluid_wcsph_get_pressures(PeWcsph* w, double* out, uint64_t n) {
    if (!w || !out) return PE_ERR_NULL;
    if (n != w->world->len()) return PE_ERR_BOUNDS;
    return guard([&] {
        w->world->get_scalar(1, out);
        return PE_OK;
    });
}

int pe_fluid_wcsph_get_kinds(PeWcsph* w, uint8_t* out, uint64_t n) {
    if (!w || !out) return PE_ERR_NULL;
    if (n != w->world->len()) return PE_ERR_BOUNDS;
    return guard([&] {
        w->world->get_kind(out);
        return PE_OK;
    });
}

int pe_fluid_wcsph_set_positions(PeWcsph* w, const double* in, uint64_t n) {
    if (!w || !in) return PE_ERR_NULL;
    if (n != w->world->len()) return PE_ERR_BOUNDS;
    return guard([&] { return w->world->set_vec(0, in) ? PE_OK : PE_ERR_ARG; });
}

int pe_fluid_wcsph_set_velocities(PeWcsph* w, const double* in, uint64_t n) {
    if (!w || !in) return PE_ERR_NULL;
    if (n != w->world->len()) return PE_ERR_BOUNDS;
    return guard([&] { return w->world->set_vec(1, in) ? PE_OK : PE_ERR_ARG; });
}

int pe_fluid_wcsph_set_densities(PeWcsph* w, const double* in, uint64_t n) {
    if (!w || !in) return PE_ERR_NULL;
    if (n != w->world->len()) return PE_ERR_BOUNDS;
    for (uint64_t i = 0; i < n; ++i)
        if (!std::isfinite(in[i])) return PE_ERR_ARG;
    return guard([&] {
        w->world->set_scalar(0, in);
        return PE_OK;
    });
}

int pe_fluid_wcsph_set_pressures(PeWcsph* w, const double* in, uint64_t n) {
    if (!w || !in) return PE_ERR_NULL;
    if (n != w->world->len()) return PE_ERR_BOUNDS;
    for (uint64_t i = 0; i < n; ++i)
        if (!std::isfinite(in[i])) return PE_ERR_ARG;
    return guard([&] {
        w->world->set_scalar(1, in);
        return PE_OK;
    });
}

int pe_fluid_wcsph_get_grid(PeWcsph* w, int32_t* keys, uint64_t* order, uint64_t n,
                            int32_t* occupied, uint64_t* ranges, uint64_t occupied_cap,
                            uint64_t* n_occupied) {
    if (!w) return PE_ERR_NULL;
    if ((keys || order) && n != w->world->len()) return PE_ERR_BOUNDS;
    return guard([&] {
        uint64_t m = 0;
        w->world->get_grid(keys, order, occupied, ranges, occupied_cap, &m);
        if (n_occupied) *n_occupied = m;
        if ((occupied || ranges) && m > occupied_cap) return PE_ERR_BOUNDS;
        return PE_OK;
    });
}

int pe_fluid_wcsph_get_neighbour_counts(PeWcsph* w, uint32_t* candidates, uint32_t* in_support,
                                        uint64_t n) {
    if (!w) return PE_ERR_NULL;
    if (n != w->world->len()) return PE_ERR_BOUNDS;
    return guard([&] {
        w->world->get_neighbour_counts(candidates, in_support);
        return PE_OK;
    });
}

int pe_fluid_wcsph_status(PeWcsph* w, uint32_t* status) {
    if (!w || !status) return PE_ERR_NULL;
    return guard([&] {
        *status = w->world->status();
        return PE_OK;
    });
}

int pe_fluid_wcsph_capacity_info(PeWcsph* w, uint64_t out[8]) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        w->world->capacity_info(out);
        return PE_OK;
    });
}

int pe_fluid_wcsph_clear_status(PeWcsph* w) {
    if (!w) return PE_ERR_NULL;
    return guard([&] {
        w->world->clear_status();
        return PE_OK;
    });
}

int pe_fluid_wcsph_diagnostics(PeWcsph* w, PeFluidDiagnostics* out) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        pe::World::Diagnostics d{};
        w->world->diagnostics(&d);
        PeFluidDiagnostics r{};
        r.total_mass = d.total_mass;
        for (int c = 0; c < 3; ++c) r.linear_momentum[c] = d.linear_momentum[c];
        r.kinetic_energy = d.kinetic_energy;
        r.gravitational_potential = d.gravitational_potential;
        r.mean_density_error = d.mean_density_error;
        r.max_density_error = d.max_density_error;
        r.v_max = d.v_max;
        r.a_max = d.a_max;
        r.hash64 = d.hash64;
        *out = r;
        return PE_OK;
    });
}

int pe_fluid_wcsph_fluid_center_of_mass(PeWcsph* w, double out[3]) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        pe::World::Diagnostics d{};
        w->world->diagnostics(&d);
        for (int c = 0; c < 3; ++c) out[c] = d.fluid_com[c];
        return PE_OK;
    });
}

int pe_fluid_wcsph_stream(PeWcsph* w, void** out) {
    if (!w || !out) return PE_ERR_NULL;
    *out = (void*)w->world->stream();
    return PE_OK;
}

int pe_fluid_wcsph_profile(PeWcsph* w, int32_t enable) {
    if (!w) return PE_ERR_NULL;
    w->world->set_profiling(enable != 0);
    return PE_OK;
}

int pe_fluid_wcsph_profile_read(PeWcsph* w, PeFluidProfile* out, int32_t reset) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        w->world->profile_read(out->ms, out->count, reset != 0);
        return PE_OK;
    });
}

int pe_fluid_wcsph_kernel_launches(PeWcsph* w, uint64_t* out, int32_t reset) {
    if (!w || !out) return PE_ERR_NULL;
    *out = w->world->kernel_launches();
    if (reset) w->world->reset_launch_count();
    return PE_OK;
}

// ---------------------------------------------------------------- helpers
double pe_fluid_kernel_w(int32_t kernel, double r, double h, int32_t dim) {
    if (kernel < PE_KERNEL_CUBIC_SPLINE || kernel > PE_KERNEL_SPIKY || !valid_dim(dim)) return NAN;
    if (h <= 0.0) return 0.0;  // kernels.rs:41
    return pe::kfn_w(pe::make_kernel_fn(kernel, h, dim), r);
}

int pe_fluid_grad_w(int32_t kernel, const double rij[3], double h, int32_t dim, double out[3]) {
    if (!rij || !out) return PE_ERR_NULL;
    if (kernel < PE_KERNEL_CUBIC_SPLINE || kernel > PE_KERNEL_SPIKY || !valid_dim(dim)) return PE_ERR_ARG;
    out[0] = out[1] = out[2] = 0.0;
    if (h <= 0.0) return PE_OK;  // kernels.rs:57
    pe::kfn_grad(pe::make_kernel_fn(kernel, h, dim), rij[0], rij[1], rij[2], &out[0], &out[1], &out[2]);
    return PE_OK;
}

double pe_fluid_tait_pressure(double rest_density, double sound_speed, double gamma, double density) {
    const double ratio = density / rest_density;
    const double b = rest_density * sound_speed * sound_speed / gamma;
    bool is_int = false;
    const int gi = pe::integer_exponent(gamma, &is_int);
    const double pw = is_int ? pe::pow_int_dd(ratio, gi) : std::pow(ratio, gamma);
    return b * (pw - 1.0);
}

double pe_fluid_pi_ij(double alpha, double beta, double eps, double h, double sound_speed,
                      const double xi[3], const double xj[3], const double vi[3], const double vj[3],
                      double rho_i, double rho_j) {
    if (!xi || !xj || !vi || !vj) return NAN;
    const double rx = xi[0] - xj[0], ry = xi[1] - xj[1], rz = xi[2] - xj[2];
    const double wx = vi[0] - vj[0], wy = vi[1] - vj[1], wz = vi[2] - vj[2];
    const double vr = wx * rx + wy * ry + wz * rz;
    if (vr >= 0.0) return 0.0;
    const double r2 = rx * rx + ry * ry + rz * rz;
    const double mu = h * vr / (r2 + eps * h * h);
    const double rho_bar = 0.5 * (rho_i + rho_j);
    return (-alpha * sound_speed * mu + beta * mu * mu) / rho_bar;
}

double pe_fluid_suggested_dt(double h, double sound_speed, double v_max, double a_max,
                             double lambda_v, double lambda_f) {
    const double dt_v = lambda_v * h / std::fmax(sound_speed + v_max, 1e-12);
    const double dt_f = a_max > 1e-12 ? lambda_f * std::sqrt(h / a_max) : INFINITY;
    return std::fmin(dt_v, dt_f);
}

const char* pe_fluid_version(void) { return "physics-engine-b200 wcsph 0.1.0 (sm_100a)"; }

}  // extern "C"

// ---------------------------------------------------------------- coupling

struct PeCoupler {
    pe::Coupler* c;
    PeWcsph* w;
};

int pe_fluid_coupler_create(PeWcsph* w, uint32_t n_bodies, uint64_t n_samples, const int64_t* body,
                            const double* local, const double* local_n, const int64_t* particle,
                            PeCoupler** out) {
    if (!w || !out) return PE_ERR_NULL;
    *out = nullptr;
    if (n_samples && (!body || !local || !local_n || !particle)) return PE_ERR_NULL;
    const uint64_t n = w->world->len();
    for (uint64_t k = 0; k < n_samples; ++k) {
        if (body[k] < 0 || (uint64_t)body[k] >= n_bodies || particle[k] < 0 || (uint64_t)particle[k] >= n)
            return PE_ERR_BOUNDS;
        if (!finite3(local + 3 * k) || !finite3(local_n + 3 * k)) return PE_ERR_ARG;
    }
    return guard([&] {
        *out = new PeCoupler{new pe::Coupler(*w->world, n_bodies, n_samples, body, local, local_n, particle), w};
        return PE_OK;
    });
}

void pe_fluid_coupler_destroy(PeCoupler* c) {
    if (!c) return;
    try {
        delete c->c;
    } catch (...) {
    }
    delete c;
}

int pe_fluid_coupler_sync(PeCoupler* c, const double* X, const double* Q, const double* V, const double* omega) {
    if (!c || (c->c->bodies() && (!X || !Q || !V || !omega))) return PE_ERR_NULL;
    for (uint32_t b = 0; b < c->c->bodies(); ++b)
        if (!finite3(X + 3 * b) || !finite3(V + 3 * b) || !finite3(omega + 3 * b) || !finite3(Q + 4 * b) ||
            !std::isfinite(Q[4 * b + 3]))
            return PE_ERR_ARG;
    return guard([&] {
        c->c->sync(X, Q, V, omega);
        return PE_OK;
    });
}

int pe_fluid_coupler_reduce(PeCoupler* c, const double* X, double* force, double* torque) {
    if (!c || (c->c->bodies() && (!X || !force || !torque))) return PE_ERR_NULL;
    return guard([&] {
        c->c->reduce(X, force, torque);
        return PE_OK;
    });
}
