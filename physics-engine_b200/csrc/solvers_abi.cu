// C ABI of the sibling solvers that share the WCSPH world's grid, lists and
// state: Position Based Fluids (pbf.rs) and divergence-free SPH (dfsph.rs).
// Same conventions as abi.cu: pe-ffi
// error codes, no unwinding across the boundary, caller-owned host buffers in
// original particle order.
#include <cmath>
#include <cstring>

#include "dfsph.cuh"
#include "handles.cuh"
#include "pbf.cuh"

using namespace peabi;

struct PePbf {
    pe::PbfSolver* s;
};

struct PeDfsph {
    pe::DfsphSolver* s;
};

namespace {

int check_pbf(const PePbfParams* p) {
    if (!p) return PE_ERR_NULL;
    if (p->density_kernel < 0 || p->density_kernel > 3 || p->grad_kernel < 0 || p->grad_kernel > 3)
        return PE_ERR_ARG;
    const double v[] = {p->epsilon_lambda, p->art_pressure_k, p->art_pressure_n, p->art_pressure_dq_over_h,
                        p->viscosity_eps, p->vorticity_eps};
    for (double d : v)
        if (!std::isfinite(d)) return PE_ERR_ARG;
    if (!finite3(p->gravity)) return PE_ERR_ARG;
    if (p->iterations > (1u << 20)) return PE_ERR_BOUNDS;
    return PE_OK;
}

pe::PbfParams to_pbf(const PePbfParams& p) {
    pe::PbfParams q{};
    q.density_kernel = p.density_kernel;
    q.grad_kernel = p.grad_kernel;
    q.iterations = p.iterations;
    q.epsilon_lambda = p.epsilon_lambda;
    q.art_pressure_k = p.art_pressure_k;
    q.art_pressure_n = p.art_pressure_n;
    q.art_pressure_dq_over_h = p.art_pressure_dq_over_h;
    q.viscosity_eps = p.viscosity_eps;
    q.vorticity_eps = p.vorticity_eps;
    for (int a = 0; a < 3; ++a) q.gravity[a] = p.gravity[a];
    q.reuse_neighbours = p.reuse_neighbours;
    return q;
}

PePbfParams from_pbf(const pe::PbfParams& q) {
    PePbfParams p{};
    p.density_kernel = q.density_kernel;
    p.grad_kernel = q.grad_kernel;
    p.iterations = q.iterations;
    p.epsilon_lambda = q.epsilon_lambda;
    p.art_pressure_k = q.art_pressure_k;
    p.art_pressure_n = q.art_pressure_n;
    p.art_pressure_dq_over_h = q.art_pressure_dq_over_h;
    p.viscosity_eps = q.viscosity_eps;
    p.vorticity_eps = q.vorticity_eps;
    for (int a = 0; a < 3; ++a) p.gravity[a] = q.gravity[a];
    p.reuse_neighbours = q.reuse_neighbours;
    return p;
}

int check_dfsph(const PeDfsphParams* p) {
    if (!p) return PE_ERR_NULL;
    if (p->kernel < 0 || p->kernel > 3) return PE_ERR_ARG;
    const double v[] = {p->density_error_tol, p->divergence_error_tol, p->xsph_epsilon, p->particle_diameter,
                        p->cfl_lambda, p->solver_omega, p->max_velocity_correction};
    for (double d : v)
        if (!std::isfinite(d)) return PE_ERR_ARG;
    for (int k = 0; k < 4; ++k)
        if (p->free_slip_set[k] && !std::isfinite(p->free_slip[k])) return PE_ERR_ARG;
    if (!finite3(p->gravity)) return PE_ERR_ARG;
    if (p->max_density_iters > (1u << 20) || p->max_divergence_iters > (1u << 20)) return PE_ERR_BOUNDS;
    return PE_OK;
}

pe::DfsphParams to_dfsph(const PeDfsphParams& p) {
    pe::DfsphParams q{};
    q.kernel = p.kernel;
    q.max_density_iters = p.max_density_iters;
    q.max_divergence_iters = p.max_divergence_iters;
    q.density_error_tol = p.density_error_tol;
    q.divergence_error_tol = p.divergence_error_tol;
    for (int a = 0; a < 3; ++a) q.gravity[a] = p.gravity[a];
    q.xsph_epsilon = p.xsph_epsilon;
    q.particle_diameter = p.particle_diameter;
    q.cfl_lambda = p.cfl_lambda;
    q.adaptive_dt = p.adaptive_dt;
    q.warm_start = p.warm_start;
    for (int k = 0; k < 4; ++k) {
        q.has_slip[k] = p.free_slip_set[k] ? 1 : 0;
        q.slip[k] = p.free_slip[k];
    }
    q.solver_omega = p.solver_omega;
    q.max_velocity_correction = p.max_velocity_correction;
    return q;
}

PeDfsphParams from_dfsph(const pe::DfsphParams& q) {
    PeDfsphParams p{};
    p.kernel = q.kernel;
    p.max_density_iters = q.max_density_iters;
    p.max_divergence_iters = q.max_divergence_iters;
    p.density_error_tol = q.density_error_tol;
    p.divergence_error_tol = q.divergence_error_tol;
    for (int a = 0; a < 3; ++a) p.gravity[a] = q.gravity[a];
    p.xsph_epsilon = q.xsph_epsilon;
    p.particle_diameter = q.particle_diameter;
    p.cfl_lambda = q.cfl_lambda;
    p.adaptive_dt = q.adaptive_dt;
    p.warm_start = q.warm_start;
    for (int k = 0; k < 4; ++k) {
        p.free_slip_set[k] = q.has_slip[k];
        p.free_slip[k] = q.slip[k];
    }
    p.solver_omega = q.solver_omega;
    p.max_velocity_correction = q.max_velocity_correction;
    return p;
}

}  // namespace

extern "C" {

int pe_fluid_pbf_params_default(PePbfParams* out) {
    if (!out) return PE_ERR_NULL;
    PePbfParams p{};
    p.density_kernel = PE_KERNEL_POLY6;
    p.grad_kernel = PE_KERNEL_SPIKY;
    p.iterations = 5;
    p.epsilon_lambda = 0.01;
    p.art_pressure_k = 0.01;
    p.art_pressure_n = 4.0;
    p.art_pressure_dq_over_h = 0.25;
    p.viscosity_eps = 0.01;
    p.vorticity_eps = 0.0;
    p.gravity[0] = 0.0;
    p.gravity[1] = 0.0;
    p.gravity[2] = -9.80665;
    p.reuse_neighbours = 1;
    *out = p;
    return PE_OK;
}

int pe_fluid_pbf_create_from_arrays(const PePbfParams* params, int32_t dim, double rest_density, double mass,
                                    double h, uint64_t n, const double* x, const double* v, const uint8_t* kind,
                                    const double* psi, const double* n_out, const PeWcsphConfig* cfg,
                                    PePbf** out) {
    if (!out) return PE_ERR_NULL;
    *out = nullptr;
    int rc = check_pbf(params);
    if (rc != PE_OK) return rc;
    rc = check_arrays(dim, rest_density, mass, h, n, x, v, kind, psi, n_out);
    if (rc != PE_OK) return rc;
    return guard([&] {
        std::vector<double> zero;
        const double* ps = psi;
        if (!ps) {
            zero.assign(n ? n : 1, 0.0);
            ps = zero.data();
        }
        auto* s = new pe::PbfSolver(to_pbf(*params), to_config(cfg), dim, rest_density, mass, h, n, x, v, kind,
                                    ps, n_out);
        *out = new PePbf{s};
        return PE_OK;
    });
}

int pe_fluid_pbf_create(const PeParticles* particles, const PePbfParams* params, const PeWcsphConfig* cfg,
                        PePbf** out) {
    if (!particles) return PE_ERR_NULL;
    const PeParticles& p = *particles;
    return pe_fluid_pbf_create_from_arrays(params, p.dim, p.rest_density, p.mass, p.h, p.len(), p.x.data(),
                                           p.v.data(), p.kind.data(), p.psi.data(), p.n_out.data(), cfg, out);
}

void pe_fluid_pbf_destroy(PePbf* w) {
    if (!w) return;
    try {
        delete w->s;
    } catch (...) {
    }
    delete w;
}

int pe_fluid_pbf_step(PePbf* w, double dt) {
    if (!w) return PE_ERR_NULL;
    if (!(std::isfinite(dt) && dt >= 0.0)) return PE_ERR_ARG;
    return guard([&] {
        w->s->step(dt);
        return status_code(w->s->world().status());
    });
}

int pe_fluid_pbf_run(PePbf* w, double dt, uint64_t steps) {
    if (!w) return PE_ERR_NULL;
    if (!(std::isfinite(dt) && dt >= 0.0)) return PE_ERR_ARG;
    return guard([&] {
        w->s->run(dt, steps);
        return status_code(w->s->world().status());
    });
}

int pe_fluid_pbf_len(const PePbf* w, uint64_t* out_len) {
    if (!w || !out_len) return PE_ERR_NULL;
    *out_len = w->s->world().len();
    return PE_OK;
}

int pe_fluid_pbf_get_time(const PePbf* w, double* t) {
    if (!w || !t) return PE_ERR_NULL;
    *t = w->s->world().time();
    return PE_OK;
}

int pe_fluid_pbf_get_params(const PePbf* w, PePbfParams* out) {
    if (!w || !out) return PE_ERR_NULL;
    *out = from_pbf(w->s->params());
    return PE_OK;
}

int pe_fluid_pbf_set_params(PePbf* w, const PePbfParams* params) {
    if (!w) return PE_ERR_NULL;
    int rc = check_pbf(params);
    if (rc != PE_OK) return rc;
    return guard([&] {
        w->s->set_params(to_pbf(*params));
        return PE_OK;
    });
}

#define PE_PBF_GET(name, call)                                        \
    int pe_fluid_pbf_##name(PePbf* w, double* out, uint64_t n) {      \
        if (!w || !out) return PE_ERR_NULL;                           \
        if (n != w->s->world().len()) return PE_ERR_BOUNDS;           \
        return guard([&] {                                            \
            call;                                                     \
            return PE_OK;                                             \
        });                                                           \
    }
PE_PBF_GET(get_positions, w->s->world().get_vec(0, out))
PE_PBF_GET(get_velocities, w->s->world().get_vec(1, out))
PE_PBF_GET(get_densities, w->s->world().get_scalar(0, out))
PE_PBF_GET(get_lambdas, w->s->get_lambda(out))
#undef PE_PBF_GET

#define PE_PBF_SET(name, which)                                           \
    int pe_fluid_pbf_##name(PePbf* w, const double* in, uint64_t n) {     \
        if (!w || !in) return PE_ERR_NULL;                                \
        if (n != w->s->world().len()) return PE_ERR_BOUNDS;               \
        return guard([&] {                                                \
            return w->s->world().set_vec(which, in) ? PE_OK : PE_ERR_ARG; \
        });                                                               \
    }
PE_PBF_SET(set_positions, 0)
PE_PBF_SET(set_velocities, 1)
#undef PE_PBF_SET

int pe_fluid_pbf_mean_density_error(PePbf* w, double* out) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        *out = w->s->mean_density_error();
        return PE_OK;
    });
}

int pe_fluid_pbf_v_max(PePbf* w, double* out) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        *out = w->s->v_max();
        return PE_OK;
    });
}

int pe_fluid_pbf_status(PePbf* w, uint32_t* status) {
    if (!w || !status) return PE_ERR_NULL;
    return guard([&] {
        *status = w->s->world().status();
        return PE_OK;
    });
}

int pe_fluid_pbf_stream(PePbf* w, void** out) {
    if (!w || !out) return PE_ERR_NULL;
    *out = (void*)w->s->world().stream();
    return PE_OK;
}

int pe_fluid_pbf_kernel_launches(PePbf* w, uint64_t* out, int32_t reset) {
    if (!w || !out) return PE_ERR_NULL;
    *out = w->s->world().kernel_launches();
    if (reset) w->s->world().reset_launch_count();
    return PE_OK;
}

// ---------------------------------------------------------------- DFSPH
int pe_fluid_dfsph_params_default(PeDfsphParams* out) {
    if (!out) return PE_ERR_NULL;
    PeDfsphParams p{};
    p.kernel = PE_KERNEL_CUBIC_SPLINE;
    p.max_density_iters = 50;
    p.max_divergence_iters = 50;
    p.density_error_tol = 0.001;
    p.divergence_error_tol = 0.001;
    p.gravity[2] = -9.80665;
    p.xsph_epsilon = 0.05;
    p.particle_diameter = 0.0;
    p.cfl_lambda = 0.4;
    p.adaptive_dt = 1;
    p.warm_start = 1;
    p.solver_omega = 1.0;
    p.max_velocity_correction = 0.0;
    *out = p;
    return PE_OK;
}

int pe_fluid_dfsph_create_from_arrays(const PeDfsphParams* params, int32_t dim, double rest_density,
                                      double mass, double h, uint64_t n, const double* x, const double* v,
                                      const uint8_t* kind, const double* psi, const double* n_out,
                                      const PeWcsphConfig* cfg, PeDfsph** out) {
    if (!out) return PE_ERR_NULL;
    *out = nullptr;
    int rc = check_dfsph(params);
    if (rc != PE_OK) return rc;
    rc = check_arrays(dim, rest_density, mass, h, n, x, v, kind, psi, n_out);
    if (rc != PE_OK) return rc;
    return guard([&] {
        std::vector<double> zero;
        const double* ps = psi;
        if (!ps) {
            zero.assign(n ? n : 1, 0.0);
            ps = zero.data();
        }
        auto* s = new pe::DfsphSolver(to_dfsph(*params), to_config(cfg), dim, rest_density, mass, h, n, x, v,
                                      kind, ps, n_out);
        *out = new PeDfsph{s};
        return PE_OK;
    });
}

int pe_fluid_dfsph_create(const PeParticles* particles, const PeDfsphParams* params, const PeWcsphConfig* cfg,
                          PeDfsph** out) {
    if (!particles) return PE_ERR_NULL;
    const PeParticles& p = *particles;
    return pe_fluid_dfsph_create_from_arrays(params, p.dim, p.rest_density, p.mass, p.h, p.len(), p.x.data(),
                                             p.v.data(), p.kind.data(), p.psi.data(), p.n_out.data(), cfg, out);
}

void pe_fluid_dfsph_destroy(PeDfsph* w) {
    if (!w) return;
    try {
        delete w->s;
    } catch (...) {
    }
    delete w;
}

int pe_fluid_dfsph_step(PeDfsph* w, double dt) {
    if (!w) return PE_ERR_NULL;
    if (!std::isfinite(dt)) return PE_ERR_ARG;
    return guard([&] {
        w->s->step(dt);
        return status_code(w->s->world().status());
    });
}

int pe_fluid_dfsph_run(PeDfsph* w, double dt, uint64_t steps) {
    if (!w) return PE_ERR_NULL;
    if (!std::isfinite(dt)) return PE_ERR_ARG;
    return guard([&] {
        w->s->run(dt, steps);
        return status_code(w->s->world().status());
    });
}

int pe_fluid_dfsph_step_adaptive(PeDfsph* w, double* dt_out) {
    if (!w) return PE_ERR_NULL;
    return guard([&] {
        const double dt = w->s->step_adaptive();
        if (dt_out) *dt_out = dt;
        return status_code(w->s->world().status());
    });
}

int pe_fluid_dfsph_suggest_dt(PeDfsph* w, double* out) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        *out = w->s->suggest_dt();
        return PE_OK;
    });
}

#define PE_DF_PHASE(name)                          \
    int pe_fluid_dfsph_##name(PeDfsph* w) {        \
        if (!w) return PE_ERR_NULL;                \
        return guard([&] {                         \
            w->s->name();                          \
            return status_code(w->s->world().status()); \
        });                                        \
    }
PE_DF_PHASE(rebuild_neighbours)
PE_DF_PHASE(compute_density)
PE_DF_PHASE(compute_alpha)
#undef PE_DF_PHASE

int pe_fluid_dfsph_len(const PeDfsph* w, uint64_t* out_len) {
    if (!w || !out_len) return PE_ERR_NULL;
    *out_len = w->s->world().len();
    return PE_OK;
}

int pe_fluid_dfsph_get_time(const PeDfsph* w, double* t) {
    if (!w || !t) return PE_ERR_NULL;
    *t = w->s->world().time();
    return PE_OK;
}

int pe_fluid_dfsph_get_last_dt(const PeDfsph* w, double* out) {
    if (!w || !out) return PE_ERR_NULL;
    *out = w->s->last_dt();
    return PE_OK;
}

int pe_fluid_dfsph_get_params(const PeDfsph* w, PeDfsphParams* out) {
    if (!w || !out) return PE_ERR_NULL;
    *out = from_dfsph(w->s->params());
    return PE_OK;
}

int pe_fluid_dfsph_set_params(PeDfsph* w, const PeDfsphParams* params) {
    if (!w) return PE_ERR_NULL;
    int rc = check_dfsph(params);
    if (rc != PE_OK) return rc;
    return guard([&] {
        w->s->set_params(to_dfsph(*params));
        return PE_OK;
    });
}

#define PE_DF_GET(name, call)                                         \
    int pe_fluid_dfsph_##name(PeDfsph* w, double* out, uint64_t n) {  \
        if (!w || !out) return PE_ERR_NULL;                           \
        if (n != w->s->world().len()) return PE_ERR_BOUNDS;           \
        return guard([&] {                                            \
            call;                                                     \
            return PE_OK;                                             \
        });                                                           \
    }
PE_DF_GET(get_positions, w->s->world().get_vec(0, out))
PE_DF_GET(get_velocities, w->s->world().get_vec(1, out))
PE_DF_GET(get_boundary_forces, w->s->world().get_vec(3, out))
PE_DF_GET(get_densities, w->s->world().get_scalar(0, out))
PE_DF_GET(get_pressures, w->s->world().get_scalar(1, out))
PE_DF_GET(get_alphas, w->s->get_alpha(out))
#undef PE_DF_GET

#define PE_DF_SET(name, which)                                            \
    int pe_fluid_dfsph_##name(PeDfsph* w, const double* in, uint64_t n) { \
        if (!w || !in) return PE_ERR_NULL;                                \
        if (n != w->s->world().len()) return PE_ERR_BOUNDS;               \
        return guard([&] {                                                \
            return w->s->world().set_vec(which, in) ? PE_OK : PE_ERR_ARG; \
        });                                                               \
    }
PE_DF_SET(set_positions, 0)
PE_DF_SET(set_velocities, 1)
#undef PE_DF_SET

int pe_fluid_dfsph_last_iterations(PeDfsph* w, uint64_t out[2]) {
    if (!w || !out) return PE_ERR_NULL;
    out[0] = w->s->last_density_iters();
    out[1] = w->s->last_divergence_iters();
    return PE_OK;
}

int pe_fluid_dfsph_mean_density_error(PeDfsph* w, double* out) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        *out = w->s->mean_density_error();
        return PE_OK;
    });
}

int pe_fluid_dfsph_v_max(PeDfsph* w, double* out) {
    if (!w || !out) return PE_ERR_NULL;
    return guard([&] {
        *out = w->s->v_max();
        return PE_OK;
    });
}

int pe_fluid_dfsph_status(PeDfsph* w, uint32_t* status) {
    if (!w || !status) return PE_ERR_NULL;
    return guard([&] {
        *status = w->s->world().status();
        return PE_OK;
    });
}

int pe_fluid_dfsph_stream(PeDfsph* w, void** out) {
    if (!w || !out) return PE_ERR_NULL;
    *out = (void*)w->s->world().stream();
    return PE_OK;
}

int pe_fluid_dfsph_kernel_launches(PeDfsph* w, uint64_t* out, int32_t reset) {
    if (!w || !out) return PE_ERR_NULL;
    *out = w->s->world().kernel_launches();
    if (reset) w->s->world().reset_launch_count();
    return PE_OK;
}

}  // extern "C"
