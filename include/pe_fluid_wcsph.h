/*
 * pe_fluid_wcsph.h — C ABI of the B200 WCSPH fluid step.
 *
 * Drop-in for the WCSPH solver path of eranyid/physics-engine's `pe-fluid`
 * crate. The reference exposes that path only as a Rust API
 * (`WcsphWorld`, crates/pe-fluid/src/wcsph.rs:58-370, and the particle
 * builders of crates/pe-fluid/src/particles.rs); its C ABI crate `pe-ffi`
 * (crates/pe-ffi/src/lib.rs) exports rigid-body worlds only. This header is
 * the C surface a `pe-ffi`-style binding of the fluid path binds, following
 * pe-ffi's conventions (docs/FFI.md:7-35):
 *   - opaque handles, `int` return codes with the same integers as
 *     crates/pe-ffi/src/error.rs:4-16 (one code added: PE_ERR_DEVICE);
 *   - no exception/unwind crosses the boundary (crates/pe-ffi/src/lib.rs:68-80);
 *   - non-finite inputs and dt <= 0 give PE_ERR_ARG, short buffers give
 *     PE_ERR_BOUNDS, null required pointers give PE_ERR_NULL;
 *   - caller-owned host buffers; getters and setters never allocate host
 *     memory for the caller; device memory is owned by the handle;
 *   - one owner thread per handle, no internal mutex.
 *
 * Arrays are in the original particle order (the order particles were pushed);
 * vectors are `[n*3]` interleaved (x0, y0, z0, x1, ...), like
 * `Particles::pack_positions` (particles.rs:137).
 */
#ifndef PE_FLUID_WCSPH_H
#define PE_FLUID_WCSPH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* Return codes (crates/pe-ffi/src/error.rs:4-16). */
#define PE_OK 0
#define PE_ERR_NULL 1
#define PE_ERR_BOUNDS 2
#define PE_ERR_ARG 3
#define PE_ERR_PANIC 4
#define PE_ERR_SCENE 5
#define PE_ERR_UNSUPPORTED 6
#define PE_ERR_DEVICE 7 /* added: a CUDA runtime call failed */

/* Sticky status bits reported by pe_fluid_wcsph_status. */
#define PE_STATUS_DOMAIN 1u            /* a particle left the dense grid domain */
#define PE_STATUS_NEIGHBOUR_OVERFLOW 2u /* a neighbour list reached its capacity */
#define PE_STATUS_NONFINITE 4u          /* a non-finite position reached the grid */
#define PE_STATUS_SLOW_UNION 8u         /* informational: a cell took the slow list path */

/* Dim (crates/pe-fluid/src/lib.rs:202). */
#define PE_DIM_2 2
#define PE_DIM_3 3

/* KernelKind (crates/pe-fluid/src/kernels.rs:19). The f64 WCSPH step takes any
 * kind (the cubic spline is the reference's default, wcsph.rs:45); the
 * single-precision form takes the cubic spline only. */
#define PE_KERNEL_CUBIC_SPLINE 0
#define PE_KERNEL_WENDLAND_C2 1
#define PE_KERNEL_POLY6 2
#define PE_KERNEL_SPIKY 3

/* ParticleKind (crates/pe-fluid/src/particles.rs:11). */
#define PE_PARTICLE_FLUID 0
#define PE_PARTICLE_BOUNDARY 1

/* WcsphParams (crates/pe-fluid/src/wcsph.rs:24-39) flattened:
 * TaitEos (eos.rs:32), MonaghanViscosity (viscosity.rs:30), Xsph
 * (viscosity.rs:77), gravity, adapt_sound_speed, and SurfaceTensionParams
 * (surface_tension.rs:38-46; the branch of wcsph.rs:261-278, f64 only). */
typedef struct PeWcsphParams {
    int32_t density_kernel;
    double eos_rest_density;
    double eos_sound_speed;
    double eos_gamma;
    double visc_alpha;
    double visc_beta;
    double visc_eps;
    double xsph_epsilon;
    double gravity[3];
    int32_t adapt_sound_speed;
    double surface_tension_sigma;          /* SurfaceTensionParams.sigma; 0 = off */
    int32_t surface_tension_model;         /* PE_SURFACE_TENSION_* */
    double surface_tension_colour_gamma;   /* SurfaceTensionParams.colour_gamma */
} PeWcsphParams;

/* SurfaceTensionModel (crates/pe-fluid/src/surface_tension.rs:27-34). */
#define PE_SURFACE_TENSION_NONE 0
#define PE_SURFACE_TENSION_AKINCI 1
#define PE_SURFACE_TENSION_COLOUR_FIELD 2

/* GPU placement and capacities (no reference counterpart; zeros = defaults). */
typedef struct PeWcsphConfig {
    int32_t device;               /* CUDA device ordinal; -1 = the current device */
    uint32_t max_neighbours;      /* first guess of list entries per particle for the
                                     neighbour-list pool (0 = 256); the first build
                                     measures the need and resizes the pool */
    uint32_t max_lower;           /* reserved, set to 0 */
    double domain_margin;         /* grid domain growth per side, fraction of extent (<0 = 0.25) */
    uint32_t domain_margin_cells; /* minimum growth per side in cells (0 = 4) */
    int32_t precision;            /* PE_PRECISION_F64 (default, the reference's bits) or
                                     PE_PRECISION_F32 (single-precision form) */
    int32_t use_graph;            /* nonzero: pe_fluid_wcsph_run replays a captured CUDA
                                     graph of six steps once the step is steady (no
                                     host synchronisation inside); same results */
} PeWcsphConfig;

#define PE_PRECISION_F64 0
/* Single-precision form: cell-local float positions and float velocities,
 * single-precision pair arithmetic with Kahan-compensated density, force and
 * XSPH sums; the grid, its sort and the sound-speed control stay f64. Not the
 * reference's bits: its error against the f64 step is measured by bench.py
 * (the f32 leg: density error, centre-of-mass and energy drift). */
#define PE_PRECISION_F32 1

/* Conservation / error reductions (crates/pe-fluid/src/diagnostics.rs:19-102,
 * wcsph.rs:350-369), computed in f64 on the device. */
typedef struct PeFluidDiagnostics {
    double total_mass;
    double linear_momentum[3];
    double kinetic_energy;
    double gravitational_potential; /* m g z with g = -gravity.z */
    double mean_density_error;
    double max_density_error;
    double v_max;
    double a_max;
    uint64_t hash64; /* particles_hash64 (diagnostics.rs:19) */
} PeFluidDiagnostics;

typedef struct PeParticles PeParticles; /* host-side Particles builder */
typedef struct PeWcsph PeWcsph;         /* one WCSPH world on one GPU */

/* ---- Particles (crates/pe-fluid/src/particles.rs) ---- */

/* Particles::new (particles.rs:52). Returns NULL on bad arguments. */
PeParticles* pe_fluid_particles_new(int32_t dim, double rest_density, double mass, double h);
void pe_fluid_particles_free(PeParticles* p);
int pe_fluid_particles_len(const PeParticles* p, uint64_t* out_len);
/* push_fluid (particles.rs:90) */
int pe_fluid_particles_push_fluid(PeParticles* p, const double x[3], const double v[3]);
/* push_boundary (particles.rs:102) / push_boundary_oriented (particles.rs:107) */
int pe_fluid_particles_push_boundary(PeParticles* p, const double x[3], double psi);
int pe_fluid_particles_push_boundary_oriented(PeParticles* p, const double x[3], double psi,
                                              const double n_out[3]);
/* fill_box (particles.rs:220) */
int pe_fluid_fill_box(PeParticles* p, const double origin[3], uint64_t nx, uint64_t ny, uint64_t nz,
                      double dx, const double v0[3]);
/* fill_box_boundary (particles.rs:286) */
int pe_fluid_fill_box_boundary(PeParticles* p, const double min[3], const double max[3], double dx,
                               uint64_t layers);
/* recomputed_akinci_psi (particles.rs:252), same summation order. */
int pe_fluid_recomputed_akinci_psi(PeParticles* p, int32_t kernel);
/* Seeded lattice jitter of the fluid particles: xoshiro256** (pe-math
 * rng.rs:14-72) seeded with `seed`, draws in particle order, x then y (then z
 * in 3-D), each U(-amplitude, amplitude), added to the position. */
int pe_fluid_particles_jitter_fluid(PeParticles* p, uint64_t seed, double amplitude);
/* Copy out SoA arrays (any pointer may be NULL); n must equal the length. */
/* count draws lo + (hi - lo) * u, u = (next >> 11) * 2^-53, in sequence from the
 * project's Xoshiro256** seeded with seed (the generator of the jitter,
 * rng.rs:14-72); used to draw seeded scene parameters. */
int pe_fluid_rng_uniform(uint64_t seed, double lo, double hi, uint64_t count, double* out);
int pe_fluid_particles_export(const PeParticles* p, double* x, double* v, uint8_t* kind, double* psi,
                              double* n_out, uint64_t n);
/* mass_from_spacing (particles.rs:166), mass_calibrated_to_rest (particles.rs:178). */
double pe_fluid_mass_from_spacing(double rest_density, double dx, int32_t dim);
double pe_fluid_mass_calibrated_to_rest(double rest_density, double dx, double h, int32_t dim,
                                        int32_t kernel);

/* ---- WCSPH world (crates/pe-fluid/src/wcsph.rs) ---- */

/* WcsphParams::water (wcsph.rs:43-53). */
int pe_fluid_wcsph_params_water(double rest_density, double sound_speed, const double gravity[3],
                                PeWcsphParams* out);
/* WcsphWorld::new (wcsph.rs:83). `cfg` may be NULL. */
int pe_fluid_wcsph_create(const PeParticles* particles, const PeWcsphParams* params,
                          const PeWcsphConfig* cfg, PeWcsph** out);
/* Same from caller arrays: kind[i] in {0 fluid, 1 boundary}; psi and n_out may
 * be NULL (0); v may be NULL (0). */
int pe_fluid_wcsph_create_from_arrays(const PeWcsphParams* params, int32_t dim, double rest_density,
                                      double mass, double h, uint64_t n, const double* x,
                                      const double* v, const uint8_t* kind, const double* psi,
                                      const double* n_out, const PeWcsphConfig* cfg, PeWcsph** out);
/* ---- Position Based Fluids (crates/pe-fluid/src/pbf.rs) ----
 * PbfParams (pbf.rs:26-53); kernels are PE_KERNEL_* values. */
typedef struct PePbfParams {
    int32_t density_kernel;
    int32_t grad_kernel;
    uint64_t iterations;
    double epsilon_lambda;
    double art_pressure_k;
    double art_pressure_n;
    double art_pressure_dq_over_h;
    double viscosity_eps;
    double vorticity_eps;
    double gravity[3];
    int32_t reuse_neighbours;
} PePbfParams;
typedef struct PePbf PePbf;
/* PbfParams::default (pbf.rs:55-74). */
int pe_fluid_pbf_params_default(PePbfParams* out);
/* PbfWorld::new (pbf.rs:112-130): grid cell = the larger support radius of the
 * two kernels. cfg: device and capacity fields only (precision f64, no graphs). */
int pe_fluid_pbf_create(const PeParticles* particles, const PePbfParams* params, const PeWcsphConfig* cfg,
                        PePbf** out);
int pe_fluid_pbf_create_from_arrays(const PePbfParams* params, int32_t dim, double rest_density, double mass,
                                    double h, uint64_t n, const double* x, const double* v, const uint8_t* kind,
                                    const double* psi, const double* n_out, const PeWcsphConfig* cfg,
                                    PePbf** out);
void pe_fluid_pbf_destroy(PePbf* w);
/* PbfWorld::step (pbf.rs:384-436); dt >= 0. */
int pe_fluid_pbf_step(PePbf* w, double dt);
int pe_fluid_pbf_run(PePbf* w, double dt, uint64_t steps);
int pe_fluid_pbf_len(const PePbf* w, uint64_t* out_len);
int pe_fluid_pbf_get_time(const PePbf* w, double* t);
int pe_fluid_pbf_get_params(const PePbf* w, PePbfParams* out);
/* The kernels' support radius is fixed at creation. */
int pe_fluid_pbf_set_params(PePbf* w, const PePbfParams* params);
/* particles.{x, v, rho} and the last iteration's lambda, original order. */
int pe_fluid_pbf_get_positions(PePbf* w, double* out, uint64_t n);
int pe_fluid_pbf_get_velocities(PePbf* w, double* out, uint64_t n);
int pe_fluid_pbf_get_densities(PePbf* w, double* out, uint64_t n);
int pe_fluid_pbf_get_lambdas(PePbf* w, double* out, uint64_t n);
int pe_fluid_pbf_set_positions(PePbf* w, const double* in, uint64_t n);
int pe_fluid_pbf_set_velocities(PePbf* w, const double* in, uint64_t n);
/* pbf.rs:440-455 mean |rho/rho0 - 1|, pbf.rs:458 v_max. */
int pe_fluid_pbf_mean_density_error(PePbf* w, double* out);
int pe_fluid_pbf_v_max(PePbf* w, double* out);
int pe_fluid_pbf_status(PePbf* w, uint32_t* status);
int pe_fluid_pbf_kernel_launches(PePbf* w, uint64_t* out, int32_t reset);
/* The CUDA stream (cudaStream_t) all of the world's work is issued on. */
int pe_fluid_pbf_stream(PePbf* w, void** out);

/* ---- Divergence-free SPH (crates/pe-fluid/src/dfsph.rs) ----
 * DfsphParams (dfsph.rs:33-80) without surface tension; the optional free-slip
 * planes x >= xmin, y >= ymin, x <= xmax, y <= ymax are free_slip[0..3],
 * active where free_slip_set[k] is nonzero. */
typedef struct PeDfsphParams {
    int32_t kernel;
    uint64_t max_density_iters;
    uint64_t max_divergence_iters;
    double density_error_tol;
    double divergence_error_tol;
    double gravity[3];
    double xsph_epsilon;
    double particle_diameter;
    double cfl_lambda;
    int32_t adaptive_dt;
    int32_t warm_start;
    int32_t free_slip_set[4];
    double free_slip[4];
    double solver_omega;
    double max_velocity_correction;
} PeDfsphParams;
typedef struct PeDfsph PeDfsph;
/* DfsphParams::default (dfsph.rs:82-104). */
int pe_fluid_dfsph_params_default(PeDfsphParams* out);
/* DfsphWorld::new (dfsph.rs:137-180): builds the grid and lists and computes
 * densities and alpha. cfg: device and capacity fields only. */
int pe_fluid_dfsph_create(const PeParticles* particles, const PeDfsphParams* params, const PeWcsphConfig* cfg,
                          PeDfsph** out);
int pe_fluid_dfsph_create_from_arrays(const PeDfsphParams* params, int32_t dim, double rest_density,
                                      double mass, double h, uint64_t n, const double* x, const double* v,
                                      const uint8_t* kind, const double* psi, const double* n_out,
                                      const PeWcsphConfig* cfg, PeDfsph** out);
void pe_fluid_dfsph_destroy(PeDfsph* w);
/* DfsphWorld::step (dfsph.rs:718-769), step_adaptive (dfsph.rs:772-784, the
 * dt used goes to *dt_out), suggest_dt (dfsph.rs:633-665). */
int pe_fluid_dfsph_step(PeDfsph* w, double dt);
int pe_fluid_dfsph_run(PeDfsph* w, double dt, uint64_t steps);
int pe_fluid_dfsph_step_adaptive(PeDfsph* w, double* dt_out);
int pe_fluid_dfsph_suggest_dt(PeDfsph* w, double* out);
/* The public phase methods (dfsph.rs:201, 214, 252). */
int pe_fluid_dfsph_rebuild_neighbours(PeDfsph* w);
int pe_fluid_dfsph_compute_density(PeDfsph* w);
int pe_fluid_dfsph_compute_alpha(PeDfsph* w);
int pe_fluid_dfsph_len(const PeDfsph* w, uint64_t* out_len);
int pe_fluid_dfsph_get_time(const PeDfsph* w, double* t);
int pe_fluid_dfsph_get_last_dt(const PeDfsph* w, double* out);
int pe_fluid_dfsph_get_params(const PeDfsph* w, PeDfsphParams* out);
int pe_fluid_dfsph_set_params(PeDfsph* w, const PeDfsphParams* params);
/* particles.{x, v, rho, p}, boundary_force, alpha; original order. */
int pe_fluid_dfsph_get_positions(PeDfsph* w, double* out, uint64_t n);
int pe_fluid_dfsph_get_velocities(PeDfsph* w, double* out, uint64_t n);
int pe_fluid_dfsph_get_densities(PeDfsph* w, double* out, uint64_t n);
int pe_fluid_dfsph_get_pressures(PeDfsph* w, double* out, uint64_t n);
int pe_fluid_dfsph_get_boundary_forces(PeDfsph* w, double* out, uint64_t n);
int pe_fluid_dfsph_get_alphas(PeDfsph* w, double* out, uint64_t n);
/* Setting state keeps the neighbour lists, as writing the reference's public
 * fields does; rebuild_neighbours refreshes them. */
int pe_fluid_dfsph_set_positions(PeDfsph* w, const double* in, uint64_t n);
int pe_fluid_dfsph_set_velocities(PeDfsph* w, const double* in, uint64_t n);
/* Iterations of the last step's density and divergence solvers. */
int pe_fluid_dfsph_last_iterations(PeDfsph* w, uint64_t out[2]);
/* diagnostics.rs:74-88 mean |rho - rho0| / rho0; dfsph.rs:792 v_max. */
int pe_fluid_dfsph_mean_density_error(PeDfsph* w, double* out);
int pe_fluid_dfsph_v_max(PeDfsph* w, double* out);
int pe_fluid_dfsph_status(PeDfsph* w, uint32_t* status);
int pe_fluid_dfsph_kernel_launches(PeDfsph* w, uint64_t* out, int32_t reset);
int pe_fluid_dfsph_stream(PeDfsph* w, void** out);

/* Fluid side of CoupledWcsphWorld::step (coupling.rs:853-866). A coupler holds
 * the rigid samples of a world: sample k is world particle particle[k] (an
 * oriented boundary sample) on body body[k] < n_bodies, at body-frame offset
 * local[3k..] with body-frame normal local_n[3k..] (FluidRigidCoupler::samples,
 * coupling.rs:42-51, insertion order). The rigid bodies stay with the caller. */
typedef struct PeCoupler PeCoupler;
int pe_fluid_coupler_create(PeWcsph* w, uint32_t n_bodies, uint64_t n_samples, const int64_t* body,
                            const double* local, const double* local_n, const int64_t* particle,
                            PeCoupler** out);
void pe_fluid_coupler_destroy(PeCoupler* c);
/* FluidRigidCoupler::sync_from_rigid (coupling.rs:289-306): per body the
 * centre of mass X (3), orientation q (4: w, x, y, z), velocity V (3) and
 * world-frame angular velocity omega (3); the samples' positions, velocities
 * and normals follow, and the next step rebuilds the grid. */
int pe_fluid_coupler_sync(PeCoupler* c, const double* X, const double* q, const double* V, const double* omega);
/* FluidRigidCoupler::reduce_with_state (coupling.rs:308-330): per body the sum
 * of its samples' boundary reactions (force, 3 per body) and of r x f with
 * r = x - X (torque, 3 per body), in sample order. */
int pe_fluid_coupler_reduce(PeCoupler* c, const double* X, double* force, double* torque);

/* Batched form (no reference counterpart; replaces a loop of WcsphWorld::step
 * over independent tanks): n_tanks tanks with the same material and physics,
 * particles stored tank-major, tank t owning particles [tank_offsets[t],
 * tank_offsets[t + 1]) (tank_offsets has n_tanks + 1 entries, 0 ... n, no tank
 * empty). Every tank keeps its own grid domain and persisted sound speed and
 * evolves exactly as a world created from its particles alone; one step call
 * advances all tanks. n_tanks = 1 with tank_offsets NULL is
 * pe_fluid_wcsph_create_from_arrays. */
int pe_fluid_wcsph_create_batch(const PeWcsphParams* params, int32_t dim, double rest_density,
                                double mass, double h, uint64_t n, const double* x, const double* v,
                                const uint8_t* kind, const double* psi, const double* n_out,
                                uint32_t n_tanks, const uint64_t* tank_offsets,
                                const PeWcsphConfig* cfg, PeWcsph** out);
void pe_fluid_wcsph_destroy(PeWcsph* w);
int pe_fluid_wcsph_tanks(PeWcsph* w, uint32_t* n_tanks);
/* The persisted sound speed of every tank (n_tanks must equal the world's). */
int pe_fluid_wcsph_get_sound_speeds(PeWcsph* w, double* out, uint32_t n_tanks);
/* Launch-shape autotuner (no reference counterpart): times the candidate block
 * sizes of the density, force and XSPH passes (64, 128, 256), and the list
 * build's tile (32 or 64 centre particles per chunk) with its CTAs per SM, on
 * the current state without advancing it, and keeps the fastest. No shape
 * changes a result bit.
 * out (may be NULL) = {density, forces, xsph block sizes, list CTAs per SM}. */
int pe_fluid_wcsph_autotune(PeWcsph* w, uint32_t out[4]);
int pe_fluid_wcsph_shapes(PeWcsph* w, uint32_t out[4]);
/* The list build's tile in use: centre particles per chunk (32 or 64). */
int pe_fluid_wcsph_list_chunk(PeWcsph* w, uint32_t* out);
/* Pair weights: the density pass keeps each neighbour entry's W(r) for the
 * XSPH pass of the same lists and positions (on by default; a device buffer
 * of twice the neighbour-list pool's bytes, the pool's bytes in the
 * single-precision form, allocated only while the device has room for it and
 * 2 GB besides). on = 0 frees it and XSPH recomputes W. The f64 step's
 * results are identical either way (the single-precision form's may differ
 * in the last bits). pe_fluid_wcsph_pair_weights reports whether the buffer
 * is in use (1) or not (0). */
int pe_fluid_wcsph_set_pair_weights(PeWcsph* w, int32_t on);
int pe_fluid_wcsph_pair_weights(PeWcsph* w, int32_t* out);
/* The buffer covers the pool's first 5/8 (1.25x the lists of a freshly sized
 * pool). A density pass that meets a list reaching past it keeps no weights
 * for that step and XSPH recomputes W; the next pe_fluid_wcsph_status (run
 * polls it every 16 steps) extends the buffer to the whole pool.
 * out = {in use (0/1), list entries covered, the last density pass met a
 * list beyond them (0/1)}. Synchronous. */
int pe_fluid_wcsph_pair_weight_info(PeWcsph* w, uint64_t out[3]);

/* WcsphWorld::step (wcsph.rs:326). Synchronous; returns PE_ERR_BOUNDS if the
 * step raised PE_STATUS_DOMAIN or PE_STATUS_NEIGHBOUR_OVERFLOW. */
int pe_fluid_wcsph_step(PeWcsph* w, double dt);
/* `steps` calls of step, checked once at the end. */
int pe_fluid_wcsph_run(PeWcsph* w, double dt, uint64_t steps);
/* Phase methods (wcsph.rs:102, 117, 157, 181, 283). */
int pe_fluid_wcsph_rebuild_grid(PeWcsph* w);
int pe_fluid_wcsph_compute_density(PeWcsph* w);
int pe_fluid_wcsph_compute_pressure(PeWcsph* w);
int pe_fluid_wcsph_compute_forces(PeWcsph* w);
int pe_fluid_wcsph_apply_xsph(PeWcsph* w);

int pe_fluid_wcsph_len(const PeWcsph* w, uint64_t* out_len);
int pe_fluid_wcsph_get_time(const PeWcsph* w, double* t);
int pe_fluid_wcsph_set_time(PeWcsph* w, double t);
/* Persisted sound speed (params.eos.sound_speed, updated by compute_pressure). */
int pe_fluid_wcsph_get_sound_speed(PeWcsph* w, double* c);
int pe_fluid_wcsph_get_params(PeWcsph* w, PeWcsphParams* out);
int pe_fluid_wcsph_set_params(PeWcsph* w, const PeWcsphParams* params);

/* State in original order. Vectors are [n*3]. */
int pe_fluid_wcsph_get_positions(PeWcsph* w, double* out, uint64_t n);
int pe_fluid_wcsph_get_velocities(PeWcsph* w, double* out, uint64_t n);
int pe_fluid_wcsph_get_accelerations(PeWcsph* w, double* out, uint64_t n);
int pe_fluid_wcsph_get_boundary_forces(PeWcsph* w, double* out, uint64_t n);
int pe_fluid_wcsph_get_densities(PeWcsph* w, double* out, uint64_t n);
int pe_fluid_wcsph_get_pressures(PeWcsph* w, double* out, uint64_t n);
int pe_fluid_wcsph_get_kinds(PeWcsph* w, uint8_t* out, uint64_t n);
/* Setting positions marks the grid stale (the next step rebuilds it). */
int pe_fluid_wcsph_set_positions(PeWcsph* w, const double* in, uint64_t n);
int pe_fluid_wcsph_set_velocities(PeWcsph* w, const double* in, uint64_t n);
int pe_fluid_wcsph_set_densities(PeWcsph* w, const double* in, uint64_t n);
int pe_fluid_wcsph_set_pressures(PeWcsph* w, const double* in, uint64_t n);

/* UniformGrid (grid.rs:32-45): keys [n*3] per original index, order [n]
 * (original indices sorted by (key, index)), occupied [m*3], ranges [m*2]
 * with m <= occupied_cap; *n_occupied receives m. Any output may be NULL. */
int pe_fluid_wcsph_get_grid(PeWcsph* w, int32_t* keys, uint64_t* order, uint64_t n,
                            int32_t* occupied, uint64_t* ranges, uint64_t occupied_cap,
                            uint64_t* n_occupied);
/* Per particle: candidate count (= neigh_lists[i].len() of the reference,
 * self included; 0 for boundary) and in-support count (j != i, r/h < 2). */
int pe_fluid_wcsph_get_neighbour_counts(PeWcsph* w, uint32_t* candidates, uint32_t* in_support,
                                        uint64_t n);

int pe_fluid_wcsph_status(PeWcsph* w, uint32_t* status);
int pe_fluid_wcsph_clear_status(PeWcsph* w);
/* Capacity introspection (no reference counterpart): out = {status bits,
 * largest neighbour-cell union seen, 16-byte list groups the last list build
 * asked for, union stage capacity, list pool capacity in 16-byte groups,
 * occupied cells, dense cells, list-build CTAs}. */
int pe_fluid_wcsph_capacity_info(PeWcsph* w, uint64_t out[8]);
/* diagnostics.rs:19-102 and wcsph.rs:350-369, reduced on the device with the
 * reference's bits: sums in original index order, the FNV-1a hash of the
 * fluid (x, v); no copy of the state to the host. */
int pe_fluid_wcsph_diagnostics(PeWcsph* w, PeFluidDiagnostics* out);
/* Fluid centre of mass (no reference counterpart): the fluid positions summed
 * in original index order on the device, divided by the fluid count. */
int pe_fluid_wcsph_fluid_center_of_mass(PeWcsph* w, double out[3]);
/* Per-phase device time, measured with CUDA events on the world's stream:
 * 0 grid build, 1 neighbour lists, 2 density, 3 pressure, 4 forces + kick/drift,
 * 5 boundary reaction forces, 6 XSPH (no reference counterpart). */
#define PE_FLUID_NUM_PHASES 7
typedef struct PeFluidProfile {
    double ms[PE_FLUID_NUM_PHASES];
    uint64_t count[PE_FLUID_NUM_PHASES];
} PeFluidProfile;
int pe_fluid_wcsph_profile(PeWcsph* w, int32_t enable);
int pe_fluid_wcsph_profile_read(PeWcsph* w, PeFluidProfile* out, int32_t reset);
/* The CUDA stream (cudaStream_t) all of the world's work is issued on. */
int pe_fluid_wcsph_stream(PeWcsph* w, void** out);
/* Kernel launches issued since creation or the last reset (accounting aid). */
int pe_fluid_wcsph_kernel_launches(PeWcsph* w, uint64_t* out, int32_t reset);

/* ---- stateless helpers ---- */
/* kernels.rs:40 w and kernels.rs:56 grad_w (every PE_KERNEL_*), eos.rs:65 pressure. */
double pe_fluid_kernel_w(int32_t kernel, double r, double h, int32_t dim);
int pe_fluid_grad_w(int32_t kernel, const double rij[3], double h, int32_t dim, double out[3]);
double pe_fluid_tait_pressure(double rest_density, double sound_speed, double gamma, double density);
/* viscosity.rs:51 pi_ij */
double pe_fluid_pi_ij(double alpha, double beta, double eps, double h, double sound_speed,
                      const double xi[3], const double xj[3], const double vi[3], const double vj[3],
                      double rho_i, double rho_j);
/* cfl.rs:36 suggested_dt */
double pe_fluid_suggested_dt(double h, double sound_speed, double v_max, double a_max,
                             double lambda_v, double lambda_f);
/* ---- allocation-free density pass (no reference counterpart) ----
 *
 * For callers that cannot allocate device memory: applications that give the
 * library a fixed device budget or route every device allocation through
 * their own allocator, and real-time loops that must not pay for cudaMalloc's
 * device-wide synchronisation. It computes what `rebuild_grid` followed by
 * `compute_density` give (wcsph.rs:102-154) for a world whose density kernel
 * is the cubic spline (PE_KERNEL_CUBIC, the WcsphParams default; no other
 * kernel is offered here), with the same bits as the world API: rho[i] for
 * every particle, rest_density for boundary samples.
 *
 * x [n*3], kind [n], psi [n] (may be NULL: every boundary sample then has
 * psi 0), n_out [n*3] (may be NULL: no sample is oriented) and the output
 * rho [n] are DEVICE pointers; `stream` is a cudaStream_t (NULL = the legacy
 * default stream). Nothing is allocated: the working memory is one fixed
 * array in the library's device image (about 18 MB per device that loads the
 * library, held until the process exits). Limits: n <=
 * PE_FLUID_NOALLOC_MAX_PARTICLES and a cell-key bounding box of at most
 * PE_FLUID_NOALLOC_MAX_CELLS cells (2h-sized cells); beyond either the call
 * returns PE_ERR_BOUNDS and leaves rho untouched. A non-finite value in x,
 * psi or n_out returns PE_ERR_ARG, rho untouched.
 *
 * Every call, with the caller's device current, looks up the array's device
 * address (cudaGetSymbolAddress, which allocates nothing). The call waits for
 * its stream once, midway (to read the key bounding box that sizes the grid).
 * All calls share the one array, which keeps the previous call's contents;
 * every call clears what must start at zero. Calls that overlap on the GPU
 * race on the array: issue them in order on one stream or otherwise
 * serialise them. */
#define PE_FLUID_NOALLOC_MAX_PARTICLES 131072u
#define PE_FLUID_NOALLOC_MAX_CELLS 262144u
int pe_fluid_density_noalloc(int32_t dim, double rest_density, double mass, double h, uint64_t n,
                             const double* x, const uint8_t* kind, const double* psi,
                             const double* n_out, double* rho, void* stream);

/* Measured FP64 issue rate of the device (no reference counterpart): independent
 * non-fused multiplies and adds, the instruction mix the step's f64 passes
 * compile to, in 1e9 operations per second. The denominator of the step's FP64
 * roofline. */
int pe_fluid_probe_fp64_rate(int32_t device, double* gops);

/* Measured cost of one phase boundary (no reference counterpart), in
 * microseconds: a kernel node of a replayed CUDA graph of `phases` nodes
 * (node_us), against a grid-wide barrier inside one cooperative persistent
 * kernel of `phases` phases (barrier_us; the barrier's wait is bounded and a
 * timeout returns PE_ERR_DEVICE). Both over the same co-resident grid with
 * token work per phase. 2 <= phases <= 4096. */
int pe_fluid_probe_phase_overhead(int32_t device, uint32_t phases, double* node_us, double* barrier_us);

/* Library version string. */
const char* pe_fluid_version(void);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* PE_FLUID_WCSPH_H */
