// Position Based Fluids on the GPU: `PbfWorld::step` of
// crates/pe-fluid/src/pbf.rs:384-436, bit for bit, on the same cell-sorted
// state, grid and neighbour lists as the WCSPH world (a World whose grid cell
// and list radius are the PBF support radius, h for poly6 / spiky).
#pragma once

#include <memory>

#include "kernel_any.cuh"
#include "world.cuh"

namespace pe {

struct PbfParams {  // pbf.rs:26-53
    int density_kernel, grad_kernel;
    uint64_t iterations;
    double epsilon_lambda, art_pressure_k, art_pressure_n, art_pressure_dq_over_h;
    double viscosity_eps, vorticity_eps;
    double gravity[3];
    int reuse_neighbours;
};

// Per-step constants of the PBF passes.
struct PbfConst {
    int dim;
    KernelFn dk, gk;           // density and gradient kernels
    double mass, rho0;
    double rho_self;           // mass * W(0)
    double mass_over_rho0;     // mass / rho0
    double eps_lambda;
    double art_k, art_n, w_dq; // artificial pressure (pbf.rs:229-235)
    int art_n_int, art_n_is_int;
    double max_corr;           // 0.4 h
    double visc_eps, vort_eps;
    double gx, gy, gz;
    double far2;  // squared distance beyond both kernels' support (with a margin)
};

class PbfSolver {
   public:
    PbfSolver(const PbfParams& prm, const WorldConfig& cfg, int dim, double rest_density, double mass, double h,
              uint64_t n, const double* x, const double* v, const uint8_t* kind, const double* psi,
              const double* n_out);
    ~PbfSolver();
    PbfSolver(const PbfSolver&) = delete;
    PbfSolver& operator=(const PbfSolver&) = delete;

    void step(double dt);
    void run(double dt, uint64_t steps);
    World& world() { return *w_; }
    const PbfParams& params() const { return prm_; }
    void set_params(const PbfParams& p);
    // pbf.rs:440-455 mean |rho / rho0 - 1| over fluid particles (sequential sum
    // in original index order, as the reference); pbf.rs:458 v_max
    double mean_density_error();
    double v_max();
    // lambda of the last constraint iteration, original order
    void get_lambda(double* out);

   private:
    void refresh_const();
    void lists(bool all_candidates);
    std::unique_ptr<World> w_;
    PbfParams prm_;
    PbfConst kc_{};
    double* lambda_ = nullptr;   // per slot
    double* lambda_orig_ = nullptr;  // the same values in original order
    double4* dp_ = nullptr;      // per slot: position correction / viscosity dv
    double4* omega_ = nullptr;   // per slot: vorticity
};

}  // namespace pe
