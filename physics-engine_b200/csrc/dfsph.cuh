// Divergence-free SPH on the GPU: `DfsphWorld` of
// crates/pe-fluid/src/dfsph.rs (constant-density and divergence-free solvers
// with warm start, XSPH on the predicted velocity, boundary reactions, free-slip
// planes), bit for bit, on the cell-sorted state, grid and neighbour lists of a
// World (grid cell = the kernel's support radius).
#pragma once

#include <memory>

#include "kernel_any.cuh"
#include "world.cuh"

namespace pe {

struct DfsphParams {  // dfsph.rs:33-80 (surface tension not provided: sigma = 0)
    int kernel;
    uint64_t max_density_iters, max_divergence_iters;
    double density_error_tol, divergence_error_tol;
    double gravity[3];
    double xsph_epsilon;
    double particle_diameter, cfl_lambda;
    int adaptive_dt, warm_start;
    int has_slip[4];  // free_slip_{xmin, ymin, xmax, ymax}
    double slip[4];
    double solver_omega, max_velocity_correction;
};

struct DfsphConst {
    int dim;
    KernelFn kf;
    double mass, rho0;
    double rho_self;     // mass * W(0)
    double eps_h;        // 0.15 h (particles.rs:132)
    double denom_floor;  // dfsph.rs:262-267
    double xsph_eps;
    double gx, gy, gz;
    double omega, dv_cap;
    int warm_start;
    int has_slip[4];
    double slip[4];
    double far2;  // squared distance beyond the kernel's support (with a margin)
};

class DfsphSolver {
   public:
    DfsphSolver(const DfsphParams& prm, const WorldConfig& cfg, int dim, double rest_density, double mass, double h,
                uint64_t n, const double* x, const double* v, const uint8_t* kind, const double* psi,
                const double* n_out);
    ~DfsphSolver();
    DfsphSolver(const DfsphSolver&) = delete;
    DfsphSolver& operator=(const DfsphSolver&) = delete;

    void step(double dt);                 // dfsph.rs:718-769
    double step_adaptive();               // dfsph.rs:772-784
    void run(double dt, uint64_t steps);
    double suggest_dt();                  // dfsph.rs:633-665
    World& world() { return *w_; }
    const DfsphParams& params() const { return prm_; }
    void set_params(const DfsphParams& p);
    double last_dt() const { return last_dt_; }
    // iterations of the last step's density and divergence solvers
    uint64_t last_density_iters() const { return it_density_; }
    uint64_t last_divergence_iters() const { return it_divergence_; }
    // the solvers' average errors of their last iteration
    double last_density_error() const { return err_density_; }
    double last_divergence_error() const { return err_divergence_; }
    uint64_t serial_sums() const { return serial_sums_; }
    void get_alpha(double* out);          // original order
    // the public phase methods (dfsph.rs:201, 214, 252)
    void rebuild_neighbours();
    void compute_density();
    void compute_alpha();
    double mean_density_error();          // diagnostics.rs:74-88
    double v_max();                       // dfsph.rs:792-800

   private:
    void refresh_const();
    void rebuild();                       // grid + lists (dfsph.rs:201-211)
    void density_and_alpha();             // dfsph.rs:214-307
    void pressure_update(double dt, bool divergence);  // dfsph.rs:422-530
    double solve_error(double dt, bool divergence);    // one error pass + its average
    uint64_t correct_density_error(double dt);         // dfsph.rs:533-584
    uint64_t correct_divergence_error(double dt);      // dfsph.rs:587-630
    void free_slip();                                  // dfsph.rs:668-715

    std::unique_ptr<World> w_;
    DfsphParams prm_;
    DfsphConst kc_{};
    uint64_t n_fluid_ = 0;
    double last_dt_ = 0.0;
    bool a_adv_set_ = false;  // the non-pressure accelerations (gravity) have been computed
    uint64_t it_density_ = 0, it_divergence_ = 0;
    double err_density_ = 0.0, err_divergence_ = 0.0;
    // per slot (valid until the next re-sort)
    double* alpha_ = nullptr;
    double* kappa_ = nullptr;
    double* kr_ = nullptr;           // kappa / max(rho, 1e-12) (boundary: 0 / rho0)
    double4* dv_ = nullptr;          // xsph scratch
    double4* react_ = nullptr;       // (F_b total, wsum) of a fluid particle's reaction
    // per original index: a solver pass's error terms, summed in index order
    double* err_orig_ = nullptr;
    double* sum_ = nullptr;          // device scalar
    double* part_ = nullptr;         // partial sums
    uint64_t serial_sums_ = 0;       // decisions that needed the sequential sum
    double* sum_host_ = nullptr;     // pinned
};

}  // namespace pe
