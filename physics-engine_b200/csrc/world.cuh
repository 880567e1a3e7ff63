// Host runtime of one WCSPH world on one GPU (the state machine behind the
// C ABI). Mirrors `WcsphWorld` (crates/pe-fluid/src/wcsph.rs:58-370): the
// same phase methods, the same step, the persisted sound speed, and
// caller-owned host buffers for every getter/setter.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "wcsph_device.cuh"

namespace pe {

struct WorldParams {
    int kernel;  // 0 = cubic spline
    double eos_rest_density, eos_sound_speed, eos_gamma;
    double visc_alpha, visc_beta, visc_eps;
    double xsph_epsilon;
    double gravity[3];
    int adapt_sound_speed;
    double surface_tension_sigma;
    int surface_tension_model;  // 0 none, 1 Akinci 2013, 2 colour field
    double surface_tension_colour_gamma;
};

struct WorldConfig {
    int device;                 // CUDA device ordinal (-1 = current)
    uint32_t max_neighbours;    // initial list-part capacity per particle (0 = 256; grows on demand)
    uint32_t max_lower;         // reserved
    double domain_margin;       // extra grid domain per side, fraction of extent (<0 = 0.25)
    uint32_t domain_margin_cells;  // minimum extra cells per side (0 = 4)
    int precision;              // 0 = f64 (reference bits), 1 = single-precision form
    int use_graph;              // run() replays captured CUDA graphs of the step
    int pair_weights;           // keep each visit entry's W for XSPH (World::set_pair_weights)
};

class CudaError : public std::runtime_error {
   public:
    explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

class Surrogate;
class Coupler;
class PbfSolver;
class DfsphSolver;

class World {
   public:
    // tank_offsets (n_tanks + 1 entries, from 0 to n) splits the particles into
    // independent tanks stepped together; null means one tank.
    World(const WorldParams& prm, const WorldConfig& cfg, int dim, double rest_density, double mass,
          double h, uint64_t n, const double* x, const double* v, const uint8_t* kind,
          const double* psi, const double* n_out, const uint64_t* tank_offsets = nullptr,
          uint32_t n_tanks = 1, double support = 0.0);
    ~World();
    World(const World&) = delete;
    World& operator=(const World&) = delete;

    // Phase methods (wcsph.rs:102, 117, 157, 181, 283) and the step (wcsph.rs:326).
    void rebuild_grid();
    void compute_density();
    void compute_pressure();
    void compute_forces();
    void apply_xsph();
    void step(double dt);
    void run(double dt, uint64_t steps);
    void synchronize();

    uint64_t len() const { return n_; }
    int dim() const { return dim_; }
    double time() const { return t_; }
    void set_time(double t) { t_ = t; }
    double sound_speed();             // tank 0
    void set_sound_speed(double c);   // every tank
    uint32_t tanks() const { return n_tanks_; }
    void get_sound_speeds(double* out);  // one per tank
    const WorldParams& params() const { return prm_; }
    void set_params(const WorldParams& p);
    double mass() const { return mass_; }
    double rest_density() const { return rho0_; }
    double smoothing_length() const { return h_; }
    bool single_precision() const { return f32_; }

    // Host-buffer access in original particle order.
    void get_vec(int which, double* out);         // 0 x, 1 v, 2 a, 3 boundary force
    // 0 x, 1 v; false (state untouched) when the input holds a non-finite value
    bool set_vec(int which, const double* in);
    void get_scalar(int which, double* out);      // 0 rho, 1 p
    void set_scalar(int which, const double* in); // 0 rho, 1 p
    void get_kind(uint8_t* out);
    void get_grid(int32_t* keys, uint64_t* order, int32_t* occupied, uint64_t* ranges,
                  uint64_t occ_cap, uint64_t* n_occupied);
    void get_neighbour_counts(uint32_t* candidates, uint32_t* in_support);
    uint32_t status();
    void clear_status();
    // diagnostics.rs:19-102 and wcsph.rs:350-369, reduced on the device with
    // the reference's bits (sums in original index order); no state copy.
    struct Diagnostics {
        double total_mass, linear_momentum[3], kinetic_energy, gravitational_potential;
        double mean_density_error, max_density_error, v_max, a_max;
        uint64_t hash64, fluid;
        double fluid_com[3];  // sum of fluid positions in index order / fluid count
    };
    void diagnostics(Diagnostics* out);
    // status, largest union, list groups the last build asked for, union stage
    // capacity, list pool groups, occupied cells, dense cells, list-build CTAs
    void capacity_info(uint64_t* out);

    // Device views (advanced use: zero-copy access from the same process).
    const StateBufs& device_state() const { return cur_; }
    const uint32_t* device_slot_of_orig() const { return slot_of_orig_; }
    cudaStream_t stream() const { return st_; }
    uint32_t kernel_launches() const { return launches_; }
    void reset_launch_count() { launches_ = 0; }

    // Per-phase device time with CUDA events on the world's stream.
    enum Phase { kGrid = 0, kLists, kDensity, kPressure, kForces, kBoundaryForce, kXsph, kNumPhases };
    void set_profiling(bool on) { profiling_ = on; }
    // Accumulated milliseconds and event-bracketed launches per phase since the
    // last reset; synchronises the stream.
    void profile_read(double* ms, uint64_t* count, bool reset);

    // Launch shapes picked by autotune(): block sizes of the density, force and
    // XSPH passes, and the list build's CTAs per SM and tile (centre particles
    // per chunk, 32 or 64). Timing repeats idempotent
    // passes on the current state, so the simulation does not advance.
    struct Shapes {
        uint32_t density, forces, xsph, list_ctas_per_sm;
        uint32_t list_chunk;  // centre particles per chunk of the list build (32 or 64)
    };
    Shapes shapes() const;
    Shapes autotune();

    // The density pass keeps each visit entry's W(r) for the XSPH pass of the
    // same lists and positions, in a buffer of twice the list pool's bytes
    // (the pool's bytes in the single-precision form) that is kept only while
    // the device has room for it (it follows the pool when that grows). Off,
    // or without the buffer, XSPH recomputes W from the neighbour's position.
    // In the f64 step the bits are the same either way.
    void set_pair_weights(bool on);
    bool pair_weights() const { return lists_.wpair != nullptr || lists_.wpair32 != nullptr; }
    // {in use, list entries the buffer covers, the last density pass met a
    // list beyond them}; synchronises the stream
    void pair_weight_info(uint64_t out[3]);

    // ---- learned surrogate (surrogate.cuh) ----
    // One step with the network's acceleration and density rate in place of
    // the pressure, viscosity and XSPH passes: v += dt a, x += dt v,
    // rho += dt drho/dt (fluid particles).
    void step_learned(Surrogate& s, double dt);
    // Rebuilds the grid and computes the SPH density of the current positions
    // (the plain step's density); returns the largest relative difference of
    // the carried fluid densities from it and keeps the SPH densities.
    double judge_density();
    struct LearnedStats {
        uint64_t windows, fallbacks, learned_steps, plain_steps;
        double max_error, last_error;
    };
    // steps in windows of judge_every: each window runs learned steps from a
    // checkpoint, is judged, and is replaced by plain steps from the
    // checkpoint when the density error exceeds bound
    void run_learned(Surrogate& s, double dt, uint64_t steps, uint32_t judge_every, double bound,
                     LearnedStats* st);
    uint32_t tank_slot_begin(uint32_t t) const { return tank_host_.at(t).slot_begin; }
    uint32_t tank_slot_end(uint32_t t) const {
        return t + 1 < n_tanks_ ? tank_host_[t + 1].slot_begin : (uint32_t)n_;
    }

   private:
    friend class Surrogate;
    friend class Coupler;
    friend class PbfSolver;
    friend class DfsphSolver;
    void save_checkpoint();
    void restore_checkpoint();
    double4 *ck_pos_ = nullptr, *ck_vel_ = nullptr;
    double* ck_p_ = nullptr;
    double ck_t_ = 0.0;
    float* judge_err_ = nullptr;
    void check(cudaError_t e, const char* what);
    void build_grid(const double4* pos_next, const double4* vel_next);
    void ensure_lists(bool visit_only = false);
    void run_density(bool visit_only = false);
    void run_pressure();
    void run_forces(bool integrate, double dt);
    void run_xsph();
    void run_surface_tension();
    void configure_surface_tension();
    double4* st_normals_ = nullptr;  // colour-field normals (surface tension)
    double4* st_a_ = nullptr;        // surface-tension accelerations
    void refresh_step_const();
    void refresh_f32();
    void configure_lists();
    void alloc_lists(unsigned long long groups);
    void invalidate_graph() { ++epoch_; }
    bool graph_capturable() const;
    bool capture_graph(double dt);
    void release_graph();
    template <typename T>
    T* alloc(size_t count);
    void gather_orig_vec(const double4* src, double* out);

    int dim_;
    double rho0_, mass_, h_;
    double support_;  // grid cell size and list radius (the WCSPH cubic spline: 2h)
    // Lists keep every candidate of the 27 (9) neighbour cells, not only those
    // in support: solvers that reuse a list while particles move (PBF's
    // constraint iterations) need the reference's complete candidate set.
    bool list_all_candidates_ = false;
    // Lists keep every boundary candidate (visit lists) and every fluid
    // candidate of boundary slots (lower lists, built for boundary slots only):
    // the DFSPH reaction weights range over those whole candidate sets.
    bool list_keep_boundary_ = false;
    uint64_t n_;
    WorldParams prm_;
    WorldConfig cfg_;
    double t_ = 0.0;
    int device_ = 0;
    cudaStream_t st_ = nullptr;

    GridDesc g_{};
    uint32_t n_tanks_ = 1;
    Tanks tanks_{};
    std::vector<TankDesc> tank_host_;
    PassShape shape_{};
    uint32_t list_ctas_per_sm_ = 0;  // 0: four times the resident count
    uint32_t list_chunk_ = 32;       // centre particles per list-build chunk
    StepConst kc_{};
    uint32_t ucap_ = 0, nl_blocks_ = 0, sms_ = 148;

    StateBufs cur_{}, alt_{};
    double4* pos_nx_ = nullptr;
    double4* vel_nx_ = nullptr;
    uint32_t* slot_of_orig_ = nullptr;
    uint32_t *cellid_ = nullptr, *tmp_old_ = nullptr, *tmp_orig_ = nullptr, *perm_ = nullptr;
    int4* key_tmp_ = nullptr;
    uint32_t *count_ = nullptr, *fill_ = nullptr, *cell_start_ = nullptr, *occ_ = nullptr;
    void* scan_tmp_ = nullptr;
    ListBufs lists_{};
    uint32_t* insup_ = nullptr;
    DeviceScalars* sc_ = nullptr;
    double* xfer_ = nullptr;  // n * 4 doubles of export/import staging
    unsigned char* diag_buf_ = nullptr;  // diagnostics: results, hash tables and maps
    std::vector<void*> allocs_;
    std::vector<void*> list_allocs_;

    // single-precision form
    bool f32_ = false;
    F32Const kf_{};
    F32Bufs fb_{};
    float4* velf_alt_ = nullptr;
    float* bf32_ = nullptr;

    bool grid_built_ = false;    // a grid exists (rebuild_grid ran at least once)
    bool grid_current_ = false;  // grid built from the current positions
    bool rho_current_ = false;   // densities computed from the current grid and positions
    bool lists_valid_ = false;   // neighbour lists match the grid and positions
    bool pair_w_on_ = false;     // keep lists_.wpair (set_pair_weights)
    bool w_valid_ = false;       // lists_.wpair holds W of the current lists and positions
    void alloc_pair_weights(unsigned long long groups);
    void free_pair_weights();
    unsigned long long pair_weight_groups() const;
    bool lists_checked_ = false; // list capacity verified for the current positions
    bool lists_sized_ = false;   // the first list sizing has been done
    bool lists_full_ = false;    // the last build wrote upper and lower lists too
    uint32_t launches_ = 0;

    // CUDA graph of kGraphSteps steps (the step's buffer rotations return to
    // their start after six steps)
    static constexpr uint32_t kGraphSteps = 6;
    cudaGraphExec_t graph_exec_ = nullptr;
    double graph_dt_ = 0.0;
    uint64_t epoch_ = 1, graph_epoch_ = 0;
    uint32_t graph_launches_ = 0;
    // the buffer rotation the graph was captured in; a replay from any other
    // rotation would read and write the wrong buffers
    struct Rotation {
        StateBufs cur, alt;
        double4* vel_nx;
        F32Bufs fb;
        float4* velf_alt;
    };
    Rotation graph_rot_{};
    Rotation rotation() const { return Rotation{cur_, alt_, vel_nx_, fb_, velf_alt_}; }
    static bool same_rotation(const Rotation& a, const Rotation& b);

    struct PhaseRec {
        int phase;
        cudaEvent_t a, b;
    };
    bool profiling_ = false;
    std::vector<PhaseRec> recs_;
    std::vector<cudaEvent_t> event_pool_;
    double prof_ms_[kNumPhases] = {};
    uint64_t prof_n_[kNumPhases] = {};
    cudaEvent_t take_event();
    void prof_begin(int phase);
    void prof_end();
    void prof_collect();
};

}  // namespace pe
