// Device data layout and kernel entry points of the B200 WCSPH step.
//
// Layout in HBM (one world):
//   * particle state in cell-sorted order ("slots"), structure of double4:
//       pos4[s] = (x, y, z, w)   w = psi for boundary samples,
//                                w = p / rho^2 for fluid (written by the
//                                pressure pass, read by the force pass)
//       vel4[s] = (vx, vy, vz, rho)
//     plus acc4 (a), bf4 (boundary reaction force), p (pressure), flags (u8:
//     bit0 boundary, bit1 oriented boundary), orig (slot -> original index),
//     nout4 (outward normal of oriented boundary samples), key4 (cell key).
//   * a dense cell grid over a fixed key box (ix-major linearisation, so the
//     linear cell order equals the reference's CellKey order), cell_start,
//     and the list of occupied cells.
//   * per-slot neighbour lists in one pool, reserved per chunk of a cell's
//     slots with exact capacities (see ListBufs): the "visit" list holds
//     in-support candidates in the reference's visiting order, flagged lower
//     where the force pass takes them from the "lower" list instead, which
//     holds, for fluid slots, the
//     fluid neighbours with a lower original index in ascending original-index
//     order, and, for boundary slots, all fluid neighbours in ascending
//     original index.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pe {

constexpr uint8_t kFlagBoundary = 1u;
constexpr uint8_t kFlagOriented = 2u;

// List entry: slot in bits 0..28, flags above.
constexpr uint32_t kEntrySlotMask = (1u << 29) - 1u;
constexpr uint32_t kEntryOriented = 1u << 29;
constexpr uint32_t kEntryLower = 1u << 30;
constexpr uint32_t kEntryBoundary = 1u << 31;
constexpr uint64_t kMaxParticles = (1ull << 29) - 1ull;

// Sticky device status bits.
constexpr uint32_t kStatusDomain = 1u;        // a particle left the grid domain
constexpr uint32_t kStatusListOverflow = 2u;  // a neighbour list hit its capacity
constexpr uint32_t kStatusNonFinite = 4u;     // non-finite position seen by the grid
constexpr uint32_t kStatusSlowUnion = 8u;     // informational: a cell used the slow list path

struct GridDesc {
    int32_t kx0, ky0, kz0;  // key of dense cell (0,0,0)
    int32_t nx, ny, nz;     // dense extents
    uint32_t ncell;         // nx*ny*nz
    double inv_cell;        // 1.0 / cell_size (grid.rs:63)
    double cell_size;
    int dim;
};

// Tanks: independent worlds stepped together. Particles are stored tank-major
// (original index = tank's first index + index within the tank); each tank has
// its own dense key box, and the boxes are laid end to end in one cell-id
// space, so the counting sort keeps every tank's particles in the tank's own
// slot range. A single world is one tank.
struct TankDesc {
    int32_t kx0, ky0, kz0;  // key of the tank's dense cell (0,0,0)
    int32_t nx, ny, nz;     // dense extents
    uint32_t cell_base;     // first global cell id of the tank
    uint32_t slot_begin;    // first slot (and original index) of the tank
};

struct Tanks {
    const TankDesc* desc;          // [count]; null selects the single box of GridDesc
    const uint16_t* slot_tank;     // [n] tank of each slot
    const uint16_t* cell_tank;     // [ncell] tank of each dense cell
    double* c;                     // [count] persisted sound speed (wcsph.rs:168)
    unsigned long long* vmax2;     // [count] max |v|^2 of the tank's fluid as u64 bits
    uint32_t count;
};

struct StepConst {
    int dim;
    int kernel;                // KernelKind (kernels.rs:19); 0 = cubic spline
    double h, mass, rho0;      // particles.h, .mass, .rest_density
    double inv_h;              // RN(1 / h), for the exact division by h
    double alpha;              // the kernel's normalisation for (h, dim)
    double rho_self;           // 0.0 + mass * W(0)
    double visc_alpha, visc_beta, eps_h2;  // eps_h2 = visc.eps * h * h
    double eos_rho0, eos_gamma;
    int gamma_int, gamma_is_int;
    double gx, gy, gz;
    double xsph_eps;
    double boundary_eps_h;     // 0.15 * h (particles.rs:132)
    int adapt_sound_speed;
    float r2_filter;           // conservative single-precision (2h)^2 bound
    // List-build modes of the sibling solvers: visit lists keep every
    // boundary candidate whatever its distance; lower lists are built for
    // boundary slots only, holding every fluid candidate.
    int keep_boundary;
    int lower_boundary_only;
};

// Surface-tension constants (surface_tension.rs:112-220), evaluated on the host
// in the reference's operand order.
struct SurfConst {
    int model;     // 1 Akinci 2013, 2 colour field
    double sm2;    // (sigma_eff * m) * m
    double nsm;    // (-sigma_eff) * m
    double coh;    // cohesion normalisation: 32 / (pi h^3) (3-D), 16 / (pi h h) (2-D)
    double gamma;  // colour_gamma
};

struct StateBufs {
    double4* pos;
    double4* vel;
    double4* acc;
    double4* bf;
    double* p;
    uint8_t* flags;
    uint32_t* orig;
    double4* nout;
    int4* key;
};

struct ListBufs {
    uint32_t* pool;                   // list entries, allocated in 16-byte groups
    uint4* desc;                      // per slot: visit list, see list_ref
    uint2* ldesc;                     // per slot: lower list, see list_ref
    uint32_t* ncand;                  // candidates examined per slot (fluid: union size)
    unsigned long long pool_groups;   // capacity of pool in 16-byte groups (< 2^32)
    uint32_t nslots;
    // W(r) of each visit entry at the entry's own index into pool, written by
    // the density pass for the XSPH pass of the same lists and positions;
    // null when the world keeps none. f64 for the f64 step, f32 for the
    // single-precision form. The buffer holds the first w_cap entries of the
    // pool (the list build fills the pool from its start); a density pass
    // that meets a list reaching beyond sets *w_short, and the XSPH pass
    // after it then recomputes W for every particle.
    double* wpair;
    float* wpair32;
    unsigned long long w_cap;
    uint32_t* w_short;
};

// List storage. The list build reserves, for each chunk of consecutive slots
// of one cell, a block of rows of `stride` 16-byte groups, where stride is the
// chunk's slot count and the number of rows covers the chunk's longest list
// (rounded up to 4 entries). Entries t..t+3 of a slot's list are one group,
// and the chunk's slots' groups of a row are contiguous, so the lanes of a
// warp reading entry t of consecutive slots read consecutive 16-byte groups.
//   desc[s]  = (group of row 0 of the visit list (chunk base + lane), stride,
//               visit count, 0)
//   ldesc[s] = (group of row 0 of the lower list, lower count | stride << 16)
enum ListKind : int { kListVisit = 0, kListLower = 2 };

struct ListRef {
    const uint32_t* p;  // entry t at p[(t >> 2) * step + (t & 3)]
    uint32_t step;      // 4 * stride (u32 units between rows)
    uint32_t n;
};

__device__ __forceinline__ ListRef list_ref(const ListBufs& l, uint32_t s, int kind) {
    ListRef r;
    if (kind == kListLower) {
        const uint2 d = __ldg(l.ldesc + s);
        r.p = l.pool + 4 * (size_t)d.x;
        r.step = 4 * (d.y >> 16);
        r.n = d.y & 0xffffu;
        return r;
    }
    const uint4 d = __ldg(l.desc + s);
    r.p = l.pool + 4 * (size_t)d.x;
    r.step = 4 * d.y;
    r.n = d.z;
    return r;
}

// Whether a slot's visit list lies within the pair-weight buffer.
__device__ __forceinline__ bool w_fits(const ListBufs& l, const ListRef& r) {
    const unsigned long long rows = (r.n + 3u) >> 2;
    return rows == 0 || (unsigned long long)(r.p - l.pool) + (rows - 1) * r.step + 4u <= l.w_cap;
}

struct DeviceScalars {
    uint32_t status;
    uint32_t nocc;                  // occupied cells
    uint32_t max_union;             // largest neighbour-cell union seen by the list build
    uint32_t pad_;                  // scratch flag (state import: a position changed)
    unsigned long long list_used;   // 16-byte groups the last list build asked for
    uint32_t import_bad;            // state import: a non-finite value was found
    uint32_t w_short;               // the density pass met a list beyond the pair-weight buffer
};

// Block size of the per-particle passes: a launch parameter, chosen by the
// world's autotuner among 64, 128 and 256.
constexpr int kMaxPassThreads = 256;
struct PassShape {
    uint32_t density = 128, forces = 128, xsph = 128;
};

// Single-precision form (sph_f32.cu).
struct F32Const {
    int dim;
    float h, inv_h, alpha, mass, rho0, rho_self, cell;
    double cell_d;
    float visc_alpha, visc_beta, eps_h2;
    double eos_rho0, eos_gamma_d;
    float inv_eos_rho0, eos_gamma;
    int gamma7;
    float gx, gy, gz, xsph_eps;
    float boundary_eps_h;  // one-sided filter of oriented boundary samples
    int adapt_sound_speed;
};

struct F32Bufs {
    float4* pos;  // cell-local position, w = p / rho^2 (fluid) or psi (boundary)
    float4* vel;  // velocity, w = rho
    uint8_t* kmod;  // cell key mod 4 per axis, two bits each (x | y << 2 | z << 4)
};

void launch_f32_from_f64(uint32_t n, double cell, const StateBufs& s, const F32Bufs& f,
                         cudaStream_t st);
void launch_density_f32(uint32_t n, uint32_t threads, const F32Const& k, const StateBufs& s,
                        const F32Bufs& f, const ListBufs& l, cudaStream_t st);
void launch_pressure_f32(uint32_t n, const F32Const& k, const Tanks& tk, const StateBufs& s,
                         const F32Bufs& f, cudaStream_t st);
void launch_forces_f32(uint32_t n, uint32_t threads, const F32Const& k, const Tanks& tk,
                       const StateBufs& s, const F32Bufs& f, const ListBufs& l, float dt,
                       double4* pos_next, double4* vel_next, float* bf, cudaStream_t st);
void launch_xsph_f32(uint32_t n, uint32_t threads, const F32Const& k, const StateBufs& s,
                     const F32Bufs& f, const ListBufs& l, float4* vel_out, cudaStream_t st,
                     bool use_w = false);

// ----- grid build -----
void launch_cell_ids(const GridDesc& g, const Tanks& tk, uint32_t n, const double4* pos_cur,
                     const double4* pos_next, const uint8_t* flags, uint32_t* cellid, int4* key_tmp,
                     uint32_t* count, DeviceScalars* sc, cudaStream_t st);
size_t scan_temp_bytes(uint32_t ncell);
void launch_scan_cells(uint32_t ncell, const uint32_t* count, uint32_t* cell_start, uint32_t* occ,
                       DeviceScalars* sc, void* temp, cudaStream_t st);
void launch_place(uint32_t n, const uint32_t* cellid, const uint32_t* cell_start, uint32_t* fill,
                  const uint32_t* orig, uint32_t* tmp_old, uint32_t* tmp_orig, cudaStream_t st);
void launch_cellsort(uint32_t ncell_max, const uint32_t* occ, const DeviceScalars* sc,
                     const uint32_t* cell_start, const uint32_t* tmp_old, const uint32_t* tmp_orig,
                     uint32_t* perm, cudaStream_t st);
void launch_gather(uint32_t n, const uint32_t* perm, const StateBufs& src, const double4* pos_next,
                   const double4* vel_next, const int4* key_tmp, const StateBufs& dst,
                   uint32_t* slot_of_orig, double rho0, cudaStream_t st);

// ----- neighbour lists -----
uint32_t nlist_union_capacity(uint32_t max_union);
size_t nlist_smem_bytes(uint32_t ucap, uint32_t chunk = 64);
void launch_surface_tension(uint32_t n, const StepConst& k, const SurfConst& c, const StateBufs& s,
                            const ListBufs& l, double4* normals, double4* out, cudaStream_t st);
// Sets the dynamic shared-memory limit of the list kernel for this stage size
// and returns how many of its CTAs fit on one SM.
// chunk = centre particles per chunk of the list build (32 or 64).
uint32_t nlist_prepare(int dim, uint32_t ucap, uint32_t chunk = 64);
void launch_nlist(const GridDesc& g, const Tanks& tk, const StepConst& k, uint32_t ucap,
                  uint32_t nblocks, const uint32_t* occ, const uint32_t* cell_start,
                  const StateBufs& s, const ListBufs& l, DeviceScalars* sc, cudaStream_t st,
                  bool visit_only = false, uint32_t chunk = 64);

// ----- SPH passes -----
void launch_density(uint32_t n, uint32_t threads, const StepConst& k, const StateBufs& s,
                    const ListBufs& l, cudaStream_t st);
void launch_vmax(uint32_t n, const Tanks& tk, const StateBufs& s, cudaStream_t st);
void launch_pressure(uint32_t n, const StepConst& k, const Tanks& tk, const StateBufs& s,
                     cudaStream_t st);
void forces_prepare();  // once per context, before the first launch_forces
void launch_forces(uint32_t n, uint32_t threads, const StepConst& k, const Tanks& tk,
                   const StateBufs& s, const ListBufs& l, bool integrate, double dt,
                   double4* pos_next, double4* vel_next, const double4* st_a, cudaStream_t st);
void launch_boundary_force(uint32_t n, const StepConst& k, const StateBufs& s, const ListBufs& l,
                           cudaStream_t st);
// use_w: l.wpair holds the W of these lists and positions (written by the
// density pass since the lists were built)
void launch_xsph(uint32_t n, uint32_t threads, const StepConst& k, const StateBufs& s,
                 const ListBufs& l, double4* vel_out, cudaStream_t st, bool use_w = false);

// ----- exports / diagnostics -----
void launch_occupied_export(const GridDesc& g, const uint32_t* occ, const DeviceScalars* sc,
                            const uint32_t* cell_start, const int4* key, int32_t* occ_keys,
                            uint64_t* ranges, cudaStream_t st);
void launch_in_support_counts(uint32_t n, const StepConst& k, const StateBufs& s,
                              const ListBufs& l, uint32_t* out, cudaStream_t st);

}  // namespace pe
