// Host runtime of the WCSPH world: allocation, the step schedule and the
// original-order import/export of state. See world.cuh.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "kernel_any.cuh"
#include "pe_math.cuh"
#include "world.cuh"

namespace pe {

namespace {

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

constexpr unsigned long long kMaxListGroups = 0xffffffffull;  // 32-bit group indices

// out[orig * 3 + c] = src[slot_of_orig[orig]].{x,y,z}
__global__ void k_export_vec(uint32_t n, const uint32_t* __restrict__ slot_of_orig,
                             const double4* __restrict__ src, double* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 v = src[slot_of_orig[i]];
    out[3 * (size_t)i] = v.x;
    out[3 * (size_t)i + 1] = v.y;
    out[3 * (size_t)i + 2] = v.z;
}

// component 3 of a double4 array (rho lives in vel.w) or a plain array
__global__ void k_export_w(uint32_t n, const uint32_t* __restrict__ slot_of_orig,
                           const double4* __restrict__ src4, const double* __restrict__ src1,
                           double* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t s = slot_of_orig[i];
    out[i] = src4 ? src4[s].w : src1[s];
}

// bad = 1 when any of the m values is not finite
__global__ void k_check_finite(uint64_t m, const double* __restrict__ in, uint32_t* bad) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        if (!isfinite(in[i])) *bad = 1u;
}

// changed (optional): set to 1 when any written component differs in its bits
// from what the slot held. Nothing is written when *bad is set.
__global__ void k_import_vec(uint32_t n, const uint32_t* __restrict__ slot_of_orig,
                             const double* __restrict__ in, double4* __restrict__ dst,
                             const uint8_t* __restrict__ flags, int only_fluid, uint32_t* changed,
                             const uint32_t* bad = nullptr) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (bad && *bad) return;
    uint32_t s = slot_of_orig[i];
    if (only_fluid && (flags[s] & kFlagBoundary)) return;
    double4 v = dst[s];
    const double x = in[3 * (size_t)i], y = in[3 * (size_t)i + 1], z = in[3 * (size_t)i + 2];
    if (changed && (__double_as_longlong(x) != __double_as_longlong(v.x) ||
                    __double_as_longlong(y) != __double_as_longlong(v.y) ||
                    __double_as_longlong(z) != __double_as_longlong(v.z)))
        *changed = 1u;
    v.x = x;
    v.y = y;
    v.z = z;
    dst[s] = v;
}

__global__ void k_import_w(uint32_t n, const uint32_t* __restrict__ slot_of_orig,
                           const double* __restrict__ in, double4* __restrict__ dst4,
                           double* __restrict__ dst1) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t s = slot_of_orig[i];
    if (dst4) dst4[s].w = in[i];
    else dst1[s] = in[i];
}

__global__ void k_export_u32(uint32_t n, const uint32_t* __restrict__ slot_of_orig,
                             const uint32_t* __restrict__ src, uint32_t* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = src[slot_of_orig[i]];
}

__global__ void k_export_keys(uint32_t n, const uint32_t* __restrict__ slot_of_orig,
                              const int4* __restrict__ key, int32_t* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int4 k = key[slot_of_orig[i]];
    out[3 * (size_t)i] = k.x;
    out[3 * (size_t)i + 1] = k.y;
    out[3 * (size_t)i + 2] = k.z;
}

__global__ void k_export_kind(uint32_t n, const uint32_t* __restrict__ slot_of_orig,
                              const uint8_t* __restrict__ flags, uint8_t* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = flags[slot_of_orig[i]] & kFlagBoundary;
}

// Fluid slots cache p / rho^2 in pos.w; refresh it after p or rho were set.
__global__ void k_refresh_pr2(uint32_t n, const uint8_t* __restrict__ flags,
                              const double* __restrict__ p, double4* __restrict__ pos,
                              const double4* __restrict__ vel) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (flags[i] & kFlagBoundary)) return;
    double rho = vel[i].w;
    pos[i].w = p[i] / (rho * rho);
}

}  // namespace

void World::check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
    }
}

template <typename T>
T* World::alloc(size_t count) {
    void* p = nullptr;
    size_t bytes = std::max<size_t>(count * sizeof(T), 256);
    check(cudaMalloc(&p, bytes), "cudaMalloc");
    allocs_.push_back(p);
    check(cudaMemsetAsync(p, 0, bytes, st_), "cudaMemsetAsync");
    return static_cast<T*>(p);
}

World::World(const WorldParams& prm, const WorldConfig& cfg, int dim, double rest_density,
             double mass, double h, uint64_t n, const double* x, const double* v,
             const uint8_t* kind, const double* psi, const double* n_out,
             const uint64_t* tank_offsets, uint32_t n_tanks, double support)
    : dim_(dim), rho0_(rest_density), mass_(mass), h_(h),
      support_(support > 0.0 ? support : kernel_support(prm.kernel, h)),
      n_(n), prm_(prm), cfg_(cfg) {
    if (cfg_.device >= 0) check(cudaSetDevice(cfg_.device), "cudaSetDevice");
    check(cudaGetDevice(&device_), "cudaGetDevice");
    // ---- tanks: contiguous particle ranges ----
    std::vector<uint64_t> toff;
    if (tank_offsets && n_tanks >= 1) {
        if (n_tanks > 65535u) throw std::length_error("too many tanks");
        toff.assign(tank_offsets, tank_offsets + n_tanks + 1);
        if (toff.front() != 0 || toff.back() != n_) throw std::invalid_argument("tank offsets");
        for (uint32_t t = 0; t < n_tanks; ++t)
            if (toff[t + 1] <= toff[t]) throw std::invalid_argument("empty or unordered tank");
    } else {
        n_tanks = 1;
        toff = {0, n_};
    }
    n_tanks_ = n_tanks;
    check(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "cudaStreamCreate");
    try {
        // ---- each tank's grid domain from its initial keys (grid.rs:62 key_of) ----
        const double cell = support_;  // support_radius, kernels.rs:32 (grid.rs:48 cell = support)
        const double inv = 1.0 / cell;
        const double frac = cfg_.domain_margin < 0.0 ? 0.25 : cfg_.domain_margin;
        const long long minc = cfg_.domain_margin_cells ? cfg_.domain_margin_cells : 4;
        tank_host_.resize(n_tanks_);
        uint64_t total_cells = 0;
        for (uint32_t t = 0; t < n_tanks_; ++t) {
            long long lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
            for (uint64_t i = toff[t]; i < toff[t + 1]; ++i) {
                long long k3[3] = {floor_i32(x[3 * i] * inv), floor_i32(x[3 * i + 1] * inv),
                                   dim_ == 2 ? 0 : floor_i32(x[3 * i + 2] * inv)};
                for (int a = 0; a < 3; ++a) {
                    if (i == toff[t] || k3[a] < lo[a]) lo[a] = k3[a];
                    if (i == toff[t] || k3[a] > hi[a]) hi[a] = k3[a];
                }
            }
            long long ext[3];
            for (int a = 0; a < 3; ++a) {
                if (dim_ == 2 && a == 2) {
                    lo[a] = hi[a] = 0;
                    ext[a] = 1;
                    continue;
                }
                long long span = hi[a] - lo[a] + 1;
                long long m = std::max<long long>(minc, (long long)std::ceil(frac * (double)span));
                lo[a] = std::max<long long>(lo[a] - m, -2147483647LL);
                hi[a] = std::min<long long>(hi[a] + m, 2147483646LL);
                ext[a] = hi[a] - lo[a] + 1;
            }
            const double ncell = (double)ext[0] * (double)ext[1] * (double)ext[2];
            if (ncell > (double)(1u << 28)) throw std::length_error("grid domain too large");
            TankDesc& td = tank_host_[t];
            td.kx0 = (int32_t)lo[0];
            td.ky0 = (int32_t)lo[1];
            td.kz0 = (int32_t)lo[2];
            td.nx = (int32_t)ext[0];
            td.ny = (int32_t)ext[1];
            td.nz = (int32_t)ext[2];
            td.cell_base = (uint32_t)total_cells;
            td.slot_begin = (uint32_t)toff[t];
            total_cells += (uint64_t)ncell;
            if (total_cells > (1ull << 31)) throw std::length_error("grid domain too large");
        }
        g_.kx0 = tank_host_[0].kx0;
        g_.ky0 = tank_host_[0].ky0;
        g_.kz0 = tank_host_[0].kz0;
        g_.nx = tank_host_[0].nx;
        g_.ny = tank_host_[0].ny;
        g_.nz = tank_host_[0].nz;
        g_.ncell = (uint32_t)total_cells;
        g_.inv_cell = inv;
        g_.cell_size = cell;
        g_.dim = dim_;

        f32_ = cfg_.precision == 1;
        pair_w_on_ = cfg_.pair_weights != 0;
        if (f32_ && prm_.surface_tension_sigma != 0.0)
            throw std::invalid_argument("surface tension needs the f64 step");
        if (f32_ && prm_.kernel != 0) throw std::invalid_argument("the single-precision form is cubic-spline only");
        refresh_step_const();
        configure_surface_tension();

        // ---- union stage capacity from the largest initial neighbour-cell union ----
        std::vector<uint32_t> cnt(g_.ncell, 0);
        std::vector<uint16_t> cell_tank(g_.ncell, 0);
        uint32_t max_union = 1;
        for (uint32_t t = 0; t < n_tanks_; ++t) {
            const TankDesc& td = tank_host_[t];
            const size_t cells_t = (size_t)td.nx * td.ny * td.nz;
            std::fill(cell_tank.begin() + td.cell_base, cell_tank.begin() + td.cell_base + cells_t,
                      (uint16_t)t);
            uint32_t* c = cnt.data() + td.cell_base;
            std::vector<uint32_t> occupied;
            for (uint64_t i = toff[t]; i < toff[t + 1]; ++i) {
                long long kx = floor_i32(x[3 * i] * inv) - td.kx0, ky = floor_i32(x[3 * i + 1] * inv) - td.ky0;
                long long kz = dim_ == 2 ? 0 : floor_i32(x[3 * i + 2] * inv) - td.kz0;
                const uint32_t lc = (uint32_t)((kx * td.ny + ky) * td.nz + kz);
                if (c[lc]++ == 0) occupied.push_back(lc);
            }
            for (uint32_t lc : occupied) {
                const int cz = (int)(lc % (uint32_t)td.nz), cy = (int)((lc / (uint32_t)td.nz) % (uint32_t)td.ny);
                const int cx = (int)(lc / ((uint32_t)td.nz * (uint32_t)td.ny));
                uint32_t u = 0;
                for (int dx = -1; dx <= 1; ++dx)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dz = (dim_ == 2 ? 0 : -1); dz <= (dim_ == 2 ? 0 : 1); ++dz) {
                            int qx = cx + dx, qy = cy + dy, qz = cz + dz;
                            if (qx < 0 || qy < 0 || qz < 0 || qx >= td.nx || qy >= td.ny || qz >= td.nz) continue;
                            u += c[((size_t)qx * td.ny + qy) * td.nz + qz];
                        }
                max_union = std::max(max_union, u);
            }
        }
        ucap_ = nlist_union_capacity(max_union);

        // ---- allocations ----
        const size_t N = std::max<uint64_t>(n_, 1);
        auto make_state = [&](StateBufs& s) {
            s.pos = alloc<double4>(N);
            s.vel = alloc<double4>(N);
            s.acc = alloc<double4>(N);
            s.bf = alloc<double4>(N);
            s.p = alloc<double>(N);
            s.flags = alloc<uint8_t>(N);
            s.orig = alloc<uint32_t>(N);
            s.nout = alloc<double4>(N);
            s.key = alloc<int4>(N);
        };
        make_state(cur_);
        make_state(alt_);
        pos_nx_ = alloc<double4>(N);
        vel_nx_ = alloc<double4>(N);
        slot_of_orig_ = alloc<uint32_t>(N);
        cellid_ = alloc<uint32_t>(N);
        tmp_old_ = alloc<uint32_t>(N);
        tmp_orig_ = alloc<uint32_t>(N);
        perm_ = alloc<uint32_t>(N);
        key_tmp_ = alloc<int4>(N);
        count_ = alloc<uint32_t>(g_.ncell);
        fill_ = alloc<uint32_t>(g_.ncell);
        cell_start_ = alloc<uint32_t>((size_t)g_.ncell + 1);
        occ_ = alloc<uint32_t>(g_.ncell);
        scan_tmp_ = alloc<unsigned char>(scan_temp_bytes(g_.ncell));
        lists_.nslots = (uint32_t)N;
        // first guess of the list pool: max_neighbours entries per slot (the
        // first build measures the need and resizes)
        const uint64_t want = cfg_.max_neighbours ? cfg_.max_neighbours : 256u;
        alloc_lists((unsigned long long)N * ((want + 3u) / 4u));
        lists_.desc = alloc<uint4>(N);
        lists_.ldesc = alloc<uint2>(N);
        lists_.ncand = alloc<uint32_t>(N);
        insup_ = alloc<uint32_t>(N);
        sc_ = alloc<DeviceScalars>(1);
        lists_.w_short = &sc_->w_short;
        {
            TankDesc* d_desc = alloc<TankDesc>(n_tanks_);
            uint16_t* d_slot_tank = alloc<uint16_t>(N);
            uint16_t* d_cell_tank = alloc<uint16_t>(g_.ncell);
            tanks_.c = alloc<double>(n_tanks_);
            tanks_.vmax2 = alloc<unsigned long long>(n_tanks_);
            std::vector<uint16_t> slot_tank(N, 0);
            for (uint32_t t = 0; t < n_tanks_; ++t)
                std::fill(slot_tank.begin() + toff[t], slot_tank.begin() + toff[t + 1], (uint16_t)t);
            std::vector<double> c0(n_tanks_, prm_.eos_sound_speed);
            check(cudaMemcpyAsync(d_desc, tank_host_.data(), sizeof(TankDesc) * n_tanks_,
                                  cudaMemcpyHostToDevice, st_), "upload");
            check(cudaMemcpyAsync(d_slot_tank, slot_tank.data(), sizeof(uint16_t) * N,
                                  cudaMemcpyHostToDevice, st_), "upload");
            check(cudaMemcpyAsync(d_cell_tank, cell_tank.data(), sizeof(uint16_t) * g_.ncell,
                                  cudaMemcpyHostToDevice, st_), "upload");
            check(cudaMemcpyAsync(tanks_.c, c0.data(), sizeof(double) * n_tanks_, cudaMemcpyHostToDevice, st_),
                  "upload");
            // the host vectors must outlive the copies
            check(cudaStreamSynchronize(st_), "upload");
            tanks_.desc = d_desc;
            tanks_.slot_tank = d_slot_tank;
            tanks_.cell_tank = d_cell_tank;
            tanks_.count = n_tanks_;
        }
        xfer_ = alloc<double>(N * 4);
        if (f32_) {
            fb_.pos = alloc<float4>(N);
            fb_.vel = alloc<float4>(N);
            fb_.kmod = alloc<uint8_t>(N);
            velf_alt_ = alloc<float4>(N);
            bf32_ = alloc<float>(4 * N);
        }

        // ---- upload in original order (slot = original index) ----
        std::vector<double4> hp(N), hv(N), hn(N);
        std::vector<uint8_t> hf(N, 0);
        std::vector<uint32_t> ho(N);
        for (uint64_t i = 0; i < n_; ++i) {
            bool b = kind[i] != 0;
            double nx = n_out ? n_out[3 * i] : 0.0, ny = n_out ? n_out[3 * i + 1] : 0.0,
                   nz = n_out ? n_out[3 * i + 2] : 0.0;
            hp[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], b ? psi[i] : 0.0);
            hv[i] = make_double4(v ? v[3 * i] : 0.0, v ? v[3 * i + 1] : 0.0, v ? v[3 * i + 2] : 0.0,
                                 rest_density);
            hn[i] = make_double4(nx, ny, nz, 0.0);
            bool oriented = b && (nx * nx + ny * ny + nz * nz) > 0.0;
            hf[i] = (b ? kFlagBoundary : 0) | (oriented ? kFlagOriented : 0);
            ho[i] = (uint32_t)i;
        }
        check(cudaMemcpyAsync(cur_.pos, hp.data(), N * sizeof(double4), cudaMemcpyHostToDevice, st_), "upload");
        check(cudaMemcpyAsync(cur_.vel, hv.data(), N * sizeof(double4), cudaMemcpyHostToDevice, st_), "upload");
        check(cudaMemcpyAsync(cur_.nout, hn.data(), N * sizeof(double4), cudaMemcpyHostToDevice, st_), "upload");
        check(cudaMemcpyAsync(cur_.flags, hf.data(), N, cudaMemcpyHostToDevice, st_), "upload");
        check(cudaMemcpyAsync(cur_.orig, ho.data(), N * sizeof(uint32_t), cudaMemcpyHostToDevice, st_), "upload");
        check(cudaMemcpyAsync(slot_of_orig_, ho.data(), N * sizeof(uint32_t), cudaMemcpyHostToDevice, st_), "upload");
        DeviceScalars hs{};
        check(cudaMemcpyAsync(sc_, &hs, sizeof(hs), cudaMemcpyHostToDevice, st_), "upload");

        // ---- launch geometry of the list build: a persistent grid ----
        int sms = 148;
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "attribute");
        sms_ = (uint32_t)sms;
        configure_lists();
        check(cudaStreamSynchronize(st_), "create");
    } catch (...) {
        for (void* p : allocs_) cudaFree(p);
        allocs_.clear();
        for (void* p : list_allocs_) cudaFree(p);
        list_allocs_.clear();
        if (st_) cudaStreamDestroy(st_);
        st_ = nullptr;
        throw;
    }
}

void World::alloc_lists(unsigned long long groups) {
    for (void* p : list_allocs_) cudaFree(p);
    list_allocs_.clear();
    lists_.pool = nullptr;
    lists_.pool_groups = 0;
    // group indices are 32-bit: at most 2^32 - 1 groups (64 GB) of entries
    groups = std::min<unsigned long long>(std::max<unsigned long long>(groups, 1024ull), kMaxListGroups);
    void* p = nullptr;
    check(cudaMalloc(&p, groups * 16ull), "cudaMalloc lists");
    list_allocs_.push_back(p);
    lists_.pool = static_cast<uint32_t*>(p);
    lists_.pool_groups = groups;
    lists_.wpair = nullptr;
    lists_.wpair32 = nullptr;
    lists_.w_cap = 0;
    w_valid_ = false;
    if (pair_w_on_) alloc_pair_weights(pair_weight_groups());
    lists_valid_ = false;
    invalidate_graph();
}

// The list build fills the pool from its start, and a freshly sized pool is
// twice the need (it grows when a build asks for more than 75%). The buffer
// covers the pool's first 5/8 (1.25x the need); a build whose lists reach
// past that is caught by the density pass (w_short: XSPH recomputes W), and
// the next status poll extends the buffer to the whole pool.
unsigned long long World::pair_weight_groups() const {
    return std::min<unsigned long long>(lists_.pool_groups, (lists_.pool_groups * 5ull + 7ull) / 8ull);
}

void World::alloc_pair_weights(unsigned long long groups) {
    if (pair_weights() || !groups) return;
    // Kept only with room to spare: the buffer is an optimisation, so it
    // gives way to the list pool (a 512-tank batch's pool alone is ~55 GB).
    const size_t bytes = (size_t)groups * 4u * (f32_ ? sizeof(float) : sizeof(double));
    constexpr size_t kHeadroom = 2ull << 30;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b < bytes + kHeadroom) {
        cudaGetLastError();
        return;
    }
    void* w = nullptr;
    if (cudaMalloc(&w, bytes) != cudaSuccess) {
        cudaGetLastError();  // no buffer: XSPH recomputes W
        return;
    }
    list_allocs_.push_back(w);
    if (f32_) lists_.wpair32 = static_cast<float*>(w);
    else lists_.wpair = static_cast<double*>(w);
    lists_.w_cap = groups * 4ull;
    w_valid_ = false;
}

void World::free_pair_weights() {
    void* const w = lists_.wpair ? (void*)lists_.wpair : (void*)lists_.wpair32;
    if (!w) return;
    check(cudaStreamSynchronize(st_), "pair weights");
    for (auto it = list_allocs_.begin(); it != list_allocs_.end(); ++it)
        if (*it == w) {
            cudaFree(*it);
            list_allocs_.erase(it);
            break;
        }
    lists_.wpair = nullptr;
    lists_.wpair32 = nullptr;
    lists_.w_cap = 0;
    w_valid_ = false;
}

void World::pair_weight_info(uint64_t out[3]) {
    DeviceScalars hs{};
    check(cudaMemcpyAsync(&hs, sc_, sizeof(hs), cudaMemcpyDeviceToHost, st_), "pair weights");
    check(cudaStreamSynchronize(st_), "pair weights");
    out[0] = pair_weights() ? 1u : 0u;
    out[1] = lists_.w_cap;
    out[2] = pair_weights() && hs.w_short ? 1u : 0u;
}

void World::set_pair_weights(bool on) {
    if (on == pair_w_on_ && (!on || pair_weights())) return;
    pair_w_on_ = on;
    if (on) alloc_pair_weights(pair_weight_groups());
    else free_pair_weights();
    invalidate_graph();  // a captured step bakes in which XSPH kernel runs
}

World::~World() {
    if (st_) cudaStreamSynchronize(st_);
    release_graph();
    for (void* p : {(void*)ck_pos_, (void*)ck_vel_, (void*)ck_p_, (void*)judge_err_})
        if (p) cudaFree(p);
    for (void* p : list_allocs_) cudaFree(p);
    for (auto& r : recs_) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : event_pool_) cudaEventDestroy(e);
    for (void* p : allocs_) cudaFree(p);
    if (st_) cudaStreamDestroy(st_);
}

cudaEvent_t World::take_event() {
    if (!event_pool_.empty()) {
        cudaEvent_t e = event_pool_.back();
        event_pool_.pop_back();
        return e;
    }
    cudaEvent_t e;
    check(cudaEventCreate(&e), "cudaEventCreate");
    return e;
}

void World::prof_begin(int phase) {
    if (!profiling_) return;
    PhaseRec r{phase, take_event(), take_event()};
    check(cudaEventRecord(r.a, st_), "cudaEventRecord");
    recs_.push_back(r);
}

void World::prof_end() {
    if (!profiling_ || recs_.empty()) return;
    check(cudaEventRecord(recs_.back().b, st_), "cudaEventRecord");
    if (recs_.size() >= 4096) prof_collect();
}

void World::prof_collect() {
    check(cudaStreamSynchronize(st_), "profile");
    for (auto& r : recs_) {
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, r.a, r.b), "cudaEventElapsedTime");
        prof_ms_[r.phase] += ms;
        prof_n_[r.phase] += 1;
        event_pool_.push_back(r.a);
        event_pool_.push_back(r.b);
    }
    recs_.clear();
}

void World::profile_read(double* ms, uint64_t* count, bool reset) {
    prof_collect();
    for (int p = 0; p < kNumPhases; ++p) {
        if (ms) ms[p] = prof_ms_[p];
        if (count) count[p] = prof_n_[p];
        if (reset) {
            prof_ms_[p] = 0.0;
            prof_n_[p] = 0;
        }
    }
}

void World::refresh_step_const() {
    StepConst k{};
    k.dim = dim_;
    k.h = h_;
    k.inv_h = 1.0 / h_;
    k.mass = mass_;
    k.rho0 = rho0_;
    k.kernel = prm_.kernel;
    const KernelFn kf = make_kernel_fn(prm_.kernel, h_, dim_);
    k.alpha = kf.alpha;
    // wcsph.rs:133-135: rho = 0.0; rho += mass * w(kern, 0.0, h, dim)
    k.rho_self = 0.0 + mass_ * kfn_w(kf, 0.0);
    k.visc_alpha = prm_.visc_alpha;
    k.visc_beta = prm_.visc_beta;
    k.eps_h2 = prm_.visc_eps * h_ * h_;  // viscosity.rs:63
    k.eos_rho0 = prm_.eos_rest_density;
    k.eos_gamma = prm_.eos_gamma;
    bool is_int = false;
    k.gamma_int = integer_exponent(prm_.eos_gamma, &is_int);
    k.gamma_is_int = is_int ? 1 : 0;
    k.gx = prm_.gravity[0];
    k.gy = prm_.gravity[1];
    k.gz = prm_.gravity[2];
    k.xsph_eps = prm_.xsph_epsilon;
    k.boundary_eps_h = 0.15 * h_;  // particles.rs:132
    k.adapt_sound_speed = prm_.adapt_sound_speed;
    double sup = support_;
    k.r2_filter = list_all_candidates_
                      ? std::numeric_limits<float>::infinity()
                      : std::nextafter((float)(sup * sup * (1.0 + 1e-4)), std::numeric_limits<float>::infinity());
    k.keep_boundary = list_keep_boundary_ ? 1 : 0;
    k.lower_boundary_only = list_keep_boundary_ ? 1 : 0;
    kc_ = k;

    F32Const f{};
    f.dim = dim_;
    f.h = (float)h_;
    f.inv_h = (float)(1.0 / h_);
    f.alpha = (float)k.alpha;
    f.mass = (float)mass_;
    f.rho0 = (float)rho0_;
    f.rho_self = (float)k.rho_self;
    f.cell = (float)(2.0 * h_);
    f.cell_d = 2.0 * h_;
    f.visc_alpha = (float)prm_.visc_alpha;
    f.visc_beta = (float)prm_.visc_beta;
    f.eps_h2 = (float)k.eps_h2;
    f.eos_rho0 = prm_.eos_rest_density;
    f.eos_gamma_d = prm_.eos_gamma;
    f.inv_eos_rho0 = (float)(1.0 / prm_.eos_rest_density);
    f.eos_gamma = (float)prm_.eos_gamma;
    f.gamma7 = prm_.eos_gamma == 7.0;
    f.gx = (float)prm_.gravity[0];
    f.gy = (float)prm_.gravity[1];
    f.gz = (float)prm_.gravity[2];
    f.xsph_eps = (float)prm_.xsph_epsilon;
    f.boundary_eps_h = (float)k.boundary_eps_h;
    f.adapt_sound_speed = prm_.adapt_sound_speed;
    kf_ = f;
    invalidate_graph();
}

void World::refresh_f32() {
    if (!f32_) return;
    launch_f32_from_f64((uint32_t)n_, 2.0 * h_, cur_, fb_, st_);
    launches_ += 1;
    check(cudaGetLastError(), "f32 state");
}

void World::set_params(const WorldParams& p) {
    if (f32_ && p.surface_tension_sigma != 0.0)
        throw std::invalid_argument("surface tension needs the f64 step");
    if (f32_ && p.kernel != 0) throw std::invalid_argument("the single-precision form is cubic-spline only");
    if (kernel_support(p.kernel, h_) != kernel_support(prm_.kernel, h_))
        throw std::invalid_argument("the kernel's support radius is fixed at creation");
    bool c_changed = p.eos_sound_speed != prm_.eos_sound_speed;
    prm_ = p;
    refresh_step_const();
    configure_surface_tension();
    if (c_changed) set_sound_speed(p.eos_sound_speed);
}

double World::sound_speed() {
    double c = 0.0;
    check(cudaMemcpyAsync(&c, tanks_.c, sizeof(double), cudaMemcpyDeviceToHost, st_), "get c");
    check(cudaStreamSynchronize(st_), "get c");
    prm_.eos_sound_speed = c;
    return c;
}

void World::get_sound_speeds(double* out) {
    check(cudaMemcpyAsync(out, tanks_.c, sizeof(double) * n_tanks_, cudaMemcpyDeviceToHost, st_), "get c");
    check(cudaStreamSynchronize(st_), "get c");
}

void World::set_sound_speed(double c) {
    prm_.eos_sound_speed = c;
    std::vector<double> all(n_tanks_, c);
    check(cudaMemcpyAsync(tanks_.c, all.data(), sizeof(double) * n_tanks_, cudaMemcpyHostToDevice, st_),
          "set c");
    check(cudaStreamSynchronize(st_), "set c");
}

void World::synchronize() { check(cudaStreamSynchronize(st_), "synchronize"); }

void World::build_grid(const double4* pos_next, const double4* vel_next) {
    const uint32_t n = (uint32_t)n_;
    prof_begin(kGrid);
    check(cudaMemsetAsync(count_, 0, sizeof(uint32_t) * g_.ncell, st_), "memset");
    check(cudaMemsetAsync(fill_, 0, sizeof(uint32_t) * g_.ncell, st_), "memset");
    launch_cell_ids(g_, tanks_, n, cur_.pos, pos_next, cur_.flags, cellid_, key_tmp_, count_, sc_, st_);
    launch_scan_cells(g_.ncell, count_, cell_start_, occ_, sc_, scan_tmp_, st_);
    launch_place(n, cellid_, cell_start_, fill_, cur_.orig, tmp_old_, tmp_orig_, st_);
    launch_cellsort(std::min<uint32_t>(g_.ncell, n ? n : 1), occ_, sc_, cell_start_, tmp_old_, tmp_orig_,
                    perm_, st_);
    launch_gather(n, perm_, cur_, pos_next, vel_next, key_tmp_, alt_, slot_of_orig_, rho0_, st_);
    launches_ += 7;
    prof_end();
    std::swap(cur_, alt_);
    grid_built_ = true;
    lists_valid_ = false;
    w_valid_ = false;
    check(cudaGetLastError(), "grid build");
}

void World::ensure_lists(bool visit_only) {
    // the f32 form and the learned step read the visit list only
    const bool build_visit_only = f32_ || visit_only;
    if (lists_valid_ && (lists_full_ || build_visit_only)) return;
    w_valid_ = false;
    if (!grid_built_) {
        // No grid yet: every neighbour query of the reference returns nothing.
        check(cudaMemsetAsync(lists_.desc, 0, sizeof(uint4) * lists_.nslots, st_), "memset");
        check(cudaMemsetAsync(lists_.ldesc, 0, sizeof(uint2) * lists_.nslots, st_), "memset");
        check(cudaMemsetAsync(lists_.ncand, 0, sizeof(uint32_t) * lists_.nslots, st_), "memset");
    } else {
        // Every pass of this loop builds into the current pool, so the loop
        // always ends with lists built in the pool they describe.
        for (int attempt = 0;; ++attempt) {
            check(cudaMemsetAsync(&sc_->list_used, 0, sizeof(unsigned long long), st_), "memset");
            prof_begin(kLists);
            launch_nlist(g_, tanks_, kc_, ucap_, nl_blocks_, occ_, cell_start_, cur_, lists_, sc_, st_,
                         build_visit_only, list_chunk_);
            prof_end();
            launches_ += 1;
            check(cudaGetLastError(), "neighbour lists");
            if (lists_checked_) break;
            // First build for these positions: size the pool from what the
            // build asked for before any pass consumes the lists.
            DeviceScalars hs{};
            check(cudaMemcpyAsync(&hs, sc_, sizeof(hs), cudaMemcpyDeviceToHost, st_), "lists");
            check(cudaStreamSynchronize(st_), "lists");
            const unsigned long long need = hs.list_used, have = lists_.pool_groups;
            const bool overflowed = need > have || (hs.status & kStatusListOverflow);
            const bool at_max = have >= kMaxListGroups;
            // The very first sizing keeps twice the need (lists grow by ~40%
            // in a few steps when a free-surface start collapses); later
            // checks (after the host moved particles) use the 75% rule that
            // runs poll, so a slowly compressing tank does not reallocate on
            // every set_positions. A pool at its maximum only has to hold the need.
            const bool fits = at_max ? need <= have
                                     : (lists_sized_ ? need * 4 <= have * 3 : need * 2 <= have);
            if (!overflowed && (fits || attempt >= 3)) {
                lists_checked_ = true;
                lists_sized_ = true;
                break;
            }
            if (overflowed && (at_max || attempt >= 3))
                throw std::length_error("neighbour lists exceed the 64 GB pool limit");
            alloc_lists(2 * need);
            if (overflowed) {
                // this build is discarded: clear its status bit
                const uint32_t keep = hs.status & ~kStatusListOverflow;
                check(cudaMemcpyAsync(&sc_->status, &keep, sizeof(uint32_t), cudaMemcpyHostToDevice, st_),
                      "status");
            }
            // rebuild into the new pool
        }
    }
    check(cudaGetLastError(), "neighbour lists");
    lists_valid_ = true;
    lists_full_ = grid_built_ && !build_visit_only;
}

void World::run_density(bool visit_only) {
    ensure_lists(visit_only);
    if (pair_weights()) check(cudaMemsetAsync(&sc_->w_short, 0, sizeof(uint32_t), st_), "memset");
    prof_begin(kDensity);
    if (f32_) launch_density_f32((uint32_t)n_, shape_.density, kf_, cur_, fb_, lists_, st_);
    else launch_density((uint32_t)n_, shape_.density, kc_, cur_, lists_, st_);
    prof_end();
    launches_ += 1;
    check(cudaGetLastError(), "density");
    w_valid_ = pair_weights();
}

void World::run_pressure() {
    prof_begin(kPressure);
    if (prm_.adapt_sound_speed)
        check(cudaMemsetAsync(tanks_.vmax2, 0, sizeof(unsigned long long) * n_tanks_, st_), "memset");
    if (f32_) {
        launch_pressure_f32((uint32_t)n_, kf_, tanks_, cur_, fb_, st_);
        launches_ += kf_.adapt_sound_speed ? 1 : 0;
    } else {
        if (kc_.adapt_sound_speed) {
            launch_vmax((uint32_t)n_, tanks_, cur_, st_);
            launches_ += 1;
        }
        launch_pressure((uint32_t)n_, kc_, tanks_, cur_, st_);
    }
    prof_end();
    launches_ += 1;
    check(cudaGetLastError(), "pressure");
}

void World::run_forces(bool integrate, double dt) {
    ensure_lists();
    if (f32_) {
        // the single-precision form always integrates into the next buffers;
        // without a kick/drift request the step is taken with dt = 0
        prof_begin(kForces);
        launch_forces_f32((uint32_t)n_, shape_.forces, kf_, tanks_, cur_, fb_, lists_,
                          integrate ? (float)dt : 0.f, pos_nx_, vel_nx_, bf32_, st_);
        prof_end();
        launches_ += 2;
    } else {
        const bool surf = prm_.surface_tension_sigma != 0.0;  // wcsph.rs:262
        if (surf) run_surface_tension();
        prof_begin(kForces);
        launch_forces((uint32_t)n_, shape_.forces, kc_, tanks_, cur_, lists_, integrate, dt, pos_nx_,
                      vel_nx_, surf ? st_a_ : nullptr, st_);
        prof_end();
        prof_begin(kBoundaryForce);
        launch_boundary_force((uint32_t)n_, kc_, cur_, lists_, st_);
        prof_end();
        launches_ += 2;
    }
    check(cudaGetLastError(), "forces");
}

// surface_tension.rs:112-220 into st_a_ (model none: zeros, which wcsph.rs:274
// still adds)
void World::run_surface_tension() {
    configure_surface_tension();
    const uint32_t n = (uint32_t)n_;
    if (prm_.surface_tension_model == 0) return;  // st_a_ holds zeros
    SurfConst c{};
    c.model = prm_.surface_tension_model;
    const double pi = 3.14159265358979311599796346854;  // f64::consts::PI
    const double sigma_eff = prm_.surface_tension_sigma * (dim_ == 2 ? 1.0 / 20.0 : 1.0);
    c.sm2 = sigma_eff * mass_ * mass_;
    c.nsm = -sigma_eff * mass_;
    c.coh = dim_ == 2 ? 16.0 / (pi * h_ * h_) : 32.0 / (pi * pow_int_dd(h_, 3));
    c.gamma = prm_.surface_tension_colour_gamma;
    launch_surface_tension(n, kc_, c, cur_, lists_, st_normals_, st_a_, st_);
    launches_ += 2;
    check(cudaGetLastError(), "surface tension");
}

// Buffers and list mode of the surface-tension branch: the Akinci curvature
// term sums over every fluid candidate of the neighbour cells, so that model
// needs lists holding all of them.
void World::configure_surface_tension() {
    const bool on = prm_.surface_tension_sigma != 0.0;
    if (on && !st_a_) {
        const size_t N = std::max<uint64_t>(n_, 1);
        st_normals_ = alloc<double4>(N);
        st_a_ = alloc<double4>(N);  // zeroed
    }
    const bool all = on && prm_.surface_tension_model == 1;
    if (all != list_all_candidates_) {
        list_all_candidates_ = all;
        refresh_step_const();
        lists_valid_ = false;
        lists_checked_ = false;
        invalidate_graph();
    }
}

void World::run_xsph() {
    if (prm_.xsph_epsilon == 0.0) return;  // wcsph.rs:285
    ensure_lists();
    prof_begin(kXsph);
    if (f32_) {
        launch_xsph_f32((uint32_t)n_, shape_.xsph, kf_, cur_, fb_, lists_, velf_alt_, st_, w_valid_);
        prof_end();
        launches_ += w_valid_ ? 2 : 1;  // with weights: the weight-reading kernel and its fallback
        check(cudaGetLastError(), "xsph");
        std::swap(fb_.vel, velf_alt_);
        return;
    }
    launch_xsph((uint32_t)n_, shape_.xsph, kc_, cur_, lists_, vel_nx_, st_, w_valid_);
    prof_end();
    launches_ += w_valid_ ? 2 : 1;  // with weights: the weight-reading kernel and its fallback
    check(cudaGetLastError(), "xsph");
    std::swap(cur_.vel, vel_nx_);
    // the swapped-out buffer of the alternate state must stay a valid full copy
    // only for the current layout, which vel_nx_ is not needed for.
}

void World::rebuild_grid() {
    build_grid(nullptr, nullptr);
    refresh_f32();
    grid_current_ = true;
    rho_current_ = false;
}

void World::compute_density() {
    run_density();
    rho_current_ = grid_current_;
}

void World::compute_pressure() { run_pressure(); }

void World::compute_forces() { run_forces(false, 0.0); }

void World::apply_xsph() { run_xsph(); }

void World::step(double dt) {
    // wcsph.rs:327-328. When the previous step ended with a grid and densities
    // of the current positions, rebuilding them reproduces the same bits, so
    // they are reused.
    if (!(grid_current_ && rho_current_)) {
        build_grid(nullptr, nullptr);
        refresh_f32();
        run_density();
    }
    run_pressure();               // wcsph.rs:329
    run_forces(true, dt);         // wcsph.rs:330-342 (kick + drift fused)
    build_grid(pos_nx_, vel_nx_); // wcsph.rs:343
    refresh_f32();
    run_density();                // wcsph.rs:344
    run_xsph();                   // wcsph.rs:345
    t_ += dt;                     // wcsph.rs:346
    grid_current_ = true;
    rho_current_ = true;
}

void World::run(double dt, uint64_t steps) {
    uint64_t s = 0, last_poll = 0;
    while (s < steps) {
        if (cfg_.use_graph && steps - s >= kGraphSteps && graph_capturable()) {
            if (!graph_exec_ || graph_dt_ != dt || graph_epoch_ != epoch_ ||
                !same_rotation(graph_rot_, rotation()))
                capture_graph(dt);
            if (graph_exec_) {
                check(cudaGraphLaunch(graph_exec_, st_), "graph launch");
                s += kGraphSteps;
                for (uint32_t k = 0; k < kGraphSteps; ++k) t_ += dt;  // wcsph.rs:346, once per step
                launches_ += graph_launches_;
                if (s - last_poll >= 16) {
                    status();
                    last_poll = s;
                }
                continue;
            }
        }
        step(dt);
        ++s;
        if (s - last_poll >= 16) {
            status();  // lets the list storage and stage grow if needed
            last_poll = s;
        }
    }
}

// A step can be captured when it issues no host synchronisation: the grid and
// densities are current (no initial rebuild), the list capacity has been
// checked for these positions, and no phase events are being recorded.
bool World::graph_capturable() const {
    return grid_current_ && rho_current_ && lists_checked_ && lists_sized_ && !profiling_ && n_ > 0;
}

void World::release_graph() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
}

// Captures kGraphSteps steps into one graph. Capturing records the launches
// without running them, so every host-side effect of the captured steps
// (buffer rotations, time, launch count) is undone afterwards and replayed
// per graph launch; the rotations return to their start after kGraphSteps
// steps, which is checked here.
bool World::same_rotation(const Rotation& a, const Rotation& b) {
    return std::memcmp(&a.cur, &b.cur, sizeof(a.cur)) == 0 && std::memcmp(&a.alt, &b.alt, sizeof(a.alt)) == 0 &&
           a.vel_nx == b.vel_nx && std::memcmp(&a.fb, &b.fb, sizeof(a.fb)) == 0 && a.velf_alt == b.velf_alt;
}

bool World::capture_graph(double dt) {
    release_graph();
    graph_rot_ = rotation();
    const StateBufs cur0 = cur_, alt0 = alt_;
    double4* const vel_nx0 = vel_nx_;
    const F32Bufs fb0 = fb_;
    float4* const velf_alt0 = velf_alt_;
    const double t0 = t_;
    const uint32_t l0 = launches_;
    cudaGraph_t graph = nullptr;
    bool ok = cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        try {
            for (uint32_t k = 0; k < kGraphSteps; ++k) step(dt);
        } catch (const std::exception&) {
            ok = false;
        }
        ok = cudaStreamEndCapture(st_, &graph) == cudaSuccess && ok;
    }
    const bool same = std::memcmp(&cur_, &cur0, sizeof(cur0)) == 0 &&
                      std::memcmp(&alt_, &alt0, sizeof(alt0)) == 0 && vel_nx_ == vel_nx0 &&
                      std::memcmp(&fb_, &fb0, sizeof(fb0)) == 0 && velf_alt_ == velf_alt0;
    graph_launches_ = launches_ - l0;
    cur_ = cur0;
    alt_ = alt0;
    vel_nx_ = vel_nx0;
    fb_ = fb0;
    velf_alt_ = velf_alt0;
    t_ = t0;
    launches_ = l0;
    cudaGetLastError();  // clear the (non-sticky) error a failed capture leaves
    if (ok && same && graph) {
        if (cudaGraphInstantiate(&graph_exec_, graph, 0) != cudaSuccess) {
            graph_exec_ = nullptr;
            cudaGetLastError();
        }
    }
    if (graph) cudaGraphDestroy(graph);
    graph_dt_ = dt;
    graph_epoch_ = epoch_;
    return graph_exec_ != nullptr;
}

void World::configure_lists() {
    uint32_t per_sm = nlist_prepare(dim_, ucap_, list_chunk_);
    check(cudaGetLastError(), "nlist prepare");
    forces_prepare();
    check(cudaGetLastError(), "force pass prepare");
    const uint32_t mult = list_ctas_per_sm_ ? list_ctas_per_sm_ : std::max<uint32_t>(per_sm, 1u) * 4u;
    nl_blocks_ = sms_ * mult;
    invalidate_graph();
}

World::Shapes World::shapes() const {
    Shapes r;
    r.density = shape_.density;
    r.forces = shape_.forces;
    r.xsph = shape_.xsph;
    r.list_ctas_per_sm = nl_blocks_ / std::max<uint32_t>(sms_, 1u);
    r.list_chunk = list_chunk_;
    return r;
}

// Times each candidate launch shape on the current state with CUDA events and
// keeps the fastest. Every timed pass is idempotent here: the list build and
// the density pass recompute the same values, the force pass writes only the
// next-state scratch buffers, and XSPH (f64) writes the scratch velocity
// buffer without the swap that would commit it. Results do not depend on the
// shapes (each particle's sums run in the same order in every shape).
World::Shapes World::autotune() {
    if (!n_) return shapes();
    if (!grid_current_) {
        build_grid(nullptr, nullptr);
        refresh_f32();
        grid_current_ = true;
        rho_current_ = false;
    }
    ensure_lists();
    const bool prof = profiling_;
    profiling_ = false;
    cudaEvent_t a = take_event(), b = take_event();
    auto time_it = [&](auto&& launch) {
        launch();  // warm
        check(cudaEventRecord(a, st_), "autotune");
        for (int r = 0; r < 3; ++r) launch();
        check(cudaEventRecord(b, st_), "autotune");
        check(cudaEventSynchronize(b), "autotune");
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, a, b), "autotune");
        return ms;
    };
    const uint32_t cand[3] = {64, 128, 256};
    const uint32_t n = (uint32_t)n_;
    auto pick = [&](uint32_t& field, auto&& launch) {
        float best = 0.f;
        uint32_t best_t = 0;
        for (uint32_t t : cand) {
            field = t;
            const float ms = time_it(launch);
            if (best_t == 0 || ms < best) {
                best = ms;
                best_t = t;
            }
        }
        field = best_t;
    };
    if (pair_weights()) check(cudaMemsetAsync(&sc_->w_short, 0, sizeof(uint32_t), st_), "memset");
    pick(shape_.density, [&] {
        if (f32_) launch_density_f32(n, shape_.density, kf_, cur_, fb_, lists_, st_);
        else launch_density(n, shape_.density, kc_, cur_, lists_, st_);
    });
    w_valid_ = pair_weights();  // the density launches wrote W for these lists
    pick(shape_.forces, [&] {
        if (f32_) launch_forces_f32(n, shape_.forces, kf_, tanks_, cur_, fb_, lists_, 0.f, pos_nx_, vel_nx_, nullptr, st_);
        else launch_forces(n, shape_.forces, kc_, tanks_, cur_, lists_, true, 0.0, pos_nx_, vel_nx_,
                           prm_.surface_tension_sigma != 0.0 ? st_a_ : nullptr, st_);
    });
    if (!f32_ && prm_.xsph_epsilon != 0.0)
        pick(shape_.xsph, [&] { launch_xsph(n, shape_.xsph, kc_, cur_, lists_, vel_nx_, st_, w_valid_); });
    // list build: tile (centre particles per chunk) x CTAs per SM (multiples
    // of the resident count). The lists' entries and order do not depend on
    // either; a smaller chunk never asks for more of the pool (each chunk
    // reserves its longest list's rows), so the pool sized at creation fits.
    {
        float best = 0.f;
        uint32_t best_m = 0, best_c = list_chunk_;
        for (uint32_t chunk : {64u, 32u}) {
            const uint32_t per_sm = std::max<uint32_t>(nlist_prepare(dim_, ucap_, chunk), 1u);
            for (uint32_t m : {1u, 2u, 4u, 8u}) {
                nl_blocks_ = sms_ * per_sm * m;
                const float ms = time_it([&] {
                    check(cudaMemsetAsync(&sc_->list_used, 0, sizeof(unsigned long long), st_), "memset");
                    launch_nlist(g_, tanks_, kc_, ucap_, nl_blocks_, occ_, cell_start_, cur_, lists_, sc_, st_,
                                 !lists_full_, chunk);
                });
                if (best_m == 0 || ms < best) {
                    best = ms;
                    best_m = per_sm * m;
                    best_c = chunk;
                }
            }
        }
        list_chunk_ = best_c;
        list_ctas_per_sm_ = best_m;
        nlist_prepare(dim_, ucap_, list_chunk_);
        nl_blocks_ = sms_ * best_m;
        // the lists in the pool now come from the last timed build; rebuild
        // them with the chosen shape so their layout is the one used from now
        check(cudaMemsetAsync(&sc_->list_used, 0, sizeof(unsigned long long), st_), "memset");
        launch_nlist(g_, tanks_, kc_, ucap_, nl_blocks_, occ_, cell_start_, cur_, lists_, sc_, st_, !lists_full_,
                     list_chunk_);
        w_valid_ = false;  // the pair weights follow the old layout
    }
    check(cudaGetLastError(), "autotune");
    event_pool_.push_back(a);
    event_pool_.push_back(b);
    profiling_ = prof;
    invalidate_graph();
    return shapes();
}

uint32_t World::status() {
    DeviceScalars hs{};
    check(cudaMemcpyAsync(&hs, sc_, sizeof(hs), cudaMemcpyDeviceToHost, st_), "status");
    check(cudaStreamSynchronize(st_), "status");
    // Grow the list storage ahead of need: the next list build uses the larger
    // capacity (the current lists are complete as long as no overflow bit is set).
    if (hs.list_used * 4 > lists_.pool_groups * 3 && lists_.pool_groups < kMaxListGroups) {
        alloc_lists(2 * hs.list_used);
        lists_checked_ = false;
    }
    // Pair weights that a density pass found too short cover the whole pool
    // from now on (XSPH recomputed W meanwhile).
    if (hs.w_short && pair_w_on_ && lists_.w_cap < lists_.pool_groups * 4ull) {
        free_pair_weights();
        alloc_pair_weights(lists_.pool_groups);
        invalidate_graph();
    }
    // Grow the shared-memory stage of the list build when the fluid has
    // packed more particles into a neighbourhood than it holds.
    if (hs.max_union > ucap_) {
        uint32_t want = nlist_union_capacity(hs.max_union);
        if (want > ucap_) {
            ucap_ = want;
            configure_lists();
        }
    }
    return hs.status;
}

void World::capacity_info(uint64_t* out) {
    DeviceScalars hs{};
    check(cudaMemcpyAsync(&hs, sc_, sizeof(hs), cudaMemcpyDeviceToHost, st_), "info");
    check(cudaStreamSynchronize(st_), "info");
    out[0] = hs.status;
    out[1] = hs.max_union;
    out[2] = hs.list_used;
    out[3] = ucap_;
    out[4] = lists_.pool_groups;
    out[5] = hs.nocc;
    out[6] = g_.ncell;
    out[7] = nl_blocks_;
}

void World::clear_status() {
    check(cudaMemsetAsync(&sc_->status, 0, sizeof(uint32_t), st_), "status");
    check(cudaStreamSynchronize(st_), "status");
}

void World::gather_orig_vec(const double4* src, double* out) {
    uint32_t n = (uint32_t)n_;
    if (!n) return;
    k_export_vec<<<blocks_for(n, 256), 256, 0, st_>>>(n, slot_of_orig_, src, xfer_);
    check(cudaMemcpyAsync(out, xfer_, sizeof(double) * 3 * n_, cudaMemcpyDeviceToHost, st_), "export");
    check(cudaStreamSynchronize(st_), "export");
}

void World::get_vec(int which, double* out) {
    const double4* src = which == 0 ? cur_.pos : which == 1 ? cur_.vel : which == 2 ? cur_.acc : cur_.bf;
    gather_orig_vec(src, out);
}

bool World::set_vec(int which, const double* in) {
    uint32_t n = (uint32_t)n_;
    if (!n) return true;
    check(cudaMemcpyAsync(xfer_, in, sizeof(double) * 3 * n_, cudaMemcpyHostToDevice, st_), "import");
    // The input is checked for non-finite values on the device (a host scan of
    // the caller's buffer costs more than the copy); a rejected input leaves
    // the state untouched.
    check(cudaMemsetAsync(&sc_->import_bad, 0, sizeof(uint32_t), st_), "import");
    k_check_finite<<<sms_ * 4, 256, 0, st_>>>(3 * n_, xfer_, &sc_->import_bad);
    // Positions that come back bit for bit as they were (a caller that reads
    // the state out and writes it back) leave the grid, lists and densities
    // valid: rebuilding them would reproduce the same bits.
    uint32_t* changed = which == 0 ? &sc_->pad_ : nullptr;
    if (changed) check(cudaMemsetAsync(changed, 0, sizeof(uint32_t), st_), "import");
    // Velocities of boundary samples are part of the state too (the reference
    // stores them; they never move), so both kinds are written.
    k_import_vec<<<blocks_for(n, 256), 256, 0, st_>>>(n, slot_of_orig_, xfer_,
                                                      which == 0 ? cur_.pos : cur_.vel, cur_.flags, 0, changed,
                                                      &sc_->import_bad);
    uint32_t flags_h[2] = {0u, 1u};  // bad, moved
    check(cudaMemcpyAsync(&flags_h[0], &sc_->import_bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, st_), "import");
    if (changed) check(cudaMemcpyAsync(&flags_h[1], changed, sizeof(uint32_t), cudaMemcpyDeviceToHost, st_), "import");
    check(cudaStreamSynchronize(st_), "import");
    if (flags_h[0]) return false;
    refresh_f32();
    if (which == 0 && flags_h[1]) {
        grid_current_ = false;
        rho_current_ = false;
        lists_valid_ = false;
        lists_checked_ = false;
    }
    return true;
}

void World::get_scalar(int which, double* out) {
    uint32_t n = (uint32_t)n_;
    if (!n) return;
    k_export_w<<<blocks_for(n, 256), 256, 0, st_>>>(n, slot_of_orig_, which == 0 ? cur_.vel : nullptr,
                                                    cur_.p, xfer_);
    check(cudaMemcpyAsync(out, xfer_, sizeof(double) * n_, cudaMemcpyDeviceToHost, st_), "export");
    check(cudaStreamSynchronize(st_), "export");
}

void World::set_scalar(int which, const double* in) {
    uint32_t n = (uint32_t)n_;
    if (!n) return;
    check(cudaMemcpyAsync(xfer_, in, sizeof(double) * n_, cudaMemcpyHostToDevice, st_), "import");
    k_import_w<<<blocks_for(n, 256), 256, 0, st_>>>(n, slot_of_orig_, xfer_,
                                                    which == 0 ? cur_.vel : nullptr, cur_.p);
    k_refresh_pr2<<<blocks_for(n, 256), 256, 0, st_>>>(n, cur_.flags, cur_.p, cur_.pos, cur_.vel);
    refresh_f32();
    check(cudaStreamSynchronize(st_), "import");
    if (which == 0) rho_current_ = false;
}

void World::get_kind(uint8_t* out) {
    uint32_t n = (uint32_t)n_;
    if (!n) return;
    uint8_t* d = reinterpret_cast<uint8_t*>(xfer_);
    k_export_kind<<<blocks_for(n, 256), 256, 0, st_>>>(n, slot_of_orig_, cur_.flags, d);
    check(cudaMemcpyAsync(out, d, n_, cudaMemcpyDeviceToHost, st_), "export");
    check(cudaStreamSynchronize(st_), "export");
}

void World::get_grid(int32_t* keys, uint64_t* order, int32_t* occupied, uint64_t* ranges,
                     uint64_t occ_cap, uint64_t* n_occupied) {
    uint32_t n = (uint32_t)n_;
    if (!grid_built_) {
        if (n_occupied) *n_occupied = 0;
        return;
    }
    DeviceScalars hs{};
    check(cudaMemcpyAsync(&hs, sc_, sizeof(hs), cudaMemcpyDeviceToHost, st_), "grid");
    check(cudaStreamSynchronize(st_), "grid");
    if (n_occupied) *n_occupied = hs.nocc;
    if (keys && n) {
        int32_t* d = reinterpret_cast<int32_t*>(xfer_);
        k_export_keys<<<blocks_for(n, 256), 256, 0, st_>>>(n, slot_of_orig_, cur_.key, d);
        check(cudaMemcpyAsync(keys, d, sizeof(int32_t) * 3 * n_, cudaMemcpyDeviceToHost, st_), "grid");
        check(cudaStreamSynchronize(st_), "grid");
    }
    if (order && n) {
        std::vector<uint32_t> o(n);
        check(cudaMemcpyAsync(o.data(), cur_.orig, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st_), "grid");
        check(cudaStreamSynchronize(st_), "grid");
        for (uint32_t s = 0; s < n; ++s) order[s] = o[s];
    }
    if ((occupied || ranges) && hs.nocc && occ_cap >= hs.nocc) {
        int32_t* dk = reinterpret_cast<int32_t*>(xfer_);
        uint64_t* dr = reinterpret_cast<uint64_t*>(pos_nx_);
        launch_occupied_export(g_, occ_, sc_, cell_start_, cur_.key, dk, dr, st_);
        if (occupied)
            check(cudaMemcpyAsync(occupied, dk, sizeof(int32_t) * 3 * hs.nocc, cudaMemcpyDeviceToHost, st_), "grid");
        if (ranges)
            check(cudaMemcpyAsync(ranges, dr, sizeof(uint64_t) * 2 * hs.nocc, cudaMemcpyDeviceToHost, st_), "grid");
        check(cudaStreamSynchronize(st_), "grid");
    }
}

void World::get_neighbour_counts(uint32_t* candidates, uint32_t* in_support) {
    uint32_t n = (uint32_t)n_;
    if (!n) return;
    ensure_lists();
    uint32_t* d = reinterpret_cast<uint32_t*>(xfer_);
    if (candidates) {
        k_export_u32<<<blocks_for(n, 256), 256, 0, st_>>>(n, slot_of_orig_, lists_.ncand, d);
        check(cudaMemcpyAsync(candidates, d, sizeof(uint32_t) * n_, cudaMemcpyDeviceToHost, st_), "counts");
        check(cudaStreamSynchronize(st_), "counts");
    }
    if (in_support) {
        launch_in_support_counts(n, kc_, cur_, lists_, insup_, st_);
        k_export_u32<<<blocks_for(n, 256), 256, 0, st_>>>(n, slot_of_orig_, insup_, d);
        check(cudaMemcpyAsync(in_support, d, sizeof(uint32_t) * n_, cudaMemcpyDeviceToHost, st_), "counts");
        check(cudaStreamSynchronize(st_), "counts");
    }
}

}  // namespace pe
