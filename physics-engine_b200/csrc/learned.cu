// The learned surrogate coupled to a world: message graph and features from a
// world's state, training targets from the plain step, the learned step, and
// the judge / fallback runner (see surrogate.cuh and world.cuh).
#include <algorithm>
#include <cmath>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "pe_math.cuh"
#include "surrogate.cuh"
#include "world.cuh"

namespace pe {

namespace {

inline unsigned blocks(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

void cu(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string("learned ") + what + ": " + cudaGetErrorString(e));
}

// Feature scaling: positions in units of h, velocities in units of c0 / 10,
// densities as 50 (rho / rho0 - 1), pressures as 5 p / B with B = rho0 c0^2 / gamma.
struct FeatScale {
    double inv_h, sv, srho, inv_rho0, sp, r2;
};

__device__ __forceinline__ bool keep_edge(const StateBufs& s, uint32_t s0, uint32_t n, uint32_t j,
                                          const double4& xi, double r2) {
    if (j < s0 || j >= s0 + n) return false;
    const double4 xj = s.pos[j];
    const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    return dx * dx + dy * dy + dz * dz <= r2;
}

__global__ void k_msg_count(uint32_t s0, uint32_t n, StateBufs s, ListBufs l, FeatScale fs, int* cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) {
        cnt[n] = 0;
        return;
    }
    const uint32_t slot = s0 + i;
    if (s.flags[slot] & kFlagBoundary) {
        cnt[i] = 0;
        return;
    }
    const double4 xi = s.pos[slot];
    const ListRef r = list_ref(l, slot, kListVisit);
    int c = 0;
    for (uint32_t t = 0; t < r.n; ++t) {
        const uint32_t j = __ldg(r.p + (size_t)(t >> 2) * r.step + (t & 3u)) & kEntrySlotMask;
        c += keep_edge(s, s0, n, j, xi, fs.r2) ? 1 : 0;
    }
    cnt[i] = c;
}

__device__ __forceinline__ float rho_feat(double rho, const FeatScale& fs) {
    return (float)((rho * fs.inv_rho0 - 1.0) * fs.srho);
}

__global__ void k_msg_fill(uint32_t s0, uint32_t n, StateBufs s, ListBufs l, FeatScale fs,
                           const int* __restrict__ row, int* __restrict__ src, int* __restrict__ dst,
                           __nv_bfloat16* __restrict__ xe) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t slot = s0 + i;
    if (s.flags[slot] & kFlagBoundary) return;
    const double4 xi = s.pos[slot], vi = s.vel[slot];
    const float rfi = rho_feat(vi.w, fs), pfi = (float)(s.p[slot] * fs.sp);
    const ListRef r = list_ref(l, slot, kListVisit);
    int k = row[i];
    for (uint32_t t = 0; t < r.n; ++t) {
        const uint32_t j = __ldg(r.p + (size_t)(t >> 2) * r.step + (t & 3u)) & kEntrySlotMask;
        if (!keep_edge(s, s0, n, j, xi, fs.r2)) continue;
        const double4 xj = s.pos[j], vj = s.vel[j];
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        float f[kEdgeFeat];
        f[0] = (float)(dx * fs.inv_h);
        f[1] = (float)(dy * fs.inv_h);
        f[2] = (float)(dz * fs.inv_h);
        f[3] = (float)(sqrt(dx * dx + dy * dy + dz * dz) * fs.inv_h);
        f[4] = (float)((vj.x - vi.x) * fs.sv);
        f[5] = (float)((vj.y - vi.y) * fs.sv);
        f[6] = (float)((vj.z - vi.z) * fs.sv);
        f[7] = rfi;
        f[8] = rho_feat(vj.w, fs);
        f[9] = pfi;
        f[10] = (float)(s.p[j] * fs.sp);
        f[11] = (s.flags[j] & kFlagBoundary) ? 1.f : 0.f;
#pragma unroll
        for (int q = 12; q < kEdgeFeat; ++q) f[q] = 0.f;
        src[k] = (int)(j - s0);
        dst[k] = (int)i;
#pragma unroll
        for (int q = 0; q < kEdgeFeat; ++q) xe[(size_t)k * kEdgeFeat + q] = __float2bfloat16_rn(f[q]);
        ++k;
    }
}

__global__ void k_node_feat(uint32_t s0, uint32_t n, StateBufs s, FeatScale fs, __nv_bfloat16* __restrict__ f,
                            uint8_t* __restrict__ fluid, uint32_t* __restrict__ orig, double* __restrict__ vrho) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t slot = s0 + i;
    const bool bnd = s.flags[slot] & kFlagBoundary;
    const double4 v = s.vel[slot];
    float q[kNodeFeat] = {(float)(v.x * fs.sv), (float)(v.y * fs.sv), (float)(v.z * fs.sv), rho_feat(v.w, fs),
                          (float)(s.p[slot] * fs.sp), bnd ? 1.f : 0.f, 0.f, 0.f};
#pragma unroll
    for (int c = 0; c < kNodeFeat; ++c) f[(size_t)i * kNodeFeat + c] = __float2bfloat16_rn(q[c]);
    fluid[i] = bnd ? 0 : 1;
    orig[i] = s.orig[slot];
    vrho[4 * (size_t)i] = v.x;
    vrho[4 * (size_t)i + 1] = v.y;
    vrho[4 * (size_t)i + 2] = v.z;
    vrho[4 * (size_t)i + 3] = v.w;
}

// raw targets: (v' - v) / dt and (rho' - rho) / dt of the fluid nodes
__global__ void k_targets(uint32_t n, const uint8_t* __restrict__ fluid, const uint32_t* __restrict__ orig,
                          const double* __restrict__ vrho, const uint32_t* __restrict__ slot_of_orig,
                          StateBufs s, double inv_dt, float* __restrict__ raw) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!fluid[i]) {
        for (int c = 0; c < kOut; ++c) raw[(size_t)i * kOut + c] = 0.f;
        return;
    }
    const double4 v = s.vel[slot_of_orig[orig[i]]];
    raw[(size_t)i * kOut + 0] = (float)((v.x - vrho[4 * (size_t)i]) * inv_dt);
    raw[(size_t)i * kOut + 1] = (float)((v.y - vrho[4 * (size_t)i + 1]) * inv_dt);
    raw[(size_t)i * kOut + 2] = (float)((v.z - vrho[4 * (size_t)i + 2]) * inv_dt);
    raw[(size_t)i * kOut + 3] = (float)((v.w - vrho[4 * (size_t)i + 3]) * inv_dt);
}

// predictions in physical units per slot: acc = (a, drho/dt), zero for boundary
__global__ void k_denorm(uint32_t s0, uint32_t n, const float* __restrict__ Y, const uint8_t* __restrict__ fluid,
                         SurrogateStats st, double4* __restrict__ acc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double r[kOut];
#pragma unroll
    for (int c = 0; c < kOut; ++c)
        r[c] = fluid[i] ? (double)Y[(size_t)i * kOutPad + c] * st.std[c] + st.mean[c] : 0.0;
    acc[s0 + i] = make_double4(r[0], r[1], r[2], r[3]);
}

__global__ void k_learned_integrate(uint32_t n, int dim, StateBufs s, double dt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (s.flags[i] & kFlagBoundary)) return;
    const double4 a = s.acc[i];
    double4 v = s.vel[i], x = s.pos[i];
    v.x += dt * a.x;
    v.y += dt * a.y;
    v.z = dim == 2 ? 0.0 : v.z + dt * a.z;
    x.x += dt * v.x;
    x.y += dt * v.y;
    x.z = dim == 2 ? 0.0 : x.z + dt * v.z;
    v.w = fmax(v.w + dt * a.w, 1e-12);
    s.vel[i] = v;
    s.pos[i] = x;
}

__global__ void k_checkpoint(uint32_t n, StateBufs s, double4* __restrict__ cp, double4* __restrict__ cv,
                             double* __restrict__ cpr, int restore) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t o = s.orig[i];
    if (restore) {
        s.pos[i] = cp[o];
        s.vel[i] = cv[o];
        s.p[i] = cpr[o];
    } else {
        cp[o] = s.pos[i];
        cv[o] = s.vel[i];
        cpr[o] = s.p[i];
    }
}

__global__ void k_rho_by_orig(uint32_t n, StateBufs s, double* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[s.orig[i]] = s.vel[i].w;
}

// max over fluid of |rho_carried - rho| / rho (non-negative floats order like their bits)
__global__ void k_judge(uint32_t n, StateBufs s, const double* __restrict__ carried, unsigned* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float e = 0.f;
    if (i < n && !(s.flags[i] & kFlagBoundary)) {
        const double rho = s.vel[i].w;
        const double d = fabs(carried[s.orig[i]] - rho) / rho;
        e = isfinite(d) ? (float)d : 3.0e38f;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
    if ((threadIdx.x & 31) == 0 && e > 0.f) atomicMax(err, __float_as_uint(e));
}

FeatScale scales_of(const World& w, double r_over_h) {
    const WorldParams& p = w.params();
    FeatScale fs;
    const double h = w.smoothing_length();
    fs.inv_h = 1.0 / h;
    fs.sv = 10.0 / p.eos_sound_speed;
    fs.srho = 50.0;
    fs.inv_rho0 = 1.0 / p.eos_rest_density;
    const double B = p.eos_rest_density * p.eos_sound_speed * p.eos_sound_speed / p.eos_gamma;
    fs.sp = 5.0 / B;
    fs.r2 = (r_over_h * h) * (r_over_h * h);
    return fs;
}

}  // namespace

// ------------------------------------------------------------ surrogate side

void Surrogate::graph_from_world(World& w, uint32_t s0, uint32_t s1) {
    if (s1 <= s0 || s1 > w.n_) throw std::invalid_argument("graph range");
    if (!(w.grid_current_ && w.rho_current_)) {  // as the step starts (wcsph.rs:327-328)
        w.build_grid(nullptr, nullptr);
        w.refresh_f32();
        w.grid_current_ = true;
        w.run_density();
        w.rho_current_ = true;
    }
    w.ensure_lists(true);
    cu(cudaStreamSynchronize(w.st_), "world");
    const uint32_t n = s1 - s0;
    const FeatScale fs = scales_of(w, r_msg_over_h_);
    int E = 0;
    for (int pass = 0; pass < 2; ++pass) {
        ensure_graph((int)n, std::max(g_.cap_e, E));
        k_msg_count<<<blocks(n + 1, 256), 256, 0, st_>>>(s0, n, w.cur_, w.lists_, fs, cnt_);
        size_t need = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, need, cnt_, g_.row, (int)n + 1, st_);
        if (need > scan_bytes_) {
            cu(cudaStreamSynchronize(st_), "scan");
            if (scan_tmp_) cudaFree(scan_tmp_);
            cu(cudaMalloc(&scan_tmp_, need), "cudaMalloc scan");
            scan_bytes_ = need;
        }
        cu(cub::DeviceScan::ExclusiveSum(scan_tmp_, scan_bytes_, cnt_, g_.row, (int)n + 1, st_), "scan");
        cu(cudaMemcpyAsync(&E, g_.row + n, sizeof(int), cudaMemcpyDeviceToHost, st_), "edges");
        cu(cudaStreamSynchronize(st_), "edges");
        if (E <= g_.cap_e) break;  // else grow (which drops the offsets) and count again
    }
    ensure_graph((int)n, E);
    k_msg_fill<<<blocks(n, 256), 256, 0, st_>>>(s0, n, w.cur_, w.lists_, fs, g_.row, g_.src, g_.dst, g_.xe);
    k_node_feat<<<blocks(n, 256), 256, 0, st_>>>(s0, n, w.cur_, fs, g_.f, g_.fluid, node_orig_, node_v_);
    cu(cudaGetLastError(), "graph");
    cu(cudaStreamSynchronize(st_), "graph");
}

void Surrogate::targets_from_world(World& w, double dt, bool update_stats) {
    cu(cudaStreamSynchronize(w.st_), "world");
    const int n = g_.n;
    k_targets<<<blocks(n, 256), 256, 0, st_>>>((uint32_t)n, g_.fluid, node_orig_, node_v_, w.slot_of_orig_,
                                                w.cur_, 1.0 / dt, raw_t_);
    std::vector<float> raw((size_t)n * kOut);
    std::vector<uint8_t> fl(n);
    cu(cudaMemcpyAsync(raw.data(), raw_t_, raw.size() * 4, cudaMemcpyDeviceToHost, st_), "targets");
    cu(cudaMemcpyAsync(fl.data(), g_.fluid, (size_t)n, cudaMemcpyDeviceToHost, st_), "targets");
    cu(cudaStreamSynchronize(st_), "targets");
    if (update_stats) {
        for (int i = 0; i < n; ++i)
            if (fl[i]) {
                for (int c = 0; c < kOut; ++c) {
                    const double v = raw[(size_t)i * kOut + c];
                    st_sum_[c] += v;
                    st_sq_[c] += v * v;
                }
                st_count_ += 1.0;
            }
        if (st_count_ > 0.0)
            for (int c = 0; c < kOut; ++c) {
                const double mean = st_sum_[c] / st_count_;
                const double var = std::max(st_sq_[c] / st_count_ - mean * mean, 0.0);
                stats_.mean[c] = (float)mean;
                stats_.std[c] = (float)std::max(std::sqrt(var), 1e-6);
            }
    }
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < kOut; ++c) {
            float& v = raw[(size_t)i * kOut + c];
            v = fl[i] ? (v - stats_.mean[c]) / stats_.std[c] : 0.f;
        }
    set_targets(raw.data());
}

void Surrogate::predict_world(World& w, double4* acc_out) {
    graph_from_world(w, 0, (uint32_t)w.n_);
    forward(false);
    k_denorm<<<blocks(g_.n, 256), 256, 0, st_>>>(0u, (uint32_t)g_.n, Y_, g_.fluid, stats_, acc_out);
    cu(cudaGetLastError(), "predict");
    cu(cudaStreamSynchronize(st_), "predict");
}

// ------------------------------------------------------------ world side

void World::step_learned(Surrogate& s, double dt) {
    if (!grid_current_) {
        build_grid(nullptr, nullptr);
        refresh_f32();
        grid_current_ = true;
    }
    ensure_lists(true);
    run_pressure();  // network inputs: p of the carried densities (per-tank c)
    s.predict_world(*this, cur_.acc);
    k_learned_integrate<<<blocks(n_, 256), 256, 0, st_>>>((uint32_t)n_, dim_, cur_, dt);
    launches_ += 1;
    check(cudaGetLastError(), "learned step");
    refresh_f32();
    t_ += dt;
    grid_current_ = false;
    rho_current_ = false;
    lists_valid_ = false;
}

double World::judge_density() {
    if (!n_) return 0.0;
    if (!judge_err_) {
        void* p = nullptr;
        check(cudaMalloc(&p, 256), "cudaMalloc");
        judge_err_ = static_cast<float*>(p);
    }
    k_rho_by_orig<<<blocks(n_, 256), 256, 0, st_>>>((uint32_t)n_, cur_, xfer_);
    build_grid(nullptr, nullptr);
    refresh_f32();
    grid_current_ = true;
    run_density(true);  // the density pass reads the visit list only
    rho_current_ = true;
    check(cudaMemsetAsync(judge_err_, 0, 4, st_), "memset");
    k_judge<<<blocks(n_, 256), 256, 0, st_>>>((uint32_t)n_, cur_, xfer_, reinterpret_cast<unsigned*>(judge_err_));
    float e = 0.f;
    check(cudaMemcpyAsync(&e, judge_err_, 4, cudaMemcpyDeviceToHost, st_), "judge");
    check(cudaStreamSynchronize(st_), "judge");
    return e;
}

void World::save_checkpoint() {
    if (!ck_pos_) {
        void* p = nullptr;
        check(cudaMalloc(&p, sizeof(double4) * std::max<uint64_t>(n_, 1)), "cudaMalloc");
        ck_pos_ = static_cast<double4*>(p);
        check(cudaMalloc(&p, sizeof(double4) * std::max<uint64_t>(n_, 1)), "cudaMalloc");
        ck_vel_ = static_cast<double4*>(p);
        check(cudaMalloc(&p, sizeof(double) * std::max<uint64_t>(n_, 1)), "cudaMalloc");
        ck_p_ = static_cast<double*>(p);
    }
    k_checkpoint<<<blocks(n_, 256), 256, 0, st_>>>((uint32_t)n_, cur_, ck_pos_, ck_vel_, ck_p_, 0);
    check(cudaGetLastError(), "checkpoint");
    ck_t_ = t_;
}

void World::restore_checkpoint() {
    k_checkpoint<<<blocks(n_, 256), 256, 0, st_>>>((uint32_t)n_, cur_, ck_pos_, ck_vel_, ck_p_, 1);
    check(cudaGetLastError(), "checkpoint");
    refresh_f32();
    t_ = ck_t_;
    grid_current_ = false;
    rho_current_ = false;
    lists_valid_ = false;
}

void World::run_learned(Surrogate& s, double dt, uint64_t steps, uint32_t judge_every, double bound,
                        LearnedStats* st) {
    LearnedStats r{};
    if (judge_every == 0) judge_every = 1;
    if (!(grid_current_ && rho_current_)) {  // wcsph.rs:327-328: the step starts from SPH densities
        build_grid(nullptr, nullptr);
        refresh_f32();
        grid_current_ = true;
        run_density();
        rho_current_ = true;
    }
    // the per-tank sound speeds of the checkpoint
    std::vector<double> c_ck(n_tanks_);
    uint64_t done = 0;
    while (done < steps) {
        const uint64_t k = std::min<uint64_t>(judge_every, steps - done);
        save_checkpoint();
        get_sound_speeds(c_ck.data());
        for (uint64_t i = 0; i < k; ++i) step_learned(s, dt);
        const double err = judge_density();
        r.last_error = err;
        r.max_error = std::max(r.max_error, err);
        ++r.windows;
        if (!(err <= bound)) {
            restore_checkpoint();
            check(cudaMemcpyAsync(tanks_.c, c_ck.data(), sizeof(double) * n_tanks_, cudaMemcpyHostToDevice, st_),
                  "c");
            run(dt, k);
            ++r.fallbacks;
            r.plain_steps += k;
        } else {
            r.learned_steps += k;
        }
        done += k;
    }
    check(cudaStreamSynchronize(st_), "learned run");
    if (st) *st = r;
}

}  // namespace pe
