// Fluid side of the WCSPH-rigid coupling (crates/pe-fluid/src/coupling.rs):
// FluidRigidCoupler::sync_from_rigid (coupling.rs:289-306) writes the rigid
// samples' boundary particles from per-body state, and
// FluidRigidCoupler::reduce_with_state (coupling.rs:308-330) sums, per body,
// its samples' boundary reactions and their torques about the body's centre of
// mass. The rigid bodies themselves (pe-rigid) stay with the caller. All
// arithmetic keeps the reference's operand order without contraction, and the
// per-body sums run in sample order, so both match the reference bit for bit.
#include <algorithm>
#include <vector>

#include "coupling.cuh"

namespace pe {

namespace {

struct DV3 {
    double x, y, z;
};

// quat.rs:119-137 to_matrix, quat.rs:102-109 rotate; q = (w, x, y, z)
__device__ __forceinline__ DV3 quat_rotate(const double* q, DV3 v) {
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    const double r00 = 1.0 - 2.0 * (y * y + z * z), r01 = 2.0 * (x * y - w * z), r02 = 2.0 * (x * z + w * y);
    const double r10 = 2.0 * (x * y + w * z), r11 = 1.0 - 2.0 * (x * x + z * z), r12 = 2.0 * (y * z - w * x);
    const double r20 = 2.0 * (x * z - w * y), r21 = 2.0 * (y * z + w * x), r22 = 1.0 - 2.0 * (x * x + y * y);
    return DV3{r00 * v.x + r01 * v.y + r02 * v.z, r10 * v.x + r11 * v.y + r12 * v.z,
               r20 * v.x + r21 * v.y + r22 * v.z};
}

// vec3.rs:87-93
__device__ __forceinline__ DV3 cross3(DV3 a, DV3 b) {
    return DV3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// bodies: X[3 b], Q[4 b], V[3 b], Om[3 b] packed as 13 doubles per body
__global__ void k_coupler_sync(uint64_t ns, int dim, const int64_t* __restrict__ body,
                               const double* __restrict__ local, const double* __restrict__ local_n,
                               const int64_t* __restrict__ particle, const double* __restrict__ bodies,
                               const uint32_t* __restrict__ slot_of_orig, StateBufs s) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ns) return;
    const double* B = bodies + 13 * body[k];
    const uint32_t slot = slot_of_orig[particle[k]];
    const DV3 r = quat_rotate(B + 3, DV3{local[3 * k], local[3 * k + 1], local[3 * k + 2]});
    const DV3 w = cross3(DV3{B[10], B[11], B[12]}, r);
    const DV3 n = quat_rotate(B + 3, DV3{local_n[3 * k], local_n[3 * k + 1], local_n[3 * k + 2]});
    double4 p = s.pos[slot], v = s.vel[slot];
    p.x = B[0] + r.x;
    p.y = B[1] + r.y;
    p.z = dim == 2 ? 0.0 : B[2] + r.z;
    v.x = B[7] + w.x;
    v.y = B[8] + w.y;
    v.z = dim == 2 ? 0.0 : B[9] + w.z;
    s.pos[slot] = p;
    s.vel[slot] = v;
    s.nout[slot] = make_double4(n.x, n.y, dim == 2 ? 0.0 : n.z, 0.0);
}

// one thread per body, its samples in order (body_start: CSR over samples grouped by body)
__global__ void k_coupler_reduce(uint32_t nb, const uint64_t* __restrict__ body_start,
                                 const int64_t* __restrict__ sample_particle, const double* __restrict__ X,
                                 const uint32_t* __restrict__ slot_of_orig, StateBufs s, double* __restrict__ out) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    DV3 f{0.0, 0.0, 0.0}, t{0.0, 0.0, 0.0};
    const DV3 xb{X[3 * b], X[3 * b + 1], X[3 * b + 2]};
    for (uint64_t k = body_start[b]; k < body_start[b + 1]; ++k) {
        const uint32_t slot = slot_of_orig[sample_particle[k]];
        const double4 fb4 = s.bf[slot], x4 = s.pos[slot];
        const DV3 fb{fb4.x, fb4.y, fb4.z};
        f = DV3{f.x + fb.x, f.y + fb.y, f.z + fb.z};
        const DV3 r{x4.x - xb.x, x4.y - xb.y, x4.z - xb.z};
        const DV3 c = cross3(r, fb);
        t = DV3{t.x + c.x, t.y + c.y, t.z + c.z};
    }
    out[6 * b] = f.x;
    out[6 * b + 1] = f.y;
    out[6 * b + 2] = f.z;
    out[6 * b + 3] = t.x;
    out[6 * b + 4] = t.y;
    out[6 * b + 5] = t.z;
}

}  // namespace

Coupler::Coupler(World& w, uint32_t n_bodies, uint64_t ns, const int64_t* body, const double* local,
                 const double* local_n, const int64_t* particle)
    : w_(w), nb_(n_bodies), ns_(ns) {
    // samples grouped by body, each group in sample order
    std::vector<uint64_t> start((size_t)nb_ + 1, 0);
    for (uint64_t k = 0; k < ns; ++k) ++start[(size_t)body[k] + 1];
    for (uint32_t b = 0; b < nb_; ++b) start[b + 1] += start[b];
    std::vector<int64_t> grouped(ns);
    std::vector<uint64_t> fill(start.begin(), start.end() - 1);
    for (uint64_t k = 0; k < ns; ++k) grouped[fill[(size_t)body[k]]++] = particle[k];
    body_ = upload(body, ns);
    local_ = upload(local, 3 * ns);
    local_n_ = upload(local_n, 3 * ns);
    particle_ = upload(particle, ns);
    start_ = upload(start.data(), start.size());
    grouped_ = upload(grouped.data(), grouped.size());
    bodies_ = alloc<double>((size_t)nb_ * 13);
    X_ = alloc<double>((size_t)nb_ * 3);
    out_ = alloc<double>((size_t)nb_ * 6);
    if (cudaStreamSynchronize(w_.st_) != cudaSuccess) throw CudaError("coupler upload");
}

Coupler::~Coupler() {
    cudaStreamSynchronize(w_.st_);
    for (void* p : keep_) cudaFree(p);
}

template <typename T>
T* Coupler::alloc(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n * sizeof(T), 16)) != cudaSuccess) throw CudaError("cudaMalloc coupler");
    keep_.push_back(p);
    return static_cast<T*>(p);
}

template <typename T>
T* Coupler::upload(const T* h, size_t n) {
    T* d = alloc<T>(n);
    if (n && cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, w_.st_) != cudaSuccess)
        throw CudaError("coupler upload");
    return d;
}

void Coupler::sync(const double* X, const double* Q, const double* V, const double* Om) {
    std::vector<double> bodies((size_t)nb_ * 13);
    for (uint32_t b = 0; b < nb_; ++b) {
        double* B = bodies.data() + 13 * (size_t)b;
        for (int c = 0; c < 3; ++c) {
            B[c] = X[3 * b + c];
            B[7 + c] = V[3 * b + c];
            B[10 + c] = Om[3 * b + c];
        }
        for (int c = 0; c < 4; ++c) B[3 + c] = Q[4 * b + c];
    }
    cudaStream_t st = w_.st_;
    w_.check(cudaMemcpyAsync(bodies_, bodies.data(), bodies.size() * sizeof(double), cudaMemcpyHostToDevice, st),
             "coupler sync");
    if (ns_)
        k_coupler_sync<<<(unsigned)((ns_ + 255) / 256), 256, 0, st>>>(ns_, w_.dim_, body_, local_, local_n_, particle_,
                                                                       bodies_, w_.slot_of_orig_, w_.cur_);
    w_.check(cudaGetLastError(), "coupler sync");
    w_.refresh_f32();
    w_.check(cudaStreamSynchronize(st), "coupler sync");  // the host buffer must outlive the copy
    // boundary samples moved: the reference rebuilds the grid in the next step
    w_.grid_current_ = false;
    w_.rho_current_ = false;
    w_.lists_valid_ = false;
    w_.lists_checked_ = false;
}

void Coupler::reduce(const double* X, double* force, double* torque) {
    cudaStream_t st = w_.st_;
    std::vector<double> out((size_t)nb_ * 6);
    w_.check(cudaMemcpyAsync(X_, X, (size_t)nb_ * 3 * sizeof(double), cudaMemcpyHostToDevice, st), "coupler reduce");
    if (nb_)
        k_coupler_reduce<<<(nb_ + 127) / 128, 128, 0, st>>>(nb_, start_, grouped_, X_, w_.slot_of_orig_, w_.cur_,
                                                             out_);
    w_.check(cudaGetLastError(), "coupler reduce");
    w_.check(cudaMemcpyAsync(out.data(), out_, out.size() * sizeof(double), cudaMemcpyDeviceToHost, st),
             "coupler reduce");
    w_.check(cudaStreamSynchronize(st), "coupler reduce");
    for (uint32_t b = 0; b < nb_; ++b)
        for (int c = 0; c < 3; ++c) {
            force[3 * b + c] = out[6 * b + c];
            torque[3 * b + c] = out[6 * b + 3 + c];
        }
}

}  // namespace pe
