// Conservation diagnostics and the state hash reduced on the device
// (crates/pe-fluid/src/diagnostics.rs:19-102, wcsph.rs:350-369), with the
// reference's bits and no copy of the particle state to the host.
//
// Sums. The reference adds the fluid particles' terms one after another in
// original index order (momentum, kinetic and potential energy, the density
// error sum). Floating-point addition is not associative, so those sums stay
// sequential: one CTA walks the particles in chunks of 1024 original indices;
// all its threads gather and form the terms of a chunk (boundary samples
// dropped by a block-wide compaction, so the chains only see fluid terms)
// while one thread per sum adds the previous chunk's terms in order from
// shared memory. The fluid centre of mass (sum of positions over the fluid
// count, no reference counterpart) is summed the same way. Skipping a boundary sample equals the reference's
// `continue`: the sums start at +0.0 and never become -0.0. Maxima (density
// error, |v|^2, |a|^2) do not depend on order and are reduced in parallel;
// NaN never wins a comparison, as in the reference's `>` and `f64::max`.
//
// Hash. FNV-1a over the bytes b of the fluid (x, v) in index order,
// h <- (h ^ b) * P (mod 2^64), is split into two parts that parallelise:
//   * the low byte l of h evolves on its own, l <- ((l ^ b) * P) mod 2^8,
//     a 256-state machine: each chunk of particles is run from all 256
//     start states (k_hash_tables), and one thread walks the chunks' tables
//     to find each chunk's start state (k_hash_starts);
//   * given l, h ^ b = h + d with d = (l ^ b) - l, so each byte is the affine
//     map h <- P h + P d: each chunk composes its maps (k_hash_affine) and one
//     thread composes the chunks' maps (k_hash_combine).
#include <cstdint>

#include "world.cuh"

namespace pe {

namespace {

constexpr int kSumThreads = 1024;
constexpr int kChains = 9;  // momentum x, y, z, kinetic energy, potential energy, density error, x, y, z
constexpr uint32_t kHashChunk = 512;     // original indices per hash chunk
constexpr int kHashTableThreads = 128;   // two start states per thread
constexpr int kHashAffineThreads = 128;
constexpr unsigned long long kFnvOffset = 0xcbf29ce484222325ULL;
constexpr unsigned long long kFnvPrime = 0x100000001b3ULL;

struct DiagDev {
    double chain[kChains];
    unsigned long long nf;
    double max_err, vmax2, amax2;
    unsigned long long hash;
};

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

__device__ __forceinline__ double dmax_non_nan(double m, double x) { return x > m ? x : m; }

__global__ void __launch_bounds__(kSumThreads)
    k_diag_sums(uint32_t n, const uint32_t* __restrict__ slot_of_orig, const double4* __restrict__ pos,
                const double4* __restrict__ vel, const double4* __restrict__ acc,
                const uint8_t* __restrict__ flags, double m, double g, double rho0, DiagDev* out) {
    extern __shared__ double sh_terms[];  // [2][kChains][kSumThreads]
    __shared__ uint32_t wcount[kSumThreads / 32];
    __shared__ uint32_t ccount[2];
    __shared__ double red[3][kSumThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t nch = (n + kSumThreads - 1) / kSumThreads;
    double chain = 0.0;  // the running sum of chain `warp` (lane 0 of warps 0..5)
    double mx_err = 0.0, mx_v2 = 0.0, mx_a2 = 0.0;
    unsigned long long nf = 0;
    for (uint32_t k = 0; k <= nch; ++k) {
        // gather chunk k (the loads stay in flight while the chains run)
        bool fl = false;
        double4 vi = make_double4(0, 0, 0, 0), xi = vi, ai = vi;
        const uint64_t i = (uint64_t)k * kSumThreads + tid;
        if (k < nch && i < n) {
            const uint32_t s = slot_of_orig[i];
            if (!(flags[s] & kFlagBoundary)) {
                fl = true;
                vi = vel[s];
                xi = pos[s];
                ai = acc[s];
            }
        }
        // add chunk k - 1 in index order
        if (k > 0 && lane == 0 && warp < kChains) {
            const double* src = sh_terms + ((k - 1) & 1) * kChains * kSumThreads + warp * kSumThreads;
            const uint32_t cnt = ccount[(k - 1) & 1];
            double s = chain;
            for (uint32_t j = 0; j < cnt; ++j) s = s + src[j];
            chain = s;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, fl);
        if (lane == 0) wcount[warp] = __popc(bal);
        __syncthreads();
        if (k < nch) {
            uint32_t off = 0, total = 0;
            for (int w = 0; w < kSumThreads / 32; ++w) {
                const uint32_t c = wcount[w];
                off += w < warp ? c : 0u;
                total += c;
            }
            if (fl) {
                const uint32_t at = off + __popc(bal & ((1u << lane) - 1u));
                double* dst = sh_terms + (k & 1) * kChains * kSumThreads;
                const double v2 = vi.x * vi.x + vi.y * vi.y + vi.z * vi.z;  // vec3.rs norm_squared
                const double e = fabs(vi.w - rho0) / rho0;                  // diagnostics.rs:79
                dst[0 * kSumThreads + at] = vi.x * m;                       // diagnostics.rs:45 (v * mass)
                dst[1 * kSumThreads + at] = vi.y * m;
                dst[2 * kSumThreads + at] = vi.z * m;
                dst[3 * kSumThreads + at] = 0.5 * m * v2;                   // diagnostics.rs:56
                dst[4 * kSumThreads + at] = m * g * xi.z;                   // diagnostics.rs:67
                dst[5 * kSumThreads + at] = e;
                dst[6 * kSumThreads + at] = xi.x;  // centre of mass (no reference counterpart)
                dst[7 * kSumThreads + at] = xi.y;
                dst[8 * kSumThreads + at] = xi.z;
                mx_err = dmax_non_nan(mx_err, e);                           // diagnostics.rs:97
                mx_v2 = dmax_non_nan(mx_v2, v2);                            // viscosity.rs:93
                mx_a2 = dmax_non_nan(mx_a2, ai.x * ai.x + ai.y * ai.y + ai.z * ai.z);  // wcsph.rs:365
            }
            if (tid == 0) {
                ccount[k & 1] = total;
                nf += total;
            }
        }
        __syncthreads();
    }
    // block maxima (order-free)
    for (int o = 16; o > 0; o >>= 1) {
        mx_err = dmax_non_nan(mx_err, __shfl_xor_sync(0xffffffffu, mx_err, o));
        mx_v2 = dmax_non_nan(mx_v2, __shfl_xor_sync(0xffffffffu, mx_v2, o));
        mx_a2 = dmax_non_nan(mx_a2, __shfl_xor_sync(0xffffffffu, mx_a2, o));
    }
    if (lane == 0) {
        red[0][warp] = mx_err;
        red[1][warp] = mx_v2;
        red[2][warp] = mx_a2;
    }
    __syncthreads();
    if (tid == 0) {
        double a = 0.0, b = 0.0, c = 0.0;
        for (int w = 0; w < kSumThreads / 32; ++w) {
            a = dmax_non_nan(a, red[0][w]);
            b = dmax_non_nan(b, red[1][w]);
            c = dmax_non_nan(c, red[2][w]);
        }
        out->max_err = a;
        out->vmax2 = b;
        out->amax2 = c;
        out->nf = nf;
    }
    if (lane == 0 && warp < kChains) out->chain[warp] = chain;
}

// Stages the fluid (x, v) of original indices [base, base + kHashChunk) as
// 64-bit words in index order (six per fluid particle); returns the count.
template <int THREADS>
__device__ uint32_t stage_hash_chunk(uint32_t n, uint64_t base, const uint32_t* __restrict__ slot_of_orig,
                                     const double4* __restrict__ pos, const double4* __restrict__ vel,
                                     const uint8_t* __restrict__ flags, unsigned long long* words,
                                     uint32_t* wcount) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int kWarps = THREADS / 32;
    uint32_t done = 0;
    for (uint32_t part = 0; part < kHashChunk / THREADS; ++part) {
        const uint64_t i = base + (uint64_t)part * THREADS + tid;
        bool fl = false;
        double4 xi = make_double4(0, 0, 0, 0), vi = xi;
        if (i < n) {
            const uint32_t s = slot_of_orig[i];
            if (!(flags[s] & kFlagBoundary)) {
                fl = true;
                xi = pos[s];
                vi = vel[s];
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, fl);
        if (lane == 0) wcount[warp] = __popc(bal);
        __syncthreads();
        uint32_t off = 0, total = 0;
        for (int w = 0; w < kWarps; ++w) {
            off += w < warp ? wcount[w] : 0u;
            total += wcount[w];
        }
        if (fl) {
            unsigned long long* d = words + 6 * (size_t)(done + off + __popc(bal & ((1u << lane) - 1u)));
            d[0] = (unsigned long long)__double_as_longlong(xi.x);
            d[1] = (unsigned long long)__double_as_longlong(xi.y);
            d[2] = (unsigned long long)__double_as_longlong(xi.z);
            d[3] = (unsigned long long)__double_as_longlong(vi.x);
            d[4] = (unsigned long long)__double_as_longlong(vi.y);
            d[5] = (unsigned long long)__double_as_longlong(vi.z);
        }
        done += total;
        __syncthreads();
    }
    return done;
}

// The low byte's state after chunk c for every start state (two per thread,
// in the 16-bit halves of one register: (l ^ b) * 0xb3 < 2^16, so the halves
// never carry into each other).
__global__ void __launch_bounds__(kHashTableThreads)
    k_hash_tables(uint32_t n, const uint32_t* __restrict__ slot_of_orig, const double4* __restrict__ pos,
                  const double4* __restrict__ vel, const uint8_t* __restrict__ flags, uint8_t* tabs,
                  uint32_t* chunk_fluid) {
    __shared__ unsigned long long words[6 * kHashChunk];
    __shared__ uint32_t wcount[kHashTableThreads / 32];
    const uint32_t c = blockIdx.x;
    const uint32_t nf = stage_hash_chunk<kHashTableThreads>(n, (uint64_t)c * kHashChunk, slot_of_orig, pos, vel,
                                                            flags, words, wcount);
    const uint32_t tid = threadIdx.x;
    uint32_t x = tid | ((tid + kHashTableThreads) << 16);
    const uint32_t nw = 6 * nf;
    for (uint32_t w = 0; w < nw; ++w) {
        const unsigned long long word = words[w];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t b = (uint32_t)(word >> (8 * k)) & 0xffu;
            x = ((x ^ (b | (b << 16))) * 0xb3u) & 0x00ff00ffu;  // P mod 2^8 = 0xb3
        }
    }
    tabs[(size_t)c * 256 + tid] = (uint8_t)(x & 0xffu);
    tabs[(size_t)c * 256 + tid + kHashTableThreads] = (uint8_t)(x >> 16);
    if (tid == 0) chunk_fluid[c] = nf;
}

// Start state of every chunk: one thread walks the tables, a slice of them
// staged in shared memory at a time.
__global__ void __launch_bounds__(256) k_hash_starts(uint32_t nch, const uint8_t* __restrict__ tabs,
                                                     uint8_t* lstart) {
    constexpr uint32_t kSlice = 64;
    __shared__ uint32_t t[kSlice * 64];
    uint32_t l = (uint32_t)(kFnvOffset & 0xffu);
    for (uint32_t c0 = 0; c0 < nch; c0 += kSlice) {
        const uint32_t cn = min(kSlice, nch - c0);
        const uint32_t* src = reinterpret_cast<const uint32_t*>(tabs + (size_t)c0 * 256);
        for (uint32_t j = threadIdx.x; j < cn * 64; j += blockDim.x) t[j] = src[j];
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint8_t* tb = reinterpret_cast<const uint8_t*>(t);
            for (uint32_t j = 0; j < cn; ++j) {
                lstart[c0 + j] = (uint8_t)l;
                l = tb[j * 256 + l];
            }
        }
        __syncthreads();
    }
}

// The affine map h -> a h + c (mod 2^64) of chunk c, from its known start
// state of the low byte.
__global__ void __launch_bounds__(kHashAffineThreads)
    k_hash_affine(uint32_t n, const uint32_t* __restrict__ slot_of_orig, const double4* __restrict__ pos,
                  const double4* __restrict__ vel, const uint8_t* __restrict__ flags,
                  const uint8_t* __restrict__ lstart, unsigned long long* amap, unsigned long long* cmap) {
    __shared__ unsigned long long words[6 * kHashChunk];
    __shared__ uint32_t wcount[kHashAffineThreads / 32];
    const uint32_t c = blockIdx.x;
    const uint32_t nf = stage_hash_chunk<kHashAffineThreads>(n, (uint64_t)c * kHashChunk, slot_of_orig, pos, vel,
                                                             flags, words, wcount);
    if (threadIdx.x != 0) return;
    unsigned long long a = 1ULL, cc = 0ULL;
    uint32_t l = lstart[c];
    const uint32_t nw = 6 * nf;
    for (uint32_t w = 0; w < nw; ++w) {
        const unsigned long long word = words[w];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t b = (uint32_t)(word >> (8 * k)) & 0xffu;
            const uint32_t lb = l ^ b;
            const unsigned long long d = (unsigned long long)((long long)lb - (long long)l);
            cc = (cc + d) * kFnvPrime;
            a = a * kFnvPrime;
            l = (lb * 0xb3u) & 0xffu;
        }
    }
    amap[c] = a;
    cmap[c] = cc;
}

__global__ void k_hash_combine(uint32_t nch, const unsigned long long* __restrict__ amap,
                               const unsigned long long* __restrict__ cmap, DiagDev* out) {
    if (threadIdx.x != 0) return;
    unsigned long long h = kFnvOffset;
    for (uint32_t c = 0; c < nch; ++c) h = amap[c] * h + cmap[c];
    out->hash = h;
}

}  // namespace

void World::diagnostics(Diagnostics* d) {
    *d = Diagnostics{};
    d->hash64 = kFnvOffset;
    const uint32_t n = (uint32_t)n_;
    if (!n) return;
    const uint32_t nch = blocks_for(n, kHashChunk);
    if (!diag_buf_) {
        void* p = nullptr;
        check(cudaMalloc(&p, 256 + (size_t)nch * (256 + 4 + 1 + 16) + 1024), "cudaMalloc");
        allocs_.push_back(p);  // freed with the world
        diag_buf_ = static_cast<unsigned char*>(p);
    }
    check(cudaFuncSetAttribute(k_diag_sums, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(2 * kChains * kSumThreads * sizeof(double))),
          "diagnostics smem");
    unsigned char* b = static_cast<unsigned char*>(diag_buf_);
    DiagDev* dd = reinterpret_cast<DiagDev*>(b);
    unsigned long long* amap = reinterpret_cast<unsigned long long*>(b + 256);
    unsigned long long* cmap = amap + nch;
    uint8_t* tabs = reinterpret_cast<uint8_t*>(cmap + nch);
    uint32_t* chunk_fluid = reinterpret_cast<uint32_t*>(tabs + (size_t)nch * 256);
    uint8_t* lstart = reinterpret_cast<uint8_t*>(chunk_fluid + nch);
    const double g = -prm_.gravity[2];
    k_diag_sums<<<1, kSumThreads, 2 * kChains * kSumThreads * sizeof(double), st_>>>(
        n, slot_of_orig_, cur_.pos, cur_.vel, cur_.acc, cur_.flags, mass_, g, rho0_, dd);
    k_hash_tables<<<nch, kHashTableThreads, 0, st_>>>(n, slot_of_orig_, cur_.pos, cur_.vel, cur_.flags, tabs,
                                                      chunk_fluid);
    k_hash_starts<<<1, 256, 0, st_>>>(nch, tabs, lstart);
    k_hash_affine<<<nch, kHashAffineThreads, 0, st_>>>(n, slot_of_orig_, cur_.pos, cur_.vel, cur_.flags, lstart,
                                                       amap, cmap);
    k_hash_combine<<<1, 32, 0, st_>>>(nch, amap, cmap, dd);
    launches_ += 5;
    check(cudaGetLastError(), "diagnostics");
    DiagDev h{};
    check(cudaMemcpyAsync(&h, dd, sizeof(h), cudaMemcpyDeviceToHost, st_), "diagnostics");
    check(cudaStreamSynchronize(st_), "diagnostics");
    d->total_mass = mass_ * (double)h.nf;  // particles.rs:159-161
    for (int a = 0; a < 3; ++a) d->linear_momentum[a] = h.chain[a];
    d->kinetic_energy = h.chain[3];
    d->gravitational_potential = h.chain[4];
    d->mean_density_error = h.nf ? h.chain[5] / (double)h.nf : 0.0;  // diagnostics.rs:84-88
    d->max_density_error = h.max_err;
    d->v_max = sqrt(h.vmax2);  // viscosity.rs:99
    d->a_max = sqrt(h.amax2);  // wcsph.rs:368
    d->hash64 = h.hash;
    d->fluid = h.nf;
    for (int a = 0; a < 3; ++a) d->fluid_com[a] = h.nf ? h.chain[6 + a] / (double)h.nf : 0.0;
}

}  // namespace pe
