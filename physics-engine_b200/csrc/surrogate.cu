// Learned surrogate: parameters, forward and backward passes of the two-hop
// message-passing network (see surrogate.cuh), Adam, and the graph built from
// a world's state. Training materialises the activations of a tank-sized
// graph; every matrix product runs on the tcgen05 GEMM (mlp_gemm.cu).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "surrogate.cuh"

namespace pe {

namespace {

constexpr float kAggScale = 1.0f / 16.0f;

inline unsigned blocks(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }
inline int round8(int v) { return (v + 7) & ~7; }

void cu(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("surrogate ") + what + ": " + cudaGetErrorString(e));
}

__global__ void k_to_bf16(size_t n, const float* __restrict__ src, __nv_bfloat16* __restrict__ dst) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

// out_i = scale * sum of rows [row_i, row_{i+1}) of in (a warp per node)
__global__ void k_segsum(int n, const int* __restrict__ row, const float* __restrict__ in, float scale,
                         float* __restrict__ out) {
    const int node = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (node >= n) return;
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int e = row[node]; e < row[node + 1]; ++e) {
        const float4 v = reinterpret_cast<const float4*>(in + (size_t)e * kWidth)[lane];
        s.x += v.x;
        s.y += v.y;
        s.z += v.z;
        s.w += v.w;
    }
    s.x *= scale;
    s.y *= scale;
    s.z *= scale;
    s.w *= scale;
    reinterpret_cast<float4*>(out + (size_t)node * kWidth)[lane] = s;
}

// [h | scale * a] as the node MLP's bf16 input
__global__ void k_concat(int n, const __nv_bfloat16* __restrict__ hb, const float* __restrict__ a, float scale,
                         __nv_bfloat16* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * 2 * kWidth) return;
    const size_t node = i / (2 * kWidth);
    const int c = (int)(i % (2 * kWidth));
    out[i] = c < kWidth ? hb[node * kWidth + c] : __float2bfloat16_rn(a[node * kWidth + c - kWidth] * scale);
}

// h += u on fluid nodes; hb_next = bf16(h)
__global__ void k_residual(int n, const float* __restrict__ u, const uint8_t* __restrict__ fluid,
                           float* __restrict__ h, __nv_bfloat16* __restrict__ hb_next) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * kWidth) return;
    float v = h[i];
    if (fluid[i / kWidth]) v += u[i];
    h[i] = v;
    hb_next[i] = __float2bfloat16_rn(v);
}

// loss = sum over fluid nodes of |y - t|^2 / nf; dY = 2 (y - t) / nf (padding columns 0)
__global__ void k_loss(int n, const float* __restrict__ Y, const float* __restrict__ T,
                       const uint8_t* __restrict__ fluid, float inv_nf, float* __restrict__ dY,
                       float* __restrict__ loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (i < n) {
#pragma unroll
        for (int c = 0; c < kOutPad; ++c) {
            float d = 0.f;
            if (c < kOut && fluid[i]) d = Y[(size_t)i * kOutPad + c] - T[(size_t)i * kOut + c];
            dY[(size_t)i * kOutPad + c] = 2.f * d * inv_nf;
            l += d * d;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l * inv_nf);
}

// dZ (fp32 [R x N]) masked in place by mask > 0; bf16 copies dZ [R8 x N] and
// dZ^T [N x R8] (zero-padded rows / columns); column sums into gbias
__global__ void k_grad_prep(int R, int R8, int N, float* __restrict__ dZ, const __nv_bfloat16* __restrict__ mask,
                            __nv_bfloat16* __restrict__ g16, __nv_bfloat16* __restrict__ gT,
                            float* __restrict__ gbias) {
    __shared__ float tile[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    float csum = 0.f;
    for (int k = ty; k < 32; k += 8) {
        const int r = r0 + k, c = c0 + tx;
        float v = 0.f;
        if (r < R && c < N) {
            v = dZ[(size_t)r * N + c];
            if (mask && !(__bfloat162float(mask[(size_t)r * N + c]) > 0.f)) v = 0.f;
            dZ[(size_t)r * N + c] = v;
        }
        if (r < R8 && c < N) g16[(size_t)r * N + c] = __float2bfloat16_rn(v);
        tile[k][tx] = v;
        csum += v;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int c = c0 + k, r = r0 + tx;
        if (c < N && r < R8) gT[(size_t)c * R8 + r] = __float2bfloat16_rn(tile[tx][k]);
    }
    if (gbias && c0 + tx < N && csum != 0.f) atomicAdd(&gbias[c0 + tx], csum);
}

// X (bf16 [R x K]) -> X^T (bf16 [K x R8]), zero columns R..R8
__global__ void k_transpose(int R, int R8, int K, const __nv_bfloat16* __restrict__ X,
                            __nv_bfloat16* __restrict__ XT) {
    __shared__ __nv_bfloat16 tile[32][34];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int k = ty; k < 32; k += 8) {
        const int r = r0 + k, c = c0 + tx;
        tile[k][tx] = (r < R && c < K) ? X[(size_t)r * K + c] : __float2bfloat16_rn(0.f);
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int c = c0 + k, r = r0 + tx;
        if (c < K && r < R8) XT[(size_t)c * R8 + r] = tile[tx][k];
    }
}

__global__ void k_mask_rows(int n, const float* __restrict__ in, const uint8_t* __restrict__ fluid,
                            float* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (size_t)n * kWidth) out[i] = fluid[i / kWidth] ? in[i] : 0.f;
}

// dHp = dH + dXN[:, :128]; da = scale * dXN[:, 128:]
__global__ void k_split_dxn(int n, const float* __restrict__ dH, const float* __restrict__ dXN, float scale,
                            float* __restrict__ dHp, float* __restrict__ da) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * kWidth) return;
    const size_t node = i / kWidth, c = i % kWidth;
    dHp[i] = dH[i] + dXN[node * 2 * kWidth + c];
    da[i] = scale * dXN[node * 2 * kWidth + kWidth + c];
}

__global__ void k_gather_rows(int E, const int* __restrict__ idx, const float* __restrict__ in,
                              float* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)E * kWidth) return;
    out[i] = in[(size_t)idx[i / kWidth] * kWidth + i % kWidth];
}

__global__ void k_scatter_add(int E, const int* __restrict__ idx, const float* __restrict__ in,
                              float* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)E * kWidth) return;
    const float v = in[i];
    if (v != 0.f) atomicAdd(&out[(size_t)idx[i / kWidth] * kWidth + i % kWidth], v);
}

__global__ void k_add(size_t n, float* __restrict__ a, const float* __restrict__ b) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] += b[i];
}

__global__ void k_adam(size_t n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float c1, float c2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
}

// bf16 copies of a master Wt [Np x K]: Wt16 (same layout) and W16 [K x Np]
__global__ void k_refresh(int Np, int K, const float* __restrict__ Wt, __nv_bfloat16* __restrict__ Wt16,
                          __nv_bfloat16* __restrict__ W16) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Np * K) return;
    const int n = i / K, k = i % K;
    const __nv_bfloat16 b = __float2bfloat16_rn(Wt[i]);
    Wt16[i] = b;
    W16[(size_t)k * Np + n] = b;
}

// host-side seeded normal numbers (xoshiro256** + Box-Muller)
struct HostRng {
    uint64_t s[4];
    explicit HostRng(uint64_t seed) {
        uint64_t z = seed;
        for (auto& v : s) {
            z += 0x9e3779b97f4a7c15ULL;
            uint64_t x = z;
            x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
            x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
            v = x ^ (x >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() { return std::sqrt(-2.0 * std::log(uniform())) * std::cos(6.283185307179586 * uniform()); }
};

}  // namespace

template <typename T>
T* Surrogate::dalloc(size_t n) {
    void* p = nullptr;
    cu(cudaMalloc(&p, std::max<size_t>(n * sizeof(T), 256)), "cudaMalloc");
    cu(cudaMemsetAsync(p, 0, std::max<size_t>(n * sizeof(T), 256), st_), "memset");
    return static_cast<T*>(p);
}

Surrogate::Surrogate(uint64_t seed, double r_msg_over_h) : r_msg_over_h_(r_msg_over_h) {
    cu(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "stream");
    own_stream_ = true;
    if (!gemm_prepare()) throw std::runtime_error("surrogate: GEMM shared-memory limit");
    if (!edge_hop_prepare()) throw std::runtime_error("surrogate: fused edge kernel shared-memory limit");
    {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess)
            cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev);
    }
    err_ = dalloc<uint32_t>(1);
    allocs_.push_back(err_);
    loss_ = dalloc<float>(1);
    allocs_.push_back(loss_);
    for (int c = 0; c < kOut; ++c) {
        stats_.mean[c] = 0.f;
        stats_.std[c] = 1.f;
    }
    alloc_params(seed);
}

Surrogate::~Surrogate() {
    if (st_) cudaStreamSynchronize(st_);
    for (void* p : allocs_) cudaFree(p);
    for (void* p : graph_allocs_) cudaFree(p);
    for (void* p : act_allocs_) cudaFree(p);
    if (part_) cudaFree(part_);
    if (scan_tmp_) cudaFree(scan_tmp_);
    if (own_stream_ && st_) cudaStreamDestroy(st_);
}

void Surrogate::alloc_params(uint64_t seed) {
    auto add = [&](const std::string& name, int K, int N, bool bias) {
        Linear L;
        L.name = name;
        L.K = K;
        L.N = N;
        L.Np = round8(N);
        L.has_bias = bias;
        layers_.push_back(L);
    };
    auto mlp = [&](const std::string& name, int K, int N) {
        add(name + ".0", K, kWidth, true);
        add(name + ".1", kWidth, kWidth, true);
        add(name + ".2", kWidth, N, true);
    };
    mlp("enc", kNodeFeat, kWidth);
    for (int l = 1; l <= 2; ++l) {
        const std::string h = "hop" + std::to_string(l);
        add(h + ".edge.a", kWidth, kWidth, false);
        add(h + ".edge.b", kWidth, kWidth, false);
        add(h + ".edge.0", kEdgeFeat, kWidth, true);
        add(h + ".edge.1", kWidth, kWidth, true);
        add(h + ".edge.2", kWidth, kWidth, true);
        mlp(h + ".node", 2 * kWidth, kWidth);
    }
    mlp("dec", kWidth, kOut);
    HostRng rng(seed);
    for (Linear& L : layers_) {
        const size_t nw = (size_t)L.Np * L.K;
        L.Wt = dalloc<float>(nw);
        L.gWt = dalloc<float>(nw);
        L.mW = dalloc<float>(nw);
        L.vW = dalloc<float>(nw);
        L.b = dalloc<float>(L.Np);
        L.gb = dalloc<float>(L.Np);
        L.mb = dalloc<float>(L.Np);
        L.vb = dalloc<float>(L.Np);
        L.Wt16 = dalloc<__nv_bfloat16>(nw);
        L.W16 = dalloc<__nv_bfloat16>(nw);
        for (void* p : {(void*)L.Wt, (void*)L.gWt, (void*)L.mW, (void*)L.vW, (void*)L.b, (void*)L.gb, (void*)L.mb,
                        (void*)L.vb, (void*)L.Wt16, (void*)L.W16})
            allocs_.push_back(p);
        // He initialisation for the ReLU layers; the decoder's output layer starts small
        const bool out_layer = L.name == "dec.2";
        const double sd = std::sqrt(2.0 / L.K) * (out_layer ? 0.1 : 1.0);
        std::vector<float> w(nw, 0.f);
        for (int n = 0; n < L.N; ++n)
            for (int k = 0; k < L.K; ++k) w[(size_t)n * L.K + k] = (float)(sd * rng.normal());
        cu(cudaMemcpyAsync(L.Wt, w.data(), nw * sizeof(float), cudaMemcpyHostToDevice, st_), "init");
        cu(cudaStreamSynchronize(st_), "init");
        refresh_bf16(L);
    }
}

void Surrogate::refresh_bf16(Linear& L) {
    const int n = L.Np * L.K;
    k_refresh<<<blocks(n, 256), 256, 0, st_>>>(L.Np, L.K, L.Wt, L.Wt16, L.W16);
}

void Surrogate::get_param(int i, float* W, float* b, bool grad) {
    const Linear& L = layers_.at(i);
    std::vector<float> wt((size_t)L.Np * L.K), bb(L.Np);
    cu(cudaMemcpyAsync(wt.data(), grad ? L.gWt : L.Wt, wt.size() * 4, cudaMemcpyDeviceToHost, st_), "get");
    cu(cudaMemcpyAsync(bb.data(), grad ? L.gb : L.b, bb.size() * 4, cudaMemcpyDeviceToHost, st_), "get");
    cu(cudaStreamSynchronize(st_), "get");
    if (W)
        for (int k = 0; k < L.K; ++k)
            for (int n = 0; n < L.N; ++n) W[(size_t)k * L.N + n] = wt[(size_t)n * L.K + k];
    if (b)
        for (int n = 0; n < L.N; ++n) b[n] = L.has_bias ? bb[n] : 0.f;
}

void Surrogate::set_param(int i, const float* W, const float* b) {
    Linear& L = layers_.at(i);
    std::vector<float> wt((size_t)L.Np * L.K, 0.f), bb(L.Np, 0.f);
    cu(cudaMemcpyAsync(wt.data(), L.Wt, wt.size() * 4, cudaMemcpyDeviceToHost, st_), "set");
    cu(cudaStreamSynchronize(st_), "set");
    if (W)
        for (int k = 0; k < L.K; ++k)
            for (int n = 0; n < L.N; ++n) wt[(size_t)n * L.K + k] = W[(size_t)k * L.N + n];
    if (b && L.has_bias)
        for (int n = 0; n < L.N; ++n) bb[n] = b[n];
    cu(cudaMemcpyAsync(L.Wt, wt.data(), wt.size() * 4, cudaMemcpyHostToDevice, st_), "set");
    if (b && L.has_bias) cu(cudaMemcpyAsync(L.b, bb.data(), bb.size() * 4, cudaMemcpyHostToDevice, st_), "set");
    cu(cudaStreamSynchronize(st_), "set");
    refresh_bf16(L);
}

void Surrogate::ensure_graph(int n, int E) {
    if (n <= g_.cap_n && E <= g_.cap_e) {
        g_.n = n;
        g_.E = E;
        return;
    }
    cu(cudaStreamSynchronize(st_), "graph");
    for (void* p : graph_allocs_) cudaFree(p);
    graph_allocs_.clear();
    if (scan_tmp_) cudaFree(scan_tmp_);
    // grow with a quarter of headroom: the edge count creeps up step by step as
    // the fluid compresses, and every growth reallocates
    const int cn = std::max(n + n / 4, g_.cap_n), ce = std::max(E + E / 4, g_.cap_e);
    auto ga = [&](size_t bytes) {
        void* p = nullptr;
        cu(cudaMalloc(&p, std::max<size_t>(bytes, 256)), "cudaMalloc graph");
        graph_allocs_.push_back(p);
        return p;
    };
    g_.row = static_cast<int*>(ga((size_t)(cn + 1) * 4));
    g_.src = static_cast<int*>(ga((size_t)ce * 4));
    g_.dst = static_cast<int*>(ga((size_t)ce * 4));
    g_.xe = static_cast<__nv_bfloat16*>(ga((size_t)ce * kEdgeFeat * 2));
    g_.f = static_cast<__nv_bfloat16*>(ga((size_t)cn * kNodeFeat * 2));
    g_.fluid = static_cast<uint8_t*>(ga((size_t)cn));
    node_orig_ = static_cast<uint32_t*>(ga((size_t)cn * 4));
    node_v_ = static_cast<double*>(ga((size_t)cn * 4 * 8));
    target_ = static_cast<float*>(ga((size_t)cn * kOut * 4));
    raw_t_ = static_cast<float*>(ga((size_t)cn * kOut * 4));
    cnt_ = static_cast<int*>(ga((size_t)(cn + 1) * 4));
    scan_tmp_ = nullptr;
    scan_bytes_ = 0;
    g_.cap_n = cn;
    g_.cap_e = ce;
    g_.n = n;
    g_.E = E;
}

void Surrogate::ensure_acts(bool train) {
    // Inference keeps one hop's edge activations and no backward buffers: at a
    // million particles (~3e7 edges) that is ~1.5 KB per edge instead of ~4.6.
    const int n = g_.n, E = g_.E;
    if (n <= act_n_ && E <= act_e_ && (act_train_ || !train)) return;
    cu(cudaStreamSynchronize(st_), "acts");
    for (void* p : act_allocs_) cudaFree(p);
    act_allocs_.clear();
    // grow with a quarter of headroom; a switch to training sizes for the
    // current graph only (training buffers cost ~3x per edge)
    const bool keep = act_train_ || !train;
    const int cn = round8(std::max(n + n / 4, keep ? act_n_ : 0));
    const int ce = round8(std::max(E + E / 4, keep ? act_e_ : 0));
    auto fa = [&](size_t count) {
        void* p = nullptr;
        cu(cudaMalloc(&p, std::max<size_t>(count * 4, 256)), "cudaMalloc acts");
        act_allocs_.push_back(p);
        return static_cast<float*>(p);
    };
    auto ba = [&](size_t count) {
        void* p = nullptr;
        cu(cudaMalloc(&p, std::max<size_t>(count * 2, 256)), "cudaMalloc acts");
        act_allocs_.push_back(p);
        return static_cast<__nv_bfloat16*>(p);
    };
    const size_t W = kWidth;
    enc_a1_ = ba(cn * W);
    enc_a2_ = ba(cn * W);
    h_ = fa(cn * W);
    for (auto& p : hb_) p = ba(cn * W);
    P_ = fa(cn * W);
    Q_ = fa(cn * W);
    for (int l = 0; l < 2; ++l) {
        eh1_[l] = (l == 0 || train) ? ba(ce * W) : eh1_[0];
        eh2_[l] = (l == 0 || train) ? ba(ce * W) : eh2_[0];
        xn_[l] = ba(cn * 2 * W);
        na1_[l] = ba(cn * W);
        na2_[l] = ba(cn * W);
    }
    M_ = fa(ce * W);
    A_ = fa(cn * W);
    U_ = fa(cn * W);
    da1_ = ba(cn * W);
    da2_ = ba(cn * W);
    Y_ = fa(cn * kOutPad);
    dY_ = fa(cn * kOutPad);
    dH_ = fa(cn * W);
    dHp_ = fa(cn * W);
    dXN_ = fa(cn * 2 * W);
    dE_ = train ? fa(ce * W) : nullptr;
    dE2_ = train ? fa(ce * W) : nullptr;
    dP_ = fa(cn * W);
    dQ_ = fa(cn * W);
    dT1_ = fa(cn * W);
    dT2_ = fa(cn * W);
    const size_t rows = train ? (size_t)std::max(cn, ce) : 0;
    gb16_ = train ? ba(rows * 2 * W) : nullptr;
    gbT_ = train ? ba(rows * 2 * W) : nullptr;
    xT_ = train ? ba(rows * 2 * W) : nullptr;
    act_n_ = cn;
    act_e_ = ce;
    act_train_ = train;
}

void Surrogate::gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* Bt, int ldb, int M, int N, int K,
                     float* Cf, __nv_bfloat16* Cb, int ldc, const float* bias, bool relu, int splits) {
    if (M <= 0 || N <= 0) return;
    if (splits > 1) {
        const size_t need = (size_t)splits * M * ldc;
        if (need > part_floats_) {
            cu(cudaStreamSynchronize(st_), "part");
            if (part_) cudaFree(part_);
            cu(cudaMalloc(&part_, need * 4), "cudaMalloc part");
            part_floats_ = need;
        }
        GemmArgs g{A, Bt, part_, nullptr, nullptr, M, N, K, lda, ldb, ldc, 0, err_};
        launch_gemm(g, splits, st_);
        launch_gemm_reduce(M, N, ldc, splits, part_, bias, relu ? 1 : 0, Cf, Cb, st_);
    } else {
        GemmArgs g{A, Bt, Cf, Cb, bias, M, N, K, lda, ldb, ldc, relu ? 1 : 0, err_};
        launch_gemm(g, 1, st_);
    }
}

void Surrogate::linear_fwd(const Linear& L, const __nv_bfloat16* X, int R, float* Yf, __nv_bfloat16* Yb,
                           bool relu) {
    gemm(X, L.K, L.Wt16, L.K, R, L.Np, L.K, Yf, Yb, L.Np, L.has_bias ? L.b : nullptr, relu);
}

void Surrogate::mlp_fwd(int first, const __nv_bfloat16* X, int R, __nv_bfloat16* A1, __nv_bfloat16* A2,
                        float* Yf) {
    linear_fwd(layers_[first], X, R, nullptr, A1, true);
    linear_fwd(layers_[first + 1], A1, R, nullptr, A2, true);
    linear_fwd(layers_[first + 2], A2, R, Yf, nullptr, false);
}

void Surrogate::forward(bool keep_for_backward) {
    ensure_acts(keep_for_backward);
    const int n = g_.n, E = g_.E;
    const size_t nW = (size_t)n * kWidth;
    mlp_fwd(0, g_.f, n, enc_a1_, enc_a2_, h_);
    k_to_bf16<<<blocks(nW, 256), 256, 0, st_>>>(nW, h_, hb_[0]);
    for (int l = 0; l < 2; ++l) {
        const int base = 3 + 8 * l;
        linear_fwd(layers_[base + 0], hb_[l], n, P_, nullptr, false);
        linear_fwd(layers_[base + 1], hb_[l], n, Q_, nullptr, false);
        if (E > 0 && fused_edges_ && !keep_for_backward) {
            // the whole edge MLP and the sum per destination in one kernel
            const Linear &L0 = layers_[base + 2], &L1 = layers_[base + 3], &L2 = layers_[base + 4];
            cu(cudaMemsetAsync(A_, 0, sizeof(float) * nW, st_), "memset");
            EdgeHopArgs ea{E, g_.src, g_.dst, g_.xe, P_, Q_, L0.Wt16, L0.b, L1.Wt16, L1.b, L2.Wt16, L2.b, A_, err_};
            launch_edge_hop(ea, sms_, st_);
        } else if (E > 0) {
            // layer 1: relu(x_e Wc + b1 + P[dst] + Q[src]), the gathers fused into the GEMM's epilogue
            const Linear& L0 = layers_[base + 2];
            GemmArgs ga{g_.xe, L0.Wt16, nullptr, eh1_[l], L0.b, E, L0.Np, L0.K, L0.K, L0.K, L0.Np, 1, err_};
            ga.add0 = P_;
            ga.idx0 = g_.dst;
            ga.add1 = Q_;
            ga.idx1 = g_.src;
            ga.ld_add = kWidth;
            launch_gemm(ga, 1, st_);
            linear_fwd(layers_[base + 3], eh1_[l], E, nullptr, eh2_[l], true);
            linear_fwd(layers_[base + 4], eh2_[l], E, M_, nullptr, false);
        }
        if (!(E > 0 && fused_edges_ && !keep_for_backward))
            k_segsum<<<blocks((size_t)n * 32, 256), 256, 0, st_>>>(n, g_.row, M_, 1.f, A_);
        k_concat<<<blocks(2 * nW, 256), 256, 0, st_>>>(n, hb_[l], A_, kAggScale, xn_[l]);
        mlp_fwd(base + 5, xn_[l], n, na1_[l], na2_[l], U_);
        k_residual<<<blocks(nW, 256), 256, 0, st_>>>(n, U_, g_.fluid, h_, hb_[l + 1]);
    }
    mlp_fwd(19, hb_[2], n, da1_, da2_, Y_);
    cu(cudaGetLastError(), "forward");
}

void Surrogate::get_outputs(float* y) {
    const int n = g_.n;
    std::vector<float> buf((size_t)n * kOutPad);
    cu(cudaMemcpyAsync(buf.data(), Y_, buf.size() * 4, cudaMemcpyDeviceToHost, st_), "outputs");
    cu(cudaStreamSynchronize(st_), "outputs");
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < kOut; ++c) y[(size_t)i * kOut + c] = buf[(size_t)i * kOutPad + c];
}

void Surrogate::linear_bwd(Linear& L, const __nv_bfloat16* X, int R, float* dZ, const __nv_bfloat16* mask,
                           float* dX) {
    if (R <= 0) return;
    const int R8 = round8(R);
    dim3 tb(32, 8);
    dim3 gz(blocks(R8, 32), blocks(L.Np, 32));
    k_grad_prep<<<gz, tb, 0, st_>>>(R, R8, L.Np, dZ, mask, gb16_, gbT_, L.has_bias ? L.gb : nullptr);
    dim3 gx(blocks(R8, 32), blocks(L.K, 32));
    k_transpose<<<gx, tb, 0, st_>>>(R, R8, L.K, X, xT_);
    // dW^T [Np x K] = dZ^T [Np x R] * X [R x K]
    const int splits = std::max(1, std::min(64, R8 / 8192));
    gemm(gbT_, R8, xT_, R8, L.Np, L.K, R8, L.gWt, nullptr, L.K, nullptr, false, splits);
    // dX [R x K] = dZ [R x Np] * W^T
    if (dX) gemm(gb16_, L.Np, L.W16, L.Np, R, L.K, L.Np, dX, nullptr, L.K, nullptr, false);
}

void Surrogate::mlp_bwd(int first, const __nv_bfloat16* X, int R, const __nv_bfloat16* A1,
                        const __nv_bfloat16* A2, float* dY, float* dX) {
    // dY [R x Np2] -> dA2 (dT1) -> masked by A2 -> dA1 (dT2) -> masked by A1 -> dX
    float* t1 = R <= g_.n ? dT1_ : dE2_;
    float* t2 = R <= g_.n ? dT2_ : dE_;
    linear_bwd(layers_[first + 2], A2, R, dY, nullptr, t1);
    linear_bwd(layers_[first + 1], A1, R, t1, A2, t2);
    linear_bwd(layers_[first + 0], X, R, t2, A1, dX);
}

void Surrogate::adam(Linear& L, float lr) {
    const float c1 = 1.f / (1.f - std::pow(0.9f, (float)adam_t_));
    const float c2 = 1.f / (1.f - std::pow(0.999f, (float)adam_t_));
    const size_t nw = (size_t)L.Np * L.K;
    k_adam<<<blocks(nw, 256), 256, 0, st_>>>(nw, L.Wt, L.gWt, L.mW, L.vW, lr, c1, c2);
    if (L.has_bias) k_adam<<<blocks(L.Np, 256), 256, 0, st_>>>(L.Np, L.b, L.gb, L.mb, L.vb, lr, c1, c2);
    refresh_bf16(L);
}

float Surrogate::train_step(float lr) {
    forward(true);
    const int n = g_.n, E = g_.E;
    const size_t nW = (size_t)n * kWidth;
    std::vector<uint8_t> fl(n);
    cu(cudaMemcpyAsync(fl.data(), g_.fluid, n, cudaMemcpyDeviceToHost, st_), "fluid");
    cu(cudaMemsetAsync(loss_, 0, 4, st_), "memset");
    for (Linear& L : layers_) cu(cudaMemsetAsync(L.gb, 0, (size_t)L.Np * 4, st_), "memset");
    cu(cudaStreamSynchronize(st_), "fluid");
    int nf = 0;
    for (uint8_t v : fl) nf += v ? 1 : 0;
    k_loss<<<blocks(n, 256), 256, 0, st_>>>(n, Y_, target_, g_.fluid, 1.f / (float)std::max(nf, 1), dY_, loss_);
    mlp_bwd(19, hb_[2], n, da1_, da2_, dY_, dH_);
    for (int l = 1; l >= 0; --l) {
        const int base = 3 + 8 * l;
        k_mask_rows<<<blocks(nW, 256), 256, 0, st_>>>(n, dH_, g_.fluid, U_);
        mlp_bwd(base + 5, xn_[l], n, na1_[l], na2_[l], U_, dXN_);
        k_split_dxn<<<blocks(nW, 256), 256, 0, st_>>>(n, dH_, dXN_, kAggScale, dHp_, A_);
        if (E > 0) {
            const size_t eW = (size_t)E * kWidth;
            k_gather_rows<<<blocks(eW, 256), 256, 0, st_>>>(E, g_.dst, A_, M_);
            linear_bwd(layers_[base + 4], eh2_[l], E, M_, nullptr, dE2_);
            linear_bwd(layers_[base + 3], eh1_[l], E, dE2_, eh2_[l], dE_);
            linear_bwd(layers_[base + 2], g_.xe, E, dE_, eh1_[l], nullptr);  // masks dE_ to dZ1
            k_segsum<<<blocks((size_t)n * 32, 256), 256, 0, st_>>>(n, g_.row, dE_, 1.f, dP_);
            cu(cudaMemsetAsync(dQ_, 0, nW * 4, st_), "memset");
            k_scatter_add<<<blocks(eW, 256), 256, 0, st_>>>(E, g_.src, dE_, dQ_);
            linear_bwd(layers_[base + 0], hb_[l], n, dP_, nullptr, dT1_);
            k_add<<<blocks(nW, 256), 256, 0, st_>>>(nW, dHp_, dT1_);
            linear_bwd(layers_[base + 1], hb_[l], n, dQ_, nullptr, dT1_);
            k_add<<<blocks(nW, 256), 256, 0, st_>>>(nW, dHp_, dT1_);
        } else {
            for (int k = 0; k < 5; ++k) {
                Linear& L = layers_[base + k];
                cu(cudaMemsetAsync(L.gWt, 0, (size_t)L.Np * L.K * 4, st_), "memset");
            }
        }
        std::swap(dH_, dHp_);
    }
    mlp_bwd(0, g_.f, n, enc_a1_, enc_a2_, dH_, nullptr);
    if (lr > 0.f) {
        ++adam_t_;
        for (Linear& L : layers_) adam(L, lr);
    }
    float loss = 0.f;
    cu(cudaMemcpyAsync(&loss, loss_, 4, cudaMemcpyDeviceToHost, st_), "loss");
    cu(cudaStreamSynchronize(st_), "train");
    cu(cudaGetLastError(), "train");
    return loss;
}

void Surrogate::set_graph(int n, int E, const int* row, const int* src, const float* f, const float* xe,
                          const uint8_t* fluid) {
    ensure_graph(n, E);
    std::vector<int> dst(E);
    for (int i = 0; i < n; ++i)
        for (int e = row[i]; e < row[i + 1]; ++e) dst[e] = i;
    std::vector<__nv_bfloat16> fb((size_t)n * kNodeFeat), xb((size_t)E * kEdgeFeat);
    for (size_t i = 0; i < fb.size(); ++i) fb[i] = __float2bfloat16_rn(f[i]);
    for (size_t i = 0; i < xb.size(); ++i) xb[i] = __float2bfloat16_rn(xe[i]);
    cu(cudaMemcpyAsync(g_.row, row, (size_t)(n + 1) * 4, cudaMemcpyHostToDevice, st_), "graph");
    if (E) {
        cu(cudaMemcpyAsync(g_.src, src, (size_t)E * 4, cudaMemcpyHostToDevice, st_), "graph");
        cu(cudaMemcpyAsync(g_.dst, dst.data(), (size_t)E * 4, cudaMemcpyHostToDevice, st_), "graph");
        cu(cudaMemcpyAsync(g_.xe, xb.data(), xb.size() * 2, cudaMemcpyHostToDevice, st_), "graph");
    }
    cu(cudaMemcpyAsync(g_.f, fb.data(), fb.size() * 2, cudaMemcpyHostToDevice, st_), "graph");
    cu(cudaMemcpyAsync(g_.fluid, fluid, (size_t)n, cudaMemcpyHostToDevice, st_), "graph");
    cu(cudaStreamSynchronize(st_), "graph");
}

void Surrogate::set_targets(const float* t) {
    cu(cudaMemcpyAsync(target_, t, (size_t)g_.n * kOut * 4, cudaMemcpyHostToDevice, st_), "targets");
    cu(cudaStreamSynchronize(st_), "targets");
}

uint32_t Surrogate::device_error() {
    uint32_t e = 0;
    cu(cudaMemcpyAsync(&e, err_, 4, cudaMemcpyDeviceToHost, st_), "err");
    cu(cudaStreamSynchronize(st_), "err");
    return e;
}

}  // namespace pe
