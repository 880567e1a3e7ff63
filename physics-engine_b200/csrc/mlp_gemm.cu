// BF16 GEMM on the 5th-generation tensor cores (tcgen05), the building block of
// the learned surrogate's MLP layers:
//
//   C[M x N] = A[M x K] * Bt[N x K]^T (+ bias[N]) (ReLU optional)
//
// A and Bt are row-major bf16 with K contiguous ("K-major" operands), C is
// fp32 and/or bf16. One CTA computes a 128 x 128 tile of C: 64-wide K slices
// of A and Bt are staged in shared memory in the 128-byte-swizzled K-major
// layout (8-row atoms of 1024 bytes, 16-byte chunk c of row r stored at chunk
// c ^ (r & 7)), two stages deep; one thread issues the four K=16
// `tcgen05.mma.kind::f16` of a slice with the fp32 accumulator in tensor
// memory (128 lanes x 128 columns) and commits them to the stage's mbarrier,
// which frees the stage for the next-but-one slice. The epilogue reads the
// accumulator with `tcgen05.ld` (warp w owns lanes 32w..32w+31, i.e. rows
// 32w..32w+31 of the tile). With gridDim.z > 1 the K range is split and each
// split writes its own fp32 partial (summed by launch_gemm_reduce).
//
// Every mbarrier wait is bounded; a wait that runs out sets bit 0 of *err, and
// the kernel still waits (bounded) for its committed MMAs before freeing its
// tensor memory and returning.
#include <cuda_bf16.h>
#include <cstdint>

#include "mlp.cuh"
#include "umma.cuh"

namespace pe {

namespace {

using namespace umma;

constexpr int kBM = kTileM, kBN = kTileN, kBK = 64;
constexpr int kGemmThreads = 128;
constexpr uint32_t kOperandBytes = kBM * kBK * 2;  // 16 KB: one operand, one stage

// One 128-row x 64-column bf16 slice of a K-major operand into the swizzled
// layout; rows >= rows_valid and columns >= k_valid read as zero.
__device__ __forceinline__ void load_slice(uint8_t* dst, const __nv_bfloat16* __restrict__ src, int ld,
                                           int row0, int rows_valid, int k0, int k_valid) {
    for (int i = threadIdx.x; i < kBM * 8; i += kGemmThreads) {
        const int r = i >> 3, c = i & 7;
        const int row = row0 + r, col = k0 + c * 8;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (row < rows_valid && col < k_valid)  // k_valid and ld are multiples of 8
            v = __ldg(reinterpret_cast<const uint4*>(src + (size_t)row * ld + col));
        *reinterpret_cast<uint4*>(dst + r * 128 + ((c ^ (r & 7)) << 4)) = v;
    }
}

__global__ void __launch_bounds__(kGemmThreads) k_gemm_bf16(GemmArgs g) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t mbar[3];
    __shared__ uint32_t s_tmem;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
    const int nk_all = (g.K + kBK - 1) / kBK;
    const int per = (nk_all + (int)gridDim.z - 1) / (int)gridDim.z;
    const int kt0 = (int)blockIdx.z * per, kt1 = min(nk_all, kt0 + per);

    if (tid == 0) {
        for (int i = 0; i < 3; ++i) mbar_init(smem_addr(&mbar[i]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                     "r"(128u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    bool ok = true;
    uint32_t phase[2] = {0u, 0u};
    uint32_t issued[2] = {0u, 0u};
    for (int kt = kt0; kt < kt1; ++kt) {
        const int s = (kt - kt0) & 1;
        if (issued[s]) {  // the MMAs that last read this stage must be done
            ok = mbar_wait(smem_addr(&mbar[s]), phase[s]) && ok;
            phase[s] ^= 1u;
            issued[s] = 0u;
        }
        uint8_t* sA = smem + (uint32_t)s * kOperandBytes;        // stages of A, then of Bt
        uint8_t* sB = smem + (uint32_t)(2 + s) * kOperandBytes;
        load_slice(sA, g.A, g.lda, m0, g.M, kt * kBK, g.K);
        load_slice(sB, g.Bt, g.ldb, n0, g.N, kt * kBK, g.K);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sB);
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk)
                umma_bf16(tmem, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32),
                          (kt > kt0 || kk > 0) ? 1u : 0u);
            umma_commit(smem_addr(&mbar[s]));
        }
        issued[s] = 1u;
    }
    // all committed MMAs complete before the accumulator is read
    if (tid == 0) umma_commit(smem_addr(&mbar[2]));
    const bool have = kt1 > kt0;
    ok = (have ? mbar_wait(smem_addr(&mbar[2]), 0u) : true) && ok;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // Epilogue: the accumulator goes through shared memory (the operand stages
    // are free once every MMA has completed) so that each warp then stores
    // whole 512-byte rows. Row r's 4-float chunk q sits at chunk q ^ (r & 31):
    // the row-per-lane writes and the chunk-per-lane reads both spread over
    // all banks.
    const bool split = gridDim.z > 1;  // raw fp32 partials, summed by k_reduce_splits
    const size_t part = (size_t)blockIdx.z * (size_t)g.M * (size_t)g.ldc;
    float4* stile = reinterpret_cast<float4*>(smem);  // 128 rows x 32 chunks
    {
        const int r = warp * 32 + lane;
#pragma unroll 1
        for (int cb = 0; cb < kBN / 32; ++cb) {
            uint32_t v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 32), v);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int q = cb * 8 + j;
                stile[r * 32 + (q ^ (r & 31))] =
                    have ? make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]),
                                       __uint_as_float(v[4 * j + 2]), __uint_as_float(v[4 * j + 3]))
                         : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
    }
    __syncthreads();
    const int col = n0 + lane * 4;
    const bool vec = (g.ldc & 3) == 0 && col + 3 < g.N;
#pragma unroll 1
    for (int r = warp; r < kBM; r += kGemmThreads / 32) {
        const int row = m0 + r;
        if (row >= g.M || col >= g.N) continue;
        const float4 c4 = stile[r * 32 + (lane ^ (r & 31))];
        float v[4] = {c4.x, c4.y, c4.z, c4.w};
        if (!split) {
            const float* a0 = g.add0 ? g.add0 + (size_t)g.idx0[row] * g.ld_add : nullptr;
            const float* a1 = g.add1 ? g.add1 + (size_t)g.idx1[row] * g.ld_add : nullptr;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (col + i >= g.N) break;
                if (g.bias) v[i] += g.bias[col + i];
                if (a0) v[i] += a0[col + i];
                if (a1) v[i] += a1[col + i];
                if (g.relu) v[i] = fmaxf(v[i], 0.f);
            }
        }
        if (vec) {
            if (g.Cf) *reinterpret_cast<float4*>(g.Cf + part + (size_t)row * g.ldc + col) = make_float4(v[0], v[1], v[2], v[3]);
            if (g.Cb && !split) {
                __nv_bfloat162 lo = __floats2bfloat162_rn(v[0], v[1]), hi = __floats2bfloat162_rn(v[2], v[3]);
                uint2 packed = make_uint2(*reinterpret_cast<uint32_t*>(&lo), *reinterpret_cast<uint32_t*>(&hi));
                *reinterpret_cast<uint2*>(g.Cb + (size_t)row * g.ldc + col) = packed;
            }
        } else {
            for (int i = 0; i < 4 && col + i < g.N; ++i) {
                if (g.Cf) g.Cf[part + (size_t)row * g.ldc + col + i] = v[i];
                if (g.Cb && !split) g.Cb[(size_t)row * g.ldc + col + i] = __float2bfloat16_rn(v[i]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u) : "memory");
    }
    if (!ok && tid == 0) atomicOr(g.err, 1u);
}

__global__ void k_reduce_splits(int M, int N, int ldc, int splits, const float* __restrict__ part,
                                const float* __restrict__ bias, int relu, float* __restrict__ Cf,
                                __nv_bfloat16* __restrict__ Cb) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)M * N) return;
    const int row = (int)(i / N), col = (int)(i % N);
    float v = 0.f;
    for (int s = 0; s < splits; ++s) v += part[(size_t)s * M * ldc + (size_t)row * ldc + col];
    if (bias) v += bias[col];
    if (relu) v = fmaxf(v, 0.f);
    if (Cf) Cf[(size_t)row * ldc + col] = v;
    if (Cb) Cb[(size_t)row * ldc + col] = __float2bfloat16_rn(v);
}

}  // namespace

size_t gemm_smem_bytes() { return 4 * (size_t)kOperandBytes + 1024; }

bool gemm_prepare() {
    return cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)gemm_smem_bytes()) == cudaSuccess;
}

void launch_gemm(const GemmArgs& g, int splits, cudaStream_t st) {
    if (g.M <= 0 || g.N <= 0) return;
    dim3 grid((g.M + kBM - 1) / kBM, (g.N + kBN - 1) / kBN, splits > 0 ? splits : 1);
    k_gemm_bf16<<<grid, kGemmThreads, gemm_smem_bytes(), st>>>(g);
}

void launch_gemm_reduce(int M, int N, int ldc, int splits, const float* part, const float* bias, int relu,
                        float* Cf, __nv_bfloat16* Cb, cudaStream_t st) {
    const size_t n = (size_t)M * N;
    if (!n) return;
    k_reduce_splits<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(M, N, ldc, splits, part, bias, relu, Cf, Cb);
}

}  // namespace pe

// ---------------------------------------------------------------- C ABI
namespace {
__device__ uint32_t g_gemm_err;
}

// Runs one GEMM on the caller's device buffers (see pe::GemmArgs) on `stream`
// and waits for it; returns 0, or 7 (device error) with *err = the kernel's
// wait-timeout flag. part (splits * M * ldc floats) is needed when splits > 1.
extern "C" __attribute__((visibility("default"))) int pe_mlp_gemm_bf16(
    const void* A, const void* Bt, float* Cf, void* Cb, const float* bias, int M, int N, int K, int lda,
    int ldb, int ldc, int relu, int splits, float* part, void* stream, uint32_t* err) {
    using namespace pe;
    if (!A || !Bt || (!Cf && !Cb) || M < 0 || N < 0 || K <= 0 || K % 8 || lda % 8 || ldb % 8 || ldc < N ||
        lda < K || ldb < K)
        return 3;
    if (splits > 1 && !part) return 1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t zero = 0;
    if (cudaMemcpyToSymbolAsync(g_gemm_err, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return 7;
    uint32_t* derr = nullptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&derr), g_gemm_err) != cudaSuccess || !gemm_prepare())
        return 7;
    GemmArgs g{static_cast<const __nv_bfloat16*>(A), static_cast<const __nv_bfloat16*>(Bt),
               splits > 1 ? part : Cf, splits > 1 ? nullptr : static_cast<__nv_bfloat16*>(Cb), bias,
               M, N, K, lda, ldb, ldc, relu, derr};
    launch_gemm(g, splits, st);
    if (splits > 1) launch_gemm_reduce(M, N, ldc, splits, part, bias, relu, Cf, static_cast<__nv_bfloat16*>(Cb), st);
    uint32_t h = 0;
    if (cudaMemcpyFromSymbolAsync(&h, g_gemm_err, sizeof(h), 0, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return 7;
    if (err) *err = h;
    return h ? 7 : 0;
}
