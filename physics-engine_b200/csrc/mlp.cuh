// Learned surrogate: tensor-core GEMM building block, the fused edge MLP and
// the message-passing network kernels (mlp_gemm.cu, edge_fused.cu, surrogate.cu).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace pe {

// C[M x N] = A[M x K] * Bt[N x K]^T (+ bias) (ReLU if relu), bf16 operands with
// K contiguous, fp32 accumulation. K, lda and ldb are multiples of 8. Cf (fp32)
// and Cb (bf16) may each be null; with split-K the fp32 partials of split z are
// written at Cf + z * M * ldc and bias / ReLU / Cb are applied by
// launch_gemm_reduce.
struct GemmArgs {
    const __nv_bfloat16* A;
    const __nv_bfloat16* Bt;
    float* Cf;
    __nv_bfloat16* Cb;
    const float* bias;
    int M, N, K, lda, ldb, ldc, relu;
    uint32_t* err;  // bit 0: a bounded wait ran out
    // optional gathered addends, added after the bias and before the ReLU:
    // C[r][c] += add0[idx0[r] * ld_add + c] + add1[idx1[r] * ld_add + c]
    const float* add0 = nullptr;
    const int* idx0 = nullptr;
    const float* add1 = nullptr;
    const int* idx1 = nullptr;
    int ld_add = 0;
};

// One hop's edge MLP fused into one persistent kernel (edge_fused.cu), for
// inference: out[dst[e]] += relu(relu(x_e Wc + b1 + P[dst[e]] + Q[src[e]]) W2
// + b2) W3 + b3 over the E edges (sorted by destination); out [n x 128] must
// be zero. P, Q fp32 [n x 128]; x_e bf16 [E x 16]; Wc, W2, W3 bf16 K-major
// ([128 x 16], [128 x 128], [128 x 128]).
struct EdgeHopArgs {
    int E;
    const int* src;
    const int* dst;
    const __nv_bfloat16* xe;
    const float* P;
    const float* Q;
    const __nv_bfloat16* Wc;
    const float* b1;
    const __nv_bfloat16* W2;
    const float* b2;
    const __nv_bfloat16* W3;
    const float* b3;
    float* out;
    uint32_t* err;  // bit 0: a bounded wait ran out
};
bool edge_hop_prepare();
void launch_edge_hop(const EdgeHopArgs& a, int sms, cudaStream_t st);

size_t gemm_smem_bytes();
bool gemm_prepare();
void launch_gemm(const GemmArgs& g, int splits, cudaStream_t st);
void launch_gemm_reduce(int M, int N, int ldc, int splits, const float* part, const float* bias, int relu,
                        float* Cf, __nv_bfloat16* Cb, cudaStream_t st);

}  // namespace pe
