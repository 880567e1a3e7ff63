// Learned surrogate: tensor-core GEMM building block and the message-passing
// network kernels (mlp_gemm.cu, surrogate.cu).
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

size_t gemm_smem_bytes();
bool gemm_prepare();
void launch_gemm(const GemmArgs& g, int splits, cudaStream_t st);
void launch_gemm_reduce(int M, int N, int ldc, int splits, const float* part, const float* bias, int relu,
                        float* Cf, __nv_bfloat16* Cb, cudaStream_t st);

}  // namespace pe
