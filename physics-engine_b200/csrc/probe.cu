// FP64 issue-rate probe: the denominator of the step's FP64 roofline. The
// step's f64 passes compile without contraction (separate DMUL and DADD, as
// the reference's no-FMA policy requires), so the attainable rate is that of
// independent non-fused multiplies and adds, measured here on the live device.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/pe_fluid_wcsph.h"

namespace {

constexpr int kChains = 8;

__global__ void k_fp64_issue(double* out, uint32_t iters, double m, double c) {
    double a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = 1.0 + 1e-3 * (double)(threadIdx.x + k);
    for (uint32_t it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = __dadd_rn(__dmul_rn(a[k], m), c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k];
    if (s == 12345.678) out[0] = s;  // keeps the chains live
}

}  // namespace

extern "C" int pe_fluid_probe_fp64_rate(int32_t device, double* gops) {
    if (!gops) return PE_ERR_NULL;
    *gops = 0.0;
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return PE_ERR_DEVICE;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return PE_ERR_DEVICE;
    double* out = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    int rc = PE_ERR_DEVICE;
    if (cudaMalloc(&out, sizeof(double)) == cudaSuccess && cudaStreamCreate(&st) == cudaSuccess &&
        cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess) {
        const uint32_t threads = 256, blocks = (uint32_t)sms * 8, iters = 1u << 14;
        k_fp64_issue<<<blocks, threads, 0, st>>>(out, 64, 0.999999, 1e-7);  // warm-up
        cudaEventRecord(a, st);
        k_fp64_issue<<<blocks, threads, 0, st>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(b, st);
        float ms = 0.0f;
        if (cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess &&
            ms > 0.0f) {
            const double ops = (double)blocks * threads * iters * kChains * 2.0;
            *gops = ops / ((double)ms * 1e-3) / 1e9;
            rc = PE_OK;
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (st) cudaStreamDestroy(st);
    if (out) cudaFree(out);
    cudaGetLastError();
    return rc;
}
