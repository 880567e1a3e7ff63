// Device probes.
//
// FP64 issue rate: the denominator of the step's FP64 roofline. The step's f64
// passes compile without contraction (separate DMUL and DADD, as the
// reference's no-FMA policy requires), so the attainable rate is that of
// independent non-fused multiplies and adds, measured here on the live device.
//
// Phase overhead: what separating two grid-wide phases costs as a kernel node
// of a replayed CUDA graph (the batched step's form) and as a grid-wide
// barrier inside one cooperative persistent kernel (the alternative). The
// barrier is this file's own, with a bounded wait that raises an error flag.
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

constexpr uint32_t kPhaseThreads = 256;
constexpr long long kBarrierSpinLimit = 1ll << 22;  // x ~64 ns: a bounded wait of ~0.3 s

// One phase's token work: each thread bumps its own word.
__device__ __forceinline__ void phase_work(uint32_t* buf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    buf[i] += 1u;
}

__global__ void k_phase_node(uint32_t* buf) { phase_work(buf); }

// Grid-wide barrier for a cooperative launch: the last block to arrive resets
// the count and advances the generation; the others wait for the generation
// to change, for a bounded number of polls, after which they set *err.
__device__ __forceinline__ void grid_barrier(uint32_t* count, volatile uint32_t* gen, uint32_t nblocks,
                                             uint32_t* err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t g = *gen;
        __threadfence();
        if (atomicAdd(count, 1u) == nblocks - 1u) {
            *count = 0u;
            __threadfence();
            atomicAdd(const_cast<uint32_t*>(gen), 1u);
        } else {
            long long it = 0;
            while (*gen == g) {
                if (++it > kBarrierSpinLimit) {
                    atomicOr(err, 1u);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

__global__ void k_phase_persistent(uint32_t* buf, uint32_t phases, uint32_t* bar, uint32_t* err) {
    for (uint32_t p = 0; p < phases; ++p) {
        phase_work(buf);
        grid_barrier(bar, bar + 1, gridDim.x, err);
        if (*(volatile uint32_t*)err) return;
    }
}

}  // namespace

extern "C" int pe_fluid_probe_phase_overhead(int32_t device, uint32_t phases, double* node_us,
                                             double* barrier_us) {
    if (!node_us || !barrier_us) return PE_ERR_NULL;
    if (phases < 2 || phases > 4096) return PE_ERR_ARG;
    *node_us = *barrier_us = 0.0;
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return PE_ERR_DEVICE;
    int dev = 0, sms = 0, coop = 0, occ = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_phase_persistent, kPhaseThreads, 0) != cudaSuccess)
        return PE_ERR_DEVICE;
    if (!coop || occ < 1) return PE_ERR_UNSUPPORTED;
    // every block co-resident (cooperative launch), a few per SM as the step's passes have
    const uint32_t blocks = (uint32_t)sms * (uint32_t)(occ < 4 ? occ : 4);
    constexpr int kReps = 50;
    uint32_t *buf = nullptr, *bar = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = PE_ERR_DEVICE;
    auto timed = [&](auto&& body, float* ms) {
        if (cudaEventRecord(a, st) != cudaSuccess) return false;
        body();
        return cudaEventRecord(b, st) == cudaSuccess && cudaEventSynchronize(b) == cudaSuccess &&
               cudaEventElapsedTime(ms, a, b) == cudaSuccess;
    };
    if (cudaMalloc(&buf, sizeof(uint32_t) * blocks * kPhaseThreads) == cudaSuccess &&
        cudaMalloc(&bar, sizeof(uint32_t) * 4) == cudaSuccess && cudaStreamCreate(&st) == cudaSuccess &&
        cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess &&
        cudaMemsetAsync(buf, 0, sizeof(uint32_t) * blocks * kPhaseThreads, st) == cudaSuccess &&
        cudaMemsetAsync(bar, 0, sizeof(uint32_t) * 4, st) == cudaSuccess) {
        // graph of `phases` kernel nodes
        bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            for (uint32_t p = 0; p < phases; ++p) k_phase_node<<<blocks, kPhaseThreads, 0, st>>>(buf);
            ok = cudaStreamEndCapture(st, &graph) == cudaSuccess &&
                 cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        }
        float ms_graph = 0.0f, ms_p = 0.0f, ms_1 = 0.0f;
        uint32_t* err = bar + 2;
        auto coop_launch = [&](uint32_t ph) {
            void* args[] = {&buf, &ph, &bar, &err};
            return cudaLaunchCooperativeKernel((const void*)k_phase_persistent, dim3(blocks), dim3(kPhaseThreads),
                                               args, 0, st) == cudaSuccess;
        };
        ok = ok && cudaGraphLaunch(exec, st) == cudaSuccess && coop_launch(phases);  // warm-up
        ok = ok && timed([&] {
            for (int r = 0; r < kReps; ++r) cudaGraphLaunch(exec, st);
        }, &ms_graph);
        ok = ok && timed([&] {
            for (int r = 0; r < kReps; ++r) coop_launch(phases);
        }, &ms_p);
        ok = ok && timed([&] {
            for (int r = 0; r < kReps; ++r) coop_launch(1);
        }, &ms_1);
        uint32_t herr = 1;
        ok = ok && cudaMemcpy(&herr, err, sizeof(uint32_t), cudaMemcpyDeviceToHost) == cudaSuccess;
        if (ok && herr == 0) {
            *node_us = 1e3 * (double)ms_graph / ((double)kReps * phases);
            *barrier_us = 1e3 * (double)(ms_p - ms_1) / ((double)kReps * (phases - 1));
            rc = PE_OK;
        }
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (st) cudaStreamDestroy(st);
    if (buf) cudaFree(buf);
    if (bar) cudaFree(bar);
    cudaGetLastError();
    return rc;
}

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
