// Fused edge MLP of one message-passing hop, for inference (the learned
// step): for every edge e = (i <- j) of the message graph (edges sorted by
// destination)
//
//   z1  = relu(x_e Wc + b1 + P[i] + Q[j])      P = h Wa, Q = h Wb (per node)
//   z2  = relu(z1 W2 + b2)
//   m_e = z2 W3 + b3
//   out[i] += m_e
//
// which the unfused path computes as three GEMM launches writing E x 128
// activations to memory (~60 GB of traffic per hop at 3.3e7 edges) and a
// segment sum. Here one persistent CTA per SM keeps Wc, W2 and W3 in shared
// memory and walks tiles of 128 edges: x_e W c is one K=16 tcgen05 MMA into
// the tensor-memory accumulator; the epilogue (thread r = edge r = TMEM lane
// r) adds b1, P[i] and Q[j] in the unfused epilogue's order, applies ReLU and
// writes bf16 into a swizzled shared-memory tile that is the A operand of
// the next 8 MMAs (K = 128), and so on; the last epilogue stages the
// messages in shared memory and sums each run of equal destinations before
// one atomic add per run and column. Activations are rounded to bf16 at the
// same points as in the unfused path; only the message sum's order differs.
//
// Every mbarrier wait is bounded; a wait that runs out sets bit 0 of *err and
// ends the tile loop of the whole CTA (at the tile's end, by a block-wide
// vote), and the CTA still waits (bounded) for its committed MMAs before
// freeing its tensor memory.
#include <cuda_bf16.h>
#include <cstdint>

#include "mlp.cuh"
#include "umma.cuh"

namespace pe {

namespace {

using namespace umma;

constexpr int kEdgeThreads = 128;        // one thread per edge of a tile (TMEM lane)
constexpr uint32_t kSlice = 128u * 128u;  // bytes of a 128-row x 64-column bf16 slice
constexpr uint32_t kOffWc = 0;                    // Wc^T [128 x 16]: chunks 0-1 of one slice
constexpr uint32_t kOffW2 = kOffWc + kSlice;      // W2^T [128 x 128]: two slices
constexpr uint32_t kOffW3 = kOffW2 + 2 * kSlice;  // W3^T: two slices
constexpr uint32_t kOffX = kOffW3 + 2 * kSlice;   // edge features [128 x 16]: chunks 0-1
constexpr uint32_t kOffA = kOffX + kSlice;        // activations [128 x 128]: two slices
constexpr uint32_t kOffStage = kOffA + 2 * kSlice;  // fp32 messages, 128 rows x 32 columns
constexpr uint32_t kStageLd = 33;                   // padded row (conflict-free both ways)
constexpr uint32_t kSmemBytes = kOffStage + 128u * kStageLd * 4u + 1024u;  // + alignment slack

__device__ __forceinline__ uint32_t sw_off(int row, int chunk) {
    return (uint32_t)row * 128u + ((uint32_t)(chunk ^ (row & 7)) << 4);
}

// Rows 0..127 of a K-major bf16 matrix (row length ld) into swizzled slices:
// 16-byte chunk c of row r goes to slice c / 8, chunk c % 8.
__device__ void stage_rows(uint8_t* dst, const __nv_bfloat16* __restrict__ src, int ld, int chunks) {
    for (int i = threadIdx.x; i < 128 * chunks; i += blockDim.x) {
        const int r = i / chunks, c = i % chunks;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(src + (size_t)r * ld + c * 8));
        *reinterpret_cast<uint4*>(dst + (uint32_t)(c >> 3) * kSlice + sw_off(r, c & 7)) = v;
    }
}

// 32 fp32 values (columns 32 cb .. 32 cb + 31 of row r) into the bf16 activation tile
__device__ __forceinline__ void put_bf16_row(uint8_t* sA, int r, int cb, const float (&x)[32]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t w[4];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            __nv_bfloat162 b = __floats2bfloat162_rn(x[q * 8 + 2 * h], x[q * 8 + 2 * h + 1]);
            w[h] = *reinterpret_cast<uint32_t*>(&b);
        }
        const int cidx = cb * 4 + q;  // 16-byte chunk of the 128-column row
        *reinterpret_cast<uint4*>(sA + (uint32_t)(cidx >> 3) * kSlice + sw_off(r, cidx & 7)) =
            make_uint4(w[0], w[1], w[2], w[3]);
    }
}

__device__ __forceinline__ void issue_k128(uint32_t tmem, const uint8_t* sA, const uint8_t* sW) {
    const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sW);
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
            umma_bf16(tmem, sw128_desc(a0 + (uint32_t)s * kSlice + kk * 32),
                      sw128_desc(b0 + (uint32_t)s * kSlice + kk * 32), (s | kk) ? 1u : 0u);
}

__global__ void __launch_bounds__(kEdgeThreads) k_edge_hop(EdgeHopArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    uint8_t* sWc = smem + kOffWc;
    uint8_t* sW2 = smem + kOffW2;
    uint8_t* sW3 = smem + kOffW3;
    uint8_t* sX = smem + kOffX;
    uint8_t* sA = smem + kOffA;
    float* sStage = reinterpret_cast<float*>(smem + kOffStage);
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_dst[kEdgeThreads];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        mbar_init(smem_addr(&mbar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                     "r"(128u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // the weights stay in shared memory for every tile of the CTA
    stage_rows(sWc, a.Wc, 16, 2);
    stage_rows(sW2, a.W2, 128, 16);
    stage_rows(sW3, a.W3, 128, 16);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's lanes

    bool ok = true;
    uint32_t phase = 0u;
    auto mma_wait = [&]() {
        const bool done = mbar_wait(smem_addr(&mbar), phase);
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        return done;
    };
    auto to_tensor = [&]() {  // generic-proxy shared writes visible to the MMAs, TMEM reads done
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    };
    const int ntiles = (a.E + kEdgeThreads - 1) / kEdgeThreads;
    // This thread's edge (row tid) of a tile: endpoints and its two 16-byte
    // chunks of edge features, loaded one tile ahead.
    auto fetch_edge = [&](int tile, int& d, int& sj, uint4& x0, uint4& x1) {
        const int e = tile * kEdgeThreads + tid;
        d = -1;
        sj = -1;
        x0 = x1 = make_uint4(0u, 0u, 0u, 0u);
        if (tile < ntiles && e < a.E) {
            d = __ldg(a.dst + e);
            sj = __ldg(a.src + e);
            x0 = __ldg(reinterpret_cast<const uint4*>(a.xe + (size_t)e * 16));
            x1 = __ldg(reinterpret_cast<const uint4*>(a.xe + (size_t)e * 16 + 8));
        }
    };
    // 32 columns (block cb) of this edge's P[dst] and Q[src] rows
    auto fetch_pq = [&](int d, int sj, int cb, float4 (&p)[8], float4 (&q)[8]) {
        const float4* P4 = reinterpret_cast<const float4*>(a.P + (size_t)(d < 0 ? 0 : d) * 128 + cb * 32);
        const float4* Q4 = reinterpret_cast<const float4*>(a.Q + (size_t)(sj < 0 ? 0 : sj) * 128 + cb * 32);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            p[i] = __ldg(P4 + i);
            q[i] = __ldg(Q4 + i);
        }
    };
    int d, sj;
    uint4 x0, x1;
    fetch_edge(blockIdx.x, d, sj, x0, x1);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        // ---- edge features and endpoints of the tile (fetched a tile ahead)
        s_dst[tid] = d;
        *reinterpret_cast<uint4*>(sX + sw_off(tid, 0)) = x0;
        *reinterpret_cast<uint4*>(sX + sw_off(tid, 1)) = x1;
        const int dc = d, sc = sj;
        to_tensor();
        // ---- layer 1: x_e Wc (one K = 16 MMA), then + b1 + P[dst] + Q[src], ReLU
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            umma_bf16(tmem, sw128_desc(smem_addr(sX)), sw128_desc(smem_addr(sWc)), 0u);
            umma_commit(smem_addr(&mbar));
        }
        // the next tile's edge and this edge's first P/Q block load while the MMA runs
        fetch_edge(tile + gridDim.x, d, sj, x0, x1);
        float4 pa[8], qa[8];
        fetch_pq(dc, sc, 0, pa, qa);
        ok = mma_wait() && ok;
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
            float4 pb[8], qb[8];
            if (cb < 3) fetch_pq(dc, sc, cb + 1, pb, qb);  // one block ahead
            uint32_t v[32];
            tmem_ld32(trow + (uint32_t)(cb * 32), v);
            float x[32];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float pv[4] = {pa[i].x, pa[i].y, pa[i].z, pa[i].w};
                const float qv[4] = {qa[i].x, qa[i].y, qa[i].z, qa[i].w};
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const int j = i * 4 + h;
                    float t = __uint_as_float(v[j]) + a.b1[cb * 32 + j];  // the unfused epilogue's order
                    t += pv[h];
                    t += qv[h];
                    x[j] = fmaxf(t, 0.f);
                }
            }
            put_bf16_row(sA, tid, cb, x);
            if (cb < 3) {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    pa[i] = pb[i];
                    qa[i] = qb[i];
                }
            }
        }
        to_tensor();
        // ---- layer 2: relu(z1 W2 + b2)
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            issue_k128(tmem, sA, sW2);
            umma_commit(smem_addr(&mbar));
        }
        ok = mma_wait() && ok;
#pragma unroll 1
        for (int cb = 0; cb < 4; ++cb) {
            uint32_t v[32];
            tmem_ld32(trow + (uint32_t)(cb * 32), v);
            float x[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) x[j] = fmaxf(__uint_as_float(v[j]) + a.b2[cb * 32 + j], 0.f);
            put_bf16_row(sA, tid, cb, x);  // the MMAs that read sA have completed
        }
        to_tensor();
        // ---- layer 3: m_e = z2 W3 + b3, summed per destination
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            issue_k128(tmem, sA, sW3);
            umma_commit(smem_addr(&mbar));
        }
        ok = mma_wait() && ok;
#pragma unroll 1
        for (int cb = 0; cb < 4; ++cb) {
            uint32_t v[32];
            tmem_ld32(trow + (uint32_t)(cb * 32), v);
#pragma unroll
            for (int j = 0; j < 32; ++j) sStage[tid * kStageLd + j] = __uint_as_float(v[j]) + a.b3[cb * 32 + j];
            __syncthreads();
            // thread (group g, column j): rows 32 g .. 32 g + 31, one atomic per run of a destination
            const int j = lane, g = warp;
            int cur = -1;
            float acc = 0.f;
            for (int rr = 0; rr < 32; ++rr) {
                const int row = g * 32 + rr, d = s_dst[row];
                if (d < 0) break;  // rows past the last edge close the tile
                if (d != cur) {
                    if (cur >= 0) atomicAdd(a.out + (size_t)cur * 128 + cb * 32 + j, acc);
                    cur = d;
                    acc = 0.f;
                }
                acc += sStage[row * kStageLd + j];
            }
            if (cur >= 0) atomicAdd(a.out + (size_t)cur * 128 + cb * 32 + j, acc);
            __syncthreads();  // the staging buffer is reused by the next column block
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        // the tile's TMEM reads and shared-memory use end before the next
        // tile; a run-out wait on any thread stops every thread (a decision
        // all threads share, so none is left at a barrier)
        ok = __syncthreads_and(ok ? 1 : 0) != 0;
        if (!ok) break;
    }
    // every committed MMA completes before the tensor memory is freed
    if (tid == 0) umma_commit(smem_addr(&mbar));
    ok = mma_wait() && ok;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u) : "memory");
    }
    if (!ok && tid == 0) atomicOr(a.err, 1u);
}

}  // namespace

bool edge_hop_prepare() {
    return cudaFuncSetAttribute(k_edge_hop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes) ==
           cudaSuccess;
}

void launch_edge_hop(const EdgeHopArgs& a, int sms, cudaStream_t st) {
    if (a.E <= 0) return;
    const int ntiles = (a.E + kEdgeThreads - 1) / kEdgeThreads;
    const int grid = ntiles < sms ? ntiles : sms;
    k_edge_hop<<<grid, kEdgeThreads, kSmemBytes, st>>>(a);
}

}  // namespace pe
