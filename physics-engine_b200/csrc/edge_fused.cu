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
// memory; its two warpgroups walk their own tiles of 128 edges, each with its
// own 128 tensor-memory columns, buffers and barriers, so one group's MMA
// waits and gathers overlap the other's epilogues. Per tile, x_e Wc is one
// K=16 tcgen05 MMA into the group's accumulator; the epilogue (thread r =
// edge r = TMEM lane r) adds b1, P[i] and Q[j] in the unfused epilogue's
// order (the next tile's endpoints and features, and the next 32-column block
// of P[i] and Q[j], are already loading), applies ReLU and
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

constexpr int kGroups = 2;             // warpgroups per CTA, each on its own tiles
constexpr int kGroupThreads = 128;     // one thread per edge of a tile (TMEM lane)
constexpr int kEdgeThreads = kGroups * kGroupThreads;
constexpr uint32_t kSlice = 128u * 128u;  // bytes of a 128-row x 64-column bf16 slice
constexpr uint32_t kOffWc = 0;                    // Wc^T [128 x 16]: chunks 0-1 of one slice
constexpr uint32_t kOffW2 = kOffWc + kSlice;      // W2^T [128 x 128]: two slices
constexpr uint32_t kOffW3 = kOffW2 + 2 * kSlice;  // W3^T: two slices
constexpr uint32_t kOffGroup = kOffW3 + 2 * kSlice;
// per warpgroup: the edge-feature slice [128 x 16] (chunks 0-1), which the
// last epilogue reuses for the fp32 messages (128 rows x 32 columns, column
// j of row r at j ^ (r & 31)), then the activation tile [128 x 128]
constexpr uint32_t kGroupBytes = 3 * kSlice;
constexpr uint32_t kSmemBytes = kOffGroup + kGroups * kGroupBytes + 1024u;  // + alignment slack

__device__ __forceinline__ uint32_t sw_off(int row, int chunk) {
    return (uint32_t)row * 128u + ((uint32_t)(chunk ^ (row & 7)) << 4);
}

// barrier of warpgroup g alone (ids 1, 2; 0 is __syncthreads')
__device__ __forceinline__ void group_sync(int g) {
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(kGroupThreads) : "memory");
}
// the same barrier, returning whether v holds on every thread of the group
__device__ __forceinline__ bool group_all(int g, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(g + 1), "r"(kGroupThreads)
        : "memory");
    return r != 0;
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
    __shared__ __align__(8) uint64_t mbar[kGroups];
    __shared__ uint32_t s_tmem;
    __shared__ int s_dst[kGroups][kGroupThreads];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = tid / kGroupThreads, gt = tid % kGroupThreads, gw = gt >> 5;
    uint8_t* sWc = smem + kOffWc;
    uint8_t* sW2 = smem + kOffW2;
    uint8_t* sW3 = smem + kOffW3;
    uint8_t* sX = smem + kOffGroup + (uint32_t)g * kGroupBytes;
    float* sStage = reinterpret_cast<float*>(sX);  // free once the tile's first MMA completed
    uint8_t* sA = sX + kSlice;
    int* dstv = s_dst[g];

    if (tid == 0) {
        for (int i = 0; i < kGroups; ++i) mbar_init(smem_addr(&mbar[i]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                     "r"(128u * kGroups)
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
    const uint32_t tmem = s_tmem + 128u * (uint32_t)g;            // this group's 128 columns
    const uint32_t trow = tmem + ((uint32_t)(gw * 32) << 16);      // this warp's lanes (warp % 4)
    const uint32_t bar = smem_addr(&mbar[g]);

    bool ok = true;
    uint32_t phase = 0u;
    auto mma_wait = [&]() {
        const bool done = mbar_wait(bar, phase);
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        return done;
    };
    auto to_tensor = [&]() {  // generic-proxy shared writes visible to the MMAs, TMEM reads done
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        group_sync(g);
    };
    const int ntiles = (a.E + kGroupThreads - 1) / kGroupThreads;
    const int stride = (int)gridDim.x * kGroups;
    // This thread's edge (row gt) of a tile: endpoints and its two 16-byte
    // chunks of edge features, loaded one tile ahead.
    auto fetch_edge = [&](int tile, int& d, int& sj, uint4& x0, uint4& x1) {
        const int e = tile * kGroupThreads + gt;
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
    const int first = (int)blockIdx.x * kGroups + g;
    fetch_edge(first, d, sj, x0, x1);
    for (int tile = first; tile < ntiles; tile += stride) {
        // ---- edge features and endpoints of the tile (fetched a tile ahead)
        dstv[gt] = d;
        *reinterpret_cast<uint4*>(sX + sw_off(gt, 0)) = x0;
        *reinterpret_cast<uint4*>(sX + sw_off(gt, 1)) = x1;
        const int dc = d, sc = sj;
        to_tensor();
        // ---- layer 1: x_e Wc (one K = 16 MMA), then + b1 + P[dst] + Q[src], ReLU
        if (gt == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            umma_bf16(tmem, sw128_desc(smem_addr(sX)), sw128_desc(smem_addr(sWc)), 0u);
            umma_commit(bar);
        }
        // the next tile's edge and this edge's first P/Q block load while the MMA runs
        fetch_edge(tile + stride, d, sj, x0, x1);
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
            put_bf16_row(sA, gt, cb, x);
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
        if (gt == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            issue_k128(tmem, sA, sW2);
            umma_commit(bar);
        }
        ok = mma_wait() && ok;
#pragma unroll 1
        for (int cb = 0; cb < 4; ++cb) {
            uint32_t v[32];
            tmem_ld32(trow + (uint32_t)(cb * 32), v);
            float x[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) x[j] = fmaxf(__uint_as_float(v[j]) + a.b2[cb * 32 + j], 0.f);
            put_bf16_row(sA, gt, cb, x);  // the MMAs that read sA have completed
        }
        to_tensor();
        // ---- layer 3: m_e = z2 W3 + b3, summed per destination
        if (gt == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            issue_k128(tmem, sA, sW3);
            umma_commit(bar);
        }
        ok = mma_wait() && ok;
#pragma unroll 1
        for (int cb = 0; cb < 4; ++cb) {
            uint32_t v[32];
            tmem_ld32(trow + (uint32_t)(cb * 32), v);
#pragma unroll
            for (int j = 0; j < 32; ++j) sStage[gt * 32 + (j ^ (gt & 31))] = __uint_as_float(v[j]) + a.b3[cb * 32 + j];
            group_sync(g);
            // thread (warp gw, column j): rows 32 gw .. 32 gw + 31, one atomic per run of a destination
            const int j = lane;
            int cur = -1;
            float acc = 0.f;
            for (int rr = 0; rr < 32; ++rr) {
                const int row = gw * 32 + rr, dd = dstv[row];
                if (dd < 0) break;  // rows past the last edge close the tile
                if (dd != cur) {
                    if (cur >= 0) atomicAdd(a.out + (size_t)cur * 128 + cb * 32 + j, acc);
                    cur = dd;
                    acc = 0.f;
                }
                acc += sStage[row * 32 + (j ^ (row & 31))];
            }
            if (cur >= 0) atomicAdd(a.out + (size_t)cur * 128 + cb * 32 + j, acc);
            group_sync(g);  // the staging buffer is reused by the next column block
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        // the tile's TMEM reads and shared-memory use end before the group's
        // next tile; a run-out wait on any thread of the group stops the whole
        // group (a decision its threads share, so none is left at a barrier)
        ok = group_all(g, ok);
        if (!ok) break;
    }
    // every committed MMA completes before the tensor memory is freed
    if (gt == 0) umma_commit(bar);
    ok = mma_wait() && ok;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s_tmem), "r"(128u * kGroups)
                     : "memory");
    }
    if (!ok && gt == 0) atomicOr(a.err, 1u);
}

}  // namespace

bool edge_hop_prepare() {
    return cudaFuncSetAttribute(k_edge_hop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes) ==
           cudaSuccess;
}

void launch_edge_hop(const EdgeHopArgs& a, int sms, cudaStream_t st) {
    if (a.E <= 0) return;
    const int ntiles = (a.E + kGroupThreads - 1) / kGroupThreads;
    const int ctas = (ntiles + kGroups - 1) / kGroups;
    const int grid = ctas < sms ? ctas : sms;
    k_edge_hop<<<grid, kEdgeThreads, kSmemBytes, st>>>(a);
}

}  // namespace pe
