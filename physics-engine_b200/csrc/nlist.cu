// Neighbour-list build: one CTA per occupied cell.
//
// Replaces the per-particle `UniformGrid::neighbours` gathers
// (crates/pe-fluid/src/grid.rs:122-140) that the reference repeats six times
// per fluid particle per step. The 27 (3-D) or 9 (2-D) neighbour cells of the
// CTA's cell are visited in the reference's (dz, dy, dx) order; their
// particles (each cell's run already in ascending original index) are staged
// in shared memory as single-precision coordinates relative to the cell
// corner, and every particle of the centre cell filters the staged union with
// a conservative squared-distance bound (`r2_filter` exceeds (2h)^2 by a
// relative 1e-4, far above the single-precision error of the staged
// coordinates), so every pair with q = r/h < 2 is kept. Extra borderline
// candidates are harmless: the f64 passes evaluate q exactly and such pairs
// contribute an exact +-0.
//
// Two lists come out per particle:
//   visit  — fluid particles only: in-support candidates (self excluded) in
//            the reference's visiting order, each flagged boundary / oriented
//            / lower (fluid with a smaller original index);
//   lower  — fluid particles: fluid neighbours with a smaller original index,
//            in ascending original index; boundary particles: all fluid
//            neighbours in ascending original index.
// The ascending-index order comes from one shared-memory bitonic sort of the
// union's fluid entries per cell, shared by all particles of the cell.
#include <climits>

#include "pe_math.cuh"
#include "wcsph_device.cuh"

namespace pe {

namespace {

constexpr int kNlThreads = 128;
constexpr uint32_t kMaxUnionStage = 8192;  // 8192 * 24 B + 4 KB = 196 KB of shared memory

__device__ __forceinline__ void emit(uint32_t* list, uint32_t slot, uint32_t t, uint32_t cap,
                                     uint32_t value) {
    if (t < cap) list[list_index(slot, t, cap)] = value;
}

// Staged word w of a union entry: original index (29 bits) | kind flags.
constexpr uint32_t kStageBoundary = 1u << 31;
constexpr uint32_t kStageOriented = 1u << 30;
constexpr uint32_t kStageOrigMask = (1u << 29) - 1u;

template <int NC>
__device__ __forceinline__ uint32_t slot_of_union(const uint32_t* s_off, const uint32_t* s_cstart,
                                                  uint32_t u) {
    // binary search of the cell q with s_off[q] <= u < s_off[q + 1]
    int lo = 0, hi = NC - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (s_off[mid] <= u) lo = mid;
        else hi = mid - 1;
    }
    return s_cstart[lo] + (u - s_off[lo]);
}

// Block-wide exclusive scan (kNlThreads threads).
__device__ __forceinline__ void block_exclusive_scan(uint32_t v, uint32_t* ex, uint32_t* total) {
    __shared__ uint32_t warp_sums[kNlThreads / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)lane >= o) incl += x;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    uint32_t before = 0, tot = 0;
#pragma unroll
    for (uint32_t w = 0; w < kNlThreads / 32; ++w) {
        if (w < warp) before += warp_sums[w];
        tot += warp_sums[w];
    }
    *ex = before + incl - v;
    *total = tot;
}

__device__ __forceinline__ uint32_t entry_flags(uint32_t w) {
    return ((w & kStageBoundary) ? kEntryBoundary : 0u) | ((w & kStageOriented) ? kEntryOriented : 0u);
}

// Shared-memory layout of one CTA (ucap = staged union capacity):
//   float4   s_pos[ucap]     local coordinates, w = original index | kind flags
//   uint32   s_ent[ucap]     list entry (slot | boundary | oriented) per position
//   uint16   s_sorted[ucap]  union positions of the fluid entries, ascending
//                            original index (radix ping-pong buffer A)
//   uint16   s_tmp[ucap]     radix ping-pong buffer B
//   uint16   s_cnt[16][kNlThreads]  radix digit counters
template <int DIM>
__global__ void __launch_bounds__(kNlThreads) k_nlist(GridDesc g, StepConst k, uint32_t ucap,
                                                      const uint32_t* __restrict__ occ,
                                                      const uint32_t* __restrict__ cell_start,
                                                      StateBufs s, ListBufs l, DeviceScalars* sc) {
    constexpr int NC = DIM == 3 ? 27 : 9;
    constexpr int CENTER = DIM == 3 ? 13 : 4;
    extern __shared__ __align__(16) unsigned char smem[];
    float4* s_pos = reinterpret_cast<float4*>(smem);
    uint32_t* s_ent = reinterpret_cast<uint32_t*>(s_pos + ucap);
    uint16_t* s_sorted = reinterpret_cast<uint16_t*>(s_ent + ucap);
    uint16_t* s_tmp = s_sorted + ucap;
    uint16_t* s_cnt = s_tmp + ucap;  // 16 * kNlThreads
    __shared__ uint32_t s_cstart[NC];
    __shared__ uint32_t s_off[NC + 1];
    __shared__ uint32_t s_nf, s_omin, s_omax;

    const float r2f = k.r2_filter;
    const uint32_t nocc = sc->nocc;
    const uint32_t tid = threadIdx.x;
    bool overflow = false;
    uint32_t max_union = 0;

    for (uint32_t it = blockIdx.x; it < nocc; it += gridDim.x) {
        const uint32_t c = occ[it];
        const int cz = (int)(c % (uint32_t)g.nz);
        const int cy = (int)((c / (uint32_t)g.nz) % (uint32_t)g.ny);
        const int cx = (int)(c / ((uint32_t)g.nz * (uint32_t)g.ny));
        if (tid < 32) {
            uint32_t st = 0, cnt = 0;
            if ((int)tid < NC) {
                int dz = DIM == 3 ? (int)tid / 9 - 1 : 0;
                int dy = DIM == 3 ? ((int)tid / 3) % 3 - 1 : (int)tid / 3 - 1;
                int dx = (int)tid % 3 - 1;
                int qx = cx + dx, qy = cy + dy, qz = cz + dz;
                if (qx >= 0 && qy >= 0 && qz >= 0 && qx < g.nx && qy < g.ny && qz < g.nz) {
                    uint32_t nc = ((uint32_t)qx * (uint32_t)g.ny + (uint32_t)qy) * (uint32_t)g.nz + (uint32_t)qz;
                    st = cell_start[nc];
                    cnt = cell_start[nc + 1] - st;
                }
            }
            uint32_t incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
                if ((int)tid >= o) incl += x;
            }
            if ((int)tid < NC) {
                s_cstart[tid] = st;
                s_off[tid + 1] = incl;
            }
            if (tid == 0) {
                s_off[0] = 0;
                s_nf = 0;
                s_omin = 0xffffffffu;
                s_omax = 0u;
            }
        }
        __syncthreads();
        const uint32_t U = s_off[NC];
        const uint32_t cs = s_cstart[CENTER];
        const uint32_t ncenter = s_off[CENTER + 1] - s_off[CENTER];
        const double ox = (double)(g.kx0 + cx) * g.cell_size;
        const double oy = (double)(g.ky0 + cy) * g.cell_size;
        const double oz = DIM == 3 ? (double)(g.kz0 + cz) * g.cell_size : 0.0;
        max_union = max(max_union, U);

        if (U <= ucap) {
            // ---- stage the union in visiting order ----
            for (uint32_t u = tid; u < U; u += blockDim.x) {
                const uint32_t slot = slot_of_union<NC>(s_off, s_cstart, u);
                const double4 p = s.pos[slot];
                const uint8_t fl = s.flags[slot];
                const uint32_t o = s.orig[slot];
                const uint32_t w = o | ((fl & kFlagBoundary) ? kStageBoundary : 0u) |
                                   ((fl & kFlagOriented) ? kStageOriented : 0u);
                s_pos[u] = make_float4((float)(p.x - ox), (float)(p.y - oy),
                                       DIM == 3 ? (float)(p.z - oz) : 0.0f, __uint_as_float(w));
                s_ent[u] = slot | entry_flags(w);
                if (!(fl & kFlagBoundary)) {
                    const uint32_t idx = atomicAdd(&s_nf, 1u);
                    s_sorted[idx] = (uint16_t)u;
                    atomicMin(&s_omin, o);
                    atomicMax(&s_omax, o);
                }
            }
            __syncthreads();
            // ---- sort the fluid positions by original index: LSD radix sort on
            // 4-bit digits of (orig - min), keys read through the positions ----
            const uint32_t nf = s_nf;
            {
                const uint32_t omin = s_omin;
                const uint32_t span = nf ? s_omax - omin : 0u;
                const int npass = span ? (32 - __clz(span) + 3) / 4 : 0;
                const uint32_t chunk = (nf + kNlThreads - 1) / kNlThreads;
                const uint32_t e0 = min(nf, tid * chunk), e1 = min(nf, e0 + chunk);
                uint16_t *src = s_sorted, *dst = s_tmp;
                for (int pass = 0; pass < npass; ++pass) {
                    const int shift = 4 * pass;
#pragma unroll
                    for (int d = 0; d < 16; ++d) s_cnt[d * kNlThreads + tid] = 0;
                    for (uint32_t e = e0; e < e1; ++e) {
                        const uint32_t o = __float_as_uint(s_pos[src[e]].w) & kStageOrigMask;
                        ++s_cnt[(((o - omin) >> shift) & 15u) * kNlThreads + tid];
                    }
                    __syncthreads();
                    {
                        // exclusive scan of the counters in (digit, thread) order
                        uint32_t v[16], sum = 0;
#pragma unroll
                        for (int q = 0; q < 16; ++q) {
                            v[q] = s_cnt[tid * 16 + q];
                            sum += v[q];
                        }
                        uint32_t ex, tot;
                        block_exclusive_scan(sum, &ex, &tot);
#pragma unroll
                        for (int q = 0; q < 16; ++q) {
                            s_cnt[tid * 16 + q] = (uint16_t)ex;
                            ex += v[q];
                        }
                    }
                    __syncthreads();
                    for (uint32_t e = e0; e < e1; ++e) {
                        const uint16_t pu = src[e];
                        const uint32_t o = __float_as_uint(s_pos[pu].w) & kStageOrigMask;
                        const uint32_t d = ((o - omin) >> shift) & 15u;
                        dst[s_cnt[d * kNlThreads + tid]++] = pu;
                    }
                    __syncthreads();
                    uint16_t* t = src;
                    src = dst;
                    dst = t;
                }
                if (src != s_sorted) {
                    for (uint32_t i = tid; i < nf; i += blockDim.x) s_sorted[i] = src[i];
                    __syncthreads();
                }
            }
            // ---- per centre particle: a "visit" thread and a "lower" thread in
            // different warps, working independently ----
            const uint32_t W = (U + 31u) >> 5;
            const bool lower_role = tid >= kNlThreads / 2;
            for (uint32_t pi = tid % (kNlThreads / 2); pi < ncenter; pi += kNlThreads / 2) {
                const uint32_t kslot = cs + pi;
                const uint32_t myu = s_off[CENTER] + pi;
                const float4 me = s_pos[myu];
                const uint32_t mw = __float_as_uint(me.w);
                const uint32_t myo = mw & kStageOrigMask;
                const bool fluid = !(mw & kStageBoundary);
                if (!lower_role) {
                    uint32_t nv = 0, nu = 0;
                    if (fluid) {
                        for (uint32_t w = 0; w < W; ++w) {
                            uint32_t m = 0;
#pragma unroll
                            for (int bit = 0; bit < 32; ++bit) {
                                const uint32_t u = (w << 5) + bit;
                                const float4 q = s_pos[u];
                                const float dx = q.x - me.x, dy = q.y - me.y, dz = q.z - me.z;
                                const float d2 = dx * dx + dy * dy + dz * dz;
                                m |= (d2 <= r2f && u < U && u != myu) ? (1u << bit) : 0u;
                            }
                            while (m) {
                                const uint32_t u = (w << 5) + (__ffs(m) - 1);
                                m &= m - 1u;
                                const uint32_t ow = __float_as_uint(s_pos[u].w);
                                uint32_t e = s_ent[u];
                                if (!(ow & kStageBoundary) && (ow & kStageOrigMask) < myo) {
                                    e |= kEntryLower;
                                } else {
                                    emit(l.upper, kslot, nu, l.capv, e);
                                    ++nu;
                                }
                                emit(l.visit, kslot, nv, l.capv, e);
                                ++nv;
                            }
                        }
                    }
                    if (nv > l.capv) { overflow = true; nv = l.capv; }
                    if (nu > l.capv) nu = l.capv;
                    l.nvisit[kslot] = nv;
                    l.nupper[kslot] = nu;
                    l.ncand[kslot] = fluid ? U : 0u;
                } else {
                    // R = number of fluid union entries with a smaller original index
                    uint32_t R = nf;
                    if (fluid) {
                        uint32_t lo = 0, hi = nf;
                        while (lo < hi) {
                            const uint32_t mid = (lo + hi) >> 1;
                            const uint32_t o = __float_as_uint(s_pos[s_sorted[mid]].w) & kStageOrigMask;
                            if (o < myo) lo = mid + 1;
                            else hi = mid;
                        }
                        R = lo;
                    }
                    uint32_t nl = 0;
                    for (uint32_t i0 = 0; i0 < R; i0 += 32) {
                        uint32_t m = 0;
#pragma unroll
                        for (int bit = 0; bit < 32; ++bit) {
                            const uint32_t i = i0 + bit;
                            const float4 q = s_pos[s_sorted[i < nf ? i : 0u]];
                            const float dx = q.x - me.x, dy = q.y - me.y, dz = q.z - me.z;
                            const float d2 = dx * dx + dy * dy + dz * dz;
                            m |= (d2 <= r2f && i < R) ? (1u << bit) : 0u;
                        }
                        while (m) {
                            const uint32_t i = i0 + (__ffs(m) - 1);
                            m &= m - 1u;
                            emit(l.lower, kslot, nl, l.capl, s_ent[s_sorted[i]] & kEntrySlotMask);
                            ++nl;
                        }
                    }
                    if (nl > l.capl) { overflow = true; nl = l.capl; }
                    l.nlower[kslot] = nl;
                }
            }
        } else {
            // ---- slow path: union larger than the shared-memory stage ----
            if (tid == 0) atomicOr(&sc->status, kStatusSlowUnion);
            const uint32_t ce = cs + ncenter;
            for (uint32_t kslot = cs + tid; kslot < ce; kslot += blockDim.x) {
                double4 pm = s.pos[kslot];
                const float mx = (float)(pm.x - ox), my = (float)(pm.y - oy),
                            mz = DIM == 3 ? (float)(pm.z - oz) : 0.0f;
                const uint32_t myo = s.orig[kslot];
                const bool fluid = !(s.flags[kslot] & kFlagBoundary);
                uint32_t nv = 0, nl = 0, nu = 0;
                if (fluid) {
                    for (int q = 0; q < NC; ++q) {
                        uint32_t q0 = s_cstart[q], q1 = q0 + (s_off[q + 1] - s_off[q]);
                        for (uint32_t slot = q0; slot < q1; ++slot) {
                            if (slot == kslot) continue;
                            double4 p = s.pos[slot];
                            float dx = (float)(p.x - ox) - mx, dy = (float)(p.y - oy) - my;
                            float dz = DIM == 3 ? (float)(p.z - oz) - mz : 0.0f;
                            if (dx * dx + dy * dy + dz * dz <= r2f) {
                                uint8_t fl = s.flags[slot];
                                uint32_t e = slot | ((fl & kFlagBoundary) ? kEntryBoundary : 0u) |
                                             ((fl & kFlagOriented) ? kEntryOriented : 0u);
                                if (!(fl & kFlagBoundary) && s.orig[slot] < myo) {
                                    e |= kEntryLower;
                                } else {
                                    emit(l.upper, kslot, nu, l.capv, e);
                                    ++nu;
                                }
                                emit(l.visit, kslot, nv, l.capv, e);
                                ++nv;
                            }
                        }
                    }
                }
                // ascending original index by repeated selection (O(U) per output)
                long long last = -1;
                for (;;) {
                    unsigned long long best = ULLONG_MAX;
                    uint32_t best_slot = 0;
                    for (int q = 0; q < NC; ++q) {
                        uint32_t q0 = s_cstart[q], q1 = q0 + (s_off[q + 1] - s_off[q]);
                        for (uint32_t slot = q0; slot < q1; ++slot) {
                            if (s.flags[slot] & kFlagBoundary) continue;
                            uint32_t o = s.orig[slot];
                            if ((long long)o <= last) continue;
                            if (fluid && o >= myo) continue;
                            if ((unsigned long long)o >= best) continue;
                            double4 p = s.pos[slot];
                            float dx = (float)(p.x - ox) - mx, dy = (float)(p.y - oy) - my;
                            float dz = DIM == 3 ? (float)(p.z - oz) - mz : 0.0f;
                            if (dx * dx + dy * dy + dz * dz <= r2f) {
                                best = o;
                                best_slot = slot;
                            }
                        }
                    }
                    if (best == ULLONG_MAX) break;
                    emit(l.lower, kslot, nl, l.capl, best_slot);
                    ++nl;
                    last = (long long)best;
                }
                if (nv > l.capv) { overflow = true; nv = l.capv; }
                if (nl > l.capl) { overflow = true; nl = l.capl; }
                if (nu > l.capv) nu = l.capv;
                l.nupper[kslot] = fluid ? nu : 0u;
                l.nvisit[kslot] = fluid ? nv : 0u;
                l.nlower[kslot] = nl;
                l.ncand[kslot] = fluid ? U : 0u;
            }
        }
        __syncthreads();  // shared memory is reused by the next cell
    }
    if (overflow) atomicOr(&sc->status, kStatusListOverflow);
    if (tid == 0 && max_union) atomicMax(&sc->max_union, max_union);
}

}  // namespace

uint32_t nlist_union_capacity(uint32_t max_union) {
    // The smallest power of two (the bitonic sort works on powers of two) that
    // holds the largest union seen, within the shared-memory limit; larger
    // unions take the slow path.
    uint32_t cap = 256;
    while (cap < max_union && cap < kMaxUnionStage) cap <<= 1;
    return cap;
}

size_t nlist_smem_bytes(uint32_t ucap) {
    return (size_t)ucap * (sizeof(float4) + sizeof(uint32_t) + 2 * sizeof(uint16_t)) +
           16 * kNlThreads * sizeof(uint16_t);
}

uint32_t nlist_prepare(int dim, uint32_t ucap) {
    size_t smem = nlist_smem_bytes(ucap);
    int blocks = 0;
    if (dim == 3) {
        cudaFuncSetAttribute(k_nlist<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_nlist<3>, kNlThreads, smem);
    } else {
        cudaFuncSetAttribute(k_nlist<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_nlist<2>, kNlThreads, smem);
    }
    return blocks > 0 ? (uint32_t)blocks : 1u;
}

void launch_nlist(const GridDesc& g, const StepConst& k, uint32_t ucap, uint32_t nblocks,
                  const uint32_t* occ, const uint32_t* cell_start, const StateBufs& s,
                  const ListBufs& l, DeviceScalars* sc, cudaStream_t st) {
    size_t smem = nlist_smem_bytes(ucap);
    if (g.dim == 3) {
        k_nlist<3><<<nblocks, kNlThreads, smem, st>>>(g, k, ucap, occ, cell_start, s, l, sc);
    } else {
        k_nlist<2><<<nblocks, kNlThreads, smem, st>>>(g, k, ucap, occ, cell_start, s, l, sc);
    }
}

}  // namespace pe
