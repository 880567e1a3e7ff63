// Neighbour-list build: CTAs per occupied cell, two kernels.
//
// Replaces the per-particle `UniformGrid::neighbours` gathers
// (crates/pe-fluid/src/grid.rs:122-140) that the reference repeats six times
// per fluid particle per step. The 27 (3-D) or 9 (2-D) neighbour cells of a
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
// k_nlist_visit writes, for fluid particles, the "visit" list (in-support
// candidates, self excluded, in visiting order, each flagged boundary /
// oriented / lower) and the "upper" list (the visit list without the entries
// flagged lower). k_nlist_lower writes the "lower" list: for fluid particles
// the fluid neighbours with a smaller original index, for boundary particles
// all fluid neighbours, both in ascending original index; the order comes
// from a shared-memory radix sort of the union's fluid entries per cell.
//
// Each centre particle is served by two threads in different warps that
// split its candidates in halves (union words, or sorted positions) and write
// to the two halves of the particle's list storage; consumers read part 0 and
// then part 1, which is the full list in order.
#include <climits>

#include "pe_math.cuh"
#include "wcsph_device.cuh"

namespace pe {

namespace {

constexpr int kNlThreads = 128;
constexpr uint32_t kHalf = kNlThreads / 2;
constexpr uint32_t kMaxUnionStage = 8192;

// Staged word w of a union entry: original index (29 bits) | kind flags.
constexpr uint32_t kStageBoundary = 1u << 31;
constexpr uint32_t kStageOriented = 1u << 30;
constexpr uint32_t kStageOrigMask = (1u << 29) - 1u;

__device__ __forceinline__ void emit(uint32_t* list, uint32_t slot, uint32_t t, uint32_t cap,
                                     uint32_t value) {
    if (t < cap) list[list_index(slot, t, cap)] = value;
}

// Base of slot s's entries in a list (entry t at base[(t & ~3) * 32 + (t & 3)]).
__device__ __forceinline__ uint32_t* slot_base(uint32_t* list, uint32_t s, uint32_t cap) {
    return list + (size_t)(s >> 5) * cap * 32u + (s & 31u) * 4u;
}

__device__ __forceinline__ void put(uint32_t* base, uint32_t t, uint32_t value) {
    base[(t & ~3u) * 32u + (t & 3u)] = value;
}

template <int NC>
__device__ __forceinline__ uint32_t slot_of_union(const uint32_t* s_off, const uint32_t* s_cstart,
                                                  uint32_t u) {
    int lo = 0, hi = NC - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (s_off[mid] <= u) lo = mid;
        else hi = mid - 1;
    }
    return s_cstart[lo] + (u - s_off[lo]);
}

__device__ __forceinline__ uint32_t entry_flags(uint32_t w) {
    return ((w & kStageBoundary) ? kEntryBoundary : 0u) | ((w & kStageOriented) ? kEntryOriented : 0u);
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
    __syncthreads();
}

struct CellUnion {
    uint32_t U, cs, ncenter, center_off;
    double ox, oy, oz;
};

// Ranges of the NC neighbour cells of dense cell c, in visiting order.
template <int DIM>
__device__ __forceinline__ CellUnion cell_union(const GridDesc& g, uint32_t c,
                                                const uint32_t* __restrict__ cell_start,
                                                uint32_t* s_cstart, uint32_t* s_off) {
    constexpr int NC = DIM == 3 ? 27 : 9;
    constexpr int CENTER = DIM == 3 ? 13 : 4;
    const uint32_t tid = threadIdx.x;
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
        if (tid == 0) s_off[0] = 0;
    }
    __syncthreads();
    CellUnion cu;
    cu.U = s_off[NC];
    cu.cs = s_cstart[CENTER];
    cu.ncenter = s_off[CENTER + 1] - s_off[CENTER];
    cu.center_off = s_off[CENTER];
    cu.ox = (double)(g.kx0 + cx) * g.cell_size;
    cu.oy = (double)(g.ky0 + cy) * g.cell_size;
    cu.oz = DIM == 3 ? (double)(g.kz0 + cz) * g.cell_size : 0.0;
    return cu;
}

template <int DIM>
__device__ __forceinline__ float4 stage_entry(const StateBufs& s, uint32_t slot, const CellUnion& cu,
                                              uint8_t* fl_out, uint32_t* orig_out) {
    const double4 p = s.pos[slot];
    const uint8_t fl = s.flags[slot];
    const uint32_t o = s.orig[slot];
    const uint32_t w = o | ((fl & kFlagBoundary) ? kStageBoundary : 0u) |
                       ((fl & kFlagOriented) ? kStageOriented : 0u);
    *fl_out = fl;
    *orig_out = o;
    return make_float4((float)(p.x - cu.ox), (float)(p.y - cu.oy),
                       DIM == 3 ? (float)(p.z - cu.oz) : 0.0f, __uint_as_float(w));
}

__device__ __forceinline__ bool within(const float4& q, const float4& me, float r2f) {
    const float dx = q.x - me.x, dy = q.y - me.y, dz = q.z - me.z;
    return dx * dx + dy * dy + dz * dz <= r2f;
}

// ----------------------------------------------------------------- visit
// Shared memory: float4 s_pos[ucap]; uint32 s_ent[ucap].
template <int DIM>
__global__ void __launch_bounds__(kNlThreads) k_nlist_visit(GridDesc g, StepConst k, uint32_t ucap,
                                                            const uint32_t* __restrict__ occ,
                                                            const uint32_t* __restrict__ cell_start,
                                                            StateBufs s, ListBufs l,
                                                            DeviceScalars* sc) {
    constexpr int NC = DIM == 3 ? 27 : 9;
    extern __shared__ __align__(16) unsigned char smem[];
    float4* s_pos = reinterpret_cast<float4*>(smem);
    uint32_t* s_ent = reinterpret_cast<uint32_t*>(s_pos + ucap);
    __shared__ uint32_t s_cstart[NC];
    __shared__ uint32_t s_off[NC + 1];

    const float r2f = k.r2_filter;
    const uint32_t nocc = sc->nocc;
    const uint32_t tid = threadIdx.x;
    const uint32_t part = tid / kHalf;
    const uint32_t half_cap = l.capv >> 1;
    const size_t n = l.nslots;
    bool overflow = false;
    uint32_t max_union = 0, longest = 0;

    for (uint32_t it = blockIdx.x; it < nocc; it += gridDim.x) {
        const CellUnion cu = cell_union<DIM>(g, occ[it], cell_start, s_cstart, s_off);
        const uint32_t U = cu.U;
        max_union = max(max_union, U);
        if (U <= ucap) {
            for (uint32_t u = tid; u < U; u += blockDim.x) {
                const uint32_t slot = slot_of_union<NC>(s_off, s_cstart, u);
                uint8_t fl;
                uint32_t o;
                const float4 q = stage_entry<DIM>(s, slot, cu, &fl, &o);
                s_pos[u] = q;
                s_ent[u] = slot | entry_flags(__float_as_uint(q.w));
            }
            __syncthreads();
            const uint32_t W = (U + 31u) >> 5, Wh = (W + 1u) >> 1;
            const uint32_t w0 = part ? Wh : 0u, w1 = part ? W : Wh;
            const uint32_t base = part * half_cap;
            for (uint32_t pi = tid % kHalf; pi < cu.ncenter; pi += kHalf) {
                const uint32_t kslot = cu.cs + pi;
                const uint32_t myu = cu.center_off + pi;
                const float4 me = s_pos[myu];
                const uint32_t mw = __float_as_uint(me.w);
                const uint32_t myo = mw & kStageOrigMask;
                uint32_t nv = 0, nu = 0;
                uint32_t* vb = slot_base(l.visit, kslot, l.capv) ;
                // no upper list storage in the single-precision form (visit list only)
                uint32_t* ub = l.upper ? slot_base(l.upper, kslot, l.capv) : nullptr;
                if (!(mw & kStageBoundary)) {
                    for (uint32_t w = w0; w < w1; ++w) {
                        uint32_t m = 0;
#pragma unroll
                        for (int bit = 0; bit < 32; ++bit)
                            m |= within(s_pos[(w << 5) + bit], me, r2f) ? (1u << bit) : 0u;
                        if (w == W - 1u && (U & 31u)) m &= (1u << (U & 31u)) - 1u;
                        if (w == (myu >> 5)) m &= ~(1u << (myu & 31u));
                        while (m) {
                            const uint32_t u = (w << 5) + (__ffs(m) - 1);
                            m &= m - 1u;
                            const uint32_t ow = __float_as_uint(s_pos[u].w);
                            uint32_t e = s_ent[u];
                            if (!(ow & kStageBoundary) && (ow & kStageOrigMask) < myo) {
                                e |= kEntryLower;
                            } else {
                                if (ub && nu < half_cap) put(ub, base + nu, e);
                                ++nu;
                            }
                            if (nv < half_cap) put(vb, base + nv, e);
                            ++nv;
                        }
                    }
                }
                longest = max(longest, nv);
                if (nv > half_cap) { overflow = true; nv = half_cap; }
                if (nu > half_cap) nu = half_cap;
                l.nvisit[part * n + kslot] = nv;
                l.nupper[part * n + kslot] = nu;
                if (part == 0) l.ncand[kslot] = (mw & kStageBoundary) ? 0u : U;
            }
        } else {
            // slow path: a union larger than the stage, straight from global memory
            if (tid == 0) atomicOr(&sc->status, kStatusSlowUnion);
            for (uint32_t kslot = cu.cs + tid; kslot < cu.cs + cu.ncenter; kslot += blockDim.x) {
                uint8_t mfl;
                uint32_t myo;
                const float4 me = stage_entry<DIM>(s, kslot, cu, &mfl, &myo);
                const bool fluid = !(mfl & kFlagBoundary);
                uint32_t nv = 0, nu = 0;
                if (fluid) {
                    for (int q = 0; q < NC; ++q) {
                        const uint32_t q0 = s_cstart[q], q1 = q0 + (s_off[q + 1] - s_off[q]);
                        for (uint32_t slot = q0; slot < q1; ++slot) {
                            if (slot == kslot) continue;
                            uint8_t fl;
                            uint32_t o;
                            const float4 qp = stage_entry<DIM>(s, slot, cu, &fl, &o);
                            if (!within(qp, me, r2f)) continue;
                            uint32_t e = slot | entry_flags(__float_as_uint(qp.w));
                            if (!(fl & kFlagBoundary) && o < myo) {
                                e |= kEntryLower;
                            } else {
                                if (l.upper && nu < half_cap) emit(l.upper, kslot, nu, l.capv, e);
                                ++nu;
                            }
                            if (nv < half_cap) emit(l.visit, kslot, nv, l.capv, e);
                            ++nv;
                        }
                    }
                }
                longest = max(longest, nv);
                if (nv > half_cap) { overflow = true; nv = half_cap; }
                if (nu > half_cap) nu = half_cap;
                l.nvisit[kslot] = nv;
                l.nupper[kslot] = nu;
                l.nvisit[n + kslot] = 0;
                l.nupper[n + kslot] = 0;
                l.ncand[kslot] = fluid ? U : 0u;
            }
        }
        __syncthreads();  // shared memory is reused by the next cell
    }
    if (overflow) atomicOr(&sc->status, kStatusListOverflow);
    if (tid == 0 && max_union) atomicMax(&sc->max_union, max_union);
    if (longest) atomicMax(&sc->max_part, longest);
}

// ----------------------------------------------------------------- lower
// Shared memory: float4 s_pos[ucap]; uint32 s_ent[ucap]; uint16 s_sorted[ucap];
// uint16 s_tmp[ucap]; uint16 s_cnt[16][kNlThreads].
template <int DIM>
__global__ void __launch_bounds__(kNlThreads) k_nlist_lower(GridDesc g, StepConst k, uint32_t ucap,
                                                            const uint32_t* __restrict__ occ,
                                                            const uint32_t* __restrict__ cell_start,
                                                            StateBufs s, ListBufs l,
                                                            DeviceScalars* sc) {
    constexpr int NC = DIM == 3 ? 27 : 9;
    extern __shared__ __align__(16) unsigned char smem[];
    float4* s_pos = reinterpret_cast<float4*>(smem);
    uint32_t* s_ent = reinterpret_cast<uint32_t*>(s_pos + ucap);
    uint16_t* s_sorted = reinterpret_cast<uint16_t*>(s_ent + ucap);
    uint16_t* s_tmp = s_sorted + ucap;
    uint16_t* s_cnt = s_tmp + ucap;
    __shared__ uint32_t s_cstart[NC];
    __shared__ uint32_t s_off[NC + 1];
    __shared__ uint32_t s_nf, s_omin, s_omax;

    const float r2f = k.r2_filter;
    const uint32_t nocc = sc->nocc;
    const uint32_t tid = threadIdx.x;
    const uint32_t part = tid / kHalf;
    const uint32_t half_cap = l.capl >> 1;
    const size_t n = l.nslots;
    bool overflow = false;
    uint32_t longest = 0;

    for (uint32_t it = blockIdx.x; it < nocc; it += gridDim.x) {
        if (tid == 0) {
            s_nf = 0;
            s_omin = 0xffffffffu;
            s_omax = 0u;
        }
        const CellUnion cu = cell_union<DIM>(g, occ[it], cell_start, s_cstart, s_off);
        const uint32_t U = cu.U;
        if (U <= ucap) {
            for (uint32_t u = tid; u < U; u += blockDim.x) {
                const uint32_t slot = slot_of_union<NC>(s_off, s_cstart, u);
                uint8_t fl;
                uint32_t o;
                s_pos[u] = stage_entry<DIM>(s, slot, cu, &fl, &o);
                s_ent[u] = slot;
                if (!(fl & kFlagBoundary)) {
                    const uint32_t idx = atomicAdd(&s_nf, 1u);
                    s_sorted[idx] = (uint16_t)u;
                    atomicMin(&s_omin, o);
                    atomicMax(&s_omax, o);
                }
            }
            __syncthreads();
            // LSD radix sort of the fluid positions on 4-bit digits of
            // (orig - min); keys are read through the positions. The keys are
            // unique, so the result does not depend on the staging order.
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
                        dst[s_cnt[(((o - omin) >> shift) & 15u) * kNlThreads + tid]++] = pu;
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
            const uint32_t base = part * half_cap;
            for (uint32_t pi = tid % kHalf; pi < cu.ncenter; pi += kHalf) {
                const uint32_t kslot = cu.cs + pi;
                const float4 me = s_pos[cu.center_off + pi];
                const uint32_t mw = __float_as_uint(me.w);
                const uint32_t myo = mw & kStageOrigMask;
                // R = number of fluid union entries below this particle's index
                uint32_t R = nf;
                if (!(mw & kStageBoundary)) {
                    uint32_t lo = 0, hi = nf;
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        const uint32_t o = __float_as_uint(s_pos[s_sorted[mid]].w) & kStageOrigMask;
                        if (o < myo) lo = mid + 1;
                        else hi = mid;
                    }
                    R = lo;
                }
                const uint32_t i_begin = part ? (R >> 1) : 0u, i_end = part ? R : (R >> 1);
                uint32_t nl = 0;
                uint32_t* lb = slot_base(l.lower, kslot, l.capl);
                for (uint32_t i0 = i_begin; i0 < i_end; i0 += 32) {
                    uint32_t m = 0;
#pragma unroll
                    for (int bit = 0; bit < 32; ++bit) {
                        const uint32_t i = i0 + bit;
                        m |= within(s_pos[s_sorted[i < nf ? i : 0u]], me, r2f) ? (1u << bit) : 0u;
                    }
                    if (i_end - i0 < 32u) m &= (1u << (i_end - i0)) - 1u;
                    while (m) {
                        const uint32_t i = i0 + (__ffs(m) - 1);
                        m &= m - 1u;
                        if (nl < half_cap) put(lb, base + nl, s_ent[s_sorted[i]]);
                        ++nl;
                    }
                }
                longest = max(longest, nl);
                if (nl > half_cap) { overflow = true; nl = half_cap; }
                l.nlower[part * n + kslot] = nl;
            }
        } else {
            // slow path: ascending original index by repeated selection
            if (tid == 0) atomicOr(&sc->status, kStatusSlowUnion);
            for (uint32_t kslot = cu.cs + tid; kslot < cu.cs + cu.ncenter; kslot += blockDim.x) {
                uint8_t mfl;
                uint32_t myo;
                const float4 me = stage_entry<DIM>(s, kslot, cu, &mfl, &myo);
                const bool fluid = !(mfl & kFlagBoundary);
                uint32_t nl = 0;
                long long last = -1;
                for (;;) {
                    unsigned long long best = ULLONG_MAX;
                    uint32_t best_slot = 0;
                    for (int q = 0; q < NC; ++q) {
                        const uint32_t q0 = s_cstart[q], q1 = q0 + (s_off[q + 1] - s_off[q]);
                        for (uint32_t slot = q0; slot < q1; ++slot) {
                            if (s.flags[slot] & kFlagBoundary) continue;
                            const uint32_t o = s.orig[slot];
                            if ((long long)o <= last || (fluid && o >= myo) ||
                                (unsigned long long)o >= best)
                                continue;
                            uint8_t fl;
                            uint32_t oo;
                            if (within(stage_entry<DIM>(s, slot, cu, &fl, &oo), me, r2f)) {
                                best = o;
                                best_slot = slot;
                            }
                        }
                    }
                    if (best == ULLONG_MAX) break;
                    if (nl < half_cap) emit(l.lower, kslot, nl, l.capl, best_slot);
                    ++nl;
                    last = (long long)best;
                }
                longest = max(longest, nl);
                if (nl > half_cap) { overflow = true; nl = half_cap; }
                l.nlower[kslot] = nl;
                l.nlower[n + kslot] = 0;
            }
        }
        __syncthreads();
    }
    if (overflow) atomicOr(&sc->status, kStatusListOverflow);
    if (longest) atomicMax(&sc->max_part, longest);
}

size_t visit_smem_bytes(uint32_t ucap) { return (size_t)ucap * (sizeof(float4) + sizeof(uint32_t)); }

}  // namespace

uint32_t nlist_union_capacity(uint32_t max_union) {
    // The smallest power of two that holds the largest union seen, within the
    // shared-memory limit; larger unions take the slow path.
    uint32_t cap = 256;
    while (cap < max_union && cap < kMaxUnionStage) cap <<= 1;
    return cap;
}

size_t nlist_smem_bytes(uint32_t ucap) {
    // the lower kernel's layout, the larger of the two
    return (size_t)ucap * (sizeof(float4) + sizeof(uint32_t) + 2 * sizeof(uint16_t)) +
           16 * kNlThreads * sizeof(uint16_t);
}

uint32_t nlist_prepare(int dim, uint32_t ucap) {
    const size_t sl = nlist_smem_bytes(ucap), sv = visit_smem_bytes(ucap);
    int bl = 0, bv = 0;
    if (dim == 3) {
        cudaFuncSetAttribute(k_nlist_lower<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sl);
        cudaFuncSetAttribute(k_nlist_visit<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sv);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bl, k_nlist_lower<3>, kNlThreads, sl);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bv, k_nlist_visit<3>, kNlThreads, sv);
    } else {
        cudaFuncSetAttribute(k_nlist_lower<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sl);
        cudaFuncSetAttribute(k_nlist_visit<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sv);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bl, k_nlist_lower<2>, kNlThreads, sl);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bv, k_nlist_visit<2>, kNlThreads, sv);
    }
    const int b = bl > bv ? bl : bv;
    return b > 0 ? (uint32_t)b : 1u;
}

void launch_nlist(const GridDesc& g, const StepConst& k, uint32_t ucap, uint32_t nblocks,
                  const uint32_t* occ, const uint32_t* cell_start, const StateBufs& s,
                  const ListBufs& l, DeviceScalars* sc, cudaStream_t st, bool visit_only) {
    const size_t sl = nlist_smem_bytes(ucap), sv = visit_smem_bytes(ucap);
    if (g.dim == 3) {
        k_nlist_visit<3><<<nblocks, kNlThreads, sv, st>>>(g, k, ucap, occ, cell_start, s, l, sc);
        if (!visit_only)
            k_nlist_lower<3><<<nblocks, kNlThreads, sl, st>>>(g, k, ucap, occ, cell_start, s, l, sc);
    } else {
        k_nlist_visit<2><<<nblocks, kNlThreads, sv, st>>>(g, k, ucap, occ, cell_start, s, l, sc);
        if (!visit_only)
            k_nlist_lower<2><<<nblocks, kNlThreads, sl, st>>>(g, k, ucap, occ, cell_start, s, l, sc);
    }
}

}  // namespace pe
