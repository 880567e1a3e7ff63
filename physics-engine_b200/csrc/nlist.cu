// Neighbour-list build: CTAs per occupied cell.
//
// Replaces the per-particle `UniformGrid::neighbours` gathers
// (crates/pe-fluid/src/grid.rs:122-140) that the reference repeats six times
// per fluid particle per step. The 27 (3-D) or 9 (2-D) neighbour cells of a
// CTA's cell are visited in the reference's (dz, dy, dx) order; their
// particles (each cell's run already in ascending original index) are staged
// in shared memory as single-precision coordinates relative to the cell
// corner, one array per coordinate, and every particle of the centre cell
// filters the staged union with a conservative squared-distance bound
// (`r2_filter` exceeds (2h)^2 by a relative 1e-4, far above the
// single-precision error of the staged coordinates), four candidates per
// 16-byte read on paired f32x2 arithmetic, so every pair with q = r/h < 2 is
// kept. Extra borderline candidates are harmless: the f64 passes evaluate q
// exactly and such pairs contribute an exact +-0.
//
// k_nlist_both writes, for fluid particles, the "visit" list (in-support
// candidates, self excluded, in visiting order, each flagged boundary /
// oriented / lower; the force pass reads its unflagged entries as the
// reference's j > i and boundary pairs) and the "lower" list: for fluid
// particles the fluid neighbours with a smaller original index, for boundary
// particles all fluid neighbours, both in ascending original index; the order
// comes from a shared-memory radix sort (9-bit digits) of the union's fluid
// entries per cell. k_nlist_visit writes the visit list alone (the passes that need no
// ascending-index order).
//
// The kernels work on chunks of up to 32 (or 64) centre particles with eight
// (or four) threads per particle; the fused kernel is compiled for three
// resident CTAs per SM (80 registers), which the 32-centre tile's shared
// memory allows. A first pass, each thread taking a quarter of the candidates
// (union words, or sorted positions), keeps the in-support bit masks in shared
// memory and counts; the chunk's longest lists size one block of the list
// pool, reserved with one atomic add; a second pass writes the entries, each
// thread a quarter of the particle's list (a quarter of the words would leave
// most of the kept candidates, which lie in the middle words, to two threads).
#include <climits>

#include "pe_math.cuh"
#include "wcsph_device.cuh"

namespace pe {

namespace {

constexpr int kNlThreads = 256;
// Centre particles per chunk (a launch shape the world's autotuner picks:
// 32, the world's default, or 64); kNlThreads / chunk threads work on each
// centre particle. kDefaultChunk is what an unknown value falls back to.
constexpr uint32_t kDefaultChunk = 64;
constexpr uint32_t kWarps = kNlThreads / 32;
// Largest stage: the fused kernel's 38 dynamic bytes per staged entry (f32
// position 16, slot 4, sort index 2, visit masks 8, lower masks or sort
// scratch 8) plus its ~2.4 KB of static shared memory must fit the 227 KB a
// CTA can opt in to on sm_100 (232,448 bytes).
constexpr uint32_t kMaxUnionStage = 5888;
static_assert(38u * kMaxUnionStage + 4096u <= 232448u, "list stage exceeds the shared-memory limit");
constexpr uint32_t kStageStep = 256;               // stage capacities are multiples of this

// Staged word w of a union entry: original index (29 bits) | kind flags.
constexpr uint32_t kStageBoundary = 1u << 31;  // the sign bit (word_mask reads it so)
constexpr uint32_t kStageOriented = 1u << 30;
constexpr uint32_t kStageOrigMask = (1u << 29) - 1u;

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
    __shared__ uint32_t warp_sums[kWarps];
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
    for (uint32_t w = 0; w < kWarps; ++w) {
        if (w < warp) before += warp_sums[w];
        tot += warp_sums[w];
    }
    *ex = before + incl - v;
    *total = tot;
    __syncthreads();
}

__device__ __forceinline__ uint32_t warp_max(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

struct CellUnion {
    uint32_t U, cs, ncenter, center_off;
    double ox, oy, oz;
};

// Ranges of the NC neighbour cells of global dense cell c, in visiting order;
// neighbours are taken inside the box of c's tank.
template <int DIM>
__device__ __forceinline__ CellUnion cell_union(const GridDesc& g, const Tanks& tk, uint32_t c,
                                                const uint32_t* __restrict__ cell_start,
                                                uint32_t* s_cstart, uint32_t* s_off) {
    constexpr int NC = DIM == 3 ? 27 : 9;
    constexpr int CENTER = DIM == 3 ? 13 : 4;
    const uint32_t tid = threadIdx.x;
    const TankDesc td = tk.desc[tk.cell_tank[c]];
    const uint32_t lc = c - td.cell_base;
    const int cz = (int)(lc % (uint32_t)td.nz);
    const int cy = (int)((lc / (uint32_t)td.nz) % (uint32_t)td.ny);
    const int cx = (int)(lc / ((uint32_t)td.nz * (uint32_t)td.ny));
    if (tid < 32) {
        uint32_t st = 0, cnt = 0;
        if ((int)tid < NC) {
            int dz = DIM == 3 ? (int)tid / 9 - 1 : 0;
            int dy = DIM == 3 ? ((int)tid / 3) % 3 - 1 : (int)tid / 3 - 1;
            int dx = (int)tid % 3 - 1;
            int qx = cx + dx, qy = cy + dy, qz = cz + dz;
            if (qx >= 0 && qy >= 0 && qz >= 0 && qx < td.nx && qy < td.ny && qz < td.nz) {
                uint32_t nc = td.cell_base +
                              ((uint32_t)qx * (uint32_t)td.ny + (uint32_t)qy) * (uint32_t)td.nz + (uint32_t)qz;
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
    cu.ox = (double)(td.kx0 + cx) * g.cell_size;
    cu.oy = (double)(td.ky0 + cy) * g.cell_size;
    cu.oz = DIM == 3 ? (double)(td.kz0 + cz) * g.cell_size : 0.0;
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

// in-support, or a boundary candidate kept whatever its distance
__device__ __forceinline__ bool keep_entry(const float4& q, const float4& me, float r2f, int keep_boundary) {
    return within(q, me, r2f) || (keep_boundary && (__float_as_uint(q.w) & kStageBoundary));
}

// The staged union in shared memory as four float arrays (cell-local x, y, z
// and the staged word orig | kind flags), so that the candidates of a word can
// be read four at a time per coordinate.
struct Stage {
    float *x, *y, *z, *w;
    __device__ __forceinline__ Stage(float* base, uint32_t ucap)
        : x(base), y(base + ucap), z(base + 2 * ucap), w(base + 3 * ucap) {}
    __device__ __forceinline__ float4 get(uint32_t u) const { return make_float4(x[u], y[u], z[u], w[u]); }
    __device__ __forceinline__ void put(uint32_t u, const float4& p) {
        x[u] = p.x;
        y[u] = p.y;
        z[u] = p.z;
        w[u] = p.w;
    }
    __device__ __forceinline__ uint32_t word(uint32_t u) const { return __float_as_uint(w[u]); }
};

// Packed single-precision pairs (two f32 in one 64-bit register) and the
// sm_100 paired arithmetic on them, each half rounded to nearest like the
// scalar instruction.
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2_sub(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// Keep mask of the 32 staged entries from position base (keep_entry per bit):
// four candidates per 16-byte read of each coordinate, their squared
// distances in two packed pairs (dx dx + dy dy + dz dz, as the scalar test).
template <bool KEEP_BOUNDARY>
__device__ __forceinline__ uint32_t word_mask(const Stage& st, uint32_t base, const float4& me, float r2f) {
    const unsigned long long mx = f2_pack(me.x, me.x), my = f2_pack(me.y, me.y), mz = f2_pack(me.z, me.z);
    uint32_t m = 0;
#pragma unroll
    for (int g = 0; g < 8; ++g) {
        const float4 X = *reinterpret_cast<const float4*>(st.x + base + 4 * g);
        const float4 Y = *reinterpret_cast<const float4*>(st.y + base + 4 * g);
        const float4 Z = *reinterpret_cast<const float4*>(st.z + base + 4 * g);
        const unsigned long long dx0 = f2_sub(f2_pack(X.x, X.y), mx), dx1 = f2_sub(f2_pack(X.z, X.w), mx);
        const unsigned long long dy0 = f2_sub(f2_pack(Y.x, Y.y), my), dy1 = f2_sub(f2_pack(Y.z, Y.w), my);
        const unsigned long long dz0 = f2_sub(f2_pack(Z.x, Z.y), mz), dz1 = f2_sub(f2_pack(Z.z, Z.w), mz);
        const unsigned long long r0 = f2_fma(dz0, dz0, f2_fma(dy0, dy0, f2_mul(dx0, dx0)));
        const unsigned long long r1 = f2_fma(dz1, dz1, f2_fma(dy1, dy1, f2_mul(dx1, dx1)));
        float a, b, c, d;
        f2_unpack(r0, a, b);
        f2_unpack(r1, c, d);
        uint32_t k4 = (a <= r2f ? 1u : 0u) | (b <= r2f ? 2u : 0u) | (c <= r2f ? 4u : 0u) | (d <= r2f ? 8u : 0u);
        if (KEEP_BOUNDARY) {
            const float4 W = *reinterpret_cast<const float4*>(st.w + base + 4 * g);
            k4 |= ((__float_as_uint(W.x) >> 31) & 1u) | (((__float_as_uint(W.y) >> 31) & 1u) << 1) |
                  (((__float_as_uint(W.z) >> 31) & 1u) << 2) | (((__float_as_uint(W.w) >> 31) & 1u) << 3);
        }
        m |= k4 << (4 * g);
    }
    return m;
}

__device__ __forceinline__ uint32_t rows_for(uint32_t n) { return (n + 3u) >> 2; }

// Reserved block of one chunk: `rows_a + rows_b` rows of `stride` groups.
struct ChunkBlock {
    unsigned long long base;  // group index of row 0, lane 0
    uint32_t rows_a, rows_b;
    bool ok;
};

// Cursor over the set bits of one centre's masks (word w at m[w * kChunk]),
// in ascending bit order: entry t of the list is the t-th set bit.
template <uint32_t kChunk>
struct MaskCursor {
    static constexpr uint32_t kWays = kNlThreads / kChunk;
    const uint32_t* m;
    uint32_t w, bits;
    // Positioned on entry t0, given this centre's per-way counts cnt[r] of the
    // way word ranges [W r / kWays, W (r + 1) / kWays); t0 < the total count.
    __device__ __forceinline__ MaskCursor(const uint32_t* masks, const uint32_t (*cnt)[kChunk], uint32_t lane,
                                          uint32_t W, uint32_t t0)
        : m(masks + lane) {
        uint32_t r = 0, acc = 0;
        while (r + 1u < kWays && acc + cnt[r][lane] <= t0) acc += cnt[r++][lane];
        w = W * r / kWays;
        bits = m[w * kChunk];
        while (acc + (uint32_t)__popc(bits) <= t0) {
            acc += __popc(bits);
            bits = m[++w * kChunk];
        }
        for (; acc < t0; ++acc) bits &= bits - 1u;
    }
    // Position of the next set bit; the caller takes no more than the count.
    __device__ __forceinline__ uint32_t next() {
        while (!bits) bits = m[++w * kChunk];
        const uint32_t u = (w << 5) + (__ffs(bits) - 1);
        bits &= bits - 1u;
        return u;
    }
};

// Every thread passes its (a, b) list lengths; thread 0 reserves the block for
// the chunk's longest ones and all threads return it.
__device__ __forceinline__ ChunkBlock reserve_chunk(const ListBufs& l, DeviceScalars* sc, uint32_t stride,
                                                    uint32_t na, uint32_t nb, uint32_t (*s_red)[2],
                                                    ChunkBlock* s_blk, bool* s_overflow) {
    const uint32_t a = warp_max(na), b = warp_max(nb);
    if ((threadIdx.x & 31u) == 0) {
        s_red[threadIdx.x >> 5][0] = a;
        s_red[threadIdx.x >> 5][1] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t ma = 0, mb = 0;
#pragma unroll
        for (uint32_t w = 0; w < kWarps; ++w) {
            ma = max(ma, s_red[w][0]);
            mb = max(mb, s_red[w][1]);
        }
        ChunkBlock blk;
        blk.rows_a = rows_for(ma);
        blk.rows_b = rows_for(mb);
        const unsigned long long groups = (unsigned long long)(blk.rows_a + blk.rows_b) * stride;
        blk.base = groups ? atomicAdd(&sc->list_used, groups) : 0ull;
        // counts, strides and row offsets are stored in 16 bits
        const bool fits16 = ma < 65536u && mb < 65536u && stride < 65536u && blk.rows_a < 65536u;
        blk.ok = fits16 && blk.base + groups <= l.pool_groups;
        if (!blk.ok) *s_overflow = true;
        *s_blk = blk;
    }
    __syncthreads();
    return *s_blk;
}

// LSD radix sort of a union's fluid positions (s_sorted[0..nf)) by original
// index, on 9-bit digits of (orig - omin) (two passes for spans below 2^18);
// keys are read through the staged words. Warp w ranks the w-th contiguous
// segment of the array, 32 entries at a time in order, grouping equal digits
// with a match, so every pass is stable; counter (digit, warp) is
// s_cnt[digit * kWarps + warp] and one exclusive scan over them in that order
// gives each group its start. The keys are unique, so the result does not
// depend on the staging order. Ends with a block barrier.
constexpr int kRadixBits = 9;
constexpr uint32_t kRadixDigits = 1u << kRadixBits;
static_assert(kRadixDigits * kWarps == 16 * kNlThreads, "radix counters fill the scan's 16 per thread");

__device__ __forceinline__ void radix_sort_by_orig(const float* s_w, uint16_t* s_sorted, uint16_t* s_tmp,
                                                   uint16_t* s_cnt, uint32_t nf, uint32_t omin, uint32_t omax) {
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t span = nf ? omax - omin : 0u;
    const int npass = span ? (32 - __clz(span) + kRadixBits - 1) / kRadixBits : 0;
    const uint32_t seg = ((nf + kWarps - 1) / kWarps + 31u) & ~31u;
    const uint32_t e0 = min(nf, warp * seg), e1 = min(nf, e0 + seg);
    uint16_t *src = s_sorted, *dst = s_tmp;
    for (int pass = 0; pass < npass; ++pass) {
        const int shift = kRadixBits * pass;
        for (uint32_t i = tid; i < kRadixDigits * kWarps; i += blockDim.x) s_cnt[i] = 0;
        __syncthreads();
        for (uint32_t b = e0; b < e1; b += 32u) {
            const uint32_t e = b + lane;
            const bool valid = e < e1;
            uint32_t d = kRadixDigits;  // lanes past the segment: a digit of their own
            if (valid) d = (((__float_as_uint(s_w[src[e]]) & kStageOrigMask) - omin) >> shift) & (kRadixDigits - 1u);
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            if (valid && lane == (uint32_t)(__ffs(peers) - 1)) s_cnt[d * kWarps + warp] += (uint16_t)__popc(peers);
            __syncwarp();
        }
        __syncthreads();
        {
            // this thread's 16 consecutive counters as two 16-byte words
            // (32-byte stride between lanes: two-way bank conflicts, not 8)
            uint4* cw = reinterpret_cast<uint4*>(s_cnt + tid * 16);
            const uint4 c0 = cw[0], c1 = cw[1];
            const uint32_t pk[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
            uint32_t sum = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) sum += (pk[j] & 0xffffu) + (pk[j] >> 16);
            uint32_t ex, tot;
            block_exclusive_scan(sum, &ex, &tot);
            uint32_t out[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t lo = ex;
                ex += pk[j] & 0xffffu;
                out[j] = lo | (ex << 16);
                ex += pk[j] >> 16;
            }
            cw[0] = make_uint4(out[0], out[1], out[2], out[3]);
            cw[1] = make_uint4(out[4], out[5], out[6], out[7]);
        }
        __syncthreads();
        for (uint32_t b = e0; b < e1; b += 32u) {
            const uint32_t e = b + lane;
            const bool valid = e < e1;
            uint32_t d = kRadixDigits;
            uint16_t pu = 0;
            if (valid) {
                pu = src[e];
                d = (((__float_as_uint(s_w[pu]) & kStageOrigMask) - omin) >> shift) & (kRadixDigits - 1u);
            }
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            uint32_t base = 0;
            if (valid) {
                base = s_cnt[d * kWarps + warp];
                dst[base + __popc(peers & ((1u << lane) - 1u))] = pu;
            }
            __syncwarp();
            if (valid && lane == (uint32_t)(__ffs(peers) - 1)) s_cnt[d * kWarps + warp] = (uint16_t)(base + __popc(peers));
            __syncwarp();
        }
        __syncthreads();
        uint16_t* t = src;
        src = dst;
        dst = t;
    }
    if (src != s_sorted) {
        for (uint32_t i = tid; i < nf; i += blockDim.x) s_sorted[i] = src[i];
    }
    __syncthreads();
}

// Slow path of the visit list for a union larger than the stage.
template <int DIM, bool LOWER_FLAGS>
__device__ __forceinline__ void visit_slow(const StepConst& k, float r2f, const CellUnion& cu, uint32_t U,
                                           const StateBufs& s, const ListBufs& l, DeviceScalars* sc,
                                           const uint32_t* s_cstart, const uint32_t* s_off, uint32_t (*s_red)[2],
                                           ChunkBlock* s_blk, bool* s_overflow) {
    constexpr int NC = DIM == 3 ? 27 : 9;
    const uint32_t tid = threadIdx.x;
    // Slow path: a union larger than the stage, straight from global
    // memory, one thread per centre particle: count, reserve, write.
    if (tid == 0) atomicOr(&sc->status, kStatusSlowUnion);
    for (uint32_t c0 = 0; c0 < cu.ncenter; c0 += kNlThreads) {
        const uint32_t nc = min((uint32_t)kNlThreads, cu.ncenter - c0);
        const bool active = tid < nc;
        const uint32_t kslot = cu.cs + c0 + tid;
        uint8_t mfl = 0;
        uint32_t myo = 0;
        float4 me = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t nv = 0;
        bool fluidc = false;
        if (active) {
            me = stage_entry<DIM>(s, kslot, cu, &mfl, &myo);
            fluidc = !(mfl & kFlagBoundary);
            if (fluidc) {
                for (int c = 0; c < NC; ++c) {
                    const uint32_t q0 = s_cstart[c], q1 = q0 + (s_off[c + 1] - s_off[c]);
                    for (uint32_t slot = q0; slot < q1; ++slot) {
                        if (slot == kslot) continue;
                        uint8_t fl;
                        uint32_t o;
                        if (keep_entry(stage_entry<DIM>(s, slot, cu, &fl, &o), me, r2f, k.keep_boundary))
                            ++nv;
                    }
                }
            }
        }
        const ChunkBlock blk = reserve_chunk(l, sc, nc, nv, 0u, s_red, s_blk, s_overflow);
        if (active) {
            const uint32_t gv = (uint32_t)blk.base + tid;
            l.desc[kslot] = blk.ok ? make_uint4(gv, nc, nv, 0u) : make_uint4(0u, 0u, 0u, 0u);
            l.ncand[kslot] = fluidc ? U : 0u;
            if (blk.ok && fluidc) {
                const size_t step = 4u * nc;
                uint32_t* pv = l.pool + 4 * (size_t)gv;
                uint32_t tv = 0;
                for (int c = 0; c < NC; ++c) {
                    const uint32_t q0 = s_cstart[c], q1 = q0 + (s_off[c + 1] - s_off[c]);
                    for (uint32_t slot = q0; slot < q1; ++slot) {
                        if (slot == kslot) continue;
                        uint8_t fl;
                        uint32_t o;
                        const float4 qp = stage_entry<DIM>(s, slot, cu, &fl, &o);
                        if (!keep_entry(qp, me, r2f, k.keep_boundary)) continue;
                        uint32_t e = slot | entry_flags(__float_as_uint(qp.w));
                        if (LOWER_FLAGS && !(fl & kFlagBoundary) && o < myo) e |= kEntryLower;
                        if (tv < nv) pv[(tv >> 2) * step + (tv & 3u)] = e;
                        ++tv;
                    }
                }
            }
        }
        __syncthreads();
    }
}

// Slow path of the lower list for a union larger than the stage.
template <int DIM>
__device__ __forceinline__ void lower_slow(const StepConst& k, float r2f, const CellUnion& cu, const StateBufs& s,
                                           const ListBufs& l, DeviceScalars* sc, const uint32_t* s_cstart,
                                           const uint32_t* s_off, uint32_t (*s_red)[2], ChunkBlock* s_blk,
                                           bool* s_overflow) {
    constexpr int NC = DIM == 3 ? 27 : 9;
    const uint32_t tid = threadIdx.x;
    // Slow path: ascending original index by repeated selection, one
    // thread per centre particle: count, reserve, write.
    if (tid == 0) atomicOr(&sc->status, kStatusSlowUnion);
    for (uint32_t c0 = 0; c0 < cu.ncenter; c0 += kNlThreads) {
        const uint32_t nc = min((uint32_t)kNlThreads, cu.ncenter - c0);
        const bool active = tid < nc;
        const uint32_t kslot = cu.cs + c0 + tid;
        uint8_t mfl = 0;
        uint32_t myo = 0;
        float4 me = make_float4(0.f, 0.f, 0.f, 0.f);
        bool fluidc = false;
        uint32_t nl = 0;
        float r2c = r2f;
        if (active) {
            me = stage_entry<DIM>(s, kslot, cu, &mfl, &myo);
            fluidc = !(mfl & kFlagBoundary);
            if (!fluidc && k.keep_boundary) r2c = __int_as_float(0x7f800000);
            if (!(fluidc && k.lower_boundary_only)) {
                for (int c = 0; c < NC; ++c) {
                    const uint32_t q0 = s_cstart[c], q1 = q0 + (s_off[c + 1] - s_off[c]);
                    for (uint32_t slot = q0; slot < q1; ++slot) {
                        uint8_t fl;
                        uint32_t o;
                        const float4 qp = stage_entry<DIM>(s, slot, cu, &fl, &o);
                        if ((fl & kFlagBoundary) || (fluidc && o >= myo)) continue;
                        if (within(qp, me, r2c)) ++nl;
                    }
                }
            }
        }
        const ChunkBlock blk = reserve_chunk(l, sc, nc, nl, 0u, s_red, s_blk, s_overflow);
        if (active) {
            const uint32_t gl = (uint32_t)blk.base + tid;
            l.ldesc[kslot] = blk.ok ? make_uint2(gl, nl | (nc << 16)) : make_uint2(0u, 0u);
            if (blk.ok) {
                const size_t step = 4u * nc;
                uint32_t* pl = l.pool + 4 * (size_t)gl;
                uint32_t tl = 0;
                long long last = -1;
                while (tl < nl) {
                    unsigned long long best = ULLONG_MAX;
                    uint32_t best_slot = 0;
                    for (int c = 0; c < NC; ++c) {
                        const uint32_t q0 = s_cstart[c], q1 = q0 + (s_off[c + 1] - s_off[c]);
                        for (uint32_t slot = q0; slot < q1; ++slot) {
                            if (s.flags[slot] & kFlagBoundary) continue;
                            const uint32_t o = s.orig[slot];
                            if ((long long)o <= last || (fluidc && o >= myo) ||
                                (unsigned long long)o >= best)
                                continue;
                            uint8_t fl;
                            uint32_t oo;
                            if (within(stage_entry<DIM>(s, slot, cu, &fl, &oo), me, r2c)) {
                                best = o;
                                best_slot = slot;
                            }
                        }
                    }
                    if (best == ULLONG_MAX) break;
                    pl[(tl >> 2) * step + (tl & 3u)] = best_slot;
                    ++tl;
                    last = (long long)best;
                }
            }
        }
        __syncthreads();
    }
}

// ----------------------------------------------------------------- visit
// Dynamic shared memory (ucap a multiple of kStageStep): float x, y, z, w[ucap] (Stage);
// uint32 s_ent[ucap]; uint32 s_mask[(ucap / 32) * kChunk] (word w of chunk
// lane c at s_mask[w * kChunk + c]).
template <int DIM, bool LOWER_FLAGS, uint32_t kChunk>
__global__ void __launch_bounds__(kNlThreads) k_nlist_visit(GridDesc g, Tanks tk, StepConst k, uint32_t ucap,
                                                            const uint32_t* __restrict__ occ,
                                                            const uint32_t* __restrict__ cell_start,
                                                            StateBufs s, ListBufs l,
                                                            DeviceScalars* sc) {
    constexpr int NC = DIM == 3 ? 27 : 9;
    constexpr uint32_t kWays = kNlThreads / kChunk;
    extern __shared__ __align__(16) unsigned char smem[];
    Stage st(reinterpret_cast<float*>(smem), ucap);
    uint32_t* s_ent = reinterpret_cast<uint32_t*>(smem) + 4 * (size_t)ucap;
    uint32_t* s_mask = s_ent + ucap;
    __shared__ uint32_t s_cstart[NC];
    __shared__ uint32_t s_off[NC + 1];
    __shared__ uint32_t s_cv[kWays][kChunk];
    __shared__ uint32_t s_red[kWarps][2];
    __shared__ ChunkBlock s_blk;
    __shared__ bool s_overflow;

    const float r2f = k.r2_filter;
    const uint32_t nocc = sc->nocc;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid % kChunk, q = tid / kChunk;
    uint32_t max_union = 0;
    if (tid == 0) s_overflow = false;

    for (uint32_t it = blockIdx.x; it < nocc; it += gridDim.x) {
        const CellUnion cu = cell_union<DIM>(g, tk, occ[it], cell_start, s_cstart, s_off);
        const uint32_t U = cu.U;
        max_union = max(max_union, U);
        if (U <= ucap) {
            for (uint32_t u = tid; u < U; u += blockDim.x) {
                const uint32_t slot = slot_of_union<NC>(s_off, s_cstart, u);
                uint8_t fl;
                uint32_t o;
                const float4 p = stage_entry<DIM>(s, slot, cu, &fl, &o);
                st.put(u, p);
                s_ent[u] = slot | entry_flags(__float_as_uint(p.w));
            }
            __syncthreads();
            const uint32_t W = (U + 31u) >> 5;
            const uint32_t wb = W * q / kWays, we = W * (q + 1) / kWays;
            for (uint32_t c0 = 0; c0 < cu.ncenter; c0 += kChunk) {
                const uint32_t nc = min(kChunk, cu.ncenter - c0);
                const bool active = lane < nc;
                const uint32_t myu = cu.center_off + c0 + lane;
                bool fluidc = false;
                uint32_t myo = 0;
                // ---- pass 1: in-support masks of this quarter's words, counts
                if (active) {
                    const float4 me = st.get(myu);
                    const uint32_t mw = __float_as_uint(me.w);
                    fluidc = !(mw & kStageBoundary);
                    myo = mw & kStageOrigMask;
                    uint32_t cv = 0;
                    if (fluidc) {
                        for (uint32_t w = wb; w < we; ++w) {
                            uint32_t m = k.keep_boundary ? word_mask<true>(st, w << 5, me, r2f)
                                                         : word_mask<false>(st, w << 5, me, r2f);
                            if (w == W - 1u && (U & 31u)) m &= (1u << (U & 31u)) - 1u;
                            if (w == (myu >> 5)) m &= ~(1u << (myu & 31u));
                            s_mask[w * kChunk + lane] = m;
                            cv += __popc(m);
                        }
                    }
                    s_cv[q][lane] = cv;
                }
                __syncthreads();
                // ---- list lengths and the chunk's block
                uint32_t nv = 0;
                if (active) {
#pragma unroll
                    for (uint32_t r = 0; r < kWays; ++r) nv += s_cv[r][lane];
                }
                const ChunkBlock blk = reserve_chunk(l, sc, nc, nv, 0u, s_red, &s_blk, &s_overflow);
                // ---- pass 2: descriptors and entries
                if (active) {
                    const uint32_t kslot = cu.cs + c0 + lane;
                    const uint32_t gv = (uint32_t)blk.base + lane;  // < pool_groups < 2^32 when ok
                    if (q == 0) {
                        l.desc[kslot] = blk.ok ? make_uint4(gv, nc, nv, 0u) : make_uint4(0u, 0u, 0u, 0u);
                        l.ncand[kslot] = fluidc ? U : 0u;
                    }
                    // entries split evenly over the centre's threads
                    const uint32_t v0 = nv * q / kWays, v1 = nv * (q + 1u) / kWays;
                    if (blk.ok && fluidc && v0 < v1) {
                        const size_t step = 4u * nc;
                        uint32_t* pv = l.pool + 4 * (size_t)gv;
                        MaskCursor<kChunk> cur(s_mask, s_cv, lane, W, v0);
                        for (uint32_t t = v0; t < v1; ++t) {
                            const uint32_t u = cur.next();
                            uint32_t e = s_ent[u];
                            if (LOWER_FLAGS) {
                                const uint32_t ow = st.word(u);
                                e |= ow < myo ? kEntryLower : 0u;  // a boundary word has bit 31 set
                            }
                            pv[(t >> 2) * step + (t & 3u)] = e;
                        }
                    }
                }
                __syncthreads();  // masks and counts are reused by the next chunk
            }
        } else {
            visit_slow<DIM, LOWER_FLAGS>(k, r2f, cu, U, s, l, sc, s_cstart, s_off, s_red, &s_blk, &s_overflow);
        }
        __syncthreads();  // shared memory is reused by the next cell
    }
    if (tid == 0 && s_overflow) atomicOr(&sc->status, kStatusListOverflow);
    if (tid == 0 && max_union) atomicMax(&sc->max_union, max_union);
}

// ----------------------------------------------------------------- both
// One pass per occupied cell for both lists: the union is staged once, the
// visit masks of a chunk's fluid centres are computed once, and a fluid
// centre's lower list is read out of its own visit mask in ascending original
// index (through the radix-sorted fluid positions); boundary centres test the
// sorted fluid positions directly. One reservation per chunk holds both lists
// (visit rows first). Dynamic shared memory: float x, y, z, w[ucap] (Stage); uint32
// s_ent[ucap] (slot | flags); uint32 s_vmask[(ucap / 32) * kChunk]; uint16
// s_sorted[ucap]; then a region used first by the radix sort and then by the
// lower masks over sorted positions.
template <int DIM, uint32_t kChunk>
__global__ void __launch_bounds__(kNlThreads, 3) k_nlist_both(GridDesc g, Tanks tk, StepConst k, uint32_t ucap,
                                                           const uint32_t* __restrict__ occ,
                                                           const uint32_t* __restrict__ cell_start,
                                                           StateBufs s, ListBufs l, DeviceScalars* sc) {
    constexpr int NC = DIM == 3 ? 27 : 9;
    constexpr uint32_t kWays = kNlThreads / kChunk;
    extern __shared__ __align__(16) unsigned char smem[];
    Stage st(reinterpret_cast<float*>(smem), ucap);
    uint32_t* s_ent = reinterpret_cast<uint32_t*>(smem) + 4 * (size_t)ucap;
    uint32_t* s_vmask = s_ent + ucap;
    uint16_t* s_sorted = reinterpret_cast<uint16_t*>(s_vmask + (ucap / 32) * kChunk);
    uint32_t* s_lmask = reinterpret_cast<uint32_t*>(s_sorted + ucap);
    uint16_t* s_tmp = reinterpret_cast<uint16_t*>(s_lmask);
    uint16_t* s_cnt = s_tmp + ucap;
    __shared__ uint32_t s_cstart[NC];
    __shared__ uint32_t s_off[NC + 1];
    __shared__ uint32_t s_nf, s_omin, s_omax;
    __shared__ uint32_t s_cv[kWays][kChunk], s_cl[kWays][kChunk];
    __shared__ uint32_t s_red[kWarps][2];
    __shared__ ChunkBlock s_blk;
    __shared__ bool s_overflow;

    const float r2f = k.r2_filter;
    const uint32_t nocc = sc->nocc;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid % kChunk, q = tid / kChunk;
    uint32_t max_union = 0;
    if (tid == 0) s_overflow = false;

    for (uint32_t it = blockIdx.x; it < nocc; it += gridDim.x) {
        if (tid == 0) {
            s_nf = 0;
            s_omin = 0xffffffffu;
            s_omax = 0u;
        }
        const CellUnion cu = cell_union<DIM>(g, tk, occ[it], cell_start, s_cstart, s_off);
        const uint32_t U = cu.U;
        max_union = max(max_union, U);
        if (U <= ucap) {
            // Stage the union; fluid entries are appended to s_sorted with one
            // shared atomic per warp, their index range reduced per warp.
            uint32_t tmin = 0xffffffffu, tmax = 0u;
            for (uint32_t u0 = 0; u0 < U; u0 += blockDim.x) {
                const uint32_t u = u0 + tid;
                bool fluid = false;
                if (u < U) {
                    const uint32_t slot = slot_of_union<NC>(s_off, s_cstart, u);
                    uint8_t fl;
                    uint32_t o;
                    const float4 p = stage_entry<DIM>(s, slot, cu, &fl, &o);
                    st.put(u, p);
                    s_ent[u] = slot | entry_flags(__float_as_uint(p.w));
                    fluid = !(fl & kFlagBoundary);
                    if (fluid) {
                        tmin = min(tmin, o);
                        tmax = max(tmax, o);
                    }
                }
                const uint32_t fm = __ballot_sync(0xffffffffu, fluid);
                uint32_t base = 0;
                if ((tid & 31u) == 0 && fm) base = atomicAdd(&s_nf, (uint32_t)__popc(fm));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (fluid) s_sorted[base + __popc(fm & ((1u << (tid & 31u)) - 1u))] = (uint16_t)u;
            }
            tmin = __reduce_min_sync(0xffffffffu, tmin);
            tmax = __reduce_max_sync(0xffffffffu, tmax);
            if ((tid & 31u) == 0 && tmin <= tmax) {
                atomicMin(&s_omin, tmin);
                atomicMax(&s_omax, tmax);
            }
            __syncthreads();
            const uint32_t nf = s_nf;
            radix_sort_by_orig(st.w, s_sorted, s_tmp, s_cnt, nf, s_omin, s_omax);
            // sorted positions past nf up to the next multiple of 32 read as
            // union position 0: the lower-mask pass reads whole words (their
            // bits past a centre's prefix are cleared)
            for (uint32_t i = nf + tid; i < ((nf + 31u) & ~31u); i += blockDim.x) s_sorted[i] = 0;
            __syncthreads();
            const uint32_t W = (U + 31u) >> 5;
            const uint32_t wb = W * q / kWays, we = W * (q + 1) / kWays;
            for (uint32_t c0 = 0; c0 < cu.ncenter; c0 += kChunk) {
                const uint32_t nc = min(kChunk, cu.ncenter - c0);
                const bool active = lane < nc;
                const uint32_t myu = cu.center_off + c0 + lane;
                bool fluidc = false;
                uint32_t myo = 0, R = 0;
                float4 me = make_float4(0.f, 0.f, 0.f, 0.f);
                // ---- pass 1a: visit masks of this quarter's union words (fluid centres)
                if (active) {
                    me = st.get(myu);
                    const uint32_t mw = __float_as_uint(me.w);
                    fluidc = !(mw & kStageBoundary);
                    myo = mw & kStageOrigMask;
                    uint32_t cv = 0;
                    if (fluidc) {
                        for (uint32_t w = wb; w < we; ++w) {
                            uint32_t m = k.keep_boundary ? word_mask<true>(st, w << 5, me, r2f)
                                                         : word_mask<false>(st, w << 5, me, r2f);
                            if (w == W - 1u && (U & 31u)) m &= (1u << (U & 31u)) - 1u;
                            if (w == (myu >> 5)) m &= ~(1u << (myu & 31u));
                            s_vmask[w * kChunk + lane] = m;
                            cv += __popc(m);
                        }
                    }
                    s_cv[q][lane] = cv;
                    // R = sorted fluid positions below this particle's index
                    // (all of them for a boundary particle)
                    if (!fluidc) {
                        R = nf;
                    } else if (!k.lower_boundary_only) {
                        uint32_t lo = 0, hi = nf;
                        while (lo < hi) {
                            const uint32_t mid = (lo + hi) >> 1;
                            const uint32_t o = st.word(s_sorted[mid]) & kStageOrigMask;
                            if (o < myo) lo = mid + 1;
                            else hi = mid;
                        }
                        R = lo;
                    }
                }
                __syncthreads();  // every quarter's visit words are in place
                // ---- pass 1b: lower masks of this quarter's sorted words
                const uint32_t WR = (R + 31u) >> 5;
                const uint32_t lb = WR * q / kWays, le = WR * (q + 1) / kWays;
                if (active) {
                    const float r2c = (!fluidc && k.keep_boundary) ? __int_as_float(0x7f800000) : r2f;
                    uint32_t cl = 0;
                    for (uint32_t w = lb; w < le; ++w) {
                        uint32_t m = 0;
                        if (fluidc) {
                            const uint4* sw = reinterpret_cast<const uint4*>(s_sorted + (w << 5));
#pragma unroll
                            for (int v = 0; v < 4; ++v) {
                                const uint4 x = sw[v];
                                const uint32_t pr[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
                                for (int h = 0; h < 8; ++h) {
                                    const uint32_t u = (pr[h >> 1] >> ((h & 1) * 16)) & 0xffffu;
                                    m |= ((s_vmask[(u >> 5) * kChunk + lane] >> (u & 31u)) & 1u) << (v * 8 + h);
                                }
                            }
                        } else {
#pragma unroll
                            for (int bit = 0; bit < 32; ++bit) {
                                const uint32_t i = (w << 5) + bit;
                                m |= within(st.get(s_sorted[i]), me, r2c) ? (1u << bit) : 0u;
                            }
                        }
                        if (w == WR - 1u && (R & 31u)) m &= (1u << (R & 31u)) - 1u;
                        s_lmask[w * kChunk + lane] = m;
                        cl += __popc(m);
                    }
                    s_cl[q][lane] = cl;
                }
                __syncthreads();
                // ---- list lengths and the chunk's block
                uint32_t nv = 0, nl = 0;
                if (active) {
#pragma unroll
                    for (uint32_t r = 0; r < kWays; ++r) {
                        nv += s_cv[r][lane];
                        nl += s_cl[r][lane];
                    }
                }
                const ChunkBlock blk = reserve_chunk(l, sc, nc, nv, nl, s_red, &s_blk, &s_overflow);
                // ---- pass 2: descriptors and entries
                if (active) {
                    const uint32_t kslot = cu.cs + c0 + lane;
                    const uint32_t gv = (uint32_t)blk.base + lane;  // < pool_groups < 2^32 when ok
                    const uint32_t gl = (uint32_t)(blk.base + (unsigned long long)blk.rows_a * nc) + lane;
                    if (q == 0) {
                        l.desc[kslot] = blk.ok ? make_uint4(gv, nc, nv, 0u) : make_uint4(0u, 0u, 0u, 0u);
                        l.ncand[kslot] = fluidc ? U : 0u;
                        l.ldesc[kslot] = blk.ok ? make_uint2(gl, nl | (nc << 16)) : make_uint2(0u, 0u);
                    }
                    if (blk.ok) {
                        const size_t step = 4u * nc;
                        // Entries are split evenly over the centre's threads
                        // (split by words, the middle ways would hold most of
                        // the kept candidates).
                        const uint32_t v0 = nv * q / kWays, v1 = nv * (q + 1u) / kWays;
                        if (fluidc && v0 < v1) {
                            uint32_t* pv = l.pool + 4 * (size_t)gv;
                            MaskCursor<kChunk> cur(s_vmask, s_cv, lane, W, v0);
                            for (uint32_t t = v0; t < v1; ++t) {
                                const uint32_t u = cur.next();
                                uint32_t e = s_ent[u];
                                const uint32_t ow = st.word(u);
                                e |= ow < myo ? kEntryLower : 0u;  // a boundary word has bit 31 set
                                pv[(t >> 2) * step + (t & 3u)] = e;
                            }
                        }
                        const uint32_t l0 = nl * q / kWays, l1 = nl * (q + 1u) / kWays;
                        if (l0 < l1) {
                            uint32_t* pl = l.pool + 4 * (size_t)gl;
                            MaskCursor<kChunk> cur(s_lmask, s_cl, lane, WR, l0);
                            for (uint32_t t = l0; t < l1; ++t)
                                pl[(t >> 2) * step + (t & 3u)] = s_ent[s_sorted[cur.next()]] & kEntrySlotMask;
                        }
                    }
                }
                __syncthreads();  // masks and counts are reused by the next chunk
            }
        } else {
            visit_slow<DIM, true>(k, r2f, cu, U, s, l, sc, s_cstart, s_off, s_red, &s_blk, &s_overflow);
            lower_slow<DIM>(k, r2f, cu, s, l, sc, s_cstart, s_off, s_red, &s_blk, &s_overflow);
        }
        __syncthreads();  // shared memory is reused by the next cell
    }
    if (tid == 0 && s_overflow) atomicOr(&sc->status, kStatusListOverflow);
    if (tid == 0 && max_union) atomicMax(&sc->max_union, max_union);
}

size_t both_smem_bytes(uint32_t ucap, uint32_t chunk) {
    const size_t sort = (size_t)ucap * sizeof(uint16_t) + 16 * kNlThreads * sizeof(uint16_t);
    const size_t mask = (size_t)(ucap / 32) * chunk * sizeof(uint32_t);
    return (size_t)ucap * (sizeof(float4) + sizeof(uint32_t) + sizeof(uint16_t)) + mask + (sort > mask ? sort : mask);
}

size_t visit_smem_bytes(uint32_t ucap, uint32_t chunk) {
    return (size_t)ucap * (sizeof(float4) + sizeof(uint32_t)) + (size_t)(ucap / 32) * chunk * sizeof(uint32_t);
}

uint32_t valid_chunk(uint32_t chunk) { return chunk == 32u ? 32u : kDefaultChunk; }

}  // namespace

uint32_t nlist_union_capacity(uint32_t max_union) {
    // The largest union seen plus an eighth, in steps of kStageStep, within
    // the shared-memory limit; larger unions take the slow path. The margin
    // is kept small so that three CTAs of the fused kernel fit an SM at the
    // 32-centre tile (at 1M: a 2,304-entry stage, 75 KB per CTA; with a
    // quarter's margin the stage was 2,560 entries and two CTAs fit).
    uint64_t want = (uint64_t)max_union + max_union / 8u;
    want = (want + kStageStep - 1) / kStageStep * kStageStep;
    if (want < kStageStep) want = kStageStep;
    if (want > kMaxUnionStage) want = kMaxUnionStage;
    return (uint32_t)want;
}

size_t nlist_smem_bytes(uint32_t ucap, uint32_t chunk) {
    chunk = valid_chunk(chunk);
    const size_t a = visit_smem_bytes(ucap, chunk), b = both_smem_bytes(ucap, chunk);
    return a > b ? a : b;
}

namespace {
template <int DIM, uint32_t C>
uint32_t prepare_for(uint32_t ucap) {
    const int sv = (int)visit_smem_bytes(ucap, C), sb = (int)both_smem_bytes(ucap, C);
    int bv = 0, bb = 0;
    cudaFuncSetAttribute(k_nlist_visit<DIM, false, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, sv);
    cudaFuncSetAttribute(k_nlist_both<DIM, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, sb);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bv, k_nlist_visit<DIM, false, C>, kNlThreads, sv);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bb, k_nlist_both<DIM, C>, kNlThreads, sb);
    const int b = bv > bb ? bv : bb;
    return b > 0 ? (uint32_t)b : 1u;
}

template <int DIM, uint32_t C>
void launch_for(const GridDesc& g, const Tanks& tk, const StepConst& k, uint32_t ucap, uint32_t nblocks,
                const uint32_t* occ, const uint32_t* cell_start, const StateBufs& s, const ListBufs& l,
                DeviceScalars* sc, cudaStream_t st, bool visit_only) {
    if (visit_only)
        k_nlist_visit<DIM, false, C><<<nblocks, kNlThreads, visit_smem_bytes(ucap, C), st>>>(
            g, tk, k, ucap, occ, cell_start, s, l, sc);
    else
        k_nlist_both<DIM, C><<<nblocks, kNlThreads, both_smem_bytes(ucap, C), st>>>(g, tk, k, ucap, occ,
                                                                                  cell_start, s, l, sc);
}
}  // namespace

uint32_t nlist_prepare(int dim, uint32_t ucap, uint32_t chunk) {
    chunk = valid_chunk(chunk);
    if (dim == 3) return chunk == 32u ? prepare_for<3, 32>(ucap) : prepare_for<3, 64>(ucap);
    return chunk == 32u ? prepare_for<2, 32>(ucap) : prepare_for<2, 64>(ucap);
}

void launch_nlist(const GridDesc& g, const Tanks& tk, const StepConst& k, uint32_t ucap,
                  uint32_t nblocks, const uint32_t* occ, const uint32_t* cell_start,
                  const StateBufs& s, const ListBufs& l, DeviceScalars* sc, cudaStream_t st,
                  bool visit_only, uint32_t chunk) {
    chunk = valid_chunk(chunk);
    if (g.dim == 3) {
        if (chunk == 32u) launch_for<3, 32>(g, tk, k, ucap, nblocks, occ, cell_start, s, l, sc, st, visit_only);
        else launch_for<3, 64>(g, tk, k, ucap, nblocks, occ, cell_start, s, l, sc, st, visit_only);
    } else {
        if (chunk == 32u) launch_for<2, 32>(g, tk, k, ucap, nblocks, occ, cell_start, s, l, sc, st, visit_only);
        else launch_for<2, 64>(g, tk, k, ucap, nblocks, occ, cell_start, s, l, sc, st, visit_only);
    }
}

}  // namespace pe
