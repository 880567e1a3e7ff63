// Deterministic uniform-grid build (replaces `UniformGrid::rebuild`,
// crates/pe-fluid/src/grid.rs:76-107, and `key_of`, grid.rs:62).
//
// The reference sorts particle indices by (CellKey, index) with a comparison
// sort. Here the same total order is produced by a counting sort over a dense
// key box: cell ids are computed with the reference's exact floor_i32 rule,
// counted with warp-aggregated atomics, scanned, placed with warp-aggregated
// atomics, and each cell's run is then ranked by original index so that the
// within-cell order is ascending original index, exactly as the reference's
// tie-break. The dense linearisation is ix-major, so ascending linear cell id
// equals ascending CellKey (the derived Ord on {ix, iy, iz}).
#include "pe_math.cuh"
#include "wcsph_device.cuh"

namespace pe {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__global__ void k_cell_ids(GridDesc g, Tanks tk, uint32_t n, const double4* __restrict__ pos_cur,
                           const double4* __restrict__ pos_next, const uint8_t* __restrict__ flags,
                           uint32_t* __restrict__ cellid, int4* __restrict__ key_tmp,
                           uint32_t* __restrict__ count, DeviceScalars* sc) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    bool active = s < n;
    uint32_t c = 0;
    if (active) {
        bool boundary = flags[s] & kFlagBoundary;
        double4 p = (pos_next != nullptr && !boundary) ? pos_next[s] : pos_cur[s];
        // grid.rs:63-70: inv = 1.0 / cell_size; key = floor_i32(p * inv)
        int32_t ix = floor_i32(p.x * g.inv_cell);
        int32_t iy = floor_i32(p.y * g.inv_cell);
        int32_t iz = g.dim == 2 ? 0 : floor_i32(p.z * g.inv_cell);
        if (!isfinite(p.x) || !isfinite(p.y) || (g.dim == 3 && !isfinite(p.z)))
            atomicOr(&sc->status, kStatusNonFinite);
        key_tmp[s] = make_int4(ix, iy, iz, 0);
        // the box of this slot's tank (slots keep their tank across re-sorts)
        TankDesc td;
        if (tk.desc) {
            td = tk.desc[tk.slot_tank[s]];
        } else {
            td.kx0 = g.kx0;
            td.ky0 = g.ky0;
            td.kz0 = g.kz0;
            td.nx = g.nx;
            td.ny = g.ny;
            td.nz = g.nz;
            td.cell_base = 0;
        }
        long long dx = (long long)ix - td.kx0, dy = (long long)iy - td.ky0, dz = (long long)iz - td.kz0;
        if (dx < 0 || dy < 0 || dz < 0 || dx >= td.nx || dy >= td.ny || dz >= td.nz) {
            atomicOr(&sc->status, kStatusDomain);
            dx = dx < 0 ? 0 : (dx >= td.nx ? td.nx - 1 : dx);
            dy = dy < 0 ? 0 : (dy >= td.ny ? td.ny - 1 : dy);
            dz = dz < 0 ? 0 : (dz >= td.nz ? td.nz - 1 : dz);
        }
        c = td.cell_base + (uint32_t)((dx * td.ny + dy) * td.nz + dz);
        cellid[s] = c;
    }
    unsigned mask = __ballot_sync(0xffffffffu, active);
    if (active) {
        unsigned peers = __match_any_sync(mask, c);
        if ((int)lane_id() == __ffs(peers) - 1) atomicAdd(&count[c], (uint32_t)__popc(peers));
    }
}

// Block-wide exclusive scan of (a, b) pairs with warp shuffles.
__device__ __forceinline__ void block_scan2(uint32_t a, uint32_t b, uint32_t* ea, uint32_t* eb,
                                            uint32_t* ta, uint32_t* tb) {
    __shared__ uint32_t wa[32], wb[32];
    uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t ia = a, ib = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t xa = __shfl_up_sync(0xffffffffu, ia, o);
        uint32_t xb = __shfl_up_sync(0xffffffffu, ib, o);
        if ((int)lane >= o) { ia += xa; ib += xb; }
    }
    if (lane == 31) { wa[warp] = ia; wb[warp] = ib; }
    __syncthreads();
    if (warp == 0) {
        uint32_t nw = blockDim.x >> 5;
        uint32_t va = lane < nw ? wa[lane] : 0u, vb = lane < nw ? wb[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t xa = __shfl_up_sync(0xffffffffu, va, o);
            uint32_t xb = __shfl_up_sync(0xffffffffu, vb, o);
            if ((int)lane >= o) { va += xa; vb += xb; }
        }
        wa[lane] = va;
        wb[lane] = vb;
    }
    __syncthreads();
    uint32_t pa = warp ? wa[warp - 1] : 0u, pb = warp ? wb[warp - 1] : 0u;
    *ea = pa + ia - a;
    *eb = pb + ib - b;
    *ta = wa[(blockDim.x >> 5) - 1];
    *tb = wb[(blockDim.x >> 5) - 1];
    __syncthreads();
}

// Pass 1: per-tile totals of (particles, occupied cells).
__global__ void k_scan_reduce(uint32_t ncell, const uint32_t* __restrict__ count,
                              uint2* __restrict__ tile_sums) {
    uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t a = 0, b = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        uint32_t c = base + i;
        uint32_t v = c < ncell ? count[c] : 0u;
        a += v;
        b += v != 0u;
    }
    uint32_t ea, eb, ta, tb;
    block_scan2(a, b, &ea, &eb, &ta, &tb);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = make_uint2(ta, tb);
}

// Pass 2: exclusive scan of the tile totals (one block, any tile count).
__global__ void k_scan_top(uint32_t ntiles, uint2* __restrict__ tile_sums, DeviceScalars* sc) {
    uint32_t carry_a = 0, carry_b = 0;
    for (uint32_t off = 0; off < ntiles; off += blockDim.x) {
        uint32_t i = off + threadIdx.x;
        uint2 v = i < ntiles ? tile_sums[i] : make_uint2(0u, 0u);
        uint32_t ea, eb, ta, tb;
        block_scan2(v.x, v.y, &ea, &eb, &ta, &tb);
        if (i < ntiles) tile_sums[i] = make_uint2(carry_a + ea, carry_b + eb);
        carry_a += ta;
        carry_b += tb;
    }
    if (threadIdx.x == 0) sc->nocc = carry_b;
}

// Pass 3: cell_start (exclusive) and the list of occupied cells in linear order.
__global__ void k_scan_down(uint32_t ncell, const uint32_t* __restrict__ count,
                            const uint2* __restrict__ tile_sums, uint32_t* __restrict__ cell_start,
                            uint32_t* __restrict__ occ) {
    uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t a = 0, b = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        uint32_t c = base + i;
        v[i] = c < ncell ? count[c] : 0u;
        a += v[i];
        b += v[i] != 0u;
    }
    uint32_t ea, eb, ta, tb;
    block_scan2(a, b, &ea, &eb, &ta, &tb);
    uint2 off = tile_sums[blockIdx.x];
    uint32_t ra = off.x + ea, rb = off.y + eb;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        uint32_t c = base + i;
        if (c < ncell) {
            cell_start[c] = ra;
            if (v[i]) occ[rb++] = c;
            ra += v[i];
        }
    }
    // The thread that owns the last cell writes the end sentinel.
    if (ncell > 0 && base <= ncell - 1 && ncell - 1 < base + kScanItems) cell_start[ncell] = ra;
}

__global__ void k_place(uint32_t n, const uint32_t* __restrict__ cellid,
                        const uint32_t* __restrict__ cell_start, uint32_t* __restrict__ fill,
                        const uint32_t* __restrict__ orig, uint32_t* __restrict__ tmp_old,
                        uint32_t* __restrict__ tmp_orig) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    bool active = s < n;
    uint32_t c = active ? cellid[s] : 0u;
    unsigned mask = __ballot_sync(0xffffffffu, active);
    if (!active) return;
    unsigned peers = __match_any_sync(mask, c);
    int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(&fill[c], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    uint32_t rank = __popc(peers & ((1u << lane_id()) - 1u));
    uint32_t pos = cell_start[c] + base + rank;
    tmp_old[pos] = s;
    tmp_orig[pos] = orig[s];
}

// One warp per occupied cell: rank each entry by original index (unique), so
// the cell's run ends up in ascending original index (grid.rs:86-87 tie-break).
__global__ void k_cellsort(const uint32_t* __restrict__ occ, const DeviceScalars* sc,
                           const uint32_t* __restrict__ cell_start,
                           const uint32_t* __restrict__ tmp_old,
                           const uint32_t* __restrict__ tmp_orig, uint32_t* __restrict__ perm) {
    uint32_t nocc = sc->nocc;
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    uint32_t lane = lane_id();
    for (uint32_t i = warp; i < nocc; i += nwarps) {
        uint32_t c = occ[i];
        uint32_t start = cell_start[c];
        uint32_t n = cell_start[c + 1] - start;
        if (n <= 32u) {
            uint32_t mine = lane < n ? tmp_orig[start + lane] : 0xffffffffu;
            uint32_t rank = 0;
            for (uint32_t f = 0; f < n; ++f) {
                uint32_t o = __shfl_sync(0xffffffffu, mine, f);
                rank += o < mine;
            }
            if (lane < n) perm[start + rank] = tmp_old[start + lane];
        } else {
            for (uint32_t e0 = 0; e0 < n; e0 += 32u) {
                uint32_t e = e0 + lane;
                uint32_t mine = e < n ? tmp_orig[start + e] : 0xffffffffu;
                uint32_t rank = 0;
                for (uint32_t f = 0; f < n; ++f) rank += tmp_orig[start + f] < mine;
                if (e < n) perm[start + rank] = tmp_old[start + e];
            }
        }
    }
}

__global__ void k_gather(uint32_t n, const uint32_t* __restrict__ perm, StateBufs src,
                         const double4* __restrict__ pos_next, const double4* __restrict__ vel_next,
                         const int4* __restrict__ key_tmp, StateBufs dst,
                         uint32_t* __restrict__ slot_of_orig) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t old = perm[s];
    uint8_t fl = src.flags[old];
    bool moved = !(fl & kFlagBoundary);
    dst.pos[s] = (moved && pos_next) ? pos_next[old] : src.pos[old];
    dst.vel[s] = (moved && vel_next) ? vel_next[old] : src.vel[old];
    dst.acc[s] = src.acc[old];
    dst.bf[s] = src.bf[old];
    dst.p[s] = src.p[old];
    dst.flags[s] = fl;
    uint32_t o = src.orig[old];
    dst.orig[s] = o;
    dst.nout[s] = src.nout[old];
    dst.key[s] = key_tmp[old];
    slot_of_orig[o] = s;
}

__global__ void k_occupied_export(const uint32_t* __restrict__ occ, const DeviceScalars* sc,
                                  const uint32_t* __restrict__ cell_start,
                                  const int4* __restrict__ key, int32_t* __restrict__ occ_keys,
                                  uint64_t* __restrict__ ranges) {
    uint32_t nocc = sc->nocc;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nocc; i += gridDim.x * blockDim.x) {
        uint32_t c = occ[i];
        uint32_t a = cell_start[c], b = cell_start[c + 1];
        int4 k = key[a];
        occ_keys[3 * (size_t)i] = k.x;
        occ_keys[3 * (size_t)i + 1] = k.y;
        occ_keys[3 * (size_t)i + 2] = k.z;
        ranges[2 * (size_t)i] = a;
        ranges[2 * (size_t)i + 1] = b;
    }
}

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

}  // namespace

void launch_cell_ids(const GridDesc& g, const Tanks& tk, uint32_t n, const double4* pos_cur,
                     const double4* pos_next, const uint8_t* flags, uint32_t* cellid, int4* key_tmp,
                     uint32_t* count, DeviceScalars* sc, cudaStream_t st) {
    if (n == 0) return;
    k_cell_ids<<<blocks_for(n, 256), 256, 0, st>>>(g, tk, n, pos_cur, pos_next, flags, cellid, key_tmp,
                                                  count, sc);
}

size_t scan_temp_bytes(uint32_t ncell) {
    return sizeof(uint2) * (size_t)((ncell + kScanTile - 1) / kScanTile + 1);
}

void launch_scan_cells(uint32_t ncell, const uint32_t* count, uint32_t* cell_start, uint32_t* occ,
                       DeviceScalars* sc, void* temp, cudaStream_t st) {
    uint32_t ntiles = (ncell + kScanTile - 1) / kScanTile;
    uint2* tiles = static_cast<uint2*>(temp);
    k_scan_reduce<<<ntiles, kScanThreads, 0, st>>>(ncell, count, tiles);
    k_scan_top<<<1, kScanThreads, 0, st>>>(ntiles, tiles, sc);
    k_scan_down<<<ntiles, kScanThreads, 0, st>>>(ncell, count, tiles, cell_start, occ);
}

void launch_place(uint32_t n, const uint32_t* cellid, const uint32_t* cell_start, uint32_t* fill,
                  const uint32_t* orig, uint32_t* tmp_old, uint32_t* tmp_orig, cudaStream_t st) {
    if (n == 0) return;
    k_place<<<blocks_for(n, 256), 256, 0, st>>>(n, cellid, cell_start, fill, orig, tmp_old, tmp_orig);
}

void launch_cellsort(uint32_t ncell_max, const uint32_t* occ, const DeviceScalars* sc,
                     const uint32_t* cell_start, const uint32_t* tmp_old, const uint32_t* tmp_orig,
                     uint32_t* perm, cudaStream_t st) {
    uint32_t warps = ncell_max < 148u * 64u ? ncell_max : 148u * 64u;
    if (warps == 0) return;
    k_cellsort<<<blocks_for((uint64_t)warps * 32u, 256), 256, 0, st>>>(occ, sc, cell_start, tmp_old,
                                                                       tmp_orig, perm);
}

void launch_gather(uint32_t n, const uint32_t* perm, const StateBufs& src, const double4* pos_next,
                   const double4* vel_next, const int4* key_tmp, const StateBufs& dst,
                   uint32_t* slot_of_orig, double /*rho0*/, cudaStream_t st) {
    if (n == 0) return;
    k_gather<<<blocks_for(n, 256), 256, 0, st>>>(n, perm, src, pos_next, vel_next, key_tmp, dst,
                                                slot_of_orig);
}

void launch_occupied_export(const GridDesc& g, const uint32_t* occ, const DeviceScalars* sc,
                            const uint32_t* cell_start, const int4* key, int32_t* occ_keys,
                            uint64_t* ranges, cudaStream_t st) {
    uint32_t blocks = blocks_for(g.ncell, 256);
    if (blocks > 148u * 8u) blocks = 148u * 8u;
    if (blocks == 0) blocks = 1;
    k_occupied_export<<<blocks, 256, 0, st>>>(occ, sc, cell_start, key, occ_keys, ranges);
}

}  // namespace pe
