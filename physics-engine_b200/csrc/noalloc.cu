// pe_fluid_density_noalloc: the density pass (grid rebuild followed by the
// density summation of wcsph.rs:102-154, cubic-spline kernel) for callers that
// cannot allocate device memory — applications that hand the library a fixed
// device budget or manage every device allocation through their own
// allocator, and real-time loops that must not pay cudaMalloc's device-wide
// synchronisation.
//
// All working memory is one file-scope __device__ array of kScratchBytes. The
// caller passes inputs and the output in its own device memory; this path
// calls no cudaMalloc, cudaFree or allocating library routine.
//
// Host code must not take the array's name as a device address: every call
// looks the address up with cudaGetSymbolAddress (with the caller's device
// current), checks it, and passes it to every kernel. The lookup allocates
// nothing, and it is not cached, so a context that was torn down and created
// again (cudaDeviceReset) never sees the previous context's address.
// Every call on a device shares the one array and leaves its contents
// behind: the counters that must start at zero are cleared on each call, and
// calls that overlap on the GPU (different streams, or threads without
// ordering) race on it — serialise them.
#include <cmath>
#include <cstdint>

#include "../../include/pe_fluid_wcsph.h"
#include "pe_math.cuh"
#include "sph_pair.cuh"
#include "wcsph_device.cuh"

namespace pe {

namespace {

constexpr uint64_t kMaxN = PE_FLUID_NOALLOC_MAX_PARTICLES;
constexpr uint64_t kMaxCells = PE_FLUID_NOALLOC_MAX_CELLS;

struct NoAllocHeader {
    DeviceScalars sc;
    int32_t kmin[3], kmax[3];
    uint32_t nonfinite;
};

// Layout of the scratch array (offsets in bytes, each 256-aligned).
constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kOffHeader = 0;
constexpr size_t kOffPos = align256(sizeof(NoAllocHeader));           // double4[kMaxN] (orig order)
constexpr size_t kOffFlags = kOffPos + align256(kMaxN * 32);           // uint8[kMaxN]
constexpr size_t kOffOrig = kOffFlags + align256(kMaxN);               // uint32[kMaxN]
constexpr size_t kOffCellId = kOffOrig + align256(kMaxN * 4);          // uint32[kMaxN]
constexpr size_t kOffKey = kOffCellId + align256(kMaxN * 4);           // int4[kMaxN]
constexpr size_t kOffTmpOld = kOffKey + align256(kMaxN * 16);          // uint32[kMaxN]
constexpr size_t kOffTmpOrig = kOffTmpOld + align256(kMaxN * 4);       // uint32[kMaxN]
constexpr size_t kOffPerm = kOffTmpOrig + align256(kMaxN * 4);         // uint32[kMaxN]
constexpr size_t kOffSPos = kOffPerm + align256(kMaxN * 4);            // double4[kMaxN] (sorted)
constexpr size_t kOffSFlags = kOffSPos + align256(kMaxN * 32);         // uint8[kMaxN]
constexpr size_t kOffSOrig = kOffSFlags + align256(kMaxN);             // uint32[kMaxN]
constexpr size_t kOffCount = kOffSOrig + align256(kMaxN * 4);         // uint32[kMaxCells]
constexpr size_t kOffFill = kOffCount + align256(kMaxCells * 4);       // uint32[kMaxCells]
constexpr size_t kOffStart = kOffFill + align256(kMaxCells * 4);       // uint32[kMaxCells + 1]
constexpr size_t kOffOcc = kOffStart + align256((kMaxCells + 1) * 4);  // uint32[kMaxCells]
constexpr size_t kOffScan = kOffOcc + align256(kMaxCells * 4);         // scan tile sums
constexpr size_t kScratchBytes = kOffScan + align256(8 * (kMaxCells / 4096 + 2));

static_assert(kScratchBytes <= (size_t)20 << 20, "the scratch array should stay modest");

static __device__ __align__(256) unsigned char g_density_scratch[kScratchBytes];

// Original-order packing of the caller's arrays, and the key bounding box.
__global__ void k_na_pack(uint32_t n, const double* __restrict__ x, const uint8_t* __restrict__ kind,
                          const double* __restrict__ psi, const double* __restrict__ n_out,
                          double inv_cell, int dim, unsigned char* scratch) {
    NoAllocHeader* hd = reinterpret_cast<NoAllocHeader*>(scratch + kOffHeader);
    double4* pos = reinterpret_cast<double4*>(scratch + kOffPos);
    uint8_t* flags = scratch + kOffFlags;
    uint32_t* orig = reinterpret_cast<uint32_t*>(scratch + kOffOrig);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double px = x[3 * (size_t)i], py = x[3 * (size_t)i + 1], pz = x[3 * (size_t)i + 2];
    const bool b = kind[i] != 0;
    const double nx = n_out ? n_out[3 * (size_t)i] : 0.0, ny = n_out ? n_out[3 * (size_t)i + 1] : 0.0,
                 nz = n_out ? n_out[3 * (size_t)i + 2] : 0.0;
    const double ps = psi ? psi[i] : 0.0;
    // pe-ffi rejects non-finite input (docs/FFI.md:29-35); the host reads the
    // flag with the key box and returns PE_ERR_ARG before the grid is sized.
    if (!(isfinite(px) && isfinite(py) && isfinite(pz) && isfinite(nx) && isfinite(ny) && isfinite(nz) &&
          isfinite(ps)))
        atomicOr(&hd->nonfinite, 1u);
    const bool oriented = b && (nx * nx + ny * ny + nz * nz) > 0.0;
    pos[i] = make_double4(px, py, pz, b ? ps : 0.0);
    flags[i] = (b ? kFlagBoundary : 0) | (oriented ? kFlagOriented : 0);
    orig[i] = i;
    const int32_t k[3] = {floor_i32(px * inv_cell), floor_i32(py * inv_cell),
                          dim == 2 ? 0 : floor_i32(pz * inv_cell)};
    for (int a = 0; a < 3; ++a) {
        atomicMin(&hd->kmin[a], k[a]);
        atomicMax(&hd->kmax[a], k[a]);
    }
}

__global__ void k_na_init_header(unsigned char* scratch) {
    NoAllocHeader* hd = reinterpret_cast<NoAllocHeader*>(scratch + kOffHeader);
    hd->sc = DeviceScalars{};
    for (int a = 0; a < 3; ++a) {
        hd->kmin[a] = 2147483647;
        hd->kmax[a] = -2147483647 - 1;
    }
    hd->nonfinite = 0;
}

// Sorted copies of the fields the density needs (perm: new slot -> old slot).
__global__ void k_na_gather(uint32_t n, unsigned char* scratch) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t* perm = reinterpret_cast<const uint32_t*>(scratch + kOffPerm);
    const uint32_t old = perm[s];
    reinterpret_cast<double4*>(scratch + kOffSPos)[s] = reinterpret_cast<const double4*>(scratch + kOffPos)[old];
    (scratch + kOffSFlags)[s] = (scratch + kOffFlags)[old];
    reinterpret_cast<uint32_t*>(scratch + kOffSOrig)[s] = reinterpret_cast<const uint32_t*>(scratch + kOffOrig)[old];
}

// Density of every sorted slot, written to rho[original index]: the 27 (9)
// neighbour cells in the reference's (dz, dy, dx) order, each cell's run in
// ascending original index, a conservative single-precision filter, and the
// reference's f64 sum for the candidates that pass it (wcsph.rs:125-153).
template <int DIM>
__global__ void k_na_density(uint32_t n, GridDesc g, StepConst k, const unsigned char* scratch,
                             const double* __restrict__ n_out, double* __restrict__ rho_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4* pos = reinterpret_cast<const double4*>(scratch + kOffSPos);
    const uint8_t* flags = scratch + kOffSFlags;
    const uint32_t* orig = reinterpret_cast<const uint32_t*>(scratch + kOffSOrig);
    const uint32_t* cell_start = reinterpret_cast<const uint32_t*>(scratch + kOffStart);
    const uint32_t* cellid = reinterpret_cast<const uint32_t*>(scratch + kOffCellId);
    const uint32_t* perm = reinterpret_cast<const uint32_t*>(scratch + kOffPerm);
    if (flags[i] & kFlagBoundary) {
        rho_out[orig[i]] = k.rho0;  // wcsph.rs:127
        return;
    }
    const double4 xi = pos[i];
    const uint32_t c = cellid[perm[i]];
    const int cz = (int)(c % (uint32_t)g.nz);
    const int cy = (int)((c / (uint32_t)g.nz) % (uint32_t)g.ny);
    const int cx = (int)(c / ((uint32_t)g.nz * (uint32_t)g.ny));
    double rho = k.rho_self;
    for (int dz = (DIM == 3 ? -1 : 0); dz <= (DIM == 3 ? 1 : 0); ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int qx = cx + dx, qy = cy + dy, qz = cz + dz;
                if (qx < 0 || qy < 0 || qz < 0 || qx >= g.nx || qy >= g.ny || qz >= g.nz) continue;
                const uint32_t q = ((uint32_t)qx * (uint32_t)g.ny + (uint32_t)qy) * (uint32_t)g.nz + (uint32_t)qz;
                for (uint32_t j = cell_start[q]; j < cell_start[q + 1]; ++j) {
                    if (j == i) continue;
                    const double4 xj = pos[j];
                    const float fx = (float)(xj.x - xi.x), fy = (float)(xj.y - xi.y),
                                fz = (float)(xj.z - xi.z);
                    if (fx * fx + fy * fy + fz * fz > k.r2_filter) continue;
                    const double ddx = xj.x - xi.x, ddy = xj.y - xi.y, ddz = xj.z - xi.z;
                    const double r = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
                    const double wij = kern_w(r, k);
                    const uint8_t fl = flags[j];
                    if (fl & kFlagOriented) {
                        const size_t oj = 3 * (size_t)orig[j];
                        const double4 nb = make_double4(n_out[oj], n_out[oj + 1], n_out[oj + 2], 0.0);
                        if (!sees_fluid(k, xj, nb, xi.x, xi.y, xi.z)) continue;
                    }
                    const double f = (fl & kFlagBoundary) ? k.rho0 * xj.w : k.mass;
                    rho += f * wij;
                }
            }
    rho_out[orig[i]] = fmax(rho, 1e-12);
}

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

// Device address of the scratch array in the current device's context,
// looked up on every call (no cache that could outlive the context).
unsigned char* scratch_for_current_device(int* err) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_density_scratch) != cudaSuccess || !p) {
        *err = PE_ERR_DEVICE;
        return nullptr;
    }
    return static_cast<unsigned char*>(p);
}

}  // namespace

}  // namespace pe

extern "C" int pe_fluid_density_noalloc(int32_t dim, double rest_density, double mass, double h,
                                        uint64_t n, const double* x, const uint8_t* kind,
                                        const double* psi, const double* n_out, double* rho,
                                        void* stream) {
    using namespace pe;
    if (dim != 2 && dim != 3) return PE_ERR_ARG;
    if (!(std::isfinite(rest_density) && rest_density > 0.0 && std::isfinite(mass) && mass > 0.0 &&
          std::isfinite(h) && h > 0.0))
        return PE_ERR_ARG;
    if (n > kMaxN) return PE_ERR_BOUNDS;
    if (n == 0) return PE_OK;
    if (!x || !kind || !rho) return PE_ERR_NULL;
    int err = PE_OK;
    unsigned char* scratch = scratch_for_current_device(&err);
    if (!scratch) return err;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t nn = (uint32_t)n;

    const double cell = 2.0 * h;       // kernels.rs:32 support_radius
    const double inv = 1.0 / cell;     // grid.rs:63
    k_na_init_header<<<1, 1, 0, st>>>(scratch);
    k_na_pack<<<blocks_for(nn, 256), 256, 0, st>>>(nn, x, kind, psi, n_out, inv, dim, scratch);
    NoAllocHeader hd{};
    if (cudaMemcpyAsync(&hd, scratch + kOffHeader, sizeof(hd), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PE_ERR_DEVICE;
    if (hd.nonfinite) return PE_ERR_ARG;
    GridDesc g{};
    g.kx0 = hd.kmin[0];
    g.ky0 = hd.kmin[1];
    g.kz0 = hd.kmin[2];
    const double ext[3] = {(double)hd.kmax[0] - hd.kmin[0] + 1, (double)hd.kmax[1] - hd.kmin[1] + 1,
                           (double)hd.kmax[2] - hd.kmin[2] + 1};
    if (ext[0] * ext[1] * ext[2] > (double)kMaxCells) return PE_ERR_BOUNDS;
    g.nx = (int32_t)ext[0];
    g.ny = (int32_t)ext[1];
    g.nz = (int32_t)ext[2];
    g.ncell = (uint32_t)(ext[0] * ext[1] * ext[2]);
    g.inv_cell = inv;
    g.cell_size = cell;
    g.dim = dim;

    StepConst k{};
    k.dim = dim;
    k.h = h;
    k.inv_h = 1.0 / h;
    k.mass = mass;
    k.rho0 = rest_density;
    k.alpha = cubic_alpha(h, dim);
    k.rho_self = 0.0 + mass * cubic_w(0.0, h, k.alpha);  // wcsph.rs:133-135
    k.boundary_eps_h = 0.15 * h;
    const double sup = 2.0 * h;
    k.r2_filter = std::nextafter((float)(sup * sup * (1.0 + 1e-4)), INFINITY);

    DeviceScalars* sc = reinterpret_cast<DeviceScalars*>(scratch + kOffHeader);
    uint32_t* count = reinterpret_cast<uint32_t*>(scratch + kOffCount);
    uint32_t* fill = reinterpret_cast<uint32_t*>(scratch + kOffFill);
    uint32_t* start = reinterpret_cast<uint32_t*>(scratch + kOffStart);
    uint32_t* occ = reinterpret_cast<uint32_t*>(scratch + kOffOcc);
    uint32_t* cellid = reinterpret_cast<uint32_t*>(scratch + kOffCellId);
    int4* key = reinterpret_cast<int4*>(scratch + kOffKey);
    // counters that must start at zero on every call
    if (cudaMemsetAsync(count, 0, sizeof(uint32_t) * g.ncell, st) != cudaSuccess ||
        cudaMemsetAsync(fill, 0, sizeof(uint32_t) * g.ncell, st) != cudaSuccess)
        return PE_ERR_DEVICE;
    launch_cell_ids(g, Tanks{}, nn, reinterpret_cast<const double4*>(scratch + kOffPos), nullptr,
                    scratch + kOffFlags, cellid, key, count, sc, st);
    launch_scan_cells(g.ncell, count, start, occ, sc, scratch + kOffScan, st);
    launch_place(nn, cellid, start, fill, reinterpret_cast<const uint32_t*>(scratch + kOffOrig),
                 reinterpret_cast<uint32_t*>(scratch + kOffTmpOld),
                 reinterpret_cast<uint32_t*>(scratch + kOffTmpOrig), st);
    launch_cellsort(g.ncell < nn ? g.ncell : nn, occ, sc, start,
                    reinterpret_cast<const uint32_t*>(scratch + kOffTmpOld),
                    reinterpret_cast<const uint32_t*>(scratch + kOffTmpOrig),
                    reinterpret_cast<uint32_t*>(scratch + kOffPerm), st);
    k_na_gather<<<blocks_for(nn, 256), 256, 0, st>>>(nn, scratch);
    if (dim == 3)
        k_na_density<3><<<blocks_for(nn, 128), 128, 0, st>>>(nn, g, k, scratch, n_out, rho);
    else
        k_na_density<2><<<blocks_for(nn, 128), 128, 0, st>>>(nn, g, k, scratch, n_out, rho);
    return cudaGetLastError() == cudaSuccess ? PE_OK : PE_ERR_DEVICE;
}
