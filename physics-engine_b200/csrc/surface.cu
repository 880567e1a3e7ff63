// Surface tension of the WCSPH step (crates/pe-fluid/src/surface_tension.rs,
// applied by wcsph.rs:261-278): colour-field normals, then the Akinci (2013)
// cohesion + curvature or the colour-field (CSF) acceleration, per fluid slot
// as gathers over the visit list in the reference's visiting order. The
// Akinci curvature term has no distance cut-off, so that model runs on lists
// holding every candidate of the neighbour cells. Compiled with --fmad=false.
#include "list_iter.cuh"
#include "pe_math.cuh"
#include "sph_pair.cuh"
#include "wcsph_device.cuh"

namespace pe {

namespace {

constexpr uint32_t kStThreads = 128;

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

// kernels.rs:56 grad_w (cubic spline) at rij = x_j - x_i
__device__ __forceinline__ void grad_cubic(const StepConst& k, double rx, double ry, double rz, double* gx,
                                           double* gy, double* gz) {
    const double r = sqrt(rx * rx + ry * ry + rz * rz);
    const double dwdr = kern_dwdr(r, k);
    if (r < 1e-30) {
        *gx = *gy = *gz = 0.0;
        return;
    }
    const double s = -dwdr / r;
    *gx = rx * s;
    *gy = ry * s;
    *gz = rz * s;
}

// surface_tension.rs:127-148 n_i = h sum_j (m / rho_j) grad W (fluid j)
__global__ void __launch_bounds__(kStThreads) k_st_normals(uint32_t n, StepConst k, StateBufs s, ListBufs l,
                                                          double4* __restrict__ normals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.flags[i] & kFlagBoundary) {
        normals[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        return;
    }
    const double4 xi = s.pos[i];
    double nx = 0.0, ny = 0.0, nz = 0.0;
    for_each_entry(list_ref(l, i, kListVisit), [&](uint32_t e) {
        if (e & kEntryBoundary) return;
        const uint32_t j = e & kEntrySlotMask;
        const double4 xj = s.pos[j];
        double gx, gy, gz;
        grad_cubic(k, xj.x - xi.x, xj.y - xi.y, xj.z - xi.z, &gx, &gy, &gz);
        const double f = k.mass / fmax(s.vel[j].w, 1e-12);
        nx = nx + gx * f;
        ny = ny + gy * f;
        nz = nz + gz * f;
    });
    normals[i] = make_double4(nx * k.h, ny * k.h, nz * k.h, 0.0);
}

// surface_tension.rs:78-103 cohesion kernel, support h
__device__ __forceinline__ double cohesion(const StepConst& k, const SurfConst& c, double r) {
    if (r <= 0.0 || r >= k.h || k.h <= 0.0) return 0.0;
    const double q = div_h(r, k);
    const double t = 1.0 - q;
    return c.coh * t * t * t * q * q * q;
}

// surface_tension.rs:152-184 Akinci cohesion + curvature
__global__ void __launch_bounds__(kStThreads) k_st_akinci(uint32_t n, StepConst k, SurfConst c, StateBufs s,
                                                         ListBufs l, const double4* __restrict__ normals,
                                                         double4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.flags[i] & kFlagBoundary) {
        out[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        return;
    }
    const double4 xi = s.pos[i], ni = normals[i];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for_each_entry(list_ref(l, i, kListVisit), [&](uint32_t e) {
        if (e & kEntryBoundary) return;
        const uint32_t j = e & kEntrySlotMask;
        const double4 xj = s.pos[j], nj = normals[j];
        const double rx = xj.x - xi.x, ry = xj.y - xi.y, rz = xj.z - xi.z;
        const double r = sqrt(rx * rx + ry * ry + rz * rz);
        if (r < 1e-12) return;
        const double hx = rx / r, hy = ry / r, hz = rz / r;
        const double a = c.sm2 * cohesion(k, c, r);
        fx = fx + hx * a;
        fy = fy + hy * a;
        fz = fz + hz * a;
        fx = fx + (ni.x - nj.x) * c.nsm;
        fy = fy + (ni.y - nj.y) * c.nsm;
        fz = fz + (ni.z - nj.z) * c.nsm;
    });
    out[i] = make_double4(fx / k.mass, fy / k.mass, fz / k.mass, 0.0);
}

// surface_tension.rs:185-218 colour-field (CSF) acceleration
__global__ void __launch_bounds__(kStThreads) k_st_colour(uint32_t n, StepConst k, SurfConst c, StateBufs s,
                                                         ListBufs l, const double4* __restrict__ normals,
                                                         double4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_double4(0.0, 0.0, 0.0, 0.0);
    if (s.flags[i] & kFlagBoundary) return;
    const double4 ni = normals[i];
    const double n_len = sqrt(ni.x * ni.x + ni.y * ni.y + ni.z * ni.z);
    if (n_len < 1e-8) return;
    const double hx = ni.x / n_len, hy = ni.y / n_len, hz = ni.z / n_len;
    const double4 xi = s.pos[i];
    double div_n = 0.0;
    for_each_entry(list_ref(l, i, kListVisit), [&](uint32_t e) {
        if (e & kEntryBoundary) return;
        const uint32_t j = e & kEntrySlotMask;
        const double4 xj = s.pos[j], nj = normals[j];
        double gx, gy, gz;
        grad_cubic(k, xj.x - xi.x, xj.y - xi.y, xj.z - xi.z, &gx, &gy, &gz);
        const double nj_len = sqrt(nj.x * nj.x + nj.y * nj.y + nj.z * nj.z);
        double jx = 0.0, jy = 0.0, jz = 0.0;
        if (nj_len > 1e-8) {
            jx = nj.x / nj_len;
            jy = nj.y / nj_len;
            jz = nj.z / nj_len;
        }
        const double dx = jx - hx, dy = jy - hy, dz = jz - hz;
        div_n += (k.mass / fmax(s.vel[j].w, 1e-12)) * (dx * gx + dy * gy + dz * gz);
    });
    const double kappa = -div_n;
    const double f = -c.gamma * kappa / fmax(s.vel[i].w, 1e-12);
    out[i] = make_double4(hx * f, hy * f, hz * f, 0.0);
}

}  // namespace

void launch_surface_tension(uint32_t n, const StepConst& k, const SurfConst& c, const StateBufs& s,
                            const ListBufs& l, double4* normals, double4* out, cudaStream_t st) {
    if (!n) return;
    const uint32_t b = blocks_for(n, kStThreads);
    k_st_normals<<<b, kStThreads, 0, st>>>(n, k, s, l, normals);
    if (c.model == 1) k_st_akinci<<<b, kStThreads, 0, st>>>(n, k, c, s, l, normals, out);
    else k_st_colour<<<b, kStThreads, 0, st>>>(n, k, c, s, l, normals, out);
}

}  // namespace pe
