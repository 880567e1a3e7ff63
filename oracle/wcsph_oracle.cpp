// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// CPU oracle: an order-exact C++ restatement of eranyid/physics-engine's
// `pe-fluid` WCSPH solver path (Rust), with its PBF and DFSPH siblings and the
// fluid side of the rigid coupling. Only the test suite, the smoke check
// and the CPU-baseline leg of bench.py load this library; the product
// (physics-engine_b200/) never links, calls or falls back to it.
//
// Every function names the reference file:line it restates. Floating-point
// statements keep the reference's operand order and association exactly
// (Rust evaluates `a * b * c` as `(a * b) * c`), and the file is compiled
// with `-ffp-contract=off` (no FMA), matching the reference's determinism
// policy (`.cargo/config.toml`, `docs/DETERMINISM.md`).
//
// Elementary functions: the reference calls the pure-Rust `libm` crate
// 0.2.16 (`Cargo.lock:524-525`), whose source is not vendored. `sqrt` is
// IEEE correctly rounded everywhere, so the C library's sqrt is bit-identical.
// `pow` (Tait EOS, `eos.rs:68`; poly6/spiky normalisation, `kernels.rs:164,190`)
// is restated as a correctly rounded integer power evaluated in binary128
// (`oracle_pow`), falling back to the C library for non-integer exponents.
// The crate's pow is documented as "nearly rounded", so the two agree except
// in rare last-ulp cases. The PBF and DFSPH restatements below reproduce the
// reference's locked tank hashes (9d9e0da856fd43d4, f1f2825b5eeaab0d), which
// pins the pow normalisations of the poly6 and spiky kernels.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <cstdint>
#include <cstring>
#include <limits>
#include <new>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------------------
// Parallel oracle helpers (threads > 1 only; one thread runs inline).
// ---------------------------------------------------------------------------
// fn(i, worker) for i in [0, n), handed out in chunks from a shared counter.
template <typename F>
static void parallel_for(size_t n, int threads, F fn, size_t chunk = 256) {
    if (threads <= 1 || n <= chunk) {
        for (size_t i = 0; i < n; ++i) fn(i, 0);
        return;
    }
    std::atomic<size_t> next{0};
    auto work = [&](int w) {
        for (;;) {
            size_t a = next.fetch_add(chunk);
            if (a >= n) return;
            size_t b = std::min(n, a + chunk);
            for (size_t i = a; i < b; ++i) fn(i, w);
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < threads; ++w) pool.emplace_back(work, w);
    work(0);
    for (auto& t : pool) t.join();
}

// Sort by a strict total order: sorted chunks merged pairwise. A total order
// has one sorted result, so this equals the sequential stable sort.
template <typename T, typename Lt>
static void parallel_sort_total(std::vector<T>& v, Lt lt, int threads) {
    const size_t n = v.size();
    if (threads <= 1 || n < 65536) {
        std::stable_sort(v.begin(), v.end(), lt);
        return;
    }
    size_t parts = 1;
    while (parts < (size_t)threads) parts *= 2;
    std::vector<size_t> cut(parts + 1);
    for (size_t k = 0; k <= parts; ++k) cut[k] = n * k / parts;
    {
        std::vector<std::thread> pool;
        for (size_t k = 0; k < parts; ++k)
            pool.emplace_back([&, k] { std::sort(v.begin() + cut[k], v.begin() + cut[k + 1], lt); });
        for (auto& t : pool) t.join();
    }
    std::vector<T> tmp(n);
    for (size_t width = 1; width < parts; width *= 2) {
        std::vector<std::thread> pool;
        for (size_t k = 0; k < parts; k += 2 * width)
            pool.emplace_back([&, k] {
                std::merge(v.begin() + cut[k], v.begin() + cut[k + width], v.begin() + cut[k + width],
                           v.begin() + cut[k + 2 * width], tmp.begin() + cut[k], lt);
            });
        for (auto& t : pool) t.join();
        v.swap(tmp);
    }
}

// ---------------------------------------------------------------------------
// pe-math Vec3 (crates/pe-math/src/vec3.rs:9-183): component-wise ops.
// ---------------------------------------------------------------------------
struct V3 {
    double x, y, z;
};
static inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
static inline V3 zero3() { return V3{0.0, 0.0, 0.0}; }
static inline V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 operator*(V3 a, double s) { return V3{a.x * s, a.y * s, a.z * s}; }
static inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
static inline V3& operator-=(V3& a, V3 b) { a = a - b; return a; }
// vec3.rs:69 norm_squared = x*x + y*y + z*z (left to right)
static inline double norm2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
// vec3.rs:63 norm = sqrt(norm_squared)
static inline double norm(V3 a) { return std::sqrt(norm2(a)); }
// vec3.rs:81 dot
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// ---------------------------------------------------------------------------
// pow restatement (see header): correctly rounded x^n for integer n.
// ---------------------------------------------------------------------------
static double pow_int_binary128(double x, long n) {
    __float128 b = x;
    __float128 r = 1;
    unsigned long e = n < 0 ? (unsigned long)(-n) : (unsigned long)n;
    while (e) {
        if (e & 1UL) r *= b;
        b *= b;
        e >>= 1;
    }
    if (n < 0) r = (__float128)1 / r;
    return (double)r;
}

double oracle_pow(double x, double y) {
    if (std::isfinite(x) && x > 0.0 && std::isfinite(y) && y == std::floor(y) &&
        std::fabs(y) <= 64.0) {
        return pow_int_binary128(x, (long)y);
    }
    return std::pow(x, y);
}

// ---------------------------------------------------------------------------
// pe-math xoshiro256** (crates/pe-math/src/rng.rs:14-72).
// ---------------------------------------------------------------------------
struct Xoshiro {
    uint64_t s[4];
};
static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
// rng.rs:25 splitmix64
static inline uint64_t splitmix64(uint64_t* st) {
    *st += 0x9e3779b97f4a7c15ULL;
    uint64_t z = *st;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
// rng.rs:35 seed
static Xoshiro xoshiro_seed(uint64_t seed) {
    Xoshiro r;
    uint64_t sm = seed;
    for (int i = 0; i < 4; ++i) r.s[i] = splitmix64(&sm);
    if (r.s[0] == 0 && r.s[1] == 0 && r.s[2] == 0 && r.s[3] == 0) r.s[0] = 0x9e3779b97f4a7c15ULL;
    return r;
}
// rng.rs:50 next_u64
static inline uint64_t xoshiro_next(Xoshiro* r) {
    uint64_t* s = r->s;
    uint64_t result = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
}
// rng.rs:64 next_f64, rng.rs:70 uniform
static inline double xoshiro_f64(Xoshiro* r) {
    return (double)(xoshiro_next(r) >> 11) * (1.0 / (double)(1ULL << 53));
}
static inline double xoshiro_uniform(Xoshiro* r, double lo, double hi) {
    return lo + (hi - lo) * xoshiro_f64(r);
}

// ---------------------------------------------------------------------------
// pe-fluid types
// ---------------------------------------------------------------------------
enum Dim { D2 = 2, D3 = 3 };                         // lib.rs:202
enum Kind : uint8_t { FLUID = 0, BOUNDARY = 1 };      // particles.rs:11
enum KernelKind { CUBIC = 0, WENDLAND = 1, POLY6 = 2, SPIKY = 3 };  // kernels.rs:19

static const double PI = 3.14159265358979311599796346854;  // f64::consts::PI

// kernels.rs:32 support_radius
static double support_radius(KernelKind k, double h) {
    return (k == CUBIC || k == WENDLAND) ? 2.0 * h : h;
}
// kernels.rs:79 cubic_alpha
static double cubic_alpha(double h, Dim dim) {
    return dim == D2 ? 10.0 / (7.0 * PI * h * h) : 1.0 / (PI * h * h * h);
}
// kernels.rs:86 cubic_spline_w
static double cubic_spline_w(double r, double h, Dim dim) {
    double q = r / h;
    if (q >= 2.0) return 0.0;
    double a = cubic_alpha(h, dim);
    if (q < 1.0) {
        return a * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
    }
    double t = 2.0 - q;
    return a * 0.25 * t * t * t;
}
// kernels.rs:102 cubic_spline_dwdr
static double cubic_spline_dwdr(double r, double h, Dim dim) {
    double q = r / h;
    if (q >= 2.0 || q <= 0.0) return 0.0;
    double a = cubic_alpha(h, dim);
    double dwdq;
    if (q < 1.0) {
        dwdq = a * (-3.0 * q + 2.25 * q * q);
    } else {
        double t = 2.0 - q;
        dwdq = a * (-0.75 * t * t);
    }
    return dwdq / h;
}
// kernels.rs:121 wendland_alpha, :129 wendland_c2_w, :139 wendland_c2_dwdr
static double wendland_alpha(double h, Dim dim) {
    return dim == D2 ? 7.0 / (4.0 * PI * h * h) : 21.0 / (16.0 * PI * h * h * h);
}
static double wendland_c2_w(double r, double h, Dim dim) {
    double q = r / h;
    if (q >= 2.0) return 0.0;
    double a = wendland_alpha(h, dim);
    double t = 1.0 - 0.5 * q;
    return a * t * t * t * t * (2.0 * q + 1.0);
}
static double wendland_c2_dwdr(double r, double h, Dim dim) {
    double q = r / h;
    if (q >= 2.0 || q <= 0.0) return 0.0;
    double a = wendland_alpha(h, dim);
    double t = 1.0 - 0.5 * q;
    double dwdq = a * (-5.0 * q) * t * t * t;
    return dwdq / h;
}
// kernels.rs:161 poly6_alpha, :169 poly6_w, :178 poly6_dwdr
static double poly6_alpha(double h, Dim dim) {
    return dim == D2 ? 4.0 / (PI * oracle_pow(h, 8.0)) : 315.0 / (64.0 * PI * oracle_pow(h, 9.0));
}
static double poly6_w(double r, double h, Dim dim) {
    if (r >= h) return 0.0;
    double a = poly6_alpha(h, dim);
    double t = h * h - r * r;
    return a * t * t * t;
}
static double poly6_dwdr(double r, double h, Dim dim) {
    if (r >= h || r <= 0.0) return 0.0;
    double a = poly6_alpha(h, dim);
    double t = h * h - r * r;
    return a * (-6.0 * r * t * t);
}
// kernels.rs:188 spiky_alpha, :196 spiky_w, :205 spiky_dwdr
static double spiky_alpha(double h, Dim dim) {
    return dim == D2 ? 10.0 / (PI * oracle_pow(h, 5.0)) : 15.0 / (PI * oracle_pow(h, 6.0));
}
static double spiky_w(double r, double h, Dim dim) {
    if (r >= h) return 0.0;
    double a = spiky_alpha(h, dim);
    double t = h - r;
    return a * t * t * t;
}
static double spiky_dwdr(double r, double h, Dim dim) {
    if (r >= h || r <= 0.0) return 0.0;
    double a = spiky_alpha(h, dim);
    double t = h - r;
    return a * (-3.0 * t * t);
}
// kernels.rs:40 w
static double kern_w(KernelKind k, double r, double h, Dim dim) {
    if (h <= 0.0 || r < 0.0) return 0.0;
    switch (k) {
        case CUBIC: return cubic_spline_w(r, h, dim);
        case WENDLAND: return wendland_c2_w(r, h, dim);
        case POLY6: return poly6_w(r, h, dim);
        default: return spiky_w(r, h, dim);
    }
}
// kernels.rs:56 grad_w (rij = r_j - r_i; returns grad_i W)
static V3 grad_w(KernelKind k, V3 rij, double h, Dim dim) {
    if (h <= 0.0) return zero3();
    double r2 = norm2(rij);
    double r = std::sqrt(r2);
    double dwdr;
    switch (k) {
        case CUBIC: dwdr = cubic_spline_dwdr(r, h, dim); break;
        case WENDLAND: dwdr = wendland_c2_dwdr(r, h, dim); break;
        case POLY6: dwdr = poly6_dwdr(r, h, dim); break;
        default: dwdr = spiky_dwdr(r, h, dim); break;
    }
    if (r < 1e-30) return zero3();
    return rij * (-dwdr / r);
}

// ---------------------------------------------------------------------------
// Particles (particles.rs:20-162)
// ---------------------------------------------------------------------------
struct Particles {
    Dim dim;
    double rest_density, mass, h;
    std::vector<V3> x, v, a;
    std::vector<double> rho, p;
    std::vector<uint8_t> kind;
    std::vector<double> psi;
    std::vector<V3> n_out;
    size_t len() const { return x.size(); }
    // particles.rs:90 push_fluid
    void push_fluid(V3 px, V3 pv) {
        x.push_back(px); v.push_back(pv); a.push_back(zero3());
        rho.push_back(rest_density); p.push_back(0.0);
        kind.push_back(FLUID); psi.push_back(0.0); n_out.push_back(zero3());
    }
    // particles.rs:102/107 push_boundary(_oriented)
    void push_boundary(V3 px, double ps, V3 n = V3{0, 0, 0}) {
        x.push_back(px); v.push_back(zero3()); a.push_back(zero3());
        rho.push_back(rest_density); p.push_back(0.0);
        kind.push_back(BOUNDARY); psi.push_back(ps); n_out.push_back(n);
    }
    // particles.rs:126 boundary_sees_fluid
    bool boundary_sees_fluid(size_t b, V3 xf) const {
        V3 n = n_out[b];
        double n2 = norm2(n);
        if (n2 <= 0.0) return true;
        double eps = 0.15 * h * std::sqrt(std::fmax(n2, 0.0));
        return dot(xf - x[b], n) > -eps;
    }
    size_t fluid_count() const {
        size_t c = 0;
        for (auto k : kind) c += (k == FLUID);
        return c;
    }
};

// particles.rs:166 mass_from_spacing
static double mass_from_spacing(double rho0, double dx, Dim dim) {
    return dim == D2 ? rho0 * dx * dx : rho0 * dx * dx * dx;
}
// particles.rs:178 mass_calibrated_to_rest
static double mass_calibrated_to_rest(double rho0, double dx, double h, Dim dim, KernelKind k) {
    double support = support_radius(k, h);
    int n = (int)std::ceil(support / dx) + 1;
    double sum_w = kern_w(k, 0.0, h, dim);
    for (int ix = -n; ix <= n; ++ix)
        for (int iy = -n; iy <= n; ++iy) {
            int z0 = dim == D2 ? 0 : -n, z1 = dim == D2 ? 0 : n;
            for (int iz = z0; iz <= z1; ++iz) {
                if (ix == 0 && iy == 0 && iz == 0) continue;
                double r = std::sqrt(((double)ix * dx) * ((double)ix * dx) +
                                     ((double)iy * dx) * ((double)iy * dx) +
                                     ((double)iz * dx) * ((double)iz * dx));
                if (r < support) sum_w += kern_w(k, r, h, dim);
            }
        }
    return sum_w < 1e-30 ? mass_from_spacing(rho0, dx, dim) : rho0 / sum_w;
}
// particles.rs:220 fill_box (iz -> iy -> ix fill order)
static void fill_box(Particles& p, V3 origin, size_t nx, size_t ny, size_t nz, double dx, V3 v0) {
    if (p.dim == D2) nz = 1;
    for (size_t iz = 0; iz < nz; ++iz)
        for (size_t iy = 0; iy < ny; ++iy)
            for (size_t ix = 0; ix < nx; ++ix)
                p.push_fluid(v3(origin.x + (double)ix * dx, origin.y + (double)iy * dx,
                                origin.z + (double)iz * dx), v0);
}
// particles.rs:252 recomputed_akinci_psi (O(N_b^2), index order)
static void recomputed_akinci_psi(Particles& p, KernelKind k) {
    double h = p.h;
    double support = support_radius(k, h);
    std::vector<size_t> bound;
    for (size_t i = 0; i < p.len(); ++i)
        if (p.kind[i] == BOUNDARY) bound.push_back(i);
    for (size_t bi : bound) {
        V3 xb = p.x[bi];
        double delta = kern_w(k, 0.0, h, p.dim);
        for (size_t bj : bound) {
            if (bj == bi) continue;
            double r = norm(p.x[bj] - xb);
            if (r < support) delta += kern_w(k, r, h, p.dim);
        }
        p.psi[bi] = delta > 1e-30 ? 1.0 / delta : 0.0;
    }
}
// particles.rs:286 fill_box_boundary
static void fill_box_boundary(Particles& p, V3 mn, V3 mx, double dx, size_t layers) {
    double psi = p.dim == D2 ? dx * dx : dx * dx * dx;
    if (layers < 1) layers = 1;
    if (p.dim == D2) {
        size_t nx = (size_t)std::round((mx.x - mn.x) / dx) + 1;
        size_t ny = (size_t)std::round((mx.y - mn.y) / dx) + 1;
        for (size_t layer = 0; layer < layers; ++layer) {
            double off = (double)layer * dx;
            for (size_t i = 0; i < nx; ++i) {
                double x = mn.x + (double)i * dx;
                p.push_boundary(v3(x, mn.y - off, 0.0), psi);
                p.push_boundary(v3(x, mx.y + off, 0.0), psi);
            }
            for (size_t j = 1; j + 1 < ny; ++j) {
                double y = mn.y + (double)j * dx;
                p.push_boundary(v3(mn.x - off, y, 0.0), psi);
                p.push_boundary(v3(mx.x + off, y, 0.0), psi);
            }
        }
        return;
    }
    size_t nx = (size_t)std::round((mx.x - mn.x) / dx) + 1;
    size_t ny = (size_t)std::round((mx.y - mn.y) / dx) + 1;
    size_t nz = (size_t)std::round((mx.z - mn.z) / dx) + 1;
    for (size_t layer = 0; layer < layers; ++layer) {
        double off = (double)layer * dx;
        for (size_t i = 0; i < nx; ++i)
            for (size_t j = 0; j < ny; ++j) {
                double x = mn.x + (double)i * dx, y = mn.y + (double)j * dx;
                p.push_boundary(v3(x, y, mn.z - off), psi);
                p.push_boundary(v3(x, y, mx.z + off), psi);
            }
        for (size_t i = 0; i < nx; ++i)
            for (size_t k = 1; k + 1 < nz; ++k) {
                double x = mn.x + (double)i * dx, z = mn.z + (double)k * dx;
                p.push_boundary(v3(x, mn.y - off, z), psi);
                p.push_boundary(v3(x, mx.y + off, z), psi);
            }
        for (size_t j = 1; j + 1 < ny; ++j)
            for (size_t k = 1; k + 1 < nz; ++k) {
                double y = mn.y + (double)j * dx, z = mn.z + (double)k * dx;
                p.push_boundary(v3(mn.x - off, y, z), psi);
                p.push_boundary(v3(mx.x + off, y, z), psi);
            }
    }
}

// ---------------------------------------------------------------------------
// Uniform grid (grid.rs:13-157)
// ---------------------------------------------------------------------------
struct CellKey {
    int32_t ix, iy, iz;
};
// Derived Ord on {ix, iy, iz}: lexicographic, ix-major (grid.rs:12).
static inline bool key_lt(const CellKey& a, const CellKey& b) {
    if (a.ix != b.ix) return a.ix < b.ix;
    if (a.iy != b.iy) return a.iy < b.iy;
    return a.iz < b.iz;
}
static inline bool key_eq(const CellKey& a, const CellKey& b) {
    return a.ix == b.ix && a.iy == b.iy && a.iz == b.iz;
}
// grid.rs:144 floor_i32
static inline int32_t floor_i32(double x) {
    if (!std::isfinite(x)) return 0;
    const double lo = (double)std::numeric_limits<int32_t>::min() + 1.0;
    const double hi = (double)std::numeric_limits<int32_t>::max() - 1.0;
    double c = x < lo ? lo : (x > hi ? hi : x);
    int32_t t = (int32_t)c;  // truncation toward zero; c is in range
    if ((double)t > c) return t == std::numeric_limits<int32_t>::min() ? t : t - 1;
    return t;
}

struct UniformGrid {
    double cell_size;
    Dim dim;
    std::vector<size_t> order;
    std::vector<CellKey> keys;
    std::vector<CellKey> occupied;
    std::vector<std::pair<size_t, size_t>> ranges;

    // grid.rs:62 key_of
    CellKey key_of(V3 p) const {
        double inv = 1.0 / cell_size;
        int32_t ix = floor_i32(p.x * inv);
        int32_t iy = floor_i32(p.y * inv);
        int32_t iz = dim == D2 ? 0 : floor_i32(p.z * inv);
        return CellKey{ix, iy, iz};
    }
    // grid.rs:76 rebuild: sort by (key, index), run-length occupied cells
    // threads > 1 (parallel oracle): the same keys and the same order, since
    // (key, index) is a total order and the sort's result is unique.
    void rebuild(const std::vector<V3>& pos, int threads = 1) {
        size_t n = pos.size();
        keys.resize(n);
        order.resize(n);
        parallel_for(n, threads, [&](size_t i, int) {
            keys[i] = key_of(pos[i]);
            order[i] = i;
        }, 4096);
        const std::vector<CellKey>& k = keys;
        auto lt = [&k](size_t a, size_t b) {
            if (key_lt(k[a], k[b])) return true;
            if (key_lt(k[b], k[a])) return false;
            return a < b;
        };
        parallel_sort_total(order, lt, threads);
        occupied.clear();
        ranges.clear();
        if (n == 0) return;
        size_t start = 0;
        CellKey cur = keys[order[0]];
        for (size_t s = 1; s < n; ++s) {
            CellKey kk = keys[order[s]];
            if (!key_eq(kk, cur)) {
                occupied.push_back(cur);
                ranges.push_back({start, s});
                start = s;
                cur = kk;
            }
        }
        occupied.push_back(cur);
        ranges.push_back({start, n});
    }
    // grid.rs:111 cell_range: binary search of the occupied keys
    bool cell_range(CellKey key, size_t* a, size_t* b) const {
        auto it = std::lower_bound(occupied.begin(), occupied.end(), key, key_lt);
        if (it == occupied.end() || !key_eq(*it, key)) return false;
        size_t idx = (size_t)(it - occupied.begin());
        *a = ranges[idx].first;
        *b = ranges[idx].second;
        return true;
    }
    // grid.rs:122 neighbours: cells in (dz, dy, dx) order, appends order[a..b]
    void neighbours(size_t i, std::vector<size_t>& out) const {
        CellKey key = keys[i];
        int dz0 = dim == D2 ? 0 : -1, dz1 = dim == D2 ? 0 : 1;
        for (int dz = dz0; dz <= dz1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    CellKey nk{key.ix + dx, key.iy + dy, key.iz + dz};
                    size_t a, b;
                    if (cell_range(nk, &a, &b))
                        for (size_t s = a; s < b; ++s) out.push_back(order[s]);
                }
    }
};

// ---------------------------------------------------------------------------
// WCSPH (wcsph.rs:24-370, eos.rs:59-80, viscosity.rs:30-100)
// ---------------------------------------------------------------------------
struct WParams {
    int32_t kernel;            // KernelKind (wcsph.rs:26)
    double eos_rest_density;   // eos.rs:34
    double eos_sound_speed;    // eos.rs:36
    double eos_gamma;          // eos.rs:38
    double visc_alpha, visc_beta, visc_eps;  // viscosity.rs:30
    double xsph_epsilon;       // viscosity.rs:77
    double gravity[3];         // wcsph.rs:34
    int32_t adapt_sound_speed; // wcsph.rs:36
    int32_t materialize_neigh_lists;  // wcsph.rs:102-113 (1 = as the reference)
    // SurfaceTensionParams (surface_tension.rs:38-46): model 0 None,
    // 1 Akinci2013, 2 ColourField
    int32_t st_model;
    double st_sigma, st_colour_gamma;
};

// surface_tension.rs:78-103 cohesion kernels (support h)
static double cohesion_kernel(double r, double h, Dim dim) {
    if (r <= 0.0 || r >= h || h <= 0.0) return 0.0;
    double q = r / h;
    double t = 1.0 - q;
    if (dim == D2) return 16.0 / (PI * h * h) * t * t * t * q * q * q;
    return 32.0 / (PI * oracle_pow(h, 3.0)) * t * t * t * q * q * q;
}

struct World {
    Particles parts;
    UniformGrid grid;
    WParams prm;
    double t = 0.0;
    // Parallel oracle (threads > 1): every per-particle loop runs on
    // std::threads and compute_forces runs as the gather of forces_gather_*; the
    // results are the sequential oracle's bits (tests check both on the same
    // scenes). Used to time the CPU baseline on large tanks.
    int threads = 1;
    // Sensitivity test hook: with rate > 0, each fluid particle's Tait power
    // moves one ulp (up or down) with probability `rate`, drawn from a seeded
    // counter per pressure pass; models a last-ulp difference of the pow.
    double pow_perturb_rate = 0.0;
    uint64_t pow_perturb_seed = 0;
    uint64_t pressure_calls = 0;
    std::vector<size_t> neigh;
    std::vector<std::vector<size_t>> neigh_lists;
    std::vector<V3> xsph_dv;
    std::vector<V3> boundary_force;
    std::vector<V3> st_normals, st_a;

    KernelKind kk() const { return (KernelKind)prm.kernel; }

    // wcsph.rs:102 rebuild_grid
    void rebuild_grid() {
        grid.rebuild(parts.x, threads);
        size_t n = parts.len();
        if (neigh_lists.size() != n) neigh_lists.resize(n);
        parallel_for(n, threads, [&](size_t i, int) {
            neigh_lists[i].clear();
            if (prm.materialize_neigh_lists && parts.kind[i] == FLUID) grid.neighbours(i, neigh_lists[i]);
        });
    }
    // wcsph.rs:117 compute_density
    void compute_density() {
        size_t n = parts.len();
        if (threads > 1) {
            std::vector<std::vector<size_t>> nb(threads);
            parallel_for(n, threads, [&](size_t i, int w) { parts.rho[i] = density_of(i, nb[w]); });
            return;
        }
        for (size_t i = 0; i < n; ++i) parts.rho[i] = density_of(i, neigh);
    }
    double density_of(size_t i, std::vector<size_t>& nb) const {
        double h = parts.h, mass = parts.mass, rho0 = parts.rest_density;
        Dim dim = parts.dim;
        if (parts.kind[i] != FLUID) return rho0;
        nb.clear();
        grid.neighbours(i, nb);
        V3 xi = parts.x[i];
        double rho = 0.0;
        rho += mass * kern_w(kk(), 0.0, h, dim);
        for (size_t j : nb) {
            if (j == i) continue;
            double r = norm(parts.x[j] - xi);
            double wij = kern_w(kk(), r, h, dim);
            if (parts.kind[j] == FLUID) {
                rho += mass * wij;
            } else if (parts.boundary_sees_fluid(j, xi)) {
                rho += rho0 * parts.psi[j] * wij;
            }
        }
        return std::fmax(rho, 1e-12);  // f64::max (NaN -> other)
    }
    // viscosity.rs:89 max_speed over fluid
    double max_speed() const {
        double m = 0.0;
        for (size_t i = 0; i < parts.len(); ++i) {
            if (parts.kind[i] != FLUID) continue;
            double s = norm2(parts.v[i]);
            if (s > m) m = s;
        }
        return std::sqrt(m);
    }
    // eos.rs:59 stiffness_b, eos.rs:65 pressure
    double eos_pressure(double density) const {
        double ratio = density / prm.eos_rest_density;
        double b = prm.eos_rest_density * prm.eos_sound_speed * prm.eos_sound_speed / prm.eos_gamma;
        return b * (oracle_pow(ratio, prm.eos_gamma) - 1.0);
    }
    // wcsph.rs:157 compute_pressure (+ eos.rs:74 ensure_sound_speed)
    void compute_pressure() {
        double c = prm.eos_sound_speed;
        if (prm.adapt_sound_speed) {
            double vmax = max_speed();
            double min_c = 10.0 * std::fmax(vmax, 0.0);
            c = c < min_c ? min_c : c;
            prm.eos_sound_speed = c;
        }
        const uint64_t call = pressure_calls++;
        parallel_for(parts.len(), threads, [&](size_t i, int) {
            parts.p[i] = parts.kind[i] == FLUID ? eos_pressure_at(parts.rho[i], i, call) : 0.0;
        }, 4096);
    }
    static uint64_t splitmix64(uint64_t z) {
        z += 0x9E3779B97F4A7C15ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    // eos_pressure, with the sensitivity hook's one-ulp move of the power
    double eos_pressure_at(double density, size_t i, uint64_t call) const {
        if (pow_perturb_rate <= 0.0) return eos_pressure(density);
        double ratio = density / prm.eos_rest_density;
        double b = prm.eos_rest_density * prm.eos_sound_speed * prm.eos_sound_speed / prm.eos_gamma;
        double pw = oracle_pow(ratio, prm.eos_gamma);
        const uint64_t r = splitmix64(pow_perturb_seed ^ splitmix64(call * 0x100000001ULL + i));
        if ((double)(r >> 11) * 0x1.0p-53 < pow_perturb_rate)
            pw = std::nextafter(pw, (r & 1) ? INFINITY : -INFINITY);
        return b * (pw - 1.0);
    }
    // viscosity.rs:51 pi_ij
    double pi_ij(double h, double c, V3 xi, V3 xj, V3 vi, V3 vj, double rhoi, double rhoj) const {
        V3 rij = xi - xj;
        V3 vij = vi - vj;
        double vr = dot(vij, rij);
        if (vr >= 0.0) return 0.0;
        double r2 = norm2(rij);
        double mu = h * vr / (r2 + prm.visc_eps * h * h);
        double rho_bar = 0.5 * (rhoi + rhoj);
        double c_bar = c;
        return (-prm.visc_alpha * c_bar * mu + prm.visc_beta * mu * mu) / rho_bar;
    }
    // wcsph.rs:181 compute_forces (surface tension branch not restated: sigma = 0)
    void compute_forces() {
        size_t n = parts.len();
        double h = parts.h, mass = parts.mass, rho0 = parts.rest_density;
        double c0 = prm.eos_sound_speed;
        Dim dim = parts.dim;
        V3 g = v3(prm.gravity[0], prm.gravity[1], prm.gravity[2]);
        if (boundary_force.size() != n) boundary_force.resize(n);
        if (threads > 1 && prm.st_sigma == 0.0) {
            forces_gather();
            return;
        }
        for (auto& a : parts.a) a = zero3();
        for (auto& f : boundary_force) f = zero3();
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) continue;
            neigh.clear();
            grid.neighbours(i, neigh);
            V3 xi = parts.x[i], vi = parts.v[i];
            double rho_i = parts.rho[i], p_i = parts.p[i];
            for (size_t j : neigh) {
                if (j == i) continue;
                V3 xj = parts.x[j];
                V3 rij = xj - xi;
                double r = norm(rij);
                if (r < 1e-30) continue;
                V3 gw = grad_w(kk(), rij, h, dim);
                if (parts.kind[j] == FLUID) {
                    if (j < i) continue;
                    double rho_j = parts.rho[j], p_j = parts.p[j];
                    V3 vj = parts.v[j];
                    double press = p_i / (rho_i * rho_i) + p_j / (rho_j * rho_j);
                    V3 f_press = gw * (-mass * press);
                    double pi = pi_ij(h, c0, xi, xj, vi, vj, rho_i, rho_j);
                    V3 f_visc = gw * (-mass * pi);
                    V3 f = f_press + f_visc;
                    parts.a[i] += f;
                    parts.a[j] -= f;
                } else {
                    if (!parts.boundary_sees_fluid(j, xi)) continue;
                    double press = p_i / (rho_i * rho_i);
                    V3 f = gw * (-(rho0 * parts.psi[j]) * press);
                    parts.a[i] += f;
                    boundary_force[j] += f * (-mass);
                }
            }
            parts.a[i] += g;
        }
        // wcsph.rs:261-278 optional surface tension
        if (prm.st_sigma != 0.0) {
            surface_tension_accel(st_normals, st_a);
            for (size_t i = 0; i < n; ++i)
                if (parts.kind[i] == FLUID) parts.a[i] += st_a[i];
        }
    }
    // Parallel form of compute_forces. The scatter above gives a[k] the
    // sequence 0 - f(i1,k) - f(i2,k) - ... (fluid i < k, ascending i), then
    // + f(k,j) (fluid j > k and boundary j, visiting order), then + g; and
    // f(i,k) = -f(k,i) bit for bit (the pressure sum and pi_ij are symmetric,
    // grad W flips sign exactly), so x - f(i,k) = x + f(k,i). A boundary
    // sample's reaction is the sum over fluid i in ascending i. The cell
    // neighbour relation is symmetric, so each particle finds those partners
    // among its own candidates.
    V3 fluid_pair_force(size_t i, size_t j, V3 gw) const {
        double rho_i = parts.rho[i], p_i = parts.p[i], rho_j = parts.rho[j], p_j = parts.p[j];
        double press = p_i / (rho_i * rho_i) + p_j / (rho_j * rho_j);
        V3 f_press = gw * (-parts.mass * press);
        double pi = pi_ij(parts.h, prm.eos_sound_speed, parts.x[i], parts.x[j], parts.v[i], parts.v[j], rho_i,
                          rho_j);
        V3 f_visc = gw * (-parts.mass * pi);
        return f_press + f_visc;
    }
    V3 gather_fluid_accel(size_t k, std::vector<size_t>& nb, std::vector<size_t>& low) const {
        const double h = parts.h, rho0 = parts.rest_density;
        const Dim dim = parts.dim;
        nb.clear();
        grid.neighbours(k, nb);
        low.clear();
        for (size_t j : nb)
            if (j < k && parts.kind[j] == FLUID) low.push_back(j);
        std::sort(low.begin(), low.end());
        const V3 xk = parts.x[k];
        V3 a = zero3();
        for (size_t i : low) {
            V3 rij = parts.x[i] - xk;
            if (norm(rij) < 1e-30) continue;
            a += fluid_pair_force(k, i, grad_w(kk(), rij, h, dim));
        }
        const double rho_k = parts.rho[k], p_k = parts.p[k];
        for (size_t j : nb) {
            if (j == k) continue;
            V3 rij = parts.x[j] - xk;
            if (norm(rij) < 1e-30) continue;
            V3 gw = grad_w(kk(), rij, h, dim);
            if (parts.kind[j] == FLUID) {
                if (j < k) continue;
                a += fluid_pair_force(k, j, gw);
            } else {
                if (!parts.boundary_sees_fluid(j, xk)) continue;
                double press = p_k / (rho_k * rho_k);
                a += gw * (-(rho0 * parts.psi[j]) * press);
            }
        }
        a += v3(prm.gravity[0], prm.gravity[1], prm.gravity[2]);
        return a;
    }
    V3 gather_boundary_force(size_t b, std::vector<size_t>& nb, std::vector<size_t>& low) const {
        const double h = parts.h, mass = parts.mass, rho0 = parts.rest_density;
        const Dim dim = parts.dim;
        nb.clear();
        grid.neighbours(b, nb);
        low.clear();
        for (size_t j : nb)
            if (parts.kind[j] == FLUID) low.push_back(j);
        std::sort(low.begin(), low.end());
        V3 f = zero3();
        for (size_t i : low) {
            V3 rij = parts.x[b] - parts.x[i];
            if (norm(rij) < 1e-30) continue;
            if (!parts.boundary_sees_fluid(b, parts.x[i])) continue;
            V3 gw = grad_w(kk(), rij, h, dim);
            double press = parts.p[i] / (parts.rho[i] * parts.rho[i]);
            V3 fi = gw * (-(rho0 * parts.psi[b]) * press);
            f += fi * (-mass);
        }
        return f;
    }
    void forces_gather() {
        const size_t n = parts.len();
        std::vector<std::vector<size_t>> nb(threads), low(threads);
        parallel_for(n, threads, [&](size_t i, int w) {
            if (parts.kind[i] == FLUID) {
                parts.a[i] = gather_fluid_accel(i, nb[w], low[w]);
                boundary_force[i] = zero3();
            } else {
                parts.a[i] = zero3();
                boundary_force[i] = gather_boundary_force(i, nb[w], low[w]);
            }
        });
    }
    // surface_tension.rs:112-220 surface_tension_accel over the grid's lists
    void surface_tension_accel(std::vector<V3>& normals, std::vector<V3>& out) {
        const size_t n = parts.len();
        normals.assign(n, zero3());
        out.assign(n, zero3());
        if (prm.st_model == 0 || prm.st_sigma == 0.0) return;
        const double h = parts.h, mass = parts.mass;
        const Dim dim = parts.dim;
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) continue;
            neigh.clear();
            grid.neighbours(i, neigh);
            V3 xi = parts.x[i];
            V3 ni = zero3();
            for (size_t j : neigh) {
                if (j == i || parts.kind[j] != FLUID) continue;
                V3 gw = grad_w(kk(), parts.x[j] - xi, h, dim);
                ni += gw * (mass / std::fmax(parts.rho[j], 1e-12));
            }
            normals[i] = ni * h;
        }
        if (prm.st_model == 1) {
            const double dim_scale = dim == D2 ? 1.0 / 20.0 : 1.0;
            const double sigma_eff = prm.st_sigma * dim_scale;
            for (size_t i = 0; i < n; ++i) {
                if (parts.kind[i] != FLUID) continue;
                neigh.clear();
                grid.neighbours(i, neigh);
                V3 xi = parts.x[i];
                V3 f = zero3();
                for (size_t j : neigh) {
                    if (j == i || parts.kind[j] != FLUID) continue;
                    V3 rij = parts.x[j] - xi;
                    double r = norm(rij);
                    if (r < 1e-12) continue;
                    V3 r_hat{rij.x / r, rij.y / r, rij.z / r};
                    double c = cohesion_kernel(r, h, dim);
                    f += r_hat * (sigma_eff * mass * mass * c);
                    f += (normals[i] - normals[j]) * (-sigma_eff * mass);
                }
                out[i] = V3{f.x / mass, f.y / mass, f.z / mass};
            }
        } else if (prm.st_model == 2) {
            const double gamma = prm.st_colour_gamma;
            for (size_t i = 0; i < n; ++i) {
                if (parts.kind[i] != FLUID) continue;
                V3 ni = normals[i];
                double n_len = norm(ni);
                if (n_len < 1e-8) continue;
                V3 n_hat{ni.x / n_len, ni.y / n_len, ni.z / n_len};
                neigh.clear();
                grid.neighbours(i, neigh);
                V3 xi = parts.x[i];
                double div_n = 0.0;
                for (size_t j : neigh) {
                    if (j == i || parts.kind[j] != FLUID) continue;
                    V3 gw = grad_w(kk(), parts.x[j] - xi, h, dim);
                    V3 nj = normals[j];
                    double nj_len = norm(nj);
                    V3 nj_hat = nj_len > 1e-8 ? V3{nj.x / nj_len, nj.y / nj_len, nj.z / nj_len} : zero3();
                    div_n += (mass / std::fmax(parts.rho[j], 1e-12)) * dot(nj_hat - n_hat, gw);
                }
                double kappa = -div_n;
                out[i] = n_hat * (-gamma * kappa / std::fmax(parts.rho[i], 1e-12));
            }
        }
    }
    // wcsph.rs:283 apply_xsph
    void apply_xsph() {
        double eps = prm.xsph_epsilon;
        if (eps == 0.0) return;
        size_t n = parts.len();
        double h = parts.h, mass = parts.mass;
        Dim dim = parts.dim;
        xsph_dv.assign(n, zero3());
        auto one = [&](size_t i, std::vector<size_t>& nb) {
            if (parts.kind[i] != FLUID) return;
            nb.clear();
            grid.neighbours(i, nb);
            V3 xi = parts.x[i], vi = parts.v[i];
            double rho_i = parts.rho[i];
            V3 dv = zero3();
            for (size_t j : nb) {
                if (j == i || parts.kind[j] != FLUID) continue;
                double r = norm(parts.x[j] - xi);
                double wij = kern_w(kk(), r, h, dim);
                double rho_bar = 0.5 * (rho_i + parts.rho[j]);
                dv += (parts.v[j] - vi) * (mass / rho_bar * wij);
            }
            xsph_dv[i] = dv * eps;
        };
        if (threads > 1) {
            std::vector<std::vector<size_t>> nb(threads);
            parallel_for(n, threads, [&](size_t i, int w) { one(i, nb[w]); });
        } else {
            for (size_t i = 0; i < n; ++i) one(i, neigh);
        }
        for (size_t i = 0; i < n; ++i)
            if (parts.kind[i] == FLUID) parts.v[i] += xsph_dv[i];
    }
    // wcsph.rs:326 step
    void step(double dt) {
        rebuild_grid();
        compute_density();
        compute_pressure();
        compute_forces();
        size_t n = parts.len();
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) continue;
            parts.v[i] += parts.a[i] * dt;
            parts.x[i] += parts.v[i] * dt;
            if (parts.dim == D2) {
                parts.x[i].z = 0.0;
                parts.v[i].z = 0.0;
            }
        }
        rebuild_grid();
        compute_density();
        apply_xsph();
        t += dt;
    }
    // wcsph.rs:361 a_max
    double a_max() const {
        double m = 0.0;
        for (size_t i = 0; i < parts.len(); ++i)
            if (parts.kind[i] == FLUID) m = std::fmax(m, norm2(parts.a[i]));
        return std::sqrt(m);
    }
};

// diagnostics.rs:10-33 FNV-1a over fluid (x, v) bits, little-endian bytes
static inline void fnv1a_f64(uint64_t* hsh, double x) {
    uint64_t bits;
    std::memcpy(&bits, &x, 8);
    for (int k = 0; k < 8; ++k) {
        *hsh ^= (bits >> (8 * k)) & 0xffULL;
        *hsh *= 0x100000001b3ULL;
    }
}
static uint64_t particles_hash64(const Particles& p) {
    uint64_t h = 0xcbf29ce484222325ULL;
    for (size_t i = 0; i < p.len(); ++i) {
        if (p.kind[i] != FLUID) continue;
        fnv1a_f64(&h, p.x[i].x); fnv1a_f64(&h, p.x[i].y); fnv1a_f64(&h, p.x[i].z);
        fnv1a_f64(&h, p.v[i].x); fnv1a_f64(&h, p.v[i].y); fnv1a_f64(&h, p.v[i].z);
    }
    return h;
}


// ---------------------------------------------------------------------------
// Position Based Fluids (pbf.rs:25-459)
// ---------------------------------------------------------------------------
static inline V3 cross(V3 a, V3 b) {  // vec3.rs:87-93
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

struct PParams {                 // pbf.rs:26-53
    int32_t density_kernel, grad_kernel;
    int64_t iterations;
    double epsilon_lambda, art_pressure_k, art_pressure_n, art_pressure_dq_over_h;
    double viscosity_eps, vorticity_eps;
    double gravity[3];
    int32_t reuse_neighbours;
};

struct PbfWorld {
    Particles parts;
    UniformGrid grid;
    PParams prm;
    double t = 0.0;
    std::vector<V3> pred, dp, dv_scratch, omega_scratch;
    std::vector<double> lambda, rho_pred;
    std::vector<std::vector<size_t>> neigh_lists;

    KernelKind dk() const { return (KernelKind)prm.density_kernel; }
    KernelKind gk() const { return (KernelKind)prm.grad_kernel; }

    // pbf.rs:112-130 new: the grid cell is the larger support radius
    PbfWorld(const Particles& p, const PParams& q) : parts(p), prm(q) {
        double s0 = support_radius(dk(), parts.h), s1 = support_radius(gk(), parts.h);
        grid.cell_size = std::fmax(s0, s1);
        grid.dim = parts.dim;
        ensure_buffers();
    }
    // pbf.rs:132-144
    void ensure_buffers() {
        size_t n = parts.len();
        pred.resize(n, zero3());
        lambda.resize(n, 0.0);
        dp.resize(n, zero3());
        rho_pred.resize(n, 0.0);
        dv_scratch.resize(n, zero3());
        omega_scratch.resize(n, zero3());
        neigh_lists.resize(n);
    }
    // pbf.rs:146-156: lists for fluid particles only
    void rebuild_neighbours(const std::vector<V3>& pos) {
        grid.rebuild(pos);
        for (size_t i = 0; i < parts.len(); ++i) {
            neigh_lists[i].clear();
            if (parts.kind[i] == FLUID) grid.neighbours(i, neigh_lists[i]);
        }
    }
    // pbf.rs:159-187
    void density_at_pred() {
        const double h = parts.h, mass = parts.mass, rho0 = parts.rest_density;
        const Dim dim = parts.dim;
        for (size_t i = 0; i < parts.len(); ++i) {
            if (parts.kind[i] != FLUID) {
                rho_pred[i] = rho0;
                parts.rho[i] = rho0;
                continue;
            }
            V3 xi = pred[i];
            double rho = mass * kern_w(dk(), 0.0, h, dim);
            for (size_t j : neigh_lists[i]) {
                if (j == i) continue;
                double r = norm(pred[j] - xi);
                double wij = kern_w(dk(), r, h, dim);
                if (parts.kind[j] == FLUID) rho += mass * wij;
                else rho += rho0 * parts.psi[j] * wij;
            }
            rho_pred[i] = std::fmax(rho, 1e-12);
            parts.rho[i] = rho_pred[i];
        }
    }
    // pbf.rs:189-227
    void compute_lambdas() {
        const double h = parts.h, mass = parts.mass, rho0 = parts.rest_density, eps = prm.epsilon_lambda;
        const Dim dim = parts.dim;
        for (size_t i = 0; i < parts.len(); ++i) {
            if (parts.kind[i] != FLUID) {
                lambda[i] = 0.0;
                continue;
            }
            double ci = rho_pred[i] / rho0 - 1.0;
            V3 xi = pred[i];
            double sum_grad_sq = 0.0;
            V3 grad_i = zero3();
            for (size_t j : neigh_lists[i]) {
                if (j == i) continue;
                V3 gw = grad_w(gk(), pred[j] - xi, h, dim);
                double scale = parts.kind[j] == FLUID ? mass / rho0 : parts.psi[j];
                V3 contrib = gw * scale;
                grad_i += contrib;
                if (parts.kind[j] == FLUID) sum_grad_sq += norm2(contrib);
            }
            sum_grad_sq += norm2(grad_i);
            lambda[i] = -ci / (sum_grad_sq + eps);
        }
    }
    // pbf.rs:229-235
    double artificial_pressure(double wij, double w_dq) const {
        if (w_dq <= 1e-30 || prm.art_pressure_k == 0.0) return 0.0;
        double ratio = std::fmin(wij / w_dq, 1.0);
        return -prm.art_pressure_k * oracle_pow(ratio, prm.art_pressure_n);
    }
    // pbf.rs:237-286
    void compute_delta_p() {
        const double h = parts.h, mass = parts.mass, rho0 = parts.rest_density;
        const Dim dim = parts.dim;
        const double dq = prm.art_pressure_dq_over_h * h;
        const double w_dq = kern_w(dk(), dq, h, dim);
        for (auto& d : dp) d = zero3();
        for (size_t i = 0; i < parts.len(); ++i) {
            if (parts.kind[i] != FLUID) continue;
            V3 xi = pred[i];
            V3 corr = zero3();
            for (size_t j : neigh_lists[i]) {
                if (j == i) continue;
                V3 rij = pred[j] - xi;
                double r = norm(rij);
                double wij = kern_w(dk(), r, h, dim);
                V3 gw = grad_w(gk(), rij, h, dim);
                double s_corr = artificial_pressure(wij, w_dq);
                if (parts.kind[j] == FLUID) {
                    double coeff = lambda[i] + lambda[j] + s_corr;
                    corr += gw * (mass / rho0 * coeff);
                } else {
                    double coeff = lambda[i] + s_corr;
                    corr += gw * (parts.psi[j] * coeff);
                }
            }
            double max_corr = 0.4 * h;
            double mag = norm(corr);
            if (mag > max_corr && mag > 0.0) corr = corr * (max_corr / mag);
            dp[i] = corr;
        }
    }
    // pbf.rs:288-381
    void apply_viscosity_and_vorticity(double dt) {
        const double h = parts.h, mass = parts.mass;
        const Dim dim = parts.dim;
        rebuild_neighbours(parts.x);
        const size_t n = parts.len();
        if (prm.viscosity_eps != 0.0) {
            for (auto& d : dv_scratch) d = zero3();
            for (size_t i = 0; i < n; ++i) {
                if (parts.kind[i] != FLUID) continue;
                V3 xi = parts.x[i], vi = parts.v[i];
                V3 corr = zero3();
                for (size_t j : neigh_lists[i]) {
                    if (j == i || parts.kind[j] != FLUID) continue;
                    double r = norm(parts.x[j] - xi);
                    double wij = kern_w(dk(), r, h, dim);
                    double rho_bar = 0.5 * (parts.rho[i] + parts.rho[j]);
                    corr += (parts.v[j] - vi) * (mass / std::fmax(rho_bar, 1e-12) * wij);
                }
                dv_scratch[i] = corr * prm.viscosity_eps;
            }
            for (size_t i = 0; i < n; ++i) parts.v[i] += dv_scratch[i];
        }
        if (prm.vorticity_eps == 0.0 || dt == 0.0) return;
        for (auto& o : omega_scratch) o = zero3();
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) continue;
            V3 xi = parts.x[i], vi = parts.v[i];
            V3 w_i = zero3();
            for (size_t j : neigh_lists[i]) {
                if (j == i || parts.kind[j] != FLUID) continue;
                V3 gw = grad_w(gk(), parts.x[j] - xi, h, dim);
                double rho_bar = 0.5 * (parts.rho[i] + parts.rho[j]);
                w_i += cross(parts.v[j] - vi, gw) * (mass / std::fmax(rho_bar, 1e-12));
            }
            omega_scratch[i] = w_i;
        }
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) continue;
            V3 xi = parts.x[i];
            V3 eta = zero3();
            double om_i = norm(omega_scratch[i]);
            for (size_t j : neigh_lists[i]) {
                if (j == i || parts.kind[j] != FLUID) continue;
                V3 gw = grad_w(gk(), parts.x[j] - xi, h, dim);
                double rho_bar = 0.5 * (parts.rho[i] + parts.rho[j]);
                eta += gw * (mass / std::fmax(rho_bar, 1e-12) * (norm(omega_scratch[j]) - om_i));
            }
            double nrm = norm(eta);
            if (nrm > 1e-12) {
                V3 n_hat{eta.x / nrm, eta.y / nrm, eta.z / nrm};
                V3 f = cross(n_hat, omega_scratch[i]) * prm.vorticity_eps;
                parts.v[i] += f * dt;
            }
        }
    }
    // pbf.rs:384-436
    void step(double dt) {
        ensure_buffers();
        const size_t n = parts.len();
        const V3 g{prm.gravity[0], prm.gravity[1], prm.gravity[2]};
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) {
                pred[i] = parts.x[i];
                continue;
            }
            parts.v[i] += g * dt;
            pred[i] = parts.x[i] + parts.v[i] * dt;
            if (parts.dim == D2) {
                pred[i].z = 0.0;
                parts.v[i].z = 0.0;
            }
        }
        rebuild_neighbours(pred);
        for (int64_t it = 0; it < prm.iterations; ++it) {
            density_at_pred();
            compute_lambdas();
            compute_delta_p();
            for (size_t i = 0; i < n; ++i)
                if (parts.kind[i] == FLUID) {
                    pred[i] += dp[i];
                    if (parts.dim == D2) pred[i].z = 0.0;
                }
            if (!prm.reuse_neighbours) rebuild_neighbours(pred);
        }
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) continue;
            if (dt > 0.0) parts.v[i] = (pred[i] - parts.x[i]) * (1.0 / dt);
            parts.x[i] = pred[i];
        }
        for (size_t i = 0; i < n; ++i) pred[i] = parts.x[i];
        rebuild_neighbours(pred);
        density_at_pred();
        apply_viscosity_and_vorticity(dt);
        t += dt;
    }
};

// ---------------------------------------------------------------------------
// Divergence-free SPH (dfsph.rs:33-800); surface tension (sigma != 0) is not
// restated.
// ---------------------------------------------------------------------------
struct DParams {                 // dfsph.rs:33-80
    int32_t kernel;
    int64_t max_density_iters, max_divergence_iters;
    double density_error_tol, divergence_error_tol;
    double gravity[3];
    double xsph_epsilon;
    double particle_diameter, cfl_lambda;
    int32_t adaptive_dt, warm_start;
    int32_t has_slip[4];         // free_slip_{xmin, ymin, xmax, ymax}.is_some()
    double slip[4];
    double solver_omega, max_velocity_correction;
};

// cfl.rs:36 suggested_dt
static double cfl_suggested_dt(double h, double c, double vmax, double amax, double lv, double lf) {
    double dt_v = lv * h / std::fmax(c + vmax, 1e-12);
    double dt_f = amax > 1e-12 ? lf * std::sqrt(h / amax) : std::numeric_limits<double>::infinity();
    return std::fmin(dt_v, dt_f);
}

struct DfsphWorld {
    Particles parts;
    UniformGrid grid;
    DParams prm;
    double t = 0.0, last_dt = 0.0;
    std::vector<double> alpha, kappa, kappa_v, kappa_warm, kappa_v_warm;
    std::vector<V3> v_star, a_adv, scratch_dv, dv_bound, boundary_force;
    std::vector<std::vector<size_t>> neigh_lists;
    std::vector<std::pair<size_t, double>> reaction_tmp;
    int64_t last_density_iters = 0, last_divergence_iters = 0;

    KernelKind kk() const { return (KernelKind)prm.kernel; }

    // dfsph.rs:137-180 new
    DfsphWorld(const Particles& p, const DParams& q) : parts(p), prm(q) {
        if (prm.particle_diameter <= 0.0) prm.particle_diameter = parts.h;
        grid.cell_size = support_radius(kk(), parts.h);
        grid.dim = parts.dim;
        if (parts.dim == D2)
            for (size_t i = 0; i < parts.len(); ++i) {
                parts.x[i].z = 0.0;
                parts.v[i].z = 0.0;
            }
        rebuild_neighbours();
        compute_density();
        compute_alpha();
    }
    // dfsph.rs:182-198
    void ensure_buffers() {
        size_t n = parts.len();
        alpha.resize(n, 0.0);
        v_star.resize(n, zero3());
        kappa.resize(n, 0.0);
        kappa_v.resize(n, 0.0);
        kappa_warm.resize(n, 0.0);
        kappa_v_warm.resize(n, 0.0);
        a_adv.resize(n, zero3());
        scratch_dv.resize(n, zero3());
        dv_bound.resize(n, zero3());
        boundary_force.resize(n, zero3());
        neigh_lists.resize(n);
    }
    // dfsph.rs:201-211
    void rebuild_neighbours() {
        ensure_buffers();
        grid.rebuild(parts.x);
        for (size_t i = 0; i < parts.len(); ++i) {
            neigh_lists[i].clear();
            if (parts.kind[i] == FLUID) grid.neighbours(i, neigh_lists[i]);
        }
    }
    // dfsph.rs:214-244
    void compute_density() {
        const double h = parts.h, mass = parts.mass, rho0 = parts.rest_density;
        const Dim dim = parts.dim;
        for (size_t i = 0; i < parts.len(); ++i) {
            if (parts.kind[i] != FLUID) {
                parts.rho[i] = rho0;
                continue;
            }
            V3 xi = parts.x[i];
            double rho = mass * kern_w(kk(), 0.0, h, dim);
            for (size_t j : neigh_lists[i]) {
                if (j == i) continue;
                double wij = kern_w(kk(), norm(parts.x[j] - xi), h, dim);
                if (parts.kind[j] == FLUID) rho += mass * wij;
                else if (parts.boundary_sees_fluid(j, xi)) rho += rho0 * parts.psi[j] * wij;
            }
            parts.rho[i] = std::fmax(rho, 1e-12);
        }
    }
    // dfsph.rs:252-307
    void compute_alpha() {
        const double h = parts.h, mass = parts.mass, rho0 = parts.rest_density;
        const Dim dim = parts.dim;
        double h_safe = std::fmax(h, 1e-12);
        double char_grad = dim == D2 ? mass / (h_safe * h_safe * h_safe) : mass / (h_safe * h_safe * h_safe * h_safe);
        double denom_floor = std::fmax(1e-6 * char_grad * char_grad, 1e-12);
        for (size_t i = 0; i < parts.len(); ++i) {
            if (parts.kind[i] != FLUID) {
                alpha[i] = 0.0;
                continue;
            }
            V3 xi = parts.x[i];
            V3 sum_grad = zero3();
            double sum_grad_sq = 0.0;
            size_t n_nbr = 0;
            for (size_t j : neigh_lists[i]) {
                if (j == i) continue;
                V3 gw = grad_w(kk(), parts.x[j] - xi, h, dim);
                double mj = parts.kind[j] == FLUID ? mass
                            : (parts.boundary_sees_fluid(j, xi) ? rho0 * parts.psi[j] : 0.0);
                if (mj == 0.0 && parts.kind[j] == BOUNDARY) continue;
                V3 g = gw * mj;
                sum_grad += g;
                sum_grad_sq += norm2(g);
                n_nbr += 1;
            }
            if (n_nbr < 2) {
                alpha[i] = 0.0;
                continue;
            }
            double denom = std::fmax(norm2(sum_grad) + sum_grad_sq, denom_floor);
            alpha[i] = parts.rho[i] / denom;
        }
    }
    // dfsph.rs:309-323
    double neighbour_mass_for(size_t i, size_t j) const {
        if (parts.kind[j] == FLUID) return parts.mass;
        return parts.boundary_sees_fluid(j, parts.x[i]) ? parts.rest_density * parts.psi[j] : 0.0;
    }
    // dfsph.rs:326-351
    double density_derivative(size_t i) const {
        const double h = parts.h;
        const Dim dim = parts.dim;
        V3 xi = parts.x[i], vi = v_star[i];
        double drho = 0.0;
        for (size_t j : neigh_lists[i]) {
            if (j == i) continue;
            double mj = neighbour_mass_for(i, j);
            if (mj == 0.0) continue;
            V3 gw = grad_w(kk(), parts.x[j] - xi, h, dim);
            V3 vj = parts.kind[j] == FLUID ? v_star[j] : parts.v[j];
            drho += mj * dot(vi - vj, gw);
        }
        return drho;
    }
    // dfsph.rs:353-379 (surface tension not restated)
    void compute_nonpressure_accel() {
        const V3 g{prm.gravity[0], prm.gravity[1], prm.gravity[2]};
        for (size_t i = 0; i < parts.len(); ++i) a_adv[i] = parts.kind[i] == FLUID ? g : zero3();
    }
    // dfsph.rs:382-416
    void apply_xsph_on_vstar() {
        const double eps = prm.xsph_epsilon;
        if (eps == 0.0) return;
        const double h = parts.h, mass = parts.mass;
        const Dim dim = parts.dim;
        for (auto& d : scratch_dv) d = zero3();
        for (size_t i = 0; i < parts.len(); ++i) {
            if (parts.kind[i] != FLUID) continue;
            V3 xi = parts.x[i], vi = v_star[i];
            double rho_i = parts.rho[i];
            V3 dv = zero3();
            for (size_t j : neigh_lists[i]) {
                if (j == i || parts.kind[j] != FLUID) continue;
                double wij = kern_w(kk(), norm(parts.x[j] - xi), h, dim);
                double rho_bar = 0.5 * (rho_i + parts.rho[j]);
                dv += (v_star[j] - vi) * (mass / std::fmax(rho_bar, 1e-12) * wij);
            }
            scratch_dv[i] = dv * eps;
        }
        for (size_t i = 0; i < parts.len(); ++i)
            if (parts.kind[i] == FLUID) v_star[i] += scratch_dv[i];
    }
    // dfsph.rs:422-530
    void apply_pressure_velocity_update(double dt, bool use_divergence) {
        const double h = parts.h;
        const Dim dim = parts.dim;
        const std::vector<double>& kap = use_divergence ? kappa_v : kappa;
        const size_t n = parts.len();
        for (auto& d : scratch_dv) d = zero3();
        for (auto& d : dv_bound) d = zero3();
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) continue;
            V3 xi = parts.x[i];
            double rho_i = std::fmax(parts.rho[i], 1e-12);
            double ki = kap[i];
            V3 dv = zero3(), dv_b = zero3();
            for (size_t j : neigh_lists[i]) {
                if (j == i) continue;
                double mj = neighbour_mass_for(i, j);
                if (mj == 0.0) continue;
                V3 gw = grad_w(kk(), parts.x[j] - xi, h, dim);
                double kj = parts.kind[j] == FLUID ? kap[j] : 0.0;
                double rho_j = parts.kind[j] == FLUID ? std::fmax(parts.rho[j], 1e-12) : parts.rest_density;
                double coeff = mj * (ki / rho_i + kj / rho_j);
                V3 term = gw * coeff;
                dv += term;
                if (parts.kind[j] == BOUNDARY) dv_b += term;
            }
            scratch_dv[i] = dv * (-dt);
            dv_bound[i] = dv_b * (-dt);
        }
        const double dv_cap = prm.max_velocity_correction, mass = parts.mass;
        const double inv_dt = 1.0 / std::fmax(dt, 1e-12);
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) continue;
            V3 dv = scratch_dv[i];
            double scale = 1.0;
            if (dv_cap > 0.0) {
                double s2 = norm2(dv);
                if (s2 > dv_cap * dv_cap) {
                    scale = dv_cap / std::sqrt(s2);
                    dv = dv * scale;
                }
            }
            V3 dv_b = dv_bound[i] * scale;
            if (norm2(dv_b) > 0.0) {
                V3 xi = parts.x[i];
                double wsum = 0.0;
                reaction_tmp.clear();
                for (size_t j : neigh_lists[i]) {
                    if (parts.kind[j] != BOUNDARY) continue;
                    if (!parts.boundary_sees_fluid(j, xi)) continue;
                    double r = norm(parts.x[j] - xi);
                    double wt = std::fmin(1.0 / std::fmax(r, 1e-9), 1e6);
                    wsum += wt;
                    reaction_tmp.push_back({j, wt});
                }
                if (wsum > 0.0) {
                    V3 fb_total = dv_b * (-mass * inv_dt);
                    for (auto& jw : reaction_tmp) boundary_force[jw.first] += fb_total * (jw.second / wsum);
                }
            }
            v_star[i] += dv;
            if (parts.dim == D2) v_star[i].z = 0.0;
        }
    }
    // dfsph.rs:533-584
    int64_t correct_density_error(double dt) {
        const size_t n = parts.len();
        const double rho0 = parts.rest_density, dt2 = dt * dt;
        int64_t iters = 0;
        if (prm.warm_start) {
            for (size_t i = 0; i < n; ++i) kappa[i] = kappa_warm[i];
            apply_pressure_velocity_update(dt, false);
        }
        std::fill(kappa_warm.begin(), kappa_warm.end(), 0.0);
        for (;;) {
            double avg_err = 0.0;
            size_t count = 0;
            for (size_t i = 0; i < n; ++i) {
                if (parts.kind[i] != FLUID) {
                    kappa[i] = 0.0;
                    continue;
                }
                double rho_star = parts.rho[i] + dt * density_derivative(i);
                double err = std::fmax(rho_star - rho0, 0.0);
                avg_err += err / rho0;
                count += 1;
                kappa[i] = prm.solver_omega * err / dt2 * alpha[i];
                if (prm.warm_start) kappa_warm[i] += kappa[i];
            }
            if (count > 0) avg_err /= (double)count;
            apply_pressure_velocity_update(dt, false);
            iters += 1;
            if ((avg_err <= prm.density_error_tol && iters >= 2) || iters >= prm.max_density_iters) break;
        }
        return iters;
    }
    // dfsph.rs:587-630
    int64_t correct_divergence_error(double dt) {
        const size_t n = parts.len();
        const double rho0 = parts.rest_density;
        int64_t iters = 0;
        if (prm.warm_start) {
            for (size_t i = 0; i < n; ++i) kappa_v[i] = kappa_v_warm[i];
            apply_pressure_velocity_update(dt, true);
        }
        std::fill(kappa_v_warm.begin(), kappa_v_warm.end(), 0.0);
        for (;;) {
            double avg = 0.0;
            size_t count = 0;
            for (size_t i = 0; i < n; ++i) {
                if (parts.kind[i] != FLUID) {
                    kappa_v[i] = 0.0;
                    continue;
                }
                double drho = std::fmax(density_derivative(i), 0.0);
                avg += drho / rho0;
                count += 1;
                kappa_v[i] = prm.solver_omega * (1.0 / dt) * drho * alpha[i];
                if (prm.warm_start) kappa_v_warm[i] += kappa_v[i];
            }
            if (count > 0) avg /= (double)count;
            apply_pressure_velocity_update(dt, true);
            iters += 1;
            if ((avg <= prm.divergence_error_tol && iters >= 1) || iters >= prm.max_divergence_iters) break;
        }
        return iters;
    }
    // dfsph.rs:633-665 suggest_dt
    double suggest_dt() const {
        double vmax = 0.0, amax = 0.0;
        for (size_t i = 0; i < parts.len(); ++i) {
            if (parts.kind[i] != FLUID) continue;
            vmax = std::fmax(vmax, norm2(parts.v[i]));
            amax = std::fmax(amax, norm2(a_adv[i]));
        }
        vmax = std::sqrt(vmax);
        amax = std::sqrt(amax);
        double d = std::fmax(prm.particle_diameter, 1e-12);
        double dt_v = prm.cfl_lambda * d / std::fmax(vmax, 1e-6);
        double dt_f = cfl_suggested_dt(parts.h, 0.0, vmax, std::fmax(amax, 1e-6), prm.cfl_lambda, 0.25);
        double r = std::fmin(dt_v, dt_f);
        return r < 1e-6 ? 1e-6 : (r > 1e-2 ? 1e-2 : r);  // f64::clamp
    }
    // dfsph.rs:668-715
    void apply_free_slip_walls() {
        if (!prm.has_slip[0] && !prm.has_slip[1] && !prm.has_slip[2] && !prm.has_slip[3]) return;
        for (size_t i = 0; i < parts.len(); ++i) {
            if (parts.kind[i] != FLUID) continue;
            V3 x = parts.x[i], v = v_star[i];
            if (prm.has_slip[0] && x.x < prm.slip[0]) {
                x.x = prm.slip[0];
                if (v.x < 0.0) v.x = 0.0;
            }
            if (prm.has_slip[1] && x.y < prm.slip[1]) {
                x.y = prm.slip[1];
                if (v.y < 0.0) v.y = 0.0;
            }
            if (prm.has_slip[2] && x.x > prm.slip[2]) {
                x.x = prm.slip[2];
                if (v.x > 0.0) v.x = 0.0;
            }
            if (prm.has_slip[3] && x.y > prm.slip[3]) {
                x.y = prm.slip[3];
                if (v.y > 0.0) v.y = 0.0;
            }
            parts.x[i] = x;
            v_star[i] = v;
        }
    }
    // dfsph.rs:718-769 step
    void step(double dt_in) {
        ensure_buffers();
        const size_t n = parts.len();
        const double dt = std::fmax(dt_in, 1e-12);
        last_dt = dt;
        for (auto& f : boundary_force) f = zero3();
        compute_nonpressure_accel();
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) {
                v_star[i] = parts.v[i];
                continue;
            }
            v_star[i] = parts.v[i] + a_adv[i] * dt;
            if (parts.dim == D2) v_star[i].z = 0.0;
        }
        apply_xsph_on_vstar();
        last_density_iters = correct_density_error(dt);
        for (size_t i = 0; i < n; ++i) {
            if (parts.kind[i] != FLUID) continue;
            parts.x[i] += v_star[i] * dt;
            if (parts.dim == D2) parts.x[i].z = 0.0;
        }
        apply_free_slip_walls();
        rebuild_neighbours();
        compute_density();
        compute_alpha();
        last_divergence_iters = correct_divergence_error(dt);
        apply_free_slip_walls();
        for (size_t i = 0; i < n; ++i)
            if (parts.kind[i] == FLUID) {
                parts.v[i] = v_star[i];
                parts.p[i] = kappa[i];
                if (parts.dim == D2) parts.v[i].z = 0.0;
            }
        t += dt;
    }
    // dfsph.rs:772-784 step_adaptive
    double step_adaptive() {
        ensure_buffers();
        compute_nonpressure_accel();
        double dt = prm.adaptive_dt ? suggest_dt() : std::fmax(last_dt, 1e-4);
        step(dt);
        return dt;
    }
};
}  // namespace oracle

// ===========================================================================
// C ABI used by the test suite (ctypes). Buffers are caller-owned, SoA in
// original particle order, `[n*3]` for vectors.
// ===========================================================================
using namespace oracle;

extern "C" {

struct OScene;  // opaque particle builder
OScene* oscene_new(int dim, double rho0, double mass, double h) {
    Particles* p = new (std::nothrow) Particles();
    if (!p) return nullptr;
    p->dim = dim == 2 ? D2 : D3;
    p->rest_density = rho0;
    p->mass = mass;
    p->h = h;
    return reinterpret_cast<OScene*>(p);
}
void oscene_free(OScene* s) { delete reinterpret_cast<Particles*>(s); }
long oscene_len(OScene* s) { return (long)reinterpret_cast<Particles*>(s)->len(); }
void oscene_push_fluid(OScene* s, const double* x, const double* v) {
    reinterpret_cast<Particles*>(s)->push_fluid(v3(x[0], x[1], x[2]), v3(v[0], v[1], v[2]));
}
void oscene_push_boundary(OScene* s, const double* x, double psi, const double* n_out) {
    V3 n = n_out ? v3(n_out[0], n_out[1], n_out[2]) : zero3();
    reinterpret_cast<Particles*>(s)->push_boundary(v3(x[0], x[1], x[2]), psi, n);
}
void oscene_fill_box(OScene* s, const double* origin, long nx, long ny, long nz, double dx,
                     const double* v0) {
    fill_box(*reinterpret_cast<Particles*>(s), v3(origin[0], origin[1], origin[2]), (size_t)nx,
             (size_t)ny, (size_t)nz, dx, v3(v0[0], v0[1], v0[2]));
}
void oscene_fill_box_boundary(OScene* s, const double* mn, const double* mx, double dx, long layers) {
    fill_box_boundary(*reinterpret_cast<Particles*>(s), v3(mn[0], mn[1], mn[2]),
                      v3(mx[0], mx[1], mx[2]), dx, (size_t)layers);
}
void oscene_recompute_psi(OScene* s, int kernel) {
    recomputed_akinci_psi(*reinterpret_cast<Particles*>(s), (KernelKind)kernel);
}
// Seeded lattice jitter of the fluid particles: xoshiro256** draws in particle
// order, x then y (then z in 3-D), each U(-amp, amp), added component-wise.
void oscene_jitter_fluid(OScene* s, uint64_t seed, double amp) {
    Particles& p = *reinterpret_cast<Particles*>(s);
    Xoshiro r = xoshiro_seed(seed);
    for (size_t i = 0; i < p.len(); ++i) {
        if (p.kind[i] != FLUID) continue;
        double jx = xoshiro_uniform(&r, -amp, amp);
        double jy = xoshiro_uniform(&r, -amp, amp);
        double jz = p.dim == D3 ? xoshiro_uniform(&r, -amp, amp) : 0.0;
        p.x[i] = p.x[i] + v3(jx, jy, jz);
    }
}
void oscene_export(OScene* s, double* x, double* v, uint8_t* kind, double* psi, double* n_out) {
    Particles& p = *reinterpret_cast<Particles*>(s);
    for (size_t i = 0; i < p.len(); ++i) {
        if (x) { x[3 * i] = p.x[i].x; x[3 * i + 1] = p.x[i].y; x[3 * i + 2] = p.x[i].z; }
        if (v) { v[3 * i] = p.v[i].x; v[3 * i + 1] = p.v[i].y; v[3 * i + 2] = p.v[i].z; }
        if (kind) kind[i] = p.kind[i];
        if (psi) psi[i] = p.psi[i];
        if (n_out) { n_out[3 * i] = p.n_out[i].x; n_out[3 * i + 1] = p.n_out[i].y; n_out[3 * i + 2] = p.n_out[i].z; }
    }
}

double o_mass_from_spacing(double rho0, double dx, int dim) {
    return mass_from_spacing(rho0, dx, dim == 2 ? D2 : D3);
}
double o_mass_calibrated_to_rest(double rho0, double dx, double h, int dim, int kernel) {
    return mass_calibrated_to_rest(rho0, dx, h, dim == 2 ? D2 : D3, (KernelKind)kernel);
}
double o_kernel_w(int kernel, double r, double h, int dim) {
    return kern_w((KernelKind)kernel, r, h, dim == 2 ? D2 : D3);
}
void o_grad_w(int kernel, const double* rij, double h, int dim, double* out) {
    V3 g = grad_w((KernelKind)kernel, v3(rij[0], rij[1], rij[2]), h, dim == 2 ? D2 : D3);
    out[0] = g.x; out[1] = g.y; out[2] = g.z;
}
double o_pow(double x, double y) { return oracle_pow(x, y); }
// viscosity.rs:51 pi_ij with explicit parameters
double o_pi_ij(double alpha, double beta, double eps, double h, double c, const double* xi,
               const double* xj, const double* vi, const double* vj, double rho_i, double rho_j) {
    World w;
    w.prm.visc_alpha = alpha;
    w.prm.visc_beta = beta;
    w.prm.visc_eps = eps;
    return w.pi_ij(h, c, v3(xi[0], xi[1], xi[2]), v3(xj[0], xj[1], xj[2]), v3(vi[0], vi[1], vi[2]),
                   v3(vj[0], vj[1], vj[2]), rho_i, rho_j);
}
// eos.rs:65 TaitEos::pressure
double o_tait_pressure(double rest_density, double sound_speed, double gamma, double density) {
    World w;
    w.prm.eos_rest_density = rest_density;
    w.prm.eos_sound_speed = sound_speed;
    w.prm.eos_gamma = gamma;
    return w.eos_pressure(density);
}
int32_t o_floor_i32(double x) { return floor_i32(x); }
uint64_t o_xoshiro_first(uint64_t seed, long n, uint64_t* out) {
    Xoshiro r = xoshiro_seed(seed);
    uint64_t last = 0;
    for (long i = 0; i < n; ++i) { last = xoshiro_next(&r); if (out) out[i] = last; }
    return last;
}

struct OWorld;
OWorld* ow_create(OScene* s, const WParams* prm) {
    World* w = new (std::nothrow) World();
    if (!w) return nullptr;
    w->parts = *reinterpret_cast<Particles*>(s);
    w->prm = *prm;
    w->grid.cell_size = support_radius((KernelKind)prm->kernel, w->parts.h);
    w->grid.dim = w->parts.dim;
    w->neigh_lists.resize(w->parts.len());
    w->boundary_force.assign(w->parts.len(), zero3());
    return reinterpret_cast<OWorld*>(w);
}
void ow_free(OWorld* w) { delete reinterpret_cast<World*>(w); }
static inline World& W(OWorld* w) { return *reinterpret_cast<World*>(w); }
long ow_len(OWorld* w) { return (long)W(w).parts.len(); }
void ow_step(OWorld* w, double dt) { W(w).step(dt); }
void ow_run(OWorld* w, double dt, long steps) { for (long k = 0; k < steps; ++k) W(w).step(dt); }
void ow_rebuild_grid(OWorld* w) { W(w).rebuild_grid(); }
void ow_compute_density(OWorld* w) { W(w).compute_density(); }
void ow_compute_pressure(OWorld* w) { W(w).compute_pressure(); }
void ow_compute_forces(OWorld* w) { W(w).compute_forces(); }
void ow_apply_xsph(OWorld* w) { W(w).apply_xsph(); }
double ow_time(OWorld* w) { return W(w).t; }
double ow_sound_speed(OWorld* w) { return W(w).prm.eos_sound_speed; }
double ow_a_max(OWorld* w) { return W(w).a_max(); }
double ow_v_max(OWorld* w) { return W(w).max_speed(); }
uint64_t ow_hash(OWorld* w) { return particles_hash64(W(w).parts); }
void ow_set_threads(OWorld* w, int threads) { W(w).threads = threads < 1 ? 1 : threads; }
void ow_set_pow_perturbation(OWorld* w, double rate, uint64_t seed) {
    W(w).pow_perturb_rate = rate;
    W(w).pow_perturb_seed = seed;
}

static void put3(const std::vector<V3>& src, double* out) {
    for (size_t i = 0; i < src.size(); ++i) {
        out[3 * i] = src[i].x; out[3 * i + 1] = src[i].y; out[3 * i + 2] = src[i].z;
    }
}
static void get3(std::vector<V3>& dst, const double* in) {
    for (size_t i = 0; i < dst.size(); ++i) dst[i] = v3(in[3 * i], in[3 * i + 1], in[3 * i + 2]);
}
void ow_get_x(OWorld* w, double* out) { put3(W(w).parts.x, out); }
void ow_get_v(OWorld* w, double* out) { put3(W(w).parts.v, out); }
void ow_get_a(OWorld* w, double* out) { put3(W(w).parts.a, out); }
void ow_get_boundary_force(OWorld* w, double* out) { put3(W(w).boundary_force, out); }

// ---- fluid side of the WCSPH-rigid coupling (coupling.rs:289-330) ----
// quat.rs:119-137 to_matrix and quat.rs:102-109 rotate, q = (w, x, y, z)
static V3 quat_rotate(const double* q, V3 v) {
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    const double r00 = 1.0 - 2.0 * (y * y + z * z), r01 = 2.0 * (x * y - w * z), r02 = 2.0 * (x * z + w * y);
    const double r10 = 2.0 * (x * y + w * z), r11 = 1.0 - 2.0 * (x * x + z * z), r12 = 2.0 * (y * z - w * x);
    const double r20 = 2.0 * (x * z - w * y), r21 = 2.0 * (y * z + w * x), r22 = 1.0 - 2.0 * (x * x + y * y);
    return V3{r00 * v.x + r01 * v.y + r02 * v.z, r10 * v.x + r11 * v.y + r12 * v.z,
              r20 * v.x + r21 * v.y + r22 * v.z};
}

// vec3.rs:87-93
static V3 cross3(V3 a, V3 b) {
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// FluidRigidCoupler::sync_from_rigid (coupling.rs:289-306): per sample, in
// order, x = X + R(q) local, v = V + omega x r, n_out = R(q) local_n; bodies
// give X (3), q (4: w, x, y, z), V (3) and the world-frame omega (3).
void o_coupler_sync(OWorld* wp, uint64_t ns, const int64_t* body, const double* local, const double* local_n,
                    const int64_t* particle, const double* X, const double* Q, const double* V,
                    const double* Om) {
    Particles& parts = W(wp).parts;
    for (uint64_t k = 0; k < ns; ++k) {
        const int64_t b = body[k], i = particle[k];
        const V3 xb{X[3 * b], X[3 * b + 1], X[3 * b + 2]}, vb{V[3 * b], V[3 * b + 1], V[3 * b + 2]};
        const V3 wb{Om[3 * b], Om[3 * b + 1], Om[3 * b + 2]};
        const V3 r = quat_rotate(Q + 4 * b, V3{local[3 * k], local[3 * k + 1], local[3 * k + 2]});
        parts.x[i] = xb + r;
        parts.v[i] = vb + cross3(wb, r);
        parts.n_out[i] = quat_rotate(Q + 4 * b, V3{local_n[3 * k], local_n[3 * k + 1], local_n[3 * k + 2]});
        if (parts.dim == D2) {
            parts.x[i].z = 0.0;
            parts.v[i].z = 0.0;
            parts.n_out[i].z = 0.0;
        }
    }
}

// FluidRigidCoupler::reduce_with_state (coupling.rs:308-330): per body the sum
// of its samples' boundary forces and of r x f with r = x - X, in sample order.
void o_coupler_reduce(OWorld* wp, uint64_t ns, const int64_t* body, const int64_t* particle, uint64_t nb,
                      const double* X, double* force, double* torque) {
    World& w = W(wp);
    std::vector<V3> f(nb, zero3()), t(nb, zero3());
    for (uint64_t k = 0; k < ns; ++k) {
        const int64_t b = body[k], i = particle[k];
        const V3 fb = (size_t)i < w.boundary_force.size() ? w.boundary_force[i] : zero3();
        f[b] += fb;
        const V3 r = w.parts.x[i] - V3{X[3 * b], X[3 * b + 1], X[3 * b + 2]};
        t[b] += cross3(r, fb);
    }
    put3(f, force);
    put3(t, torque);
}
void ow_get_rho(OWorld* w, double* out) { std::copy(W(w).parts.rho.begin(), W(w).parts.rho.end(), out); }
void ow_get_p(OWorld* w, double* out) { std::copy(W(w).parts.p.begin(), W(w).parts.p.end(), out); }
void ow_set_x(OWorld* w, const double* in) { get3(W(w).parts.x, in); }
void ow_set_v(OWorld* w, const double* in) { get3(W(w).parts.v, in); }
void ow_set_rho(OWorld* w, const double* in) { std::copy(in, in + W(w).parts.len(), W(w).parts.rho.begin()); }
void ow_set_p(OWorld* w, const double* in) { std::copy(in, in + W(w).parts.len(), W(w).parts.p.begin()); }

// Grid export: keys [n*3] per original index, order [n], occupied [m*3],
// ranges [m*2]; ow_grid_occupied_count gives m.
long ow_grid_occupied_count(OWorld* w) { return (long)W(w).grid.occupied.size(); }
void ow_get_grid(OWorld* w, int32_t* keys, int64_t* order, int32_t* occupied, int64_t* ranges) {
    UniformGrid& g = W(w).grid;
    for (size_t i = 0; i < g.keys.size(); ++i) {
        if (keys) { keys[3 * i] = g.keys[i].ix; keys[3 * i + 1] = g.keys[i].iy; keys[3 * i + 2] = g.keys[i].iz; }
    }
    for (size_t s = 0; s < g.order.size(); ++s) if (order) order[s] = (int64_t)g.order[s];
    for (size_t c = 0; c < g.occupied.size(); ++c) {
        if (occupied) { occupied[3 * c] = g.occupied[c].ix; occupied[3 * c + 1] = g.occupied[c].iy; occupied[3 * c + 2] = g.occupied[c].iz; }
        if (ranges) { ranges[2 * c] = (int64_t)g.ranges[c].first; ranges[2 * c + 1] = (int64_t)g.ranges[c].second; }
    }
}
// Per-particle candidate count (= neigh_lists[i].len(), self included; 0 for
// boundary) and in-support count (j != i with q = r/h < 2, kernel support).
void ow_neighbour_counts(OWorld* w, int32_t* candidates, int32_t* in_support) {
    World& wd = W(w);
    std::vector<size_t> tmp;
    double h = wd.parts.h;
    for (size_t i = 0; i < wd.parts.len(); ++i) {
        if (wd.parts.kind[i] != FLUID) {
            if (candidates) candidates[i] = 0;
            if (in_support) in_support[i] = 0;
            continue;
        }
        tmp.clear();
        wd.grid.neighbours(i, tmp);
        if (candidates) candidates[i] = (int32_t)tmp.size();
        if (in_support) {
            int32_t c = 0;
            for (size_t j : tmp) {
                if (j == i) continue;
                double r = norm(wd.parts.x[j] - wd.parts.x[i]);
                if (r / h < 2.0) ++c;
            }
            in_support[i] = c;
        }
    }
}

// Diagnostics (diagnostics.rs:35-102), cfl.rs:36 suggested_dt.
double o_total_mass(OWorld* w) { return W(w).parts.mass * (double)W(w).parts.fluid_count(); }
void o_linear_momentum(OWorld* w, double* out) {
    Particles& p = W(w).parts;
    V3 m = zero3();
    for (size_t i = 0; i < p.len(); ++i) if (p.kind[i] == FLUID) m += p.v[i] * p.mass;
    out[0] = m.x; out[1] = m.y; out[2] = m.z;
}
double o_kinetic_energy(OWorld* w) {
    Particles& p = W(w).parts;
    double ke = 0.0;
    for (size_t i = 0; i < p.len(); ++i) if (p.kind[i] == FLUID) ke += 0.5 * p.mass * norm2(p.v[i]);
    return ke;
}
double o_gravitational_potential(OWorld* w, double g) {
    Particles& p = W(w).parts;
    double pe = 0.0;
    for (size_t i = 0; i < p.len(); ++i) if (p.kind[i] == FLUID) pe += p.mass * g * p.x[i].z;
    return pe;
}
double o_mean_density_error(OWorld* w) {
    Particles& p = W(w).parts;
    double s = 0.0;
    size_t n = 0;
    for (size_t i = 0; i < p.len(); ++i)
        if (p.kind[i] == FLUID) { s += std::fabs(p.rho[i] - p.rest_density) / p.rest_density; ++n; }
    return n == 0 ? 0.0 : s / (double)n;
}
double o_max_density_error(OWorld* w) {
    Particles& p = W(w).parts;
    double m = 0.0;
    for (size_t i = 0; i < p.len(); ++i)
        if (p.kind[i] == FLUID) {
            double e = std::fabs(p.rho[i] - p.rest_density) / p.rest_density;
            if (e > m) m = e;
        }
    return m;
}
double o_suggested_dt(double h, double c, double vmax, double amax, double lv, double lf) {
    double dt_v = lv * h / std::fmax(c + vmax, 1e-12);
    double dt_f = amax > 1e-12 ? lf * std::sqrt(h / amax) : std::numeric_limits<double>::infinity();
    return std::fmin(dt_v, dt_f);
}


// ---- PBF (pbf.rs) ----
struct OPbf;
static PbfWorld& P(OPbf* w) { return *reinterpret_cast<PbfWorld*>(w); }
OPbf* opbf_create(OScene* s, const PParams* prm) {
    return reinterpret_cast<OPbf*>(new PbfWorld(*reinterpret_cast<Particles*>(s), *prm));
}
void opbf_free(OPbf* w) { delete reinterpret_cast<PbfWorld*>(w); }
void opbf_run(OPbf* w, double dt, long steps) {
    for (long k = 0; k < steps; ++k) P(w).step(dt);
}
uint64_t opbf_hash(OPbf* w) { return particles_hash64(P(w).parts); }
double opbf_time(OPbf* w) { return P(w).t; }
void opbf_get_x(OPbf* w, double* out) { put3(P(w).parts.x, out); }
void opbf_get_v(OPbf* w, double* out) { put3(P(w).parts.v, out); }
void opbf_get_rho(OPbf* w, double* out) { std::copy(P(w).parts.rho.begin(), P(w).parts.rho.end(), out); }
void opbf_get_lambda(OPbf* w, double* out) { std::copy(P(w).lambda.begin(), P(w).lambda.end(), out); }

// ---- DFSPH (dfsph.rs) ----
struct ODfsph;
static DfsphWorld& D(ODfsph* w) { return *reinterpret_cast<DfsphWorld*>(w); }
ODfsph* odfsph_create(OScene* s, const DParams* prm) {
    return reinterpret_cast<ODfsph*>(new DfsphWorld(*reinterpret_cast<Particles*>(s), *prm));
}
void odfsph_free(ODfsph* w) { delete reinterpret_cast<DfsphWorld*>(w); }
void odfsph_run(ODfsph* w, double dt, long steps) {
    for (long k = 0; k < steps; ++k) D(w).step(dt);
}
double odfsph_step_adaptive(ODfsph* w) { return D(w).step_adaptive(); }
uint64_t odfsph_hash(ODfsph* w) { return particles_hash64(D(w).parts); }
double odfsph_time(ODfsph* w) { return D(w).t; }
void odfsph_iters(ODfsph* w, int64_t* out) {
    out[0] = D(w).last_density_iters;
    out[1] = D(w).last_divergence_iters;
}
void odfsph_get_x(ODfsph* w, double* out) { put3(D(w).parts.x, out); }
void odfsph_get_v(ODfsph* w, double* out) { put3(D(w).parts.v, out); }
void odfsph_get_boundary_force(ODfsph* w, double* out) { put3(D(w).boundary_force, out); }
void odfsph_get_rho(ODfsph* w, double* out) { std::copy(D(w).parts.rho.begin(), D(w).parts.rho.end(), out); }
void odfsph_get_p(ODfsph* w, double* out) { std::copy(D(w).parts.p.begin(), D(w).parts.p.end(), out); }
void odfsph_get_alpha(ODfsph* w, double* out) { std::copy(D(w).alpha.begin(), D(w).alpha.end(), out); }
}  // extern "C"
