// Opaque C-ABI handles and argument helpers shared by the ABI translation units.
#pragma once

#include <cmath>
#include <new>
#include <stdexcept>
#include <vector>

#include "../../include/pe_fluid_wcsph.h"
#include "world.cuh"

struct PeWcsph {
    pe::World* world;
};

struct PeParticles {
    int32_t dim;
    double rest_density, mass, h;
    std::vector<double> x, v, psi, n_out;  // [n*3], [n*3], [n], [n*3]
    std::vector<uint8_t> kind;
    uint64_t len() const { return kind.size(); }
};

namespace peabi {

// Runs f, mapping C++ exceptions to the pe-ffi error codes (nothing unwinds
// across the C boundary).
template <class F>
int guard(F&& f) {
    try {
        return f();
    } catch (const pe::CudaError&) {
        return PE_ERR_DEVICE;
    } catch (const std::length_error&) {
        return PE_ERR_BOUNDS;
    } catch (const std::invalid_argument&) {
        return PE_ERR_ARG;
    } catch (const std::bad_alloc&) {
        return PE_ERR_DEVICE;
    } catch (...) {
        return PE_ERR_PANIC;
    }
}

inline bool finite3(const double* a) {
    return std::isfinite(a[0]) && std::isfinite(a[1]) && std::isfinite(a[2]);
}

inline bool valid_dim(int32_t d) { return d == PE_DIM_2 || d == PE_DIM_3; }

inline int status_code(uint32_t st) {
    if (st & (PE_STATUS_DOMAIN | PE_STATUS_NEIGHBOUR_OVERFLOW)) return PE_ERR_BOUNDS;
    if (st & PE_STATUS_NONFINITE) return PE_ERR_ARG;
    return PE_OK;
}

inline pe::WorldConfig to_config(const PeWcsphConfig* c) {
    pe::WorldConfig w{};
    w.device = c ? c->device : -1;
    w.max_neighbours = c ? c->max_neighbours : 0;
    w.max_lower = c ? c->max_lower : 0;
    w.domain_margin = c ? c->domain_margin : -1.0;
    w.domain_margin_cells = c ? c->domain_margin_cells : 0;
    w.precision = c ? c->precision : 0;
    w.use_graph = c ? c->use_graph : 0;
    if (!c) w.domain_margin = -1.0;
    return w;
}

// Validates the particle arrays of a create call (the reference's builders
// only ever produce finite positions and kinds 0 / 1).
inline int check_arrays(int32_t dim, double rest_density, double mass, double h, uint64_t n, const double* x,
                        const double* v, const uint8_t* kind, const double* psi, const double* n_out) {
    if (!valid_dim(dim)) return PE_ERR_ARG;
    if (!(std::isfinite(rest_density) && rest_density > 0.0 && std::isfinite(mass) && mass > 0.0 &&
          std::isfinite(h) && h > 0.0))
        return PE_ERR_ARG;
    if (n > pe::kMaxParticles) return PE_ERR_BOUNDS;
    if (n && (!x || !kind)) return PE_ERR_NULL;
    for (uint64_t i = 0; i < n; ++i) {
        if (!finite3(x + 3 * i) || (v && !finite3(v + 3 * i))) return PE_ERR_ARG;
        if (kind[i] > 1) return PE_ERR_ARG;
        if (psi && !std::isfinite(psi[i])) return PE_ERR_ARG;
        if (n_out && !finite3(n_out + 3 * i)) return PE_ERR_ARG;
    }
    return PE_OK;
}

}  // namespace peabi
