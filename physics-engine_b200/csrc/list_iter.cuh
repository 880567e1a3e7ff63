// Walking a slot's neighbour list in order (see ListRef), shared by the SPH
// passes of every solver.
#pragma once

#include "wcsph_device.cuh"

namespace pe {

// Calls f(entry) over a slot's list in order, with the loads of the next two
// entries issued before the current one is processed.
template <class F>
__device__ __forceinline__ void for_each_entry(const ListRef r, F&& f) {
    const uint32_t n = r.n;
    if (n == 0) return;
    auto at = [&](uint32_t t) { return __ldg(r.p + (size_t)(t >> 2) * r.step + (t & 3u)); };
    uint32_t e0 = at(0), e1 = n > 1 ? at(1) : 0u;
    for (uint32_t t = 0; t < n; ++t) {
        const uint32_t e = e0;
        e0 = e1;
        if (t + 2 < n) e1 = at(t + 2);
        f(e);
    }
}

// Calls f(entry, data) over a slot's list in order, where data = load(entry)
// is issued one entry ahead: the gather of the next neighbour's state is in
// flight while the current pair is computed.
template <class Load, class F>
__device__ __forceinline__ void for_each_loaded(const ListRef r, Load&& load, F&& f) {
    const uint32_t n = r.n;
    if (n == 0) return;
    auto at = [&](uint32_t t) { return __ldg(r.p + (size_t)(t >> 2) * r.step + (t & 3u)); };
    uint32_t e0 = at(0), e1 = n > 1 ? at(1) : 0u;
    auto d0 = load(e0);
    for (uint32_t t = 0; t < n; ++t) {
        const uint32_t e = e0;
        const auto d = d0;
        if (t + 1 < n) {
            e0 = e1;
            d0 = load(e1);
            if (t + 2 < n) e1 = at(t + 2);
        }
        f(e, d);
    }
}

}  // namespace pe
