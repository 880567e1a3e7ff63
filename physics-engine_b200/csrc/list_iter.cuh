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

// Calls f(t, entry, data) over a slot's list in order (t the entry's
// position), where data = load(t, entry) is issued one entry ahead: the
// gather of the next neighbour's state is in flight while the current pair
// is computed. load sees t = 0, 1, 2, ... in order.
template <class Load, class F>
__device__ __forceinline__ void for_each_loaded_t(const ListRef r, Load&& load, F&& f) {
    const uint32_t n = r.n;
    if (n == 0) return;
    auto at = [&](uint32_t t) { return __ldg(r.p + (size_t)(t >> 2) * r.step + (t & 3u)); };
    uint32_t e0 = at(0), e1 = n > 1 ? at(1) : 0u;
    auto d0 = load(0u, e0);
    for (uint32_t t = 0; t < n; ++t) {
        const uint32_t e = e0;
        const auto d = d0;
        if (t + 1 < n) {
            e0 = e1;
            d0 = load(t + 1, e1);
            if (t + 2 < n) e1 = at(t + 2);
        }
        f(t, e, d);
    }
}

// for_each_loaded_t without the positions.
template <class Load, class F>
__device__ __forceinline__ void for_each_loaded(const ListRef r, Load&& load, F&& f) {
    for_each_loaded_t(
        r, [&](uint32_t, uint32_t e) { return load(e); },
        [&](uint32_t, uint32_t e, const auto& d) { f(e, d); });
}

// Calls f(t, entry, data) over a slot's list in order (t the entry's
// position), data = load(t, entry), with the data of the next two entries in
// flight.
template <class Load, class F>
__device__ __forceinline__ void for_each_loaded2_t(const ListRef r, Load&& load, F&& f) {
    const uint32_t n = r.n;
    if (n == 0) return;
    auto at = [&](uint32_t t) { return __ldg(r.p + (size_t)(t >> 2) * r.step + (t & 3u)); };
    uint32_t e0 = at(0), e1 = n > 1 ? at(1) : 0u, e2 = n > 2 ? at(2) : 0u;
    auto d0 = load(0u, e0);
    auto d1 = n > 1 ? load(1u, e1) : d0;
    for (uint32_t t = 0; t < n; ++t) {
        const uint32_t e = e0;
        const auto d = d0;
        e0 = e1;
        d0 = d1;
        if (t + 2 < n) {
            e1 = e2;
            d1 = load(t + 2, e2);
            if (t + 3 < n) e2 = at(t + 3);
        }
        f(t, e, d);
    }
}

// for_each_loaded with the data of the next two entries in flight.
template <class Load, class F>
__device__ __forceinline__ void for_each_loaded2(const ListRef r, Load&& load, F&& f) {
    for_each_loaded2_t(
        r, [&](uint32_t, uint32_t e) { return load(e); },
        [&](uint32_t, uint32_t e, const auto& d) { f(e, d); });
}

// Entries a chunk compacts at most (see for_each_kept).
constexpr uint32_t kKeepChunk = 32;

// Calls f(entry, data) in list order over the entries keep(entry, data)
// accepts, data = load(entry). The list is taken in chunks of kKeepChunk; each
// chunk's accepted entries are first compacted into this thread's column of
// buf (kKeepChunk rows of blockDim.x entries, shared memory), so a warp runs
// its f loop over accepted entries only instead of idling on the rejected ones
// at each lane's own positions.
template <class Load, class Keep, class F>
__device__ __forceinline__ void for_each_kept(const ListRef r, uint32_t* buf, Load&& load, Keep&& keep, F&& f) {
    const uint32_t n = r.n, tid = threadIdx.x, bd = blockDim.x;
    auto at = [&](uint32_t t) { return __ldg(r.p + (size_t)(t >> 2) * r.step + (t & 3u)); };
    for (uint32_t t0 = 0; t0 < n; t0 += kKeepChunk) {
        const uint32_t t1 = min(n, t0 + kKeepChunk);
        uint32_t c = 0;
        for (uint32_t t = t0; t < t1; ++t) {
            const uint32_t e = at(t);
            if (keep(e, load(e))) buf[(c++) * bd + tid] = e;
        }
        if (c == 0) continue;
        uint32_t e = buf[tid];
        auto d = load(e);
        for (uint32_t u = 0; u < c; ++u) {
            const uint32_t ec = e;
            const auto dc = d;
            if (u + 1 < c) {
                e = buf[(u + 1) * bd + tid];
                d = load(e);
            }
            f(ec, dc);
        }
    }
}

}  // namespace pe
