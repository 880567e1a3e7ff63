// C ABI of the learned surrogate (include/pe_fluid_surrogate.h).
#include <cmath>
#include <cstring>
#include <new>
#include <stdexcept>

#include "../../include/pe_fluid_surrogate.h"
#include "handles.cuh"
#include "surrogate.cuh"

struct PeSurrogate {
    pe::Surrogate* s;
};

namespace {

template <class F>
int guard_s(F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return PE_ERR_DEVICE;
    } catch (const std::length_error&) {
        return PE_ERR_BOUNDS;
    } catch (const std::out_of_range&) {
        return PE_ERR_BOUNDS;
    } catch (const std::invalid_argument&) {
        return PE_ERR_ARG;
    } catch (...) {
        return PE_ERR_DEVICE;
    }
}

}  // namespace

int pe_surrogate_create(uint64_t seed, double r_msg_over_h, PeSurrogate** out) {
    if (!out) return PE_ERR_NULL;
    *out = nullptr;
    if (!(r_msg_over_h > 0.0 && r_msg_over_h <= 2.0)) return PE_ERR_ARG;
    return guard_s([&] {
        *out = new PeSurrogate{new pe::Surrogate(seed, r_msg_over_h)};
        return PE_OK;
    });
}

void pe_surrogate_destroy(PeSurrogate* s) {
    if (!s) return;
    try {
        delete s->s;
    } catch (...) {
    }
    delete s;
}

int pe_surrogate_num_params(PeSurrogate* s, int32_t* n) {
    if (!s || !n) return PE_ERR_NULL;
    *n = s->s->num_params();
    return PE_OK;
}

int pe_surrogate_param_info(PeSurrogate* s, int32_t i, char* name, int32_t name_cap, int32_t* K, int32_t* N,
                            int32_t* has_bias) {
    if (!s) return PE_ERR_NULL;
    if (i < 0 || i >= s->s->num_params()) return PE_ERR_BOUNDS;
    const pe::Linear& L = s->s->param(i);
    if (name && name_cap > 0) {
        std::strncpy(name, L.name.c_str(), (size_t)name_cap - 1);
        name[name_cap - 1] = 0;
    }
    if (K) *K = L.K;
    if (N) *N = L.N;
    if (has_bias) *has_bias = L.has_bias ? 1 : 0;
    return PE_OK;
}

int pe_surrogate_get_param(PeSurrogate* s, int32_t i, float* W, float* b) {
    if (!s) return PE_ERR_NULL;
    if (i < 0 || i >= s->s->num_params()) return PE_ERR_BOUNDS;
    return guard_s([&] {
        s->s->get_param(i, W, b, false);
        return PE_OK;
    });
}

int pe_surrogate_set_param(PeSurrogate* s, int32_t i, const float* W, const float* b) {
    if (!s) return PE_ERR_NULL;
    if (i < 0 || i >= s->s->num_params()) return PE_ERR_BOUNDS;
    return guard_s([&] {
        s->s->set_param(i, W, b);
        return PE_OK;
    });
}

int pe_surrogate_get_grad(PeSurrogate* s, int32_t i, float* W, float* b) {
    if (!s) return PE_ERR_NULL;
    if (i < 0 || i >= s->s->num_params()) return PE_ERR_BOUNDS;
    return guard_s([&] {
        s->s->get_param(i, W, b, true);
        return PE_OK;
    });
}

int pe_surrogate_set_graph(PeSurrogate* s, int32_t n, int32_t E, const int32_t* row, const int32_t* src,
                           const float* f, const float* xe, const uint8_t* fluid) {
    if (!s || !row || !f || !fluid || (E > 0 && (!src || !xe))) return PE_ERR_NULL;
    if (n <= 0 || E < 0 || row[0] != 0 || row[n] != E) return PE_ERR_ARG;
    for (int32_t i = 0; i < n; ++i)
        if (row[i + 1] < row[i]) return PE_ERR_ARG;
    for (int32_t e = 0; e < E; ++e)
        if (src[e] < 0 || src[e] >= n) return PE_ERR_BOUNDS;
    return guard_s([&] {
        s->s->set_graph(n, E, row, src, f, xe, fluid);
        return PE_OK;
    });
}

int pe_surrogate_set_targets(PeSurrogate* s, const float* t) {
    if (!s || !t) return PE_ERR_NULL;
    return guard_s([&] {
        s->s->set_targets(t);
        return PE_OK;
    });
}

int pe_surrogate_forward(PeSurrogate* s, float* y) {
    if (!s || !y) return PE_ERR_NULL;
    return guard_s([&] {
        s->s->forward(false);
        s->s->get_outputs(y);
        return s->s->device_error() ? PE_ERR_DEVICE : PE_OK;
    });
}

int pe_surrogate_set_fused_edges(PeSurrogate* s, int32_t on) {
    if (!s) return PE_ERR_NULL;
    s->s->set_fused_edges(on != 0);
    return PE_OK;
}

int pe_surrogate_train_step(PeSurrogate* s, float lr, float* loss) {
    if (!s) return PE_ERR_NULL;
    return guard_s([&] {
        const float l = s->s->train_step(lr);
        if (loss) *loss = l;
        return s->s->device_error() ? PE_ERR_DEVICE : PE_OK;
    });
}

int pe_surrogate_get_stats(PeSurrogate* s, float mean[4], float std_[4]) {
    if (!s || !mean || !std_) return PE_ERR_NULL;
    const pe::SurrogateStats& st = s->s->stats();
    for (int c = 0; c < 4; ++c) {
        mean[c] = st.mean[c];
        std_[c] = st.std[c];
    }
    return PE_OK;
}

int pe_surrogate_set_stats(PeSurrogate* s, const float mean[4], const float std_[4]) {
    if (!s || !mean || !std_) return PE_ERR_NULL;
    pe::SurrogateStats st;
    for (int c = 0; c < 4; ++c) {
        if (!(std_[c] > 0.f) || !std::isfinite(mean[c])) return PE_ERR_ARG;
        st.mean[c] = mean[c];
        st.std[c] = std_[c];
    }
    s->s->set_stats(st);
    return PE_OK;
}

int pe_surrogate_graph_from_world(PeSurrogate* s, PeWcsph* w, uint32_t slot_begin, uint32_t slot_end) {
    if (!s || !w) return PE_ERR_NULL;
    if (slot_end <= slot_begin || slot_end > w->world->len()) return PE_ERR_BOUNDS;
    return guard_s([&] {
        s->s->graph_from_world(*w->world, slot_begin, slot_end);
        return PE_OK;
    });
}

int pe_surrogate_targets_from_world(PeSurrogate* s, PeWcsph* w, double dt, int32_t update_stats) {
    if (!s || !w) return PE_ERR_NULL;
    if (!(std::isfinite(dt) && dt > 0.0)) return PE_ERR_ARG;
    return guard_s([&] {
        s->s->targets_from_world(*w->world, dt, update_stats != 0);
        return PE_OK;
    });
}

int pe_fluid_wcsph_tank_range(PeWcsph* w, uint32_t tank, uint32_t* slot_begin, uint32_t* slot_end) {
    if (!w || !slot_begin || !slot_end) return PE_ERR_NULL;
    if (tank >= w->world->tanks()) return PE_ERR_BOUNDS;
    *slot_begin = w->world->tank_slot_begin(tank);
    *slot_end = w->world->tank_slot_end(tank);
    return PE_OK;
}

int pe_fluid_wcsph_step_learned(PeWcsph* w, PeSurrogate* s, double dt) {
    if (!w || !s) return PE_ERR_NULL;
    if (!(std::isfinite(dt) && dt > 0.0)) return PE_ERR_ARG;
    return guard_s([&] {
        w->world->step_learned(*s->s, dt);
        const uint32_t st = w->world->status();
        return (st & (PE_STATUS_DOMAIN | PE_STATUS_NEIGHBOUR_OVERFLOW)) ? PE_ERR_BOUNDS
               : (st & PE_STATUS_NONFINITE)                            ? PE_ERR_ARG
                                                                       : PE_OK;
    });
}

int pe_fluid_wcsph_judge_density(PeWcsph* w, double* max_rel_error) {
    if (!w || !max_rel_error) return PE_ERR_NULL;
    return guard_s([&] {
        *max_rel_error = w->world->judge_density();
        return PE_OK;
    });
}

int pe_fluid_wcsph_run_learned(PeWcsph* w, PeSurrogate* s, double dt, uint64_t steps, uint32_t judge_every,
                               double bound, double out[6]) {
    if (!w || !s) return PE_ERR_NULL;
    if (!(std::isfinite(dt) && dt > 0.0) || !(bound > 0.0) || judge_every == 0) return PE_ERR_ARG;
    return guard_s([&] {
        pe::World::LearnedStats st{};
        w->world->run_learned(*s->s, dt, steps, judge_every, bound, &st);
        if (out) {
            out[0] = (double)st.windows;
            out[1] = (double)st.fallbacks;
            out[2] = (double)st.learned_steps;
            out[3] = (double)st.plain_steps;
            out[4] = st.max_error;
            out[5] = st.last_error;
        }
        const uint32_t code = w->world->status();
        return (code & (PE_STATUS_DOMAIN | PE_STATUS_NEIGHBOUR_OVERFLOW)) ? PE_ERR_BOUNDS
               : (code & PE_STATUS_NONFINITE)                            ? PE_ERR_ARG
                                                                         : PE_OK;
    });
}
