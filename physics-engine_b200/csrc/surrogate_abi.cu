// C ABI of the learned surrogate (include/pe_fluid_surrogate.h).
#include <cstring>
#include <new>
#include <stdexcept>

#include "../../include/pe_fluid_surrogate.h"
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

int pe_surrogate_train_step(PeSurrogate* s, float lr, float* loss) {
    if (!s) return PE_ERR_NULL;
    return guard_s([&] {
        const float l = s->s->train_step(lr);
        if (loss) *loss = l;
        return s->s->device_error() ? PE_ERR_DEVICE : PE_OK;
    });
}
