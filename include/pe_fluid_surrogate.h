/* Learned surrogate of the WCSPH step (no reference counterpart).
 *
 * A two-hop message-passing network over the particles' neighbour graph
 * predicts each fluid particle's acceleration and density rate; BF16 weights
 * on the tensor cores with fp32 accumulation, trained on the GPU on rollouts
 * of the plain step. The plain step judges it every k steps and replaces it
 * when the density error exceeds a bound (pe_fluid_wcsph_run_learned).
 * Return codes are those of pe_fluid_wcsph.h. */
#ifndef PE_FLUID_SURROGATE_H
#define PE_FLUID_SURROGATE_H

#include <stdint.h>

#include "pe_fluid_wcsph.h"

#ifdef __cplusplus
extern "C" {
#endif
#pragma GCC visibility push(default)

typedef struct PeSurrogate PeSurrogate;

/* Network with He-initialised weights from seed; edges join particles closer
 * than r_msg_over_h * h. */
int pe_surrogate_create(uint64_t seed, double r_msg_over_h, PeSurrogate** out);
void pe_surrogate_destroy(PeSurrogate* s);

/* Parameters: linear layers in network order, W is K x N row-major (inputs x
 * outputs), b has N entries (zeros for the bias-free layers). */
int pe_surrogate_num_params(PeSurrogate* s, int32_t* n);
int pe_surrogate_param_info(PeSurrogate* s, int32_t i, char* name, int32_t name_cap, int32_t* K, int32_t* N,
                            int32_t* has_bias);
int pe_surrogate_get_param(PeSurrogate* s, int32_t i, float* W, float* b);
int pe_surrogate_set_param(PeSurrogate* s, int32_t i, const float* W, const float* b);
/* Gradient of the last pe_surrogate_train_step's loss, same layout. */
int pe_surrogate_get_grad(PeSurrogate* s, int32_t i, float* W, float* b);

/* An explicit graph: n nodes (features f, n x 8), E edges sorted by
 * destination (row: n + 1 offsets, src: E sources, xe: E x 16 features). */
int pe_surrogate_set_graph(PeSurrogate* s, int32_t n, int32_t E, const int32_t* row, const int32_t* src,
                           const float* f, const float* xe, const uint8_t* fluid);
int pe_surrogate_set_targets(PeSurrogate* s, const float* t); /* n x 4, normalised */
int pe_surrogate_forward(PeSurrogate* s, float* y);
/* Inference runs each hop's edge MLP and its sum per destination as one fused
 * tensor-core kernel (on = 1, the default) or as the three GEMMs and the
 * segment sum that training uses (on = 0); the two differ only in the order
 * of the fp32 message sums. */
int pe_surrogate_set_fused_edges(PeSurrogate* s, int32_t on);           /* n x 4, normalised */
/* Forward, loss (mean over fluid nodes of the squared error), backward; one
 * Adam step when lr > 0. */
int pe_surrogate_train_step(PeSurrogate* s, float lr, float* loss);

/* Target normalisation (per output: mean and standard deviation). */
int pe_surrogate_get_stats(PeSurrogate* s, float mean[4], float std_[4]);
int pe_surrogate_set_stats(PeSurrogate* s, const float mean[4], const float std_[4]);

/* Training on the plain step: the graph of slots [slot_begin, slot_end) of a
 * world (a tank's range, pe_fluid_wcsph_tank_range), then, after the world
 * took one plain step of dt, that graph's targets (velocity change and density
 * change per dt); update_stats refits the normalisation first. */
int pe_surrogate_graph_from_world(PeSurrogate* s, PeWcsph* w, uint32_t slot_begin, uint32_t slot_end);
int pe_surrogate_targets_from_world(PeSurrogate* s, PeWcsph* w, double dt, int32_t update_stats);
int pe_fluid_wcsph_tank_range(PeWcsph* w, uint32_t tank, uint32_t* slot_begin, uint32_t* slot_end);

/* One learned step of all particles: the network's acceleration and density
 * rate replace the pressure, viscosity and XSPH passes (v += dt a, x += dt v,
 * rho += dt drho/dt). */
int pe_fluid_wcsph_step_learned(PeWcsph* w, PeSurrogate* s, double dt);
/* The plain step's SPH density of the current positions replaces the carried
 * densities; *max_rel_error = max over fluid of |carried - SPH| / SPH. */
int pe_fluid_wcsph_judge_density(PeWcsph* w, double* max_rel_error);
/* steps in windows of judge_every learned steps; after each window the plain
 * density judges it, and a window whose error exceeds bound is rerun from its
 * start with the plain step. out (may be NULL) = {windows, fallbacks, learned
 * steps, plain steps, largest error, last error}. */
int pe_fluid_wcsph_run_learned(PeWcsph* w, PeSurrogate* s, double dt, uint64_t steps, uint32_t judge_every,
                               double bound, double out[6]);

/* The tensor-core GEMM the network runs on, on caller device buffers (a test
 * and benchmark entry): C[M x N] = A[M x K] * Bt[N x K]^T (+ bias) (ReLU), bf16
 * A and Bt with K contiguous, fp32 Cf and/or bf16 Cb; part (splits * M * ldc
 * floats) when splits > 1. Synchronous on stream; *err = wait-timeout flag. */
int pe_mlp_gemm_bf16(const void* A, const void* Bt, float* Cf, void* Cb, const float* bias, int M, int N, int K,
                     int lda, int ldb, int ldc, int relu, int splits, float* part, void* stream, uint32_t* err);

#pragma GCC visibility pop
#ifdef __cplusplus
}
#endif
#endif
