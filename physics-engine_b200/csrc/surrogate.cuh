// Learned surrogate of the WCSPH step: a two-hop message-passing network over
// the particles' neighbour graph that predicts each fluid particle's
// acceleration and density rate. BF16 weights and activations on the tensor
// cores (mlp_gemm.cu), fp32 accumulation, fp32 master weights with Adam.
//
//   h0_i  = enc(f_i)                                   f: 8 node features
//   hop l = 1, 2, edges e = (i <- j), i fluid:
//     z_e   = h_i Wa + h_j Wb + x_e Wc + b1            x_e: 16 edge features
//     m_e   = relu(relu(z_e) W2 + b2) W3 + b3
//     h_l,i = h_{l-1},i + node_l([h_{l-1},i, (sum_e m_e) / 16])
//   y_i   = dec(h2_i)                                  (a_x, a_y, a_z, drho/dt), normalised
//
// Every MLP is Linear-ReLU-Linear-ReLU-Linear with hidden width 128.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "mlp.cuh"

namespace pe {

class World;

constexpr int kWidth = 128;
constexpr int kNodeFeat = 8;
constexpr int kEdgeFeat = 16;
constexpr int kOut = 4;
constexpr int kOutPad = 8;  // the decoder's last layer is padded to 8 outputs (zero weights)

struct Linear {
    std::string name;
    int K = 0, N = 0, Np = 0;   // inputs, outputs, outputs padded to a multiple of 8
    bool has_bias = true;
    float* Wt = nullptr;        // fp32 master, [Np x K]
    float* b = nullptr;         // fp32 [Np]
    __nv_bfloat16* Wt16 = nullptr;  // bf16 [Np x K]: forward operand
    __nv_bfloat16* W16 = nullptr;   // bf16 [K x Np]: input-gradient operand
    float* gWt = nullptr;       // gradients
    float* gb = nullptr;
    float *mW = nullptr, *vW = nullptr, *mb = nullptr, *vb = nullptr;  // Adam moments
};

// The message graph of a range of nodes: edges sorted by destination.
struct MsgGraph {
    int n = 0, E = 0;
    int* row = nullptr;              // [n + 1]
    int* src = nullptr;              // [E]
    int* dst = nullptr;              // [E]
    __nv_bfloat16* xe = nullptr;     // [E x 16]
    __nv_bfloat16* f = nullptr;      // [n x 8]
    uint8_t* fluid = nullptr;        // [n]
    int cap_n = 0, cap_e = 0;
};

struct SurrogateStats {
    float mean[kOut], std[kOut];     // target normalisation
};

class Surrogate {
   public:
    explicit Surrogate(uint64_t seed, double r_msg_over_h = 1.0);
    ~Surrogate();
    Surrogate(const Surrogate&) = delete;
    Surrogate& operator=(const Surrogate&) = delete;

    // parameters in the order of the network description; W is [K x N] row-major
    int num_params() const { return (int)layers_.size(); }
    const Linear& param(int i) const { return layers_[i]; }
    void get_param(int i, float* W, float* b, bool grad);
    void set_param(int i, const float* W, const float* b);

    // graph from host arrays (tests): row [n+1], src [E], f [n x 8], xe [E x 16]
    void set_graph(int n, int E, const int* row, const int* src, const float* f, const float* xe,
                   const uint8_t* fluid);
    void set_targets(const float* t);  // [n x 4], already normalised

    // forward on the current graph (outputs [n x 4], normalised)
    void forward(bool keep_for_backward);
    void get_outputs(float* y);
    // forward + backward; with lr > 0 also one Adam step. Returns the loss.
    float train_step(float lr);

    // ---- coupling to a world ----
    // graph and features of slots [s0, s1) of w's current state (neighbour
    // lists must be current); keeps the nodes' original indices for targets
    void graph_from_world(World& w, uint32_t s0, uint32_t s1);
    // normalised targets of the current graph's fluid nodes from w's state one
    // step of dt later; with update_stats these targets join the moments the
    // normalisation is fitted on (all update_stats calls so far) and it is refit
    void targets_from_world(World& w, double dt, bool update_stats);
    // predicted acceleration and density rate per slot of w (whole world),
    // written to acc (double4 per slot, w = drho/dt)
    void predict_world(World& w, double4* acc_out);

    double r_msg() const { return r_msg_over_h_; }
    const SurrogateStats& stats() const { return stats_; }
    void set_stats(const SurrogateStats& s) { stats_ = s; }
    cudaStream_t stream() const { return st_; }
    void set_stream(cudaStream_t s) { st_ = s; }
    uint32_t device_error();
    // inference (forward without backward) runs each hop's edge MLP as one
    // fused kernel (edge_fused.cu) when on; off: the three GEMMs and the
    // segment sum that training uses
    void set_fused_edges(bool on) { fused_edges_ = on; }
    bool fused_edges() const { return fused_edges_; }

   private:
    void alloc_params(uint64_t seed);
    void ensure_graph(int n, int E);
    void ensure_acts(bool train);
    void refresh_bf16(Linear& L);
    void gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* Bt, int ldb, int M, int N, int K, float* Cf,
              __nv_bfloat16* Cb, int ldc, const float* bias, bool relu, int splits = 1);
    void linear_fwd(const Linear& L, const __nv_bfloat16* X, int R, float* Yf, __nv_bfloat16* Yb, bool relu);
    void mlp_fwd(int first, const __nv_bfloat16* X, int R, __nv_bfloat16* A1, __nv_bfloat16* A2, float* Yf);
    // backward of one Linear: dZ fp32 [R x Np] (masked by mask > 0 if mask) ->
    // grads; dX fp32 [R x K] if dX
    void linear_bwd(Linear& L, const __nv_bfloat16* X, int R, float* dZ, const __nv_bfloat16* mask, float* dX);
    void mlp_bwd(int first, const __nv_bfloat16* X, int R, const __nv_bfloat16* A1, const __nv_bfloat16* A2,
                 float* dY, float* dX);
    void adam(Linear& L, float lr);
    template <typename T>
    T* dalloc(size_t n);

    std::vector<Linear> layers_;
    std::vector<void*> allocs_;
    std::vector<void*> graph_allocs_, act_allocs_;
    cudaStream_t st_ = nullptr;
    bool own_stream_ = false;
    double r_msg_over_h_;
    SurrogateStats stats_{};
    double st_sum_[kOut] = {}, st_sq_[kOut] = {};  // moments of every target fitted so far
    double st_count_ = 0.0;
    int adam_t_ = 0;
    uint32_t* err_ = nullptr;
    bool fused_edges_ = true;
    int sms_ = 148;
    float* loss_ = nullptr;
    float* part_ = nullptr;
    size_t part_floats_ = 0;

    MsgGraph g_;
    uint32_t* node_orig_ = nullptr;   // original index of each graph node
    double* node_v_ = nullptr;        // [n x 4]: velocity, density at the graph's time
    float* raw_t_ = nullptr;          // [n x 4] targets before normalisation
    int* cnt_ = nullptr;              // [n + 1] edges per node, then CSR offsets
    void* scan_tmp_ = nullptr;
    size_t scan_bytes_ = 0;
    float* target_ = nullptr;         // [n x 4] normalised targets
    // activations (rows: nodes or edges)
    int act_n_ = 0, act_e_ = 0;
    bool act_train_ = false;
    __nv_bfloat16 *enc_a1_ = nullptr, *enc_a2_ = nullptr;
    float* h_ = nullptr;                   // latent fp32 [n x 128]
    __nv_bfloat16* hb_[3] = {};            // latent bf16 per level
    float *P_ = nullptr, *Q_ = nullptr;    // [n x 128]
    __nv_bfloat16 *eh1_[2] = {}, *eh2_[2] = {};  // per hop, [E x 128]
    float* M_ = nullptr;                   // [E x 128]
    float* A_ = nullptr;                   // [n x 128]
    __nv_bfloat16* xn_[2] = {};            // per hop, [n x 256]
    __nv_bfloat16 *na1_[2] = {}, *na2_[2] = {};
    float* U_ = nullptr;                   // [n x 128]
    __nv_bfloat16 *da1_ = nullptr, *da2_ = nullptr;
    float* Y_ = nullptr;                   // [n x 8]
    // backward scratch
    float *dY_ = nullptr, *dH_ = nullptr, *dHp_ = nullptr, *dXN_ = nullptr, *dE_ = nullptr, *dE2_ = nullptr;
    float *dP_ = nullptr, *dQ_ = nullptr, *dT1_ = nullptr, *dT2_ = nullptr;
    __nv_bfloat16 *gb16_ = nullptr, *gbT_ = nullptr, *xT_ = nullptr;
};

}  // namespace pe
