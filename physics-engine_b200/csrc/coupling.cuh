// Fluid side of the WCSPH-rigid coupling (coupling.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "world.cuh"

namespace pe {

// Rigid samples of a world: sample k is particle particle[k] of the world, on
// body body[k] at body-frame offset local[k] with body-frame normal local_n[k]
// (FluidRigidCoupler::samples, coupling.rs:42-51, in insertion order).
class Coupler {
   public:
    Coupler(World& w, uint32_t n_bodies, uint64_t ns, const int64_t* body, const double* local,
            const double* local_n, const int64_t* particle);
    ~Coupler();
    Coupler(const Coupler&) = delete;
    Coupler& operator=(const Coupler&) = delete;
    // sync_from_rigid: X (3), q (4: w, x, y, z), V (3), world-frame omega (3) per body
    void sync(const double* X, const double* Q, const double* V, const double* Om);
    // reduce_with_state: per body force and torque about X, 3 doubles each
    void reduce(const double* X, double* force, double* torque);
    uint32_t bodies() const { return nb_; }

   private:
    template <typename T>
    T* alloc(size_t n);
    template <typename T>
    T* upload(const T* h, size_t n);
    World& w_;
    uint32_t nb_;
    uint64_t ns_;
    std::vector<void*> keep_;
    const int64_t *body_ = nullptr, *particle_ = nullptr, *grouped_ = nullptr;
    const double *local_ = nullptr, *local_n_ = nullptr;
    const uint64_t* start_ = nullptr;
    double *bodies_ = nullptr, *X_ = nullptr, *out_ = nullptr;
};

}  // namespace pe
