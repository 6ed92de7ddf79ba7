// pbf_particles.hpp — C++ facade over the C ABI in pbf.h with the method
// names and span arguments of the reference's sim::Particles<float,3>
// (Simulation/Source/particles.h:256-487), so the reference's time-step loop
// (Simulation/Source/main.cpp:71-124) compiles against it unchanged.
//
// Spans are any type with .begin/.end members — the reference's IndexSpan
// (Vec<std::size_t,2>, Common/vec.h:706) or sim::gpu::IndexSpan below.  A
// nonzero status from the C ABI becomes std::runtime_error, as the reference
// reports failures (Common/array.h:128-129).
#pragma once

#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "pbf.h"

namespace sim {
namespace gpu {

struct IndexSpan {
  std::size_t begin, end;
};

// Parameter accessors the reference's driver loop uses (parameters.h:262-264).
class Parameters {
 public:
  explicit Parameters(const pbf_params& p) : p_(p) {}
  std::size_t solve_step_count() const { return (std::size_t)p_.solve_steps; }
  float time_step() const { return p_.time_step; }
  float rest_density() const { return p_.rest_density; }
  const pbf_params& raw() const { return p_; }
  pbf_params& raw() { return p_; }

 private:
  pbf_params p_;
};

class Particles {
 public:
  Particles(const pbf_params& params, std::size_t capacity) : capacity_(capacity) {
    if (pbf_create(&params, capacity, &ctx_) != PBF_OK)
      throw std::runtime_error(std::string("pbf_create: ") + pbf_create_error());
  }
  ~Particles() { pbf_destroy(ctx_); }
  Particles(const Particles&) = delete;
  Particles& operator=(const Particles&) = delete;

  // particles.h:76-86
  std::size_t local_count() const { return pbf_count(ctx_); }
  std::size_t max_local_count() const { return capacity_; }
  std::size_t available() const { return capacity_ - local_count(); }

  // State in the reference's Vec<float,3> AoS layout (x* = x on upload).
  void upload(const float* x_aos, const float* v_aos, std::size_t n) { check(pbf_upload(ctx_, x_aos, v_aos, n)); }
  void download(float* x_aos, float* v_aos, float* rho = nullptr, float* lambda = nullptr) {
    check(pbf_download(ctx_, x_aos, v_aos, rho, lambda));
  }
  std::vector<float> array(int which) {
    const bool vec = which <= PBF_ARRAY_SCRATCH;
    std::vector<float> out(local_count() * (vec ? 3 : 1));
    check(pbf_get_array(ctx_, which, out.data()));
    return out;
  }

  // particles.h:184-199 (add) and 231-250 (construct_fluid): append particles;
  // throws past the capacity, as the reference does.
  void add(const float* x_aos, const float* v_aos, std::size_t k) { check(pbf_add_particles(ctx_, x_aos, v_aos, k)); }
  std::size_t construct_fluid(const float fluid_min[3], const float fluid_max[3],
                              const float velocity[3] = nullptr) {
    std::size_t added = 0;
    check(pbf_construct_fluid(ctx_, fluid_min, fluid_max, velocity, &added));
    return added;
  }

  // Output frames and checkpoints (pbf.h: state files).
  void save(const char* path) { check(pbf_save_state(ctx_, path)); }
  void load(const char* path) { check(pbf_load_state(ctx_, path)); }

  // The stages.
  template <class S> void apply_external_forces(const S& s) { check(pbf_apply_external_forces(ctx_, s.begin, s.end)); }
  template <class S> void predict_positions(const S& s) { check(pbf_predict_positions(ctx_, s.begin, s.end)); }
  template <class B, class F> void find_neighbors(const B& bin, const F& fill) {
    check(pbf_find_neighbors(ctx_, bin.begin, bin.end, fill.begin, fill.end));
  }
  template <class S> void compute_densities(const S& s) { check(pbf_compute_densities(ctx_, s.begin, s.end)); }
  template <class S> void compute_pressure_lambdas(const S& s) {
    check(pbf_compute_pressure_lambdas(ctx_, s.begin, s.end));
  }
  template <class S> void compute_pressure_dps(const S& s, const int substep) {
    check(pbf_compute_pressure_dps(ctx_, s.begin, s.end, substep));
  }
  template <class S> void update_position_stars(const S& s) { check(pbf_update_position_stars(ctx_, s.begin, s.end)); }
  template <class S> void update_velocities(const S& s) { check(pbf_update_velocities(ctx_, s.begin, s.end)); }
  template <class C, class S> void apply_surface_tension(const C& color, const S& st) {
    check(pbf_apply_surface_tension(ctx_, color.begin, color.end, st.begin, st.end));
  }
  template <class S> void apply_viscosity(const S& s) { check(pbf_apply_viscosity(ctx_, s.begin, s.end)); }
  template <class S> void compute_vorticity(const S& s) { check(pbf_compute_vorticity(ctx_, s.begin, s.end)); }
  template <class S> void apply_vorticity(const S& s) { check(pbf_apply_vorticity(ctx_, s.begin, s.end)); }
  template <class S> void update_positions(const S& s) { check(pbf_update_positions(ctx_, s.begin, s.end)); }

  // The whole step, fused and replayed from a CUDA graph.
  void step(int nsteps = 1) { check(pbf_step(ctx_, nsteps)); }
  pbf_stats_t stats() {
    pbf_stats_t st;
    check(pbf_stats(ctx_, &st));
    return st;
  }
  pbf_ctx* handle() { return ctx_; }

 private:
  void check(int rc) {
    if (rc != PBF_OK) throw std::runtime_error(pbf_last_error(ctx_));
  }
  pbf_ctx* ctx_ = nullptr;
  std::size_t capacity_;
};

}  // namespace gpu
}  // namespace sim
