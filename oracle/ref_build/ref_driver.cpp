// Test-infrastructure driver around the reference's OWN PBF implementation.
//
// This file is compiled together with the unmodified reference headers
// (Simulation/Source/particles.h, neighbors.h, neighbors.cpp and Common/*) by
// oracle/ref_build/Makefile into oracle/_ref/libpbf_ref*.so.  It is the
// checker the restated oracle and the CUDA path are pinned against, and the
// timed CPU baseline; nothing in the product links it.
//
// It replaces the reference's MPI/renderer driver (Simulation/Source/main.cpp)
// with a single-rank loop over the span [0, N), exactly as the reference's own
// serial tests drive Particles (Simulation/Tests/Serial/particle_test.cpp:227-267):
// no Distributor, so resident_span() == local_span() == [0, N).
//
// Private members of sim::Neighbors (bin ids, particle ids, bin bounds) are
// read for parity dumps; the access specifier is widened here only.
#include <omp.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <future>
#include <iostream>
#include <limits>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>

// System headers the reference headers pull in are included first so that the
// access-specifier override below reaches the reference's own classes only.
#include "thrust/binary_search.h"
#include "thrust/execution_policy.h"
#include "thrust/for_each.h"
#include "thrust/iterator/counting_iterator.h"
#include "thrust/partition.h"
#include "thrust/sort.h"
#include <boost/algorithm/string/trim.hpp>
#include <boost/lexical_cast.hpp>
#include <boost/property_tree/ini_parser.hpp>
#include <boost/property_tree/ptree.hpp>

#define private public
#include "parameters.h"
#include "particles.h"
#undef private

namespace {
using Real = float;
constexpr Dimension Dim = three_dimensional;
using Params = sim::Parameters<Real, Dim>;
using Parts = sim::Particles<Real, Dim>;
using V3 = Vec<Real, Dim>;

struct RefSim {
  Params* params = nullptr;
  Parts* parts = nullptr;
  std::string error;
};

thread_local std::string g_error;
}  // namespace

extern "C" {

// Plain-data parameter block; field meaning follows Common/parameters.h:550-573.
// A value <= 0 for smoothing_radius / neighbor_bin_spacing / rest_spacing lets
// derive_from_input() (parameters.h:123-148) derive it, as an absent INI key does.
typedef struct {
  float time_step, gravity, gamma, visc_c, lambda_epsilon, k_stiff, vorticity_coef;
  float smoothing_radius, neighbor_bin_spacing, rest_spacing;
  float boundary_min[3], boundary_max[3];
  float fluid_min[3], fluid_max[3];
  float mover_center[3];
  uint64_t solve_steps, max_particles_local, global_particle_count;
  float rest_density;  // > 0: written over the derived rest_density_ (parameters.h:557)
} ref_params_t;

const char* ref_last_error(void) { return g_error.c_str(); }

void ref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : omp_get_num_procs()); }
int ref_get_threads(void) { return omp_get_max_threads(); }

static Params* make_params(const ref_params_t* p) {
  auto* q = new Params();
  q->simulation_mode_ = Params::Mode::EDIT_VIEW;
  q->execution_mode_ = sim::ExecutionMode::CPU;
  q->solve_step_count_ = p->solve_steps;
  q->time_step_ = p->time_step;
  q->initial_global_particle_count_ = p->global_particle_count;
  q->max_particles_local_ = p->max_particles_local;
  q->neighbor_bin_spacing_ = p->neighbor_bin_spacing > 0 ? p->neighbor_bin_spacing : -1.0f;
  q->gravity_ = p->gravity;
  q->gamma_ = p->gamma;
  q->visc_c_ = p->visc_c;
  q->lambda_epsilon_ = p->lambda_epsilon;
  q->k_stiff_ = p->k_stiff;
  q->rest_density_ = -1.0f;
  q->vorticity_coef_ = p->vorticity_coef;
  q->smoothing_radius_ = p->smoothing_radius > 0 ? p->smoothing_radius : -1.0f;
  q->particle_rest_spacing_ = p->rest_spacing > 0 ? p->rest_spacing : -1.0f;
  for (int i = 0; i < 3; ++i) {
    q->boundary_.min[i] = p->boundary_min[i];
    q->boundary_.max[i] = p->boundary_max[i];
    q->initial_fluid_.min[i] = p->fluid_min[i];
    q->initial_fluid_.max[i] = p->fluid_max[i];
    q->mover_center_[i] = p->mover_center[i];
  }
  q->derive_from_input();
  if (p->rest_density > 0) q->rest_density_ = p->rest_density;
  return q;
}

// Read the derived parameters back (parameters.h:123-148).
int ref_derived(const ref_params_t* p, float out[8]) {
  try {
    Params* q = make_params(p);
    out[0] = q->particle_rest_spacing_;
    out[1] = q->particle_radius_;
    out[2] = q->smoothing_radius_;
    out[3] = q->neighbor_bin_spacing_;
    out[4] = q->rest_density_;
    out[5] = q->rest_mass_;
    out[6] = q->max_speed_;
    out[7] = (float)q->solve_step_count_;
    delete q;
    return 0;
  } catch (std::exception const& e) {
    g_error = e.what();
    return -1;
  }
}

// Parameters from an INI file through the reference's own read_INI (parameters.h:92-119).
int ref_derived_from_ini(const char* path, float out[8], uint64_t counts[3]) {
  try {
    Params q{std::string(path)};
    out[0] = q.particle_rest_spacing_;
    out[1] = q.particle_radius_;
    out[2] = q.smoothing_radius_;
    out[3] = q.neighbor_bin_spacing_;
    out[4] = q.rest_density_;
    out[5] = q.rest_mass_;
    out[6] = q.max_speed_;
    out[7] = q.gravity_;
    counts[0] = q.max_particles_local_;
    counts[1] = q.initial_global_particle_count_;
    counts[2] = q.solve_step_count_;
    return 0;
  } catch (std::exception const& e) {
    g_error = e.what();
    return -1;
  }
}

void* ref_create(const ref_params_t* p) {
  try {
    auto* s = new RefSim();
    s->params = make_params(p);
    s->parts = new Parts(*s->params);
    return s;
  } catch (std::exception const& e) {
    g_error = e.what();
    return nullptr;
  }
}

void ref_destroy(void* h) {
  auto* s = static_cast<RefSim*>(h);
  if (!s) return;
  delete s->parts;
  delete s->params;
  delete s;
}

void ref_set_rest_density(void* h, float rho0) { static_cast<RefSim*>(h)->params->rest_density_ = rho0; }

float ref_get_param(void* h, int which) {
  auto* q = static_cast<RefSim*>(h)->params;
  switch (which) {
    case 0: return q->rest_density_;
    case 1: return q->smoothing_radius_;
    case 2: return q->neighbor_bin_spacing_;
    case 3: return q->max_speed_;
    case 4: return q->particle_rest_spacing_;
    default: return -1.0f;
  }
}

// construct_fluid over the INI's InitialFluid box (particles.h:231-250).
int64_t ref_construct_fluid(void* h) {
  auto* s = static_cast<RefSim*>(h);
  try {
    return (int64_t)s->parts->construct_fluid(s->params->initial_fluid());
  } catch (std::exception const& e) {
    g_error = e.what();
    return -1;
  }
}

// construct_fluid over a given box with an initial velocity (particles.h:231-250),
// as the multi-rank driver's distribute_fluid calls it (distributor.h:318-353).
int64_t ref_construct_fluid_box(void* h, const float mn[3], const float mx[3], const float vel[3]) {
  auto* s = static_cast<RefSim*>(h);
  try {
    AABB<Real, Dim> box;
    box.min = V3{mn[0], mn[1], mn[2]};
    box.max = V3{mx[0], mx[1], mx[2]};
    return (int64_t)s->parts->construct_fluid(box, V3{vel[0], vel[1], vel[2]});
  } catch (std::exception const& e) {
    g_error = e.what();
    return -1;
  }
}

// Append particles with x* = x (particles.h:161-176).
int ref_add(void* h, const float* x, const float* v, uint64_t n) {
  auto* s = static_cast<RefSim*>(h);
  try {
    for (uint64_t i = 0; i < n; ++i) {
      V3 xp{x[3 * i], x[3 * i + 1], x[3 * i + 2]};
      V3 vp{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
      s->parts->add(xp, xp, vp);
    }
    return 0;
  } catch (std::exception const& e) {
    g_error = e.what();
    return -1;
  }
}

uint64_t ref_count(void* h) { return static_cast<RefSim*>(h)->parts->local_count(); }

// Drop the last k particles (particles.h:146-154): the multi-rank driver's
// halo invalidation and OOB removal.
int ref_remove(void* h, uint64_t k) {
  auto* p = static_cast<RefSim*>(h)->parts;
  if (k > p->local_count()) {
    g_error = "ref_remove: more particles than held";
    return -1;
  }
  p->remove(k);
  return 0;
}

// Overwrite per-particle arrays (AoS float3) of the current particles.
// which: 0 positions, 1 position_stars, 2 velocities, 3 scratch
int ref_set_vec(void* h, int which, const float* src) {
  auto* p = static_cast<RefSim*>(h)->parts;
  sim::Array<V3>* a = which == 0 ? &p->positions_ : which == 1 ? &p->position_stars_
                    : which == 2 ? &p->velocities_ : &p->scratch_;
  for (size_t i = 0; i < p->local_count(); ++i)
    (*a)[i] = V3{src[3 * i], src[3 * i + 1], src[3 * i + 2]};
  return 0;
}

int ref_get_vec(void* h, int which, float* dst) {
  auto* p = static_cast<RefSim*>(h)->parts;
  sim::Array<V3>* a = which == 0 ? &p->positions_ : which == 1 ? &p->position_stars_
                    : which == 2 ? &p->velocities_ : &p->scratch_;
  for (size_t i = 0; i < p->local_count(); ++i) {
    dst[3 * i] = (*a)[i].x;
    dst[3 * i + 1] = (*a)[i].y;
    dst[3 * i + 2] = (*a)[i].z;
  }
  return 0;
}

// which: 0 densities, 1 lambdas
int ref_get_scalar(void* h, int which, float* dst) {
  auto* p = static_cast<RefSim*>(h)->parts;
  sim::Array<Real>* a = which == 0 ? &p->densities_ : &p->lambdas_;
  for (size_t i = 0; i < p->local_count(); ++i) dst[i] = (*a)[i];
  return 0;
}

int ref_set_scalar(void* h, int which, const float* src) {
  auto* p = static_cast<RefSim*>(h)->parts;
  sim::Array<Real>* a = which == 0 ? &p->densities_ : &p->lambdas_;
  for (size_t i = 0; i < p->local_count(); ++i) (*a)[i] = src[i];
  return 0;
}

// Neighbor grid dimensions (neighbors.h:69-71).
void ref_bin_dims(void* h, uint64_t out[3]) {
  auto d = static_cast<RefSim*>(h)->parts->neighbors_.bin_dimensions();
  out[0] = d.x;
  out[1] = d.y;
  out[2] = d.z;
}

uint64_t ref_bin_id(void* h, const float p[3]) {
  return static_cast<RefSim*>(h)->parts->neighbors_.calculate_bin_id(V3{p[0], p[1], p[2]});
}

// Neighbor lists as int32 [N][cap] (entries past count are left untouched) and
// counts (neighbors.h:41-44).
int ref_get_neighbors(void* h, int32_t* idx, int32_t* count, int cap) {
  auto* p = static_cast<RefSim*>(h)->parts;
  for (size_t i = 0; i < p->local_count(); ++i) {
    const sim::NeighborList& l = p->neighbors_[i];
    count[i] = l.count;
    for (int k = 0; k < l.count && k < cap; ++k) idx[i * cap + k] = (int32_t)l.neighbor_indices[k];
  }
  return 0;
}

// Sorted bin ids and particle ids after sort_bins (neighbors.h:130-132) and
// begin/end of every bin (neighbors.h:137-148).
int ref_get_bins(void* h, uint64_t* sorted_keys, uint64_t* particle_ids, uint64_t* bin_begin,
                 uint64_t* bin_end) {
  auto* p = static_cast<RefSim*>(h)->parts;
  auto& nb = p->neighbors_;
  const size_t n = p->local_count();
  for (size_t i = 0; i < n; ++i) {
    if (sorted_keys) sorted_keys[i] = nb.bin_ids_[i];
    if (particle_ids) particle_ids[i] = nb.particle_ids_[i];
  }
  const size_t nbins = product(nb.bin_dimensions_);
  for (size_t b = 0; b < nbins; ++b) {
    if (bin_begin) bin_begin[b] = nb.begin_indices_[b];
    if (bin_end) bin_end[b] = nb.end_indices_[b];
  }
  return 0;
}

// One stage of the step, named as in Simulation/Source/particles.h.
//  0 apply_external_forces   1 predict_positions   2 find_neighbors
//  3 compute_densities       4 compute_pressure_lambdas
//  5 compute_pressure_dps    6 update_position_stars
//  7 update_velocities       8 apply_surface_tension
//  9 apply_viscosity        10 compute_vorticity  11 apply_vorticity
// 12 update_positions
int ref_stage(void* h, int stage, int sub) {
  auto* s = static_cast<RefSim*>(h);
  auto* p = s->parts;
  const IndexSpan span{0, p->local_count()};
  try {
    switch (stage) {
      case 0: p->apply_external_forces(span); break;
      case 1: p->predict_positions(span); break;
      case 2: p->find_neighbors(span, span); break;
      case 3: p->compute_densities(span); break;
      case 4: p->compute_pressure_lambdas(span); break;
      case 5: p->compute_pressure_dps(span, sub); break;
      case 6: p->update_position_stars(span); break;
      case 7: p->update_velocities(span); break;
      case 8: p->apply_surface_tension(span, span); break;
      case 9: p->apply_viscosity(span); break;
      case 10: p->compute_vorticity(span); break;
      case 11: p->apply_vorticity(span); break;
      case 12: p->update_positions(span); break;
      default: g_error = "unknown stage"; return -1;
    }
    return 0;
  } catch (std::exception const& e) {
    g_error = e.what();
    return -1;
  }
}

// One stage over explicit spans, as the multi-rank driver calls them
// (Simulation/Source/main.adios: resident and local spans): [a0, a1) is the
// stage's span; [b0, b1) the second span of find_neighbors (fill) and
// apply_surface_tension.  Stage numbers as in ref_stage.
int ref_stage_span(void* h, int stage, int sub, uint64_t a0, uint64_t a1, uint64_t b0, uint64_t b1) {
  auto* p = static_cast<RefSim*>(h)->parts;
  const IndexSpan a{a0, a1}, b{b0, b1};
  try {
    switch (stage) {
      case 0: p->apply_external_forces(a); break;
      case 1: p->predict_positions(a); break;
      case 2: p->find_neighbors(a, b); break;
      case 3: p->compute_densities(a); break;
      case 4: p->compute_pressure_lambdas(a); break;
      case 5: p->compute_pressure_dps(a, sub); break;
      case 6: p->update_position_stars(a); break;
      case 7: p->update_velocities(a); break;
      case 8: p->apply_surface_tension(a, b); break;
      case 9: p->apply_viscosity(a); break;
      case 10: p->compute_vorticity(a); break;
      case 11: p->apply_vorticity(a); break;
      case 12: p->update_positions(a); break;
      default: g_error = "unknown stage"; return -1;
    }
    return 0;
  } catch (std::exception const& e) {
    g_error = e.what();
    return -1;
  }
}

// The per-step stage order of Simulation/Source/main.cpp:71-124 on a single
// rank (domain_sync and the renderer/halo calls are MPI-only and absent).
int ref_step(void* h, int nsteps) {
  auto* s = static_cast<RefSim*>(h);
  auto* p = s->parts;
  const IndexSpan span{0, p->local_count()};
  try {
    for (int step = 0; step < nsteps; ++step) {
      p->apply_external_forces(span);
      p->predict_positions(span);
      p->find_neighbors(span, span);
      for (unsigned int sub = 0; sub < s->params->solve_step_count(); sub++) {
        p->compute_densities(span);
        p->compute_pressure_lambdas(span);
        p->compute_pressure_dps(span, sub);
        p->update_position_stars(span);
      }
      p->update_velocities(span);
      p->apply_surface_tension(span, span);
      p->apply_viscosity(span);
      p->compute_vorticity(span);
      p->apply_vorticity(span);
      p->apply_viscosity(span);
      p->update_positions(span);
    }
    return 0;
  } catch (std::exception const& e) {
    g_error = e.what();
    return -1;
  }
}

// Wall time of ref_step(h, nsteps) in seconds (std::chrono::steady_clock).
double ref_time_steps(void* h, int nsteps) {
  const auto t0 = std::chrono::steady_clock::now();
  if (ref_step(h, nsteps) != 0) return -1.0;
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
