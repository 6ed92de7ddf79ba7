/*
 * pbf_oracle.c — CPU restatement of the reference's PBF step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 * The product library never links or calls it.
 *
 * It restates, in plain C and in the reference's floating-point operation
 * order (no FMA contraction: built with -ffp-contract=off), the functions of
 * AdamSimpson/SPH-CPP that make up one PBF time step:
 *   Common/parameters.h:123-148   derive_from_input
 *   Common/vec.h:476-507,526,622  dot / magnitude / cross
 *   Common/aabb.h:213-219         bin_count_in_volume
 *   Simulation/Source/kernels.h   Poly6, Del_Spikey, C_Spline (3D)
 *   Simulation/Source/neighbors.h calculate_bin_id, sort, bin bounds, fill
 *   Simulation/Source/particles.h every stage, apply_boundary_conditions
 *   Simulation/Source/main.cpp:71-124  stage order of one step
 * Parity is pinned by tests/test_oracle_ref.py against the reference itself,
 * compiled from its own sources into oracle/_ref/ (oracle/ref_build/Makefile),
 * and by the golden vectors under tests/golden/ generated from that build.
 *
 * Two documented departures, each selectable:
 *  - XSPH viscosity (particles.h:436-447) updates velocities in place while
 *    neighbours read them, and compute_densities (particles.h:303-305) nudges
 *    a particle sitting on a neighbour in place while others read it, so the
 *    reference's result depends on thread order.  visc_mode 1 reproduces its
 *    single-thread order (in place, index order); visc_mode 0 is the GPU's
 *    deterministic order (Jacobi: read old, write new after the pass).
 *  - s_corr (scorr_k > 0) is the Macklin & Mueller 2013 artificial-pressure
 *    term, absent from the reference's compute_pressure_dps.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/pbf.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct {
  float x, y, z;
} v3;

static inline v3 v3_sub(v3 a, v3 b) {
  v3 r = {a.x - b.x, a.y - b.y, a.z - b.z};
  return r;
}
/* dot accumulates from 0 in x, y, z order (vec.h:476-483). */
static inline float v3_mag2(v3 a) {
  float d = 0.0f;
  d += a.x * a.x;
  d += a.y * a.y;
  d += a.z * a.z;
  return d;
}
static inline float v3_mag(v3 a) { return sqrtf(v3_mag2(a)); } /* vec.h:500-504 */
static inline v3 v3_cross(v3 l, v3 r) {                         /* vec.h:622-630 */
  v3 c;
  c.x = l.y * r.z - l.z * r.y;
  c.y = l.z * r.x - l.x * r.z;
  c.z = l.x * r.y - l.y * r.x;
  return c;
}

/* ---------------- kernels.h (3D) ---------------- */
typedef struct {
  float h, poly6_norm, spikey_norm, cspline_norm;
} kern_t;

static kern_t make_kern(float h) {
  kern_t k;
  k.h = h;
  k.poly6_norm = (float)(315.0 / (64.0 * M_PI * pow(h, 9.0))); /* kernels.h:61-62 */
  k.spikey_norm = (float)(-45.0 / (M_PI * pow(h, 6.0)));       /* kernels.h:159-160 */
  k.cspline_norm = (float)(32.0 / (M_PI * pow(h, 9.0)));       /* kernels.h:217-218 */
  return k;
}

/* Poly6 (kernels.h:64-70) */
static inline float poly6(const kern_t* k, float r) {
  if (r > k->h) return 0.0f;
  const float a = k->h * k->h - r * r;
  return k->poly6_norm * a * a * a;
}

/* Del_Spikey (kernels.h:163-172); eps = FLT_EPSILON (kernels.h:161) */
static inline v3 del_spikey(const kern_t* k, v3 p, v3 q) {
  const v3 r = v3_sub(p, q);
  const float rm = v3_mag(r);
  v3 out = {0.0f, 0.0f, 0.0f};
  if (rm > k->h) return out;
  const float s = k->spikey_norm * (k->h - rm) * (k->h - rm);
  const float den = rm + FLT_EPSILON;
  out.x = (s * r.x) / den;
  out.y = (s * r.y) / den;
  out.z = (s * r.z) / den;
  return out;
}

/* C_Spline (kernels.h:220-228); the r <= h/2 branch is evaluated in double
 * because its leading literal 2.0 is a double. */
static inline float c_spline(const kern_t* k, float r) {
  const float h = k->h;
  if (r > h) return 0.0f;
  if (r <= h * 0.5f) {
    const float hr = h - r;
    const double t = 2.0 * hr * hr * hr * r * r * r;
    const float h6 = h * h * h * h * h * h / 64.0f;
    return (float)(k->cspline_norm * (t - h6));
  }
  return k->cspline_norm * (h - r) * (h - r) * (h - r) * r * r * r;
}

/* ---------------- parameters.h:123-148 ---------------- */
int oracle_params_derive(pbf_params* p, float rest_spacing, float rho_override) {
  if (!p || !(rest_spacing > 0.0f)) return PBF_ERR_ARG;
  p->particle_rest_spacing = rest_spacing;
  if (p->smoothing_radius <= 0.0f) p->smoothing_radius = (float)(1.8 * (double)rest_spacing);
  if (p->neighbor_bin_spacing <= 0.0f)
    p->neighbor_bin_spacing = (float)(1.2 * (double)p->smoothing_radius);
  p->rest_mass = 1.0f;
  const float volume = powf(rest_spacing, 3.0f);
  p->rest_density = rho_override > 0.0f ? rho_override : p->rest_mass / volume;
  p->max_speed =
      (float)(0.5 * (double)p->smoothing_radius * (double)p->solve_steps / (double)p->time_step);
  return PBF_OK;
}

/* ---------------- scene: construct_fluid + seeded jitter ---------------- */
static uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* aabb.h:213-219 */
int oracle_lattice_dims(const float mn[3], const float mx[3], float spacing, int64_t out[3]) {
  for (int a = 0; a < 3; ++a) {
    const float c = floorf((mx[a] - mn[a]) / spacing);
    out[a] = c > 0.0f ? (int64_t)c : 0;
  }
  return PBF_OK;
}

/* particles.h:231-250 plus jitter u in [-amp, amp): u = (2*r24*2^-24 - 1)*amp */
int oracle_build_lattice(const float mn[3], const int64_t d[3], float spacing, float amp,
                         uint64_t seed, float* x) {
  const float half = spacing / 2.0f;
  int64_t i = 0;
  for (int64_t z = 0; z < d[2]; ++z)
    for (int64_t y = 0; y < d[1]; ++y)
      for (int64_t xx = 0; xx < d[0]; ++xx, ++i) {
        const int64_t c[3] = {xx, y, z};
        for (int a = 0; a < 3; ++a) {
          float v = (float)c[a] * spacing + mn[a];
          v += half;
          if (amp != 0.0f) {
            const uint64_t r = splitmix64(seed + 0x9E3779B97F4A7C15ull * (uint64_t)(3 * i + a));
            const float u = (float)(r >> 40) * 0x1p-24f;
            const float j = (u * 2.0f - 1.0f) * amp;
            v += j;
          }
          x[3 * i + a] = v;
        }
      }
  return PBF_OK;
}

/* ---------------- simulation state ---------------- */
typedef struct {
  pbf_params p;
  kern_t k;
  size_t n, cap_particles;
  int cap;         /* neighbor cap */
  int visc_mode;   /* 0 Jacobi, 1 in-place index order */
  int64_t dims[3]; /* neighbors.h:69-71 */
  int64_t nbins;
  v3 *x, *xs, *v, *scratch, *vtmp;
  float *rho, *lam;
  uint32_t *keys, *sorted_keys, *ids, *bin_begin, *bin_end;
  int32_t *nbr, *nbr_count;
  int have_lists;
} oracle_t;

static int64_t grid_dim(float extent, float s) {
  /* ceil(extent / s) + 2 in float, cast to size_t (neighbors.h:69-71) */
  return (int64_t)(ceilf(extent / s) + 2.0f);
}

int oracle_grid_dims(const pbf_params* p, int64_t out[3]) {
  for (int a = 0; a < 3; ++a)
    out[a] = grid_dim(p->boundary_max[a] - p->boundary_min[a], p->neighbor_bin_spacing);
  return PBF_OK;
}

void* oracle_create(const pbf_params* p, size_t capacity) {
  oracle_t* o = (oracle_t*)calloc(1, sizeof(oracle_t));
  if (!o) return NULL;
  o->p = *p;
  o->k = make_kern(p->smoothing_radius);
  o->cap_particles = capacity;
  o->cap = p->neighbor_cap > 0 ? p->neighbor_cap : 60;
  oracle_grid_dims(p, o->dims);
  o->nbins = o->dims[0] * o->dims[1] * o->dims[2];
  o->x = (v3*)calloc(capacity, sizeof(v3));
  o->xs = (v3*)calloc(capacity, sizeof(v3));
  o->v = (v3*)calloc(capacity, sizeof(v3));
  o->vtmp = (v3*)calloc(capacity, sizeof(v3));
  o->scratch = (v3*)calloc(capacity, sizeof(v3));
  o->rho = (float*)calloc(capacity, sizeof(float));
  o->lam = (float*)calloc(capacity, sizeof(float));
  o->keys = (uint32_t*)calloc(capacity, sizeof(uint32_t));
  o->sorted_keys = (uint32_t*)calloc(capacity, sizeof(uint32_t));
  o->ids = (uint32_t*)calloc(capacity, sizeof(uint32_t));
  o->bin_begin = (uint32_t*)calloc((size_t)o->nbins + 1, sizeof(uint32_t));
  o->bin_end = (uint32_t*)calloc((size_t)o->nbins + 1, sizeof(uint32_t));
  o->nbr = (int32_t*)malloc(capacity * (size_t)o->cap * sizeof(int32_t));
  o->nbr_count = (int32_t*)calloc(capacity, sizeof(int32_t));
  return o;
}

void oracle_destroy(void* h) {
  oracle_t* o = (oracle_t*)h;
  if (!o) return;
  free(o->x); free(o->xs); free(o->v); free(o->vtmp); free(o->scratch);
  free(o->rho); free(o->lam); free(o->keys); free(o->sorted_keys); free(o->ids);
  free(o->bin_begin); free(o->bin_end); free(o->nbr); free(o->nbr_count);
  free(o);
}

void oracle_set_visc_mode(void* h, int mode) { ((oracle_t*)h)->visc_mode = mode; }
void oracle_set_params(void* h, const pbf_params* p) {
  oracle_t* o = (oracle_t*)h;
  o->p = *p;
  o->k = make_kern(p->smoothing_radius);
}

/* particles.h:184-199: x* = x, everything else zero */
int oracle_set_state(void* h, const float* x, const float* v, size_t n) {
  oracle_t* o = (oracle_t*)h;
  if (n > o->cap_particles) return PBF_ERR_CAPACITY;
  o->n = n;
  memcpy(o->x, x, n * sizeof(v3));
  memcpy(o->xs, x, n * sizeof(v3));
  if (v) memcpy(o->v, v, n * sizeof(v3)); else memset(o->v, 0, n * sizeof(v3));
  memset(o->scratch, 0, n * sizeof(v3));
  memset(o->rho, 0, n * sizeof(float));
  memset(o->lam, 0, n * sizeof(float));
  o->have_lists = 0;
  return PBF_OK;
}

/* which: PBF_ARRAY_* */
int oracle_get(void* h, int which, float* out) {
  oracle_t* o = (oracle_t*)h;
  switch (which) {
    case PBF_ARRAY_POSITIONS: memcpy(out, o->x, o->n * sizeof(v3)); break;
    case PBF_ARRAY_POSITION_STARS: memcpy(out, o->xs, o->n * sizeof(v3)); break;
    case PBF_ARRAY_VELOCITIES: memcpy(out, o->v, o->n * sizeof(v3)); break;
    case PBF_ARRAY_SCRATCH: memcpy(out, o->scratch, o->n * sizeof(v3)); break;
    case PBF_ARRAY_DENSITIES: memcpy(out, o->rho, o->n * sizeof(float)); break;
    case PBF_ARRAY_LAMBDAS: memcpy(out, o->lam, o->n * sizeof(float)); break;
    default: return PBF_ERR_ARG;
  }
  return PBF_OK;
}

int oracle_set(void* h, int which, const float* in) {
  oracle_t* o = (oracle_t*)h;
  switch (which) {
    case PBF_ARRAY_POSITIONS: memcpy(o->x, in, o->n * sizeof(v3)); break;
    case PBF_ARRAY_POSITION_STARS: memcpy(o->xs, in, o->n * sizeof(v3)); break;
    case PBF_ARRAY_VELOCITIES: memcpy(o->v, in, o->n * sizeof(v3)); break;
    case PBF_ARRAY_SCRATCH: memcpy(o->scratch, in, o->n * sizeof(v3)); break;
    case PBF_ARRAY_DENSITIES: memcpy(o->rho, in, o->n * sizeof(float)); break;
    case PBF_ARRAY_LAMBDAS: memcpy(o->lam, in, o->n * sizeof(float)); break;
    default: return PBF_ERR_ARG;
  }
  return PBF_OK;
}

/* apply_boundary_conditions (particles.h:510-526) */
static inline v3 apply_bc(const pbf_params* p, v3 pos) {
  const float mr = p->mover_radius;
  const v3 mc = {p->mover_center[0], p->mover_center[1], p->mover_center[2]};
  const float dr2 = v3_mag2(v3_sub(pos, mc));
  if (dr2 < mr * mr) {
    const float dr = sqrtf(dr2);
    const float a = mr - dr;
    const v3 d = v3_sub(pos, mc);
    pos.x += (a * d.x) / dr;
    pos.y += (a * d.y) / dr;
    pos.z += (a * d.z) / dr;
  }
  /* clamp_in_place (vec.h:671-675, utility_math.h:52-57) */
  float* c = &pos.x;
  for (int i = 0; i < 3; ++i) {
    if (c[i] < p->boundary_min[i]) c[i] = p->boundary_min[i];
    else if (c[i] > p->boundary_max[i]) c[i] = p->boundary_max[i];
  }
  return pos;
}

/* calculate_bin_id 3D (neighbors.h:109-114) */
static inline int64_t bin_id(const oracle_t* o, v3 pt) {
  const float s = o->p.neighbor_bin_spacing;
  const float bx = floorf((pt.x + s) / s), by = floorf((pt.y + s) / s), bz = floorf((pt.z + s) / s);
  const int64_t ix = (int64_t)bx, iy = (int64_t)by, iz = (int64_t)bz;
  return o->dims[0] * o->dims[1] * iz + (iy * o->dims[0] + ix);
}

uint64_t oracle_bin_id(void* h, const float p[3]) {
  v3 pt = {p[0], p[1], p[2]};
  return (uint64_t)bin_id((oracle_t*)h, pt);
}

/* ---------------- stages ---------------- */

/* particles.h:263-270 */
static void st_external(oracle_t* o) {
  const float g = o->p.gravity, dt = o->p.time_step;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)o->n; ++i) o->v[i].y += g * dt;
}

/* particles.h:275-287 */
static void st_predict(oracle_t* o) {
  const float dt = o->p.time_step;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)o->n; ++i) {
    v3 s = o->x[i];
    s.x += o->v[i].x * dt;
    s.y += o->v[i].y * dt;
    s.z += o->v[i].z * dt;
    o->xs[i] = apply_bc(&o->p, s);
  }
}

/* Neighbors::find (neighbors.h:241-248): bins, stable sort by key, bin bounds,
 * fixed-cap lists.  The stable sort_by_key is a counting sort over bin ids
 * (ties keep ascending particle id, as the stable sort does). */
static int st_find_neighbors(oracle_t* o) {
  const int64_t n = (int64_t)o->n, B = o->nbins;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t b = bin_id(o, o->xs[i]);
    if (b < 0 || b >= B) return PBF_ERR_PARAMS;
    o->keys[i] = (uint32_t)b;
  }
  memset(o->bin_begin, 0, (size_t)(B + 1) * sizeof(uint32_t));
  for (int64_t i = 0; i < n; ++i) o->bin_begin[o->keys[i] + 1]++;
  for (int64_t b = 0; b < B; ++b) o->bin_begin[b + 1] += o->bin_begin[b];
  for (int64_t b = 0; b < B; ++b) o->bin_end[b] = o->bin_begin[b + 1];
  /* scatter using bin_end as a cursor copy */
  uint32_t* cursor = (uint32_t*)malloc((size_t)B * sizeof(uint32_t));
  memcpy(cursor, o->bin_begin, (size_t)B * sizeof(uint32_t));
  for (int64_t i = 0; i < n; ++i) {
    const uint32_t slot = cursor[o->keys[i]]++;
    o->ids[slot] = (uint32_t)i;
    o->sorted_keys[slot] = o->keys[i];
  }
  free(cursor);

  /* fill_neighbors (neighbors.h:197-230) */
  const float s = o->p.neighbor_bin_spacing;
  const float r2max = s * s;
  const int cap = o->cap;
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t p = 0; p < n; ++p) {
    const v3 xp = o->xs[p];
    int count = 0;
    int32_t* list = o->nbr + (size_t)p * cap;
    /* calculate_neighbor_indices 3D (neighbors.h:172-185): i (x) outer, k (z) inner */
    for (int i = -1; i < 2; i++)
      for (int j = -1; j < 2; j++)
        for (int kk = -1; kk < 2; kk++) {
          v3 nc;
          nc.x = xp.x + (float)i * s;
          nc.y = xp.y + (float)j * s;
          nc.z = xp.z + (float)kk * s;
          const int64_t nb = bin_id(o, nc);
          if (nb < 0 || nb >= B) continue; /* never for a validated grid */
          const uint32_t b0 = o->bin_begin[nb], b1 = o->bin_end[nb];
          for (uint32_t jj = b0; jj < b1; ++jj) {
            const uint32_t q = o->ids[jj];
            if ((int64_t)q == p) continue;
            const float d2 = v3_mag2(v3_sub(xp, o->xs[q]));
            if (d2 < r2max && count < cap) list[count++] = (int32_t)q;
          }
        }
    o->nbr_count[p] = count;
  }
  o->have_lists = 1;
  return PBF_OK;
}

/* particles.h:292-313, with the coincident-neighbour nudge of 303-305.
 * The reference nudges position_stars_[p] in place while other threads read
 * it.  visc_mode 1 (the reference's single-thread order): a serial loop, in
 * place.  visc_mode 0 (GPU semantics, deterministic): each particle sums with
 * its own nudged position; every nudge is written back after the pass. */
static float density_of(const oracle_t* o, int64_t p, v3* xp_io, const v3* xs) {
  const float W0 = poly6(&o->k, 0.0f);
  const float m = o->p.rest_mass, dt = o->p.time_step;
  float d = m * W0;
  v3 xp = *xp_io;
  const int32_t* list = o->nbr + (size_t)p * o->cap;
  for (int c = 0; c < o->nbr_count[p]; ++c) {
    const int32_t q = list[c];
    const v3 xq = xs[q];
    if ((double)v3_mag(v3_sub(xp, xq)) < 0.00000001) {
      const v3 vp = o->v[p];
      xp.x -= vp.x * dt / 50.0f;
      xp.y -= vp.y * dt / 50.0f;
      xp.z -= vp.z * dt / 50.0f;
    }
    const float rm = v3_mag(v3_sub(xp, xq));
    d += m * poly6(&o->k, rm);
  }
  *xp_io = xp;
  return d;
}

static void st_densities(oracle_t* o) {
  if (o->visc_mode == 1) {
    for (int64_t p = 0; p < (int64_t)o->n; ++p) {
      v3 xp = o->xs[p];
      o->rho[p] = density_of(o, p, &xp, o->xs);
      o->xs[p] = xp;
    }
    return;
  }
  v3* out = o->vtmp;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)o->n; ++p) {
    v3 xp = o->xs[p];
    o->rho[p] = density_of(o, p, &xp, o->xs);
    out[p] = xp;
  }
  memcpy(o->xs, out, o->n * sizeof(v3));
}

/* particles.h:318-342 */
static void st_lambdas(oracle_t* o) {
  const float rho0 = o->p.rest_density, eps = o->p.lambda_epsilon;
  const int cap = o->cap;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)o->n; ++p) {
    const float constraint = o->rho[p] / rho0 - 1.0f;
    const float Cp = constraint < 0.0f ? 0.0f : constraint;
    float sumC = 0.0f;
    v3 sg = {0.0f, 0.0f, 0.0f};
    const float sc = -1.0f / rho0;
    const int32_t* list = o->nbr + (size_t)p * cap;
    for (int c = 0; c < o->nbr_count[p]; ++c) {
      const v3 dw = del_spikey(&o->k, o->xs[p], o->xs[list[c]]);
      const v3 g = {sc * dw.x, sc * dw.y, sc * dw.z};
      sg.x -= g.x;
      sg.y -= g.y;
      sg.z -= g.z;
      sumC += v3_mag2(g);
    }
    sumC += v3_mag2(sg);
    o->lam[p] = -Cp / (sumC + eps);
  }
}

/* particles.h:348-358; optional s_corr (not in the reference) */
static void st_dps(oracle_t* o) {
  const float rho0 = o->p.rest_density;
  const int cap = o->cap;
  const int scorr = o->p.scorr_k > 0.0f;
  const float wdq = scorr ? poly6(&o->k, o->p.scorr_dq * o->p.smoothing_radius) : 1.0f;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)o->n; ++p) {
    v3 dp = {0.0f, 0.0f, 0.0f};
    const int32_t* list = o->nbr + (size_t)p * cap;
    for (int c = 0; c < o->nbr_count[p]; ++c) {
      const int32_t q = list[c];
      float l = o->lam[p] + o->lam[q];
      if (scorr) {
        const float w = poly6(&o->k, v3_mag(v3_sub(o->xs[p], o->xs[q])));
        l += -o->p.scorr_k * powf(w / wdq, o->p.scorr_n);
      }
      const v3 dw = del_spikey(&o->k, o->xs[p], o->xs[q]);
      dp.x += l * dw.x;
      dp.y += l * dw.y;
      dp.z += l * dw.z;
    }
    const float s = 1.0f / rho0;
    o->scratch[p].x = s * dp.x;
    o->scratch[p].y = s * dp.y;
    o->scratch[p].z = s * dp.z;
  }
}

/* particles.h:363-370 */
static void st_update_xs(oracle_t* o) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)o->n; ++p) {
    v3 s = o->xs[p];
    s.x += o->scratch[p].x;
    s.y += o->scratch[p].y;
    s.z += o->scratch[p].z;
    o->xs[p] = apply_bc(&o->p, s);
  }
}

/* particles.h:375-385 */
static void st_update_v(oracle_t* o) {
  const float dt = o->p.time_step;
  const double thr = 0.000001 * (double)o->p.max_speed;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)o->n; ++p) {
    v3 v;
    v.x = (o->xs[p].x - o->x[p].x) / dt;
    v.y = (o->xs[p].y - o->x[p].y) / dt;
    v.z = (o->xs[p].z - o->x[p].z) / dt;
    if ((double)v3_mag2(v) < thr) v.x = v.y = v.z = 0.0f;
    o->v[p] = v;
  }
}

/* particles.h:390-394 */
static void st_update_x(oracle_t* o) { memcpy(o->x, o->xs, o->n * sizeof(v3)); }

/* particles.h:400-431 */
static void st_surface_tension(oracle_t* o) {
  const int cap = o->cap;
  const float h = o->p.smoothing_radius, gamma = o->p.gamma, dt = o->p.time_step;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)o->n; ++p) {
    v3 color = {0.0f, 0.0f, 0.0f};
    const int32_t* list = o->nbr + (size_t)p * cap;
    for (int c = 0; c < o->nbr_count[p]; ++c) {
      const int32_t q = list[c];
      const v3 dw = del_spikey(&o->k, o->xs[p], o->xs[q]);
      color.x += dw.x / o->rho[q];
      color.y += dw.y / o->rho[q];
      color.z += dw.z / o->rho[q];
    }
    o->scratch[p].x = h * color.x;
    o->scratch[p].y = h * color.y;
    o->scratch[p].z = h * color.z;
  }
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)o->n; ++p) {
    v3 f = {0.0f, 0.0f, 0.0f};
    const int32_t* list = o->nbr + (size_t)p * cap;
    for (int c = 0; c < o->nbr_count[p]; ++c) {
      const int32_t q = list[c];
      const v3 r = v3_sub(o->xs[p], o->xs[q]);
      float rm = v3_mag(r);
      if ((double)rm < (double)h * 0.000001) rm = (float)((double)h * 0.000001);
      const float cs = -gamma * c_spline(&o->k, rm);
      const v3 coh = {(cs * r.x) / rm, (cs * r.y) / rm, (cs * r.z) / rm};
      const v3 cur = {-gamma * (o->scratch[p].x - o->scratch[q].x),
                      -gamma * (o->scratch[p].y - o->scratch[q].y),
                      -gamma * (o->scratch[p].z - o->scratch[q].z)};
      const float K = (float)(2.0 * (double)o->p.rest_density / (double)(o->rho[p] + o->rho[q]));
      f.x += K * (coh.x + cur.x);
      f.y += K * (coh.y + cur.y);
      f.z += K * (coh.z + cur.z);
    }
    o->v[p].x += f.x / o->rho[p] * dt;
    o->v[p].y += f.y / o->rho[p] * dt;
    o->v[p].z += f.z / o->rho[p] * dt;
  }
}

/* particles.h:436-447 (see visc_mode in the header comment) */
static v3 visc_dv(const oracle_t* o, int64_t p, const v3* vel) {
  v3 dv = {0.0f, 0.0f, 0.0f};
  const int32_t* list = o->nbr + (size_t)p * o->cap;
  for (int c = 0; c < o->nbr_count[p]; ++c) {
    const int32_t q = list[c];
    const float w = poly6(&o->k, v3_mag(v3_sub(o->xs[p], o->xs[q])));
    dv.x += (vel[q].x - vel[p].x) * w / o->rho[q];
    dv.y += (vel[q].y - vel[p].y) * w / o->rho[q];
    dv.z += (vel[q].z - vel[p].z) * w / o->rho[q];
  }
  return dv;
}

static void st_viscosity(oracle_t* o) {
  const float c = o->p.visc_c;
  if (o->visc_mode == 1) {
    for (int64_t p = 0; p < (int64_t)o->n; ++p) {
      const v3 dv = visc_dv(o, p, o->v);
      o->v[p].x += c * dv.x;
      o->v[p].y += c * dv.y;
      o->v[p].z += c * dv.z;
    }
    return;
  }
  memcpy(o->vtmp, o->v, o->n * sizeof(v3));
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)o->n; ++p) {
    const v3 dv = visc_dv(o, p, o->vtmp);
    o->v[p].x = o->vtmp[p].x + c * dv.x;
    o->v[p].y = o->vtmp[p].y + c * dv.y;
    o->v[p].z = o->vtmp[p].z + c * dv.z;
  }
}

/* particles.h:452-466 */
static void st_vorticity(oracle_t* o) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)o->n; ++p) {
    v3 w = {0.0f, 0.0f, 0.0f};
    const int32_t* list = o->nbr + (size_t)p * o->cap;
    for (int c = 0; c < o->nbr_count[p]; ++c) {
      const int32_t q = list[c];
      const v3 del = del_spikey(&o->k, o->xs[p], o->xs[q]);
      const v3 vd = v3_sub(o->v[q], o->v[p]);
      const v3 cr = v3_cross(vd, del);
      w.x += cr.x;
      w.y += cr.y;
      w.z += cr.z;
    }
    o->scratch[p] = w;
  }
}

/* particles.h:471-487 */
static void st_apply_vorticity(oracle_t* o) {
  const float ve = o->p.vorticity_coef, dt = o->p.time_step;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)o->n; ++p) {
    v3 eta = {0.0f, 0.0f, 0.0f};
    const int32_t* list = o->nbr + (size_t)p * o->cap;
    for (int c = 0; c < o->nbr_count[p]; ++c) {
      const int32_t q = list[c];
      const v3 del = del_spikey(&o->k, o->xs[p], o->xs[q]);
      const float vm = v3_mag(o->scratch[q]);
      eta.x += vm * del.x;
      eta.y += vm * del.y;
      eta.z += vm * del.z;
    }
    const float den = v3_mag(eta) + FLT_EPSILON;
    const v3 N = {eta.x / den, eta.y / den, eta.z / den};
    const v3 cr = v3_cross(N, o->scratch[p]);
    o->v[p].x += cr.x * ve * dt;
    o->v[p].y += cr.y * ve * dt;
    o->v[p].z += cr.z * ve * dt;
  }
}

/* Stage numbering shared with the reference driver (oracle/ref_build). */
int oracle_stage(void* h, int stage, int sub) {
  oracle_t* o = (oracle_t*)h;
  (void)sub; /* compute_pressure_dps ignores its substep (particles.h:348-358) */
  if (stage >= 3 && stage != 7 && stage != 12 && !o->have_lists) return PBF_ERR_STATE;
  switch (stage) {
    case 0: st_external(o); break;
    case 1: st_predict(o); break;
    case 2: return st_find_neighbors(o);
    case 3: st_densities(o); break;
    case 4: st_lambdas(o); break;
    case 5: st_dps(o); break;
    case 6: st_update_xs(o); break;
    case 7: st_update_v(o); break;
    case 8: st_surface_tension(o); break;
    case 9: st_viscosity(o); break;
    case 10: st_vorticity(o); break;
    case 11: st_apply_vorticity(o); break;
    case 12: st_update_x(o); break;
    default: return PBF_ERR_ARG;
  }
  return PBF_OK;
}

/* One step in the order of Simulation/Source/main.cpp:71-124. */
int oracle_step(void* h, int nsteps) {
  oracle_t* o = (oracle_t*)h;
  for (int s = 0; s < nsteps; ++s) {
    st_external(o);
    st_predict(o);
    int rc = st_find_neighbors(o);
    if (rc) return rc;
    for (int sub = 0; sub < o->p.solve_steps; ++sub) {
      st_densities(o);
      st_lambdas(o);
      st_dps(o);
      st_update_xs(o);
    }
    st_update_v(o);
    if (o->p.gamma != 0.0f) st_surface_tension(o); /* exact no-op at gamma = 0 */
    st_viscosity(o);
    st_vorticity(o);
    st_apply_vorticity(o);
    st_viscosity(o);
    st_update_x(o);
  }
  return PBF_OK;
}

/* Lists as [N][cap] original indices (-1 past count) and counts. */
int oracle_get_neighbors(void* h, int32_t* idx, int32_t* count) {
  oracle_t* o = (oracle_t*)h;
  for (size_t p = 0; p < o->n; ++p) {
    if (count) count[p] = o->nbr_count[p];
    if (idx)
      for (int c = 0; c < o->cap; ++c)
        idx[p * o->cap + c] = c < o->nbr_count[p] ? o->nbr[p * o->cap + c] : -1;
  }
  return PBF_OK;
}

int oracle_get_bins(void* h, uint32_t* sorted_keys, uint32_t* ids, uint32_t* begin, uint32_t* end) {
  oracle_t* o = (oracle_t*)h;
  if (sorted_keys) memcpy(sorted_keys, o->sorted_keys, o->n * sizeof(uint32_t));
  if (ids) memcpy(ids, o->ids, o->n * sizeof(uint32_t));
  if (begin) memcpy(begin, o->bin_begin, (size_t)o->nbins * sizeof(uint32_t));
  if (end) memcpy(end, o->bin_end, (size_t)o->nbins * sizeof(uint32_t));
  return PBF_OK;
}

int64_t oracle_num_bins(void* h) { return ((oracle_t*)h)->nbins; }

/* Residual statistics: density of the current x* over the current lists
 * (particles.h:292-313 without the nudge), clamped error max(rho/rho0-1, 0),
 * kinetic energy and centre of mass of x. */
int oracle_stats(void* h, pbf_stats_t* st) {
  oracle_t* o = (oracle_t*)h;
  memset(st, 0, sizeof(*st));
  st->n = o->n;
  if (!o->have_lists) return PBF_ERR_STATE;
  const float W0 = poly6(&o->k, 0.0f);
  const float m = o->p.rest_mass;
  double sum_err = 0.0, max_err = 0.0, ke = 0.0, cx = 0.0, cy = 0.0, cz = 0.0, nn = 0.0;
  uint64_t hits = 0;
  for (size_t p = 0; p < o->n; ++p) {
    float d = m * W0;
    const int32_t* list = o->nbr + p * o->cap;
    for (int c = 0; c < o->nbr_count[p]; ++c)
      d += m * poly6(&o->k, v3_mag(v3_sub(o->xs[p], o->xs[list[c]])));
    double e = (double)d / (double)o->p.rest_density - 1.0;
    if (e < 0.0) e = 0.0;
    sum_err += e;
    if (e > max_err) max_err = e;
    const v3 v = o->v[p];
    ke += 0.5 * (double)m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
    cx += o->x[p].x;
    cy += o->x[p].y;
    cz += o->x[p].z;
    nn += o->nbr_count[p];
    if (o->nbr_count[p] >= o->cap) hits++;
  }
  const double n = o->n ? (double)o->n : 1.0;
  st->mean_density_error = sum_err / n;
  st->max_density_error = max_err;
  st->kinetic_energy = ke;
  st->center_of_mass[0] = cx / n;
  st->center_of_mass[1] = cy / n;
  st->center_of_mass[2] = cz / n;
  st->mean_neighbors = nn / n;
  st->cap_hits = hits;
  return PBF_OK;
}

/* Exposed kernels for the kernel known-answer tests (kernels_test.cpp). */
float oracle_poly6(float h, float r) {
  const kern_t k = make_kern(h);
  return poly6(&k, r);
}
void oracle_del_spikey(float h, const float p[3], const float q[3], float out[3]) {
  const kern_t k = make_kern(h);
  const v3 a = {p[0], p[1], p[2]}, b = {q[0], q[1], q[2]};
  const v3 r = del_spikey(&k, a, b);
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
float oracle_c_spline(float h, float r) {
  const kern_t k = make_kern(h);
  return c_spline(&k, r);
}

/* Rest density of the centre particle of an unjittered (2r+1)^3 lattice,
 * built and summed exactly as the reference would on that lattice:
 * construct_fluid positions, find_neighbors, compute_densities. */
int oracle_lattice_rest_density(const pbf_params* p, float spacing, float* out) {
  const int r = 4;
  const int64_t d[3] = {2 * r + 1, 2 * r + 1, 2 * r + 1};
  const int64_t n = d[0] * d[1] * d[2];
  pbf_params q = *p;
  const float mn[3] = {0.0f, 0.0f, 0.0f};
  for (int a = 0; a < 3; ++a) {
    q.boundary_min[a] = 0.0f;
    q.boundary_max[a] = (float)d[a] * spacing;
  }
  float* x = (float*)malloc((size_t)n * 3 * sizeof(float));
  oracle_build_lattice(mn, d, spacing, 0.0f, 0, x);
  void* h = oracle_create(&q, (size_t)n);
  oracle_set_state(h, x, NULL, (size_t)n);
  int rc = st_find_neighbors((oracle_t*)h);
  if (rc == 0) {
    st_densities((oracle_t*)h);
    const int64_t c = (int64_t)r * d[0] * d[1] + (int64_t)r * d[0] + r;
    *out = ((oracle_t*)h)->rho[c];
  }
  oracle_destroy(h);
  free(x);
  return rc;
}
