// Host-side parameter derivation, INI schema and scene construction for the
// B200 PBF step.  No GPU is touched here.
//
// Mirrors the reference's Common/parameters.h (read_INI 92-119,
// derive_from_input 123-148), Common/aabb.h:213-219 (bin_count_in_volume) and
// Simulation/Source/particles.h:231-250 (construct_fluid), in the same
// floating-point operation order, so a scene built here is bit-identical to
// the reference's construct_fluid output.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/pbf.h"
#include "pbf_internal.h"

namespace pbf {

// Shared float rules of the hot path (neighbors.h:69-71, 109-114).
int64_t grid_dim(float extent, float s) { return (int64_t)(std::ceil(extent / s) + 2.0f); }

int64_t axis_bin(float c, float s) { return (int64_t)std::floor((c + s) / s); }

}  // namespace pbf

namespace {

std::string trim(const std::string& s) {
  const char* ws = " \t\r\n";
  const auto b = s.find_first_not_of(ws);
  if (b == std::string::npos) return "";
  const auto e = s.find_last_not_of(ws);
  return s.substr(b, e - b + 1);
}

uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

void pbf_params_init(pbf_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->time_step = -1.0f;
  p->gravity = -1.0f;
  p->gamma = -1.0f;
  p->visc_c = -1.0f;
  p->lambda_epsilon = -1.0f;
  p->vorticity_coef = -1.0f;
  p->smoothing_radius = -1.0f;
  p->neighbor_bin_spacing = -1.0f;
  p->rest_density = -1.0f;
  p->rest_mass = 1.0f;
  p->max_speed = -1.0f;
  p->particle_rest_spacing = -1.0f;
  p->mover_radius = 0.2f;  // particles.h:515
  p->solve_steps = -1;
  p->neighbor_cap = 60;  // neighbors.h:39
  p->scorr_k = 0.0f;
  p->scorr_n = 4.0f;
  p->scorr_dq = 0.2f;
  p->solver = 0;
  p->residual_tol = 0.01f;
  p->max_iterations = 8;
  p->residual_sample = 1;
}

// parameters.h:123-148
int pbf_params_derive(pbf_params* p, float rest_spacing, float rest_density_override) {
  if (!p || !(rest_spacing > 0.0f)) return PBF_ERR_ARG;
  p->particle_rest_spacing = rest_spacing;
  if (p->smoothing_radius <= 0.0f) p->smoothing_radius = (float)(1.8 * (double)rest_spacing);
  if (p->neighbor_bin_spacing <= 0.0f)
    p->neighbor_bin_spacing = (float)(1.2 * (double)p->smoothing_radius);
  p->rest_mass = 1.0f;
  const float volume = std::pow(rest_spacing, 3.0f);
  p->rest_density = rest_density_override > 0.0f ? rest_density_override : p->rest_mass / volume;
  p->max_speed = (float)(0.5 * (double)p->smoothing_radius * (double)p->solve_steps /
                         (double)p->time_step);
  return PBF_OK;
}

// parameters.h:92-119 key set; missing keys stay -1 as in the reference.
int pbf_params_from_ini(const char* path, pbf_params* p, float fluid_min[3], float fluid_max[3]) {
  if (!path || !p) return PBF_ERR_ARG;
  std::ifstream in(path);
  if (!in) return PBF_ERR_IO;
  std::map<std::string, std::string> kv;
  std::string line, section;
  while (std::getline(in, line)) {
    line = trim(line);
    if (line.empty() || line[0] == ';' || line[0] == '#') continue;
    if (line.front() == '[' && line.back() == ']') {
      section = trim(line.substr(1, line.size() - 2));
      continue;
    }
    const auto eq = line.find('=');
    if (eq == std::string::npos) continue;
    kv[section + "." + trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
  }
  auto getf = [&](const char* key, float dflt) {
    auto it = kv.find(key);
    if (it == kv.end()) return dflt;
    return std::stof(it->second);
  };
  auto geti = [&](const char* key, double dflt) {
    auto it = kv.find(key);
    if (it == kv.end()) return dflt;
    return std::stod(it->second);
  };
  auto getv = [&](const char* key, float out[3]) {
    out[0] = out[1] = out[2] = 0.0f;
    auto it = kv.find(key);
    if (it == kv.end()) return;
    std::stringstream ss(it->second);
    std::string item;
    for (int i = 0; i < 3 && std::getline(ss, item, ','); ++i) out[i] = std::stof(trim(item));
  };
  pbf_params_init(p);
  p->solve_steps = (int32_t)geti("SimParameters.number_solve_steps", -1);
  p->time_step = getf("SimParameters.time_step", -1.0f);
  const double global_count = geti("SimParameters.global_particle_count", -1);
  p->neighbor_bin_spacing = getf("SimParameters.neighbor_bin_spacing", -1.0f);
  p->neighbor_cap = (int32_t)geti("SimParameters.neighbor_cap", 60);
  p->exact_math = (int32_t)geti("SimParameters.exact_math", 0);
  p->gravity = getf("PhysicalParameters.g", -1.0f);
  p->gamma = getf("PhysicalParameters.gamma", -1.0f);
  p->visc_c = getf("PhysicalParameters.visc_c", -1.0f);
  p->lambda_epsilon = getf("PhysicalParameters.lambda_epsilon", -1.0f);
  p->vorticity_coef = getf("PhysicalParameters.vorticity_coef", -1.0f);
  p->smoothing_radius = getf("PhysicalParameters.smoothing_radius", -1.0f);
  const float spacing_key = getf("PhysicalParameters.rest_spacing", -1.0f);
  const float rho_key = getf("PhysicalParameters.rest_density_override", -1.0f);
  p->scorr_k = getf("PhysicalParameters.scorr_k", 0.0f);
  p->scorr_n = getf("PhysicalParameters.scorr_n", 4.0f);
  p->scorr_dq = getf("PhysicalParameters.scorr_dq", 0.2f);
  getv("Boundary.min", p->boundary_min);
  getv("Boundary.max", p->boundary_max);
  float fmin[3], fmax[3];
  getv("InitialFluid.min", fmin);
  getv("InitialFluid.max", fmax);
  getv("Mover.center", p->mover_center);
  if (fluid_min) std::memcpy(fluid_min, fmin, sizeof(fmin));
  if (fluid_max) std::memcpy(fluid_max, fmax, sizeof(fmax));
  float spacing = spacing_key;
  if (spacing <= 0.0f) {
    // parameters.h:124-125: (volume / count)^(1/Dim)
    const float volume = (fmax[0] - fmin[0]) * (fmax[1] - fmin[1]) * (fmax[2] - fmin[2]);
    spacing = (float)std::pow(volume / (float)(uint64_t)global_count, 1.0 / 3.0);
  }
  return pbf_params_derive(p, spacing, rho_key);
}

int pbf_lattice_dims(const float mn[3], const float mx[3], float spacing, int64_t out[3]) {
  if (!mn || !mx || !out || !(spacing > 0.0f)) return PBF_ERR_ARG;
  for (int a = 0; a < 3; ++a) {
    const float c = std::floor((mx[a] - mn[a]) / spacing);
    out[a] = c > 0.0f ? (int64_t)c : 0;
  }
  return PBF_OK;
}

// particles.h:231-250 + seeded jitter (SplitMix64 counter stream).
int pbf_build_lattice(const float mn[3], const int64_t d[3], float spacing, float amp,
                      uint64_t seed, float* x) {
  if (!mn || !d || !x || !(spacing > 0.0f)) return PBF_ERR_ARG;
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

int pbf_grid_dims(const pbf_params* p, int64_t out[3]) {
  if (!p || !out || !(p->neighbor_bin_spacing > 0.0f)) return PBF_ERR_ARG;
  for (int a = 0; a < 3; ++a)
    out[a] = pbf::grid_dim(p->boundary_max[a] - p->boundary_min[a], p->neighbor_bin_spacing);
  return PBF_OK;
}

// Centre-particle density of an unjittered (2r+1)^3 lattice with r = 4, as
// the reference's find_neighbors + compute_densities produce it
// (neighbors.h:197-230, particles.h:292-313): lattice positions from
// construct_fluid, neighbours in the 27-bin order with the strict s^2 test
// and the cap, Poly6 summed in list order.
int pbf_lattice_rest_density(const pbf_params* p, float spacing, float* rho0_out) {
  if (!p || !rho0_out || !(spacing > 0.0f) || !(p->smoothing_radius > 0.0f) ||
      !(p->neighbor_bin_spacing > 0.0f))
    return PBF_ERR_ARG;
  const int r = 4, n1 = 2 * r + 1;
  const int64_t d[3] = {n1, n1, n1};
  const int64_t n = (int64_t)n1 * n1 * n1;
  const float mn[3] = {0.0f, 0.0f, 0.0f};
  std::vector<float> x((size_t)n * 3);
  pbf_build_lattice(mn, d, spacing, 0.0f, 0, x.data());
  const float s = p->neighbor_bin_spacing, h = p->smoothing_radius;
  int64_t gd[3];
  for (int a = 0; a < 3; ++a) gd[a] = pbf::grid_dim((float)n1 * spacing - 0.0f, s);
  auto bin = [&](float px, float py, float pz) {
    return gd[0] * gd[1] * pbf::axis_bin(pz, s) + (pbf::axis_bin(py, s) * gd[0] + pbf::axis_bin(px, s));
  };
  // stable counting sort of particle ids by bin
  const int64_t B = gd[0] * gd[1] * gd[2];
  std::vector<int64_t> start(B + 1, 0), keys(n), ids(n);
  for (int64_t i = 0; i < n; ++i) {
    keys[i] = bin(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
    if (keys[i] < 0 || keys[i] >= B) return PBF_ERR_PARAMS;
    start[keys[i] + 1]++;
  }
  for (int64_t b = 0; b < B; ++b) start[b + 1] += start[b];
  std::vector<int64_t> cur(start.begin(), start.end() - 1);
  for (int64_t i = 0; i < n; ++i) ids[cur[keys[i]]++] = i;
  const int64_t c = (int64_t)r * n1 * n1 + (int64_t)r * n1 + r;
  const float px = x[3 * c], py = x[3 * c + 1], pz = x[3 * c + 2];
  const double norm_d = 315.0 / (64.0 * M_PI * std::pow((double)h, 9.0));
  const float norm = (float)norm_d;
  auto poly6 = [&](float rm) {
    if (rm > h) return 0.0f;
    const float a = h * h - rm * rm;
    return norm * a * a * a;
  };
  const float m = p->rest_mass > 0.0f ? p->rest_mass : 1.0f;
  float density = m * poly6(0.0f);
  int count = 0;
  const int cap = p->neighbor_cap > 0 ? p->neighbor_cap : 60;
  for (int i = -1; i < 2; i++)
    for (int j = -1; j < 2; j++)
      for (int k = -1; k < 2; k++) {
        const int64_t nb = bin(px + (float)i * s, py + (float)j * s, pz + (float)k * s);
        if (nb < 0 || nb >= B) continue;
        for (int64_t jj = start[nb]; jj < start[nb + 1]; ++jj) {
          const int64_t q = ids[jj];
          if (q == c) continue;
          float dx = px - x[3 * q], dy = py - x[3 * q + 1], dz = pz - x[3 * q + 2];
          float d2 = 0.0f;
          d2 += dx * dx;
          d2 += dy * dy;
          d2 += dz * dz;
          if (d2 < s * s && count < cap) {
            ++count;
            density += m * poly6(std::sqrt(d2));
          }
        }
      }
  *rho0_out = density;
  return PBF_OK;
}

}  // extern "C"
