// pbf_run — headless single-rank driver of the B200 PBF step.
//
// Replaces the reference's MPI/renderer driver (Simulation/Source/main.cpp)
// for one GPU: reads the reference's INI schema, builds the initial fluid as
// construct_fluid does (particles.h:231-250), then runs the time-step loop of
// main.cpp:71-124 — stage for stage through sim::gpu::Particles, or fused
// (--fused) through the graph-captured step — and prints statistics.
//
//   pbf_run params.ini [steps] [--fused] [--jitter AMP] [--seed S] [--dump out.bin]
//           [--save state.pbf] [--resume state.pbf] [--frames K PREFIX]
//
// --dump writes the final positions and velocities as raw float32 AoS
// (N x 3 each, after a uint64 N); --frames writes a state file (pbf.h) every
// K steps as PREFIX_<step>.pbf: the headless stand-ins for the reference's
// renderer gather / ADIOS position output (distributor.h:742-750).  --save
// writes the final state, --resume starts from a state file instead of the
// INI's initial fluid (the parameters then come from the file).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <vector>

#include "../../include/pbf_particles.hpp"

int main(int argc, char* argv[]) {
  try {
    if (argc < 2) {
      std::fprintf(stderr, "usage: %s params.ini [steps] [--fused] [--jitter AMP] [--seed S] [--dump F]\n", argv[0]);
      return 2;
    }
    int steps = argc > 2 && argv[2][0] != '-' ? std::atoi(argv[2]) : 10;
    bool fused = false;
    float jitter = 0.0f;
    uint64_t seed = 0;
    const char* dump = nullptr;
    const char* save = nullptr;
    const char* resume = nullptr;
    const char* frame_prefix = nullptr;
    int frame_every = 0;
    for (int i = 2; i < argc; ++i) {
      if (!std::strcmp(argv[i], "--fused")) fused = true;
      else if (!std::strcmp(argv[i], "--jitter") && i + 1 < argc) jitter = (float)std::atof(argv[++i]);
      else if (!std::strcmp(argv[i], "--seed") && i + 1 < argc) seed = std::strtoull(argv[++i], nullptr, 10);
      else if (!std::strcmp(argv[i], "--dump") && i + 1 < argc) dump = argv[++i];
      else if (!std::strcmp(argv[i], "--save") && i + 1 < argc) save = argv[++i];
      else if (!std::strcmp(argv[i], "--resume") && i + 1 < argc) resume = argv[++i];
      else if (!std::strcmp(argv[i], "--frames") && i + 2 < argc) {
        frame_every = std::atoi(argv[++i]);
        frame_prefix = argv[++i];
      }
    }
    pbf_params raw;
    float fmin[3], fmax[3];
    if (pbf_params_from_ini(argv[1], &raw, fmin, fmax) != PBF_OK) {
      std::fprintf(stderr, "cannot read %s\n", argv[1]);
      return 1;
    }
    float rho0 = 0.0f;
    if (pbf_lattice_rest_density(&raw, raw.particle_rest_spacing, &rho0) == PBF_OK) raw.rest_density = rho0;
    auto* parameters = new sim::gpu::Parameters(raw);
    size_t n = 0;
    std::vector<float> x, v;
    sim::gpu::Particles* particles = nullptr;
    if (resume) {
      // the particle count is the uint64 at byte 16 of the state file's header
      FILE* f = std::fopen(resume, "rb");
      uint64_t nn = 0;
      const bool ok = f && std::fseek(f, 16, SEEK_SET) == 0 && std::fread(&nn, sizeof(nn), 1, f) == 1;
      if (f) std::fclose(f);
      if (!ok) throw std::runtime_error(std::string("cannot read ") + resume);
      n = (size_t)nn;
      particles = new sim::gpu::Particles(parameters->raw(), n > 0 ? n : 1);
      particles->load(resume);
      x.resize(3 * n);
      v.resize(3 * n);
    } else {
      int64_t dims[3];
      pbf_lattice_dims(fmin, fmax, raw.particle_rest_spacing, dims);
      n = (size_t)(dims[0] * dims[1] * dims[2]);
      x.assign(3 * n, 0.0f);
      v.assign(3 * n, 0.0f);
      pbf_build_lattice(fmin, dims, raw.particle_rest_spacing, jitter * raw.smoothing_radius, seed, x.data());
      particles = new sim::gpu::Particles(parameters->raw(), n);
      particles->upload(x.data(), v.data(), n);
    }

    const sim::gpu::IndexSpan resident_span{0, n}, local_span{0, n};
    const uint64_t first_step = pbf_step_count(particles->handle());  // > 0 after --resume of a fused run
    for (int frame = 0; frame < steps; ++frame) {
      if (frame_every > 0 && frame % frame_every == 0) {
        char name[4096];
        std::snprintf(name, sizeof(name), "%s_%06llu.pbf", frame_prefix,
                      (unsigned long long)(first_step + (uint64_t)frame));
        particles->save(name);
      }
      if (fused) {
        particles->step(1);
        continue;
      }
      // Simulation/Source/main.cpp:71-124, single rank (domain_sync is MPI-only)
      particles->apply_external_forces(resident_span);
      particles->predict_positions(resident_span);
      particles->find_neighbors(local_span, resident_span);
      for (unsigned int sub = 0; sub < parameters->solve_step_count(); sub++) {
        particles->compute_densities(resident_span);
        particles->compute_pressure_lambdas(resident_span);
        particles->compute_pressure_dps(resident_span, sub);
        particles->update_position_stars(resident_span);
      }
      particles->update_velocities(local_span);
      particles->apply_surface_tension(local_span, resident_span);
      particles->apply_viscosity(resident_span);
      particles->compute_vorticity(resident_span);
      particles->apply_vorticity(resident_span);
      particles->apply_viscosity(resident_span);
      particles->update_positions(resident_span);
    }
    const pbf_stats_t st = particles->stats();
    std::printf("particles %zu steps %d mean_density_error %.6g max_density_error %.6g kinetic_energy %.9g "
                "com %.7g %.7g %.7g mean_neighbors %.4f flags %u\n",
                n, steps, st.mean_density_error, st.max_density_error, st.kinetic_energy, st.center_of_mass[0],
                st.center_of_mass[1], st.center_of_mass[2], st.mean_neighbors, st.error_flags);
    if (save) particles->save(save);
    if (dump) {
      particles->download(x.data(), v.data());
      FILE* f = std::fopen(dump, "wb");
      if (!f) throw std::runtime_error("cannot open dump file");
      const uint64_t nn = n;
      std::fwrite(&nn, sizeof(nn), 1, f);
      std::fwrite(x.data(), sizeof(float), 3 * n, f);
      std::fwrite(v.data(), sizeof(float), 3 * n, f);
      std::fclose(f);
    }
    delete particles;
    delete parameters;
  } catch (std::exception const& exception) {
    std::printf("Aborting: %s\n", exception.what());
    return 1;
  }
  return 0;
}
