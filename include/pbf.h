/*
 * pbf.h — C ABI of the B200 position-based-fluids (PBF) step.
 *
 * Drop-in for the per-stage call surface of the reference's
 * sim::Particles<float,3> (Simulation/Source/particles.h:256-487), which the
 * reference reaches through sim::algorithms (Common/sim_algorithms.h:38-260).
 * A generic lambda-taking template cannot cross a C ABI, so the boundary keeps
 * the *stage* surface: one exported function per Particles stage, plus a fused,
 * CUDA-graph-captured whole step.  include/pbf_particles.hpp wraps this in a
 * C++ class with the reference's method names.
 *
 * Conventions
 *  - Every function returns 0 on success or a negative PBF_ERR_* code; the
 *    message is available from pbf_last_error(ctx).  No C++ exception crosses
 *    the ABI (the reference throws std::runtime_error, array.h:128-129; the
 *    C++ facade turns a nonzero status back into std::runtime_error).
 *  - Host arrays are the reference's Vec<float,3> layout: 12-byte AoS float[3]
 *    (Common/vec.h:184-192), indexed by the reference's particle index.
 *  - Work is stream-ordered on the context's own CUDA stream; functions that
 *    return host data synchronise that stream.  One context per host thread;
 *    a context is not re-entrant.
 *  - Spans: the reference's IndexSpan arguments, [b, e) over reference
 *    indices.  A single rank passes [0, N).  A multi-rank driver (the x-slab
 *    decomposition, Simulation/Source/main.adios) passes [0, R) for its R
 *    resident particles, the first R reference indices; the others are halo
 *    particles: the stage reads them as neighbours and leaves them as they
 *    are.  find_neighbors bins every held particle (its bin span must be
 *    [0, N)) and fills lists for its fill span only (the others get empty
 *    lists).  Spans not starting at 0 or ending past N return PBF_ERR_SPAN.
 *    The fused pbf_step always covers every particle.
 *  - Device memory is owned by the context (allocated once in pbf_create,
 *    sized by capacity); the caller keeps ownership of its host arrays.
 */
#ifndef PBF_B200_H
#define PBF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PBF_OK 0
#define PBF_ERR_ARG -1        /* bad argument (null pointer, size) */
#define PBF_ERR_CUDA -2       /* CUDA runtime error */
#define PBF_ERR_CAPACITY -3   /* n > capacity (reference: array.h:128-129) */
#define PBF_ERR_SPAN -4       /* span not [0, e) with e <= N */
#define PBF_ERR_PARAMS -5     /* parameters outside what the reference grid supports */
#define PBF_ERR_STATE -6      /* call out of order (e.g. no neighbor lists yet) */
#define PBF_ERR_DEVICE -7     /* device-side check tripped (see pbf_stats_t.error_flags) */
#define PBF_ERR_IO -8         /* INI or state file unreadable, or a short write */

/* Device-side error flag bits (pbf_stats_t.error_flags). */
#define PBF_FLAG_KEY_RANGE 1u     /* a bin id fell outside the grid; clamped */
#define PBF_FLAG_NONFINITE 2u     /* a non-finite position was hashed */
#define PBF_FLAG_WAIT_TIMEOUT 4u  /* a kernel gave up a bounded wait (tensor cores, persistent step); that launch's results are invalid */

/*
 * Parameter block.  Field meaning follows the reference's public
 * Parameters<float,3> fields (Common/parameters.h:550-573); pbf_params_derive
 * fills the derived ones the way Parameters::derive_from_input does
 * (parameters.h:123-148).
 */
typedef struct pbf_params {
  float time_step;            /* dt                                   (parameters.h:564) */
  float gravity;              /* g, applied to v.y                    (particles.h:268)  */
  float gamma;                /* surface tension; 0 = stage is a no-op (particles.h:400-431) */
  float visc_c;               /* XSPH coefficient                     (particles.h:445)  */
  float lambda_epsilon;       /* constraint-force-mixing epsilon      (particles.h:340)  */
  float vorticity_coef;       /* vorticity confinement epsilon        (particles.h:484)  */
  float smoothing_radius;     /* h                                    (parameters.h:555) */
  float neighbor_bin_spacing; /* s, grid cell edge and list radius    (neighbors.h:198)  */
  float rest_density;         /* rho0                                 (parameters.h:557) */
  float rest_mass;            /* m                                    (parameters.h:558) */
  float max_speed;            /* 0.5*h*K/dt, velocity clamp scale     (parameters.h:145) */
  float particle_rest_spacing;/* lattice spacing                      (parameters.h:553) */
  float boundary_min[3];      /* wall clamp box                       (particles.h:525)  */
  float boundary_max[3];
  float mover_center[3];      /* mover sphere centre                  (particles.h:517)  */
  float mover_radius;         /* 0.2 in the reference                 (particles.h:515)  */
  int32_t solve_steps;        /* K Jacobi iterations                  (main.cpp:82)      */
  int32_t neighbor_cap;       /* 60 in the reference (MAX_NEIGHBORS, neighbors.h:39); <= 64 */
  /* Artificial-pressure term s_corr = -k (W(r)/W(dq))^n (Macklin & Mueller
   * 2013).  Not in the reference (particles.h:348-358 has none): k = 0 keeps
   * reference parity. */
  float scorr_k;
  float scorr_n;
  float scorr_dq;             /* as a fraction of h */
  /* 1: every kernel evaluates in the reference's operation order with
   * IEEE-rounded add/mul/div/sqrt and no FMA (bit-identical to the reference's
   * CPU build on the same inputs); 0: fast math in the physics gathers
   * (reciprocals, FMA), results within the 1e-5 parity tolerance.  The
   * neighbor search, predict and boundary clamp are always exact. */
  int32_t exact_math;
  /* Solver: 0 = the reference's K plain Jacobi iterations; 1 = learned warm
   * start: iteration 1 takes lambda from the per-particle MLP (pbf_mlp_*),
   * then plain iterations run while the mean clamped density error exceeds
   * residual_tol, at most max_iterations in all (fast math only).  With
   * residual_tol <= 0 the count is fixed: exactly max_iterations, the
   * network's and max_iterations - 1 plain ones, with no residual checks. */
  int32_t solver;
  float residual_tol;
  int32_t max_iterations;
  /* Learned solver's residual checks: 1 (or less) = the mean over every
   * particle, each check the next iteration's density/lambda pass as well;
   * S > 1 = the mean over every S-th run of 32 consecutive sorted slots (an
   * estimate from a spatially spread sample), and the full density/lambda
   * pass runs only when another iteration follows. */
  int32_t residual_sample;
} pbf_params;

/* Physics statistics of the current state (a residual density pass over the
 * current positions with the current neighbor lists; no state is modified). */
typedef struct pbf_stats_t {
  uint64_t n;
  double mean_density_error;  /* mean_i max(rho_i/rho0 - 1, 0) (clamped constraint, particles.h:325) */
  double max_density_error;   /* max_i  max(rho_i/rho0 - 1, 0) */
  double kinetic_energy;      /* sum_i 0.5 m |v_i|^2 */
  double center_of_mass[3];   /* mean_i x_i */
  double mean_neighbors;      /* mean list length */
  uint64_t cap_hits;          /* particles whose list is at the cap */
  uint32_t error_flags;       /* PBF_FLAG_* bits raised since the last pbf_stats */
  uint32_t solver_iterations; /* Jacobi iterations the last step ran */
  double solver_residual;     /* learned solver: mean clamped density error at its last check */
  uint32_t tiles;             /* 32-particle tiles of the last list fill that wrote staging (0: none) */
  uint32_t tiles_staged;      /* of those, the tiles the staged gathers read from shared memory */
  uint32_t lists_slot_order;  /* fast math: 1 if the last list fill walked the bins in slot order (few lists
                                 at the cap), 0 if in the reference's order */
} pbf_stats_t;

typedef struct pbf_ctx pbf_ctx;

/* ---- parameters and scene construction (host only, no GPU needed) ---- */

/* Reference defaults for the keys the INI may omit: mover radius 0.2,
 * neighbor cap 60, rest mass 1, s_corr off; everything else -1 as the
 * reference's read_INI leaves an absent key (parameters.h:96-118). */
void pbf_params_init(pbf_params* p);

/* Derive spacing-dependent fields as Parameters::derive_from_input does
 * (parameters.h:123-148): h = 1.8*spacing if h <= 0, s = 1.2*h if s <= 0,
 * m = 1, rho0 = m/spacing^3 (unless rest_density_override > 0),
 * max_speed = 0.5*h*K/dt. */
int pbf_params_derive(pbf_params* p, float rest_spacing, float rest_density_override);

/* Read the reference's INI schema (parameters.h:92-119) into p and the
 * initial-fluid box; derives as above.  fluid_min/fluid_max may be NULL. */
int pbf_params_from_ini(const char* path, pbf_params* p, float fluid_min[3], float fluid_max[3]);

/* Lattice counts per axis = floor(extent/spacing) (aabb.h:213-219). */
int pbf_lattice_dims(const float fluid_min[3], const float fluid_max[3], float spacing,
                     int64_t dims_out[3]);

/* construct_fluid (particles.h:231-250): z outer, x inner,
 * x = (idx*spacing + min) + spacing/2, then a seeded jitter, uniform in
 * [-amp, +amp) per axis, from SplitMix64 over (seed, 3*index + axis).
 * x_out holds dims[0]*dims[1]*dims[2] AoS float3 entries. */
int pbf_build_lattice(const float fluid_min[3], const int64_t dims[3], float spacing,
                      float jitter_amp, uint64_t seed, float* x_out);

/* Density of the centre particle of an unjittered spacing-lattice of
 * (2r+1)^3 particles, computed with the reference's Poly6 sum
 * (particles.h:292-313) in its neighbor-list order: the "rest density from an
 * interior lattice particle" convention.  Host computation. */
int pbf_lattice_rest_density(const pbf_params* p, float spacing, float* rho0_out);

/* Grid dimensions the reference builds for p (neighbors.h:69-71). */
int pbf_grid_dims(const pbf_params* p, int64_t dims_out[3]);

/* ---- context ---- */

/* Allocates every device buffer for up to `capacity` particles on the current
 * CUDA device and validates p against the reference grid (box min >= 0 and
 * all hashed bins in range). */
int pbf_create(const pbf_params* p, size_t capacity, pbf_ctx** out);
void pbf_destroy(pbf_ctx* ctx);
const char* pbf_last_error(const pbf_ctx* ctx);
/* Message of the last pbf_create failure (no context exists then). */
const char* pbf_create_error(void);

/* Replace the parameters (same capacity; grid must not grow). */
int pbf_set_params(pbf_ctx* ctx, const pbf_params* p);
int pbf_get_params(const pbf_ctx* ctx, pbf_params* p);

/* Host AoS float3 state in; x* = x (particles.h:184-199).  v may be NULL (zero).
 * Fast math: also starts the list-order choice afresh (slot order first), so
 * steps from an uploaded state do not depend on what the context ran before. */
int pbf_upload(pbf_ctx* ctx, const float* x_aos, const float* v_aos, size_t n);
/* Download in the reference's particle order; any pointer may be NULL. */
int pbf_download(pbf_ctx* ctx, float* x_aos, float* v_aos, float* rho, float* lambda);
size_t pbf_count(const pbf_ctx* ctx);

/* Per-array access in the reference's particle order (parity and tests). */
#define PBF_ARRAY_POSITIONS 0
#define PBF_ARRAY_POSITION_STARS 1
#define PBF_ARRAY_VELOCITIES 2
#define PBF_ARRAY_SCRATCH 3      /* Vec scratch: dp, vorticity or color field */
#define PBF_ARRAY_DENSITIES 4    /* scalar */
#define PBF_ARRAY_LAMBDAS 5      /* scalar */
int pbf_get_array(pbf_ctx* ctx, int which, float* host_out);
int pbf_set_array(pbf_ctx* ctx, int which, const float* host_in);

/* ---- stages: one per sim::Particles method, same span semantics ---- */
int pbf_apply_external_forces(pbf_ctx* ctx, size_t b, size_t e);      /* particles.h:263-270 */
int pbf_predict_positions(pbf_ctx* ctx, size_t b, size_t e);          /* particles.h:275-287 */
int pbf_find_neighbors(pbf_ctx* ctx, size_t bin_b, size_t bin_e,
                       size_t fill_b, size_t fill_e);                  /* particles.h:256-258 */
int pbf_compute_densities(pbf_ctx* ctx, size_t b, size_t e);          /* particles.h:292-313 */
int pbf_compute_pressure_lambdas(pbf_ctx* ctx, size_t b, size_t e);   /* particles.h:318-342 */
int pbf_compute_pressure_dps(pbf_ctx* ctx, size_t b, size_t e, int substep); /* 348-358 */
int pbf_update_position_stars(pbf_ctx* ctx, size_t b, size_t e);      /* particles.h:363-370 */
int pbf_update_velocities(pbf_ctx* ctx, size_t b, size_t e);          /* particles.h:375-385 */
int pbf_apply_surface_tension(pbf_ctx* ctx, size_t color_b, size_t color_e,
                              size_t st_b, size_t st_e);               /* particles.h:400-431 */
int pbf_apply_viscosity(pbf_ctx* ctx, size_t b, size_t e);            /* particles.h:436-447 */
int pbf_compute_vorticity(pbf_ctx* ctx, size_t b, size_t e);          /* particles.h:452-466 */
int pbf_apply_vorticity(pbf_ctx* ctx, size_t b, size_t e);            /* particles.h:471-487 */
int pbf_update_positions(pbf_ctx* ctx, size_t b, size_t e);           /* particles.h:390-394 */

/* The whole step of Simulation/Source/main.cpp:71-124 (single rank), fused
 * and captured once as a CUDA graph per nsteps, then replayed. */
int pbf_step(pbf_ctx* ctx, int nsteps);

/* Parity exports in the reference's index space (synchronous):
 *  idx   [N][cap] neighbor indices, entries past count set to -1 (neighbors.h:41-44)
 *  count [N]
 *  sorted_ids [N]   particle ids in sorted-bin order (neighbors.h:130-132)
 *  sorted_keys [N]  bin id of each sorted entry
 *  bin_begin/bin_end [B]  lower/upper bound of every bin (neighbors.h:137-148)
 * Any pointer may be NULL.  idx is in the reference's order (x offset outer)
 * whatever order the fast fill walked in (pbf_stats_t.lists_slot_order). */
int pbf_get_neighbors(pbf_ctx* ctx, int32_t* idx, int32_t* count);
int pbf_get_bins(pbf_ctx* ctx, uint32_t* sorted_keys, uint32_t* sorted_ids,
                 uint32_t* bin_begin, uint32_t* bin_end);
int64_t pbf_num_bins(const pbf_ctx* ctx);

int pbf_stats(pbf_ctx* ctx, pbf_stats_t* out);

/* Device synchronisation of the context stream. */
int pbf_sync(pbf_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or CUDA events after the context's kernels. */
int pbf_get_stream(pbf_ctx* ctx, void** stream_out);

/* ---- instrumentation ---- */
/* Per-kernel device time: with timing on, pbf_step launches the step's
 * kernels one by one (no graph) and records a CUDA event around each.
 * pbf_kernel_times returns, per kernel family, launches and total ms since
 * the last reset.  names[i] points to static strings. */
int pbf_set_timing(pbf_ctx* ctx, int on);
int pbf_kernel_times(pbf_ctx* ctx, int max_kinds, const char** names, int64_t* launches,
                     double* total_ms, int* n_kinds);
int pbf_reset_timing(pbf_ctx* ctx);
/* Number of kernel launches one pbf_step(ctx, 1) issues. */
int pbf_launches_per_step(pbf_ctx* ctx, int64_t* out);

/* ---- growing the particle set (the emitter) ----
 * pbf_add_particles replaces Particles::add (particles.h:184-199) for k host
 * particles (AoS xyz; v may be NULL for zero velocity): they get the next
 * reference indices n .. n+k-1, x* = x.  PBF_ERR_CAPACITY past the capacity
 * (the reference throws), PBF_ERR_STATE on a batch of scenes.
 * pbf_construct_fluid replaces Particles::construct_fluid (particles.h:231-250):
 * the lattice of the box at particle_rest_spacing, z outer / x inner, point =
 * index*spacing + min + spacing/2, all with `velocity` (NULL: zero); *added =
 * the count.  The reference's emitter (distributor.h:357-369) is this call on
 * the box of extent 1.1*spacing centred at the emitter, once per step while
 * it is active.  A changed count drops the captured step graphs. */
int pbf_add_particles(pbf_ctx* ctx, const float* x, const float* v, size_t k);
int pbf_construct_fluid(pbf_ctx* ctx, const float fluid_min[3], const float fluid_max[3],
                        const float velocity[3], size_t* added);
/* Steps advanced by pbf_step on this context (restored by pbf_load_state). */
uint64_t pbf_step_count(const pbf_ctx* ctx);

/* ---- state files: output frames and checkpoints ----
 * No counterpart in the reference (its output path is the renderer sync and
 * ADIOS, distributor.h:742-750, adios_writer.h; it has no checkpoint).  One
 * little-endian file: a 104-byte header
 *   char magic[8] = "PBFSTATE"; uint32 version = 1; uint32 sizeof(pbf_params);
 *   uint64 n; uint64 steps; uint32 flags (bit 0: network present); uint32 0;
 *   pbf_tuning (3 x 5 int32); uint32 0
 * then the pbf_params block, then in the reference's particle order
 *   float x[n][3], v[n][3], density[n], lambda[n], lambda_history[n]
 * (lambda_history: the lambda the learned solver applied in the last step),
 * then, with flag bit 0, float network[PBF_MLP_PARAMS], norm[PBF_MLP_NORM].
 * pbf_load_state restores parameters, launch shapes, particles and network
 * into a context with room for them; the steps that follow are bit-identical
 * to those the saved context would have taken. */
int pbf_save_state(pbf_ctx* ctx, const char* path);
int pbf_load_state(pbf_ctx* ctx, const char* path);

/* ---- batched scenes ----
 * No counterpart in the reference (one scene per process there).  One context
 * advances `nscenes` independent scenes in the same launches: each scene has
 * its own box (boundary_min/max, with the single-scene rules: min >= 0, the
 * grid must cover the box) and its own bin grid; all share the physics of the
 * parameter block, whose boundary fields are ignored.  Particles are
 * uploaded, downloaded and indexed as the scenes concatenated in order (scene
 * i holds particles [sum of the counts before i, + count_i)); pbf_upload takes
 * exactly the sum of the counts.  The bin keys of scene i follow those of
 * scenes 0..i-1, so sorted keys and bin bounds (pbf_get_bins) are in that
 * global key space.  A scene's bins, lists and particle arithmetic are those
 * of a context created for it alone with the same launch shapes.  The learned
 * solver's residual check is the batch's mean.  pbf_set_params keeps the
 * scenes' boxes. */
typedef struct {
  float boundary_min[3];
  float boundary_max[3];
  size_t count;  /* particles of the scene */
} pbf_scene;
int pbf_create_batch(const pbf_params* p, const pbf_scene* scenes, int nscenes, pbf_ctx** out);
/* Scenes of a batch context; 0 for a single-scene context. */
int pbf_scene_count(const pbf_ctx* ctx);
/* pbf_stats over one scene's particles (scene 0 of a single-scene context is
 * the whole set); the error flags are reported, not cleared. */
int pbf_scene_stats(pbf_ctx* ctx, int scene, pbf_stats_t* out);

/* ---- launch shapes of the fast-math gather kernels ----
 * No counterpart in the reference (its loops are OpenMP for_each_index).
 * Each family of gather kernels runs with `lanes` threads per particle
 * walking one neighbor list together (2, 4 or 8) in blocks of `block` threads
 * (128 or 256), either reading the neighbours' records from global memory or,
 * `staged` (4 lanes, 128 threads only), from shared memory: each block copies
 * the neighbour bins of its 32-particle tile there first and walks 16-bit
 * lists of staging indices the list fill writes beside the int32 lists.  The
 * shape changes only the order of floating-point sums inside a particle (fast
 * math), never the lists; exact_math kernels run one thread per particle and
 * ignore it.  Default: 2 lanes x 128 threads for density/lambda and delta-p,
 * 2 x 256 for XSPH and vorticity apply, 4 x 256 for vorticity (the autotuner's
 * choice on the 1M dam), not staged. */
enum {
  PBF_TUNE_DENSITY = 0,          /* density + lambda, and the learned solver's residual check */
  PBF_TUNE_DELTA_P = 1,          /* position delta + x* update */
  PBF_TUNE_VISCOSITY = 2,        /* both XSPH passes */
  PBF_TUNE_VORTICITY = 3,
  PBF_TUNE_APPLY_VORTICITY = 4,
  PBF_TUNE_FAMILIES = 5
};
#define PBF_TUNE_CANDIDATES 7  /* (lanes, block, staged) = (4,128,0) (4,256,0) (8,128,0) (8,256,0) (2,128,0) (2,256,0) (4,128,1) */
typedef struct {
  int lanes[PBF_TUNE_FAMILIES];
  int block[PBF_TUNE_FAMILIES];
  int staged[PBF_TUNE_FAMILIES];
} pbf_tuning;
int pbf_get_tuning(const pbf_ctx* ctx, pbf_tuning* out);
/* PBF_ERR_ARG for a shape outside the candidates; drops captured graphs. */
int pbf_set_tuning(pbf_ctx* ctx, const pbf_tuning* t);
/* Autotuner: from the current particle state, runs `steps` (>= 1) timed
 * steps per candidate shape after one untimed step, restoring the state before
 * each candidate and at the end; applies and returns (chosen, may be NULL) the
 * fastest shape of each family.  ms (may be NULL) receives
 * [PBF_TUNE_CANDIDATES][PBF_TUNE_FAMILIES] device ms per step.  The particle
 * state (positions, velocities, the learned solver's lambda history) is left
 * as found; neighbor lists and statistics need a new step.  Kernel timing
 * totals are reset. */
int pbf_autotune(pbf_ctx* ctx, int steps, pbf_tuning* chosen, double* ms);

/* ---- learned warm start: the per-particle MLP ----
 * 12 -> 64 -> 64 -> 1, GELU, BF16 tensor-core GEMMs with FP32 accumulation.
 * Parameters are fp32 masters in the order W1[64][12], b1[64], W2[64][64],
 * b2[64], w3[64], b3 (PBF_MLP_PARAMS floats); the normalisation block is
 * mean[12], inv_std[12], label_scale (PBF_MLP_NORM floats).  Features of a
 * particle at the first Jacobi iteration (raw, before normalisation):
 *   0 neighbours/64   1 C = max(rho/rho0-1, 0)   2 rho/rho0 - 1
 *   3 S = sum|grad C_j|^2 + |grad C_i|^2         4 plain lambda -C/(S+eps)
 *   5 lambda the particle received in the previous step
 *   6 |grad C_i|^2 / S   7 share of neighbours closer than h
 *   8 v_y dt/h   9 |v| dt/h   10 height above the floor / h (<= 4)
 *   11 distance to the nearest wall / h (<= 4)
 * The label is the sum of the lambdas the plain solver applies over its K
 * iterations; the network predicts label/label_scale. */
#define PBF_MLP_FEATURES 12
#define PBF_MLP_PARAMS 5057
#define PBF_MLP_NORM 25
int pbf_mlp_init(pbf_ctx* ctx, uint64_t seed);
int pbf_mlp_get(pbf_ctx* ctx, float* params, float* norm);
int pbf_mlp_set(pbf_ctx* ctx, const float* params, const float* norm);
/* With recording on, fused plain steps keep the last step's features and
 * labels on the device; pbf_get_training_data copies them out (slot order). */
int pbf_set_recording(pbf_ctx* ctx, int on);
int pbf_get_training_data(pbf_ctx* ctx, float* features, float* labels);
/* adam_steps Adam updates (beta 0.9/0.999, eps 1e-8) on batches of `batch`
 * samples drawn from the recorded step with a counter-based RNG; the mean
 * squared error of the last batch is returned in *loss. */
int pbf_mlp_train(pbf_ctx* ctx, int adam_steps, int batch, float lr, uint64_t seed, float* loss);
/* Gradient of the mean squared error over n host samples (normalised
 * features, targets in network units) with the current parameters. */
int pbf_mlp_gradients(pbf_ctx* ctx, const float* features, const float* targets, size_t n, float* grad,
                      float* loss);
/* Network output for n host samples of normalised features. */
int pbf_mlp_predict(pbf_ctx* ctx, const float* features, size_t n, float* y);
/* Self-test of the network kernel's failure path; no counterpart in the
 * reference.  One 128-row tile is launched with its tensor-core MMAs and
 * their completion signal left out, so every bounded wait of the kernel on
 * that signal gives up.  The kernel then raises PBF_FLAG_WAIT_TIMEOUT in
 * *flags (its own status word, not the context's error flags), frees its
 * tensor memory and returns; the context stays usable.  Needs a network
 * (pbf_mlp_init or pbf_mlp_set) and a capacity of at least 278 particles. */
int pbf_selftest_mlp_wait_timeout(pbf_ctx* ctx, uint32_t* flags);

/* ---- persistent step (batches of scenes) ----
 * No counterpart in the reference.  With enable = 1, each step of a batch
 * context (pbf_create_batch) runs all its gather passes (the K Jacobi
 * iterations of density/lambda and delta-p, both XSPH passes, vorticity and
 * its application) as ONE persistent launch after the list fill, instead of
 * one launch per pass: blocks take (pass, tile) tasks from a queue, and a tile
 * waits only until the previous pass has finished in the scenes it covers, so
 * each scene goes through the passes at its own pace within the step.  The
 * gathers run at fixed shapes (2 lanes per particle, 4 for vorticity, 128
 * threads); the results are those of the launch-per-pass step at the same
 * shapes, bit for bit.  Every wait is bounded (2 s); a launch that gives one
 * up raises PBF_FLAG_WAIT_TIMEOUT (pbf_stats) and its step's results are
 * invalid.  Applies to fast math, the plain solver with 1..16 iterations, no
 * surface tension and no s_corr: PBF_ERR_PARAMS otherwise, PBF_ERR_STATE on a
 * one-scene context; a later pbf_set_params outside these runs the
 * launch-per-pass step until it is back inside.  enable = 0 turns it off.
 * Drops captured graphs. */
int pbf_set_persistent(pbf_ctx* ctx, int enable);
/* Self-test of the persistent step's failure path; no counterpart in the
 * reference.  Runs the persistent kernel's scheduler alone (no particle data
 * is read or written) on two 4-tile passes whose dependency is never met,
 * with a 2 ms bound: every waiting block gives up, raises
 * PBF_FLAG_WAIT_TIMEOUT in *flags (its own status word, not the context's
 * error flags) and returns; the context stays usable. */
int pbf_selftest_persistent_wait_timeout(pbf_ctx* ctx, uint32_t* flags);

/* ---- scene groups ----
 * No counterpart in the reference.  Independent contexts (one scene each)
 * advanced together by ONE graph launch: the graph holds every member's
 * nsteps-step chain as a child graph, with no dependency between members, so
 * each scene advances at its own pace.  Each member's results are its own
 * pbf_step results, bit for bit.  The launch runs on the group's stream,
 * after each member's pending work; each member's later work waits for it.
 * Members must have per-kernel timing off; the graph is cached per nsteps and
 * rebuilt when a member's particle count or parameters change.  Members stay
 * owned by the caller and must outlive the group. */
typedef struct pbf_group pbf_group;
int pbf_group_create(pbf_ctx* const* ctxs, int n, pbf_group** out);
int pbf_group_step(pbf_group* g, int nsteps);
int pbf_group_sync(pbf_group* g);
int pbf_group_get_stream(pbf_group* g, void** stream_out);
void pbf_group_destroy(pbf_group* g);

/* ---- neighbor search that allocates nothing ----
 * No counterpart in the reference.  For callers that may not allocate device
 * memory: hosts that own every device allocation (their own pool or a fixed
 * budget) and callers that cannot afford the device-wide synchronisation of
 * cudaMalloc/cudaFree.  Builds the reference's neighbor lists (the same lists
 * as pbf_find_neighbors + pbf_get_neighbors) for a caller-owned device point
 * set, using only a file-scope device array of PBF_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until the process exits.  The sort is
 * the regular path's stable radix sort (linear in n however the points crowd
 * into bins) and crowded bins are walked run by run over bit-identical
 * positions, so no input makes the search quadratic in a bin's population
 * beyond the distance tests the reference itself makes.
 *   d_x     device, n x 3 floats (AoS), the positions to bin
 *   d_nbr   device, n x neighbor_cap int32: reference indices, -1 past the count
 *   d_cnt   device, n int32 counts
 *   d_flags device, one uint32 (may be NULL: nothing reported): receives the
 *           call's PBF_FLAG_* bits, PBF_FLAG_KEY_RANGE when a position is
 *           non-finite or outside the bin grid (its bins are clamped into the
 *           grid, as the regular path does, and the lists are not the
 *           reference's for such input)
 *   stream  a cudaStream_t (NULL: the legacy default stream); the work is
 *           enqueued there and the call returns without synchronising, so
 *           read *d_flags after the stream has reached it.
 * Limits: n <= PBF_NOALLOC_MAX_PARTICLES and a grid of at most
 * PBF_NOALLOC_MAX_BINS bins; larger inputs return PBF_ERR_CAPACITY with the
 * message in pbf_last_error(NULL).  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture.  Every call reuses the same array: calls that overlap
 * on the GPU (other streams, other host threads) race — serialise them. */
#define PBF_NOALLOC_MAX_PARTICLES 65536
#define PBF_NOALLOC_MAX_BINS 262144
#define PBF_NOALLOC_SCRATCH_BYTES 5506560
int pbf_find_neighbors_noalloc(const pbf_params* p, const float* d_x, size_t n, int32_t* d_nbr,
                               int32_t* d_cnt, uint32_t* d_flags, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PBF_B200_H */
