/*
 * ommb200 -- C ABI of the B200-native force and integration engine for the openmm-rs hot
 * path: NonbondedForce (PME, LJ with cutoff and switching, no-cutoff), GBSAOBCForce,
 * HarmonicBond/AngleForce and LangevinMiddleIntegrator with SETTLE, driven through a
 * Context with step / getState.
 *
 * Every entry point returns an int status (OMMB200_OK or a negative OMMB200_ERR_* code) and
 * never aborts; ommb200_last_error() gives the message of the calling thread's last failure.
 * Handles are opaque; a Context takes ownership of the System and Integrator passed to it
 * (as openmm-core's Context::new moves them in, context.rs:83-87) and a System takes
 * ownership of each Force added to it (system.rs:201-204).  Host arrays are copied in/out.
 * A Context is not thread-safe; use one per host thread.  All reference citations are
 * relative to mogura-rs/openmm-rs/crates/openmm-core/src.
 */
#ifndef OMMB200_H
#define OMMB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (constraints.rs:12-21 ConstraintError; asserts become INVALID_ARG) ---- */
#define OMMB200_OK 0
#define OMMB200_ERR_INVALID_ARG (-1)
#define OMMB200_ERR_CONSTRAINT (-2)
#define OMMB200_ERR_NONFINITE (-3)
#define OMMB200_ERR_NLIST_OVERFLOW (-4)
#define OMMB200_ERR_TIMEOUT (-5)
#define OMMB200_ERR_CUDA (-6)
#define OMMB200_ERR_UNSUPPORTED (-7)
#define OMMB200_ERR_OUT_OF_MEMORY (-8)

/* NonbondedMethod (forces/nonbonded.rs:19-33) */
#define OMMB200_NO_CUTOFF 0
#define OMMB200_CUTOFF_NON_PERIODIC 1
#define OMMB200_CUTOFF_PERIODIC 2
#define OMMB200_EWALD 3 /* accepted by the setter, rejected at Context creation */
#define OMMB200_PME 4
#define OMMB200_LJPME 5 /* accepted by the setter, rejected at Context creation */

/* GBSAOBCMethod (forces/gbsa_obc.rs:11-17) */
#define OMMB200_GBSA_NO_CUTOFF 0
#define OMMB200_GBSA_CUTOFF_NON_PERIODIC 1
#define OMMB200_GBSA_CUTOFF_PERIODIC 2

/* arithmetic of the force kernels */
#define OMMB200_PRECISION_MIXED 0  /* FP32 pair/spline math, 64-bit fixed-point accumulation */
#define OMMB200_PRECISION_DOUBLE 1 /* the same kernels entirely in FP64 */

/* getState flags (state.rs:7-14) plus the virial, which the reference lacks */
#define OMMB200_STATE_POSITIONS 1
#define OMMB200_STATE_VELOCITIES 2
#define OMMB200_STATE_FORCES 4
#define OMMB200_STATE_ENERGY 8
#define OMMB200_STATE_VIRIAL 16

typedef struct ommb200_system ommb200_system;
typedef struct ommb200_force ommb200_force;
typedef struct ommb200_integrator ommb200_integrator;
typedef struct ommb200_context ommb200_context;

typedef struct {
  int precision;              /* OMMB200_PRECISION_* (default MIXED) */
  int device;                 /* CUDA device ordinal (default 0) */
  int use_cuda_graph;         /* capture the step in a CUDA graph (default 1) */
  double neighbor_skin;       /* Verlet skin in nm; <= 0 picks the tuned default */
  int steps_per_graph;        /* steps captured per graph launch; <= 0 picks the default */
  int pme_bricks;             /* brick-owned PME gather (rectangular periodic boxes):
                                 -1 when the grid has two bricks per SM or more (default), 0 never,
                                 1 whenever the box allows; the forces are the same either way */
  double prune_margin;        /* nm, pruned pair list between rebuilds (periodic rectangular
                                 boxes): entries beyond cutoff + margin of their half block are
                                 dropped until a particle moves margin / 2; 0 = off; < 0 picks
                                 the default (off; ommb200_context_autotune may turn it on) */
  int pair_cull;              /* mixed precision, periodic rectangular boxes without a pruned
                                 list: the pair kernel drops, at every evaluation, the entries
                                 beyond the cutoff of their half block's current bounding box
                                 and packs the rest into full rounds; a warp takes runs of this
                                 many tiles of one block.  0 = off (every listed entry is
                                 evaluated); < 0 picks by size (64 when the list gives each
                                 resident warp about 40 tiles or more, else off;
                                 ommb200_context_autotune may change it); at most 64.  The pair
                                 set is the same either way */
} ommb200_options;

typedef struct {
  double time;                /* ps */
  int64_t step_count;
  double potential_energy;    /* kJ/mol, valid if OMMB200_STATE_ENERGY was requested */
  double kinetic_energy;      /* kJ/mol (context.rs:1107-1163, LFMiddle offset 0) */
  double box[9];              /* periodic box rows a, b, c in nm */
  double virial[9];           /* -dU/d(strain), kJ/mol, if OMMB200_STATE_VIRIAL */
} ommb200_state_info;

/* ---- library ---- */
const char* ommb200_last_error(void);
const char* ommb200_version(void);
void ommb200_default_options(ommb200_options* out);

/* ---- System (system.rs:43-233) ---- */
int ommb200_system_create(ommb200_system** out);                       /* System::new */
int ommb200_system_destroy(ommb200_system* system);
int ommb200_system_add_particle(ommb200_system* s, double mass, int* index); /* system.rs:64-72 */
int ommb200_system_num_particles(const ommb200_system* s, int* out);
int ommb200_system_add_constraint(ommb200_system* s, int p1, int p2, double distance,
                                  int* index);                          /* add_constraint */
int ommb200_system_set_default_periodic_box_vectors(ommb200_system* s, const double a[3],
                                                    const double b[3], const double c[3]);
int ommb200_system_add_force(ommb200_system* s, ommb200_force* force, int* index); /* add_force */

/* ---- forces: common (forces/mod.rs:142-246 force_group / name) ---- */
int ommb200_force_destroy(ommb200_force* force); /* only for forces not added to a System */
int ommb200_force_set_group(ommb200_force* force, int group);
int ommb200_force_get_group(const ommb200_force* force, int* group);

/* ---- NonbondedForce (forces/nonbonded.rs:122-658) ---- */
int ommb200_nonbonded_create(ommb200_force** out);                          /* new, 122-159 */
int ommb200_nonbonded_add_particle(ommb200_force* f, double charge, double sigma,
                                   double epsilon, int* index);             /* 162-173 */
int ommb200_nonbonded_set_particle_parameters(ommb200_force* f, int index, double charge,
                                              double sigma, double epsilon); /* 175-184 */
int ommb200_nonbonded_get_particle_parameters(const ommb200_force* f, int index,
                                              double* charge, double* sigma, double* epsilon);
int ommb200_nonbonded_num_particles(const ommb200_force* f, int* out);
int ommb200_nonbonded_add_exception(ommb200_force* f, int p1, int p2, double charge_prod,
                                    double sigma, double epsilon, int* index); /* 195-214 */
int ommb200_nonbonded_num_exceptions(const ommb200_force* f, int* out);
int ommb200_nonbonded_create_exceptions_from_bonds(ommb200_force* f, int n_bonds,
                                                   const int* bonds /* 2*n_bonds */,
                                                   double coulomb14_scale,
                                                   double lj14_scale); /* 434-500 */
int ommb200_nonbonded_set_method(ommb200_force* f, int method);           /* 502-504 */
int ommb200_nonbonded_set_cutoff_distance(ommb200_force* f, double cutoff); /* 521-528 */
int ommb200_nonbonded_set_reaction_field_dielectric(ommb200_force* f, double eps); /* 534-540 */
int ommb200_nonbonded_set_ewald_error_tolerance(ommb200_force* f, double tol); /* 546-552 */
int ommb200_nonbonded_set_exceptions_use_periodic_boundary_conditions(ommb200_force* f,
                                                                      int periodic); /* 558 */
int ommb200_nonbonded_set_use_dispersion_correction(ommb200_force* f, int enabled); /* 572 */
int ommb200_nonbonded_set_use_switching_function(ommb200_force* f, int enabled);  /* 578 */
int ommb200_nonbonded_set_switching_distance(ommb200_force* f, double distance);  /* 585 */
int ommb200_nonbonded_set_pme_parameters(ommb200_force* f, double alpha, int nx, int ny,
                                         int nz);                              /* 597-611 */
int ommb200_nonbonded_set_reciprocal_space_force_group(ommb200_force* f, int group); /* 111 */
int ommb200_nonbonded_set_include_direct_space(ommb200_force* f, int enabled);      /* 123 */

/* ---- GBSAOBCForce (forces/gbsa_obc.rs:61-133) ---- */
int ommb200_gbsa_obc_create(ommb200_force** out);
int ommb200_gbsa_obc_add_particle(ommb200_force* f, double charge, double radius,
                                  double scaling_factor, int* index);
int ommb200_gbsa_obc_set_particle_parameters(ommb200_force* f, int index, double charge,
                                             double radius, double scaling_factor);
int ommb200_gbsa_obc_set_method(ommb200_force* f, int method);
int ommb200_gbsa_obc_set_cutoff_distance(ommb200_force* f, double cutoff);
int ommb200_gbsa_obc_set_solvent_dielectric(ommb200_force* f, double value);
int ommb200_gbsa_obc_set_solute_dielectric(ommb200_force* f, double value);
int ommb200_gbsa_obc_set_surface_area_energy(ommb200_force* f, double value);

/* ---- HarmonicBondForce (forces/harmonic_bond.rs) / HarmonicAngleForce ---- */
int ommb200_harmonic_bond_create(ommb200_force** out);
int ommb200_harmonic_bond_add_bond(ommb200_force* f, int p1, int p2, double length, double k,
                                   int* index);
int ommb200_harmonic_bond_set_uses_pbc(ommb200_force* f, int use_pbc);
int ommb200_harmonic_angle_create(ommb200_force** out);
int ommb200_harmonic_angle_add_angle(ommb200_force* f, int p1, int p2, int p3, double angle,
                                     double k, int* index);
int ommb200_harmonic_angle_set_uses_pbc(ommb200_force* f, int use_pbc);

/* ---- MonteCarloBarostat (forces/barostat.rs) ----
 * Isotropic Monte Carlo volume moves: every `frequency` steps (counted by the barostat itself,
 * 76-86) the box and the positions (molecule centroids when molecules are scaled as rigid,
 * else every particle) are scaled by (V'/V)^(1/3) with V' - V uniform in +-volume_scale,
 * and the move is accepted by the Metropolis test on dE + P dV - N kT ln(V'/V) with E over
 * the integrator's force groups (context/program.rs:5-47).  Needs a periodic System; not in
 * batches.  The random stream is the engine's own counter-based one (Philox4x32-10 keyed by
 * the seed), not the reference's ChaCha12 sequence. */
int ommb200_monte_carlo_barostat_create(double pressure, double temperature, int frequency,
                                        ommb200_force** out);                   /* new, 63-85 */
int ommb200_monte_carlo_barostat_set_default_pressure(ommb200_force* f, double pressure); /* 90 */
int ommb200_monte_carlo_barostat_get_default_pressure(const ommb200_force* f, double* out);
int ommb200_monte_carlo_barostat_set_default_temperature(ommb200_force* f, double t);   /* 94 */
int ommb200_monte_carlo_barostat_get_default_temperature(const ommb200_force* f, double* out);
/* 98-101: a change reaches the Contexts that already hold this barostat */
int ommb200_monte_carlo_barostat_set_frequency(ommb200_force* f, int frequency);
int ommb200_monte_carlo_barostat_get_frequency(const ommb200_force* f, int* out);
int ommb200_monte_carlo_barostat_set_scale_molecules_as_rigid(ommb200_force* f, int rigid); /* 106 */
int ommb200_monte_carlo_barostat_get_scale_molecules_as_rigid(const ommb200_force* f, int* out);
int ommb200_monte_carlo_barostat_set_random_number_seed(ommb200_force* f, int seed);   /* 112 */
int ommb200_monte_carlo_barostat_get_random_number_seed(const ommb200_force* f, int* out);

/* ---- learned Born radii for GBSAOBCForce (no reference counterpart) ----
 * With learned radii enabled (NoCutoff GBSA only), the O(N^2) descreening passes are replaced
 * by a switched short-range integral (cutoff 2.0 nm, switch from 1.8 nm) plus a network tail
 * predicted from 32 radial symmetry functions per particle (cutoff 1.2 nm).  Every judge_interval MD steps the
 * exact pass runs as judge: that step uses exact radii, the network is trained on the exact
 * radii (train_steps Adam steps, batches of 4,096 particles, lr 1e-3) and it is used for the
 * following steps only if its largest per-particle radius relative error was at most
 * radius_tolerance. */
int ommb200_gbsa_obc_set_learned_radii(ommb200_force* f, int enabled, int judge_interval,
                                       double radius_tolerance, int train_steps);

/* ---- LangevinMiddleIntegrator (integrators/langevin.rs:14-102) ---- */
int ommb200_langevin_middle_create(double temperature, double friction, double step_size,
                                   ommb200_integrator** out);              /* new, 44-67 */
int ommb200_integrator_destroy(ommb200_integrator* integrator); /* if not owned by a Context */
int ommb200_integrator_set_random_number_seed(ommb200_integrator* i, int seed);     /* 33-35 */
int ommb200_integrator_set_constraint_tolerance(ommb200_integrator* i, double tol); /* 73-79 */
int ommb200_integrator_set_temperature(ommb200_integrator* i, double t);            /* 83-89 */
int ommb200_integrator_set_friction(ommb200_integrator* i, double f);              /* 90-96 */
int ommb200_integrator_set_step_size(ommb200_integrator* i, double dt);            /* 97-102 */
int ommb200_integrator_set_integration_force_groups(ommb200_integrator* i, uint32_t groups);

/* ---- Context (context.rs:83-1163) ---- */
/* Context::new (83-161): takes ownership of system and integrator (also on failure). */
int ommb200_context_create(ommb200_system* system, ommb200_integrator* integrator,
                           const ommb200_options* options, ommb200_context** out);
int ommb200_context_destroy(ommb200_context* ctx);
int ommb200_context_num_particles(const ommb200_context* ctx, int* out);
int ommb200_context_set_positions(ommb200_context* ctx, const double* positions, int n); /* 163 */
int ommb200_context_set_velocities(ommb200_context* ctx, const double* velocities, int n);
/* set_velocities_to_temperature (182-223): Maxwell-Boltzmann draw, half-step force offset,
 * velocity constraints at tolerance 1e-5. */
int ommb200_context_set_velocities_to_temperature(ommb200_context* ctx, double temperature,
                                                  int seed);
int ommb200_context_set_periodic_box_vectors(ommb200_context* ctx, const double a[3],
                                             const double b[3], const double c[3]); /* 241 */
int ommb200_context_set_time(ommb200_context* ctx, double time);
int ommb200_context_set_step_count(ommb200_context* ctx, int64_t steps);
int ommb200_context_apply_constraints(ommb200_context* ctx, double tolerance);  /* 767-776 */
int ommb200_context_apply_velocity_constraints(ommb200_context* ctx, double tolerance);
/* try_step (800-805): returns OMMB200_ERR_CONSTRAINT / _NONFINITE on failure. */
int ommb200_context_step(ommb200_context* ctx, int steps);
/* set_parameter / get_parameter (251-268): the global parameters of the System's forces
 * ("MonteCarloPressure" in bar, "MonteCarloTemperature" in K); unknown names are
 * OMMB200_ERR_INVALID_ARG. */
int ommb200_context_set_parameter(ommb200_context* ctx, const char* name, double value);
int ommb200_context_get_parameter(ommb200_context* ctx, const char* name, double* value);
/* Barostat bookkeeping (no reference counterpart): attempted / accepted moves since the
 * Context was created, the current volume step, and the last move: volumes before and after,
 * energy change, Metropolis work and the uniform draw compared with exp(-work/kT) (-1 when
 * the work was not positive). */
typedef struct {
  uint64_t attempted, accepted;
  double volume_scale;
  int last_accepted;
  double last_old_volume, last_new_volume, last_energy_change, last_work, last_uniform;
} ommb200_barostat_stats;
int ommb200_context_get_barostat_stats(ommb200_context* ctx, ommb200_barostat_stats* out);
/* try_get_state_options (1041-1105): any of the output arrays (3*N doubles) may be NULL. */
int ommb200_context_get_state(ommb200_context* ctx, int flags, uint32_t groups,
                              double* positions, double* velocities, double* forces,
                              ommb200_state_info* info);
/* context.rs:689-705 update_nonbonded_force_parameters (nonbonded.rs:721-767): copy the
 * particle and exception parameters of `source` (a NonbondedForce handle the caller keeps)
 * into the Context's NonbondedForce.  Same particle and exception counts, same exception
 * pairs, and no excluded pair may become an interacting one (OMMB200_ERR_INVALID_ARG). */
int ommb200_context_update_nonbonded_parameters(ommb200_context* ctx, const ommb200_force* source);
/* context.rs:680-687 update_gbsa_obc_force_parameters (gbsa_obc.rs:134-141): charges, radii
 * and scale factors of `source` (same particle count). */
int ommb200_context_update_gbsa_obc_parameters(ommb200_context* ctx, const ommb200_force* source);
/* Checkpoints (the reference's set_state, context.rs:274-293, restores positions, velocities,
 * box and time but not the random stream): the complete dynamic state as opaque bytes --
 * positions, velocities, box, time, step count, random-stream counter and seed, neighbour-list
 * reference positions and learned-radii network / optimiser.  Loading it into a Context built
 * from the same System and options continues the trajectory bit for bit. */
int ommb200_context_checkpoint_size(const ommb200_context* ctx, int64_t* bytes);
int ommb200_context_create_checkpoint(ommb200_context* ctx, void* buffer, int64_t bytes);
int ommb200_context_load_checkpoint(ommb200_context* ctx, const void* buffer, int64_t bytes);
/* Autotuner (no reference counterpart): times trial_steps MD steps from the current state
 * for each candidate Verlet skin (which sets the neighbour-list rebuild interval), tile width
 * (rectangular periodic boxes: 16 neighbour entries per half of a 32-particle block, or 32 per
 * block) and pair-kernel grid, keeps the fastest and restores positions, velocities and the
 * random stream, so the trajectory is unchanged.  Outputs may be NULL. */
int ommb200_context_autotune(ommb200_context* ctx, int trial_steps, double* skin,
                             int* pair_ctas_per_sm, double* ms_per_step);
/* The current tuning choices (no reference counterpart); outputs may be NULL. */
int ommb200_context_get_tuning(ommb200_context* ctx, double* skin, int* pair_ctas_per_sm,
                               int* tile_entries);
/* PME parameters frozen at Context creation (nonbonded.rs:1078-1106). */
int ommb200_context_get_pme_parameters(const ommb200_context* ctx, double* alpha, int* nx,
                                       int* ny, int* nz);
/* Which PME gather form runs (no reference counterpart): *bricks_in_use = 1 for the
 * brick-owned form, 0 for the eight-lanes-per-particle one; *bricks = grid bricks of kBrickEdge^3 points (0 without
 * PME).  Outputs may be NULL. */
int ommb200_context_get_pme_layout(const ommb200_context* ctx, int* bricks_in_use, int* bricks);

/* Learned-radii state of a Context whose GBSAOBCForce uses learned radii. */
typedef struct {
  int64_t judges;            /* exact-pass judgements so far */
  int64_t learned_steps;     /* MD steps whose radii came from the network */
  int64_t exact_steps;       /* MD steps whose radii came from the exact pass */
  int active;                /* the network passed the last judgement */
  double last_radius_error;  /* largest per-particle radius relative error, last judgement */
  double last_loss;          /* normalised mean squared error of the last training batch */
} ommb200_learned_radii_stats;
int ommb200_context_get_learned_radii_stats(ommb200_context* ctx,
                                            ommb200_learned_radii_stats* out);
/* The network parameters (host float [OMMB200_RADII_MLP_PARAMS], layout below). */
int ommb200_context_get_radii_mlp_params(ommb200_context* ctx, float* params);
int ommb200_context_set_radii_mlp_params(ommb200_context* ctx, const float* params);

/* ---- batches of independent systems (no reference counterpart) ----
 * One Context over n_systems independent Systems: each step() advances all of them with one
 * set of launches (the reference runs one Context per System).  The Systems must carry the
 * same force kinds with the same global settings (method, cutoff, dielectrics, switching,
 * groups) and, when there is more than one, be non-periodic; particle counts may differ.  The
 * batch's particles are the Systems' particles concatenated in order: positions, velocities
 * and forces of get_state / set_positions use that order, and every Context call behaves as
 * for one System whose energy is the sum over the batch.  Particles of different Systems never
 * interact.  Takes ownership of every System and the integrator (also on failure).  The
 * random stream is per particle, so a System's trajectory depends on its offset in the batch. */
int ommb200_context_create_batch(ommb200_system* const* systems, int n_systems,
                                 ommb200_integrator* integrator, const ommb200_options* options,
                                 ommb200_context** out);
int ommb200_context_num_systems(const ommb200_context* ctx, int* out);
/* First particle and particle count of System `index` within the batch. */
int ommb200_context_system_range(const ommb200_context* ctx, int index, int* first, int* count);
/* Potential (of force groups `groups`) and kinetic energy of each System, kJ/mol; arrays of
 * n_systems doubles, either may be NULL. */
int ommb200_context_get_system_energies(ommb200_context* ctx, uint32_t groups,
                                        double* potential, double* kinetic);

/* ---- allocation-free force evaluation (no counterpart in the reference) ----
 * For callers that must not allocate device memory: code inside another framework's memory
 * pool, whose accounting a private allocation would bypass, or a plugin that may only use the
 * buffers it is handed.  Evaluates NonbondedForce forces and energy of a non-periodic system without
 * exceptions (method OMMB200_NO_CUTOFF or OMMB200_CUTOFF_NON_PERIODIC) with the Context's
 * mixed-precision arithmetic; with a cutoff, LJ is cut plainly (no switching function) and the
 * electrostatics are the reaction field.  All pointers are device pointers on the current
 * device: positions[3n], charges[n], sigmas[n], epsilons[n] in; forces[3n] and energy[1] out.
 * Work is enqueued on `stream` (a cudaStream_t; NULL = legacy default stream) and not
 * synchronised.  n is at most 8192: the scratch is a 384 KiB static device array that every GPU
 * loading the library keeps until exit.  The first call in each CUDA context looks up that
 * array's address (the array is loaded per context); make it before any stream capture.  Calls
 * share the array, so calls that overlap on the GPU race. */
int ommb200_nonbonded_forces_noalloc(int n, const double* positions, const double* charges,
                                     const double* sigmas, const double* epsilons, int method,
                                     double cutoff, double reaction_field_dielectric,
                                     double* forces, double* energy, void* stream);

/* ---- learned Born radii network (no reference counterpart) ----
 * Per particle: 32 radial symmetry-function features -> 64 -> 64 -> 1 (tanh), predicting the
 * long-range tail of the OBC descreening integral.  BF16 tensor-core kernels with FP32
 * accumulation.  Parameters are a flat float block of OMMB200_RADII_MLP_PARAMS values:
 * W1[32][64], b1[64], W2[64][64], b2[64], w3[64], b3 (the first OMMB200_RADII_MLP_TRAINABLE
 * are trained), then feature mean[32], feature 1/std[32], target mean, target scale.
 * All pointers are device pointers; work runs on `stream` (a cudaStream_t, NULL = legacy
 * default) and the call returns after it completes. */
#define OMMB200_RADII_MLP_PARAMS 6403
#define OMMB200_RADII_MLP_TRAINABLE 6337
/* tail[n] and, if not NULL, d tail / d features [n][32] from features [n][32]. */
int ommb200_radii_mlp_forward(int n, const float* features, const float* params, float* tail,
                              float* dtail_dfeatures, void* stream);
/* `steps` Adam steps (lr, beta 0.9 / 0.999, eps 1e-8) on the mean squared error of the
 * normalised target over batches of `batch` particles (a multiple of 128) drawn from the n
 * rows by `seed` (all rows in order when batch == n).  adam_moments [2][TRAINABLE] (m then v)
 * and *adam_step are updated with the parameters.  grad_out [TRAINABLE] (may be NULL)
 * receives the last batch's gradient, loss_out [steps] (may be NULL) each batch's loss. */
int ommb200_radii_mlp_train(int n, const float* features, const float* targets, float* params,
                            float* adam_moments, int* adam_step, int steps, int batch,
                            double learning_rate, uint64_t seed, float* grad_out,
                            float* loss_out, void* stream);

/* ---- diagnostics (no reference counterpart) ---- */
/* The interacting nonbonded pair set at the current positions, as evaluated by the pair
 * kernel itself: (i, j) with i < j in original particle indices, unsorted.  Writes up to
 * max_pairs pairs and the total count. */
int ommb200_context_debug_pair_list(ommb200_context* ctx, int64_t max_pairs, int32_t* pairs,
                                    int64_t* count);
/* Per-kernel device time of the last step() call in ms, summed over launches; names are
 * written as a ';'-separated list.  Only filled when profiling was enabled. */
int ommb200_context_set_profiling(ommb200_context* ctx, int enabled);
int ommb200_context_kernel_times(ommb200_context* ctx, int max_entries, char* names,
                                 int names_len, double* ms, int* launches, int* count);
/* Neighbour-list state after the last force evaluation: tiles (32 x 32 pair blocks) the pair
 * kernel evaluates, 32-slot particle blocks in use, tiles of the last rebuild carrying exclusion
 * masks, and list rebuilds so far. */
int ommb200_context_nlist_stats(ommb200_context* ctx, int* tiles, int* blocks, int* masked,
                                int64_t* rebuilds);
/* Neighbour-list capacities (no reference counterpart; the reference builds its cell lists on
 * the host at every evaluation): tile slots, particles one x-y column may hold, and how many
 * times an overflow made them grow (the steps or the evaluation then ran again). */
int ommb200_context_nlist_capacity(ommb200_context* ctx, int* tile_capacity, int* column_capacity,
                                   int* regrows);
/* The pruned pair list of periodic rectangular boxes (no reference counterpart): tiles of the
 * last rebuild (the pair kernel's tiles are in ommb200_context_nlist_stats), prunes so far, and
 * the margin beyond the cutoff the pruned list keeps (0 when the pair kernel reads the rebuild's
 * tiles directly). */
int ommb200_context_nlist_prune_stats(ommb200_context* ctx, int* rebuild_tiles, int64_t* prunes,
                                      double* margin);
/* The culling pair kernel (ommb200_options.pair_cull; no reference counterpart): tiles per
 * warp run as this Context uses it now (0 when the pair kernel evaluates every listed entry),
 * and the rounds it has run since the Context was created, each 2 x 16 x 16 pair slots (a self
 * tile runs two).  Either output may be NULL. */
int ommb200_context_get_pair_cull(ommb200_context* ctx, int* tiles_per_run, int64_t* rounds);
/* The cudaStream_t every kernel of this Context is launched on (for CUDA-event timing). */
int ommb200_context_get_stream(ommb200_context* ctx, void** stream);
/* Diagnostics (no reference counterpart): the number of polls after which the tensor-core
 * kernels stop waiting for their MMAs, set their status to OMMB200_ERR_TIMEOUT and return, so
 * that the time-out path can be exercised; polls < 0 restores the default (about a
 * millisecond).  Kernels captured in a Context's CUDA graph keep the limit of their capture. */
int ommb200_set_tensor_core_wait_limit(long long polls);
/* Measured FP32 FMA throughput of the device (TFLOP/s, FMA = 2 flops): the roofline
 * denominator of the FP32 pair kernel. */
int ommb200_measure_fp32_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* OMMB200_H */
