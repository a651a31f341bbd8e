/*
 * f64 CPU oracle for the openmm-rs hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain C++ double precision, the reference's CPU algorithm for
 * NonbondedForce (PME / cutoff / no-cutoff), the PME reciprocal sum, the cell-list pair
 * enumeration, GBSAOBCForce, HarmonicBond/AngleForce, LangevinMiddleIntegrator and the
 * SHAKE/RATTLE constraint solver of mogura-rs/openmm-rs (crates/openmm-core).  Each function
 * cites the file:line it follows.  It adds three things the reference does not have: an
 * analytic SETTLE (Miyamoto & Kollman, J. Comput. Chem. 13:952, 1992), the analytic virial
 * -dU/d(strain), and the Philox4x32-10 Gaussian stream (Salmon et al., SC'11) that the CUDA
 * engine uses, so that CPU and GPU trajectories can be compared step by step.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu-baseline arm may load this library.
 * The product (openmm-rs_b200/) never calls it.
 *
 * Parity pinning: the reference ships no golden vectors (its OpenMM-generated fixtures need
 * an external OpenMM checkout) and cannot be compiled here (no Rust toolchain).  The oracle
 * is pinned by the reference's own analytic known-answer tests and finite-difference tests,
 * restated in tests/test_oracle.py; PME is cross-checked against an independent direct Ewald
 * sum.  Absolute FFT/erfc values are therefore pinned only by self-consistency.
 */
#ifndef OMMB200_ORACLE_H
#define OMMB200_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORC_NO_CUTOFF = 0,
  ORC_CUTOFF_NONPERIODIC = 1,
  ORC_CUTOFF_PERIODIC = 2,
  ORC_EWALD = 3, /* not restated (out of scope); rejected */
  ORC_PME = 4
};

typedef struct {
  int method;
  double cutoff;
  double ewald_tolerance;
  double reaction_field_dielectric;
  int use_switching;
  double switching_distance;
  int use_dispersion_correction;
  int exceptions_use_pbc;
  int use_neighbor_cells;
  double pme_alpha; /* > 0 overrides the tolerance rule */
  int pme_grid[3];
  int include_direct;
  int include_reciprocal;
} orc_nonbonded_options;

/* nonbonded.rs:647-658 */
void orc_pme_parameters(double cutoff, double tolerance, const double box[9], double* alpha,
                        int dims[3]);

/* nonbonded.rs:771-1042.  forces (3n) and virial (9, may be NULL) are overwritten.
 * Returns 0 on success, <0 on invalid input. */
int orc_nonbonded(int n, const double* pos, const double* charge, const double* sigma,
                  const double* epsilon, int n_exc, const int* exc_i, const int* exc_j,
                  const double* exc_qq, const double* exc_sigma, const double* exc_eps,
                  const orc_nonbonded_options* opt, const double* box, double* forces,
                  double* energy, double* virial, int threads);

/* nonbonded.rs:660-719: dispersion coefficient C such that E_disp = C / V. */
double orc_dispersion_coefficient(int n, const double* sigma, const double* epsilon,
                                  double cutoff, int use_switching, double switching_distance);

/* pme.rs:31-61 + 305-425: reciprocal energy and forces (forces are ADDED to). */
double orc_pme_reciprocal(int n, const double* pos, const double* charge, const double box[9],
                          double alpha, const int dims[3], double* forces, double* virial);

/* Independent check: direct Ewald reciprocal sum over |m_d| <= kmax (any triclinic box). */
double orc_ewald_reciprocal(int n, const double* pos, const double* charge, const double box[9],
                            double alpha, int kmax, double* forces);

/* neighbors.rs:96-181 + nonbonded.rs:842-864: the interacting pair set (i<j, not excluded,
 * r^2 < cutoff^2 after minimum image).  Writes up to max_pairs (i,j) pairs; returns count. */
int64_t orc_pair_set(int n, const double* pos, double cutoff, const double* box, int use_pbc,
                     int n_exc, const int* exc_i, const int* exc_j, int use_cells,
                     int64_t max_pairs, int32_t* pairs);

/* gbsa_obc.rs:151-309. forces (3n) overwritten; born (n, may be NULL) receives radii. */
int orc_gbsa_obc(int n, const double* pos, const double* charge, const double* radius,
                 const double* scale, int method, double cutoff, double solvent_dielectric,
                 double solute_dielectric, double surface_area_energy, const double* box,
                 double* forces, double* energy, double* born, double* virial);

/* Learned Born radii (no reference counterpart): radial symmetry functions G [n][nf] over all
 * other particles within rc; and GB energy/forces (NoCutoff, gbsa_obc.rs:184-309) with the
 * HCT integral replaced by I_short (switched from rs to rc) + tail, features within rf, tail
 * and d tail/dG given
 * per particle.  short_out / full_out (may be NULL) receive I_short and the exact integral. */
int orc_radial_features(int n, const double* pos, int nf, double mu0, double dmu, double eta,
                        double rc, double* features);
int orc_learned_gbsa(int n, const double* pos, const double* charge, const double* radius,
                     const double* scale, double solvent_dielectric, double solute_dielectric,
                     double surface_area_energy, double rs, double rc, double rf, int nf,
                     double mu0,
                     double dmu, double eta, const double* tail, const double* dtail_dg,
                     double* forces, double* energy, double* born, double* short_out,
                     double* full_out);

/* harmonic_bond.rs:102-144 and harmonic_angle.rs:102-175; forces ADDED to. */
double orc_harmonic_bond(int nb, const int* bi, const int* bj, const double* length,
                         const double* k, const double* pos, int use_pbc, const double* box,
                         double* forces, double* virial);
double orc_harmonic_angle(int na, const int* ai, const int* aj, const int* ak,
                          const double* angle, const double* k, const double* pos, int use_pbc,
                          const double* box, double* forces, double* virial);

/* Philox4x32-10 and the engine's Gaussian stream: 3 normals per atom per step. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_gaussian_noise(uint64_t seed, uint64_t stream, uint64_t step, int n, double* out);

/* constraints.rs:81-156 (Gauss-Seidel SHAKE / RATTLE).  Returns 0, or a negative code:
 * -1 nonconvergence, -2 singular, -3 nonfinite, -4 coincident reference. */
int orc_constraints_solve(int nc, const int* ci, const int* cj, const double* distance,
                          const double* masses, const double* reference, double* values,
                          int velocities, double tolerance);

/* Analytic SETTLE (positions) and the exact rigid-water velocity projection. */
int orc_settle_positions(int nw, const int* atoms /*3*nw: O,H,H*/, double d_oh, double d_hh,
                         const double* masses, const double* reference, double* positions);
int orc_settle_velocities(int nw, const int* atoms, const double* masses,
                          const double* positions, double* velocities);

/* langevin.rs:216-278 (+ integrators/mod.rs:232-268): one LFMiddle step with the given
 * normals.  constraint_mode 0 = SHAKE/RATTLE (reference), 1 = SETTLE for the given waters
 * (other constraints absent). */
int orc_lfmiddle_step(int n, double* pos, double* vel, const double* forces,
                      const double* masses, double dt, double temperature, double friction,
                      const double* noise, int nc, const int* ci, const int* cj,
                      const double* distance, double tolerance, int constraint_mode, int nw,
                      const int* waters, double d_oh, double d_hh);

/* context.rs:1107-1163 with a zero time offset. */
double orc_kinetic_energy(int n, const double* vel, const double* masses);

/* Wall-clock helper for the CPU baseline. */
double orc_wtime(void);
int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
