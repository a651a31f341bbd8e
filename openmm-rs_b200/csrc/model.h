// Host-side definitions mirroring openmm-core's System / Force / Integrator objects
// (crates/openmm-core/src/system.rs, forces/nonbonded.rs, forces/gbsa_obc.rs,
// forces/harmonic_bond.rs, forces/harmonic_angle.rs, integrators/langevin.rs).  These hold
// parameters only; the Engine (engine.h) turns them into device buffers at Context creation,
// which, like the reference's Context::new (context.rs:83-161), takes ownership of both.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace ommb200 {

// Error raised by setters and Context creation; carries an OMMB200_ERR_* code.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

enum ForceKind { kNonbonded = 1, kGbsaObc = 2, kHarmonicBond = 3, kHarmonicAngle = 4,
                 kMonteCarloBarostat = 5 };

// NonbondedMethod (nonbonded.rs:19-33); Ewald and LJPME are not engine methods.
enum NonbondedMethod { kNoCutoff = 0, kCutoffNonPeriodic = 1, kCutoffPeriodic = 2, kEwald = 3,
                       kPME = 4, kLJPME = 5 };

struct ForceDef {
  explicit ForceDef(ForceKind k) : kind(k) {}
  virtual ~ForceDef() = default;
  ForceKind kind;
  int force_group = 0;
  std::string name;
  bool owned_by_system = false;
};

struct ExceptionDef {
  int p1, p2;
  double charge_prod, sigma, epsilon;
};

struct NonbondedDef : ForceDef {
  NonbondedDef() : ForceDef(kNonbonded) { name = "NonbondedForce"; }
  std::vector<double> charge, sigma, epsilon;
  std::vector<ExceptionDef> exceptions;
  int method = kNoCutoff;
  double cutoff = 1.0;
  double reaction_field_dielectric = 78.3;
  double ewald_error_tolerance = 5e-4;
  bool exceptions_use_pbc = false;
  bool use_dispersion_correction = true;
  bool use_switching = false;
  double switching_distance = -1.0;
  double pme_alpha = 0.0;  // 0: derive from the tolerance rule at Context creation
  std::array<int, 3> pme_grid{{0, 0, 0}};
  int reciprocal_force_group = -1;
  bool include_direct_space = true;

  bool periodic() const {
    return method == kCutoffPeriodic || method == kEwald || method == kPME || method == kLJPME;
  }
  int add_particle(double q, double s, double e);
  int add_exception(int p1, int p2, double qq, double s, double e);
  void create_exceptions_from_bonds(const std::vector<std::pair<int, int>>& bonds,
                                    double coulomb14, double lj14);
  // nonbonded.rs:647-658
  void effective_pme_parameters(const double box[9], double* alpha, int dims[3]) const;
};

// Learned Born radii (no reference counterpart): a network predicts the long-range tail of the
// HCT integral; the exact pass judges it every `judge_interval` MD steps.
struct LearnedRadiiDef {
  bool enabled = false;
  int judge_interval = 50;
  double radius_tolerance = 0.01;  // largest per-particle radius relative error allowed
  int train_steps = 10;            // Adam steps after each judge
  int batch = 4096;                // particles per Adam step
  double learning_rate = 1e-3;
  int seed = 1;
};

struct GbsaObcDef : ForceDef {
  GbsaObcDef() : ForceDef(kGbsaObc) { name = "GBSAOBCForce"; }
  std::vector<double> charge, radius, scale;
  int method = 0;  // 0 NoCutoff, 1 CutoffNonPeriodic, 2 CutoffPeriodic
  double cutoff = 1.0;
  double solvent_dielectric = 78.3;
  double solute_dielectric = 1.0;
  double surface_area_energy = 2.25936;
  LearnedRadiiDef learned;
};

struct BondDef {
  int p1, p2;
  double length, k;
};
struct HarmonicBondDef : ForceDef {
  HarmonicBondDef() : ForceDef(kHarmonicBond) { name = "HarmonicBondForce"; }
  std::vector<BondDef> bonds;
  bool use_pbc = false;
};

struct AngleDef {
  int p1, p2, p3;
  double angle, k;
};
struct HarmonicAngleDef : ForceDef {
  HarmonicAngleDef() : ForceDef(kHarmonicAngle) { name = "HarmonicAngleForce"; }
  std::vector<AngleDef> angles;
  bool use_pbc = false;
};

// MonteCarloBarostat (forces/barostat.rs:44-110): isotropic Monte Carlo volume moves every
// `frequency` steps at `pressure` (bar) and `temperature` (K).  The Context reads `frequency`
// from this object at every step, so changing it later reaches existing Contexts (the
// reference shares it through an atomic, barostat.rs:98-101).
struct BarostatDef : ForceDef {
  BarostatDef() : ForceDef(kMonteCarloBarostat) { name = "MonteCarloBarostat"; }
  double default_pressure = 1.0;
  double default_temperature = 300.0;
  int frequency = 25;
  bool scale_molecules_as_rigid = true;  // barostat.rs:78
  int random_seed = 0;                   // 0: pick from OS entropy at Context creation
};

struct ConstraintDef {
  int p1, p2;
  double distance;
};

struct SystemDef {
  std::vector<double> masses;
  std::vector<ConstraintDef> constraints;
  double box[9] = {2.0, 0, 0, 0, 2.0, 0, 0, 0, 2.0};  // system.rs:50 default 2 nm cube
  std::vector<std::unique_ptr<ForceDef>> forces;
  int add_particle(double mass);
  int add_constraint(int p1, int p2, double distance);
  void set_default_box(const double a[3], const double b[3], const double c[3]);
};

// LangevinMiddleIntegrator (integrators/langevin.rs:14-102).
struct IntegratorDef {
  double temperature = 300.0;
  double friction = 1.0;
  double step_size = 0.002;
  double constraint_tolerance = 1e-5;
  int random_seed = 0;  // 0: pick from OS entropy at Context creation (random.rs:40-46)
  uint32_t integration_force_groups = 0xffffffffu;
  bool owned_by_context = false;
};

void validate_box(const double box[9]);  // system.rs:13-38

// A contiguous particle range of the merged System that came from one input System.
struct Segment {
  int first, count;
};

// Concatenates independent Systems into one, with every force kind merged into a single
// force whose particles, exceptions, bonds and angles are offset per input System.  The
// inputs must carry the same force kinds with the same global settings, and must not be
// periodic when there is more than one.  `segments` receives each input's particle range.
std::unique_ptr<SystemDef> merge_systems(std::vector<std::unique_ptr<SystemDef>> systems,
                                         std::vector<Segment>* segments);

}  // namespace ommb200
