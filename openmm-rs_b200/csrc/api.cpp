// extern "C" boundary: every entry point validates its arguments, catches every exception
// and returns an OMMB200_* status; nothing aborts the caller.
#include <cmath>
#include <cstring>
#include <new>
#include <set>
#include <string>

#include "../../include/ommb200.h"
#include "engine.h"
#include "model.h"

using namespace ommb200;

struct ommb200_context {
  std::unique_ptr<Engine> engine;
};

namespace {

thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

void require(bool ok, const char* msg) {
  if (!ok) throw Error(OMMB200_ERR_INVALID_ARG, msg);
}

template <class F>
int guarded(F&& fn) {
  try {
    fn();
    return OMMB200_OK;
  } catch (const Error& e) {
    set_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return OMMB200_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    set_error(e.what());
    return OMMB200_ERR_CUDA;
  } catch (...) {
    set_error("unknown failure");
    return OMMB200_ERR_CUDA;
  }
}

ForceDef* as_force(ommb200_force* f) { return reinterpret_cast<ForceDef*>(f); }
const ForceDef* as_force(const ommb200_force* f) { return reinterpret_cast<const ForceDef*>(f); }

template <class T, ForceKind K>
T* force_of(ommb200_force* f) {
  require(f != nullptr, "null force handle");
  ForceDef* d = as_force(f);
  require(d->kind == K, "force handle has the wrong type for this call");
  return static_cast<T*>(d);
}
template <class T, ForceKind K>
const T* force_of(const ommb200_force* f) {
  require(f != nullptr, "null force handle");
  const ForceDef* d = as_force(f);
  require(d->kind == K, "force handle has the wrong type for this call");
  return static_cast<const T*>(d);
}

NonbondedDef* nbf(ommb200_force* f) { return force_of<NonbondedDef, kNonbonded>(f); }
const NonbondedDef* nbf(const ommb200_force* f) { return force_of<NonbondedDef, kNonbonded>(f); }
GbsaObcDef* gbf(ommb200_force* f) { return force_of<GbsaObcDef, kGbsaObc>(f); }

SystemDef* sysdef(ommb200_system* s) { return reinterpret_cast<SystemDef*>(s); }
const SystemDef* sysdef(const ommb200_system* s) { return reinterpret_cast<const SystemDef*>(s); }
IntegratorDef* integdef(ommb200_integrator* i) { return reinterpret_cast<IntegratorDef*>(i); }

void set_out(int* out, int v) {
  if (out) *out = v;
}
void set_out(double* out, double v) {
  if (out) *out = v;
}
void require_pressure(double p) { require(std::isfinite(p), "pressure must be finite"); }
void require_temperature(double t) {
  require(std::isfinite(t) && t >= 0.0, "temperature must be nonnegative and finite");
}
BarostatDef* barostat_of(ommb200_force* f) { return force_of<BarostatDef, kMonteCarloBarostat>(f); }
const BarostatDef* barostat_of(const ommb200_force* f) {
  return force_of<BarostatDef, kMonteCarloBarostat>(f);
}

void check_cuda(cudaError_t e) {
  if (e != cudaSuccess) throw Error(OMMB200_ERR_CUDA, cudaGetErrorString(e));
}
// Runs `launch(status)` on `stream` and waits; device faults and kernel status become codes.
template <class F>
void run_standalone(void* stream, F&& launch) {
  int* status = nullptr;
  check_cuda(cudaMalloc(&status, sizeof(int)));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int code = 0;
  try {
    check_cuda(cudaMemsetAsync(status, 0, sizeof(int), s));
    launch(status);
    check_cuda(cudaGetLastError());
    check_cuda(cudaMemcpyAsync(&code, status, sizeof(int), cudaMemcpyDeviceToHost, s));
    check_cuda(cudaStreamSynchronize(s));
  } catch (...) {
    cudaFree(status);
    throw;
  }
  cudaFree(status);
  if (code != 0) throw Error(OMMB200_ERR_TIMEOUT, "tensor-core wait timed out");
}
int device_sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}
}  // namespace

extern "C" {

const char* ommb200_last_error(void) { return g_last_error.c_str(); }
const char* ommb200_version(void) { return "ommb200 0.1 (sm_100a)"; }

void ommb200_default_options(ommb200_options* out) {
  if (!out) return;
  out->precision = OMMB200_PRECISION_MIXED;
  out->device = 0;
  out->use_cuda_graph = 1;
  out->neighbor_skin = 0.0;
  out->steps_per_graph = 0;
  out->pme_bricks = -1;
  out->prune_margin = -1.0;
  out->pair_cull = -1;
}

// ---- System -----------------------------------------------------------------------------
int ommb200_system_create(ommb200_system** out) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    *out = reinterpret_cast<ommb200_system*>(new SystemDef());
  });
}
int ommb200_system_destroy(ommb200_system* s) {
  return guarded([&] { delete sysdef(s); });
}
int ommb200_system_add_particle(ommb200_system* s, double mass, int* index) {
  return guarded([&] {
    require(s != nullptr, "null system handle");
    set_out(index, sysdef(s)->add_particle(mass));
  });
}
int ommb200_system_num_particles(const ommb200_system* s, int* out) {
  return guarded([&] {
    require(s && out, "null argument");
    *out = (int)sysdef(s)->masses.size();
  });
}
int ommb200_system_add_constraint(ommb200_system* s, int p1, int p2, double distance, int* index) {
  return guarded([&] {
    require(s != nullptr, "null system handle");
    set_out(index, sysdef(s)->add_constraint(p1, p2, distance));
  });
}
int ommb200_system_set_default_periodic_box_vectors(ommb200_system* s, const double a[3],
                                                    const double b[3], const double c[3]) {
  return guarded([&] {
    require(s && a && b && c, "null argument");
    sysdef(s)->set_default_box(a, b, c);
  });
}
int ommb200_system_add_force(ommb200_system* s, ommb200_force* force, int* index) {
  return guarded([&] {
    require(s && force, "null argument");
    ForceDef* f = as_force(force);
    require(!f->owned_by_system, "force already belongs to a System");
    f->owned_by_system = true;
    sysdef(s)->forces.emplace_back(f);
    set_out(index, (int)sysdef(s)->forces.size() - 1);
  });
}

// ---- forces: common ---------------------------------------------------------------------
int ommb200_force_destroy(ommb200_force* force) {
  return guarded([&] {
    if (!force) return;
    require(!as_force(force)->owned_by_system, "force is owned by a System");
    delete as_force(force);
  });
}
int ommb200_force_set_group(ommb200_force* force, int group) {
  return guarded([&] {
    require(force != nullptr, "null force handle");
    require(group >= 0 && group < 32, "force group must be between 0 and 31");
    as_force(force)->force_group = group;
  });
}
int ommb200_force_get_group(const ommb200_force* force, int* group) {
  return guarded([&] {
    require(force && group, "null argument");
    *group = as_force(force)->force_group;
  });
}

// ---- NonbondedForce ---------------------------------------------------------------------
int ommb200_nonbonded_create(ommb200_force** out) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    *out = reinterpret_cast<ommb200_force*>(static_cast<ForceDef*>(new NonbondedDef()));
  });
}
int ommb200_nonbonded_add_particle(ommb200_force* f, double q, double s, double e, int* index) {
  return guarded([&] { set_out(index, nbf(f)->add_particle(q, s, e)); });
}
int ommb200_nonbonded_set_particle_parameters(ommb200_force* f, int index, double q, double s,
                                              double e) {
  return guarded([&] {
    NonbondedDef* d = nbf(f);
    require(index >= 0 && index < (int)d->charge.size(), "particle index out of range");
    require(std::isfinite(q) && std::isfinite(s) && std::isfinite(e) && s >= 0.0 && e >= 0.0,
            "nonbonded parameters must be finite with nonnegative sigma and epsilon");
    d->charge[index] = q;
    d->sigma[index] = s;
    d->epsilon[index] = e;
  });
}
int ommb200_nonbonded_get_particle_parameters(const ommb200_force* f, int index, double* q,
                                              double* s, double* e) {
  return guarded([&] {
    const NonbondedDef* d = nbf(f);
    require(index >= 0 && index < (int)d->charge.size(), "particle index out of range");
    if (q) *q = d->charge[index];
    if (s) *s = d->sigma[index];
    if (e) *e = d->epsilon[index];
  });
}
int ommb200_nonbonded_num_particles(const ommb200_force* f, int* out) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    *out = (int)nbf(f)->charge.size();
  });
}
int ommb200_nonbonded_add_exception(ommb200_force* f, int p1, int p2, double qq, double s,
                                    double e, int* index) {
  return guarded([&] { set_out(index, nbf(f)->add_exception(p1, p2, qq, s, e)); });
}
int ommb200_nonbonded_num_exceptions(const ommb200_force* f, int* out) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    *out = (int)nbf(f)->exceptions.size();
  });
}
int ommb200_nonbonded_create_exceptions_from_bonds(ommb200_force* f, int n_bonds, const int* bonds,
                                                   double coulomb14, double lj14) {
  return guarded([&] {
    require(n_bonds >= 0 && (n_bonds == 0 || bonds), "invalid bond list");
    std::vector<std::pair<int, int>> b(n_bonds);
    for (int i = 0; i < n_bonds; ++i) b[i] = {bonds[2 * i], bonds[2 * i + 1]};
    nbf(f)->create_exceptions_from_bonds(b, coulomb14, lj14);
  });
}
int ommb200_nonbonded_set_method(ommb200_force* f, int method) {
  return guarded([&] {
    require(method >= OMMB200_NO_CUTOFF && method <= OMMB200_LJPME, "unknown nonbonded method");
    nbf(f)->method = method;
  });
}
int ommb200_nonbonded_set_cutoff_distance(ommb200_force* f, double cutoff) {
  return guarded([&] {
    require(std::isfinite(cutoff) && cutoff > 0.0, "cutoff must be positive and finite");
    nbf(f)->cutoff = cutoff;
  });
}
int ommb200_nonbonded_set_reaction_field_dielectric(ommb200_force* f, double eps) {
  return guarded([&] {
    require(!std::isnan(eps) && eps >= 1.0, "reaction field dielectric must be at least one");
    nbf(f)->reaction_field_dielectric = eps;
  });
}
int ommb200_nonbonded_set_ewald_error_tolerance(ommb200_force* f, double tol) {
  return guarded([&] {
    require(std::isfinite(tol) && tol > 0.0 && tol < 0.5, "Ewald tolerance must be between zero and one half");
    nbf(f)->ewald_error_tolerance = tol;
  });
}
int ommb200_nonbonded_set_exceptions_use_periodic_boundary_conditions(ommb200_force* f, int periodic) {
  return guarded([&] { nbf(f)->exceptions_use_pbc = periodic != 0; });
}
int ommb200_nonbonded_set_use_dispersion_correction(ommb200_force* f, int enabled) {
  return guarded([&] { nbf(f)->use_dispersion_correction = enabled != 0; });
}
int ommb200_nonbonded_set_use_switching_function(ommb200_force* f, int enabled) {
  return guarded([&] { nbf(f)->use_switching = enabled != 0; });
}
int ommb200_nonbonded_set_switching_distance(ommb200_force* f, double distance) {
  return guarded([&] {
    require(std::isfinite(distance) && distance >= 0.0, "switching distance must be nonnegative and finite");
    nbf(f)->switching_distance = distance;
  });
}
int ommb200_nonbonded_set_pme_parameters(ommb200_force* f, double alpha, int nx, int ny, int nz) {
  return guarded([&] {
    require(std::isfinite(alpha) && alpha >= 0.0, "PME alpha must be nonnegative and finite");
    require(alpha == 0.0 || (nx >= 5 && ny >= 5 && nz >= 5), "PME grid dimensions must be at least five");
    NonbondedDef* d = nbf(f);
    d->pme_alpha = alpha;
    d->pme_grid = {alpha == 0.0 ? 0 : nx, alpha == 0.0 ? 0 : ny, alpha == 0.0 ? 0 : nz};
  });
}
int ommb200_nonbonded_set_reciprocal_space_force_group(ommb200_force* f, int group) {
  return guarded([&] {
    require(group >= -1 && group < 32, "reciprocal force group must be between -1 and 31");
    nbf(f)->reciprocal_force_group = group;
  });
}
int ommb200_nonbonded_set_include_direct_space(ommb200_force* f, int enabled) {
  return guarded([&] { nbf(f)->include_direct_space = enabled != 0; });
}

// ---- GBSAOBCForce -----------------------------------------------------------------------
int ommb200_gbsa_obc_create(ommb200_force** out) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    *out = reinterpret_cast<ommb200_force*>(static_cast<ForceDef*>(new GbsaObcDef()));
  });
}
int ommb200_gbsa_obc_add_particle(ommb200_force* f, double q, double radius, double scale, int* index) {
  return guarded([&] {
    GbsaObcDef* d = gbf(f);
    d->charge.push_back(q);
    d->radius.push_back(radius);
    d->scale.push_back(scale);
    set_out(index, (int)d->charge.size() - 1);
  });
}
int ommb200_gbsa_obc_set_particle_parameters(ommb200_force* f, int index, double q, double radius,
                                             double scale) {
  return guarded([&] {
    GbsaObcDef* d = gbf(f);
    require(index >= 0 && index < (int)d->charge.size(), "particle index out of range");
    d->charge[index] = q;
    d->radius[index] = radius;
    d->scale[index] = scale;
  });
}
int ommb200_gbsa_obc_set_method(ommb200_force* f, int method) {
  return guarded([&] {
    require(method >= 0 && method <= 2, "unknown GBSA method");
    gbf(f)->method = method;
  });
}
int ommb200_gbsa_obc_set_cutoff_distance(ommb200_force* f, double cutoff) {
  return guarded([&] { gbf(f)->cutoff = cutoff; });
}
int ommb200_gbsa_obc_set_solvent_dielectric(ommb200_force* f, double value) {
  return guarded([&] { gbf(f)->solvent_dielectric = value; });
}
int ommb200_gbsa_obc_set_solute_dielectric(ommb200_force* f, double value) {
  return guarded([&] { gbf(f)->solute_dielectric = value; });
}
int ommb200_gbsa_obc_set_surface_area_energy(ommb200_force* f, double value) {
  return guarded([&] { gbf(f)->surface_area_energy = value; });
}
int ommb200_gbsa_obc_set_learned_radii(ommb200_force* f, int enabled, int judge_interval,
                                       double radius_tolerance, int train_steps) {
  return guarded([&] {
    GbsaObcDef* g = gbf(f);
    require(judge_interval >= 1, "judge interval must be at least one step");
    require(std::isfinite(radius_tolerance) && radius_tolerance > 0.0,
            "radius tolerance must be positive and finite");
    require(train_steps >= 0, "training steps must be nonnegative");
    g->learned.enabled = enabled != 0;
    g->learned.judge_interval = judge_interval;
    g->learned.radius_tolerance = radius_tolerance;
    g->learned.train_steps = train_steps;
  });
}

// ---- bonded -----------------------------------------------------------------------------
int ommb200_harmonic_bond_create(ommb200_force** out) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    *out = reinterpret_cast<ommb200_force*>(static_cast<ForceDef*>(new HarmonicBondDef()));
  });
}
int ommb200_harmonic_bond_add_bond(ommb200_force* f, int p1, int p2, double length, double k, int* index) {
  return guarded([&] {
    auto* d = force_of<HarmonicBondDef, kHarmonicBond>(f);
    d->bonds.push_back({p1, p2, length, k});
    set_out(index, (int)d->bonds.size() - 1);
  });
}
int ommb200_harmonic_bond_set_uses_pbc(ommb200_force* f, int use_pbc) {
  return guarded([&] { force_of<HarmonicBondDef, kHarmonicBond>(f)->use_pbc = use_pbc != 0; });
}
int ommb200_harmonic_angle_create(ommb200_force** out) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    *out = reinterpret_cast<ommb200_force*>(static_cast<ForceDef*>(new HarmonicAngleDef()));
  });
}
int ommb200_harmonic_angle_add_angle(ommb200_force* f, int p1, int p2, int p3, double angle,
                                     double k, int* index) {
  return guarded([&] {
    auto* d = force_of<HarmonicAngleDef, kHarmonicAngle>(f);
    d->angles.push_back({p1, p2, p3, angle, k});
    set_out(index, (int)d->angles.size() - 1);
  });
}
int ommb200_harmonic_angle_set_uses_pbc(ommb200_force* f, int use_pbc) {
  return guarded([&] { force_of<HarmonicAngleDef, kHarmonicAngle>(f)->use_pbc = use_pbc != 0; });
}

// ---- MonteCarloBarostat (forces/barostat.rs:63-119) -------------------------------------------

int ommb200_monte_carlo_barostat_create(double pressure, double temperature, int frequency,
                                        ommb200_force** out) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    require_pressure(pressure);
    require_temperature(temperature);
    require(frequency >= 0, "frequency must be nonnegative");
    auto* d = new BarostatDef();
    d->default_pressure = pressure;
    d->default_temperature = temperature;
    d->frequency = frequency;
    *out = reinterpret_cast<ommb200_force*>(static_cast<ForceDef*>(d));
  });
}
int ommb200_monte_carlo_barostat_set_default_pressure(ommb200_force* f, double pressure) {
  return guarded([&] {
    require_pressure(pressure);
    barostat_of(f)->default_pressure = pressure;
  });
}
int ommb200_monte_carlo_barostat_get_default_pressure(const ommb200_force* f, double* out) {
  return guarded([&] { set_out(out, barostat_of(f)->default_pressure); });
}
int ommb200_monte_carlo_barostat_set_default_temperature(ommb200_force* f, double t) {
  return guarded([&] {
    require_temperature(t);
    barostat_of(f)->default_temperature = t;
  });
}
int ommb200_monte_carlo_barostat_get_default_temperature(const ommb200_force* f, double* out) {
  return guarded([&] { set_out(out, barostat_of(f)->default_temperature); });
}
int ommb200_monte_carlo_barostat_set_frequency(ommb200_force* f, int frequency) {
  return guarded([&] {
    require(frequency >= 0, "frequency must be nonnegative");
    barostat_of(f)->frequency = frequency;
  });
}
int ommb200_monte_carlo_barostat_get_frequency(const ommb200_force* f, int* out) {
  return guarded([&] { set_out(out, barostat_of(f)->frequency); });
}
int ommb200_monte_carlo_barostat_set_scale_molecules_as_rigid(ommb200_force* f, int rigid) {
  return guarded([&] { barostat_of(f)->scale_molecules_as_rigid = rigid != 0; });
}
int ommb200_monte_carlo_barostat_get_scale_molecules_as_rigid(const ommb200_force* f, int* out) {
  return guarded([&] { set_out(out, barostat_of(f)->scale_molecules_as_rigid ? 1 : 0); });
}
int ommb200_monte_carlo_barostat_set_random_number_seed(ommb200_force* f, int seed) {
  return guarded([&] { barostat_of(f)->random_seed = seed; });
}
int ommb200_monte_carlo_barostat_get_random_number_seed(const ommb200_force* f, int* out) {
  return guarded([&] { set_out(out, barostat_of(f)->random_seed); });
}

// ---- LangevinMiddleIntegrator -----------------------------------------------------------
int ommb200_langevin_middle_create(double temperature, double friction, double step_size,
                                   ommb200_integrator** out) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    require(std::isfinite(temperature) && temperature >= 0.0, "temperature must be nonnegative and finite");
    require(std::isfinite(friction) && friction >= 0.0, "friction must be nonnegative and finite");
    require(std::isfinite(step_size) && step_size > 0.0, "step size must be positive and finite");
    auto* i = new IntegratorDef();
    i->temperature = temperature;
    i->friction = friction;
    i->step_size = step_size;
    *out = reinterpret_cast<ommb200_integrator*>(i);
  });
}
int ommb200_integrator_destroy(ommb200_integrator* i) {
  return guarded([&] {
    if (!i) return;
    require(!integdef(i)->owned_by_context, "integrator is owned by a Context");
    delete integdef(i);
  });
}
int ommb200_integrator_set_random_number_seed(ommb200_integrator* i, int seed) {
  return guarded([&] {
    require(i != nullptr, "null integrator handle");
    integdef(i)->random_seed = seed;
  });
}
int ommb200_integrator_set_constraint_tolerance(ommb200_integrator* i, double tol) {
  return guarded([&] {
    require(i != nullptr, "null integrator handle");
    require(std::isfinite(tol) && tol > 0.0 && tol < 1.0, "constraint tolerance must be between zero and one");
    integdef(i)->constraint_tolerance = tol;
  });
}
int ommb200_integrator_set_temperature(ommb200_integrator* i, double t) {
  return guarded([&] {
    require(i != nullptr, "null integrator handle");
    require(std::isfinite(t) && t >= 0.0, "temperature must be nonnegative and finite");
    integdef(i)->temperature = t;
  });
}
int ommb200_integrator_set_friction(ommb200_integrator* i, double f) {
  return guarded([&] {
    require(i != nullptr, "null integrator handle");
    require(std::isfinite(f) && f >= 0.0, "friction must be nonnegative and finite");
    integdef(i)->friction = f;
  });
}
int ommb200_integrator_set_step_size(ommb200_integrator* i, double dt) {
  return guarded([&] {
    require(i != nullptr, "null integrator handle");
    require(std::isfinite(dt) && dt > 0.0, "step size must be positive and finite");
    integdef(i)->step_size = dt;
  });
}
int ommb200_integrator_set_integration_force_groups(ommb200_integrator* i, uint32_t groups) {
  return guarded([&] {
    require(i != nullptr, "null integrator handle");
    integdef(i)->integration_force_groups = groups;
  });
}

// ---- Context ----------------------------------------------------------------------------
static EngineOptions engine_options(const ommb200_options* options) {
  ommb200_options o;
  ommb200_default_options(&o);
  if (options) o = *options;
  require(o.precision == OMMB200_PRECISION_MIXED || o.precision == OMMB200_PRECISION_DOUBLE,
          "unknown precision");
  require(o.pme_bricks >= -1 && o.pme_bricks <= 1, "pme_bricks must be -1, 0 or 1");
  require(std::isfinite(o.prune_margin) && o.prune_margin <= 0.5,
          "prune_margin must be finite and at most 0.5 nm");
  require(o.pair_cull >= -1 && o.pair_cull <= 64, "pair_cull must be -1, 0 or 1-64 tiles");
  EngineOptions eo;
  eo.precision = o.precision;
  eo.device = o.device;
  eo.use_graph = o.use_cuda_graph != 0;
  eo.skin = o.neighbor_skin;
  eo.steps_per_graph = o.steps_per_graph;
  eo.pme_bricks = o.pme_bricks;
  eo.prune_margin = o.prune_margin;
  eo.pair_cull = o.pair_cull;
  return eo;
}

int ommb200_context_create(ommb200_system* system, ommb200_integrator* integrator,
                           const ommb200_options* options, ommb200_context** out) {
  std::unique_ptr<SystemDef> sys(sysdef(system));
  std::unique_ptr<IntegratorDef> integ(integdef(integrator));
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    *out = nullptr;
    require(sys != nullptr && integ != nullptr, "null system or integrator handle");
    integ->owned_by_context = true;
    auto ctx = std::make_unique<ommb200_context>();
    ctx->engine = std::make_unique<Engine>(std::move(sys), std::move(integ), engine_options(options));
    *out = ctx.release();
  });
}
int ommb200_context_create_batch(ommb200_system* const* systems, int n_systems,
                                 ommb200_integrator* integrator, const ommb200_options* options,
                                 ommb200_context** out) {
  std::vector<std::unique_ptr<SystemDef>> defs;
  std::set<ommb200_system*> seen;
  bool repeated = false;
  if (systems)
    for (int k = 0; k < n_systems; ++k) {
      const bool fresh = seen.insert(systems[k]).second;
      repeated = repeated || !fresh;
      defs.emplace_back(fresh ? sysdef(systems[k]) : nullptr);
    }
  std::unique_ptr<IntegratorDef> integ(integdef(integrator));
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    *out = nullptr;
    require(systems != nullptr && n_systems > 0, "a batch needs at least one System");
    require(!repeated, "a System handle appears more than once in the batch");
    for (auto& d : defs) require(d != nullptr, "null system handle");
    require(integ != nullptr, "null integrator handle");
    integ->owned_by_context = true;
    std::vector<Segment> segments;
    std::unique_ptr<SystemDef> merged = merge_systems(std::move(defs), &segments);
    auto ctx = std::make_unique<ommb200_context>();
    ctx->engine = std::make_unique<Engine>(std::move(merged), std::move(integ),
                                           engine_options(options), segments);
    *out = ctx.release();
  });
}
int ommb200_context_destroy(ommb200_context* ctx) {
  return guarded([&] { delete ctx; });
}

#define OMMB200_CTX                                   \
  require(ctx != nullptr && ctx->engine, "null context handle"); \
  Engine& E = *ctx->engine

int ommb200_context_num_particles(const ommb200_context* ctx, int* out) {
  return guarded([&] {
    require(ctx && ctx->engine && out, "null argument");
    *out = ctx->engine->num_particles();
  });
}
int ommb200_context_set_positions(ommb200_context* ctx, const double* positions, int n) {
  return guarded([&] {
    OMMB200_CTX;
    require(positions != nullptr && n == E.num_particles(), "positions must have shape [N, 3]");
    E.set_positions(positions);
  });
}
int ommb200_context_set_velocities(ommb200_context* ctx, const double* velocities, int n) {
  return guarded([&] {
    OMMB200_CTX;
    require(velocities != nullptr && n == E.num_particles(), "velocities must have shape [N, 3]");
    E.set_velocities(velocities);
  });
}
int ommb200_context_set_velocities_to_temperature(ommb200_context* ctx, double temperature, int seed) {
  return guarded([&] {
    OMMB200_CTX;
    E.set_velocities_to_temperature(temperature, seed);
  });
}
int ommb200_context_set_periodic_box_vectors(ommb200_context* ctx, const double a[3],
                                             const double b[3], const double c[3]) {
  return guarded([&] {
    OMMB200_CTX;
    require(a && b && c, "null box vector");
    const double box[9] = {a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]};
    E.set_box(box);
  });
}
int ommb200_context_set_time(ommb200_context* ctx, double time) {
  return guarded([&] {
    OMMB200_CTX;
    E.set_time(time);
  });
}
int ommb200_context_set_step_count(ommb200_context* ctx, int64_t steps) {
  return guarded([&] {
    OMMB200_CTX;
    E.set_step_count(steps);
  });
}
int ommb200_context_apply_constraints(ommb200_context* ctx, double tolerance) {
  return guarded([&] {
    OMMB200_CTX;
    E.apply_constraints(tolerance);
  });
}
int ommb200_context_apply_velocity_constraints(ommb200_context* ctx, double tolerance) {
  return guarded([&] {
    OMMB200_CTX;
    E.apply_velocity_constraints(tolerance);
  });
}
int ommb200_context_step(ommb200_context* ctx, int steps) {
  return guarded([&] {
    OMMB200_CTX;
    require(steps >= 0, "step count must be nonnegative");
    E.step(steps);
  });
}
int ommb200_context_set_parameter(ommb200_context* ctx, const char* name, double value) {
  return guarded([&] {
    OMMB200_CTX;
    require(name != nullptr, "null parameter name");
    E.set_parameter(name, value);
  });
}
int ommb200_context_get_parameter(ommb200_context* ctx, const char* name, double* value) {
  return guarded([&] {
    OMMB200_CTX;
    require(name != nullptr && value != nullptr, "null argument");
    *value = E.get_parameter(name);
  });
}
int ommb200_context_get_barostat_stats(ommb200_context* ctx, ommb200_barostat_stats* out) {
  return guarded([&] {
    OMMB200_CTX;
    require(out != nullptr, "null output pointer");
    E.barostat_stats(out);
  });
}
int ommb200_context_get_state(ommb200_context* ctx, int flags, uint32_t groups, double* positions,
                              double* velocities, double* forces, ommb200_state_info* info) {
  return guarded([&] {
    OMMB200_CTX;
    E.get_state(flags, groups, (flags & OMMB200_STATE_POSITIONS) ? positions : nullptr,
                (flags & OMMB200_STATE_VELOCITIES) ? velocities : nullptr,
                (flags & OMMB200_STATE_FORCES) ? forces : nullptr, info);
  });
}
int ommb200_context_get_pme_parameters(const ommb200_context* ctx, double* alpha, int* nx, int* ny,
                                       int* nz) {
  return guarded([&] {
    require(ctx && ctx->engine && alpha && nx && ny && nz, "null argument");
    ctx->engine->pme_parameters(alpha, nx, ny, nz);
  });
}
int ommb200_context_get_pme_layout(const ommb200_context* ctx, int* bricks_in_use, int* bricks) {
  return guarded([&] {
    require(ctx && ctx->engine, "null argument");
    ctx->engine->pme_layout(bricks_in_use, bricks);
  });
}

int ommb200_radii_mlp_forward(int n, const float* features, const float* params, float* tail,
                              float* dtail_dfeatures, void* stream) {
  return guarded([&] {
    require(n > 0 && features && params && tail, "invalid arguments");
    run_standalone(stream, [&](int* status) {
      launch_mlp_infer(n, features, params, tail, dtail_dfeatures, status, device_sm_count(),
                       static_cast<cudaStream_t>(stream));
    });
  });
}
int ommb200_radii_mlp_train(int n, const float* features, const float* targets, float* params,
                            float* adam_moments, int* adam_step, int steps, int batch,
                            double learning_rate, uint64_t seed, float* grad_out,
                            float* loss_out, void* stream) {
  return guarded([&] {
    require(n > 0 && features && targets && params && adam_moments && adam_step,
            "invalid arguments");
    require(steps > 0 && batch >= 128 && batch % 128 == 0,
            "batch must be a positive multiple of 128 and steps positive");
    require(std::isfinite(learning_rate) && learning_rate >= 0.0, "invalid learning rate");
    run_standalone(stream, [&](int* status) {
      launch_mlp_train(n, features, targets, params, adam_moments,
                       adam_moments + kRadiiMlpTrainable, adam_step, steps, batch,
                       (float)learning_rate, seed, grad_out, loss_out, status,
                       static_cast<cudaStream_t>(stream));
    });
  });
}

int ommb200_context_update_nonbonded_parameters(ommb200_context* ctx, const ommb200_force* source) {
  return guarded([&] {
    OMMB200_CTX;
    E.update_nonbonded(*nbf(source));
  });
}
int ommb200_context_update_gbsa_obc_parameters(ommb200_context* ctx, const ommb200_force* source) {
  return guarded([&] {
    OMMB200_CTX;
    E.update_gbsa(*force_of<GbsaObcDef, kGbsaObc>(source));
  });
}
int ommb200_context_checkpoint_size(const ommb200_context* ctx, int64_t* bytes) {
  return guarded([&] {
    require(ctx && ctx->engine && bytes, "null argument");
    *bytes = (int64_t)ctx->engine->checkpoint_bytes();
  });
}
int ommb200_context_create_checkpoint(ommb200_context* ctx, void* buffer, int64_t bytes) {
  return guarded([&] {
    OMMB200_CTX;
    require(buffer != nullptr && bytes >= 0, "invalid buffer");
    E.save_checkpoint(static_cast<uint8_t*>(buffer), (size_t)bytes);
  });
}
int ommb200_context_load_checkpoint(ommb200_context* ctx, const void* buffer, int64_t bytes) {
  return guarded([&] {
    OMMB200_CTX;
    require(buffer != nullptr && bytes >= 0, "invalid buffer");
    E.load_checkpoint(static_cast<const uint8_t*>(buffer), (size_t)bytes);
  });
}
int ommb200_context_get_learned_radii_stats(ommb200_context* ctx,
                                            ommb200_learned_radii_stats* out) {
  return guarded([&] {
    OMMB200_CTX;
    require(out != nullptr, "null output");
    E.learned_stats(out);
  });
}
int ommb200_context_get_radii_mlp_params(ommb200_context* ctx, float* params) {
  return guarded([&] {
    OMMB200_CTX;
    require(params != nullptr, "null output");
    E.learned_params(params);
  });
}
int ommb200_context_set_radii_mlp_params(ommb200_context* ctx, const float* params) {
  return guarded([&] {
    OMMB200_CTX;
    require(params != nullptr, "null input");
    for (int i = 0; i < OMMB200_RADII_MLP_PARAMS; ++i)
      require(std::isfinite(params[i]), "network parameters must be finite");
    E.set_learned_params(params);
  });
}
int ommb200_context_num_systems(const ommb200_context* ctx, int* out) {
  return guarded([&] {
    require(ctx && ctx->engine && out, "null argument");
    *out = ctx->engine->num_segments();
  });
}
int ommb200_context_system_range(const ommb200_context* ctx, int index, int* first, int* count) {
  return guarded([&] {
    require(ctx && ctx->engine && first && count, "null argument");
    require(index >= 0 && index < ctx->engine->num_segments(), "system index out of range");
    const Segment g = ctx->engine->segment(index);
    *first = g.first;
    *count = g.count;
  });
}
int ommb200_context_get_system_energies(ommb200_context* ctx, uint32_t groups, double* potential,
                                        double* kinetic) {
  return guarded([&] {
    OMMB200_CTX;
    E.segment_energies(groups, potential, kinetic);
  });
}
int ommb200_context_debug_pair_list(ommb200_context* ctx, int64_t max_pairs, int32_t* pairs,
                                    int64_t* count) {
  return guarded([&] {
    OMMB200_CTX;
    require(max_pairs >= 0 && count != nullptr, "invalid arguments");
    *count = E.debug_pair_list(max_pairs, pairs);
  });
}
int ommb200_context_set_profiling(ommb200_context* ctx, int enabled) {
  return guarded([&] {
    OMMB200_CTX;
    E.set_profiling(enabled != 0);
  });
}
int ommb200_context_kernel_times(ommb200_context* ctx, int max_entries, char* names, int names_len,
                                 double* ms, int* launches, int* count) {
  return guarded([&] {
    OMMB200_CTX;
    require(count != nullptr, "null count pointer");
    auto t = E.kernel_times();
    *count = (int)t.size();
    std::string joined;
    for (int i = 0; i < (int)t.size() && i < max_entries; ++i) {
      if (ms) ms[i] = t[i].ms;
      if (launches) launches[i] = t[i].launches;
      if (i) joined += ';';
      joined += t[i].name;
    }
    if (names && names_len > 0) {
      std::strncpy(names, joined.c_str(), names_len - 1);
      names[names_len - 1] = '\0';
    }
  });
}
int ommb200_context_autotune(ommb200_context* ctx, int trial_steps, double* skin,
                             int* pair_ctas_per_sm, double* ms_per_step) {
  return guarded([&] {
    OMMB200_CTX;
    E.autotune(trial_steps, skin, pair_ctas_per_sm, ms_per_step);
  });
}
int ommb200_context_get_tuning(ommb200_context* ctx, double* skin, int* pair_ctas_per_sm,
                               int* tile_entries) {
  return guarded([&] {
    OMMB200_CTX;
    E.tuning(skin, pair_ctas_per_sm, tile_entries);
  });
}
int ommb200_context_nlist_stats(ommb200_context* ctx, int* tiles, int* blocks, int* masked,
                                int64_t* rebuilds) {
  return guarded([&] {
    OMMB200_CTX;
    E.nlist_stats(tiles, blocks, masked, rebuilds);
  });
}
int ommb200_set_tensor_core_wait_limit(long long polls) {
  return guarded([&] { set_tensor_wait_limit(polls); });
}
int ommb200_context_nlist_capacity(ommb200_context* ctx, int* tile_capacity, int* column_capacity,
                                   int* regrows) {
  return guarded([&] {
    OMMB200_CTX;
    E.nlist_capacity(tile_capacity, column_capacity, regrows);
  });
}
int ommb200_context_nlist_prune_stats(ommb200_context* ctx, int* rebuild_tiles, int64_t* prunes,
                                      double* margin) {
  return guarded([&] {
    OMMB200_CTX;
    E.nlist_prune_stats(rebuild_tiles, prunes, margin);
  });
}
int ommb200_context_get_pair_cull(ommb200_context* ctx, int* tiles_per_run, int64_t* rounds) {
  return guarded([&] {
    OMMB200_CTX;
    E.pair_cull_stats(tiles_per_run, rounds);
  });
}
int ommb200_context_get_stream(ommb200_context* ctx, void** stream) {
  return guarded([&] {
    OMMB200_CTX;
    require(stream != nullptr, "null output pointer");
    *stream = (void*)E.stream();
  });
}
int ommb200_nonbonded_forces_noalloc(int n, const double* positions, const double* charges,
                                     const double* sigmas, const double* epsilons, int method,
                                     double cutoff, double reaction_field_dielectric,
                                     double* forces, double* energy, void* stream) {
  return guarded([&] {
    nonbonded_forces_noalloc(n, positions, charges, sigmas, epsilons, method, cutoff,
                             reaction_field_dielectric, forces, energy, (cudaStream_t)stream);
  });
}
int ommb200_measure_fp32_peak(int device, double* tflops) {
  return guarded([&] {
    require(tflops != nullptr, "null output pointer");
    *tflops = measure_fp32_peak(device);
  });
}

}  // extern "C"
