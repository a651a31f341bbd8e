// Host-side parameter objects; validation mirrors the reference's asserts, reported as
// OMMB200_ERR_INVALID_ARG instead of panics.
#include "model.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <set>

#include "../../include/ommb200.h"

namespace ommb200 {

static void require(bool ok, const char* msg, int code = OMMB200_ERR_INVALID_ARG) {
  if (!ok) throw Error(code, msg);
}

// nonbonded.rs:1245-1255
static void validate_particle_parameters(double q, double s, double e) {
  require(std::isfinite(q) && std::isfinite(s) && std::isfinite(e) && s >= 0.0 && e >= 0.0,
          "nonbonded parameters must be finite with nonnegative sigma and epsilon");
}

int NonbondedDef::add_particle(double q, double s, double e) {
  validate_particle_parameters(q, s, e);
  charge.push_back(q);
  sigma.push_back(s);
  epsilon.push_back(e);
  return (int)charge.size() - 1;
}

int NonbondedDef::add_exception(int p1, int p2, double qq, double s, double e) {
  validate_particle_parameters(qq, s, e);
  exceptions.push_back({p1, p2, qq, s, e});
  return (int)exceptions.size() - 1;
}

// nonbonded.rs:434-500: 1-2 and 1-3 pairs become exclusions, 1-4 pairs scaled exceptions.
void NonbondedDef::create_exceptions_from_bonds(const std::vector<std::pair<int, int>>& bonds,
                                                double coulomb14, double lj14) {
  const int n = (int)charge.size();
  std::vector<std::vector<int>> nb(n);
  for (auto& b : bonds) {
    require(b.first >= 0 && b.first < n && b.second >= 0 && b.second < n,
            "bonded particle index out of range");
    nb[b.first].push_back(b.second);
    nb[b.second].push_back(b.first);
  }
  std::set<std::pair<int, int>> excl, p14;
  for (int i = 0; i < n; ++i) {
    for (int j : nb[i])
      if (i < j) excl.insert({i, j});
    for (int j : nb[i])
      for (int k : nb[j])
        if (k != i) excl.insert({std::min(i, k), std::max(i, k)});
    for (int j : nb[i])
      for (int k : nb[j]) {
        if (k == i) continue;
        for (int l : nb[k]) {
          if (l == j || l == i) continue;
          std::pair<int, int> key{std::min(i, l), std::max(i, l)};
          if (!excl.count(key)) p14.insert(key);
        }
      }
  }
  for (auto& e : excl) add_exception(e.first, e.second, 0.0, 0.5 * (sigma[e.first] + sigma[e.second]), 0.0);
  for (auto& p : p14) {
    if (excl.count(p)) continue;
    add_exception(p.first, p.second, coulomb14 * charge[p.first] * charge[p.second],
                  0.5 * (sigma[p.first] + sigma[p.second]),
                  lj14 * std::sqrt(epsilon[p.first] * epsilon[p.second]));
  }
}

void NonbondedDef::effective_pme_parameters(const double box[9], double* alpha, int dims[3]) const {
  if (pme_alpha > 0.0) {
    *alpha = pme_alpha;
    for (int a = 0; a < 3; ++a) dims[a] = pme_grid[a];
    return;
  }
  const double a = std::sqrt(-std::log(2.0 * ewald_error_tolerance)) / cutoff;
  *alpha = a;
  for (int axis = 0; axis < 3; ++axis) {
    double d = std::ceil(2.0 * a * box[3 * axis + axis] /
                         (3.0 * std::pow(ewald_error_tolerance, 0.2)));
    dims[axis] = (int)std::max(d, 6.0);
  }
}

int SystemDef::add_particle(double mass) {
  require(std::isfinite(mass) && mass >= 0.0, "particle mass must be nonnegative and finite");
  masses.push_back(mass);
  return (int)masses.size() - 1;
}

int SystemDef::add_constraint(int p1, int p2, double distance) {
  constraints.push_back({p1, p2, distance});
  return (int)constraints.size() - 1;
}

void validate_box(const double b[9]) {
  require(b[1] == 0.0 && b[2] == 0.0, "first periodic box vector must be parallel to x");
  require(b[5] == 0.0, "second periodic box vector must be in the x-y plane");
  require(b[0] > 0.0 && b[4] > 0.0 && b[8] > 0.0 && b[0] >= 2.0 * std::fabs(b[3]) &&
              b[0] >= 2.0 * std::fabs(b[6]) && b[4] >= 2.0 * std::fabs(b[7]),
          "periodic box vectors must be in reduced form");
}

std::unique_ptr<SystemDef> merge_systems(std::vector<std::unique_ptr<SystemDef>> systems,
                                         std::vector<Segment>* segments) {
  require(!systems.empty(), "a batch needs at least one System");
  auto out = std::make_unique<SystemDef>();
  std::copy(systems[0]->box, systems[0]->box + 9, out->box);
  NonbondedDef* nb = nullptr;
  GbsaObcDef* gb = nullptr;
  HarmonicBondDef* hb = nullptr;
  HarmonicAngleDef* ha = nullptr;
  std::vector<int> kinds0;
  for (size_t k = 0; k < systems.size(); ++k) {
    SystemDef& s = *systems[k];
    require(s.masses.size() > 0, "every System of a batch needs particles");
    const int off = (int)out->masses.size();
    segments->push_back({off, (int)s.masses.size()});
    out->masses.insert(out->masses.end(), s.masses.begin(), s.masses.end());
    for (auto& c : s.constraints) out->constraints.push_back({c.p1 + off, c.p2 + off, c.distance});
    std::vector<int> kinds;
    for (auto& f : s.forces) kinds.push_back(f->kind);
    std::sort(kinds.begin(), kinds.end());
    kinds.erase(std::unique(kinds.begin(), kinds.end()), kinds.end());
    if (k == 0) kinds0 = kinds;
    require(kinds == kinds0, "every System of a batch must carry the same force kinds");
    for (auto& f : s.forces) {
      switch (f->kind) {
        case kNonbonded: {
          auto* src = static_cast<NonbondedDef*>(f.get());
          if (!nb) {
            nb = new NonbondedDef(*src);
            nb->charge.clear();
            nb->sigma.clear();
            nb->epsilon.clear();
            nb->exceptions.clear();
            nb->owned_by_system = true;
            out->forces.emplace_back(nb);
          }
          require(src->method == nb->method && src->cutoff == nb->cutoff &&
                      src->reaction_field_dielectric == nb->reaction_field_dielectric &&
                      src->use_switching == nb->use_switching &&
                      src->switching_distance == nb->switching_distance &&
                      src->force_group == nb->force_group &&
                      src->include_direct_space == nb->include_direct_space,
                  "the NonbondedForces of a batch must share their global settings");
          require((int)src->charge.size() == (int)s.masses.size(),
                  "NonbondedForce must have one parameter record per particle");
          nb->charge.insert(nb->charge.end(), src->charge.begin(), src->charge.end());
          nb->sigma.insert(nb->sigma.end(), src->sigma.begin(), src->sigma.end());
          nb->epsilon.insert(nb->epsilon.end(), src->epsilon.begin(), src->epsilon.end());
          for (auto e : src->exceptions) {
            e.p1 += off;
            e.p2 += off;
            nb->exceptions.push_back(e);
          }
          break;
        }
        case kGbsaObc: {
          auto* src = static_cast<GbsaObcDef*>(f.get());
          if (!gb) {
            gb = new GbsaObcDef(*src);
            gb->charge.clear();
            gb->radius.clear();
            gb->scale.clear();
            gb->owned_by_system = true;
            out->forces.emplace_back(gb);
          }
          require(src->method == gb->method && src->cutoff == gb->cutoff &&
                      src->solvent_dielectric == gb->solvent_dielectric &&
                      src->solute_dielectric == gb->solute_dielectric &&
                      src->surface_area_energy == gb->surface_area_energy &&
                      src->force_group == gb->force_group &&
                      src->learned.enabled == gb->learned.enabled &&
                      src->learned.judge_interval == gb->learned.judge_interval &&
                      src->learned.radius_tolerance == gb->learned.radius_tolerance &&
                      src->learned.train_steps == gb->learned.train_steps,
                  "the GBSAOBCForces of a batch must share their global settings");
          gb->charge.insert(gb->charge.end(), src->charge.begin(), src->charge.end());
          gb->radius.insert(gb->radius.end(), src->radius.begin(), src->radius.end());
          gb->scale.insert(gb->scale.end(), src->scale.begin(), src->scale.end());
          break;
        }
        case kHarmonicBond: {
          auto* src = static_cast<HarmonicBondDef*>(f.get());
          if (!hb) {
            hb = new HarmonicBondDef();
            hb->force_group = src->force_group;
            hb->use_pbc = src->use_pbc;
            hb->owned_by_system = true;
            out->forces.emplace_back(hb);
          }
          require(src->force_group == hb->force_group && src->use_pbc == hb->use_pbc,
                  "the HarmonicBondForces of a batch must share group and periodicity");
          for (auto b : src->bonds) hb->bonds.push_back({b.p1 + off, b.p2 + off, b.length, b.k});
          break;
        }
        case kMonteCarloBarostat:
          throw Error(OMMB200_ERR_UNSUPPORTED, "a batch cannot carry a MonteCarloBarostat");
        case kHarmonicAngle: {
          auto* src = static_cast<HarmonicAngleDef*>(f.get());
          if (!ha) {
            ha = new HarmonicAngleDef();
            ha->force_group = src->force_group;
            ha->use_pbc = src->use_pbc;
            ha->owned_by_system = true;
            out->forces.emplace_back(ha);
          }
          require(src->force_group == ha->force_group && src->use_pbc == ha->use_pbc,
                  "the HarmonicAngleForces of a batch must share group and periodicity");
          for (auto a : src->angles)
            ha->angles.push_back({a.p1 + off, a.p2 + off, a.p3 + off, a.angle, a.k});
          break;
        }
      }
    }
  }
  if (systems.size() > 1) {
    if (nb) require(!nb->periodic(), "a batch of several Systems must be non-periodic", OMMB200_ERR_UNSUPPORTED);
    if (gb) require(gb->method != 2, "a batch of several Systems must be non-periodic", OMMB200_ERR_UNSUPPORTED);
  }
  return out;
}

void SystemDef::set_default_box(const double a[3], const double b[3], const double c[3]) {
  double nb[9] = {a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]};
  validate_box(nb);
  std::copy(nb, nb + 9, box);
}

}  // namespace ommb200
