// Host-side parameter objects; validation mirrors the reference's asserts, reported as
// OMMB200_ERR_INVALID_ARG instead of panics.
#include "model.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <set>

#include "../../include/ommb200.h"

namespace ommb200 {

static void require(bool ok, const char* msg) {
  if (!ok) throw Error(OMMB200_ERR_INVALID_ARG, msg);
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

void SystemDef::set_default_box(const double a[3], const double b[3], const double c[3]) {
  double nb[9] = {a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]};
  validate_box(nb);
  std::copy(nb, nb + 9, box);
}

}  // namespace ommb200
