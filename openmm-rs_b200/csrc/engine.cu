// Context engine: buffers, the per-step launch sequence and its CUDA graph, getState.
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <random>
#include <functional>
#include <set>

namespace ommb200 {

#define OMMB200_CK(call)                                                                    \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw Error(OMMB200_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)
#define OMMB200_CKFFT(call)                                                                 \
  do {                                                                                      \
    cufftResult r_ = (call);                                                                \
    if (r_ != CUFFT_SUCCESS)                                                                \
      throw Error(OMMB200_ERR_CUDA, std::string(#call) + ": cuFFT status " +                 \
                                        std::to_string((int)r_));                           \
  } while (0)

DeviceArena::~DeviceArena() {
  for (void* p : ptrs_) cudaFree(p);
}

void* DeviceArena::alloc_bytes(size_t bytes) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(e == cudaErrorMemoryAllocation ? OMMB200_ERR_OUT_OF_MEMORY : OMMB200_ERR_CUDA,
                std::string("device allocation of ") + std::to_string(bytes) +
                    " bytes failed: " + cudaGetErrorString(e));
  }
  ptrs_.push_back(p);
  OMMB200_CK(cudaMemset(p, 0, bytes));
  return p;
}

namespace {

// the message becomes a string only when the check fails (set_positions checks 3N values)
void require(bool ok, const char* msg, int code = OMMB200_ERR_INVALID_ARG) {
  if (!ok) throw Error(code, msg);
}

Box<double> make_box(const double b[9]) {
  Box<double> r;
  r.ax = b[0];
  r.bx = b[3];
  r.by = b[4];
  r.cx = b[6];
  r.cy = b[7];
  r.cz = b[8];
  r.inv_ax = 1.0 / r.ax;
  r.inv_by = 1.0 / r.by;
  r.inv_cz = 1.0 / r.cz;
  return r;
}

template <class Real>
Box<Real> cast_box(const Box<double>& b) {
  Box<Real> r;
  r.ax = (Real)b.ax;
  r.bx = (Real)b.bx;
  r.by = (Real)b.by;
  r.cx = (Real)b.cx;
  r.cy = (Real)b.cy;
  r.cz = (Real)b.cz;
  r.inv_ax = (Real)b.inv_ax;
  r.inv_by = (Real)b.inv_by;
  r.inv_cz = (Real)b.inv_cz;
  return r;
}

// pme.rs:176-199
void reciprocal_box(const double* bv, double recip[3][3], double* volume) {
  auto cross = [](const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  double bc[3], ca[3], ab[3];
  cross(bv + 3, bv + 6, bc);
  cross(bv + 6, bv, ca);
  cross(bv, bv + 3, ab);
  const double v = bv[0] * bc[0] + bv[1] * bc[1] + bv[2] * bc[2];
  for (int i = 0; i < 3; ++i) {
    recip[0][i] = bc[i] / v;
    recip[1][i] = ca[i] / v;
    recip[2][i] = ab[i] / v;
  }
  *volume = v;
}

// pme.rs:151-174 (host copy, used for the B-spline moduli)
void spline5_host(double f, double w[5]) {
  w[0] = 1.0 - f;
  w[1] = f;
  w[2] = w[3] = w[4] = 0.0;
  for (int order = 3; order <= 5; ++order) {
    const double den = order - 1;
    w[order - 1] = f * w[order - 2] / den;
    for (int i = order - 2; i >= 1; --i)
      w[i] = ((f + (order - 1 - i)) * w[i - 1] + ((i + 1) - f) * w[i]) / den;
    w[0] *= (1.0 - f) / den;
  }
}

// pme.rs:240-259
std::vector<double> bspline_moduli(int n) {
  double w[5];
  spline5_host(0.0, w);
  std::vector<double> v(n);
  for (int k = 0; k < n; ++k) {
    double re = 0.0, im = 0.0;
    for (int i = 0; i < 5; ++i) {
      const double ang = 2.0 * kPiD * (double)k * (double)i / (double)n;
      re += w[i] * std::cos(ang);
      im += w[i] * std::sin(ang);
    }
    v[k] = re * re + im * im;
  }
  for (int k = 0; k < n; ++k)
    if (v[k] < 1e-7) v[k] = 0.5 * (v[(k + n - 1) % n] + v[(k + 1) % n]);
  return v;
}

// nonbonded.rs:660-719 (no parameter offsets): E_disp = C / V.
double dispersion_coefficient(const NonbondedDef& nb) {
  double moments[13] = {0}, diagonal[13] = {0};
  for (size_t i = 0; i < nb.sigma.size(); ++i) {
    double power = 1.0;
    for (int k = 0; k <= 12; ++k) {
      moments[k] += std::sqrt(nb.epsilon[i]) * power;
      diagonal[k] += nb.epsilon[i] * power;
      power *= nb.sigma[i];
    }
  }
  auto pair_moment = [&](int power) {
    double coefficient = 1.0, sum = 0.0;
    for (int k = 0; k <= power; ++k) {
      sum += coefficient * moments[k] * moments[power - k];
      coefficient *= (double)(power - k) / (double)(k + 1);
    }
    return sum / std::pow(2.0, power) + diagonal[power];
  };
  const double rc = nb.cutoff, rs = nb.switching_distance;
  auto integral = [&](int power) {
    const double tail = std::pow(rc, 3 - power) / (double)(power - 3);
    if (!nb.use_switching) return tail;
    auto f = [&](double r) {
      const double t = (r - rs) / (rc - rs);
      return t * t * t * (10.0 + t * (-15.0 + 6.0 * t)) * std::pow(r, 2 - power);
    };
    // adaptive Simpson, nonbonded.rs:1290-1336
    struct S {
      static double rec(const decltype(f)& fn, double a, double b, double fa, double fm, double fb,
                        double est, double tol, int depth) {
        const double m = 0.5 * (a + b);
        const double fl = fn(0.5 * (a + m)), fr = fn(0.5 * (m + b));
        const double left = (m - a) / 6.0 * (fa + 4.0 * fl + fm);
        const double right = (b - m) / 6.0 * (fm + 4.0 * fr + fb);
        const double diff = left + right - est;
        if (depth == 0 || std::fabs(diff) <= 15.0 * tol) return left + right + diff / 15.0;
        return rec(fn, a, m, fa, fl, fm, left, 0.5 * tol, depth - 1) +
               rec(fn, m, b, fm, fr, fb, right, 0.5 * tol, depth - 1);
      }
    };
    const double fa = f(rs), fm = f(0.5 * (rs + rc)), fb = f(rc);
    const double est = (rc - rs) / 6.0 * (fa + 4.0 * fm + fb);
    return tail + S::rec(f, rs, rc, fa, fm, fb, est, 1e-11 * std::max(std::fabs(est), 1e-12), 20);
  };
  const double nn = (double)nb.sigma.size();
  return 8.0 * kPiD * nn / (nn + 1.0) *
         (pair_moment(12) * integral(12) - pair_moment(6) * integral(6));
}

}  // namespace

Engine::Engine(std::unique_ptr<SystemDef> system, std::unique_ptr<IntegratorDef> integrator,
               const EngineOptions& options, std::vector<Segment> segments)
    : sys_(std::move(system)), integ_(std::move(integrator)), opt_(options),
      segments_(std::move(segments)) {
  n_ = (int)sys_->masses.size();
  require(n_ > 0, "cannot create a context for a system with no particles");
  if (segments_.empty()) segments_.push_back({0, n_});
  dp_ = opt_.precision == OMMB200_PRECISION_DOUBLE;
  std::copy(sys_->box, sys_->box + 9, box_);
  int devices = 0;
  OMMB200_CK(cudaGetDeviceCount(&devices));
  require(opt_.device >= 0 && opt_.device < devices, "CUDA device ordinal out of range");
  OMMB200_CK(cudaSetDevice(opt_.device));
  OMMB200_CK(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, opt_.device));
  OMMB200_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  {
    // the reciprocal-space chain (spread, transform, gather) is a sequence of small kernels that
    // runs beside the pair kernel: its CTAs go ahead of queued pair CTAs
    int lowest = 0, greatest = 0;
    OMMB200_CK(cudaDeviceGetStreamPriorityRange(&lowest, &greatest));
    OMMB200_CK(cudaStreamCreateWithPriority(&pme_stream_, cudaStreamNonBlocking, greatest));
  }
  OMMB200_CK(cudaStreamCreateWithFlags(&aux_stream_, cudaStreamNonBlocking));
  OMMB200_CK(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
  OMMB200_CK(cudaEventCreateWithFlags(&join_ev_, cudaEventDisableTiming));
  if (integ_->random_seed != 0) {
    seed_ = (uint32_t)integ_->random_seed;
  } else {
    std::random_device rd;
    seed_ = ((uint64_t)rd() << 32) | rd();
  }
  host_masses_ = sys_->masses;
  pos_ = mem_.alloc<double>(3 * (size_t)n_);
  vel_ = mem_.alloc<double>(3 * (size_t)n_);
  scratch3_ = mem_.alloc<double>(3 * (size_t)n_);
  inv_mass_ = mem_.alloc<double>(n_);
  force_ = mem_.alloc<long long>(3 * (size_t)n_);
  energy_ = mem_.alloc<long long>(8 * segments_.size());
  status_ = mem_.alloc<int>(1);
  rebuild_ = mem_.alloc<int>(1);
  rng_step_ = mem_.alloc<unsigned long long>(1);
  std::vector<double> im(n_);
  for (int i = 0; i < n_; ++i) im[i] = host_masses_[i] == 0.0 ? 0.0 : 1.0 / host_masses_[i];
  OMMB200_CK(cudaMemcpy(inv_mass_, im.data(), sizeof(double) * n_, cudaMemcpyHostToDevice));

  const NonbondedDef* nb = nullptr;
  for (auto& f : sys_->forces) {
    switch (f->kind) {
      case kNonbonded:
        require(nb == nullptr, "only one NonbondedForce per System is supported",
                OMMB200_ERR_UNSUPPORTED);
        nb = static_cast<const NonbondedDef*>(f.get());
        break;
      case kGbsaObc:
        require(gb_def_ == nullptr, "only one GBSAOBCForce per System is supported",
                OMMB200_ERR_UNSUPPORTED);
        gb_def_ = static_cast<const GbsaObcDef*>(f.get());
        break;
      case kMonteCarloBarostat:
        require(bar_def_ == nullptr, "only one MonteCarloBarostat per System is supported",
                OMMB200_ERR_UNSUPPORTED);
        bar_def_ = static_cast<BarostatDef*>(f.get());
        break;
      default:
        break;
    }
    require(f->force_group >= 0 && f->force_group < 32, "force group must be in 0..31");
  }
  build_static_layout();
  if (nb) setup_nonbonded(*nb);
  if (gb_def_) setup_gbsa(*gb_def_);
  setup_bonded();
  setup_integrator();
  update_box_dependents();
  if (bar_def_) setup_barostat(*bar_def_);
  const int one = 1;
  OMMB200_CK(cudaMemcpy(rebuild_, &one, sizeof(int), cudaMemcpyHostToDevice));
}

Engine::~Engine() {
  destroy_graph();
  if (fft_ready_) {
    cufftDestroy(fft_fwd_);
    cufftDestroy(fft_inv_);
  }
  for (auto& p : pending_) {
    cudaEventDestroy(p.start);
    cudaEventDestroy(p.stop);
  }
  for (auto e : event_pool_) cudaEventDestroy(e);
  if (fork_ev_) cudaEventDestroy(fork_ev_);
  if (join_ev_) cudaEventDestroy(join_ev_);
  if (pme_stream_) cudaStreamDestroy(pme_stream_);
  if (aux_stream_) cudaStreamDestroy(aux_stream_);
  if (stream_) cudaStreamDestroy(stream_);
}

// nonbonded.rs:1055-1107 (initialize) + device layout.
void Engine::setup_nonbonded(const NonbondedDef& nb) {
  nb_ = &nb;
  require((int)nb.charge.size() == n_, "NonbondedForce must have one parameter record per particle");
  require(nb.method != kEwald && nb.method != kLJPME,
          "NonbondedForce methods Ewald and LJPME are not engine methods; use PME",
          OMMB200_ERR_UNSUPPORTED);
  require(nb.method >= kNoCutoff && nb.method <= kLJPME, "unknown nonbonded method");
  std::set<std::pair<int, int>> seen;
  for (auto& e : nb.exceptions) {
    require(e.p1 >= 0 && e.p1 < n_ && e.p2 >= 0 && e.p2 < n_, "exception particle index out of range");
    require(seen.insert({std::min(e.p1, e.p2), std::max(e.p1, e.p2)}).second, "duplicate exception pair");
  }
  if (nb.use_switching)
    require(nb.switching_distance >= 0.0 && nb.switching_distance < nb.cutoff,
            "switching distance must be between zero and cutoff");
  nb_periodic_ = nb.periodic();
  nb_pme_ = nb.method == kPME;
  elec_ = nb_pme_ ? kElecEwald : (nb.method == kNoCutoff ? kElecCoulomb : kElecReactionField);
  if (nb_periodic_) {
    validate_box(box_);
    for (int a = 0; a < 3; ++a)
      require(nb.cutoff <= 0.5 * box_[4 * a], "cutoff must not exceed half the periodic box size");
  }
  if (nb_pme_) {
    nb.effective_pme_parameters(box_, &alpha_, grid_);
    for (int a = 0; a < 3; ++a) require(grid_[a] >= 5, "PME grid dimensions must be at least five");
  }

  // per-particle parameters and exceptions (uploaded by upload_nonbonded_parameters)
  qscaled_ = mem_.alloc<double>(n_);
  charge_ = mem_.alloc<double>(n_);
  half_sigma_ = mem_.alloc<double>(n_);
  sqrt_eps_ = mem_.alloc<double>(n_);
  // exceptions: excluded from the pair kernel, evaluated in f64 (nonbonded.rs:995-1036)
  n_exceptions_ = (int)nb.exceptions.size();
  std::vector<int2> ep(std::max(n_exceptions_, 1));
  std::vector<std::vector<int>> partners(n_);
  for (int k = 0; k < n_exceptions_; ++k) {
    const auto& e = nb.exceptions[k];
    ep[k] = make_int2(e.p1, e.p2);
    partners[e.p1].push_back(e.p2);
    partners[e.p2].push_back(e.p1);
  }
  exc_pairs_ = mem_.alloc<int2>(ep.size());
  exc_params_ = mem_.alloc<double4>(ep.size());
  OMMB200_CK(cudaMemcpy(exc_pairs_, ep.data(), sizeof(int2) * ep.size(), cudaMemcpyHostToDevice));
  std::vector<int> xs(n_ + 1, 0), xl;
  for (int i = 0; i < n_; ++i) {
    xs[i] = (int)xl.size();
    xl.insert(xl.end(), partners[i].begin(), partners[i].end());
  }
  xs[n_] = (int)xl.size();
  int* excl_start = mem_.alloc<int>(n_ + 1);
  int* excl_list = mem_.alloc<int>(std::max<size_t>(xl.size(), 1));
  OMMB200_CK(cudaMemcpy(excl_start, xs.data(), 4 * (n_ + 1), cudaMemcpyHostToDevice));
  if (!xl.empty())
    OMMB200_CK(cudaMemcpy(excl_list, xl.data(), 4 * xl.size(), cudaMemcpyHostToDevice));

  // slots and tiles
  NlistArgs& a = nl_;
  a = NlistArgs{};
  a.n_atoms = n_;
  a.pos = pos_;
  a.excl_start = excl_start;
  a.excl_list = excl_list;
  a.rebuild = rebuild_;
  a.status = status_;
  a.periodic = nb_periodic_;
  a.cutoff = nb.cutoff;
  a.min_width = std::min(box_[0], std::min(box_[4], box_[8]));
  a.n_blocks = mem_.alloc<int>(1);
  a.rebuild_count = mem_.alloc<unsigned long long>(1);
  a.n_tiles = mem_.alloc<int>(1);
  a.n_masks = mem_.alloc<int>(1);
  if (nb_periodic_) {
    skin_ = opt_.skin > 0.0 ? opt_.skin : 0.1;
    a.skin = skin_;
    a.halves = 1;
    double recip[3][3], vol;
    reciprocal_box(box_, recip, &vol);
    const double density = n_ / vol;
    // x-y columns ~0.62 nm wide: z-sorted blocks of 32 become ~0.6 x 0.6 x 0.8 nm bricks.
    // Tall boxes get narrower columns so a column stays within the per-column sort's
    // shared-memory capacity (4096 keys).
    const double width = std::min(0.62, std::sqrt(1500.0 / (density * box_[8])));
    for (int d = 0; d < 2; ++d)
      a.n_col[d] = std::max(1, std::min(4096, (int)std::floor(box_[4 * d] / width)));
    a.n_cols = a.n_col[0] * a.n_col[1];
    const double col_area = (box_[0] / a.n_col[0]) * (box_[4] / a.n_col[1]);
    list_density_ = density;
    list_col_w_[0] = box_[0] / a.n_col[0];
    list_col_w_[1] = box_[4] / a.n_col[1];
    const double expected = density * col_area * box_[8];
    a.col_max = std::max(64, (int)std::min(4096.0, 2.5 * expected + 64));
    a.slot_capacity = ((n_ + 31 * a.n_cols) + 31) / 32 * 32;
    a.pos_ref = mem_.alloc<double>(3 * (size_t)n_);
    a.column = mem_.alloc<int>(n_);
    a.zkey = mem_.alloc<float>(n_);
    a.col_count = mem_.alloc<int>(a.n_cols);
    a.col_start = mem_.alloc<int>(a.n_cols + 1);
    a.col_scatter = mem_.alloc<int>(a.n_cols + 1);
    a.col_cursor = mem_.alloc<int>(a.n_cols);
    a.scratch_atoms = mem_.alloc<int>(n_);
    const long long blocks = a.slot_capacity / 32;
    // sized for the largest skin the autotuner may pick
    const double reach = nb.cutoff + std::max(skin_, kMaxTunedSkin);
    const double wx = box_[0] / a.n_col[0], wy = box_[4] / a.n_col[1];
    const double hz = 32.0 / (density * wx * wy);
    const double gathered = density * (wx + 2 * reach) * (wy + 2 * reach) * (hz + 2 * reach) / 2.0;
    // rectangular boxes pack 16 entries per half of a block and tile, triclinic ones 32
    const bool halves = box_[3] == 0.0 && box_[6] == 0.0 && box_[7] == 0.0;
    const double per_tile = halves ? 16.0 : 32.0;
    const long long per_block = (long long)(1.5 * gathered / per_tile) + 8;
    const bool small_box = a.min_width < 2.0 * (reach + 2.0);
    const long long all_pairs = (blocks * (blocks + 1) / 2 + blocks) * (halves ? 2 : 1);
    a.tile_capacity = (int)std::min<long long>(all_pairs, small_box ? all_pairs : blocks * per_block);
    // a masked tile holds an exclusion or a padding slot: at most one per exception plus two
    // per block (self tile, last partial neighbour tile) with 32-entry tiles; with halves a
    // block's longer half can leave several tiles half padded, so every tile gets a slot
    a.mask_capacity = halves ? a.tile_capacity
                             : (int)std::min<long long>(a.tile_capacity,
                                                        (long long)n_exceptions_ + 2 * blocks + 64);
  } else {
    a.slot_capacity = static_slots_;
    long long tiles = 0;
    for (const Segment& g : segments_) {
      const long long b = (g.count + 31) / 32;
      tiles += b * (b + 1) / 2;
    }
    a.tile_capacity = (int)tiles;
    a.mask_capacity = a.tile_capacity;
  }
  n_slots_ = a.slot_capacity;
  n_blocks_ = n_slots_ / 32;
  a.sorted_atom = mem_.alloc<int>(n_slots_);
  a.atom_slot = mem_.alloc<int>(n_);
  a.image = mem_.alloc<int>(3 * (size_t)n_);
  a.slot_wpos = mem_.alloc<double4>(n_slots_);
  a.block_center = mem_.alloc<double>(3 * (size_t)n_blocks_);
  a.block_half = mem_.alloc<double>(3 * (size_t)n_blocks_);
  if (nb_periodic_) {  // replaced by the first rebuild
    std::vector<int> sorted(n_slots_, -1);
    for (int i = 0; i < n_; ++i) sorted[i] = i;
    OMMB200_CK(cudaMemcpy(a.sorted_atom, sorted.data(), 4 * n_slots_, cudaMemcpyHostToDevice));
    OMMB200_CK(cudaMemcpy(a.atom_slot, sorted.data(), 4 * n_, cudaMemcpyHostToDevice));
  } else {
    OMMB200_CK(cudaMemcpy(a.sorted_atom, static_slot_atom_.data(), 4 * n_slots_, cudaMemcpyHostToDevice));
    OMMB200_CK(cudaMemcpy(a.atom_slot, static_atom_slot_.data(), 4 * n_, cudaMemcpyHostToDevice));
  }
  a.tiles = mem_.alloc<int4>(a.tile_capacity);
  a.entries = mem_.alloc_bytes((size_t)(dp_ ? 32 : 16) * 32 * (size_t)a.tile_capacity);
  a.masks = mem_.alloc<uint32_t>(32 * (size_t)a.mask_capacity);
  if (nb_periodic_) {  // the pruned pair list (used while pruning() holds)
    a.block_tiles = mem_.alloc<int>(2 * (size_t)(n_slots_ / 32));
    prune_flag_ = mem_.alloc<int>(1);
    pos_prune_ = mem_.alloc<double>(3 * (size_t)n_);
    prune_count_ = mem_.alloc<unsigned long long>(1);
    prune_n_tiles_ = mem_.alloc<int>(1);
    prune_done_ = mem_.alloc<unsigned>(1);
    a.prune = prune_flag_;
    prune_margin_ = opt_.prune_margin >= 0.0 ? opt_.prune_margin : kDefaultPruneMargin;
    if (prune_margin_ > 0.0) alloc_pruned_list();
    cull_tiles_ = opt_.pair_cull >= 0 ? opt_.pair_cull : 0;  // < 0: set by size below
    cull_work_ = mem_.alloc<int>(2);
    OMMB200_CK(cudaMemset(cull_work_, 0, 2 * sizeof(int)));
    cull_rounds_ = mem_.alloc<unsigned long long>(1);
    OMMB200_CK(cudaMemset(cull_rounds_, 0, sizeof(unsigned long long)));
  }
  posq_ = mem_.alloc_bytes((dp_ ? 32 : 16) * (size_t)n_slots_);
  ljp_ = mem_.alloc_bytes((dp_ ? 16 : 8) * (size_t)n_slots_);
  if (!nb_periodic_) build_static_tiles();
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, opt_.device);
  sm_count_ = dev_sms;
  pair_grid_ = dev_sms * 8;
  if (nb_periodic_ && opt_.pair_cull < 0) {  // by size: runs pay off with many tiles per warp
    const double tiles = 0.5 * tiles_per_block_max() * n_ / 32.0;
    const double warps = dev_sms * 5.0 * 4.0;  // resident warps of the culling kernel
    cull_tiles_ = tiles / warps >= kCullMinTilesPerWarp ? kDefaultCullTiles : 0;
  }

  if (nb_pme_) {
    const long long g = (long long)grid_[0] * grid_[1] * grid_[2];
    const long long gk = (long long)grid_[0] * grid_[1] * (grid_[2] / 2 + 1);
    const size_t rs = dp_ ? 8 : 4;
    pme_fixed_ = mem_.alloc<long long>(g);
    pme_real_ = mem_.alloc_bytes(rs * g);
    pme_k_ = mem_.alloc_bytes(2 * rs * gk);
    influence_ = mem_.alloc_bytes(rs * gk);
    moduli_ = mem_.alloc<double>(grid_[0] + grid_[1] + grid_[2]);
    // own transform while every axis factors into radices 2, 3, 4, 5, 7, 8 and the
    // plane kernels' buffers fit in shared memory; cuFFT otherwise
    own_fft_ = true;
    for (int d = 0; d < 3; ++d) {
      int m = grid_[d], k = 0;
      for (int r : {8, 4, 2, 3, 5, 7})
        while (m % r == 0 && k < 16) {
          fft_.rad[d][k++] = r;
          m /= r;
        }
      fft_.nrad[d] = k;
      if (m != 1) own_fft_ = false;
    }
    if (own_fft_) {
      fft_.pencils_x = 8;
      const int ny = grid_[1], nz = grid_[2], nzh = nz / 2 + 1, nyp = (ny + 1) / 2;
      auto items = [&](int d, int pencils) {  // most butterflies of one stage of axis d
        int most = 0;
        for (int k = 0; k < fft_.nrad[d]; ++k) most = std::max(most, pencils * grid_[d] / fft_.rad[d][k]);
        return most;
      };
      auto block = [](int want, int lo, int hi) { return std::min(hi, std::max(lo, (want + 31) / 32 * 32)); };
      // plane kernels: a third of a plane's elements per thread pass (copies), at least one
      // butterfly per thread in every stage (256-thread CTAs, which would fit beside the pair
      // kernel's CTAs, measured slower); x pass: at least the butterflies of a stage
      fft_.threads[0] = fft_.threads[2] =
          block(std::max(std::max(items(2, nyp), items(1, nzh)), nzh * ny / 3), 128, 512);
      fft_.threads[1] = block(std::max(items(0, fft_.pencils_x), fft_.pencils_x * grid_[0] / 4), 64, 256);
      PmeArgs<float> pf{};
      PmeArgs<double> pd{};
      pf.nx = pd.nx = grid_[0];
      pf.ny = pd.ny = grid_[1];
      pf.nz = pd.nz = grid_[2];
      const size_t need = dp_ ? std::max(pme_transform_smem(pd, fft_, 0), pme_transform_smem(pd, fft_, 1))
                              : std::max(pme_transform_smem(pf, fft_, 0), pme_transform_smem(pf, fft_, 1));
      own_fft_ = need <= 200 * 1024;
      if (own_fft_) {
        if (dp_)
          prepare_pme_transform(pd, fft_);
        else
          prepare_pme_transform(pf, fft_);
        OMMB200_CK(cudaGetLastError());
      }
    }
    if (own_fft_) {
      for (int d = 0; d < 3; ++d) {
        const int n = grid_[d];
        std::vector<double> tw(2 * (size_t)n);
        for (int m = 0; m < n; ++m) {
          const double ang = 2.0 * kPiD * (double)m / (double)n;
          tw[2 * m] = std::cos(ang);
          tw[2 * m + 1] = -std::sin(ang);
        }
        void* dtw = mem_.alloc_bytes((dp_ ? 16 : 8) * (size_t)n);
        if (dp_) {
          OMMB200_CK(cudaMemcpy(dtw, tw.data(), 16 * (size_t)n, cudaMemcpyHostToDevice));
        } else {
          std::vector<float> f(tw.begin(), tw.end());
          OMMB200_CK(cudaMemcpy(dtw, f.data(), 8 * (size_t)n, cudaMemcpyHostToDevice));
        }
        fft_.tw[d] = dtw;
      }
    } else {
      OMMB200_CKFFT(cufftPlan3d(&fft_fwd_, grid_[0], grid_[1], grid_[2], dp_ ? CUFFT_D2Z : CUFFT_R2C));
      OMMB200_CKFFT(cufftPlan3d(&fft_inv_, grid_[0], grid_[1], grid_[2], dp_ ? CUFFT_Z2D : CUFFT_C2R));
      fft_ready_ = true;
      OMMB200_CKFFT(cufftSetStream(fft_fwd_, stream_));
      OMMB200_CKFFT(cufftSetStream(fft_inv_, stream_));
    }
    std::vector<double> mod;
    for (int d = 0; d < 3; ++d) {
      auto m = bspline_moduli(grid_[d]);
      mod.insert(mod.end(), m.begin(), m.end());
    }
    OMMB200_CK(cudaMemcpy(moduli_, mod.data(), 8 * mod.size(), cudaMemcpyHostToDevice));
    if (nb_periodic_ && nl_.n_cols > 0) {  // the brick form's slot ranges
      for (int d = 0; d < 3; ++d) {
        bricks_.grid[d] = grid_[d];
        bricks_.nb[d] = (grid_[d] + kBrickEdge - 1) / kBrickEdge;
      }
      bricks_.n_col[0] = nl_.n_col[0];
      bricks_.n_col[1] = nl_.n_col[1];
      bricks_.ranges = mem_.alloc<int2>(2 * (size_t)nl_.n_cols * bricks_.nb[2]);
      bricks_.n_slots = nl_.slot_capacity;
      bricks_.base = mem_.alloc<int4>((size_t)nl_.slot_capacity);
      bricks_.frac = mem_.alloc_bytes((dp_ ? 32 : 16) * (size_t)nl_.slot_capacity);
    }
  }
  upload_nonbonded_parameters(nb);
}

// Per-particle parameters, exception parameters and the parameter-dependent constants (self
// energy, dispersion coefficient); the pair set and the tile masks do not depend on them.
void Engine::upload_nonbonded_parameters(const NonbondedDef& nb) {
  const double sk = std::sqrt(kOne4PiEps0);
  std::vector<double> qs(n_), hs(n_), se(n_);
  for (int i = 0; i < n_; ++i) {
    qs[i] = nb.charge[i] * sk;
    hs[i] = 0.5 * nb.sigma[i];
    se[i] = 2.0 * std::sqrt(nb.epsilon[i]);  // pair product = 4 sqrt(eps_i eps_j)
  }
  OMMB200_CK(cudaMemcpy(qscaled_, qs.data(), 8 * n_, cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(charge_, nb.charge.data(), 8 * n_, cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(half_sigma_, hs.data(), 8 * n_, cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(sqrt_eps_, se.data(), 8 * n_, cudaMemcpyHostToDevice));
  std::vector<double4> epar(std::max(n_exceptions_, 1));
  for (int k = 0; k < n_exceptions_; ++k) {
    const auto& e = nb.exceptions[k];
    epar[k] = make_double4(e.charge_prod * kOne4PiEps0, e.sigma, e.epsilon,
                           nb.charge[e.p1] * nb.charge[e.p2] * kOne4PiEps0);
  }
  OMMB200_CK(cudaMemcpy(exc_params_, epar.data(), sizeof(double4) * epar.size(), cudaMemcpyHostToDevice));
  dispersion_coeff_ =
      (nb_periodic_ && nb.use_dispersion_correction) ? dispersion_coefficient(nb) : 0.0;
  double q2 = 0.0;
  for (double q : nb.charge) q2 += q * q;
  self_energy_ = nb_pme_ ? -kOne4PiEps0 * alpha_ / std::sqrt(kPiD) * q2 : 0.0;
  if (nb_pme_ && volume_ > 0.0) {  // after Context creation: the neutralising term
    double qt = 0.0;
    for (double q : nb.charge) qt += q;
    plasma_energy_ = kOne4PiEps0 * kPiD * qt * qt / (2.0 * alpha_ * alpha_ * volume_);
  }
}

// context.rs:689-705 / nonbonded.rs:721-767: new particle and exception parameters, same
// particles, same exception pairs, and no excluded pair may become an interacting one.
void Engine::update_nonbonded(const NonbondedDef& src) {
  require(nb_ != nullptr, "the System has no NonbondedForce");
  NonbondedDef& nb = *const_cast<NonbondedDef*>(nb_);
  require(src.charge.size() == nb.charge.size(), "particle count must match");
  require(src.exceptions.size() == nb.exceptions.size(), "exception count must match");
  for (size_t k = 0; k < nb.exceptions.size(); ++k) {
    const ExceptionDef &o = nb.exceptions[k], &e = src.exceptions[k];
    require(o.p1 == e.p1 && o.p2 == e.p2, "exception particle indices must not change");
    require(o.charge_prod != 0.0 || o.epsilon != 0.0 || (e.charge_prod == 0.0 && e.epsilon == 0.0),
            "excluded exceptions cannot become non-excluded without reinitialization");
  }
  for (size_t i = 0; i < src.charge.size(); ++i)
    require(std::isfinite(src.charge[i]) && std::isfinite(src.sigma[i]) &&
                std::isfinite(src.epsilon[i]) && src.sigma[i] >= 0.0 && src.epsilon[i] >= 0.0,
            "nonbonded parameters must be finite with nonnegative sigma and epsilon");
  sync();
  nb.charge = src.charge;
  nb.sigma = src.sigma;
  nb.epsilon = src.epsilon;
  nb.exceptions = src.exceptions;
  upload_nonbonded_parameters(nb);
  if (packed_by_integrator()) {
    pack_slots(pos_, stream_);
    sync();
  }
}

// context.rs:680-687 / gbsa_obc.rs:134-141: new charges, radii and scale factors.
void Engine::update_gbsa(const GbsaObcDef& src) {
  require(gb_def_ != nullptr, "the System has no GBSAOBCForce");
  GbsaObcDef& g = *const_cast<GbsaObcDef*>(gb_def_);
  require(src.charge.size() == g.charge.size(), "particle count must match");
  for (size_t i = 0; i < src.charge.size(); ++i) {
    require(std::isfinite(src.charge[i]), "GBSA charges must be finite");
    require(std::isfinite(src.radius[i]) && src.radius[i] > 0.0,
            "GBSA radii must be positive and finite");
    require(std::isfinite(src.scale[i]) && src.scale[i] > 0.0,
            "GBSA scaling factors must be positive and finite");
  }
  sync();
  g.charge = src.charge;
  g.radius = src.radius;
  g.scale = src.scale;
  OMMB200_CK(cudaMemcpy(const_cast<double*>(gb_.charge), g.charge.data(), 8 * n_, cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(const_cast<double*>(gb_.radius), g.radius.data(), 8 * n_, cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(const_cast<double*>(gb_.scale), g.scale.data(), 8 * n_, cudaMemcpyHostToDevice));
}

// Segment-padded slot order and every block pair within one segment as a tile:
// non-periodic methods, built once.  Pairs across segments (independent systems of a batch)
// have no tile, so they never interact.
void Engine::build_static_tiles() {
  NlistArgs& a = nl_;
  std::vector<int4> tiles;
  std::vector<uint32_t> masks;
  std::vector<float4> entry_f;
  std::vector<double4> entry_d;
  std::vector<std::vector<int>> partners(n_);
  for (auto& e : nb_->exceptions) {
    partners[e.p1].push_back(e.p2);
    partners[e.p2].push_back(e.p1);
  }
  for (int I = 0; I < n_blocks_; ++I)
    for (int J = I; J < n_blocks_ && static_block_seg_[J] == static_block_seg_[I]; ++J) {
      uint32_t m[32];
      bool any = false;
      uint32_t pad = 0;
      for (int k = 0; k < 32; ++k)
        if (static_slot_atom_[32 * J + k] < 0) pad |= 1u << k;
      for (int l = 0; l < 32; ++l) {
        const int ai = static_slot_atom_[32 * I + l];
        uint32_t v = pad;
        if (ai < 0) {
          v = 0xffffffffu;
        } else {
          for (int p : partners[ai]) {
            const int sp = static_atom_slot_[p];
            if (sp / 32 == J) v |= 1u << (sp % 32);
          }
        }
        m[l] = v;
        any = any || v != 0;
      }
      int slot = -1, flags = I == J ? kTileSelf : 0;
      if (any) {
        slot = (int)(masks.size() / 32);
        masks.insert(masks.end(), m, m + 32);
        flags |= kTileHasMask;
      }
      tiles.push_back(make_int4(I, flags, slot, 0));
      // entries: the 32 slots of block J in its own (shared, unshifted) frame
      for (int k = 0; k < 32; ++k) {
        const int s = static_slot_atom_[32 * J + k] >= 0 ? 32 * J + k : -1;
        if (dp_) {
          entry_d.push_back(make_double4(0.0, 0.0, 0.0, (double)s));
        } else {
          float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
          std::memcpy(&e.w, &s, sizeof(int));
          entry_f.push_back(e);
        }
      }
    }
  const int nt = (int)tiles.size(), nm = (int)(masks.size() / 32);
  static_tile_count_ = nt;
  const int nb = n_blocks_;
  OMMB200_CK(cudaMemcpy(a.tiles, tiles.data(), sizeof(int4) * nt, cudaMemcpyHostToDevice));
  if (dp_)
    OMMB200_CK(cudaMemcpy(a.entries, entry_d.data(), sizeof(double4) * entry_d.size(), cudaMemcpyHostToDevice));
  else
    OMMB200_CK(cudaMemcpy(a.entries, entry_f.data(), sizeof(float4) * entry_f.size(), cudaMemcpyHostToDevice));
  if (nm) OMMB200_CK(cudaMemcpy(a.masks, masks.data(), 4 * masks.size(), cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(a.n_tiles, &nt, 4, cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(a.n_masks, &nm, 4, cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(a.n_blocks, &nb, 4, cudaMemcpyHostToDevice));
}

void Engine::setup_bonded() {
  for (auto& f : sys_->forces) {
    if (f->kind == kHarmonicBond) {
      auto* b = static_cast<const HarmonicBondDef*>(f.get());
      if (b->bonds.empty()) continue;
      std::vector<int2> idx;
      std::vector<double2> prm;
      for (auto& x : b->bonds) {
        require(x.p1 >= 0 && x.p1 < n_ && x.p2 >= 0 && x.p2 < n_, "bonded particle index out of range");
        idx.push_back(make_int2(x.p1, x.p2));
        prm.push_back(make_double2(x.length, x.k));
      }
      BondedLaunch L{};
      L.group = f->force_group;
      L.args.n_bonds = (int)idx.size();
      int2* di = mem_.alloc<int2>(idx.size());
      double2* dp = mem_.alloc<double2>(prm.size());
      OMMB200_CK(cudaMemcpy(di, idx.data(), sizeof(int2) * idx.size(), cudaMemcpyHostToDevice));
      OMMB200_CK(cudaMemcpy(dp, prm.data(), sizeof(double2) * prm.size(), cudaMemcpyHostToDevice));
      L.args.bonds = di;
      L.args.bond_params = dp;
      L.args.bond_pbc = b->use_pbc;
      bonded_.push_back(L);
    } else if (f->kind == kHarmonicAngle) {
      auto* g = static_cast<const HarmonicAngleDef*>(f.get());
      if (g->angles.empty()) continue;
      std::vector<int4> idx;
      std::vector<double2> prm;
      for (auto& x : g->angles) {
        require(x.p1 >= 0 && x.p1 < n_ && x.p2 >= 0 && x.p2 < n_ && x.p3 >= 0 && x.p3 < n_,
                "bonded particle index out of range");
        idx.push_back(make_int4(x.p1, x.p2, x.p3, 0));
        prm.push_back(make_double2(x.angle, x.k));
      }
      BondedLaunch L{};
      L.group = f->force_group;
      L.args.n_angles = (int)idx.size();
      int4* di = mem_.alloc<int4>(idx.size());
      double2* dp = mem_.alloc<double2>(prm.size());
      OMMB200_CK(cudaMemcpy(di, idx.data(), sizeof(int4) * idx.size(), cudaMemcpyHostToDevice));
      OMMB200_CK(cudaMemcpy(dp, prm.data(), sizeof(double2) * prm.size(), cudaMemcpyHostToDevice));
      L.args.angles = di;
      L.args.angle_params = dp;
      L.args.angle_pbc = g->use_pbc;
      bonded_.push_back(L);
    }
  }
  for (auto& L : bonded_) {
    L.args.pos = pos_;
    L.args.force = force_;
    L.args.energy = energy_;
    L.args.n_atoms_for_force = n_;
    L.args.atom_segment = segments_.size() > 1 ? d_atom_segment_ : nullptr;
  }
}

// Segment-padded slot order: segment s occupies a run of whole 32-slot blocks.
void Engine::build_static_layout() {
  static_slot_atom_.clear();
  static_block_seg_.clear();
  static_atom_slot_.assign(n_, -1);
  std::vector<int> atom_seg(n_, 0);
  for (size_t s = 0; s < segments_.size(); ++s) {
    const Segment g = segments_[s];
    require(g.first >= 0 && g.count > 0 && g.first + g.count <= n_, "invalid system range");
    const int start = (int)static_slot_atom_.size();
    const int padded = (g.count + 31) / 32 * 32;
    static_slot_atom_.resize(start + padded, -1);
    for (int i = 0; i < g.count; ++i) {
      static_slot_atom_[start + i] = g.first + i;
      static_atom_slot_[g.first + i] = start + i;
      atom_seg[g.first + i] = (int)s;
    }
    for (int b = 0; b < padded / 32; ++b) static_block_seg_.push_back((int)s);
  }
  static_slots_ = (int)static_slot_atom_.size();
  d_block_segment_ = mem_.alloc<int>(static_block_seg_.size());
  d_atom_segment_ = mem_.alloc<int>(n_);
  OMMB200_CK(cudaMemcpy(d_block_segment_, static_block_seg_.data(), 4 * static_block_seg_.size(),
                        cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(d_atom_segment_, atom_seg.data(), 4 * (size_t)n_, cudaMemcpyHostToDevice));
}

// gbsa_obc.rs:313-343 (initialize) + device layout: the segment-padded slot order, every
// block pair of a segment as a tile.
void Engine::setup_gbsa(const GbsaObcDef& g) {
  require((int)g.charge.size() == n_, "GBSA particle count must match System");
  for (int i = 0; i < n_; ++i) {
    require(std::isfinite(g.charge[i]), "GBSA charges must be finite");
    require(std::isfinite(g.radius[i]) && g.radius[i] > 0.0, "GBSA radii must be positive and finite");
    require(std::isfinite(g.scale[i]) && g.scale[i] > 0.0,
            "GBSA scaling factors must be positive and finite");
  }
  require(std::isfinite(g.solvent_dielectric) && std::isfinite(g.solute_dielectric) &&
              std::isfinite(g.surface_area_energy),
          "GBSA global settings must be finite");
  if (g.method != 0) require(std::isfinite(g.cutoff) && g.cutoff > 0.0, "GBSA cutoff must be positive and finite");
  if (g.method == 2) {
    validate_box(box_);
    for (int a = 0; a < 3; ++a)
      require(box_[4 * a] >= 2.0 * g.cutoff, "GBSA cutoff exceeds half a periodic box width");
  }
  GbArgs& a = gb_;
  a = GbArgs{};
  a.n_atoms = n_;
  a.n_slots = static_slots_;
  const int blocks = static_slots_ / 32;
  std::vector<int2> tiles;
  for (int I = 0; I < blocks; ++I)
    for (int J = I; J < blocks && static_block_seg_[J] == static_block_seg_[I]; ++J)
      tiles.push_back(make_int2(I, J));
  a.n_tiles = (int)tiles.size();
  int2* dt = mem_.alloc<int2>(tiles.size());
  int* dsa = mem_.alloc<int>(a.n_slots);
  OMMB200_CK(cudaMemcpy(dt, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(dsa, static_slot_atom_.data(), 4 * static_slot_atom_.size(),
                        cudaMemcpyHostToDevice));
  a.tiles = dt;
  a.slot_atom = dsa;
  a.block_segment = d_block_segment_;
  a.atom_segment = d_atom_segment_;
  double* q = mem_.alloc<double>(n_);
  double* r = mem_.alloc<double>(n_);
  double* s = mem_.alloc<double>(n_);
  OMMB200_CK(cudaMemcpy(q, g.charge.data(), 8 * n_, cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(r, g.radius.data(), 8 * n_, cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(s, g.scale.data(), 8 * n_, cudaMemcpyHostToDevice));
  a.pos = pos_;
  a.charge = q;
  a.radius = r;
  a.scale = s;
  // gbsa_obc.rs:214-218
  a.prefactor = (g.solute_dielectric != 0.0 && g.solvent_dielectric != 0.0)
                    ? -kOne4PiEps0 * (1.0 / g.solute_dielectric - 1.0 / g.solvent_dielectric)
                    : 0.0;
  a.prefactor_sign = a.prefactor < 0.0 ? -1.0 : (a.prefactor > 0.0 ? 1.0 : 0.0);
  a.charge_scale = std::sqrt(std::fabs(a.prefactor));
  a.surface = 4.0 * kPiD * g.surface_area_energy;
  a.periodic = g.method == 2;
  a.use_cutoff = g.method != 0;
  a.cutoff = g.cutoff;
  const size_t rs = dp_ ? 8 : 4;
  a.posq = mem_.alloc_bytes(4 * rs * a.n_slots);
  a.params = mem_.alloc_bytes(2 * rs * a.n_slots);
  a.born_slot = mem_.alloc_bytes(2 * rs * a.n_slots);  // R, 1 / R
  a.dedr_slot = mem_.alloc_bytes(rs * a.n_slots);
  a.born_sum = mem_.alloc<long long>(n_);
  a.dedr_sum = mem_.alloc<long long>(n_);
  a.born_radius = mem_.alloc<double>(n_);
  a.chain = mem_.alloc<double>(n_);
  a.dedr_self = mem_.alloc<double>(n_);
  a.force = force_;
  a.energy = energy_;
  // a NoCutoff NonbondedForce over the same segment-padded tiles joins GB pass 2 (one distance
  // and one force rotation per pair instead of two kernels)
  if (nb_ && nb_->method == kNoCutoff && !nb_periodic_ && g.method == 0 &&
      static_tile_count_ == a.n_tiles) {
    nb_gb_fusable_ = true;
    a.nb_tiles = nl_.tiles;
    a.nb_masks = nl_.masks;
    a.nb_charge = qscaled_;
    a.nb_half_sigma = half_sigma_;
    a.nb_two_sqrt_eps = sqrt_eps_;
    a.nb_params = mem_.alloc_bytes(4 * rs * a.n_slots);
  }
  if (g.learned.enabled) setup_learned(g.learned);
}

// Learned radii: per-block short-range lists over the segment-padded blocks, network
// parameters (deterministic Xavier-normal start from the seed) and training state.
void Engine::setup_learned(const LearnedRadiiDef& def) {
  require(gb_def_->method == 0, "learned Born radii need a NoCutoff GBSAOBCForce",
          OMMB200_ERR_UNSUPPORTED);
  learned_ = true;
  LearnedGbArgs& L = lr_;
  L = LearnedGbArgs{};
  L.n_atoms = n_;
  L.n_blocks = static_slots_ / 32;
  std::vector<int> first(L.n_blocks), count(L.n_blocks);
  int max_blocks = 1;
  for (int b = 0; b < L.n_blocks;) {
    int e = b;
    while (e < L.n_blocks && static_block_seg_[e] == static_block_seg_[b]) ++e;
    for (int k = b; k < e; ++k) {
      first[k] = b;
      count[k] = e - b;
    }
    max_blocks = std::max(max_blocks, e - b);
    b = e;
  }
  L.max_nbr = max_blocks;
  int* dfirst = mem_.alloc<int>(L.n_blocks);
  int* dcount = mem_.alloc<int>(L.n_blocks);
  OMMB200_CK(cudaMemcpy(dfirst, first.data(), 4 * first.size(), cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(dcount, count.data(), 4 * count.size(), cudaMemcpyHostToDevice));
  L.block_first = dfirst;
  L.block_count = dcount;
  L.block_box = mem_.alloc<float4>(2 * (size_t)L.n_blocks);
  L.nbr = mem_.alloc<int>((size_t)L.n_blocks * L.max_nbr);
  L.nbr_count = mem_.alloc<int>(2 * (size_t)L.n_blocks);
  L.rc = 2.0f;
  L.rs = 1.8f;
  L.rf = 1.2f;
  L.features = mem_.alloc<float>((size_t)n_ * kRadiiFeatures);
  L.tail = mem_.alloc<float>(n_);
  L.dtail = mem_.alloc<float>((size_t)n_ * kRadiiFeatures);
  L.short_sum = mem_.alloc<long long>(n_);
  L.params = mem_.alloc<float>(kRadiiMlpParams);
  L.moments = mem_.alloc<float>(2 * kRadiiMlpTrainable);
  L.adam_t = mem_.alloc<int>(1);
  L.snap_features = mem_.alloc<float>((size_t)n_ * kRadiiFeatures);
  L.snap_target = mem_.alloc<float>(n_);
  L.train_steps = def.train_steps;
  L.loss = mem_.alloc<float>(std::max(1, def.train_steps));
  L.batch = def.batch;
  L.judge_interval = def.judge_interval;
  L.learning_rate = (float)def.learning_rate;
  L.tolerance = (float)def.radius_tolerance;
  L.seed = (unsigned long long)(uint32_t)def.seed * 0x9E3779B97F4A7C15ull + 1ull;
  L.n_segments = (int)segments_.size();
  std::vector<int> sf, sc;
  for (const Segment& g : segments_) {
    sf.push_back(g.first);
    sc.push_back(g.count);
  }
  int* dsf = mem_.alloc<int>(sf.size());
  int* dsc = mem_.alloc<int>(sc.size());
  OMMB200_CK(cudaMemcpy(dsf, sf.data(), 4 * sf.size(), cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(dsc, sc.data(), 4 * sc.size(), cudaMemcpyHostToDevice));
  L.seg_first = dsf;
  L.seg_count = dsc;
  L.seg_offset = mem_.alloc<float>(sf.size());
  L.state = mem_.alloc<LearnedState>(1);
  L.step = rng_step_;
  L.status = status_;
  // Xavier-normal weights (Box-Muller on a 64-bit LCG stream), zero biases, identity
  // normalisation until the first judge fixes it
  std::vector<float> p(kRadiiMlpParams, 0.f);
  uint64_t st = L.seed;
  auto uniform = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return ((st >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  };
  auto normal = [&]() {
    const double u = uniform(), v = uniform();
    return std::sqrt(-2.0 * std::log(u)) * std::cos(2.0 * kPiD * v);
  };
  for (int i = 0; i < 32 * 64; ++i) p[i] = (float)(normal() / std::sqrt(32.0));
  for (int i = 0; i < 64 * 64; ++i) p[2112 + i] = (float)(normal() / std::sqrt(64.0));
  for (int i = 0; i < 64; ++i) p[6272 + i] = (float)(0.1 * normal() / std::sqrt(64.0));
  for (int f = 0; f < 32; ++f) p[kRadiiMlpOffInvStd + f] = 1.f;
  p[kRadiiMlpOffTScale] = 1.f;
  OMMB200_CK(cudaMemcpy(L.params, p.data(), 4 * p.size(), cudaMemcpyHostToDevice));
  gb_.use_learned = &L.state->use_learned;
  gb_.short_sum = L.short_sum;
  gb_.tail = L.tail;
  gb_.seg_offset = L.seg_offset;
}

void Engine::learned_stats(ommb200_learned_radii_stats* out) {
  *out = ommb200_learned_radii_stats{};
  if (!learned_) return;
  LearnedState st{};
  float loss = 0.f;
  OMMB200_CK(cudaMemcpyAsync(&st, lr_.state, sizeof(st), cudaMemcpyDeviceToHost, stream_));
  if (lr_.train_steps > 0)
    OMMB200_CK(cudaMemcpyAsync(&loss, lr_.loss + lr_.train_steps - 1, 4, cudaMemcpyDeviceToHost,
                               stream_));
  sync();
  out->judges = (int64_t)st.judges;
  out->learned_steps = (int64_t)st.learned_evals;
  out->exact_steps = (int64_t)st.exact_evals;
  out->active = st.active;
  out->last_radius_error = st.last_error;
  out->last_loss = loss;
}

void Engine::learned_params(float* out) {
  require(learned_, "the Context has no learned Born radii", OMMB200_ERR_UNSUPPORTED);
  OMMB200_CK(cudaMemcpyAsync(out, lr_.params, 4 * kRadiiMlpParams, cudaMemcpyDeviceToHost, stream_));
  sync();
}

// Installs given parameters (normalisation included) and trusts them until the next judge.
void Engine::set_learned_params(const float* in) {
  require(learned_, "the Context has no learned Born radii", OMMB200_ERR_UNSUPPORTED);
  OMMB200_CK(cudaMemcpyAsync(lr_.params, in, 4 * kRadiiMlpParams, cudaMemcpyHostToDevice, stream_));
  OMMB200_CK(cudaMemsetAsync(lr_.seg_offset, 0, 4 * (size_t)lr_.n_segments, stream_));
  LearnedState st{};
  OMMB200_CK(cudaMemcpyAsync(&st, lr_.state, sizeof(st), cudaMemcpyDeviceToHost, stream_));
  sync();
  st.initialized = 1;
  st.active = 1;
  OMMB200_CK(cudaMemcpyAsync(lr_.state, &st, sizeof(st), cudaMemcpyHostToDevice, stream_));
  sync();
}

// constraints.rs:35-75 validation, then SETTLE waters / free particles / SHAKE clusters.
void Engine::setup_integrator() {
  const IntegratorDef& it = *integ_;
  require(std::isfinite(it.temperature) && it.temperature >= 0.0, "temperature must be nonnegative and finite");
  require(std::isfinite(it.friction) && it.friction >= 0.0, "friction must be nonnegative and finite");
  require(std::isfinite(it.step_size) && it.step_size > 0.0, "step size must be positive and finite");
  std::set<std::pair<int, int>> seen;
  std::vector<ConstraintDef> active;
  for (auto& c : sys_->constraints) {
    require(c.p1 >= 0 && c.p1 < n_ && c.p2 >= 0 && c.p2 < n_ && c.p1 != c.p2,
            "constraint particle indices must be distinct and valid", OMMB200_ERR_CONSTRAINT);
    require(std::isfinite(c.distance) && c.distance > 0.0,
            "constraint distance must be positive and finite", OMMB200_ERR_CONSTRAINT);
    require(seen.insert({std::min(c.p1, c.p2), std::max(c.p1, c.p2)}).second,
            "duplicate constraint between the same particles", OMMB200_ERR_CONSTRAINT);
    require((host_masses_[c.p1] == 0.0) == (host_masses_[c.p2] == 0.0),
            "a constraint cannot connect a massive and massless particle", OMMB200_ERR_CONSTRAINT);
    if (host_masses_[c.p1] != 0.0) active.push_back(c);
  }
  // connected components of the constraint graph
  std::vector<int> parent(n_);
  std::iota(parent.begin(), parent.end(), 0);
  std::function<int(int)> root = [&](int x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  };
  for (auto& c : active) parent[root(c.p1)] = root(c.p2);
  std::map<int, std::vector<int>> comp_cons;
  std::map<int, std::set<int>> comp_atoms;
  for (size_t k = 0; k < active.size(); ++k) {
    const int r = root(active[k].p1);
    comp_cons[r].push_back((int)k);
    comp_atoms[r].insert(active[k].p1);
    comp_atoms[r].insert(active[k].p2);
  }
  std::vector<int4> waters;
  std::vector<int> free_atoms, cstart{0}, astart{0}, catoms;
  std::vector<int2> cpairs;
  std::vector<double> cd2;
  bool have_geom = false;
  auto same = [](double a, double b) { return std::fabs(a - b) <= 1e-12 * std::max(std::fabs(a), std::fabs(b)); };
  for (auto& kv : comp_cons) {
    const auto& cons = kv.second;
    const auto& atoms = comp_atoms[kv.first];
    bool is_water = false;
    if (cons.size() == 3 && atoms.size() == 3) {
      // the oxygen is the atom in two constraints of equal length
      for (int o : atoms) {
        std::vector<int> hs;
        std::vector<double> d_oh;
        double d_hh = -1.0;
        for (int k : cons) {
          const auto& c = active[k];
          if (c.p1 == o || c.p2 == o) {
            hs.push_back(c.p1 == o ? c.p2 : c.p1);
            d_oh.push_back(c.distance);
          } else {
            d_hh = c.distance;
          }
        }
        if (hs.size() != 2 || d_hh <= 0.0 || !same(d_oh[0], d_oh[1])) continue;
        if (!same(host_masses_[hs[0]], host_masses_[hs[1]])) continue;
        if (!(d_hh < 2.0 * d_oh[0])) continue;
        WaterGeometry g{d_oh[0], d_hh, host_masses_[o], host_masses_[hs[0]]};
        if (!have_geom) {
          geom_ = g;
          have_geom = true;
        }
        if (same(g.d_oh, geom_.d_oh) && same(g.d_hh, geom_.d_hh) && same(g.m_o, geom_.m_o) &&
            same(g.m_h, geom_.m_h)) {
          waters.push_back(make_int4(o, hs[0], hs[1], 0));
          is_water = true;
        }
        break;
      }
    }
    if (is_water) continue;
    for (int k : cons) {
      cpairs.push_back(make_int2(active[k].p1, active[k].p2));
      cd2.push_back(active[k].distance * active[k].distance);
    }
    cstart.push_back((int)cpairs.size());
    catoms.insert(catoms.end(), atoms.begin(), atoms.end());
    astart.push_back((int)catoms.size());
  }
  std::vector<char> constrained(n_, 0);
  for (auto& c : active) constrained[c.p1] = constrained[c.p2] = 1;
  for (int i = 0; i < n_; ++i)
    if (!constrained[i] && host_masses_[i] != 0.0) free_atoms.push_back(i);
  n_water_ = (int)waters.size();
  n_free_ = (int)free_atoms.size();
  n_clusters_ = (int)cstart.size() - 1;
  water_ = mem_.alloc<int4>(waters.size());
  free_atoms_ = mem_.alloc<int>(free_atoms.size());
  cluster_start_ = mem_.alloc<int>(cstart.size());
  cluster_pairs_ = mem_.alloc<int2>(cpairs.size());
  cluster_dist2_ = mem_.alloc<double>(cd2.size());
  cluster_atom_start_ = mem_.alloc<int>(astart.size());
  cluster_atoms_ = mem_.alloc<int>(catoms.size());
  auto up = [](void* d, const void* h, size_t bytes) {
    if (bytes) OMMB200_CK(cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice));
  };
  up(water_, waters.data(), sizeof(int4) * waters.size());
  up(free_atoms_, free_atoms.data(), 4 * free_atoms.size());
  up(cluster_start_, cstart.data(), 4 * cstart.size());
  up(cluster_pairs_, cpairs.data(), sizeof(int2) * cpairs.size());
  up(cluster_dist2_, cd2.data(), 8 * cd2.size());
  up(cluster_atom_start_, astart.data(), 4 * astart.size());
  up(cluster_atoms_, catoms.data(), 4 * catoms.size());
}

void Engine::update_box_dependents() {
  reciprocal_box(box_, recip_, &volume_);
  nl_.box = make_box(box_);
  nl_.min_width = std::min(box_[0], std::min(box_[4], box_[8]));
  nl_.max_cand = 0;
  if (nb_periodic_ && box_[3] == 0.0 && box_[6] == 0.0 && box_[7] == 0.0) {
    // candidate blocks of one block in the column-neighbourhood kernel, for the largest skin
    // the autotuner may pick.  At most every block of every column in reach; expected, per
    // column the blocks (each ~32 / (density * column area) tall) whose z-extent comes within
    // reach of I's, twice over.  The kernel keeps its candidates in shared memory, so the
    // expected count (not the bound) sets how many of its CTAs share an SM; a block with more
    // candidates reports an overflow and the list grows (`cand_scale_`).
    const double reach = nb_->cutoff + std::max(skin_, kMaxTunedSkin);
    const int nx = nl_.n_col[0], ny = nl_.n_col[1];
    const int kx = (int)std::floor(reach * nx / box_[0] + 1e-6) + 1;
    const int ky = (int)std::floor(reach * ny / box_[4] + 1e-6) + 1;
    const long long cols = (long long)std::min(nx, 2 * kx + 1) * std::min(ny, 2 * ky + 1);
    const long long bound = cols * (nl_.col_max / 32 + 1);
    const double column_area = (box_[0] / nx) * (box_[4] / ny);
    const double block_height = 32.0 / (n_ / volume_ * column_area);
    const double per_column = (2.0 * reach + 2.0 * block_height) / block_height + 2.0;
    const long long expected = (long long)std::ceil(2.0 * cand_scale_ * cols * per_column);
    const long long cand = std::min(bound, expected);
    if (cand * 48 <= 200 * 1024) nl_.max_cand = (int)cand;
  }
  for (auto& L : bonded_) L.args.box = make_box(box_);
  gb_.boxd = make_box(box_);
  gb_.boxf = cast_box<float>(gb_.boxd);
  if (!nb_) return;
  if (nb_pme_) {
    PmeRecip r;
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) r.m[a][c] = recip_[a][c];
    if (dp_)
      launch_pme_influence(static_cast<double*>(influence_), moduli_, grid_[0], grid_[1],
                           grid_[2], r, alpha_, volume_, stream_);
    else
      launch_pme_influence(static_cast<float*>(influence_), moduli_, grid_[0], grid_[1],
                           grid_[2], r, alpha_, volume_, stream_);
    OMMB200_CK(cudaGetLastError());
    double qt = 0.0;
    for (double q : nb_->charge) qt += q;
    plasma_energy_ = kOne4PiEps0 * kPiD * qt * qt / (2.0 * alpha_ * alpha_ * volume_);
  }
  update_bricks();
}

// Brick-owned PME gather (large grids in rectangular boxes): chosen while the box is rectangular,
// a brick's columns fit kBrickMaxRanges and the grid has at least two bricks per SM (or the
// option asks for it).  A change of choice drops the captured graph and asks for a rebuild (the
// slot ranges are made with the list).
void Engine::update_bricks() {
  const bool before = use_bricks_;
  bool use = false;
  if (bricks_.ranges && opt_.pme_bricks != 0 && box_[3] == 0.0 && box_[6] == 0.0 &&
      box_[7] == 0.0) {
    const double drift = 0.5 * std::max(skin_, kMaxTunedSkin), slack = 1e-3;
    int cols[2] = {1, 1};
    for (int d = 0; d < 3; ++d) {
      bricks_.len[d] = box_[4 * d];
      bricks_.cell[d] = box_[4 * d] / grid_[d];
      bricks_.below[d] = drift + slack;  // a stencil starting in the brick: its base point
    }
    bricks_.above = drift + slack;
    for (int d = 0; d < 2; ++d) {
      const double w = bricks_.len[d] / nl_.n_col[d];
      const double span = kBrickEdge * bricks_.cell[d] + bricks_.below[d] + bricks_.above;
      cols[d] = std::min(nl_.n_col[d], (int)std::floor(span / w) + 2);
    }
    const long long n = (long long)bricks_.nb[0] * bricks_.nb[1] * bricks_.nb[2];
    use = 2 * cols[0] * cols[1] <= kBrickMaxRanges &&
          (opt_.pme_bricks == 1 || n >= 2LL * sm_count_);
  }
  use_bricks_ = use;
  if (use == before) return;
  destroy_graph();
  const int one = 1;
  OMMB200_CK(cudaMemcpy(rebuild_, &one, 4, cudaMemcpyHostToDevice));
}

void Engine::destroy_graph() {
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  if (graph_) cudaGraphDestroy(graph_);
  graph_exec_ = nullptr;
  graph_ = nullptr;
  graph_steps_ = 0;
}

void Engine::sync() { OMMB200_CK(cudaStreamSynchronize(stream_)); }

int Engine::take_status() {
  int st = 0;
  OMMB200_CK(cudaMemcpy(&st, status_, sizeof(int), cudaMemcpyDeviceToHost));
  if (st == 0) return 0;
  const int zero = 0;
  OMMB200_CK(cudaMemcpy(status_, &zero, sizeof(int), cudaMemcpyHostToDevice));
  return st;
}

void Engine::check_status() { raise_status(take_status()); }

void Engine::raise_status(int st) {
  switch (st) {
    case 0:
      return;
    case kStatusTimeout:
      throw Error(OMMB200_ERR_TIMEOUT, "a tensor-core wait timed out");
    case kStatusConstraint:
      throw Error(OMMB200_ERR_CONSTRAINT, "constraint projection failed (no rigid solution or no convergence in 1000 iterations)");
    case kStatusNonfinite:
      throw Error(OMMB200_ERR_NONFINITE, "a position or velocity became nonfinite");
    case kStatusTileOverflow:
      throw Error(OMMB200_ERR_NLIST_OVERFLOW,
                  "neighbour tile list exceeded its capacity and cannot grow further");
    default:
      throw Error(OMMB200_ERR_CUDA, "device reported status " + std::to_string(st));
  }
}

bool Engine::grow_neighbor_capacity() {
  if (!nb_periodic_) return false;
  NlistArgs& a = nl_;
  int demand_tiles = 0, demand_masks = 0;
  OMMB200_CK(cudaMemcpy(&demand_tiles, a.n_tiles, sizeof(int), cudaMemcpyDeviceToHost));
  OMMB200_CK(cudaMemcpy(&demand_masks, a.n_masks, sizeof(int), cudaMemcpyDeviceToHost));
  bool grew = false;
  // per-column sort: the keys of one column live in shared memory, at most 4096
  if (a.col_max < 4096) {
    a.col_max = std::min(4096, 2 * a.col_max);
    grew = true;
  }
  // tiles and masks: half again as many as the failed build asked for (it counts its whole
  // demand even past the capacity), and at least 1.5 times the current arrays
  const long long blocks = a.slot_capacity / 32;
  const long long all_pairs = (blocks * (blocks + 1) / 2 + blocks) * 2;
  const long long want =
      std::min<long long>(all_pairs, std::max<long long>(3LL * demand_tiles / 2, 3LL * a.tile_capacity / 2));
  if (want > a.tile_capacity && want < (1LL << 31) / 32) {
    a.tile_capacity = (int)want;
    a.tiles = mem_.alloc<int4>(a.tile_capacity);
    a.entries = mem_.alloc_bytes((size_t)(dp_ ? 32 : 16) * 32 * (size_t)a.tile_capacity);
    grew = true;
  }
  const long long want_masks = std::min<long long>(
      a.tile_capacity, std::max<long long>(3LL * demand_masks / 2, 3LL * a.mask_capacity / 2));
  if (want_masks > a.mask_capacity) {
    a.mask_capacity = (int)want_masks;
    a.masks = mem_.alloc<uint32_t>(32 * (size_t)a.mask_capacity);
    grew = true;
  }
  if (nl_.max_cand > 0 && cand_scale_ < 64) {  // the builder's candidate arrays
    cand_scale_ *= 2;
    grew = true;
  }
  if (!grew) return false;
  ++regrows_;
  if (prune_tiles_) alloc_pruned_list();  // the pruned list holds at most the rebuild's tiles
  update_box_dependents();  // the candidate capacity follows the column size
  destroy_graph();          // the captured launches hold the old arrays
  const int one = 1;
  OMMB200_CK(cudaMemcpy(rebuild_, &one, sizeof(int), cudaMemcpyHostToDevice));
  return true;
}

void Engine::prof_begin(const char* name) {
  if (!profiling_) return;
  if (event_pool_.size() < 2) {
    for (int k = 0; k < 64; ++k) {
      cudaEvent_t e;
      OMMB200_CK(cudaEventCreate(&e));
      event_pool_.push_back(e);
    }
  }
  current_prof_ = name;
  current_start_ = event_pool_.back();
  event_pool_.pop_back();
  OMMB200_CK(cudaEventRecord(current_start_, stream_));
}

void Engine::prof_end() {
  if (!profiling_ || !current_start_) return;
  cudaEvent_t stop = event_pool_.back();
  event_pool_.pop_back();
  OMMB200_CK(cudaEventRecord(stop, stream_));
  pending_.push_back({current_prof_, current_start_, stop});
  current_start_ = nullptr;
}

void Engine::harvest_profile() {
  for (auto& p : pending_) {
    float ms = 0.f;
    OMMB200_CK(cudaEventElapsedTime(&ms, p.start, p.stop));
    auto it = std::find_if(kernel_times_.begin(), kernel_times_.end(),
                           [&](const KernelTime& k) { return k.name == p.name; });
    if (it == kernel_times_.end()) kernel_times_.push_back({p.name, (double)ms, 1});
    else {
      it->ms += ms;
      it->launches += 1;
    }
    event_pool_.push_back(p.start);
    event_pool_.push_back(p.stop);
  }
  pending_.clear();
}

void Engine::set_profiling(bool enabled) {
  profiling_ = enabled;
  kernel_times_.clear();
}

// In a captured step the neighbour-list rebuild is the body of an IF node whose condition a
// one-thread kernel copies from the rebuild flag, so steps without a rebuild skip its nine
// launches instead of running them as early-exit kernels.
void Engine::enqueue_conditional_rebuild() {
  cudaStreamCaptureStatus st;
  cudaGraph_t cap = nullptr;
  OMMB200_CK(cudaStreamGetCaptureInfo(stream_, &st, nullptr, &cap, nullptr, nullptr));
  cudaGraphConditionalHandle handle;
  OMMB200_CK(cudaGraphConditionalHandleCreate(&handle, cap, 0, cudaGraphCondAssignDefault));
  launch_nlist_condition(nl_, handle, stream_);
  enqueue_conditional_body(handle, [&](cudaStream_t s) {
    launch_nlist_rebuild(nl_, dp_, s, with_new_list(nl_));
  });
}

// An IF node at the current point of the captured stream; its body is `body`'s launches,
// captured on the auxiliary stream, and runs when `handle` (set by a kernel just before) is set.
void Engine::enqueue_conditional_body(cudaGraphConditionalHandle handle,
                                      const std::function<void(cudaStream_t)>& body) {
  cudaStreamCaptureStatus st;
  cudaGraph_t cap = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  OMMB200_CK(cudaStreamGetCaptureInfo(stream_, &st, nullptr, &cap, &deps, &nd));
  cudaGraphNodeParams params{};
  params.type = cudaGraphNodeTypeConditional;
  params.conditional.handle = handle;
  params.conditional.type = cudaGraphCondTypeIf;
  params.conditional.size = 1;
  cudaGraphNode_t node;
  OMMB200_CK(cudaGraphAddNode(&node, cap, deps, nd, &params));
  OMMB200_CK(cudaStreamUpdateCaptureDependencies(stream_, &node, 1,
                                                 cudaStreamSetCaptureDependencies));
  cudaGraph_t graph = params.conditional.phGraph_out[0];
  OMMB200_CK(cudaStreamBeginCaptureToGraph(aux_stream_, graph, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal));
  body(aux_stream_);
  cudaGraph_t done = nullptr;
  OMMB200_CK(cudaStreamEndCapture(aux_stream_, &done));
}

bool Engine::culling() const {
  return cull_tiles_ > 0 && !dp_ && !pruning() && nb_periodic_ && nl_.block_tiles && nl_.halves &&
         nl_.max_cand > 0 && elec_ != kElecCoulomb && segments_.size() <= 1 && box_[3] == 0.0 &&
         box_[6] == 0.0 && box_[7] == 0.0;
}

double Engine::tiles_per_block_max() const {
  // entries per half block: particles within cutoff + skin of a wx x wy x hz/2 box (its
  // Minkowski sum with that sphere).  A block lists only the blocks after it, so the first
  // blocks of the order hold all of them, twice the mean
  const double a = list_col_w_[0], b = list_col_w_[1];
  const double c = 16.0 / std::max(1e-9, list_density_ * a * b);
  const double r = nb_->cutoff + skin_;
  const double vol = a * b * c + 2.0 * (a * b + b * c + c * a) * r + kPiD * (a + b + c) * r * r +
                     4.0 / 3.0 * kPiD * r * r * r;
  return 1.0 + list_density_ * vol / 16.0;
}

int Engine::cull_chunks() const {
  // runs cover the largest block with a margin, so the last one, which takes whatever is
  // left, stays short
  return std::max(1, (int)std::ceil(1.25 * tiles_per_block_max() / std::max(1, cull_tiles_)));
}

bool Engine::pruning() const {
  return prune_margin_ > 0.0 && prune_tiles_ && nb_periodic_ && nl_.block_tiles && nl_.halves && nl_.max_cand > 0 && box_[3] == 0.0 &&
         box_[6] == 0.0 && box_[7] == 0.0;
}

void Engine::ensure_pruned_list() {
  if (!prune_tiles_ && nl_.block_tiles) alloc_pruned_list();
}

void Engine::alloc_pruned_list() {
  prune_capacity_ = nl_.tile_capacity;
  prune_tiles_ = mem_.alloc<int4>(prune_capacity_);
  prune_entries_ = mem_.alloc_bytes((size_t)(dp_ ? 32 : 16) * 32 * (size_t)prune_capacity_);
  prune_masks_ = mem_.alloc<uint32_t>(32 * (size_t)prune_capacity_);
  prune_cols_ = mem_.alloc<uint32_t>(32 * (size_t)prune_capacity_);
  prune_keep_ = mem_.alloc<uint32_t>((size_t)prune_capacity_);
}

PruneArgs Engine::prune_args() const {
  PruneArgs p{};
  p.tiles = prune_tiles_;
  p.entries = prune_entries_;
  p.masks = prune_masks_;
  p.cols = prune_cols_;
  p.keep = prune_keep_;
  p.done = prune_done_;
  p.n_tiles = prune_n_tiles_;
  p.capacity = prune_capacity_;
  p.sm_count = sm_count_;
  p.prune = prune_flag_;
  p.pos_prune = pos_prune_;
  p.posq = posq_;
  const double reach = nb_->cutoff + prune_margin_ + kPruneAllowance;
  p.reach2 = reach * reach;
  p.prune_count = prune_count_;
  return p;
}

template <class Real>
void Engine::enqueue_nonbonded(bool energy, bool direct, bool reciprocal, bool dump, bool pairs) {
  const NonbondedDef& nb = *nb_;
  if (nb_periodic_) {
    prof_begin("nlist_rebuild");
    if (capturing_)
      enqueue_conditional_rebuild();
    else
      launch_nlist_rebuild(nl_, dp_, stream_, with_new_list(nl_));
    prof_end();
  }
  // fork: PME on its own stream (serialised on the main stream while profiling, so that
  // per-kernel events time one kernel at a time)
  const bool pme = reciprocal && nb_pme_;
  cudaStream_t ps = (pme && !profiling_) ? pme_stream_ : stream_;
  if (ps != stream_) {
    OMMB200_CK(cudaEventRecord(fork_ev_, stream_));
    OMMB200_CK(cudaStreamWaitEvent(ps, fork_ev_, 0));
  }
  // the reciprocal chain is enqueued first, so its kernels reach the GPU ahead of the direct
  // chain's (the two orders measured within run-to-run spread of each other)
  if (reciprocal && nb_pme_) {
    PmeArgs<Real> m{};
    m.n_atoms = n_;
    m.order = nl_.sorted_atom;
    m.n_order = n_slots_;
    m.pos = pos_;
    m.charge = charge_;
    m.nx = grid_[0];
    m.ny = grid_[1];
    m.nz = grid_[2];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) m.recip[r][c] = recip_[r][c];
    m.grid_fixed = pme_fixed_;
    m.grid_real = static_cast<Real*>(pme_real_);
    m.grid_k = pme_k_;
    m.influence = static_cast<const Real*>(influence_);
    m.moduli = moduli_;
    m.force = force_;
    m.energy = energy_;
    m.alpha = alpha_;
    m.volume = volume_;
    prof_begin("pme_spread");
    launch_pme_spread<Real>(m, ps);
    prof_end();
    if (own_fft_) {
      prof_begin("pme_transform");
      launch_pme_transform<Real>(m, fft_, energy, ps);
      prof_end();
    } else {
    prof_begin("pme_convert");
    launch_pme_convert<Real>(m, ps);
    prof_end();
    OMMB200_CKFFT(cufftSetStream(fft_fwd_, ps));
    OMMB200_CKFFT(cufftSetStream(fft_inv_, ps));
    prof_begin("pme_fft_forward");
    if (dp_)
      OMMB200_CKFFT(cufftExecD2Z(fft_fwd_, (cufftDoubleReal*)pme_real_, (cufftDoubleComplex*)pme_k_));
    else
      OMMB200_CKFFT(cufftExecR2C(fft_fwd_, (cufftReal*)pme_real_, (cufftComplex*)pme_k_));
    prof_end();
    prof_begin("pme_convolve");
    launch_pme_convolve<Real>(m, energy, ps);
    prof_end();
    prof_begin("pme_fft_inverse");
    if (dp_)
      OMMB200_CKFFT(cufftExecZ2D(fft_inv_, (cufftDoubleComplex*)pme_k_, (cufftDoubleReal*)pme_real_));
    else
      OMMB200_CKFFT(cufftExecC2R(fft_inv_, (cufftComplex*)pme_k_, (cufftReal*)pme_real_));
    prof_end();
    }
    prof_begin("pme_gather");
    if (use_bricks_) {
      launch_pme_brick_stencils<Real>(m, bricks_, nl_, ps);
      launch_pme_gather_bricks<Real>(m, bricks_, nl_, ps);
    } else
      launch_pme_gather<Real>(m, ps);
    prof_end();
  }
  // the exclusion corrections first: a small kernel that leaves SMs free while the reciprocal
  // chain starts beside it, before the pair kernel fills every SM
  if (direct && n_exceptions_) {
    ExceptionArgs e{};
    e.n = n_exceptions_;
    e.pairs = exc_pairs_;
    e.params = exc_params_;
    e.pos = pos_;
    e.force = force_;
    e.energy = energy_;
    e.atom_segment = segments_.size() > 1 ? d_atom_segment_ : nullptr;
    e.box = nl_.box;
    e.use_pbc = nb_periodic_ && nb.exceptions_use_pbc;
    e.ewald = nb_pme_;
    e.alpha = alpha_;
    e.n_atoms_for_force = n_;
    prof_begin("exceptions");
    launch_exceptions(e, energy, stream_);
    prof_end();
  }
  if (direct && pairs) {
    if (!packed_by_integrator()) {
      prof_begin("pack");
      launch_pack<Real>(n_slots_, nl_.sorted_atom, pos_, nl_.image, nl_.block_center, qscaled_,
                        half_sigma_, sqrt_eps_, posq_, ljp_, nl_.box, stream_);
      prof_end();
    }
    const bool pruned = pruning();
    if (pruned) {  // a pending prune (after a rebuild, or once a particle moved margin / 2)
      const PruneArgs pa = prune_args();
      prof_begin("nlist_prune");
      if (capturing_) {
        cudaStreamCaptureStatus st;
        cudaGraph_t cap = nullptr;
        OMMB200_CK(cudaStreamGetCaptureInfo(stream_, &st, nullptr, &cap, nullptr, nullptr));
        cudaGraphConditionalHandle handle;
        OMMB200_CK(cudaGraphConditionalHandleCreate(&handle, cap, 0, cudaGraphCondAssignDefault));
        launch_prune_condition(pa, handle, stream_);
        enqueue_conditional_body(handle, [&](cudaStream_t s) { launch_nlist_prune(nl_, pa, dp_, s); });
      } else {
        launch_nlist_prune(nl_, pa, dp_, stream_);
      }
      prof_end();
    }
    PairArgs<Real> p{};
    p.n_atoms = n_;
    p.sorted_atom = nl_.sorted_atom;
    p.pos = pos_;
    p.posq = posq_;
    p.ljp = ljp_;
    p.tiles = pruned ? prune_tiles_ : nl_.tiles;
    p.entries = pruned ? prune_entries_ : nl_.entries;
    p.masks = pruned ? prune_masks_ : nl_.masks;
    p.n_tiles = pruned ? prune_n_tiles_ : nl_.n_tiles;
    p.tile_capacity = pruned ? prune_capacity_ : nl_.tile_capacity;
    p.force = force_;
    p.energy = energy_;
    p.block_segment = segments_.size() > 1 ? d_block_segment_ : nullptr;
    p.box = cast_box<Real>(nl_.box);
    p.box_exact = nl_.box;
    p.periodic = nb_periodic_;
    p.use_cutoff = nb.method != kNoCutoff;
    const double rc = nb.cutoff;
    p.cutoff2 = (Real)(rc * rc);
    p.cutoff2_exact = rc * rc;
    p.band = (Real)(rc * rc * (dp_ ? 1e-10 : 1e-4));
    p.alpha = (Real)alpha_;
    // the FP32 kernel evaluates exp(-alpha^2 r^2) as exp2(-alpha^2 log2(e) r^2)
    p.exp_scale = (Real)(-alpha_ * alpha_ * (dp_ ? 1.0 : 1.4426950408889634));
    p.two_alpha_sqrtpi = (Real)(2.0 * alpha_ / std::sqrt(kPiD));
    if (elec_ == kElecReactionField) {
      const double eps = nb.reaction_field_dielectric, rc3 = rc * rc * rc;
      double krf, crf;
      if (std::isinf(eps)) {
        krf = 0.5 / rc3;
        crf = 1.5 / rc;
      } else {
        krf = (eps - 1.0) / (2.0 * eps + 1.0) / rc3;
        crf = (3.0 * eps) / (2.0 * eps + 1.0) / rc;
      }
      p.krf = (Real)krf;
      p.crf = (Real)crf;
    }
    p.use_switching = (nb.method != kNoCutoff) && nb.use_switching;
    if (p.use_switching) {
      p.switch_r = (Real)nb.switching_distance;
      p.switch_inv_width = (Real)(1.0 / (rc - nb.switching_distance));
    }
    p.pair_dump = dump_pairs_;
    p.pair_count = dump_count_;
    p.pair_capacity = dump_capacity_;
    if (culling()) {
      p.cull_tiles = cull_tiles_;
      p.cull_chunks = cull_chunks();
      // pairs at r^2 >= rc^2 + band are outside whatever the f64 decision says; the factor
      // covers the rounding of the sum
      p.cull2 = (Real)((rc * rc + (double)p.band) * (1.0 + 1e-5));
      p.n_blocks = nl_.n_blocks;
      p.block_tiles = nl_.block_tiles;
      p.cull_work = cull_work_;
      p.cull_rounds = cull_rounds_;
    }
    prof_begin("pair");
    launch_pair<Real>(p, elec_, energy, dump, pair_grid_, stream_);
    prof_end();
  }
  if (ps != stream_) {  // join
    OMMB200_CK(cudaEventRecord(join_ev_, ps));
    OMMB200_CK(cudaStreamWaitEvent(stream_, join_ev_, 0));
  }
}

void Engine::compute_forces(bool energy, uint32_t groups, bool in_step, int step_offset) {
  // inside a captured group of steps the previous step's integrator left the forces zeroed
  if (!(in_step && capturing_ && step_offset > 0)) {
    prof_begin("zero_forces");
    OMMB200_CK(cudaMemsetAsync(force_, 0, sizeof(long long) * 3 * (size_t)n_, stream_));
    prof_end();
  }
  gb_.fuse_nonbonded = 0;
  if (nb_) {
    const int g = nb_->force_group;
    const int rg = nb_->reciprocal_force_group < 0 ? g : nb_->reciprocal_force_group;
    const bool direct = nb_->include_direct_space && ((groups >> g) & 1u);
    const bool recip = nb_pme_ && ((groups >> rg) & 1u);
    // the pair terms go to GB pass 2 when both forces are evaluated (not while dumping pairs)
    const bool fuse = nb_gb_fusable_ && direct && !dump_mode_ &&
                      ((groups >> gb_def_->force_group) & 1u);
    gb_.fuse_nonbonded = fuse ? 1 : 0;
    if (dp_)
      enqueue_nonbonded<double>(energy, direct, recip, dump_mode_, !fuse);
    else
      enqueue_nonbonded<float>(energy, direct, recip, dump_mode_, !fuse);
  }
  if (gb_def_ && ((groups >> gb_def_->force_group) & 1u)) {
    auto gb = [&](int phase, const char* name) {
      prof_begin(name);
      if (dp_)
        launch_gbsa_phase<double>(gb_, phase, energy, sm_count_, stream_);
      else
        launch_gbsa_phase<float>(gb_, phase, energy, sm_count_, stream_);
      prof_end();
    };
    auto lr = [&](int phase, const char* name) {
      if (!learned_) return;
      prof_begin(name);
      if (dp_)
        launch_learned_phase<double>(lr_, gb_, phase, sm_count_, stream_);
      else
        launch_learned_phase<float>(lr_, gb_, phase, sm_count_, stream_);
      prof_end();
    };
    if (learned_) {
      prof_begin("lr_control");
      launch_learned_control(lr_, in_step, step_offset, stream_);
      prof_end();
    }
    gb(kGbPack, "gb_pack");
    lr(kLrLists, "lr_lists");
    lr(kLrFeatures, "lr_features");
    lr(kLrInfer, "lr_infer");
    gb(kGbPass1, "gb_descreening");
    gb(kGbRadii, "gb_radii");
    gb(kGbPass2, "gb_pairs");
    gb(kGbChain, "gb_chain");
    gb(kGbPass3, "gb_descreening_forces");
    lr(kLrForces, "lr_forces");
    lr(kLrJudge, "lr_judge");
    lr(kLrTrain, "lr_train");
    lr(kLrOffsets, "lr_offsets");
  }
  for (auto& L : bonded_) {
    if (!((groups >> L.group) & 1u)) continue;
    prof_begin("bonded");
    launch_bonded(L.args, energy, stream_);
    prof_end();
  }
}

IntegrateArgs Engine::integrate_args(int step_offset) const {
  IntegrateArgs a{};
  a.n_atoms = n_;
  a.n_water = n_water_;
  a.water = water_;
  a.geom = geom_;
  a.n_free = n_free_;
  a.free_atoms = free_atoms_;
  a.n_clusters = n_clusters_;
  a.cluster_start = cluster_start_;
  a.cluster_pairs = cluster_pairs_;
  a.cluster_dist2 = cluster_dist2_;
  a.cluster_atom_start = cluster_atom_start_;
  a.cluster_atoms = cluster_atoms_;
  a.pos = pos_;
  a.vel = vel_;
  a.scratch = scratch3_;
  a.force = force_;
  a.inv_mass = inv_mass_;
  a.dt = integ_->step_size;
  a.decay = std::exp(-integ_->friction * integ_->step_size);
  a.noise_var = kBoltzmann * integ_->temperature * -std::expm1(-2.0 * integ_->friction * integ_->step_size);
  a.tolerance = integ_->constraint_tolerance;
  a.seed = seed_;
  a.rng_step = rng_step_;
  a.step_offset = step_offset;
  a.pos_ref = nb_periodic_ ? nl_.pos_ref : nullptr;
  a.half_skin2 = 0.25 * skin_ * skin_;
  a.rebuild = rebuild_;
  a.status = status_;
  if (pruning() && a.pos_ref) {
    a.pos_prune = pos_prune_;
    a.half_margin2 = 0.25 * prune_margin_ * prune_margin_;
    a.prune = prune_flag_;
  }
  return a;
}

void Engine::enqueue_step(int step_offset) {
  compute_forces(false, integ_->integration_force_groups, true, step_offset);
  IntegrateArgs a = integrate_args(step_offset);
  a.zero_force = 1;
  if (packed_by_integrator()) {
    a.posq = posq_;
    a.posq_double = dp_ ? 1 : 0;
    a.atom_slot = nl_.atom_slot;
    a.image = nl_.image;
    a.block_center = nl_.block_center;
    a.qscaled = qscaled_;
    a.pbox = nl_.box;
  }
  prof_begin("integrate");
  launch_integrate(a, stream_);
  prof_end();
}

// Periodic lists: the integrator writes the pair kernel's packed coordinates of the moved
// particles, and the pack kernel runs only with a rebuild (new slots, images and centres) or
// after new parameters or a checkpoint.  Every other change of the positions asks for a rebuild.
bool Engine::packed_by_integrator() const { return nb_ && nb_periodic_ && segments_.size() <= 1; }

std::function<void(cudaStream_t)> Engine::with_new_list(const NlistArgs& list) {
  return [this, list](cudaStream_t s) {
    if (use_bricks_) launch_pme_brick_ranges(list, bricks_, s);
    if (packed_by_integrator()) pack_slots(list.pos, s, list.rebuild);
  };
}

void Engine::pack_slots(const double* pos, cudaStream_t s, const int* only_after_rebuild) {
  if (dp_)
    launch_pack<double>(n_slots_, nl_.sorted_atom, pos, nl_.image, nl_.block_center, qscaled_,
                        half_sigma_, sqrt_eps_, posq_, ljp_, nl_.box, s, only_after_rebuild);
  else
    launch_pack<float>(n_slots_, nl_.sorted_atom, pos, nl_.image, nl_.block_center, qscaled_,
                       half_sigma_, sqrt_eps_, posq_, ljp_, nl_.box, s, only_after_rebuild);
}

void Engine::run_graph_steps(int launches) {
  const int k = graph_steps_;
  if (!graph_exec_) {
    OMMB200_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    capturing_ = true;
    try {
      for (int s = 0; s < k; ++s) enqueue_step(s);
      launch_advance_counter(rng_step_, k, stream_);
    } catch (...) {
      capturing_ = false;
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream_, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    capturing_ = false;
    OMMB200_CK(cudaStreamEndCapture(stream_, &graph_));
    OMMB200_CK(cudaGraphInstantiate(&graph_exec_, graph_, cudaGraphInstantiateFlagUseNodePriority));
  }
  for (int i = 0; i < launches; ++i) OMMB200_CK(cudaGraphLaunch(graph_exec_, stream_));
}

void Engine::step(int steps) {
  if (steps <= 0) return;
  if (!bar_def_) {
    run_steps(steps);
    return;
  }
  // the barostat counts every step and moves at the start of the step that brings its
  // counter to the frequency, read live (barostat.rs:76-81, context.rs:904)
  int done = 0;
  while (done < steps) {
    const uint64_t f = (uint64_t)std::max(0, bar_def_->frequency);
    int chunk = steps - done;
    if (f > 0) chunk = (int)std::min<uint64_t>(chunk, bar_counter_ + 1 >= f ? 0 : f - 1 - bar_counter_);
    if (chunk > 0) {
      run_steps(chunk);
      bar_counter_ += (uint64_t)chunk;
      done += chunk;
      continue;
    }
    bar_counter_ = 0;
    barostat_move();
    run_steps(1);
    done += 1;
  }
}

// A batch of steps that overflows the periodic neighbour list (a density fluctuation, a clumpy
// start) is not lost: the list's capacities grow, the state saved at the start of the batch is
// restored and the batch runs again.  Forces do not depend on the tile list (the pair set is
// decided pair by pair, the sums are fixed point), so the re-run is the run that had enough room.
void Engine::run_steps(int steps) {
  const int k = opt_.steps_per_graph > 0 ? opt_.steps_per_graph : 20;
  for (int attempt = 0;; ++attempt) {
    const bool guarded = nb_periodic_;
    if (guarded) save_dynamic_state(step_snapshot_);
    int remaining = steps;
    if (opt_.use_graph && !profiling_ && steps >= k) {
      if (graph_steps_ != k) destroy_graph();
      graph_steps_ = k;
      run_graph_steps(steps / k);
      remaining = steps % k;
    }
    for (int s = 0; s < remaining; ++s) {
      enqueue_step(0);
      launch_advance_counter(rng_step_, 1, stream_);
    }
    OMMB200_CK(cudaGetLastError());
    sync();
    harvest_profile();
    const int st = take_status();
    if (st == kStatusTileOverflow && guarded && grow_neighbor_capacity()) {
      restore_dynamic_state(step_snapshot_);
      continue;
    }
    time_ += steps * integ_->step_size;
    step_count_ += steps;
    raise_status(st);
    return;
  }
}

void Engine::set_positions(const double* xyz) {
  for (size_t i = 0; i < 3 * (size_t)n_; ++i)
    require(std::isfinite(xyz[i]), "particle positions must be finite");  // neighbors.rs:107-110
  OMMB200_CK(cudaMemcpyAsync(pos_, xyz, sizeof(double) * 3 * (size_t)n_, cudaMemcpyHostToDevice, stream_));
  const int one = 1;
  OMMB200_CK(cudaMemcpyAsync(rebuild_, &one, sizeof(int), cudaMemcpyHostToDevice, stream_));
  sync();
}

void Engine::set_velocities(const double* v) {
  OMMB200_CK(cudaMemcpyAsync(vel_, v, sizeof(double) * 3 * (size_t)n_, cudaMemcpyHostToDevice, stream_));
  sync();
}

// context.rs:182-223
void Engine::set_velocities_to_temperature(double temperature, int seed) {
  require(std::isfinite(temperature) && temperature >= 0.0, "temperature must be nonnegative and finite");
  const uint64_t key = seed != 0 ? (uint64_t)(uint32_t)seed : seed_;
  std::vector<double> v(3 * (size_t)n_, 0.0);
  const uint64_t draw = velocity_draws_++;
  for (int i = 0; i < n_; ++i) {
    if (host_masses_[i] == 0.0) continue;
    uint32_t c[4] = {(uint32_t)i, (uint32_t)draw, (uint32_t)(draw >> 32), 1u};
    philox4x32_10(c, (uint32_t)key, (uint32_t)(key >> 32));
    const double s = 2.3283064365386962890625e-10;
    const double u0 = (c[0] + 0.5) * s, u1 = (c[1] + 0.5) * s, u2 = (c[2] + 0.5) * s, u3 = (c[3] + 0.5) * s;
    const double m0 = std::sqrt(-2.0 * std::log(u0)), m1 = std::sqrt(-2.0 * std::log(u2));
    const double scale = std::sqrt(kBoltzmann * temperature / host_masses_[i]);
    v[3 * i] = scale * m0 * std::cos(2.0 * kPiD * u1);
    v[3 * i + 1] = scale * m0 * std::sin(2.0 * kPiD * u1);
    v[3 * i + 2] = scale * m1 * std::cos(2.0 * kPiD * u3);
  }
  // LFMiddle velocity_time_offset = dt/2 (langevin.rs:204-206): v -= F/m * dt/2
  const double offset = 0.5 * integ_->step_size;
  compute_forces_checked(false, 0xffffffffu);
  std::vector<long long> f(3 * (size_t)n_);
  OMMB200_CK(cudaMemcpyAsync(f.data(), force_, 8 * f.size(), cudaMemcpyDeviceToHost, stream_));
  sync();
  for (int i = 0; i < n_; ++i) {
    if (host_masses_[i] == 0.0) continue;
    for (int c = 0; c < 3; ++c) v[3 * i + c] -= (double)f[(size_t)c * n_ + i] * kForceScaleInv / host_masses_[i] * offset;
  }
  set_velocities(v.data());
  apply_velocity_constraints(1e-5);
}

void Engine::set_box(const double b[9]) {
  validate_box(b);
  if (nb_ && nb_periodic_)
    for (int a = 0; a < 3; ++a)
      require(nb_->cutoff <= 0.5 * b[4 * a], "cutoff must not exceed half the periodic box size");
  std::copy(b, b + 9, box_);
  destroy_graph();
  update_box_dependents();
  const int one = 1;
  OMMB200_CK(cudaMemcpy(rebuild_, &one, sizeof(int), cudaMemcpyHostToDevice));
}

void Engine::apply_constraints(double tolerance) {
  require(std::isfinite(tolerance) && tolerance > 0.0 && tolerance < 1.0,
          "constraint tolerance must be finite and between zero and one", OMMB200_ERR_CONSTRAINT);
  OMMB200_CK(cudaMemcpyAsync(scratch3_, pos_, 24 * (size_t)n_, cudaMemcpyDeviceToDevice, stream_));
  IntegrateArgs a = integrate_args(0);
  a.tolerance = tolerance;
  launch_constrain_positions(a, scratch3_, stream_);
  const int one = 1;
  OMMB200_CK(cudaMemcpyAsync(rebuild_, &one, sizeof(int), cudaMemcpyHostToDevice, stream_));
  sync();
  check_status();
}

void Engine::apply_velocity_constraints(double tolerance) {
  require(std::isfinite(tolerance) && tolerance > 0.0 && tolerance < 1.0,
          "constraint tolerance must be finite and between zero and one", OMMB200_ERR_CONSTRAINT);
  IntegrateArgs a = integrate_args(0);
  a.tolerance = tolerance;
  launch_constrain_velocities(a, stream_);
  sync();
  check_status();
}

// Forces (into `forces`, may be null) and, with `energy`, the fixed-point energy/virial
// terms of every segment: [8 * segment + (energy, virial xx yy zz xy xz yz)].
// compute_forces with the energy sums zeroed first, synchronised, and run again after the
// neighbour list grew when it overflowed; any other device error is raised.
void Engine::compute_forces_checked(bool energy, uint32_t groups) {
  for (;;) {
    OMMB200_CK(cudaMemsetAsync(energy_, 0, 8 * segments_.size() * sizeof(long long), stream_));
    compute_forces(energy, groups);
    sync();
    const int st = take_status();
    if (st == kStatusTileOverflow && grow_neighbor_capacity()) continue;
    raise_status(st);
    return;
  }
}

std::vector<long long> Engine::evaluate(bool energy, uint32_t groups, double* forces) {
  const size_t nterms = 8 * segments_.size();
  compute_forces_checked(energy, groups);
  if (forces) {
    std::vector<long long> f(3 * (size_t)n_);
    OMMB200_CK(cudaMemcpyAsync(f.data(), force_, 8 * f.size(), cudaMemcpyDeviceToHost, stream_));
    sync();
    for (int i = 0; i < n_; ++i)
      for (int c = 0; c < 3; ++c) forces[3 * i + c] = (double)f[(size_t)c * n_ + i] * kForceScaleInv;
  }
  std::vector<long long> terms(nterms);
  OMMB200_CK(cudaMemcpyAsync(terms.data(), energy_, 8 * nterms, cudaMemcpyDeviceToHost, stream_));
  sync();
  harvest_profile();
  check_status();
  return terms;
}

void Engine::segment_energies(uint32_t groups, double* potential, double* kinetic) {
  const int ns = (int)segments_.size();
  if (ns == 1) {  // one system: the full getState energy, long-range corrections included
    ommb200_state_info info{};
    get_state(OMMB200_STATE_ENERGY, groups, nullptr, nullptr, nullptr, &info);
    if (potential) potential[0] = info.potential_energy;
    if (kinetic) kinetic[0] = info.kinetic_energy;
    return;
  }
  if (potential) {
    std::vector<long long> terms = evaluate(true, groups, nullptr);
    for (int s = 0; s < ns; ++s) potential[s] = (double)terms[8 * s] * kEnergyScaleInv;
  }
  if (kinetic) {
    std::vector<double> v(3 * (size_t)n_);
    OMMB200_CK(cudaMemcpyAsync(v.data(), vel_, 24 * (size_t)n_, cudaMemcpyDeviceToHost, stream_));
    sync();
    for (int s = 0; s < ns; ++s) {
      double ke = 0.0;
      for (int i = segments_[s].first; i < segments_[s].first + segments_[s].count; ++i)
        ke += host_masses_[i] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
      kinetic[s] = 0.5 * ke;
    }
  }
}

void Engine::get_state(int flags, uint32_t groups, double* pos, double* vel, double* forces,
                       ommb200_state_info* info) {
  const bool need_forces = flags & (OMMB200_STATE_FORCES | OMMB200_STATE_ENERGY | OMMB200_STATE_VIRIAL);
  const bool need_energy = flags & (OMMB200_STATE_ENERGY | OMMB200_STATE_VIRIAL);
  long long e[8] = {0};
  if (need_forces) {
    std::vector<long long> terms = evaluate(need_energy, groups, forces);
    for (size_t k = 0; k < terms.size(); ++k) e[k % 8] += terms[k];
  }
  std::vector<double> vtmp;
  double* vout = vel;
  if (!vout && info) {
    vtmp.resize(3 * (size_t)n_);
    vout = vtmp.data();
  }
  if (pos) OMMB200_CK(cudaMemcpyAsync(pos, pos_, 24 * (size_t)n_, cudaMemcpyDeviceToHost, stream_));
  if (vout) OMMB200_CK(cudaMemcpyAsync(vout, vel_, 24 * (size_t)n_, cudaMemcpyDeviceToHost, stream_));
  sync();
  if (!info) return;
  info->time = time_;
  info->step_count = step_count_;
  std::copy(box_, box_ + 9, info->box);
  double ke = 0.0;
  for (int i = 0; i < n_; ++i)
    ke += host_masses_[i] * (vout[3 * i] * vout[3 * i] + vout[3 * i + 1] * vout[3 * i + 1] + vout[3 * i + 2] * vout[3 * i + 2]);
  info->kinetic_energy = 0.5 * ke;
  double w[6];
  const double pe = assemble_energy(e, need_energy ? groups : 0u, w);
  info->potential_energy = need_energy ? pe : 0.0;
  const double vir[9] = {w[0], w[3], w[4], w[3], w[1], w[5], w[4], w[5], w[2]};
  std::copy(vir, vir + 9, info->virial);
}

double Engine::assemble_energy(const long long e[8], uint32_t groups, double w[6]) const {
  double pe = (double)e[0] * kEnergyScaleInv;
  for (int c = 0; c < 6; ++c) w[c] = (double)e[1 + c] * kEnergyScaleInv;
  if (groups && nb_) {
    const int g = nb_->force_group;
    const int rg = nb_->reciprocal_force_group < 0 ? g : nb_->reciprocal_force_group;
    const bool direct = nb_->include_direct_space && ((groups >> g) & 1u);
    const bool recip = nb_pme_ && ((groups >> rg) & 1u);
    if (recip) {
      pe += self_energy_ - plasma_energy_;
      for (int c = 0; c < 3; ++c) w[c] -= plasma_energy_;
    }
    if (direct && nb_periodic_ && nb_->use_dispersion_correction) {
      const double ed = dispersion_coeff_ / volume_;
      pe += ed;
      for (int c = 0; c < 3; ++c) w[c] += ed;
    }
  }
  return pe;
}

double Engine::potential_energy(uint32_t groups) {
  long long e[8] = {0};
  const std::vector<long long> terms = evaluate(true, groups, nullptr);
  for (size_t k = 0; k < terms.size(); ++k) e[k % 8] += terms[k];
  double w[6];
  return assemble_energy(e, groups, w);
}

// ---- MonteCarloBarostat ---------------------------------------------------------------------
// barostat.rs:198-213 (initialize) and context.rs:95-101; molecules as system.rs:100-141 finds
// them: particles joined by constraints and by HarmonicBondForce bonds, each molecule's atoms
// in increasing order, molecules ordered by their first atom.
void Engine::setup_barostat(BarostatDef& def) {
  bool periodic = nb_ && nb_periodic_;
  if (gb_def_ && gb_def_->method == 2) periodic = true;
  for (auto& f : sys_->forces) {
    if (f->kind == kHarmonicBond && static_cast<const HarmonicBondDef*>(f.get())->use_pbc)
      periodic = true;
    if (f->kind == kHarmonicAngle && static_cast<const HarmonicAngleDef*>(f.get())->use_pbc)
      periodic = true;
  }
  require(periodic, "a barostat cannot be used with a non-periodic system");
  bar_def_ = &def;
  bar_rigid_ = def.scale_molecules_as_rigid;
  bar_pressure_ = def.default_pressure;
  bar_temperature_ = def.default_temperature;
  bar_volume_scale_ = 0.01 * box_[0] * box_[4] * box_[8];
  bar_counter_ = bar_window_attempted_ = bar_window_accepted_ = 0;
  bar_attempted_ = bar_accepted_ = bar_draws_ = 0;
  if (def.random_seed == 0) {
    std::random_device rd;
    bar_seed_ = ((uint64_t)rd() << 32) | rd();
  } else {
    bar_seed_ = (uint64_t)(uint32_t)def.random_seed;
  }
  std::vector<int> parent(n_);
  std::iota(parent.begin(), parent.end(), 0);
  auto root = [&](int p) {
    while (parent[p] != p) {
      parent[p] = parent[parent[p]];
      p = parent[p];
    }
    return p;
  };
  auto join = [&](int a, int b) {
    a = root(a);
    b = root(b);
    parent[std::max(a, b)] = std::min(a, b);
  };
  for (auto& c : sys_->constraints) join(c.p1, c.p2);
  for (auto& f : sys_->forces)
    if (f->kind == kHarmonicBond)
      for (auto& b : static_cast<const HarmonicBondDef*>(f.get())->bonds) join(b.p1, b.p2);
  std::vector<std::vector<int>> groups(n_);
  for (int i = 0; i < n_; ++i) groups[root(i)].push_back(i);
  std::vector<int> start(1, 0), atoms;
  for (auto& g : groups) {
    if (g.empty()) continue;
    atoms.insert(atoms.end(), g.begin(), g.end());
    start.push_back((int)atoms.size());
  }
  n_molecules_ = (int)start.size() - 1;
  bar_scaled_ = bar_rigid_ ? n_molecules_ : n_;
  mol_start_ = mem_.alloc<int>(start.size());
  mol_atoms_ = mem_.alloc<int>(std::max<size_t>(1, atoms.size()));
  OMMB200_CK(cudaMemcpy(mol_start_, start.data(), 4 * start.size(), cudaMemcpyHostToDevice));
  OMMB200_CK(cudaMemcpy(mol_atoms_, atoms.data(), 4 * atoms.size(), cudaMemcpyHostToDevice));
  bar_saved_ = mem_.alloc<double>(3 * (size_t)n_);
  bar_last_ = ommb200_barostat_stats{};
  bar_last_.last_uniform = -1.0;
}

// The engine's own uniform stream for the barostat: Philox4x32-10 keyed by the seed, one
// counter value per draw, 53 bits per uniform in [0, 1).
double Engine::barostat_uniform() {
  uint32_t c[4] = {(uint32_t)bar_draws_, (uint32_t)(bar_draws_ >> 32), 0x6d636261u, 0u};
  philox4x32_10(c, (uint32_t)bar_seed_, (uint32_t)(bar_seed_ >> 32));
  ++bar_draws_;
  const uint64_t v = ((((uint64_t)c[0]) << 32) | c[1]) >> 11;
  return (double)v * (1.0 / 9007199254740992.0);
}

// barostat.rs:172-189: every 10 attempts the volume step shrinks by 1.1 below a quarter
// accepted and grows by 1.1 (at most 0.3 of the volume) above three quarters.
void Engine::barostat_record(bool accepted, double previous_volume) {
  ++bar_attempted_;
  bar_accepted_ += accepted ? 1 : 0;
  ++bar_window_attempted_;
  bar_window_accepted_ += accepted ? 1 : 0;
  bar_last_.last_accepted = accepted ? 1 : 0;
  if (bar_window_attempted_ >= 10) {
    const double fraction = (double)bar_window_accepted_ / (double)bar_window_attempted_;
    if (fraction < 0.25) {
      bar_volume_scale_ /= 1.1;
    } else if (fraction > 0.75) {
      bar_volume_scale_ = std::min(bar_volume_scale_ * 1.1, previous_volume * 0.3);
    } else {
      return;
    }
    bar_window_attempted_ = bar_window_accepted_ = 0;
  }
}

// barostat.rs:121-169 and context/program.rs:5-47: propose a uniform scaling of the box and
// the positions, compare the integrator's force groups' energy before and after, accept by
// the Metropolis test; a rejected move restores positions and box.
void Engine::barostat_move() {
  constexpr double kBarNm3ToKjPerMol = 0.0602214076;  // barostat.rs:13
  const uint32_t groups = integ_->integration_force_groups;
  const double v_old = box_[0] * box_[4] * box_[8];
  const double v_new = v_old + bar_volume_scale_ * 2.0 * (barostat_uniform() - 0.5);
  bar_last_.last_old_volume = v_old;
  bar_last_.last_new_volume = v_new;
  bar_last_.last_energy_change = 0.0;
  bar_last_.last_work = NAN;
  bar_last_.last_uniform = -1.0;
  if (!std::isfinite(v_new) || v_new <= 0.0) {
    barostat_record(false, v_old);
    return;
  }
  const double scale = std::cbrt(v_new / v_old);
  double old_box[9], new_box[9];
  std::copy(box_, box_ + 9, old_box);
  for (int k = 0; k < 9; ++k) new_box[k] = box_[k] * scale;
  // a box the cutoff no longer fits is not evaluated: the move is rejected
  bool fits = true;
  if (nb_ && nb_periodic_)
    for (int a = 0; a < 3; ++a) fits = fits && nb_->cutoff <= 0.5 * new_box[4 * a];
  if (gb_def_ && gb_def_->method == 2)
    for (int a = 0; a < 3; ++a) fits = fits && 2.0 * gb_def_->cutoff <= new_box[4 * a];
  if (!fits) {
    barostat_record(false, v_old);
    return;
  }
  const double e_old = potential_energy(groups);
  const size_t bytes = 24 * (size_t)n_;
  const int one = 1;
  OMMB200_CK(cudaMemcpyAsync(bar_saved_, pos_, bytes, cudaMemcpyDeviceToDevice, stream_));
  launch_scale_positions(pos_, n_, mol_start_, mol_atoms_, n_molecules_, scale, bar_rigid_, stream_);
  std::copy(new_box, new_box + 9, box_);
  update_box_dependents();
  OMMB200_CK(cudaMemcpyAsync(rebuild_, &one, sizeof(int), cudaMemcpyHostToDevice, stream_));
  const double e_new = potential_energy(groups);
  const double kt = kBoltzmann * bar_temperature_;
  const double work = (e_new - e_old) + bar_pressure_ * kBarNm3ToKjPerMol * (v_new - v_old) -
                      (double)bar_scaled_ * kt * std::log(v_new / v_old);
  bool accepted;
  if (std::isnan(work)) {
    accepted = false;
  } else if (work <= 0.0) {
    accepted = true;
  } else {
    const double u = barostat_uniform();
    bar_last_.last_uniform = u;
    accepted = kt > 0.0 && u <= std::exp(-work / kt);
  }
  bar_last_.last_energy_change = e_new - e_old;
  bar_last_.last_work = work;
  barostat_record(accepted, v_old);
  if (accepted) {
    destroy_graph();  // captured launches carry the old box
  } else {
    OMMB200_CK(cudaMemcpyAsync(pos_, bar_saved_, bytes, cudaMemcpyDeviceToDevice, stream_));
    std::copy(old_box, old_box + 9, box_);
    update_box_dependents();
    OMMB200_CK(cudaMemcpyAsync(rebuild_, &one, sizeof(int), cudaMemcpyHostToDevice, stream_));
  }
  sync();
  check_status();
}

void Engine::set_parameter(const std::string& name, double value) {
  if (bar_def_ && name == "MonteCarloPressure") {  // barostat.rs:253-257
    require(std::isfinite(value), "pressure must be finite");
    bar_pressure_ = value;
    return;
  }
  if (bar_def_ && name == "MonteCarloTemperature") {  // barostat.rs:258-264
    require(std::isfinite(value) && value >= 0.0, "temperature must be nonnegative and finite");
    bar_temperature_ = value;
    return;
  }
  throw Error(OMMB200_ERR_INVALID_ARG, "unknown global parameter '" + name + "'");
}

double Engine::get_parameter(const std::string& name) const {
  if (bar_def_ && name == "MonteCarloPressure") return bar_pressure_;
  if (bar_def_ && name == "MonteCarloTemperature") return bar_temperature_;
  throw Error(OMMB200_ERR_INVALID_ARG, "unknown global parameter '" + name + "'");
}

void Engine::barostat_stats(ommb200_barostat_stats* out) const {
  require(bar_def_ != nullptr, "the System has no MonteCarloBarostat");
  *out = bar_last_;
  out->attempted = bar_attempted_;
  out->accepted = bar_accepted_;
  out->volume_scale = bar_volume_scale_;
}

// The dynamic state a re-run must start from: positions, velocities, the random-stream
// counter and, with learned radii (they train during steps), the network, its optimiser and the
// control block.  Host-side time and step counts are untouched.
void Engine::save_dynamic_state(DynamicSnapshot& snap) {
  const size_t bytes = 24 * (size_t)n_;
  if (!snap.x) {
    snap.x = mem_.alloc<double>(3 * (size_t)n_);
    snap.v = mem_.alloc<double>(3 * (size_t)n_);
    if (learned_) snap.lr = mem_.alloc<float>(kRadiiMlpParams + 2 * kRadiiMlpTrainable + 1 + segments_.size());
  }
  OMMB200_CK(cudaMemcpyAsync(snap.x, pos_, bytes, cudaMemcpyDeviceToDevice, stream_));
  OMMB200_CK(cudaMemcpyAsync(snap.v, vel_, bytes, cudaMemcpyDeviceToDevice, stream_));
  OMMB200_CK(cudaMemcpyAsync(&snap.rng, rng_step_, 8, cudaMemcpyDeviceToHost, stream_));
  if (learned_) {
    const size_t at = kRadiiMlpParams + 2 * kRadiiMlpTrainable;
    OMMB200_CK(cudaMemcpyAsync(snap.lr, lr_.params, 4 * kRadiiMlpParams, cudaMemcpyDeviceToDevice, stream_));
    OMMB200_CK(cudaMemcpyAsync(snap.lr + kRadiiMlpParams, lr_.moments, 8 * kRadiiMlpTrainable,
                               cudaMemcpyDeviceToDevice, stream_));
    OMMB200_CK(cudaMemcpyAsync(snap.lr + at, lr_.adam_t, 4, cudaMemcpyDeviceToDevice, stream_));
    OMMB200_CK(cudaMemcpyAsync(snap.lr + at + 1, lr_.seg_offset, 4 * segments_.size(),
                               cudaMemcpyDeviceToDevice, stream_));
    OMMB200_CK(cudaMemcpyAsync(&snap.state, lr_.state, sizeof(snap.state), cudaMemcpyDeviceToHost,
                               stream_));
  }
  sync();
}

// Puts the saved state back and requests a neighbour-list rebuild from it.
void Engine::restore_dynamic_state(const DynamicSnapshot& snap) {
  const size_t bytes = 24 * (size_t)n_;
  OMMB200_CK(cudaMemcpyAsync(pos_, snap.x, bytes, cudaMemcpyDeviceToDevice, stream_));
  OMMB200_CK(cudaMemcpyAsync(vel_, snap.v, bytes, cudaMemcpyDeviceToDevice, stream_));
  OMMB200_CK(cudaMemcpyAsync(rng_step_, &snap.rng, 8, cudaMemcpyHostToDevice, stream_));
  const int one = 1;
  OMMB200_CK(cudaMemcpyAsync(rebuild_, &one, sizeof(int), cudaMemcpyHostToDevice, stream_));
  if (learned_) {
    const size_t at = kRadiiMlpParams + 2 * kRadiiMlpTrainable;
    OMMB200_CK(cudaMemcpyAsync(lr_.params, snap.lr, 4 * kRadiiMlpParams, cudaMemcpyDeviceToDevice, stream_));
    OMMB200_CK(cudaMemcpyAsync(lr_.moments, snap.lr + kRadiiMlpParams, 8 * kRadiiMlpTrainable,
                               cudaMemcpyDeviceToDevice, stream_));
    OMMB200_CK(cudaMemcpyAsync(lr_.adam_t, snap.lr + at, 4, cudaMemcpyDeviceToDevice, stream_));
    OMMB200_CK(cudaMemcpyAsync(lr_.seg_offset, snap.lr + at + 1, 4 * segments_.size(),
                               cudaMemcpyDeviceToDevice, stream_));
    OMMB200_CK(cudaMemcpyAsync(lr_.state, &snap.state, sizeof(snap.state), cudaMemcpyHostToDevice,
                               stream_));
  }
  sync();
}

void Engine::autotune(int trial_steps, double* skin_out, int* ctas_out, double* ms_out) {
  require(trial_steps > 0, "autotune needs a positive number of trial steps");
  DynamicSnapshot saved;
  save_dynamic_state(saved);
  const double time0 = time_;
  const int64_t steps0 = step_count_;
  const bool prof = profiling_;
  profiling_ = false;
  cudaEvent_t t0, t1;
  OMMB200_CK(cudaEventCreate(&t0));
  OMMB200_CK(cudaEventCreate(&t1));
  auto restore = [&]() {
    restore_dynamic_state(saved);
    time_ = time0;
    step_count_ = steps0;
  };
  auto trial = [&](double skin, int ctas) {
    skin_ = skin;
    nl_.skin = skin;
    pair_grid_ = sm_count_ * ctas;
    destroy_graph();
    restore();
    // barostat moves stay out of the trials (run_steps does not count barostat steps)
    run_steps(std::min(trial_steps, 40));  // warm-up, builds the graph
    OMMB200_CK(cudaEventRecord(t0, stream_));
    run_steps(trial_steps);
    OMMB200_CK(cudaEventRecord(t1, stream_));
    OMMB200_CK(cudaEventSynchronize(t1));
    float ms = 0.f;
    OMMB200_CK(cudaEventElapsedTime(&ms, t0, t1));
    return (double)ms / trial_steps;
  };
  double best_skin = skin_, best_ms = 1e30, best_margin = prune_margin_;
  int best_ctas = pair_grid_ / std::max(1, sm_count_);
  int best_halves = nl_.halves;
  int best_cull = cull_tiles_;
  // culling pair kernel: tiles per warp run (0 = off); it runs only without a pruned list
  auto tune_cull = [&]() {
    if (!(nb_ && nb_periodic_ && nl_.block_tiles && nl_.max_cand > 0 && nl_.halves) || dp_ ||
        prune_margin_ > 0.0)
      return;
    for (int c : kTunedCullTiles) {
      cull_tiles_ = c;
      const double ms = trial(best_skin, best_ctas);
      if (ms < best_ms) {
        best_ms = ms;
        best_cull = c;
      }
    }
    cull_tiles_ = best_cull;
  };
  // pruned-list margin (0 = no pruning), where the list builder records each block's tiles
  auto tune_margin = [&]() {
    if (!(nb_ && nb_periodic_ && nl_.block_tiles && nl_.max_cand > 0 && nl_.halves)) return;
    for (double m : kTunedPruneMargins) {
      if (m > 0.0) ensure_pruned_list();
      prune_margin_ = m;
      const double ms = trial(best_skin, best_ctas);
      if (ms < best_ms) {
        best_ms = ms;
        best_margin = m;
      }
    }
    prune_margin_ = best_margin;
  };
  try {
    tune_cull();
    tune_margin();
    if (nb_ && nb_periodic_) {
      for (double s : kTunedSkins) {
        const double ms = trial(s, best_ctas);
        if (ms < best_ms) {
          best_ms = ms;
          best_skin = s;
        }
      }
    }
    // tile width: 16 entries per half block against 32 per block (rectangular boxes)
    if (nb_ && nb_periodic_ && nl_.max_cand > 0) {
      for (int h : {1, 0}) {
        nl_.halves = h;
        const double ms = trial(best_skin, best_ctas);
        if (ms < best_ms) {
          best_ms = ms;
          best_halves = h;
        }
      }
      nl_.halves = best_halves;
    }
    tune_margin();  // again, for the chosen skin and tile width
    // pair-kernel grid, jointly with the culling kernel's run length: its warps stay resident
    // until the work runs out, so a smaller grid leaves SMs to the reciprocal chain beside it
    if (nb_) {
      const bool cull_ok = nb_periodic_ && nl_.block_tiles && nl_.max_cand > 0 && nl_.halves &&
                           !dp_ && best_margin == 0.0;
      const std::vector<int> culls = cull_ok ? std::vector<int>(std::begin(kTunedCullTiles),
                                                                std::end(kTunedCullTiles))
                                             : std::vector<int>{cull_tiles_};
      for (int k : culls) {
        cull_tiles_ = k;
        for (int c : kTunedPairCtasPerSm) {
          const double ms = trial(best_skin, c);
          if (ms < best_ms) {
            best_ms = ms;
            best_ctas = c;
            best_cull = k;
          }
        }
      }
      cull_tiles_ = best_cull;
    }
  } catch (...) {
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    profiling_ = prof;
    throw;
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  skin_ = best_skin;
  nl_.skin = best_skin;
  nl_.halves = best_halves;
  prune_margin_ = best_margin;
  cull_tiles_ = best_cull;
  pair_grid_ = sm_count_ * best_ctas;
  destroy_graph();
  restore();
  profiling_ = prof;
  if (skin_out) *skin_out = best_skin;
  if (ctas_out) *ctas_out = best_ctas;
  if (ms_out) *ms_out = best_ms;
}

void Engine::tuning(double* skin, int* pair_ctas_per_sm, int* tile_entries) const {
  if (skin) *skin = skin_;
  if (pair_ctas_per_sm) *pair_ctas_per_sm = pair_grid_ / std::max(1, sm_count_);
  const bool rect = nb_ && nb_periodic_ && nl_.max_cand > 0;
  if (tile_entries) *tile_entries = rect && nl_.halves ? 16 : 32;
}

void Engine::nlist_capacity(int* tile_capacity, int* column_capacity, int* regrows) const {
  if (tile_capacity) *tile_capacity = nl_.tile_capacity;
  if (column_capacity) *column_capacity = nb_periodic_ ? nl_.col_max : 0;
  if (regrows) *regrows = regrows_;
}

void Engine::pair_cull_stats(int* tiles_per_run, int64_t* rounds) {
  unsigned long long r = 0;
  if (cull_rounds_) {
    OMMB200_CK(cudaMemcpyAsync(&r, cull_rounds_, 8, cudaMemcpyDeviceToHost, stream_));
    sync();
  }
  if (tiles_per_run) *tiles_per_run = culling() ? cull_tiles_ : 0;
  if (rounds) *rounds = (int64_t)r;
}

void Engine::nlist_prune_stats(int* rebuild_tiles, int64_t* prunes, double* margin) {
  int t = 0;
  unsigned long long c = 0;
  if (nb_ && nb_periodic_) {
    OMMB200_CK(cudaMemcpyAsync(&t, nl_.n_tiles, 4, cudaMemcpyDeviceToHost, stream_));
    OMMB200_CK(cudaMemcpyAsync(&c, prune_count_, 8, cudaMemcpyDeviceToHost, stream_));
    sync();
  }
  if (rebuild_tiles) *rebuild_tiles = t;
  if (prunes) *prunes = pruning() ? (int64_t)c : 0;
  if (margin) *margin = pruning() ? prune_margin_ : 0.0;
}

void Engine::nlist_stats(int* tiles, int* blocks, int* masked, int64_t* rebuilds) {
  int v[3] = {0, 0, 0};
  unsigned long long r = 0;
  if (nb_) {
    // the tiles the pair kernel evaluates: the pruned list's while pruning
    OMMB200_CK(cudaMemcpyAsync(&v[0], pruning() ? prune_n_tiles_ : nl_.n_tiles, 4,
                               cudaMemcpyDeviceToHost, stream_));
    OMMB200_CK(cudaMemcpyAsync(&v[1], nl_.n_blocks, 4, cudaMemcpyDeviceToHost, stream_));
    OMMB200_CK(cudaMemcpyAsync(&v[2], nl_.n_masks, 4, cudaMemcpyDeviceToHost, stream_));
    OMMB200_CK(cudaMemcpyAsync(&r, nl_.rebuild_count, 8, cudaMemcpyDeviceToHost, stream_));
    sync();
  }
  if (tiles) *tiles = v[0];
  if (blocks) *blocks = v[1];
  if (masked) *masked = v[2];
  if (rebuilds) *rebuilds = (int64_t)r;
}

void Engine::pme_layout(int* bricks_in_use, int* bricks) const {
  if (bricks_in_use) *bricks_in_use = use_bricks_ ? 1 : 0;
  if (bricks) *bricks = bricks_.ranges ? bricks_.nb[0] * bricks_.nb[1] * bricks_.nb[2] : 0;
}

void Engine::pme_parameters(double* alpha, int* nx, int* ny, int* nz) const {
  *alpha = alpha_;
  *nx = grid_[0];
  *ny = grid_[1];
  *nz = grid_[2];
}

int64_t Engine::debug_pair_list(int64_t max_pairs, int32_t* pairs) {
  require(nb_ != nullptr, "the System has no NonbondedForce");
  if (max_pairs > dump_capacity_) {
    dump_pairs_ = mem_.alloc<int32_t>(2 * (size_t)std::max<int64_t>(max_pairs, 1));
    dump_capacity_ = max_pairs;
  }
  if (!dump_count_) dump_count_ = mem_.alloc<unsigned long long>(1);
  OMMB200_CK(cudaMemsetAsync(dump_count_, 0, 8, stream_));
  dump_mode_ = true;
  try {
    for (;;) {  // an overflowing list grows and the dump starts again
      OMMB200_CK(cudaMemsetAsync(dump_count_, 0, 8, stream_));
      compute_forces(false, 0xffffffffu);
      sync();
      const int st = take_status();
      if (st == kStatusTileOverflow && grow_neighbor_capacity()) continue;
      raise_status(st);
      break;
    }
  } catch (...) {
    dump_mode_ = false;
    throw;
  }
  dump_mode_ = false;
  unsigned long long count = 0;
  OMMB200_CK(cudaMemcpyAsync(&count, dump_count_, 8, cudaMemcpyDeviceToHost, stream_));
  sync();
  const int64_t take = std::min<int64_t>((int64_t)count, max_pairs);
  if (take > 0 && pairs)
    OMMB200_CK(cudaMemcpy(pairs, dump_pairs_, 8 * (size_t)take, cudaMemcpyDeviceToHost));
  harvest_profile();
  check_status();
  return (int64_t)count;
}

}  // namespace ommb200

namespace ommb200 {

namespace {
struct CheckpointHeader {
  char magic[8];
  uint32_t version;
  int32_t n_atoms, n_segments, precision, learned, dynamic_list, rebuild_flag, pair_grid, halves;
  int32_t prune_flag, cull_tiles;
  double time;
  int64_t step_count;
  double box[9];
  uint64_t seed, velocity_draws, rng_step;
  double skin;
  double prune_margin;
  // barostat (zero without one): step counter, volume step and its window, totals, stream
  uint64_t bar_counter, bar_window_attempted, bar_window_accepted, bar_attempted, bar_accepted;
  uint64_t bar_seed, bar_draws;
  double bar_volume_scale, bar_pressure, bar_temperature;
};
constexpr char kCheckpointMagic[8] = {'O', 'M', 'B', '2', 'C', 'K', 'P', 'T'};
constexpr uint32_t kCheckpointVersion = 7;
}  // namespace

size_t Engine::checkpoint_bytes() const {
  size_t b = sizeof(CheckpointHeader) + 2 * 24 * (size_t)n_;
  if (nb_periodic_) b += 2 * 24 * (size_t)n_;  // rebuild and prune reference positions
  if (learned_)
    b += 4 * (size_t)(kRadiiMlpParams + 2 * kRadiiMlpTrainable + 1 + segments_.size() + 1) +
         sizeof(LearnedState);
  return b;
}

void Engine::save_checkpoint(uint8_t* out, size_t bytes) {
  require(bytes >= checkpoint_bytes(), "checkpoint buffer too small");
  CheckpointHeader h{};
  std::memcpy(h.magic, kCheckpointMagic, 8);
  h.version = kCheckpointVersion;
  h.n_atoms = n_;
  h.n_segments = (int32_t)segments_.size();
  h.precision = opt_.precision;
  h.learned = learned_ ? 1 : 0;
  h.dynamic_list = nb_periodic_ ? 1 : 0;
  h.pair_grid = pair_grid_;
  h.halves = nl_.halves;
  h.time = time_;
  h.step_count = step_count_;
  std::copy(box_, box_ + 9, h.box);
  h.seed = seed_;
  h.velocity_draws = velocity_draws_;
  h.skin = skin_;
  h.prune_margin = prune_margin_;
  h.cull_tiles = cull_tiles_;
  h.bar_counter = bar_counter_;
  h.bar_window_attempted = bar_window_attempted_;
  h.bar_window_accepted = bar_window_accepted_;
  h.bar_attempted = bar_attempted_;
  h.bar_accepted = bar_accepted_;
  h.bar_seed = bar_seed_;
  h.bar_draws = bar_draws_;
  h.bar_volume_scale = bar_volume_scale_;
  h.bar_pressure = bar_pressure_;
  h.bar_temperature = bar_temperature_;
  int flag = 0, prune_flag = 0;
  OMMB200_CK(cudaMemcpyAsync(&h.rng_step, rng_step_, 8, cudaMemcpyDeviceToHost, stream_));
  OMMB200_CK(cudaMemcpyAsync(&flag, rebuild_, 4, cudaMemcpyDeviceToHost, stream_));
  if (prune_flag_)
    OMMB200_CK(cudaMemcpyAsync(&prune_flag, prune_flag_, 4, cudaMemcpyDeviceToHost, stream_));
  uint8_t* p = out + sizeof(CheckpointHeader);
  auto take = [&](const void* dev, size_t n) {
    OMMB200_CK(cudaMemcpyAsync(p, dev, n, cudaMemcpyDeviceToHost, stream_));
    p += n;
  };
  take(pos_, 24 * (size_t)n_);
  take(vel_, 24 * (size_t)n_);
  if (nb_periodic_) {
    take(nl_.pos_ref, 24 * (size_t)n_);
    take(pos_prune_, 24 * (size_t)n_);
  }
  if (learned_) {
    take(lr_.params, 4 * kRadiiMlpParams);
    take(lr_.moments, 8 * kRadiiMlpTrainable);
    take(lr_.adam_t, 4);
    take(lr_.seg_offset, 4 * segments_.size());
    take(lr_.state, sizeof(LearnedState));
    take(lr_.loss + std::max(0, lr_.train_steps - 1), 4);  // last training loss (a judge may skip training)
  }
  sync();
  h.rebuild_flag = flag;
  h.prune_flag = prune_flag;
  std::memcpy(out, &h, sizeof(h));
}

void Engine::load_checkpoint(const uint8_t* in, size_t bytes) {
  require(bytes >= sizeof(CheckpointHeader), "checkpoint too short");
  CheckpointHeader h;
  std::memcpy(&h, in, sizeof(h));
  require(std::memcmp(h.magic, kCheckpointMagic, 8) == 0 && h.version == kCheckpointVersion,
          "not a checkpoint of this engine version");
  require(h.n_atoms == n_ && h.n_segments == (int32_t)segments_.size() &&
              h.precision == opt_.precision && h.learned == (learned_ ? 1 : 0) &&
              h.dynamic_list == (nb_periodic_ ? 1 : 0),
          "checkpoint was written by a Context of a different System or configuration");
  require(bytes >= checkpoint_bytes(), "checkpoint too short");
  for (double x : h.box) require(std::isfinite(x), "checkpoint box is not finite");
  destroy_graph();
  sync();
  const uint8_t* p = in + sizeof(CheckpointHeader);
  auto put = [&](void* dev, size_t n) {
    OMMB200_CK(cudaMemcpy(dev, p, n, cudaMemcpyHostToDevice));
    p += n;
  };
  put(pos_, 24 * (size_t)n_);
  put(vel_, 24 * (size_t)n_);
  std::copy(h.box, h.box + 9, box_);
  update_box_dependents();
  time_ = h.time;
  step_count_ = h.step_count;
  if (bar_def_) {
    bar_counter_ = h.bar_counter;
    bar_window_attempted_ = h.bar_window_attempted;
    bar_window_accepted_ = h.bar_window_accepted;
    bar_attempted_ = h.bar_attempted;
    bar_accepted_ = h.bar_accepted;
    bar_seed_ = h.bar_seed;
    bar_draws_ = h.bar_draws;
    bar_volume_scale_ = h.bar_volume_scale;
    bar_pressure_ = h.bar_pressure;
    bar_temperature_ = h.bar_temperature;
  }
  seed_ = h.seed;
  velocity_draws_ = h.velocity_draws;
  OMMB200_CK(cudaMemcpy(rng_step_, &h.rng_step, 8, cudaMemcpyHostToDevice));
  if (nb_periodic_) {
    skin_ = h.skin;
    nl_.skin = h.skin;
    prune_margin_ = h.prune_margin;
    cull_tiles_ = h.cull_tiles;
    if (prune_margin_ > 0.0) ensure_pruned_list();
    update_bricks();
    pair_grid_ = h.pair_grid;
    nl_.halves = h.halves;
    put(nl_.pos_ref, 24 * (size_t)n_);
    // rebuild the neighbour list from the saved reference positions: the same input as the
    // original run's last rebuild, so the tiles (and every force sum) are the same
    NlistArgs from_ref = nl_;
    from_ref.pos = nl_.pos_ref;
    const int one = 1;
    OMMB200_CK(cudaMemcpy(rebuild_, &one, 4, cudaMemcpyHostToDevice));
    launch_nlist_rebuild(from_ref, dp_, stream_, with_new_list(from_ref));
    // and the pruned list from the positions of the original run's last prune (its tiles hold
    // the same entries, so every per-tile sum rounds the same)
    put(pos_prune_, 24 * (size_t)n_);
    if (pruning() && nb_) {
      NlistArgs from_prune = nl_;
      from_prune.pos = pos_prune_;
      OMMB200_CK(cudaMemcpy(prune_flag_, &one, 4, cudaMemcpyHostToDevice));
      if (dp_)
        launch_pack<double>(n_slots_, nl_.sorted_atom, pos_prune_, nl_.image, nl_.block_center,
                            qscaled_, half_sigma_, sqrt_eps_, posq_, ljp_, nl_.box, stream_);
      else
        launch_pack<float>(n_slots_, nl_.sorted_atom, pos_prune_, nl_.image, nl_.block_center,
                           qscaled_, half_sigma_, sqrt_eps_, posq_, ljp_, nl_.box, stream_);
      launch_nlist_prune(from_prune, prune_args(), dp_, stream_);
    }
    if (packed_by_integrator() && nb_) pack_slots(pos_, stream_);  // the saved run's last step wrote these
    sync();
    OMMB200_CK(cudaMemcpy(rebuild_, &h.rebuild_flag, 4, cudaMemcpyHostToDevice));
    OMMB200_CK(cudaMemcpy(prune_flag_, &h.prune_flag, 4, cudaMemcpyHostToDevice));
  }
  if (learned_) {
    put(lr_.params, 4 * kRadiiMlpParams);
    put(lr_.moments, 8 * kRadiiMlpTrainable);
    put(lr_.adam_t, 4);
    put(lr_.seg_offset, 4 * segments_.size());
    put(lr_.state, sizeof(LearnedState));
    put(lr_.loss + std::max(0, lr_.train_steps - 1), 4);
  }
  check_status();
}

}  // namespace ommb200
