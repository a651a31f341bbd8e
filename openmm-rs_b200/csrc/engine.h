// The Context engine: device-resident state of one System plus the launch sequence of an MD
// step (context.rs:878-928 try_step_once: forces, then the integrator) and of getState.
#pragma once

#include <cufft.h>

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "../../include/ommb200.h"
#include "kernels.h"
#include "model.h"

namespace ommb200 {

// Owns every device allocation of an Engine; memory is zeroed on allocation.
double measure_fp32_peak(int device);  // diagnostics.cu
// noalloc.cu: NonbondedForce forces with scratch in a static device array (no allocation)
void nonbonded_forces_noalloc(int n, const double* pos, const double* q, const double* sigma,
                              const double* eps, int method, double cutoff, double rf_dielectric,
                              double* forces, double* energy, cudaStream_t stream);

// Verlet skins and pair-kernel CTAs per SM the autotuner tries.
constexpr double kTunedSkins[] = {0.06, 0.08, 0.1, 0.13, 0.16, 0.2};
constexpr double kMaxTunedSkin = 0.2;
constexpr int kTunedPairCtasPerSm[] = {2, 3, 4, 6, 7, 8, 9, 10, 11, 12};
// Margins of the pruned pair list (nm) the autotuner tries: entries within cutoff + margin of
// their half block stay, and a particle that moves margin / 2 requests the next prune, so a
// wider margin prunes less often and leaves more pairs for the pair kernel; 0 turns pruning
// off (the pair kernel reads the rebuild's list).  The allowance absorbs the FP32 rounding of
// the prune's distances.
constexpr double kTunedPruneMargins[] = {0.0, 0.05, 0.08, 0.12};
constexpr double kDefaultPruneMargin = 0.0;
constexpr double kPruneAllowance = 1e-4;
// Culling pair kernel (FP32, periodic rectangular boxes, no pruned list): a warp takes a run
// of this many consecutive tiles of one block; 0 reads every tile's entries as they are
// (pair_kernel_x2).  By default it runs with kDefaultCullTiles when the list gives a resident
// warp about kCullMinTilesPerWarp tiles or more (below that each tile's loads are exposed);
// the autotuner tries the values below.
constexpr int kDefaultCullTiles = 64;
constexpr double kCullMinTilesPerWarp = 40.0;
constexpr int kTunedCullTiles[] = {0, 4, 8, 16, 32, 64};

class DeviceArena {
 public:
  ~DeviceArena();
  void* alloc_bytes(size_t bytes);
  template <class T>
  T* alloc(size_t count) {
    return static_cast<T*>(alloc_bytes(sizeof(T) * (count ? count : 1)));
  }

 private:
  std::vector<void*> ptrs_;
};

struct EngineOptions {
  int precision = OMMB200_PRECISION_MIXED;
  int device = 0;
  bool use_graph = true;
  double skin = 0.0;
  int steps_per_graph = 0;
  int pme_bricks = -1;  // brick-owned PME gather: -1 by grid size, 0 off, 1 on
  double prune_margin = -1.0;  // nm; 0 off, < 0 the default
  int pair_cull = -1;  // culling pair kernel: tiles per sub-chunk; 0 off, < 0 the default
};

// Device state that a re-run of MD steps starts from (Engine::save_dynamic_state).
struct DynamicSnapshot {
  double* x = nullptr;
  double* v = nullptr;
  float* lr = nullptr;  // learned radii: network, optimiser moments and step, system offsets
  unsigned long long rng = 0;
  LearnedState state{};
};

class Engine {
 public:
  // `segments`: particle ranges of independent systems merged into `system` (a batch);
  // empty = one system.
  Engine(std::unique_ptr<SystemDef> system, std::unique_ptr<IntegratorDef> integrator,
         const EngineOptions& options, std::vector<Segment> segments = {});
  int num_segments() const { return (int)segments_.size(); }
  Segment segment(int s) const { return segments_.at(s); }
  // Per-system potential and kinetic energy of the included force groups.
  void segment_energies(uint32_t groups, double* potential, double* kinetic);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  int num_particles() const { return n_; }
  void set_positions(const double* xyz);
  void set_velocities(const double* v);
  void set_velocities_to_temperature(double temperature, int seed);
  void set_box(const double box[9]);
  void set_time(double t) { time_ = t; }
  void set_step_count(int64_t s) { step_count_ = s; }
  void apply_constraints(double tolerance);
  void apply_velocity_constraints(double tolerance);
  void step(int steps);
  void get_state(int flags, uint32_t groups, double* pos, double* vel, double* forces,
                 ommb200_state_info* info);
  void pme_parameters(double* alpha, int* nx, int* ny, int* nz) const;
  void pme_layout(int* bricks_in_use, int* bricks) const;
  void nlist_stats(int* tiles, int* blocks, int* masked, int64_t* rebuilds);
  void nlist_capacity(int* tile_capacity, int* column_capacity, int* regrows) const;
  void nlist_prune_stats(int* rebuild_tiles, int64_t* prunes, double* margin);
  // tiles per warp run of the culling pair kernel (0 when it does not run) and the rounds it
  // has run so far (each 2 x 16 x 16 pair slots)
  void pair_cull_stats(int* tiles_per_run, int64_t* rounds);
  // current skin, pair-kernel CTAs per SM and neighbour entries per i-group (16: halves of
  // 32-particle blocks; 32: whole blocks)
  void tuning(double* skin, int* pair_ctas_per_sm, int* tile_entries) const;
  // Times `trial_steps` MD steps for each candidate skin and pair-kernel grid from the
  // current state, keeps the fastest, and restores the state (positions, velocities, RNG
  // counter), so the trajectory is the same as without tuning.
  void autotune(int trial_steps, double* skin, int* pair_ctas_per_sm, double* ms_per_step);
  int64_t debug_pair_list(int64_t max_pairs, int32_t* pairs);
  void set_profiling(bool enabled);
  struct KernelTime {
    std::string name;
    double ms;
    int launches;
  };
  std::vector<KernelTime> kernel_times() const { return kernel_times_; }
  cudaStream_t stream() const { return stream_; }
  // context.rs:680-705: live parameter updates of the Context's NonbondedForce / GBSAOBCForce
  void update_nonbonded(const NonbondedDef& src);
  void update_gbsa(const GbsaObcDef& src);
  // Complete dynamic state (positions, velocities, box, time, step count, random-stream
  // counter, neighbour-list reference, learned-radii network and optimiser) as bytes;
  // loading it into a Context of the same System continues the trajectory bit for bit.
  size_t checkpoint_bytes() const;
  void save_checkpoint(uint8_t* out, size_t bytes);
  void load_checkpoint(const uint8_t* in, size_t bytes);
  // context.rs:251-268: global parameters of the System's forces (the barostat's pressure and
  // temperature)
  void set_parameter(const std::string& name, double value);
  double get_parameter(const std::string& name) const;
  void barostat_stats(ommb200_barostat_stats* out) const;
  // learned Born radii: counters of the device control block, last judge error and loss
  void learned_stats(ommb200_learned_radii_stats* out);
  void learned_params(float* out);
  void set_learned_params(const float* in);

 private:
  void setup_nonbonded(const NonbondedDef& nb);
  void setup_bonded();
  void setup_gbsa(const GbsaObcDef& gb);
  void build_static_layout();
  void setup_integrator();
  void update_box_dependents();
  void update_bricks();
  bool packed_by_integrator() const;
  // the launches that follow a neighbour-list build of `list` (brick ranges, gated pack)
  std::function<void(cudaStream_t)> with_new_list(const NlistArgs& list);
  void pack_slots(const double* pos, cudaStream_t s, const int* only_after_rebuild = nullptr);
  void build_static_tiles();
  void enqueue_conditional_rebuild();
  void enqueue_conditional_body(cudaGraphConditionalHandle handle,
                                const std::function<void(cudaStream_t)>& body);
  // The pair kernel runs on the pruned list: periodic rectangular boxes whose rebuild packs 16
  // entries per half block (the builder that records each block's tiles).
  bool pruning() const;
  // whether the culling pair kernel runs, and its sub-chunks per block (tiles per block
  // estimated from the density, the column widths and the cutoff + skin)
  bool culling() const;
  int cull_chunks() const;
  double tiles_per_block_max() const;  // estimate from the density and the cutoff + skin
  void alloc_pruned_list();
  void ensure_pruned_list();  // the pruned list's arrays, allocated on first use
  PruneArgs prune_args() const;
  // `in_step`: an MD step's evaluation (the learned radii may judge and train there);
  // `step_offset`: its position inside the captured group of steps.
  void compute_forces(bool energy, uint32_t groups, bool in_step = false, int step_offset = 0);
  void compute_forces_checked(bool energy, uint32_t groups);
  void setup_learned(const LearnedRadiiDef& def);
  void upload_nonbonded_parameters(const NonbondedDef& nb);
  std::vector<long long> evaluate(bool energy, uint32_t groups, double* forces);
  void enqueue_step(int step_offset);
  void run_steps(int steps);
  void run_graph_steps(int graph_launches);
  // MonteCarloBarostat (forces/barostat.rs, context/program.rs:5-47)
  void setup_barostat(BarostatDef& def);
  void barostat_move();
  void barostat_record(bool accepted, double previous_volume);
  double barostat_uniform();
  // potential energy of `groups` (forces evaluated into the Context's buffers)
  double potential_energy(uint32_t groups);
  // long-range corrections added to the fixed-point sums e[8] (energy, virial) of `groups`
  double assemble_energy(const long long e[8], uint32_t groups, double w[6]) const;
  void check_status();
  // Reads and clears the device status word; raise_status throws its error (0: none).
  int take_status();
  void raise_status(int status);
  // After a neighbour-list overflow: larger tile and mask arrays and per-column sort, and a
  // rebuild requested; false when nothing can grow any more.
  bool grow_neighbor_capacity();
  void save_dynamic_state(DynamicSnapshot& snap);
  void restore_dynamic_state(const DynamicSnapshot& snap);
  void sync();
  void destroy_graph();
  template <class Real>
  void enqueue_nonbonded(bool energy, bool direct, bool reciprocal, bool dump, bool pairs);
  void prof_begin(const char* name);
  void prof_end();
  void harvest_profile();
  IntegrateArgs integrate_args(int step_offset) const;

  std::unique_ptr<SystemDef> sys_;
  std::unique_ptr<IntegratorDef> integ_;
  EngineOptions opt_;
  bool dp_ = false;
  int n_ = 0;
  double box_[9];
  // barostat state: the live definition (frequency), Context values of pressure and
  // temperature, step counter since the last move, volume step and its 10-attempt window,
  // totals, random stream (seed, draws), last move; molecules as CSR lists of atoms
  BarostatDef* bar_def_ = nullptr;
  bool bar_rigid_ = true;  // captured at Context creation (barostat.rs:104-108)
  double bar_pressure_ = 0.0, bar_temperature_ = 0.0, bar_volume_scale_ = 0.0;
  uint64_t bar_counter_ = 0, bar_window_attempted_ = 0, bar_window_accepted_ = 0;
  uint64_t bar_attempted_ = 0, bar_accepted_ = 0, bar_seed_ = 0, bar_draws_ = 0;
  ommb200_barostat_stats bar_last_{};
  int n_molecules_ = 0, bar_scaled_ = 0;
  int* mol_start_ = nullptr;
  int* mol_atoms_ = nullptr;
  double* bar_saved_ = nullptr;
  double time_ = 0.0;
  int64_t step_count_ = 0;
  uint64_t seed_ = 0;
  uint64_t velocity_draws_ = 0;
  cudaStream_t stream_ = nullptr;
  // PME runs on its own stream, forked after the neighbour-list rebuild and joined before
  // the integrator, so it overlaps the real-space pair kernel (also inside the CUDA graph).
  cudaStream_t pme_stream_ = nullptr;
  cudaEvent_t fork_ev_ = nullptr, join_ev_ = nullptr;
  cudaStream_t aux_stream_ = nullptr;  // captures conditional-node bodies
  bool capturing_ = false;             // a step group is being captured into the graph
  DeviceArena mem_;

  // state
  double* pos_ = nullptr;
  double* vel_ = nullptr;
  double* inv_mass_ = nullptr;
  double* scratch3_ = nullptr;
  long long* force_ = nullptr;
  long long* energy_ = nullptr;  // [8 * segments]: energy, virial (6), unused
  int* status_ = nullptr;
  int* rebuild_ = nullptr;
  unsigned long long* rng_step_ = nullptr;
  std::vector<double> host_masses_;

  // nonbonded
  const NonbondedDef* nb_ = nullptr;
  bool nb_periodic_ = false;
  bool nb_pme_ = false;
  int elec_ = kElecCoulomb;
  int n_blocks_ = 0, n_slots_ = 0;
  NlistArgs nl_{};
  double* qscaled_ = nullptr;
  double* charge_ = nullptr;
  double* half_sigma_ = nullptr;
  double* sqrt_eps_ = nullptr;  // 2 sqrt(epsilon)
  int static_tile_count_ = 0;    // tiles of the non-periodic (segment-padded) pair list
  bool nb_gb_fusable_ = false;   // NoCutoff pair terms can run inside GB pass 2
  void* posq_ = nullptr;
  void* ljp_ = nullptr;
  bool params_packed_ = false;
  double alpha_ = 0.0;
  int grid_[3] = {0, 0, 0};
  double recip_[3][3];
  double volume_ = 0.0;
  double self_energy_ = 0.0, plasma_energy_ = 0.0, dispersion_coeff_ = 0.0;
  long long* pme_fixed_ = nullptr;
  void* pme_real_ = nullptr;
  void* pme_k_ = nullptr;
  void* influence_ = nullptr;
  double* moduli_ = nullptr;
  cufftHandle fft_fwd_ = 0, fft_inv_ = 0;
  bool fft_ready_ = false;
  bool own_fft_ = false;  // the engine's pencil transform instead of cuFFT
  PmeFft fft_{};
  int n_exceptions_ = 0;
  int2* exc_pairs_ = nullptr;
  double4* exc_params_ = nullptr;
  int32_t* dump_pairs_ = nullptr;
  unsigned long long* dump_count_ = nullptr;
  long long dump_capacity_ = 0;
  bool dump_mode_ = false;
  int pair_grid_ = 0;
  int sm_count_ = 148;
  // pruned pair list (PruneArgs): inner tiles, entries, masks, exclusion columns, counters
  int4* prune_tiles_ = nullptr;
  void* prune_entries_ = nullptr;
  uint32_t* prune_masks_ = nullptr;
  uint32_t* prune_cols_ = nullptr;
  uint32_t* prune_keep_ = nullptr;
  double prune_margin_ = kDefaultPruneMargin;  // 0: no pruning
  int cull_tiles_ = 0;  // culling pair kernel's run length in tiles (0: off)
  int* cull_work_ = nullptr;  // its work counters (zero between launches)
  unsigned long long* cull_rounds_ = nullptr;  // its rounds so far
  double list_density_ = 0.0, list_col_w_[2] = {0.0, 0.0};  // for the tiles-per-block estimate
  int cand_scale_ = 1;  // growth of the list builder's candidate arrays after overflows
  PmeBricks bricks_{};      // brick-owned PME gather: geometry, slot ranges, stencils
  bool use_bricks_ = false;
  unsigned* prune_done_ = nullptr;
  int* prune_n_tiles_ = nullptr;
  int prune_capacity_ = 0;
  int* prune_flag_ = nullptr;
  double* pos_prune_ = nullptr;
  unsigned long long* prune_count_ = nullptr;

  // segments (independent systems) and the segment-padded slot order shared by the
  // non-periodic nonbonded tiles and GBSA: every segment starts on a 32-slot boundary
  std::vector<Segment> segments_;
  std::vector<int> static_slot_atom_;   // [static_slots_], -1 = padding
  std::vector<int> static_atom_slot_;   // [n_]
  std::vector<int> static_block_seg_;   // [static_slots_ / 32]
  int static_slots_ = 0;
  int* d_block_segment_ = nullptr;
  int* d_atom_segment_ = nullptr;

  // GBSAOBCForce
  const GbsaObcDef* gb_def_ = nullptr;
  GbArgs gb_{};
  // learned Born radii
  bool learned_ = false;
  LearnedGbArgs lr_{};

  // bonded terms, one launch per force
  struct BondedLaunch {
    BondedArgs args;
    int group;
  };
  std::vector<BondedLaunch> bonded_;

  // integrator
  int n_water_ = 0, n_free_ = 0, n_clusters_ = 0;
  int4* water_ = nullptr;
  WaterGeometry geom_{};
  int* free_atoms_ = nullptr;
  int* cluster_start_ = nullptr;
  int2* cluster_pairs_ = nullptr;
  double* cluster_dist2_ = nullptr;
  int* cluster_atom_start_ = nullptr;
  int* cluster_atoms_ = nullptr;
  double skin_ = 0.0;

  DynamicSnapshot step_snapshot_;  // start of the current run_steps batch (periodic systems)
  int regrows_ = 0;                 // neighbour-list capacity increases so far

  // graph
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  int graph_steps_ = 0;

  // profiling
  bool profiling_ = false;
  struct PendingEvent {
    std::string name;
    cudaEvent_t start, stop;
  };
  std::vector<PendingEvent> pending_;
  std::vector<cudaEvent_t> event_pool_;
  std::vector<KernelTime> kernel_times_;
  std::string current_prof_;
  cudaEvent_t current_start_ = nullptr;
};

}  // namespace ommb200
