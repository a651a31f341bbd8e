// Argument blocks and launchers of the engine's CUDA kernels.  Every launcher enqueues on the
// given stream and never synchronizes, so a whole MD step can be captured in a CUDA graph.
#pragma once

#include <algorithm>
#include <functional>
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include "common.cuh"

namespace ommb200 {

// ---- neighbour tiles -------------------------------------------------------------------
// Particles live in 32-slot blocks of a spatially sorted order.  A tile pairs the 32 slots
// of block I with 32 "entries": either block I itself (self tile) or up to 32 j-particles
// gathered from blocks J > I, each entry carrying the offset of its block's frame from I's.
enum TileFlags : int {
  kTileHasMask = 1,    // exclusion/padding mask stored at masks[32 * mask_slot]
  kTilePairImage = 2,  // apply the minimum image per pair (small boxes)
  kTileSelf = 4,       // entries are block I itself; each pair is seen twice
  kTileHalves = 8,     // entries 0-15 pair with slots 0-15 of I only, entries 16-31 with 16-31
};

struct NlistArgs {
  int n_atoms;        // particles of the system
  int slot_capacity;  // multiple of 32: N + 31 * columns
  const double* pos;  // [3N] master positions
  double* pos_ref;    // [3N] positions at the last rebuild
  int* image;         // [3N] lattice image n of each particle at the last rebuild
  int* column;        // [N] x-y column of each particle
  float* zkey;        // [N] wrapped z of each particle
  int* col_count;     // [n_cols] particles per column (zero between rebuilds)
  int* col_start;     // [n_cols + 1] first slot of each column (columns padded to blocks)
  int* col_scatter;   // [n_cols + 1] unpadded prefix, for the scatter
  int* col_cursor;    // [n_cols] scatter cursor (zero between rebuilds)
  int* scratch_atoms; // [N] unordered scatter
  int* n_blocks;      // device: blocks in use after the last rebuild
  int* sorted_atom;   // [slot_capacity] particle in each slot, -1 for padding
  int* atom_slot;     // [N] inverse of sorted_atom
  double4* slot_wpos;    // [slot_capacity] wrapped rebuild position of each slot (w = 0)
  double* block_center;  // [3 * slot_capacity / 32]
  double* block_half;    // [3 * slot_capacity / 32] half extents of the bounding box
  int4* tiles;           // [tile_capacity] (I, flags, mask_slot, 0)
  void* entries;         // [32 * tile_capacity] float4/double4: shift xyz, slot (as int bits
                         //   for float4, as a double for double4); slot -1 = padding
  uint32_t* masks;       // [32 * mask_capacity]
  int* n_tiles;          // device counter
  int* n_masks;          // device counter
  int tile_capacity, mask_capacity;
  const int* excl_start;  // [N + 1] CSR of excluded partners (both directions)
  const int* excl_list;
  int* rebuild;           // nonzero: rebuild before the next force evaluation
  unsigned long long* rebuild_count;
  int* status;
  Box<double> box;
  int periodic;
  double cutoff;      // interaction cutoff (nm)
  double skin;        // Verlet skin (nm)
  double min_width;   // shortest lattice vector bound: min(ax, by, cz)
  int n_col[2];       // x-y column grid of the sort
  int n_cols;
  int col_max;        // largest column the per-column sort accepts
  int max_cand;       // candidate blocks one block can have (rectangular boxes), 0 = unknown
  int halves;         // rectangular boxes: 16 entries per half of a block (else 32 per block)
  int* block_tiles;   // [2 * blocks] first tile and tile count of each block (halves builder)
  int* prune;         // null, or set by every rebuild: the pruned list must be made again
};

// Pruned list: the rebuild's tiles cut down to the entries within cutoff + margin of a particle
// of their half block at the current positions (the pair kernel's list while pruning is on).
struct PruneArgs {
  int4* tiles;          // [capacity] (I, flags, mask slot = tile index, 0)
  void* entries;        // [32 * capacity] as the rebuild's entries
  uint32_t* masks;      // [32 * capacity]
  uint32_t* cols;       // [32 * capacity] scratch: exclusion column (bit per i-slot) per entry
  uint32_t* keep;       // [rebuild tile capacity] scratch: kept entries of each rebuild tile
  unsigned* done;       // scratch: placement CTAs finished (the last one closes the prune)
  int* n_tiles;         // tiles in use
  int capacity;
  int sm_count;         // grid of the keep pass
  int* prune;           // nonzero: prune before this evaluation's pair kernel
  double* pos_prune;    // [3N] positions at the last prune
  const void* posq;     // this evaluation's packed particles
  double reach2;        // (cutoff + margin + a rounding allowance)^2
  unsigned long long* prune_count;
};

// `with_list` (may be empty) enqueues launches that need the new list and must run only on a
// rebuild: it is called after the list is built and before the rebuild flag clears, so its
// kernels can gate on the flag (the brick gather's slot ranges, the pack of the new slots).
void launch_nlist_rebuild(const NlistArgs& a, bool double_entries, cudaStream_t s,
                          const std::function<void(cudaStream_t)>& with_list = {});
void launch_nlist_prune(const NlistArgs& a, const PruneArgs& p, bool double_entries,
                        cudaStream_t s);
// Sets `handle` to whether a prune is pending (the graph form of the early-exit prune kernels).
void launch_prune_condition(const PruneArgs& p, cudaGraphConditionalHandle handle, cudaStream_t s);
// Sets `handle` (a conditional graph node's condition) to whether a rebuild is pending.
void launch_nlist_condition(const NlistArgs& a, cudaGraphConditionalHandle handle,
                            cudaStream_t s);

// ---- nonbonded pair kernel -------------------------------------------------------------
enum ElecKind : int { kElecEwald = 0, kElecReactionField = 1, kElecCoulomb = 2 };

template <class Real>
struct PairArgs {
  int n_atoms;
  const int* sorted_atom;
  const double* pos;
  const void* posq;     // [slots] float4/double4: block-local xyz, q * sqrt(ke)
  const void* ljp;      // [slots] float2/double2: sigma / 2, 2 sqrt(epsilon)
  const int4* tiles;
  const void* entries;
  const uint32_t* masks;
  const int* n_tiles;
  int tile_capacity;
  long long* force;     // [3][N] fixed point
  long long* energy;    // [7]: energy, virial xx yy zz xy xz yz (fixed point)
  const int* block_segment;  // batch: system of each block, energy at energy[8 * system]
  Box<Real> box;
  Box<double> box_exact;
  int periodic;
  int use_cutoff;
  Real cutoff2;
  double cutoff2_exact;
  Real band;            // |r2 - rc2| below this is decided in f64 by the reference formula
  Real alpha, two_alpha_sqrtpi;
  Real exp_scale;       // -alpha^2 (times log2 e in the FP32 form, which uses exp2)
  Real krf, crf;
  int use_switching;
  Real switch_r, switch_inv_width;
  int32_t* pair_dump;   // diagnostics
  unsigned long long* pair_count;
  long long pair_capacity;
  // culling form (FP32, periodic halves-tile lists from the CTA builder): cull_tiles > 0 runs
  // pair_kernel_cull over sub-chunks of cull_tiles tiles, cull_chunks per block (the last
  // takes the rest); entries farther than sqrt(cull2) from their half block's box are dropped
  int cull_tiles;
  int cull_chunks;
  Real cull2;
  const int* n_blocks;     // device: blocks in use
  const int* block_tiles;  // [2 * blocks] first tile and tile count of each block
  int* cull_work;          // [2] zero between launches: next sub-chunk, warps finished
  unsigned long long* cull_rounds;  // rounds run (each 2 x 16 x 16 pair slots), accumulated
};

template <class Real>
void launch_pair(const PairArgs<Real>& a, int elec, bool energy, bool dump, int grid,
                 cudaStream_t s);

// Packing of block-local coordinates and LJ parameters into the sorted slots; with
// `only_after_rebuild` set, only when that rebuild flag is set (between rebuilds of a periodic
// list the integrator writes the packed coordinates).
template <class Real>
void launch_pack(int n_slots, const int* sorted_atom, const double* pos, const int* image,
                 const double* block_center, const double* qscaled, const double* half_sigma,
                 const double* two_sqrt_eps, void* posq, void* ljp, const Box<double>& box,
                 cudaStream_t s, const int* only_after_rebuild = nullptr);

// ---- PME -------------------------------------------------------------------------------
template <class Real>
struct PmeArgs {
  int n_atoms;
  const int* order;     // particle visiting order (sorted slots) or nullptr
  int n_order;
  const double* pos;
  const double* charge;
  int nx, ny, nz;
  double recip[3][3];
  long long* grid_fixed;  // [nx*ny*nz]
  Real* grid_real;        // [nx*ny*nz]
  void* grid_k;           // [nx*ny*(nz/2+1)] complex
  const Real* influence;  // [nx*ny*(nz/2+1)]
  const double* moduli;   // [nx + ny + nz] B-spline moduli |b(m)|^2 (pme.rs:240-259)
  long long* force;
  long long* energy;
  double alpha, volume;
};

template <class Real>
void launch_pme_spread(const PmeArgs<Real>& a, cudaStream_t s);

// Brick-owned PME gather for rectangular boxes: the grid is cut into bricks of kBrickEdge^3
// points (the last brick of an axis may be shorter) and one CTA gathers the particles whose
// stencil starts in its brick.  The particles that can reach a brick until the next
// neighbour-list rebuild are found through the rebuild's x-y columns (z-sorted): for each
// column and z layer of bricks, the slot ranges (two where the layer's reach wraps the box) of
// the particles whose rebuild position lies within the layer's reach, made at every rebuild.
constexpr int kBrickEdge = 14;
constexpr int kBrickMaxRanges = 256;  // slot ranges one brick gathers (columns x 2)
struct PmeBricks {
  int2* ranges;        // [n_cols * nb[2] * 2] (first slot, end slot)
  int4* base;          // [slots] this step's stencil base point per axis, w = 1 for a charged
                       //   particle with a finite position (0: it touches no grid point)
  void* frac;          // [slots] Real4: stencil fractions per axis, w = the charge as Real
  int n_slots;
  int nb[3];           // bricks per axis
  int grid[3];         // grid points per axis
  int n_col[2];        // x-y columns of the neighbour-list sort
  double len[3];       // box edge lengths (nm)
  double cell[3];      // grid spacing (nm)
  double below[3];     // reach of a brick below its lower faces: drift (plus slack)
  double above;        // reach above its upper faces: drift (plus slack)
};
void launch_pme_brick_ranges(const NlistArgs& a, const PmeBricks& b, cudaStream_t s);
template <class Real>
void launch_pme_brick_stencils(const PmeArgs<Real>& a, const PmeBricks& b, const NlistArgs& nl,
                               cudaStream_t s);
template <class Real>
void launch_pme_gather_bricks(const PmeArgs<Real>& a, const PmeBricks& b, const NlistArgs& nl,
                              cudaStream_t s);
// Influence table on the half spectrum for the current reciprocal box (device, f64 math).
struct PmeRecip {
  double m[3][3];
};
template <class Real>
void launch_pme_influence(Real* out, const double* moduli, int nx, int ny, int nz,
                          const PmeRecip& recip, double alpha, double volume, cudaStream_t s);
// Plan of the engine's own grid transform (it replaces the conversion kernel, the cuFFT pair
// and the convolution kernel): per axis the radices of the Stockham stages and
// the twiddle table W_n^m = exp(-2 pi i m / n), m < n (Real2 elements); block sizes of the
// forward-plane, x-pass and inverse-plane kernels; kz pencils per x-pass CTA.
struct PmeFft {
  int nrad[3];
  int rad[3][16];
  int threads[3];
  int pencils_x;
  const void* tw[3];
};
template <class Real>
size_t pme_transform_smem(const PmeArgs<Real>& a, const PmeFft& f, int kernel);
template <class Real>
void prepare_pme_transform(const PmeArgs<Real>& a, const PmeFft& f);
template <class Real>
void launch_pme_transform(const PmeArgs<Real>& a, const PmeFft& f, bool energy, cudaStream_t s);
template <class Real>
void launch_pme_convert(const PmeArgs<Real>& a, cudaStream_t s);
template <class Real>
void launch_pme_convolve(const PmeArgs<Real>& a, bool energy, cudaStream_t s);
template <class Real>
void launch_pme_gather(const PmeArgs<Real>& a, cudaStream_t s);

// ---- GBSAOBCForce --------------------------------------------------------------------------
// Particles in segment-padded slot order (one segment per independent system); tiles pair
// 32-slot blocks of the same segment.  energy[8 * segment] receives each segment's energy.
struct GbArgs {
  int n_atoms, n_slots, n_tiles;
  const int2* tiles;          // (I, J), I <= J
  const int* slot_atom;       // [n_slots], -1 = padding
  const int* block_segment;   // [n_slots / 32]
  const int* atom_segment;    // [n_atoms]
  const double* pos;
  const double* charge;
  const double* radius;
  const double* scale;
  double prefactor;           // -ke (1/eps_solute - 1/eps_solvent), gbsa_obc.rs:214-218
  double prefactor_sign;      // sign of the prefactor; charges are packed as q sqrt|prefactor|
  double charge_scale;        // sqrt|prefactor|
  double surface;             // 4 pi * surface-area energy
  int periodic, use_cutoff;
  double cutoff;
  Box<double> boxd;
  Box<float> boxf;
  void* posq;                 // [n_slots] Real4: x, y, z, q sqrt|prefactor|
  void* params;               // [n_slots] Real2: rho - 0.009, s (rho - 0.009)
  void* born_slot;            // [n_slots] Real2: Born radius and its reciprocal
  void* dedr_slot;            // [n_slots] Real: dE/dR R^2 chain
  long long* born_sum;        // [n_atoms] descreening sums, 2^-40
  long long* dedr_sum;        // [n_atoms] pair dE/dR sums, 2^-32
  double* born_radius;        // [n_atoms]
  double* chain;              // [n_atoms]
  double* dedr_self;          // [n_atoms]
  long long* force;
  long long* energy;
  // learned radii (null when off): while *use_learned is set the radii come from
  // I_short + tail and the exact descreening passes 1 and 3 are skipped
  const int* use_learned;
  const long long* short_sum;  // [n_atoms] switched short-range integral, 2^-40
  const float* tail;           // [n_atoms] network tail
  const float* seg_offset;     // [segments] tail offset per system
  // NonbondedForce (NoCutoff) fused into pass 2 while fuse_nonbonded is set: its tiles are the
  // GB tiles in the same order (every block pair of a segment), with their exclusion masks
  int fuse_nonbonded;
  const int4* nb_tiles;           // [n_tiles] (I, flags, mask slot, 0)
  const uint32_t* nb_masks;       // 32 per masked tile
  const double* nb_charge;        // [n_atoms] q sqrt(ke)
  const double* nb_half_sigma;    // [n_atoms] sigma / 2
  const double* nb_two_sqrt_eps;  // [n_atoms] 2 sqrt(epsilon)
  void* nb_params;                // [n_slots] Real4: q sqrt(ke), sigma / 2, 2 sqrt(eps), 0
};

// ---- learned Born radii (learned_gb.cu) -----------------------------------------------------
// Device control block of the learned-radii path.
struct LearnedState {
  int use_learned;  // this evaluation takes its radii from the network
  int judge;        // this evaluation judges the network against the exact pass
  int need;         // use_learned | judge: features and network run
  int active;       // the network passed the last judge
  int initialized;  // feature / target normalisation fixed
  int train;        // this judge retrains the network (first judge, or error above half the
                    // tolerance)
  unsigned long long judges, learned_evals, exact_evals;
  unsigned int max_err_bits;  // judge scratch: largest radius relative error (float bits)
  float last_error;           // largest per-particle radius relative error at the last judge
};
struct LearnedGbArgs {
  int n_atoms, n_blocks, max_nbr;
  const int* block_first;   // [n_blocks] first block of the block's segment
  const int* block_count;   // [n_blocks] blocks of that segment
  float4* block_box;        // [n_blocks][2] centre, half extents
  int* nbr;                 // [n_blocks][max_nbr] near blocks from the front, far from the back
  int* nbr_count;           // [n_blocks][2] near (within rf) and far (rf..rc) block counts
  float rc, rs;             // short-range integral cutoff and switch start (nm)
  float rf;                 // feature cutoff (nm), at most rc
  float* features;          // [n_atoms][32]
  float* tail;              // [n_atoms]
  float* dtail;             // [n_atoms][32] d tail / d features
  long long* short_sum;     // [n_atoms] switched short-range HCT integral, 2^-40
  float* params;            // [kRadiiMlpParams]
  float* moments;           // [2][kRadiiMlpTrainable]
  int* adam_t;
  float* snap_features;     // [n_atoms][32] judge snapshot
  float* snap_target;       // [n_atoms] exact minus short-range integral
  float* loss;              // [train_steps]
  int n_segments;           // independent systems (segments of the batch)
  const int* seg_first;     // [n_segments] first particle
  const int* seg_count;     // [n_segments] particles
  float* seg_offset;        // [n_segments] tail offset fixed at the last judge
  int train_steps, batch, judge_interval;
  float learning_rate, tolerance;
  unsigned long long seed;
  LearnedState* state;
  const unsigned long long* step;  // MD step counter
  int* status;                     // engine status word (tensor-core wait timeouts)
};
// Decides this evaluation's mode (judge every judge_interval MD steps when allowed).
void launch_learned_control(const LearnedGbArgs& a, bool judge_allowed, int step_offset,
                            cudaStream_t s);
// The learned-radii launches, in step order: lists (block boxes and short-range block lists),
// features (+ I_short), infer (network tail and gradient) before the GB radii; forces (learned
// evaluations), judge (+ normalisation), train and offsets (judge evaluations) after the chain
// step.  Every kernel returns at once when its evaluation does not need it.
enum LearnedPhase : int { kLrLists, kLrFeatures, kLrInfer, kLrForces, kLrJudge, kLrTrain,
                          kLrOffsets };
template <class Real>
void launch_learned_phase(const LearnedGbArgs& a, const GbArgs& g, int phase, int sm_count,
                          cudaStream_t s);

// GBSAOBCForce launches, in step order.
enum GbPhase : int { kGbPack, kGbPass1, kGbRadii, kGbPass2, kGbChain, kGbPass3 };
template <class Real>
void launch_gbsa_phase(const GbArgs& a, int phase, bool energy, int sm_count, cudaStream_t s);

// ---- exceptions and bonded terms (exceptions always in f64) ------------------------------
struct ExceptionArgs {
  int n;
  const int2* pairs;
  const double4* params;  // (charge_prod * ke, sigma, epsilon, q_i q_j * ke)
  const double* pos;
  long long* force;
  long long* energy;
  Box<double> box;
  int use_pbc;
  int ewald;
  double alpha;
  int n_atoms_for_force;  // row stride of the [3][N] force array
  const int* atom_segment;  // batch: system of each particle, energy at energy[8 * system]
};
void launch_exceptions(const ExceptionArgs& a, bool energy, cudaStream_t s);

struct BondedArgs {
  int n_bonds;
  const int2* bonds;
  const double2* bond_params;  // (length, k)
  int bond_pbc;
  int n_angles;
  const int4* angles;
  const double2* angle_params;  // (theta0, k)
  int angle_pbc;
  const double* pos;
  long long* force;
  long long* energy;
  Box<double> box;
  int n_atoms_for_force;
  const int* atom_segment;  // batch: system of each particle, energy at energy[8 * system]
};
void launch_bonded(const BondedArgs& a, bool energy, cudaStream_t s);

// ---- integration -----------------------------------------------------------------------
struct WaterGeometry {
  double d_oh, d_hh, m_o, m_h;
};

struct IntegrateArgs {
  int n_atoms;
  int n_water;
  const int4* water;  // (O, H1, H2, unused)
  WaterGeometry geom;
  int n_free;
  const int* free_atoms;
  int n_clusters;
  const int* cluster_start;       // [n_clusters + 1] into the constraint arrays
  const int2* cluster_pairs;      // constraint particle pairs
  const double* cluster_dist2;    // squared distances
  const int* cluster_atom_start;  // [n_clusters + 1] into cluster_atoms
  const int* cluster_atoms;
  double* pos;
  double* vel;
  double* scratch;                // [3N] SHAKE reference / proposal buffer
  long long* force;
  const double* inv_mass;
  double dt, decay, noise_var;    // noise_var = kT (1 - decay^2)
  double tolerance;
  uint64_t seed;
  const unsigned long long* rng_step;
  int step_offset;
  const double* pos_ref;          // neighbour-list reference positions (may be null)
  double half_skin2;
  int* rebuild;
  int* status;
  const double* pos_prune;        // positions at the last prune of the pair list (may be null)
  double half_margin2;            // (margin / 2)^2: a particle moved farther requests a prune
  int* prune;
  // MD steps only: the step zeroes every force it consumed (the next step's evaluation needs
  // no clearing), and, where `posq` is set (periodic lists), writes each moved particle's new
  // block-local position and charge into its slot of the pair kernel's packed coordinates
  int zero_force;
  void* posq;                     // float4 or double4 per slot
  int posq_double;
  const int* atom_slot;
  const int* image;               // lattice image of each particle at the last rebuild
  const double* block_center;
  const double* qscaled;
  Box<double> pbox;
};
void launch_integrate(const IntegrateArgs& a, cudaStream_t s);
// Barostat volume move: positions scaled, per particle or per molecule (CSR lists of atoms)
void launch_scale_positions(double* pos, int n_atoms, const int* mol_start, const int* mol_atoms,
                            int n_molecules, double scale, bool rigid, cudaStream_t s);
void launch_advance_counter(unsigned long long* counter, int by, cudaStream_t s);

// Velocity / position constraint projections used outside the step (apply_constraints,
// set_velocities_to_temperature).
void launch_constrain_positions(const IntegrateArgs& a, const double* reference, cudaStream_t s);
void launch_constrain_velocities(const IntegrateArgs& a, cudaStream_t s);

// ---- learned Born radii network (radii_mlp.cu) ------------------------------------------
// Flat float parameter block: W1[32][64], b1[64], W2[64][64], b2[64], w3[64], b3 (trainable),
// then feature mean[32], feature 1/std[32], target mean, target scale.
constexpr int kRadiiMlpParams = 6403;
constexpr int kRadiiMlpTrainable = 6337;
constexpr int kRadiiMlpOffMean = 6337, kRadiiMlpOffInvStd = 6369, kRadiiMlpOffTMean = 6401,
              kRadiiMlpOffTScale = 6402;
constexpr int kRadiiFeatures = 32;
// tail[n] = network output in integral units; dtail[n][32] = d tail / d features (may be null).
// `gate` (may be null): the kernel does nothing while *gate == 0.
void launch_mlp_infer(int n, const float* features, const float* params, float* tail,
                      float* dtail, int* status, int sm_count, cudaStream_t s,
                      const int* gate = nullptr);
// `steps` Adam steps on batches of `batch` (multiple of 128) particles drawn from the n
// snapshot rows (all of them in order when batch == n).  adam_m / adam_v hold the moments of
// the trainable block, *adam_t the step count; grad_out (may be null) receives the gradient of
// the last batch, loss_out[steps] (may be null) each batch's mean squared error.
// Polls of the tensor-core kernels' MMA completion waits (polls < 0: the default, about a
// millisecond); a smaller limit makes them give up, set the time-out status and return.
void set_tensor_wait_limit(long long polls);
void launch_mlp_train(int n, const float* features, const float* targets, float* params,
                      float* adam_m, float* adam_v, int* adam_t, int steps, int batch, float lr,
                      unsigned long long seed, float* grad_out, float* loss_out, int* status,
                      cudaStream_t s, const int* gate = nullptr);

}  // namespace ommb200
