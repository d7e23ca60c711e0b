// Device-side data of one pdgpu context and the kernel launchers shared by
// the FP64 kernels (pdgpu_kernels.cu), the mixed-precision bond loop
// (pdgpu_mixed.cu) and the host runtime (pdgpu_runtime.cu).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/pdgpu.h"

namespace pdgpu {

// node flag bits
enum : uint8_t {
  NODE_ACTIVE = 1,   // in d_fPdCompNodes: integrated, peridynamic force computed
  NODE_SEARCH = 2,   // searches for contact candidates (non-wall, computeForce, not all fixed)
  NODE_WALL = 4,     // node of a wall
  NODE_PARTICLE = 8, // node of a non-wall particle (receives particle damping)
  NODE_SEARCH0 = 16, // searched at DEMModel::init (before the two_particle override)
  NODE_UBC = 32,     // has displacement boundary-condition entries (ubc_of)
  NODE_FBC = 64,     // has force boundary-condition entries (fbc_of)
};

// device error codes (CtrlState::error)
enum : int {
  DEV_OK = 0,
  DEV_ERR_CONTACT_OVERFLOW = 1,
  DEV_ERR_WALLPAIR_OVERFLOW = 2,
  DEV_ERR_CELL_OVERFLOW = 3,
  DEV_ERR_NONFINITE = 4,
  DEV_ERR_STAGE_TIMEOUT = 5,  // a bond tile's bulk copies did not complete
  DEV_ERR_BARRIER_TIMEOUT = 6,  // a grid-wide barrier of the contact rebuild gave up
};

struct DevParticle {
  int64_t start, end, center;
  int32_t type, zone, compute_force, all_fixed, material, pad;
  double horizon, h, density, rc, kn, bound_r;
  double check_low, check_up;  // horizon -/+ 0.5 h (volume correction bounds)
  double mat[6];
};

struct ContactPair {
  double rc, kn, mu, betan, kappa;
};

constexpr int kDampGroup = 4;  // particles per damping CTA, at most (static shared memory)

struct DampParticle {
  double bound_r, density;
  int32_t zone, type;
  int32_t q0, q1;  // the particles of its scene (all particles outside an ensemble)
};

struct Influence {
  int32_t type;
  int32_t pad;
  double p0, p1;  // const: a0 | linear: a0, a1 | gaussian: alpha, beta
};

// Step control, resident on the device so that a whole step can be replayed
// from a CUDA graph without host work.
struct CtrlState {
  int64_t n;
  double time;
  // contact neighbour search (DEMModel::updateContactNeighborSearchParameters)
  int64_t interval, counter, init_calls;
  double radius;
  double max_velocity;
  unsigned long long vmax_bits;  // running max of |v| (non-negative doubles compare as integers)
  double static_vmax;            // |v| max over nodes that are never integrated
  int32_t update;                // this step rebuilds the contact candidate lists
  int32_t first_bc;              // zero-displacement sets still to be applied
  int64_t updates;
  int64_t entries;
  // device-side error word; once set, every kernel returns immediately
  int32_t error;
  int32_t pad;
  int64_t error_info;
  // post-processing results of the latest test step
  double reaction, contact_reaction, penetration;
  double pen_dist, max_y, contact_area_radius;
  int64_t history_count;
  int64_t c_nnodes;  // nodes with a non-empty contact candidate list
  // CTAs finished in the fused step kernels (the last one runs the serial tail)
  uint32_t begin_done, end_done;
  // tile claims and finished CTAs of the persistent bond loop (reset by its last CTA)
  uint32_t tile_next, tile_done;
  // learned surrogate: this step the bond loop runs for every particle and
  // the surrogate is judged against it (every sur_interval-th step)
  int32_t sur_check;
  int32_t pad2;
  // grid-wide barrier of the cooperative contact rebuild: arrivals of the
  // current barrier and the barriers passed so far
  uint32_t bar_count, bar_gen;
};

// Cell grid fixed at set-up; nodes outside are clamped to the border cells,
// which keeps every pair within one cell of each other in each direction.
struct Grid {
  double lo[3];
  double inv_cell;
  int32_t dims[3];
  int32_t ncells;
};

struct BcSetDev {
  int32_t time_fn, spatial_fn, dir_mask, zero;
  double tp[4];
  double sp[2];
};

// Per-particle constants of the FP32 bond loop (mixed precision form).
struct MixParticle {
  int64_t start;
  int32_t material, irreversible;
  float inv_horizon, check_low, check_up, inv_h;
  float rc, kn;
  float k_force;   // RNP: 4 C beta / invFactor | PMB, PD elastic: c | PD state: unused
  float beta, rbar, factor_sc, s0;
  float K, G;
  // util::isGreater(a, b) for a, b > 0 is a > b / (1 - 1e-5): thresholds
  float low_thr;   // volume correction applies beyond it (horizon - h/2)
  float fsc_thr;   // RNP: bond breaks when |S| sqrt(r) / rbar exceeds it
  float s0_thr;    // PMB: bond breaks when |S| exceeds it (s0 + 1e-10)
  float inv_rbar, inv_s0;  // damage Z = |S| / critical stretch
  float j0, j1;    // influence J(r): j0 + j1 r (constant, linear) | j0 2^(j1 r^2) (Gaussian)
  float tf_coef, am_coef;  // PD state: 3K - 5G and 15G
  float cu_h;      // check_up / h: corrected volume factor is cu_h - r / h
  float kj0, kj1;  // law constant times j0, j1 (PD state: j0, j1)
  float fsc_q;     // RNP: breaks when S^2 r exceeds (fsc_thr rbar)^2
  float nbeta_l2e; // RNP: -beta log2(e), exp(-beta r S^2) = 2^(nbeta_l2e S^2 r)
};

// One CTA of the tiled bond loop: nodes [node_begin, node_end) of one
// particle, whose bonds reach node indices inside [win_begin, win_end).
struct BondTile {
  int32_t particle;
  int32_t slots;  // symmetric mixed bond loop: bonds (i, j) with both nodes in the tile, i < j
  int64_t node_begin, node_end, win_begin, win_end;
  int64_t bond_begin, bond_end;  // pd_row[node_begin], pd_row[node_end]
  int64_t center;                // the particle's centre node
};

// one problem of a grouped tensor-core GEMM: C = act(A B^T + bias), A M x K
// and B N x K BF16 row-major, C FP32 (Cf) and/or BF16 (Cb)
struct GemmProblem {
  const void *A, *B;
  const float *bias;
  float *Cf;
  void *Cb;
  int32_t lda, ldb, ldc, M, N, K, act, pad;
};

// a particle of a surrogate zone: first node, centre node, orientation
// (cos, sin), 1 / scale, force scale, squared gate floor
struct SurPart {
  int64_t start, center;
  int32_t particle, pad;
  double c, s, inv_scale, fscale, floor2;
};

struct DevData {
  int32_t dim;
  int32_t precision;
  int64_t n_nodes;
  int32_t n_particles;
  int32_t n_zones;
  double dt;
  double gravity[3];
  int32_t gravity_on;
  int32_t time_scheme;

  // nodes (stride 2 doubles in 2-D, 4 in 3-D)
  double *xref, *x, *u, *v, *f;
  double *vol, *mx, *theta, *vmag;
  float *Z;
  int32_t *ptid;
  uint8_t *fix, *flags;

  // particles, contact, influence
  DevParticle *particles;
  ContactPair *contact;  // n_zones * n_zones
  Influence inf;

  // peridynamic bonds (CSR, one bit per bond: 1 = broken)
  int64_t n_bonds;
  int64_t *pd_row;
  int32_t *pd_col;
  uint32_t *bond_bits;

  // contact candidates (CSR)
  double max_contact_r, search_factor;
  double rc_max;  // largest contact radius of the zone-pair table (the contact pass's distance pre-filter)
  int64_t search_interval;
  int64_t contact_cap;
  int64_t *c_row;
  int32_t *c_col;
  int32_t *c_own;  // per candidate entry: its node (written with c_col)
  unsigned long long *phase_ns;  // rebuild phase clock (null: off), kRebuildPhases marks
  uint8_t *c_hit;  // per candidate entry, this step: inside the largest contact radius
  int64_t *c_cnt;  // per-node candidate counts of the last rebuild
  int64_t *c_tmp;  // N+1 scratch for the compaction scan
  int32_t *c_nodes;  // nodes with candidates, ascending
  int32_t contact_grid;  // blocks of the contact node pass
  Grid grid;
  int32_t *cell_of, *cell_cnt, *cell_start, *cell_fill, *cell_tmp, *cell_nodes;
  int32_t *cell_pid;  // contact rebuild: the particle of a cell's nodes when they share one, else -1
  int64_t cell_cap;  // max nodes in one cell handled by the in-cell sort

  // particle-wall damping pairs
  int32_t wp_cap;
  int32_t *wp, *wp_cnt;
  double *fdamp;  // n_particles * 4
  // contact force sum per node (node-vector layout), written by the contact
  // pass beside the bond loop and folded into f (then cleared) by the
  // external-force pass
  double *fc;
  // short dependency chains for the contact and damping passes
  int2 *c_span;          // [c_row[i], c_row[i + 1]) of compacted node t = c_nodes[t]
  uint16_t *nzone;        // zone of each node's particle
  DampParticle *dpart;   // per particle: bounding radius, density, zone, type
  // damping CTAs: group g holds particles damp_group[g] .. damp_group[g + 1] - 1
  // (consecutive, one scene, at most kDampGroup); null: one particle per CTA
  int32_t *damp_group;
  int32_t n_damp_groups;
  double *pcen;          // per particle, this step: {x, y, z, bounding radius, vx, vy, vz, -}
  float4 *pcen32;        // the same centre and bounding radius in FP32 (damping pre-filter)

  // boundary conditions: per BC node, a run of entries applied in set order
  int32_t n_ubc_sets, n_fbc_sets;
  BcSetDev *ubc_sets, *fbc_sets;
  int32_t n_ubc_nodes, n_fbc_nodes;
  int32_t *ubc_node, *ubc_row, *ubc_set;
  double *ubc_val;
  uint8_t *ubc_once;
  int32_t *fbc_node, *fbc_row, *fbc_set;
  double *fbc_val;
  int32_t *ubc_of, *fbc_of;  // per node: its row in the BC tables (valid where NODE_UBC / NODE_FBC)

  // initial condition
  int32_t ic_active;
  double ic_v[3];
  uint8_t *ic_particle;  // per particle: in the IC list

  // post-processing
  int32_t test;
  int64_t test_wall;
  int32_t test_dir;
  int64_t test_interval;
  int64_t history_cap;
  double *history;        // [cap][4]: t, delta, reaction, contact reaction
  double *cr_partial;     // contact-reaction partial sums per contact block
  int32_t cr_blocks;

  CtrlState *ctrl;

  // mixed-precision bond loop: particle-local FP32 reference coordinates,
  // FP32 volumes, particle-local 16-bit neighbour offsets when they fit
  uint16_t *pd_col16;
  // symmetric mixed bond loop (2-D): per bond, each node's row reordered as
  // [bonds to later nodes of its tile | bonds leaving the tile | bonds to
  // earlier nodes of its tile]; sym_col holds the particle-local neighbour
  // of the first two kinds and, for the third, the tile-local slot in which
  // the earlier node's thread leaves this node's share of their bond;
  // sym_pos the entry's offset in the node's row of pd_col.  sym_meta per
  // node: {first slot of its bonds to later nodes, count of those | count
  // of the first two kinds << 16}.
  uint16_t *sym_col, *sym_pos;
  uint2 *sym_meta;
  int32_t use_sym;
  // mixed bond loop, per-node form: position p of a tile processes node
  // node_order[p], the tile's nodes ordered by row length, longest first
  // (null: node order)
  int32_t *node_order;
  MixParticle *mixp;
  float4 *xv_mixed;  // per node {x, y, z, vol}: reference coordinates minus the centre's, FP32
  int32_t use16;
  float inf_p0, inf_p1;

  // the step a restart resumes from (pdgpu_restart), -1 without one
  int64_t restart_step;

  // batched ensemble (pdgpu_set_scenes): independent scenes side by side in
  // one model.  Per scene its node range and test wall; per particle whether
  // it is a scene's test wall; per compacted contact node its term of the
  // wall reaction; per scene the compressive-test history [cap][4].
  int32_t n_scenes;
  int64_t *scene_node;
  int32_t *scene_wall;
  uint8_t *pwall_test;
  double *cr_t;
  double *scene_hist;
  int64_t scene_hist_cap;

  // learned surrogate (pdgpu_set_surrogate): per particle the gate's verdict
  // at the last check, and whether the last contact-list rebuild found
  // contact candidates of its nodes (within contact radius plus skin, so no
  // contact can start before the next rebuild); the check interval (0 = no
  // surrogate) and whether the proximity flags are kept.  A particle is on
  // the surrogate when sur_on && !sur_near.
  uint8_t *sur_on;
  uint8_t *sur_near;
  // with the surrogate, one bond-loop launch over all tiles and a contact
  // rebuild every step: the rebuild kernel lists the tiles of the particles
  // off the surrogate (tile_live[0 .. *tile_live_n)), and the bond loop
  // claims from that list off check steps; tile_particle[t] is tile t's
  // particle.  Null otherwise.
  int32_t *tile_live;
  uint32_t *tile_live_n;
  const int32_t *tile_particle;
  int32_t n_tile_live_src;
  int32_t sur_interval;
  int32_t sur_near_gate;
};

// ---- launchers (all asynchronous on `s`) ----
// tensor-core GEMM of the surrogate: C = act(A B^T + bias) (pdgpu_tc.cu)
int launch_tc_gemm(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const float *bias,
                   int act, float *Cf, void *Cb, int ldc, int *err, cudaStream_t s);
int launch_tc_gemm_grouped(const GemmProblem *probs, int n_probs, int max_m, int max_n, int ncol, int *err,
                           cudaStream_t s);
// learned surrogate around the GEMMs (pdgpu_surrogate.cu)
void launch_sur_gather(const double *u, const SurPart *parts, int P, int n_nodes, void *A, int lda, float *Af,
                       cudaStream_t s);

// one surrogate shape as the per-step kernels see it (one launch covers
// every shape: blockIdx.y is the shape, blockIdx.x the particle row)
struct SurShapeDev {
  const SurPart *parts;
  int32_t P, n_nodes, kpad, pad;
  const void *phiT;  // 32 x kpad BF16; the CUDA-core chain's copy: 32 rows of
                     // sur_n_chunks(n_nodes) x 256 BF16, K-permuted (sur_kperm)
  void *xy;          // (P + 1) x 64 BF16: [network output | projected input]
  float *F;          // (P + 1) x kpad FP32: body-frame forces (check steps)
  float *xpart;      // (P + 1) x n_chunks x 32 FP32: the projection's partial sums
  int32_t n_chunks, pad2;
  // the CUDA-core chain's warp-MMA operands, BF16 row-major [out][in] with
  // each row's 16-bit pairs permuted within chunks of 64 inputs (32 for a
  // 32-input row) so that one lane's fragments of a chunk are contiguous
  // (sur_kperm): layer weights, the lift [kpad][64]; FP32 biases
  const void *w1m, *w2m, *w3m;
  const float *b1, *b2, *b3;
  const void *liftm;
};

int sm_count();  // SMs of the current device

// Position of 16-bit pair w (0 <= w < 32 or 16) in a K-permuted chunk of a
// row: a chunk holds ks m16n8k16 k-steps (4 for 64 inputs, 2 for 32); pair w
// = 8 kl + 4 h + t (k-step kl, fragment register h, lane t of a quad) goes
// to t * 2 ks + 2 kl + h, so that lane t's 2 ks pairs are adjacent.
__host__ __device__ inline int sur_kperm(int w, int ks) { return (w % 4) * 2 * ks + 2 * (w / 8) + (w / 4) % 2; }

// The surrogate's chain on CUDA cores, every shape in one launch per stage,
// the shapes by value in the kernel parameters (at most kMaxSurShapes):
// gather + projection in node chunks (sur_n_chunks(n_nodes) partial sums
// per row), the three layers, and the lift fused with the scatter into f
// (ordinary steps; on check steps into F, compared with the bond loop by
// launch_sur_check_all after it).
constexpr int kMaxSurShapes = 16;
struct SurShapes {
  SurShapeDev s[kMaxSurShapes];
  int32_t n;
};
int sur_n_chunks(int n_nodes);
void launch_sur_gather_project(const double *u, const SurShapes &shapes, int max_p, int max_nodes, cudaStream_t s);
void launch_sur_mlp(const SurShapes &shapes, int max_p, cudaStream_t s);
void launch_sur_lift_scatter(double *f, const SurShapes &shapes, int max_p, int max_nodes, const uint8_t *on,
                             const uint8_t *near, const CtrlState *ctrl, unsigned long long *count, cudaStream_t s);
void launch_sur_check_all(const DevData &d, const SurShapes &shapes, double *err2, float z_gate, double err_gate,
                          cudaStream_t s);
// the tensor-core chain's scatter (F from the lift GEMM) and gate
void launch_sur_scatter_all(double *f, const SurShapeDev *shapes, int n_shapes, int max_p, const uint8_t *on,
                            const uint8_t *near, const CtrlState *ctrl, double *err2, unsigned long long *count,
                            cudaStream_t s);
void launch_sur_gate_all(const DevData &d, const SurShapeDev *shapes, int n_shapes, int max_p, const double *err2,
                         float z_gate, double err_gate, cudaStream_t s);

void launch_pack_vec(const DevData &d, const double *aos3, double *dst, cudaStream_t s);
void launch_unpack_vec(const DevData &d, const double *src, double *aos3, cudaStream_t s);
void launch_apply_ic(const DevData &d, cudaStream_t s);
void launch_integrate(const DevData &d, int half_kick_only, cudaStream_t s);  // CD or Verlet first half
void launch_verlet_second(const DevData &d, cudaStream_t s);
void launch_ctrl(const DevData &d, int mode, cudaStream_t s);  // mode 0 step, 1 prelude, 2 init list
// integrate + displacement BC + step control (last CTA)
void launch_step_begin(const DevData &d, int verlet, cudaStream_t s);
// external forces + force BC (+ Verlet second half) + post-processing (last CTA)
void launch_step_end(const DevData &d, int verlet, int post, cudaStream_t s);
void launch_bc(const DevData &d, cudaStream_t s);
void launch_mixed_setup(const DevData &d, cudaStream_t s);
// symmetric layout: per node its tile (node_tile) -> counts (n_up, n_uo into
// sym_meta.y) -> slot bases from an exclusive scan of n_up (scan, N + 1) ->
// reordered rows; tiles get their slot counts
void launch_sym_count(const DevData &d, const BondTile *tiles, const int32_t *node_tile, int64_t *n_up,
                      cudaStream_t s);
void launch_sym_fill(const DevData &d, BondTile *tiles, int n_tiles, const int32_t *node_tile,
                     const int64_t *scan, cudaStream_t s);
void launch_node_tiles(const BondTile *tiles, int n_tiles, int32_t *node_tile, cudaStream_t s);
void launch_sym_bits(const DevData &d, const BondTile *tiles, const int32_t *node_tile, cudaStream_t s);
void launch_tile_windows(const DevData &d, BondTile *tiles, int n_tiles, cudaStream_t s);
// tiled bond loop (pdgpu_bonds_fp64.cu / pdgpu_bonds_mixed.cu)
void launch_pd_tiled_fp64(const DevData &d, const BondTile *tiles, int n_tiles, int lanes,
                          size_t smem, cudaStream_t s);
void launch_prepass_tiled_fp64(const DevData &d, const BondTile *tiles, int n_tiles, int lanes,
                               size_t smem, cudaStream_t s);
// law_begin[m] .. law_begin[m + 1]: the tiles of material law m (PDGPU_MAT_*)
void launch_pd_tiled_mixed(const DevData &d, const BondTile *tiles, const int *law_begin, int lanes,
                           size_t smem, cudaStream_t s);
void launch_prepass_tiled_mixed(const DevData &d, const BondTile *tiles, int n_tiles, int lanes,
                                size_t smem, cudaStream_t s);
// persistent PD state pre-pass of the mixed form over the state-based tiles
void launch_prepass_mixed(const DevData &d, const BondTile *tiles, const int *law_begin, int lanes,
                          size_t smem, cudaStream_t s);
size_t tile_smem_fp64(int dim, bool state, int64_t window);
size_t tile_smem_mixed(int dim, bool state, int64_t window);       // state pre-pass
size_t tile_smem_mixed_main(int dim, bool state, bool col16, const BondTile &t, bool sym = false);
int set_tile_smem_limit_fp64(int dim, size_t bytes);
int set_tile_smem_limit_mixed(int dim, size_t bytes);

void launch_contact_force(const DevData &d, int lanes, cudaStream_t s);
void launch_contact_owner(const DevData &d, cudaStream_t s);
// strain and stress at the quadrature points of linear triangles (2-D):
// three entries per element, nq <= 3 points (pts: xi, eta per point)
cudaError_t launch_strain_tri(const DevData &d, int64_t n_elem, const int64_t *conn, int nq, const double *pts,
                              const double *nu, const double *lam, const double *mu, const uint8_t *plane_strain,
                              double *xq, double *strain, double *stress, cudaStream_t s);
// the same for linear tetrahedra (3-D), the one-point rule
cudaError_t launch_strain_tet(const DevData &d, int64_t n_elem, const int64_t *conn, const double *nu,
                              const double *lam, const double *mu, double *xq, double *strain, double *stress,
                              cudaStream_t s);
constexpr int kRebuildPhases = 16;
int rebuild_grid_blocks(const DevData &d, int lanes);
cudaError_t launch_contact_rebuild(const DevData &d, int64_t *bsum, int grid, int lanes, int init,
                                   cudaStream_t s);
void launch_damping(const DevData &d, cudaStream_t s);
void launch_scene_post(const DevData &d, cudaStream_t s);  // per-scene test output of an ensemble
void launch_external(const DevData &d, cudaStream_t s);
void launch_postprocess(const DevData &d, cudaStream_t s);
void launch_build_pd(const DevData &d, double cell, int64_t *row_tmp, int32_t *cnt, void *scan_tmp,
                     size_t scan_bytes, int pass, cudaStream_t s);
void launch_compute_mx(const DevData &d, cudaStream_t s);
size_t scan_temp_bytes(int64_t n);
void launch_vec_reduce_check(const DevData &d, cudaStream_t s);

}  // namespace pdgpu
