// Host runtime of the pdgpu C ABI: context, uploads, the step sequence of
// DEMModel::integrate / integrateStep / computeForces, CUDA-graph replay,
// downloads and per-kernel timing.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "pdgpu_internal.h"

using namespace pdgpu;

namespace {

constexpr int kMaxTimed = 64;
constexpr int64_t kHistoryCap = 1 << 16;
constexpr int64_t kSceneHistCap = 1 << 12;  // test records per scene of an ensemble
// tail padding of the bond arrays: the bond loop copies whole 16-byte
// blocks of neighbour columns and bitmap words around each tile's range
constexpr int64_t kBondPad = 16;
constexpr int64_t kBitPad = 8;
constexpr int64_t kRowPad = 2;

struct TimedLaunch {
  int slot;
  cudaEvent_t a, b;
};

}  // namespace

struct pdgpu_ctx {
  pdgpu_desc desc{};
  cudaStream_t stream = nullptr;
  DevData d{};
  std::string err;

  bool nodes = false, particles = false, bonds = false, mx = false, contact = false;
  bool prepared = false, contact_init = false, begun = false;

  // host copies used for set-up
  std::vector<double> xref;      // N*3
  std::vector<int32_t> ptid;     // N
  std::vector<uint8_t> fix;      // N
  std::vector<double> vol_host;  // N, copied for output on first use
  std::vector<DevParticle> hp;   // particles
  std::vector<double> vmag0;     // initial |v|
  std::vector<uint8_t> ic_sel;   // per particle
  std::vector<BcSetDev> ubc_sets, fbc_sets;
  struct Entry {
    int32_t node, set;
    double val;
    uint8_t once;
  };
  std::vector<Entry> ubc_e, fbc_e;

  // scratch
  double *stage = nullptr;  // N*3 AoS staging
  void *scan_tmp = nullptr;
  size_t scan_bytes = 0;
  int pd_lanes = 0, contact_lanes = 1;
  int contact_ctas = 2;  // CTAs per SM of the contact node pass (two fit beside the bond loop)
  int64_t *rebuild_bsum = nullptr;
  int rebuild_grid = 0;
  // tiled bond loop
  BondTile *tiles = nullptr;
  int n_tiles = 0;
  size_t tile_smem = 0, tile_smem_state = 0;  // pre-pass stage; FP64 bond loop with m_x, theta
  size_t tile_smem_pd = 0;                     // the bond-loop launch
  size_t tile_smem_sym = 0;                    // the symmetric bond-loop launch (mixed, 2-D)
  int bond_scheme = 0;  // 0: per node, 1: symmetric where it applies, 2: per node longest row first
  int32_t *node_tile = nullptr;                // per node its bond tile (-1: none), symmetric form
  int tile_law[5] = {0, 0, 0, 0, 0};           // tiles of law m: [tile_law[m], tile_law[m + 1])
  int64_t tile_nodes = 0;  // nodes per tile (0 = chosen at set-up)
  bool state_prepass = false;

  // graph replay
  cudaGraphExec_t gexec = nullptr;
  int graph_steps = 0;
  // contact and damping run on `branch` beside the bond loop on `stream`
  cudaStream_t branch = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

  // batched ensemble (pdgpu_set_scenes): particle offsets (CSR) and test walls
  std::vector<int64_t> scene_poff, scene_walls;

  // learned surrogate (pdgpu_set_surrogate): per shape its particles, BF16
  // weights and the activations of the chain (P + 1 rows: row P is a zero
  // input, whose output the scatter subtracts)
  struct SurShape {
    int n_nodes = 0, kpad = 0, P = 0;
    SurPart *parts = nullptr;
    void *phiT = nullptr, *lift = nullptr, *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
    float *b1 = nullptr, *b2 = nullptr, *b3 = nullptr;
    void *A = nullptr, *xy = nullptr, *h1 = nullptr, *h2 = nullptr;
    float *F = nullptr, *xpart = nullptr;
    void *w1m = nullptr, *w2m = nullptr, *w3m = nullptr, *liftm = nullptr;  // CUDA-core chain layouts
    void *phim = nullptr;
  };
  std::vector<SurShape> sur;
  GemmProblem *sur_probs = nullptr;  // device: 5 stages x shapes
  int sur_max_p = 0, sur_max_k = 0;
  bool sur_fused = false;  // the CUDA-core chain runs
  int sur_chain = 0;       // requested chain: 0 CUDA cores, 1 tensor-core GEMMs
  SurShapeDev *sur_dev = nullptr;  // device: the shapes as the tensor-core chain's kernels see them
  SurShapes sur_shapes{};          // the same, by value for the CUDA-core chain
  int sur_max_rows = 0;            // largest particle count of a shape
  int sur_max_nodes = 0;           // largest node count of a shape
  double *sur_err2 = nullptr;        // per particle: squared error, squared norm (last check)
  int32_t *sur_errflag = nullptr;    // a tensor-core wait timed out
  unsigned long long *sur_count = nullptr;  // particle-steps on the surrogate, covered
  float sur_z_gate = 0.5f;
  double sur_err_gate = 0.05;
  cudaStream_t sur_stream = nullptr;
  cudaEvent_t ev_sur0 = nullptr, ev_sur1 = nullptr;

  // asynchronous VTU output (pdgpu_write_vtu_async): a device copy of the
  // state taken on the context stream, its download on out_stream into
  // pinned buffers, the file written by out_thread
  cudaStream_t out_stream = nullptr;
  cudaEvent_t ev_out0 = nullptr, ev_out1 = nullptr;
  double *out_dev = nullptr, *out_host = nullptr;  // [4 * stride * N + 2 * N + 1] doubles
  size_t out_doubles = 0;
  std::thread out_thread;
  int out_rc = 0;
  std::string out_err;

  // timing
  bool timing = false;
  std::vector<TimedLaunch> pending;
  std::vector<cudaEvent_t> pool;
  const char *names[kMaxTimed] = {};
  double ms[kMaxTimed] = {};
  int64_t launches[kMaxTimed] = {};
  int n_names = 0;

  // allocations to free
  std::vector<void *> allocs;
};

namespace {

int fail(pdgpu_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e__ = (call);                                                          \
    if (e__ != cudaSuccess)                                                            \
      return fail(ctx, PDGPU_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e__), \
                  __FILE__, __LINE__);                                                 \
  } while (0)

template <class T>
int dalloc(pdgpu_ctx *ctx, T **p, size_t count) {
  void *q = nullptr;
  size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess)
    return fail(ctx, PDGPU_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
  ctx->allocs.push_back(q);
  *p = (T *)q;
  return PDGPU_OK;
}

template <class T>
void dfree(pdgpu_ctx *ctx, T *&p) {
  if (!p) return;
  auto it = std::find(ctx->allocs.begin(), ctx->allocs.end(), (void *)p);
  if (it != ctx->allocs.end()) ctx->allocs.erase(it);
  cudaFree(p);
  p = nullptr;
}

#define TRY(x)                \
  do {                        \
    int r__ = (x);            \
    if (r__ != PDGPU_OK) return r__; \
  } while (0)

int stride(const pdgpu_ctx *ctx) { return ctx->desc.dim == 2 ? 2 : 4; }

// ---- timing ----
int timed_slot(pdgpu_ctx *c, const char *name) {
  for (int i = 0; i < c->n_names; i++)
    if (c->names[i] == name || std::strcmp(c->names[i], name) == 0) return i;
  if (c->n_names >= kMaxTimed) return -1;
  c->names[c->n_names] = name;
  return c->n_names++;
}

cudaEvent_t take_event(pdgpu_ctx *c) {
  if (!c->pool.empty()) {
    cudaEvent_t e = c->pool.back();
    c->pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

template <class F>
void run_on(pdgpu_ctx *c, cudaStream_t s, const char *name, F &&f) {
  if (!c->timing) {
    f();
    return;
  }
  const int slot = timed_slot(c, name);
  cudaEvent_t a = take_event(c), b = take_event(c);
  cudaEventRecord(a, s);
  f();
  cudaEventRecord(b, s);
  c->pending.push_back({slot, a, b});
}

template <class F>
void run(pdgpu_ctx *c, const char *name, F &&f) {
  run_on(c, c->stream, name, f);
}

void resolve_timing(pdgpu_ctx *c) {
  if (c->pending.empty()) return;
  cudaStreamSynchronize(c->stream);
  for (auto &t : c->pending) {
    float m = 0.f;
    cudaEventElapsedTime(&m, t.a, t.b);
    if (t.slot >= 0) {
      c->ms[t.slot] += m;
      c->launches[t.slot] += 1;
    }
    c->pool.push_back(t.a);
    c->pool.push_back(t.b);
  }
  c->pending.clear();
}

// ---- spatial factors of BC sets (particleULoading.cpp:146-172,
//      particleFLoading.cpp:112-134), evaluated once on the host ----
bool h_greater(double a, double b) {
  return (a - b) > ((std::abs(a) < std::abs(b) ? std::abs(b) : std::abs(a)) * 1.0e-5);
}
bool h_less(double a, double b) {
  return (b - a) > ((std::abs(a) < std::abs(b) ? std::abs(b) : std::abs(a)) * 1.0e-5);
}
// util::hatFunction (function.cpp:24-42)
double hat(double x, double lo, double hi) {
  if (h_greater(x, lo - 1.0E-12) && h_less(x, hi + 1.0E-12)) {
    const double mid = 0.5 * (lo + hi);
    const double l = mid - lo;
    if (l < 1.0E-12) return 1.0;
    if (h_less(x, mid)) return (x - lo) / l;
    return (hi - x) / l;
  }
  return 0.0;
}

double spatial_u(const BcSetDev &bc, const double *x, const double *box) {
  double umax = bc.tp[0];
  const double kPi = 3.14159265358979323846;
  switch (bc.spatial_fn) {
    case PDGPU_SPACE_HAT_X: umax = bc.sp[0] * hat(x[0], box[0], box[3]); break;
    case PDGPU_SPACE_HAT_Y: umax = bc.sp[0] * hat(x[1], box[1], box[4]); break;
    case PDGPU_SPACE_SIN_X: umax = umax * std::sin(kPi * bc.sp[0] * x[0]); break;
    case PDGPU_SPACE_SIN_Y: umax = umax * std::sin(kPi * bc.sp[0] * x[1]); break;
    case PDGPU_SPACE_LINEAR_X: umax = umax * bc.sp[0] * x[0]; break;
    case PDGPU_SPACE_LINEAR_Y: umax = umax * bc.sp[0] * x[1]; break;
    default: break;
  }
  return umax;
}

double spatial_f(const BcSetDev &bc, const double *x, const double *box) {
  double fmax = 1.0;
  const double kPi = 3.14159265358979323846;
  switch (bc.spatial_fn) {
    case PDGPU_SPACE_HAT_X: fmax = bc.sp[0] * hat(x[0], box[0], box[3]); break;
    case PDGPU_SPACE_HAT_Y: fmax = bc.sp[0] * hat(x[1], box[1], box[4]); break;
    case PDGPU_SPACE_SIN_X: fmax = bc.sp[0] * std::sin(kPi * bc.sp[0] * x[0]); break;
    case PDGPU_SPACE_SIN_Y: fmax = bc.sp[0] * std::sin(kPi * bc.sp[0] * x[1]); break;
    case PDGPU_SPACE_LINEAR_X: fmax = bc.sp[0] * bc.sp[0] * x[0]; break;
    case PDGPU_SPACE_LINEAR_Y: fmax = bc.sp[0] * bc.sp[0] * x[1]; break;
    default: break;
  }
  return fmax;
}

int add_bc(pdgpu_ctx *ctx, bool disp, const pdgpu_bc_set *set, const uint8_t *psel,
           const uint8_t *nsel, const double *pbox) {
  if (!ctx || !set || !psel || !nsel || !pbox) return fail(ctx, PDGPU_ERR_ARG, "add_bc: null argument");
  if (!ctx->nodes || !ctx->particles)
    return fail(ctx, PDGPU_ERR_STATE, "add_bc: upload nodes and particles first");
  if (ctx->prepared) return fail(ctx, PDGPU_ERR_STATE, "add_bc: boundary conditions are fixed once stepping starts");
  BcSetDev b{};
  b.time_fn = set->time_fn;
  b.spatial_fn = set->spatial_fn;
  b.dir_mask = set->dir_mask;
  b.zero = set->zero;
  for (int q = 0; q < 4; q++) b.tp[q] = set->time_params[q];
  for (int q = 0; q < 2; q++) b.sp[q] = set->spatial_params[q];
  auto &sets = disp ? ctx->ubc_sets : ctx->fbc_sets;
  auto &ent = disp ? ctx->ubc_e : ctx->fbc_e;
  const int sidx = (int)sets.size();
  sets.push_back(b);
  const int64_t np = (int64_t)ctx->hp.size();
  for (int64_t p = 0; p < np; p++) {
    if (!psel[p]) continue;
    // zero-displacement sets act once, at the first apply() call, which the
    // reference makes for particle 0 only (particleULoading.cpp:120-131)
    if (disp && b.zero && p != 0) continue;
    for (int64_t i = ctx->hp[p].start; i < ctx->hp[p].end; i++) {
      if (!nsel[i]) continue;
      const double *x = &ctx->xref[3 * i];
      const double v = disp ? spatial_u(b, x, pbox + 6 * p) : spatial_f(b, x, pbox + 6 * p);
      ent.push_back({(int32_t)i, sidx, v, (uint8_t)(disp && b.zero ? 1 : 0)});
    }
  }
  return PDGPU_OK;
}

int upload_bc_tables(pdgpu_ctx *ctx, bool disp) {
  auto &ent = disp ? ctx->ubc_e : ctx->fbc_e;
  auto &sets = disp ? ctx->ubc_sets : ctx->fbc_sets;
  std::stable_sort(ent.begin(), ent.end(), [](const pdgpu_ctx::Entry &a, const pdgpu_ctx::Entry &b) {
    return a.node < b.node;
  });
  std::vector<int32_t> nodes, row{0}, set;
  std::vector<double> val;
  std::vector<uint8_t> once;
  for (size_t k = 0; k < ent.size(); k++) {
    if (k == 0 || ent[k].node != ent[k - 1].node) {
      if (k) row.push_back((int32_t)k);
      nodes.push_back(ent[k].node);
    }
    set.push_back(ent[k].set);
    val.push_back(ent[k].val);
    once.push_back(ent[k].once);
  }
  if (!ent.empty()) row.push_back((int32_t)ent.size());
  DevData &d = ctx->d;
  BcSetDev *dsets;
  int32_t *dn, *dr, *ds;
  double *dv;
  TRY(dalloc(ctx, &dsets, sets.size()));
  TRY(dalloc(ctx, &dn, nodes.size()));
  TRY(dalloc(ctx, &dr, row.size()));
  TRY(dalloc(ctx, &ds, set.size()));
  TRY(dalloc(ctx, &dv, val.size()));
  if (!sets.empty()) CK(cudaMemcpy(dsets, sets.data(), sets.size() * sizeof(BcSetDev), cudaMemcpyHostToDevice));
  if (!nodes.empty()) {
    CK(cudaMemcpy(dn, nodes.data(), nodes.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dr, row.data(), row.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ds, set.data(), set.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dv, val.data(), val.size() * 8, cudaMemcpyHostToDevice));
  }
  if (disp) {
    uint8_t *donce;
    TRY(dalloc(ctx, &donce, once.size()));
    if (!once.empty()) CK(cudaMemcpy(donce, once.data(), once.size(), cudaMemcpyHostToDevice));
    d.n_ubc_sets = (int32_t)sets.size();
    d.ubc_sets = dsets;
    d.n_ubc_nodes = (int32_t)nodes.size();
    d.ubc_node = dn;
    d.ubc_row = dr;
    d.ubc_set = ds;
    d.ubc_val = dv;
    d.ubc_once = donce;
  } else {
    d.n_fbc_sets = (int32_t)sets.size();
    d.fbc_sets = dsets;
    d.n_fbc_nodes = (int32_t)nodes.size();
    d.fbc_node = dn;
    d.fbc_row = dr;
    d.fbc_set = ds;
    d.fbc_val = dv;
  }
  return PDGPU_OK;
}

// Grid of cells at least `cell` wide over the current positions (with a
// margin); positions outside are clamped to the border cells.
int make_grid(pdgpu_ctx *ctx, double cell, Grid *g) {
  const int dim = ctx->desc.dim;
  std::vector<double> x(3 * ctx->d.n_nodes);
  std::vector<double> tmp((size_t)stride(ctx) * ctx->d.n_nodes);
  CK(cudaMemcpy(tmp.data(), ctx->d.x, tmp.size() * 8, cudaMemcpyDeviceToHost));
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < ctx->d.n_nodes; i++)
    for (int q = 0; q < dim; q++) {
      lo[q] = std::min(lo[q], tmp[stride(ctx) * i + q]);
      hi[q] = std::max(hi[q], tmp[stride(ctx) * i + q]);
    }
  const int64_t limit = dim == 2 ? (int64_t)1 << 24 : (int64_t)1 << 26;
  for (;;) {
    int64_t total = 1;
    for (int q = 0; q < 3; q++) {
      if (q < dim) {
        const double margin = 4.0 * cell + 0.05 * (hi[q] - lo[q]);
        g->lo[q] = lo[q] - margin;
        g->dims[q] = (int32_t)std::max<double>(1.0, std::floor((hi[q] - lo[q] + 2 * margin) / cell));
      } else {
        g->lo[q] = 0.0;
        g->dims[q] = 1;
      }
      total *= g->dims[q];
    }
    if (total <= limit) {
      g->ncells = (int32_t)total;
      break;
    }
    cell *= 1.5;
  }
  // a cell is at least `cell` wide: floor() above can only widen it
  g->inv_cell = 1.0 / cell;
  for (int q = 0; q < dim; q++) {
    const double ext = (double)g->dims[q] * cell;
    (void)ext;
  }
  return PDGPU_OK;
}

int ensure_cells(pdgpu_ctx *ctx, const Grid &g) {
  DevData &d = ctx->d;
  if (d.cell_cnt && d.grid.ncells >= g.ncells) {
    d.grid = g;
    return PDGPU_OK;
  }
  dfree(ctx, d.cell_cnt);
  dfree(ctx, d.cell_start);
  dfree(ctx, d.cell_fill);
  dfree(ctx, d.cell_pid);
  TRY(dalloc(ctx, &d.cell_cnt, (size_t)g.ncells + 1));
  TRY(dalloc(ctx, &d.cell_start, (size_t)g.ncells + 1));
  TRY(dalloc(ctx, &d.cell_fill, (size_t)g.ncells + 1));
  TRY(dalloc(ctx, &d.cell_pid, (size_t)g.ncells + 1));
  CK(cudaMemset(d.cell_cnt, 0, ((size_t)g.ncells + 1) * 4));
  CK(cudaMemset(d.cell_fill, 0, ((size_t)g.ncells + 1) * 4));
  d.grid = g;
  const size_t need = scan_temp_bytes(std::max<int64_t>(d.n_nodes, (int64_t)g.ncells + 1) + 1);
  if (need > ctx->scan_bytes) {
    if (ctx->scan_tmp) {
      auto it = std::find(ctx->allocs.begin(), ctx->allocs.end(), ctx->scan_tmp);
      if (it != ctx->allocs.end()) ctx->allocs.erase(it);
      cudaFree(ctx->scan_tmp);
      ctx->scan_tmp = nullptr;
    }
    char *t;
    TRY(dalloc(ctx, &t, need));
    ctx->scan_tmp = t;
    ctx->scan_bytes = need;
  }
  return PDGPU_OK;
}

int read_ctrl(pdgpu_ctx *ctx, CtrlState *c) {
  CK(cudaMemcpyAsync(c, ctx->d.ctrl, sizeof(CtrlState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PDGPU_OK;
}

int device_error(pdgpu_ctx *ctx) {
  CtrlState c;
  TRY(read_ctrl(ctx, &c));
  switch (c.error) {
    case DEV_OK: return PDGPU_OK;
    case DEV_ERR_CONTACT_OVERFLOW:
      return fail(ctx, PDGPU_ERR_OVERFLOW,
                  "contact candidate list needs %lld entries, capacity is %lld (step %lld); "
                  "raise pdgpu_desc.contact_capacity",
                  (long long)c.error_info, (long long)ctx->d.contact_cap, (long long)c.n);
    case DEV_ERR_WALLPAIR_OVERFLOW:
      return fail(ctx, PDGPU_ERR_OVERFLOW,
                  "particle %lld has more particle-wall pairs than wall_pair_capacity=%d (step %lld)",
                  (long long)c.error_info, ctx->d.wp_cap, (long long)c.n);
    case DEV_ERR_STAGE_TIMEOUT:
      return fail(ctx, PDGPU_ERR_CUDA, "bond tile %lld: shared-memory bulk copies did not complete",
                  (long long)c.error_info);
    case DEV_ERR_BARRIER_TIMEOUT:
      return fail(ctx, PDGPU_ERR_CUDA, "contact-list rebuild: a grid-wide barrier gave up waiting (step %lld)",
                  (long long)c.n);
    case DEV_ERR_NONFINITE:
      return fail(ctx, PDGPU_ERR_NAN, "weighted volume of node %lld is too close to zero",
                  (long long)c.error_info);
    default:
      return fail(ctx, PDGPU_ERR_STATE, "device error %d (info %lld)", c.error, (long long)c.error_info);
  }
}

// FP32 constants per particle for the mixed-precision bond loop
int prepare_mixed(pdgpu_ctx *ctx) {
  DevData &d = ctx->d;
  const int64_t N = d.n_nodes;
  std::vector<MixParticle> mp(ctx->hp.size());
  bool fits16 = true;
  for (size_t k = 0; k < ctx->hp.size(); k++) {
    const DevParticle &P = ctx->hp[k];
    MixParticle &M = mp[k];
    M = MixParticle{};
    M.start = P.start;
    M.material = P.material;
    M.inv_horizon = (float)(1.0 / P.horizon);
    M.check_low = (float)P.check_low;
    M.check_up = (float)P.check_up;
    M.inv_h = (float)(1.0 / P.h);
    M.rc = (float)P.rc;
    M.kn = (float)P.kn;
    const double rel = 1.0 - 1.0e-5;  // util::isGreater's relative tolerance
    M.low_thr = (float)(P.check_low / rel);
    switch (P.material) {
      case PDGPU_MAT_RNP:
        M.k_force = (float)(4.0 * P.mat[0] * P.mat[1] / P.mat[3]);
        M.beta = (float)P.mat[1];
        M.rbar = (float)P.mat[2];
        M.factor_sc = (float)P.mat[4];
        M.irreversible = P.mat[5] != 0.0;
        M.inv_rbar = (float)(1.0 / P.mat[2]);
        M.fsc_thr = (float)(P.mat[4] / rel);
        break;
      case PDGPU_MAT_PMB:
        M.k_force = (float)P.mat[0];
        M.s0 = (float)P.mat[1];
        M.inv_s0 = (float)(1.0 / P.mat[1]);
        M.s0_thr = (float)((P.mat[1] + 1.0e-10) / rel);
        break;
      case PDGPU_MAT_PDELASTIC: M.k_force = (float)P.mat[0]; break;
      default:
        M.K = (float)P.mat[0];
        M.G = (float)P.mat[1];
        M.s0 = (float)P.mat[2];
        M.inv_s0 = (float)(1.0 / P.mat[2]);
        M.s0_thr = (float)((P.mat[2] + 1.0e-10) / rel);  // the pre-pass breaks bonds beyond it
        M.tf_coef = (float)(3.0 * P.mat[0] - 5.0 * P.mat[1]);
        M.am_coef = (float)(15.0 * P.mat[1]);
        break;
    }
    // influence function J(r / horizon) (material.h:273-288)
    const double ih = 1.0 / P.horizon;
    if (d.inf.type == PDGPU_INF_GAUSSIAN) {
      M.j0 = (float)d.inf.p0;
      M.j1 = (float)(-ih * ih / d.inf.p1 * 1.4426950408889634);  // exponent in base 2
    } else if (d.inf.type == PDGPU_INF_LINEAR) {
      M.j0 = (float)d.inf.p0;
      M.j1 = (float)(d.inf.p1 * ih);
    } else {
      M.j0 = (float)d.inf.p0;
      M.j1 = 0.f;
    }
    M.cu_h = (float)(P.check_up / P.h);
    const double kf = P.material == PDGPU_MAT_PDSTATE ? 1.0 : (double)M.k_force;
    M.kj0 = (float)(kf * d.inf.p0);
    M.kj1 = d.inf.type == PDGPU_INF_LINEAR ? (float)(kf * d.inf.p1 * ih) : 0.f;
    if (P.material == PDGPU_MAT_RNP) {
      const double t = (P.mat[4] / rel) * P.mat[2];
      M.fsc_q = (float)(t * t);
      M.nbeta_l2e = (float)(-P.mat[1] * 1.4426950408889634);
    }
    if (P.compute_force && P.end - P.start > 65536) fits16 = false;
  }
  TRY(dalloc(ctx, &d.mixp, mp.size()));
  CK(cudaMemcpy(d.mixp, mp.data(), mp.size() * sizeof(MixParticle), cudaMemcpyHostToDevice));
  d.use16 = fits16 ? 1 : 0;
  if (fits16) TRY(dalloc(ctx, &d.pd_col16, d.n_bonds + kBondPad));
  TRY(dalloc(ctx, &d.xv_mixed, N));
  d.inf_p0 = (float)d.inf.p0;
  d.inf_p1 = (float)d.inf.p1;
  launch_mixed_setup(d, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return PDGPU_OK;
}

// Tiles of the bond loop: every force-computing particle is cut into runs of
// tile_nodes consecutive nodes; the device finds each tile's neighbour window
// and the largest window fixes the shared-memory stage.
// The learned surrogate's list of bond-loop tiles (written each step by the
// contact rebuild kernel, read by the bond loop): kept when the surrogate is
// set, the steps rebuild contact lists (multi-particle scenes) and one
// bond-loop launch covers every tile (a single material law).
int setup_tile_list(pdgpu_ctx *ctx) {
  DevData &d = ctx->d;
  if (d.tile_live) {
    dfree(ctx, d.tile_live);
    dfree(ctx, d.tile_live_n);
    int32_t *tp0 = const_cast<int32_t *>(d.tile_particle);
    dfree(ctx, tp0);
    d.tile_live = nullptr;
    d.tile_live_n = nullptr;
    d.tile_particle = nullptr;
    d.n_tile_live_src = 0;
  }
  int laws = 0;
  for (int m = 0; m < 4; m++) laws += ctx->tile_law[m + 1] > ctx->tile_law[m];
  if (ctx->sur.empty() || !ctx->desc.multi_particle || !ctx->tiles || ctx->n_tiles <= 0 || laws != 1)
    return PDGPU_OK;
  std::vector<BondTile> t((size_t)ctx->n_tiles);
  CK(cudaMemcpy(t.data(), ctx->tiles, t.size() * sizeof(BondTile), cudaMemcpyDeviceToHost));
  std::vector<int32_t> part(t.size());
  for (size_t k = 0; k < t.size(); k++) part[k] = t[k].particle;
  int32_t *tp;
  TRY(dalloc(ctx, &tp, part.size()));
  CK(cudaMemcpy(tp, part.data(), part.size() * 4, cudaMemcpyHostToDevice));
  TRY(dalloc(ctx, &d.tile_live, part.size()));
  TRY(dalloc(ctx, &d.tile_live_n, 1));
  CK(cudaMemset(d.tile_live_n, 0, 4));
  d.tile_particle = tp;
  d.n_tile_live_src = ctx->n_tiles;
  return PDGPU_OK;
}

int prepare_tiles(pdgpu_ctx *ctx) {
  DevData &d = ctx->d;
  const bool mixed = d.precision == PDGPU_PREC_MIXED;
  const size_t limit = 227 * 1024 - 1024;  // dynamic stage; static shared memory on top
  // default: every thread of the 256-thread CTA has a node, and at least
  // 128 (2-D) or 96 (3-D) nodes per tile
  const int64_t tn0 = ctx->tile_nodes > 0 ? ctx->tile_nodes
                                          : std::max<int64_t>(d.dim == 2 ? 128 : 96, 256 / ctx->pd_lanes);
  for (int64_t tn : {tn0, (int64_t)64, (int64_t)32, (int64_t)16}) {
    std::vector<BondTile> t;
    for (size_t p = 0; p < ctx->hp.size(); p++) {
      const DevParticle &P = ctx->hp[p];
      if (!P.compute_force) continue;
      for (int64_t a = P.start; a < P.end; a += tn) {
        BondTile b{};
        b.particle = (int32_t)p;
        b.node_begin = a;
        b.node_end = std::min(P.end, a + tn);
        b.center = P.center;
        t.push_back(b);
      }
    }
    // ordered by material law: one bond-loop launch per law
    std::stable_sort(t.begin(), t.end(), [&](const BondTile &a, const BondTile &b) {
      return ctx->hp[a.particle].material < ctx->hp[b.particle].material;
    });
    for (int m = 0; m <= 4; m++) {
      ctx->tile_law[m] = 0;
      for (auto &b : t) ctx->tile_law[m] += ctx->hp[b.particle].material < m;
    }
    if (ctx->tiles) dfree(ctx, ctx->tiles);
    ctx->n_tiles = (int)t.size();
    if (t.empty()) return PDGPU_OK;
    TRY(dalloc(ctx, &ctx->tiles, t.size()));
    CK(cudaMemcpyAsync(ctx->tiles, t.data(), t.size() * sizeof(BondTile), cudaMemcpyHostToDevice,
                       ctx->stream));
    launch_tile_windows(d, ctx->tiles, ctx->n_tiles, ctx->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(t.data(), ctx->tiles, t.size() * sizeof(BondTile), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // every tile's window must hold its own nodes and fit the stage
    int64_t wmax = 0;
    for (auto &b : t) {
      const DevParticle &P = ctx->hp[b.particle];
      if (b.win_begin < 0 || b.win_end > d.n_nodes || b.win_begin > b.node_begin ||
          b.win_end < b.node_end || b.win_begin < P.start || b.win_end > P.end)
        return fail(ctx, PDGPU_ERR_STATE, "bond tile window [%lld, %lld) inconsistent with nodes [%lld, %lld)",
                    (long long)b.win_begin, (long long)b.win_end, (long long)b.node_begin,
                    (long long)b.node_end);
      if (b.bond_begin < 0 || b.bond_end < b.bond_begin || b.bond_end > d.n_bonds)
        return fail(ctx, PDGPU_ERR_STATE, "bond tile bonds [%lld, %lld) outside [0, %lld)",
                    (long long)b.bond_begin, (long long)b.bond_end, (long long)d.n_bonds);
      wmax = std::max(wmax, b.win_end - b.win_begin);
    }
    const size_t sm = mixed ? tile_smem_mixed(d.dim, false, wmax) : tile_smem_fp64(d.dim, false, wmax);
    const size_t ss = mixed ? tile_smem_mixed(d.dim, true, wmax) : tile_smem_fp64(d.dim, true, wmax);
    // bytes of the bond-loop launch: the FP64 form stages the window only;
    // the mixed form also holds each tile's columns and bitmap words
    size_t pd = ctx->state_prepass ? ss : sm;
    if (mixed) {
      pd = 0;
      for (auto &b : t)
        pd = std::max(pd, tile_smem_mixed_main(d.dim, ctx->hp[b.particle].material == PDGPU_MAT_PDSTATE,
                                               d.use16 != 0, b));
    }
    const size_t need = std::max(pd, ctx->state_prepass ? sm : (size_t)0);
    if (need > limit) continue;
    const int rc = mixed ? set_tile_smem_limit_mixed(d.dim, need) : set_tile_smem_limit_fp64(d.dim, need);
    if (rc != 0) return fail(ctx, PDGPU_ERR_CUDA, "cannot raise the shared-memory limit to %zu bytes", need);
    ctx->tile_smem = sm;
    ctx->tile_smem_state = ss;
    ctx->tile_smem_pd = pd;
    ctx->tile_nodes = tn;
    return setup_tile_list(ctx);
  }
  return fail(ctx, PDGPU_ERR_ARG,
              "a particle's bonds reach too far in node order for the shared-memory stage; "
              "order each particle's nodes spatially");
}

// Bond scheme 2: the per-node mixed bond loop walks each tile's nodes longest
// row first (stable), so the lanes of a warp have rows of similar length
// where in node order the short rows of a particle's rim idle the lanes
// beside them.  Each node's own sum is untouched, so results do not change.
// (On the 2-D compressive test node order measured ~5 % faster: the order
// scatters a warp's node records across the staged window.)
int prepare_order(pdgpu_ctx *ctx) {
  DevData &d = ctx->d;
  if (d.precision != PDGPU_PREC_MIXED || d.use_sym || ctx->bond_scheme != 2 || ctx->n_tiles == 0)
    return PDGPU_OK;
  const int64_t N = d.n_nodes;
  std::vector<int64_t> row((size_t)N + 1);
  CK(cudaMemcpy(row.data(), d.pd_row, ((size_t)N + 1) * 8, cudaMemcpyDeviceToHost));
  std::vector<BondTile> t((size_t)ctx->n_tiles);
  CK(cudaMemcpy(t.data(), ctx->tiles, t.size() * sizeof(BondTile), cudaMemcpyDeviceToHost));
  std::vector<int32_t> order((size_t)N);
  for (int64_t i = 0; i < N; i++) order[i] = (int32_t)i;
  for (const auto &b : t)
    std::stable_sort(order.begin() + b.node_begin, order.begin() + b.node_end, [&](int32_t a, int32_t c) {
      return row[a + 1] - row[a] > row[c + 1] - row[c];
    });
  if (!d.node_order) TRY(dalloc(ctx, &d.node_order, (size_t)N));
  CK(cudaMemcpy(d.node_order, order.data(), (size_t)N * 4, cudaMemcpyHostToDevice));
  return PDGPU_OK;
}

// both directions of a bond between two nodes of one tile share their broken
// state in the symmetric form (see k_sym_bits)
int sym_bits(pdgpu_ctx *ctx) {
  if (!ctx->d.use_sym) return PDGPU_OK;
  launch_sym_bits(ctx->d, ctx->tiles, ctx->node_tile, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return PDGPU_OK;
}

// The symmetric layout of the mixed 2-D bond loop (see pdgpu_bonds_mixed.cu):
// built on the device from the tiles and neighbour lists; used when every
// row and every tile's slot count fits 16 bits and the stage with the slots
// fits shared memory, else the per-node form stays.
int prepare_sym(pdgpu_ctx *ctx) {
  DevData &d = ctx->d;
  d.use_sym = 0;
  if (d.precision != PDGPU_PREC_MIXED || d.dim != 2 || !d.use16 || ctx->bond_scheme != 1 || ctx->n_tiles == 0)
    return PDGPU_OK;
  const int64_t N = d.n_nodes;
  std::vector<int64_t> row((size_t)N + 1);
  CK(cudaMemcpy(row.data(), d.pd_row, ((size_t)N + 1) * 8, cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < N; i++)
    if (row[i + 1] - row[i] >= 65536) return PDGPU_OK;
  if (!d.sym_col) {
    TRY(dalloc(ctx, &d.sym_col, d.n_bonds + kBondPad));
    TRY(dalloc(ctx, &d.sym_pos, d.n_bonds + kBondPad));
    TRY(dalloc(ctx, &d.sym_meta, (size_t)N + 2));
    CK(cudaMemset(d.sym_col, 0, (d.n_bonds + kBondPad) * 2));
    CK(cudaMemset(d.sym_pos, 0, (d.n_bonds + kBondPad) * 2));
    CK(cudaMemset(d.sym_meta, 0, ((size_t)N + 2) * sizeof(uint2)));
  }
  int64_t *n_up = nullptr, *scan_d = nullptr;
  if (!ctx->node_tile) TRY(dalloc(ctx, &ctx->node_tile, (size_t)N));
  int32_t *node_tile = ctx->node_tile;
  TRY(dalloc(ctx, &n_up, (size_t)N));
  TRY(dalloc(ctx, &scan_d, (size_t)N + 1));
  CK(cudaMemsetAsync(node_tile, 0xff, (size_t)N * 4, ctx->stream));
  launch_node_tiles(ctx->tiles, ctx->n_tiles, node_tile, ctx->stream);
  launch_sym_count(d, ctx->tiles, node_tile, n_up, ctx->stream);
  CK(cudaGetLastError());
  std::vector<int64_t> up((size_t)N), scan((size_t)N + 1, 0);
  CK(cudaMemcpyAsync(up.data(), n_up, (size_t)N * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int64_t i = 0; i < N; i++) scan[i + 1] = scan[i] + up[i];
  CK(cudaMemcpyAsync(scan_d, scan.data(), ((size_t)N + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
  launch_sym_fill(d, ctx->tiles, ctx->n_tiles, node_tile, scan_d, ctx->stream);
  CK(cudaGetLastError());
  std::vector<BondTile> t((size_t)ctx->n_tiles);
  CK(cudaMemcpyAsync(t.data(), ctx->tiles, t.size() * sizeof(BondTile), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  dfree(ctx, n_up);
  dfree(ctx, scan_d);
  size_t need = 0;
  for (auto &b : t) {
    if (b.slots < 0 || b.slots > 65535) return PDGPU_OK;
    need = std::max(need, tile_smem_mixed_main(2, ctx->hp[b.particle].material == PDGPU_MAT_PDSTATE, true, b, true));
  }
  const size_t limit = 227 * 1024 - 1024;
  if (need > limit) return PDGPU_OK;
  if (set_tile_smem_limit_mixed(2, std::max(need, ctx->tile_smem_pd)) != 0)
    return fail(ctx, PDGPU_ERR_CUDA, "cannot raise the shared-memory limit to %zu bytes", need);
  ctx->tile_smem_sym = need;
  d.use_sym = 1;
  return sym_bits(ctx);
}

// flags, BC tables, grid and contact buffers: done once before stepping
int prepare(pdgpu_ctx *ctx) {
  if (ctx->prepared) return PDGPU_OK;
  if (!ctx->nodes || !ctx->particles)
    return fail(ctx, PDGPU_ERR_STATE, "upload nodes and particles before stepping");
  if (!ctx->bonds) return fail(ctx, PDGPU_ERR_STATE, "peridynamic neighbour lists missing");
  if (!ctx->mx) return fail(ctx, PDGPU_ERR_STATE, "weighted volume m_x missing");
  if (ctx->desc.multi_particle && !ctx->contact)
    return fail(ctx, PDGPU_ERR_STATE, "contact parameters missing for a multi-particle run");
  DevData &d = ctx->d;
  const int64_t N = d.n_nodes;
  // node flags
  std::vector<uint8_t> flags(N, 0);
  double svmax = 0.0;
  int64_t nsearch = 0;
  for (size_t p = 0; p < ctx->hp.size(); p++) {
    const DevParticle &P = ctx->hp[p];
    for (int64_t i = P.start; i < P.end; i++) {
      uint8_t f = 0;
      if (P.compute_force) f |= NODE_ACTIVE;
      if (P.type == 1) f |= NODE_WALL;
      else f |= NODE_PARTICLE;
      if (P.type == 0 && P.compute_force && !P.all_fixed) f |= NODE_SEARCH;
      // DEMModel::init searches before the two_particle override
      if (P.type == 0 && !P.all_fixed) f |= NODE_SEARCH0;
      if (f & NODE_SEARCH) nsearch++;
      flags[i] = f;
      if (!(f & NODE_ACTIVE)) svmax = std::max(svmax, ctx->vmag0[i]);
    }
  }
  // BC tables (entries sorted by node), then the per-node BC rows
  TRY(upload_bc_tables(ctx, true));
  TRY(upload_bc_tables(ctx, false));
  for (int disp = 1; disp >= 0; disp--) {
    const auto &ent = disp ? ctx->ubc_e : ctx->fbc_e;
    std::vector<int32_t> of((size_t)N, -1);
    int32_t t = -1;
    for (size_t k = 0; k < ent.size(); k++) {
      if (k == 0 || ent[k].node != ent[k - 1].node) t++;
      of[ent[k].node] = t;
      flags[ent[k].node] |= disp ? NODE_UBC : NODE_FBC;
    }
    int32_t *dof;
    TRY(dalloc(ctx, &dof, (size_t)N));
    CK(cudaMemcpy(dof, of.data(), (size_t)N * 4, cudaMemcpyHostToDevice));
    (disp ? d.ubc_of : d.fbc_of) = dof;
  }
  TRY(dalloc(ctx, &d.flags, N));
  CK(cudaMemcpy(d.flags, flags.data(), N, cudaMemcpyHostToDevice));
  // IC particle flags
  TRY(dalloc(ctx, &d.ic_particle, ctx->hp.size()));
  if (ctx->ic_sel.size() != ctx->hp.size()) ctx->ic_sel.assign(ctx->hp.size(), 0);
  CK(cudaMemcpy(d.ic_particle, ctx->ic_sel.data(), ctx->hp.size(), cudaMemcpyHostToDevice));
  // lanes per node from the average bonds per node (measured on B200: the
  // FP32 form runs fastest with a thread per node at ~23 bonds per node)
  const double bpn = N ? (double)d.n_bonds / (double)N : 0.0;
  if (ctx->pd_lanes <= 0)
    ctx->pd_lanes = d.precision == PDGPU_PREC_MIXED ? (bpn > 48 ? 4 : 1)
                                                    : (bpn > 48 ? 32 : (bpn > 20 ? 8 : 4));
  // contact buffers
  {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // four CTAs per SM: the pass is bound by the latency of its gathers (a
    // cold L2 after every step), so it wants many candidates in flight; the
    // CTAs that find no free slot beside the bond loop start as it drains
    d.contact_grid = ctx->contact_ctas * (sms > 0 ? sms : 148);
  }
  d.cr_blocks = d.contact_grid;
  TRY(dalloc(ctx, &d.cr_partial, (size_t)d.cr_blocks + 1));
  CK(cudaMemset(d.cr_partial, 0, ((size_t)d.cr_blocks + 1) * 8));
  TRY(dalloc(ctx, &d.history, (size_t)kHistoryCap * 4));
  d.history_cap = kHistoryCap;
  TRY(dalloc(ctx, &d.fdamp, ctx->hp.size() * 4));
  CK(cudaMemset(d.fdamp, 0, ctx->hp.size() * 4 * 8));
  if (ctx->desc.multi_particle) {
    const size_t st = d.dim == 2 ? 2 : 4;
    TRY(dalloc(ctx, &d.fc, st * (size_t)N));
    CK(cudaMemset(d.fc, 0, st * (size_t)N * 8));
    if (!ctx->branch) {
      // highest priority: the branch's few latency-bound CTAs are scheduled
      // ahead of the bond loop's remaining tiles
      int lo = 0, hi = 0;
      CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
      CK(cudaStreamCreateWithPriority(&ctx->branch, cudaStreamDefault, hi));
    }
    if (!ctx->ev_fork) CK(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    if (!ctx->ev_join) CK(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  }
  TRY(dalloc(ctx, &d.c_row, (size_t)N + 1));
  CK(cudaMemset(d.c_row, 0, ((size_t)N + 1) * 8));
  TRY(dalloc(ctx, &d.c_cnt, (size_t)N));
  CK(cudaMemset(d.c_cnt, 0, (size_t)N * 8));
  TRY(dalloc(ctx, &d.c_tmp, (size_t)N + 1));
  TRY(dalloc(ctx, &d.c_nodes, (size_t)N));
  TRY(dalloc(ctx, &d.c_span, (size_t)N));
  CK(cudaMemset(d.c_span, 0, (size_t)N * sizeof(int2)));
  {
    // per-node zone and compact per-particle damping constants
    if (d.n_zones > 65535) return fail(ctx, PDGPU_ERR_ARG, "at most 65535 contact zones");
    std::vector<uint16_t> nz((size_t)N, 0);
    std::vector<DampParticle> dp(ctx->hp.size());
    const int ns = ctx->scene_poff.empty() ? 1 : (int)ctx->scene_poff.size() - 1;
    for (int sc = 0; sc < ns; sc++) {
      const int32_t q0 = ctx->scene_poff.empty() ? 0 : (int32_t)ctx->scene_poff[sc];
      const int32_t q1 = ctx->scene_poff.empty() ? (int32_t)ctx->hp.size() : (int32_t)ctx->scene_poff[sc + 1];
      for (int32_t p = q0; p < q1; p++) {
        const DevParticle &P = ctx->hp[p];
        for (int64_t i = P.start; i < P.end; i++) nz[i] = (uint16_t)P.zone;
        dp[p] = DampParticle{P.bound_r, P.density, P.zone, P.type, q0, q1};
      }
    }
    TRY(dalloc(ctx, &d.nzone, (size_t)N));
    CK(cudaMemcpy(d.nzone, nz.data(), (size_t)N * 2, cudaMemcpyHostToDevice));
    if (ns > 1) {
      // batched ensemble: scene node ranges, test walls and histories
      std::vector<int64_t> sn(ns + 1);
      std::vector<int32_t> sw(ns);
      std::vector<uint8_t> pw(ctx->hp.size(), 0);
      for (int sc = 0; sc < ns; sc++) {
        sn[sc] = ctx->hp[ctx->scene_poff[sc]].start;
        sw[sc] = (int32_t)ctx->scene_walls[sc];
        if (sw[sc] >= 0) pw[sw[sc]] = 1;
      }
      sn[ns] = N;
      d.n_scenes = ns;
      TRY(dalloc(ctx, &d.scene_node, sn.size()));
      CK(cudaMemcpy(d.scene_node, sn.data(), sn.size() * 8, cudaMemcpyHostToDevice));
      TRY(dalloc(ctx, &d.scene_wall, sw.size()));
      CK(cudaMemcpy(d.scene_wall, sw.data(), sw.size() * 4, cudaMemcpyHostToDevice));
      TRY(dalloc(ctx, &d.pwall_test, pw.size()));
      CK(cudaMemcpy(d.pwall_test, pw.data(), pw.size(), cudaMemcpyHostToDevice));
      TRY(dalloc(ctx, &d.cr_t, (size_t)N));
      CK(cudaMemset(d.cr_t, 0, (size_t)N * 8));
      d.scene_hist_cap = kSceneHistCap;
      TRY(dalloc(ctx, &d.scene_hist, (size_t)ns * kSceneHistCap * 4));
      CK(cudaMemset(d.scene_hist, 0, (size_t)ns * kSceneHistCap * 4 * 8));
      d.test_dir = ctx->desc.test_dir;
      d.test_interval = ctx->desc.test_interval > 0 ? ctx->desc.test_interval : 1;
    }
    TRY(dalloc(ctx, &d.dpart, dp.size()));
    CK(cudaMemcpy(d.dpart, dp.data(), dp.size() * sizeof(DampParticle), cudaMemcpyHostToDevice));
    // damping CTAs: with many particles, groups of consecutive particles of
    // one scene share each particle record they load (about 400 groups)
    const int group = std::min(kDampGroup, std::max(1, (int)(dp.size() / 400)));
    if (group > 1) {
      std::vector<int32_t> g{0};
      for (size_t p = 0; p < dp.size();) {
        size_t e = p + 1;
        while (e < dp.size() && (int)(e - p) < group && dp[e].q0 == dp[p].q0 && dp[e].q1 == dp[p].q1) e++;
        g.push_back((int32_t)e);
        p = e;
      }
      d.n_damp_groups = (int32_t)g.size() - 1;
      TRY(dalloc(ctx, &d.damp_group, g.size()));
      CK(cudaMemcpy(d.damp_group, g.data(), g.size() * 4, cudaMemcpyHostToDevice));
    }
    TRY(dalloc(ctx, &d.pcen, 8 * dp.size()));
    CK(cudaMemset(d.pcen, 0, 8 * dp.size() * 8));
    TRY(dalloc(ctx, &d.pcen32, dp.size()));
    CK(cudaMemset(d.pcen32, 0, dp.size() * sizeof(float4)));
  }
  if (ctx->desc.multi_particle) {
    d.contact_cap = ctx->desc.contact_capacity > 0 ? ctx->desc.contact_capacity
                                                   : std::max<int64_t>(64 * nsearch, 1 << 20);
    TRY(dalloc(ctx, &d.c_col, (size_t)d.contact_cap));
    TRY(dalloc(ctx, &d.c_own, (size_t)d.contact_cap));
    TRY(dalloc(ctx, &d.c_hit, (size_t)d.contact_cap));
    d.wp_cap = ctx->desc.wall_pair_capacity > 0 ? (int32_t)ctx->desc.wall_pair_capacity : 2048;
    if (d.wp_cap > 4096) return fail(ctx, PDGPU_ERR_ARG, "wall_pair_capacity is limited to 4096");
    TRY(dalloc(ctx, &d.wp, ctx->hp.size() * (size_t)d.wp_cap));
    TRY(dalloc(ctx, &d.wp_cnt, ctx->hp.size()));
    CK(cudaMemset(d.wp_cnt, 0, ctx->hp.size() * 4));
    TRY(dalloc(ctx, &d.cell_of, N));
    TRY(dalloc(ctx, &d.cell_tmp, N));
    TRY(dalloc(ctx, &d.cell_nodes, N));
    Grid g{};
    const double cell = std::max(1.0, ctx->desc.search_factor) * ctx->desc.max_contact_r;
    if (!(cell > 0)) return fail(ctx, PDGPU_ERR_ARG, "max_contact_r must be positive");
    TRY(make_grid(ctx, cell, &g));
    TRY(ensure_cells(ctx, g));
    ctx->rebuild_grid = rebuild_grid_blocks(d, ctx->contact_lanes);
    TRY(dalloc(ctx, &ctx->rebuild_bsum, (size_t)ctx->rebuild_grid + 1));
  }
  // step control
  CtrlState c{};
  c.interval = ctx->desc.search_interval;
  c.radius = ctx->desc.search_factor * ctx->desc.max_contact_r;
  c.static_vmax = svmax;
  c.first_bc = 1;
  CK(cudaMemcpy(d.ctrl, &c, sizeof c, cudaMemcpyHostToDevice));
  // the state pre-pass runs when particle 0 is state-based (demModel.cpp:607-610)
  ctx->state_prepass = !ctx->hp.empty() && ctx->hp[0].material == PDGPU_MAT_PDSTATE;
  if (d.precision == PDGPU_PREC_MIXED) TRY(prepare_mixed(ctx));
  TRY(prepare_tiles(ctx));
  TRY(prepare_sym(ctx));
  TRY(prepare_order(ctx));
  ctx->prepared = true;
  return PDGPU_OK;
}

// DEMModel::computeForces (demModel.cpp:462-600)
// DEMModel::computePeridynamicForces (demModel.cpp:602-789): state pre-pass
// and bond loop; writes f (peridynamic part) and Z, may break bonds
void pd_forces(pdgpu_ctx *ctx) {
  DevData &d = ctx->d;
  cudaStream_t s = ctx->stream;
  const bool mixed = d.precision == PDGPU_PREC_MIXED;
  if (ctx->state_prepass) {
    if (mixed)
      run(ctx, "pd_prepass_mixed", [&] {
        launch_prepass_mixed(d, ctx->tiles, ctx->tile_law, ctx->pd_lanes, ctx->tile_smem_pd, s);
      });
    else
      run(ctx, "pd_prepass", [&] {
        launch_prepass_tiled_fp64(d, ctx->tiles, ctx->n_tiles, ctx->pd_lanes, ctx->tile_smem, s);
      });
  }
  const size_t smem = d.use_sym ? ctx->tile_smem_sym : ctx->tile_smem_pd;
  if (mixed)
    run(ctx, "pd_force_mixed", [&] {
      launch_pd_tiled_mixed(d, ctx->tiles, ctx->tile_law, ctx->pd_lanes, smem, s);
    });
  else
    run(ctx, "pd_force", [&] {
      launch_pd_tiled_fp64(d, ctx->tiles, ctx->n_tiles, ctx->pd_lanes, smem, s);
    });
}

// The learned surrogate's chain for every particle of its zones, on its own
// stream beside the bond loop: gather the body-frame displacements, project
// (x = A phi^T), the three layers (y), and lift [y | x] to body-frame forces.
void sur_forward(pdgpu_ctx *ctx, cudaStream_t s) {
  const DevData &d = ctx->d;
  const int ns = (int)ctx->sur.size();
  const int pm = ctx->sur_max_p, km = ctx->sur_max_k;
  if (ctx->sur_fused) {
    // CUDA cores, every shape in one launch per stage: gather + projection
    // (a long reduction of little work per row, which tensor-core tiles walk
    // serially on a few CTAs), the three layers (a few rows per SM), and the
    // lift with the scatter into f for the particles whose tiles the bond
    // loop skips
    launch_sur_gather_project(d.u, ctx->sur_shapes, ctx->sur_max_rows, ctx->sur_max_nodes, s);
    launch_sur_mlp(ctx->sur_shapes, ctx->sur_max_rows, s);
    launch_sur_lift_scatter(d.f, ctx->sur_shapes, ctx->sur_max_rows, ctx->sur_max_nodes, d.sur_on, d.sur_near,
                            d.ctrl, ctx->sur_count, s);
    return;
  }
  for (auto &S : ctx->sur) launch_sur_gather(d.u, S.parts, S.P, S.n_nodes, S.A, S.kpad, nullptr, s);
  launch_tc_gemm_grouped(ctx->sur_probs + 0 * ns, ns, pm, 32, 32, ctx->sur_errflag, s);  // projection
  // 64-column tiles: four (layers) and kpad / 64 (lift) CTAs per 128-row
  // tile instead of one and kpad / 256
  launch_tc_gemm_grouped(ctx->sur_probs + 1 * ns, ns, pm, 256, 64, ctx->sur_errflag, s);  // layer 1
  launch_tc_gemm_grouped(ctx->sur_probs + 2 * ns, ns, pm, 256, 64, ctx->sur_errflag, s);  // layer 2
  launch_tc_gemm_grouped(ctx->sur_probs + 3 * ns, ns, pm, 32, 32, ctx->sur_errflag, s);   // layer 3
  launch_tc_gemm_grouped(ctx->sur_probs + 4 * ns, ns, pm, km, 64, ctx->sur_errflag, s);   // lift
}

// After the bond loop: on check steps the comparison with the bond loop and
// the gate; with the tensor-core chain also the surrogate forces into f on
// ordinary steps.
void sur_apply(pdgpu_ctx *ctx, cudaStream_t s) {
  const DevData &d = ctx->d;
  const int ns = (int)ctx->sur.size();
  if (ctx->sur_fused) {
    launch_sur_check_all(d, ctx->sur_shapes, ctx->sur_err2, ctx->sur_z_gate, ctx->sur_err_gate, s);
    return;
  }
  launch_sur_scatter_all(d.f, ctx->sur_dev, ns, ctx->sur_max_rows, d.sur_on, d.sur_near, d.ctrl, ctx->sur_err2,
                         ctx->sur_count, s);
  launch_sur_gate_all(d, ctx->sur_dev, ns, ctx->sur_max_rows, ctx->sur_err2, ctx->sur_z_gate, ctx->sur_err_gate, s);
}

// Contact forces and particle damping depend on positions and velocities
// only, not on the bond loop's forces: they run on the branch stream while
// the bond loop runs, and the external-force pass (after the join) adds
// their results to f in the reference's order: bond forces, contact forces,
// damping, external forces.
void compute_forces(pdgpu_ctx *ctx, bool step) {
  DevData &d = ctx->d;
  cudaStream_t s = ctx->stream;
  if (ctx->desc.multi_particle) {
    // the cooperative rebuild stays on the main stream, ahead of the fork
    run(ctx, "contact_update", [&] {
      launch_contact_rebuild(d, ctx->rebuild_bsum, ctx->rebuild_grid, ctx->contact_lanes, 0, s);
    });
    cudaEventRecord(ctx->ev_fork, s);
    cudaStreamWaitEvent(ctx->branch, ctx->ev_fork, 0);
    run_on(ctx, ctx->branch, "contact_force", [&] { launch_contact_force(d, ctx->contact_lanes, ctx->branch); });
    run_on(ctx, ctx->branch, "damping", [&] { launch_damping(d, ctx->branch); });
    cudaEventRecord(ctx->ev_join, ctx->branch);
  }
  const bool sur = step && !ctx->sur.empty();
  if (sur) {
    cudaEventRecord(ctx->ev_sur0, s);
    cudaStreamWaitEvent(ctx->sur_stream, ctx->ev_sur0, 0);
    run_on(ctx, ctx->sur_stream, "surrogate", [&] { sur_forward(ctx, ctx->sur_stream); });
    cudaEventRecord(ctx->ev_sur1, ctx->sur_stream);
  }
  pd_forces(ctx);
  if (sur) {
    cudaStreamWaitEvent(s, ctx->ev_sur1, 0);
    run(ctx, "surrogate_apply", [&] { sur_apply(ctx, s); });
  }
  if (ctx->desc.multi_particle) cudaStreamWaitEvent(s, ctx->ev_join, 0);
  // external forces and force BC; in a step also the Verlet second half and
  // the post-processing
  const bool verlet = ctx->desc.time_scheme == 1;
  run(ctx, "step_end", [&] { launch_step_end(d, step && verlet, step ? 1 : 0, s); });
  if (step && d.n_scenes > 1) run(ctx, "scene_post", [&] { launch_scene_post(d, s); });
}

// DEMModel::integrateStep (demModel.cpp:342-460) + post-processing
void one_step(pdgpu_ctx *ctx) {
  DevData &d = ctx->d;
  cudaStream_t s = ctx->stream;
  const bool verlet = ctx->desc.time_scheme == 1;
  // integrate, displacement BC, step control
  run(ctx, "step_begin", [&] { launch_step_begin(d, verlet ? 1 : 0, s); });
  compute_forces(ctx, true);
}

// One step inside a graph under capture: the same kernels as one_step,
// captured without the timing events.
cudaError_t graph_step(pdgpu_ctx *ctx, const char **where) {
  DevData &d = ctx->d;
  cudaStream_t s = ctx->stream;
  const bool verlet = ctx->desc.time_scheme == 1;
  const bool mixed = d.precision == PDGPU_PREC_MIXED;
  launch_step_begin(d, verlet ? 1 : 0, s);
  cudaError_t e = cudaSuccess;
  if (ctx->desc.multi_particle) {
    // contact-list rebuild: the single-launch cooperative kernel, which exits
    // at once on steps without a rebuild; on the main path, where nothing
    // else runs beside its grid-wide syncs
    *where = "contact-list rebuild";
    e = launch_contact_rebuild(d, ctx->rebuild_bsum, ctx->rebuild_grid, ctx->contact_lanes, 0, s);
    if (e != cudaSuccess) return e;
    // branch (captured first, so its kernels are dispatched ahead of the bond
    // loop's tiles): contact forces, then damping
    *where = "fork";
    e = cudaEventRecord(ctx->ev_fork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->branch, ctx->ev_fork, 0);
    if (e != cudaSuccess) return e;
    launch_contact_force(d, ctx->contact_lanes, ctx->branch);
    launch_damping(d, ctx->branch);
    e = cudaEventRecord(ctx->ev_join, ctx->branch);
    if (e != cudaSuccess) return e;
  }
  // surrogate chain beside the bond loop
  const bool sur = !ctx->sur.empty();
  if (sur) {
    *where = "surrogate fork";
    e = cudaEventRecord(ctx->ev_sur0, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->sur_stream, ctx->ev_sur0, 0);
    if (e != cudaSuccess) return e;
    sur_forward(ctx, ctx->sur_stream);
    e = cudaEventRecord(ctx->ev_sur1, ctx->sur_stream);
    if (e != cudaSuccess) return e;
  }
  // main: bond loop
  if (ctx->state_prepass) {
    if (mixed) launch_prepass_mixed(d, ctx->tiles, ctx->tile_law, ctx->pd_lanes, ctx->tile_smem_pd, s);
    else launch_prepass_tiled_fp64(d, ctx->tiles, ctx->n_tiles, ctx->pd_lanes, ctx->tile_smem, s);
  }
  const size_t smem = d.use_sym ? ctx->tile_smem_sym : ctx->tile_smem_pd;
  if (mixed) launch_pd_tiled_mixed(d, ctx->tiles, ctx->tile_law, ctx->pd_lanes, smem, s);
  else launch_pd_tiled_fp64(d, ctx->tiles, ctx->n_tiles, ctx->pd_lanes, smem, s);
  if (sur) {
    *where = "surrogate join";
    e = cudaStreamWaitEvent(s, ctx->ev_sur1, 0);
    if (e != cudaSuccess) return e;
    sur_apply(ctx, s);
  }
  if (ctx->desc.multi_particle) {
    *where = "join";
    e = cudaStreamWaitEvent(s, ctx->ev_join, 0);
    if (e != cudaSuccess) return e;
  }
  *where = "kernels after the join";
  launch_step_end(d, verlet ? 1 : 0, 1, s);
  launch_scene_post(d, s);
  return cudaGetLastError();
}

int build_graph(pdgpu_ctx *ctx, int steps) {
  cudaStream_t s = ctx->stream;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const char *where = "graph_step";
  cudaError_t e = cudaSuccess;
  int k = 0;
  for (; k < steps && e == cudaSuccess; k++) e = graph_step(ctx, &where);
  const cudaError_t e2 = cudaStreamEndCapture(s, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(ctx, PDGPU_ERR_CUDA, "graph capture failed in %s (step %d of %d): %s",
                e != cudaSuccess ? where : "cudaStreamEndCapture", k, steps,
                cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  e = cudaGraphInstantiate(&ctx->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(ctx, PDGPU_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
  ctx->graph_steps = steps;
  return PDGPU_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int pdgpu_device_check(int device, char *msg, size_t len) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  auto say = [&](const char *t) {
    if (msg && len) snprintf(msg, len, "%s", t);
  };
  if (e != cudaSuccess || n <= device) {
    say("no CUDA device visible");
    return PDGPU_ERR_NODEVICE;
  }
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) {
    say("cudaGetDeviceProperties failed");
    return PDGPU_ERR_NODEVICE;
  }
  if (p.major != 10 || p.minor != 0) {
    char b[128];
    snprintf(b, sizeof b, "device %d is sm_%d%d; this library is built for sm_100a", device, p.major,
             p.minor);
    say(b);
    return PDGPU_ERR_NODEVICE;
  }
  say(p.name);
  return PDGPU_OK;
}

int pdgpu_create(const pdgpu_desc *desc, pdgpu_ctx **out) {
  if (!desc || !out) return PDGPU_ERR_ARG;
  *out = nullptr;
  if (desc->dim != 2 && desc->dim != 3) return PDGPU_ERR_ARG;
  if (!(desc->dt > 0)) return PDGPU_ERR_ARG;
  if (desc->precision != PDGPU_PREC_FP64 && desc->precision != PDGPU_PREC_MIXED) return PDGPU_ERR_ARG;
  int rc = pdgpu_device_check(desc->device, nullptr, 0);
  if (rc != PDGPU_OK) return rc;
  auto *ctx = new pdgpu_ctx();
  ctx->desc = *desc;
  // a blocking stream: ordered with the legacy default stream, so plain
  // cudaMemcpy/cudaMemset calls of the set-up path never race the kernels
  if (cudaSetDevice(desc->device) != cudaSuccess || cudaStreamCreate(&ctx->stream) != cudaSuccess) {
    delete ctx;
    return PDGPU_ERR_CUDA;
  }
  DevData &d = ctx->d;
  d.dim = desc->dim;
  d.precision = desc->precision;
  d.dt = desc->dt;
  d.restart_step = -1;
  for (int q = 0; q < 3; q++) d.gravity[q] = desc->gravity[q];
  const double gl = std::sqrt(desc->gravity[0] * desc->gravity[0] + desc->gravity[1] * desc->gravity[1] +
                              desc->gravity[2] * desc->gravity[2]);
  d.gravity_on = gl > 1.0E-8;  // demModel.cpp:797
  d.time_scheme = desc->time_scheme;
  d.max_contact_r = desc->max_contact_r;
  d.search_factor = desc->search_factor;
  d.search_interval = desc->search_interval;
  d.test = desc->test;
  d.test_wall = desc->test_wall;
  d.test_dir = desc->test_dir;
  d.test_interval = desc->test_interval > 0 ? desc->test_interval : 1;
  if (dalloc(ctx, &d.ctrl, 1) != PDGPU_OK) {
    pdgpu_destroy(ctx);
    return PDGPU_ERR_NOMEM;
  }
  cudaMemset(d.ctrl, 0, sizeof(CtrlState));
  *out = ctx;
  return PDGPU_OK;
}

void pdgpu_destroy(pdgpu_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->desc.device);
  if (ctx->out_thread.joinable()) ctx->out_thread.join();
  if (ctx->out_stream) cudaStreamDestroy(ctx->out_stream);
  if (ctx->ev_out0) cudaEventDestroy(ctx->ev_out0);
  if (ctx->ev_out1) cudaEventDestroy(ctx->ev_out1);
  if (ctx->out_host) cudaFreeHost(ctx->out_host);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->branch) cudaStreamDestroy(ctx->branch);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  if (ctx->sur_stream) cudaStreamDestroy(ctx->sur_stream);
  if (ctx->ev_sur0) cudaEventDestroy(ctx->ev_sur0);
  if (ctx->ev_sur1) cudaEventDestroy(ctx->ev_sur1);
  for (auto &t : ctx->pending) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  for (auto e : ctx->pool) cudaEventDestroy(e);
  for (void *p : ctx->allocs) cudaFree(p);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int pdgpu_last_error(const pdgpu_ctx *ctx, char *buf, size_t len) {
  if (!ctx || !buf || !len) return PDGPU_ERR_ARG;
  snprintf(buf, len, "%s", ctx->err.c_str());
  return PDGPU_OK;
}

int pdgpu_upload_nodes(pdgpu_ctx *ctx, int64_t n, const double *xref, const double *x,
                       const double *u, const double *v, const double *vol, const uint8_t *fix,
                       const uint64_t *pt_id) {
  if (!ctx) return PDGPU_ERR_ARG;
  if (n <= 0 || n >= INT32_MAX || !xref || !vol || !fix || !pt_id)
    return fail(ctx, PDGPU_ERR_ARG, "upload_nodes: bad arguments (n=%lld)", (long long)n);
  if (ctx->nodes) return fail(ctx, PDGPU_ERR_STATE, "upload_nodes: nodes already uploaded");
  CK(cudaSetDevice(ctx->desc.device));
  DevData &d = ctx->d;
  d.n_nodes = n;
  const size_t sv = (size_t)stride(ctx) * n;
  TRY(dalloc(ctx, &d.xref, sv));
  TRY(dalloc(ctx, &d.x, sv));
  TRY(dalloc(ctx, &d.u, sv));
  TRY(dalloc(ctx, &d.v, sv));
  TRY(dalloc(ctx, &d.f, sv));
  TRY(dalloc(ctx, &d.vol, n));
  TRY(dalloc(ctx, &d.mx, n));
  TRY(dalloc(ctx, &d.theta, n));
  TRY(dalloc(ctx, &d.vmag, n));
  TRY(dalloc(ctx, &d.Z, n));
  TRY(dalloc(ctx, &d.ptid, n));
  TRY(dalloc(ctx, &d.fix, n));
  TRY(dalloc(ctx, &ctx->stage, (size_t)3 * n));
  CK(cudaMemset(d.f, 0, sv * 8));
  CK(cudaMemset(d.mx, 0, n * 8));
  CK(cudaMemset(d.theta, 0, n * 8));
  CK(cudaMemset(d.Z, 0, n * 4));
  CK(cudaMemset(d.xref, 0, sv * 8));
  cudaStream_t s = ctx->stream;
  auto put = [&](const double *src, double *dst) -> int {
    CK(cudaMemcpyAsync(ctx->stage, src, (size_t)3 * n * 8, cudaMemcpyHostToDevice, s));
    launch_pack_vec(d, ctx->stage, dst, s);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    return PDGPU_OK;
  };
  TRY(put(xref, d.xref));
  TRY(put(x ? x : xref, d.x));
  if (u) TRY(put(u, d.u));
  else CK(cudaMemset(d.u, 0, sv * 8));
  if (v) TRY(put(v, d.v));
  else CK(cudaMemset(d.v, 0, sv * 8));
  CK(cudaMemcpy(d.vol, vol, n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.fix, fix, n, cudaMemcpyHostToDevice));
  ctx->ptid.resize(n);
  for (int64_t i = 0; i < n; i++) {
    if (pt_id[i] > (uint64_t)INT32_MAX) return fail(ctx, PDGPU_ERR_ARG, "particle id out of range");
    ctx->ptid[i] = (int32_t)pt_id[i];
  }
  CK(cudaMemcpy(d.ptid, ctx->ptid.data(), n * 4, cudaMemcpyHostToDevice));
  ctx->xref.assign(xref, xref + 3 * n);
  ctx->fix.assign(fix, fix + n);
  ctx->vmag0.assign(n, 0.0);
  if (v)
    for (int64_t i = 0; i < n; i++)
      ctx->vmag0[i] = std::sqrt(v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
  // |v| as held by ModelData::d_vMag at upload (zero after init)
  CK(cudaMemcpy(d.vmag, ctx->vmag0.data(), n * 8, cudaMemcpyHostToDevice));
  ctx->nodes = true;
  return PDGPU_OK;
}

int pdgpu_upload_particles(pdgpu_ctx *ctx, int64_t np, const pdgpu_particle *p) {
  if (!ctx) return PDGPU_ERR_ARG;
  if (!ctx->nodes) return fail(ctx, PDGPU_ERR_STATE, "upload_particles: upload nodes first");
  if (np <= 0 || !p) return fail(ctx, PDGPU_ERR_ARG, "upload_particles: bad arguments");
  if (ctx->particles) return fail(ctx, PDGPU_ERR_STATE, "upload_particles: already uploaded");
  ctx->hp.resize(np);
  for (int64_t k = 0; k < np; k++) {
    DevParticle &P = ctx->hp[k];
    P = DevParticle{};
    P.start = p[k].glob_start;
    P.end = p[k].glob_end;
    P.center = p[k].center_node;
    if (P.start < 0 || P.end > ctx->d.n_nodes || P.start >= P.end || P.center < P.start || P.center >= P.end)
      return fail(ctx, PDGPU_ERR_ARG, "particle %lld: bad node range", (long long)k);
    P.type = p[k].type;
    P.zone = p[k].zone;
    P.compute_force = p[k].compute_force;
    P.all_fixed = p[k].all_dofs_constrained;
    P.material = p[k].material;
    if (P.material < 0 || P.material > 3) return fail(ctx, PDGPU_ERR_ARG, "particle %lld: bad material", (long long)k);
    P.horizon = p[k].horizon;
    P.h = p[k].h;
    P.density = p[k].density;
    P.rc = p[k].rc;
    P.kn = p[k].kn;
    P.bound_r = p[k].bound_r;
    // bounds of the volume correction (demModel.cpp:636-637, 708-709)
    P.check_up = P.horizon + 0.5 * P.h;
    P.check_low = P.horizon - 0.5 * P.h;
    for (int q = 0; q < 6; q++) P.mat[q] = p[k].mat[q];
    for (int64_t i = P.start; i < P.end; i++)
      if (ctx->ptid[i] != (int32_t)k)
        return fail(ctx, PDGPU_ERR_ARG, "node %lld: particle id %d does not match particle range %lld",
                    (long long)i, ctx->ptid[i], (long long)k);
  }
  DevData &d = ctx->d;
  d.n_particles = (int32_t)np;
  TRY(dalloc(ctx, &d.particles, np));
  CK(cudaMemcpy(d.particles, ctx->hp.data(), np * sizeof(DevParticle), cudaMemcpyHostToDevice));
  ctx->particles = true;
  return PDGPU_OK;
}

int pdgpu_set_influence(pdgpu_ctx *ctx, int32_t type, const double params[2]) {
  if (!ctx || !params || type < 0 || type > 2) return fail(ctx, PDGPU_ERR_ARG, "set_influence: bad arguments");
  ctx->d.inf.type = type;
  ctx->d.inf.p0 = params[0];
  ctx->d.inf.p1 = params[1];
  return PDGPU_OK;
}

int pdgpu_upload_contact(pdgpu_ctx *ctx, int32_t nz, const double *rc, const double *kn,
                         const double *mu, const double *betan, const double *kappa) {
  if (!ctx || nz <= 0 || !rc || !kn || !mu || !betan || !kappa)
    return fail(ctx, PDGPU_ERR_ARG, "upload_contact: bad arguments");
  std::vector<ContactPair> cp((size_t)nz * nz);
  double rc_max = 0.0;
  for (size_t k = 0; k < cp.size(); k++) {
    cp[k] = {rc[k], kn[k], mu[k], betan[k], kappa[k]};
    if (rc[k] > rc_max) rc_max = rc[k];  // a NaN radius is skipped: is_less(R, NaN) never holds
  }
  DevData &d = ctx->d;
  d.rc_max = rc_max;
  if (!d.contact) TRY(dalloc(ctx, &d.contact, cp.size()));
  CK(cudaMemcpy(d.contact, cp.data(), cp.size() * sizeof(ContactPair), cudaMemcpyHostToDevice));
  d.n_zones = nz;
  for (auto &P : ctx->hp)
    if (P.zone < 0 || P.zone >= nz) return fail(ctx, PDGPU_ERR_ARG, "particle zone out of range");
  ctx->contact = true;
  return PDGPU_OK;
}

int pdgpu_upload_pd_neighbors(pdgpu_ctx *ctx, const uint64_t *rowptr, const uint64_t *col,
                              const uint8_t *bond_state) {
  if (!ctx || !rowptr || !col) return fail(ctx, PDGPU_ERR_ARG, "upload_pd_neighbors: null argument");
  if (!ctx->nodes) return fail(ctx, PDGPU_ERR_STATE, "upload nodes first");
  if (ctx->bonds) return fail(ctx, PDGPU_ERR_STATE, "neighbour lists already set");
  DevData &d = ctx->d;
  const int64_t N = d.n_nodes;
  const int64_t B = (int64_t)rowptr[N];
  std::vector<int64_t> row(N + 1);
  std::vector<int32_t> c32(B);
  for (int64_t i = 0; i <= N; i++) {
    row[i] = (int64_t)rowptr[i];
    if (i && row[i] < row[i - 1]) return fail(ctx, PDGPU_ERR_ARG, "rowptr not monotone at %lld", (long long)i);
  }
  for (int64_t k = 0; k < B; k++) {
    if (col[k] >= (uint64_t)N) return fail(ctx, PDGPU_ERR_ARG, "neighbour index out of range");
    c32[k] = (int32_t)col[k];
  }
  std::vector<uint32_t> bits((B + 31) / 32 + kBitPad, 0u);
  if (bond_state)
    for (int64_t k = 0; k < B; k++)
      if (bond_state[k]) bits[k >> 5] |= 1u << (k & 31);
  d.n_bonds = B;
  TRY(dalloc(ctx, &d.pd_row, N + 1 + kRowPad));
  TRY(dalloc(ctx, &d.pd_col, B + kBondPad));
  TRY(dalloc(ctx, &d.bond_bits, bits.size()));
  CK(cudaMemcpy(d.pd_row, row.data(), (N + 1) * 8, cudaMemcpyHostToDevice));
  if (B) CK(cudaMemcpy(d.pd_col, c32.data(), B * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d.bond_bits, bits.data(), bits.size() * 4, cudaMemcpyHostToDevice));
  ctx->bonds = true;
  return PDGPU_OK;
}

int pdgpu_build_pd_neighbors(pdgpu_ctx *ctx) {
  if (!ctx) return PDGPU_ERR_ARG;
  if (!ctx->nodes || !ctx->particles) return fail(ctx, PDGPU_ERR_STATE, "upload nodes and particles first");
  if (ctx->bonds) return fail(ctx, PDGPU_ERR_STATE, "neighbour lists already set");
  DevData &d = ctx->d;
  const int64_t N = d.n_nodes;
  double hmax = 0.0;
  for (auto &P : ctx->hp) hmax = std::max(hmax, P.horizon);
  if (!(hmax > 0)) return fail(ctx, PDGPU_ERR_ARG, "horizon must be positive");
  Grid g{};
  TRY(make_grid(ctx, hmax, &g));
  if (!d.cell_of) TRY(dalloc(ctx, &d.cell_of, N));
  if (!d.cell_tmp) TRY(dalloc(ctx, &d.cell_tmp, N));
  if (!d.cell_nodes) TRY(dalloc(ctx, &d.cell_nodes, N));
  TRY(ensure_cells(ctx, g));
  TRY(dalloc(ctx, &d.pd_row, N + 1 + kRowPad));
  CK(cudaMemset(d.pd_row, 0, (N + 1) * 8));
  // the cell kernels run only when ctrl.update is set
  CtrlState c{};
  c.update = 1;
  CK(cudaMemcpy(d.ctrl, &c, sizeof c, cudaMemcpyHostToDevice));
  launch_build_pd(d, hmax, d.pd_row, nullptr, ctx->scan_tmp, ctx->scan_bytes, 0, ctx->stream);
  CK(cudaGetLastError());
  int64_t B = 0;
  CK(cudaMemcpyAsync(&B, d.pd_row + N, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  d.n_bonds = B;
  TRY(dalloc(ctx, &d.pd_col, B + kBondPad));
  int32_t *tmp;
  TRY(dalloc(ctx, &tmp, B));
  launch_build_pd(d, hmax, d.pd_row, tmp, ctx->scan_tmp, ctx->scan_bytes, 1, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  dfree(ctx, tmp);
  TRY(dalloc(ctx, &d.bond_bits, (B + 31) / 32 + kBitPad));
  CK(cudaMemset(d.bond_bits, 0, ((B + 31) / 32 + kBitPad) * 4));
  CtrlState z{};
  CK(cudaMemcpy(d.ctrl, &z, sizeof z, cudaMemcpyHostToDevice));
  ctx->bonds = true;
  return PDGPU_OK;
}

int pdgpu_upload_mx(pdgpu_ctx *ctx, const double *mx) {
  if (!ctx || !mx) return fail(ctx, PDGPU_ERR_ARG, "upload_mx: null argument");
  if (!ctx->nodes) return fail(ctx, PDGPU_ERR_STATE, "upload nodes first");
  CK(cudaMemcpy(ctx->d.mx, mx, ctx->d.n_nodes * 8, cudaMemcpyHostToDevice));
  ctx->mx = true;
  return PDGPU_OK;
}

int pdgpu_compute_mx(pdgpu_ctx *ctx) {
  if (!ctx) return PDGPU_ERR_ARG;
  if (!ctx->bonds || !ctx->particles) return fail(ctx, PDGPU_ERR_STATE, "neighbour lists and particles first");
  CtrlState z{};
  CK(cudaMemcpy(ctx->d.ctrl, &z, sizeof z, cudaMemcpyHostToDevice));
  launch_compute_mx(ctx->d, ctx->stream);
  CK(cudaGetLastError());
  TRY(device_error(ctx));
  ctx->mx = true;
  return PDGPU_OK;
}

int pdgpu_add_displacement_bc(pdgpu_ctx *ctx, const pdgpu_bc_set *set, const uint8_t *psel,
                              const uint8_t *nsel, const double *pbox) {
  return add_bc(ctx, true, set, psel, nsel, pbox);
}

int pdgpu_add_force_bc(pdgpu_ctx *ctx, const pdgpu_bc_set *set, const uint8_t *psel,
                       const uint8_t *nsel, const double *pbox) {
  return add_bc(ctx, false, set, psel, nsel, pbox);
}

int pdgpu_set_initial_condition(pdgpu_ctx *ctx, const double vel[3], const uint64_t *plist,
                                int64_t n) {
  if (!ctx || !vel || (n > 0 && !plist)) return fail(ctx, PDGPU_ERR_ARG, "set_initial_condition: bad arguments");
  if (!ctx->particles) return fail(ctx, PDGPU_ERR_STATE, "upload particles first");
  ctx->ic_sel.assign(ctx->hp.size(), 0);
  for (int64_t k = 0; k < n; k++) {
    if (plist[k] >= ctx->hp.size()) return fail(ctx, PDGPU_ERR_ARG, "IC particle out of range");
    ctx->ic_sel[plist[k]] = 1;
  }
  ctx->d.ic_active = 1;
  for (int q = 0; q < 3; q++) ctx->d.ic_v[q] = vel[q];
  return PDGPU_OK;
}

int pdgpu_init_contact(pdgpu_ctx *ctx) {
  if (!ctx) return PDGPU_ERR_ARG;
  TRY(prepare(ctx));
  if (!ctx->desc.multi_particle) return PDGPU_OK;
  if (ctx->contact_init) return fail(ctx, PDGPU_ERR_STATE, "contact lists already initialised");
  launch_ctrl(ctx->d, 2, ctx->stream);
  CK(launch_contact_rebuild(ctx->d, ctx->rebuild_bsum, ctx->rebuild_grid, ctx->contact_lanes, 1,
                            ctx->stream));
  // no bond loop follows this rebuild: clear the surrogate's tile list
  if (ctx->d.tile_live) CK(cudaMemsetAsync(ctx->d.tile_live_n, 0, 4, ctx->stream));
  TRY(device_error(ctx));
  ctx->contact_init = true;
  return PDGPU_OK;
}

int pdgpu_integrate_begin(pdgpu_ctx *ctx) {
  if (!ctx) return PDGPU_ERR_ARG;
  TRY(prepare(ctx));
  if (ctx->desc.multi_particle && !ctx->contact_init) TRY(pdgpu_init_contact(ctx));
  if (ctx->begun) return fail(ctx, PDGPU_ERR_STATE, "integrate_begin called twice");
  DevData &d = ctx->d;
  cudaStream_t s = ctx->stream;
  if (d.restart_step > 0) {
    // DEMModel::restart (demModel.cpp:84-102): step and time of the restart
    CtrlState c;
    CK(cudaMemcpy(&c, d.ctrl, sizeof c, cudaMemcpyDeviceToHost));
    c.n = d.restart_step;
    c.time = (double)d.restart_step * d.dt;
    CK(cudaMemcpy(d.ctrl, &c, sizeof c, cudaMemcpyHostToDevice));
  }
  // DEMModel::integrate (demModel.cpp:277-283): the initial condition only at step 0
  if (d.ic_active && d.restart_step <= 0) run(ctx, "initial_condition", [&] { launch_apply_ic(d, s); });
  run(ctx, "displacement_bc", [&] { launch_bc(d, s); });
  run(ctx, "ctrl", [&] { launch_ctrl(d, 1, s); });
  compute_forces(ctx, false);
  CK(cudaGetLastError());
  TRY(device_error(ctx));
  ctx->begun = true;
  return PDGPU_OK;
}

int pdgpu_step(pdgpu_ctx *ctx, int64_t nsteps) {
  if (!ctx || nsteps < 0) return PDGPU_ERR_ARG;
  if (!ctx->begun) return fail(ctx, PDGPU_ERR_STATE, "call pdgpu_integrate_begin first");
  for (int64_t k = 0; k < nsteps; k++) one_step(ctx);
  CK(cudaGetLastError());
  return PDGPU_OK;
}

int pdgpu_step_graph(pdgpu_ctx *ctx, int64_t nsteps, int32_t graph_steps) {
  if (!ctx || nsteps < 0 || graph_steps <= 0) return PDGPU_ERR_ARG;
  if (!ctx->begun) return fail(ctx, PDGPU_ERR_STATE, "call pdgpu_integrate_begin first");
  if (ctx->gexec && ctx->graph_steps != graph_steps) {
    cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
  }
  if (!ctx->gexec) TRY(build_graph(ctx, graph_steps));
  int64_t left = nsteps;
  while (left >= graph_steps) {
    CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
    left -= graph_steps;
  }
  for (int64_t k = 0; k < left; k++) one_step(ctx);
  CK(cudaGetLastError());
  return PDGPU_OK;
}

int pdgpu_step_kernel_count(pdgpu_ctx *ctx, int64_t *count) {
  if (!ctx || !count) return PDGPU_ERR_ARG;
  if (!ctx->begun) return fail(ctx, PDGPU_ERR_STATE, "call pdgpu_integrate_begin first");
  const bool was_timing = ctx->timing;
  ctx->timing = false;
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  one_step(ctx);
  CK(cudaStreamEndCapture(ctx->stream, &g));
  ctx->timing = was_timing;
  size_t n = 0;
  CK(cudaGraphGetNodes(g, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  CK(cudaGraphGetNodes(g, nodes.data(), &n));
  int64_t k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    CK(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) k++;
  }
  cudaGraphDestroy(g);
  *count = k;
  return PDGPU_OK;
}

int pdgpu_sync(pdgpu_ctx *ctx) {
  if (!ctx) return PDGPU_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  resolve_timing(ctx);
  return device_error(ctx);
}

int pdgpu_download(pdgpu_ctx *ctx, int32_t field, void *dst) {
  if (!ctx || !dst) return PDGPU_ERR_ARG;
  if (!ctx->nodes) return fail(ctx, PDGPU_ERR_STATE, "no nodes");
  DevData &d = ctx->d;
  const int64_t N = d.n_nodes;
  cudaStream_t s = ctx->stream;
  double *vec = nullptr;
  switch (field) {
    case PDGPU_FIELD_X: vec = d.x; break;
    case PDGPU_FIELD_U: vec = d.u; break;
    case PDGPU_FIELD_V: vec = d.v; break;
    case PDGPU_FIELD_F: vec = d.f; break;
    case PDGPU_FIELD_Z: CK(cudaMemcpyAsync(dst, d.Z, N * 4, cudaMemcpyDeviceToHost, s)); break;
    case PDGPU_FIELD_VMAG: CK(cudaMemcpyAsync(dst, d.vmag, N * 8, cudaMemcpyDeviceToHost, s)); break;
    case PDGPU_FIELD_THETA: CK(cudaMemcpyAsync(dst, d.theta, N * 8, cudaMemcpyDeviceToHost, s)); break;
    case PDGPU_FIELD_MX: CK(cudaMemcpyAsync(dst, d.mx, N * 8, cudaMemcpyDeviceToHost, s)); break;
    case PDGPU_FIELD_FIX: CK(cudaMemcpyAsync(dst, d.fix, N, cudaMemcpyDeviceToHost, s)); break;
    case PDGPU_FIELD_BONDS: {
      if (!ctx->bonds) return fail(ctx, PDGPU_ERR_STATE, "no bonds");
      std::vector<uint32_t> bits((d.n_bonds + 31) / 32 + 1);
      CK(cudaMemcpyAsync(bits.data(), d.bond_bits, bits.size() * 4, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      uint8_t *o = (uint8_t *)dst;
      for (int64_t k = 0; k < d.n_bonds; k++) o[k] = (bits[k >> 5] >> (k & 31)) & 1u;
      return PDGPU_OK;
    }
    default: return fail(ctx, PDGPU_ERR_ARG, "download: unknown field %d", field);
  }
  if (vec) {
    launch_unpack_vec(d, vec, ctx->stage, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, ctx->stage, (size_t)3 * N * 8, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  return PDGPU_OK;
}

// ---- VTU output and restart ----
}  // extern "C"

namespace {

// one appended block: UInt64 byte count, then the bytes
struct VtuArray {
  std::string name, type;
  int comps;
  std::vector<unsigned char> bytes;
  std::vector<std::string> comp_names;  // optional; x, y, z for three components
};

template <typename T>
VtuArray vtu_array(const std::string &name, const char *type, int comps, const std::vector<T> &v) {
  VtuArray a{name, type, comps, {}};
  a.bytes.resize(v.size() * sizeof(T));
  if (!v.empty()) std::memcpy(a.bytes.data(), v.data(), a.bytes.size());
  return a;
}

bool has_tag(const std::string &tags, const char *tag) {
  size_t b = 0;
  while (b <= tags.size()) {
    size_t e = tags.find(',', b);
    if (e == std::string::npos) e = tags.size();
    std::string t = tags.substr(b, e - b);
    while (!t.empty() && t.front() == ' ') t.erase(t.begin());
    while (!t.empty() && t.back() == ' ') t.pop_back();
    if (t == tag) return true;
    b = e + 1;
  }
  return false;
}

// host copy of what one .vtu file holds (AoS util::Point arrays)
struct VtuFrame {
  int64_t n = 0;
  double time = 0.;
  std::vector<double> x, u, v, f, theta;
  std::vector<float> Z;
};

bool write_points_vtu(const char *path, int64_t N, double t, const std::vector<double> &points,
                      const std::vector<VtuArray> &pdata, std::string *err);

// The arrays of VtkParticleWriter::appendNodes (vtkParticleWriter.cpp:39-270),
// in its order, as raw appended VTK XML.  Host work only (safe on another
// thread: reads the frame and the context's constant host arrays).
bool write_frame(const pdgpu_ctx *ctx, const VtuFrame &fr, const std::string &T, const char *path,
                 std::string *err) {
  const int64_t N = fr.n;
  std::vector<VtuArray> pdata;
  auto vec3 = [&](const std::vector<double> &src, const char *name, bool times_vol) {
    std::vector<double> v(src);
    if (times_vol)
      for (int64_t i = 0; i < N; i++)
        for (int q = 0; q < 3; q++) v[3 * i + q] *= ctx->vol_host[i];
    pdata.push_back(vtu_array(name, "Float64", 3, v));
  };
  if (has_tag(T, "Displacement")) vec3(fr.u, "Displacement", false);
  if (has_tag(T, "Velocity")) vec3(fr.v, "Velocity", false);
  if (has_tag(T, "Force_Density")) vec3(fr.f, "Force_Density", false);
  if (has_tag(T, "Force")) vec3(fr.f, "Force", true);
  if (has_tag(T, "Fixity")) {
    std::vector<double> v(N);
    for (int64_t i = 0; i < N; i++) v[i] = (double)ctx->fix[i];
    pdata.push_back(vtu_array("Fixity", "Float64", 1, v));
  }
  if (has_tag(T, "Particle_ID")) {
    std::vector<double> v(N);
    for (int64_t i = 0; i < N; i++) v[i] = (double)ctx->ptid[i];
    pdata.push_back(vtu_array("Particle_ID", "Float64", 1, v));
  }
  if (has_tag(T, "Zone_ID")) {
    std::vector<double> v(N);
    for (int64_t i = 0; i < N; i++) v[i] = (double)ctx->hp[ctx->ptid[i]].zone;
    pdata.push_back(vtu_array("Zone_ID", "Float64", 1, v));
  }
  if (has_tag(T, "Nodal_Volume")) pdata.push_back(vtu_array("Nodal_Volume", "Float64", 1, ctx->vol_host));
  if (has_tag(T, "Damage_Z"))
    pdata.push_back(vtu_array("Damage_Z", "Float64", 1, std::vector<double>(fr.Z.begin(), fr.Z.end())));
  if (has_tag(T, "Theta") && !fr.theta.empty()) pdata.push_back(vtu_array("Theta", "Float64", 1, fr.theta));
  return write_points_vtu(path, N, fr.time, fr.x, pdata, err);
}

// A points-only unstructured grid (no cells) with a TIME field and the given
// point arrays, as raw appended VTK XML.
bool write_points_vtu(const char *path, int64_t N, double t, const std::vector<double> &points,
                      const std::vector<VtuArray> &pdata, std::string *err) {
  const VtuArray time = vtu_array("TIME", "Float64", 1, std::vector<double>{t});
  const VtuArray pts = vtu_array("Points", "Float64", 3, points);
  const VtuArray conn = vtu_array("connectivity", "Int64", 1, std::vector<int64_t>{});
  const VtuArray offs = vtu_array("offsets", "Int64", 1, std::vector<int64_t>{});
  const VtuArray types = vtu_array("types", "UInt8", 1, std::vector<uint8_t>{});
  std::vector<const VtuArray *> order{&time};
  for (auto &a : pdata) order.push_back(&a);
  order.push_back(&pts);
  order.push_back(&conn);
  order.push_back(&offs);
  order.push_back(&types);
  std::vector<uint64_t> off(order.size());
  uint64_t o = 0;
  for (size_t k = 0; k < order.size(); k++) {
    off[k] = o;
    o += 8 + order[k]->bytes.size();
  }
  auto decl = [&](size_t k, int64_t tuples) {
    const VtuArray &a = *order[k];
    std::string s = "<DataArray type=\"" + a.type + "\" Name=\"" + a.name + "\"";
    if (a.comps > 1) {
      s += " NumberOfComponents=\"" + std::to_string(a.comps) + "\"";
      if (!a.comp_names.empty()) {
        for (size_t c = 0; c < a.comp_names.size(); c++)
          s += " ComponentName" + std::to_string(c) + "=\"" + a.comp_names[c] + "\"";
      } else if (a.comps == 3) {
        s += " ComponentName0=\"x\" ComponentName1=\"y\" ComponentName2=\"z\"";
      }
    }
    if (tuples >= 0) s += " NumberOfTuples=\"" + std::to_string(tuples) + "\"";
    s += " format=\"appended\" offset=\"" + std::to_string(off[k]) + "\"/>\n";
    return s;
  };
  std::string head = "<?xml version=\"1.0\"?>\n"
                     "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" "
                     "header_type=\"UInt64\">\n<UnstructuredGrid>\n<FieldData>\n";
  head += decl(0, 1);
  head += "</FieldData>\n<Piece NumberOfPoints=\"" + std::to_string(N) + "\" NumberOfCells=\"0\">\n<PointData>\n";
  for (size_t k = 1; k <= pdata.size(); k++) head += decl(k, -1);
  head += "</PointData>\n<Points>\n" + decl(pdata.size() + 1, -1) + "</Points>\n<Cells>\n";
  for (size_t k = pdata.size() + 2; k < order.size(); k++) head += decl(k, -1);
  head += "</Cells>\n</Piece>\n</UnstructuredGrid>\n<AppendedData encoding=\"raw\">\n_";
  FILE *f = std::fopen(path, "wb");
  if (!f) {
    *err = std::string("cannot open ") + path;
    return false;
  }
  bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
  for (auto *a : order) {
    const uint64_t nb = a->bytes.size();
    ok = ok && std::fwrite(&nb, 8, 1, f) == 1;
    if (nb) ok = ok && std::fwrite(a->bytes.data(), 1, nb, f) == nb;
  }
  const char *tail = "\n</AppendedData>\n</VTKFile>\n";
  ok = ok && std::fwrite(tail, 1, std::strlen(tail), f) == std::strlen(tail);
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) *err = std::string("write to ") + path + " failed";
  return ok;
}

// the nodal volumes on the host (constant; copied once)
int host_volumes(pdgpu_ctx *ctx) {
  if ((int64_t)ctx->vol_host.size() == ctx->d.n_nodes) return PDGPU_OK;
  ctx->vol_host.resize((size_t)ctx->d.n_nodes);
  CK(cudaMemcpy(ctx->vol_host.data(), ctx->d.vol, (size_t)ctx->d.n_nodes * 8, cudaMemcpyDeviceToHost));
  return PDGPU_OK;
}

std::string xml_attr(const std::string &tag, const char *key) {
  const std::string k = std::string(key) + "=\"";
  const size_t p = tag.find(k);
  if (p == std::string::npos) return "";
  const size_t q = tag.find('"', p + k.size());
  return q == std::string::npos ? "" : tag.substr(p + k.size(), q - p - k.size());
}

}  // namespace

extern "C" {

int pdgpu_write_vtu(pdgpu_ctx *ctx, const char *path, const char *tags) {
  if (!ctx || !path) return PDGPU_ERR_ARG;
  if (!ctx->nodes || !ctx->particles) return fail(ctx, PDGPU_ERR_STATE, "write_vtu: no nodes");
  const std::string T = tags ? tags : "";
  const int64_t N = ctx->d.n_nodes;
  VtuFrame fr;
  fr.n = N;
  fr.x.resize(3 * N);
  TRY(pdgpu_download(ctx, PDGPU_FIELD_X, fr.x.data()));
  if (has_tag(T, "Displacement")) {
    fr.u.resize(3 * N);
    TRY(pdgpu_download(ctx, PDGPU_FIELD_U, fr.u.data()));
  }
  if (has_tag(T, "Velocity")) {
    fr.v.resize(3 * N);
    TRY(pdgpu_download(ctx, PDGPU_FIELD_V, fr.v.data()));
  }
  if (has_tag(T, "Force_Density") || has_tag(T, "Force")) {
    fr.f.resize(3 * N);
    TRY(pdgpu_download(ctx, PDGPU_FIELD_F, fr.f.data()));
  }
  if (has_tag(T, "Damage_Z")) {
    fr.Z.resize(N);
    TRY(pdgpu_download(ctx, PDGPU_FIELD_Z, fr.Z.data()));
  }
  if (has_tag(T, "Theta") && ctx->d.theta) {
    fr.theta.resize(N);
    TRY(pdgpu_download(ctx, PDGPU_FIELD_THETA, fr.theta.data()));
  }
  TRY(host_volumes(ctx));
  pdgpu_scalars sc{};
  TRY(pdgpu_get_scalars(ctx, &sc));
  fr.time = sc.time;
  std::string err;
  if (!write_frame(ctx, fr, T, path, &err)) return fail(ctx, PDGPU_ERR_ARG, "write_vtu: %s", err.c_str());
  return PDGPU_OK;
}

int pdgpu_write_vtu_async(pdgpu_ctx *ctx, const char *path, const char *tags) {
  if (!ctx || !path) return PDGPU_ERR_ARG;
  if (!ctx->nodes || !ctx->particles) return fail(ctx, PDGPU_ERR_STATE, "write_vtu_async: no nodes");
  // one file in flight: the previous one is finished first
  TRY(pdgpu_output_wait(ctx));
  TRY(host_volumes(ctx));
  DevData &d = ctx->d;
  const int64_t N = d.n_nodes;
  const int64_t st = d.dim == 2 ? 2 : 4;
  // staging layout in doubles: x, u, v, f (device node-vector layout),
  // theta, Z (floats, packed), time
  const size_t o_th = (size_t)(4 * st * N), o_z = o_th + (size_t)N, o_t = o_z + (size_t)(N + 1) / 2;
  const size_t need = o_t + 1;
  if (ctx->out_doubles < need) {
    if (ctx->out_dev) dfree(ctx, ctx->out_dev);
    if (ctx->out_host) cudaFreeHost(ctx->out_host);
    ctx->out_host = nullptr;
    ctx->out_doubles = 0;
    TRY(dalloc(ctx, &ctx->out_dev, need));
    CK(cudaMallocHost((void **)&ctx->out_host, need * 8));
    ctx->out_doubles = need;
  }
  if (!ctx->out_stream) CK(cudaStreamCreateWithFlags(&ctx->out_stream, cudaStreamNonBlocking));
  if (!ctx->ev_out0) CK(cudaEventCreateWithFlags(&ctx->ev_out0, cudaEventDisableTiming));
  if (!ctx->ev_out1) CK(cudaEventCreateWithFlags(&ctx->ev_out1, cudaEventDisableTiming));
  // the state as of now, in stream order on the context stream (a device
  // copy: the steps issued next do not wait for the download or the file)
  cudaStream_t s = ctx->stream;
  const size_t vb = (size_t)(st * N) * 8;
  double *o = ctx->out_dev;
  CK(cudaMemcpyAsync(o, d.x, vb, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(o + st * N, d.u, vb, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(o + 2 * st * N, d.v, vb, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(o + 3 * st * N, d.f, vb, cudaMemcpyDeviceToDevice, s));
  if (d.theta) CK(cudaMemcpyAsync(o + o_th, d.theta, (size_t)N * 8, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(o + o_z, d.Z, (size_t)N * 4, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(o + o_t, reinterpret_cast<const char *>(d.ctrl) + offsetof(CtrlState, time), 8,
                     cudaMemcpyDeviceToDevice, s));
  CK(cudaEventRecord(ctx->ev_out0, s));
  CK(cudaStreamWaitEvent(ctx->out_stream, ctx->ev_out0, 0));
  CK(cudaMemcpyAsync(ctx->out_host, o, need * 8, cudaMemcpyDeviceToHost, ctx->out_stream));
  CK(cudaEventRecord(ctx->ev_out1, ctx->out_stream));
  ctx->out_rc = PDGPU_OK;
  ctx->out_err.clear();
  const std::string P = path, T = tags ? tags : "";
  const int dim = d.dim, dev = ctx->desc.device;
  const bool has_theta = d.theta != nullptr;
  ctx->out_thread = std::thread([ctx, P, T, N, st, dim, dev, has_theta, o_th, o_z, o_t]() {
    cudaSetDevice(dev);
    const cudaError_t e = cudaEventSynchronize(ctx->ev_out1);
    if (e != cudaSuccess) {
      ctx->out_rc = PDGPU_ERR_CUDA;
      ctx->out_err = std::string("write_vtu_async: download failed: ") + cudaGetErrorString(e);
      return;
    }
    const double *h = ctx->out_host;
    VtuFrame fr;
    fr.n = N;
    fr.time = h[o_t];
    auto aos = [&](int k, std::vector<double> *out) {
      out->assign((size_t)(3 * N), 0.0);
      const double *src = h + k * st * N;
      for (int64_t i = 0; i < N; i++)
        for (int q = 0; q < dim; q++) (*out)[3 * i + q] = src[st * i + q];
    };
    aos(0, &fr.x);
    if (has_tag(T, "Displacement")) aos(1, &fr.u);
    if (has_tag(T, "Velocity")) aos(2, &fr.v);
    if (has_tag(T, "Force_Density") || has_tag(T, "Force")) aos(3, &fr.f);
    if (has_tag(T, "Theta") && has_theta) fr.theta.assign(h + o_th, h + o_th + N);
    if (has_tag(T, "Damage_Z")) {
      const float *z = reinterpret_cast<const float *>(h + o_z);
      fr.Z.assign(z, z + N);
    }
    std::string err;
    if (!write_frame(ctx, fr, T, P.c_str(), &err)) {
      ctx->out_rc = PDGPU_ERR_ARG;
      ctx->out_err = "write_vtu_async: " + err;
    }
  });
  return PDGPU_OK;
}

int pdgpu_output_wait(pdgpu_ctx *ctx) {
  if (!ctx) return PDGPU_ERR_ARG;
  if (ctx->out_thread.joinable()) ctx->out_thread.join();
  if (ctx->out_rc != PDGPU_OK) {
    const int rc = ctx->out_rc;
    ctx->out_rc = PDGPU_OK;
    return fail(ctx, rc, "%s", ctx->out_err.c_str());
  }
  return PDGPU_OK;
}

int pdgpu_restart(pdgpu_ctx *ctx, const char *path, int64_t step) {
  if (!ctx || !path || step < 0) return PDGPU_ERR_ARG;
  if (ctx->begun) return fail(ctx, PDGPU_ERR_STATE, "restart before pdgpu_integrate_begin");
  if (!ctx->nodes) return fail(ctx, PDGPU_ERR_STATE, "restart: upload nodes first");
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(ctx, PDGPU_ERR_ARG, "restart: cannot open %s", path);
  std::string buf;
  {
    std::vector<char> chunk(1 << 20);
    size_t n;
    while ((n = std::fread(chunk.data(), 1, chunk.size(), f)) > 0) buf.append(chunk.data(), n);
    std::fclose(f);
  }
  const size_t app = buf.find("<AppendedData encoding=\"raw\">");
  const size_t base = app == std::string::npos ? std::string::npos : buf.find('_', app);
  if (base == std::string::npos)
    return fail(ctx, PDGPU_ERR_ARG, "restart: %s has no raw appended data (files of pdgpu_write_vtu)", path);
  const int64_t N = ctx->d.n_nodes;
  const std::string np = xml_attr(buf.substr(0, app), "NumberOfPoints");
  if (np.empty() || std::stoll(np) != N)
    return fail(ctx, PDGPU_ERR_ARG, "restart: %s has %s points, the model %lld", path, np.c_str(), (long long)N);
  // DataArray name -> its block of N x 3 doubles
  auto block = [&](const char *name, std::vector<double> *out) -> bool {
    const std::string key = std::string("Name=\"") + name + "\"";
    size_t p = buf.find(key);
    if (p == std::string::npos || p > app) return false;
    const size_t b = buf.rfind('<', p), e = buf.find('>', p);
    const std::string tag = buf.substr(b, e - b);
    if (xml_attr(tag, "type") != "Float64" || xml_attr(tag, "NumberOfComponents") != "3") return false;
    const uint64_t off = std::stoull(xml_attr(tag, "offset"));
    const size_t at = base + 1 + off;
    uint64_t nb = 0;
    if (at + 8 > buf.size()) return false;
    std::memcpy(&nb, buf.data() + at, 8);
    if (nb != (uint64_t)N * 24 || at + 8 + nb > buf.size()) return false;
    out->resize(3 * N);
    std::memcpy(out->data(), buf.data() + at + 8, nb);
    return true;
  };
  // VtkParticleReader::readNodes (vtkParticleReader.cpp:41-120): current
  // positions, displacement (else x - x_ref) and velocity (required)
  std::vector<double> x, u, v;
  if (!block("Points", &x)) return fail(ctx, PDGPU_ERR_ARG, "restart: no Float64 points in %s", path);
  if (!block("Velocity", &v)) return fail(ctx, PDGPU_ERR_ARG, "restart: no Velocity array in %s", path);
  if (!block("Displacement", &u)) {
    u.resize(3 * N);
    for (int64_t k = 0; k < 3 * N; k++) u[k] = x[k] - ctx->xref[k];
  }
  TRY(pdgpu_upload_field(ctx, PDGPU_FIELD_X, x.data()));
  TRY(pdgpu_upload_field(ctx, PDGPU_FIELD_U, u.data()));
  TRY(pdgpu_upload_field(ctx, PDGPU_FIELD_V, v.data()));
  ctx->d.restart_step = step;
  if (ctx->gexec) {
    cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
  }
  return PDGPU_OK;
}

int pdgpu_set_surrogate(pdgpu_ctx *ctx, int32_t n_shapes, const pdgpu_sur_shape *shapes, const double *fscale,
                        const double *floor, const double *orient, const double *scale, int32_t check_interval,
                        double z_gate, double err_gate, int32_t near_gate) {
  if (!ctx || n_shapes <= 0 || !shapes || !fscale || !floor || !orient || !scale || check_interval <= 0)
    return PDGPU_ERR_ARG;
  if (ctx->desc.precision != PDGPU_PREC_MIXED || ctx->desc.dim != 2)
    return fail(ctx, PDGPU_ERR_ARG, "the learned surrogate needs the mixed-precision form in 2-D");
  if (ctx->begun || !ctx->sur.empty())
    return fail(ctx, PDGPU_ERR_STATE, "set the surrogate once, before integrate_begin");
  if (!ctx->particles) return fail(ctx, PDGPU_ERR_STATE, "upload particles first");
  DevData &d = ctx->d;
  // FP32 rows x cols -> BF16 rows_out x ld_out on the device (zero padded)
  auto bf = [&](const float *src, size_t rows, size_t cols, size_t ld_out, size_t rows_out, void **dst) -> int {
    std::vector<__nv_bfloat16> h(rows_out * ld_out, __float2bfloat16(0.f));
    for (size_t r = 0; r < rows; r++)
      for (size_t c = 0; c < cols; c++) h[r * ld_out + c] = __float2bfloat16(src[r * cols + c]);
    __nv_bfloat16 *p;
    TRY(dalloc(ctx, &p, h.size()));
    CK(cudaMemcpy(p, h.data(), h.size() * 2, cudaMemcpyHostToDevice));
    *dst = p;
    return PDGPU_OK;
  };
  auto f32 = [&](const float *src, size_t n, float **dst) -> int {
    TRY(dalloc(ctx, dst, n));
    CK(cudaMemcpy(*dst, src, n * 4, cudaMemcpyHostToDevice));
    return PDGPU_OK;
  };
  std::vector<GemmProblem> probs(5 * (size_t)n_shapes);
  for (int k = 0; k < n_shapes; k++) {
    const pdgpu_sur_shape &in = shapes[k];
    if (in.n_nodes <= 0 || !in.phi_t || !in.psi || !in.w1 || !in.b1 || !in.w2 || !in.b2 || !in.w3 || !in.b3)
      return fail(ctx, PDGPU_ERR_ARG, "surrogate shape %d incomplete", k);
    pdgpu_ctx::SurShape S;
    S.n_nodes = in.n_nodes;
    const int K = 2 * in.n_nodes;
    S.kpad = (K + 15) / 16 * 16;
    std::vector<SurPart> parts;
    for (size_t p = 0; p < ctx->hp.size(); p++) {
      const DevParticle &P = ctx->hp[p];
      if (P.zone != in.zone || P.type != 0 || !P.compute_force) continue;
      if (P.end - P.start != in.n_nodes)
        return fail(ctx, PDGPU_ERR_ARG, "particle %zu of zone %d has %lld nodes, the surrogate %d", p, in.zone,
                    (long long)(P.end - P.start), in.n_nodes);
      SurPart q{};
      q.start = P.start;
      q.center = P.center;
      q.particle = (int32_t)p;
      q.c = std::cos(orient[p]);
      q.s = std::sin(orient[p]);
      q.inv_scale = 1.0 / scale[p];
      q.fscale = fscale[p];
      q.floor2 = floor[p] * floor[p];
      parts.push_back(q);
    }
    S.P = (int)parts.size();
    if (S.P == 0) return fail(ctx, PDGPU_ERR_ARG, "no force-computing particle in surrogate zone %d", in.zone);
    TRY(dalloc(ctx, &S.parts, parts.size()));
    CK(cudaMemcpy(S.parts, parts.data(), parts.size() * sizeof(SurPart), cudaMemcpyHostToDevice));
    TRY(bf(in.phi_t, 32, K, S.kpad, 32, &S.phiT));
    TRY(bf(in.psi, K, 64, 64, S.kpad, &S.lift));
    TRY(bf(in.w1, 256, 32, 32, 256, &S.w1));
    TRY(bf(in.w2, 256, 256, 256, 256, &S.w2));
    TRY(bf(in.w3, 32, 256, 256, 32, &S.w3));
    TRY(f32(in.b1, 256, &S.b1));
    TRY(f32(in.b2, 256, &S.b2));
    TRY(f32(in.b3, 32, &S.b3));
    // CUDA-core chain: warp-MMA operands with K permuted in chunks of 64
    // inputs (sur_kperm)
    auto kperm = [&](const float *src, int rows, int rows_pad, int K, void **dst) -> int {
      std::vector<float> h((size_t)rows_pad * K, 0.f);
      const int cw = std::min(K, 64) / 2, ks = cw / 8;  // pairs and k-steps per chunk
      for (int r = 0; r < rows; r++)
        for (int c = 0; c < K; c++) {
          const int chunk = c / (2 * cw), pw = (c % (2 * cw)) / 2;
          h[(size_t)r * K + chunk * 2 * cw + 2 * sur_kperm(pw, ks) + c % 2] = src[(size_t)r * K + c];
        }
      return bf(h.data(), 1, h.size(), h.size(), 1, dst);
    };
    TRY(kperm(in.w1, 256, 256, 32, &S.w1m));
    TRY(kperm(in.w2, 256, 256, 256, &S.w2m));
    TRY(kperm(in.w3, 32, 32, 256, &S.w3m));
    TRY(kperm(in.psi, K, S.kpad, 64, &S.liftm));
    {
      // phi^T rows padded with zeros to whole 128-node chunks of the projection
      const int kc = sur_n_chunks(in.n_nodes) * 256;
      std::vector<float> h((size_t)32 * kc, 0.f);
      for (int j = 0; j < 32; j++)
        for (int c = 0; c < K; c++) h[(size_t)j * kc + c] = in.phi_t[(size_t)j * K + c];
      TRY(kperm(h.data(), 32, 32, kc, &S.phim));
    }
    const int M = S.P + 1;  // row P: the zero input
    __nv_bfloat16 *A, *xy, *h1, *h2;
    TRY(dalloc(ctx, &A, (size_t)M * S.kpad));
    CK(cudaMemset(A, 0, (size_t)M * S.kpad * 2));
    TRY(dalloc(ctx, &xy, (size_t)M * 64));  // [network output | projected input]
    TRY(dalloc(ctx, &h1, (size_t)M * 256));
    TRY(dalloc(ctx, &h2, (size_t)M * 256));
    TRY(dalloc(ctx, &S.F, (size_t)M * S.kpad));
    TRY(dalloc(ctx, &S.xpart, (size_t)M * sur_n_chunks(S.n_nodes) * 32));
    S.A = A, S.xy = xy, S.h1 = h1, S.h2 = h2;
    // x = A phi^T -> xy[:, 32:64]; h1 = tanh(x W1^T + b1); h2 = tanh(h1 W2^T + b2);
    // y = h2 W3^T + b3 -> xy[:, 0:32]; F = xy lift^T
    probs[0 * n_shapes + k] = GemmProblem{A, S.phiT, nullptr, nullptr, xy + 32, S.kpad, S.kpad, 64, M, 32, S.kpad, 0, 0};
    probs[1 * n_shapes + k] = GemmProblem{xy + 32, S.w1, S.b1, nullptr, h1, 64, 32, 256, M, 256, 32, 1, 0};
    probs[2 * n_shapes + k] = GemmProblem{h1, S.w2, S.b2, nullptr, h2, 256, 256, 256, M, 256, 256, 1, 0};
    probs[3 * n_shapes + k] = GemmProblem{h2, S.w3, S.b3, nullptr, xy, 256, 256, 64, M, 32, 256, 0, 0};
    probs[4 * n_shapes + k] = GemmProblem{xy, S.lift, nullptr, S.F, nullptr, 64, 64, S.kpad, M, S.kpad, 64, 0, 0};
    ctx->sur_max_p = std::max(ctx->sur_max_p, M);
    ctx->sur_max_k = std::max(ctx->sur_max_k, S.kpad);
    ctx->sur.push_back(S);
  }
  TRY(dalloc(ctx, &ctx->sur_probs, probs.size()));
  CK(cudaMemcpy(ctx->sur_probs, probs.data(), probs.size() * sizeof(GemmProblem), cudaMemcpyHostToDevice));
  ctx->sur_fused = ctx->sur_chain == 0 && n_shapes <= kMaxSurShapes;
  std::vector<SurShapeDev> sd;
  for (auto &S : ctx->sur) {
    sd.push_back(SurShapeDev{S.parts, S.P, S.n_nodes, S.kpad, 0, ctx->sur_chain == 0 ? S.phim : S.phiT, S.xy, S.F, S.xpart,
                             sur_n_chunks(S.n_nodes), 0, S.w1m, S.w2m, S.w3m, S.b1, S.b2, S.b3, S.liftm});
    ctx->sur_max_rows = std::max(ctx->sur_max_rows, S.P);
    ctx->sur_max_nodes = std::max(ctx->sur_max_nodes, S.n_nodes);
  }
  if (ctx->sur_fused) {
    ctx->sur_shapes.n = (int32_t)sd.size();
    for (size_t k = 0; k < sd.size(); k++) ctx->sur_shapes.s[k] = sd[k];
  }
  TRY(dalloc(ctx, &ctx->sur_dev, sd.size()));
  CK(cudaMemcpy(ctx->sur_dev, sd.data(), sd.size() * sizeof(SurShapeDev), cudaMemcpyHostToDevice));
  TRY(dalloc(ctx, &ctx->sur_err2, 2 * ctx->hp.size()));
  CK(cudaMemset(ctx->sur_err2, 0, 2 * ctx->hp.size() * 8));
  TRY(dalloc(ctx, &ctx->sur_errflag, 1));
  CK(cudaMemset(ctx->sur_errflag, 0, 4));
  TRY(dalloc(ctx, &ctx->sur_count, 2));
  CK(cudaMemset(ctx->sur_count, 0, 16));
  TRY(dalloc(ctx, &d.sur_on, ctx->hp.size()));
  CK(cudaMemset(d.sur_on, 0, ctx->hp.size()));  // on only after a check step passes the gate
  TRY(dalloc(ctx, &d.sur_near, ctx->hp.size()));
  // with the proximity gate: near until the first contact-list rebuild
  CK(cudaMemset(d.sur_near, near_gate ? 1 : 0, ctx->hp.size()));
  d.sur_near_gate = near_gate ? 1 : 0;
  d.sur_interval = check_interval;
  ctx->sur_z_gate = (float)z_gate;
  ctx->sur_err_gate = err_gate;
  CK(cudaStreamCreateWithFlags(&ctx->sur_stream, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&ctx->ev_sur0, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&ctx->ev_sur1, cudaEventDisableTiming));
  if (ctx->gexec) {
    cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
  }
  return setup_tile_list(ctx);  // when the bond tiles exist already
}

int pdgpu_surrogate_stats(pdgpu_ctx *ctx, int64_t *n_on, int64_t *n_total, int64_t *steps_on,
                          int64_t *steps_total) {
  if (!ctx || !n_on || !n_total || !steps_on || !steps_total) return PDGPU_ERR_ARG;
  *n_on = *n_total = *steps_on = *steps_total = 0;
  if (ctx->sur.empty()) return PDGPU_OK;
  const size_t np = ctx->hp.size();
  std::vector<uint8_t> on(np), near(np);
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(on.data(), ctx->d.sur_on, np, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(near.data(), ctx->d.sur_near, np, cudaMemcpyDeviceToHost));
  for (size_t p = 0; p < np; p++) *n_on += on[p] && !near[p];
  for (auto &S : ctx->sur) *n_total += S.P;
  unsigned long long cnt[2];
  CK(cudaMemcpy(cnt, ctx->sur_count, 16, cudaMemcpyDeviceToHost));
  *steps_on = (int64_t)cnt[0];
  *steps_total = (int64_t)cnt[1];
  int32_t flag = 0;
  CK(cudaMemcpy(&flag, ctx->sur_errflag, 4, cudaMemcpyDeviceToHost));
  if (flag) return fail(ctx, PDGPU_ERR_CUDA, "a tensor-core wait of the surrogate timed out");
  return PDGPU_OK;
}

int pdgpu_set_scenes(pdgpu_ctx *ctx, int32_t n_scenes, const int64_t *particle_offsets, const int64_t *test_walls) {
  if (!ctx || n_scenes <= 0 || !particle_offsets || !test_walls) return PDGPU_ERR_ARG;
  if (ctx->prepared || ctx->begun) return fail(ctx, PDGPU_ERR_STATE, "set the scenes before the first step");
  if (!ctx->particles) return fail(ctx, PDGPU_ERR_STATE, "upload particles first");
  const int64_t np = (int64_t)ctx->hp.size();
  if (particle_offsets[0] != 0 || particle_offsets[n_scenes] != np)
    return fail(ctx, PDGPU_ERR_ARG, "scene offsets must run from 0 to the number of particles");
  for (int s = 0; s < n_scenes; s++) {
    if (particle_offsets[s + 1] <= particle_offsets[s]) return fail(ctx, PDGPU_ERR_ARG, "scene %d is empty", s);
    const int64_t w = test_walls[s];
    if (w >= 0 && (w < particle_offsets[s] || w >= particle_offsets[s + 1]))
      return fail(ctx, PDGPU_ERR_ARG, "test wall of scene %d lies outside it", s);
  }
  ctx->scene_poff.assign(particle_offsets, particle_offsets + n_scenes + 1);
  ctx->scene_walls.assign(test_walls, test_walls + n_scenes);
  return PDGPU_OK;
}

int pdgpu_get_scene_history(pdgpu_ctx *ctx, int32_t scene, double *t, double *delta, double *force,
                            double *cforce, int64_t cap, int64_t *count) {
  if (!ctx || !count) return PDGPU_ERR_ARG;
  const DevData &d = ctx->d;
  if (d.n_scenes <= 1 || scene < 0 || scene >= d.n_scenes) return fail(ctx, PDGPU_ERR_ARG, "no scene %d", scene);
  CK(cudaStreamSynchronize(ctx->stream));
  CtrlState c;
  CK(cudaMemcpy(&c, d.ctrl, sizeof(c), cudaMemcpyDeviceToHost));
  const int64_t recorded = c.n >= d.test_interval ? c.n / d.test_interval : 0;
  *count = std::min<int64_t>(recorded, d.scene_hist_cap);
  const int64_t n = std::min<int64_t>(cap, *count);
  if (n <= 0 || !t || !delta || !force || !cforce) return PDGPU_OK;
  std::vector<double> h((size_t)n * 4);
  CK(cudaMemcpy(h.data(), d.scene_hist + 4 * (int64_t)scene * d.scene_hist_cap, h.size() * 8,
                cudaMemcpyDeviceToHost));
  for (int64_t k = 0; k < n; k++) {
    t[k] = h[4 * k];
    delta[k] = h[4 * k + 1];
    force[k] = h[4 * k + 2];
    cforce[k] = h[4 * k + 3];
  }
  return PDGPU_OK;
}

int pdgpu_surrogate_errors(pdgpu_ctx *ctx, double *err2, int64_t n) {
  if (!ctx || !err2 || n != 2 * (int64_t)ctx->hp.size()) return PDGPU_ERR_ARG;
  if (ctx->sur.empty()) return fail(ctx, PDGPU_ERR_STATE, "no surrogate set");
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(err2, ctx->sur_err2, (size_t)n * 8, cudaMemcpyDeviceToHost));
  return PDGPU_OK;
}

int pdgpu_compute_pd_forces(pdgpu_ctx *ctx) {
  if (!ctx) return PDGPU_ERR_ARG;
  TRY(prepare(ctx));
  pd_forces(ctx);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return device_error(ctx);
}

int pdgpu_upload_field(pdgpu_ctx *ctx, int32_t field, const void *src) {
  if (!ctx || !src) return PDGPU_ERR_ARG;
  DevData &d = ctx->d;
  if (field == PDGPU_FIELD_BONDS) {
    if (!ctx->bonds) return fail(ctx, PDGPU_ERR_STATE, "upload the neighbour lists first");
    const uint8_t *b = static_cast<const uint8_t *>(src);
    std::vector<uint32_t> bits((d.n_bonds + 31) / 32 + kBitPad, 0u);
    for (int64_t k = 0; k < d.n_bonds; k++)
      if (b[k]) bits[k >> 5] |= 1u << (k & 31);
    CK(cudaMemcpyAsync(d.bond_bits, bits.data(), bits.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return sym_bits(ctx);
  }
  double *vec = field == PDGPU_FIELD_X ? d.x : field == PDGPU_FIELD_U ? d.u : field == PDGPU_FIELD_V ? d.v : nullptr;
  if (!vec) return fail(ctx, PDGPU_ERR_ARG, "upload_field: only x, u, v and bonds can be written");
  CK(cudaMemcpyAsync(ctx->stage, src, (size_t)3 * d.n_nodes * 8, cudaMemcpyHostToDevice, ctx->stream));
  launch_pack_vec(d, ctx->stage, vec, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return PDGPU_OK;
}

int pdgpu_get_scalars(pdgpu_ctx *ctx, pdgpu_scalars *out) {
  if (!ctx || !out) return PDGPU_ERR_ARG;
  CtrlState c;
  TRY(read_ctrl(ctx, &c));
  std::memset(out, 0, sizeof *out);
  out->n = c.n;
  out->time = c.time;
  out->reaction = c.reaction;
  out->contact_reaction = c.contact_reaction;
  out->wall_penetration = c.penetration;
  out->max_velocity = c.max_velocity;
  out->contact_search_radius = c.radius;
  out->contact_update_interval = c.interval;
  out->contact_counter = c.counter;
  out->contact_updates = c.updates;
  out->contact_entries = c.entries;
  out->pen_dist = c.pen_dist;
  out->max_y = c.max_y;
  out->contact_area_radius = c.contact_area_radius;
  if (ctx->bonds && ctx->d.n_bonds) {
    std::vector<uint32_t> bits((ctx->d.n_bonds + 31) / 32 + 1);
    CK(cudaMemcpy(bits.data(), ctx->d.bond_bits, bits.size() * 4, cudaMemcpyDeviceToHost));
    int64_t nb = 0;
    for (auto w : bits) nb += __builtin_popcount(w);
    out->broken_bonds = nb;
  }
  return c.error ? device_error(ctx) : PDGPU_OK;
}

int pdgpu_step_host(pdgpu_ctx *ctx, double *u, double *v, double *x, double *f, int64_t nsteps,
                    pdgpu_scalars *out) {
  if (!ctx || !u || !v || !x || !f) return PDGPU_ERR_ARG;
  if (!ctx->begun) return fail(ctx, PDGPU_ERR_STATE, "call pdgpu_integrate_begin first");
  DevData &d = ctx->d;
  cudaStream_t s = ctx->stream;
  const size_t bytes = (size_t)3 * d.n_nodes * 8;
  double *vecs[3] = {d.u, d.v, d.x};
  double *hosts[3] = {u, v, x};
  for (int k = 0; k < 3; k++) {
    CK(cudaMemcpyAsync(ctx->stage, hosts[k], bytes, cudaMemcpyHostToDevice, s));
    launch_pack_vec(d, ctx->stage, vecs[k], s);
  }
  // replay of the step graph (one step per replay unless a longer graph exists)
  TRY(pdgpu_step_graph(ctx, nsteps, ctx->gexec ? ctx->graph_steps : 1));
  double *outs[4] = {d.u, d.v, d.x, d.f};
  double *hout[4] = {u, v, x, f};
  for (int k = 0; k < 4; k++) {
    launch_unpack_vec(d, outs[k], ctx->stage, s);
    CK(cudaMemcpyAsync(hout[k], ctx->stage, bytes, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  if (out) return pdgpu_get_scalars(ctx, out);
  return device_error(ctx);
}

int pdgpu_get_history(pdgpu_ctx *ctx, double *t, double *delta, double *force, double *cforce,
                      int64_t cap, int64_t *count) {
  if (!ctx || !count) return PDGPU_ERR_ARG;
  CtrlState c;
  TRY(read_ctrl(ctx, &c));
  *count = c.history_count;
  const int64_t n = std::min<int64_t>({cap, c.history_count, ctx->d.history_cap});
  if (n <= 0 || !ctx->d.history) return PDGPU_OK;
  std::vector<double> h(4 * n);
  CK(cudaMemcpy(h.data(), ctx->d.history, h.size() * 8, cudaMemcpyDeviceToHost));
  for (int64_t k = 0; k < n; k++) {
    if (t) t[k] = h[4 * k];
    if (delta) delta[k] = h[4 * k + 1];
    if (force) force[k] = h[4 * k + 2];
    if (cforce) cforce[k] = h[4 * k + 3];
  }
  return PDGPU_OK;
}

int pdgpu_download_contact(pdgpu_ctx *ctx, uint64_t *rowptr, uint64_t *col) {
  if (!ctx || !rowptr) return PDGPU_ERR_ARG;
  DevData &d = ctx->d;
  if (!d.c_row) return fail(ctx, PDGPU_ERR_STATE, "no contact lists");
  std::vector<int64_t> row(d.n_nodes + 1);
  CK(cudaMemcpy(row.data(), d.c_row, row.size() * 8, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < row.size(); i++) rowptr[i] = (uint64_t)row[i];
  const int64_t E = row.back();
  if (col && E > 0) {
    std::vector<int32_t> c(E);
    CK(cudaMemcpy(c.data(), d.c_col, E * 4, cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < E; k++) col[k] = (uint64_t)c[k];
  }
  return PDGPU_OK;
}

int pdgpu_num_bonds(pdgpu_ctx *ctx, int64_t *n) {
  if (!ctx || !n) return PDGPU_ERR_ARG;
  *n = ctx->d.n_bonds;
  return PDGPU_OK;
}

int pdgpu_download_pd_neighbors(pdgpu_ctx *ctx, uint64_t *rowptr, uint64_t *col) {
  if (!ctx || !rowptr || !col) return PDGPU_ERR_ARG;
  DevData &d = ctx->d;
  if (!ctx->bonds) return fail(ctx, PDGPU_ERR_STATE, "no bonds");
  std::vector<int64_t> row(d.n_nodes + 1);
  std::vector<int32_t> c(d.n_bonds);
  CK(cudaMemcpy(row.data(), d.pd_row, row.size() * 8, cudaMemcpyDeviceToHost));
  if (d.n_bonds) CK(cudaMemcpy(c.data(), d.pd_col, c.size() * 4, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < row.size(); i++) rowptr[i] = (uint64_t)row[i];
  for (size_t k = 0; k < c.size(); k++) col[k] = (uint64_t)c[k];
  return PDGPU_OK;
}

int pdgpu_set_tuning(pdgpu_ctx *ctx, int32_t pd_lanes, int32_t contact_lanes) {
  if (!ctx) return PDGPU_ERR_ARG;
  if (ctx->prepared && contact_lanes) return fail(ctx, PDGPU_ERR_STATE, "set_tuning: contact lanes are fixed once stepping starts");
  const bool mixed = ctx->desc.precision == PDGPU_PREC_MIXED;
  if (pd_lanes && !((mixed && (pd_lanes == 1 || pd_lanes == 2)) || pd_lanes == 4 || pd_lanes == 8 ||
                    pd_lanes == 16 || pd_lanes == 32))
    return fail(ctx, PDGPU_ERR_ARG, "set_tuning: pd_lanes must be 4, 8, 16 or 32 (also 1 or 2 in the mixed form)");
  if (ctx->prepared && pd_lanes) return fail(ctx, PDGPU_ERR_STATE, "set_tuning: lanes are fixed once stepping starts");
  if (contact_lanes && contact_lanes != 1 && contact_lanes != 2 && contact_lanes != 4 && contact_lanes != 8 &&
      contact_lanes != 32)
    return fail(ctx, PDGPU_ERR_ARG, "set_tuning: contact_lanes must be 1, 2, 4, 8 or 32");
  if (pd_lanes) ctx->pd_lanes = pd_lanes;
  if (contact_lanes) ctx->contact_lanes = contact_lanes;
  if (ctx->gexec) {
    cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
  }
  return PDGPU_OK;
}

int pdgpu_set_tile_nodes(pdgpu_ctx *ctx, int32_t nodes) {
  if (!ctx || nodes < 0 || nodes > 4096) return PDGPU_ERR_ARG;
  if (ctx->prepared) return fail(ctx, PDGPU_ERR_STATE, "set_tile_nodes: tiles are fixed once stepping starts");
  ctx->tile_nodes = nodes;
  return PDGPU_OK;
}

int pdgpu_set_contact_grid(pdgpu_ctx *ctx, int32_t ctas_per_sm) {
  if (!ctx || ctas_per_sm < 1 || ctas_per_sm > 16) return PDGPU_ERR_ARG;
  if (ctx->prepared) return fail(ctx, PDGPU_ERR_STATE, "set_contact_grid: set it before the first step");
  ctx->contact_ctas = ctas_per_sm;
  return PDGPU_OK;
}

int pdgpu_set_surrogate_chain(pdgpu_ctx *ctx, int32_t kind) {
  if (!ctx || kind < 0 || kind > 1) return PDGPU_ERR_ARG;
  if (!ctx->sur.empty()) return fail(ctx, PDGPU_ERR_STATE, "set_surrogate_chain: set it before set_surrogate");
  ctx->sur_chain = kind;
  return PDGPU_OK;
}

int pdgpu_set_bond_scheme(pdgpu_ctx *ctx, int32_t scheme) {
  if (!ctx || scheme < 0 || scheme > 2) return PDGPU_ERR_ARG;
  if (ctx->prepared) return fail(ctx, PDGPU_ERR_STATE, "set_bond_scheme: set it before the first step");
  ctx->bond_scheme = scheme;
  return PDGPU_OK;
}

int pdgpu_bond_scheme(pdgpu_ctx *ctx, int32_t *scheme) {
  if (!ctx || !scheme) return PDGPU_ERR_ARG;
  TRY(prepare(ctx));
  *scheme = ctx->d.use_sym ? 1 : (ctx->d.node_order ? 2 : 0);
  return PDGPU_OK;
}

int pdgpu_get_stream(pdgpu_ctx *ctx, void **stream) {
  if (!ctx || !stream) return PDGPU_ERR_ARG;
  *stream = (void *)ctx->stream;
  return PDGPU_OK;
}

int pdgpu_enable_timing(pdgpu_ctx *ctx, int32_t on) {
  if (!ctx) return PDGPU_ERR_ARG;
  resolve_timing(ctx);
  ctx->timing = on != 0;
  for (int i = 0; i < kMaxTimed; i++) {
    ctx->ms[i] = 0.0;
    ctx->launches[i] = 0;
  }
  return PDGPU_OK;
}

}  // extern "C"

namespace {

// host side of the strain/stress output: checks, device copies of the
// element data, the kernel, the three entries per element back to the host
int strain_stress(pdgpu_ctx *ctx, const char *who, int nv, int64_t n_elements, const int64_t *conn, int32_t nq,
                  const double *ref_points, const double *nu, const double *lambda, const double *mu,
                  const uint8_t *plane_strain, double *xq, double *strain, double *stress) {
  if (!ctx || n_elements < 0 || (n_elements > 0 && (!conn || (nv == 3 && (!ref_points || !plane_strain)) || !nu ||
                                                    !lambda || !mu || !xq || !strain || !stress)))
    return PDGPU_ERR_ARG;
  if (!ctx->nodes) return fail(ctx, PDGPU_ERR_STATE, "%s: upload nodes first", who);
  DevData &d = ctx->d;
  if (d.dim != (nv == 3 ? 2 : 3))
    return fail(ctx, PDGPU_ERR_ARG, "%s: %s need a %d-D context", who, nv == 3 ? "triangles" : "tetrahedra",
                nv == 3 ? 2 : 3);
  if (nv == 3 && (nq < 1 || nq > 3))
    return fail(ctx, PDGPU_ERR_ARG, "%s: %d quadrature points (the reference keeps three entries per triangle; "
                "rules of 1 or 3 points)", who, nq);
  for (int64_t k = 0; k < (int64_t)nv * n_elements; k++)
    if (conn[k] < 0 || conn[k] >= d.n_nodes)
      return fail(ctx, PDGPU_ERR_ARG, "%s: element %lld names node %lld of %lld", who, (long long)(k / nv),
                  (long long)conn[k], (long long)d.n_nodes);
  if (n_elements == 0) return PDGPU_OK;
  const size_t m = (size_t)n_elements;
  int64_t *dconn = nullptr;
  double *dmat = nullptr, *dout = nullptr;
  uint8_t *dps = nullptr;
  cudaError_t e = cudaMalloc(&dconn, (size_t)nv * m * sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMalloc(&dmat, 3 * m * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dps, m);
  if (e == cudaSuccess) e = cudaMalloc(&dout, 3 * m * 15 * sizeof(double));
  cudaStream_t s = ctx->stream;
  if (e == cudaSuccess) e = cudaMemcpyAsync(dconn, conn, (size_t)nv * m * sizeof(int64_t), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dmat, nu, m * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dmat + m, lambda, m * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dmat + 2 * m, mu, m * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && nv == 3) e = cudaMemcpyAsync(dps, plane_strain, m, cudaMemcpyHostToDevice, s);
  double *oxq = dout, *ost = dout + 9 * m, *oss = dout + 27 * m;
  if (e == cudaSuccess)
    e = nv == 3 ? launch_strain_tri(d, n_elements, dconn, nq, ref_points, dmat, dmat + m, dmat + 2 * m, dps, oxq,
                                    ost, oss, s)
                : launch_strain_tet(d, n_elements, dconn, dmat, dmat + m, dmat + 2 * m, oxq, ost, oss, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(xq, oxq, 9 * m * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(strain, ost, 18 * m * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(stress, oss, 18 * m * sizeof(double), cudaMemcpyDeviceToHost, s);
  const cudaError_t es = cudaStreamSynchronize(s);
  cudaFree(dconn);
  cudaFree(dmat);
  cudaFree(dps);
  cudaFree(dout);
  if (e != cudaSuccess || es != cudaSuccess)
    return fail(ctx, PDGPU_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e != cudaSuccess ? e : es));
  return device_error(ctx);
}

}  // namespace

extern "C" {

int pdgpu_strain_stress_tri(pdgpu_ctx *ctx, int64_t n_elements, const int64_t *conn, int32_t nq,
                            const double *ref_points, const double *nu, const double *lambda, const double *mu,
                            const uint8_t *plane_strain, double *xq, double *strain, double *stress) {
  return strain_stress(ctx, "strain_stress_tri", 3, n_elements, conn, nq, ref_points, nu, lambda, mu, plane_strain,
                       xq, strain, stress);
}

int pdgpu_strain_stress_tet(pdgpu_ctx *ctx, int64_t n_elements, const int64_t *conn, const double *nu,
                            const double *lambda, const double *mu, double *xq, double *strain, double *stress) {
  return strain_stress(ctx, "strain_stress_tet", 4, n_elements, conn, 1, nullptr, nu, lambda, mu, nullptr, xq,
                       strain, stress);
}

int pdgpu_write_strain_vtu(pdgpu_ctx *ctx, const char *path, int64_t n_points, const double *xq,
                           const double *strain, const double *stress) {
  if (!ctx || !path || n_points < 0 || (n_points > 0 && (!xq || !strain || !stress))) return PDGPU_ERR_ARG;
  CtrlState c;
  TRY(read_ctrl(ctx, &c));
  const size_t n = (size_t)n_points;
  std::vector<VtuArray> pdata;
  const std::vector<std::string> names{"xx", "yy", "zz", "yz", "xz", "xy"};
  pdata.push_back(vtu_array("Strain", "Float64", 6, std::vector<double>(strain, strain + 6 * n)));
  pdata.back().comp_names = names;
  pdata.push_back(vtu_array("Stress", "Float64", 6, std::vector<double>(stress, stress + 6 * n)));
  pdata.back().comp_names = names;
  std::string err;
  if (!write_points_vtu(path, n_points, c.time, std::vector<double>(xq, xq + 3 * n), pdata, &err))
    return fail(ctx, PDGPU_ERR_ARG, "write_strain_vtu: %s", err.c_str());
  return PDGPU_OK;
}

int pdgpu_enable_rebuild_phases(pdgpu_ctx *ctx, int32_t on) {
  if (!ctx) return PDGPU_ERR_ARG;
  DevData &d = ctx->d;
  if (on && !d.phase_ns) {
    TRY(dalloc(ctx, &d.phase_ns, (size_t)kRebuildPhases));
    CK(cudaMemset(d.phase_ns, 0, kRebuildPhases * sizeof(unsigned long long)));
  } else if (!on && d.phase_ns) {
    CK(cudaStreamSynchronize(ctx->stream));
    d.phase_ns = nullptr;  // the buffer stays with the context's allocations
  }
  if (ctx->gexec) {  // kernels in a graph hold the DevData they were captured with
    cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
  }
  return PDGPU_OK;
}

int pdgpu_rebuild_phases(pdgpu_ctx *ctx, int64_t *ns, int32_t cap, int32_t *count) {
  if (!ctx || !count || cap < 0 || (cap > 0 && !ns)) return PDGPU_ERR_ARG;
  *count = 0;
  if (!ctx->d.phase_ns) return PDGPU_OK;
  unsigned long long h[kRebuildPhases];
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(h, ctx->d.phase_ns, sizeof h, cudaMemcpyDeviceToHost));
  int n = 0;
  while (n < kRebuildPhases && h[n] != 0) n++;
  for (int k = 0; k < n && k < cap; k++) ns[k] = (int64_t)h[k];
  *count = n < cap ? n : cap;
  return PDGPU_OK;
}

int pdgpu_kernel_times(pdgpu_ctx *ctx, int32_t maxk, const char **names, double *ms,
                       int64_t *launches, int32_t *count) {
  if (!ctx || !count) return PDGPU_ERR_ARG;
  resolve_timing(ctx);
  const int n = std::min(maxk, ctx->n_names);
  for (int i = 0; i < n; i++) {
    if (names) names[i] = ctx->names[i];
    if (ms) ms[i] = ctx->ms[i];
    if (launches) launches[i] = ctx->launches[i];
  }
  *count = n;
  return PDGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// State snapshot (no counterpart in the reference, whose restart
// demModel.cpp:84-102 reads positions and velocities back and resets every
// bond to intact).  A snapshot taken between steps holds everything a step
// reads that earlier steps wrote, so a context loaded from it continues
// exactly as the saved one would have: x, u, v, f, damage, |v|, dilatation,
// the bond-broken bits, the step-control state (step, time, contact-search
// counters, post-processing results), the contact candidate lists and the
// particle-wall damping pairs of the last rebuild, the compressive-test
// history, and the learned surrogate's per-particle flags.
//
// File layout (little-endian):
//   SnapHeader
//   portable part, for any loader (util::Point layout):
//     x, u, v      [N][3] double each
//     broken bonds [n_broken][2] uint64 (i, j): pairs, so the bond order of
//                  the loader's own neighbour lists does not matter
//   device part (this library's layout; same scene and capacities):
//     x, u, v, f   [N][stride] double; Z [N] float; vmag, theta [N] double
//     bond bits    [n_words] uint32
//     CtrlState
//     contact: row [N+1] int64, count [N] int64, nodes [N] int32,
//              spans [N] int2, columns [entries] int32,
//              wall pairs [Np][wp_cap] int32, wall pair counts [Np] int32
//     history [hist][4] double; scene history [n_scenes][cap][4] double
//     surrogate flags: on [Np] uint8, near [Np] uint8 (when set)
// ---------------------------------------------------------------------------
namespace {

struct SnapHeader {
  char magic[8];        // "PDSNAP01"
  int64_t dim, n_nodes, n_bonds, n_particles;
  int64_t stride;       // doubles per node vector on the device (2 or 4)
  int64_t n_broken;     // pairs in the portable part
  int64_t n_words;      // bond-bit words in the device part
  int64_t entries;      // contact candidate entries
  int64_t wp_cap;       // particle-wall pair capacity per particle
  int64_t history;      // compressive-test records
  int64_t n_scenes, scene_hist_cap;
  int64_t surrogate;    // 1: surrogate flags follow
  int64_t multi_particle;
  // the step, and the contact-search state a loader of the portable part
  // needs (ModelData::d_n, d_time, d_contNeighUpdateInterval,
  // d_contNeighTimestepCounter, d_contNeighSearchRadius, d_maxVelocity)
  int64_t step;
  double time;
  int64_t contact_interval, contact_counter;
  double contact_radius, max_velocity;
  int64_t ctrl_bytes;   // sizeof(CtrlState) of the writer
};

template <typename T>
int dl(pdgpu_ctx *ctx, std::vector<T> *h, const T *d, size_t n) {
  h->resize(n);
  if (n) CK(cudaMemcpyAsync(h->data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  return PDGPU_OK;
}

template <typename T>
int ul(pdgpu_ctx *ctx, T *d, const std::vector<T> &h) {
  if (!h.empty()) CK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  return PDGPU_OK;
}

template <typename T>
bool wr(FILE *f, const std::vector<T> &v) {
  return v.empty() || std::fwrite(v.data(), sizeof(T), v.size(), f) == v.size();
}

template <typename T>
bool rd(FILE *f, std::vector<T> *v, size_t n) {
  v->resize(n);
  return n == 0 || std::fread(v->data(), sizeof(T), n, f) == n;
}

}  // namespace

extern "C" {

int pdgpu_save_state(pdgpu_ctx *ctx, const char *path) {
  if (!ctx || !path) return PDGPU_ERR_ARG;
  if (!ctx->begun) return fail(ctx, PDGPU_ERR_STATE, "save_state: call pdgpu_integrate_begin first");
  TRY(device_error(ctx));
  DevData &d = ctx->d;
  const int64_t N = d.n_nodes, B = d.n_bonds, st = d.dim == 2 ? 2 : 4;
  const int64_t Np = (int64_t)ctx->hp.size(), nw = (B + 31) / 32;
  const bool multi = ctx->desc.multi_particle != 0;
  CtrlState c;
  TRY(read_ctrl(ctx, &c));
  // portable part
  std::vector<double> xa(3 * N), ua(3 * N), va(3 * N);
  TRY(pdgpu_download(ctx, PDGPU_FIELD_X, xa.data()));
  TRY(pdgpu_download(ctx, PDGPU_FIELD_U, ua.data()));
  TRY(pdgpu_download(ctx, PDGPU_FIELD_V, va.data()));
  std::vector<uint32_t> bits;
  std::vector<int64_t> prow;
  std::vector<int32_t> pcol;
  TRY(dl(ctx, &bits, d.bond_bits, (size_t)nw));
  TRY(dl(ctx, &prow, d.pd_row, (size_t)N + 1));
  TRY(dl(ctx, &pcol, d.pd_col, (size_t)B));
  // device part
  std::vector<double> x, u, v, f, vmag, theta;
  std::vector<float> Z;
  TRY(dl(ctx, &x, d.x, (size_t)(st * N)));
  TRY(dl(ctx, &u, d.u, (size_t)(st * N)));
  TRY(dl(ctx, &v, d.v, (size_t)(st * N)));
  TRY(dl(ctx, &f, d.f, (size_t)(st * N)));
  TRY(dl(ctx, &Z, d.Z, (size_t)N));
  TRY(dl(ctx, &vmag, d.vmag, (size_t)N));
  TRY(dl(ctx, &theta, d.theta, (size_t)N));
  std::vector<int64_t> crow, ccnt;
  std::vector<int32_t> cnodes, cspan, ccol, wp, wpc;
  if (multi) {
    TRY(dl(ctx, &crow, d.c_row, (size_t)N + 1));
    TRY(dl(ctx, &ccnt, d.c_cnt, (size_t)N));
    TRY(dl(ctx, &cnodes, d.c_nodes, (size_t)N));
    TRY(dl(ctx, &cspan, reinterpret_cast<const int32_t *>(d.c_span), (size_t)(2 * N)));
    TRY(dl(ctx, &wp, d.wp, (size_t)(Np * d.wp_cap)));
    TRY(dl(ctx, &wpc, d.wp_cnt, (size_t)Np));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  if (multi) TRY(dl(ctx, &ccol, d.c_col, (size_t)crow[N]));
  const int64_t nh = std::min<int64_t>(c.history_count, d.history_cap);
  std::vector<double> hist, shist;
  TRY(dl(ctx, &hist, d.history, (size_t)(4 * std::max<int64_t>(nh, 0))));
  if (d.n_scenes > 1) TRY(dl(ctx, &shist, d.scene_hist, (size_t)(d.n_scenes * d.scene_hist_cap * 4)));
  std::vector<uint8_t> son, snear;
  if (d.sur_on) {
    TRY(dl(ctx, &son, d.sur_on, (size_t)Np));
    TRY(dl(ctx, &snear, d.sur_near, (size_t)Np));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  std::vector<uint64_t> pairs;
  for (int64_t i = 0; i < N; i++)
    for (int64_t k = prow[i]; k < prow[i + 1]; k++)
      if ((bits[k >> 5] >> (k & 31)) & 1u) {
        pairs.push_back((uint64_t)i);
        pairs.push_back((uint64_t)pcol[k]);
      }
  SnapHeader h{};
  std::memcpy(h.magic, "PDSNAP01", 8);
  h.dim = d.dim;
  h.n_nodes = N;
  h.n_bonds = B;
  h.n_particles = Np;
  h.stride = st;
  h.n_broken = (int64_t)pairs.size() / 2;
  h.n_words = nw;
  h.entries = multi ? crow[N] : 0;
  h.wp_cap = multi ? d.wp_cap : 0;
  h.history = std::max<int64_t>(nh, 0);
  h.n_scenes = d.n_scenes;
  h.scene_hist_cap = d.n_scenes > 1 ? d.scene_hist_cap : 0;
  h.surrogate = d.sur_on ? 1 : 0;
  h.multi_particle = multi ? 1 : 0;
  h.step = c.n;
  h.time = c.time;
  h.contact_interval = c.interval;
  h.contact_counter = c.counter;
  h.contact_radius = c.radius;
  h.max_velocity = c.max_velocity;
  h.ctrl_bytes = (int64_t)sizeof(CtrlState);
  FILE *fo = std::fopen(path, "wb");
  if (!fo) return fail(ctx, PDGPU_ERR_ARG, "save_state: cannot write %s", path);
  bool ok = std::fwrite(&h, sizeof h, 1, fo) == 1 && wr(fo, xa) && wr(fo, ua) && wr(fo, va) && wr(fo, pairs) &&
            wr(fo, x) && wr(fo, u) && wr(fo, v) && wr(fo, f) && wr(fo, Z) && wr(fo, vmag) && wr(fo, theta) &&
            wr(fo, bits) && std::fwrite(&c, sizeof c, 1, fo) == 1;
  if (ok && multi) ok = wr(fo, crow) && wr(fo, ccnt) && wr(fo, cnodes) && wr(fo, cspan) && wr(fo, ccol) &&
                        wr(fo, wp) && wr(fo, wpc);
  if (ok) ok = wr(fo, hist) && wr(fo, shist) && wr(fo, son) && wr(fo, snear);
  ok = (std::fclose(fo) == 0) && ok;
  if (!ok) return fail(ctx, PDGPU_ERR_ARG, "save_state: writing %s failed", path);
  return PDGPU_OK;
}

int pdgpu_load_state(pdgpu_ctx *ctx, const char *path) {
  if (!ctx || !path) return PDGPU_ERR_ARG;
  if (ctx->begun)
    return fail(ctx, PDGPU_ERR_STATE, "load_state takes the place of pdgpu_integrate_begin: the model has started");
  TRY(prepare(ctx));
  const bool multi = ctx->desc.multi_particle != 0;
  if (multi && !ctx->contact_init) TRY(pdgpu_init_contact(ctx));
  DevData &d = ctx->d;
  const int64_t N = d.n_nodes, B = d.n_bonds, st = d.dim == 2 ? 2 : 4;
  const int64_t Np = (int64_t)ctx->hp.size(), nw = (B + 31) / 32;
  FILE *fi = std::fopen(path, "rb");
  if (!fi) return fail(ctx, PDGPU_ERR_ARG, "load_state: cannot open %s", path);
  SnapHeader h{};
  bool ok = std::fread(&h, sizeof h, 1, fi) == 1 && std::memcmp(h.magic, "PDSNAP01", 8) == 0;
  if (!ok) {
    std::fclose(fi);
    return fail(ctx, PDGPU_ERR_ARG, "load_state: %s is not a pdgpu state snapshot", path);
  }
  const char *why = nullptr;
  if (h.dim != d.dim || h.n_nodes != N || h.n_bonds != B || h.n_particles != Np || h.stride != st)
    why = "it holds another scene (dimension, nodes, bonds or particles differ)";
  else if (h.n_words != nw || h.ctrl_bytes != (int64_t)sizeof(CtrlState))
    why = "it was written by an incompatible library";
  else if (h.multi_particle != (multi ? 1 : 0))
    why = "contact is on in one model and off in the other";
  else if (multi && (h.entries > d.contact_cap || h.wp_cap != d.wp_cap))
    why = "its contact lists do not fit this model's capacities";
  else if (h.n_scenes != d.n_scenes || (d.n_scenes > 1 && h.scene_hist_cap != d.scene_hist_cap))
    why = "its scene layout differs";
  if (why) {
    std::fclose(fi);
    return fail(ctx, PDGPU_ERR_ARG, "load_state: %s: %s", path, why);
  }
  std::vector<double> skip, x, u, v, f, vmag, theta, hist, shist;
  std::vector<uint64_t> pairs;
  std::vector<float> Z;
  std::vector<uint32_t> bits;
  std::vector<int64_t> crow, ccnt;
  std::vector<int32_t> cnodes, cspan, ccol, wp, wpc;
  std::vector<uint8_t> son, snear;
  CtrlState c;
  ok = rd(fi, &skip, (size_t)(9 * N)) && rd(fi, &pairs, (size_t)(2 * h.n_broken)) &&
       rd(fi, &x, (size_t)(st * N)) && rd(fi, &u, (size_t)(st * N)) && rd(fi, &v, (size_t)(st * N)) &&
       rd(fi, &f, (size_t)(st * N)) && rd(fi, &Z, (size_t)N) && rd(fi, &vmag, (size_t)N) &&
       rd(fi, &theta, (size_t)N) && rd(fi, &bits, (size_t)nw) && std::fread(&c, sizeof c, 1, fi) == 1;
  if (ok && multi)
    ok = rd(fi, &crow, (size_t)N + 1) && rd(fi, &ccnt, (size_t)N) && rd(fi, &cnodes, (size_t)N) &&
         rd(fi, &cspan, (size_t)(2 * N)) && rd(fi, &ccol, (size_t)h.entries) &&
         rd(fi, &wp, (size_t)(Np * d.wp_cap)) && rd(fi, &wpc, (size_t)Np);
  if (ok)
    ok = rd(fi, &hist, (size_t)(4 * h.history)) &&
         rd(fi, &shist, (size_t)(h.n_scenes > 1 ? h.n_scenes * h.scene_hist_cap * 4 : 0));
  if (ok && h.surrogate) ok = rd(fi, &son, (size_t)Np) && rd(fi, &snear, (size_t)Np);
  std::fclose(fi);
  if (!ok) return fail(ctx, PDGPU_ERR_ARG, "load_state: %s is truncated", path);
  if (multi && (crow[0] != 0 || crow[N] != h.entries))
    return fail(ctx, PDGPU_ERR_ARG, "load_state: %s: contact row offsets are inconsistent", path);
  if (h.history > d.history_cap) return fail(ctx, PDGPU_ERR_ARG, "load_state: %s: history too long", path);
  // the step resumes from the saved state: no restart rule, nothing in flight
  c.error = 0;
  c.error_info = 0;
  c.begin_done = c.end_done = 0;
  c.tile_next = c.tile_done = 0;
  c.bar_count = 0;
  d.restart_step = -1;
  TRY(ul(ctx, d.x, x));
  TRY(ul(ctx, d.u, u));
  TRY(ul(ctx, d.v, v));
  TRY(ul(ctx, d.f, f));
  TRY(ul(ctx, d.Z, Z));
  TRY(ul(ctx, d.vmag, vmag));
  TRY(ul(ctx, d.theta, theta));
  TRY(ul(ctx, d.bond_bits, bits));
  CK(cudaMemcpyAsync(d.ctrl, &c, sizeof c, cudaMemcpyHostToDevice, ctx->stream));
  if (multi) {
    TRY(ul(ctx, d.c_row, crow));
    TRY(ul(ctx, d.c_cnt, ccnt));
    TRY(ul(ctx, d.c_nodes, cnodes));
    TRY(ul(ctx, reinterpret_cast<int32_t *>(d.c_span), cspan));
    TRY(ul(ctx, d.c_col, ccol));
    launch_contact_owner(d, ctx->stream);
    CK(cudaGetLastError());
    TRY(ul(ctx, d.wp, wp));
    TRY(ul(ctx, d.wp_cnt, wpc));
    CK(cudaMemsetAsync(d.fc, 0, (size_t)(st * N) * 8, ctx->stream));
  }
  TRY(ul(ctx, d.history, hist));
  if (d.n_scenes > 1) TRY(ul(ctx, d.scene_hist, shist));
  if (d.sur_on && h.surrogate) {
    TRY(ul(ctx, d.sur_on, son));
    TRY(ul(ctx, d.sur_near, snear));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->gexec) {
    cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
  }
  TRY(sym_bits(ctx));
  ctx->begun = true;
  return PDGPU_OK;
}

}  // extern "C"
