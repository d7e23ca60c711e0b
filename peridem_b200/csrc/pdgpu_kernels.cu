// FP64 kernels of the explicit step.  This file is compiled with
// --fmad=false: every product and sum rounds separately, as in the
// reference's x86-64 build (no -march, so no FMA contraction), which keeps
// the bond-break, contact and neighbour-search decisions bit-identical to
// the reference for the same inputs.
//
// Layout in HBM: node vectors are stored with a stride of 2 doubles in 2-D
// (double2) and 4 doubles in 3-D (double4, last lane unused), so one node is
// one aligned 16- or 32-byte access; peridynamic bonds are CSR (int64 row
// offsets, int32 columns) with one broken-bit per bond in a uint32 bitmap.
#include <cooperative_groups.h>
#include <cub/cub.cuh>

#include <cfloat>
#include <cstdint>

#include "pdgpu_internal.h"

namespace pdgpu {

namespace {

constexpr double kPi = 3.14159265358979323846;  // M_PI
constexpr int kBlock = 256;

// util::isGreater / util::isLess with COMPARE_EPS = 1e-5
// (src/util/function.cpp:15-23, function.h:18)
__device__ __forceinline__ bool is_greater(double a, double b) {
  const double fa = fabs(a), fb = fabs(b);
  return (a - b) > ((fa < fb ? fb : fa) * 1.0e-5);
}
__device__ __forceinline__ bool is_less(double a, double b) {
  const double fa = fabs(a), fb = fabs(b);
  return (b - a) > ((fa < fb ? fb : fa) * 1.0e-5);
}

template <int DIM>
__device__ __forceinline__ void ldv(const double *__restrict__ a, int64_t i, double (&o)[3]) {
  if constexpr (DIM == 2) {
    const double2 t = reinterpret_cast<const double2 *>(a)[i];
    o[0] = t.x;
    o[1] = t.y;
    o[2] = 0.0;
  } else {
    const double2 *p = reinterpret_cast<const double2 *>(a) + 2 * i;
    const double2 t0 = p[0], t1 = p[1];
    o[0] = t0.x;
    o[1] = t0.y;
    o[2] = t1.x;
  }
}

template <int DIM>
__device__ __forceinline__ void ldg_v(const double *__restrict__ a, int64_t i, double (&o)[3]) {
  if constexpr (DIM == 2) {
    const double2 t = __ldg(reinterpret_cast<const double2 *>(a) + i);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = 0.0;
  } else {
    const double2 *p = reinterpret_cast<const double2 *>(a) + 2 * i;
    const double2 t0 = __ldg(p), t1 = __ldg(p + 1);
    o[0] = t0.x;
    o[1] = t0.y;
    o[2] = t1.x;
  }
}

template <int DIM>
__device__ __forceinline__ void stv(double *__restrict__ a, int64_t i, const double (&o)[3]) {
  if constexpr (DIM == 2) {
    reinterpret_cast<double2 *>(a)[i] = make_double2(o[0], o[1]);
  } else {
    double2 *p = reinterpret_cast<double2 *>(a) + 2 * i;
    p[0] = make_double2(o[0], o[1]);
    p[1] = make_double2(o[2], 0.0);
  }
}

// util::Point::length / dot: ((x*x + y*y) + z*z); the z term is an exact
// no-op in 2-D (z = 0), so it is skipped there.
template <int DIM>
__device__ __forceinline__ double dot3(const double (&a)[3], const double (&b)[3]) {
  double s = a[0] * b[0] + a[1] * b[1];
  if constexpr (DIM == 3) s = s + a[2] * b[2];
  return s;
}
template <int DIM>
__device__ __forceinline__ double len3(const double (&a)[3]) {
  return sqrt(dot3<DIM>(a, a));
}

// J(r / horizon) of the process-wide influence function
// (influenceFn.cpp:21-23, 55-57, 86-88; material.h:431-433)
__device__ __forceinline__ double influence(const Influence &f, double r, double horizon) {
  const double q = r / horizon;
  if (f.type == PDGPU_INF_LINEAR) return f.p0 + f.p1 * q;
  if (f.type == PDGPU_INF_CONST) return f.p0;
  return f.p0 * exp(-q * q / f.p1);
}

template <int LPN>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (LPN == 32) {
    return 0xffffffffu;
  } else {
    const unsigned lane = threadIdx.x & 31u;
    return ((1u << LPN) - 1u) << (lane / LPN * LPN);
  }
}

template <int LPN>
__device__ __forceinline__ double group_sum(double v, unsigned m) {
#pragma unroll
  for (int o = LPN / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o);
  return v;
}
template <int LPN>
__device__ __forceinline__ double group_max(double v, unsigned m) {
#pragma unroll
  for (int o = LPN / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(m, v, o));
  return v;
}
template <int LPN>
__device__ __forceinline__ int64_t group_sum_i(int64_t v, unsigned m) {
#pragma unroll
  for (int o = LPN / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o);
  return v;
}

__device__ __forceinline__ void set_error(CtrlState *c, int code, int64_t info) {
  if (atomicCAS(&c->error, 0, code) == 0) c->error_info = info;
}

// non-negative doubles order like their bit patterns
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *a, double v) {
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

template <int DIM>
__device__ __forceinline__ int cell_coord(double x, const Grid &g, int d) {
  double c = floor((x - g.lo[d]) * g.inv_cell);
  if (c < 0.0) c = 0.0;
  const double hi = (double)(g.dims[d] - 1);
  if (c > hi) c = hi;
  return (int)c;
}

template <int DIM>
__device__ __forceinline__ int cell_index(const double (&p)[3], const Grid &g) {
  int c = cell_coord<DIM>(p[0], g, 0) + g.dims[0] * cell_coord<DIM>(p[1], g, 1);
  if constexpr (DIM == 3) c += g.dims[0] * g.dims[1] * cell_coord<DIM>(p[2], g, 2);
  return c;
}

// ---------------------------------------------------------------------------
// layout conversion
// ---------------------------------------------------------------------------

template <int DIM>
__global__ void k_pack(const double *__restrict__ aos3, double *__restrict__ dst, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double o[3] = {aos3[3 * i], aos3[3 * i + 1], aos3[3 * i + 2]};
  stv<DIM>(dst, i, o);
}

template <int DIM>
__global__ void k_unpack(const double *__restrict__ src, double *__restrict__ aos3, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double o[3];
  ldv<DIM>(src, i, o);
  aos3[3 * i] = o[0];
  aos3[3 * i + 1] = o[1];
  aos3[3 * i + 2] = (DIM == 3) ? o[2] : 0.0;
}

// ---------------------------------------------------------------------------
// DEMModel::applyInitialCondition (demModel.cpp:1068-1095): every node of a
// listed particle gets the IC velocity (all three components).
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void k_apply_ic(DevData d) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_nodes) return;
  if (!d.ic_particle[d.ptid[i]]) return;
  double o[3] = {d.ic_v[0], d.ic_v[1], d.ic_v[2]};
  stv<DIM>(d.v, i, o);
}

// ---------------------------------------------------------------------------
// DEMModel::integrateCD (demModel.cpp:349-390) and the first half of
// DEMModel::integrateVerlet (:392-424), over d_fPdCompNodes, free dofs only.
// Also folds |v| into the running maximum that the contact-search control
// reads (updateContactNeighborSearchParameters, :1862-1883).
// ---------------------------------------------------------------------------
template <int DIM, bool VERLET>
__global__ void __launch_bounds__(kBlock) k_integrate(DevData d) {
  __shared__ double smax[kBlock / 32];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double vm = 0.0;
  if (i < d.n_nodes && (d.flags[i] & NODE_ACTIVE) && !d.ctrl->error) {
    const double rho = d.particles[d.ptid[i]].density;
    const uint8_t fix = d.fix[i];
    double v[3], u[3], x[3], f[3];
    ldv<DIM>(d.v, i, v);
    ldv<DIM>(d.u, i, u);
    ldv<DIM>(d.x, i, x);
    ldv<DIM>(d.f, i, f);
    const double dt = d.dt;
    const double k = VERLET ? 0.5 * (dt / rho) : dt / rho;
#pragma unroll
    for (int dof = 0; dof < DIM; dof++) {
      if (!((fix >> dof) & 1u)) {
        v[dof] += k * f[dof];
        u[dof] += dt * v[dof];
        x[dof] += dt * v[dof];
      }
    }
    stv<DIM>(d.v, i, v);
    stv<DIM>(d.u, i, u);
    stv<DIM>(d.x, i, x);
    vm = len3<DIM>(v);
    d.vmag[i] = vm;
  }
  // block max of |v| -> one atomic per block
  for (int o = 16; o > 0; o >>= 1) vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, o));
  if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = vm;
  __syncthreads();
  if (threadIdx.x < 32) {
    double m = threadIdx.x < kBlock / 32 ? smax[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0 && m > 0.0) atomic_max_nonneg(&d.ctrl->vmax_bits, m);
  }
}

// second half kick of DEMModel::integrateVerlet (:436-459)
template <int DIM>
__global__ void k_verlet_second(DevData d) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_nodes || !(d.flags[i] & NODE_ACTIVE) || d.ctrl->error) return;
  const double rho = d.particles[d.ptid[i]].density;
  const uint8_t fix = d.fix[i];
  double v[3], f[3];
  ldv<DIM>(d.v, i, v);
  ldv<DIM>(d.f, i, f);
  const double k = 0.5 * (d.dt / rho);
#pragma unroll
  for (int dof = 0; dof < DIM; dof++)
    if (!((fix >> dof) & 1u)) v[dof] += k * f[dof];
  stv<DIM>(d.v, i, v);
  d.vmag[i] = len3<DIM>(v);
}

// ---------------------------------------------------------------------------
// Step control (one thread): time advance (integrateCD :381-383) and the
// contact-list update decision of
// DEMModel::updateContactNeighborSearchParameters (demModel.cpp:1808-1955).
// mode 0: a time step; 1: the computeForces call of the integrate() prelude;
// 2: the contact list build of DEMModel::init.
// ---------------------------------------------------------------------------
// the fields the step control changes, written back in one go
__device__ __forceinline__ void ctrl_commit(CtrlState *dst, const CtrlState &c) {
  dst->n = c.n;
  dst->time = c.time;
  dst->first_bc = c.first_bc;
  dst->init_calls = c.init_calls;
  dst->counter = c.counter;
  dst->interval = c.interval;
  dst->radius = c.radius;
  dst->max_velocity = c.max_velocity;
  dst->update = c.update;
  dst->sur_check = c.sur_check;
}

// pre: a copy of the state taken earlier in the same kernel (its fields are
// written only here), or null to read it now
__device__ __noinline__ void ctrl_step(const DevData &d, int mode, const CtrlState *pre = nullptr) {
  CtrlState *cp = d.ctrl;
  CtrlState c = pre ? *pre : *cp;  // one pass over the state instead of a chain of loads
  if (c.error) return;
  if (mode == 0) {
    c.n += 1;
    c.time += d.dt;
    c.first_bc = 0;
  }
  // learned surrogate: every sur_interval-th step (and the first) re-judges
  // it with the full bond loop
  c.sur_check = d.sur_interval > 0 && (c.n % d.sur_interval == 0 || c.n <= 1);
  // read and reset atomically: other CTAs raised it with atomicMax
  const double vmax_now =
      fmax(__longlong_as_double((long long)atomicExch(&cp->vmax_bits, 0ull)), c.static_vmax);
  if (!d.n_zones) {  // single particle: no contact
    c.update = 0;
    ctrl_commit(cp, c);
    return;
  }
  const int64_t n = c.n;
  if (n == 0) {
    c.init_calls += 1;
    if (c.init_calls == 1) {
      c.update = 1;
      ctrl_commit(cp, c);
      return;
    }
    if (c.init_calls == 2) {
      c.counter += 1;
      c.update = ((c.counter - 1) % c.interval) == 0;
      ctrl_commit(cp, c);
      return;
    }
  }
  // restart: the counter of the restart step (demModel.cpp:1833-1837)
  if (d.restart_step >= 0 && n == d.restart_step) c.counter = n % c.interval;
  if (c.interval == 1) {
    c.radius = d.max_contact_r;
    c.counter += 1;
    c.update = ((c.counter - 1) % c.interval) == 0;
    ctrl_commit(cp, c);
    return;
  }
  const int64_t upi = c.interval > 5 ? (int64_t)(0.2 * (double)c.interval) : 1;
  if (c.counter > 0 && c.counter % upi != 0) {
    c.counter += 1;
    c.update = ((c.counter - 1) % c.interval) == 0;
    ctrl_commit(cp, c);
    return;
  }
  c.max_velocity = vmax_now;
  const double safety = d.search_factor > 5 ? d.search_factor : 10.0;
  const double r_contact = d.search_factor * d.max_contact_r;
  const double r_vel = c.max_velocity * d.dt * (double)d.search_interval * safety;
  if (is_greater(r_vel, r_contact)) {
    c.interval = (int64_t)(d.max_contact_r / (c.max_velocity * d.dt));
    c.radius = r_contact;
    c.counter = 0;
    if (c.interval < 1) {
      c.interval = 1;
      c.radius = d.max_contact_r;
    }
  } else {
    c.radius = c.interval < 2 ? d.max_contact_r : r_contact;
  }
  c.counter += 1;
  c.update = ((c.counter - 1) % c.interval) == 0;
  ctrl_commit(cp, c);
}

__global__ void k_ctrl(const __grid_constant__ DevData d, int mode) { ctrl_step(d, mode); }


// ---------------------------------------------------------------------------
// DEMModel::computeExternalDisplacementBC -> ParticleULoading::apply
// (particleULoading.cpp:115-230).  One thread per BC node applies that node's
// sets in deck order; the spatial factor of each (node, set) is precomputed
// on the host from the reference configuration.
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __noinline__ void apply_ubc(const DevData &d, int t, int64_t i, double time, int first,
                                          double (&u)[3], double (&v)[3], double (&x)[3]) {
  double xr[3];
  ldg_v<DIM>(d.xref, i, xr);
  for (int e = d.ubc_row[t]; e < d.ubc_row[t + 1]; e++) {
    if (d.ubc_once[e] && !first) continue;
    const BcSetDev bc = d.ubc_sets[d.ubc_set[e]];
    const double umax = d.ubc_val[e];
    double du = 0.0, dv = 0.0;
    switch (bc.time_fn) {
      case PDGPU_TIME_CONSTANT: du = umax; break;
      case PDGPU_TIME_LINEAR: du = umax * time; dv = umax; break;
      case PDGPU_TIME_QUADRATIC:
        du = umax * time + bc.tp[1] * time * time;
        dv = umax + bc.tp[1] * time;
        break;
      case PDGPU_TIME_SIN: {
        const double a = kPi * bc.tp[1];
        du = umax * sin(a * time);
        dv = umax * a * cos(a * time);
        break;
      }
      default: break;
    }
    double ui[3] = {0.0, 0.0, 0.0}, vi[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < 3; q++)
      if ((bc.dir_mask >> q) & 1) {
        ui[q] = du;
        vi[q] = dv;
      }
    if (bc.time_fn == PDGPU_TIME_ROTATION) {
      const double dx0 = xr[0] - bc.tp[1], dx1 = xr[1] - bc.tp[2];
      const double th = bc.tp[0] * time;
      const double ct = cos(th), st = sin(th);
      // util::rotate2D / derRotate2D (transformation.cpp:53-65)
      const double r0 = dx0 * ct - dx1 * st, r1 = dx0 * st + dx1 * ct;
      const double d0 = -dx0 * st - dx1 * ct, d1 = dx0 * ct - dx1 * st;
      ui[0] += r0 - dx0;
      ui[1] += r1 - dx1;
      ui[2] += 0.0 - (xr[2] - bc.tp[3]);
      vi[0] += bc.tp[0] * d0;
      vi[1] += bc.tp[0] * d1;
      vi[2] += bc.tp[0] * 0.0;
    }
    for (int q = 0; q < DIM; q++)
      if ((bc.dir_mask >> q) & 1) {
        u[q] = ui[q];
        v[q] = vi[q];
        x[q] = ui[q] + xr[q];
      }
  }
}

template <int DIM>
__global__ void k_bc(const __grid_constant__ DevData d) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.n_ubc_nodes || d.ctrl->error) return;
  const int64_t i = d.ubc_node[t];
  double u[3], v[3], x[3];
  ldv<DIM>(d.u, i, u);
  ldv<DIM>(d.v, i, v);
  ldv<DIM>(d.x, i, x);
  apply_ubc<DIM>(d, t, i, d.ctrl->time, d.ctrl->first_bc, u, v, x);
  stv<DIM>(d.u, i, u);
  stv<DIM>(d.v, i, v);
  stv<DIM>(d.x, i, x);
}

// ---------------------------------------------------------------------------
// First kernel of a step: integrateCD / the first Verlet half (as k_integrate),
// then the displacement BC of each BC node at the step's new time (as k_bc
// after k_ctrl: zero-displacement sets are not re-applied), then — in the
// last CTA to finish — the step control (as k_ctrl, mode 0).
// ---------------------------------------------------------------------------
constexpr int kBeginNodes = 2;  // nodes per thread of the step-begin kernel

template <int DIM, bool VERLET>
__global__ void __launch_bounds__(kBlock) k_step_begin(const __grid_constant__ DevData d) {
  __shared__ double smax[kBlock / 32];
  __shared__ int last;
  __shared__ __align__(8) CtrlState s_ctrl;
  static_assert(sizeof(CtrlState) % 8 == 0 && sizeof(CtrlState) / 8 <= kBlock, "CtrlState copy");
  // every block copies the step-control state now, while its nodes load: the
  // last block's step control then starts without a chain of cold loads
  if (threadIdx.x < sizeof(CtrlState) / 8)
    reinterpret_cast<uint64_t *>(&s_ctrl)[threadIdx.x] = reinterpret_cast<const uint64_t *>(d.ctrl)[threadIdx.x];
  // CTAs run in reverse node order: the boundary-condition nodes (walls, at
  // the end of the node array) then start in the first wave.  Each thread
  // takes kBeginNodes nodes, kBlock apart, and issues every load of all of
  // them before the first update.
  const int64_t base = (int64_t)(gridDim.x - 1 - blockIdx.x) * (kBlock * kBeginNodes) + threadIdx.x;
  double vm = 0.0;
  if (!d.ctrl->error) {
    uint8_t fl[kBeginNodes], fix[kBeginNodes];
    int32_t pid[kBeginNodes];
    double v[kBeginNodes][3], u[kBeginNodes][3], x[kBeginNodes][3], f[kBeginNodes][3];
#pragma unroll
    for (int k = 0; k < kBeginNodes; k++) {
      const int64_t i = base + (int64_t)k * kBlock;
      fl[k] = 0;
      if (i < d.n_nodes) {
        fl[k] = d.flags[i];
        fix[k] = d.fix[i];
        pid[k] = d.ptid[i];
        ldv<DIM>(d.v, i, v[k]);
        ldv<DIM>(d.u, i, u[k]);
        ldv<DIM>(d.x, i, x[k]);
        ldv<DIM>(d.f, i, f[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < kBeginNodes; k++) {
      const int64_t i = base + (int64_t)k * kBlock;
      if (!(fl[k] & (NODE_ACTIVE | NODE_UBC))) continue;
      if (fl[k] & NODE_ACTIVE) {
        const double rho = d.particles[pid[k]].density;
        const double dt = d.dt;
        const double kk = VERLET ? 0.5 * (dt / rho) : dt / rho;
#pragma unroll
        for (int dof = 0; dof < DIM; dof++) {
          if (!((fix[k] >> dof) & 1u)) {
            v[k][dof] += kk * f[k][dof];
            u[k][dof] += dt * v[k][dof];
            x[k][dof] += dt * v[k][dof];
          }
        }
        const double m = len3<DIM>(v[k]);
        vm = fmax(vm, m);
        d.vmag[i] = m;
      }
      // the step control advances time by dt before the BC pass (through
      // copies: only they have their address taken, so the per-node arrays
      // stay in registers)
      if (fl[k] & NODE_UBC) {
        double ub[3], vb[3], xb[3];
#pragma unroll
        for (int q = 0; q < 3; q++) ub[q] = u[k][q], vb[q] = v[k][q], xb[q] = x[k][q];
        apply_ubc<DIM>(d, d.ubc_of[i], i, d.ctrl->time + d.dt, 0, ub, vb, xb);
#pragma unroll
        for (int q = 0; q < 3; q++) u[k][q] = ub[q], v[k][q] = vb[q], x[k][q] = xb[q];
      }
      stv<DIM>(d.v, i, v[k]);
      stv<DIM>(d.u, i, u[k]);
      stv<DIM>(d.x, i, x[k]);
    }
  }
  // block max of |v| -> one atomic per block
  for (int o = 16; o > 0; o >>= 1) vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, o));
  if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = vm;
  __syncthreads();
  if (threadIdx.x < 32) {
    double m = threadIdx.x < kBlock / 32 ? smax[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) {
      if (m > 0.0) atomic_max_nonneg(&d.ctrl->vmax_bits, m);
      __threadfence();
      last = atomicAdd(&d.ctrl->begin_done, 1u) == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    d.ctrl->begin_done = 0u;
    ctrl_step(d, 0, &s_ctrl);
  }
}

// ---------------------------------------------------------------------------
// Contact candidate lists: DEMModel::updateContactNeighborlist
// (demModel.cpp:1696-1756) with the kd-tree exclude-tag radius search
// (nsearch.h:278-301; strict  sum_d (q_d - p_d)^2 < r*r  of
// nanoflann.hpp:611-621 / nflannSetup.h:272) replaced by a cell list.
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void k_cell_count(DevData d, const double *__restrict__ pos, Grid g) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_nodes) return;
  if (d.ctrl->error || !d.ctrl->update) return;
  double p[3];
  ldv<DIM>(pos, i, p);
  const int c = cell_index<DIM>(p, g);
  d.cell_of[i] = c;
  atomicAdd(d.cell_cnt + c, 1);
}

__global__ void k_cell_scatter(DevData d) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_nodes) return;
  if (d.ctrl->error || !d.ctrl->update) return;
  const int c = d.cell_of[i];
  const int pos = d.cell_start[c] + atomicAdd(d.cell_fill + c, 1);
  d.cell_tmp[pos] = (int32_t)i;
}

// one warp per cell: order the cell's nodes by index (rank counting), so
// candidate lists do not depend on atomic arrival order
__global__ void k_cell_sort(DevData d) {
  const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= d.grid.ncells) return;
  if (d.ctrl->error || !d.ctrl->update) return;
  const int s = d.cell_start[c], e = d.cell_start[c + 1];
  for (int a = s + lane; a < e; a += 32) {
    const int32_t va = d.cell_tmp[a];
    int rank = 0;
    for (int b = s; b < e; b++) rank += d.cell_tmp[b] < va;
    d.cell_nodes[s + rank] = va;
  }
  if (lane == 0) d.cell_fill[c] = 0;
}

__global__ void k_zero_cells(DevData d) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > d.grid.ncells) return;
  if (!d.ctrl->update) return;
  d.cell_cnt[c] = 0;
}





// ---------------------------------------------------------------------------
// The whole contact-list rebuild as one cooperative launch: every phase is
// separated by a grid-wide barrier of the cooperative launch (all blocks are
// co-resident by construction).  On steps without a rebuild every block
// returns after reading the control word, so the rebuild costs one launch.
// ---------------------------------------------------------------------------
namespace cg = cooperative_groups;
constexpr int kCoopBlock = 256;

// Grid-wide barrier with a bounded wait: thread 0 of each block arrives on
// a counter in the step-control state; the last to arrive resets it and
// advances the generation the others poll.  All blocks of the cooperative
// launch are resident, so the wait ends unless a block faulted; after
// kBarWaitNs of the GPU's global timer (far beyond any phase of a rebuild)
// the block records DEV_ERR_BARRIER_TIMEOUT and every block leaves the
// rebuild at its next barrier (the step's later kernels see the error word
// and do nothing).  Returns false when the rebuild must stop.
constexpr unsigned long long kBarWaitNs = 30ull * 1000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ bool grid_bar(CtrlState *c) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *gen = &c->bar_gen;
    const unsigned g0 = *gen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(&c->bar_count, 1u) == gridDim.x - 1) {
      atomicExch(&c->bar_count, 0u);
      __threadfence();
      atomicAdd(&c->bar_gen, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      unsigned polls = 0;
      while (*gen == g0) {
        // the clock is read every 256 polls; the poll count is a second,
        // clock-independent bound (2^31 polls of at least a few ns each)
        if ((++polls & 255u) == 0 && (global_ns() - t0 > kBarWaitNs || polls > (1u << 31))) {
          ok = 0;
          atomicCAS(&c->error, 0, DEV_ERR_BARRIER_TIMEOUT);
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
    s_ok = ok && !((volatile int *)&c->error)[0];
  }
  __syncthreads();
  return s_ok != 0;
}

// exclusive scan over the whole grid: out[i] = sum_{k<i} in(k) for
// i = 0..n, each block scanning one contiguous chunk; false when a barrier
// gave up
template <class Tout, class F>
__device__ bool grid_scan(CtrlState *gc, F in, Tout *out, int64_t n, int64_t *bsum) {
  __shared__ int64_t wsum[kCoopBlock / 32];
  __shared__ int64_t carry;
  const int64_t nb = gridDim.x;
  const int64_t chunk = (n + nb - 1) / nb;
  const int64_t b0 = blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // block totals
  int64_t t = 0;
  for (int64_t k = b0 + threadIdx.x; k < b1; k += blockDim.x) t += (int64_t)in(k);
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (lane == 0) wsum[warp] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t s = 0;
    for (int w = 0; w < kCoopBlock / 32; w++) s += wsum[w];
    bsum[blockIdx.x] = s;
  }
  if (!grid_bar(gc)) return false;
  {
    // carry = sum of the earlier blocks' totals, summed by the whole block
    // (integers: any order gives the same sum); read past L1, which may
    // hold this array from an earlier scan of the same launch
    int64_t s = 0;
    for (int64_t b = threadIdx.x; b < blockIdx.x; b += blockDim.x) s += __ldcg(bsum + b);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) wsum[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t c = 0;
      for (int w = 0; w < kCoopBlock / 32; w++) c += wsum[w];
      carry = c;
    }
    __syncthreads();
  }
  for (int64_t base = b0; base < b1; base += blockDim.x) {
    const int64_t k = base + threadIdx.x;
    const int64_t v = k < b1 ? (int64_t)in(k) : 0;
    int64_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int64_t woff = 0;
    for (int w = 0; w < warp; w++) woff += wsum[w];
    if (k < b1) out[k] = (Tout)(carry + woff + incl - v);
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t s = 0;
      for (int w = 0; w < kCoopBlock / 32; w++) s += wsum[w];
      carry += s;
    }
    __syncthreads();
  }
  if (blockIdx.x == nb - 1 && threadIdx.x == 0) out[n] = (Tout)carry;
  return grid_bar(gc);
}


// Candidate pass, cell-centric: a warp takes a centre cell and stages its
// neighbourhood (the 3^DIM cells around it, z, y, x ascending; each cell's
// nodes ascending) in its own slice of shared memory, in chunks; every
// searching node of the centre cell scans the staged list in that order with
// the strict test sum_d (q_d - p_d)^2 < r^2 (nanoflann's L2 order), skipping
// nodes of its own particle.  Each node's candidates thus come in (cell, node
// index) order.  COUNT writes c_cnt for every node; FILL writes the columns.
// Per-warp staging of the candidate pass, in dynamic shared memory: a chunk
// of neighbourhood entries (position, node, particle) and the state of up to
// kCandCentres centre nodes (position, particle, running count / output slot).
constexpr int kCandChunk = 256;
constexpr int kCandCentres = 64;

template <int DIM>
struct CandWarp {
  double x[DIM][kCandChunk];
  double q[DIM][kCandCentres];
  int64_t out[kCandCentres];
  int32_t j[kCandChunk], p[kCandChunk];
  int32_t ci[kCandCentres], pi[kCandCentres];
  int32_t nb_s[DIM == 3 ? 27 : 9], nb_off[(DIM == 3 ? 27 : 9) + 1];
};

template <int DIM>
constexpr size_t cand_stage_bytes() {
  return sizeof(CandWarp<DIM>) * (kCoopBlock / 32);
}

template <int DIM, int LPN, bool FILL>
__device__ void cand_cells(const DevData &d, uint8_t search_bit, CandWarp<DIM> *stage) {
  constexpr int kWarps = kCoopBlock / 32;
  constexpr int kNb = DIM == 3 ? 27 : 9;
  const int wl = threadIdx.x >> 5, l32 = threadIdx.x & 31;
  CandWarp<DIM> &W = stage[wl];
  const Grid G = d.grid;
  const double r = d.ctrl->radius;
  const double r2 = r * r;
  const int lane = threadIdx.x % LPN;
  const unsigned gm = group_mask<LPN>();
  const unsigned lane_base = (threadIdx.x & 31u) / LPN * LPN;
  constexpr int kGroups = 32 / LPN;
  const int grp = l32 / LPN;
  const int64_t nwarps = (int64_t)gridDim.x * kWarps;
  for (int64_t c = (int64_t)blockIdx.x * kWarps + wl; c < G.ncells; c += nwarps) {
    const int s_c = d.cell_start[c], e_c = d.cell_start[c + 1];
    if (s_c == e_c) continue;  // warp-uniform
    {
      // lane t takes neighbour cell t in traversal order (z, y, x
      // ascending); cells outside the grid contribute no nodes
      const int t = l32;
      const int cx0 = (int)(c % G.dims[0]);
      const int cy0 = (int)((c / G.dims[0]) % G.dims[1]);
      const int cz0 = DIM == 3 ? (int)(c / ((int64_t)G.dims[0] * G.dims[1])) : 0;
      int a = 0, cnt = 0;
      const int32_t pc_cell = d.cell_pid[c];
      if (t < kNb) {
        const int cx = cx0 + t % 3 - 1, cy = cy0 + (t / 3) % 3 - 1, cz = DIM == 3 ? cz0 + t / 9 - 1 : 0;
        if (cx >= 0 && cx < G.dims[0] && cy >= 0 && cy < G.dims[1] && cz >= 0 &&
            cz < (DIM == 3 ? G.dims[2] : 1)) {
          const int cell = cx + G.dims[0] * (cy + G.dims[1] * cz);
          // a centre cell of one particle finds nothing in a neighbour cell
          // of that same particle
          if (pc_cell < 0 || d.cell_pid[cell] != pc_cell) {
            a = d.cell_start[cell];
            cnt = d.cell_start[cell + 1] - a;
          }
        }
      }
      int incl = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (t >= o) incl += y;
      }
      if (t < kNb) {
        W.nb_s[t] = a;
        W.nb_off[t] = incl - cnt;
      }
      if (t == kNb - 1) W.nb_off[kNb] = incl;
    }
    __syncwarp();
    const int total = W.nb_off[kNb];
    if (total == 0) {
      // every neighbour cell culled: no candidate for any node of this cell
      for (int a = s_c + l32; a < e_c; a += 32) d.c_cnt[d.cell_nodes[a]] = 0;
      __syncwarp();  // the warp's stage is reused by the next cell
      continue;
    }
    // centre nodes in sets of up to kCandCentres (one set unless the cell is crowded)
    for (int sb = s_c; sb < e_c; sb += kCandCentres) {
      const int nc = min(kCandCentres, e_c - sb);
      // particle of the centre cell's first node: a chunk whose entries and
      // searching centres all belong to it cannot produce a candidate
      const int32_t pc = d.ptid[d.cell_nodes[sb]];
      bool mixed_centres = false;
      for (int a = l32; a < nc; a += 32) {
        const int32_t i = d.cell_nodes[sb + a];
        const bool search = (d.flags[i] & search_bit) != 0;
        double q[3];
        ldv<DIM>(d.x, i, q);
#pragma unroll
        for (int t = 0; t < DIM; t++) W.q[t][a] = q[t];
        W.ci[a] = i;
        W.pi[a] = search ? d.ptid[i] : -2;  // -2: not searching
        W.out[a] = FILL && search ? d.c_row[i] : 0;
        if (search && W.pi[a] != pc) mixed_centres = true;
      }
      mixed_centres = __any_sync(0xffffffffu, mixed_centres);
      for (int base = 0; base < total; base += kCandChunk) {
        const int n = min(kCandChunk, total - base);
        __syncwarp();  // the previous chunk is no longer read
        for (int a = l32; a < n; a += 32) {
          const int g = base + a;
          int k = 0;
          while (k + 1 < kNb && W.nb_off[k + 1] <= g) k++;
          const int32_t j = d.cell_nodes[W.nb_s[k] + (g - W.nb_off[k])];
          double p[3];
          ldv<DIM>(d.x, j, p);
#pragma unroll
          for (int t = 0; t < DIM; t++) W.x[t][a] = p[t];
          W.j[a] = j;
          W.p[a] = d.ptid[j];
        }
        __syncwarp();
        bool other = mixed_centres;
        for (int a = l32; a < n && !other; a += 32) other = W.p[a] != pc;
        if (!__any_sync(0xffffffffu, other)) continue;  // one particle only: no candidates here
        for (int cb = 0; cb < nc; cb += kGroups) {
          const int cc = cb + grp;
          const int32_t pi = cc < nc ? W.pi[cc] : -2;
          const bool search = pi != -2;
          double q[3] = {0.0, 0.0, 0.0};
          int64_t out = 0, out_end = 0;
          if (search) {
#pragma unroll
            for (int t = 0; t < DIM; t++) q[t] = W.q[t][cc];
            out = W.out[cc];
            if (FILL) out_end = d.c_row[W.ci[cc] + 1];
          }
          for (int b0 = 0; b0 < n; b0 += LPN) {
            const int a = b0 + lane;
            bool hit = false;
            int32_t j = -1;
            if (search && a < n) {
              j = W.j[a];
              if (W.p[a] != pi) {
                double dd = 0.0;
#pragma unroll
                for (int t = 0; t < DIM; t++) {
                  const double df = q[t] - W.x[t][a];
                  dd += df * df;
                }
                hit = dd < r2;
              }
            }
            const unsigned bal = (__ballot_sync(gm, hit) & gm) >> lane_base;
            if (FILL && hit) {
              const int64_t at = out + __popc(bal & ((1u << lane) - 1u));
              if (at < out_end && at < d.contact_cap) d.c_col[at] = j;
            }
            out += __popc(bal);
          }
          __syncwarp(gm);
          if (search && lane == 0) W.out[cc] = out;
        }
      }
      __syncwarp();
      if (!FILL)
        for (int a = l32; a < nc; a += 32) d.c_cnt[W.ci[a]] = W.pi[a] != -2 ? W.out[a] : 0;
    }
    __syncwarp();  // the warp's stage is reused by the next cell
  }
}

// Fill pass over the nodes that have candidates (c_nodes[0, nn)): a warp per
// node walks the same neighbourhood in the same order as the count pass and
// writes the columns.  Lane t first takes neighbour cell t (empty when it
// lies outside the grid or holds only nodes of this node's particle); the
// cells' node ranges, concatenated in traversal order, are then walked 32
// entries at a time, so each entry costs one chain of loads (its node, then
// that node's particle and position) whatever cell it sits in.
template <int DIM>
__device__ void cand_fill_nodes(const DevData &d, int64_t nn) {
  constexpr int kNb = DIM == 3 ? 27 : 9;
  const Grid G = d.grid;
  const double r = d.ctrl->radius;
  const double r2 = r * r;
  const int l32 = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (kCoopBlock / 32);
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nn; t += nwarps) {
    const int32_t i = d.c_nodes[t];
    double q[3];
    ldv<DIM>(d.x, i, q);
    const int32_t pi = d.ptid[i];
    int64_t out = d.c_row[i];
    const int64_t out_end = d.c_row[i + 1];
    for (int64_t e = out + l32; e < out_end && e < d.contact_cap; e += 32) d.c_own[e] = i;
    const int cx0 = cell_coord<DIM>(q[0], G, 0), cy0 = cell_coord<DIM>(q[1], G, 1);
    const int cz0 = DIM == 3 ? cell_coord<DIM>(q[2], G, 2) : 0;
    int a = 0, cnt = 0;
    if (l32 < kNb) {
      const int cx = cx0 + l32 % 3 - 1, cy = cy0 + (l32 / 3) % 3 - 1, cz = DIM == 3 ? cz0 + l32 / 9 - 1 : 0;
      if (cx >= 0 && cx < G.dims[0] && cy >= 0 && cy < G.dims[1] && cz >= 0 && cz < (DIM == 3 ? G.dims[2] : 1)) {
        const int cell = cx + G.dims[0] * (cy + G.dims[1] * cz);
        if (d.cell_pid[cell] != pi) {  // a cell of this node's particle only holds no candidate
          a = d.cell_start[cell];
          cnt = d.cell_start[cell + 1] - a;
        }
      }
    }
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (l32 >= o) incl += y;
    }
    int inc[kNb];
#pragma unroll
    for (int c = 0; c < kNb; c++) inc[c] = __shfl_sync(0xffffffffu, incl, c);
    const int total = inc[kNb - 1];
    for (int base = 0; base < total; base += 32) {
      const int g = base + l32;
      int k = 0;
#pragma unroll
      for (int c = 0; c < kNb; c++) k += inc[c] <= g;
      const int ak = __shfl_sync(0xffffffffu, a, k & 31);
      const int ek = __shfl_sync(0xffffffffu, incl - cnt, k & 31);
      bool hit = false;
      int32_t j = -1;
      if (g < total) {
        j = d.cell_nodes[ak + (g - ek)];
        if (d.ptid[j] != pi) {
          double p[3];
          ldv<DIM>(d.x, j, p);
          double dd = 0.0;
#pragma unroll
          for (int u = 0; u < DIM; u++) {
            const double df = q[u] - p[u];
            dd += df * df;
          }
          hit = dd < r2;
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, hit);
      if (hit) {
        const int64_t at = out + __popc(bal & ((1u << l32) - 1u));
        if (at < out_end && at < d.contact_cap) d.c_col[at] = j;
      }
      out += __popc(bal);
    }
  }
}

// The learned surrogate's list of the tiles the bond loop runs this step:
// those of the particles not on the surrogate (sur_on && !sur_near is the
// test the surrogate's scatter applies).  The order follows the atomic
// claims; each tile's forces do not depend on it.
__device__ void list_live_tiles(const DevData &d) {
  if (!d.tile_live) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < d.n_tile_live_src; t += gridDim.x * blockDim.x) {
    const int p = d.tile_particle[t];
    if (d.sur_on[p] && !d.sur_near[p]) continue;
    const unsigned k = atomicAdd(d.tile_live_n, 1u);
    if (k < (unsigned)d.n_tile_live_src) d.tile_live[k] = t;
  }
}

template <int DIM, int LPN>
__global__ void __launch_bounds__(kCoopBlock) k_contact_rebuild(DevData d, uint8_t search_bit,
                                                               int64_t *bsum) {
  extern __shared__ __align__(16) unsigned char cand_smem[];
  CandWarp<DIM> *stage = reinterpret_cast<CandWarp<DIM> *>(cand_smem);
  if (d.ctrl->error) return;
  if (!d.ctrl->update) {
    list_live_tiles(d);
    return;
  }
  CtrlState *gc = d.ctrl;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // phase clock (profiling): the first CTA's time past each barrier
  int mark = 0;
  auto stamp = [&]() {
    if (d.phase_ns && tid == 0 && mark < kRebuildPhases) d.phase_ns[mark] = global_ns();
    mark++;
  };
  stamp();
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  const int64_t N = d.n_nodes;
  const Grid G = d.grid;
  for (int64_t c = tid; c <= G.ncells; c += nth) {
    d.cell_cnt[c] = 0;
    d.cell_fill[c] = 0;
  }
  if (d.sur_near_gate)
    for (int64_t p = tid; p < d.n_particles; p += nth) d.sur_near[p] = 0;
  if (!grid_bar(gc)) return;
  stamp();
  for (int64_t i = tid; i < N; i += nth) {
    double p[3];
    ldv<DIM>(d.x, i, p);
    const int c = cell_index<DIM>(p, G);
    d.cell_of[i] = c;
    atomicAdd(d.cell_cnt + c, 1);
  }
  if (!grid_bar(gc)) return;
  stamp();
  const int32_t *cc = d.cell_cnt;
  if (!grid_scan<int32_t>(gc, [cc](int64_t k) { return cc[k]; }, d.cell_start, G.ncells, bsum)) return;
  stamp();
  for (int64_t i = tid; i < N; i += nth) {
    const int c = d.cell_of[i];
    d.cell_tmp[d.cell_start[c] + atomicAdd(d.cell_fill + c, 1)] = (int32_t)i;
  }
  if (!grid_bar(gc)) return;
  stamp();
  {
    // per cell: its nodes in index order (rank counting) and, when they all
    // belong to one particle, that particle (no candidate joins two nodes
    // of one particle, so the searches skip a cell of the searching node's
    // own particle)
    const int lane = threadIdx.x & 31;
    for (int64_t c = tid >> 5; c < G.ncells; c += nth >> 5) {
      const int s = d.cell_start[c], e = d.cell_start[c + 1];
      int32_t pmin = INT32_MAX, pmax = -1;
      for (int a = s + lane; a < e; a += 32) {
        const int32_t va = d.cell_tmp[a];
        int rank = 0;
        for (int b = s; b < e; b++) rank += d.cell_tmp[b] < va;
        d.cell_nodes[s + rank] = va;
        const int32_t p = d.ptid[va];
        pmin = min(pmin, p);
        pmax = max(pmax, p);
      }
      for (int o = 16; o > 0; o >>= 1) {
        pmin = min(pmin, __shfl_xor_sync(0xffffffffu, pmin, o));
        pmax = max(pmax, __shfl_xor_sync(0xffffffffu, pmax, o));
      }
      if (lane == 0) d.cell_pid[c] = (e > s && pmin == pmax) ? pmin : -1;
    }
  }
  if (!grid_bar(gc)) return;
  stamp();
  cand_cells<DIM, LPN, false>(d, search_bit, stage);
  if (!grid_bar(gc)) return;
  stamp();
  const int64_t *cn = d.c_cnt;
  if (!grid_scan<int64_t>(gc, [cn](int64_t k) { return cn[k]; }, d.c_row, N, bsum)) return;
  stamp();
  if (!grid_scan<int64_t>(gc, [cn](int64_t k) { return (int64_t)(cn[k] > 0); }, d.c_tmp, N, bsum)) return;
  stamp();
  for (int64_t i = tid; i < N; i += nth)
    if (cn[i] > 0) {
      d.c_nodes[d.c_tmp[i]] = (int32_t)i;
      d.c_span[d.c_tmp[i]] = make_int2((int)d.c_row[i], (int)d.c_row[i + 1]);
      if (d.sur_near_gate) d.sur_near[d.ptid[i]] = 1;  // every writer stores the same value
    }
  if (tid == 0) d.ctrl->c_nnodes = d.c_tmp[N];
  if (!grid_bar(gc)) return;  // the compacted list is complete
  list_live_tiles(d);          // the proximity flags are final
  stamp();
  cand_fill_nodes<DIM>(d, d.c_tmp[N]);
  stamp();  // the first CTA's share of the fill done
  if (tid == 0) {
    const int64_t total = d.c_row[N];
    d.ctrl->entries = total;
    d.ctrl->updates += 1;
    if (total > d.contact_cap) set_error(d.ctrl, DEV_ERR_CONTACT_OVERFLOW, total);
  }
}

// ---------------------------------------------------------------------------
// Distance pass ahead of the contact node pass: one thread per candidate
// entry marks the entries inside the largest contact radius of the zone-pair
// table (R < rc_max; every pair the node pass can accept, is_less(R, rc),
// has R < rc <= rc_max, and R is computed by the same operations there).
// Flat over the entries, so each thread carries one gather chain instead of
// a node's whole candidate row.
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void __launch_bounds__(kBlock) k_contact_near(DevData d) {
  if (d.ctrl->error) return;
  const int64_t E = d.ctrl->entries < d.contact_cap ? d.ctrl->entries : d.contact_cap;
  const double rmax = d.rc_max;
  for (int64_t e = (int64_t)blockIdx.x * kBlock + threadIdx.x; e < E; e += (int64_t)gridDim.x * kBlock) {
    const int32_t i = d.c_own[e], j = d.c_col[e];
    double yi[3], yj[3], yji[3];
    ldv<DIM>(d.x, i, yi);
    ldv<DIM>(d.x, j, yj);
#pragma unroll
    for (int q = 0; q < 3; q++) yji[q] = yj[q] - yi[q];
    d.c_hit[e] = len3<DIM>(yji) < rmax ? 1 : 0;
  }
}

// the node of every candidate entry, from the compacted lists (after a
// state snapshot restores them)
__global__ void k_contact_owner(DevData d) {
  const int64_t nn = d.ctrl->c_nnodes;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nn; t += (int64_t)gridDim.x * blockDim.x) {
    const int32_t i = d.c_nodes[t];
    const int2 sp = d.c_span[t];
    for (int64_t e = sp.x; e < sp.y && e < d.contact_cap; e++) d.c_own[e] = i;
  }
}

// ---------------------------------------------------------------------------
// Node pass of DEMModel::computeContactForces (demModel.cpp:832-934):
// penalty normal force + Coulomb-type friction for candidates inside the
// zone-pair contact radius; f_i += sum.  Particle-wall pairs inside the
// contact radius are recorded for the particle-wall damping (:994-1017),
// and the test wall's contact reaction is summed per block.
// ---------------------------------------------------------------------------
constexpr int kZonePairsSmem = 256;

// Every load a candidate needs is issued together: the compacted node and
// its candidate span (speculatively, before the node count arrives), then the
// node's own data with its candidate columns, then all of each candidate's
// data at once; the zone-pair table sits in shared memory.  The first
// threads also gather the particle centres for the damping pass.
template <int DIM, int LPN>
__global__ void __launch_bounds__(kBlock) k_contact(DevData d) {
  __shared__ ContactPair cps[kZonePairsSmem];
  __shared__ double scr[kBlock / LPN];
  const int lane = threadIdx.x % LPN;
  const int nz = d.n_zones;
  const bool tab = nz * nz <= kZonePairsSmem;
  const int64_t gstride = (int64_t)gridDim.x * (kBlock / LPN);
  int64_t t = (int64_t)blockIdx.x * (kBlock / LPN) + threadIdx.x / LPN;
  int32_t i_next = t < d.n_nodes ? d.c_nodes[t] : 0;
  int2 sp_next = t < d.n_nodes ? d.c_span[t] : make_int2(0, 0);
  const int64_t nn_raw = d.ctrl->c_nnodes;
  const int err = d.ctrl->error;
  if (tab)
    for (int a = threadIdx.x; a < nz * nz; a += kBlock) cps[a] = d.contact[a];
  {
    // particle centres (position, velocity) of this step for the damping pass
    for (int64_t p = (int64_t)blockIdx.x * kBlock + threadIdx.x; p < d.n_particles;
         p += (int64_t)gridDim.x * kBlock) {
      const int64_t c = d.particles[p].center;
      double xc[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
      ldv<DIM>(d.x, c, xc);
      ldv<DIM>(d.v, c, vc);
      double *o = d.pcen + 8 * p;  // {x, y, z, bounding radius, vx, vy, vz, -}
#pragma unroll
      for (int q = 0; q < 3; q++) {
        o[q] = xc[q];
        o[4 + q] = vc[q];
      }
      o[3] = d.dpart[p].bound_r;
      d.pcen32[p] = make_float4((float)xc[0], (float)xc[1], (float)xc[2], (float)o[3]);
    }
  }
  __syncthreads();
  const int64_t nn = err ? 0 : nn_raw;
  double crd_acc = 0.0;
  for (; t < nn; t += gstride) {
    const int64_t i = i_next;
    const int2 sp = sp_next;
    if (t + gstride < nn) {
      i_next = d.c_nodes[t + gstride];
      sp_next = d.c_span[t + gstride];
    }
    const unsigned gm = group_mask<LPN>();
    const int32_t pi = d.ptid[i];
    const int zi = d.nzone[i];
    double yi[3], vi[3];
    ldv<DIM>(d.x, i, yi);
    ldv<DIM>(d.v, i, vi);
    double fx = 0.0, fy = 0.0, fz = 0.0, crd = 0.0;
    for (int k = sp.x + lane; k < sp.y; k += LPN) {
      // most candidates lie in the search skin, beyond every zone pair's
      // contact radius: k_contact_near marked the others
      if (!d.c_hit[k]) continue;
      const int32_t j = d.c_col[k];
      double yj[3];
      ldv<DIM>(d.x, j, yj);
      double yji[3];
#pragma unroll
      for (int q = 0; q < 3; q++) yji[q] = yj[q] - yi[q];
      const double R = len3<DIM>(yji);
      double vj[3];
      ldv<DIM>(d.v, j, vj);
      const double volj = d.vol[j];
      const int32_t pj = d.ptid[j];
      const int zj = d.nzone[j];
      const bool wall = (d.flags[j] & NODE_WALL) != 0;
      const ContactPair cp = tab ? cps[zi * nz + zj] : d.contact[zi * nz + zj];
      if (is_less(R, cp.rc)) {
        double vji[3], en[3], et[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
          vji[q] = vj[q] - vi[q];
          en[q] = yji[q] / R;
        }
        const double vn = dot3<DIM>(vji, en);
#pragma unroll
        for (int q = 0; q < 3; q++) et[q] = vji[q] - vn * en[q];
        const double etl = len3<DIM>(et);
        if (is_greater(etl, 0.)) {
#pragma unroll
          for (int q = 0; q < 3; q++) et[q] = et[q] / etl;
        } else {
          et[0] = et[1] = et[2] = 0.0;
        }
        double sf = cp.kn * (R - cp.rc) * volj;
        if (sf > 0.) sf = 0.;
        const double mf = cp.mu * sf;
        const double cx = sf * en[0], cy = sf * en[1], cz = sf * en[2];
        fx += cx;
        fy += cy;
        if constexpr (DIM == 3) fz += cz;
        fx += mf * et[0];
        fy += mf * et[1];
        if constexpr (DIM == 3) fz += mf * et[2];
        if (wall) {
          const int slot = atomicAdd(d.wp_cnt + pi, 1);
          if (slot < d.wp_cap) d.wp[(int64_t)pi * d.wp_cap + slot] = j;
          else set_error(d.ctrl, DEV_ERR_WALLPAIR_OVERFLOW, pi);
        }
        if (d.pwall_test ? d.pwall_test[pj] != 0 : pj == d.test_wall) {
          const int td = d.test_dir;
          crd += td == 0 ? cx + mf * et[0] : (td == 1 ? cy + mf * et[1] : cz + mf * et[2]);
        }
      }
    }
    fx = group_sum<LPN>(fx, gm);
    fy = group_sum<LPN>(fy, gm);
    if constexpr (DIM == 3) fz = group_sum<LPN>(fz, gm);
    crd = group_sum<LPN>(crd, gm);
    if (lane == 0) {
      const double f[3] = {fx, fy, fz};
      stv<DIM>(d.fc, i, f);
      crd_acc += crd * d.vol[i];
      if (d.cr_t) d.cr_t[t] = crd * d.vol[i];
    }
  }
  // deterministic per-block partial of the test wall's contact reaction
  if (lane == 0) scr[threadIdx.x / LPN] = crd_acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int g = 0; g < kBlock / LPN; g++) sum += scr[g];
    d.cr_partial[blockIdx.x] = sum;
  }
}

// ---------------------------------------------------------------------------
// The contact node pass in one kernel, warp-cooperative (the default, one
// lane per node): a warp takes 32 consecutive compacted nodes, whose
// candidate rows are consecutive in the entry array, and walks their
// entries 32 at a time, coalesced.  Each lane finds its entry's node among
// the warp's (binary search over the row starts, held one per lane), takes
// that node's position and velocity by shuffle, and reads only the
// candidate's position unless the pair is inside the largest contact
// radius.  The rare contributions are then handed, in entry order, to the
// lane that owns the node, which adds them in the reference's order (normal
// part, then friction part, candidate by candidate).  Results equal the
// node pass with one lane per node.
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void __launch_bounds__(kBlock) k_contact_warp(DevData d) {
  __shared__ ContactPair cps[kZonePairsSmem];
  __shared__ double scr[kBlock];
  const int l32 = threadIdx.x & 31;
  const int nz = d.n_zones;
  const bool tab = nz * nz <= kZonePairsSmem;
  const int64_t nn_raw = d.ctrl->c_nnodes;
  const int err = d.ctrl->error;
  if (tab)
    for (int a = threadIdx.x; a < nz * nz; a += kBlock) cps[a] = d.contact[a];
  for (int64_t p = (int64_t)blockIdx.x * kBlock + threadIdx.x; p < d.n_particles; p += (int64_t)gridDim.x * kBlock) {
    // particle centres (position, velocity) of this step for the damping pass
    const int64_t c = d.particles[p].center;
    double xc[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
    ldv<DIM>(d.x, c, xc);
    ldv<DIM>(d.v, c, vc);
    // record {x, y, z, bounding radius, vx, vy, vz, -}: the damping pass's
    // pair search reads only the first 32 bytes
    double *o = d.pcen + 8 * p;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      o[q] = xc[q];
      o[4 + q] = vc[q];
    }
    o[3] = d.dpart[p].bound_r;
    d.pcen32[p] = make_float4((float)xc[0], (float)xc[1], (float)xc[2], (float)o[3]);
  }
  __syncthreads();
  const int64_t nn = err ? 0 : nn_raw;
  const double rmax = d.rc_max;
  const int64_t nwarps = (int64_t)gridDim.x * (kBlock / 32);
  double crd_acc = 0.0;
  for (int64_t w = ((int64_t)blockIdx.x * kBlock + threadIdx.x) >> 5; w * 32 < nn; w += nwarps) {
    const int64_t t = w * 32 + l32;
    const bool own = t < nn;
    const int nval = (int)min((int64_t)32, nn - w * 32);  // lanes with a node
    int32_t i = 0;
    int2 sp = make_int2(0, 0);
    double yi[3] = {0, 0, 0}, vi[3] = {0, 0, 0};
    int32_t pi = -1;
    int zi = 0;
    if (own) {
      i = d.c_nodes[t];
      sp = d.c_span[t];
      pi = d.ptid[i];
      zi = d.nzone[i];
      ldv<DIM>(d.x, i, yi);
      ldv<DIM>(d.v, i, vi);
    }
    const int e0 = __shfl_sync(0xffffffffu, sp.x, 0);
    const int e1 = __shfl_sync(0xffffffffu, sp.y, nval - 1);
    double fx = 0.0, fy = 0.0, fz = 0.0, crd = 0.0;
    for (int base = e0; base < e1; base += 32) {
      const int e = base + l32;
      // the entry's node: the last lane whose row starts at or before e
      int o = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int cnd = o + step;
        const int st = __shfl_sync(0xffffffffu, sp.x, cnd & 31);
        if (cnd < nval && st <= e) o = cnd;
      }
      double yo[3], vo[3];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        yo[q] = __shfl_sync(0xffffffffu, yi[q], o);
        vo[q] = __shfl_sync(0xffffffffu, vi[q], o);
      }
      const int32_t po = __shfl_sync(0xffffffffu, pi, o);
      const int zo = __shfl_sync(0xffffffffu, zi, o);
      double cxn = 0.0, cyn = 0.0, czn = 0.0, cxt = 0.0, cyt = 0.0, czt = 0.0, cr = 0.0;
      bool contrib = false;
      if (e < e1) {
        const int32_t j = d.c_col[e];
        double yj[3];
        ldv<DIM>(d.x, j, yj);
        double yji[3];
#pragma unroll
        for (int q = 0; q < 3; q++) yji[q] = yj[q] - yo[q];
        const double R = len3<DIM>(yji);
        if (R < rmax) {
          double vj[3];
          ldv<DIM>(d.v, j, vj);
          const double volj = d.vol[j];
          const int32_t pj = d.ptid[j];
          const int zj = d.nzone[j];
          const bool wall = (d.flags[j] & NODE_WALL) != 0;
          const ContactPair cp = tab ? cps[zo * nz + zj] : d.contact[zo * nz + zj];
          if (is_less(R, cp.rc)) {
            double vji[3], en[3], et[3];
#pragma unroll
            for (int q = 0; q < 3; q++) {
              vji[q] = vj[q] - vo[q];
              en[q] = yji[q] / R;
            }
            const double vn = dot3<DIM>(vji, en);
#pragma unroll
            for (int q = 0; q < 3; q++) et[q] = vji[q] - vn * en[q];
            const double etl = len3<DIM>(et);
            if (is_greater(etl, 0.)) {
#pragma unroll
              for (int q = 0; q < 3; q++) et[q] = et[q] / etl;
            } else {
              et[0] = et[1] = et[2] = 0.0;
            }
            double sf = cp.kn * (R - cp.rc) * volj;
            if (sf > 0.) sf = 0.;
            const double mf = cp.mu * sf;
            cxn = sf * en[0];
            cyn = sf * en[1];
            czn = sf * en[2];
            cxt = mf * et[0];
            cyt = mf * et[1];
            czt = mf * et[2];
            contrib = true;
            if (wall) {
              const int slot = atomicAdd(d.wp_cnt + po, 1);
              if (slot < d.wp_cap) d.wp[(int64_t)po * d.wp_cap + slot] = j;
              else set_error(d.ctrl, DEV_ERR_WALLPAIR_OVERFLOW, po);
            }
            if (d.pwall_test ? d.pwall_test[pj] != 0 : pj == d.test_wall) {
              const int td = d.test_dir;
              cr = td == 0 ? cxn + cxt : (td == 1 ? cyn + cyt : czn + czt);
            } else {
              cr = -0.0;  // marks "no test-wall term" (never added)
            }
          }
        }
      }
      // hand the contributions to their nodes' lanes in entry order
      unsigned m = __ballot_sync(0xffffffffu, contrib);
      while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        const int dst = __shfl_sync(0xffffffffu, o, src);
        const double ax = __shfl_sync(0xffffffffu, cxn, src), ay = __shfl_sync(0xffffffffu, cyn, src);
        const double bx = __shfl_sync(0xffffffffu, cxt, src), by = __shfl_sync(0xffffffffu, cyt, src);
        const double c = __shfl_sync(0xffffffffu, cr, src);
        double az = 0.0, bz = 0.0;
        if constexpr (DIM == 3) {
          az = __shfl_sync(0xffffffffu, czn, src);
          bz = __shfl_sync(0xffffffffu, czt, src);
        }
        if (l32 == dst) {
          fx += ax;
          fy += ay;
          if constexpr (DIM == 3) fz += az;
          fx += bx;
          fy += by;
          if constexpr (DIM == 3) fz += bz;
          if (!(c == 0.0 && signbit(c))) crd += c;
        }
      }
    }
    if (own) {
      if (fx != 0.0 || fy != 0.0 || (DIM == 3 && fz != 0.0)) {
        const double f[3] = {fx, fy, fz};
        stv<DIM>(d.fc, i, f);
      }
      crd_acc += crd * d.vol[i];
      if (d.cr_t) d.cr_t[t] = crd * d.vol[i];
    }
  }
  // deterministic per-block partial of the test wall's contact reaction
  scr[threadIdx.x] = crd_acc;
  __syncthreads();
  for (int h = kBlock / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) scr[threadIdx.x] += scr[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) d.cr_partial[blockIdx.x] = scr[0];
}

// ---------------------------------------------------------------------------
// Particle damping of DEMModel::computeContactForces (demModel.cpp:937-1050):
// particle-particle through particle centres and particle-wall through the
// condensed wall nodes.  One block per particle; the force density is applied
// to all nodes of the particle by k_external.
// ---------------------------------------------------------------------------
constexpr int kDampBlock = 128;
constexpr int kWallSort = 4096;

// One CTA per group of up to kDampGroup consecutive particles of one scene
// (d.damp_group; one particle per CTA without it): each particle record
// loaded in the particle-particle loop serves the whole group.  A thread
// visits the same particles q in the same order for every member as the
// one-particle form, and keeps a partial sum per member and component in
// shared memory, so the sums are those of the one-particle form bit for bit.
__global__ void __launch_bounds__(kDampBlock) k_damping(DevData d, int dim) {
  __shared__ int32_t wn[kWallSort];
  __shared__ double red[3][kDampBlock / 32];
  __shared__ ContactPair cps[kZonePairsSmem];
  __shared__ double s_acc[kDampGroup][3][kDampBlock];  // member, component, thread
  __shared__ double s_c[kDampGroup][8];                // centre (3), centre velocity (3), radius, density
  __shared__ int s_zone[kDampGroup], s_type[kDampGroup];
  __shared__ float4 s_cf[kDampGroup];                  // FP32 centre and radius
  const int p0 = d.damp_group ? d.damp_group[blockIdx.x] : (int)blockIdx.x;
  const int np = d.damp_group ? d.damp_group[blockIdx.x + 1] - p0 : 1;
  const int nz = d.n_zones;
  const bool tab = nz * nz <= kZonePairsSmem;
  if (tab)
    for (int a = threadIdx.x; a < nz * nz; a += blockDim.x) cps[a] = d.contact[a];
  if ((int)threadIdx.x < np) {
    const int p = p0 + threadIdx.x;
    const DampParticle P = d.dpart[p];
    for (int q = 0; q < 3; q++) {
      s_c[threadIdx.x][q] = d.pcen[8 * p + q];
      s_c[threadIdx.x][3 + q] = d.pcen[8 * p + 4 + q];
    }
    s_c[threadIdx.x][6] = P.bound_r;
    s_c[threadIdx.x][7] = P.density;
    s_cf[threadIdx.x] = d.pcen32[p];
    s_zone[threadIdx.x] = P.zone;
    s_type[threadIdx.x] = P.type;
  }
  for (int e = threadIdx.x; e < kDampGroup * 3 * kDampBlock; e += blockDim.x) (&s_acc[0][0][0])[e] = 0.0;
  __syncthreads();
  bool any = false;
  for (int k = 0; k < np; k++) any |= s_type[k] == 0;
  if (!any) return;
  if (d.ctrl->error) return;
  const DampParticle G = d.dpart[p0];  // the group's scene: its particles q0 .. q1 - 1
  // particle-particle, over the particles of the scene: first the 16-byte
  // FP32 {centre, radius} record, against the largest reach any zone pair
  // allows with a 10 % margin over the FP64 test below (coordinates rounded
  // to FP32 move a distance by far less), so that only pairs that test can
  // pass read the FP64 record; kDampBatch records in flight per thread, each
  // thread visiting its particles in increasing order
  constexpr int kDampBatch = 4;
  const float rc_f = (float)(1.01 * d.rc_max);
  for (int qb = G.q0 + threadIdx.x; qb < G.q1; qb += kDampBatch * blockDim.x) {
    float4 cf[kDampBatch];
#pragma unroll
    for (int t = 0; t < kDampBatch; t++) {
      const int q = qb + t * (int)blockDim.x;
      cf[t] = q < G.q1 ? d.pcen32[q] : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int t = 0; t < kDampBatch; t++) {
      const int q = qb + t * (int)blockDim.x;
      if (q >= G.q1) continue;
      for (int k = 0; k < np; k++) {
        if (s_type[k] != 0 || q == p0 + k) continue;
        const float4 pf = s_cf[k];
        const float ex = cf[t].x - pf.x, ey = cf[t].y - pf.y, ez = cf[t].z - pf.z;
        const float rm = cf[t].w + pf.w + rc_f;
        if (ex * ex + ey * ey + ez * ez > 1.17f * rm * rm) continue;
        const double2 c01 = *reinterpret_cast<const double2 *>(d.pcen + 8 * q);
        const double2 c2r = *reinterpret_cast<const double2 *>(d.pcen + 8 * q + 2);
        const double *C = s_c[k];
        const double Ri = C[6];
        double xcj[3] = {c01.x - C[0], c01.y - C[1], c2r.x - C[2]};
        const double d2 = xcj[0] * xcj[0] + xcj[1] * xcj[1] + xcj[2] * xcj[2];
        const double reach_max = c2r.y + Ri + 1.01 * d.rc_max;
        if (d2 > 1.0625 * reach_max * reach_max) continue;
        const DampParticle Q = d.dpart[q];
        if (Q.type != 0) continue;
        const double Rj = Q.bound_r;
        double vcj[3];
        for (int c = 0; c < 3; c++) vcj[c] = d.pcen[8 * q + 4 + c] - C[3 + c];
        const ContactPair cp = tab ? cps[s_zone[k] * nz + Q.zone] : d.contact[s_zone[k] * nz + Q.zone];
        const double reach = Rj + Ri + 1.01 * cp.rc;
        // pairs well beyond the reach cannot pass the relative-tolerance test
        if (d2 > 1.0625 * reach * reach) continue;
        const double dist = sqrt(d2);
        if (is_less(dist, reach)) {
          const double vol_pi = kPi * Ri * Ri;
          const double vol_pj = kPi * Rj * Rj;
          const double m1 = C[7] * vol_pi, m2 = Q.density * vol_pj;
          const double meq = 2. * m1 * m2 / (m1 + m2);  // util::equivalentMass
          const double bn = cp.betan * sqrt(cp.kappa * cp.rc * meq);
          double hat[3] = {0.0, 0.0, 0.0};
          if (is_greater(dist, 0.))
            for (int c = 0; c < 3; c++) hat[c] = xcj[c] / dist;
          double vm = vcj[0] * hat[0] + vcj[1] * hat[1] + vcj[2] * hat[2];
          if (vm > 0.) vm = 0.;
          for (int c = 0; c < 3; c++) s_acc[k][c][threadIdx.x] += bn * vm * hat[c] / vol_pi;
        }
      }
    }
  }
  // per member: particle-wall (unique wall nodes within the contact radius
  // of any node), then the block reduction
  const int st = dim == 2 ? 2 : 4;
  for (int k = 0; k < np; k++) {
    if (s_type[k] != 0) continue;  // uniform over the CTA
    const int p = p0 + k;
    const double *C = s_c[k];
    const double Ri = C[6], vol_pi = kPi * Ri * Ri, rhoi = C[7];
    int nw = d.wp_cnt[p];
    if (nw > d.wp_cap) nw = d.wp_cap;
    if (nw > kWallSort) nw = kWallSort;  // capacity is validated on the host
    int sz = 1;
    while (sz < nw) sz <<= 1;
    for (int a = threadIdx.x; a < sz; a += blockDim.x)
      wn[a] = a < nw ? d.wp[(int64_t)p * d.wp_cap + a] : INT32_MAX;
    __syncthreads();
    for (int kk = 2; kk <= sz; kk <<= 1)
      for (int jj = kk >> 1; jj > 0; jj >>= 1) {
        for (int a = threadIdx.x; a < sz; a += blockDim.x) {
          const int b = a ^ jj;
          if (b > a) {
            const bool up = (a & kk) == 0;
            const int32_t va = wn[a], vb = wn[b];
            if ((va > vb) == up) {
              wn[a] = vb;
              wn[b] = va;
            }
          }
        }
        __syncthreads();
      }
    double acc[3] = {s_acc[k][0][threadIdx.x], s_acc[k][1][threadIdx.x], s_acc[k][2][threadIdx.x]};
    for (int a = threadIdx.x; a < nw; a += blockDim.x) {
      const int32_t w = wn[a];
      if (a > 0 && wn[a - 1] == w) continue;
      const int zk = d.nzone[w];
      const ContactPair cp = tab ? cps[s_zone[k] * nz + zk] : d.contact[s_zone[k] * nz + zk];
      const double meq = rhoi * vol_pi;
      const double bn = cp.betan * sqrt(cp.kappa * cp.rc * meq);
      double xk[3] = {0, 0, 0}, vk[3] = {0, 0, 0};
      for (int t = 0; t < dim; t++) {
        xk[t] = d.x[st * (int64_t)w + t] - C[t];
        vk[t] = d.v[st * (int64_t)w + t] - C[3 + t];
      }
      const double l = sqrt(xk[0] * xk[0] + xk[1] * xk[1] + xk[2] * xk[2]);
      double hat[3] = {0.0, 0.0, 0.0};
      if (is_greater(l, 0.))
        for (int t = 0; t < 3; t++) hat[t] = xk[t] / l;
      double vm = vk[0] * hat[0] + vk[1] * hat[1] + vk[2] * hat[2];
      if (vm > 0.) vm = 0.;
      for (int t = 0; t < 3; t++) acc[t] += bn * vm * hat[t] / vol_pi;
    }
    // block reduction (fixed order)
    for (int t = 0; t < 3; t++) {
      double v = acc[t];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if ((threadIdx.x & 31) == 0) red[t][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int t = 0; t < 3; t++) {
        double s = 0.0;
        for (int w = 0; w < kDampBlock / 32; w++) s += red[t][w];
        d.fdamp[4 * p + t] = s;
      }
      d.wp_cnt[p] = 0;
    }
    __syncthreads();  // before wn and red are reused
  }
}

// ---------------------------------------------------------------------------
// Damping force to all nodes of each particle (demModel.cpp:1053-1064), then
// DEMModel::computeExternalForces (:791-812): gravity, then force BCs
// (ParticleFLoading::apply, particleFLoading.cpp:85-173).
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void k_external(DevData d) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_nodes || d.ctrl->error) return;
  // nodes outside d_fPdCompNodes carry no peridynamic or contact force: the
  // reference zeroes f for all nodes at the start of computeForces (:473-478)
  double f[3] = {0.0, 0.0, 0.0};
  const uint8_t fl = d.flags[i];
  if (fl & NODE_ACTIVE) {
    ldv<DIM>(d.f, i, f);
    // contact forces (computeContactForces adds them after the bond loop);
    // only searching nodes can carry one
    if (d.fc && (fl & (NODE_SEARCH | NODE_SEARCH0))) {
      double c[3];
      ldv<DIM>(d.fc, i, c);
      if (c[0] != 0.0 || c[1] != 0.0 || (DIM == 3 && c[2] != 0.0)) {
#pragma unroll
        for (int q = 0; q < DIM; q++) f[q] += c[q];
        const double z[3] = {0.0, 0.0, 0.0};
        stv<DIM>(d.fc, i, z);
      }
    }
  }
  const int32_t p = d.ptid[i];
  if (d.flags[i] & NODE_PARTICLE) {
#pragma unroll
    for (int q = 0; q < DIM; q++) f[q] += d.fdamp[4 * p + q];
  }
  if (d.gravity_on) {
    const double rho = d.particles[p].density;
#pragma unroll
    for (int q = 0; q < DIM; q++) f[q] += rho * d.gravity[q];
  }
  stv<DIM>(d.f, i, f);
}

template <int DIM>
__device__ __noinline__ void apply_fbc(const DevData &d, int t, double time, double (&f)[3]) {
  for (int e = d.fbc_row[t]; e < d.fbc_row[t + 1]; e++) {
    const BcSetDev bc = d.fbc_sets[d.fbc_set[e]];
    double fmax = d.fbc_val[e];
    switch (bc.time_fn) {
      case PDGPU_TIME_LINEAR: fmax *= time; break;
      case PDGPU_TIME_LINEAR_STEP: {
        // util::linearStepFunc (function.cpp:62-85)
        const double x1 = bc.tp[1], x2 = bc.tp[2];
        const double period = floor(time / (x1 + x2));
        const double val =
            is_less(time, period * (x1 + x2) + x1) ? time - period * x2 : (period + 1.) * x1;
        fmax *= val;
        break;
      }
      case PDGPU_TIME_LINEAR_SLOW_FAST:
        if (is_greater(time, bc.tp[1])) fmax *= bc.tp[3] * time;
        else fmax *= bc.tp[2] * time;
        break;
      case PDGPU_TIME_SIN: fmax *= sin(kPi * bc.tp[1] * time); break;
      default: break;
    }
    fmax *= bc.tp[0];
    for (int q = 0; q < DIM; q++)
      if ((bc.dir_mask >> q) & 1) f[q] += fmax;
  }
}

template <int DIM>
__global__ void k_force_bc(const __grid_constant__ DevData d) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.n_fbc_nodes || d.ctrl->error) return;
  const int64_t i = d.fbc_node[t];
  double f[3];
  ldv<DIM>(d.f, i, f);
  apply_fbc<DIM>(d, t, d.ctrl->time, f);
  stv<DIM>(d.f, i, f);
}

// ---------------------------------------------------------------------------
// Post-processing every test_interval steps: DEMModel::ppCompressiveTest
// (demModel.cpp:2202-2250) or ppTwoParticleTest (:2096-2149).
// ---------------------------------------------------------------------------
// The test's post-processing (demModel.cpp ppCompressiveTest / ppTwoParticleTest)
// run by one 1024-thread block; forces of the current step are read past L1,
// since other CTAs of the same kernel may have written them.
template <int DIM>
__device__ __noinline__ void postprocess_block(const DevData &d) {
  // sums are formed as by a 1024-thread block (per-thread strided partials,
  // warp butterflies, then the 32 warp sums in order), whatever blockDim is
  constexpr int kV = 1024;
  __shared__ double red[2][kV / 32];
  CtrlState *c = d.ctrl;
  if (c->error) return;
  const int64_t n = c->n;
  if (!(n % d.test_interval == 0 && n >= d.test_interval)) return;
  const int st = DIM == 2 ? 2 : 4;
  if (d.test == PDGPU_TEST_COMPRESSIVE) {
    const DevParticle W = d.particles[d.test_wall];
    const int dir = d.test_dir;
    for (int vt = threadIdx.x; vt < kV; vt += blockDim.x) {
      double s = 0.0;
      for (int64_t i = W.start + vt; i < W.end; i += kV) s += __ldcg(d.f + st * i + dir) * d.vol[i];
      double cr = 0.0;
      for (int b = vt; b < d.cr_blocks; b += kV) cr += d.cr_partial[b];
      for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        cr += __shfl_xor_sync(0xffffffffu, cr, o);
      }
      if ((vt & 31) == 0) {
        red[0][vt >> 5] = s;
        red[1][vt >> 5] = cr;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double rs = 0.0, rc = 0.0;
      for (int w = 0; w < kV / 32; w++) {
        rs += red[0][w];
        rc += red[1][w];
      }
      const double delta = d.x[st * W.start + dir] - d.xref[st * W.start + dir];
      c->reaction = rs;
      c->contact_reaction = -rc;
      c->penetration = delta;
      const int64_t h = c->history_count;
      if (h < d.history_cap) {
        d.history[4 * h] = c->time;
        d.history[4 * h + 1] = delta;
        d.history[4 * h + 2] = rs;
        d.history[4 * h + 3] = -rc;
      }
      c->history_count = h + 1;
    }
  } else if (d.test == PDGPU_TEST_TWO_PARTICLE && d.n_particles >= 2) {
    const DevParticle P0 = d.particles[0], P1 = d.particles[1];
    for (int vt = threadIdx.x; vt < kV; vt += blockDim.x) {
      double m = -DBL_MAX;
      for (int64_t i = P1.start + vt; i < P1.end; i += kV) m = fmax(m, d.x[st * i + 1]);
      for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      if ((vt & 31) == 0) red[0][vt >> 5] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double my = -DBL_MAX;
      for (int w = 0; w < kV / 32; w++) my = fmax(my, red[0][w]);
      double dx[3] = {0, 0, 0};
      for (int q = 0; q < DIM; q++) dx[q] = d.x[st * P1.center + q] - d.x[st * P0.center + q];
      const double r = P0.bound_r;
      const ContactPair cp = d.contact[P0.zone * d.n_zones + P1.zone];
      const double re = r + cp.rc;
      double pen = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]) - re - r;
      double car = 0.0;
      if (is_less(pen, 0.)) car = sqrt(re * re - (re + pen) * (re + pen));
      else if (is_greater(pen, 0.)) {
        pen = 0.;
        car = 0.;
      }
      c->pen_dist = pen;
      c->contact_area_radius = car;
      c->max_y = is_less(0.0, my) ? my : 0.0;
    }
  }
}

// Compressive-test output of every scene of a batched ensemble, one CTA per
// scene (the single-scene form is postprocess_block): the test wall's
// reaction sum f vol over its nodes, the contact reaction summed over the
// scene's run of the compacted contact nodes (ascending node ids, so each
// scene's nodes form one run), and the wall's displacement.
template <int DIM>
__global__ void __launch_bounds__(256) k_scene_post(const __grid_constant__ DevData d) {
  __shared__ double red[2][8];
  __shared__ int64_t range[2];
  const CtrlState *c = d.ctrl;
  if (c->error) return;
  const int64_t n = c->n;
  if (!(n % d.test_interval == 0 && n >= d.test_interval)) return;
  const int64_t h = n / d.test_interval - 1;
  const int s = blockIdx.x;
  if (h >= d.scene_hist_cap || s >= d.n_scenes || d.scene_wall[s] < 0) return;
  const int st = DIM == 2 ? 2 : 4;
  const DevParticle W = d.particles[d.scene_wall[s]];
  const int dir = d.test_dir;
  const int64_t nn = c->c_nnodes;
  if (threadIdx.x < 2) {
    const int64_t key = d.scene_node[s + threadIdx.x];
    int64_t lo = 0, hi = nn;  // first compacted index whose node is >= key
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (d.c_nodes[mid] < key) lo = mid + 1;
      else hi = mid;
    }
    range[threadIdx.x] = lo;
  }
  __syncthreads();
  double rs = 0.0, rc = 0.0;
  for (int64_t i = W.start + threadIdx.x; i < W.end; i += blockDim.x) rs += d.f[st * i + dir] * d.vol[i];
  for (int64_t t = range[0] + threadIdx.x; t < range[1]; t += blockDim.x) rc += d.cr_t[t];
  for (int o = 16; o > 0; o >>= 1) {
    rs += __shfl_xor_sync(0xffffffffu, rs, o);
    rc += __shfl_xor_sync(0xffffffffu, rc, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = rs;
    red[1][threadIdx.x >> 5] = rc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < 8; w++) {
      a += red[0][w];
      b += red[1][w];
    }
    double *o = d.scene_hist + 4 * ((int64_t)s * d.scene_hist_cap + h);
    o[0] = c->time;
    o[1] = d.x[st * W.start + dir] - d.xref[st * W.start + dir];
    o[2] = a;
    o[3] = -b;
  }
}

template <int DIM>
__global__ void __launch_bounds__(1024) k_postprocess(const __grid_constant__ DevData d) {
  postprocess_block<DIM>(d);
}

// ---------------------------------------------------------------------------
// Last kernel of a step: per node, the external-force pass
// (as k_external: bond forces, then contact forces, damping, gravity), the
// force BC (as k_force_bc) and, for velocity Verlet, the second half kick (as
// k_verlet_second); then the last CTA to finish runs the post-processing (as
// k_postprocess) when `post` is set.
// ---------------------------------------------------------------------------
constexpr int kEndNodes = 2;  // nodes per thread of the step-end kernel

template <int DIM, bool VERLET>
__global__ void __launch_bounds__(kBlock) k_step_end(const __grid_constant__ DevData d, int post) {
  __shared__ int last;
  const int64_t n_step = d.ctrl->n;
  // each thread takes kEndNodes nodes, kBlock apart, and issues the node
  // loads of all of them (independent of their flags) before the sums
  const int64_t base = (int64_t)blockIdx.x * (kBlock * kEndNodes) + threadIdx.x;
  if (!d.ctrl->error) {
    uint8_t fl[kEndNodes];
    int32_t pid[kEndNodes];
    double fa[kEndNodes][3];
#pragma unroll
    for (int k = 0; k < kEndNodes; k++) {
      const int64_t i = base + (int64_t)k * kBlock;
      fl[k] = 0;
      pid[k] = 0;
      if (i < d.n_nodes) {
        fl[k] = d.flags[i];
        pid[k] = d.ptid[i];
        ldv<DIM>(d.f, i, fa[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < kEndNodes; k++) {
      const int64_t i = base + (int64_t)k * kBlock;
      if (i >= d.n_nodes) continue;
      const int32_t p = pid[k];
      double f[3] = {0.0, 0.0, 0.0};
      // the contact force only where the node searches (elsewhere it is never
      // written and its lines are cold)
      if (fl[k] & NODE_ACTIVE) {
#pragma unroll
        for (int q = 0; q < DIM; q++) f[q] = fa[k][q];
        if (d.fc && (fl[k] & (NODE_SEARCH | NODE_SEARCH0))) {
          double c[3];
          ldv<DIM>(d.fc, i, c);
          if (c[0] != 0.0 || c[1] != 0.0 || (DIM == 3 && c[2] != 0.0)) {
#pragma unroll
            for (int q = 0; q < DIM; q++) f[q] += c[q];
            const double z[3] = {0.0, 0.0, 0.0};
            stv<DIM>(d.fc, i, z);
          }
        }
      }
      if (fl[k] & NODE_PARTICLE) {
#pragma unroll
        for (int q = 0; q < DIM; q++) f[q] += d.fdamp[4 * p + q];
      }
      double rho = 0.0;
      if (d.gravity_on || (VERLET && (fl[k] & NODE_ACTIVE))) rho = d.particles[p].density;
      if (d.gravity_on) {
#pragma unroll
        for (int q = 0; q < DIM; q++) f[q] += rho * d.gravity[q];
      }
      if (fl[k] & NODE_FBC) {  // through a copy, so that f stays in registers
        double fb[3] = {f[0], f[1], f[2]};
        apply_fbc<DIM>(d, d.fbc_of[i], d.ctrl->time, fb);
#pragma unroll
        for (int q = 0; q < 3; q++) f[q] = fb[q];
      }
      stv<DIM>(d.f, i, f);
      if (VERLET && (fl[k] & NODE_ACTIVE)) {
        const uint8_t fix = d.fix[i];
        double v[3];
        ldv<DIM>(d.v, i, v);
        const double kk = 0.5 * (d.dt / rho);
#pragma unroll
        for (int dof = 0; dof < DIM; dof++)
          if (!((fix >> dof) & 1u)) v[dof] += kk * f[dof];
        stv<DIM>(d.v, i, v);
        d.vmag[i] = len3<DIM>(v);
      }
    }
  }
  // the post-processing tail only on the steps that record test output
  if (!post || d.test == PDGPU_TEST_NONE) return;
  if (!(n_step % d.test_interval == 0 && n_step >= d.test_interval)) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&d.ctrl->end_done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last) {
    __threadfence();
    if (threadIdx.x == 0) d.ctrl->end_done = 0u;
    postprocess_block<DIM>(d);
  }
}

// ---------------------------------------------------------------------------
// Set-up kernels
// ---------------------------------------------------------------------------

// DEMModel::updatePeridynamicNeighborlist (demModel.cpp:1659-1694): same
// particle, j != i, strict squared distance against horizon^2, computed in
// nanoflann's order (query minus point, dims 0..2).
template <int DIM, int LPN, bool FILL>
__global__ void __launch_bounds__(kBlock) k_pd_cand(DevData d, Grid g, int64_t *row) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / LPN;
  const int lane = threadIdx.x % LPN;
  if (i >= d.n_nodes) return;
  const unsigned gm = group_mask<LPN>();
  const unsigned lane_base = (threadIdx.x & 31u) / LPN * LPN;
  double q[3];
  ldv<DIM>(d.x, i, q);
  const int32_t pi = d.ptid[i];
  const double r = d.particles[pi].horizon;
  const double r2 = r * r;
  int c[3] = {cell_coord<DIM>(q[0], g, 0), cell_coord<DIM>(q[1], g, 1),
              DIM == 3 ? cell_coord<DIM>(q[2], g, 2) : 0};
  int64_t out = FILL ? row[i] : 0;
  int64_t count = 0;
  const int zlo = DIM == 3 ? max(c[2] - 1, 0) : 0;
  const int zhi = DIM == 3 ? min(c[2] + 1, g.dims[2] - 1) : 0;
  for (int cz = zlo; cz <= zhi; cz++)
    for (int cy = max(c[1] - 1, 0); cy <= min(c[1] + 1, g.dims[1] - 1); cy++)
      for (int cx = max(c[0] - 1, 0); cx <= min(c[0] + 1, g.dims[0] - 1); cx++) {
        const int cell = cx + g.dims[0] * (cy + g.dims[1] * cz);
        const int s = d.cell_start[cell], e = d.cell_start[cell + 1];
        for (int base = s; base < e; base += LPN) {
          const int a = base + lane;
          bool hit = false;
          int32_t j = -1;
          if (a < e) {
            j = d.cell_nodes[a];
            if (j != i && d.ptid[j] == pi) {
              double p[3];
              ldv<DIM>(d.x, j, p);
              double dd = 0.0;
#pragma unroll
              for (int t = 0; t < DIM; t++) {
                const double df = q[t] - p[t];
                dd += df * df;
              }
              hit = dd < r2;
            }
          }
          const unsigned bal = (__ballot_sync(gm, hit) & gm) >> lane_base;
          if (FILL) {
            if (hit) d.pd_col[out + __popc(bal & ((1u << lane) - 1u))] = j;
            out += __popc(bal);
          } else {
            count += __popc(bal);
          }
        }
      }
  if (!FILL && lane == 0) row[i + 1] = count;
}

// order each node's neighbour list by node index (one warp per node)
__global__ void k_pd_sort_rows(DevData d, int32_t *tmp) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= d.n_nodes) return;
  const int64_t s = d.pd_row[i], e = d.pd_row[i + 1];
  for (int64_t a = s + lane; a < e; a += 32) tmp[a] = d.pd_col[a];
  __syncwarp();
  for (int64_t a = s + lane; a < e; a += 32) {
    const int32_t va = tmp[a];
    int64_t rank = 0;
    for (int64_t b = s; b < e; b++) rank += tmp[b] < va;
    d.pd_col[s + rank] = va;
  }
}

// material::computeStateMxI (materialUtil.cpp:21-73).  One thread per node
// sums its row in list order, as the reference does, so that with the
// reference's own neighbour order the result is the reference's to the bit
// (FP64, no FMA contraction in this unit).
template <int DIM, int LPN>
__global__ void k_mx(DevData d) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / LPN;
  const int lane = threadIdx.x % LPN;
  if (i >= d.n_nodes) return;
  const unsigned gm = group_mask<LPN>();
  const DevParticle &P = d.particles[d.ptid[i]];
  double xi[3];
  ldv<DIM>(d.xref, i, xi);
  double m = 0.0;
  for (int64_t k = d.pd_row[i] + lane; k < d.pd_row[i + 1]; k += LPN) {
    const int32_t j = d.pd_col[k];
    double xj[3], dx[3];
    ldv<DIM>(d.xref, j, xj);
    for (int q = 0; q < 3; q++) dx[q] = xj[q] - xi[q];
    const double rji = len3<DIM>(dx);
    if (is_greater(rji, P.horizon)) continue;
    double volj = d.vol[j];
    if (is_greater(rji, P.check_low)) volj *= (P.check_up - rji) / P.h;
    m += rji * rji * influence(d.inf, rji, P.horizon) * volj;
  }
  m = group_sum<LPN>(m, gm);
  if (lane == 0) {
    d.mx[i] = m;
    if (is_less(m, 1.0e-18)) set_error(d.ctrl, DEV_ERR_NONFINITE, i);
  }
}

inline unsigned blocks_for(int64_t n, int per_block) {
  return (unsigned)((n + per_block - 1) / per_block);
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

#define PDGPU_DIM_DISPATCH(d, KERNEL, ...)            \
  do {                                               \
    if ((d).dim == 2) KERNEL<2> __VA_ARGS__;         \
    else KERNEL<3> __VA_ARGS__;                      \
  } while (0)

void launch_pack_vec(const DevData &d, const double *aos3, double *dst, cudaStream_t s) {
  PDGPU_DIM_DISPATCH(d, k_pack, <<<blocks_for(d.n_nodes, kBlock), kBlock, 0, s>>>(aos3, dst, d.n_nodes));
}
void launch_unpack_vec(const DevData &d, const double *src, double *aos3, cudaStream_t s) {
  PDGPU_DIM_DISPATCH(d, k_unpack, <<<blocks_for(d.n_nodes, kBlock), kBlock, 0, s>>>(src, aos3, d.n_nodes));
}
void launch_apply_ic(const DevData &d, cudaStream_t s) {
  PDGPU_DIM_DISPATCH(d, k_apply_ic, <<<blocks_for(d.n_nodes, kBlock), kBlock, 0, s>>>(d));
}
void launch_integrate(const DevData &d, int verlet, cudaStream_t s) {
  const unsigned g = blocks_for(d.n_nodes, kBlock);
  if (d.dim == 2) {
    if (verlet) k_integrate<2, true><<<g, kBlock, 0, s>>>(d);
    else k_integrate<2, false><<<g, kBlock, 0, s>>>(d);
  } else {
    if (verlet) k_integrate<3, true><<<g, kBlock, 0, s>>>(d);
    else k_integrate<3, false><<<g, kBlock, 0, s>>>(d);
  }
}
void launch_verlet_second(const DevData &d, cudaStream_t s) {
  PDGPU_DIM_DISPATCH(d, k_verlet_second, <<<blocks_for(d.n_nodes, kBlock), kBlock, 0, s>>>(d));
}
void launch_ctrl(const DevData &d, int mode, cudaStream_t s) { k_ctrl<<<1, 1, 0, s>>>(d, mode); }
void launch_bc(const DevData &d, cudaStream_t s) {
  if (!d.n_ubc_nodes) return;
  PDGPU_DIM_DISPATCH(d, k_bc, <<<blocks_for(d.n_ubc_nodes, 128), 128, 0, s>>>(d));
}

size_t scan_temp_bytes(int64_t n) {
  size_t a = 0, b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, a, (int32_t *)nullptr, (int32_t *)nullptr, (int)n);
  cub::DeviceScan::InclusiveSum(nullptr, b, (int64_t *)nullptr, (int64_t *)nullptr, n);
  return a > b ? a : b;
}


template <int DIM, int LPN>
static cudaError_t rebuild_dim(const DevData &d, uint8_t bit, int64_t *bsum, int grid,
                               cudaStream_t s) {
  DevData dd = d;
  void *args[] = {(void *)&dd, (void *)&bit, (void *)&bsum};
  return cudaLaunchCooperativeKernel((const void *)k_contact_rebuild<DIM, LPN>, dim3(grid),
                                     dim3(kCoopBlock), args, cand_stage_bytes<DIM>(), s);
}

int rebuild_grid_blocks(const DevData &d, int lanes) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const void *f;
  if (d.dim == 2) f = lanes <= 8 ? (const void *)k_contact_rebuild<2, 8> : (const void *)k_contact_rebuild<2, 32>;
  else f = lanes <= 8 ? (const void *)k_contact_rebuild<3, 8> : (const void *)k_contact_rebuild<3, 32>;
  const size_t dyn = d.dim == 2 ? cand_stage_bytes<2>() : cand_stage_bytes<3>();
  cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, f, kCoopBlock, dyn);
  return sms * (per > 0 ? per : 1);
}

cudaError_t launch_contact_rebuild(const DevData &d, int64_t *bsum, int grid, int lanes, int init,
                                   cudaStream_t s) {
  const uint8_t bit = init ? NODE_SEARCH0 : NODE_SEARCH;
  if (d.dim == 2) return lanes <= 8 ? rebuild_dim<2, 8>(d, bit, bsum, grid, s) : rebuild_dim<2, 32>(d, bit, bsum, grid, s);
  return lanes <= 8 ? rebuild_dim<3, 8>(d, bit, bsum, grid, s) : rebuild_dim<3, 32>(d, bit, bsum, grid, s);
}

int sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

void launch_contact_owner(const DevData &d, cudaStream_t s) {
  k_contact_owner<<<sm_count() * 4, kBlock, 0, s>>>(d);
}

void launch_contact_force(const DevData &d, int lanes, cudaStream_t s) {
  const unsigned g = (unsigned)d.contact_grid;
  if (lanes == 1) {  // one kernel, a warp per 32 nodes
    if (d.dim == 2) k_contact_warp<2><<<g, kBlock, 0, s>>>(d);
    else k_contact_warp<3><<<g, kBlock, 0, s>>>(d);
    return;
  }
  // the distance pass: eight CTAs per SM, grid-stride over the entries
  if (d.dim == 2) k_contact_near<2><<<sm_count() * 8, kBlock, 0, s>>>(d);
  else k_contact_near<3><<<sm_count() * 8, kBlock, 0, s>>>(d);
  if (d.dim == 2) {
    if (lanes == 1) k_contact<2, 1><<<g, kBlock, 0, s>>>(d);
    else if (lanes == 2) k_contact<2, 2><<<g, kBlock, 0, s>>>(d);
    else if (lanes == 4) k_contact<2, 4><<<g, kBlock, 0, s>>>(d);
    else if (lanes == 8) k_contact<2, 8><<<g, kBlock, 0, s>>>(d);
    else k_contact<2, 32><<<g, kBlock, 0, s>>>(d);
  } else {
    if (lanes == 1) k_contact<3, 1><<<g, kBlock, 0, s>>>(d);
    else if (lanes == 2) k_contact<3, 2><<<g, kBlock, 0, s>>>(d);
    else if (lanes == 4) k_contact<3, 4><<<g, kBlock, 0, s>>>(d);
    else if (lanes == 8) k_contact<3, 8><<<g, kBlock, 0, s>>>(d);
    else k_contact<3, 32><<<g, kBlock, 0, s>>>(d);
  }
}

void launch_scene_post(const DevData &d, cudaStream_t s) {
  if (d.n_scenes <= 1) return;
  if (d.dim == 2) k_scene_post<2><<<d.n_scenes, 256, 0, s>>>(d);
  else k_scene_post<3><<<d.n_scenes, 256, 0, s>>>(d);
}

void launch_damping(const DevData &d, cudaStream_t s) {
  if (d.n_particles <= 0) return;
  k_damping<<<d.damp_group ? d.n_damp_groups : d.n_particles, kDampBlock, 0, s>>>(d, d.dim);
}

void launch_external(const DevData &d, cudaStream_t s) {
  PDGPU_DIM_DISPATCH(d, k_external, <<<blocks_for(d.n_nodes, kBlock), kBlock, 0, s>>>(d));
  if (d.n_fbc_nodes)
    PDGPU_DIM_DISPATCH(d, k_force_bc, <<<blocks_for(d.n_fbc_nodes, 128), 128, 0, s>>>(d));
}

void launch_step_begin(const DevData &d, int verlet, cudaStream_t s) {
  const unsigned g = blocks_for(d.n_nodes, kBlock * kBeginNodes);
  if (d.dim == 2) {
    if (verlet) k_step_begin<2, true><<<g, kBlock, 0, s>>>(d);
    else k_step_begin<2, false><<<g, kBlock, 0, s>>>(d);
  } else {
    if (verlet) k_step_begin<3, true><<<g, kBlock, 0, s>>>(d);
    else k_step_begin<3, false><<<g, kBlock, 0, s>>>(d);
  }
}

void launch_step_end(const DevData &d, int verlet, int post, cudaStream_t s) {
  const unsigned g = blocks_for(d.n_nodes, kBlock * kEndNodes);
  if (d.dim == 2) {
    if (verlet) k_step_end<2, true><<<g, kBlock, 0, s>>>(d, post);
    else k_step_end<2, false><<<g, kBlock, 0, s>>>(d, post);
  } else {
    if (verlet) k_step_end<3, true><<<g, kBlock, 0, s>>>(d, post);
    else k_step_end<3, false><<<g, kBlock, 0, s>>>(d, post);
  }
}

void launch_postprocess(const DevData &d, cudaStream_t s) {
  if (d.test == PDGPU_TEST_NONE) return;
  PDGPU_DIM_DISPATCH(d, k_postprocess, <<<1, 1024, 0, s>>>(d));
}

void launch_build_pd(const DevData &d, double cell, int64_t *row, int32_t *tmp, void *scan_tmp,
                     size_t scan_bytes, int pass, cudaStream_t s) {
  // pass 0: grid + counts; pass 1: fill + sort rows.  d.grid holds the
  // horizon-sized grid built by the caller; d.ctrl->update must be 1.
  const int lanes = d.dim == 2 ? 8 : 32;
  const unsigned g = blocks_for(d.n_nodes * lanes, kBlock);
  (void)cell;
  if (pass == 0) {
    const unsigned gn = blocks_for(d.n_nodes, kBlock);
    k_zero_cells<<<blocks_for(d.grid.ncells + 1, kBlock), kBlock, 0, s>>>(d);
    PDGPU_DIM_DISPATCH(d, k_cell_count, <<<gn, kBlock, 0, s>>>(d, d.x, d.grid));
    cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, d.cell_cnt, d.cell_start, d.grid.ncells + 1, s);
    k_cell_scatter<<<gn, kBlock, 0, s>>>(d);
    k_cell_sort<<<blocks_for((int64_t)d.grid.ncells * 32, kBlock), kBlock, 0, s>>>(d);
    if (d.dim == 2) k_pd_cand<2, 8, false><<<g, kBlock, 0, s>>>(d, d.grid, row);
    else k_pd_cand<3, 32, false><<<g, kBlock, 0, s>>>(d, d.grid, row);
    cub::DeviceScan::InclusiveSum(scan_tmp, scan_bytes, row + 1, row + 1, d.n_nodes, s);
  } else {
    if (d.dim == 2) k_pd_cand<2, 8, true><<<g, kBlock, 0, s>>>(d, d.grid, row);
    else k_pd_cand<3, 32, true><<<g, kBlock, 0, s>>>(d, d.grid, row);
    k_pd_sort_rows<<<blocks_for(d.n_nodes * 32, kBlock), kBlock, 0, s>>>(d, tmp);
  }
}

void launch_compute_mx(const DevData &d, cudaStream_t s) {
  const unsigned g = blocks_for(d.n_nodes, kBlock);
  if (d.dim == 2) k_mx<2, 1><<<g, kBlock, 0, s>>>(d);
  else k_mx<3, 1><<<g, kBlock, 0, s>>>(d);
}

}  // namespace pdgpu
