/*
 * pdoracle.c — CPU restatement of the reference's explicit step.
 * ORACLE TEST INFRASTRUCTURE ONLY (see pdoracle.h).
 *
 * Points are three doubles as in util::Point (src/util/point.h); every
 * expression keeps the reference's left-to-right evaluation order.
 */
#include "pdoracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI 3.14159265358979323846 /* M_PI */

typedef struct {
  double x, y, z;
} pt;

static pt P3(double x, double y, double z) {
  pt p = {x, y, z};
  return p;
}
static pt add(pt a, pt b) { return P3(a.x + b.x, a.y + b.y, a.z + b.z); }
static pt sub(pt a, pt b) { return P3(a.x - b.x, a.y - b.y, a.z - b.z); }
static pt scl(double s, pt a) { return P3(s * a.x, s * a.y, s * a.z); }
static pt dvs(pt a, double s) { return P3(a.x / s, a.y / s, a.z / s); }
/* util::Point::dot / length (point.h:118, 132) */
static double dot(pt a, pt b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double len(pt a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static double comp(pt a, int d) { return d == 0 ? a.x : d == 1 ? a.y : a.z; }
static void setc(pt *a, int d, double v) {
  if (d == 0) a->x = v;
  else if (d == 1) a->y = v;
  else a->z = v;
}

/* util::isGreater / isLess, COMPARE_EPS = 1e-5 (function.cpp:15-23) */
static int is_greater(double a, double b) {
  return (a - b) > ((fabs(a) < fabs(b) ? fabs(b) : fabs(a)) * 1.0e-5);
}
static int is_less(double a, double b) {
  return (b - a) > ((fabs(a) < fabs(b) ? fabs(b) : fabs(a)) * 1.0e-5);
}

struct po_model {
  po_scene s;
  int64_t N, Np, B;
  pt *x, *u, *v, *f;
  double *vmag, *theta, *mx;
  float *Z;
  uint8_t *bonds;
  uint8_t *active, *search, *search0;
  /* contact candidates (ModelData::d_neighC) as CSR */
  int64_t *c_row;
  int64_t *c_col;
  int64_t c_cap;
  /* time and contact control (ModelData) */
  int64_t n;
  double time;
  int64_t interval, counter, init_calls;
  double radius, max_velocity;
  uint8_t *zero_applied;
  /* post-processing */
  double reaction, penetration, contact_reaction, pen_dist, max_y, car;
  /* per-particle damping scratch */
  int64_t *wall_list;
  int64_t wall_cap;
};

static pt node(const double *a, int64_t i) { return P3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }

/* J(r / horizon) (influenceFn.cpp:21-23, 55-57, 86-88; material.h:431-433) */
static double infl(const po_scene *s, double r, double horizon) {
  const double q = r / horizon;
  if (s->inf_type == 1) return s->inf_params[0] + s->inf_params[1] * q;
  if (s->inf_type == 0) return s->inf_params[0];
  return s->inf_params[0] * exp(-q * q / s->inf_params[1]);
}

/* Material::getSc (material.h:415-417, 801, 1144, 1459) */
static double get_sc(const po_scene *s, int32_t p, double r) {
  const double *mat = s->p_mat + 6 * p;
  switch (s->p_material[p]) {
    case 0: return mat[2] / sqrt(r);
    case 1: return mat[1];
    case 2: return DBL_MAX;
    default: return mat[2];
  }
}

/* Material::getS (material.h:405-407 RNP; 791-793 / 1134-1136 / 1449-1451) */
static double get_s(const po_scene *s, int32_t p, pt dx, pt du) {
  if (s->p_material[p] == 0) return dot(dx, du) / dot(dx, dx);
  return (len(add(dx, du)) - len(dx)) / len(dx);
}

/* Material::getBondForceDirection (material.h:394-397; 780-783, ...) */
static pt get_dir(const po_scene *s, int32_t p, pt dx, pt du) {
  if (s->p_material[p] == 0) return dvs(dx, len(dx));
  return dvs(add(dx, du), len(add(dx, du)));
}

po_model *po_create(const po_scene *s) {
  po_model *m = (po_model *)calloc(1, sizeof(po_model));
  m->s = *s;
  m->N = s->n_nodes;
  m->Np = s->n_particles;
  m->B = (int64_t)s->pd_rowptr[m->N];
  m->x = (pt *)calloc(m->N, sizeof(pt));
  m->u = (pt *)calloc(m->N, sizeof(pt));
  m->v = (pt *)calloc(m->N, sizeof(pt));
  m->f = (pt *)calloc(m->N, sizeof(pt));
  m->vmag = (double *)calloc(m->N, sizeof(double));
  m->theta = (double *)calloc(m->N, sizeof(double));
  m->mx = (double *)calloc(m->N, sizeof(double));
  m->Z = (float *)calloc(m->N, sizeof(float));
  m->bonds = (uint8_t *)calloc(m->B + 1, 1);
  m->active = (uint8_t *)calloc(m->N, 1);
  m->search = (uint8_t *)calloc(m->N, 1);
  m->search0 = (uint8_t *)calloc(m->N, 1);
  m->c_row = (int64_t *)calloc(m->N + 1, sizeof(int64_t));
  m->c_cap = 1024;
  m->c_col = (int64_t *)malloc(m->c_cap * sizeof(int64_t));
  m->zero_applied = (uint8_t *)calloc(s->n_ubc + 1, 1);
  m->wall_cap = 1024;
  m->wall_list = (int64_t *)malloc(m->wall_cap * sizeof(int64_t));
  for (int64_t i = 0; i < m->N; i++) {
    m->x[i] = node(s->xref, i);
    m->mx[i] = s->mx[i];
  }
  for (int64_t p = 0; p < m->Np; p++)
    for (int64_t i = s->p_start[p]; i < s->p_end[p]; i++) {
      /* d_fPdCompNodes (demModel.cpp:234-241) */
      m->active[i] = s->p_compute_force[p] ? 1 : 0;
      /* searching nodes of updateContactNeighborlist (:1720-1729) */
      m->search[i] = (s->p_type[p] == 0 && s->p_compute_force[p] && !s->p_all_fixed[p]);
      /* at DEMModel::init, before the two_particle override (:218-220) */
      m->search0[i] = (s->p_type[p] == 0 && !s->p_all_fixed[p]);
    }
  /* DEMModel::init (:183-184) */
  m->interval = s->search_interval;
  m->radius = s->search_factor * s->max_contact_r;
  return m;
}

void po_destroy(po_model *m) {
  if (!m) return;
  free(m->x); free(m->u); free(m->v); free(m->f); free(m->vmag); free(m->theta); free(m->mx);
  free(m->Z); free(m->bonds); free(m->active); free(m->search); free(m->search0);
  free(m->c_row); free(m->c_col); free(m->zero_applied); free(m->wall_list);
  free(m);
}

/* ------------------------------------------------------------------------
 * DEMModel::computePeridynamicForces (demModel.cpp:602-789)
 * ------------------------------------------------------------------------ */
static void pd_forces(po_model *m) {
  const po_scene *s = &m->s;
  /* state-based pre-pass (:610-679), when particle 0 is state-based */
  if (m->Np > 0 && s->p_material[0] == 3) {
    for (int64_t i = 0; i < m->N; i++) {
      if (!m->active[i]) continue;
      const int32_t p = (int32_t)s->ptid[i];
      if (s->p_material[p] != 3) continue;
      const double horizon = s->p_horizon[p], h = s->p_h[p];
      const pt xi = node(s->xref, i), ui = m->u[i];
      const double mm = m->mx[i];
      double theta = 0.;
      const double up = horizon + 0.5 * h, low = horizon - 0.5 * h;
      for (int64_t k = (int64_t)s->pd_rowptr[i]; k < (int64_t)s->pd_rowptr[i + 1]; k++) {
        const int64_t j = (int64_t)s->pd_col[k];
        const pt xj = node(s->xref, j), uj = m->u[j];
        const double rji = len(sub(xj, xi));
        const double cl = len(sub(add(sub(xj, xi), uj), ui)) - rji;
        const double sv = cl / rji;
        const double sc = get_sc(s, p, rji);
        int fs = m->bonds[k];
        if (!fs && is_greater(fabs(sv), sc + 1.0e-10)) fs = 1;
        m->bonds[k] = (uint8_t)fs;
        if (!fs) {
          double volj = s->vol[j];
          if (is_greater(rji, low)) volj *= (up - rji) / h;
          theta += rji * cl * infl(s, rji, horizon) * volj;
        }
      }
      m->theta[i] = 3. * theta / mm;
    }
  }
  /* main pass (:685-788) */
  for (int64_t i = 0; i < m->N; i++) {
    if (!m->active[i]) continue;
    const int32_t p = (int32_t)s->ptid[i];
    const double *mat = s->p_mat + 6 * p;
    const int mt = s->p_material[p];
    const double horizon = s->p_horizon[p], h = s->p_h[p];
    const pt xi = node(s->xref, i), ui = m->u[i];
    const double mi = m->mx[i], thi = m->theta[i];
    const double up = horizon + 0.5 * h, low = horizon - 0.5 * h;
    pt force = P3(0., 0., 0.);
    float Zi = 0.f;
    for (int64_t k = (int64_t)s->pd_rowptr[i]; k < (int64_t)s->pd_rowptr[i + 1]; k++) {
      const int64_t j = (int64_t)s->pd_col[k];
      int fs = m->bonds[k];
      const pt xj = node(s->xref, j), uj = m->u[j];
      double volj = s->vol[j];
      const double rji = len(sub(xj, xi));
      const double Sji = get_s(s, p, sub(xj, xi), sub(uj, ui));
      if (!fs) {
        if (is_greater(rji, low)) volj *= (up - rji) / h;
        if (mt == 3) {
          /* PdState::getBondEF (material.h:1415-1429) for i and for j */
          const double J = infl(s, rji, horizon);
          const double cl = Sji * rji;
          const double K = mat[0], G = mat[1];
          const double ai = 15. * G / mi;
          const double fi = (3. * K / mi) - ai / 3.;
          const double efi = J * (rji * thi * fi + cl * ai);
          const double mj = m->mx[j], thj = m->theta[j];
          const double aj = 15. * G / mj;
          const double fj = (3. * K / mj) - aj / 3.;
          const double efj = J * (rji * thj * fj + cl * aj);
          const double sf = (efi + efj) * volj;
          force = add(force, scl(sf, get_dir(s, p, sub(xj, xi), sub(uj, ui))));
        } else {
          double ef = 0.;
          const double J = infl(s, rji, horizon);
          if (mt == 0) {
            /* RnpMaterial::getBondEF with break_bonds (material.h:342-361) */
            if (mat[5] != 0. && !fs && is_greater(fabs(Sji), mat[4] * get_sc(s, p, rji))) fs = 1;
            if (!fs) ef = J * 4. * Sji * mat[0] * mat[1] * exp(-mat[1] * rji * Sji * Sji) / mat[3];
          } else if (mt == 1) {
            /* PmbMaterial::getBondEF (material.h:732-753) */
            if (!fs && is_greater(fabs(Sji), mat[1] + 1.0e-10)) fs = 1;
            if (!fs) ef = J * mat[0] * Sji;
          } else {
            /* PdElastic::getBondEF (material.h:1090-1097) */
            ef = J * mat[0] * Sji;
          }
          m->bonds[k] = (uint8_t)fs;
          const double sf = ef * volj;
          force = add(force, scl(sf, get_dir(s, p, sub(xj, xi), sub(uj, ui))));
        }
      } else {
        /* internal normal contact of a broken bond (:760-768) */
        const pt yji = sub(add(xj, uj), add(xi, ui));
        const double R = len(yji);
        double sf = s->p_kn[p] * volj * (R - s->p_rc[p]) / R;
        if (sf > 0.) sf = 0.;
        force = add(force, scl(sf, yji));
      }
      /* damage (:770-773) */
      const double Sc = get_sc(s, p, rji);
      if (is_greater(fabs(Sji / Sc), (double)Zi)) Zi = (float)fabs(Sji / Sc);
    }
    m->f[i] = force;
    m->Z[i] = Zi;
  }
}

/* ------------------------------------------------------------------------
 * DEMModel::updateContactNeighborSearchParameters (demModel.cpp:1808-1955)
 * ------------------------------------------------------------------------ */
static int contact_params(po_model *m) {
  const po_scene *s = &m->s;
  if (m->n == 0) {
    m->init_calls += 1;
    if (m->init_calls == 1) return 1;
    if (m->init_calls == 2) {
      m->counter++;
      return (m->counter - 1) % m->interval == 0;
    }
  }
  if (m->interval == 1) {
    m->radius = s->max_contact_r;
    m->counter++;
    return (m->counter - 1) % m->interval == 0;
  }
  const int64_t upi = m->interval > 5 ? (int64_t)(0.2 * (double)m->interval) : 1;
  if (m->counter > 0 && m->counter % upi != 0) {
    m->counter++;
    return (m->counter - 1) % m->interval == 0;
  }
  /* maximum |v| per particle, then over particles (:1862-1883) */
  double vmax = 0.;
  for (int64_t p = 0; p < m->Np; p++) {
    double pm = m->vmag[s->p_start[p]];
    for (int64_t i = s->p_start[p]; i < s->p_end[p]; i++)
      if (m->vmag[i] > pm) pm = m->vmag[i];
    if (p == 0 || pm > vmax) vmax = pm;
  }
  m->max_velocity = vmax;
  const double safety = s->search_factor > 5 ? s->search_factor : 10;
  const double r_contact = s->search_factor * s->max_contact_r;
  const double r_vel = m->max_velocity * s->dt * (double)s->search_interval * safety;
  if (is_greater(r_vel, r_contact)) {
    m->interval = (int64_t)(s->max_contact_r / (m->max_velocity * s->dt));
    m->radius = r_contact;
    m->counter = 0;
    if (m->interval < 1) {
      m->interval = 1;
      m->radius = s->max_contact_r;
    }
  } else {
    m->radius = m->interval < 2 ? s->max_contact_r : r_contact;
  }
  m->counter++;
  return (m->counter - 1) % m->interval == 0;
}

/* DEMModel::updateContactNeighborlist (:1696-1756): brute-force radius
 * search with the kd-tree's strict test sum_d (q_d - p_d)^2 < r*r
 * (nanoflann.hpp:611-621, nflannSetup.h:272), other particles only. */
static void contact_search(po_model *m, const uint8_t *searching) {
  const po_scene *s = &m->s;
  const double r2 = m->radius * m->radius;
  int64_t e = 0;
  for (int64_t i = 0; i < m->N; i++) {
    m->c_row[i] = e;
    if (!searching[i]) continue;
    const pt q = m->x[i];
    for (int64_t j = 0; j < m->N; j++) {
      if (s->ptid[j] == s->ptid[i]) continue;
      const double d0 = q.x - m->x[j].x, d1 = q.y - m->x[j].y, d2 = q.z - m->x[j].z;
      double dd = 0.;
      dd += d0 * d0;
      dd += d1 * d1;
      dd += d2 * d2;
      if (dd < r2) {
        if (e >= m->c_cap) {
          m->c_cap *= 2;
          m->c_col = (int64_t *)realloc(m->c_col, m->c_cap * sizeof(int64_t));
        }
        m->c_col[e++] = j;
      }
    }
  }
  m->c_row[m->N] = e;
}

static const double *cpair(const po_scene *s, const double *a, int32_t zi, int32_t zj) {
  return a + (int64_t)zi * s->n_zones + zj;
}

/* ------------------------------------------------------------------------
 * DEMModel::computeContactForces (demModel.cpp:820-1066)
 * ------------------------------------------------------------------------ */
static void contact_forces(po_model *m) {
  const po_scene *s = &m->s;
  /* node pass (:832-934) over d_fContCompNodes */
  for (int64_t i = 0; i < m->N; i++) {
    if (!m->active[i]) continue;
    const int32_t pi = (int32_t)s->ptid[i];
    const pt yi = m->x[i], vi = m->v[i];
    pt force = P3(0., 0., 0.);
    for (int64_t k = m->c_row[i]; k < m->c_row[i + 1]; k++) {
      const int64_t j = m->c_col[k];
      const pt yj = m->x[j];
      const double Rji = len(sub(yj, yi));
      const int32_t pj = (int32_t)s->ptid[j];
      const int both_walls = s->p_type[pi] == 1 && s->p_type[pj] == 1;
      if (j == i || pj == pi || both_walls) continue;
      const int32_t zi = s->p_zone[pi], zj = s->p_zone[pj];
      const double rc = *cpair(s, s->c_rc, zi, zj);
      if (is_less(Rji, rc)) {
        const pt yji = sub(m->x[j], yi);
        const double volj = s->vol[j];
        const pt vji = sub(m->v[j], vi);
        const pt en = dvs(yji, Rji);
        const double vn = dot(vji, en);
        pt et = sub(vji, scl(vn, en));
        if (is_greater(len(et), 0.)) et = dvs(et, len(et));
        else et = P3(0., 0., 0.);
        double sf = *cpair(s, s->c_kn, zi, zj) * (Rji - rc) * volj;
        if (sf > 0.) sf = 0.;
        force = add(force, scl(sf, en));
        force = add(force, scl(*cpair(s, s->c_mu, zi, zj) * sf, et));
        if (pj == s->test_wall) {
          const pt c = add(scl(sf, en), scl(*cpair(s, s->c_mu, zi, zj) * sf, et));
          m->contact_reaction -= comp(c, s->test_dir) * s->vol[i];
        }
      }
    }
    m->f[i] = add(m->f[i], force);
  }
  /* particle damping (:937-1065) */
  for (int64_t p = 0; p < m->Np; p++) {
    if (s->p_type[p] != 0) continue;
    const double Ri = s->p_bound_r[p];
    const double vol_pi = PI * Ri * Ri;
    const pt xc = m->x[s->p_center[p]], vc = m->v[s->p_center[p]];
    const double rhoi = s->p_density[p];
    pt force = P3(0., 0., 0.);
    for (int64_t q = 0; q < m->Np; q++) {
      if (s->p_type[q] != 0 || q == p) continue;
      const double Rj = s->p_bound_r[q];
      const pt xcji = sub(m->x[s->p_center[q]], xc);
      const double dist = len(xcji);
      const int32_t zi = s->p_zone[p], zj = s->p_zone[q];
      const double rc = *cpair(s, s->c_rc, zi, zj);
      if (is_less(dist, Rj + Ri + 1.01 * rc)) {
        const double vol_pj = PI * Rj * Rj;
        const double rhoj = s->p_density[q];
        const double m1 = rhoi * vol_pi, m2 = rhoj * vol_pj;
        const double meq = 2. * m1 * m2 / (m1 + m2);
        const double bn = *cpair(s, s->c_betan, zi, zj) * sqrt(*cpair(s, s->c_kappa, zi, zj) * rc * meq);
        pt hat = P3(0., 0., 0.);
        if (is_greater(dist, 0.)) hat = dvs(xcji, dist);
        const pt vcji = sub(m->v[s->p_center[q]], vc);
        double vm = dot(vcji, hat);
        if (vm > 0.) vm = 0.;
        force = add(force, dvs(scl(bn * vm, hat), vol_pi));
      }
    }
    /* wall nodes within Rc of a node of p, first-occurrence order (:994-1017) */
    int64_t nw = 0;
    for (int64_t jn = s->p_start[p]; jn < s->p_end[p]; jn++) {
      const pt yj = m->x[jn];
      for (int64_t k = m->c_row[jn]; k < m->c_row[jn + 1]; k++) {
        const int64_t kid = m->c_col[k];
        const int32_t pk = (int32_t)s->ptid[kid];
        if (s->p_type[pk] != 1) continue;
        const double Rjk = len(sub(m->x[kid], yj));
        if (!is_less(Rjk, *cpair(s, s->c_rc, s->p_zone[p], s->p_zone[pk]))) continue;
        int seen = 0;
        for (int64_t a = 0; a < nw; a++)
          if (m->wall_list[a] == kid) {
            seen = 1;
            break;
          }
        if (seen) continue;
        if (nw >= m->wall_cap) {
          m->wall_cap *= 2;
          m->wall_list = (int64_t *)realloc(m->wall_list, m->wall_cap * sizeof(int64_t));
        }
        m->wall_list[nw++] = kid;
      }
    }
    for (int64_t a = 0; a < nw; a++) {
      const int64_t j = m->wall_list[a];
      const int32_t pj = (int32_t)s->ptid[j];
      const double meq = rhoi * vol_pi;
      const int32_t zi = s->p_zone[p], zj = s->p_zone[pj];
      const double rc = *cpair(s, s->c_rc, zi, zj);
      const double bn = *cpair(s, s->c_betan, zi, zj) * sqrt(*cpair(s, s->c_kappa, zi, zj) * rc * meq);
      const pt xcji = sub(m->x[j], xc);
      pt hat = P3(0., 0., 0.);
      if (is_greater(len(xcji), 0.)) hat = dvs(xcji, len(xcji));
      const pt vcji = sub(m->v[j], vc);
      double vm = dot(vcji, hat);
      if (vm > 0.) vm = 0.;
      force = add(force, dvs(scl(bn * vm, hat), vol_pi));
    }
    for (int64_t i = s->p_start[p]; i < s->p_end[p]; i++) m->f[i] = add(m->f[i], force);
  }
}

/* ------------------------------------------------------------------------
 * DEMModel::computeExternalForces (demModel.cpp:791-812) with
 * ParticleFLoading::apply (particleFLoading.cpp:85-173)
 * ------------------------------------------------------------------------ */
static double hat_fn(double x, double lo, double hi) {
  /* util::hatFunction (function.cpp:24-42) */
  if (is_greater(x, lo - 1.0E-12) && is_less(x, hi + 1.0E-12)) {
    const double mid = 0.5 * (lo + hi);
    const double l = mid - lo;
    if (l < 1.0E-12) return 1.0;
    if (is_less(x, mid)) return (x - lo) / l;
    return (hi - x) / l;
  }
  return 0.0;
}

static void external_forces(po_model *m) {
  const po_scene *s = &m->s;
  const pt g = P3(s->gravity[0], s->gravity[1], s->gravity[2]);
  if (len(g) > 1.0E-8)
    for (int64_t i = 0; i < m->N; i++) m->f[i] = add(m->f[i], scl(s->p_density[s->ptid[i]], g));
  for (int64_t p = 0; p < m->Np; p++)
    for (int32_t b = 0; b < s->n_fbc; b++) {
      const po_bc *bc = &s->fbc[b];
      if (!bc->particle_sel[p]) continue;
      const double *box = bc->particle_box + 6 * p;
      for (int64_t i = s->p_start[p]; i < s->p_end[p]; i++) {
        if (!bc->node_sel[i]) continue;
        const pt x = node(s->xref, i);
        double fmax = 1.0;
        const double *sp = bc->spatial_params;
        switch (bc->spatial_fn) {
          case 1: fmax = sp[0] * hat_fn(x.x, box[0], box[3]); break;
          case 2: fmax = sp[0] * hat_fn(x.y, box[1], box[4]); break;
          case 3: fmax = sp[0] * sin(PI * sp[0] * x.x); break;
          case 4: fmax = sp[0] * sin(PI * sp[0] * x.y); break;
          case 5: fmax = sp[0] * sp[0] * x.x; break;
          case 6: fmax = sp[0] * sp[0] * x.y; break;
          default: break;
        }
        const double t = m->time, *tp = bc->time_params;
        if (bc->time_fn == 1) fmax *= t;
        else if (bc->time_fn == 5) {
          const double period = floor(t / (tp[1] + tp[2]));
          fmax *= is_less(t, period * (tp[1] + tp[2]) + tp[1]) ? t - period * tp[2] : (period + 1.) * tp[1];
        } else if (bc->time_fn == 6) {
          if (is_greater(t, tp[1])) fmax *= tp[3] * t;
          else fmax *= tp[2] * t;
        } else if (bc->time_fn == 3) {
          fmax *= sin(PI * tp[1] * t);
        }
        fmax *= tp[0];
        pt fi = P3(0., 0., 0.);
        for (int d = 0; d < 3; d++)
          if ((bc->dir_mask >> d) & 1) setc(&fi, d, fmax);
        m->f[i] = add(m->f[i], fi);
      }
    }
}

/* DEMModel::computeForces (demModel.cpp:462-600) */
static void compute_forces(po_model *m) {
  for (int64_t i = 0; i < m->N; i++) m->f[i] = P3(0., 0., 0.);
  m->contact_reaction = 0.;
  pd_forces(m);
  if (m->s.multi_particle) {
    if (contact_params(m)) contact_search(m, m->search);
    contact_forces(m);
  }
  external_forces(m);
}

/* ParticleULoading::apply for every particle (particleULoading.cpp:115-230) */
static void displacement_bc(po_model *m) {
  const po_scene *s = &m->s;
  for (int64_t p = 0; p < m->Np; p++)
    for (int32_t b = 0; b < s->n_ubc; b++) {
      const po_bc *bc = &s->ubc[b];
      if (bc->zero && m->zero_applied[b]) continue;
      if (bc->zero) m->zero_applied[b] = 1;
      if (!bc->particle_sel[p]) continue;
      const double *box = bc->particle_box + 6 * p;
      for (int64_t i = s->p_start[p]; i < s->p_end[p]; i++) {
        if (!bc->node_sel[i]) continue;
        const pt x = node(s->xref, i);
        const double *tp = bc->time_params, *sp = bc->spatial_params;
        double umax = tp[0], du = 0., dv = 0.;
        switch (bc->spatial_fn) {
          case 1: umax = sp[0] * hat_fn(x.x, box[0], box[3]); break;
          case 2: umax = sp[0] * hat_fn(x.y, box[1], box[4]); break;
          case 3: umax = umax * sin(PI * sp[0] * x.x); break;
          case 4: umax = umax * sin(PI * sp[0] * x.y); break;
          case 5: umax = umax * sp[0] * x.x; break;
          case 6: umax = umax * sp[0] * x.y; break;
          default: break;
        }
        const double t = m->time;
        if (bc->time_fn == 0) du = umax;
        else if (bc->time_fn == 1) {
          du = umax * t;
          dv = umax;
        } else if (bc->time_fn == 2) {
          du = umax * t + tp[1] * t * t;
          dv = umax + tp[1] * t;
        } else if (bc->time_fn == 3) {
          const double a = PI * tp[1];
          du = umax * sin(a * t);
          dv = umax * a * cos(a * t);
        }
        pt ui = P3(0., 0., 0.), vi = P3(0., 0., 0.);
        for (int d = 0; d < 3; d++)
          if ((bc->dir_mask >> d) & 1) {
            setc(&ui, d, du);
            setc(&vi, d, dv);
          }
        if (bc->time_fn == 4) {
          const pt x0 = P3(tp[1], tp[2], tp[3]);
          const pt dx = sub(x, x0);
          const double th = tp[0] * t;
          const pt rx = P3(dx.x * cos(th) - dx.y * sin(th), dx.x * sin(th) + dx.y * cos(th), 0.0);
          const pt drx = P3(-dx.x * sin(th) - dx.y * cos(th), dx.x * cos(th) - dx.y * sin(th), 0.0);
          ui = add(ui, sub(rx, dx));
          vi = add(vi, scl(tp[0], drx));
        }
        for (int d = 0; d < 3; d++)
          if ((bc->dir_mask >> d) & 1) {
            setc(&m->u[i], d, comp(ui, d));
            setc(&m->v[i], d, comp(vi, d));
            setc(&m->x[i], d, comp(ui, d) + comp(x, d));
          }
      }
    }
}

static void postprocess(po_model *m) {
  const po_scene *s = &m->s;
  if (!(m->n % s->test_interval == 0 && m->n >= s->test_interval)) return;
  if (s->test == 2) {
    /* ppCompressiveTest (demModel.cpp:2202-2250) */
    const int64_t w0 = s->p_start[s->test_wall];
    m->penetration = comp(m->x[w0], s->test_dir) - s->xref[3 * w0 + s->test_dir];
    double r = 0.;
    for (int64_t i = s->p_start[s->test_wall]; i < s->p_end[s->test_wall]; i++)
      r += comp(m->f[i], s->test_dir) * s->vol[i];
    m->reaction = r;
  } else if (s->test == 1 && m->Np >= 2) {
    /* ppTwoParticleTest (demModel.cpp:2096-2149) */
    const pt xc0 = m->x[s->p_center[0]], xc1 = m->x[s->p_center[1]];
    const double r = s->p_bound_r[0];
    const double re = r + *cpair(s, s->c_rc, s->p_zone[0], s->p_zone[1]);
    double pen = len(sub(xc1, xc0)) - re - r, car = 0.;
    if (is_less(pen, 0.)) car = sqrt(pow(re, 2.) - pow(re + pen, 2.));
    else if (is_greater(pen, 0.)) {
      pen = 0.;
      car = 0.;
    }
    double my_loc = m->x[s->p_start[1]].y;
    for (int64_t i = s->p_start[1]; i < s->p_end[1]; i++)
      if (is_less(my_loc, m->x[i].y)) my_loc = m->x[i].y;
    double my = 0.;
    if (is_less(my, my_loc)) my = my_loc;
    m->pen_dist = pen;
    m->car = car;
    m->max_y = my;
  }
}

static void integrate_kick_drift(po_model *m, double factor) {
  const po_scene *s = &m->s;
  const double dt = s->dt;
  for (int64_t i = 0; i < m->N; i++) {
    if (!m->active[i]) continue;
    const double rho = s->p_density[s->ptid[i]];
    const uint8_t fix = s->fix[i];
    for (int dof = 0; dof < s->dim; dof++) {
      if (!((fix >> dof) & 1u)) {
        const double k = factor == 1.0 ? (dt / rho) : 0.5 * (dt / rho);
        setc(&m->v[i], dof, comp(m->v[i], dof) + k * comp(m->f[i], dof));
        setc(&m->u[i], dof, comp(m->u[i], dof) + dt * comp(m->v[i], dof));
        setc(&m->x[i], dof, comp(m->x[i], dof) + dt * comp(m->v[i], dof));
      }
    }
    m->vmag[i] = len(m->v[i]);
  }
}

void po_integrate_begin(po_model *m) {
  const po_scene *s = &m->s;
  /* DEMModel::init: the first contact list (demModel.cpp:181-189) */
  if (s->multi_particle && contact_params(m)) contact_search(m, m->search0);
  /* DEMModel::integrate prelude (:277-283) */
  if (s->ic_active)
    for (int64_t p = 0; p < m->Np; p++)
      if (s->ic_particle[p])
        for (int64_t i = s->p_start[p]; i < s->p_end[p]; i++)
          m->v[i] = P3(s->ic_v[0], s->ic_v[1], s->ic_v[2]);
  displacement_bc(m);
  compute_forces(m);
}

void po_step(po_model *m, int64_t nsteps) {
  const po_scene *s = &m->s;
  for (int64_t k = 0; k < nsteps; k++) {
    if (s->time_scheme == 1) {
      /* DEMModel::integrateVerlet (:392-460) */
      integrate_kick_drift(m, 0.5);
      m->n++;
      m->time += s->dt;
      displacement_bc(m);
      compute_forces(m);
      for (int64_t i = 0; i < m->N; i++) {
        if (!m->active[i]) continue;
        const double rho = s->p_density[s->ptid[i]];
        for (int dof = 0; dof < s->dim; dof++)
          if (!((s->fix[i] >> dof) & 1u))
            setc(&m->v[i], dof, comp(m->v[i], dof) + 0.5 * (s->dt / rho) * comp(m->f[i], dof));
        m->vmag[i] = len(m->v[i]);
      }
    } else {
      /* DEMModel::integrateCD (:349-390) */
      integrate_kick_drift(m, 1.0);
      m->n++;
      m->time += s->dt;
      displacement_bc(m);
      compute_forces(m);
    }
    postprocess(m);
  }
}

double *po_x(po_model *m) { return (double *)m->x; }
double *po_u(po_model *m) { return (double *)m->u; }
double *po_v(po_model *m) { return (double *)m->v; }
double *po_f(po_model *m) { return (double *)m->f; }
float *po_Z(po_model *m) { return m->Z; }
double *po_theta(po_model *m) { return m->theta; }
double *po_vmag(po_model *m) { return m->vmag; }
uint8_t *po_bonds(po_model *m) { return m->bonds; }
int64_t po_n(po_model *m) { return m->n; }
double po_time(po_model *m) { return m->time; }

void po_contact_state(po_model *m, int64_t *interval, int64_t *counter, double *radius,
                      double *max_velocity) {
  if (interval) *interval = m->interval;
  if (counter) *counter = m->counter;
  if (radius) *radius = m->radius;
  if (max_velocity) *max_velocity = m->max_velocity;
}

int64_t po_contact_entries(po_model *m) { return m->c_row[m->N]; }

void po_contact_lists(po_model *m, uint64_t *rowptr, uint64_t *col) {
  for (int64_t i = 0; i <= m->N; i++) rowptr[i] = (uint64_t)m->c_row[i];
  if (col)
    for (int64_t k = 0; k < m->c_row[m->N]; k++) col[k] = (uint64_t)m->c_col[k];
}

void po_test_values(po_model *m, double *reaction, double *penetration, double *contact_reaction,
                    double *pen_dist, double *max_y) {
  if (reaction) *reaction = m->reaction;
  if (penetration) *penetration = m->penetration;
  if (contact_reaction) *contact_reaction = m->contact_reaction;
  if (pen_dist) *pen_dist = m->pen_dist;
  if (max_y) *max_y = m->max_y;
}

/* DEMModel::updatePeridynamicNeighborlist (demModel.cpp:1659-1694):
 * same particle, j != i, strict sum_d (x_i - x_j)^2 < horizon^2; lists in
 * node order. */
static int pd_hit(const po_scene *s, int64_t i, int64_t j) {
  if (j == i || s->ptid[j] != s->ptid[i]) return 0;
  const double r = s->p_horizon[s->ptid[i]];
  const double d0 = s->xref[3 * i] - s->xref[3 * j];
  const double d1 = s->xref[3 * i + 1] - s->xref[3 * j + 1];
  const double d2 = s->xref[3 * i + 2] - s->xref[3 * j + 2];
  double dd = 0.;
  dd += d0 * d0;
  dd += d1 * d1;
  dd += d2 * d2;
  return dd < r * r;
}

int64_t po_count_pd_neighbors(const po_scene *s) {
  int64_t c = 0;
  for (int64_t p = 0; p < s->n_particles; p++)
    for (int64_t i = s->p_start[p]; i < s->p_end[p]; i++)
      for (int64_t j = s->p_start[p]; j < s->p_end[p]; j++) c += pd_hit(s, i, j);
  return c;
}

void po_build_pd_neighbors(const po_scene *s, uint64_t *rowptr, uint64_t *col) {
  int64_t e = 0;
  for (int64_t i = 0; i < s->n_nodes; i++) {
    rowptr[i] = (uint64_t)e;
    const int64_t p = (int64_t)s->ptid[i];
    for (int64_t j = s->p_start[p]; j < s->p_end[p]; j++)
      if (pd_hit(s, i, j)) col[e++] = (uint64_t)j;
  }
  rowptr[s->n_nodes] = (uint64_t)e;
}

/* material::computeStateMxI (materialUtil.cpp:21-73) */
void po_compute_mx(const po_scene *s, double *mx) {
  for (int64_t i = 0; i < s->n_nodes; i++) {
    const int64_t p = (int64_t)s->ptid[i];
    const double horizon = s->p_horizon[p], h = s->p_h[p];
    const double up = horizon + 0.5 * h, low = horizon - 0.5 * h;
    const pt xi = node(s->xref, i);
    double m = 0.;
    for (uint64_t k = s->pd_rowptr[i]; k < s->pd_rowptr[i + 1]; k++) {
      const int64_t j = (int64_t)s->pd_col[k];
      const double rji = len(sub(node(s->xref, j), xi));
      if (is_greater(rji, horizon)) continue;
      double volj = s->vol[j];
      if (is_greater(rji, low)) volj *= (up - rji) / h;
      m += pow(rji, 2) * infl(s, rji, horizon) * volj;
    }
    mx[i] = m;
  }
}
