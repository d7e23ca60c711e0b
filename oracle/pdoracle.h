/*
 * pdoracle — a plain-C, single-threaded restatement of the reference's
 * explicit step (model::DEMModel, src/model/dem/demModel.cpp), used as the
 * CPU checker of the CUDA path.
 *
 * ORACLE TEST INFRASTRUCTURE ONLY: tests, the smoke check and the CPU
 * baseline of the benchmark call it; the product library never does.
 *
 * The model keeps the reference's arithmetic order operation by operation
 * (compiled with -ffp-contract=off, like the reference's x86-64 build), so
 * for the same neighbour-list order it reproduces the reference's results;
 * contact candidate lists are rebuilt here by brute force in node order.
 */
#ifndef PDORACLE_H
#define PDORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct po_bc {
  int32_t time_fn, spatial_fn, dir_mask, zero;
  double time_params[4];
  double spatial_params[2];
  const uint8_t *particle_sel; /* [Np] */
  const uint8_t *node_sel;     /* [N]  */
  const double *particle_box;  /* [Np*6] */
} po_bc;

/* The scene as ModelData holds it after DEMModel::init. */
typedef struct po_scene {
  int32_t dim, time_scheme, multi_particle, test;
  double dt;
  double gravity[3];
  int64_t n_nodes, n_particles;
  const double *xref, *vol; /* [N*3], [N] */
  const uint8_t *fix;       /* [N] */
  const uint64_t *ptid;     /* [N] */
  /* particles */
  const int64_t *p_start, *p_end, *p_center;
  const int32_t *p_type, *p_zone, *p_compute_force, *p_all_fixed, *p_material;
  const double *p_horizon, *p_h, *p_density, *p_rc, *p_kn, *p_bound_r;
  const double *p_mat; /* [Np*6] */
  int32_t inf_type;
  double inf_params[2];
  /* contact */
  int32_t n_zones;
  const double *c_rc, *c_kn, *c_mu, *c_betan, *c_kappa;
  double max_contact_r, search_factor;
  int64_t search_interval;
  /* test */
  int64_t test_wall, test_interval;
  int32_t test_dir;
  /* bonds (CSR) and weighted volume */
  const uint64_t *pd_rowptr, *pd_col;
  const double *mx;
  /* boundary conditions and initial condition */
  int32_t n_ubc, n_fbc;
  const po_bc *ubc, *fbc;
  int32_t ic_active;
  double ic_v[3];
  const uint8_t *ic_particle; /* [Np] */
} po_scene;

typedef struct po_model po_model;

po_model *po_create(const po_scene *s);
void po_destroy(po_model *m);
void po_integrate_begin(po_model *m);
void po_step(po_model *m, int64_t nsteps);

/* state access (pointers stay valid for the model's lifetime) */
double *po_x(po_model *m);
double *po_u(po_model *m);
double *po_v(po_model *m);
double *po_f(po_model *m);
float *po_Z(po_model *m);
double *po_theta(po_model *m);
double *po_vmag(po_model *m);
uint8_t *po_bonds(po_model *m);
int64_t po_n(po_model *m);
double po_time(po_model *m);
/* contact control and post-processing results */
void po_contact_state(po_model *m, int64_t *interval, int64_t *counter, double *radius,
                      double *max_velocity);
int64_t po_contact_entries(po_model *m);
void po_contact_lists(po_model *m, uint64_t *rowptr, uint64_t *col);
void po_test_values(po_model *m, double *reaction, double *penetration, double *contact_reaction,
                    double *pen_dist, double *max_y);

/* set-up helpers restated from the reference */
int64_t po_count_pd_neighbors(const po_scene *s);
void po_build_pd_neighbors(const po_scene *s, uint64_t *rowptr, uint64_t *col);
void po_compute_mx(const po_scene *s, double *mx);

#ifdef __cplusplus
}
#endif

#endif
