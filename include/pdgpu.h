/*
 * pdgpu — B200 (sm_100a) explicit time step for PeriDEM, behind a plain C ABI.
 *
 * The entry points below replace, one for one, the virtual steps of the
 * reference's model::DEMModel (src/model/dem/demModel.h:74-233): a host-side
 * DEMModel subclass keeps the reference's own set-up (DEMModel::init), copies
 * ModelData into a context with the pdgpu_upload_* calls, and from then on
 * calls pdgpu_integrate_begin / pdgpu_step instead of
 * DEMModel::integrate / integrateStep.  All arrays are the reference's own
 * layouts: node vectors are util::Point (3 contiguous doubles, also in 2-D),
 * indices are size_t (uint64), fixity is the uint8 bit mask of
 * ModelData::d_fix.
 *
 * Every call returns PDGPU_OK (0) or a negative PDGPU_ERR_* code; the message
 * of the last failure is available from pdgpu_last_error().  The library owns
 * all device memory; it copies caller buffers on upload and writes caller
 * buffers on download, and keeps no caller pointer.  One context is used by
 * one host thread at a time; work runs on the context's own CUDA stream.
 */
#ifndef PDGPU_H
#define PDGPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PDGPU_API __attribute__((visibility("default")))
#else
#define PDGPU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define PDGPU_OK 0
#define PDGPU_ERR_ARG (-1)      /* bad argument or call order */
#define PDGPU_ERR_CUDA (-2)     /* a CUDA runtime call failed */
#define PDGPU_ERR_NOMEM (-3)    /* device allocation failed */
#define PDGPU_ERR_OVERFLOW (-4) /* a device list outgrew its capacity */
#define PDGPU_ERR_NAN (-5)      /* non-finite force or position detected */
#define PDGPU_ERR_STATE (-6)    /* context not ready for this call */
#define PDGPU_ERR_NODEVICE (-7) /* no CUDA device / wrong architecture */

/* material laws (src/material/mparticle/material.h) */
#define PDGPU_MAT_RNP 0       /* RnpMaterial, "RNPBond" (material.h:251-659)     */
#define PDGPU_MAT_PMB 1       /* PmbMaterial, "PMBBond" (material.h:665-1019)    */
#define PDGPU_MAT_PDELASTIC 2 /* PdElastic, "PDElasticBond" (material.h:1025-1324) */
#define PDGPU_MAT_PDSTATE 3   /* PdState, "PDState" (material.h:1330-1724)       */

/* influence functions (src/material/mparticle/influenceFn.cpp:13-122) */
#define PDGPU_INF_CONST 0
#define PDGPU_INF_LINEAR 1
#define PDGPU_INF_GAUSSIAN 2

/* time functions of a boundary-condition set (particleULoading.cpp:115-230,
 * particleFLoading.cpp:85-173) */
#define PDGPU_TIME_CONSTANT 0
#define PDGPU_TIME_LINEAR 1
#define PDGPU_TIME_QUADRATIC 2
#define PDGPU_TIME_SIN 3
#define PDGPU_TIME_ROTATION 4
#define PDGPU_TIME_LINEAR_STEP 5
#define PDGPU_TIME_LINEAR_SLOW_FAST 6

/* spatial functions of a boundary-condition set */
#define PDGPU_SPACE_CONSTANT 0
#define PDGPU_SPACE_HAT_X 1
#define PDGPU_SPACE_HAT_Y 2
#define PDGPU_SPACE_SIN_X 3
#define PDGPU_SPACE_SIN_Y 4
#define PDGPU_SPACE_LINEAR_X 5
#define PDGPU_SPACE_LINEAR_Y 6

/* post-processing test (DEMModel::integrate, demModel.cpp:304-313) */
#define PDGPU_TEST_NONE 0
#define PDGPU_TEST_TWO_PARTICLE 1
#define PDGPU_TEST_COMPRESSIVE 2

/* arithmetic of the bond loop */
#define PDGPU_PREC_FP64 0  /* plain FP64 everywhere: the drop-in form */
#define PDGPU_PREC_MIXED 1 /* FP32 bond loop on particle-local coordinates,
                              FP64 integration and reductions */

/* fields for pdgpu_download / pdgpu_upload_field */
#define PDGPU_FIELD_X 0       /* double[N*3] current position  (d_x)      */
#define PDGPU_FIELD_U 1       /* double[N*3] displacement      (d_u)      */
#define PDGPU_FIELD_V 2       /* double[N*3] velocity          (d_v)      */
#define PDGPU_FIELD_F 3       /* double[N*3] force density     (d_f)      */
#define PDGPU_FIELD_Z 4       /* float[N]    damage            (d_Z)      */
#define PDGPU_FIELD_VMAG 5    /* double[N]   |v|               (d_vMag)   */
#define PDGPU_FIELD_THETA 6   /* double[N]   dilatation        (d_thetaX) */
#define PDGPU_FIELD_MX 7      /* double[N]   weighted volume   (d_mX)     */
#define PDGPU_FIELD_BONDS 8   /* uint8[B]    1 = broken, in neighbour-list order */
#define PDGPU_FIELD_FIX 9     /* uint8[N]    fixity mask       (d_fix)    */

/* Context description: the scalar parts of the reference's ModelDeck,
 * ParticleDeck (gravity, neighbour search, test) and OutputDeck. */
typedef struct pdgpu_desc {
  int32_t dim;             /* ModelDeck::d_dim: 2 or 3 */
  int32_t time_scheme;     /* 0 central_difference, 1 velocity_verlet */
  int32_t precision;       /* PDGPU_PREC_* */
  int32_t device;          /* CUDA device ordinal */
  double dt;               /* ModelDeck::d_dt */
  double gravity[3];       /* ParticleDeck::d_gravity */
  int32_t multi_particle;  /* Input::isMultiParticle(): contact on/off */
  int32_t test;            /* PDGPU_TEST_* */
  int64_t test_wall;       /* ParticleDeck::d_particleIdCompressiveTest */
  int32_t test_dir;        /* ParticleDeck::d_particleForceDirectionCompressiveTest - 1 */
  int32_t pad0;
  int64_t test_interval;   /* OutputDeck::d_dtTestOut */
  double search_factor;    /* PNeighborDeck::d_sFactor */
  int64_t search_interval; /* PNeighborDeck::d_neighUpdateInterval */
  double max_contact_r;    /* ModelData::d_maxContactR (after setupContact) */
  /* Capacities (0 = library default: 64 candidates per searching node, at
   * least 2^20 entries; 2048 wall pairs per particle, at most 4096).  A list
   * that outgrows its capacity is not written past it: the step stops with
   * PDGPU_ERR_OVERFLOW, and pdgpu_last_error names the size needed; create
   * the context again with a larger capacity. */
  int64_t contact_capacity;   /* total contact candidate entries */
  int64_t wall_pair_capacity; /* particle-wall node pairs per particle */
} pdgpu_desc;

/* One particle or wall (particle::BaseParticle, baseParticle.cpp:60-189). */
typedef struct pdgpu_particle {
  int64_t glob_start;    /* d_globStart */
  int64_t glob_end;      /* d_globEnd */
  int64_t center_node;   /* d_globStart + RefParticle::getCenterNodeId() */
  int32_t type;          /* d_typeIndex: 0 particle, 1 wall */
  int32_t zone;          /* d_zoneId */
  int32_t compute_force; /* d_computeForce (after the two_particle override) */
  int32_t all_dofs_constrained; /* d_allDofsConstrained */
  int32_t material;      /* PDGPU_MAT_* */
  int32_t pad0;
  double horizon;        /* d_horizon */
  double h;              /* d_h (mesh size) */
  double density;        /* d_density */
  double rc;             /* d_Rc, internal contact radius of broken bonds */
  double kn;             /* d_Kn, internal contact stiffness */
  double bound_r;        /* d_geom_p->boundingRadius() */
  /* Bond-law constants of d_material_p:
   *   RNP:        {C, beta, rbar, invFactor, factorSc, irreversible(0/1)}
   *   PMB:        {c, s0}
   *   PDElastic:  {c}
   *   PDState:    {K, G, s0}                                            */
  double mat[6];
} pdgpu_particle;

/* One boundary-condition set (inp::PBCData, src/inp/pdecks/pBCData.h). */
typedef struct pdgpu_bc_set {
  int32_t time_fn;       /* PDGPU_TIME_* */
  int32_t spatial_fn;    /* PDGPU_SPACE_* */
  int32_t dir_mask;      /* bit d set = direction d+1 is in d_direction */
  int32_t zero;          /* d_isDisplacementZero */
  double time_params[4]; /* d_timeFnParams (unused entries 0) */
  double spatial_params[2];
} pdgpu_bc_set;

/* Scalars after the last step. */
typedef struct pdgpu_scalars {
  int64_t n;                     /* ModelData::d_n */
  double time;                   /* ModelData::d_time */
  double reaction;               /* last ppCompressiveTest reaction (reference definition) */
  double contact_reaction;       /* -sum over particle nodes of (contact force from the test wall)*vol */
  double wall_penetration;       /* last ppCompressiveTest penetration */
  double max_velocity;           /* ModelData::d_maxVelocity */
  double contact_search_radius;  /* d_contNeighSearchRadius */
  int64_t contact_update_interval; /* d_contNeighUpdateInterval */
  int64_t contact_counter;       /* d_contNeighTimestepCounter */
  int64_t contact_updates;       /* contact list rebuilds so far */
  int64_t contact_entries;       /* current contact candidate entries */
  int64_t broken_bonds;          /* bonds with the broken bit set */
  double pen_dist;               /* ppTwoParticleTest key data */
  double max_y;
  double contact_area_radius;
} pdgpu_scalars;

/* A zone's material deck (inp::MaterialDeck, src/inp/decks/materialDeck.h),
 * the values pdgpu_material_constants derives the bond-law constants from.
 * Values not given are negative, as in the deck. */
typedef struct pdgpu_material_deck {
  int32_t law;          /* PDGPU_MAT_* (d_materialType) */
  int32_t irreversible; /* d_irreversibleBondBreak */
  double E, K, G, nu;   /* d_matData.d_E, d_K, d_G, d_nu */
  double Gc;            /* d_matData.d_Gc */
  double check_sc_factor; /* d_checkScFactor */
} pdgpu_material_deck;

typedef struct pdgpu_ctx pdgpu_ctx;

/* Library / device check.  Returns PDGPU_OK when a device of compute
 * capability 10.0 is visible. */
PDGPU_API int pdgpu_device_check(int device, char *msg, size_t msg_len);

/* Deck-level constants for a host that holds only the input decks (no
 * device work; no counterpart call in the reference, whose material
 * constructors compute these into private members):
 *   pdgpu_influence_params: the influence function's two parameters from the
 *     deck's type and parameter list (influenceFn.cpp:13-85 defaults), as
 *     pdgpu_set_influence takes them;
 *   pdgpu_material_constants: pdgpu_particle.mat for a particle of the given
 *     horizon (RnpMaterial material.h:541-620, PmbMaterial :919-997,
 *     PdElastic :1257-1305, PdState :1579-1700, same evaluation order) and
 *     the bulk modulus BaseParticle uses for the internal contact stiffness
 *     of broken bonds (baseParticle.cpp:156-179). */
PDGPU_API int pdgpu_influence_params(int32_t type, int32_t n_params, const double *params, int32_t dim,
                                     double out[2]);
PDGPU_API int pdgpu_material_constants(const pdgpu_material_deck *deck, int32_t dim, double horizon,
                                       int32_t inf_type, const double inf_params[2], double mat[6],
                                       double *bulk_modulus);

/* Mesh size of every particle on the device (no context needed):
 * util::computeMeshSize (src/util/geom.cpp:578-604), the d_h that
 * BaseParticle sets (baseParticle.cpp:146) and from which the horizon and the
 * contact radii follow.  Same result as the reference's O(n^2) scan, record
 * for record: starting from |x_start - x_start+1|, the pairs of the
 * particle's nodes in (i, j) scan order replace the guess when
 * util::isLess(distance, guess).  x is a host array of n_nodes util::Points;
 * particle p owns nodes [particle_start[p], particle_end[p]); h receives
 * n_particles values (0 for a particle of fewer than two nodes).  Blocking;
 * allocates its scratch on `device` and frees it before returning. */
PDGPU_API int pdgpu_mesh_size(int32_t device, const double *x, int64_t n_nodes, const int64_t *particle_start,
                              const int64_t *particle_end, int64_t n_particles, double *h);

/* Context lifetime: the DEMModel constructor / destructor. */
PDGPU_API int pdgpu_create(const pdgpu_desc *desc, pdgpu_ctx **out);
PDGPU_API void pdgpu_destroy(pdgpu_ctx *ctx);
PDGPU_API int pdgpu_last_error(const pdgpu_ctx *ctx, char *buf, size_t len);

/* Node data after DEMModel::init (ModelData::d_xRef, d_x, d_u, d_v, d_vol,
 * d_fix, d_ptId; modelData.h:531-760).  Any of x/u/v may be NULL (x defaults
 * to xref, u and v to 0). */
PDGPU_API int pdgpu_upload_nodes(pdgpu_ctx *ctx, int64_t n_nodes, const double *xref, const double *x,
                       const double *u, const double *v, const double *vol, const uint8_t *fix,
                       const uint64_t *pt_id);

/* Particles and walls (ModelData::d_particlesListTypeAll). */
PDGPU_API int pdgpu_upload_particles(pdgpu_ctx *ctx, int64_t n_particles, const pdgpu_particle *particles);

/* The process-wide influence function (material.h:23-54). */
PDGPU_API int pdgpu_set_influence(pdgpu_ctx *ctx, int32_t type, const double params[2]);

/* Contact parameters per zone pair after DEMModel::setupContact
 * (demModel.cpp:1531-1600): row-major n_zones x n_zones arrays of
 * ContactPairDeck::d_contactR, d_Kn, d_mu, d_betan, d_kappa. */
PDGPU_API int pdgpu_upload_contact(pdgpu_ctx *ctx, int32_t n_zones, const double *rc, const double *kn,
                         const double *mu, const double *betan, const double *kappa);

/* Peridynamic neighbour lists (ModelData::d_neighPd) in CSR form, in the
 * caller's order; bond_state (optional) gives the geometry::Fracture bits
 * one byte per bond.  Replaces DEMModel::updatePeridynamicNeighborlist. */
PDGPU_API int pdgpu_upload_pd_neighbors(pdgpu_ctx *ctx, const uint64_t *rowptr, const uint64_t *col,
                              const uint8_t *bond_state);

/* Builds the peridynamic neighbour lists on the device instead
 * (DEMModel::updatePeridynamicNeighborlist, demModel.cpp:1659-1694, with the
 * kd-tree include-tag search of nsearch.h:340-364 replaced by a cell list;
 * same strict squared-distance test, so the same sets).  Lists are sorted
 * by node index. */
PDGPU_API int pdgpu_build_pd_neighbors(pdgpu_ctx *ctx);

/* Weighted volume m_x: upload (ModelData::d_mX) or compute on the device
 * (material::computeStateMx, materialUtil.cpp:211-245). */
PDGPU_API int pdgpu_upload_mx(pdgpu_ctx *ctx, const double *mx);
PDGPU_API int pdgpu_compute_mx(pdgpu_ctx *ctx);

/* Boundary conditions (ParticleULoading / ParticleFLoading).  particle_sel
 * [n_particles] is needToProcessParticle() per particle; node_sel [n_nodes]
 * is needToComputeDof() per node; particle_box [n_particles*6] is the box
 * (lo xyz, hi xyz) the spatial function uses for each particle. */
PDGPU_API int pdgpu_add_displacement_bc(pdgpu_ctx *ctx, const pdgpu_bc_set *set, const uint8_t *particle_sel,
                              const uint8_t *node_sel, const double *particle_box);
PDGPU_API int pdgpu_add_force_bc(pdgpu_ctx *ctx, const pdgpu_bc_set *set, const uint8_t *particle_sel,
                       const uint8_t *node_sel, const double *particle_box);

/* Initial condition (PICDeck; DEMModel::applyInitialCondition). */
PDGPU_API int pdgpu_set_initial_condition(pdgpu_ctx *ctx, const double velocity[3],
                                const uint64_t *particle_list, int64_t n_list);

/* Contact neighbour list of DEMModel::init (demModel.cpp:181-189): builds the
 * first contact candidate lists.  Call after all uploads. */
PDGPU_API int pdgpu_init_contact(pdgpu_ctx *ctx);

/* The prelude of DEMModel::integrate (demModel.cpp:277-283):
 * applyInitialCondition (if n == 0), computeExternalDisplacementBC,
 * computeForces. */
PDGPU_API int pdgpu_integrate_begin(pdgpu_ctx *ctx);

/* nsteps x (DEMModel::integrateStep + ppTwoParticleTest / ppCompressiveTest),
 * demModel.cpp:285-324.  Runs asynchronously on the context stream; errors
 * found on the device are reported by the next synchronising call. */
PDGPU_API int pdgpu_step(pdgpu_ctx *ctx, int64_t nsteps);

/* Same as pdgpu_step, issued as replays of a CUDA graph of `graph_steps`
 * steps captured on first use (kernels only; no host work per step). */
PDGPU_API int pdgpu_step_graph(pdgpu_ctx *ctx, int64_t nsteps, int32_t graph_steps);

/* Number of kernels one pdgpu_step step launches (counted from a captured
 * graph of one step; nothing runs). */
PDGPU_API int pdgpu_step_kernel_count(pdgpu_ctx *ctx, int64_t *count);

/* Waits for the context stream and reports device-side errors. */
PDGPU_API int pdgpu_sync(pdgpu_ctx *ctx);

/* Copies a field into a caller buffer (blocking). */
PDGPU_API int pdgpu_download(pdgpu_ctx *ctx, int32_t field, void *dst);

/* Overwrites u, v or x (N*3 doubles), or the bond state (PDGPU_FIELD_BONDS,
 * uint8[B], 1 = broken), from a caller buffer (blocking); used by the
 * host-buffer step below and by restarts. */
PDGPU_API int pdgpu_upload_field(pdgpu_ctx *ctx, int32_t field, const void *src);

/* DEMModel::output (demModel.cpp:1962-2024) with
 * rw::writer::VtkParticleWriter::appendNodes (vtkParticleWriter.cpp:39-270):
 * writes the current state to an XML UnstructuredGrid file `path` (.vtu):
 * the current positions as points (no cells), the model time as the field
 * array TIME, and one point array per tag named in the comma-separated
 * `tags` among Displacement, Velocity, Force_Density, Force (f vol), Fixity,
 * Particle_ID, Zone_ID, Nodal_Volume, Damage_Z, Theta (other tags are
 * ignored, as in the reference).  Data are appended raw (Float64, UInt64
 * block headers).  Blocking. */
PDGPU_API int pdgpu_write_vtu(pdgpu_ctx *ctx, const char *path, const char *tags);

/* DEMModel::output without stopping the step loop (no counterpart in the
 * reference, whose output blocks): the state as of this call (in stream
 * order) is copied on the device, downloaded on a stream of its own and
 * written by a host thread to `path`, exactly as pdgpu_write_vtu would; the
 * call returns at once and steps issued after it run meanwhile.  One file is
 * in flight at a time (a second call waits for the first);
 * pdgpu_output_wait waits for it and reports its status. */
PDGPU_API int pdgpu_write_vtu_async(pdgpu_ctx *ctx, const char *path, const char *tags);
PDGPU_API int pdgpu_output_wait(pdgpu_ctx *ctx);

/* DEMModel::restart (demModel.cpp:84-102) with
 * rw::reader::VtkParticleReader::readNodes (vtkParticleReader.cpp:41-120):
 * reads the points (current positions), Displacement (else x - x_ref) and
 * Velocity of a file written by pdgpu_write_vtu, and makes
 * pdgpu_integrate_begin resume at `step` (time step * dt; no initial
 * condition; the contact-search counter of the restart step as in
 * demModel.cpp:1833-1837).  Like the reference, the bond states are not
 * restored from the file; a host that keeps them saves them with
 * pdgpu_download(PDGPU_FIELD_BONDS) and writes them back with
 * pdgpu_upload_field (or passes them to pdgpu_upload_pd_neighbors) before
 * pdgpu_integrate_begin.  Call before pdgpu_integrate_begin. */
PDGPU_API int pdgpu_restart(pdgpu_ctx *ctx, const char *path, int64_t step);

/* State snapshot: a restart that keeps everything (no counterpart in the
 * reference, whose DEMModel::restart, demModel.cpp:84-102, restores positions
 * and velocities only and resets every bond to intact).
 *
 * pdgpu_save_state writes, between steps (after pdgpu_integrate_begin),
 * everything a step reads that earlier steps wrote: x, u, v, f, Z, |v|,
 * dilatation, the bond-broken bits, the step and time, the contact-search
 * control, the contact candidate lists and particle-wall damping pairs of
 * the last rebuild, the compressive-test history and the learned
 * surrogate's per-particle flags.  Blocking.  The file starts with a
 * portable part that any host can read without this library: a fixed
 * header (step, time, contact-search interval, counter, radius, max
 * velocity), x, u, v as util::Point arrays, and the broken bonds as (i, j)
 * node pairs, independent of neighbour-list order.
 *
 * pdgpu_load_state takes the place of pdgpu_integrate_begin on a context
 * with the same scene uploaded (same nodes, bonds, particles, contact
 * capacities; either precision): the context continues exactly as the saved
 * one would have.  A file of another scene is refused with PDGPU_ERR_ARG. */
PDGPU_API int pdgpu_save_state(pdgpu_ctx *ctx, const char *path);
PDGPU_API int pdgpu_load_state(pdgpu_ctx *ctx, const char *path);

/* DEMModel::computePeridynamicForces (demModel.cpp:602-789) alone on the
 * current state: the state-based pre-pass and the bond loop write the
 * peridynamic force density f and damage Z and may break bonds; contact,
 * damping and external forces are not added.  Blocking. */
PDGPU_API int pdgpu_compute_pd_forces(pdgpu_ctx *ctx);

/* One reference-facing step on host buffers, as a DEMModel::integrateStep
 * override that keeps ModelData on the host: uploads u, v, x from the caller
 * (N*3 doubles each), runs nsteps steps, downloads u, v, x and f back into
 * the same buffers, and fills *out (may be NULL). */
PDGPU_API int pdgpu_step_host(pdgpu_ctx *ctx, double *u, double *v, double *x, double *f, int64_t nsteps,
                    pdgpu_scalars *out);

PDGPU_API int pdgpu_get_scalars(pdgpu_ctx *ctx, pdgpu_scalars *out);

/* The ppCompressiveTest history (time, wall penetration, reaction) recorded
 * every test_interval steps; writes up to cap rows, sets *count to the
 * number recorded so far. */
PDGPU_API int pdgpu_get_history(pdgpu_ctx *ctx, double *t, double *delta, double *force,
                      double *contact_force, int64_t cap, int64_t *count);

/* Contact candidate lists (ModelData::d_neighC) in CSR form: rowptr has
 * N+1 entries; col must hold scalars.contact_entries entries. */
PDGPU_API int pdgpu_download_contact(pdgpu_ctx *ctx, uint64_t *rowptr, uint64_t *col);

/* Peridynamic neighbour lists as held on the device. */
PDGPU_API int pdgpu_num_bonds(pdgpu_ctx *ctx, int64_t *n_bonds);
PDGPU_API int pdgpu_download_pd_neighbors(pdgpu_ctx *ctx, uint64_t *rowptr, uint64_t *col);

/* Launch shape of the bond loop and the contact kernel: lanes per node
 * (4, 8, 16 or 32 for the bond loop, also 1 or 2 in the mixed form; 1, 2,
 * 4, 8 or 32 for the contact pass, default 1).  With 1 the contact pass is
 * one warp-cooperative kernel: a warp walks the candidate entries of 32
 * nodes, coalesced, and each node's lane adds its contributions in list
 * order; with more, a flat distance pass marks the entries inside the
 * largest contact radius and a node pass sums them with that many lanes
 * per node.  0 keeps the current choice.  Set before the first step. */
PDGPU_API int pdgpu_set_tuning(pdgpu_ctx *ctx, int32_t pd_lanes, int32_t contact_lanes);

/* CTAs per SM of the contact node pass (1..16, default 2); it runs beside
 * the bond loop and is bound by the latency of its gathers.  Set before the
 * first step. */
PDGPU_API int pdgpu_set_contact_grid(pdgpu_ctx *ctx, int32_t ctas_per_sm);

/* Nodes per bond-loop tile (one CTA each); 0 = automatic.  Set before the
 * first step; tiles shrink by themselves when a window outgrows shared
 * memory. */
PDGPU_API int pdgpu_set_tile_nodes(pdgpu_ctx *ctx, int32_t nodes);

/* How the mixed-precision bond loop visits bonds (no counterpart in the
 * reference): 0 (default) evaluates every bond from both ends, a tile's
 * nodes in node order; 2 the same with each tile's nodes taken longest row
 * first (results identical to 0); 1 (2-D) evaluates a bond whose two nodes
 * share a tile once and hands the far node its share through shared memory
 * (where rows and tiles fit its 16-bit layout: fewer bond evaluations, but
 * more shared memory per tile and a barrier between the two halves).  Set
 * before the first step.  pdgpu_bond_scheme reports the one in use (it
 * prepares the context). */
PDGPU_API int pdgpu_set_bond_scheme(pdgpu_ctx *ctx, int32_t scheme);
PDGPU_API int pdgpu_bond_scheme(pdgpu_ctx *ctx, int32_t *scheme);

/* The context's CUDA stream (a cudaStream_t) for callers that time work. */
PDGPU_API int pdgpu_get_stream(pdgpu_ctx *ctx, void **stream);

/* Per-kernel device time accumulated since the last reset (CUDA events
 * around each launch when enabled); names are static strings. */
PDGPU_API int pdgpu_enable_timing(pdgpu_ctx *ctx, int32_t on);
PDGPU_API int pdgpu_kernel_times(pdgpu_ctx *ctx, int32_t max_kernels, const char **names, double *ms,
                       int64_t *launches, int32_t *count);

/* Strain and stress at the quadrature points of linear triangles (2-D) from
 * the context's current displacement: the Strain_Stress output of
 * DEMModel::output (demModel.cpp:2026-2072), i.e. fe::getCurrentQuadPoints
 * and fe::getStrainStress (fe/meshUtil.cpp:170-420) with
 * fe::TriElem::getQuadDatas (fe/triElem.cpp:60-95), evaluated on the GPU in
 * the reference's order (strain and stress as 32-bit floats, as
 * util::SymMatrix3 keeps them, returned widened to double).  conn[3e..3e+2]
 * are element e's global node ids; ref_points (xi, eta per point) the
 * reference-triangle quadrature points, nq = 1 or 3 (the reference's rules of
 * order 1 and 2); nu, lambda, mu and plane_strain per element (the
 * particle material's Material::computeMaterialProperties and deck flag).
 * Writes three entries per element, as the reference stores them (entries
 * past the rule's points zero): xq[3 (3e + q) + c] the current position,
 * strain and stress[6 (3e + q) + k] with k = xx, yy, zz, yz, xz, xy.
 * Synchronous; host buffers. */
PDGPU_API int pdgpu_strain_stress_tri(pdgpu_ctx *ctx, int64_t n_elements, const int64_t *conn, int32_t nq,
                                      const double *ref_points, const double *nu, const double *lambda,
                                      const double *mu, const uint8_t *plane_strain, double *xq, double *strain,
                                      double *stress);

/* The same for linear tetrahedra (3-D, conn[4e..4e+3]) with the one-point
 * rule (the centroid), the reference's only tetrahedron rule that fits the
 * three entries it stores per element (fe::TetElem, fe/tetElem.cpp: J^-1 by
 * util::inv, derivatives by util::dot); entries 1 and 2 of each element zero. */
PDGPU_API int pdgpu_strain_stress_tet(pdgpu_ctx *ctx, int64_t n_elements, const int64_t *conn, const double *nu,
                                      const double *lambda, const double *mu, double *xq, double *strain,
                                      double *stress);

/* The file VtkParticleWriter::appendStrainStress writes
 * (vtkParticleWriter.cpp:444-495, output_strain_<n>.vtu): the quadrature
 * points as points (no cells), point arrays Strain and Stress of six
 * components named xx, yy, zz, yz, xz, xy, and the context's time as TIME,
 * as raw appended VTK XML (pdgpu_write_vtu's format). */
PDGPU_API int pdgpu_write_strain_vtu(pdgpu_ctx *ctx, const char *path, int64_t n_points, const double *xq,
                                     const double *strain, const double *stress);

/* Phase clock of the contact-list rebuild (a profiling aid): with on != 0
 * every later rebuild records the GPU global timer (ns) as its first CTA
 * passes each grid-wide barrier, in order: start, cells cleared, nodes
 * counted per cell, cell offsets scanned, nodes scattered, cells sorted,
 * candidates counted, row offsets scanned, compaction offsets scanned,
 * lists compacted, and the first CTA's share of the fill done (11 marks).
 * pdgpu_rebuild_phases copies the marks of the latest rebuild (up to cap)
 * and sets *count. */
PDGPU_API int pdgpu_enable_rebuild_phases(pdgpu_ctx *ctx, int32_t on);
PDGPU_API int pdgpu_rebuild_phases(pdgpu_ctx *ctx, int64_t *ns, int32_t cap, int32_t *count);

/* A batched ensemble (no counterpart in the reference, which runs one scene
 * per process): the uploaded nodes and particles hold n_scenes independent
 * scenes, each a contiguous run of particles (particle_offsets, n_scenes + 1
 * entries from 0 to the particle count; nodes follow their particles), far
 * enough apart that no contact candidate joins two scenes, with zone ids
 * distinct per scene and a block-diagonal contact table.  All scenes share
 * dt and advance together: one bond-loop launch over every scene's tiles,
 * one contact pass, one graph per step.  Particle damping pairs stay within
 * a scene.  test_walls[s] is the particle of scene s whose compressive-test
 * output (ppCompressiveTest: time, wall displacement, reaction sum f vol,
 * contact reaction) is recorded every test_interval steps (-1: none), in
 * test_dir; up to 4096 records per scene.  Call before the first step. */
PDGPU_API int pdgpu_set_scenes(pdgpu_ctx *ctx, int32_t n_scenes, const int64_t *particle_offsets,
                               const int64_t *test_walls);

/* The compressive-test records of one scene of an ensemble (like
 * pdgpu_get_history); *count = records so far (at most 4096). */
PDGPU_API int pdgpu_get_scene_history(pdgpu_ctx *ctx, int32_t scene, double *t, double *delta, double *force,
                                      double *cforce, int64_t cap, int64_t *count);

/* Building block of the learned surrogate (no counterpart in the
 * reference): C = act(A B^T + bias) on the tensor cores (tcgen05, BF16
 * operands, FP32 accumulation).  A is M x K and B is N x K, both row-major
 * BF16 device arrays with K contiguous (lda, ldb in elements, multiples of
 * 8); K and N multiples of 16.  bias (N floats) may be NULL; act 0 = none,
 * 1 = tanh.  C (ldc) is written as FP32 (Cf) and/or BF16 (Cb).  *err (device
 * int) is set to 1 if the kernel's bounded waits time out.  Asynchronous on
 * `stream`. */
PDGPU_API int pdgpu_tc_gemm(const void *A, int32_t lda, const void *B, int32_t ldb, int32_t M, int32_t N,
                            int32_t K, const float *bias, int32_t act, float *Cf, void *Cb, int32_t ldc,
                            int32_t *err, void *stream);

/* The learned surrogate of the bond loop (no counterpart in the reference;
 * mixed-precision form, 2-D).  Per zone ("shape": particles sharing a
 * reference mesh, scaled and rotated), a particle's displacement in its body
 * frame, u_b = R(-orient) (u_i - u_centre) / scale (2 n_nodes values in the
 * particle's node order), is projected on 32 displacement modes (phi_t,
 * 32 x 2 n_nodes) to x, mapped by an MLP 32-256-256-32 (tanh, tanh, linear;
 * weights W[out][in]) to y, and [y, x] is lifted (psi, 2 n_nodes x 64: the
 * force modes of the network's output, then the tangent force of each
 * displacement mode) to the body-frame force f_b; f_i = fscale R(orient) f_b.
 * Zero deformation gives exactly zero force (the chain's output for a zero
 * input is subtracted).  Every check_interval steps the bond loop runs for
 * all particles; a particle then keeps the surrogate until the next check
 * only if none of its bonds is broken, its damage Z stays below z_gate
 * (0.5 = half the critical stretch) and |f_surrogate - f| < err_gate
 * max(|f|, floor).  With near_gate != 0 a particle also stays on the bond
 * loop while the last contact-list rebuild found contact candidates of its
 * nodes (within contact radius plus skin, so no contact starts on a
 * surrogate particle).  Per-particle arrays fscale, floor, orient, scale are
 * indexed by particle.  All arrays are host FP32/FP64 and are copied
 * (weights to BF16).  Call once, before pdgpu_integrate_begin. */
typedef struct {
  int32_t zone, n_nodes;
  const float *phi_t, *psi;
  const float *w1, *b1; /* 256 x 32, 256 */
  const float *w2, *b2; /* 256 x 256, 256 */
  const float *w3, *b3; /* 32 x 256, 32 */
} pdgpu_sur_shape;

PDGPU_API int pdgpu_set_surrogate(pdgpu_ctx *ctx, int32_t n_shapes, const pdgpu_sur_shape *shapes,
                                  const double *fscale, const double *floor, const double *orient,
                                  const double *scale, int32_t check_interval, double z_gate,
                                  double err_gate, int32_t near_gate);

/* Which kernels evaluate the surrogate in the step (call before
 * pdgpu_set_surrogate; no counterpart in the reference): 0 (default) CUDA
 * cores, four launches per step — gather with projection, the three layers,
 * and the lift with the scatter into f beside the bond loop; 1 the tcgen05
 * GEMMs the training uses (projection, layers and lift as grouped GEMMs, the
 * scatter after the bond loop).  Both take BF16 operands with FP32
 * accumulation and round activations to BF16; they differ in summation
 * order only. */
PDGPU_API int pdgpu_set_surrogate_chain(pdgpu_ctx *ctx, int32_t kind);

/* Particles on the surrogate now and particles it covers; and, summed over
 * the steps so far, particle-steps whose force came from the surrogate and
 * particle-steps of the particles it covers. */
PDGPU_API int pdgpu_surrogate_stats(pdgpu_ctx *ctx, int64_t *n_on, int64_t *n_total, int64_t *steps_on,
                                    int64_t *steps_total);

/* The last check step's comparison per particle: err2[2p] = sum over the
 * particle's nodes of |f_surrogate - f|^2, err2[2p + 1] = sum of |f|^2 (f the
 * bond loop's force density); zeros outside the surrogate's zones.
 * n = 2 x number of particles. */
PDGPU_API int pdgpu_surrogate_errors(pdgpu_ctx *ctx, double *err2, int64_t n);

/* Training building blocks of the surrogate on caller-owned device arrays
 * (no counterpart in the reference), asynchronous on `stream`:
 *   mse_grad:   dY = scale (Y - T) as FP32 and BF16; *loss += sum (Y - T)^2
 *   tanh_back:  dZ = dH (1 - H^2) as FP32 and BF16 (H = tanh of the layer)
 *   colsum:     out[c] = sum_r X[r][c] (bias gradients; X rows x cols FP32)
 *   transpose:  out (cols x rows) = in (rows x cols)^T, BF16
 *   adam:       Adam step `step` (1-based) on FP32 p with moments m, v;
 *               wb (may be NULL) receives p as BF16 */
PDGPU_API int pdgpu_sur_mse_grad(const float *Y, const float *T, int64_t n, float scale, float *dY, void *dYb,
                                 double *loss, void *stream);
PDGPU_API int pdgpu_sur_tanh_back(const float *dH, const float *H, int64_t n, float *dZ, void *dZb, void *stream);
PDGPU_API int pdgpu_sur_colsum(const float *X, int32_t rows, int32_t cols, float *out, void *stream);
PDGPU_API int pdgpu_sur_transpose(const void *in, int32_t rows, int32_t cols, void *out, void *stream);
PDGPU_API int pdgpu_sur_adam(float *p, float *m, float *v, const float *g, int64_t n, float lr, float beta1,
                             float beta2, float eps, int32_t step, void *wb, void *stream);

/* Peridynamic neighbour lists built WITHOUT ANY DEVICE ALLOCATION, for
 * callers that cannot call cudaMalloc: a host whose device memory is held by
 * another allocator (a framework's caching allocator that owns the GPU), or
 * a code path where allocation is not allowed.  No counterpart in the
 * reference (its kd-tree search is host code).
 *
 * Inputs and outputs are caller-owned DEVICE buffers: x (n_nodes*3 doubles,
 * util::Point layout), particle (n_nodes particle ids), horizon (one per
 * particle id); rowptr receives n_nodes+1 offsets and col up to col_capacity
 * neighbour indices.  The sets equal pdgpu_build_pd_neighbors' (same
 * particle, j != i, strict |x_i - x_j|^2 < horizon^2), rows ascending.
 * Pass col = NULL to learn the size in *n_bonds.
 *
 * The call BLOCKS THE HOST: work runs on `stream` (a cudaStream_t, NULL =
 * the default stream), and the call waits for that stream three times and
 * returns when the lists are written.  It cannot be captured into a CUDA
 * graph: it returns PDGPU_ERR_STATE when `stream` is capturing (or, for the
 * default stream, when another stream captures in global mode); a host with
 * a capture in progress passes a non-default stream that is not capturing.
 *
 * Limits: n_nodes <= 262144; at most 1024 neighbours per node (the size
 * query already returns PDGPU_ERR_OVERFLOW beyond that); at most 8192 nodes
 * in one grid cell of the search (cells are about one horizon wide, and
 * grow coarser when the domain spans more than 2^20 of them; a sparse
 * domain that crowds more nodes into one cell is refused with
 * PDGPU_ERR_ARG).  Scratch is a 16 MiB static device array that every GPU
 * loading this library keeps until the process exits; the first call on a
 * device looks its address up, and the call must not be used on a device
 * after cudaDeviceReset in the same process.  All calls share that array,
 * so calls that overlap on the GPU race.  Errors come back as a code and a
 * message in err. */
PDGPU_API int pdgpu_build_neighbors_noalloc(const double *x, const uint32_t *particle,
                                            const double *horizon, int64_t n_nodes, int32_t dim,
                                            uint64_t *rowptr, uint32_t *col, int64_t col_capacity,
                                            int64_t *n_bonds, void *stream, char *err,
                                            size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* PDGPU_H */
