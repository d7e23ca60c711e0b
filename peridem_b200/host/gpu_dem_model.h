// gpu_dem_model.h — model::GpuDEMModel, the drop-in subclass of PeriDEM's
// model::DEMModel (src/model/dem/demModel.h:74-233) that runs the explicit
// step on a B200 through libpdgpu (include/pdgpu.h).
//
// The reference's own DEMModel::init sets the scene up (decks, meshes,
// particles, materials, neighbour lists, m_x, loading); integrate() then
// copies ModelData into a pdgpu context once and advances it on the GPU.
// Between the test-output and output steps the device runs on its own; at
// those steps the state is copied back into ModelData and the reference's
// own ppTwoParticleTest / ppCompressiveTest / output run on it, as in
// DEMModel::integrate (demModel.cpp:268-340).
//
// Nothing in the reference is modified: every member read here is public,
// and the bond-law constants (private in the material classes) are derived
// from the zones' material decks by pdgpu_material_constants, then checked
// against each live material's public getSc().
//
// Build: include this header after the reference's headers are on the
// include path (src/, external/, external/fmt/include) with include/ of this
// repository; link libpdgpu.so.
#ifndef PDGPU_GPU_DEM_MODEL_H
#define PDGPU_GPU_DEM_MODEL_H

#include "model/dem/demModel.h"
#include "particle/baseParticle.h"
// the decks read below (after demModel.h, which brings in what they use)
#include "inp/decks/materialDeck.h"
#include "inp/decks/modelDeck.h"
#include "inp/decks/outputDeck.h"
#include "inp/pdecks/contactDeck.h"
#include "inp/pdecks/particleDeck.h"
#include "loading/particleULoading.h"
#include "material/mparticle/material.h"
#include "pdgpu.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

namespace model {

class GpuDEMModel : public DEMModel {
public:
  using DEMModel::DEMModel;

  // arithmetic of the bond loop (PDGPU_PREC_FP64 is the drop-in form)
  int32_t d_precision = PDGPU_PREC_FP64;
  // steps per CUDA-graph replay between host events
  int32_t d_graphSteps = 64;
  // a .vtu file (pdgpu_write_vtu) to write the final state into, if not empty
  std::string d_finalVtu;

  void integrate() override {
    upload();
    // integrate() prelude: applyInitialCondition, displacement BC, forces
    check(pdgpu_integrate_begin(d_ctx), "integrate_begin");
    download();
    if (d_outputDeck_p->d_performOut) output();
    const size_t Nt = d_modelDeck_p->d_Nt;
    const size_t test_every = std::max<size_t>(1, d_outputDeck_p->d_dtTestOut);
    const size_t out_every = std::max<size_t>(1, d_outputDeck_p->d_dtOut);
    const bool two_particle = d_pDeck_p->d_testName == "two_particle";
    const bool compressive = d_pDeck_p->d_testName == "compressive_test";
    while (d_n < Nt) {
      // advance on the device to the next step at which the host acts
      size_t next = Nt;
      if (two_particle || compressive) next = std::min(next, (d_n / test_every + 1) * test_every);
      if (d_outputDeck_p->d_performOut) next = std::min(next, (d_n / out_every + 1) * out_every);
      const size_t k = next - d_n;
      check(pdgpu_step_graph(d_ctx, (int64_t)k, (int32_t)std::min<size_t>(k, (size_t)d_graphSteps)),
            "step_graph");
      check(pdgpu_sync(d_ctx), "sync");
      pdgpu_scalars sc{};
      check(pdgpu_get_scalars(d_ctx, &sc), "get_scalars");
      d_n = (size_t)sc.n;
      d_time = sc.time;  // the device sums dt step by step, as the reference does
      const bool test_step = (two_particle || compressive) && d_n % test_every == 0;
      const bool out_step = d_outputDeck_p->d_performOut && d_n % out_every == 0;
      if (test_step || out_step || d_n >= Nt) download();
      // the reference's own post-processing on the downloaded state
      if (test_step && two_particle) ppTwoParticleTest();
      if (test_step && compressive) ppCompressiveTest();
      if (out_step) output();
    }
    if (!d_finalVtu.empty())
      check(pdgpu_write_vtu(d_ctx, d_finalVtu.c_str(),
                            "Displacement,Velocity,Force_Density,Force,Damage_Z,Particle_ID,Nodal_Volume"),
            "write_vtu");
    pdgpu_destroy(d_ctx);
    d_ctx = nullptr;
  }

private:
  pdgpu_ctx *d_ctx = nullptr;

  void check(int rc, const char *what) {
    if (rc == PDGPU_OK) return;
    char buf[512] = {0};
    if (d_ctx) pdgpu_last_error(d_ctx, buf, sizeof buf);
    std::cerr << "pdgpu: " << what << " failed (" << rc << "): " << buf << "\n";
    std::exit(1);
  }

  void upload() {
    pdgpu_desc desc{};
    desc.dim = (int32_t)d_modelDeck_p->d_dim;
    desc.time_scheme = d_modelDeck_p->d_timeDiscretization == "velocity_verlet" ? 1 : 0;
    desc.precision = d_precision;
    desc.dt = d_modelDeck_p->d_dt;
    desc.gravity[0] = d_pDeck_p->d_gravity.d_x;
    desc.gravity[1] = d_pDeck_p->d_gravity.d_y;
    desc.gravity[2] = d_pDeck_p->d_gravity.d_z;
    desc.multi_particle = d_input_p->isMultiParticle() ? 1 : 0;
    desc.test = d_pDeck_p->d_testName == "two_particle"       ? PDGPU_TEST_TWO_PARTICLE
                : d_pDeck_p->d_testName == "compressive_test" ? PDGPU_TEST_COMPRESSIVE
                                                              : PDGPU_TEST_NONE;
    desc.test_wall = (int64_t)d_pDeck_p->d_particleIdCompressiveTest;
    desc.test_dir = (int32_t)d_pDeck_p->d_particleForceDirectionCompressiveTest - 1;
    desc.test_interval = (int64_t)d_outputDeck_p->d_dtTestOut;
    desc.search_factor = d_pDeck_p->d_pNeighDeck.d_sFactor;
    desc.search_interval = (int64_t)d_pDeck_p->d_pNeighDeck.d_neighUpdateInterval;
    desc.max_contact_r = d_maxContactR;
    check(pdgpu_create(&desc, &d_ctx), "create");

    // util::Point is three doubles; size_t is uint64
    const auto N = (int64_t)d_x.size();
    check(pdgpu_upload_nodes(d_ctx, N, &d_xRef[0].d_x, &d_x[0].d_x, &d_u[0].d_x, &d_v[0].d_x, d_vol.data(),
                             d_fix.data(), reinterpret_cast<const uint64_t *>(d_ptId.data())),
          "upload_nodes");

    // the influence function of the first material (material.h:23-54: one
    // per process, set by the first material constructed)
    const auto &md0 = d_pDeck_p->d_particleZones[d_particlesListTypeAll[0]->d_zoneId].d_matDeck;
    const int32_t inf_type = (int32_t)md0.d_influenceFnType;
    double inf[2] = {0., 0.};
    check(pdgpu_influence_params(inf_type, (int32_t)md0.d_influenceFnParams.size(),
                                 md0.d_influenceFnParams.data(), desc.dim, inf),
          "influence_params");

    std::vector<pdgpu_particle> ps;
    for (auto *p : d_particlesListTypeAll) {
      pdgpu_particle q{};
      q.glob_start = (int64_t)p->d_globStart;
      q.glob_end = (int64_t)p->d_globEnd;
      q.center_node = (int64_t)(p->d_globStart + p->getCenterNodeId());
      q.type = (int32_t)p->d_typeIndex;
      q.zone = (int32_t)p->d_zoneId;
      q.compute_force = p->d_computeForce ? 1 : 0;
      q.all_dofs_constrained = p->d_allDofsConstrained ? 1 : 0;
      q.horizon = p->getHorizon();
      q.h = p->getMeshSize();
      q.density = p->getDensity();
      q.rc = p->d_Rc;
      q.kn = p->d_Kn;
      q.bound_r = p->d_geom_p->boundingRadius();
      bondLaw(p, desc.dim, inf_type, inf, q);
      ps.push_back(q);
    }
    check(pdgpu_upload_particles(d_ctx, (int64_t)ps.size(), ps.data()), "upload_particles");
    check(pdgpu_set_influence(d_ctx, inf_type, inf), "set_influence");

    // contact pairs after setupContact (demModel.cpp:1531-1600)
    const auto nz = d_cDeck_p->d_data.size();
    std::vector<double> rc, kn, mu, bn, ka;
    for (size_t i = 0; i < nz; i++)
      for (size_t j = 0; j < nz; j++) {
        const auto &c = d_cDeck_p->d_data[i][j];
        rc.push_back(c.d_contactR);
        kn.push_back(c.d_Kn);
        mu.push_back(c.d_mu);
        bn.push_back(c.d_betan);
        ka.push_back(c.d_kappa);
      }
    if (desc.multi_particle)
      check(pdgpu_upload_contact(d_ctx, (int32_t)nz, rc.data(), kn.data(), mu.data(), bn.data(), ka.data()),
            "upload_contact");

    // peridynamic neighbour lists (d_neighPd) in the kd-tree's order, and m_x
    std::vector<uint64_t> row{0}, col;
    for (auto &l : d_neighPd) {
      col.insert(col.end(), l.begin(), l.end());
      row.push_back(col.size());
    }
    check(pdgpu_upload_pd_neighbors(d_ctx, row.data(), col.data(), nullptr), "upload_pd_neighbors");
    check(pdgpu_upload_mx(d_ctx, d_mX.data()), "upload_mx");

    // boundary conditions: selections evaluated by the reference's own
    // loading classes (needToProcessParticle / needToComputeDof)
    addBCs(d_pDeck_p->d_dispDeck, true);
    addBCs(d_pDeck_p->d_forceDeck, false);
    if (d_pDeck_p->d_icDeck.d_icActive) {
      const auto &ic = d_pDeck_p->d_icDeck;
      double v[3] = {ic.d_icVec.d_x, ic.d_icVec.d_y, ic.d_icVec.d_z};
      check(pdgpu_set_initial_condition(d_ctx, v, reinterpret_cast<const uint64_t *>(ic.d_pList.data()),
                                        (int64_t)ic.d_pList.size()),
            "set_initial_condition");
    }
    if (desc.multi_particle) check(pdgpu_init_contact(d_ctx), "init_contact");
  }

  void download() {
    check(pdgpu_download(d_ctx, PDGPU_FIELD_X, &d_x[0].d_x), "download x");
    check(pdgpu_download(d_ctx, PDGPU_FIELD_U, &d_u[0].d_x), "download u");
    check(pdgpu_download(d_ctx, PDGPU_FIELD_V, &d_v[0].d_x), "download v");
    check(pdgpu_download(d_ctx, PDGPU_FIELD_F, &d_f[0].d_x), "download f");
    check(pdgpu_download(d_ctx, PDGPU_FIELD_Z, d_Z.data()), "download Z");
    check(pdgpu_download(d_ctx, PDGPU_FIELD_VMAG, d_vMag.data()), "download |v|");
  }

  // the bond law by the material's class (public types) and its constants
  // from the zone's material deck (pdgpu_material_constants), checked
  // against the live material's public critical stretch
  void bondLaw(particle::BaseParticle *p, int32_t dim, int32_t inf_type, const double inf[2],
               pdgpu_particle &q) {
    const material::Material *m = p->d_material_p.get();
    int32_t law = -1;
    if (dynamic_cast<const material::RnpMaterial *>(m)) law = PDGPU_MAT_RNP;
    else if (dynamic_cast<const material::PmbMaterial *>(m)) law = PDGPU_MAT_PMB;
    else if (dynamic_cast<const material::PdElastic *>(m)) law = PDGPU_MAT_PDELASTIC;
    else if (dynamic_cast<const material::PdState *>(m)) law = PDGPU_MAT_PDSTATE;
    if (law < 0) check(PDGPU_ERR_ARG, "unknown material class");
    const auto &md = d_pDeck_p->d_particleZones[p->d_zoneId].d_matDeck;
    pdgpu_material_deck deck{};
    deck.law = law;
    deck.irreversible = md.d_irreversibleBondBreak ? 1 : 0;
    deck.E = md.d_matData.d_E;
    deck.K = md.d_matData.d_K;
    deck.G = md.d_matData.d_G;
    deck.nu = md.d_matData.d_nu;
    deck.Gc = md.d_matData.d_Gc;
    deck.check_sc_factor = md.d_checkScFactor;
    q.material = law;
    check(pdgpu_material_constants(&deck, dim, q.horizon, inf_type, inf, q.mat, nullptr), "material_constants");
    // the critical stretch the live material reports must be ours
    const double r = q.horizon;
    const double sc = law == PDGPU_MAT_RNP ? q.mat[2] / std::sqrt(r)
                      : law == PDGPU_MAT_PMB ? q.mat[1]
                      : law == PDGPU_MAT_PDSTATE ? q.mat[2]
                                                 : m->getSc(r);
    if (sc != m->getSc(r)) {
      std::cerr << "pdgpu: bond-law constants of particle " << p->getId()
                << " disagree with its material (critical stretch " << sc << " vs " << m->getSc(r) << ")\n";
      std::exit(1);
    }
  }

  static int32_t timeCode(const std::string &t) {
    static const char *names[] = {"constant", "linear", "quadratic", "sin", "rotation", "linear_step",
                                  "linear_slow_fast"};
    for (int32_t i = 0; i < 7; i++)
      if (t == names[i]) return i;  // PDGPU_TIME_*, same order
    return 99;                      // unrecognised: no time factor, as in the reference
  }
  static int32_t spatialCode(const std::string &t) {
    static const char *names[] = {"constant", "hat_x", "hat_y", "sin_x", "sin_y", "linear_x", "linear_y"};
    for (int32_t i = 0; i < 7; i++)
      if (t == names[i]) return i;  // PDGPU_SPACE_*, same order
    return PDGPU_SPACE_CONSTANT;
  }

  // one pdgpu BC set per deck set, with the particle and node selections
  // evaluated by the reference's own loading class (needToProcessParticle /
  // needToComputeDof; the force-loading predicates are the same)
  void addBCs(std::vector<inp::PBCData> &sets, bool displacement) {
    const size_t N = d_x.size(), np = d_particlesListTypeAll.size();
    loading::ParticleULoading ul(sets);
    for (const auto &bc : sets) {
      pdgpu_bc_set b{};
      b.time_fn = timeCode(bc.d_timeFnType);
      b.spatial_fn = spatialCode(bc.d_spatialFnType);
      for (auto dir : bc.d_direction) b.dir_mask |= 1 << (dir - 1);
      b.zero = bc.d_isDisplacementZero ? 1 : 0;
      for (size_t k = 0; k < 4 && k < bc.d_timeFnParams.size(); k++) b.time_params[k] = bc.d_timeFnParams[k];
      for (size_t k = 0; k < 2 && k < bc.d_spatialFnParams.size(); k++)
        b.spatial_params[k] = bc.d_spatialFnParams[k];
      std::vector<uint8_t> proc(np, 0), mask(N, 0);
      std::vector<double> box(6 * np, 0.);
      for (auto *p : d_particlesListTypeAll) {
        const bool pr = ul.needToProcessParticle(p->getId(), bc);
        proc[p->getId()] = pr ? 1 : 0;
        const auto bx = bc.d_isRegionActive ? bc.d_regionGeomData.d_geom_p->box() : p->d_geom_p->box();
        for (int k = 0; k < 3; k++) {
          box[6 * p->getId() + k] = bx.first[k];
          box[6 * p->getId() + 3 + k] = bx.second[k];
        }
        if (!pr) continue;
        for (size_t i = 0; i < p->getNumNodes(); i++)
          if (ul.needToComputeDof(p->getXRefLocal(i), p->getId(), bc)) mask[p->getNodeId(i)] = 1;
      }
      check(displacement ? pdgpu_add_displacement_bc(d_ctx, &b, proc.data(), mask.data(), box.data())
                         : pdgpu_add_force_bc(d_ctx, &b, proc.data(), mask.data(), box.data()),
            "add_bc");
    }
  }
};

}  // namespace model

#endif  // PDGPU_GPU_DEM_MODEL_H
