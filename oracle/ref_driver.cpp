// peridem_ref: runs the reference's own model::DEMModel on a YAML deck and
// dumps its state, so that tests can compare the CUDA path against it.
//
// ORACLE TEST INFRASTRUCTURE ONLY.  This file is compiled (by oracle/Makefile)
// against the reference's own sources, unchanged; nothing here is part of the
// product library, and the product never calls it.
//
// Usage:
//   peridem_ref -i deck.yaml [-nThreads T] [-dump DIR] [-steps K]
//               [-dumpSteps a,b,c] [-time K]
//
//   -dump DIR      write DIR/init.bin (state after DEMModel::init and the
//                  first computeForces of DEMModel::integrate, i.e. step 0)
//                  and DIR/step_<n>.bin for every n in -dumpSteps.
//   -steps K       number of integrateStep() calls (default: the deck's Nt).
//   -time K        time K steady-state steps (after one warm-up step) and print
//                  one JSON line with node-steps/s.
//   -load FILE     before the first step, put the model into the state of a
//                  pdgpu state snapshot (its portable part: step, time,
//                  contact-search interval and radius, x, u, v and the broken
//                  bonds as node pairs); the contact lists are rebuilt at the
//                  first contact update.  Used to time the reference from the
//                  same loaded state as the GPU.
//
// The step loop below follows model::DEMModel::integrate
// (src/model/dem/demModel.cpp:268-340): applyInitialCondition,
// computeExternalDisplacementBC, computeForces, then integrateStep +
// post-processing per step.  VTU output is not available (no VTK here), so
// decks run with Perform_Out: false.

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <functional>
#include <future>
#include <iomanip>
#include <iostream>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <optional>
#include <queue>
#include <random>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <variant>
#include <vector>
#include <fmt/format.h>
#include <taskflow/taskflow/taskflow.hpp>
#include <taskflow/taskflow/algorithm/for_each.hpp>

// The material classes keep their derived bond-law constants private; the
// dump needs them verbatim, so only this header is opened up.  Every class in
// it is polymorphic, so its layout does not depend on access specifiers.
#define private public
#define protected public
#include "material/mparticle/material.h"
#undef private
#undef protected

#include "model/dem/demModel.h"
#include "particle/baseParticle.h"
#include "inp/input.h"
#include "inp/decks/modelDeck.h"
#include "inp/decks/outputDeck.h"
#include "inp/pdecks/contactDeck.h"
#include "inp/pdecks/particleDeck.h"
#include "util/parallelUtil.h"
#include "util/geomObjects.h"

namespace {

// ---- tagged binary dump: magic, then records (name, dtype, count, data) ----
enum DType : uint32_t { F64 = 0, F32 = 1, U8 = 2, I64 = 3 };

struct Dump {
  std::ofstream f;
  explicit Dump(const std::string &path) : f(path, std::ios::binary) {
    if (!f) {
      std::cerr << "peridem_ref: cannot write " << path << "\n";
      std::exit(2);
    }
    f.write("PDDUMP01", 8);
  }
  void rec(const std::string &name, DType t, uint64_t n, const void *data, size_t esz) {
    uint32_t l = (uint32_t)name.size();
    f.write((const char *)&l, 4);
    f.write(name.data(), l);
    f.write((const char *)&t, 4);
    f.write((const char *)&n, 8);
    if (n) f.write((const char *)data, (std::streamsize)(n * esz));
  }
  void f64(const std::string &n, const std::vector<double> &v) { rec(n, F64, v.size(), v.data(), 8); }
  void f32(const std::string &n, const std::vector<float> &v) { rec(n, F32, v.size(), v.data(), 4); }
  void u8(const std::string &n, const std::vector<uint8_t> &v) { rec(n, U8, v.size(), v.data(), 1); }
  void i64(const std::string &n, const std::vector<int64_t> &v) { rec(n, I64, v.size(), v.data(), 8); }
  void s(const std::string &n, double v) { f64(n, {v}); }
  void si(const std::string &n, int64_t v) { i64(n, {v}); }
  void pts(const std::string &n, const std::vector<util::Point> &p) {
    std::vector<double> v(3 * p.size());
    for (size_t i = 0; i < p.size(); i++) {
      v[3 * i] = p[i].d_x;
      v[3 * i + 1] = p[i].d_y;
      v[3 * i + 2] = p[i].d_z;
    }
    f64(n, v);
  }
};

void csr(Dump &d, const std::string &name, const std::vector<std::vector<size_t>> &l, size_t n) {
  std::vector<int64_t> rp(n + 1, 0), col;
  for (size_t i = 0; i < n; i++) {
    if (i < l.size())
      for (auto j : l[i]) col.push_back((int64_t)j);
    rp[i + 1] = (int64_t)col.size();
  }
  d.i64(name + "_rowptr", rp);
  d.i64(name + "_col", col);
}

int timeCode(const std::string &t) {
  static const char *names[] = {"constant", "linear", "quadratic", "sin", "rotation",
                                "linear_step", "linear_slow_fast"};
  for (int i = 0; i < 7; i++)
    if (t == names[i]) return i;
  return -1;  // unrecognised: the reference applies no time factor
}

int spatialCode(const std::string &t) {
  static const char *names[] = {"constant", "hat_x", "hat_y", "sin_x", "sin_y", "linear_x",
                                "linear_y"};
  for (int i = 0; i < 7; i++)
    if (t == names[i]) return i;
  return 0;
}

class DumpModel : public model::DEMModel {
public:
  using model::DEMModel::DEMModel;

  void dumpInit(const std::string &path) {
    Dump d(path);
    const size_t N = d_x.size();
    const size_t Np = d_particlesListTypeAll.size();
    d.si("dim", (int64_t)d_modelDeck_p->d_dim);
    d.si("N", (int64_t)N);
    d.si("Np", (int64_t)Np);
    d.s("dt", d_modelDeck_p->d_dt);
    d.si("Nt", (int64_t)d_modelDeck_p->d_Nt);
    d.si("time_disc", d_modelDeck_p->d_timeDiscretization == "velocity_verlet" ? 1 : 0);
    d.f64("gravity", {d_pDeck_p->d_gravity.d_x, d_pDeck_p->d_gravity.d_y, d_pDeck_p->d_gravity.d_z});
    d.s("hMin", d_hMin);
    d.s("hMax", d_hMax);
    d.s("maxContactR", d_maxContactR);
    d.s("sFactor", d_pDeck_p->d_pNeighDeck.d_sFactor);
    d.si("neighUpdateInterval", (int64_t)d_pDeck_p->d_pNeighDeck.d_neighUpdateInterval);
    d.si("is_multi", d_input_p->isMultiParticle() ? 1 : 0);
    int test = 0;
    if (d_pDeck_p->d_testName == "two_particle") test = 1;
    else if (d_pDeck_p->d_testName == "compressive_test") test = 2;
    d.si("test", test);
    d.si("cmp_wall", (int64_t)d_pDeck_p->d_particleIdCompressiveTest);
    d.si("cmp_dir", (int64_t)d_pDeck_p->d_particleForceDirectionCompressiveTest - 1);
    d.si("dtTestOut", (int64_t)d_outputDeck_p->d_dtTestOut);

    // nodes
    d.pts("xRef", d_xRef);
    d.f64("vol", d_vol);
    d.u8("fix", d_fix);
    std::vector<int64_t> pt(d_ptId.begin(), d_ptId.end());
    d.i64("ptId", pt);
    d.f64("mX", d_mX);

    // peridynamic neighbour lists in the reference's (kd-tree) order
    csr(d, "pd", d_neighPd, N);

    // particles
    std::vector<int64_t> gs, ge, ty, zo, cf, ad, cn, mt;
    std::vector<double> hz, hh, rho, rc, kn, br, mp;
    for (auto *p : d_particlesListTypeAll) {
      gs.push_back((int64_t)p->d_globStart);
      ge.push_back((int64_t)p->d_globEnd);
      ty.push_back(p->d_typeIndex);
      zo.push_back((int64_t)p->d_zoneId);
      cf.push_back(p->d_computeForce ? 1 : 0);
      ad.push_back(p->d_allDofsConstrained ? 1 : 0);
      cn.push_back((int64_t)(p->d_globStart + p->getCenterNodeId()));
      hz.push_back(p->getHorizon());
      hh.push_back(p->getMeshSize());
      rho.push_back(p->getDensity());
      rc.push_back(p->d_Rc);
      kn.push_back(p->d_Kn);
      br.push_back(p->d_geom_p->boundingRadius());
      std::array<double, 8> prm{};
      const material::Material *m = p->d_material_p.get();
      int code = -1;
      if (auto *r = dynamic_cast<const material::RnpMaterial *>(m)) {
        code = 0;
        prm = {r->d_C, r->d_beta, r->d_rbar, r->d_invFactor, r->d_factorSc,
               r->d_irrevBondBreak ? 1. : 0., r->d_horizon, r->d_density};
      } else if (auto *q = dynamic_cast<const material::PmbMaterial *>(m)) {
        code = 1;
        prm = {q->d_c, q->d_s0, 0, 0, 0, 0, q->d_horizon, q->d_density};
      } else if (auto *e = dynamic_cast<const material::PdElastic *>(m)) {
        code = 2;
        prm = {e->d_c, 0, 0, 0, 0, 0, e->d_horizon, e->d_density};
      } else if (auto *s = dynamic_cast<const material::PdState *>(m)) {
        code = 3;
        prm = {s->d_K, s->d_G, s->d_s0, 0, 0, 0, s->d_horizon, s->d_density};
      }
      mt.push_back(code);
      mp.insert(mp.end(), prm.begin(), prm.end());
    }
    d.i64("p_globStart", gs);
    d.i64("p_globEnd", ge);
    d.i64("p_type", ty);
    d.i64("p_zone", zo);
    d.i64("p_computeForce", cf);
    d.i64("p_allDofsConstrained", ad);
    d.i64("p_center", cn);
    d.f64("p_horizon", hz);
    d.f64("p_h", hh);
    d.f64("p_density", rho);
    d.f64("p_Rc", rc);
    d.f64("p_Kn", kn);
    d.f64("p_boundR", br);
    d.i64("p_mat_type", mt);
    d.f64("p_mat_params", mp);

    // influence function.  The reference keeps one per process in a
    // translation-unit-local singleton (material.h:23-54) that the first
    // material constructed sets, so it is rebuilt here from that material's
    // deck and then checked against the live materials through their public
    // getInfFn().
    {
      const auto &md = d_pDeck_p->d_particleZones[d_particlesListTypeAll[0]->d_zoneId].d_matDeck;
      int code = (int)md.d_influenceFnType;
      size_t dim = d_modelDeck_p->d_dim;
      std::shared_ptr<material::BaseInfluenceFn> fn;
      std::vector<double> prm(2, 0.);
      if (code == 0) {
        auto c = std::make_shared<material::ConstInfluenceFn>(md.d_influenceFnParams, dim);
        prm = {c->d_a0, 0.};
        fn = c;
      } else if (code == 1) {
        auto l = std::make_shared<material::LinearInfluenceFn>(md.d_influenceFnParams, dim);
        prm = {l->d_a0, l->d_a1};
        fn = l;
      } else if (code == 2) {
        auto g = std::make_shared<material::GaussianInfluenceFn>(md.d_influenceFnParams, dim);
        prm = {g->d_alpha, g->d_beta};
        fn = g;
      }
      for (auto *p : d_particlesListTypeAll) {
        double hz = p->getHorizon();
        for (double q : {0., 0.1, 0.37, 0.5, 0.93, 1.}) {
          double r = q * hz;
          if (p->d_material_p->getInfFn(r) != fn->getInfFn(r / hz)) {
            std::cerr << "peridem_ref: influence function of particle " << p->getId()
                      << " does not match its deck\n";
            std::exit(3);
          }
        }
      }
      d.si("inf_type", code);
      d.f64("inf_params", prm);
    }

    // contact parameters per zone pair, after DEMModel::setupContact
    {
      size_t nz = d_cDeck_p->d_data.size();
      std::vector<double> R, K, mu, bn, ka, eps;
      for (size_t i = 0; i < nz; i++)
        for (size_t j = 0; j < nz; j++) {
          const auto &c = d_cDeck_p->d_data[i][j];
          R.push_back(c.d_contactR);
          K.push_back(c.d_Kn);
          mu.push_back(c.d_mu);
          bn.push_back(c.d_betan);
          ka.push_back(c.d_kappa);
          eps.push_back(c.d_eps);
        }
      d.si("nzones", (int64_t)nz);
      d.f64("c_Rc", R);
      d.f64("c_Kn", K);
      d.f64("c_mu", mu);
      d.f64("c_betan", bn);
      d.f64("c_kappa", ka);
      d.f64("c_eps", eps);
    }

    // displacement and force boundary conditions, with the node/particle
    // selection evaluated by the reference's own loading classes
    dumpBC(d, "ubc", d_pDeck_p->d_dispDeck, true);
    dumpBC(d, "fbc", d_pDeck_p->d_forceDeck, false);

    // initial condition
    d.si("ic_active", d_pDeck_p->d_icDeck.d_icActive ? 1 : 0);
    d.f64("ic_v", {d_pDeck_p->d_icDeck.d_icVec.d_x, d_pDeck_p->d_icDeck.d_icVec.d_y,
                   d_pDeck_p->d_icDeck.d_icVec.d_z});
    std::vector<int64_t> icl(d_pDeck_p->d_icDeck.d_pList.begin(), d_pDeck_p->d_icDeck.d_pList.end());
    d.i64("ic_plist", icl);

    dumpState(d);
  }

  void dumpBC(Dump &d, const std::string &pre, std::vector<inp::PBCData> &sets, bool disp) {
    const size_t N = d_x.size();
    d.si(pre + "_nsets", (int64_t)sets.size());
    loading::ParticleULoading ul(sets);
    for (size_t s = 0; s < sets.size(); s++) {
      const auto &bc = sets[s];
      std::string k = pre + "_" + std::to_string(s) + "_";
      d.si(k + "time", timeCode(bc.d_timeFnType));
      d.f64(k + "time_params", bc.d_timeFnParams);
      d.si(k + "spatial", spatialCode(bc.d_spatialFnType));
      d.f64(k + "spatial_params", bc.d_spatialFnParams);
      std::vector<int64_t> dirs(bc.d_direction.begin(), bc.d_direction.end());
      d.i64(k + "dirs", dirs);
      d.si(k + "zero", bc.d_isDisplacementZero ? 1 : 0);
      d.si(k + "region", bc.d_isRegionActive ? 1 : 0);
      // selection, evaluated with the loading class's own predicates (the
      // force-loading predicates are textually the same)
      std::vector<uint8_t> proc(d_particlesListTypeAll.size(), 0), mask(N, 0);
      std::vector<double> box(6 * d_particlesListTypeAll.size(), 0.);
      for (auto *p : d_particlesListTypeAll) {
        bool pr = ul.needToProcessParticle(p->getId(), bc);
        proc[p->getId()] = pr ? 1 : 0;
        auto b = bc.d_isRegionActive ? bc.d_regionGeomData.d_geom_p->box() : p->d_geom_p->box();
        for (int q = 0; q < 3; q++) {
          box[6 * p->getId() + q] = b.first[q];
          box[6 * p->getId() + 3 + q] = b.second[q];
        }
        if (!pr) continue;
        for (size_t i = 0; i < p->getNumNodes(); i++)
          if (ul.needToComputeDof(p->getXRefLocal(i), p->getId(), bc))
            mask[p->getNodeId(i)] = 1;
      }
      d.u8(k + "proc", proc);
      d.u8(k + "mask", mask);
      d.f64(k + "box", box);
    }
    (void)disp;
  }

  void dumpState(Dump &d) {
    const size_t N = d_x.size();
    d.si("n", (int64_t)d_n);
    d.s("time", d_time);
    d.pts("x", d_x);
    d.pts("u", d_u);
    d.pts("v", d_v);
    d.pts("f", d_f);
    d.f64("vMag", d_vMag);
    d.f64("thetaX", d_thetaX);
    d.f32("Z", d_Z);
    d.u8("fix_now", d_fix);
    // bond states in neighbour-list order, one byte per bond
    std::vector<uint8_t> bs;
    if (d_fracture_p)
      for (size_t i = 0; i < N; i++)
        for (size_t k = 0; k < d_neighPd[i].size(); k++)
          bs.push_back(d_fracture_p->getBondState(i, k) ? 1 : 0);
    d.u8("bond_state", bs);
    csr(d, "c", d_neighC, N);
    d.si("contNeighUpdateInterval", (int64_t)d_contNeighUpdateInterval);
    d.s("contNeighSearchRadius", d_contNeighSearchRadius);
    d.si("contNeighTimestepCounter", (int64_t)d_contNeighTimestepCounter);
    d.s("maxVelocity", d_maxVelocity);
    d.s("reaction", d_dbgData.count("tot_reaction_force") ? getKeyData("tot_reaction_force") : 0.);
    d.s("wall_penetration", d_dbgData.count("wall_penetration") ? getKeyData("wall_penetration") : 0.);
    d.s("pen_dist", d_dbgData.count("pen_dist") ? getKeyData("pen_dist") : 0.);
    d.s("max_y", d_dbgData.count("max_y") ? getKeyData("max_y") : 0.);
  }

  // the portable part of a pdgpu state snapshot (SnapHeader of the
  // library's pdgpu_runtime.cu, then x, u, v and broken (i, j) pairs)
  void loadState(const std::string &path) {
    struct Head {
      char magic[8];
      int64_t dim, n_nodes, n_bonds, n_particles, stride, n_broken, n_words, entries, wp_cap, history,
          n_scenes, scene_hist_cap, surrogate, multi_particle, step;
      double time;
      int64_t contact_interval, contact_counter;
      double contact_radius, max_velocity;
      int64_t ctrl_bytes;
    } h{};
    std::ifstream f(path, std::ios::binary);
    if (!f.read((char *)&h, sizeof h) || std::memcmp(h.magic, "PDSNAP01", 8) != 0) {
      std::cerr << "peridem_ref: " << path << " is not a state snapshot\n";
      std::exit(2);
    }
    const size_t N = d_x.size();
    if ((size_t)h.n_nodes != N) {
      std::cerr << "peridem_ref: snapshot has " << h.n_nodes << " nodes, the deck " << N << "\n";
      std::exit(2);
    }
    std::vector<double> a(3 * N);
    for (auto *dst : {&d_x, &d_u, &d_v}) {
      f.read((char *)a.data(), (std::streamsize)(a.size() * 8));
      for (size_t i = 0; i < N; i++) (*dst)[i] = util::Point(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
    }
    std::vector<uint64_t> pr(2 * (size_t)h.n_broken);
    f.read((char *)pr.data(), (std::streamsize)(pr.size() * 8));
    if (!f) {
      std::cerr << "peridem_ref: " << path << " is truncated\n";
      std::exit(2);
    }
    for (size_t k = 0; k < (size_t)h.n_broken; k++) {
      const size_t i = pr[2 * k], j = pr[2 * k + 1];
      const auto &nb = d_neighPd[i];
      auto it = std::find(nb.begin(), nb.end(), j);
      if (it == nb.end()) {
        std::cerr << "peridem_ref: snapshot bond (" << i << ", " << j << ") is not a bond of the deck\n";
        std::exit(2);
      }
      d_fracture_p->setBondState(i, (size_t)(it - nb.begin()), true);
    }
    for (size_t i = 0; i < N; i++) d_vMag[i] = d_v[i].length();
    d_n = (size_t)h.step;
    d_time = h.time;
    d_contNeighUpdateInterval = (size_t)h.contact_interval;
    d_contNeighSearchRadius = h.contact_radius;
    d_maxVelocity = h.max_velocity;
    // counter 0: the next contact update step rebuilds the lists from the
    // loaded positions (demModel.cpp:1808-1955)
    d_contNeighTimestepCounter = 0;
  }

  // post-processing exactly as the reference's integrate() loop does it
  void postStep() {
    if (d_pDeck_p->d_testName == "two_particle")
      ppTwoParticleTest();
    else if (d_pDeck_p->d_testName == "compressive_test")
      ppCompressiveTest();
  }
};

std::vector<long> parseList(const std::string &s) {
  std::vector<long> out;
  std::stringstream ss(s);
  std::string tok;
  while (std::getline(ss, tok, ','))
    if (!tok.empty()) out.push_back(std::stol(tok));
  return out;
}

}  // namespace

int main(int argc, char **argv) {
  std::string deck_file, dump_dir, dump_steps, load_file;
  long steps = -1, time_steps = 0;
  unsigned threads = 1;
  for (int a = 1; a < argc; a++) {
    std::string k = argv[a];
    auto next = [&]() -> std::string {
      if (a + 1 >= argc) {
        std::cerr << "peridem_ref: missing value for " << k << "\n";
        std::exit(2);
      }
      return argv[++a];
    };
    if (k == "-i") deck_file = next();
    else if (k == "-nThreads") threads = (unsigned)std::stoul(next());
    else if (k == "-dump") dump_dir = next();
    else if (k == "-steps") steps = std::stol(next());
    else if (k == "-dumpSteps") dump_steps = next();
    else if (k == "-time") time_steps = std::stol(next());
    else if (k == "-load") load_file = next();
    else {
      std::cerr << "peridem_ref: unknown option " << k << "\n";
      return 2;
    }
  }
  if (deck_file.empty()) {
    std::cerr << "usage: peridem_ref -i deck.yaml [-nThreads T] [-dump DIR] [-steps K] "
                 "[-dumpSteps a,b] [-time K] [-load FILE]\n";
    return 2;
  }

  util::parallel::initNThreads(threads);
  auto *deck = new inp::Input(deck_file);
  auto *dem = new DumpModel(deck);  // never deleted: particles hold aliases of it

  auto t0 = std::chrono::steady_clock::now();
  dem->init();
  auto t1 = std::chrono::steady_clock::now();
  if (!load_file.empty()) dem->loadState(load_file);

  // the first part of DEMModel::integrate()
  if (dem->d_n == 0) dem->applyInitialCondition();
  dem->computeExternalDisplacementBC();
  dem->computeForces();

  auto wanted = parseList(dump_steps);
  std::set<long> want(wanted.begin(), wanted.end());
  if (!dump_dir.empty()) dem->dumpInit(dump_dir + "/init.bin");

  if (time_steps > 0) {
    // one warm-up step, then K timed steps (steady state)
    dem->integrateStep();
    dem->postStep();
    auto a = std::chrono::steady_clock::now();
    for (long s = 0; s < time_steps; s++) {
      dem->integrateStep();
      dem->postStep();
    }
    auto b = std::chrono::steady_clock::now();
    double sec = std::chrono::duration<double>(b - a).count();
    double n = (double)dem->d_x.size();
    std::printf("{\"nodes\": %.0f, \"steps\": %ld, \"seconds\": %.6f, \"node_steps_per_s\": %.6e, "
                "\"threads\": %u, \"init_seconds\": %.3f}\n",
                n, time_steps, sec, n * (double)time_steps / sec, threads,
                std::chrono::duration<double>(t1 - t0).count());
    return 0;
  }

  long nsteps = steps >= 0 ? steps : (long)dem->d_modelDeck_p->d_Nt;
  for (long s = 0; s < nsteps; s++) {
    dem->integrateStep();
    dem->postStep();
    if (!dump_dir.empty() && want.count((long)dem->d_n)) {
      Dump d(dump_dir + "/step_" + std::to_string(dem->d_n) + ".bin");
      dem->dumpState(d);
    }
  }
  return 0;
}
