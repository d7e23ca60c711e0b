// pdgpu_peridem: PeriDEM's command-line program (src/main.cpp:25-79) with
// model::GpuDEMModel in place of model::DEMModel, so the same YAML input
// runs its explicit steps on a B200.
//
//   pdgpu_peridem -i input.yaml [-nThreads N] [-precision fp64|mixed]
//                 [-finalVtu file.vtu] [-steps K]
//
// -nThreads sets the host threads of the reference's set-up, as in PeriDEM;
// -precision picks the bond loop's arithmetic (fp64, the default, is the
// drop-in form); -finalVtu writes the last state with pdgpu_write_vtu;
// -steps overrides the deck's number of time steps.  At the end one line
// of JSON reports the step, the time and the post-processing key data the
// reference's own ppTwoParticleTest / ppCompressiveTest computed on the
// GPU's state.
#include <chrono>
#include <cstdio>
#include <iostream>
#include <string>

#include "gpu_dem_model.h"
#include "inp/input.h"
#include "util/parallelUtil.h"

namespace {

class Driver : public model::GpuDEMModel {
public:
  using model::GpuDEMModel::GpuDEMModel;
  void setSteps(long k) {
    if (k >= 0) d_modelDeck_p->d_Nt = (size_t)k;
  }
  double key(const std::string &k) { return d_dbgData.count(k) ? getKeyData(k) : 0.0; }
  size_t step() const { return d_n; }
  double time() const { return d_time; }
};

}  // namespace

int main(int argc, char **argv) {
  std::string deck_file, precision = "fp64", vtu;
  unsigned threads = 1;
  long steps = -1;
  for (int a = 1; a < argc; a++) {
    const std::string k = argv[a];
    auto next = [&]() -> std::string {
      if (a + 1 >= argc) {
        std::cerr << "pdgpu_peridem: missing value for " << k << "\n";
        std::exit(2);
      }
      return argv[++a];
    };
    if (k == "-i") deck_file = next();
    else if (k == "-nThreads") threads = (unsigned)std::stoul(next());
    else if (k == "-precision") precision = next();
    else if (k == "-finalVtu") vtu = next();
    else if (k == "-steps") steps = std::stol(next());
    else {
      std::cerr << "pdgpu_peridem: unknown option " << k << "\n";
      return 2;
    }
  }
  if (deck_file.empty() || (precision != "fp64" && precision != "mixed")) {
    std::cerr << "usage: pdgpu_peridem -i input.yaml [-nThreads N] [-precision fp64|mixed] "
                 "[-finalVtu file.vtu] [-steps K]\n";
    return 2;
  }
  util::parallel::initNThreads(threads);
  auto *deck = new inp::Input(deck_file);
  if (!deck->isPeriDEM()) {
    std::cerr << "PeriDEM model not found in input file.\n";
    return 1;
  }
  auto t0 = std::chrono::steady_clock::now();
  auto *dem = new Driver(deck);  // kept alive: particles hold aliases of it
  dem->setSteps(steps);
  dem->d_precision = precision == "mixed" ? PDGPU_PREC_MIXED : PDGPU_PREC_FP64;
  dem->d_finalVtu = vtu;
  dem->run(deck);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::printf("{\"n\": %zu, \"time\": %.17g, \"reaction\": %.17g, \"wall_penetration\": %.17g, "
              "\"pen_dist\": %.17g, \"max_y\": %.17g, \"seconds\": %.3f}\n",
              dem->step(), dem->time(), dem->key("tot_reaction_force"), dem->key("wall_penetration"),
              dem->key("pen_dist"), dem->key("max_y"), secs);
  return 0;
}
