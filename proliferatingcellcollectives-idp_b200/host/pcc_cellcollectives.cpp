// Command-line driver over the device library: the reference program's
// options (code/cpp/src/util/CLIParser.h:296-365, "-name value" pairs, names
// matched case-insensitively like PETSc's options database) and its main loop
// (main.cpp:18-77, spatial/Domain.cpp:120-209) with the colony resident on one
// GPU.  VTK logging is not part of this path; -out writes the final cells as
// CSV.
//
//   pcc_cellcollectives -mode hard|soft [-dt 1e-2] [-end_radius 50] [-xi 1] [-tau 1]
//       [-l0 1] [-lambda 1e-2] [-kcc 2e4] [-tolerance 1e-3] [-max_bbpgd_iterations 5e5]
//       [-max_recursive_iterations 50] [-linked_cell_size 2.2*l0] [-cfl_factor 0.5]
//       [-seed 0] [-fixed_dt 0|1] [-dt_cap 0] [-ghosts single_rank|none] [-max_steps N]
//       [-device 0] [-out cells.csv]
#include <strings.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <random>
#include <string>

#include "pcc_adapter.hpp"

namespace {

struct Options {
  std::map<std::string, std::string> kv;
  bool has(const char* k) const {
    for (auto& p : kv)
      if (strcasecmp(p.first.c_str(), k) == 0) return true;
    return false;
  }
  std::string get(const char* k, const std::string& def) const {
    for (auto& p : kv)
      if (strcasecmp(p.first.c_str(), k) == 0) return p.second;
    return def;
  }
  double num(const char* k, double def) const {
    std::string s = get(k, "");
    return s.empty() ? def : std::strtod(s.c_str(), nullptr);
  }
};

Options parse(int argc, char** argv) {
  Options o;
  for (int i = 1; i < argc; ++i) {
    if (argv[i][0] != '-') continue;
    std::string v;
    if (i + 1 < argc && (argv[i + 1][0] != '-' || std::isdigit((unsigned char)argv[i + 1][1]) || argv[i + 1][1] == '.'))
      v = argv[++i];
    o.kv[argv[i - (v.empty() ? 0 : 1)]] = v;
  }
  return o;
}

}  // namespace

int main(int argc, char** argv) {
  Options o = parse(argc, argv);
  std::string mode = o.get("-mode", "");
  if (mode.empty()) {
    std::fprintf(stderr, "Error: Required parameter -mode not provided. Use -help for usage information.\n");
    return 1;
  }
  pcc_params p;
  pcc_default_params(&p);
  if (strcasecmp(mode.c_str(), "soft") == 0)
    p.mode = PCC_MODE_SOFT;
  else if (strcasecmp(mode.c_str(), "hard") == 0)
    p.mode = PCC_MODE_HARD;
  else {
    std::fprintf(stderr, "Invalid mode: %s\n", mode.c_str());
    return 1;
  }
  p.dt = o.num("-dt", p.dt);
  p.end_radius = o.num("-end_radius", p.end_radius);
  p.xi = o.num("-xi", p.xi);
  p.tau = o.num("-tau", p.tau);
  p.l0 = o.num("-l0", p.l0);
  p.lambda = o.num("-lambda", p.lambda);
  p.kcc = o.num("-kcc", p.kcc);
  p.tolerance = o.num("-tolerance", p.tolerance);
  p.max_bbpgd_iterations = (long long)o.num("-max_bbpgd_iterations", (double)p.max_bbpgd_iterations);
  p.max_recursive_iterations = (long long)o.num("-max_recursive_iterations", (double)p.max_recursive_iterations);
  p.linked_cell_size = o.has("-linked_cell_size") ? o.num("-linked_cell_size", 0) : 2.2 * p.l0;
  p.cfl_factor = o.num("-cfl_factor", p.cfl_factor);
  p.seed = (unsigned long long)o.num("-seed", 0);
  p.fixed_dt = (int)o.num("-fixed_dt", 0);
  p.dt_cap = o.num("-dt_cap", 0);
  p.ghost_mode = strcasecmp(o.get("-ghosts", "single_rank").c_str(), "none") == 0 ? PCC_GHOSTS_NONE
                                                                                   : PCC_GHOSTS_SINGLE_RANK;
  const long long max_steps = (long long)o.num("-max_steps", 1e12);
  const int device = (int)o.num("-device", 0);

  try {
    pcc::DeviceColony dev(p, device);
    // first cell (main.cpp:27-30), orientation theta ~ U[0, pi) from the seed
    std::mt19937_64 rng(p.seed);
    const double theta = std::uniform_real_distribution<double>(0.0, M_PI)(rng);
    pcc::ParticleState c0;
    c0.quaternion = {std::cos(theta / 2), 0, 0, std::sin(theta / 2)};
    c0.length = p.l0;
    c0.l0 = p.l0;
    c0.diameter = p.l0 / 2;
    dev.upload({c0});
    auto t0 = std::chrono::steady_clock::now(), tlast = t0;
    double cell_steps = 0, radius = 0;
    long long steps = 0, bbpgd = 0;
    pcc_step_stats st{};
    while (radius < p.end_radius && steps < max_steps) {
      st = dev.step();
      radius = st.colony_radius;
      cell_steps += (double)st.n_cells;
      bbpgd += st.bbpgd_iterations;
      ++steps;
      auto now = std::chrono::steady_clock::now();
      if (std::chrono::duration<double>(now - tlast).count() > 1.0) {
        tlast = now;
        std::printf("step %lld  cells %lld  radius %.3f  dt %.3g  relcp %d  bbpgd %lld  overlap %.2e\n", steps,
                    st.n_cells, radius, st.dt_used, st.relcp_iterations, st.bbpgd_iterations, st.max_overlap);
        std::fflush(stdout);
      }
    }
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("done: %lld steps, %lld cells, radius %.3f, sim time %.4f, %.3f s wall, %.4g cell-steps/s, "
                "%lld BBPGD iterations\n",
                steps, st.n_cells, radius, st.sim_time, wall, cell_steps / wall, bbpgd);
    std::string out = o.get("-out", "");
    if (!out.empty()) {
      std::vector<pcc::ParticleState> ps;
      dev.download(ps);
      FILE* f = std::fopen(out.c_str(), "w");
      if (!f) throw std::runtime_error("cannot write " + out);
      std::fprintf(f, "gid,x,y,z,q0,q1,q2,q3,length,ldot,impedance,stress,age\n");
      for (auto& c : ps)
        std::fprintf(f, "%d,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%d\n", c.gid,
                     c.position[0], c.position[1], c.position[2], c.quaternion[0], c.quaternion[1], c.quaternion[2],
                     c.quaternion[3], c.length, c.ldot, c.impedance, c.stress, c.age);
      std::fclose(f);
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 2;
  }
  return 0;
}
