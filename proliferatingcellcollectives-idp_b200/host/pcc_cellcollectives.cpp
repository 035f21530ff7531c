// Command-line driver over the device library: the reference program's
// options (code/cpp/src/util/CLIParser.h:296-365, "-name value" pairs, names
// matched case-insensitively like PETSc's options database) and its main loop
// (main.cpp:18-77, spatial/Domain.cpp:120-209) with the colony resident on one
// GPU.  Output follows the reference: ./vtk_output_<mode>/ gets the parameters
// file at start and particles / ghost_particles / simulation files at step 0,
// whenever the colony radius grew by -log_every_colony_radius_delta or the
// simulated time by -log_every_sim_time_delta since the last log, and at the
// end (Domain.cpp:188-200); the files are written by a background thread while
// the colony steps on.  -starter_vtk <dir or file> restarts from the latest
// state of a VTK output directory (Domain::initializeFromVTK, Domain.cpp:650-690).
// -no_vtk turns the output off; -out writes the final cells as CSV.
//
//   pcc_cellcollectives -mode hard|soft [-dt 1e-2] [-end_radius 50] [-xi 1] [-tau 1]
//       [-l0 1] [-lambda 1e-2] [-kcc 2e4] [-temperature 0] [-monolayer true]
//       [-tolerance 1e-3] [-max_bbpgd_iterations 5e5]
//       [-max_recursive_iterations 50] [-linked_cell_size 2.2*l0] [-cfl_factor 0.5]
//       [-log_every_colony_radius_delta 0.5] [-log_every_sim_time_delta 1e5]
//       [-starter_vtk path] [-no_vtk] [-precision fp64|mixed] [-log_bbgd_trace]
//       [-seed 0] [-fixed_dt 0|1] [-dt_cap 0] [-ghosts single_rank|none] [-max_steps N]
//       [-device 0] [-out cells.csv]
#include <dirent.h>
#include <strings.h>

#include <sys/stat.h>

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

// The options and their defaults (the reference's -help, util/CLIParser.h:13-160,
// plus this driver's own switches).
static void print_help(const pcc_params& p) {
  auto row = [](const char* name, const char* what, const std::string& def) {
    std::printf("  %-32s %-52s [default: %s]\n", name, what, def.c_str());
  };
  auto num = [](double v) {
    char b[32];
    std::snprintf(b, sizeof b, "%g", v);
    return std::string(b);
  };
  std::printf("\nAvailable parameters:\n\nSimulation:\n");
  row("-mode hard|soft", "Collision model (required)", "none");
  row("-dt", "Time step", num(p.dt));
  row("-end_radius", "Colony radius at which the run stops", num(p.end_radius));
  row("-log_every_colony_radius_delta", "Log after the radius grew by this much (0: off)",
      num(p.log_every_colony_radius_delta));
  row("-log_every_sim_time_delta", "Log after this much simulated time (0: off)", num(p.log_every_sim_time_delta));
  row("-cfl_factor", "CFL factor of the adaptive time step", num(p.cfl_factor));
  row("-log_bbgd_trace", "Write a BBPGD trace on every 10th step to ./logs", "false");
  row("-starter_vtk", "Restart from a VTK output directory or file", "none");
  std::printf("\nPhysics:\n");
  row("-xi", "Drag coefficient", num(p.xi));
  row("-tau", "Growth time constant", num(p.tau));
  row("-l0", "Reference length", num(p.l0));
  row("-lambda", "Stress sensitivity of growth", num(p.lambda));
  row("-kcc", "Soft-model contact stiffness", num(p.kcc));
  row("-temperature", "Simulation temperature (Brownian rotational kicks)", num(p.temperature));
  row("-monolayer", "Brownian kicks about z only", p.monolayer ? "true" : "false");
  std::printf("\nSolver:\n");
  row("-tolerance", "BBPGD residual and ReLCP overlap tolerance", num(p.tolerance));
  row("-max_bbpgd_iterations", "BBPGD iteration cap", num((double)p.max_bbpgd_iterations));
  row("-max_recursive_iterations", "ReLCP phase cap", num((double)p.max_recursive_iterations));
  row("-linked_cell_size", "Broadphase bin edge", "2.2 * l0");
  std::printf("\nThis driver:\n");
  row("-precision fp64|mixed", "BBPGD operand precision", "fp64");
  row("-seed", "Seed of the first cell's orientation and the divisions", "0");
  row("-fixed_dt 0|1", "Keep dt fixed instead of adapting it", "0");
  row("-dt_cap", "Upper bound of the adapted dt (0: none)", "0");
  row("-ghosts single_rank|none", "Self-ghost copies of the one-rank decomposition", "single_rank");
  row("-max_steps", "Step cap", "none");
  row("-device", "CUDA device", "0");
  row("-no_vtk", "Write no VTK output", "false");
  row("-out", "Write the final cells as CSV", "none");
}

int main(int argc, char** argv) {
  Options o = parse(argc, argv);
  pcc_params p;
  pcc_default_params(&p);
  if (o.has("-help")) {
    print_help(p);
    return 0;
  }
  std::string mode = o.get("-mode", "");
  if (mode.empty()) {
    std::printf("Error: Required parameter -mode not provided. Use -help for usage information.\n");
    return 1;
  }
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
  p.temperature = o.num("-temperature", p.temperature);
  if (o.has("-monolayer")) {
    const std::string v = o.get("-monolayer", "");
    p.monolayer = (v.empty() || v == "1" || strcasecmp(v.c_str(), "true") == 0) ? 1 : 0;
  }
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
  p.log_every_colony_radius_delta = o.num("-log_every_colony_radius_delta", p.log_every_colony_radius_delta);
  p.log_every_sim_time_delta = o.num("-log_every_sim_time_delta", p.log_every_sim_time_delta);
  p.precision = strcasecmp(o.get("-precision", "fp64").c_str(), "mixed") == 0 ? PCC_PRECISION_MIXED
                                                                               : PCC_PRECISION_FP64;
  // -log_bbgd_trace [true|1]: BBPGD trace of every 10th step into ./logs
  if (o.has("-log_bbgd_trace")) {
    const std::string v = o.get("-log_bbgd_trace", "");
    p.log_bbpgd_trace = (v.empty() || v == "1" || strcasecmp(v.c_str(), "true") == 0) ? 1 : 0;
  }
  const long long max_steps = (long long)o.num("-max_steps", 1e12);
  const int device = (int)o.num("-device", 0);
  const bool vtk = !o.has("-no_vtk");
  const std::string starter = o.get("-starter_vtk", "");
  const std::string outdir = "./vtk_output_" + std::string(p.mode == PCC_MODE_HARD ? "hard" : "soft");

  try {
    pcc::DeviceColony dev(p, device);
    long long iter = 0;
    double sim_time = 0;
    if (!starter.empty()) {
      size_t n = 0;
      long long step0 = 0;
      double dt_file = 0;
      if (pcc_vtk_load(starter.c_str(), nullptr, 0, &n, &sim_time, &step0, &dt_file) != PCC_OK)
        throw std::runtime_error("VTK path must be a file or directory with a VTK state: " + starter);
      std::vector<double> buf(10 * (n + 1));
      std::vector<int> age(n + 1);
      std::vector<double> fv(12 * (n + 1));
      pcc_cells c{};
      double* b = buf.data();
      c.x = b;
      c.y = b + (n + 1);
      c.z = b + 2 * (n + 1);
      c.q0 = b + 3 * (n + 1);
      c.q1 = b + 4 * (n + 1);
      c.q2 = b + 5 * (n + 1);
      c.q3 = b + 6 * (n + 1);
      c.length = b + 7 * (n + 1);
      c.l0 = b + 8 * (n + 1);
      c.diameter = b + 9 * (n + 1);
      c.age = age.data();
      c.force = fv.data();
      c.velocity = fv.data() + 6 * (n + 1);
      pcc_vtk_load(starter.c_str(), &c, n, &n, &sim_time, &step0, &dt_file);
      std::printf("Loading %zu particles from VTK state at time %.2f s (iter %lld)\n", n, sim_time, step0);
      if (pcc_upload_cells(dev.handle(), &c, n) != PCC_OK) throw std::runtime_error("pcc_upload_cells failed");
      iter = step0;
      pcc_set_clock(dev.handle(), sim_time, iter);
    } else {
      // first cell (main.cpp:27-30), orientation theta ~ U[0, pi) from the seed
      std::mt19937_64 rng(p.seed);
      const double theta = std::uniform_real_distribution<double>(0.0, M_PI)(rng);
      pcc::ParticleState c0;
      c0.quaternion = {std::cos(theta / 2), 0, 0, std::sin(theta / 2)};
      c0.length = p.l0;
      c0.l0 = p.l0;
      c0.diameter = p.l0 / 2;
      dev.upload({c0});
    }
    // loggers count their own files from the starting iteration (VTK.h:190-240)
    unsigned long long log_index = (unsigned long long)iter;
    if (vtk) {
      if (starter.empty()) {
        // a fresh run clears earlier output of the same prefixes (VTK.h:209-231)
        const char* prefixes[] = {"particles", "ghost_particles", "simulation", "parameters"};
        for (const char* sub : {"", "/data"}) {
          const std::string d = outdir + sub;
          if (DIR* dp = opendir(d.c_str())) {
            while (dirent* de = readdir(dp)) {
              const std::string f = de->d_name;
              const bool ext = f.size() > 5 && (f.compare(f.size() - 5, 5, ".pvtu") == 0 ||
                                                f.compare(f.size() - 4, 4, ".vtu") == 0);
              for (const char* pre : prefixes)
                if (ext && f.rfind(pre, 0) == 0) std::remove((d + "/" + f).c_str());
            }
            closedir(dp);
          }
        }
      }
      if (pcc_vtk_write_parameters(outdir.c_str(), (unsigned long long)iter, &p) != PCC_OK)
        throw std::runtime_error("cannot write " + outdir);
    }
    auto t0 = std::chrono::steady_clock::now(), tlast = t0, tlog = t0;
    double cell_steps = 0, radius = 0, radius_last_log = 0, time_last_log = sim_time;
    long long steps = 0, bbpgd = 0;
    pcc_step_stats st{};
    while (radius < p.end_radius && steps < max_steps) {
      st = dev.step();
      radius = st.colony_radius;
      cell_steps += (double)st.n_cells;
      bbpgd += st.bbpgd_iterations;
      ++steps;
      auto now = std::chrono::steady_clock::now();
      const bool by_radius =
          p.log_every_colony_radius_delta && radius - radius_last_log > p.log_every_colony_radius_delta;
      const bool by_time = p.log_every_sim_time_delta && st.sim_time - time_last_log > p.log_every_sim_time_delta;
      if (vtk && (by_radius || by_time || iter == 0 || radius >= p.end_radius)) {
        pcc_sim_record r{};
        r.simulation_time_s = st.sim_time;
        r.time_since_last_log_s = std::chrono::duration<double>(now - tlog).count();
        r.step = (unsigned long long)iter;
        r.num_particles = (int)st.n_cells;
        r.num_constraints = (unsigned long long)st.n_constraints;
        r.colony_radius = radius;
        r.recursive_iterations = st.relcp_iterations;
        r.bbpgd_iterations = (unsigned long long)st.bbpgd_iterations;
        r.max_overlap = st.max_overlap;
        r.residual = st.residual;
        r.dt_s = st.dt_next;
        r.cpu_time_s = std::chrono::duration<double>(now - t0).count();
        r.load_imbalance = 1.0;
        if (pcc_log_vtk(dev.handle(), outdir.c_str(), log_index++, &r) != PCC_OK)
          throw std::runtime_error("pcc_log_vtk failed");
        radius_last_log = radius;
        time_last_log = st.sim_time;
        tlog = now;
        std::printf("  Logged data at Colony radius = %.3f, Simulation time = %.3f \n", radius, st.sim_time);
      }
      ++iter;
      if (std::chrono::duration<double>(now - tlast).count() > 1.0) {
        tlast = now;
        std::printf("step %lld  cells %lld  radius %.3f  dt %.3g  relcp %d  bbpgd %lld  overlap %.2e\n", steps,
                    st.n_cells, radius, st.dt_used, st.relcp_iterations, st.bbpgd_iterations, st.max_overlap);
        std::fflush(stdout);
      }
    }
    if (vtk && pcc_log_vtk_wait(dev.handle()) != PCC_OK) throw std::runtime_error("writing VTK output failed");
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
