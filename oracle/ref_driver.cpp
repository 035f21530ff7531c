// C entry points over the reference simulator's own sources, compiled in place
// (code/cpp/src of the reference project) against the single-rank PETSc/MPI
// stand-ins in oracle/shim.  This is the pinned CPU oracle: the solver, the
// collision detector, the particle update and the driver glue below are the
// reference's code; this file only sequences one Domain::run iteration
// (spatial/Domain.cpp:120-153) with the logging left out, plus two switches the
// reference lacks (a fixed time step and a cap on the adapted one).
//
// Test infrastructure: only tests/, the smoke check and the CPU baseline of
// bench.py load the library built from this file.
// Every standard header the reference headers pull in is included before the
// access-widening defines below, so no library type is compiled with them.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <optional>
#include <random>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include <petsc.h>

#include "util/Config.h"
#define private public
#define protected public
#include "spatial/Domain.h"
#undef private
#undef protected
#include "dynamics/Constraint.h"
#include "loader/VTKStateLoader.h"
#include "logger/SimulationLogger.h"
#include "pcc_gpu.h"
#include "simulation/Particle.h"
#include "simulation/ParticleManager.h"
#include "util/ArrayMath.h"
#include "util/Quaternion.h"

// ------------------------------------------------------------ seeded random_device
static unsigned long long g_div_seed = 0;
static unsigned long long g_div_next = 0;

extern "C" unsigned int pcc_division_seed(unsigned long long seed, unsigned long long k) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (k + 1ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (unsigned int)(z & 0xffffffffULL);
}
extern "C" void pcc_ref_set_division_stream(unsigned long long seed, unsigned long long next_index) {
  g_div_seed = seed;
  g_div_next = next_index;
}
extern "C" unsigned long long pcc_ref_division_index(void) { return g_div_next; }
std::pcc_seeded_random_device::result_type std::pcc_seeded_random_device::operator()() {
  return pcc_division_seed(g_div_seed, g_div_next++);
}

// Library draw of the k-th division length, through the same std:: classes
// Particle::divide uses (simulation/Particle.cpp:128-135).
extern "C" double pcc_ref_division_length(unsigned long long seed, unsigned long long k, double len) {
  double half = len / 2;
  std::mt19937 gen(pcc_division_seed(seed, k));
  std::uniform_real_distribution<> dis(half * 0.98, half * 1.02);
  return dis(gen);
}

// The reference's process-wide Brownian generator (dynamics/Physics.cpp:19).
// A colony handle reseeds it with the default seed when it is created, so each
// handle draws the stream a fresh reference process would.
extern std::mt19937 gen;

// ------------------------------------------------------------ colony handle
namespace {
struct RefColony {
  SimulationParameters params;
  std::string outdir;
  std::unique_ptr<Domain> domain;
  int ghost_mode = PCC_GHOSTS_SINGLE_RANK;
  int fixed_dt = 0;
  double dt_cap = 0;
  double colony_radius = 0;
  unsigned long long seed = 0, div_index = 0;
  std::vector<Constraint> last_constraints;
  std::string err;
};

void fill_params(SimulationParameters& sp, const pcc_params* p) {
  sp.sim_config = {};
  sp.sim_config.dt_s = p->dt;
  sp.sim_config.end_radius = p->end_radius;
  sp.sim_config.log_every_sim_time_delta = 0;
  sp.sim_config.log_every_colony_radius_delta = 0;
  sp.sim_config.log_bbgd_trace = p->log_bbpgd_trace != 0;
  sp.sim_config.min_box_size = {p->l0 + 1, p->l0 + 1, 0};
  sp.physics_config.xi = p->xi;
  sp.physics_config.TAU = p->tau;
  sp.physics_config.l0 = p->l0;
  sp.physics_config.LAMBDA = p->lambda;
  sp.physics_config.temperature = p->temperature;
  sp.physics_config.kcc = p->kcc;
  sp.physics_config.monolayer = p->monolayer ? PETSC_TRUE : PETSC_FALSE;
  sp.solver_config.tolerance = p->tolerance;
  sp.solver_config.max_bbpgd_iterations = (size_t)p->max_bbpgd_iterations;
  sp.solver_config.max_recursive_iterations = (size_t)p->max_recursive_iterations;
  sp.solver_config.linked_cell_size = p->linked_cell_size;
  sp.solver_config.growth_factor = 1.5;
  sp.solver_config.particle_preallocation_factor = 20;
  sp.solver_config.cfl_factor = p->cfl_factor;
  sp.mode = p->mode == PCC_MODE_SOFT ? "soft" : "hard";
}

double colony_radius_of(Domain& d) {
  // spatial/Domain.cpp:148-153
  auto& pm = *d.particle_manager_;
  double r = 0.0;
  for (const auto& p : pm.local_particles)
    r = std::max(r, utils::ArrayMath::magnitude(pm.collision_detector_.getParticleEndpoints(p).second));
  return r;
}
}  // namespace

extern "C" {

void* pcc_ref_create(const pcc_params* p, const char* outdir) {
  auto* c = new RefColony();
  gen.seed(std::mt19937::default_seed);
  fill_params(c->params, p);
  c->ghost_mode = p->ghost_mode;
  c->fixed_dt = p->fixed_dt;
  c->dt_cap = p->dt_cap;
  c->seed = p->seed;
  c->outdir = outdir ? outdir : "/tmp/pcc_ref_out";
  // The Domain constructor creates ./vtk_output_<mode> and writes a parameter
  // file there; build it inside the scratch folder, then restore the cwd.
  std::error_code ec;
  std::filesystem::create_directories(c->outdir, ec);
  auto cwd = std::filesystem::current_path();
  std::filesystem::current_path(c->outdir, ec);
  c->domain = std::make_unique<Domain>(c->params, false, 0, c->params.mode);
  std::filesystem::current_path(cwd, ec);
  return c;
}

void pcc_ref_destroy(void* h) { delete static_cast<RefColony*>(h); }
const char* pcc_ref_last_error(void* h) { return static_cast<RefColony*>(h)->err.c_str(); }

// Replace the colony by n cells (global ids 0..n-1 in the given order).
int pcc_ref_set_cells(void* h, const pcc_cells* cells, size_t n) {
  auto* c = static_cast<RefColony*>(h);
  auto& pm = *c->domain->particle_manager_;
  pm.local_particles.clear();
  pm.ghost_particles.clear();
  for (size_t i = 0; i < n; ++i) {
    Particle p((PetscInt)i, {cells->x[i], cells->y[i], cells->z[i]},
               {cells->q0[i], cells->q1[i], cells->q2[i], cells->q3[i]}, cells->length[i], cells->l0[i],
               cells->diameter[i]);
    if (cells->age) p.getData().age = cells->age[i];
    p.getData().ldot = cells->ldot ? cells->ldot[i] : 0.0;
    if (cells->impedance) p.setImpedance(cells->impedance[i]);
    if (cells->stress) p.setStress(cells->stress[i]);
    pm.local_particles.push_back(p);
  }
  c->domain->global_particle_count = (int)n;
  pm.global_particle_count = (PetscInt)n;
  c->colony_radius = colony_radius_of(*c->domain);
  return 0;
}

int pcc_ref_get_cells(void* h, pcc_cells* out, size_t cap, size_t* n) {
  auto* c = static_cast<RefColony*>(h);
  auto& pm = *c->domain->particle_manager_;
  *n = pm.local_particles.size();
  if (cap < *n) return PCC_ERR_CAPACITY;
  for (size_t i = 0; i < *n; ++i) {
    const Particle& p = pm.local_particles[i];
    const auto& d = p.getData();
    out->x[i] = d.position[0];
    out->y[i] = d.position[1];
    out->z[i] = d.position[2];
    out->q0[i] = d.quaternion[0];
    out->q1[i] = d.quaternion[1];
    out->q2[i] = d.quaternion[2];
    out->q3[i] = d.quaternion[3];
    out->length[i] = d.length;
    out->l0[i] = d.l0;
    out->diameter[i] = d.diameter;
    if (out->ldot) out->ldot[i] = d.ldot;
    if (out->impedance) out->impedance[i] = p.getImpedance();
    if (out->stress) out->stress[i] = p.getStress();
    if (out->age) out->age[i] = d.age;
    if (out->num_constraints) out->num_constraints[i] = p.getNumConstraints();
    if (out->force) {
      for (int k = 0; k < 3; ++k) out->force[6 * i + k] = p.getForce()[k];
      for (int k = 0; k < 3; ++k) out->force[6 * i + 3 + k] = p.getTorque()[k];
    }
    if (out->velocity) {
      for (int k = 0; k < 3; ++k) out->velocity[6 * i + k] = p.getVelocityLinear()[k];
      for (int k = 0; k < 3; ++k) out->velocity[6 * i + 3 + k] = p.getVelocityAngular()[k];
    }
  }
  return 0;
}

static void exchange_ghosts(RefColony* c) {
  if (c->ghost_mode == PCC_GHOSTS_SINGLE_RANK)
    c->domain->exchangeGhostParticles();  // spatial/Domain.cpp:339-403 at world size 1
  else
    c->domain->particle_manager_->ghost_particles.clear();
}

// ParticleManager::step on the current cells (which keep their order and ids).
int pcc_ref_solve(void* h, double dt, int iter, pcc_step_stats* st) {
  auto* c = static_cast<RefColony*>(h);
  Domain& d = *c->domain;
  c->params.sim_config.dt_s = dt;
  pcc_ref_set_division_stream(c->seed, c->div_index);
  auto fn = [c, &d]() {
    d.rebalance();
    exchange_ghosts(c);
  };
  // a BBPGD trace is written to ./logs: run inside the scratch folder
  std::error_code ec;
  auto cwd = std::filesystem::current_path();
  std::filesystem::current_path(c->outdir, ec);
  struct Back {
    std::filesystem::path p;
    ~Back() {
      std::error_code e2;
      std::filesystem::current_path(p, e2);
    }
  } back{cwd};
  try {
    auto sol = d.particle_manager_->step(iter, fn);
    c->last_constraints = std::move(sol.constraints);
    if (st) {
      st->relcp_iterations = sol.constraint_iterations;
      st->bbpgd_iterations = (long long)sol.bbpgd_iterations;
      st->residual = sol.residual;
      st->max_overlap = sol.max_overlap;
      st->n_constraints = (long long)c->last_constraints.size();
      st->n_cells = (long long)d.particle_manager_->local_particles.size();
      st->dt_used = dt;
    }
  } catch (const std::exception& e) {
    c->err = e.what();
    std::string w = e.what();
    if (w.find("BBPGD") != std::string::npos) return PCC_ERR_NOCONV_BBPGD;
    if (w.find("constraint iterations") != std::string::npos) return PCC_ERR_NOCONV_RELCP;
    return PCC_ERR_INVALID;
  }
  return 0;
}

// One Domain::run iteration (spatial/Domain.cpp:125-153) without logging.
int pcc_ref_step(void* h, pcc_step_stats* st) {
  auto* c = static_cast<RefColony*>(h);
  Domain& d = *c->domain;
  auto& pm = *d.particle_manager_;
  pcc_ref_set_division_stream(c->seed, c->div_index);
  auto new_particles = pm.divideParticles();
  c->div_index = pcc_ref_division_index();
  d.queueNewParticles(new_particles);
  d.commitNewParticles();
  d.rebalance();
  d.assignGlobalIDs();
  pm.global_particle_count = d.global_particle_count;
  double dt = c->params.sim_config.dt_s;
  pcc_step_stats local{};
  int rc = pcc_ref_solve(h, dt, (int)d.iter, &local);
  if (rc) return rc;
  d.simulation_time_seconds_ += dt;
  if (!c->fixed_dt) {
    d.adaptDt();
    if (c->dt_cap > 0 && c->params.sim_config.dt_s > c->dt_cap) c->params.sim_config.dt_s = c->dt_cap;
  }
  c->colony_radius = colony_radius_of(d);
  d.iter++;
  local.n_divided = (long long)new_particles.size();
  local.dt_next = c->params.sim_config.dt_s;
  local.colony_radius = c->colony_radius;
  local.sim_time = d.simulation_time_seconds_;
  if (st) *st = local;
  return 0;
}

int pcc_ref_run(void* h, double end_radius, long long max_steps, long long* steps_done, double* cell_steps,
                pcc_step_stats* last) {
  auto* c = static_cast<RefColony*>(h);
  long long s = 0;
  double cs = 0;
  pcc_step_stats st{};
  while (c->colony_radius < end_radius && s < max_steps) {
    int rc = pcc_ref_step(h, &st);
    if (rc) return rc;
    cs += (double)st.n_cells;
    ++s;
  }
  if (steps_done) *steps_done = s;
  if (cell_steps) *cell_steps = cs;
  if (last) *last = st;
  return 0;
}

static void export_constraints(const std::vector<Constraint>& cs, pcc_contacts* out) {
  for (size_t k = 0; k < cs.size(); ++k) {
    const Constraint& c = cs[k];
    out->gid_i[k] = c.gidI;
    out->gid_j[k] = c.gidJ;
    out->sd[k] = c.signed_distance;
    for (int a = 0; a < 3; ++a) {
      out->normal[3 * k + a] = c.normI[a];
      out->r_i[3 * k + a] = c.rPosI[a];
      out->r_j[3 * k + a] = c.rPosJ[a];
      out->contact_point[3 * k + a] = c.contactPoint[a];
    }
    out->stress_i[k] = c.stressI;
    out->stress_j[k] = c.stressJ;
    out->gamma[k] = c.gamma;
    out->phase[k] = c.iteration;
  }
}

// CollisionDetector::detectCollisions on the current cells (with the ghost
// copies of the chosen mode in place).
int pcc_ref_detect(void* h, double tol, int phase, pcc_contacts* out, size_t cap, size_t* n) {
  auto* c = static_cast<RefColony*>(h);
  auto& pm = *c->domain->particle_manager_;
  exchange_ghosts(c);
  pm.collision_detector_.reset();
  auto cs = pm.collision_detector_.detectCollisions(pm, phase, tol);
  *n = cs.size();
  if (cap < cs.size()) return PCC_ERR_CAPACITY;
  export_constraints(cs, out);
  return 0;
}

int pcc_ref_get_constraints(void* h, pcc_contacts* out, size_t cap, size_t* n) {
  auto* c = static_cast<RefColony*>(h);
  *n = c->last_constraints.size();
  if (cap < *n) return PCC_ERR_CAPACITY;
  export_constraints(c->last_constraints, out);
  return 0;
}

// The log point of Domain::run (spatial/Domain.cpp:192-196) on the current
// state: particles, ghost particles and the simulation record, written by the
// reference's loggers under <outdir>/vtk_output_<mode>.
int pcc_ref_log_vtk(void* h, const pcc_sim_record* r) {
  auto* c = static_cast<RefColony*>(h);
  std::error_code ec;
  auto cwd = std::filesystem::current_path();
  std::filesystem::current_path(c->outdir, ec);
  if (ec) return PCC_ERR_INVALID;
  Domain& d = *c->domain;
  d.particle_logger_->log(d.particle_manager_->local_particles);
  d.ghost_particle_logger_->log(d.particle_manager_->ghost_particles);
  vtk::SimulationStep st{};
  st.simulation_time_s = r->simulation_time_s;
  st.time_since_last_log_s = r->time_since_last_log_s;
  st.step = (size_t)r->step;
  st.num_particles = r->num_particles;
  st.num_constraints = (size_t)r->num_constraints;
  st.colony_radius = r->colony_radius;
  st.recursive_iterations = r->recursive_iterations;
  st.bbpgd_iterations = (size_t)r->bbpgd_iterations;
  st.max_overlap = r->max_overlap;
  st.residual = r->residual;
  st.dt_s = r->dt_s;
  st.memory_usage_mb = r->memory_usage_mb;
  st.peak_memory_mb = r->peak_memory_mb;
  st.cpu_time_s = r->cpu_time_s;
  st.mpi_comm_time_s = r->mpi_comm_time_s;
  st.load_imbalance = r->load_imbalance;
  d.simulation_logger_->log(st);
  std::filesystem::current_path(cwd, ec);
  return 0;
}

// vtk::VTKStateLoader::loadLatestState on a VTK output directory: the cells
// as the loader builds them (global ids in file order).
int pcc_ref_load_vtk(const char* dir, pcc_cells* out, size_t cap, size_t* n, double* sim_time, long long* step,
                     double* dt) {
  try {
    vtk::VTKStateLoader loader(dir);
    auto state = loader.loadLatestState();
    *n = state.particles.size();
    if (sim_time) *sim_time = state.simulation_time_s;
    if (step) *step = state.step;
    if (dt) *dt = state.dt_s;
    if (!out) return 0;
    if (cap < *n) return PCC_ERR_CAPACITY;
    for (size_t i = 0; i < *n; ++i) {
      const Particle& p = state.particles[i];
      const auto& d = p.getData();
      out->x[i] = d.position[0];
      out->y[i] = d.position[1];
      out->z[i] = d.position[2];
      out->q0[i] = d.quaternion[0];
      out->q1[i] = d.quaternion[1];
      out->q2[i] = d.quaternion[2];
      out->q3[i] = d.quaternion[3];
      out->length[i] = d.length;
      out->l0[i] = d.l0;
      out->diameter[i] = d.diameter;
      if (out->age) out->age[i] = d.age;
      if (out->force) {
        for (int k = 0; k < 3; ++k) out->force[6 * i + k] = p.getForce()[k];
        for (int k = 0; k < 3; ++k) out->force[6 * i + 3 + k] = p.getTorque()[k];
      }
      if (out->velocity) {
        for (int k = 0; k < 3; ++k) out->velocity[6 * i + k] = p.getVelocityLinear()[k];
        for (int k = 0; k < 3; ++k) out->velocity[6 * i + 3 + k] = p.getVelocityAngular()[k];
      }
    }
    return 0;
  } catch (const std::exception&) {
    return PCC_ERR_INVALID;
  }
}

double pcc_ref_get_dt(void* h) { return static_cast<RefColony*>(h)->params.sim_config.dt_s; }
void pcc_ref_set_dt(void* h, double dt) { static_cast<RefColony*>(h)->params.sim_config.dt_s = dt; }
double pcc_ref_colony_radius(void* h) { return static_cast<RefColony*>(h)->colony_radius; }
unsigned long long pcc_ref_division_count(void* h) { return static_cast<RefColony*>(h)->div_index; }

}  // extern "C"
