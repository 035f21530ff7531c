// C++ host face of the device library for the reference driver.
//
// The reference's ParticleManager::step (code/cpp/src/simulation/ParticleManager.cpp:150-166)
// calls solveHardModel / solveSoftPotential (dynamics/models/Hard.h:9, Soft.h:8)
// on its AoS particle vector and gets a SolverSolution back
// (simulation/ParticleManager.h:33-39).  This header offers the same calls over
// the C ABI in pcc_gpu.h: the particles are copied to the device colony, the
// solver runs there, and positions, quaternions, lengths, growth rates,
// impedances, stresses, forces and velocities are copied back into the same
// vector.  Failures throw std::runtime_error with the reference's messages.
#pragma once

#include <array>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "pcc_gpu.h"

namespace pcc {

// The per-cell state the reference keeps in Particle / ParticleData
// (simulation/Particle.h:12-166, simulation/ParticleData.h:8-17).
struct ParticleState {
  int gid = 0;
  std::array<double, 3> position{};
  std::array<double, 4> quaternion{1, 0, 0, 0};
  double length = 1, l0 = 1, ldot = 0, diameter = 0.5;
  int age = 1;
  double impedance = 0, stress = 0;
  std::array<double, 3> force{}, torque{}, velocity_linear{}, velocity_angular{};
};

// dynamics/Constraint.h:6-49
struct ConstraintRecord {
  double signed_distance;
  int gidI, gidJ;
  std::array<double, 3> normI, rPosI, rPosJ, contactPoint;
  double stressI, stressJ;
  int iteration;
  double gamma;
};

// simulation/ParticleManager.h:33-39
struct SolverSolution {
  std::vector<ConstraintRecord> constraints;
  int constraint_iterations = 0;
  size_t bbpgd_iterations = 0;
  double residual = 0;
  double max_overlap = 0;
};

inline void check(pcc_status rc, const pcc_ctx* ctx, const char* what) {
  if (rc == PCC_OK) return;
  if (rc == PCC_ERR_NOCONV_BBPGD) throw std::runtime_error("BBPGD did not converge");
  if (rc == PCC_ERR_NOCONV_RELCP) throw std::runtime_error("Maximum number of constraint iterations reached");
  throw std::runtime_error(std::string(what) + ": " + (ctx ? pcc_last_error(ctx) : "") + " (status " +
                           std::to_string(rc) + ")");
}

// One colony resident on one GPU (RAII over pcc_ctx).
class DeviceColony {
 public:
  explicit DeviceColony(const pcc_params& p, int device = 0) {
    check(pcc_create(&p, device, &ctx_), nullptr, "pcc_create");
  }
  ~DeviceColony() { pcc_destroy(ctx_); }
  DeviceColony(const DeviceColony&) = delete;
  DeviceColony& operator=(const DeviceColony&) = delete;

  pcc_ctx* handle() { return ctx_; }

  void upload(const std::vector<ParticleState>& ps) {
    const size_t n = ps.size();
    resize(n);
    for (size_t i = 0; i < n; ++i) {
      const auto& p = ps[i];
      x_[i] = p.position[0];
      y_[i] = p.position[1];
      z_[i] = p.position[2];
      q0_[i] = p.quaternion[0];
      q1_[i] = p.quaternion[1];
      q2_[i] = p.quaternion[2];
      q3_[i] = p.quaternion[3];
      len_[i] = p.length;
      l0_[i] = p.l0;
      d_[i] = p.diameter;
      ldot_[i] = p.ldot;
      imp_[i] = p.impedance;
      st_[i] = p.stress;
      age_[i] = p.age;
      for (int k = 0; k < 3; ++k) {
        f_[6 * i + k] = p.force[k];
        f_[6 * i + 3 + k] = p.torque[k];
        v_[6 * i + k] = p.velocity_linear[k];
        v_[6 * i + 3 + k] = p.velocity_angular[k];
      }
    }
    pcc_cells c = view();
    check(pcc_upload_cells(ctx_, &c, n), ctx_, "pcc_upload_cells");
  }

  void download(std::vector<ParticleState>& ps) {
    size_t n = 0;
    check(pcc_cell_count(ctx_, &n), ctx_, "pcc_cell_count");
    resize(n);
    pcc_cells c = view();
    check(pcc_download_cells(ctx_, &c, n, &n), ctx_, "pcc_download_cells");
    ps.resize(n);
    for (size_t i = 0; i < n; ++i) {
      auto& p = ps[i];
      p.gid = (int)i;
      p.position = {x_[i], y_[i], z_[i]};
      p.quaternion = {q0_[i], q1_[i], q2_[i], q3_[i]};
      p.length = len_[i];
      p.l0 = l0_[i];
      p.diameter = d_[i];
      p.ldot = ldot_[i];
      p.impedance = imp_[i];
      p.stress = st_[i];
      p.age = age_[i];
      for (int k = 0; k < 3; ++k) {
        p.force[k] = f_[6 * i + k];
        p.torque[k] = f_[6 * i + 3 + k];
        p.velocity_linear[k] = v_[6 * i + k];
        p.velocity_angular[k] = v_[6 * i + 3 + k];
      }
    }
  }

  std::vector<ConstraintRecord> constraints() {
    size_t n = 0;
    check(pcc_get_constraints(ctx_, nullptr, 0, &n), ctx_, "pcc_get_constraints");
    std::vector<int> gi(n), gj(n), ph(n);
    std::vector<double> sd(n), nn(3 * n), ri(3 * n), rj(3 * n), cp(3 * n), si(n), sj(n), g(n);
    pcc_contacts c{gi.data(), gj.data(), sd.data(), nn.data(), ri.data(), rj.data(), cp.data(), si.data(), sj.data(),
                   g.data(), ph.data()};
    check(pcc_get_constraints(ctx_, &c, n, &n), ctx_, "pcc_get_constraints");
    std::vector<ConstraintRecord> out(n);
    for (size_t k = 0; k < n; ++k) {
      auto& r = out[k];
      r.signed_distance = sd[k];
      r.gidI = gi[k];
      r.gidJ = gj[k];
      for (int a = 0; a < 3; ++a) {
        r.normI[a] = nn[3 * k + a];
        r.rPosI[a] = ri[3 * k + a];
        r.rPosJ[a] = rj[3 * k + a];
        r.contactPoint[a] = cp[3 * k + a];
      }
      r.stressI = si[k];
      r.stressJ = sj[k];
      r.iteration = ph[k];
      r.gamma = g[k];
    }
    return out;
  }

  // ParticleManager::step on device-resident cells.
  SolverSolution solve(double dt, int iter, bool with_constraints) {
    pcc_step_stats st{};
    check(pcc_solve(ctx_, dt, iter, &st), ctx_, "pcc_solve");
    SolverSolution s;
    s.constraint_iterations = st.relcp_iterations;
    s.bbpgd_iterations = (size_t)st.bbpgd_iterations;
    s.residual = st.residual;
    s.max_overlap = st.max_overlap;
    if (with_constraints) s.constraints = constraints();
    return s;
  }

  pcc_step_stats step() {
    pcc_step_stats st{};
    check(pcc_step(ctx_, &st), ctx_, "pcc_step");
    return st;
  }

 private:
  void resize(size_t n) {
    for (auto* v : {&x_, &y_, &z_, &q0_, &q1_, &q2_, &q3_, &len_, &l0_, &d_, &ldot_, &imp_, &st_}) v->resize(n + 1);
    f_.resize(6 * n + 6);
    v_.resize(6 * n + 6);
    age_.resize(n + 1);
  }
  pcc_cells view() {
    return pcc_cells{x_.data(), y_.data(), z_.data(), q0_.data(), q1_.data(), q2_.data(),  q3_.data(), len_.data(),
                     l0_.data(), d_.data(), ldot_.data(), imp_.data(), st_.data(), age_.data(), f_.data(), v_.data()};
  }
  pcc_ctx* ctx_ = nullptr;
  std::vector<double> x_, y_, z_, q0_, q1_, q2_, q3_, len_, l0_, d_, ldot_, imp_, st_, f_, v_;
  std::vector<int> age_;
};

// The reference's solver entry points on an AoS particle vector that the
// caller owns (cells in global-id order), as ParticleManager::step calls them.
inline SolverSolution solveHardModel(DeviceColony& dev, std::vector<ParticleState>& local_particles, double dt,
                                     int iter) {
  dev.upload(local_particles);
  SolverSolution s = dev.solve(dt, iter, true);
  dev.download(local_particles);
  return s;
}

inline SolverSolution solveSoftPotential(DeviceColony& dev, std::vector<ParticleState>& local_particles, double dt,
                                         int iter) {
  return solveHardModel(dev, local_particles, dt, iter);  // the context's mode selects the model
}

}  // namespace pcc
