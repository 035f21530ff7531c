// C ABI of the collision hot path (include/pcc_gpu.h): context management,
// state transfer and the host-side sequencing of one solver call / one step.
//
// Host orchestration mirrors the reference: solveHardModel's ReLCP loop
// (dynamics/models/Hard.cpp:91-192), solveSoftPotential (Soft.cpp:21-114) and
// one Domain::run iteration (spatial/Domain.cpp:125-153).  Every numeric pass
// runs on the device; the host reads back only the scalars that steer the
// loop (new-constraint count, largest overlap, BBPGD exit state, colony radius).
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "pcc_kernels.hpp"

namespace pcc {

cudaError_t CellBufs::reserve(size_t n, size_t keep, cudaStream_t s) {
  cudaError_t e;
  DevBuf<double>* d[] = {&x, &y, &z, &q0, &q1, &q2, &q3, &len, &l0, &diam, &ldot, &imp, &stress};
  for (auto* b : d)
    if ((e = b->reserve(n + 1, keep, s))) return e;
  if ((e = force.reserve(6 * (n + 1), 6 * keep, s))) return e;
  if ((e = vel.reserve(6 * (n + 1), 6 * keep, s))) return e;
  if ((e = age.reserve(n + 1, keep, s))) return e;
  if ((e = ncons.reserve(n + 1, keep, s))) return e;
  return cudaSuccess;
}

CellsView CellBufs::view() {
  return CellsView{x.p, y.p, z.p, q0.p, q1.p, q2.p, q3.p, len.p, l0.p, diam.p, ldot.p, imp.p, stress.p, age.p,
                   force.p, vel.p, ncons.p};
}

template <typename T>
static void swap_buf(DevBuf<T>& a, DevBuf<T>& b) {
  T* p = a.p;
  size_t c = a.cap;
  a.p = b.p;
  a.cap = b.cap;
  b.p = p;
  b.cap = c;
}

void CellBufs::swap(CellBufs& o) {
  swap_buf(x, o.x);
  swap_buf(y, o.y);
  swap_buf(z, o.z);
  swap_buf(q0, o.q0);
  swap_buf(q1, o.q1);
  swap_buf(q2, o.q2);
  swap_buf(q3, o.q3);
  swap_buf(len, o.len);
  swap_buf(l0, o.l0);
  swap_buf(diam, o.diam);
  swap_buf(ldot, o.ldot);
  swap_buf(imp, o.imp);
  swap_buf(stress, o.stress);
  swap_buf(force, o.force);
  swap_buf(vel, o.vel);
  swap_buf(age, o.age);
  swap_buf(ncons, o.ncons);
}

cudaError_t ConsBufs::reserve(size_t n, size_t keep, cudaStream_t s) {
  cudaError_t e;
  DevBuf<int>* ib[] = {&gi, &gj, &phase};
  for (auto* b : ib)
    if ((e = b->reserve(n + 1, keep, s))) return e;
  DevBuf<double>* db[] = {&sd, &gamma, &nx, &ny, &nz, &tix, &tiy, &tiz, &tjx, &tjy, &tjz, &rix, &riy,
                          &riz, &rjx, &rjy, &rjz, &cpx, &cpy, &cpz, &si, &sj};
  for (auto* b : db)
    if ((e = b->reserve(n + 1, keep, s))) return e;
  return cudaSuccess;
}

ConsView ConsBufs::view() {
  return ConsView{gi.p,  gj.p,  phase.p, sd.p,  gamma.p, nx.p,  ny.p,  nz.p,  tix.p, tiy.p, tiz.p, tjx.p,
                  tjy.p, tjz.p, rix.p,   riy.p, riz.p,   rjx.p, rjy.p, rjz.p, cpx.p, cpy.p, cpz.p, si.p, sj.p};
}

}  // namespace pcc

using namespace pcc;

namespace {

pcc_status fail(pcc_ctx* ctx, pcc_status code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

pcc_status cuda_fail(pcc_ctx* ctx, cudaError_t e, const char* where) {
  std::string m = std::string(where) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return fail(ctx, PCC_ERR_NOMEM, m);
  return fail(ctx, PCC_ERR_CUDA, m);
}

// Reads the device status word; a raised flag becomes an error code.
pcc_status check_device(pcc_ctx* ctx, const char* where) {
  cudaError_t e = cudaMemcpyAsync(ctx->status_host, ctx->status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (!e) e = cudaStreamSynchronize(ctx->stream);
  if (e) return cuda_fail(ctx, e, where);
  unsigned f = ctx->status_host->flags;
  if (!f) return PCC_OK;
  char buf[160];
  std::snprintf(buf, sizeof buf, "%s: device check failed (flags 0x%x at site %d)", where, f, ctx->status_host->where);
  cudaMemsetAsync(ctx->status, 0, sizeof(DevStatus), ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  if (f & kDevErrTimeout) return fail(ctx, PCC_ERR_TIMEOUT, buf);
  if (f & kDevErrCapacity) return fail(ctx, PCC_ERR_CAPACITY, buf);
  if (f & kDevErrNan) return fail(ctx, PCC_ERR_NAN, buf);
  return fail(ctx, PCC_ERR_BOUNDS, buf);
}

// Adds the device time since ev[2] to the detection account.
void profile_detect(pcc_ctx* ctx) {
  if (!ctx->profiling) return;
  cudaEventRecord(ctx->ev[3], ctx->stream);
  cudaEventSynchronize(ctx->ev[3]);
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
  ctx->prof.detect_ms += ms;
}

#define CU(call, where)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
  } while (0)

// The ReLCP loop (Hard.cpp:91-192).  Host round trips: the detection pass of
// each phase synchronises once (twice when it rebins); the largest overlap of
// the earlier phases' constraints and the previous BBPGD launch's scalars ride
// on that synchronisation instead of waiting on their own.  end_check: read
// the device status before returning (a step defers it to its own single
// end-of-step synchronisation).
pcc_status solve_hard(pcc_ctx* ctx, double dt, int iter, pcc_step_stats* st, bool end_check) {
  const double tol = ctx->params.tolerance;
  int phase = 0;
  // BBPGD trace on every 10th step (dynamics/models/Hard.cpp:107-111); a new
  // logger clears the earlier trace files
  ctx->trace_active = (ctx->params.log_bbpgd_trace == 1 && iter % 10 == 0) || ctx->params.log_bbpgd_trace == 2;
  if (ctx->trace_active) {
    ctx->trace_host.clear();
    vtk_clear_prefix(ctx->trace_dir, "bbpgdtrace");
  }
  long long total_it = 0;
  double res = 0.0, max_ov = 0.0;
  ctx->ncons = 0;
  ctx->bbpgd_pending = false;
  CU(reset_ldot(ctx), "reset");
  CU(mobility(ctx), "mobility");
  // U_ext: Brownian kicks at ReLCP phase 0 only (Hard.cpp:138-143, Physics.cpp:68)
  CU(brownian_draw(ctx), "brownian");
  // reads the scalars of a BBPGD launch after a synchronisation point
  auto collect = [&]() -> pcc_status {
    if (!ctx->bbpgd_pending) return PCC_OK;
    long long it = 0;
    int status = 0;
    bbpgd_collect(ctx, &it, &res, &status);
    total_it += it;
    if (status == PCC_ERR_NOCONV_BBPGD) return fail(ctx, status, "BBPGD did not converge");
    if (status) {
      pcc_status dev = check_device(ctx, "bbpgd");
      return dev ? dev : fail(ctx, status, "BBPGD device error");
    }
    return PCC_OK;
  };
  while ((long long)phase < ctx->params.max_recursive_iterations) {
    const size_t before = ctx->ncons;
    if (before) CU(max_overlap_enqueue(ctx, 0, before), "max_overlap");
    size_t added = 0;
    double ov_new = 0.0;
    if (ctx->profiling) cudaEventRecord(ctx->ev[2], ctx->stream);
    CU(detect_contacts(ctx, phase == 0 ? .25 : tol, phase, phase > 0, &added, &ov_new), "detect");
    if (ctx->n == 0) CU(cudaStreamSynchronize(ctx->stream), "detect");  // an empty colony's detection did not wait
    pcc_status rc = collect();  // the previous phase's BBPGD, now complete
    if (rc) return rc;
    double ov_old = 0.0;
    if (before) std::memcpy(&ov_old, ctx->pinned_ll + kSlotMaxOld, sizeof ov_old);
    max_ov = ov_old < ov_new ? ov_new : ov_old;
    if (max_ov <= tol && phase > 0) {
      profile_detect(ctx);
      break;
    }
    CU(build_incidence(ctx), "incidence");
    profile_detect(ctx);
    ctx->trace_phase = phase;
    long long it = 0;
    int status = 0;
    CU(bbpgd_solve(ctx, dt, &it, &res, &status, /*defer=*/true), "bbpgd");
    ctx->uext_active = false;
    if (!ctx->bbpgd_pending) {  // a traced solve synchronised and was read already
      total_it += it;
      if (status == PCC_ERR_NOCONV_BBPGD) return fail(ctx, status, "BBPGD did not converge");
      if (status) {
        pcc_status dev = check_device(ctx, "bbpgd");
        return dev ? dev : fail(ctx, status, "BBPGD device error");
      }
    }
    CU(apply_hard_solution(ctx, dt), "move");
    ++phase;
  }
  if (ctx->bbpgd_pending) {  // the loop ran out of phases right after a solve
    CU(cudaStreamSynchronize(ctx->stream), "bbpgd");
    pcc_status rc = collect();
    if (rc) return rc;
  }
  if (ctx->trace_active) {
    ctx->trace_active = false;
    // BBPGDLogger("logs", "bbpgdtrace", true): the third argument lands on the
    // logger's starting index, so files count from 1 (logger/BBPGDLogger.h:23-27)
    if (!vtk_write_trace(ctx->trace_dir, 1, ctx->trace_host))
      return fail(ctx, PCC_ERR_INVALID, "cannot write the BBPGD trace files");
  }
  CU(grow_cells(ctx, dt), "grow");
  if (end_check) {
    pcc_status rc = check_device(ctx, "hard step");
    if (rc) return rc;
  }
  if (st) {
    st->relcp_iterations = phase;
    st->bbpgd_iterations = total_it;
    st->residual = res;
    st->max_overlap = max_ov;
    st->n_constraints = (long long)ctx->ncons;
    st->n_cells = (long long)ctx->n;
  }
  if ((long long)phase == ctx->params.max_recursive_iterations)
    return fail(ctx, PCC_ERR_NOCONV_RELCP, "Maximum number of constraint iterations reached");
  return PCC_OK;
}

pcc_status solve_soft(pcc_ctx* ctx, double dt, pcc_step_stats* st, bool end_check) {
  ctx->ncons = 0;
  CU(reset_ldot(ctx), "reset");
  CU(brownian_draw(ctx), "brownian");  // Soft.cpp:94
  size_t added = 0;
  double max_ov = 0.0;
  if (ctx->profiling) cudaEventRecord(ctx->ev[2], ctx->stream);
  CU(detect_contacts(ctx, 0.0, 0, false, &added, &max_ov), "detect");
  CU(build_incidence(ctx), "incidence");
  profile_detect(ctx);
  CU(soft_forces_and_move(ctx, dt), "soft");
  ctx->uext_active = false;
  CU(grow_cells(ctx, dt), "grow");
  if (end_check) {
    pcc_status rc = check_device(ctx, "soft step");
    if (rc) return rc;
  }
  if (st) {
    st->relcp_iterations = 0;
    st->bbpgd_iterations = 0;
    st->residual = max_ov;
    st->max_overlap = max_ov;
    st->n_constraints = (long long)ctx->ncons;
    st->n_cells = (long long)ctx->n;
  }
  return PCC_OK;
}

// One solver call (ParticleManager::step).
pcc_status solve(pcc_ctx* ctx, double dt, int iter, pcc_step_stats* out, bool end_check) {
  pcc_step_stats st;
  std::memset(&st, 0, sizeof st);
  ctx->div_known = false;  // lengths change
  if (ctx->profiling) cudaEventRecord(ctx->ev[4], ctx->stream);
  if (ctx->n) CU(cudaMemsetAsync(ctx->cells.ncons.p, 0, ctx->n * sizeof(int), ctx->stream), "reset");  // Particle::reset
  pcc_status rc = ctx->params.mode == PCC_MODE_SOFT ? solve_soft(ctx, dt, &st, end_check)
                                                    : solve_hard(ctx, dt, iter, &st, end_check);
  st.dt_used = dt;
  if (ctx->profiling) {
    cudaEventRecord(ctx->ev[5], ctx->stream);
    cudaEventSynchronize(ctx->ev[5]);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev[4], ctx->ev[5]);
    ctx->prof.solve_ms += ms;
    ctx->prof.solves++;
    ctx->prof.cell_solves += (double)st.n_cells;
  }
  if (out) *out = st;
  return rc;
}

pcc_status download_contacts(pcc_ctx* ctx, size_t m, pcc_contacts* o) {
  cudaStream_t s = ctx->stream;
  auto cp_d = [&](double* dst, const double* src) {
    if (dst) cudaMemcpyAsync(dst, src, m * sizeof(double), cudaMemcpyDeviceToHost, s);
  };
  auto cp_i = [&](int* dst, const int* src) {
    if (dst) cudaMemcpyAsync(dst, src, m * sizeof(int), cudaMemcpyDeviceToHost, s);
  };
  ConsView v = ctx->cons.view();
  cp_i(o->gid_i, v.gi);
  cp_i(o->gid_j, v.gj);
  cp_i(o->phase, v.phase);
  cp_d(o->sd, v.sd);
  cp_d(o->stress_i, v.si);
  cp_d(o->stress_j, v.sj);
  cp_d(o->gamma, v.gamma);
  std::vector<double> tmp(3 * m);
  const double* trip[4][3] = {{v.nx, v.ny, v.nz}, {v.rix, v.riy, v.riz}, {v.rjx, v.rjy, v.rjz}, {v.cpx, v.cpy, v.cpz}};
  double* outs[4] = {o->normal, o->r_i, o->r_j, o->contact_point};
  cudaError_t e = cudaStreamSynchronize(s);
  if (e) return cuda_fail(ctx, e, "download contacts");
  for (int f = 0; f < 4; ++f) {
    if (!outs[f]) continue;
    for (int d = 0; d < 3; ++d) cudaMemcpyAsync(tmp.data() + d * m, trip[f][d], m * sizeof(double), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e) return cuda_fail(ctx, e, "download contacts");
    for (size_t k = 0; k < m; ++k)
      for (int d = 0; d < 3; ++d) outs[f][3 * k + d] = tmp[d * m + k];
  }
  return PCC_OK;
}

}  // namespace

extern "C" {

void pcc_default_params(pcc_params* p) {
  std::memset(p, 0, sizeof *p);
  p->dt = 1e-2;
  p->end_radius = 50;
  p->xi = 1;
  p->tau = 1;
  p->l0 = 1.0;
  p->lambda = 1e-2;
  p->temperature = 0.0;
  p->kcc = 20000;
  p->monolayer = 1;
  p->tolerance = 1e-3;
  p->max_bbpgd_iterations = 500000;
  p->max_recursive_iterations = 50;
  p->linked_cell_size = 2.2 * p->l0;
  p->cfl_factor = 0.5;
  p->mode = PCC_MODE_HARD;
  p->ghost_mode = PCC_GHOSTS_SINGLE_RANK;
  p->log_every_colony_radius_delta = 0.5;
  p->log_every_sim_time_delta = 100000;
}

pcc_status pcc_create(const pcc_params* params, int device, pcc_ctx** out) {
  if (!params || !out) return PCC_ERR_INVALID;
  *out = nullptr;
  if (!(params->temperature >= 0)) return PCC_ERR_INVALID;
  if (params->mode != PCC_MODE_HARD && params->mode != PCC_MODE_SOFT) return PCC_ERR_INVALID;
  if (params->precision != PCC_PRECISION_FP64 && params->precision != PCC_PRECISION_MIXED) return PCC_ERR_INVALID;
  if (!(params->linked_cell_size > 0) || !(params->xi > 0) || !(params->tau > 0)) return PCC_ERR_INVALID;
  pcc_ctx* ctx = new (std::nothrow) pcc_ctx();
  if (!ctx) return PCC_ERR_NOMEM;
  ctx->params = *params;
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (!e) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (!e) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (!e) {
    // keep freed stream-ordered blocks cached in the process (no return to
    // the driver at every synchronisation)
    cudaMemPool_t pool;
    unsigned long long keep_all = ~0ULL;
    e = cudaDeviceGetDefaultMemPool(&pool, device);
    if (!e) e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep_all);
  }
  if (!e) e = cudaMallocAsync(&ctx->status, sizeof(DevStatus), ctx->stream);
  if (!e) e = cudaMallocHost(&ctx->status_host, sizeof(DevStatus));
  if (!e) e = cudaMallocHost(&ctx->pinned_ll, 64 * sizeof(long long));
  if (!e) e = cudaMallocHost(&ctx->scal_host, sizeof(SolverScalars));
  if (!e) e = cudaMemsetAsync(ctx->status, 0, sizeof(DevStatus), ctx->stream);
  if (!e && params->capacity_hint > 0) e = ctx->cells.reserve((size_t)params->capacity_hint, 0, ctx->stream);
  if (!e) e = cudaStreamSynchronize(ctx->stream);
  if (e) {
    std::fprintf(stderr, "pcc_create: %s\n", cudaGetErrorString(e));
    pcc_destroy(ctx);
    return e == cudaErrorMemoryAllocation ? PCC_ERR_NOMEM : PCC_ERR_CUDA;
  }
  *out = ctx;
  return PCC_OK;
}

pcc_status pcc_destroy(pcc_ctx* ctx) {
  if (!ctx) return PCC_OK;
  cudaSetDevice(ctx->device);
  vtk_writer_shutdown(ctx);
  if (ctx->vtk_stream) {
    cudaStreamSynchronize(ctx->vtk_stream);
    cudaStreamDestroy(ctx->vtk_stream);
  }
  if (ctx->vtk_ev) cudaEventDestroy(ctx->vtk_ev);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& e : ctx->ev)
    if (e) cudaEventDestroy(e);
  if (ctx->status) cudaFreeAsync(ctx->status, ctx->stream);
  if (ctx->status_host) cudaFreeHost(ctx->status_host);
  if (ctx->pinned_ll) cudaFreeHost(ctx->pinned_ll);
  if (ctx->scal_host) cudaFreeHost(ctx->scal_host);
  if (ctx->brown_host) cudaFreeHost(ctx->brown_host);
  cudaStream_t s = ctx->stream;
  delete ctx;  // device buffers are freed on the context's stream
  if (s) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  return PCC_OK;
}

const char* pcc_last_error(const pcc_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

pcc_status pcc_set_dt(pcc_ctx* ctx, double dt) {
  if (!ctx || !(dt > 0)) return PCC_ERR_INVALID;
  ctx->params.dt = dt;
  return PCC_OK;
}

pcc_status pcc_get_dt(const pcc_ctx* ctx, double* dt) {
  if (!ctx || !dt) return PCC_ERR_INVALID;
  *dt = ctx->params.dt;
  return PCC_OK;
}

pcc_status pcc_upload_cells(pcc_ctx* ctx, const pcc_cells* c, size_t n) {
  if (!ctx || !c) return PCC_ERR_INVALID;
  if (n > 0x3fffffff) return fail(ctx, PCC_ERR_INVALID, "too many cells (ids are 32-bit)");
  if (n && (!c->x || !c->y || !c->z || !c->q0 || !c->q1 || !c->q2 || !c->q3 || !c->length || !c->l0 || !c->diameter))
    return fail(ctx, PCC_ERR_INVALID, "pcc_upload_cells: required array missing");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  CU(ctx->cells.reserve(n, 0, s), "upload");
  auto h2d = [&](double* dst, const double* src, size_t cnt) {
    if (src)
      cudaMemcpyAsync(dst, src, cnt * sizeof(double), cudaMemcpyHostToDevice, s);
    else
      cudaMemsetAsync(dst, 0, cnt * sizeof(double), s);
  };
  CellsView v = ctx->cells.view();
  h2d(v.x, c->x, n);
  h2d(v.y, c->y, n);
  h2d(v.z, c->z, n);
  h2d(v.q0, c->q0, n);
  h2d(v.q1, c->q1, n);
  h2d(v.q2, c->q2, n);
  h2d(v.q3, c->q3, n);
  h2d(v.len, c->length, n);
  h2d(v.l0, c->l0, n);
  h2d(v.diam, c->diameter, n);
  h2d(v.ldot, c->ldot, n);
  h2d(v.imp, c->impedance, n);
  h2d(v.stress, c->stress, n);
  h2d(v.force, c->force, 6 * n);
  h2d(v.vel, c->velocity, 6 * n);
  if (c->age)
    cudaMemcpyAsync(v.age, c->age, n * sizeof(int), cudaMemcpyHostToDevice, s);
  else {
    std::vector<int> ones(n ? n : 1, 1);
    cudaMemcpyAsync(v.age, ones.data(), n * sizeof(int), cudaMemcpyHostToDevice, s);
    CU(cudaStreamSynchronize(s), "upload");
  }
  if (n) cudaMemsetAsync(v.ncons, 0, n * sizeof(int), s);
  ctx->n = n;
  ctx->ncons = 0;
  ctx->div_known = false;
  CU(cudaStreamSynchronize(s), "upload");
  CU(colony_radius(ctx, &ctx->radius), "radius");
  return PCC_OK;
}

pcc_status pcc_cell_count(const pcc_ctx* ctx, size_t* n) {
  if (!ctx || !n) return PCC_ERR_INVALID;
  *n = ctx->n;
  return PCC_OK;
}

pcc_status pcc_download_cells(pcc_ctx* ctx, pcc_cells* c, size_t cap, size_t* n) {
  if (!ctx || !c || !n) return PCC_ERR_INVALID;
  *n = ctx->n;
  if (cap < ctx->n) return fail(ctx, PCC_ERR_CAPACITY, "pcc_download_cells: buffer too small");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const size_t m = ctx->n;
  CellsView v = ctx->cells.view();
  auto d2h = [&](double* dst, const double* src, size_t cnt) {
    if (dst && cnt) cudaMemcpyAsync(dst, src, cnt * sizeof(double), cudaMemcpyDeviceToHost, s);
  };
  d2h(c->x, v.x, m);
  d2h(c->y, v.y, m);
  d2h(c->z, v.z, m);
  d2h(c->q0, v.q0, m);
  d2h(c->q1, v.q1, m);
  d2h(c->q2, v.q2, m);
  d2h(c->q3, v.q3, m);
  d2h(c->length, v.len, m);
  d2h(c->l0, v.l0, m);
  d2h(c->diameter, v.diam, m);
  d2h(c->ldot, v.ldot, m);
  d2h(c->impedance, v.imp, m);
  d2h(c->stress, v.stress, m);
  d2h(c->force, v.force, 6 * m);
  d2h(c->velocity, v.vel, 6 * m);
  if (c->age && m) cudaMemcpyAsync(c->age, v.age, m * sizeof(int), cudaMemcpyDeviceToHost, s);
  if (c->num_constraints && m) cudaMemcpyAsync(c->num_constraints, v.ncons, m * sizeof(int), cudaMemcpyDeviceToHost, s);
  CU(cudaStreamSynchronize(s), "download");
  return PCC_OK;
}

pcc_status pcc_solve(pcc_ctx* ctx, double dt, int iter, pcc_step_stats* out) {
  if (!ctx || !(dt > 0)) return PCC_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return solve(ctx, dt, iter, out, /*end_check=*/true);
}

// One Domain::run iteration (Domain.cpp:125-153).  The end-of-step work --
// the device status, the adaptDt median, the colony radius and the division
// count of the next step -- comes back in one copy after one synchronisation;
// the next step's divisions use that count without waiting again.
pcc_status pcc_step(pcc_ctx* ctx, pcc_step_stats* out) {
  if (!ctx) return PCC_ERR_INVALID;
  cudaSetDevice(ctx->device);
  pcc_step_stats st;
  std::memset(&st, 0, sizeof st);
  size_t added = 0;
  CU(divide_cells(ctx, &added), "divide");
  CU(sort_cells_by_x(ctx), "sort");
  const double dt = ctx->params.dt;
  pcc_status rc = solve(ctx, dt, (int)ctx->iter, &st, /*end_check=*/false);
  if (rc) {
    if (out) *out = st;
    return rc;
  }
  ctx->sim_time += dt;
  if (!ctx->params.fixed_dt) CU(adapt_dt_enqueue(ctx), "adapt_dt");
  CU(radius_enqueue(ctx), "radius");
  CU(division_count_enqueue(ctx), "divide");
  CU(cudaMemcpyAsync(ctx->status_host, ctx->status, sizeof(DevStatus), cudaMemcpyDeviceToHost, ctx->stream), "step");
  CU(cudaStreamSynchronize(ctx->stream), "step");
  if (ctx->status_host->flags) {
    rc = check_device(ctx, ctx->params.mode == PCC_MODE_SOFT ? "soft step" : "hard step");
    if (rc) {
      if (out) *out = st;
      return rc;
    }
  }
  if (!ctx->params.fixed_dt) {
    adapt_dt_collect(ctx);
    if (ctx->params.dt_cap > 0 && ctx->params.dt > ctx->params.dt_cap) ctx->params.dt = ctx->params.dt_cap;
  }
  ctx->radius = radius_collect(ctx);
  ctx->div_next = (size_t) * reinterpret_cast<int*>(ctx->pinned_ll + kSlotDivs);
  ctx->div_known = true;
  ctx->iter++;
  st.n_divided = (long long)added;
  st.dt_used = dt;
  st.dt_next = ctx->params.dt;
  st.colony_radius = ctx->radius;
  st.sim_time = ctx->sim_time;
  if (out) *out = st;
  return PCC_OK;
}

pcc_status pcc_run(pcc_ctx* ctx, double end_radius, long long max_steps, long long* steps_done, double* cell_steps,
                   pcc_step_stats* last) {
  if (!ctx) return PCC_ERR_INVALID;
  long long s = 0;
  double cs = 0;
  pcc_step_stats st;
  std::memset(&st, 0, sizeof st);
  pcc_status rc = PCC_OK;
  while (ctx->radius < end_radius && s < max_steps) {
    rc = pcc_step(ctx, &st);
    if (rc) break;
    cs += (double)st.n_cells;
    ++s;
  }
  if (steps_done) *steps_done = s;
  if (cell_steps) *cell_steps = cs;
  if (last) *last = st;
  return rc;
}

pcc_status pcc_detect_contacts(pcc_ctx* ctx, double tol, int phase, pcc_contacts* out, size_t cap, size_t* n) {
  if (!ctx || !n) return PCC_ERR_INVALID;
  cudaSetDevice(ctx->device);
  ctx->ncons = 0;
  size_t added = 0;
  double mo = 0;
  CU(detect_contacts(ctx, tol, phase, false, &added, &mo), "detect");
  pcc_status rc = check_device(ctx, "detect");
  if (rc) return rc;
  *n = ctx->ncons;
  if (!out) return PCC_OK;
  if (cap < ctx->ncons) return fail(ctx, PCC_ERR_CAPACITY, "pcc_detect_contacts: buffer too small");
  return download_contacts(ctx, ctx->ncons, out);
}

pcc_status pcc_get_constraints(pcc_ctx* ctx, pcc_contacts* out, size_t cap, size_t* n) {
  if (!ctx || !n) return PCC_ERR_INVALID;
  cudaSetDevice(ctx->device);
  *n = ctx->ncons;
  if (!out) return PCC_OK;
  if (cap < ctx->ncons) return fail(ctx, PCC_ERR_CAPACITY, "pcc_get_constraints: buffer too small");
  return download_contacts(ctx, ctx->ncons, out);
}

pcc_status pcc_bbpgd_frozen(pcc_ctx* ctx, double dt, int repeats, long long* iterations, double* residual,
                            float* ms_per_solve) {
  if (!ctx || repeats < 1) return PCC_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  ctx->ncons = 0;
  size_t added = 0;
  double mo = 0;
  CU(reset_ldot(ctx), "reset");
  CU(mobility(ctx), "mobility");
  CU(detect_contacts(ctx, 0.25, 0, false, &added, &mo), "detect");
  CU(build_incidence(ctx), "incidence");
  const size_t m = ctx->ncons;
  DevBuf<double> sd0, g0;
  CU(sd0.reserve(m + 1, 0, s), "frozen");
  CU(g0.reserve(m + 1, 0, s), "frozen");
  CU(cudaMemcpyAsync(sd0.p, ctx->cons.sd.p, m * sizeof(double), cudaMemcpyDeviceToDevice, s), "frozen");
  CU(cudaMemcpyAsync(g0.p, ctx->cons.gamma.p, m * sizeof(double), cudaMemcpyDeviceToDevice, s), "frozen");
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float total = 0;
  long long it = 0;
  double res = 0;
  for (int r = 0; r <= repeats; ++r) {  // solve 0 is an untimed warm-up (buffers, occupancy query)
    cudaMemcpyAsync(ctx->cons.sd.p, sd0.p, m * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(ctx->cons.gamma.p, g0.p, m * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaEventRecord(a, s);
    int status = 0;
    cudaError_t e = bbpgd_solve(ctx, dt, &it, &res, &status);
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (r > 0) total += ms;
    if (e) {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      return cuda_fail(ctx, e, "bbpgd");
    }
    if (status) {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      return fail(ctx, status, "BBPGD did not converge");
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (iterations) *iterations = it;
  if (residual) *residual = res;
  if (ms_per_solve) *ms_per_solve = total / repeats;
  return check_device(ctx, "bbpgd_frozen");
}

pcc_status pcc_soft_forces_frozen(pcc_ctx* ctx, int repeats, float* ms_per_assembly) {
  if (!ctx || repeats < 1) return PCC_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  ctx->ncons = 0;
  size_t added = 0;
  double mo = 0;
  CU(detect_contacts(ctx, 0.0, 0, false, &added, &mo), "detect");
  CU(build_incidence(ctx), "incidence");
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, s);
  for (int r = 0; r < repeats; ++r) {
    cudaError_t e = soft_assemble(ctx);
    if (e) {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      return cuda_fail(ctx, e, "soft");
    }
  }
  cudaEventRecord(b, s);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (ms_per_assembly) *ms_per_assembly = ms / repeats;
  return check_device(ctx, "soft_frozen");
}

pcc_status pcc_set_profiling(pcc_ctx* ctx, int on) {
  if (!ctx) return PCC_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (on && !ctx->ev[0]) {
    for (auto& e : ctx->ev) CU(cudaEventCreate(&e), "profiling");
  }
  ctx->profiling = on != 0;
  return PCC_OK;
}

pcc_status pcc_reset_profile(pcc_ctx* ctx) {
  if (!ctx) return PCC_ERR_INVALID;
  std::memset(&ctx->prof, 0, sizeof ctx->prof);
  return PCC_OK;
}

pcc_status pcc_get_profile(const pcc_ctx* ctx, pcc_profile* out) {
  if (!ctx || !out) return PCC_ERR_INVALID;
  *out = ctx->prof;
  return PCC_OK;
}

pcc_status pcc_set_trace_dir(pcc_ctx* ctx, const char* dir) {
  if (!ctx || !dir || !*dir) return PCC_ERR_INVALID;
  ctx->trace_dir = dir;
  return PCC_OK;
}

pcc_status pcc_get_bbpgd_trace(const pcc_ctx* ctx, pcc_bbpgd_trace_step* out, size_t cap, size_t* n) {
  if (!ctx || !n) return PCC_ERR_INVALID;
  *n = ctx->trace_host.size();
  if (!out) return PCC_OK;
  if (cap < *n) return PCC_ERR_CAPACITY;
  std::memcpy(out, ctx->trace_host.data(), *n * sizeof(pcc_bbpgd_trace_step));
  return PCC_OK;
}

void* pcc_get_stream(const pcc_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

long long pcc_launch_count(const pcc_ctx* ctx) { return ctx ? ctx->launches : 0; }

}  // extern "C"
