// Batched and served colonies: many independent colony jobs in flight on one
// GPU at once (continuous batching).
//
// Each admitted job gets its own context (device state), its own non-blocking
// CUDA stream and its own host thread, which drives the job's steps through
// the same pcc_step path as a single colony.  Small colonies are bound by
// per-step latency (kernel launches, a few small read-backs per ReLCP phase),
// so running many at once lets their kernels overlap on the device and
// multiplies aggregate throughput.  Jobs are admitted in arrival order when
// (a) they have arrived, (b) a slot is free and (c) their projected device
// footprint at their final radius fits in the HBM budget next to the jobs in
// flight; a finishing job frees its slot and budget for the next one.  Jobs
// share nothing on the device, and every kernel's result is independent of
// timing, so a job's result is bit-identical alone and in any mix.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "pcc_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

// Projected device bytes of a colony grown to radius R: about 4.5 R^2 cells
// (the reference's 301,116 cells at R = 260), each with its state, up to ~17
// accumulated constraints per cell late in a step, the solver's packed copies
// and scratch -- 5 KiB per cell in total -- plus a fixed per-context part.
double projected_footprint(double radius) {
  const double cells = 4.5 * radius * radius + 64.0;
  return cells * 5120.0 + 32.0 * 1024 * 1024;
}

// theta ~ U[0, pi) from the job seed (splitmix64 finaliser, 53-bit mantissa).
double seed_angle(unsigned long long seed) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0) * M_PI;
}

void run_job(const pcc_job& job, int device, Clock::time_point t0, pcc_job_result* r) {
  auto since = [&](Clock::time_point t) { return std::chrono::duration<double>(t - t0).count(); };
  r->start_s = since(Clock::now());
  pcc_ctx* ctx = nullptr;
  pcc_status rc = pcc_create(&job.params, device, &ctx);
  if (rc == PCC_OK) {
    const double th = seed_angle(job.params.seed);
    double x = 0, y = 0, z = 0, q0 = std::cos(th / 2), q1 = 0, q2 = 0, q3 = std::sin(th / 2);
    double len = job.params.l0, l0 = job.params.l0, d = job.params.l0 / 2;
    pcc_cells c;
    std::memset(&c, 0, sizeof c);
    c.x = &x;
    c.y = &y;
    c.z = &z;
    c.q0 = &q0;
    c.q1 = &q1;
    c.q2 = &q2;
    c.q3 = &q3;
    c.length = &len;
    c.l0 = &l0;
    c.diameter = &d;
    rc = pcc_upload_cells(ctx, &c, 1);
  }
  long long steps = 0;
  double cs = 0;
  pcc_step_stats st;
  std::memset(&st, 0, sizeof st);
  if (rc == PCC_OK) {
    const long long cap = job.max_steps > 0 ? job.max_steps : (1LL << 62);
    long long bb = 0;
    while (st.colony_radius < job.end_radius && steps < cap) {
      pcc_get_dt(ctx, &r->dt);
      rc = pcc_step(ctx, &st);
      if (rc != PCC_OK) break;
      cs += (double)st.n_cells;
      bb += st.bbpgd_iterations;
      if (st.bbpgd_iterations > r->max_step_bbpgd) r->max_step_bbpgd = st.bbpgd_iterations;
      r->radius = st.colony_radius;
      ++steps;
    }
    r->bbpgd_iterations = bb;
  }
  if (ctx) {
    size_t n = 0;
    pcc_cell_count(ctx, &n);
    std::vector<double> buf(10 * (n + 1));
    pcc_cells o;
    std::memset(&o, 0, sizeof o);
    double* p = buf.data();
    o.x = p;
    o.y = p + (n + 1);
    o.z = p + 2 * (n + 1);
    o.q0 = p + 3 * (n + 1);
    o.q1 = p + 4 * (n + 1);
    o.q2 = p + 5 * (n + 1);
    o.q3 = p + 6 * (n + 1);
    o.length = p + 7 * (n + 1);
    o.l0 = p + 8 * (n + 1);
    o.diameter = p + 9 * (n + 1);
    if (pcc_download_cells(ctx, &o, n, &n) != PCC_OK) n = 0;
    double sum = 0;
    for (size_t i = 0; i < n; ++i)
      sum += o.x[i] + o.y[i] + o.z[i] + o.q0[i] + o.q1[i] + o.q2[i] + o.q3[i] + o.length[i];
    r->checksum = sum;
    r->cells = (long long)n;
  }
  if (ctx) pcc_destroy(ctx);
  r->status = rc;
  r->steps = steps;
  r->cell_steps = cs;
  r->finish_s = since(Clock::now());
}

}  // namespace

extern "C" pcc_status pcc_serve(const pcc_job* jobs, size_t n_jobs, int slots, double hbm_budget_bytes, int device,
                                pcc_job_result* results, double* wall_s) {
  if ((!jobs && n_jobs) || (!results && n_jobs) || slots < 1) return PCC_ERR_INVALID;
  std::vector<size_t> order(n_jobs);
  for (size_t i = 0; i < n_jobs; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return jobs[a].arrival_s < jobs[b].arrival_s; });
  for (size_t i = 0; i < n_jobs; ++i) {
    std::memset(&results[i], 0, sizeof(pcc_job_result));
    results[i].arrival_s = jobs[i].arrival_s;
    results[i].footprint_bytes = projected_footprint(jobs[i].end_radius);
    if (results[i].footprint_bytes > hbm_budget_bytes) return PCC_ERR_CAPACITY;
  }
  std::mutex mu;
  std::condition_variable cv;
  int in_flight = 0;
  double used = 0;
  std::vector<std::thread> threads;
  threads.reserve(n_jobs);
  const auto t0 = Clock::now();
  size_t next = 0;
  std::unique_lock<std::mutex> lock(mu);
  while (next < n_jobs) {
    const size_t j = order[next];
    const double now = std::chrono::duration<double>(Clock::now() - t0).count();
    const double need = results[j].footprint_bytes;
    if (jobs[j].arrival_s > now) {
      cv.wait_for(lock, std::chrono::duration<double>(jobs[j].arrival_s - now));
      continue;
    }
    if (in_flight >= slots || used + need > hbm_budget_bytes) {
      cv.wait(lock);
      continue;
    }
    ++in_flight;
    used += need;
    ++next;
    threads.emplace_back([&, j, need] {
      run_job(jobs[j], device, t0, &results[j]);
      std::lock_guard<std::mutex> g(mu);
      --in_flight;
      used -= need;
      cv.notify_all();
    });
  }
  cv.wait(lock, [&] { return in_flight == 0; });
  lock.unlock();
  for (auto& t : threads) t.join();
  if (wall_s) *wall_s = std::chrono::duration<double>(Clock::now() - t0).count();
  for (size_t i = 0; i < n_jobs; ++i)
    if (results[i].status != PCC_OK) return results[i].status;
  return PCC_OK;
}
