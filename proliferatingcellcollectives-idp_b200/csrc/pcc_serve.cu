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
#include <deque>
#include <mutex>
#include <new>
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

// ----------------------------------------------------------------- request loop
// The same admission and execution as pcc_serve, as a long-lived server that
// takes jobs while it runs: pcc_server_submit queues a job (its arrival time
// is the submit time), a scheduler thread admits queued jobs in submit order
// as slots and HBM budget free up, each admitted job runs on its own context,
// stream and thread, and pcc_server_poll hands back finished results.
struct pcc_server {
  int slots = 1;
  double budget = 0;
  int device = 0;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::pair<unsigned long long, pcc_job>> queue;
  std::deque<std::pair<unsigned long long, pcc_job_result>> done;
  std::vector<std::thread> workers;
  std::thread scheduler;
  int in_flight = 0;
  double used = 0;
  bool stop = false;
  unsigned long long next_id = 1;
};

namespace {

void server_loop(pcc_server* sv) {
  std::unique_lock<std::mutex> lock(sv->mu);
  for (;;) {
    sv->cv.wait(lock, [&] {
      if (sv->stop && sv->queue.empty()) return true;
      if (sv->queue.empty()) return false;
      const double need = projected_footprint(sv->queue.front().second.end_radius);
      return sv->in_flight < sv->slots && sv->used + need <= sv->budget;
    });
    if (sv->queue.empty()) return;  // stopping with nothing queued
    auto item = sv->queue.front();
    sv->queue.pop_front();
    const double need = projected_footprint(item.second.end_radius);
    ++sv->in_flight;
    sv->used += need;
    sv->workers.emplace_back([sv, item, need] {
      pcc_job_result r;
      std::memset(&r, 0, sizeof r);
      r.arrival_s = item.second.arrival_s;
      r.footprint_bytes = need;
      run_job(item.second, sv->device, sv->t0, &r);
      std::lock_guard<std::mutex> g(sv->mu);
      sv->done.emplace_back(item.first, r);
      --sv->in_flight;
      sv->used -= need;
      sv->cv.notify_all();
    });
  }
}

}  // namespace

extern "C" {

pcc_status pcc_server_create(int slots, double hbm_budget_bytes, int device, pcc_server** out) {
  if (!out || slots < 1 || !(hbm_budget_bytes > 0)) return PCC_ERR_INVALID;
  auto* sv = new (std::nothrow) pcc_server();
  if (!sv) return PCC_ERR_NOMEM;
  sv->slots = slots;
  sv->budget = hbm_budget_bytes;
  sv->device = device;
  sv->t0 = Clock::now();
  sv->scheduler = std::thread(server_loop, sv);
  *out = sv;
  return PCC_OK;
}

pcc_status pcc_server_submit(pcc_server* sv, const pcc_job* job, unsigned long long* id) {
  if (!sv || !job) return PCC_ERR_INVALID;
  if (projected_footprint(job->end_radius) > sv->budget) return PCC_ERR_CAPACITY;
  std::lock_guard<std::mutex> g(sv->mu);
  if (sv->stop) return PCC_ERR_INVALID;
  pcc_job j = *job;
  j.arrival_s = std::chrono::duration<double>(Clock::now() - sv->t0).count();
  const unsigned long long k = sv->next_id++;
  sv->queue.emplace_back(k, j);
  if (id) *id = k;
  sv->cv.notify_all();
  return PCC_OK;
}

pcc_status pcc_server_poll(pcc_server* sv, pcc_job_result* out, unsigned long long* ids, size_t cap, size_t* n,
                           double wait_s) {
  if (!sv || !n || (cap && (!out || !ids))) return PCC_ERR_INVALID;
  std::unique_lock<std::mutex> lock(sv->mu);
  if (sv->done.empty() && wait_s > 0)
    sv->cv.wait_for(lock, std::chrono::duration<double>(wait_s), [&] { return !sv->done.empty(); });
  size_t k = 0;
  while (k < cap && !sv->done.empty()) {
    ids[k] = sv->done.front().first;
    out[k] = sv->done.front().second;
    sv->done.pop_front();
    ++k;
  }
  *n = k;
  return PCC_OK;
}

pcc_status pcc_server_pending(pcc_server* sv, size_t* queued, size_t* running) {
  if (!sv) return PCC_ERR_INVALID;
  std::lock_guard<std::mutex> g(sv->mu);
  if (queued) *queued = sv->queue.size();
  if (running) *running = (size_t)sv->in_flight;
  return PCC_OK;
}

pcc_status pcc_server_destroy(pcc_server* sv) {
  if (!sv) return PCC_OK;
  {
    std::lock_guard<std::mutex> g(sv->mu);
    sv->stop = true;
  }
  sv->cv.notify_all();
  if (sv->scheduler.joinable()) sv->scheduler.join();  // admits what was queued, then exits
  for (auto& t : sv->workers) t.join();
  delete sv;
  return PCC_OK;
}

}  // extern "C"

// ----------------------------------------------------------------- lockstep batch
// Many colonies stepped together: each colony is a context with its own
// stream; pcc_batch_step advances every colony by one step, the colonies
// spread over a pool of host threads so their kernels overlap on the device,
// and returns when all are done.  A colony's trajectory is the one it has
// alone (contexts share nothing).
struct pcc_batch {
  std::vector<pcc_ctx*> ctx;
  std::vector<std::thread> pool;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  size_t next = 0, finished = 0, total = 0;
  unsigned long long epoch = 0;
  bool stop = false;
  pcc_step_stats* out = nullptr;
  std::vector<pcc_status> rc;
};

namespace {

void batch_worker(pcc_batch* b) {
  unsigned long long seen = 0;
  std::unique_lock<std::mutex> lock(b->mu);
  for (;;) {
    b->cv_work.wait(lock, [&] { return b->stop || (b->epoch != seen && b->next < b->total); });
    if (b->stop) return;
    const size_t k = b->next++;
    if (b->next >= b->total) seen = b->epoch;
    lock.unlock();
    pcc_step_stats st;
    std::memset(&st, 0, sizeof st);
    const pcc_status r = pcc_step(b->ctx[k], &st);
    lock.lock();
    b->rc[k] = r;
    if (b->out) b->out[k] = st;
    if (++b->finished == b->total) b->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

pcc_status pcc_batch_create(const pcc_params* per_colony, int n, int device, pcc_batch** out) {
  if (!per_colony || n < 1 || !out) return PCC_ERR_INVALID;
  *out = nullptr;
  auto* b = new (std::nothrow) pcc_batch();
  if (!b) return PCC_ERR_NOMEM;
  for (int k = 0; k < n; ++k) {
    pcc_ctx* c = nullptr;
    const pcc_status r = pcc_create(&per_colony[k], device, &c);
    if (r != PCC_OK) {
      for (auto* x : b->ctx) pcc_destroy(x);
      delete b;
      return r;
    }
    b->ctx.push_back(c);
  }
  b->rc.assign((size_t)n, PCC_OK);
  const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
  const int workers = std::min<int>(n, (int)std::min(64u, 2 * hw));
  for (int w = 0; w < workers; ++w) b->pool.emplace_back(batch_worker, b);
  *out = b;
  return PCC_OK;
}

pcc_status pcc_batch_context(pcc_batch* b, int k, pcc_ctx** ctx) {
  if (!b || !ctx || k < 0 || (size_t)k >= b->ctx.size()) return PCC_ERR_INVALID;
  *ctx = b->ctx[(size_t)k];
  return PCC_OK;
}

pcc_status pcc_batch_step(pcc_batch* b, pcc_step_stats* out) {
  if (!b) return PCC_ERR_INVALID;
  std::unique_lock<std::mutex> lock(b->mu);
  b->out = out;
  b->total = b->ctx.size();
  b->next = 0;
  b->finished = 0;
  ++b->epoch;
  b->cv_work.notify_all();
  b->cv_done.wait(lock, [&] { return b->finished == b->total; });
  b->out = nullptr;
  for (const pcc_status r : b->rc)
    if (r != PCC_OK) return r;
  return PCC_OK;
}

pcc_status pcc_batch_destroy(pcc_batch* b) {
  if (!b) return PCC_OK;
  {
    std::lock_guard<std::mutex> g(b->mu);
    b->stop = true;
  }
  b->cv_work.notify_all();
  for (auto& t : b->pool) t.join();
  for (auto* c : b->ctx) pcc_destroy(c);
  delete b;
  return PCC_OK;
}

}  // extern "C"
