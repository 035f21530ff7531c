// Per-step cell updates (sm_100a): growth, division with device-side append
// of daughters, the x-sort that renumbers cells, colony radius and the CFL
// time-step adaptation.
#include <cmath>
#include <cstring>

#include "pcc_kernels.hpp"

namespace pcc {

namespace {

// ---------------------------------------------------------------- division draw
__host__ __device__ inline unsigned division_seed(unsigned long long seed, unsigned long long k) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (k + 1ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (unsigned)(z & 0xffffffffULL);
}

// First two outputs of MT19937 seeded with s (Matsumoto & Nishimura's
// init_genrand, one in-place twist of words 0 and 1, tempering).
__host__ __device__ inline void mt19937_first_two(unsigned s, unsigned out[2]) {
  unsigned m0 = s, m1 = 0, m2 = 0, m397 = 0, m398 = 0, prev = s;
  for (unsigned i = 1; i < 399; ++i) {
    unsigned v = 1812433253u * (prev ^ (prev >> 30)) + i;
    if (i == 1) m1 = v;
    if (i == 2) m2 = v;
    if (i == 397) m397 = v;
    if (i == 398) m398 = v;
    prev = v;
  }
  const unsigned a[2] = {m0, m1}, b[2] = {m1, m2}, c[2] = {m397, m398};
  for (int k = 0; k < 2; ++k) {
    unsigned y = (a[k] & 0x80000000u) | (b[k] & 0x7fffffffu);
    unsigned v = c[k] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    v ^= v >> 11;
    v ^= (v << 7) & 0x9d2c5680u;
    v ^= (v << 15) & 0xefc60000u;
    v ^= v >> 18;
    out[k] = v;
  }
}

#ifdef __CUDA_ARCH__
#define PCC_ADD(a, b) __dadd_rn(a, b)
#define PCC_MUL(a, b) __dmul_rn(a, b)
#define PCC_DIV(a, b) __ddiv_rn(a, b)
#else
#define PCC_ADD(a, b) ((a) + (b))
#define PCC_MUL(a, b) ((a) * (b))
#define PCC_DIV(a, b) ((a) / (b))
#endif

// Left-daughter length of the k-th division (simulation/Particle.cpp:128-135):
// std::uniform_real_distribution over [0.98, 1.02] * len/2 fed by
// std::mt19937 seeded with division_seed(seed, k); the canonical double is
// (x0 + x1 * 2^32) / 2^64 kept below 1 (two 32-bit draws for 53 bits).
__host__ __device__ inline double division_length(unsigned long long seed, unsigned long long k, double len) {
  unsigned x[2];
  mt19937_first_two(division_seed(seed, k), x);
  double sum = 0.0;
  sum = PCC_ADD(sum, PCC_MUL((double)x[0], 1.0));
  sum = PCC_ADD(sum, PCC_MUL((double)x[1], 4294967296.0));
  double u = PCC_DIV(sum, 18446744073709551616.0);
  if (u >= 1.0) u = 0.99999999999999988898;  // nextafter(1, 0)
  const double half = PCC_DIV(len, 2.0);
  const double a = PCC_MUL(half, 0.98), b = PCC_MUL(half, 1.02);
  return PCC_ADD(PCC_MUL(u, b - a), a);
}

__global__ void k_div_flag(const double* __restrict__ len, const double* __restrict__ l0, long long n,
                           int* __restrict__ flag) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flag[i] = len[i] >= mul(2.0, l0[i]) ? 1 : 0;
}

// Particle::divide (simulation/Particle.cpp:122-150): the parent becomes the
// left daughter in place, the right daughter is appended at n + rank, where
// rank counts dividing cells in id order (ParticleManager::divideParticles,
// ParticleManager.cpp:139-148, and Domain::commitNewParticles, Domain.cpp:55-67).
__global__ void k_divide(CellsView c, long long n, const int* __restrict__ flag, const int* __restrict__ off,
                         unsigned long long seed, unsigned long long base) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  const long long k = off[i];
  const double len = c.len[i];
  const double l1 = division_length(seed, base + (unsigned long long)k, len);
  const double l2 = sub(len, l1);
  double t[3];
  cell_axis(c.q0[i], c.q1[i], c.q2[i], c.q3[i], t);
  const double h1 = dvd(l1, 2.0), h2 = dvd(l2, 2.0);
  const double p[3] = {c.x[i], c.y[i], c.z[i]};
  const long long j = n + k;
  c.x[j] = add(p[0], mul(t[0], h2));
  c.y[j] = add(p[1], mul(t[1], h2));
  c.z[j] = add(p[2], mul(t[2], h2));
  c.x[i] = sub(p[0], mul(t[0], h1));
  c.y[i] = sub(p[1], mul(t[1], h1));
  c.z[i] = sub(p[2], mul(t[2], h1));
  c.q0[j] = c.q0[i];
  c.q1[j] = c.q1[i];
  c.q2[j] = c.q2[i];
  c.q3[j] = c.q3[i];
  c.len[i] = l1;
  c.len[j] = l2;
  c.l0[j] = c.l0[i];
  c.diam[j] = c.diam[i];
  const int age = c.age[i] + 1;
  c.age[i] = age;
  c.age[j] = age;
  c.ncons[j] = 0;
  c.ldot[j] = 0.0;
  c.imp[j] = 0.0;
  c.stress[j] = 0.0;
  for (int d = 0; d < 6; ++d) {
    c.force[6 * j + d] = 0.0;
    c.vel[6 * j + d] = 0.0;
  }
}

__global__ void k_x_keys(const double* __restrict__ x, long long n, unsigned long long* __restrict__ keys,
                         int* __restrict__ vals) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = double_key(x[i]);
  vals[i] = (int)i;
}

__global__ void k_gather_cells(CellsView src, CellsView dst, const int* __restrict__ perm, long long n) {
  long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int i = perm[j];
  dst.x[j] = src.x[i];
  dst.y[j] = src.y[i];
  dst.z[j] = src.z[i];
  dst.q0[j] = src.q0[i];
  dst.q1[j] = src.q1[i];
  dst.q2[j] = src.q2[i];
  dst.q3[j] = src.q3[i];
  dst.len[j] = src.len[i];
  dst.l0[j] = src.l0[i];
  dst.diam[j] = src.diam[i];
  dst.ldot[j] = src.ldot[i];
  dst.imp[j] = src.imp[i];
  dst.stress[j] = src.stress[i];
  dst.age[j] = src.age[i];
  dst.ncons[j] = src.ncons[i];
  for (int d = 0; d < 6; ++d) {
    dst.force[6 * j + d] = src.force[6 * (long long)i + d];
    dst.vel[6 * j + d] = src.vel[6 * (long long)i + d];
  }
}

__global__ void k_grow(double* __restrict__ len, const double* __restrict__ l0, const double* __restrict__ ldot,
                       long long n, double dt) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double l = add(len[i], mul(dt, ldot[i]));
  const double cap = mul(2.0, l0[i]);
  if (l > cap) l = cap;
  len[i] = l;
}

// max over cells of |x + (len/2 - d/2) t| (spatial/Domain.cpp:148-153)
__global__ void k_radius(CellsView c, long long n, DevStatus* st) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double m = 0.0;
  if (i < n) {
    double t[3];
    cell_axis(c.q0[i], c.q1[i], c.q2[i], c.q3[i], t);
    const double half = sub(dvd(c.len[i], 2.0), dvd(c.diam[i], 2.0));
    const double e[3] = {add(c.x[i], mul(t[0], half)), add(c.y[i], mul(t[1], half)), add(c.z[i], mul(t[2], half))};
    m = __dsqrt_rn(dot3(e, e));
  }
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_down_sync(0xffffffffu, m, o);
    m = m < w ? w : m;
  }
  if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(&st->max_bits, (unsigned long long)__double_as_longlong(m));
}

// |v| + ldot per cell as an ordered key (Domain::adaptDt, spatial/Domain.cpp:73-77)
__global__ void k_speed_keys(CellsView c, long long n, unsigned long long* __restrict__ keys, int* __restrict__ vals) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* v = c.vel + 6 * i;
  const double vv[3] = {v[0], v[1], v[2]};
  const double s = add(__dsqrt_rn(dot3(vv, vv)), c.ldot[i]);
  keys[i] = double_key(s);
  vals[i] = (int)i;
}

double key_to_double(unsigned long long k) {
  unsigned long long b = (k & 0x8000000000000000ULL) ? (k & 0x7fffffffffffffffULL) : ~k;
  double d;
  std::memcpy(&d, &b, sizeof d);
  return d;
}

}  // namespace

cudaError_t reset_ldot(pcc_ctx* ctx) {
  if (!ctx->n) return cudaSuccess;
  return cudaMemsetAsync(ctx->cells.ldot.p, 0, ctx->n * sizeof(double), ctx->stream);
}

cudaError_t grow_cells(pcc_ctx* ctx, double dt) {
  if (!ctx->n) return cudaSuccess;
  k_grow<<<grid_for(ctx->n), kBlock, 0, ctx->stream>>>(ctx->cells.len.p, ctx->cells.l0.p, ctx->cells.ldot.p,
                                                       (long long)ctx->n, dt);
  ctx->launches++;
  return cudaGetLastError();
}

cudaError_t division_count_enqueue(pcc_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->n;
  cudaError_t e;
  if ((e = ctx->div_flag.reserve(n + 1, 0, s)) || (e = ctx->div_off.reserve(n + 1, 0, s))) return e;
  if (n) {
    k_div_flag<<<grid_for(n), kBlock, 0, s>>>(ctx->cells.len.p, ctx->cells.l0.p, (long long)n, ctx->div_flag.p);
    ctx->launches++;
  }
  if ((e = exclusive_scan(ctx, ctx->div_flag.p, ctx->div_off.p, n))) return e;
  return cudaMemcpyAsync(ctx->pinned_ll + kSlotDivs, ctx->div_off.p + n, sizeof(int), cudaMemcpyDeviceToHost, s);
}

cudaError_t divide_cells(pcc_ctx* ctx, size_t* added) {
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->n;
  cudaError_t e;
  *added = 0;
  if (!n) return cudaSuccess;
  size_t k;
  if (ctx->div_known) {  // counted at the end of the previous step, on these very cells
    k = ctx->div_next;
  } else {
    if ((e = division_count_enqueue(ctx))) return e;
    if ((e = cudaStreamSynchronize(s))) return e;
    k = (size_t) * reinterpret_cast<int*>(ctx->pinned_ll + kSlotDivs);
  }
  ctx->div_known = false;
  if (!k) return cudaSuccess;
  if ((e = ctx->cells.reserve(n + k, n, s))) return e;
  k_divide<<<grid_for(n), kBlock, 0, s>>>(ctx->cells.view(), (long long)n, ctx->div_flag.p, ctx->div_off.p,
                                          ctx->params.seed, ctx->div_index);
  ctx->launches++;
  ctx->div_index += k;
  ctx->n = n + k;
  *added = k;
  return cudaGetLastError();
}

cudaError_t sort_cells_by_x(pcc_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->n;
  cudaError_t e;
  if (n <= 1) return cudaSuccess;
  if ((e = ctx->keys.reserve(n, 0, s)) || (e = ctx->perm.reserve(n, 0, s))) return e;
  if ((e = ctx->cells_alt.reserve(n, 0, s))) return e;
  k_x_keys<<<grid_for(n), kBlock, 0, s>>>(ctx->cells.x.p, (long long)n, ctx->keys.p, ctx->perm.p);
  ctx->launches++;
  if ((e = radix_sort_pairs(ctx, ctx->keys.p, ctx->perm.p, n, 64))) return e;
  k_gather_cells<<<grid_for(n), kBlock, 0, s>>>(ctx->cells.view(), ctx->cells_alt.view(), ctx->perm.p, (long long)n);
  ctx->launches++;
  ctx->cells.swap(ctx->cells_alt);
  return cudaGetLastError();
}

cudaError_t radius_enqueue(pcc_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  cudaMemsetAsync(&ctx->status->max_bits, 0, sizeof(unsigned long long), s);
  if (ctx->n) {
    k_radius<<<grid_for(ctx->n), kBlock, 0, s>>>(ctx->cells.view(), (long long)ctx->n, ctx->status);
    ctx->launches++;
  }
  return cudaMemcpyAsync(ctx->pinned_ll + kSlotRadius, &ctx->status->max_bits, sizeof(unsigned long long),
                         cudaMemcpyDeviceToHost, s);
}

double radius_collect(pcc_ctx* ctx) {
  double r;
  std::memcpy(&r, ctx->pinned_ll + kSlotRadius, sizeof r);
  return r;
}

cudaError_t colony_radius(pcc_ctx* ctx, double* out) {
  cudaError_t e = radius_enqueue(ctx);
  if (!e) e = cudaStreamSynchronize(ctx->stream);
  if (e) return e;
  *out = radius_collect(ctx);
  return cudaSuccess;
}

// Domain::adaptDt (spatial/Domain.cpp:69-118): median of |v| + ldot (for an
// even count, the mean of the two middle values), dt* = cfl*tol/median,
// dt <- clamp(0.99 dt + 0.01 dt*, 0.9 dt, 1.1 dt).  The enqueue half sorts the
// speeds on the device and queues the copy of the middle keys; the collect
// half, after the caller's synchronisation, does the host arithmetic.
cudaError_t adapt_dt_enqueue(pcc_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->n;
  cudaError_t e;
  if (!n) return cudaSuccess;
  if ((e = ctx->keys.reserve(n, 0, s)) || (e = ctx->perm.reserve(n, 0, s))) return e;
  k_speed_keys<<<grid_for(n), kBlock, 0, s>>>(ctx->cells.view(), (long long)n, ctx->keys.p, ctx->perm.p);
  ctx->launches++;
  if ((e = radix_sort_pairs(ctx, ctx->keys.p, ctx->perm.p, n, 64))) return e;
  const size_t lo = n % 2 == 0 ? n / 2 - 1 : n / 2;
  return cudaMemcpyAsync(ctx->pinned_ll + kSlotMedian, ctx->keys.p + lo,
                         2 * sizeof(unsigned long long) - (n == 1 ? sizeof(unsigned long long) : 0),
                         cudaMemcpyDeviceToHost, s);
}

void adapt_dt_collect(pcc_ctx* ctx) {
  const size_t n = ctx->n;
  if (!n) return;
  const unsigned long long* pk = reinterpret_cast<const unsigned long long*>(ctx->pinned_ll + kSlotMedian);
  double med;
  if (n % 2 == 0) {
    const double lower = key_to_double(pk[0]), upper = key_to_double(pk[1]);
    med = 0.5 * (lower + upper);
  } else {
    med = key_to_double(pk[0]);
  }
  const double gmed = med / 1;
  if (gmed == 0.0) return;
  const double cfl = ctx->params.cfl_factor * ctx->params.tolerance;
  const double cap_dt = cfl / gmed;
  const double dt = ctx->params.dt;
  volatile double t1 = dt * (1.0 - 0.01);
  volatile double t2 = 0.01 * cap_dt;
  double nd = t1 + t2;
  const double lo_dt = 0.9 * dt, hi_dt = 1.1 * dt;
  nd = nd < lo_dt ? lo_dt : (hi_dt < nd ? hi_dt : nd);
  ctx->params.dt = nd;
}

cudaError_t adapt_dt(pcc_ctx* ctx) {
  cudaError_t e = adapt_dt_enqueue(ctx);
  if (!e) e = cudaStreamSynchronize(ctx->stream);
  if (e) return e;
  adapt_dt_collect(ctx);
  return cudaSuccess;
}

}  // namespace pcc

extern "C" unsigned int pcc_division_seed(unsigned long long seed, unsigned long long k) {
  return pcc::division_seed(seed, k);
}

extern "C" double pcc_division_length_host(unsigned long long seed, unsigned long long k, double len) {
  return pcc::division_length(seed, k, len);
}
