// Device helpers shared by the BBPGD kernels (general 3D form in
// pcc_solver.cu, planar forms in pcc_planar.cu): the projection, PETSc's
// VecScale special cases, the bounded grid barriers, the projected-gradient
// residual term, the Barzilai-Borwein step and the BBPGD trace record.
#pragma once

#include <cfloat>
#include <cmath>

#include "pcc_kernels.hpp"

namespace pcc {

constexpr long long kSpinLimit = 1LL << 26;
constexpr int kTraceWidth = 8;  // it, residual, step size, linear, quadratic, growth, total, -
// Work decomposition shared by the general and planar solvers (identical
// values from both): kLanes lanes per cell in the cell pass (lane l takes
// the cell's incidence entries l, l + kLanes, ...); the constraints are cut
// into chunk_count(m) reduction chunks of nearly equal size, chunk ch
// covering [chunk_lo(ch), chunk_lo(ch + 1)) (starts rounded down to a
// multiple of 32, so a warp's loads start on a line), thread t of a 256-thread unit
// taking the chunk's constraints lo + t, lo + t + 256, ... and summing its
// terms in that order before the unit's fixed shuffle tree.  The count
// depends on the constraint count alone: one constraint per thread while
// that needs at most kChunkTarget chunks, else kChunkTarget chunks (one
// round of a grid of four 256-thread blocks on each of 148 SMs, so every
// block reduces one chunk per iteration), else as many as keep a thread at
// kMaxPerThread constraints.  Nothing depends on the grid.
constexpr int kLanes = 2;
constexpr long long kChunkTarget = 592;  // 4 blocks on each of 148 SMs
constexpr int kMaxPerThread = 8;
__host__ __device__ inline long long chunk_count(long long m, long long target = kChunkTarget) {
  long long c = (m + kBlock - 1) / kBlock;
  if (c > target) c = target;
  const long long most = (long long)kBlock * kMaxPerThread;
  if (c < (m + most - 1) / most) c = (m + most - 1) / most;
  return c < 1 ? 1 : c;
}
__host__ __device__ inline long long chunk_lo(long long ch, long long m, long long nchunks) {
  return ch >= nchunks ? m : (ch * m / nchunks) & ~31LL;
}
constexpr int kCtaThreads = 4 * kBlock;  // one-CTA form: four 256-thread units
constexpr int kCtaUnits = kCtaThreads / kBlock;
constexpr unsigned kFull = 0xffffffffu;

// gamma_k = max(gamma_{k-1} - alpha g_{k-1}, 0): VecWAXPY with PETSc's special
// cases for the coefficient, then VecPointwiseMax against 0.
__device__ __forceinline__ double project(double gp, double g, double alpha) {
  const double a = -alpha;
  double v;
  if (a == 1.0) v = add(gp, g);
  else if (a == -1.0) v = sub(gp, g);
  else if (a == 0.0) v = gp;
  else v = add(mul(a, g), gp);
  return v < 0.0 ? 0.0 : v;
}

// VecScale(x, a) for one entry.
__device__ __forceinline__ double vscale(double a, double x) {
  if (a == 1.0) return x;
  if (a == 0.0) return 0.0;
  return mul(a, x);
}

// Grid barrier of a cooperative launch.  Every block adds one to a
// monotonic arrival counter; the k-th barrier of the launch is passed once the
// counter reaches k * blocks, so the last arrival's own atomic releases it
// (no reset, no second write).  sync_reduce additionally lets the last
// arriving block run `reduce` (all its threads) and then publish the
// barrier's ordinal in `released`, which the other blocks wait for.  Waits
// spin at most kSpinLimit times, then raise kDevErrTimeout and report false.
__device__ __forceinline__ unsigned long long atom_add_release(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.add.release.gpu.global.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned long long atom_add_acq_rel(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// The block's writes before a barrier are ordered before thread 0's release
// by the preceding bar.sync (the release is cumulative); thread 0's acquire,
// followed by bar.sync, orders the other blocks' writes before every thread's
// later reads.
struct GridBarrier {
  SolverScalars* sc;
  DevStatus* st;
  unsigned nblocks;
  unsigned long long k = 0;  // barriers passed so far (the same in every block)

  __device__ bool sync() {
    ++k;
    if (nblocks == 1) {  // one block: a block barrier orders its global writes
      __syncthreads();
      return true;
    }
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
      s_ok = 1;
      const unsigned long long target = k * nblocks;
      if (atom_add_acq_rel(&sc->arrive, 1ULL) + 1 != target) {
        long long spins = 0;
        while (ld_acquire(&sc->arrive) < target) {
          __nanosleep(32);
          if (++spins > kSpinLimit) {
            raise_error(st, kDevErrTimeout, 20);
            s_ok = 0;
            break;
          }
        }
      }
    }
    __syncthreads();
    return s_ok;
  }

  template <typename R>
  __device__ bool sync_reduce(R reduce) {
    ++k;
    if (nblocks == 1) {
      __syncthreads();
      reduce();
      __syncthreads();
      return true;
    }
    __shared__ int s_last, s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
      s_ok = 1;
      s_last = atom_add_acq_rel(&sc->arrive, 1ULL) + 1 == k * nblocks;
    }
    __syncthreads();
    if (s_last) {
      reduce();
      __syncthreads();
      if (threadIdx.x == 0) st_release(&sc->released, k);
    } else if (threadIdx.x == 0) {
      long long spins = 0;
      while (ld_acquire(&sc->released) < k) {
        __nanosleep(32);
        if (++spins > kSpinLimit) {
          raise_error(st, kDevErrTimeout, 21);
          s_ok = 0;
          break;
        }
      }
    }
    __syncthreads();
    return s_ok;
  }
};

__device__ __forceinline__ double proj_grad_abs(double g, double gam) {
  double v = gam > 0 ? g : (g < 0.0 ? g : 0.0);
  return fabs(v);
}

// Fixed-shape block reduction of 4 values (sum, sum, sum, max).
__device__ __forceinline__ void block_reduce4(double v[4], double* sm) {
  const int t = threadIdx.x;
#pragma unroll
  for (int q = 0; q < 4; ++q) sm[q * kBlock + t] = v[q];
  __syncthreads();
  for (int w = kBlock / 2; w > 0; w >>= 1) {
    if (t < w) {
      sm[t] = add(sm[t], sm[t + w]);
      sm[kBlock + t] = add(sm[kBlock + t], sm[kBlock + t + w]);
      sm[2 * kBlock + t] = add(sm[2 * kBlock + t], sm[2 * kBlock + t + w]);
      double x = sm[3 * kBlock + t], y = sm[3 * kBlock + t + w];
      sm[3 * kBlock + t] = x < y ? y : x;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) v[q] = sm[q * kBlock];
  __syncthreads();
}

// Energy of the BBPGD trace (HardModelGradient::energy, HardModelGradient.cpp:160-203)
// from the block partials of the cell terms and the chunk partials of the
// linear term; written by the last block of a barrier.
__device__ __forceinline__ void trace_record(double* sm, const double* tr_part, unsigned nb, long long nchunks,
                                             double dt, double lambda, double tau, long long it, double res,
                                             double alpha, double* out, long long cap) {
  double v[4] = {0, 0, 0, 0};
  for (long long b = threadIdx.x; b < (long long)nb; b += kBlock) {
    v[0] = add(v[0], ldcg(tr_part + 2 * b));
    v[1] = add(v[1], ldcg(tr_part + 2 * b + 1));
  }
  for (long long ch = threadIdx.x; ch < nchunks; ch += kBlock) v[2] = add(v[2], ldcg(tr_part + 2 * nb + ch));
  block_reduce4(v, sm);
  if (threadIdx.x == 0 && it < cap) {
    const double lin = v[2];
    const double quad = mul(v[0], dvd(dt, 2.0));
    const double growth = mul(v[1], dvd(dt, mul(lambda, tau)));
    double* r = out + (long long)kTraceWidth * it;
    r[0] = (double)it;
    r[1] = res;
    r[2] = alpha;
    r[3] = lin;
    r[4] = quad;
    r[5] = growth;
    r[6] = add(add(lin, quad), growth);
    r[7] = 0.0;
  }
}

// Step size of the next iteration from the reduced sums (sum dgam^2,
// sum dgam*dg, sum dg^2): BB1 on even, BB2 on odd iterations
// (solver/BBPGD.cpp:98-112), with the reference's +10 eps guard on a tiny
// denominator.  Both BB quotients are >= 0 in exact arithmetic (the gradient
// is monotone); near convergence rounding can make the numerator a tiny
// negative number, and a negative step lifts an inactive constraint to
// gamma ~ 1e-26 > 0, where the projected residual counts its full positive
// gradient and never returns below tol.  The step is clamped at 0.
__device__ __forceinline__ double bb_step(const double v[4], long long it) {
  double num, den;
  if (it % 2 == 0) {
    num = v[0];
    den = v[1];
  } else {
    den = v[2];
    num = v[1];
  }
  if (fabs(den) < 10 * DBL_EPSILON) den = add(den, 10 * DBL_EPSILON);
  const double step = dvd(num, den);
  return step > 0.0 ? step : 0.0;
}

// Work units.  A unit is 256 threads; chunk ch belongs to unit ch % units.
struct GridUnits {  // the multi-block kernel: one unit per block
  static constexpr bool kGrid = true;
  __device__ static unsigned units() { return gridDim.x; }
  __device__ static unsigned unit() { return blockIdx.x; }
  __device__ static int t() { return threadIdx.x; }
  __device__ static void sync() { __syncthreads(); }
  __device__ static long long warp() { return ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
  __device__ static long long warps() { return ((long long)gridDim.x * blockDim.x) >> 5; }
};
struct CtaUnits {  // the one-CTA kernel: four units in one block, each with its own named barrier
  static constexpr bool kGrid = false;
  __device__ static unsigned units() { return kCtaUnits; }
  __device__ static unsigned unit() { return threadIdx.x / kBlock; }
  __device__ static int t() { return threadIdx.x % kBlock; }
  __device__ static void sync() { asm volatile("bar.sync %0, %1;" ::"r"(unit() + 1), "r"(kBlock) : "memory"); }
  __device__ static long long warp() { return threadIdx.x >> 5; }
  __device__ static long long warps() { return kCtaThreads / 32; }
};

// (sum, sum, sum, max) over a warp by an xor tree (every lane ends with the same bits).
__device__ __forceinline__ void warp_reduce4(double v[4]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v[0] = add(v[0], __shfl_xor_sync(kFull, v[0], o));
    v[1] = add(v[1], __shfl_xor_sync(kFull, v[1], o));
    v[2] = add(v[2], __shfl_xor_sync(kFull, v[2], o));
    const double y = __shfl_xor_sync(kFull, v[3], o);
    v[3] = v[3] < y ? y : v[3];
  }
}

// A unit's 256 values into thread 0 of the unit: the warp tree, then an xor
// tree over the unit's 8 warp results.  sm: 32 doubles of this unit.
template <class U>
__device__ __forceinline__ void unit_reduce4(double v[4], double* sm) {
  warp_reduce4(v);
  const int t = U::t(), lane = t & 31, w = t >> 5;
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) sm[4 * w + q] = v[q];
  }
  U::sync();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = lane < kBlock / 32 ? sm[4 * lane + q] : 0.0;
#pragma unroll
    for (int o = kBlock / 64; o > 0; o >>= 1) {
      v[0] = add(v[0], __shfl_xor_sync(kFull, v[0], o));
      v[1] = add(v[1], __shfl_xor_sync(kFull, v[1], o));
      v[2] = add(v[2], __shfl_xor_sync(kFull, v[2], o));
      const double y = __shfl_xor_sync(kFull, v[3], o);
      v[3] = v[3] < y ? y : v[3];
    }
  }
  U::sync();  // sm is reused by the next call
}

// Sum of the chunk partials by one unit (thread t takes chunks t, t + 256, ...).
template <class U>
__device__ __forceinline__ void reduce_partials(const double4* partials, long long nchunks, double v[4], double* sm) {
  v[0] = v[1] = v[2] = v[3] = 0.0;
  for (long long ch = U::t(); ch < nchunks; ch += kBlock) {
    const double4 q = ldcg(partials + ch);
    v[0] = add(v[0], q.x);
    v[1] = add(v[1], q.y);
    v[2] = add(v[2], q.z);
    v[3] = v[3] < q.w ? q.w : v[3];
  }
  unit_reduce4<U>(v, sm);
}

}  // namespace pcc
