// Planar BBPGD solver (sm_100a): the hard model's Barzilai-Borwein projected
// gradient (solver/BBPGD.cpp:32-127, gradient of
// dynamics/models/hard/HardModelGradient.cpp:89-158) for a colony whose cells
// all lie in z = 0 and rotate about z only.  Then a D row has three non-zero
// entries per side (n_x, n_y and the z torque arm) and U three per cell
// (u_x, u_y, w_z); every other term of the general kernel is an exact zero,
// and a running sum that starts at +0 is unchanged by adding a signed zero,
// so skipping them gives the general kernel's values.
//
// One persistent launch runs the whole solve.  Each iteration is two passes
// separated by grid barriers:
//   cell pass: kLanes lanes per cell walk the cell's incidence entries
//     (ascending constraint order, lane l takes entries l, l + kLanes, ...),
//     each entry a coalesced read of its D row and the constraint's
//     gamma_old, and a read of the (gamma, g) pair of the previous iteration
//     from the constraint itself (entry 2c + side); gamma_k =
//     max(gamma_{k-1} - alpha g_{k-1}, 0) is formed on the fly, the lanes'
//     sums of F = D^T (gamma_k - gamma_old) and sigma = L^T gamma_k are combined
//     by a fixed shuffle tree, and the first lane forms U = M F, the growth
//     rate and its change;
//   constraint pass: a few constraints per thread in fixed chunks
//     (chunk_count, chunk_lo), phi_next = Phi + dt D U - dt L dldot, the new
//     (gamma_k, g_k) written over the constraint's previous pair, and the
//     three Barzilai-Borwein dot products and the residual reduced per chunk
//     by a fixed shuffle tree.
// The (gamma, g) pairs are updated in place: the cell pass reads them before
// the first barrier and the constraint pass rewrites them after it, and each
// constraint's pair is read and rewritten by the same thread.  Gathering the
// pairs costs a 32-byte sector per scattered read; pushing copies to the two
// incidence entries instead (sequential reads in the cell pass) cost the same
// sector per scattered 16-byte write and measured 1.5-1.65x slower per
// iteration once the constraint set is several times the L2.  On residual
// iterations (the only ones that can end the solve) the
// constraint pass also stores gamma_{k-1}, the iterate the reference returns,
// and phi_next, so nothing has to be kept from the previous iteration.
// After the second barrier every block reduces the chunk partials in the same
// fixed order (in the traced form the last block to arrive does, and
// publishes the step size and the convergence decision).  The
// work of a chunk and of a cell never depends on which block does it, so the
// result does not depend on the grid size: the one-CTA form for small
// colonies (four 256-thread units in one block, named barriers instead of
// grid barriers) gives the multi-block kernel's values bit for bit.
//
// Real = double is the plain FP64 method.  Real = float is the
// mixed-precision form: D, L, M, U and the D / M products in FP32, while
// gamma, the gradient, Phi / phi_next, sigma = L^T gamma, the BB dot products
// and the residual stay FP64.
#include <cfloat>
#include <cmath>

#include "pcc_bbpgd.cuh"
#include "pcc_kernels.hpp"

namespace pcc {

namespace {

constexpr int kCtaCells = 1024;            // the one-CTA form up to this many cells ...
constexpr int kCtaConstraints = 4096;      // ... and constraints
// Co-resident blocks per SM of the multi-block form and the chunk target that
// goes with it (one chunk per block per iteration), per operand precision.
template <class Real>
struct Occupancy {
  static constexpr int kBlocksPerSm = 4;
  static constexpr long long kChunks = kChunkTarget;
};
// the general (FP64) kernel cuts its chunks with the default target
static_assert(Occupancy<double>::kChunks == kChunkTarget, "FP64 chunks must match the general kernel's");

template <class Real>
struct PT;
template <>
struct PT<double> {
  using V2 = double2;
  using V4 = double4;
};
template <>
struct PT<float> {
  using V2 = float2;
  using V4 = float4;
};

template <class V4>
__device__ __forceinline__ V4 mk4(double a, double b, double c, double d);
template <>
__device__ __forceinline__ double4 mk4<double4>(double a, double b, double c, double d) {
  return make_double4(a, b, c, d);
}
template <>
__device__ __forceinline__ float4 mk4<float4>(double a, double b, double c, double d) {
  return make_float4((float)a, (float)b, (float)c, (float)d);
}
template <class V2>
__device__ __forceinline__ V2 mk2(double a, double b);
template <>
__device__ __forceinline__ double2 mk2<double2>(double a, double b) {
  return make_double2(a, b);
}
template <>
__device__ __forceinline__ float2 mk2<float2>(double a, double b) {
  return make_float2((float)a, (float)b);
}

template <class Real>
struct PArgs {
  using V2 = typename PT<Real>::V2;
  using V4 = typename PT<Real>::V4;
  long long m, n;
  // per constraint
  const int2* ij;
  const V2 *nn, *tt, *ss;  // (n_x, n_y), (t_iz, t_jz), (s_i, s_j)
  double* phi;             // Phi on entry, phi_next of the returned iterate on exit
  double* gamma;           // gamma_0 on entry, gamma_{k-1} on exit
  double* phin;            // phi_next of the last residual iteration
  double2* gg;             // (gamma, g) of the last iteration
  // per incidence entry
  const int* inc_off;
  const V4* inc;           // (D_x, D_y, D_t, s) of that side
  const double* gold;      // gamma_old of the entry's constraint
  const int* ent;          // the entry's constraint and side (2c + side)
  // per cell
  const V4* cell;          // (M_lin, M_rot, len, ldot_prev)
  V4* u;                   // (u_x, u_y, w_z, dldot)
  const double* uext;      // rotational U_ext, 3 per cell (z used: monolayer kicks); null: zero
  double *U, *F, *sig, *ldot, *imp;  // general-layout outputs, written on residual iterations
  double dt, lambda, tau, tol;
  long long max_it;
  double4* partials;       // one per chunk: (sum dgam^2, sum dgam*dg, sum dg^2, max residual)
  long long nchunks;       // chunk_count(m)
  SolverScalars* sc;
  DevStatus* st_err;
  // BBPGD trace (-log_bbgd_trace), as in the general kernel
  int trace;
  double* tr_part;
  double* trace_out;
  long long trace_cap;
};

__device__ __forceinline__ double lane_add(double a, double b) { return add(a, b); }
__device__ __forceinline__ float lane_add(float a, float b) { return __fadd_rn(a, b); }

// Lane sums of one cell over its incidence entries.
template <class Real>
struct CellAcc {
  Real f0 = 0, f1 = 0, f5 = 0;
  double sg = 0.0, g0 = 0.0, g1 = 0.0, g5 = 0.0;
};

// Cell pass.  mode 0: gamma = gamma_0 (the initial gradient); mode 1: gamma_k
// projected from the entries' (gamma, g) with step alpha.  A lane group
// takes one cell per round and loads the next cell's incidence range and
// record while it walks the current cell's entries, so the two loads are in
// flight together; each cell's sums do not depend on which group takes it.
template <class Real, class U, int kTr>
__device__ __forceinline__ void cell_pass(const PArgs<Real>& a, int mode, double alpha, bool final, double* eq,
                                          double* eg, int set = 0) {
  using V4 = typename PT<Real>::V4;
  constexpr bool kF64 = sizeof(Real) == 8;
  const int lane = threadIdx.x & 31, gl = lane % kLanes;
  constexpr long long kCellsPerWarp = 32 / kLanes;
  auto accumulate = [&](CellAcc<Real>& A, int k) {
    const V4 d = a.inc[k];
    const double go = a.gold[k];
    double gc = go;
    if (mode != 0) {
      const double2 s = ldcg(a.gg + (a.ent[k] >> 1));
      gc = project(s.x, s.y, alpha);
    }
    const double diff = sub(gc, go);
    if constexpr (kF64) {
      A.f0 = add(A.f0, mul(d.x, diff));
      A.f1 = add(A.f1, mul(d.y, diff));
      A.f5 = add(A.f5, mul(d.z, diff));
      A.sg = add(A.sg, mul(d.w, gc));
    } else {
      const float df = (float)diff;
      A.f0 = fmaf(d.x, df, A.f0);
      A.f1 = fmaf(d.y, df, A.f1);
      A.f5 = fmaf(d.z, df, A.f5);
      A.sg = fma((double)d.w, gc, A.sg);
    }
    if constexpr (kTr) {
      A.g0 = add(A.g0, mul((double)d.x, gc));
      A.g1 = add(A.g1, mul((double)d.y, gc));
      A.g5 = add(A.g5, mul((double)d.z, gc));
    }
  };
  auto combine = [&](CellAcc<Real>& A) {  // fixed shuffle tree over the group's lanes
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) {
      A.f0 = lane_add(A.f0, __shfl_xor_sync(kFull, A.f0, o));
      A.f1 = lane_add(A.f1, __shfl_xor_sync(kFull, A.f1, o));
      A.f5 = lane_add(A.f5, __shfl_xor_sync(kFull, A.f5, o));
      A.sg = add(A.sg, __shfl_xor_sync(kFull, A.sg, o));
      if constexpr (kTr) {
        A.g0 = add(A.g0, __shfl_xor_sync(kFull, A.g0, o));
        A.g1 = add(A.g1, __shfl_xor_sync(kFull, A.g1, o));
        A.g5 = add(A.g5, __shfl_xor_sync(kFull, A.g5, o));
      }
    }
  };
  auto finish = [&](long long p, const CellAcc<Real>& A, const V4& cl, double uez) {
    double ux, uy, wz;
    if constexpr (kF64) {
      ux = add(add(0.0, mul(cl.x, A.f0)), 0.0);
      uy = add(add(0.0, mul(cl.x, A.f1)), 0.0);
      wz = add(add(0.0, mul(cl.y, A.f5)), uez);  // U = U_ext + M F (HardModelGradient.cpp:21)
    } else {
      ux = cl.x * A.f0;
      uy = cl.x * A.f1;
      wz = (double)(cl.y * A.f5) + uez;
    }
    const double im = exp(vscale(-a.lambda, A.sg));
    const double ld = vscale(dvd(1.0, a.tau), mul((double)cl.z, im));
    a.u[p] = mk4<V4>(ux, uy, wz, sub(ld, (double)cl.w));
    if constexpr (kTr) {
      const double ml = cl.x, mr = cl.y;
      *eq = add(*eq, add(add(mul(A.g0, mul(ml, A.g0)), mul(A.g1, mul(ml, A.g1))), mul(A.g5, mul(mr, A.g5))));
      *eg = add(*eg, mul((double)cl.z, im));
    }
    if (final) {
      double* Up = a.U + 6 * p;
      double* Fp = a.F + 6 * p;
      Up[0] = ux;
      Up[1] = uy;
      Up[2] = 0.0;
      Up[3] = 0.0;
      Up[4] = 0.0;
      Up[5] = wz;
      Fp[0] = A.f0;
      Fp[1] = A.f1;
      Fp[2] = 0.0;
      Fp[3] = 0.0;
      Fp[4] = 0.0;
      Fp[5] = A.f5;
      a.sig[p] = A.sg;
      a.ldot[p] = ld;
      a.imp[p] = im;
    }
  };
  // Cell units: unit u is the cells [16 u, 16 u + 16), one per lane group of
  // a warp.  Warp w (of W) starts with unit w; the untraced multi-block pass
  // then draws its further units from kTakeGroups counters of counter set
  // `set` (warp w from counter w % kTakeGroups, whose units are W + (w % kTakeGroups) +
  // kTakeGroups j), so blocks that run fast take more cells and the pass ends
  // with the memory system still busy; the other forms keep the static order
  // w, w + W, w + 2W, ...  A unit is drawn one round ahead (the first draw
  // alongside the first unit's loads) and its cells' ranges are loaded one
  // round ahead of their use.  Which warp does a cell changes nothing in its
  // sums.
  constexpr bool kDyn = !kTr && U::kGrid;
  const long long W = U::warps(), units = (a.n + kCellsPerWarp - 1) / kCellsPerWarp;
  const int grp = (int)(U::warp() % kTakeGroups);
  unsigned long long* take = kDyn ? &a.sc->take[set][grp][0] : nullptr;
  long long ucur = U::warp(), unext = ucur + W;
  long long p = ucur * kCellsPerWarp + lane / kLanes;
  int b = 0, e = 0;
  V4 cl{};
  double uez = 0.0;
  if constexpr (kDyn) {
    unext = units;
    if (ucur < units && lane == 0) unext = W + grp + kTakeGroups * (long long)atomicAdd(take, 1ULL);
  }
  if (p < a.n) {
    b = a.inc_off[p];
    e = a.inc_off[p + 1];
    cl = a.cell[p];
    if (a.uext) uez = a.uext[3 * p + 2];
  }
  if constexpr (kDyn) unext = __shfl_sync(kFull, unext, 0);
  while (ucur < units) {
    long long uafter = unext + W;
    if constexpr (kDyn) {
      uafter = units;
      if (unext < units && lane == 0) uafter = W + grp + kTakeGroups * (long long)atomicAdd(take, 1ULL);
    }
    const long long pn = unext * kCellsPerWarp + lane / kLanes;
    int bn = 0, en = 0;
    V4 cln{};
    double uezn = 0.0;
    if (pn < a.n) {
      bn = a.inc_off[pn];
      en = a.inc_off[pn + 1];
      cln = a.cell[pn];
      if (a.uext) uezn = a.uext[3 * pn + 2];
    }
    CellAcc<Real> A;
    for (int k = b + gl; k < e; k += kLanes) accumulate(A, k);
    combine(A);
    if (gl == 0 && p < a.n) finish(p, A, cl, uez);
    if constexpr (kDyn) uafter = __shfl_sync(kFull, uafter, 0);
    ucur = unext;
    unext = uafter;
    p = pn;
    b = bn;
    e = en;
    cl = cln;
    uez = uezn;
  }
}

// phi_next of constraint c given U and dldot (MatMult row c in ascending
// columns: gi < gj, so the i block first; VecMAXPY(phi_next, {dt, -dt}, ...)).
// Zeroes counter set `set` of the cell-unit counters.  Iteration k's cell
// pass draws from set k % 2; set (k + 1) % 2 was last drawn from by iteration
// k - 1, so one thread zeroes it between the two barriers of iteration k and
// the second barrier orders that before iteration k + 1 draws from it.
__device__ __forceinline__ void reset_take(SolverScalars* sc, int set) {
#pragma unroll
  for (int g = 0; g < kTakeGroups; ++g) sc->take[set][g][0] = 0;
}

template <class Real>
__device__ __forceinline__ double planar_grad(const PArgs<Real>& a, long long c) {
  const int2 ij = a.ij[c];
  const auto n = a.nn[c];
  const auto t = a.tt[c];
  const auto s = a.ss[c];
  const auto ui = ldcg(a.u + ij.x);
  const auto uj = ldcg(a.u + ij.y);
  if constexpr (sizeof(Real) == 8) {
    double pd = 0.0;
    pd = add(pd, mul(n.x, ui.x));
    pd = add(pd, mul(n.y, ui.y));
    pd = add(pd, mul(t.x, ui.z));
    pd = add(pd, mul(-n.x, uj.x));
    pd = add(pd, mul(-n.y, uj.y));
    pd = add(pd, mul(t.y, uj.z));
    double gr = 0.0;
    gr = add(gr, mul(s.x, ui.w));
    gr = add(gr, mul(s.y, uj.w));
    return add(a.phi[c], add(mul(a.dt, pd), mul(-a.dt, gr)));
  } else {
    float pd = n.x * ui.x;
    pd = fmaf(n.y, ui.y, pd);
    pd = fmaf(t.x, ui.z, pd);
    pd = fmaf(-n.x, uj.x, pd);
    pd = fmaf(-n.y, uj.y, pd);
    pd = fmaf(t.y, uj.z, pd);
    const float gr = fmaf(s.y, uj.w, s.x * ui.w);
    return a.phi[c] + a.dt * ((double)pd - (double)gr);
  }
}

// Constraint pass: new (gamma, g) over the constraint's pair and its two
// incidence entries, chunk partials.  mode 0 evaluates g at gamma_0 (residual
// only).
template <class Real, class U, int kTr>
__device__ __forceinline__ void constraint_pass(const PArgs<Real>& a, int mode, double alpha, bool check, double* sm,
                                                double* smt) {
  double2* gg = a.gg;
  for (long long ch = U::unit(); ch < a.nchunks; ch += U::units()) {
    double v[4] = {0, 0, 0, 0};
    double lin = 0.0;
    const long long hi = chunk_lo(ch + 1, a.m, a.nchunks);
#pragma unroll 2
    for (long long c = chunk_lo(ch, a.m, a.nchunks) + U::t(); c < hi; c += kBlock) {
      const double2 s = gg[c];
      const double gam = mode == 0 ? s.x : project(s.x, s.y, alpha);
      const double g = planar_grad(a, c);
      const double2 r = make_double2(gam, g);
      gg[c] = r;
      if (mode != 0 && check) {  // what the solve returns if it ends here (Hard.cpp:170, BBPGD.cpp:124)
        a.gamma[c] = s.x;
        a.phin[c] = g;
      }
      if (mode != 0) {
        const double dgm = sub(gam, s.x), dg = sub(g, s.y);
        v[0] = add(v[0], mul(dgm, dgm));
        v[1] = add(v[1], mul(dgm, dg));
        v[2] = add(v[2], mul(dg, dg));
      }
      if (mode == 0 || check) {
        const double rr = proj_grad_abs(g, gam);
        v[3] = v[3] < rr ? rr : v[3];
      }
      if constexpr (kTr) lin = add(lin, mul(gam, a.phi[c]));
    }
    unit_reduce4<U>(v, sm);
    if (U::t() == 0) a.partials[ch] = make_double4(v[0], v[1], v[2], v[3]);
    if constexpr (kTr) {
      if (a.trace) {
        double w[4] = {lin, 0, 0, 0};
        block_reduce4(w, smt);
        if (threadIdx.x == 0) a.tr_part[2 * gridDim.x + ch] = w[0];
      }
    }
  }
}

__device__ __forceinline__ void trace_cells(double* smt, double eq, double eg, double* tr_part) {
  double v[4] = {eq, eg, 0, 0};
  block_reduce4(v, smt);
  if (threadIdx.x == 0) {
    tr_part[2 * blockIdx.x] = v[0];
    tr_part[2 * blockIdx.x + 1] = v[1];
  }
}

// Occupancy<Real>::kBlocksPerSm blocks per SM fit the register file, which
// the chunk sizing (Occupancy<Real>::kChunks) assumes.
template <class Real, int kTr>
__global__ void __launch_bounds__(kBlock, kTr ? 1 : Occupancy<Real>::kBlocksPerSm) k_bbpgd_planar(PArgs<Real> a) {
  __shared__ double sm[4 * (kBlock / 32)];
  __shared__ double smt[kTr ? 4 * kBlock : 1];
  const int TR = kTr ? a.trace : 0;
  const unsigned nb = gridDim.x;
  SolverScalars* sc = a.sc;
  GridBarrier bar{sc, a.st_err, nb};
  if constexpr (!kTr) {
    // Untraced: every block reduces the chunk partials itself after a plain
    // grid barrier, in the same fixed order, so every block holds the same
    // bits of the step size and of the convergence decision and nothing is
    // published between blocks.  Block 0 records the scalars for the host
    // and zeroes the cell-unit counters of the next iteration.
    __shared__ double s_v[4];
    auto reduce_all = [&](double v[4]) {
      reduce_partials<GridUnits>(a.partials, a.nchunks, v, sm);
      if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) s_v[q] = v[q];
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < 4; ++q) v[q] = s_v[q];
    };
    const bool recorder = blockIdx.x == 0 && threadIdx.x == 0;
    cell_pass<Real, GridUnits, 0>(a, 0, 0.0, false, nullptr, nullptr, 0);
    if (!bar.sync()) return;
    if (recorder) reset_take(sc, 1);
    constraint_pass<Real, GridUnits, 0>(a, 0, 0.0, true, sm, nullptr);
    if (!bar.sync()) return;
    double v[4];
    reduce_all(v);
    double alpha = 1.0 / v[3];
    if (recorder) {
      sc->res0 = v[3];
      sc->residual = v[3];
      sc->alpha = alpha;
    }
    long long it = 1;
    bool conv = false;
    while (it < a.max_it) {
      const bool check = (it % 10) == 0;
      cell_pass<Real, GridUnits, 0>(a, 1, alpha, check, nullptr, nullptr, (int)(it & 1));
      if (!bar.sync()) return;
      if (recorder) reset_take(sc, (int)((it + 1) & 1));
      constraint_pass<Real, GridUnits, 0>(a, 1, alpha, check, sm, nullptr);
      if (!bar.sync()) return;
      reduce_all(v);
      if (check && v[3] <= a.tol) conv = true;
      if (!conv) alpha = bb_step(v, it);
      if (recorder) {
        if (check) sc->residual = v[3];
        sc->alpha = alpha;
        sc->converged = conv ? 1 : 0;
        sc->iterations = it;
      }
      if (conv) break;
      ++it;
    }
    if (recorder) sc->iterations = it;
    if (!conv) return;
    const long long tid = (long long)blockIdx.x * kBlock + threadIdx.x, stride = (long long)nb * kBlock;
    for (long long c = tid; c < a.m; c += stride) a.phi[c] = ldcg(a.phin + c);
    return;
  }

  // gradient at gamma_0 and the initial residual (BBPGD.cpp:40-44)
  {
    double eq = 0.0, eg = 0.0;
    cell_pass<Real, GridUnits, kTr>(a, 0, 0.0, false, &eq, &eg);
    if (TR) trace_cells(smt, eq, eg, a.tr_part);
  }
  if (!bar.sync()) return;
  constraint_pass<Real, GridUnits, kTr>(a, 0, 0.0, true, sm, smt);
  auto reduce_init = [&]() {
    double v[4];
    reduce_partials<GridUnits>(a.partials, a.nchunks, v, sm);
    if (threadIdx.x == 0) {
      sc->res0 = v[3];
      sc->residual = v[3];
      sc->alpha = 1.0 / v[3];
      sc->converged = 0;
    }
    if (TR)
      trace_record(smt, a.tr_part, nb, a.nchunks, a.dt, a.lambda, a.tau, 0, v[3], 1.0 / v[3], a.trace_out,
                   a.trace_cap);
  };
  if (!bar.sync_reduce(reduce_init)) return;

  long long it = 1;
  while (it < a.max_it) {
    const double alpha = *(volatile double*)&sc->alpha;
    // with the trace on the residual is evaluated (and tested) every iteration (BBPGD.cpp:73)
    const bool check = (it % 10) == 0 || TR;
    {
      double eq = 0.0, eg = 0.0;
      cell_pass<Real, GridUnits, kTr>(a, 1, alpha, check, &eq, &eg);
      if (TR) trace_cells(smt, eq, eg, a.tr_part);
    }
    if (!bar.sync()) return;
    constraint_pass<Real, GridUnits, kTr>(a, 1, alpha, check, sm, smt);
    auto reduce_iter = [&]() {
      double v[4];
      reduce_partials<GridUnits>(a.partials, a.nchunks, v, sm);
      if (TR)
        trace_record(smt, a.tr_part, nb, a.nchunks, a.dt, a.lambda, a.tau, it, v[3], alpha, a.trace_out,
                     a.trace_cap);
      if (threadIdx.x == 0) {
        int conv = 0;
        if (check) {
          sc->residual = v[3];
          // a recording-only trace (trace == 2) keeps the every-10th test
          if (v[3] <= a.tol && (TR != 2 || it % 10 == 0)) conv = 1;
        }
        if (!conv) sc->alpha = bb_step(v, it);
        sc->converged = conv;
        sc->iterations = it;
      }
    };
    if (!bar.sync_reduce(reduce_iter)) return;
    if (*(volatile int*)&sc->converged) break;
    ++it;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->iterations = it;
  if (!*(volatile int*)&sc->converged) return;
  // returned result (Hard.cpp:170 with BBPGD.cpp:124): gamma_{k-1} (stored by
  // the last constraint pass), phi of gamma_k
  const long long tid = (long long)blockIdx.x * kBlock + threadIdx.x, stride = (long long)nb * kBlock;
  for (long long c = tid; c < a.m; c += stride) a.phi[c] = ldcg(a.phin + c);
}

// One-CTA form for colonies of up to kCtaCells cells and kCtaConstraints
// constraints: the same passes over four units, block barriers instead of
// grid barriers, unit 0 reducing the chunk partials.  An ordinary launch, so
// many small colonies' solves run side by side.
template <class Real>
__global__ void __launch_bounds__(kCtaThreads, 1) k_bbpgd_planar_cta(PArgs<Real> a) {
  __shared__ double sm[kCtaUnits][4 * (kBlock / 32)];
  __shared__ double s_alpha;
  __shared__ int s_conv;
  const unsigned unit = CtaUnits::unit();
  SolverScalars* sc = a.sc;

  cell_pass<Real, CtaUnits, 0>(a, 0, 0.0, false, nullptr, nullptr);
  __syncthreads();
  constraint_pass<Real, CtaUnits, 0>(a, 0, 0.0, true, sm[unit], nullptr);
  __syncthreads();
  if (unit == 0) {
    double v[4];
    reduce_partials<CtaUnits>(a.partials, a.nchunks, v, sm[0]);
    if (threadIdx.x == 0) {
      sc->res0 = v[3];
      sc->residual = v[3];
      s_alpha = 1.0 / v[3];
      s_conv = 0;
    }
  }
  __syncthreads();

  long long it = 1;
  while (it < a.max_it) {
    const double alpha = s_alpha;
    const bool check = (it % 10) == 0;
    cell_pass<Real, CtaUnits, 0>(a, 1, alpha, check, nullptr, nullptr);
    __syncthreads();
    constraint_pass<Real, CtaUnits, 0>(a, 1, alpha, check, sm[unit], nullptr);
    __syncthreads();
    if (unit == 0) {
      double v[4];
      reduce_partials<CtaUnits>(a.partials, a.nchunks, v, sm[0]);
      if (threadIdx.x == 0) {
        int conv = 0;
        if (check) {
          sc->residual = v[3];
          if (v[3] <= a.tol) conv = 1;
        }
        if (!conv) s_alpha = bb_step(v, it);
        s_conv = conv;
        sc->iterations = it;
      }
    }
    __syncthreads();
    if (s_conv) break;
    ++it;
  }
  if (threadIdx.x == 0) {
    sc->iterations = it;
    sc->converged = s_conv;
    sc->alpha = s_alpha;
  }
  if (!s_conv) return;
  for (long long c = threadIdx.x; c < a.m; c += kCtaThreads) a.phi[c] = a.phin[c];
}

// ---------------------------------------------------------------- packing
template <class Real>
__global__ void k_pack_planar_cons(ConsView cs, long long m, int2* __restrict__ ij,
                                   typename PT<Real>::V2* __restrict__ nn, typename PT<Real>::V2* __restrict__ tt,
                                   typename PT<Real>::V2* __restrict__ ss, double2* __restrict__ gg0) {
  using V2 = typename PT<Real>::V2;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m) return;
  ij[c] = make_int2(cs.gi[c], cs.gj[c]);
  nn[c] = mk2<V2>(cs.nx[c], cs.ny[c]);
  tt[c] = mk2<V2>(cs.tiz[c], cs.tjz[c]);
  ss[c] = mk2<V2>(cs.si[c], cs.sj[c]);
  gg0[c] = make_double2(cs.gamma[c], 0.0);
}

// Per incidence entry: its side's D row and the constraint's gamma_old.
template <class Real>
__global__ void k_pack_planar_inc(ConsView cs, const int* __restrict__ inc_ent, long long ne,
                                  typename PT<Real>::V4* __restrict__ inc, double* __restrict__ gold) {
  using V4 = typename PT<Real>::V4;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne) return;
  const int ent = inc_ent[k];
  const long long c = ent >> 1;
  const int side = ent & 1;
  if (side == 0)
    inc[k] = mk4<V4>(cs.nx[c], cs.ny[c], cs.tiz[c], cs.si[c]);
  else
    inc[k] = mk4<V4>(-cs.nx[c], -cs.ny[c], cs.tjz[c], cs.sj[c]);
  gold[k] = cs.gamma[c];
}

template <class Real>
__global__ void k_pack_planar_cells(const double* __restrict__ Ml, const double* __restrict__ Mr,
                                    const double* __restrict__ len, const double* __restrict__ ldot_prev, long long n,
                                    typename PT<Real>::V4* __restrict__ cell) {
  using V4 = typename PT<Real>::V4;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  cell[p] = mk4<V4>(Ml[p], Mr[p], len[p], ldot_prev[p]);
}

template <class Real>
struct PlanarBufs;
template <>
struct PlanarBufs<double> {
  static pcc::DevBuf<double2>& nn(pcc_ctx* c) { return c->p_n; }
  static pcc::DevBuf<double2>& tt(pcc_ctx* c) { return c->p_t; }
  static pcc::DevBuf<double2>& ss(pcc_ctx* c) { return c->p_s; }
  static pcc::DevBuf<double4>& inc(pcc_ctx* c) { return c->p_inc; }
  static pcc::DevBuf<double4>& cell(pcc_ctx* c) { return c->p_cell; }
  static pcc::DevBuf<double4>& u(pcc_ctx* c) { return c->p_u; }
};
template <>
struct PlanarBufs<float> {
  static pcc::DevBuf<float2>& nn(pcc_ctx* c) { return c->pf_n; }
  static pcc::DevBuf<float2>& tt(pcc_ctx* c) { return c->pf_t; }
  static pcc::DevBuf<float2>& ss(pcc_ctx* c) { return c->pf_s; }
  static pcc::DevBuf<float4>& inc(pcc_ctx* c) { return c->pf_inc; }
  static pcc::DevBuf<float4>& cell(pcc_ctx* c) { return c->pf_cell; }
  static pcc::DevBuf<float4>& u(pcc_ctx* c) { return c->pf_u; }
};

template <class Real>
cudaError_t launch(pcc_ctx* ctx, double dt, const PlanarTrace& tr, int* kind) {
  using B = PlanarBufs<Real>;
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->n, m = ctx->ncons, ne = 2 * m;
  const size_t mm = m + 1, nn = n + 1;
  cudaError_t e;
  if ((e = ctx->p_ij.reserve(mm, 0, s)) || (e = ctx->p_gg.reserve(mm, 0, s)) || (e = ctx->p_phin.reserve(mm, 0, s)) ||
      (e = ctx->p_gold.reserve(ne + 1, 0, s)))
    return e;
  if ((e = B::nn(ctx).reserve(mm, 0, s)) || (e = B::tt(ctx).reserve(mm, 0, s)) || (e = B::ss(ctx).reserve(mm, 0, s)) ||
      (e = B::inc(ctx).reserve(ne + 1, 0, s)) || (e = B::cell(ctx).reserve(nn, 0, s)) ||
      (e = B::u(ctx).reserve(nn, 0, s)))
    return e;
  const long long nchunks = chunk_count((long long)m, Occupancy<Real>::kChunks);
  if ((e = ctx->partials.reserve(4 * (nchunks + 1), 0, s))) return e;
  ConsView cv = ctx->cons.view();
  if (m) {
    k_pack_planar_cons<Real><<<grid_for((long long)m), kBlock, 0, s>>>(cv, (long long)m, ctx->p_ij.p, B::nn(ctx).p,
                                                                       B::tt(ctx).p, B::ss(ctx).p, ctx->p_gg.p);
    k_pack_planar_inc<Real><<<grid_for((long long)ne), kBlock, 0, s>>>(cv, ctx->inc_ent.p, (long long)ne,
                                                                       B::inc(ctx).p, ctx->p_gold.p);
    ctx->launches += 2;
  }
  if (n) {
    k_pack_planar_cells<Real><<<grid_for((long long)n), kBlock, 0, s>>>(
        ctx->Mlin.p, ctx->Mrot.p, ctx->cells.len.p, ctx->cells.ldot.p, (long long)n, B::cell(ctx).p);
    ctx->launches++;
  }
  PArgs<Real> a;
  a.m = (long long)m;
  a.n = (long long)n;
  a.ij = ctx->p_ij.p;
  a.nn = B::nn(ctx).p;
  a.tt = B::tt(ctx).p;
  a.ss = B::ss(ctx).p;
  a.phi = cv.sd;
  a.gamma = cv.gamma;
  a.phin = ctx->p_phin.p;
  a.gg = ctx->p_gg.p;
  a.inc_off = ctx->inc_off.p;
  a.inc = B::inc(ctx).p;
  a.gold = ctx->p_gold.p;
  a.cell = B::cell(ctx).p;
  a.u = B::u(ctx).p;
  a.uext = ctx->uext_active ? ctx->uext.p : nullptr;
  a.U = ctx->U.p;
  a.F = ctx->F.p;
  a.sig = ctx->sig.p;
  a.ldot = ctx->ldot_new.p;
  a.imp = ctx->imp_new.p;
  a.dt = dt;
  a.lambda = ctx->params.lambda;
  a.tau = ctx->params.tau;
  a.tol = ctx->params.tolerance;
  a.max_it = ctx->params.max_bbpgd_iterations;
  a.partials = reinterpret_cast<double4*>(ctx->partials.p);
  a.nchunks = nchunks;
  a.ent = ctx->inc_ent.p;
  a.sc = ctx->scal.p;
  a.st_err = ctx->status;
  a.trace = tr.trace;
  a.tr_part = tr.tr_part;
  a.trace_out = tr.trace_out;
  a.trace_cap = tr.trace_cap;
  void* args[] = {&a};
  if (ctx->profiling) cudaEventRecord(ctx->ev[0], s);
  if (!tr.trace && n <= (size_t)kCtaCells && m <= (size_t)kCtaConstraints) {
    *kind = 0;
    return cudaLaunchKernel((const void*)k_bbpgd_planar_cta<Real>, dim3(1), dim3(kCtaThreads), args, 0, s);
  }
  const void* kern = tr.trace ? (const void*)k_bbpgd_planar<Real, 1> : (const void*)k_bbpgd_planar<Real, 0>;
  int& coop = tr.trace ? (sizeof(Real) == 8 ? ctx->coop_planar_tr : ctx->coop_mixed_tr)
                       : (sizeof(Real) == 8 ? ctx->coop_blocks_planar : ctx->coop_blocks_mixed);
  if (coop == 0) {
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, 0))) return e;
    // at most kMaxBlocksPerSm blocks per SM: both grid barriers of an
    // iteration cost more with more arriving blocks than the extra resident
    // warps hide
    const int cap = Occupancy<Real>::kBlocksPerSm;
    coop = (per_sm < cap ? per_sm : cap) * ctx->num_sms;
  }
  long long want = (long long)grid_for((long long)n * kLanes);
  if (nchunks > want) want = nchunks;
  if (want > coop) want = coop;
  if (want < 1) want = 1;
  *kind = want > 1 ? 1 : 0;
  if (want == 1) return cudaLaunchKernel(kern, dim3(1), dim3(kBlock), args, 0, s);
  return cudaLaunchCooperativeKernel(kern, dim3((unsigned)want), dim3(kBlock), args, 0, s);
}

}  // namespace

long long planar_chunks(size_t m) {  // the larger of the two precisions' counts
  const long long a = chunk_count((long long)m, Occupancy<double>::kChunks);
  const long long b = chunk_count((long long)m, Occupancy<float>::kChunks);
  return a > b ? a : b;
}

cudaError_t planar_bbpgd(pcc_ctx* ctx, double dt, bool mixed, const PlanarTrace& tr, int* kind) {
  return mixed ? launch<float>(ctx, dt, tr, kind) : launch<double>(ctx, dt, tr, kind);
}

}  // namespace pcc
