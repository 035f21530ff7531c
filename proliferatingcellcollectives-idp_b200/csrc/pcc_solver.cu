// Hard-model BBPGD solver for non-planar colonies, the per-step solver glue
// and the soft-model force assembly (sm_100a).
//
// The BBPGD solve (solver/BBPGD.cpp:32-127 with the gradient of
// dynamics/models/hard/HardModelGradient.cpp:89-158) runs as ONE persistent
// cooperative kernel per ReLCP phase.  Each iteration is two grid-wide passes:
//   cell pass, kLanes lanes per cell: F = D^T (gamma - gamma_old) and
//     sigma = L^T gamma over the cell's incidence list (lane l takes entries
//     l, l + kLanes, ... in ascending constraint order; the lanes' sums meet
//     in a fixed shuffle tree; no atomics), U = M F, growth rate and its change;
//   constraint pass, one thread per constraint: phi_next = Phi + dt D U -
//     dt L dldot, the projected-gradient residual and the three
//     Barzilai-Borwein dot products, reduced per fixed chunk of constraints
//     (chunk_count, chunk_lo).
// The projection gamma_k = max(gamma_{k-1} - alpha g_{k-1}, 0) is recomputed
// where it is needed (both passes), so no extra pass stores it.  The last block
// to reach a barrier reduces the chunk partials in a fixed order and publishes
// alpha and the convergence decision: results do not depend on the grid size
// or on which block arrives last.  The decomposition and every reduction tree
// are those of the planar kernels (pcc_planar.cu), which skip only exact
// zeros, so a planar colony gives the same bits on either path.  Barrier
// waits are bounded; a wait that runs out raises kDevErrTimeout and the
// kernel returns.
#include <cfloat>
#include <cmath>

#include "pcc_bbpgd.cuh"
#include "pcc_kernels.hpp"

namespace pcc {

namespace {

constexpr int kOneBlockCells = 1024;      // otherwise one 256-thread block up to this many cells ...
constexpr int kOneBlockConstraints = 4096;  // ... and constraints

struct SolverArgs {
  // constraints
  long long m;
  const int *gi, *gj;
  const double *nx, *ny, *nz, *tix, *tiy, *tiz, *tjx, *tjy, *tjz, *si, *sj;
  double *phi;    // Phi on entry; phi_next of the returned iterate on exit
  double *gamma;  // gamma_0 on entry (also gamma_old); gamma_{k-1} on exit
  double *gam[2], *g[2];
  // cells
  long long n;
  const int *inc_off, *inc_ent;
  const double *Mlin, *Mrot, *len, *ldot_prev;
  const double* uext;  // rotational U_ext, 3 per cell (Brownian kicks at ReLCP phase 0); null: zero
  double *U, *dl, *F, *sig, *ldot, *imp;
  double dt, lambda, tau, tol;
  long long max_it;
  double* partials;  // 4 per chunk
  long long nchunks;
  SolverScalars* sc;
  DevStatus* st;
  // BBPGD trace (-log_bbgd_trace): residual every iteration and the energy
  // terms; 1 tests convergence at every iteration as the reference does while
  // tracing, 2 records without changing when convergence is tested
  int trace;
  double* tr_part;     // 2 per block (cell terms), then 1 per chunk (linear term)
  double* trace_out;   // kTraceWidth per iteration
  long long trace_cap; // iterations that fit
};



// Cell pass.  mode 0: gamma = gamma_0; mode 1: gamma_k projected from
// (gam_prev, g_prev, alpha).  Writes U and dldot; with `final` also F, sigma,
// ldot and impedance.
template <int kTr>
__device__ __forceinline__ void cell_pass(const SolverArgs& a, int mode, const double* gprev_gam,
                                          const double* gprev_g, double alpha, bool final, double* eq, double* eg) {
  const int lane = threadIdx.x & 31, gl = lane % kLanes;
  constexpr long long kCellsPerWarp = 32 / kLanes;
  for (long long pw = GridUnits::warp() * kCellsPerWarp; pw < a.n; pw += GridUnits::warps() * kCellsPerWarp) {
    const long long p = pw + lane / kLanes;
    int b = 0, e = 0;
    if (p < a.n) {
      b = a.inc_off[p];
      e = a.inc_off[p + 1];
    }
    double F[6] = {0, 0, 0, 0, 0, 0};
    double Fg[6] = {0, 0, 0, 0, 0, 0};  // D^T gamma (trace only)
    double sg = 0.0;
    for (int k = b + gl; k < e; k += kLanes) {
      const int ent = a.inc_ent[k];
      const long long c = ent >> 1;
      const int side = ent & 1;
      const double gold = a.gamma[c];
      const double gc = mode == 0 ? gold : project(ldcg(gprev_gam + c), ldcg(gprev_g + c), alpha);
      const double diff = sub(gc, gold);
      double D[6];
      if (side == 0) {
        D[0] = a.nx[c];
        D[1] = a.ny[c];
        D[2] = a.nz[c];
        D[3] = a.tix[c];
        D[4] = a.tiy[c];
        D[5] = a.tiz[c];
      } else {
        D[0] = -a.nx[c];
        D[1] = -a.ny[c];
        D[2] = -a.nz[c];
        D[3] = a.tjx[c];
        D[4] = a.tjy[c];
        D[5] = a.tjz[c];
      }
#pragma unroll
      for (int q = 0; q < 6; ++q) F[q] = add(F[q], mul(D[q], diff));
      sg = add(sg, mul(side == 0 ? a.si[c] : a.sj[c], gc));
      if constexpr (kTr) {
#pragma unroll
        for (int q = 0; q < 6; ++q) Fg[q] = add(Fg[q], mul(D[q], gc));
      }
    }
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) {
#pragma unroll
      for (int q = 0; q < 6; ++q) F[q] = add(F[q], __shfl_xor_sync(kFull, F[q], o));
      sg = add(sg, __shfl_xor_sync(kFull, sg, o));
      if constexpr (kTr) {
#pragma unroll
        for (int q = 0; q < 6; ++q) Fg[q] = add(Fg[q], __shfl_xor_sync(kFull, Fg[q], o));
      }
    }
    if (gl != 0 || p >= a.n) continue;
    const double ml = a.Mlin[p], mr = a.Mrot[p];
    double* U = a.U + 6 * p;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const double uc = add(0.0, mul(q < 3 ? ml : mr, F[q]));
      // U = U_ext + M F (VecWAXPY, HardModelGradient.cpp:21); U_ext is rotational only
      U[q] = add(uc, (q >= 3 && a.uext) ? a.uext[3 * p + q - 3] : 0.0);
    }
    const double im = exp(vscale(-a.lambda, sg));
    const double ld = vscale(dvd(1.0, a.tau), mul(a.len[p], im));
    a.dl[p] = sub(ld, a.ldot_prev[p]);
    if constexpr (kTr) {
#pragma unroll
      for (int q = 0; q < 6; ++q) *eq = add(*eq, mul(Fg[q], mul(q < 3 ? ml : mr, Fg[q])));
      *eg = add(*eg, mul(a.len[p], im));
    }
    if (final) {
#pragma unroll
      for (int q = 0; q < 6; ++q) a.F[6 * p + q] = F[q];
      a.sig[p] = sg;
      a.ldot[p] = ld;
      a.imp[p] = im;
    }
  }
}

// Pass B value for constraint c: phi_next(gamma) given U and dldot.
__device__ __forceinline__ double constraint_grad(const SolverArgs& a, long long c) {
  const int i = a.gi[c], j = a.gj[c];
  const double* Ui = a.U + 6 * (long long)i;
  const double* Uj = a.U + 6 * (long long)j;
  const double Di[6] = {a.nx[c], a.ny[c], a.nz[c], a.tix[c], a.tiy[c], a.tiz[c]};
  const double Dj[6] = {-a.nx[c], -a.ny[c], -a.nz[c], a.tjx[c], a.tjy[c], a.tjz[c]};
  double pd = 0.0;
  // MatMult row c: ascending columns; gi < gj for every emitted constraint
  if (i < j) {
#pragma unroll
    for (int q = 0; q < 6; ++q) pd = add(pd, mul(Di[q], ldcg(Ui + q)));
#pragma unroll
    for (int q = 0; q < 6; ++q) pd = add(pd, mul(Dj[q], ldcg(Uj + q)));
  } else {
#pragma unroll
    for (int q = 0; q < 6; ++q) pd = add(pd, mul(Dj[q], ldcg(Uj + q)));
#pragma unroll
    for (int q = 0; q < 6; ++q) pd = add(pd, mul(Di[q], ldcg(Ui + q)));
  }
  double gr = 0.0;
  if (i < j) {
    gr = add(gr, mul(a.si[c], ldcg(a.dl + i)));
    gr = add(gr, mul(a.sj[c], ldcg(a.dl + j)));
  } else {
    gr = add(gr, mul(a.sj[c], ldcg(a.dl + j)));
    gr = add(gr, mul(a.si[c], ldcg(a.dl + i)));
  }
  // VecMAXPY(phi_next, {dt, -dt}, {phidot, growth})
  return add(a.phi[c], add(mul(a.dt, pd), mul(-a.dt, gr)));
}

// Block partials of the cell energy terms (all threads of the block call).
__device__ __forceinline__ void trace_cells(double* sm, double eq, double eg, double* tr_part) {
  double v[4] = {eq, eg, 0, 0};
  block_reduce4(v, sm);
  if (threadIdx.x == 0) {
    tr_part[2 * blockIdx.x] = v[0];
    tr_part[2 * blockIdx.x + 1] = v[1];
  }
}

__device__ __forceinline__ void trace_chunk(double* sm, double lin, double* tr_part, unsigned nb, long long ch) {
  double v[4] = {lin, 0, 0, 0};
  block_reduce4(v, sm);
  if (threadIdx.x == 0) tr_part[2 * nb + ch] = v[0];
}

// Constraint pass over the chunks of this block: new (gamma, g) into
// (gam_out, g_out) and the chunk partials; mode 0 evaluates g at gamma_0
// (residual only).
template <int kTr>
__device__ __forceinline__ void constraint_pass(const SolverArgs& a, int mode, const double* gp, const double* gg,
                                                double* gam_out, double* g_out, double alpha, bool check, double* sm,
                                                double* smt) {
  double4* partials = reinterpret_cast<double4*>(a.partials);
  for (long long ch = blockIdx.x; ch < a.nchunks; ch += gridDim.x) {
    double v[4] = {0, 0, 0, 0};  // sum dgam^2, sum dgam*dg, sum dg^2, max residual
    double lin = 0.0;
    const long long hi = chunk_lo(ch + 1, a.m, a.nchunks);
    for (long long c = chunk_lo(ch, a.m, a.nchunks) + threadIdx.x; c < hi; c += kBlock) {
      const double gpc = mode == 0 ? a.gamma[c] : ldcg(gp + c), ggc = mode == 0 ? 0.0 : ldcg(gg + c);
      const double gam = mode == 0 ? gpc : project(gpc, ggc, alpha);
      const double g = constraint_grad(a, c);
      gam_out[c] = gam;
      g_out[c] = g;
      if (mode != 0) {
        const double dgm = sub(gam, gpc), dg = sub(g, ggc);
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
    unit_reduce4<GridUnits>(v, sm);
    if (threadIdx.x == 0) partials[ch] = make_double4(v[0], v[1], v[2], v[3]);
    if constexpr (kTr) {
      if (a.trace) trace_chunk(smt, lin, a.tr_part, gridDim.x, ch);
    }
  }
}

// kTr = 1 compiles the trace hooks in; the untraced kernel carries none of them.
template <int kTr>
__global__ void __launch_bounds__(kBlock) k_bbpgd(SolverArgs a) {
  const int TR = kTr ? a.trace : 0;
  __shared__ double sm[4 * (kBlock / 32)];
  __shared__ double smt[kTr ? 4 * kBlock : 1];
  const unsigned nb = gridDim.x;
  const long long tid = (long long)blockIdx.x * kBlock + threadIdx.x;
  const long long stride = (long long)nb * kBlock;
  SolverScalars* sc = a.sc;
  GridBarrier bar{sc, a.st, nb};
  const double4* partials = reinterpret_cast<const double4*>(a.partials);

  // ---- gradient at gamma_0 and the initial residual (BBPGD.cpp:40-44)
  {
    double eq = 0.0, eg = 0.0;
    cell_pass<kTr>(a, 0, nullptr, nullptr, 0.0, false, &eq, &eg);
    if (TR) trace_cells(smt, eq, eg, a.tr_part);
  }
  if (!bar.sync()) return;
  constraint_pass<kTr>(a, 0, nullptr, nullptr, a.gam[0], a.g[0], 0.0, true, sm, smt);
  auto reduce_init = [&]() {
    double v[4];
    reduce_partials<GridUnits>(partials, a.nchunks, v, sm);
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

  int p = 0;  // buffer of gamma_{k-1}, g_{k-1}
  long long it = 1;
  while (it < a.max_it) {
    const double alpha = *(volatile double*)&sc->alpha;
    // with the trace on the residual is evaluated (and tested) every iteration (BBPGD.cpp:73)
    const bool check = (it % 10) == 0 || TR;
    {
      double eq = 0.0, eg = 0.0;
      cell_pass<kTr>(a, 1, a.gam[p], a.g[p], alpha, check, &eq, &eg);
      if (TR) trace_cells(smt, eq, eg, a.tr_part);
    }
    if (!bar.sync()) return;
    constraint_pass<kTr>(a, 1, a.gam[p], a.g[p], a.gam[1 - p], a.g[1 - p], alpha, check, sm, smt);
    auto reduce_iter = [&]() {
      double v[4];
      reduce_partials<GridUnits>(partials, a.nchunks, v, sm);
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
        if (!conv) sc->alpha = bb_step(v, it);  // BBPGD.cpp:98-112
        sc->converged = conv;
        sc->iterations = it;
      }
    };
    if (!bar.sync_reduce(reduce_iter)) return;
    if (*(volatile int*)&sc->converged) break;
    p = 1 - p;
    ++it;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->iterations = it;
  if (!*(volatile int*)&sc->converged) return;
  // Returned result (Hard.cpp:170 with BBPGD.cpp:124): gamma_{k-1}, phi(gamma_k).
  for (long long c = tid; c < a.m; c += stride) {
    a.gamma[c] = ldcg(a.gam[p] + c);
    a.phi[c] = ldcg(a.g[1 - p] + c);
  }
}

// Cell update after a solve: dC = G U (Physics.cpp:220-265), Euler step and
// quaternion normalisation (simulation/Particle.cpp:37-57, 110-120), force,
// velocity and growth parameters (ParticleManager.cpp:29-130).
__global__ void k_move(CellsView c, long long n, const double* __restrict__ U, const double* __restrict__ F,
                       const double* __restrict__ ldot, const double* __restrict__ imp, const double* __restrict__ sig,
                       double dt) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = c.q0[i], wx = c.q1[i], wy = c.q2[i], wz = c.q3[i];
  const double* u = U + 6 * i;
  double dC[7];
  for (int k = 0; k < 3; ++k) dC[k] = add(0.0, mul(1.0, u[k]));
  const double xi[4][3] = {{mul(-0.5, wx), mul(-0.5, wy), mul(-0.5, wz)},
                           {mul(0.5, s), mul(-0.5, wz), mul(0.5, wy)},
                           {mul(0.5, wz), mul(0.5, s), mul(-0.5, wx)},
                           {mul(-0.5, wy), mul(0.5, wx), mul(0.5, s)}};
  for (int r = 0; r < 4; ++r) {
    double acc = 0.0;
    for (int k = 0; k < 3; ++k) acc = add(acc, mul(xi[r][k], u[3 + k]));
    dC[3 + r] = acc;
  }
  c.x[i] = add(c.x[i], mul(dt, dC[0]));
  c.y[i] = add(c.y[i], mul(dt, dC[1]));
  c.z[i] = add(c.z[i], mul(dt, dC[2]));
  double q[4] = {add(s, mul(dt, dC[3])), add(wx, mul(dt, dC[4])), add(wy, mul(dt, dC[5])), add(wz, mul(dt, dC[6]))};
  double nrm = __dsqrt_rn(add(add(add(mul(q[0], q[0]), mul(q[1], q[1])), mul(q[2], q[2])), mul(q[3], q[3])));
  c.q0[i] = dvd(q[0], nrm);
  c.q1[i] = dvd(q[1], nrm);
  c.q2[i] = dvd(q[2], nrm);
  c.q3[i] = dvd(q[3], nrm);
  for (int k = 0; k < 6; ++k) {
    c.force[6 * i + k] = F[6 * i + k];
    c.vel[6 * i + k] = u[k];
  }
  c.ldot[i] = ldot[i];
  c.imp[i] = imp[i];
  c.stress[i] = sig[i];
}

__global__ void k_max_overlap(const double* __restrict__ sd, long long from, long long to,
                              unsigned long long* __restrict__ dst) {
  long long c = from + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (c < to) v = sd[c] < 0 ? -sd[c] : 0.0;
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_down_sync(0xffffffffu, v, o);
    v = v < w ? w : v;
  }
  if ((threadIdx.x & 31) == 0 && v > 0.0) atomicMax(dst, (unsigned long long)__double_as_longlong(v));
}

// x^1.5 correctly rounded in practice: sqrt with its exact residual and the
// exact error of the product (error-free transformations), one final rounding.
__device__ __forceinline__ double pow15(double x) {
  const double s = __dsqrt_rn(x);
  const double r = fma(-s, s, x);           // x - s^2, exact
  const double ds = r / (2.0 * s);          // sqrt(x) ~ s + ds
  const double p = x * s;
  const double pe = fma(x, s, -p);          // x*s - p, exact
  return p + (pe + x * ds);
}

// Soft model, per contact: Hertz force magnitude (dynamics/models/Soft.cpp:46-60)
__global__ void k_soft_fel(ConsView cs, long long m, const double* __restrict__ diam, double kcc,
                           double* __restrict__ fel) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m) return;
  const double overlap = -cs.sd[c];
  if (overlap <= 0.00) {
    fel[c] = 0.0;
    return;
  }
  const double R1 = dvd(diam[cs.gi[c]], 2.0), R2 = dvd(diam[cs.gj[c]], 2.0);
  const double R_eff = __dsqrt_rn(dvd(mul(R1, R2), add(R1, R2)));
  fel[c] = mul(mul(R_eff, kcc), pow15(overlap));
}

// Soft model, per cell: force, torque and stress summed over the incident
// contacts -- a segmented reduction over the incidence list: kLanes lanes per
// cell, lane l taking the cell's entries l, l + kLanes, ... in ascending
// contact order, the lanes' sums combined by a fixed shuffle tree -- then
// U = M F, dC = G U and the move, growth rate (first lane).
__global__ void k_soft_cell(CellsView c, long long n, ConsView cs, const int* __restrict__ inc_off,
                            const int* __restrict__ inc_ent, const double* __restrict__ fel, double xi, double lambda,
                            double tau, double dt, int move, const double* __restrict__ uext) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int gl = (int)(t % kLanes);
  const long long i = t / kLanes;
  // every lane of a group takes part in the shuffles: the group's cell is past
  // the end only for whole groups, which return together
  if (i >= n) return;
  double F[6] = {0, 0, 0, 0, 0, 0};
  double sg = 0.0;
  for (int k = inc_off[i] + gl; k < inc_off[i + 1]; k += kLanes) {
    const int ent = inc_ent[k];
    const long long q = ent >> 1;
    if (-cs.sd[q] <= 0.00) continue;  // Soft.cpp:49 skips non-overlapping contacts
    const double fe = fel[q];
    const double fi[3] = {mul(cs.nx[q], fe), mul(cs.ny[q], fe), mul(cs.nz[q], fe)};
    double f[3], r[3];
    if ((ent & 1) == 0) {
      f[0] = fi[0];
      f[1] = fi[1];
      f[2] = fi[2];
      r[0] = cs.rix[q];
      r[1] = cs.riy[q];
      r[2] = cs.riz[q];
    } else {
      f[0] = -fi[0];
      f[1] = -fi[1];
      f[2] = -fi[2];
      r[0] = cs.rjx[q];
      r[1] = cs.rjy[q];
      r[2] = cs.rjz[q];
    }
    double tq[3];
    cross3(r, f, tq);
    for (int d = 0; d < 3; ++d) F[d] = add(F[d], f[d]);
    for (int d = 0; d < 3; ++d) F[3 + d] = add(F[3 + d], tq[d]);
    sg = add(sg, mul((ent & 1) == 0 ? cs.si[q] : cs.sj[q], fe));
  }
  // a group's lanes are consecutive threads of one warp (kLanes divides 32)
  const unsigned gmask = ((1u << kLanes) - 1u) << (threadIdx.x & 31 & ~(kLanes - 1));
#pragma unroll
  for (int o = kLanes / 2; o > 0; o >>= 1) {
#pragma unroll
    for (int d = 0; d < 6; ++d) F[d] = add(F[d], __shfl_xor_sync(gmask, F[d], o));
    sg = add(sg, __shfl_xor_sync(gmask, sg, o));
  }
  if (gl != 0) return;
  if (!move) {
    for (int d = 0; d < 6; ++d) c.force[6 * i + d] = F[d];
    c.stress[i] = sg;
    return;
  }
  // Mobility (Physics.cpp:192-218)
  const double l = c.len[i];
  const double ml = dvd(1.0, mul(l, xi));
  const double mr = dvd(12.0, mul(mul(mul(l, l), l), xi));
  double u[6];
  // U = U_ext + M F (Soft.cpp:14-15); U_ext is rotational only
  for (int d = 0; d < 6; ++d)
    u[d] = add(add(0.0, mul(d < 3 ? ml : mr, F[d])), (d >= 3 && uext) ? uext[3 * i + d - 3] : 0.0);
  const double s = c.q0[i], wx = c.q1[i], wy = c.q2[i], wz = c.q3[i];
  double dC[7];
  for (int k = 0; k < 3; ++k) dC[k] = add(0.0, mul(1.0, u[k]));
  const double xm[4][3] = {{mul(-0.5, wx), mul(-0.5, wy), mul(-0.5, wz)},
                           {mul(0.5, s), mul(-0.5, wz), mul(0.5, wy)},
                           {mul(0.5, wz), mul(0.5, s), mul(-0.5, wx)},
                           {mul(-0.5, wy), mul(0.5, wx), mul(0.5, s)}};
  for (int rr = 0; rr < 4; ++rr) {
    double acc = 0.0;
    for (int k = 0; k < 3; ++k) acc = add(acc, mul(xm[rr][k], u[3 + k]));
    dC[3 + rr] = acc;
  }
  c.x[i] = add(c.x[i], mul(dt, dC[0]));
  c.y[i] = add(c.y[i], mul(dt, dC[1]));
  c.z[i] = add(c.z[i], mul(dt, dC[2]));
  double qq[4] = {add(s, mul(dt, dC[3])), add(wx, mul(dt, dC[4])), add(wy, mul(dt, dC[5])), add(wz, mul(dt, dC[6]))};
  double nrm = __dsqrt_rn(add(add(add(mul(qq[0], qq[0]), mul(qq[1], qq[1])), mul(qq[2], qq[2])), mul(qq[3], qq[3])));
  c.q0[i] = dvd(qq[0], nrm);
  c.q1[i] = dvd(qq[1], nrm);
  c.q2[i] = dvd(qq[2], nrm);
  c.q3[i] = dvd(qq[3], nrm);
  for (int d = 0; d < 6; ++d) {
    c.force[6 * i + d] = F[d];
    c.vel[6 * i + d] = u[d];
  }
  // calculate_growth_rate_vector (HardModelGradient.cpp:43-52)
  const double im = exp(vscale(-lambda, sg));
  c.stress[i] = sg;
  c.imp[i] = im;
  c.ldot[i] = vscale(dvd(1.0, tau), mul(l, im));
}

__global__ void k_mobility(const double* __restrict__ len, long long n, double xi, double* __restrict__ Ml,
                           double* __restrict__ Mr) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double l = len[i];
  Ml[i] = dvd(1.0, mul(l, xi));
  Mr[i] = dvd(12.0, mul(mul(mul(l, l), l), xi));
}

// U_ext of one draw (Particle::calculateBrownianVelocity, Particle.cpp:174-190):
// coef = T u1 u_k from the host, times the impedance three times in the
// reference's left-to-right order, added into a zeroed vector (VecSetValues
// ADD_VALUES, Physics.cpp:73-75).  Monolayer kicks have only the z component.
__global__ void k_uext(const double* __restrict__ coef, const double* __restrict__ imp, long long n, int monolayer,
                       double* __restrict__ uext) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double im = imp[i];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double v = (monolayer && k < 2) ? 0.0 : mul(mul(mul(coef[3 * i + k], im), im), im);
    uext[3 * i + k] = add(0.0, v);
  }
}

}  // namespace

cudaError_t brownian_draw(pcc_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->n;
  ctx->uext_active = false;
  if (!(ctx->params.temperature > 0) || n == 0) return cudaSuccess;
  cudaError_t e;
  if ((e = ctx->uext.reserve(3 * n + 3, 0, s)) || (e = ctx->brown_coef.reserve(3 * n + 3, 0, s))) return e;
  if (ctx->brown_host_cap < 3 * n) {
    if (ctx->brown_host) {
      if ((e = cudaStreamSynchronize(s))) return e;  // the last upload may still read it
      cudaFreeHost(ctx->brown_host);
      ctx->brown_host = nullptr;
      ctx->brown_host_cap = 0;
    }
    const size_t cap = 3 * n + 3 * n / 2 + 192;
    if ((e = cudaMallocHost(&ctx->brown_host, cap * sizeof(double)))) return e;
    ctx->brown_host_cap = cap;
  } else {
    if ((e = cudaStreamSynchronize(s))) return e;  // the staging buffer is reused
  }
  // one uniform_real_distribution(-1, 1) per call, as Particle::calculateBrownianVelocity;
  // the draw order is the particle order, i.e. global-id order after the x-sort
  const double T = ctx->params.temperature;
  const bool mono = ctx->params.monolayer != 0;
  double* h = ctx->brown_host;
  for (size_t i = 0; i < n; ++i) {
    std::uniform_real_distribution<double> dist(-1.0, 1.0);
    const double rot = T * dist(ctx->brown_gen);
    if (mono) {
      h[3 * i] = 0.0;
      h[3 * i + 1] = 0.0;
      h[3 * i + 2] = rot * dist(ctx->brown_gen);
    } else {
      h[3 * i] = rot * dist(ctx->brown_gen);
      h[3 * i + 1] = rot * dist(ctx->brown_gen);
      h[3 * i + 2] = rot * dist(ctx->brown_gen);
    }
  }
  if ((e = cudaMemcpyAsync(ctx->brown_coef.p, h, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s))) return e;
  k_uext<<<grid_for((long long)n), kBlock, 0, s>>>(ctx->brown_coef.p, ctx->cells.imp.p, (long long)n, mono ? 1 : 0,
                                                   ctx->uext.p);
  ctx->launches++;
  ctx->uext_active = true;
  return cudaGetLastError();
}

cudaError_t mobility(pcc_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  if ((e = ctx->Mlin.reserve(ctx->n + 1, 0, s))) return e;
  if ((e = ctx->Mrot.reserve(ctx->n + 1, 0, s))) return e;
  if (ctx->n) {
    k_mobility<<<grid_for(ctx->n), kBlock, 0, s>>>(ctx->cells.len.p, (long long)ctx->n, ctx->params.xi,
                                                   ctx->Mlin.p, ctx->Mrot.p);
    ctx->launches++;
  }
  return cudaGetLastError();
}

cudaError_t bbpgd_solve(pcc_ctx* ctx, double dt, long long* iterations, double* residual, int* status,
                        bool defer) {
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->n, m = ctx->ncons;
  cudaError_t e;
  const size_t mm = m + 1, nn = n + 1;
  if ((e = ctx->U.reserve(6 * nn, 0, s)) || (e = ctx->dldot.reserve(nn, 0, s)) || (e = ctx->F.reserve(6 * nn, 0, s)) ||
      (e = ctx->sig.reserve(nn, 0, s)) || (e = ctx->ldot_new.reserve(nn, 0, s)) || (e = ctx->imp_new.reserve(nn, 0, s)))
    return e;
  if ((e = ctx->scal.reserve(1, 0, s))) return e;
  cudaMemsetAsync(ctx->scal.p, 0, sizeof(SolverScalars), s);
  const long long nchunks = chunk_count((long long)m);  // the FP64 planar kernel's chunks
  const bool tracing = ctx->trace_active;
  long long trace_cap = 0;
  if (tracing) {
    trace_cap = ctx->params.max_bbpgd_iterations + 1;
    if (trace_cap > (1LL << 22)) trace_cap = 1LL << 22;
    if ((e = ctx->trace_dev.reserve((size_t)(kTraceWidth * trace_cap), 0, s))) return e;
    // 2 per block of the largest grid, 1 per chunk (the planar chunks are the smaller)
    if ((e = ctx->tr_part.reserve((size_t)(2 * 8 * ctx->num_sms * 8 + planar_chunks(m) + 1), 0, s))) return e;
  }
  const int trace = tracing ? (ctx->params.log_bbpgd_trace == 2 ? 2 : 1) : 0;

  // out-of-plane Brownian kicks (-monolayer off) leave the planar form
  const bool planar = ctx->planar && ctx->params.solver_variant != PCC_SOLVER_GENERAL &&
                      !(ctx->uext_active && !ctx->params.monolayer);
  const bool mixed = planar && ctx->params.precision == PCC_PRECISION_MIXED;
  int kind = 0;
  if (planar) {  // records ev[0] itself, after packing its operands
    const PlanarTrace tr{trace, ctx->tr_part.p, ctx->trace_dev.p, trace_cap};
    e = planar_bbpgd(ctx, dt, mixed, tr, &kind);
  } else {
    if ((e = ctx->gam_a.reserve(mm, 0, s)) || (e = ctx->gam_b.reserve(mm, 0, s)) || (e = ctx->g_a.reserve(mm, 0, s)) ||
        (e = ctx->g_b.reserve(mm, 0, s)))
      return e;
    if ((e = ctx->partials.reserve(4 * (nchunks + 1), 0, s))) return e;
    SolverArgs a;
    ConsView cv = ctx->cons.view();
    a.m = (long long)m;
    a.gi = cv.gi;
    a.gj = cv.gj;
    a.nx = cv.nx;
    a.ny = cv.ny;
    a.nz = cv.nz;
    a.tix = cv.tix;
    a.tiy = cv.tiy;
    a.tiz = cv.tiz;
    a.tjx = cv.tjx;
    a.tjy = cv.tjy;
    a.tjz = cv.tjz;
    a.si = cv.si;
    a.sj = cv.sj;
    a.phi = cv.sd;
    a.gamma = cv.gamma;
    a.gam[0] = ctx->gam_a.p;
    a.gam[1] = ctx->gam_b.p;
    a.g[0] = ctx->g_a.p;
    a.g[1] = ctx->g_b.p;
    a.n = (long long)n;
    a.inc_off = ctx->inc_off.p;
    a.inc_ent = ctx->inc_ent.p;
    a.Mlin = ctx->Mlin.p;
    a.Mrot = ctx->Mrot.p;
    a.len = ctx->cells.len.p;
    a.ldot_prev = ctx->cells.ldot.p;
    a.uext = ctx->uext_active ? ctx->uext.p : nullptr;
    a.U = ctx->U.p;
    a.dl = ctx->dldot.p;
    a.F = ctx->F.p;
    a.sig = ctx->sig.p;
    a.ldot = ctx->ldot_new.p;
    a.imp = ctx->imp_new.p;
    a.dt = dt;
    a.lambda = ctx->params.lambda;
    a.tau = ctx->params.tau;
    a.tol = ctx->params.tolerance;
    a.max_it = ctx->params.max_bbpgd_iterations;
    a.partials = ctx->partials.p;
    a.nchunks = nchunks;
    a.sc = ctx->scal.p;
    a.st = ctx->status;
    a.trace = trace;
    a.tr_part = ctx->tr_part.p;
    a.trace_out = ctx->trace_dev.p;
    a.trace_cap = trace_cap;
    const void* kern = tracing ? (const void*)k_bbpgd<1> : (const void*)k_bbpgd<0>;
    int& coop = ctx->coop_blocks;
    if (coop == 0) {
      int per_sm = 0;
      if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, 0))) return e;
      // at most 4 blocks per SM: the two grid barriers of every iteration cost
      // more with more arriving blocks than the extra resident warps hide
      coop = (per_sm < 4 ? per_sm : 4) * ctx->num_sms;
    }
    long long want = (long long)grid_for((long long)n * kLanes);
    if (nchunks > want) want = nchunks;
    if (want > coop) want = coop;
    // Small colonies run in one block: its barriers are block barriers, it
    // needs no co-residency guarantee, so it is an ordinary launch that runs
    // beside other colonies' kernels.  The result does not depend on the grid.
    if (n <= (size_t)kOneBlockCells && m <= (size_t)kOneBlockConstraints) want = 1;
    if (want < 1) want = 1;
    void* args[] = {&a};
    if (ctx->profiling) cudaEventRecord(ctx->ev[0], s);
    if (want == 1)
      e = cudaLaunchKernel(kern, dim3(1), dim3(kBlock), args, 0, s);
    else
      e = cudaLaunchCooperativeKernel(kern, dim3((unsigned)want), dim3(kBlock), args, 0, s);
    kind = want > 1 ? 1 : 0;
  }
  ctx->launches++;
  if (e) return e;
  if (kind)
    ctx->prof.bbpgd_grid_launches++;
  else
    ctx->prof.bbpgd_cta_launches++;
  if (ctx->profiling) cudaEventRecord(ctx->ev[1], s);
  // 312 B per constraint and 288 B per cell in FP64; the FP32 operand terms halve
  ctx->bbpgd_pending_bytes = mixed ? 192.0 * (double)m + 144.0 * (double)n : 312.0 * (double)m + 288.0 * (double)n;
  if ((e = cudaMemcpyAsync(ctx->scal_host, ctx->scal.p, kScalarsCopied, cudaMemcpyDeviceToHost, s))) return e;
  if ((e = cudaMemcpyAsync(ctx->status_host, ctx->status, sizeof(DevStatus), cudaMemcpyDeviceToHost, s))) return e;
  ctx->bbpgd_pending = true;
  if (defer && !tracing) return cudaSuccess;  // read at the caller's next synchronisation
  if ((e = cudaStreamSynchronize(s))) return e;
  const long long it_done = ctx->scal_host->iterations;
  bbpgd_collect(ctx, iterations, residual, status);
  if (tracing) {
    // records 0 .. the last iteration run (BBPGD.cpp:55-81)
    long long nrec = it_done + 1;
    if (nrec > trace_cap) nrec = trace_cap;
    std::vector<double> rec((size_t)(kTraceWidth * nrec));
    if ((e = cudaMemcpy(rec.data(), ctx->trace_dev.p, rec.size() * sizeof(double), cudaMemcpyDeviceToHost)))
      return e;
    for (long long k = 0; k < nrec; ++k) {
      const double* r = rec.data() + kTraceWidth * k;
      pcc_bbpgd_trace_step t;
      t.step = (unsigned long long)k;
      t.recursive_iteration = (unsigned long long)ctx->trace_phase;
      t.total_constraints = (unsigned long long)m;
      t.residual = r[1];
      t.step_size = r[2];
      t.linear = r[3];
      t.quadratic = r[4];
      t.growth = r[5];
      t.total = r[6];
      ctx->trace_host.push_back(t);
    }
  }
  return cudaSuccess;
}

void bbpgd_collect(pcc_ctx* ctx, long long* iterations, double* residual, int* status) {
  const SolverScalars& host = *ctx->scal_host;
  ctx->bbpgd_pending = false;
  *iterations = host.iterations;
  *residual = host.residual;
  if (ctx->profiling) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    ctx->prof.bbpgd_launches++;
    ctx->prof.bbpgd_iterations += host.iterations;
    ctx->prof.bbpgd_ms += ms;
    ctx->prof.bbpgd_algo_bytes += (double)host.iterations * ctx->bbpgd_pending_bytes;
  }
  if (ctx->status_host->flags)
    *status = (ctx->status_host->flags & kDevErrTimeout) ? PCC_ERR_TIMEOUT : PCC_ERR_BOUNDS;
  else
    *status = host.converged ? PCC_OK : PCC_ERR_NOCONV_BBPGD;
}

cudaError_t apply_hard_solution(pcc_ctx* ctx, double dt) {
  if (!ctx->n) return cudaSuccess;
  k_move<<<grid_for(ctx->n), kBlock, 0, ctx->stream>>>(ctx->cells.view(), (long long)ctx->n, ctx->U.p, ctx->F.p,
                                                       ctx->ldot_new.p, ctx->imp_new.p, ctx->sig.p, dt);
  ctx->launches++;
  return cudaGetLastError();
}

cudaError_t max_overlap_enqueue(pcc_ctx* ctx, size_t from, size_t to) {
  cudaStream_t s = ctx->stream;
  cudaMemsetAsync(&ctx->status->maxold_bits, 0, sizeof(unsigned long long), s);
  if (to > from) {
    k_max_overlap<<<grid_for((long long)(to - from)), kBlock, 0, s>>>(ctx->cons.sd.p, (long long)from, (long long)to,
                                                                     &ctx->status->maxold_bits);
    ctx->launches++;
  }
  return cudaMemcpyAsync(ctx->pinned_ll + kSlotMaxOld, &ctx->status->maxold_bits, sizeof(unsigned long long),
                         cudaMemcpyDeviceToHost, s);
}

cudaError_t soft_assemble(pcc_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  const size_t m = ctx->ncons;
  if ((e = ctx->fel.reserve(m + 1, 0, s))) return e;
  if (m) {
    k_soft_fel<<<grid_for(m), kBlock, 0, s>>>(ctx->cons.view(), (long long)m, ctx->cells.diam.p, ctx->params.kcc,
                                              ctx->fel.p);
    ctx->launches++;
  }
  if (ctx->n) {
    k_soft_cell<<<grid_for((long long)ctx->n * kLanes), kBlock, 0, s>>>(
        ctx->cells.view(), (long long)ctx->n, ctx->cons.view(), ctx->inc_off.p, ctx->inc_ent.p, ctx->fel.p,
        ctx->params.xi, ctx->params.lambda, ctx->params.tau, 0.0, 0, nullptr);
    ctx->launches++;
  }
  return cudaGetLastError();
}

cudaError_t soft_forces_and_move(pcc_ctx* ctx, double dt) {
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  const size_t m = ctx->ncons;
  if ((e = ctx->fel.reserve(m + 1, 0, s))) return e;
  if (m) {
    k_soft_fel<<<grid_for(m), kBlock, 0, s>>>(ctx->cons.view(), (long long)m, ctx->cells.diam.p, ctx->params.kcc,
                                              ctx->fel.p);
    ctx->launches++;
  }
  if (ctx->n) {
    k_soft_cell<<<grid_for((long long)ctx->n * kLanes), kBlock, 0, s>>>(
        ctx->cells.view(), (long long)ctx->n, ctx->cons.view(), ctx->inc_off.p, ctx->inc_ent.p, ctx->fel.p,
        ctx->params.xi, ctx->params.lambda, ctx->params.tau, dt, 1, ctx->uext_active ? ctx->uext.p : nullptr);
    ctx->launches++;
  }
  return cudaGetLastError();
}

}  // namespace pcc
