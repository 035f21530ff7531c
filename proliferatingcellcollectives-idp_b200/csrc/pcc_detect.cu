// Broadphase + narrowphase contact detection (sm_100a).
//
// Replaces SpatialGrid::findPotentialCollisions (spatial/SpatialGrid.cpp:58-121)
// and CollisionDetector::tryCreateConstraint (spatial/CollisionDetector.cpp:201-311)
// of the reference.  Cells are binned on their centres exactly like the
// reference grid (origin -1, edge linked_cell_size, floor), so the candidate
// pairs -- every unordered pair in the same or an adjacent bin of the
// 27-stencil -- are the same set.  Binning is a counting sort: atomic counts,
// an exclusive scan, an atomic scatter and a per-bin sort by id, which makes
// the bin contents (and everything downstream) deterministic.  Each cell's
// geometry is packed once per phase in bin order so the neighbour scans read
// contiguous 32-byte groups.  The full pass scans the stencil once, counts
// the constraints and records each cell's partners within a wider reach in a
// candidate list; the emit pass and the later ReLCP phases of the same step
// walk those lists (with the reference's bin-adjacency test on the current
// bins and a displacement bound that proves no other pair can qualify).
// Counts are scanned into offsets, so constraints come out grouped by the
// smaller id in a fixed order, without atomics on the output.
#include <cmath>

#include "pcc_kernels.hpp"

namespace pcc {

namespace {

constexpr int kPack = 16;  // doubles per packed cell record
// record layout: [x y z len | sx sy sz diam | ex ey ez gid | tx ty tz ghost]
constexpr int kList = 32;  // candidate partners kept per cell
constexpr double kListReach = 0.25;  // list reach beyond contact: the first ReLCP phase's tolerance
enum : unsigned { kListOverflow = 1u, kListStale = 2u };

// Warp-wide max of a non-negative double folded into *dst (all lanes call).
__device__ __forceinline__ void warp_max_into(unsigned long long* dst, double v) {
  for (int o = 16; o > 0; o >>= 1) {
    const double u = __shfl_xor_sync(0xffffffffu, v, o);
    v = v < u ? u : v;
  }
  if ((threadIdx.x & 31) == 0 && v > 0.0) atomicMax(dst, (unsigned long long)__double_as_longlong(v));
}

// Bins every cell on its centre (origin -1, edge h, floor: the reference
// grid), decides its self-ghost, and folds the bin bounding box, the
// planarity flag, the longest cell and (when xref is given) the largest
// squared displacement since xref into the status, one atomic per warp.
__global__ void k_bin(CellsView c, size_t n, double h, int ghost_mode, const double* __restrict__ xref,
                      int* __restrict__ binxyz, int* __restrict__ bbox, int* __restrict__ ghost, DevStatus* st) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < n;
  int bx = 0, by = 0, bz = 0, nonplanar = 0;
  double len = 0.0, drift2 = 0.0;
  if (live) {
    const double x = c.x[i], y = c.y[i], z = c.z[i];
    bx = (int)floor(dvd(sub(x, -1.0), h));
    by = (int)floor(dvd(sub(y, -1.0), h));
    bz = (int)floor(dvd(sub(z, -1.0), h));
    binxyz[3 * i] = bx;
    binxyz[3 * i + 1] = by;
    binxyz[3 * i + 2] = bz;
    len = c.len[i];
    if (xref) {
      const double dx = x - xref[3 * i], dy = y - xref[3 * i + 1], dz = z - xref[3 * i + 2];
      drift2 = dx * dx + dy * dy + dz * dz;
    }
    // planar colony (z = 0, rotation about z only): the solver may use its 2D form
    nonplanar = (z != 0.0 || c.q1[i] != 0.0 || c.q2[i] != 0.0) ? 1 : 0;
    int g = 0;
    if (ghost_mode == PCC_GHOSTS_SINGLE_RANK) {
      // Domain::exchangeGhostParticles at world size 1 (spatial/Domain.cpp:339-403)
      // with calculateDistanceToAngularBoundary (263-290) for the sector [0, 360).
      double ang = dvd(mul(atan2(y, x), 180.0), M_PI);
      if (ang < 0) ang += 360.0;
      double radius = __dsqrt_rn(add(mul(x, x), mul(y, y)));
      if (radius >= 8.0) {
        double dmin = ang - 0.0, dmax = 360.0 - ang;
        while (dmin > 180.0) dmin -= 360.0;
        while (dmin < -180.0) dmin += 360.0;
        while (dmax > 180.0) dmax -= 360.0;
        while (dmax < -180.0) dmax += 360.0;
        double dist = 0.0;
        if (!(dmin >= 0 && dmax >= 0)) {
          double m = fabs(dmin) < fabs(dmax) ? fabs(dmin) : fabs(dmax);
          dist = mul(radius, sin(dvd(mul(m, M_PI), 180.0)));
        }
        g = dist < 2.5 ? 1 : 0;
      }
    }
    ghost[i] = g;
  }
  const unsigned full = 0xffffffffu;
  const int big = 2147483647, small = -2147483647 - 1;
  const int mnx = __reduce_min_sync(full, live ? bx : big), mny = __reduce_min_sync(full, live ? by : big),
            mnz = __reduce_min_sync(full, live ? bz : big);
  const int mxx = __reduce_max_sync(full, live ? bx : small), mxy = __reduce_max_sync(full, live ? by : small),
            mxz = __reduce_max_sync(full, live ? bz : small);
  const unsigned np = __reduce_or_sync(full, (unsigned)nonplanar);
  if ((threadIdx.x & 31) == 0 && mnx != big) {
    atomicMin(&bbox[0], mnx);
    atomicMin(&bbox[1], mny);
    atomicMin(&bbox[2], mnz);
    atomicMax(&bbox[3], mxx);
    atomicMax(&bbox[4], mxy);
    atomicMax(&bbox[5], mxz);
    if (np) atomicOr(&bbox[6], 1);
  }
  warp_max_into(&st->lmax_bits, len);
  if (xref) warp_max_into(&st->drift_bits, drift2);
}

struct Grid {
  int mx, my, mz, nx, ny, nz;
};

__device__ __forceinline__ Grid grid_from(const int* bbox) {
  Grid g;
  g.mx = bbox[0];
  g.my = bbox[1];
  g.mz = bbox[2];
  g.nx = bbox[3] - bbox[0] + 1;
  g.ny = bbox[4] - bbox[1] + 1;
  g.nz = bbox[5] - bbox[2] + 1;
  return g;
}

// Bin counts with warp-aggregated atomics: the lanes of a warp that fall in
// the same bin (cells are in x-sorted order, so neighbours often do) find
// each other with __match_any_sync and one of them adds the group's size.
__global__ void k_bin_count(const int* __restrict__ binxyz, size_t n, const int* __restrict__ bbox,
                            int* __restrict__ key, int* __restrict__ cnt) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < n;
  int k = -1;
  if (live) {
    const Grid g = grid_from(bbox);
    k = ((binxyz[3 * i + 2] - g.mz) * g.ny + (binxyz[3 * i + 1] - g.my)) * g.nx + (binxyz[3 * i] - g.mx);
    key[i] = k;
  }
  const unsigned peers = __match_any_sync(0xffffffffu, k);
  const int leader = __ffs(peers) - 1;
  if (live && (int)(threadIdx.x & 31) == leader) atomicAdd(&cnt[k], __popc(peers));
}

// Scatter into the bins: one atomic per group of same-bin lanes reserves the
// group's slots, each lane takes the slot of its rank in the group (the order
// inside a bin is fixed afterwards by k_segment_sort).
__global__ void k_bin_scatter(const int* __restrict__ key, size_t n, const int* __restrict__ off,
                              int* __restrict__ cursor, int* __restrict__ cells) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < n;
  const int k = live ? key[i] : -1;
  const unsigned peers = __match_any_sync(0xffffffffu, k);
  const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
  int base = 0;
  if (live && lane == leader) base = atomicAdd(&cursor[k], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  if (live) cells[off[k] + base + __popc(peers & ((1u << lane) - 1u))] = (int)i;
}

// Sort each segment [off[s], off[s+1]) ascending (segments are short).
__global__ void k_segment_sort(const int* __restrict__ off, size_t nseg, int* __restrict__ v) {
  size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  int b = off[s], e = off[s + 1];
  for (int i = b + 1; i < e; ++i) {
    int x = v[i];
    int j = i - 1;
    while (j >= b && v[j] > x) {
      v[j + 1] = v[j];
      --j;
    }
    v[j + 1] = x;
  }
}

__global__ void k_pack(CellsView c, const int* __restrict__ slot_cell, const int* __restrict__ ghost, size_t n,
                       double* __restrict__ pk) {
  size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int i = slot_cell[s];
  double t[3];
  cell_axis(c.q0[i], c.q1[i], c.q2[i], c.q3[i], t);
  const double len = c.len[i], diam = c.diam[i];
  // CollisionDetector::getParticleEndpoints (spatial/CollisionDetector.cpp:61-75)
  const double half = sub(dvd(len, 2.0), dvd(diam, 2.0));
  const double p[3] = {c.x[i], c.y[i], c.z[i]};
  double* r = pk + s * kPack;
  r[0] = p[0];
  r[1] = p[1];
  r[2] = p[2];
  r[3] = len;
  for (int d = 0; d < 3; ++d) {
    double hv = mul(t[d], half);
    r[4 + d] = sub(p[d], hv);
    r[8 + d] = add(p[d], hv);
    r[12 + d] = t[d];
  }
  r[7] = diam;
  r[11] = (double)i;
  r[15] = (double)ghost[i];
}

// Closest points of two segments: Eberly's branch scheme for segment-segment
// distance (the variant the reference uses, util/SpherocylinderCell.h:64-261),
// restated with non-contracting IEEE operations.
__device__ void segment_closest(const double P0[3], const double P1[3], const double Q0[3], const double Q1[3],
                                double c0[3], double c1[3], double* dist) {
  double Pd[3], Qd[3], PQ[3];
  for (int k = 0; k < 3; ++k) {
    Pd[k] = sub(P1[k], P0[k]);
    Qd[k] = sub(Q1[k], Q0[k]);
    PQ[k] = sub(P0[k], Q0[k]);
  }
  const double a = dot3(Pd, Pd), b = dot3(Pd, Qd), c = dot3(Qd, Qd);
  const double d = dot3(Pd, PQ), e = dot3(Qd, PQ);
  const double det = sub(mul(a, c), mul(b, b));
  double s = 0.0, t = 0.0;
  if (det > 0.0) {
    const double bte = mul(b, e), ctd = mul(c, d);
    if (bte <= ctd) {
      s = 0.0;
      if (e <= 0.0) {
        t = 0.0;
        double nd = -d;
        if (nd >= a) s = 1.0;
        else if (nd > 0.0) s = dvd(nd, a);
      } else if (e < c) {
        t = dvd(e, c);
      } else {
        t = 1.0;
        double bmd = sub(b, d);
        if (bmd >= a) s = 1.0;
        else if (bmd > 0.0) s = dvd(bmd, a);
      }
    } else {
      s = sub(bte, ctd);
      if (s >= det) {
        s = 1.0;
        double bpe = add(b, e);
        if (bpe <= 0.0) {
          t = 0.0;
          double nd = -d;
          if (nd <= 0.0) s = 0.0;
          else if (nd < a) s = dvd(nd, a);
        } else if (bpe < c) {
          t = dvd(bpe, c);
        } else {
          t = 1.0;
          double bmd = sub(b, d);
          if (bmd <= 0.0) s = 0.0;
          else if (bmd < a) s = dvd(bmd, a);
        }
      } else {
        const double ate = mul(a, e), btd = mul(b, d);
        if (ate <= btd) {
          t = 0.0;
          double nd = -d;
          if (nd <= 0.0) s = 0.0;
          else if (nd >= a) s = 1.0;
          else s = dvd(nd, a);
        } else {
          t = sub(ate, btd);
          if (t >= det) {
            t = 1.0;
            double bmd = sub(b, d);
            if (bmd <= 0.0) s = 0.0;
            else if (bmd >= a) s = 1.0;
            else s = dvd(bmd, a);
          } else {
            s = dvd(s, det);
            t = dvd(t, det);
          }
        }
      }
    }
  } else {
    if (e <= 0.0) {
      t = 0.0;
      double nd = -d;
      if (nd <= 0.0) s = 0.0;
      else if (nd >= a) s = 1.0;
      else s = dvd(nd, a);
    } else if (e >= c) {
      t = 1.0;
      double bmd = sub(b, d);
      if (bmd <= 0.0) s = 0.0;
      else if (bmd >= a) s = 1.0;
      else s = dvd(bmd, a);
    } else {
      s = 0.0;
      t = dvd(e, c);
    }
  }
  double diff[3];
  for (int k = 0; k < 3; ++k) {
    c0[k] = add(P0[k], mul(Pd[k], s));
    c1[k] = add(Q0[k], mul(Qd[k], t));
    diff[k] = sub(c0[k], c1[k]);
  }
  *dist = __dsqrt_rn(dot3(diff, diff));
}


struct PairGeom {
  double sd, n[3], cp[3], ri[3], rj[3], si, sj;
};

// The centre-distance prefilter of tryCreateConstraint
// (spatial/CollisionDetector.cpp:210-213): the pair is dropped when
// sqrt(|x_a - x_b|^2) > (l_a + l_b)/2 + tol.  sqrt is correctly rounded and
// monotone, so away from the boundary the squared distance decides; within a
// relative 1e-9 of it the exact test runs.  (l_a + l_b) * 0.5 equals
// (l_a + l_b) / 2 exactly.
__device__ __forceinline__ bool rough_pass(const double4& a0, const double4& b0, double tol) {
  const double dv[3] = {sub(a0.x, b0.x), sub(a0.y, b0.y), sub(a0.z, b0.z)};
  const double d2 = dot3(dv, dv);
  const double reach = add(mul(add(a0.w, b0.w), 0.5), tol);
  const double r2 = reach * reach;
  if (d2 > r2 * (1.0 + 1e-9)) return false;
  if (d2 < r2 * (1.0 - 1e-9)) return true;
  return !(__dsqrt_rn(d2) > reach);
}

// The rest of tryCreateConstraint for a pair (I, J) = (A, B) that passed the
// prefilter.  With full == false only the separation is computed.
__device__ __forceinline__ bool pair_geom(const double* __restrict__ A, const double* __restrict__ B, double tol,
                                          bool full, PairGeom* o) {
  const double4 a1 = *reinterpret_cast<const double4*>(A + 4);
  const double4 a2 = *reinterpret_cast<const double4*>(A + 8);
  const double4 b1 = *reinterpret_cast<const double4*>(B + 4);
  const double4 b2 = *reinterpret_cast<const double4*>(B + 8);
  const double P0[3] = {a1.x, a1.y, a1.z}, P1[3] = {a2.x, a2.y, a2.z};
  const double Q0[3] = {b1.x, b1.y, b1.z}, Q1[3] = {b2.x, b2.y, b2.z};
  double c0[3], c1[3], dist;
  segment_closest(P0, P1, Q0, Q1, c0, c1, &dist);
  const double sd = sub(dist, dvd(add(a1.w, b1.w), 2.0));
  if (sd > tol) return false;
  o->sd = sd;
  if (!full) return true;
  double diff[3];
  for (int k = 0; k < 3; ++k) {
    o->cp[k] = mul(add(c0[k], c1[k]), 0.5);
    diff[k] = sub(c0[k], c1[k]);
  }
  // ArrayMath::normalize (util/ArrayMath.h:219-231)
  const double mag = __dsqrt_rn(dot3(diff, diff));
  if (mag > 2.220446049250313e-16) {
    const double inv = dvd(1.0, mag);
    for (int k = 0; k < 3; ++k) o->n[k] = mul(diff[k], inv);
  } else {
    o->n[0] = 1.0;
    o->n[1] = 0.0;
    o->n[2] = 0.0;
  }
  const double4 a0 = *reinterpret_cast<const double4*>(A);
  const double4 b0 = *reinterpret_cast<const double4*>(B);
  const double4 a3 = *reinterpret_cast<const double4*>(A + 12);
  const double4 b3 = *reinterpret_cast<const double4*>(B + 12);
  const double ta[3] = {a3.x, a3.y, a3.z}, tb[3] = {b3.x, b3.y, b3.z};
  const double nn[3] = {-o->n[0], -o->n[1], -o->n[2]};
  o->si = mul(0.5, fabs(dot3(o->n, ta)));
  o->sj = mul(0.5, fabs(dot3(nn, tb)));
  const double pa[3] = {a0.x, a0.y, a0.z}, pb[3] = {b0.x, b0.y, b0.z};
  for (int k = 0; k < 3; ++k) {
    o->ri[k] = sub(o->cp[k], pa[k]);
    o->rj[k] = sub(o->cp[k], pb[k]);
  }
  return true;
}

// Writes `copies` identical constraint rows for the pair (a, b) from row w on
// (a second copy stands for the partner's self-ghost).  Returns false when the
// rows would pass `cap`.
__device__ __forceinline__ bool emit_rows(ConsView cs, size_t& w, size_t cap, int a, int b, int phase, int copies,
                                          const PairGeom& pg, DevStatus* st) {
  double ti[3], tj[3];
  const double nj[3] = {-pg.n[0], -pg.n[1], -pg.n[2]};
  cross3(pg.ri, pg.n, ti);
  cross3(pg.rj, nj, tj);
  for (int k = 0; k < copies; ++k, ++w) {
    if (w >= cap) {
      raise_error(st, kDevErrCapacity, 10);
      return false;
    }
    cs.gi[w] = a;
    cs.gj[w] = b;
    cs.phase[w] = phase;
    cs.sd[w] = pg.sd;
    cs.gamma[w] = pg.sd >= 0.0 ? 0.0 : mul(-pg.sd, 5e2);
    cs.nx[w] = pg.n[0];
    cs.ny[w] = pg.n[1];
    cs.nz[w] = pg.n[2];
    cs.tix[w] = ti[0];
    cs.tiy[w] = ti[1];
    cs.tiz[w] = ti[2];
    cs.tjx[w] = tj[0];
    cs.tjy[w] = tj[1];
    cs.tjz[w] = tj[2];
    cs.rix[w] = pg.ri[0];
    cs.riy[w] = pg.ri[1];
    cs.riz[w] = pg.ri[2];
    cs.rjx[w] = pg.rj[0];
    cs.rjy[w] = pg.rj[1];
    cs.rjz[w] = pg.rj[2];
    cs.cpx[w] = pg.cp[0];
    cs.cpy[w] = pg.cp[1];
    cs.cpz[w] = pg.cp[2];
    cs.si[w] = pg.si;
    cs.sj[w] = pg.sj;
  }
  return true;
}

// Bin of the cell at slot s: the last bin whose offset is <= s.
__device__ __forceinline__ int bin_of_slot(const int* __restrict__ bin_off, int nbins, int s) {
  int lo = 0, hi = nbins;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (bin_off[mid] <= s) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Full neighbourhood pass of a phase: one thread per cell in bin order scans
// the 27-stencil for partners with a larger id (the candidate pairs of
// SpatialGrid::findPotentialCollisions, spatial/SpatialGrid.cpp:58-121).  For
// each pair that passes tryCreateConstraint it counts the constraints the
// smaller id emits (a second copy when the partner has a self-ghost), tracks
// the largest overlap, and adds to Particle::num_constraints of both cells
// (CollisionDetector.cpp:243-244, ghost copies included; the count of a cell
// that has a self-ghost lands on the copy and is lost, as in the reference).
// Every partner within the wider reach tol_list is appended to the cell's
// candidate list (slots of the packed records, stored list-major), so the
// emit pass and the later ReLCP phases of the step need no stencil scan.
// The cell's position at list time is kept in xref.
__global__ void k_scan_count(const double* __restrict__ pk, const int* __restrict__ bin_off,
                             const int* __restrict__ bbox, size_t n, double tol, double tol_list,
                             int* __restrict__ cnt, int* __restrict__ ncontacts, int* __restrict__ plist,
                             int* __restrict__ plist_n, double* __restrict__ xref, DevStatus* st) {
  const size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double maxov = 0.0;
  if (s < n) {
    const Grid g = grid_from(bbox);
    const double* A = pk + s * kPack;
    const int a = (int)A[11];
    const double4 a0 = *reinterpret_cast<const double4*>(A);
    xref[3 * (size_t)a] = a0.x;
    xref[3 * (size_t)a + 1] = a0.y;
    xref[3 * (size_t)a + 2] = a0.z;
    const int bin = bin_of_slot(bin_off, g.nx * g.ny * g.nz, (int)s);
    const int bx = bin % g.nx, by = (bin / g.nx) % g.ny, bz = bin / (g.nx * g.ny);
    const int ga = A[15] != 0.0;
    int count = 0, nl = 0;
    for (int dz = -1; dz <= 1; ++dz) {
      const int z = bz + dz;
      if (z < 0 || z >= g.nz) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int y = by + dy;
        if (y < 0 || y >= g.ny) continue;
        // the (up to) three bins of a stencil row hold consecutive slots
        const int x0 = bx > 0 ? bx - 1 : 0, x1 = bx + 1 < g.nx ? bx + 1 : g.nx - 1;
        const int row = (z * g.ny + y) * g.nx;
        const int e = bin_off[row + x1 + 1];
        for (int s2 = bin_off[row + x0]; s2 < e; ++s2) {
          const double* B = pk + (size_t)s2 * kPack;
          const int b = (int)B[11];
          if (b <= a) continue;
          const double4 b0 = *reinterpret_cast<const double4*>(B);
          if (!rough_pass(a0, b0, tol_list)) continue;
          if (nl < kList) plist[(size_t)nl * n + a] = s2;
          ++nl;
          if (tol < tol_list && !rough_pass(a0, b0, tol)) continue;
          PairGeom pg;
          if (!pair_geom(A, B, tol, false, &pg)) continue;
          const int gb = B[15] != 0.0;
          count += 1 + gb;
          const double ov = pg.sd < 0 ? -pg.sd : 0.0;
          maxov = maxov < ov ? ov : maxov;
          if (!ga) atomicAdd(&ncontacts[a], 1 + gb);
          if (!gb) atomicAdd(&ncontacts[b], 1 + ga);
        }
      }
    }
    cnt[a] = count;
    plist_n[a] = nl;
    if (nl > kList) atomicOr(&st->list_flags, kListOverflow);
  }
  warp_max_into(&st->max_bits, maxov);
}

// Count (kEmit = false) or emit pass over the candidate lists, one thread per
// cell in id order; the emit order per cell is the list order, which is the
// stencil order of the full pass.
//
// In a later ReLCP phase of the step (adjacent = true) the lists are reused
// without rebinning the colony.  A listed pair is a candidate only if the two
// cells' current bins are neighbours, which is the reference's test.  A pair
// that is not listed cannot be a candidate that passes: with D the largest
// displacement of any cell since the lists were built and L the longest cell,
// a pair within (l_a + l_b)/2 + tol now was within (l_a + l_b)/2 + tol + 2D
// then, which is inside the list reach when tol + 2D < tol_list, and closer
// than one bin edge h (so in neighbouring bins) when L + tol + 2D < h.  If
// either bound fails the pass does nothing and flags the lists stale; the
// caller then runs the full pass.
template <bool kEmit>
__global__ void k_list_pass(const double* __restrict__ pk, const int* __restrict__ slot_of, size_t n, double tol,
                            int phase, bool adjacent, double tol_list, double h, const int* __restrict__ binxyz,
                            const int* __restrict__ plist, const int* __restrict__ plist_n, int* __restrict__ cnt,
                            int* __restrict__ ncontacts, const int* __restrict__ off, ConsView cs, size_t base,
                            size_t cap, DevStatus* st) {
  const size_t a = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (!kEmit && adjacent) {
    const double d2 = __longlong_as_double((long long)__ldcg(&st->drift_bits));
    const double lmax = __longlong_as_double((long long)__ldcg(&st->lmax_bits));
    const double reach = tol + 2.0 * sqrt(d2);
    if (!(reach < tol_list - 1e-6 && lmax + reach < h - 1e-6)) {
      if (a == 0) atomicOr(&st->list_flags, kListStale);
      return;
    }
  }
  double maxov = 0.0;
  if (a < n) {
    const double* A = pk + (size_t)slot_of[a] * kPack;
    const double4 a0 = *reinterpret_cast<const double4*>(A);
    const int ga = A[15] != 0.0;
    const int nl = min(plist_n[a], kList);  // lists in use never overflowed
    int bxa = 0, bya = 0, bza = 0;
    if (adjacent) {
      bxa = binxyz[3 * a];
      bya = binxyz[3 * a + 1];
      bza = binxyz[3 * a + 2];
    }
    int count = 0;
    size_t w = kEmit ? base + (size_t)off[a] : 0;
    for (int k = 0; k < nl; ++k) {
      const int s2 = plist[(size_t)k * n + a];
      const double* B = pk + (size_t)s2 * kPack;
      const int b = (int)B[11];
      if (adjacent) {
        const int ex = binxyz[3 * (size_t)b] - bxa, ey = binxyz[3 * (size_t)b + 1] - bya,
                  ez = binxyz[3 * (size_t)b + 2] - bza;
        if (ex < -1 || ex > 1 || ey < -1 || ey > 1 || ez < -1 || ez > 1) continue;
      }
      const double4 b0 = *reinterpret_cast<const double4*>(B);
      if (!rough_pass(a0, b0, tol)) continue;
      PairGeom pg;
      if (!pair_geom(A, B, tol, kEmit, &pg)) continue;
      const int gb = B[15] != 0.0;
      if (kEmit) {
        if (!emit_rows(cs, w, cap, (int)a, b, phase, 1 + gb, pg, st)) break;
      } else {
        count += 1 + gb;
        const double ov = pg.sd < 0 ? -pg.sd : 0.0;
        maxov = maxov < ov ? ov : maxov;
        if (!ga) atomicAdd(&ncontacts[a], 1 + gb);
        if (!gb) atomicAdd(&ncontacts[b], 1 + ga);
      }
    }
    if (!kEmit) cnt[a] = count;
  }
  if (!kEmit) warp_max_into(&st->max_bits, maxov);
}

// Emit pass over the 27-stencil, for a phase whose candidate lists overflowed.
__global__ void k_stencil_emit(const double* __restrict__ pk, const int* __restrict__ bin_off,
                               const int* __restrict__ bbox, size_t n, double tol, int phase,
                               const int* __restrict__ off, ConsView cs, size_t base, size_t cap, DevStatus* st) {
  const size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const Grid g = grid_from(bbox);
  const double* A = pk + s * kPack;
  const int a = (int)A[11];
  const double4 a0 = *reinterpret_cast<const double4*>(A);
  const int bin = bin_of_slot(bin_off, g.nx * g.ny * g.nz, (int)s);
  const int bx = bin % g.nx, by = (bin / g.nx) % g.ny, bz = bin / (g.nx * g.ny);
  size_t w = base + (size_t)off[a];
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = bz + dz;
    if (z < 0 || z >= g.nz) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int y = by + dy;
      if (y < 0 || y >= g.ny) continue;
      const int x0 = bx > 0 ? bx - 1 : 0, x1 = bx + 1 < g.nx ? bx + 1 : g.nx - 1;
      const int row = (z * g.ny + y) * g.nx;
      const int e = bin_off[row + x1 + 1];
      for (int s2 = bin_off[row + x0]; s2 < e; ++s2) {
        const double* B = pk + (size_t)s2 * kPack;
        const int b = (int)B[11];
        if (b <= a) continue;
        const double4 b0 = *reinterpret_cast<const double4*>(B);
        if (!rough_pass(a0, b0, tol)) continue;
        PairGeom pg;
        if (!pair_geom(A, B, tol, true, &pg)) continue;
        if (!emit_rows(cs, w, cap, a, b, phase, 1 + (B[15] != 0.0 ? 1 : 0), pg, st)) return;
      }
    }
  }
}

__global__ void k_slot_of(const int* __restrict__ slot_cell, size_t n, int* __restrict__ slot_of) {
  const size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) slot_of[slot_cell[s]] = (int)s;
}

__global__ void k_inc_count(const int* __restrict__ gi, const int* __restrict__ gj, size_t m, int* __restrict__ cnt) {
  size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m) return;
  atomicAdd(&cnt[gi[c]], 1);
  atomicAdd(&cnt[gj[c]], 1);
}

__global__ void k_inc_fill(const int* __restrict__ gi, const int* __restrict__ gj, size_t m,
                           const int* __restrict__ off, int* __restrict__ cursor, int* __restrict__ ent) {
  size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m) return;
  int a = gi[c], b = gj[c];
  ent[off[a] + atomicAdd(&cursor[a], 1)] = (int)(2 * c);
  ent[off[b] + atomicAdd(&cursor[b], 1)] = (int)(2 * c + 1);
}

}  // namespace

cudaError_t detect_contacts(pcc_ctx* ctx, double tol, int phase, bool reuse, size_t* added,
                            double* max_overlap_new) {
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->n;
  cudaError_t e;
  *added = 0;
  *max_overlap_new = 0.0;
  if (!reuse) ctx->list_valid = false;
  if (n == 0) return cudaSuccess;
  int* pinned = reinterpret_cast<int*>(ctx->pinned_ll);
  static const int init[7] = {2147483647, 2147483647, 2147483647, -2147483647 - 1, -2147483647 - 1,
                              -2147483647 - 1, 0};
  const double h = ctx->params.linked_cell_size;
  const double tol_list = tol > kListReach ? tol : kListReach;
  bool use_list = reuse && ctx->list_valid && ctx->list_n == n;
  if ((e = ctx->bin_of.reserve(3 * n, 0, s))) return e;
  if ((e = ctx->ghost.reserve(n, 0, s))) return e;
  if ((e = ctx->bbox.reserve(8, 0, s))) return e;
  if ((e = ctx->cand_cnt.reserve(n + 1, 0, s))) return e;
  if ((e = ctx->cand_off.reserve(n + 1, 0, s))) return e;
  if ((e = ctx->pk.reserve(n * kPack, 0, s))) return e;
  if ((e = ctx->plist.reserve(n * kList, 0, s))) return e;
  if ((e = ctx->plist_n.reserve(n + 1, 0, s))) return e;
  if ((e = ctx->slot_of.reserve(n + 1, 0, s))) return e;
  if ((e = ctx->xref.reserve(3 * n, 0, s))) return e;
  for (;;) {
    cudaMemcpyAsync(ctx->bbox.p, init, sizeof init, cudaMemcpyHostToDevice, s);  // pageable: staged at once
    cudaMemsetAsync(&ctx->status->max_bits, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(&ctx->status->list_flags, 0, 3 * sizeof(unsigned long long), s);
    k_bin<<<grid_for(n), kBlock, 0, s>>>(ctx->cells.view(), n, h, ctx->params.ghost_mode,
                                          use_list ? ctx->xref.p : nullptr, ctx->bin_of.p, ctx->bbox.p, ctx->ghost.p,
                                          ctx->status);
    ctx->launches++;
    if (use_list) {
      // the slots of the pass that built the lists: bin_cells still maps slot -> cell
      k_pack<<<grid_for(n), kBlock, 0, s>>>(ctx->cells.view(), ctx->bin_cells.p, ctx->ghost.p, n, ctx->pk.p);
      k_list_pass<false><<<grid_for(n), kBlock, 0, s>>>(
          ctx->pk.p, ctx->slot_of.p, n, tol, phase, true, ctx->list_tol, h, ctx->bin_of.p, ctx->plist.p,
          ctx->plist_n.p, ctx->cand_cnt.p, ctx->cells.ncons.p, nullptr, ConsView{}, 0, 0, ctx->status);
      ctx->launches += 2;
    } else {
      cudaMemcpyAsync(pinned, ctx->bbox.p, 7 * sizeof(int), cudaMemcpyDeviceToHost, s);
      if ((e = cudaStreamSynchronize(s))) return e;
      ctx->planar = pinned[6] == 0;
      const long long nx = (long long)pinned[3] - pinned[0] + 1, ny = (long long)pinned[4] - pinned[1] + 1,
                      nz = (long long)pinned[5] - pinned[2] + 1;
      const long long nbins = nx * ny * nz;
      if (nbins <= 0 || nbins > (1LL << 30)) {
        ctx->err = "broadphase grid too large (cells spread over more than 2^30 bins)";
        return cudaErrorInvalidValue;
      }
      if ((e = ctx->bin_cnt.reserve(nbins + 1, 0, s))) return e;
      if ((e = ctx->bin_cursor.reserve(nbins + 1, 0, s))) return e;
      if ((e = ctx->bin_off.reserve(nbins + 1, 0, s))) return e;
      if ((e = ctx->bin_cells.reserve(n, 0, s))) return e;
      int* key = ctx->cand_cnt.p;  // per-cell bin key until the pair pass
      cudaMemsetAsync(ctx->bin_cnt.p, 0, (nbins + 1) * sizeof(int), s);
      cudaMemsetAsync(ctx->bin_cursor.p, 0, (nbins + 1) * sizeof(int), s);
      k_bin_count<<<grid_for(n), kBlock, 0, s>>>(ctx->bin_of.p, n, ctx->bbox.p, key, ctx->bin_cnt.p);
      if ((e = exclusive_scan(ctx, ctx->bin_cnt.p, ctx->bin_off.p, (size_t)nbins))) return e;
      k_bin_scatter<<<grid_for(n), kBlock, 0, s>>>(key, n, ctx->bin_off.p, ctx->bin_cursor.p, ctx->bin_cells.p);
      k_segment_sort<<<grid_for(nbins), kBlock, 0, s>>>(ctx->bin_off.p, (size_t)nbins, ctx->bin_cells.p);
      k_pack<<<grid_for(n), kBlock, 0, s>>>(ctx->cells.view(), ctx->bin_cells.p, ctx->ghost.p, n, ctx->pk.p);
      k_slot_of<<<grid_for(n), kBlock, 0, s>>>(ctx->bin_cells.p, n, ctx->slot_of.p);
      k_scan_count<<<grid_for(n), kBlock, 0, s>>>(ctx->pk.p, ctx->bin_off.p, ctx->bbox.p, n, tol, tol_list,
                                                   ctx->cand_cnt.p, ctx->cells.ncons.p, ctx->plist.p,
                                                   ctx->plist_n.p, ctx->xref.p, ctx->status);
      ctx->launches += 6;
    }
    if ((e = exclusive_scan(ctx, ctx->cand_cnt.p, ctx->cand_off.p, n))) return e;
    cudaMemcpyAsync(pinned, ctx->cand_off.p + n, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(ctx->pinned_ll + 1, &ctx->status->max_bits, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                    s);
    cudaMemcpyAsync(pinned + 4, &ctx->status->list_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    // k_bin folds the planarity of the current cells on every pass: cells
    // that left the plane since the last full pass (out-of-plane Brownian
    // kicks) must take the general solver
    cudaMemcpyAsync(pinned + 5, ctx->bbox.p + 6, sizeof(int), cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s))) return e;
    ctx->planar = pinned[5] == 0;
    const unsigned flags = (unsigned)pinned[4];
    if (use_list && (flags & kListStale)) {
      // cells moved too far since the lists were built: rebin this phase
      use_list = false;
      ctx->list_valid = false;
      continue;
    }
    const bool listed = use_list || (flags & kListOverflow) == 0;
    if (use_list) ctx->prof.detect_list_passes++;
    else ctx->prof.detect_full_passes++;
    if (!use_list) {
      ctx->list_valid = listed;
      ctx->list_n = n;
      ctx->list_tol = tol_list;
    }
    const size_t m = (size_t)pinned[0];
    unsigned long long bits = (unsigned long long)ctx->pinned_ll[1];
    double mo;
    memcpy(&mo, &bits, sizeof mo);
    *max_overlap_new = mo;
    *added = m;
    if (m == 0) return cudaSuccess;
    if ((e = ctx->cons.reserve(ctx->ncons + m, ctx->ncons, s))) return e;
    if (listed) {
      k_list_pass<true><<<grid_for(n), kBlock, 0, s>>>(ctx->pk.p, ctx->slot_of.p, n, tol, phase, use_list, tol_list,
                                                      h, ctx->bin_of.p, ctx->plist.p, ctx->plist_n.p, nullptr,
                                                      nullptr, ctx->cand_off.p, ctx->cons.view(), ctx->ncons,
                                                      ctx->ncons + m, ctx->status);
    } else {
      k_stencil_emit<<<grid_for(n), kBlock, 0, s>>>(ctx->pk.p, ctx->bin_off.p, ctx->bbox.p, n, tol, phase,
                                                    ctx->cand_off.p, ctx->cons.view(), ctx->ncons, ctx->ncons + m,
                                                    ctx->status);
    }
    ctx->launches++;
    ctx->ncons += m;
    return cudaGetLastError();
  }
}

cudaError_t build_incidence(pcc_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->n, m = ctx->ncons;
  cudaError_t e;
  if ((e = ctx->inc_cnt.reserve(n + 1, 0, s))) return e;
  if ((e = ctx->inc_off.reserve(n + 1, 0, s))) return e;
  if ((e = ctx->inc_ent.reserve(2 * m + 1, 0, s))) return e;
  if ((e = ctx->bin_cursor.reserve(n + 1, 0, s))) return e;
  cudaMemsetAsync(ctx->inc_cnt.p, 0, (n + 1) * sizeof(int), s);
  cudaMemsetAsync(ctx->bin_cursor.p, 0, (n + 1) * sizeof(int), s);
  if (m) {
    k_inc_count<<<grid_for(m), kBlock, 0, s>>>(ctx->cons.gi.p, ctx->cons.gj.p, m, ctx->inc_cnt.p);
    ctx->launches++;
  }
  if ((e = exclusive_scan(ctx, ctx->inc_cnt.p, ctx->inc_off.p, n))) return e;
  if (m) {
    k_inc_fill<<<grid_for(m), kBlock, 0, s>>>(ctx->cons.gi.p, ctx->cons.gj.p, m, ctx->inc_off.p, ctx->bin_cursor.p,
                                              ctx->inc_ent.p);
    k_segment_sort<<<grid_for(n), kBlock, 0, s>>>(ctx->inc_off.p, n, ctx->inc_ent.p);
    ctx->launches += 2;
  }
  return cudaGetLastError();
}

}  // namespace pcc
