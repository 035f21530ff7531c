/*
 * Plain-C restatement of the reference's collision hot path at one rank (the
 * CPU oracle).  TEST INFRASTRUCTURE ONLY: the product library never links or
 * calls this file.
 *
 * Citations are file:line inside code/cpp/src of the reference project.
 * Build strict (-O2 -ffp-contract=off, no fast-math): every expression keeps
 * the reference's operation order, and the sparse products follow PETSc's
 * sequential AIJ kernels (row sums in ascending column order from 0.0;
 * transpose products scatter row by row).
 */
#define _GNU_SOURCE
#include "pcc_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int gi, gj;
  double sd;
  double n[3], ri[3], rj[3], cp[3];
  double si, sj, gamma;
  int phase;
} cons_t;

typedef struct {
  double x[3];
  double q[4];
  double len, l0, diam, ldot, imp, stress;
  int age;
  int nc; /* Particle::num_constraints_ */
  double force[6], vel[6];
} cell_t;

struct pcco_colony {
  pcc_params p;
  cell_t* cells;
  size_t n, cap;
  cons_t* cons; /* constraint set of the last solve */
  size_t ncons, capcons;
  unsigned long long div_index;
  size_t iter;
  double sim_time, radius;
  char err[256];
};

/* ------------------------------------------------------------------ vectors */
static void* xrealloc(void* p, size_t bytes) {
  void* q = realloc(p, bytes ? bytes : 1);
  if (!q) {
    fprintf(stderr, "pcc_oracle: out of memory\n");
    abort();
  }
  return q;
}

/* utils::Quaternion::rotateVectorOfPositions with v = (1,0,0) (util/Quaternion.cpp:7-38) */
static void direction(const double q[4], double t[3]) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  const double vx = 1.0, vy = 0.0, vz = 0.0;
  const double c1x = y * vz - z * vy, c1y = z * vx - x * vz, c1z = x * vy - y * vx;
  const double c2x = y * c1z - z * c1y, c2y = z * c1x - x * c1z, c2z = x * c1y - y * c1x;
  t[0] = vx + 2.0 * w * c1x + 2.0 * c2x;
  t[1] = vy + 2.0 * w * c1y + 2.0 * c2y;
  t[2] = vz + 2.0 * w * c1z + 2.0 * c2z;
}

static double dot3(const double a[3], const double b[3]) {
  double r = 0;
  for (int d = 0; d < 3; ++d) r += a[d] * b[d];
  return r;
}

/* ArrayMath::normalize (util/ArrayMath.h:219-231) */
static void normalize3(const double a[3], double out[3]) {
  double mag = sqrt(dot3(a, a));
  if (mag > DBL_EPSILON) {
    double inv = 1.0 / mag;
    for (int d = 0; d < 3; ++d) out[d] = a[d] * inv;
  } else {
    out[0] = 1.0;
    out[1] = 0.0;
    out[2] = 0.0;
  }
}

static void cross3(const double a[3], const double b[3], double r[3]) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}

/* CollisionDetector::getParticleEndpoints (spatial/CollisionDetector.cpp:61-75) */
static void endpoints(const cell_t* c, double s[3], double e[3]) {
  double t[3];
  direction(c->q, t);
  double half = c->len / 2 - c->diam / 2;
  for (int d = 0; d < 3; ++d) {
    double hv = t[d] * half;
    s[d] = c->x[d] - hv;
    e[d] = c->x[d] + hv;
  }
}

/* Closest points of two segments, Eberly's non-robust branch scheme
 * ("Distance between two line segments", Geometric Tools; the variant the
 * reference calls, util/SpherocylinderCell.h:64-261). */
static void segment_closest(const double P0[3], const double P1[3], const double Q0[3], const double Q1[3],
                            double c0[3], double c1[3], double* dist) {
  double Pd[3], Qd[3], PQ[3];
  for (int d = 0; d < 3; ++d) {
    Pd[d] = P1[d] - P0[d];
    Qd[d] = Q1[d] - Q0[d];
    PQ[d] = P0[d] - Q0[d];
  }
  const double a = dot3(Pd, Pd), b = dot3(Pd, Qd), c = dot3(Qd, Qd);
  const double d = dot3(Pd, PQ), e = dot3(Qd, PQ);
  const double det = a * c - b * b;
  double s = 0.0, t = 0.0;
  if (det > 0.0) {
    const double bte = b * e, ctd = c * d;
    if (bte <= ctd) { /* s <= 0 */
      s = 0.0;
      if (e <= 0.0) {
        t = 0.0;
        double nd = -d;
        if (nd >= a) s = 1.0;
        else if (nd > 0.0) s = nd / a;
      } else if (e < c) {
        t = e / c;
      } else {
        t = 1.0;
        double bmd = b - d;
        if (bmd >= a) s = 1.0;
        else if (bmd > 0.0) s = bmd / a;
      }
    } else {
      s = bte - ctd;
      if (s >= det) { /* s >= 1 */
        s = 1.0;
        double bpe = b + e;
        if (bpe <= 0.0) {
          t = 0.0;
          double nd = -d;
          if (nd <= 0.0) s = 0.0;
          else if (nd < a) s = nd / a;
        } else if (bpe < c) {
          t = bpe / c;
        } else {
          t = 1.0;
          double bmd = b - d;
          if (bmd <= 0.0) s = 0.0;
          else if (bmd < a) s = bmd / a;
        }
      } else { /* 0 < s < 1 */
        const double ate = a * e, btd = b * d;
        if (ate <= btd) {
          t = 0.0;
          double nd = -d;
          if (nd <= 0.0) s = 0.0;
          else if (nd >= a) s = 1.0;
          else s = nd / a;
        } else {
          t = ate - btd;
          if (t >= det) {
            t = 1.0;
            double bmd = b - d;
            if (bmd <= 0.0) s = 0.0;
            else if (bmd >= a) s = 1.0;
            else s = bmd / a;
          } else {
            s /= det;
            t /= det;
          }
        }
      }
    }
  } else { /* parallel */
    if (e <= 0.0) {
      t = 0.0;
      double nd = -d;
      if (nd <= 0.0) s = 0.0;
      else if (nd >= a) s = 1.0;
      else s = nd / a;
    } else if (e >= c) {
      t = 1.0;
      double bmd = b - d;
      if (bmd <= 0.0) s = 0.0;
      else if (bmd >= a) s = 1.0;
      else s = bmd / a;
    } else {
      s = 0.0;
      t = e / c;
    }
  }
  double diff[3];
  for (int k = 0; k < 3; ++k) {
    c0[k] = P0[k] + Pd[k] * s;
    c1[k] = Q0[k] + Qd[k] * t;
    diff[k] = c0[k] - c1[k];
  }
  *dist = sqrt(dot3(diff, diff));
}

/* ------------------------------------------------------------------ ghosts */
/* calculateDistanceToAngularBoundary (spatial/Domain.cpp:263-290) */
static double norm_angle(double a) {
  while (a > 180.0) a -= 360.0;
  while (a < -180.0) a += 360.0;
  return a;
}
static double dist_to_sector(double radius, double ang, double lo, double hi) {
  double dmin = norm_angle(ang - lo), dmax = norm_angle(hi - ang);
  if (dmin >= 0 && dmax >= 0) return 0.0;
  double m = fabs(dmin) < fabs(dmax) ? fabs(dmin) : fabs(dmax);
  double rad = m * M_PI / 180.0;
  return radius * sin(rad);
}
/* Domain::exchangeGhostParticles at world size 1 (spatial/Domain.cpp:339-403):
 * the only "neighbour" rank is rank 0 itself, owning [0, 360) degrees. */
static int is_self_ghost(const cell_t* c) {
  const double center_radius = 8, buffer = 2.5;
  double ang = atan2(c->x[1], c->x[0]) * 180.0 / M_PI;
  if (ang < 0) ang += 360.0;
  double radius = sqrt(c->x[0] * c->x[0] + c->x[1] * c->x[1]);
  if (radius >= center_radius) {
    if (dist_to_sector(radius, ang, 0.0, 360.0) < buffer) return 1;
  }
  return 0;
}

/* ------------------------------------------------------------------ detection */
typedef struct {
  int bx, by, bz, idx;
} binrec_t;

static int binrec_cmp(const void* A, const void* B) {
  const binrec_t *a = A, *b = B;
  if (a->bx != b->bx) return a->bx < b->bx ? -1 : 1;
  if (a->by != b->by) return a->by < b->by ? -1 : 1;
  if (a->bz != b->bz) return a->bz < b->bz ? -1 : 1;
  return a->idx < b->idx ? -1 : (a->idx > b->idx);
}

typedef struct {
  double key;
  size_t seq;
} sortkey_t;

static int cons_cmp_x(const void* A, const void* B) {
  const cons_t *a = A, *b = B;
  if (a->cp[0] < b->cp[0]) return -1;
  if (a->cp[0] > b->cp[0]) return 1;
  if (a->gi != b->gi) return a->gi < b->gi ? -1 : 1;
  return a->gj < b->gj ? -1 : (a->gj > b->gj);
}

/* CollisionDetector::tryCreateConstraint (spatial/CollisionDetector.cpp:201-311)
 * for the pair (I, J) = (a, b).  Returns 1 when a constraint is emitted. */
static int try_constraint(const cell_t* A, const cell_t* B, int ia, int ib, double tol, int phase, cons_t* out) {
  double d3[3] = {A->x[0] - B->x[0], A->x[1] - B->x[1], A->x[2] - B->x[2]};
  double rough = sqrt(dot3(d3, d3));
  if (rough > (A->len + B->len) / 2.0 + tol) return 0;
  double as[3], ae[3], bs[3], be[3], c0[3], c1[3], dist;
  endpoints(A, as, ae);
  endpoints(B, bs, be);
  segment_closest(as, ae, bs, be, c0, c1, &dist);
  double sum_radii = (A->diam + B->diam) / 2.0;
  double sd = dist - sum_radii;
  if (sd > tol) return 0;
  double cp[3], diff[3], ta[3], tb[3], nn[3];
  for (int d = 0; d < 3; ++d) cp[d] = (c0[d] + c1[d]) * 0.5;
  for (int d = 0; d < 3; ++d) diff[d] = c0[d] - c1[d];
  direction(A->q, ta);
  direction(B->q, tb);
  normalize3(diff, out->n);
  for (int d = 0; d < 3; ++d) nn[d] = -out->n[d];
  out->si = 0.5 * fabs(dot3(out->n, ta));
  out->sj = 0.5 * fabs(dot3(nn, tb));
  for (int d = 0; d < 3; ++d) {
    out->ri[d] = cp[d] - A->x[d];
    out->rj[d] = cp[d] - B->x[d];
    out->cp[d] = cp[d];
  }
  out->gi = ia;
  out->gj = ib;
  out->sd = sd;
  out->phase = phase;
  out->gamma = sd >= 0.0 ? 0.0 : -sd * 5e2;
  return 1;
}

/* CollisionDetector::detectCollisions (spatial/CollisionDetector.cpp:84-111)
 * with SpatialGrid::findPotentialCollisions (spatial/SpatialGrid.cpp:58-121):
 * all unordered pairs of cells binned (origin -1, edge linked_cell_size) into
 * the same or adjacent bins of the 27-stencil, then a sort by contact-point x.
 * With ghost_mode SINGLE_RANK a contact is emitted twice when its larger-id
 * cell has a self-ghost copy (the ownership rule at :261-275 accepts exactly
 * one of the two local-ghost pairs the copy adds). */
static cons_t* detect(pcco_colony* col, double tol, int phase, size_t* nout) {
  const size_t n = col->n;
  const double h = col->p.linked_cell_size;
  binrec_t* br = xrealloc(NULL, sizeof(binrec_t) * (n ? n : 1));
  char* ghost = xrealloc(NULL, n ? n : 1);
  for (size_t i = 0; i < n; ++i) {
    const cell_t* c = &col->cells[i];
    br[i].bx = (int)floor((c->x[0] - (-1.0)) / h);
    br[i].by = (int)floor((c->x[1] - (-1.0)) / h);
    br[i].bz = (int)floor((c->x[2] - (-1.0)) / h);
    br[i].idx = (int)i;
    ghost[i] = (char)(col->p.ghost_mode == PCC_GHOSTS_SINGLE_RANK ? is_self_ghost(c) : 0);
  }
  binrec_t* sorted = xrealloc(NULL, sizeof(binrec_t) * (n ? n : 1));
  memcpy(sorted, br, sizeof(binrec_t) * n);
  qsort(sorted, n, sizeof(binrec_t), binrec_cmp);
  size_t cap = 64, cnt = 0;
  cons_t* out = xrealloc(NULL, sizeof(cons_t) * cap);
  for (size_t a = 0; a < n; ++a) {
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          binrec_t key = {br[a].bx + dx, br[a].by + dy, br[a].bz + dz, -1};
          /* lower bound of the bin in the sorted list */
          size_t lo = 0, hi = n;
          while (lo < hi) {
            size_t mid = (lo + hi) / 2;
            if (binrec_cmp(&sorted[mid], &key) < 0) lo = mid + 1;
            else hi = mid;
          }
          for (size_t k = lo; k < n; ++k) {
            const binrec_t* r = &sorted[k];
            if (r->bx != key.bx || r->by != key.by || r->bz != key.bz) break;
            size_t b = (size_t)r->idx;
            if (b <= a) continue;
            cons_t cs;
            if (!try_constraint(&col->cells[a], &col->cells[b], (int)a, (int)b, tol, phase, &cs)) continue;
            /* incrementNumConstraints (CollisionDetector.cpp:243-244) runs for every
             * passing candidate, including the variants with ghost copies; counts
             * of a cell that has a self-ghost go to the ghost copy and are lost. */
            if (!ghost[a]) col->cells[a].nc += 1 + ghost[b];
            if (!ghost[b]) col->cells[b].nc += 1 + ghost[a];
            int copies = 1 + (ghost[b] ? 1 : 0);
            for (int k2 = 0; k2 < copies; ++k2) {
              if (cnt == cap) {
                cap *= 2;
                out = xrealloc(out, sizeof(cons_t) * cap);
              }
              out[cnt++] = cs;
            }
          }
        }
  }
  /* stable order by contact x; ties (identical ghost duplicates) by ids */
  qsort(out, cnt, sizeof(cons_t), cons_cmp_x);
  free(br);
  free(sorted);
  free(ghost);
  *nout = cnt;
  return out;
}

/* ------------------------------------------------------------------ sparse algebra */
/* Row c of D (Physics.cpp:118-154): [n, r_i x n] at columns 6i..6i+5 and
 * [-n, r_j x (-n)] at 6j..6j+5, stored in ascending column order. */
typedef struct {
  int col0, col1;      /* first cell of the row's two blocks, ascending */
  double v0[6], v1[6]; /* values of the blocks */
  double l0, l1;       /* L row (Physics.cpp:174-190) in the same column order */
} drow_t;

static void build_rows(const cons_t* cs, size_t m, drow_t* rows) {
  for (size_t c = 0; c < m; ++c) {
    const cons_t* k = &cs[c];
    double ni[3], nj[3], ti[3], tj[3], Fi[6], Fj[6];
    for (int d = 0; d < 3; ++d) {
      ni[d] = k->n[d];
      nj[d] = -k->n[d];
    }
    cross3(k->ri, ni, ti);
    cross3(k->rj, nj, tj);
    for (int d = 0; d < 3; ++d) {
      Fi[d] = ni[d];
      Fi[3 + d] = ti[d];
      Fj[d] = nj[d];
      Fj[3 + d] = tj[d];
    }
    drow_t* r = &rows[c];
    if (k->gi < k->gj) {
      r->col0 = k->gi;
      r->col1 = k->gj;
      memcpy(r->v0, Fi, sizeof Fi);
      memcpy(r->v1, Fj, sizeof Fj);
      r->l0 = k->si;
      r->l1 = k->sj;
    } else {
      r->col0 = k->gj;
      r->col1 = k->gi;
      memcpy(r->v0, Fj, sizeof Fj);
      memcpy(r->v1, Fi, sizeof Fi);
      r->l0 = k->sj;
      r->l1 = k->si;
    }
  }
}

/* y = D x  (MatMult, y has m entries, x has 6n) */
static void D_mult(const drow_t* R, size_t m, const double* x, double* y) {
  for (size_t c = 0; c < m; ++c) {
    double s = 0.0;
    for (int k = 0; k < 6; ++k) s += R[c].v0[k] * x[6 * R[c].col0 + k];
    for (int k = 0; k < 6; ++k) s += R[c].v1[k] * x[6 * R[c].col1 + k];
    y[c] = s;
  }
}
/* y = D^T x  (MatMultTranspose) */
static void D_multT(const drow_t* R, size_t m, size_t n, const double* x, double* y) {
  memset(y, 0, sizeof(double) * 6 * n);
  for (size_t c = 0; c < m; ++c) {
    const double alpha = x[c];
    for (int k = 0; k < 6; ++k) y[6 * R[c].col0 + k] += R[c].v0[k] * alpha;
    for (int k = 0; k < 6; ++k) y[6 * R[c].col1 + k] += R[c].v1[k] * alpha;
  }
}
static void L_mult(const drow_t* R, size_t m, const double* x, double* y) {
  for (size_t c = 0; c < m; ++c) {
    double s = 0.0;
    s += R[c].l0 * x[R[c].col0];
    s += R[c].l1 * x[R[c].col1];
    y[c] = s;
  }
}
static void L_multT(const drow_t* R, size_t m, size_t n, const double* x, double* y) {
  memset(y, 0, sizeof(double) * n);
  for (size_t c = 0; c < m; ++c) {
    const double alpha = x[c];
    y[R[c].col0] += R[c].l0 * alpha;
    y[R[c].col1] += R[c].l1 * alpha;
  }
}

/* VecWAXPY(w, a, x, y): w = a*x + y with PETSc's special cases */
static void waxpy(size_t n, double a, const double* x, const double* y, double* w) {
  if (a == 1.0)
    for (size_t i = 0; i < n; ++i) w[i] = y[i] + x[i];
  else if (a == -1.0)
    for (size_t i = 0; i < n; ++i) w[i] = y[i] - x[i];
  else if (a == 0.0)
    for (size_t i = 0; i < n; ++i) w[i] = y[i];
  else
    for (size_t i = 0; i < n; ++i) w[i] = a * x[i] + y[i];
}
static void vscale(size_t n, double a, double* x) {
  if (a == 1.0) return;
  if (a == 0.0) {
    memset(x, 0, sizeof(double) * n);
    return;
  }
  for (size_t i = 0; i < n; ++i) x[i] = a * x[i];
}

/* Mobility (Physics.cpp:192-218): 1/(l xi) for the 3 linear, 12/(l^3 xi) for
 * the 3 angular entries, applied as MatMult of a diagonal AIJ. */
static void mobility(const pcco_colony* col, double* Mdiag) {
  for (size_t i = 0; i < col->n; ++i) {
    double l = col->cells[i].len, xi = col->p.xi;
    double inv_len = 1.0 / (l * xi);
    double inv_len3_x_12 = 12.0 / (l * l * l * xi);
    for (int k = 0; k < 3; ++k) Mdiag[6 * i + k] = inv_len;
    for (int k = 3; k < 6; ++k) Mdiag[6 * i + k] = inv_len3_x_12;
  }
}
static void diag_mult(size_t n6, const double* M, const double* x, double* y) {
  for (size_t r = 0; r < n6; ++r) {
    double s = 0.0;
    s += M[r] * x[r];
    y[r] = s;
  }
}

/* dC = G U (Physics.cpp:220-265): 7 rows per cell, Xi(q)/2 for the quaternion */
static void G_mult(const pcco_colony* col, const double* U, double* dC) {
  for (size_t i = 0; i < col->n; ++i) {
    const double* q = col->cells[i].q;
    const double s = q[0], wx = q[1], wy = q[2], wz = q[3];
    for (int k = 0; k < 3; ++k) {
      double acc = 0.0;
      acc += 1 * U[6 * i + k];
      dC[7 * i + k] = acc;
    }
    const double xi[4][3] = {{-0.5 * wx, -0.5 * wy, -0.5 * wz},
                             {0.5 * s, -0.5 * wz, 0.5 * wy},
                             {0.5 * wz, 0.5 * s, -0.5 * wx},
                             {-0.5 * wy, 0.5 * wx, 0.5 * s}};
    for (int r = 0; r < 4; ++r) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc += xi[r][k] * U[6 * i + 3 + k];
      dC[7 * i + 3 + r] = acc;
    }
  }
}

/* ParticleManager::moveLocalParticlesFromSolution (simulation/ParticleManager.cpp:29-87)
 * with Particle::eulerStepPosition (simulation/Particle.cpp:37-57, 110-120). */
static void move_cells(pcco_colony* col, const double* dC, const double* F, const double* U, double dt) {
  for (size_t i = 0; i < col->n; ++i) {
    cell_t* c = &col->cells[i];
    const double* v = &dC[7 * i];
    for (int k = 0; k < 3; ++k) c->x[k] += dt * v[k];
    for (int k = 0; k < 4; ++k) c->q[k] += dt * v[3 + k];
    double norm = sqrt(c->q[0] * c->q[0] + c->q[1] * c->q[1] + c->q[2] * c->q[2] + c->q[3] * c->q[3]);
    for (int k = 0; k < 4; ++k) c->q[k] /= norm;
    for (int k = 0; k < 6; ++k) {
      c->force[k] = F[6 * i + k];
      c->vel[k] = U[6 * i + k];
    }
  }
}

/* ------------------------------------------------------------------ hard model */
typedef struct {
  size_t m, n;
  const drow_t* R;
  const double *M, *Uext, *phi, *gold, *len, *ldot_prev;
  double dt, lambda, tau;
  /* workspace (Workspace.h) */
  double *gdiff, *F, *Uc, *U, *phidot, *stress, *imp, *ldot, *ldiff, *growth, *phinext;
} grad_t;

/* HardModelGradient::gradient (dynamics/models/hard/HardModelGradient.cpp:89-121) */
static double* gradient(grad_t* g, const double* gamma) {
  const size_t m = g->m, n = g->n;
  waxpy(m, -1.0, g->gold, gamma, g->gdiff);
  D_multT(g->R, m, n, g->gdiff, g->F);
  diag_mult(6 * n, g->M, g->F, g->Uc);
  waxpy(6 * n, 1.0, g->Uext, g->Uc, g->U);
  D_mult(g->R, m, g->U, g->phidot);
  L_multT(g->R, m, n, gamma, g->stress);
  memcpy(g->imp, g->stress, sizeof(double) * n);
  vscale(n, -g->lambda, g->imp);
  for (size_t i = 0; i < n; ++i) g->imp[i] = exp(g->imp[i]);
  for (size_t i = 0; i < n; ++i) g->ldot[i] = g->len[i] * g->imp[i];
  vscale(n, 1 / g->tau, g->ldot);
  waxpy(n, -1.0, g->ldot_prev, g->ldot, g->ldiff);
  L_mult(g->R, m, g->ldiff, g->growth);
  memcpy(g->phinext, g->phi, sizeof(double) * m);
  const double a0 = g->dt, a1 = -g->dt;
  for (size_t i = 0; i < m; ++i) g->phinext[i] += a0 * g->phidot[i] + a1 * g->growth[i];
  return g->phinext;
}

/* HardModelGradient::residual (HardModelGradient.cpp:123-158) */
static double residual(size_t m, const double* grad, const double* gamma) {
  double res = 0.0;
  for (size_t i = 0; i < m; ++i) {
    double v;
    if (gamma[i] > 0)
      v = grad[i];
    else
      v = grad[i] < 0.0 ? grad[i] : 0.0;
    double av = fabs(v);
    res = res < av ? av : res;
  }
  return res;
}

/* BBPGD (solver/BBPGD.cpp:32-127).  gamma holds gamma_0 on entry and the
 * iterate before the converged one on return (the stored result of the
 * reference); the gradient workspace holds the converged iterate's values. */
static int bbpgd(grad_t* g, double* gamma, double tol, long long max_it, long long* iters, double* res_out) {
  const size_t m = g->m;
  double* gprev = xrealloc(NULL, sizeof(double) * (m ? m : 1));
  double* gam_i = xrealloc(NULL, sizeof(double) * (m ? m : 1));
  double* dgam = xrealloc(NULL, sizeof(double) * (m ? m : 1));
  double* dphi = xrealloc(NULL, sizeof(double) * (m ? m : 1));
  double* gam_prev = gamma;
  double* gi;
  memcpy(gprev, gradient(g, gam_prev), sizeof(double) * m);
  double res = residual(m, gprev, gam_prev);
  double alpha = 1.0 / res;
  long long it = 1;
  int rc = 0;
  while (it < max_it) {
    waxpy(m, -alpha, gprev, gam_prev, gam_i);
    for (size_t i = 0; i < m; ++i) gam_i[i] = gam_i[i] < 0.0 ? 0.0 : gam_i[i];
    gi = gradient(g, gam_i);
    if (it % 10 == 0) {
      res = residual(m, gi, gam_i);
      if (res <= tol) break;
    }
    waxpy(m, -1.0, gam_prev, gam_i, dgam);
    waxpy(m, -1.0, gprev, gi, dphi);
    double num = 0.0, den = 0.0;
    if (it % 2 == 0) {
      for (size_t i = 0; i < m; ++i) {
        num += dgam[i] * dgam[i];
        den += dgam[i] * dphi[i];
      }
    } else {
      for (size_t i = 0; i < m; ++i) {
        den += dphi[i] * dphi[i];
        num += dphi[i] * dgam[i];
      }
    }
    if (fabs(den) < 10 * DBL_EPSILON) den += 10 * DBL_EPSILON;
    alpha = num / den;
    /* swap(gamma_prev, gamma_i); swap(g_prev, g_i) */
    double* t = gam_prev;
    gam_prev = gam_i;
    gam_i = t;
    memcpy(gprev, gi, sizeof(double) * m);
    ++it;
  }
  if (it == max_it) rc = PCC_ERR_NOCONV_BBPGD;
  if (gam_prev != gamma) memcpy(gamma, gam_prev, sizeof(double) * m);
  free(gprev);
  free(gam_prev == gamma ? gam_i : gam_prev);
  free(dgam);
  free(dphi);
  *iters = it;
  *res_out = res;
  return rc;
}

static void append_cons(pcco_colony* col, const cons_t* add, size_t k) {
  if (col->ncons + k > col->capcons) {
    col->capcons = (col->ncons + k) * 2;
    col->cons = xrealloc(col->cons, sizeof(cons_t) * col->capcons);
  }
  memcpy(col->cons + col->ncons, add, sizeof(cons_t) * k);
  col->ncons += k;
}

static double max_overlap_of(const cons_t* cs, size_t m) {
  double acc = 0.0;
  for (size_t c = 0; c < m; ++c) {
    double v = cs[c].sd < 0 ? -cs[c].sd : 0;
    acc = acc < v ? v : acc;
  }
  return acc;
}

/* Particle::updateLength via ParticleManager::grow (simulation/Particle.cpp:59-65) */
static void grow_cells(pcco_colony* col, double dt) {
  for (size_t i = 0; i < col->n; ++i) {
    cell_t* c = &col->cells[i];
    c->len += dt * c->ldot;
    if (c->len > 2 * c->l0) c->len = 2 * c->l0;
  }
}

/* solveHardModel (dynamics/models/Hard.cpp:91-192) */
static int solve_hard(pcco_colony* col, double dt, pcc_step_stats* st) {
  const size_t n = col->n;
  const double tol = col->p.tolerance;
  int phase = 0;
  long long total_it = 0;
  double res = 0.0, max_ov = 0.0;
  int rc = 0;
  col->ncons = 0;
  for (size_t i = 0; i < n; ++i) col->cells[i].ldot = 0.0;
  double* Mdiag = xrealloc(NULL, sizeof(double) * 6 * (n ? n : 1));
  double* Uext = calloc(6 * (n ? n : 1), sizeof(double));
  double* len = xrealloc(NULL, sizeof(double) * (n ? n : 1));
  double* ldot_prev = xrealloc(NULL, sizeof(double) * (n ? n : 1));
  double* dC = xrealloc(NULL, sizeof(double) * 7 * (n ? n : 1));
  double* nvec[9];
  for (int k = 0; k < 9; ++k) nvec[k] = xrealloc(NULL, sizeof(double) * 6 * (n ? n : 1));
  while ((long long)phase < col->p.max_recursive_iterations) {
    size_t nnew = 0;
    cons_t* fresh = detect(col, phase == 0 ? .25 : tol, phase, &nnew);
    append_cons(col, fresh, nnew);
    free(fresh);
    max_ov = max_overlap_of(col->cons, col->ncons);
    if (max_ov <= tol && phase > 0) break;
    const size_t m = col->ncons;
    drow_t* R = xrealloc(NULL, sizeof(drow_t) * (m ? m : 1));
    build_rows(col->cons, m, R);
    mobility(col, Mdiag);
    for (size_t i = 0; i < n; ++i) {
      len[i] = col->cells[i].len;
      ldot_prev[i] = col->cells[i].ldot;
    }
    double *phi = xrealloc(NULL, sizeof(double) * (m ? m : 1)), *gam = xrealloc(NULL, sizeof(double) * (m ? m : 1));
    double* gold = xrealloc(NULL, sizeof(double) * (m ? m : 1));
    double* cbuf[5];
    for (int k = 0; k < 5; ++k) cbuf[k] = xrealloc(NULL, sizeof(double) * (m ? m : 1));
    for (size_t c = 0; c < m; ++c) {
      phi[c] = col->cons[c].sd;
      gam[c] = col->cons[c].gamma;
    }
    memcpy(gold, gam, sizeof(double) * m);
    grad_t g = {.m = m, .n = n, .R = R, .M = Mdiag, .Uext = Uext, .phi = phi, .gold = gold, .len = len,
                .ldot_prev = ldot_prev, .dt = dt, .lambda = col->p.lambda, .tau = col->p.tau,
                .gdiff = cbuf[0], .F = nvec[0], .Uc = nvec[1], .U = nvec[2], .phidot = cbuf[1],
                .stress = nvec[3], .imp = nvec[4], .ldot = nvec[5], .ldiff = nvec[6], .growth = cbuf[2],
                .phinext = cbuf[3]};
    long long it = 0;
    rc = bbpgd(&g, gam, tol, col->p.max_bbpgd_iterations, &it, &res);
    total_it += it;
    if (rc == 0) {
      G_mult(col, g.U, dC);
      move_cells(col, dC, g.F, g.U, dt);
      for (size_t i = 0; i < n; ++i) {
        col->cells[i].imp = g.imp[i];
        col->cells[i].stress = g.stress[i];
        col->cells[i].ldot = g.ldot[i];
      }
      for (size_t c = 0; c < m; ++c) {
        col->cons[c].gamma = gam[c];
        col->cons[c].sd = g.phinext[c];
      }
    }
    free(R);
    free(phi);
    free(gam);
    free(gold);
    for (int k = 0; k < 5; ++k) free(cbuf[k]);
    if (rc) {
      snprintf(col->err, sizeof col->err, "BBPGD did not converge");
      break;
    }
    phase++;
  }
  if (rc == 0) {
    grow_cells(col, dt);
    if ((long long)phase == col->p.max_recursive_iterations) {
      rc = PCC_ERR_NOCONV_RELCP;
      snprintf(col->err, sizeof col->err, "Maximum number of constraint iterations reached");
    }
  }
  free(Mdiag);
  free(Uext);
  free(len);
  free(ldot_prev);
  free(dC);
  for (int k = 0; k < 9; ++k) free(nvec[k]);
  if (st) {
    st->relcp_iterations = phase;
    st->bbpgd_iterations = total_it;
    st->residual = res;
    st->max_overlap = max_ov;
    st->n_constraints = (long long)col->ncons;
    st->n_cells = (long long)n;
  }
  return rc;
}

/* ------------------------------------------------------------------ soft model */
/* solveSoftPotential (dynamics/models/Soft.cpp:21-114) */
static int solve_soft(pcco_colony* col, double dt, pcc_step_stats* st) {
  const size_t n = col->n;
  size_t m = 0;
  cons_t* cs = detect(col, 0, 0, &m);
  col->ncons = 0;
  append_cons(col, cs, m);
  free(cs);
  double max_ov = max_overlap_of(col->cons, m);
  double* F = calloc(6 * (n ? n : 1), sizeof(double));
  double* stress = calloc(n ? n : 1, sizeof(double));
  for (size_t c = 0; c < m; ++c) {
    const cons_t* k = &col->cons[c];
    double overlap = -k->sd;
    if (overlap <= 0.00) continue;
    double R1 = col->cells[k->gi].diam / 2.0, R2 = col->cells[k->gj].diam / 2.0;
    double R_eff = sqrt(R1 * R2 / (R1 + R2));
    double F_el = R_eff * col->p.kcc * pow(overlap, 1.5);
    double fi[3], fj[3], ti[3], tj[3];
    for (int d = 0; d < 3; ++d) fi[d] = k->n[d] * F_el;
    for (int d = 0; d < 3; ++d) fj[d] = -fi[d];
    cross3(k->ri, fi, ti);
    cross3(k->rj, fj, tj);
    for (int d = 0; d < 3; ++d) {
      F[6 * k->gi + d] += fi[d];
    }
    for (int d = 0; d < 3; ++d) F[6 * k->gi + 3 + d] += ti[d];
    for (int d = 0; d < 3; ++d) F[6 * k->gj + d] += fj[d];
    for (int d = 0; d < 3; ++d) F[6 * k->gj + 3 + d] += tj[d];
    stress[k->gi] += k->si * F_el;
    stress[k->gj] += k->sj * F_el;
  }
  double* M = xrealloc(NULL, sizeof(double) * 6 * (n ? n : 1));
  double* Uc = xrealloc(NULL, sizeof(double) * 6 * (n ? n : 1));
  double* U = xrealloc(NULL, sizeof(double) * 6 * (n ? n : 1));
  double* Uext = calloc(6 * (n ? n : 1), sizeof(double));
  double* dC = xrealloc(NULL, sizeof(double) * 7 * (n ? n : 1));
  mobility(col, M);
  diag_mult(6 * n, M, F, Uc);
  waxpy(6 * n, 1.0, Uext, Uc, U);
  G_mult(col, U, dC);
  move_cells(col, dC, F, U, dt);
  /* calculate_growth_rate_vector (HardModelGradient.cpp:43-52) */
  for (size_t i = 0; i < n; ++i) {
    double imp = stress[i];
    col->cells[i].stress = stress[i];
    col->cells[i].imp = imp;
  }
  double* imp = xrealloc(NULL, sizeof(double) * (n ? n : 1));
  for (size_t i = 0; i < n; ++i) imp[i] = stress[i];
  vscale(n, -col->p.lambda, imp);
  for (size_t i = 0; i < n; ++i) imp[i] = exp(imp[i]);
  double* ld = xrealloc(NULL, sizeof(double) * (n ? n : 1));
  for (size_t i = 0; i < n; ++i) ld[i] = col->cells[i].len * imp[i];
  vscale(n, 1 / col->p.tau, ld);
  for (size_t i = 0; i < n; ++i) {
    col->cells[i].imp = imp[i];
    col->cells[i].ldot = ld[i];
  }
  grow_cells(col, dt);
  free(F);
  free(stress);
  free(M);
  free(Uc);
  free(U);
  free(Uext);
  free(dC);
  free(imp);
  free(ld);
  if (st) {
    st->relcp_iterations = 0;
    st->bbpgd_iterations = 0;
    st->residual = max_ov;
    st->max_overlap = max_ov;
    st->n_constraints = (long long)m;
    st->n_cells = (long long)n;
  }
  return 0;
}

/* ------------------------------------------------------------------ division RNG */
unsigned int pcco_division_seed(unsigned long long seed, unsigned long long k) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (k + 1ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (unsigned int)(z & 0xffffffffULL);
}

/* The first two outputs of MT19937 seeded with s (Matsumoto & Nishimura 1998,
 * init_genrand), i.e. what std::mt19937(s) returns on its first two calls. */
static void mt19937_first_two(uint32_t s, uint32_t out[2]) {
  uint32_t mt[399];
  mt[0] = s;
  for (uint32_t i = 1; i < 399; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i;
  for (int k = 0; k < 2; ++k) {
    uint32_t y = (mt[k] & 0x80000000u) | (mt[k + 1] & 0x7fffffffu);
    uint32_t v = mt[k + 397] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    v ^= v >> 11;
    v ^= (v << 7) & 0x9d2c5680u;
    v ^= (v << 15) & 0xefc60000u;
    v ^= v >> 18;
    out[k] = v;
  }
}

/* Particle::divide's draw (simulation/Particle.cpp:128-135): a 53-bit
 * canonical double from two 32-bit outputs (libstdc++ generate_canonical:
 * (x0 + x1*2^32) / 2^64, kept below 1), scaled to [0.98, 1.02] * len/2. */
double pcco_division_length(unsigned long long seed, unsigned long long k, double len) {
  uint32_t x[2];
  mt19937_first_two(pcco_division_seed(seed, k), x);
  double sum = 0.0, tmp = 1.0;
  sum += (double)x[0] * tmp;
  tmp *= 4294967296.0;
  sum += (double)x[1] * tmp;
  tmp *= 4294967296.0;
  double u = sum / tmp;
  if (u >= 1.0) u = nextafter(1.0, 0.0);
  double half = len / 2;
  double a = half * 0.98, b = half * 1.02;
  return u * (b - a) + a;
}

/* ------------------------------------------------------------------ driver */
static int cell_x_cmp(const void* A, const void* B) {
  const cell_t *a = A, *b = B;
  if (a->x[0] < b->x[0]) return -1;
  if (a->x[0] > b->x[0]) return 1;
  return 0;
}

/* ParticleManager::divideParticles + Particle::divide + Domain::commitNewParticles
 * (simulation/ParticleManager.cpp:139-148, simulation/Particle.cpp:122-150,
 * spatial/Domain.cpp:55-67) */
static size_t divide_cells(pcco_colony* col) {
  size_t n0 = col->n, added = 0;
  for (size_t i = 0; i < n0; ++i)
    if (col->cells[i].len >= 2 * col->cells[i].l0) ++added;
  if (!added) return 0;
  if (col->n + added > col->cap) {
    col->cap = (col->n + added) * 2;
    col->cells = xrealloc(col->cells, sizeof(cell_t) * col->cap);
  }
  for (size_t i = 0; i < n0; ++i) {
    cell_t* c = &col->cells[i];
    if (c->len < 2 * c->l0) continue;
    double l1 = pcco_division_length(col->p.seed, col->div_index++, c->len);
    double l2 = c->len - l1;
    double t[3], left[3], right[3];
    direction(c->q, t);
    for (int d = 0; d < 3; ++d) {
      left[d] = c->x[d] - t[d] * (l1 / 2);
      right[d] = c->x[d] + t[d] * (l2 / 2);
    }
    cell_t nc;
    memset(&nc, 0, sizeof nc);
    memcpy(nc.x, right, sizeof right);
    memcpy(nc.q, c->q, sizeof nc.q);
    nc.len = l2;
    nc.l0 = c->l0;
    nc.diam = c->diam;
    memcpy(c->x, left, sizeof left);
    c->len = l1;
    c->age++;
    nc.age = c->age;
    col->cells[col->n++] = nc;
  }
  return added;
}

/* Domain::adaptDt (spatial/Domain.cpp:69-118) */
static int dbl_cmp(const void* A, const void* B) {
  double a = *(const double*)A, b = *(const double*)B;
  return a < b ? -1 : (a > b);
}
static void adapt_dt(pcco_colony* col) {
  size_t n = col->n;
  if (!n) return;
  double* v = xrealloc(NULL, sizeof(double) * n);
  for (size_t i = 0; i < n; ++i) {
    const double* u = col->cells[i].vel;
    v[i] = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) + col->cells[i].ldot;
  }
  qsort(v, n, sizeof(double), dbl_cmp);
  double med = v[n / 2];
  if (n % 2 == 0) med = 0.5 * (v[n / 2 - 1] + med);
  free(v);
  double gmed = med / 1;
  if (gmed == 0.0) return;
  double cfl = col->p.cfl_factor * col->p.tolerance;
  double cap_dt = cfl / gmed;
  double dt = col->p.dt;
  double nd = dt * (1.0 - 0.01) + 0.01 * cap_dt;
  double lo = 0.9 * dt, hi = 1.1 * dt;
  nd = nd < lo ? lo : (hi < nd ? hi : nd);
  col->p.dt = nd;
}

static double colony_radius(const pcco_colony* col) {
  double r = 0.0;
  for (size_t i = 0; i < col->n; ++i) {
    double s[3], e[3];
    endpoints(&col->cells[i], s, e);
    double m = sqrt(dot3(e, e));
    r = r < m ? m : r;
  }
  return r;
}

/* ------------------------------------------------------------------ API */
pcco_colony* pcco_create(const pcc_params* p) {
  pcco_colony* c = calloc(1, sizeof *c);
  c->p = *p;
  return c;
}
void pcco_destroy(pcco_colony* c) {
  if (!c) return;
  free(c->cells);
  free(c->cons);
  free(c);
}
const char* pcco_last_error(pcco_colony* c) { return c->err; }

int pcco_set_cells(pcco_colony* c, const pcc_cells* s, size_t n) {
  if (n > c->cap) {
    c->cap = n * 2 + 16;
    c->cells = xrealloc(c->cells, sizeof(cell_t) * c->cap);
  }
  c->n = n;
  for (size_t i = 0; i < n; ++i) {
    cell_t* x = &c->cells[i];
    memset(x, 0, sizeof *x);
    x->x[0] = s->x[i];
    x->x[1] = s->y[i];
    x->x[2] = s->z[i];
    x->q[0] = s->q0[i];
    x->q[1] = s->q1[i];
    x->q[2] = s->q2[i];
    x->q[3] = s->q3[i];
    x->len = s->length[i];
    x->l0 = s->l0[i];
    x->diam = s->diameter[i];
    x->ldot = s->ldot ? s->ldot[i] : 0.0;
    x->imp = s->impedance ? s->impedance[i] : 0.0;
    x->stress = s->stress ? s->stress[i] : 0.0;
    x->age = s->age ? s->age[i] : 1;
  }
  c->radius = colony_radius(c);
  return 0;
}

int pcco_get_cells(pcco_colony* c, pcc_cells* o, size_t cap, size_t* n) {
  *n = c->n;
  if (cap < c->n) return PCC_ERR_CAPACITY;
  for (size_t i = 0; i < c->n; ++i) {
    const cell_t* x = &c->cells[i];
    o->x[i] = x->x[0];
    o->y[i] = x->x[1];
    o->z[i] = x->x[2];
    o->q0[i] = x->q[0];
    o->q1[i] = x->q[1];
    o->q2[i] = x->q[2];
    o->q3[i] = x->q[3];
    o->length[i] = x->len;
    o->l0[i] = x->l0;
    o->diameter[i] = x->diam;
    if (o->ldot) o->ldot[i] = x->ldot;
    if (o->impedance) o->impedance[i] = x->imp;
    if (o->stress) o->stress[i] = x->stress;
    if (o->age) o->age[i] = x->age;
    if (o->num_constraints) o->num_constraints[i] = x->nc;
    if (o->force) memcpy(o->force + 6 * i, x->force, sizeof x->force);
    if (o->velocity) memcpy(o->velocity + 6 * i, x->vel, sizeof x->vel);
  }
  return 0;
}

int pcco_solve(pcco_colony* c, double dt, int iter, pcc_step_stats* st) {
  (void)iter;
  if (c->p.temperature > 0) {
    snprintf(c->err, sizeof c->err, "temperature > 0 (Brownian kicks) is not restated");
    return PCC_ERR_INVALID;
  }
  for (size_t i = 0; i < c->n; ++i) { /* Particle::reset (Particle.h:146-149) */
    c->cells[i].ldot = 0.0;
    c->cells[i].nc = 0;
  }
  int rc = c->p.mode == PCC_MODE_SOFT ? solve_soft(c, dt, st) : solve_hard(c, dt, st);
  if (st) st->dt_used = dt;
  return rc;
}

/* One Domain::run iteration at one rank (spatial/Domain.cpp:125-153) */
int pcco_step(pcco_colony* c, pcc_step_stats* st) {
  pcc_step_stats local;
  memset(&local, 0, sizeof local);
  size_t added = divide_cells(c);
  /* Domain::assignGlobalIDs: order by x (ties keep their order), ids 0..n-1 */
  size_t n = c->n;
  typedef struct {
    cell_t c;
    size_t k;
  } tagged_t;
  tagged_t* tg = xrealloc(NULL, sizeof(tagged_t) * (n ? n : 1));
  for (size_t i = 0; i < n; ++i) {
    tg[i].c = c->cells[i];
    tg[i].k = i;
  }
  /* stable merge of (x, previous index) keys */
  for (size_t w = 1; w < n; w *= 2) {
    tagged_t* tmp = xrealloc(NULL, sizeof(tagged_t) * n);
    for (size_t lo = 0; lo < n; lo += 2 * w) {
      size_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
      size_t a = lo, b = mid, o = lo;
      while (a < mid && b < hi) tmp[o++] = (cell_x_cmp(&tg[b].c, &tg[a].c) < 0) ? tg[b++] : tg[a++];
      while (a < mid) tmp[o++] = tg[a++];
      while (b < hi) tmp[o++] = tg[b++];
    }
    memcpy(tg, tmp, sizeof(tagged_t) * n);
    free(tmp);
  }
  for (size_t i = 0; i < n; ++i) c->cells[i] = tg[i].c;
  free(tg);
  double dt = c->p.dt;
  int rc = pcco_solve(c, dt, (int)c->iter, &local);
  if (rc) return rc;
  c->sim_time += dt;
  if (!c->p.fixed_dt) {
    adapt_dt(c);
    if (c->p.dt_cap > 0 && c->p.dt > c->p.dt_cap) c->p.dt = c->p.dt_cap;
  }
  c->radius = colony_radius(c);
  c->iter++;
  local.n_divided = (long long)added;
  local.dt_used = dt;
  local.dt_next = c->p.dt;
  local.colony_radius = c->radius;
  local.sim_time = c->sim_time;
  if (st) *st = local;
  return 0;
}

int pcco_run(pcco_colony* c, double end_radius, long long max_steps, long long* steps_done, double* cell_steps,
             pcc_step_stats* last) {
  long long s = 0;
  double cs = 0;
  pcc_step_stats st;
  memset(&st, 0, sizeof st);
  while (c->radius < end_radius && s < max_steps) {
    int rc = pcco_step(c, &st);
    if (rc) return rc;
    cs += (double)st.n_cells;
    ++s;
  }
  if (steps_done) *steps_done = s;
  if (cell_steps) *cell_steps = cs;
  if (last) *last = st;
  return 0;
}

static void export_cons(const cons_t* cs, size_t m, pcc_contacts* o) {
  for (size_t k = 0; k < m; ++k) {
    o->gid_i[k] = cs[k].gi;
    o->gid_j[k] = cs[k].gj;
    o->sd[k] = cs[k].sd;
    for (int d = 0; d < 3; ++d) {
      o->normal[3 * k + d] = cs[k].n[d];
      o->r_i[3 * k + d] = cs[k].ri[d];
      o->r_j[3 * k + d] = cs[k].rj[d];
      o->contact_point[3 * k + d] = cs[k].cp[d];
    }
    o->stress_i[k] = cs[k].si;
    o->stress_j[k] = cs[k].sj;
    o->gamma[k] = cs[k].gamma;
    o->phase[k] = cs[k].phase;
  }
}

int pcco_detect(pcco_colony* c, double tol, int phase, pcc_contacts* out, size_t cap, size_t* n) {
  size_t m = 0;
  cons_t* cs = detect(c, tol, phase, &m);
  *n = m;
  if (cap < m) {
    free(cs);
    return PCC_ERR_CAPACITY;
  }
  export_cons(cs, m, out);
  free(cs);
  return 0;
}

int pcco_get_constraints(pcco_colony* c, pcc_contacts* out, size_t cap, size_t* n) {
  *n = c->ncons;
  if (cap < c->ncons) return PCC_ERR_CAPACITY;
  export_cons(c->cons, c->ncons, out);
  return 0;
}

double pcco_get_dt(pcco_colony* c) { return c->p.dt; }
void pcco_set_dt(pcco_colony* c, double dt) { c->p.dt = dt; }
double pcco_colony_radius(pcco_colony* c) { return c->radius; }
unsigned long long pcco_division_count(pcco_colony* c) { return c->div_index; }
