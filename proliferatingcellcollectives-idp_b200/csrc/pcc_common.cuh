// Shared device-side definitions of the collision hot path (sm_100a).
//
// Cells live in structure-of-arrays form in global-id order (ids are ranks of
// the x-sort, spatial/Domain.cpp:492-508 of the reference).  Constraints live
// in structure-of-arrays form, appended phase by phase within a step.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pcc_gpu.h"

namespace pcc {

constexpr int kBlock = 256;

// Error codes raised on the device (bitmask in DevStatus::flags).
enum : unsigned {
  kDevErrBounds = 1u << 0,     // an index fell outside its buffer
  kDevErrTimeout = 1u << 1,    // a bounded spin-wait gave up
  kDevErrCapacity = 1u << 2,   // a per-call capacity was exceeded
  kDevErrNan = 1u << 3,        // non-finite values appeared
};

struct DevStatus {
  unsigned flags;
  int where;
  unsigned long long max_bits;    // running max of a non-negative double (bit pattern)
  unsigned list_flags;            // contact detection: candidate lists overflowed / stale
  unsigned pad;
  unsigned long long drift_bits;  // largest squared displacement since the lists were built
  unsigned long long lmax_bits;   // longest cell
  unsigned long long maxold_bits; // largest overlap of the constraints of earlier ReLCP phases
};

// Cell arrays (device pointers).
struct CellsView {
  double *x, *y, *z, *q0, *q1, *q2, *q3;
  double *len, *l0, *diam, *ldot, *imp, *stress;
  int* age;
  double* force;  // 6 per cell
  double* vel;    // 6 per cell
  int* ncons;     // contacts counted during the last solve (Particle::getNumConstraints)
};

// Constraint arrays (device pointers).  D row of constraint c
// (dynamics/Physics.cpp:118-154): [n, ti] at cell gi and [-n, tj] at cell gj
// with ti = ri x n and tj = rj x (-n).
struct ConsView {
  int *gi, *gj, *phase;
  double *sd, *gamma;
  double *nx, *ny, *nz;
  double *tix, *tiy, *tiz, *tjx, *tjy, *tjz;
  double *rix, *riy, *riz, *rjx, *rjy, *rjz;
  double *cpx, *cpy, *cpz;
  double *si, *sj;
};

// IEEE round-to-nearest arithmetic without contraction, so the geometry and
// the state update round exactly like the reference's strict build.
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// Unit axis of a cell: the quaternion applied to (1,0,0)
// (util/Quaternion.cpp:7-38, evaluated in the same order).
__device__ __forceinline__ void cell_axis(double w, double x, double y, double z, double t[3]) {
  const double vx = 1.0, vy = 0.0, vz = 0.0;
  const double c1x = sub(mul(y, vz), mul(z, vy));
  const double c1y = sub(mul(z, vx), mul(x, vz));
  const double c1z = sub(mul(x, vy), mul(y, vx));
  const double c2x = sub(mul(y, c1z), mul(z, c1y));
  const double c2y = sub(mul(z, c1x), mul(x, c1z));
  const double c2z = sub(mul(x, c1y), mul(y, c1x));
  const double w2 = mul(2.0, w);
  t[0] = add(add(vx, mul(w2, c1x)), mul(2.0, c2x));
  t[1] = add(add(vy, mul(w2, c1y)), mul(2.0, c2y));
  t[2] = add(add(vz, mul(w2, c1z)), mul(2.0, c2z));
}

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  double r = 0.0;
  r = add(r, mul(a[0], b[0]));
  r = add(r, mul(a[1], b[1]));
  r = add(r, mul(a[2], b[2]));
  return r;
}

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double r[3]) {
  r[0] = sub(mul(a[1], b[2]), mul(a[2], b[1]));
  r[1] = sub(mul(a[2], b[0]), mul(a[0], b[2]));
  r[2] = sub(mul(a[0], b[1]), mul(a[1], b[0]));
}

// Loads that bypass L1: data produced by other blocks of the same
// persistent kernel after a grid barrier.
template <typename T>
__device__ __forceinline__ T ldcg(const T* p) {
  return __ldcg(p);
}
template <>
__device__ __forceinline__ double4 ldcg<double4>(const double4* p) {
  const double2 lo = __ldcg(reinterpret_cast<const double2*>(p));
  const double2 hi = __ldcg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(lo.x, lo.y, hi.x, hi.y);
}

__device__ __forceinline__ void raise_error(DevStatus* st, unsigned flag, int where) {
  atomicOr(&st->flags, flag);
  atomicExch(&st->where, where);
}

// Monotone map of a double to an unsigned 64-bit key (ascending order
// preserved, -0 before +0).
__device__ __forceinline__ unsigned long long double_key(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}

inline unsigned grid_for(long long n, int block = kBlock) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 2147483647LL) g = 2147483647LL;
  return (unsigned)g;
}

}  // namespace pcc
