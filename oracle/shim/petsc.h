// Single-rank, sequential stand-in for the subset of the PETSc API that the
// reference simulator calls, used only to compile the reference's own sources
// in place as a CPU test oracle (there is no PETSc in this environment).
//
// Test infrastructure: nothing in the product library includes this file.
// The arithmetic order below defines the oracle's rounding and follows
// PETSc's sequential kernels as documented:
//   MatMult (AIJ)          y[r] = sum over the row's entries in ascending column
//                          order, accumulated from 0.0;
//   MatMultTranspose (AIJ) y = 0; rows in ascending order scatter y[c] += a*x[r];
//   VecWAXPY               special cases a = 1, -1, 0 as y+x, y-x, y;
//   VecMAXPY (2 vectors)   y[i] += a0*x0[i] + a1*x1[i];
//   VecDot / VecSum        one sequential loop.
// Values set with INSERT_VALUES/ADD_VALUES into a matrix are stashed per
// (row, column) and compressed into a column-sorted CSR at assembly, as
// SeqAIJ does; explicit zeros are stored.
#pragma once

// The real petsc.h pulls in the C headers <math.h> and <stdlib.h> (petscmath.h,
// petscsys.h).  In C++ those wrappers also place the std::abs overloads in the
// global namespace, so an unqualified abs(double) in the reference (for example
// the stress weights in spatial/CollisionDetector.cpp:258-259) is the floating
// point overload.  Include them here too, or abs would bind to int abs(int).
#include <math.h>
#include <stdlib.h>

#include <mpi.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <strings.h>
#include <map>
#include <string>
#include <utility>
#include <vector>

typedef int PetscInt;
typedef int PetscMPIInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef double PetscLogDouble;
typedef int PetscErrorCode;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef enum { INSERT_VALUES = 1, ADD_VALUES = 2 } InsertMode;
typedef enum { SCATTER_FORWARD = 0 } ScatterMode;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum { PETSC_COPY_VALUES = 0, PETSC_OWN_POINTER = 1, PETSC_USE_POINTER = 2 } PetscCopyMode;
typedef const char* MatType;
typedef const char* VecType;

#define MATAIJ "aij"
#define VECSTANDARD "standard"
#define PETSC_COMM_WORLD MPI_COMM_WORLD
#define PETSC_COMM_SELF MPI_COMM_SELF
#define PETSC_DECIDE (-1)
#define PETSC_DETERMINE (-1)
#define PETSC_MAX_PATH_LEN 4096
#define MPIU_INT MPI_INT
#define PetscRealPart(a) (a)
#define PetscMax(a, b) (((a) < (b)) ? (b) : (a))
#define PetscMin(a, b) (((a) < (b)) ? (a) : (b))
#define PetscCallAbort(comm, ...)                                                          \
  do {                                                                                     \
    PetscErrorCode pcc_shim_ierr_ = (PetscErrorCode)(__VA_ARGS__);                         \
    if (pcc_shim_ierr_) {                                                                  \
      std::fprintf(stderr, "PETSc shim error %d at %s:%d\n", pcc_shim_ierr_, __FILE__, __LINE__); \
      std::abort();                                                                        \
    }                                                                                      \
  } while (0)

struct _p_Vec {
  std::vector<double> a;
};
typedef _p_Vec* Vec;

struct _p_Mat {
  PetscInt rows = 0, cols = 0;
  std::map<std::pair<PetscInt, PetscInt>, double> stash;
  std::vector<PetscInt> rowptr, colidx;
  std::vector<double> val;
  bool assembled = false;
};
typedef _p_Mat* Mat;

struct _p_IS {
  std::vector<PetscInt> idx;
};
typedef _p_IS* IS;
struct _p_ISLocalToGlobalMapping {};
typedef _p_ISLocalToGlobalMapping* ISLocalToGlobalMapping;

struct _p_VecScatter {
  std::vector<PetscInt> from;
};
typedef _p_VecScatter* VecScatter;

typedef int PetscViewer;
#define PETSC_VIEWER_STDOUT_WORLD 0

namespace pcc_petsc_shim {
struct Options {
  std::vector<std::pair<std::string, std::string>> kv;  // "-name" -> value ("" if flag only)
  const std::string* find(const char* name) const {
    // PETSc option names are matched case-insensitively.
    for (auto it = kv.rbegin(); it != kv.rend(); ++it) {
      if (strcasecmp(it->first.c_str(), name) == 0) return &it->second;
    }
    return nullptr;
  }
};
inline Options& options() {
  static Options o;
  return o;
}
inline bool& quiet() {
  static bool q = std::getenv("PCC_SHIM_VERBOSE") == nullptr;
  return q;
}
}  // namespace pcc_petsc_shim

inline PetscErrorCode PetscOptionsInsertArgs(int argc, char** argv) {
  auto& o = pcc_petsc_shim::options();
  for (int i = 1; i < argc; ++i) {
    if (argv[i][0] != '-') continue;
    std::string name = argv[i];
    std::string value;
    if (i + 1 < argc && (argv[i + 1][0] != '-' || (argv[i + 1][1] >= '0' && argv[i + 1][1] <= '9') ||
                         argv[i + 1][1] == '.')) {
      value = argv[++i];
    }
    o.kv.emplace_back(name, value);
  }
  return 0;
}
inline PetscErrorCode PetscOptionsClearAll() {
  pcc_petsc_shim::options().kv.clear();
  return 0;
}
inline PetscErrorCode PetscOptionsSetValue(void*, const char* name, const char* value) {
  pcc_petsc_shim::options().kv.emplace_back(name, value ? value : "");
  return 0;
}
inline PetscErrorCode PetscInitialize(int* argc, char*** argv, const char*, const char*) {
  if (argc && argv) PetscOptionsInsertArgs(*argc, *argv);
  return 0;
}
inline PetscErrorCode PetscFinalize() { return 0; }
inline PetscErrorCode PetscLogDefaultBegin() { return 0; }
inline PetscErrorCode PetscMemorySetGetMaximumUsage() { return 0; }
inline PetscErrorCode PetscMemoryGetCurrentUsage(PetscLogDouble* m) { *m = 0; return 0; }
inline PetscErrorCode PetscMemoryGetMaximumUsage(PetscLogDouble* m) { *m = 0; return 0; }
inline PetscErrorCode PetscPrintf(MPI_Comm, const char* fmt, ...) {
  if (pcc_petsc_shim::quiet()) return 0;
  va_list ap;
  va_start(ap, fmt);
  std::vfprintf(stdout, fmt, ap);
  va_end(ap);
  return 0;
}
inline PetscErrorCode PetscOptionsHasName(void*, const char*, const char* name, PetscBool* set) {
  *set = pcc_petsc_shim::options().find(name) ? PETSC_TRUE : PETSC_FALSE;
  return 0;
}
inline PetscErrorCode PetscOptionsGetReal(void*, const char*, const char* name, PetscReal* v, PetscBool* set) {
  const std::string* s = pcc_petsc_shim::options().find(name);
  if (set) *set = PETSC_FALSE;
  if (s && !s->empty()) {
    *v = std::strtod(s->c_str(), nullptr);
    if (set) *set = PETSC_TRUE;
  }
  return 0;
}
template <typename T>
inline PetscErrorCode PetscOptionsGetInt(void*, const char*, const char* name, T* v, PetscBool* set) {
  const std::string* s = pcc_petsc_shim::options().find(name);
  if (set) *set = PETSC_FALSE;
  if (s && !s->empty()) {
    *v = (T)std::strtoll(s->c_str(), nullptr, 10);
    if (set) *set = PETSC_TRUE;
  }
  return 0;
}
inline PetscErrorCode PetscOptionsGetBool(void*, const char*, const char* name, PetscBool* v, PetscBool* set) {
  const std::string* s = pcc_petsc_shim::options().find(name);
  if (set) *set = PETSC_FALSE;
  if (s) {
    *v = (s->empty() || *s == "1" || strcasecmp(s->c_str(), "true") == 0 || strcasecmp(s->c_str(), "yes") == 0)
             ? PETSC_TRUE
             : PETSC_FALSE;
    if (set) *set = PETSC_TRUE;
  }
  return 0;
}
inline PetscErrorCode PetscOptionsGetBool(void* o, const char* p, const char* name, bool* v, PetscBool* set) {
  PetscBool b = *v ? PETSC_TRUE : PETSC_FALSE;
  PetscErrorCode e = PetscOptionsGetBool(o, p, name, &b, set);
  *v = b == PETSC_TRUE;
  return e;
}
inline PetscErrorCode PetscOptionsGetString(void*, const char*, const char* name, char* buf, size_t len,
                                            PetscBool* set) {
  const std::string* s = pcc_petsc_shim::options().find(name);
  if (set) *set = PETSC_FALSE;
  if (s) {
    std::snprintf(buf, len, "%s", s->c_str());
    if (set) *set = PETSC_TRUE;
  }
  return 0;
}

// ----------------------------------------------------------------- Vec
inline PetscErrorCode VecCreate(MPI_Comm, Vec* v) { *v = new _p_Vec(); return 0; }
inline PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt n, Vec* v) {
  *v = new _p_Vec();
  (*v)->a.assign((size_t)n, 0.0);
  return 0;
}
inline PetscErrorCode VecSetSizes(Vec v, PetscInt local, PetscInt global) {
  v->a.assign((size_t)(local >= 0 ? local : global), 0.0);
  return 0;
}
inline PetscErrorCode VecSetFromOptions(Vec) { return 0; }
inline PetscErrorCode VecSetType(Vec, VecType) { return 0; }
inline PetscErrorCode VecDuplicate(Vec x, Vec* y) {
  *y = new _p_Vec();
  (*y)->a.assign(x->a.size(), 0.0);
  return 0;
}
inline PetscErrorCode VecDestroy(Vec* v) {
  delete *v;
  *v = nullptr;
  return 0;
}
inline PetscErrorCode VecCopy(Vec x, Vec y) { y->a = x->a; return 0; }
inline PetscErrorCode VecZeroEntries(Vec v) { std::fill(v->a.begin(), v->a.end(), 0.0); return 0; }
inline PetscErrorCode VecGetSize(Vec v, PetscInt* n) { *n = (PetscInt)v->a.size(); return 0; }
inline PetscErrorCode VecGetLocalSize(Vec v, PetscInt* n) { *n = (PetscInt)v->a.size(); return 0; }
inline PetscErrorCode VecGetOwnershipRange(Vec v, PetscInt* lo, PetscInt* hi) {
  *lo = 0;
  *hi = (PetscInt)v->a.size();
  return 0;
}
inline PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar** p) { *p = v->a.data(); return 0; }
inline PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar** p) { *p = nullptr; return 0; }
inline PetscErrorCode VecGetArray(Vec v, PetscScalar** p) { *p = v->a.data(); return 0; }
inline PetscErrorCode VecRestoreArray(Vec, PetscScalar** p) { *p = nullptr; return 0; }
inline PetscErrorCode VecSetValue(Vec v, PetscInt i, PetscScalar x, InsertMode m) {
  if (m == ADD_VALUES)
    v->a.at((size_t)i) += x;
  else
    v->a.at((size_t)i) = x;
  return 0;
}
inline PetscErrorCode VecSetValues(Vec v, PetscInt n, const PetscInt* idx, const PetscScalar* x, InsertMode m) {
  for (PetscInt k = 0; k < n; ++k) VecSetValue(v, idx[k], x[k], m);
  return 0;
}
inline PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
inline PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
inline PetscErrorCode VecWAXPY(Vec w, PetscScalar alpha, Vec x, Vec y) {
  const size_t n = x->a.size();
  w->a.resize(n);
  if (alpha == 1.0) {
    for (size_t i = 0; i < n; ++i) w->a[i] = y->a[i] + x->a[i];
  } else if (alpha == -1.0) {
    for (size_t i = 0; i < n; ++i) w->a[i] = y->a[i] - x->a[i];
  } else if (alpha == 0.0) {
    for (size_t i = 0; i < n; ++i) w->a[i] = y->a[i];
  } else {
    for (size_t i = 0; i < n; ++i) w->a[i] = alpha * x->a[i] + y->a[i];
  }
  return 0;
}
inline PetscErrorCode VecPointwiseMax(Vec w, Vec x, Vec y) {
  for (size_t i = 0; i < w->a.size(); ++i) w->a[i] = PetscMax(x->a[i], y->a[i]);
  return 0;
}
inline PetscErrorCode VecPointwiseMult(Vec w, Vec x, Vec y) {
  for (size_t i = 0; i < w->a.size(); ++i) w->a[i] = x->a[i] * y->a[i];
  return 0;
}
inline PetscErrorCode VecScale(Vec x, PetscScalar alpha) {
  if (alpha == 1.0) return 0;
  if (alpha == 0.0) return VecZeroEntries(x);
  for (double& v : x->a) v = alpha * v;
  return 0;
}
inline PetscErrorCode VecExp(Vec x) {
  for (double& v : x->a) v = std::exp(v);
  return 0;
}
inline PetscErrorCode VecMAXPY(Vec y, PetscInt nv, const PetscScalar* alpha, Vec* x) {
  PetscInt j = 0;
  for (; j + 1 < nv; j += 2) {
    const double a0 = alpha[j], a1 = alpha[j + 1];
    const double *x0 = x[j]->a.data(), *x1 = x[j + 1]->a.data();
    for (size_t i = 0; i < y->a.size(); ++i) y->a[i] += a0 * x0[i] + a1 * x1[i];
  }
  for (; j < nv; ++j) {
    const double a0 = alpha[j];
    const double* x0 = x[j]->a.data();
    for (size_t i = 0; i < y->a.size(); ++i) y->a[i] += a0 * x0[i];
  }
  return 0;
}
inline PetscErrorCode VecDot(Vec x, Vec y, PetscScalar* r) {
  double s = 0.0;
  for (size_t i = 0; i < x->a.size(); ++i) s += y->a[i] * x->a[i];
  *r = s;
  return 0;
}
inline PetscErrorCode VecSum(Vec x, PetscScalar* r) {
  double s = 0.0;
  for (double v : x->a) s += v;
  *r = s;
  return 0;
}
inline PetscErrorCode VecView(Vec, PetscViewer) { return 0; }

// ----------------------------------------------------------------- IS / VecScatter
inline PetscErrorCode ISCreateGeneral(MPI_Comm, PetscInt n, const PetscInt* idx, PetscCopyMode, IS* is) {
  *is = new _p_IS();
  (*is)->idx.assign(idx, idx + n);
  return 0;
}
inline PetscErrorCode ISDestroy(IS* is) {
  delete *is;
  *is = nullptr;
  return 0;
}
inline PetscErrorCode ISLocalToGlobalMappingDestroy(ISLocalToGlobalMapping* m) {
  delete *m;
  *m = nullptr;
  return 0;
}
inline PetscErrorCode VecScatterCreate(Vec, IS from, Vec, IS, VecScatter* sc) {
  *sc = new _p_VecScatter();
  (*sc)->from = from->idx;
  return 0;
}
inline PetscErrorCode VecScatterBegin(VecScatter sc, Vec x, Vec y, InsertMode m, ScatterMode) {
  for (size_t k = 0; k < sc->from.size(); ++k) {
    if (m == ADD_VALUES)
      y->a[k] += x->a.at((size_t)sc->from[k]);
    else
      y->a[k] = x->a.at((size_t)sc->from[k]);
  }
  return 0;
}
inline PetscErrorCode VecScatterEnd(VecScatter, Vec, Vec, InsertMode, ScatterMode) { return 0; }
inline PetscErrorCode VecScatterDestroy(VecScatter* sc) {
  delete *sc;
  *sc = nullptr;
  return 0;
}
inline PetscErrorCode VecGetSubVector(Vec x, IS is, Vec* y) {
  *y = new _p_Vec();
  for (PetscInt i : is->idx) (*y)->a.push_back(x->a.at((size_t)i));
  return 0;
}
inline PetscErrorCode VecRestoreSubVector(Vec x, IS is, Vec* y) {
  for (size_t k = 0; k < is->idx.size(); ++k) x->a[(size_t)is->idx[k]] = (*y)->a[k];
  delete *y;
  *y = nullptr;
  return 0;
}

// ----------------------------------------------------------------- Mat (AIJ)
inline PetscErrorCode MatCreate(MPI_Comm, Mat* A) { *A = new _p_Mat(); return 0; }
inline PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt M, PetscInt N) {
  A->rows = m >= 0 ? m : M;
  A->cols = n >= 0 ? n : N;
  return 0;
}
inline PetscErrorCode MatSetType(Mat, MatType) { return 0; }
inline PetscErrorCode MatSetFromOptions(Mat) { return 0; }
inline PetscErrorCode MatMPIAIJSetPreallocation(Mat, PetscInt, const PetscInt*, PetscInt, const PetscInt*) { return 0; }
inline PetscErrorCode MatSeqAIJSetPreallocation(Mat, PetscInt, const PetscInt*) { return 0; }
inline PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt* im, PetscInt n, const PetscInt* in,
                                   const PetscScalar* v, InsertMode mode) {
  A->assembled = false;
  for (PetscInt r = 0; r < m; ++r) {
    for (PetscInt c = 0; c < n; ++c) {
      if (im[r] < 0 || in[c] < 0) continue;  // negative indices are ignored, as in PETSc
      if (im[r] >= A->rows || in[c] >= A->cols) {
        std::fprintf(stderr, "PETSc shim: MatSetValues (%d,%d) outside %dx%d\n", im[r], in[c], A->rows, A->cols);
        std::abort();
      }
      auto key = std::make_pair(im[r], in[c]);
      if (mode == ADD_VALUES)
        A->stash[key] += v[r * n + c];
      else
        A->stash[key] = v[r * n + c];
    }
  }
  return 0;
}
inline PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode m) {
  return MatSetValues(A, 1, &i, 1, &j, &v, m);
}
inline PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
inline PetscErrorCode MatAssemblyEnd(Mat A, MatAssemblyType) {
  A->rowptr.assign((size_t)A->rows + 1, 0);
  A->colidx.clear();
  A->val.clear();
  for (auto& kv : A->stash) A->rowptr[(size_t)kv.first.first + 1]++;
  for (PetscInt r = 0; r < A->rows; ++r) A->rowptr[(size_t)r + 1] += A->rowptr[(size_t)r];
  for (auto& kv : A->stash) {  // std::map iterates (row, col) ascending
    A->colidx.push_back(kv.first.second);
    A->val.push_back(kv.second);
  }
  A->assembled = true;
  return 0;
}
inline PetscErrorCode MatMult(Mat A, Vec x, Vec y) {
  y->a.resize((size_t)A->rows);
  for (PetscInt r = 0; r < A->rows; ++r) {
    double sum = 0.0;
    for (PetscInt k = A->rowptr[(size_t)r]; k < A->rowptr[(size_t)r + 1]; ++k)
      sum += A->val[(size_t)k] * x->a[(size_t)A->colidx[(size_t)k]];
    y->a[(size_t)r] = sum;
  }
  return 0;
}
inline PetscErrorCode MatMultTranspose(Mat A, Vec x, Vec y) {
  y->a.assign((size_t)A->cols, 0.0);
  for (PetscInt r = 0; r < A->rows; ++r) {
    const double alpha = x->a[(size_t)r];
    for (PetscInt k = A->rowptr[(size_t)r]; k < A->rowptr[(size_t)r + 1]; ++k)
      y->a[(size_t)A->colidx[(size_t)k]] += A->val[(size_t)k] * alpha;
  }
  return 0;
}
inline PetscErrorCode MatGetOwnershipRange(Mat A, PetscInt* lo, PetscInt* hi) {
  *lo = 0;
  *hi = A->rows;
  return 0;
}
inline PetscErrorCode MatGetOwnershipRangeColumn(Mat A, PetscInt* lo, PetscInt* hi) {
  *lo = 0;
  *hi = A->cols;
  return 0;
}
inline PetscErrorCode MatGetLocalSize(Mat A, PetscInt* m, PetscInt* n) {
  if (m) *m = A->rows;
  if (n) *n = A->cols;
  return 0;
}
inline PetscErrorCode MatGetSize(Mat A, PetscInt* m, PetscInt* n) { return MatGetLocalSize(A, m, n); }
inline PetscErrorCode MatCreateVecs(Mat A, Vec* right, Vec* left) {
  if (right) VecCreateSeq(PETSC_COMM_SELF, A->cols, right);
  if (left) VecCreateSeq(PETSC_COMM_SELF, A->rows, left);
  return 0;
}
inline PetscErrorCode MatDestroy(Mat* A) {
  delete *A;
  *A = nullptr;
  return 0;
}
inline PetscErrorCode MatView(Mat, PetscViewer) { return 0; }
