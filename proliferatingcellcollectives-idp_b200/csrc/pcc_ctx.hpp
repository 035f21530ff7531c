// Host-side context of one resident colony: device buffers, stream and the
// per-step orchestration state.  Internal to libpcc_gpu.so.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <random>
#include <string>
#include <vector>

#include "pcc_common.cuh"
#include "pcc_gpu.h"

namespace pcc {

// Growable device buffer in stream-ordered memory: growth allocates, copies
// the first `keep` elements and frees the old block on the owning stream, so
// it never synchronises the device (colonies that grow side by side in one
// process keep running while another reallocates).
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  cudaStream_t owner = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFreeAsync(p, owner);
  }
  cudaError_t reserve(size_t n, size_t keep, cudaStream_t s) {
    if (n <= cap) return cudaSuccess;
    size_t nc = cap ? cap : 64;
    while (nc < n) nc = nc + nc / 2 + 64;
    T* q = nullptr;
    cudaError_t e = cudaMallocAsync(&q, nc * sizeof(T), s);
    if (e != cudaSuccess) return e;
    if (p && keep) {
      e = cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return e;
    }
    if (p) cudaFreeAsync(p, s);
    p = q;
    cap = nc;
    owner = s;
    return cudaSuccess;
  }
};

// All per-cell arrays (one set; the x-sort gathers into a second set and swaps).
struct CellBufs {
  DevBuf<double> x, y, z, q0, q1, q2, q3, len, l0, diam, ldot, imp, stress, force, vel;
  DevBuf<int> age, ncons;
  cudaError_t reserve(size_t n, size_t keep, cudaStream_t s);
  CellsView view();
  void swap(CellBufs& o);
};

struct ConsBufs {
  DevBuf<int> gi, gj, phase;
  DevBuf<double> sd, gamma, nx, ny, nz, tix, tiy, tiz, tjx, tjy, tjz, rix, riy, riz, rjx, rjy, rjz, cpx, cpy,
      cpz, si, sj;
  cudaError_t reserve(size_t n, size_t keep, cudaStream_t s);
  ConsView view();
};

// Grid barrier + reduction scratch of the persistent solver kernel.
// The arrival counter sits on a cache line of its own: every block adds to
// it at every grid barrier, while the release word and the scalars that the
// blocks read after a release share the next line.
constexpr int kTakeGroups = 8;
struct SolverScalars {
  unsigned long long arrive;     // block arrivals at grid barriers, monotonic within a launch
  unsigned long long pad0[15];
  unsigned long long released;   // ordinal of the last barrier whose reduction was published
  int converged;                 // 1 once the residual test passed
  int pad;
  long long iterations;          // BBPGD iteration count at exit
  double alpha;                  // current step size
  double residual;               // last evaluated residual
  double res0;                   // initial residual
  // cell-unit counters of the multi-block planar cell pass, two sets used by
  // alternate iterations, one counter per 128-byte line; not copied back
  alignas(128) unsigned long long take[2][kTakeGroups][16];
};
constexpr size_t kScalarsCopied = offsetof(SolverScalars, take);
static_assert(offsetof(SolverScalars, take) == 256, "counters start on their own line");

}  // namespace pcc

struct pcc_vtk_writer_state;

struct pcc_ctx {
  pcc_params params{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  int num_sms = 0;
  std::string err;

  size_t n = 0;  // resident cells
  pcc::CellBufs cells, cells_alt;

  // constraints accumulated during the current step
  size_t ncons = 0;
  pcc::ConsBufs cons;

  // detection scratch
  pcc::DevBuf<int> bin_of, bin_cnt, bin_off, bin_cursor, bin_cells, cand_cnt, cand_off;
  pcc::DevBuf<double> pk;  // packed per-cell geometry in bin order
  pcc::DevBuf<int> ghost;
  pcc::DevBuf<int> bbox;   // [6] min/max bin coordinates, [7] non-planar flag
  // candidate partner lists of the last full neighbourhood pass (list-major)
  pcc::DevBuf<int> plist, plist_n, slot_of;
  pcc::DevBuf<double> xref;  // cell positions when the lists were built
  bool list_valid = false;
  size_t list_n = 0;
  double list_tol = 0.0;

  // incidence CSR (cell -> constraint sides)
  pcc::DevBuf<int> inc_cnt, inc_off, inc_ent;

  // solver scratch
  pcc::DevBuf<double> gam_a, gam_b, g_a, g_b, gam_old;
  pcc::DevBuf<double> U, dldot, F, sig, ldot_new, imp_new, Mlin, Mrot, ldot_prev;
  pcc::DevBuf<double> partials;
  pcc::DevBuf<pcc::SolverScalars> scal;
  pcc::DevBuf<double> fel;  // soft: Hertz force magnitude per contact
  // packed operands of the planar solver
  pcc::DevBuf<int2> p_ij;
  pcc::DevBuf<double2> p_n, p_t, p_s, p_gg;
  pcc::DevBuf<double> p_gold, p_phin;
  pcc::DevBuf<double4> p_inc, p_cell, p_u;
  // ... their FP32 forms (mixed precision)
  pcc::DevBuf<float2> pf_n, pf_t, pf_s;
  pcc::DevBuf<float4> pf_inc, pf_cell, pf_u;
  bool planar = false;  // set by the last binning pass

  // Brownian external velocity (Physics.cpp:59-81, Particle.cpp:174-190): the
  // reference draws it from one process-wide std::mt19937 with the default
  // seed (Physics.cpp:19); each context holds that generator for its colony.
  std::mt19937 brown_gen;
  pcc::DevBuf<double> uext;             // 3 per cell: rotational U_ext (x, y, z)
  pcc::DevBuf<double> brown_coef;       // 3 per cell: T u1 u_k of this draw
  double* brown_host = nullptr;         // pinned staging of brown_coef
  size_t brown_host_cap = 0;
  bool uext_active = false;             // U_ext is non-zero in the current solve

  // step scratch
  pcc::DevBuf<int> div_flag, div_off;
  pcc::DevBuf<unsigned long long> keys, keys_alt;
  pcc::DevBuf<int> perm, perm_alt, sort_hist;
  pcc::DevBuf<int> scan_tmp;
  pcc::DevBuf<double> red;  // small reductions

  // host round trips: values enqueued for the next synchronisation point
  pcc::SolverScalars* scal_host = nullptr;  // pinned: BBPGD scalars of a launch not yet read
  bool bbpgd_pending = false;               // a BBPGD launch whose scalars are still on their way
  double bbpgd_pending_bytes = 0.0;         // its algorithmic bytes per iteration
  bool div_known = false;                   // div_flag / div_off / div_next describe the resident cells
  size_t div_next = 0;                      // divisions the next step commits

  pcc::DevStatus* status = nullptr;  // device
  pcc::DevStatus* status_host = nullptr;  // pinned mirror
  long long* pinned_ll = nullptr;         // pinned scratch for small read-backs
  double* pinned_d = nullptr;

  unsigned long long div_index = 0;  // divisions so far (RNG stream position)
  long long iter = 0;
  double sim_time = 0, radius = 0;
  long long launches = 0;
  int coop_blocks = 0;         // co-resident blocks of the general solver kernel
  int coop_blocks_planar = 0;  // ... of the planar one
  int coop_blocks_mixed = 0;   // ... of its mixed-precision form
  int coop_planar_tr = 0;      // ... and of their traced forms
  int coop_mixed_tr = 0;

  // VTK output: device snapshot, side stream and background writer
  pcc::DevBuf<double> vtk_dev;
  pcc::DevBuf<int> vtk_idev;
  cudaStream_t vtk_stream = nullptr;
  cudaEvent_t vtk_ev = nullptr;
  pcc_vtk_writer_state* vtk_writer = nullptr;

  // BBPGD trace of the current / last traced solve
  bool trace_active = false;
  int trace_phase = 0;
  std::string trace_dir = "logs";
  pcc::DevBuf<double> tr_part, trace_dev;
  std::vector<pcc_bbpgd_trace_step> trace_host;

  bool profiling = false;
  pcc_profile prof{};
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};
