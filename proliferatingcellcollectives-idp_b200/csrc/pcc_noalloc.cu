// Soft-model force assembly that allocates no device memory.
//
// Who needs this: a host that hands this library only memory it already owns
// and forbids it from allocating -- for instance a serving loop that admits
// colonies against a fixed HBM budget and accounts every byte through its own
// pool, or a latency-critical stepping loop that shares the GPU with other
// colonies' streams, where a cudaMalloc/cudaFree (cudaFree waits for the whole
// device) would stall work that is not its own.  pcc_soft_forces_noalloc takes
// the contacts and cell diameters in device buffers the caller owns and writes
// force/torque and stress into caller-owned device buffers.  Its intermediates
// (Hertz magnitudes, per-cell incidence lists) live in one file-scope device
// array, g_noalloc_scratch, of fixed size; nothing here calls cudaMalloc,
// cudaFree or any allocating library routine.
//
// Limits and sharing: at most kNoallocMaxCells cells and kNoallocMaxContacts
// contacts per call (larger calls return PCC_ERR_CAPACITY before touching the
// GPU).  Every gid_i / gid_j must be a cell index in [0, n): a contact with an
// id outside that range is skipped on the device (no scratch or output entry
// is touched for it), a flag in the scratch records it, and the call returns
// PCC_ERR_BOUNDS.  To read that flag the call waits for its own work on
// `stream` before it returns.  Every call on a device uses the same scratch
// array, which keeps the previous call's contents; the counters and the flag
// that must start at zero are cleared on the caller's stream at the start of
// each call.  Calls that overlap on the
// GPU (two streams, or two host threads) race on the scratch and must not be
// issued concurrently on one device.
//
// The first call on each device resolves the device address of the scratch
// array with cudaGetSymbolAddress while that device is current (the host-side
// name of a __device__ array is only a stand-in and must never be passed to a
// kernel); later calls reuse the cached address.  Make the first call on a
// device before any stream capture on it.  With lazy module loading (the
// CUDA 12 default) that first call, and the first launch of each kernel here,
// may also make the driver load this file's device code, which takes device
// memory of the driver's own; warm calls allocate nothing.
#include <cstdio>
#include <mutex>

#include "pcc_common.cuh"

namespace {

constexpr long long kNoallocMaxCells = 65536;
constexpr long long kNoallocMaxContacts = 393216;
constexpr int kNoallocMaxDevices = 64;

// Scratch layout (bytes, each part 256-byte aligned):
//   fel       kNoallocMaxContacts doubles     Hertz force magnitudes
//   cnt       kNoallocMaxCells + 1 ints        incidence counts  (cleared per call)
//   cursor    kNoallocMaxCells + 1 ints        fill cursors      (cleared per call)
//   off       kNoallocMaxCells + 1 ints        incidence offsets
//   ent       2 kNoallocMaxContacts ints       incidence entries (2c + side)
//   flag      1 unsigned                       out-of-range contact seen (cleared per call)
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kFelBytes = align256(sizeof(double) * kNoallocMaxContacts);
constexpr size_t kCellIntBytes = align256(sizeof(int) * (kNoallocMaxCells + 1));
constexpr size_t kEntBytes = align256(sizeof(int) * 2 * kNoallocMaxContacts);
constexpr size_t kFlagBytes = 256;
constexpr size_t kScratchBytes = kFelBytes + 3 * kCellIntBytes + kEntBytes + kFlagBytes;  // 6.75 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoallocMaxDevices] = {};

__device__ __forceinline__ double pow15_na(double x) {
  const double s = __dsqrt_rn(x);
  const double r = fma(-s, s, x);
  const double ds = r / (2.0 * s);
  const double p = x * s;
  const double pe = fma(x, s, -p);
  return p + (pe + x * ds);
}

// A contact whose ids are not both cell indices in [0, n) is left out.
__device__ __forceinline__ bool na_ids_ok(int a, int b, long long n) {
  return (unsigned)a < (unsigned long long)n && (unsigned)b < (unsigned long long)n;
}

__global__ void k_na_fel(const int* __restrict__ gi, const int* __restrict__ gj, const double* __restrict__ sd,
                         long long m, long long n, const double* __restrict__ diam, double kcc,
                         double* __restrict__ fel, int* __restrict__ cnt, unsigned* __restrict__ flag) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m) return;
  const int a = gi[c], b = gj[c];
  if (!na_ids_ok(a, b, n)) {
    fel[c] = 0.0;
    atomicOr(flag, 1u);
    return;
  }
  atomicAdd(&cnt[a], 1);
  atomicAdd(&cnt[b], 1);
  const double overlap = -sd[c];
  if (overlap <= 0.00) {
    fel[c] = 0.0;
    return;
  }
  const double R1 = pcc::dvd(diam[a], 2.0), R2 = pcc::dvd(diam[b], 2.0);
  const double R_eff = __dsqrt_rn(pcc::dvd(pcc::mul(R1, R2), pcc::add(R1, R2)));
  fel[c] = pcc::mul(pcc::mul(R_eff, kcc), pow15_na(overlap));
}

// Exclusive scan of n+1 counts by one block (n is at most kNoallocMaxCells).
__global__ void k_na_scan(const int* __restrict__ cnt, long long n, int* __restrict__ off) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  const long long per = (n + 1 + 1023) / 1024;
  const long long b = t * per, e = (b + per < n + 1) ? b + per : n + 1;
  int s = 0;
  for (long long i = b; i < e; ++i) s += cnt[i];
  part[t] = s;
  __syncthreads();
  for (int w = 1; w < 1024; w <<= 1) {
    int v = t >= w ? part[t - w] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = t ? part[t - 1] : 0;
  for (long long i = b; i < e; ++i) {
    off[i] = run;
    run += cnt[i];
  }
}

__global__ void k_na_fill(const int* __restrict__ gi, const int* __restrict__ gj, long long m, long long n,
                          const int* __restrict__ off, int* __restrict__ cursor, int* __restrict__ ent) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m) return;
  const int a = gi[c], b = gj[c];
  if (!na_ids_ok(a, b, n)) return;
  ent[off[a] + atomicAdd(&cursor[a], 1)] = (int)(2 * c);
  ent[off[b] + atomicAdd(&cursor[b], 1)] = (int)(2 * c + 1);
}

// Per cell: sort its incidence entries (short lists) into ascending contact
// order, then add the force, torque and stress of each overlapping contact in
// that order (the order of the reference's VecSetValues ADD stream per cell).
__global__ void k_na_gather(long long n, const int* __restrict__ off, int* __restrict__ ent,
                            const double* __restrict__ sd, const double* __restrict__ normal,
                            const double* __restrict__ r_i, const double* __restrict__ r_j,
                            const double* __restrict__ s_i, const double* __restrict__ s_j,
                            const double* __restrict__ fel, double* __restrict__ force, double* __restrict__ stress) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = off[i], e = off[i + 1];
  for (int k = b + 1; k < e; ++k) {
    int x = ent[k], j = k - 1;
    while (j >= b && ent[j] > x) {
      ent[j + 1] = ent[j];
      --j;
    }
    ent[j + 1] = x;
  }
  double F[6] = {0, 0, 0, 0, 0, 0};
  double sg = 0.0;
  for (int k = b; k < e; ++k) {
    const int en = ent[k];
    const long long q = en >> 1;
    if (-sd[q] <= 0.00) continue;
    const double fe = fel[q];
    const double fi[3] = {pcc::mul(normal[3 * q], fe), pcc::mul(normal[3 * q + 1], fe),
                          pcc::mul(normal[3 * q + 2], fe)};
    double f[3], r[3], t[3];
    const double* rr = (en & 1) == 0 ? r_i + 3 * q : r_j + 3 * q;
    for (int d = 0; d < 3; ++d) {
      f[d] = (en & 1) == 0 ? fi[d] : -fi[d];
      r[d] = rr[d];
    }
    pcc::cross3(r, f, t);
    for (int d = 0; d < 3; ++d) F[d] = pcc::add(F[d], f[d]);
    for (int d = 0; d < 3; ++d) F[3 + d] = pcc::add(F[3 + d], t[d]);
    sg = pcc::add(sg, pcc::mul((en & 1) == 0 ? s_i[q] : s_j[q], fe));
  }
  for (int d = 0; d < 6; ++d) force[6 * i + d] = F[d];
  stress[i] = sg;
}

}  // namespace

extern "C" pcc_status pcc_soft_forces_noalloc(const int* gid_i, const int* gid_j, const double* sd,
                                              const double* normal, const double* r_i, const double* r_j,
                                              const double* stress_i, const double* stress_j, size_t m,
                                              const double* diameter, size_t n, double kcc, double* force,
                                              double* stress, void* stream) {
  if ((long long)n > kNoallocMaxCells || (long long)m > kNoallocMaxContacts) {
    std::fprintf(stderr,
                 "pcc_soft_forces_noalloc: %zu cells / %zu contacts exceed the fixed scratch "
                 "(at most %lld cells and %lld contacts)\n",
                 n, m, kNoallocMaxCells, kNoallocMaxContacts);
    return PCC_ERR_CAPACITY;
  }
  if (n == 0) return PCC_OK;
  if (!diameter || !force || !stress || (m && (!gid_i || !gid_j || !sd || !normal || !r_i || !r_j || !stress_i ||
                                               !stress_j)))
    return PCC_ERR_INVALID;
  // an error left pending by earlier work in the process is not this call's:
  // report it without launching (and without clearing it)
  if (cudaPeekAtLastError() != cudaSuccess) return PCC_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoallocMaxDevices) return PCC_ERR_CUDA;
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        std::fprintf(stderr, "pcc_soft_forces_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        return PCC_ERR_CUDA;
      }
      g_noalloc_ptr[dev] = p;
    }
    base = g_noalloc_ptr[dev];
  }
  unsigned char* b = static_cast<unsigned char*>(base);
  double* fel = reinterpret_cast<double*>(b);
  int* cnt = reinterpret_cast<int*>(b + kFelBytes);
  int* cursor = reinterpret_cast<int*>(b + kFelBytes + kCellIntBytes);
  int* off = reinterpret_cast<int*>(b + kFelBytes + 2 * kCellIntBytes);
  int* ent = reinterpret_cast<int*>(b + kFelBytes + 3 * kCellIntBytes);
  unsigned* flag = reinterpret_cast<unsigned*>(b + kFelBytes + 3 * kCellIntBytes + kEntBytes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // counters and the bounds flag from the previous call must start at zero
  if (cudaMemsetAsync(cnt, 0, sizeof(int) * (n + 1), s) != cudaSuccess ||
      cudaMemsetAsync(cursor, 0, sizeof(int) * (n + 1), s) != cudaSuccess ||
      cudaMemsetAsync(flag, 0, sizeof(unsigned), s) != cudaSuccess)
    return PCC_ERR_CUDA;
  const int T = pcc::kBlock;
  if (m) {
    k_na_fel<<<pcc::grid_for((long long)m, T), T, 0, s>>>(gid_i, gid_j, sd, (long long)m, (long long)n, diameter, kcc,
                                                          fel, cnt, flag);
    if (cudaGetLastError() != cudaSuccess) return PCC_ERR_CUDA;
  }
  k_na_scan<<<1, 1024, 0, s>>>(cnt, (long long)n, off);
  if (cudaGetLastError() != cudaSuccess) return PCC_ERR_CUDA;
  if (m) {
    k_na_fill<<<pcc::grid_for((long long)m, T), T, 0, s>>>(gid_i, gid_j, (long long)m, (long long)n, off, cursor,
                                                           ent);
    if (cudaGetLastError() != cudaSuccess) return PCC_ERR_CUDA;
  }
  k_na_gather<<<pcc::grid_for((long long)n, T), T, 0, s>>>((long long)n, off, ent, sd, normal, r_i, r_j, stress_i,
                                                           stress_j, fel, force, stress);
  if (cudaGetLastError() != cudaSuccess) return PCC_ERR_CUDA;
  unsigned host_flag = 0;
  if (cudaMemcpyAsync(&host_flag, flag, sizeof host_flag, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return PCC_ERR_CUDA;
  return host_flag ? PCC_ERR_BOUNDS : PCC_OK;
}
