// Device-wide exclusive scan and stable LSD radix sort (hand-written; used by
// the broadphase bins, the incidence lists, divisions and the x-sort that
// renumbers cells every step).
#include "pcc_kernels.hpp"

namespace pcc {

namespace {

constexpr int kScanItems = 8;                      // items per thread
constexpr int kScanTile = kBlock * kScanItems;     // 2048 per block

__device__ __forceinline__ int block_exclusive_scan(int v, int* smem, int* total) {
  // Warp-shuffle scan of one value per thread across a 256-thread block.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (kBlock / 32) ? smem[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < (kBlock / 32)) smem[lane] = w;
  }
  __syncthreads();
  int base = warp ? smem[warp - 1] : 0;
  *total = smem[kBlock / 32 - 1];
  __syncthreads();
  return base + x - v;
}

__global__ void k_scan_reduce(const int* __restrict__ in, size_t n, int* __restrict__ bsum) {
  __shared__ int sm[kBlock / 32];
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += in[base + k];
  int tot;
  block_exclusive_scan(s, sm, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void k_scan_blocks(int* bsum, int nb, int* total_out) {
  __shared__ int sm[kBlock / 32];
  int carry = 0;
  for (int base = 0; base < nb; base += kBlock) {
    int i = base + threadIdx.x;
    int v = i < nb ? bsum[i] : 0;
    int tot;
    int ex = block_exclusive_scan(v, sm, &tot);
    if (i < nb) bsum[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_apply(const int* __restrict__ in, size_t n, const int* __restrict__ boff, int* __restrict__ out) {
  __shared__ int sm[kBlock / 32];
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  int tot;
  int ex = block_exclusive_scan(s, sm, &tot) + boff[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = ex;
    ex += v[k];
  }
}

// ---------------------------------------------------------------- radix sort
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kSortItems = 8;
constexpr int kSortTile = kBlock * kSortItems;  // sub-tiles of kBlock, in order
constexpr int kWarps = kBlock / 32;

__global__ void k_radix_hist(const unsigned long long* __restrict__ keys, size_t n, int shift, int nblocks,
                             int* __restrict__ hist) {
  __shared__ int cnt[kRadix];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  size_t base = (size_t)blockIdx.x * kSortTile;
  for (int k = 0; k < kSortItems; ++k) {
    size_t i = base + (size_t)k * kBlock + threadIdx.x;
    if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & (kRadix - 1)], 1);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void k_radix_scatter(const unsigned long long* __restrict__ keys, const int* __restrict__ vals, size_t n,
                                int shift, int nblocks, const int* __restrict__ offs,
                                unsigned long long* __restrict__ keys_out, int* __restrict__ vals_out) {
  __shared__ int warp_cnt[kWarps][kRadix];
  __shared__ int warp_pre[kWarps][kRadix];
  __shared__ int running[kRadix];
  __shared__ int sub_total[kRadix];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  running[t] = offs[(size_t)t * nblocks + blockIdx.x];
  for (int k = 0; k < kWarps; ++k) warp_cnt[k][t] = 0;
  __syncthreads();
  const unsigned lt_mask = (1u << lane) - 1u;
  size_t base = (size_t)blockIdx.x * kSortTile;
  for (int k = 0; k < kSortItems; ++k) {
    size_t i = base + (size_t)k * kBlock + t;
    bool valid = i < n;
    unsigned long long key = valid ? keys[i] : 0ULL;
    int val = valid ? vals[i] : 0;
    int d = valid ? (int)((key >> shift) & (kRadix - 1)) : kRadix;  // kRadix = no digit
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int rank_w = __popc(peers & lt_mask);
    int leader = __ffs(peers) - 1;
    if (valid && lane == leader) warp_cnt[w][d] = __popc(peers);
    __syncthreads();
    {
      int run = 0;
#pragma unroll
      for (int ww = 0; ww < kWarps; ++ww) {
        int c = warp_cnt[ww][t];
        warp_pre[ww][t] = run;
        run += c;
      }
      sub_total[t] = run;
    }
    __syncthreads();
    if (valid) {
      int pos = running[d] + warp_pre[w][d] + rank_w;
      keys_out[pos] = key;
      vals_out[pos] = val;
    }
    __syncthreads();
    running[t] += sub_total[t];
#pragma unroll
    for (int ww = 0; ww < kWarps; ++ww) warp_cnt[ww][t] = 0;
    __syncthreads();
  }
}

}  // namespace

cudaError_t exclusive_scan(pcc_ctx* ctx, const int* in, int* out, size_t n) {
  cudaStream_t s = ctx->stream;
  size_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 0) nb = 1;
  cudaError_t e = ctx->scan_tmp.reserve(nb + 1, 0, s);
  if (e) return e;
  int* bsum = ctx->scan_tmp.p;
  k_scan_reduce<<<(unsigned)nb, kBlock, 0, s>>>(in, n, bsum);
  k_scan_blocks<<<1, kBlock, 0, s>>>(bsum, (int)nb, out + n);
  k_scan_apply<<<(unsigned)nb, kBlock, 0, s>>>(in, n, bsum, out);
  ctx->launches += 3;
  return cudaGetLastError();
}

cudaError_t radix_sort_pairs(pcc_ctx* ctx, unsigned long long* keys, int* vals, size_t n, int bits) {
  if (n <= 1) return cudaSuccess;
  cudaStream_t s = ctx->stream;
  int nblocks = (int)((n + kSortTile - 1) / kSortTile);
  size_t hn = (size_t)kRadix * nblocks;
  cudaError_t e;
  if ((e = ctx->keys_alt.reserve(n, 0, s))) return e;
  if ((e = ctx->perm_alt.reserve(n, 0, s))) return e;
  if ((e = ctx->sort_hist.reserve(2 * hn + 1, 0, s))) return e;
  unsigned long long *ka = keys, *kb = ctx->keys_alt.p;
  int *va = vals, *vb = ctx->perm_alt.p;
  int* hist = ctx->sort_hist.p;
  int* offs = ctx->sort_hist.p + hn;
  int passes = (bits + kRadixBits - 1) / kRadixBits;
  for (int p = 0; p < passes; ++p) {
    int shift = p * kRadixBits;
    k_radix_hist<<<nblocks, kBlock, 0, s>>>(ka, n, shift, nblocks, hist);
    ctx->launches++;
    if ((e = exclusive_scan(ctx, hist, offs, hn))) return e;
    k_radix_scatter<<<nblocks, kBlock, 0, s>>>(ka, va, n, shift, nblocks, offs, kb, vb);
    ctx->launches++;
    unsigned long long* tk = ka;
    ka = kb;
    kb = tk;
    int* tv = va;
    va = vb;
    vb = tv;
  }
  if (ka != keys) {
    cudaMemcpyAsync(keys, ka, n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(vals, va, n * sizeof(int), cudaMemcpyDeviceToDevice, s);
  }
  return cudaGetLastError();
}

}  // namespace pcc
