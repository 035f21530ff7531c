// Host-side check of the BBPGD reduction chunks (pcc_bbpgd.cuh), which every
// solver form (multi-block, one-CTA, general 3D) must cut the same way: for
// constraint counts m over a wide range, chunk_lo partitions [0, m) into
// chunk_count(m) non-empty ranges whose starts are multiples of 32, with at
// most max(target, ceil(m / (256 kMaxPerThread))) chunks and one per 256
// constraints while that stays under the target.  Built by nvcc and run on
// the CPU (no device code runs); prints "ok <cases>" or the first failure.
#include <cstdio>

#include "pcc_bbpgd.cuh"

static int check(long long m, long long target) {
  const long long nc = pcc::chunk_count(m, target);
  const long long per_block = pcc::kBlock, most = per_block * pcc::kMaxPerThread;
  const long long by_block = (m + per_block - 1) / per_block, by_most = (m + most - 1) / most;
  long long want = by_block < target ? by_block : target;
  if (want < by_most) want = by_most;
  if (want < 1) want = 1;
  if (nc != want) return printf("m=%lld target=%lld: %lld chunks, expected %lld\n", m, target, nc, want), 1;
  if (pcc::chunk_lo(0, m, nc) != 0 || pcc::chunk_lo(nc, m, nc) != m)
    return printf("m=%lld: chunks do not cover [0, m)\n", m), 1;
  for (long long ch = 0; ch < nc; ++ch) {
    const long long lo = pcc::chunk_lo(ch, m, nc), hi = pcc::chunk_lo(ch + 1, m, nc);
    if (lo % 32 != 0) return printf("m=%lld chunk %lld starts at %lld\n", m, ch, lo), 1;
    if (m > 0 && hi <= lo) return printf("m=%lld chunk %lld is empty\n", m, ch), 1;
  }
  return 0;
}

int main() {
  long long cases = 0;
  const long long targets[] = {pcc::kChunkTarget, 444, 740};
  for (long long target : targets) {
    for (long long m = 0; m <= 20000; ++m, ++cases)
      if (check(m, target)) return 1;
    for (long long m = 20001; m <= 50000000; m = m * 21 / 20 + 7, ++cases)
      if (check(m, target)) return 1;
    const long long edges[] = {256 * target - 1, 256 * target, 256 * target + 1, 2048 * target - 1,
                               2048 * target, 2048 * target + 1, 614255, 921639, 5677993};
    for (long long m : edges) {
      ++cases;
      if (check(m, target)) return 1;
    }
  }
  if (pcc::chunk_count(614255) != pcc::chunk_count(614255, pcc::kChunkTarget)) return printf("default target\n"), 1;
  printf("ok %lld\n", cases);
  return 0;
}
