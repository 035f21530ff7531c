// Force-included (g++ -include) when the reference sources are compiled as
// the CPU oracle.  Particle::divide draws the daughter length from
// std::mt19937 seeded by std::random_device (simulation/Particle.cpp:131-135),
// which is not reproducible.  This header swaps std::random_device for a
// counter-based stand-in: the k-th construction-and-call in the process
// returns pcc_division_seed(seed, k), the same 32-bit seed sequence the device
// path uses, so both sides draw identical lengths for the k-th division.
//
// Test infrastructure only.
#pragma once
#include <cstdint>
#include <random>
#include <string>

extern "C" void pcc_ref_set_division_stream(unsigned long long seed, unsigned long long next_index);
extern "C" unsigned long long pcc_ref_division_index(void);

namespace std {
struct pcc_seeded_random_device {
  using result_type = unsigned int;
  pcc_seeded_random_device() {}
  explicit pcc_seeded_random_device(const std::string&) {}
  static constexpr result_type min() { return 0; }
  static constexpr result_type max() { return 0xffffffffu; }
  double entropy() const noexcept { return 0.0; }
  result_type operator()();
};
}  // namespace std

#define random_device pcc_seeded_random_device
