// ref_xoro_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own xoroshiro128+ engine (ModelG/xoroshiro128plus.h,
// compiled from its source where it lies; it needs only the C++ standard
// library) through the construction NoiseGenerator performs
// (NoiseGenerator.h:68-81: std::seed_seq{baseSeed} -> seeds[rank] ->
// xoroshiro128plus::seed(uint64)) and the three libstdc++ distributions it uses
// (:99-105, :150-155).  Its output pins the oracle's restated engine.
//
// Output (text, one record per line):
//   seeds <base> <size> <s_0> ... <s_size-1>
//   raw   <base> <rank> <size> <n> <u64> ...
//   unif  <base> <rank> <size> <n> <%.17g> ...
//   var1  <base> <rank> <size> <n> ...
//   norm  <base> <rank> <size> <n> ...
//   state <seed64> <s0> <s1> <n> <u64> ...     engine seeded directly
#include "xoroshiro128plus.h"

#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <random>
#include <sstream>
#include <vector>

static xoroshiro128plus make(int base, int rank, int size) {
  std::seed_seq seq = {base};
  std::vector<unsigned int> seeds(size, 0);
  seq.generate(seeds.begin(), seeds.end());
  xoroshiro128plus g;
  g.seed(seeds[rank]);
  return g;
}

int main() {
  const int bases[] = {10, 2021, 122335456};
  const int sizes[] = {1, 4};
  const int n = 64;
  for (int base : bases)
    for (int size : sizes) {
      std::seed_seq seq = {base};
      std::vector<unsigned int> seeds(size, 0);
      seq.generate(seeds.begin(), seeds.end());
      printf("seeds %d %d", base, size);
      for (unsigned s : seeds) printf(" %u", s);
      printf("\n");
      for (int rank = 0; rank < size; ++rank) {
        {
          auto g = make(base, rank, size);
          printf("raw %d %d %d %d", base, rank, size, n);
          for (int i = 0; i < n; ++i) printf(" %" PRIu64, g());
          printf("\n");
        }
        {
          auto g = make(base, rank, size);
          std::uniform_real_distribution<double> u;
          printf("unif %d %d %d %d", base, rank, size, n);
          for (int i = 0; i < n; ++i) printf(" %.17g", u(g));
          printf("\n");
        }
        {
          auto g = make(base, rank, size);
          std::uniform_real_distribution<double> v(-std::sqrt(3.), std::sqrt(3.));
          printf("var1 %d %d %d %d", base, rank, size, n);
          for (int i = 0; i < n; ++i) printf(" %.17g", v(g));
          printf("\n");
        }
        {
          auto g = make(base, rank, size);
          std::normal_distribution<double> d;
          printf("norm %d %d %d %d", base, rank, size, n);
          for (int i = 0; i < n; ++i) printf(" %.17g", d(g));
          printf("\n");
        }
      }
    }
  const uint64_t direct[] = {0, 1, 10, 122335456, 0xFFFFFFFFull};
  for (uint64_t s : direct) {
    xoroshiro128plus g;
    g.seed(s);
    std::ostringstream os;
    os << g;  // stream format of the .rng restart file (xoroshiro128plus.h:137-142)
    printf("state %" PRIu64 " %s %d", s, os.str().c_str(), n);
    for (int i = 0; i < n; ++i) printf(" %" PRIu64, g());
    printf("\n");
  }
  return 0;
}
