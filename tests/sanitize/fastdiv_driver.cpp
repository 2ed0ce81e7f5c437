// Host check of the kernels' flat-index division (exo::FastDiv in
// exocubed_b200/csrc/exo_internal.h, the same host/device code the kernels
// run), built with AddressSanitizer and UndefinedBehaviorSanitizer by
// tests/test_sanitizers_host.py: FastDiv(d)(n) == n / d for every divisor the
// kernels use (L, N, nc1 = L + 6, nc2 = nc3 = N + 6) across its valid range
// n < 2^40 / (d - 1), including the flat indices of large grids with thin
// columns, whose 72-bit products overflowed a plain 64-bit multiply.  Exit
// status 0 when all hold.
#include <cstdint>
#include <cstdio>
#include <random>

#include "../../exocubed_b200/csrc/exo_internal.h"

static uint64_t limit_of(uint64_t d) {
  uint64_t lim = d > 1 ? (1ull << 40) / (d - 1) : (1ull << 32);
  return lim < (1ull << 32) ? lim : (1ull << 32);
}

static int check(unsigned d, std::mt19937_64& rng, long* count) {
  const exo::FastDiv f = exo::make_fastdiv(d);
  const uint64_t lim = limit_of(d);
  auto one = [&](uint64_t n) {
    if (n >= lim) return 0;
    ++*count;
    const unsigned q = f((unsigned)n);
    if (q != (unsigned)(n / d)) {
      std::printf("FastDiv(%u)(%llu) = %u, want %llu\n", d, (unsigned long long)n, q,
                  (unsigned long long)(n / d));
      return 1;
    }
    return 0;
  };
  int bad = 0;
  for (uint64_t n = 0; n < 4096; ++n) bad += one(n);
  for (uint64_t k = 1; k < 64; ++k) {  // around multiples of d and the range end
    bad += one(k * d - 1) + one(k * d) + one(k * d + 1);
    bad += one(lim - k);
  }
  std::uniform_int_distribution<uint64_t> u(0, lim - 1);
  for (int k = 0; k < 20000; ++k) bad += one(u(rng));
  return bad;
}

int main() {
  std::mt19937_64 rng(12345);
  long count = 0;
  int bad = 0;
  for (unsigned d = 1; d <= 1100; ++d) bad += check(d, rng, &count);
  for (unsigned d = 1100; d <= 12000; d += 37) bad += check(d, rng, &count);
  // the update kernel's split of a 1700^2 x 6 x L = 1 grid (flat index up to
  // 6 N^2 L - 1 by L, then N, then N)
  {
    const unsigned N = 1700, L = 1;
    const exo::FastDiv fl = exo::make_fastdiv(L), fn = exo::make_fastdiv(N);
    const unsigned tid = 6u * N * N * L - 1;
    const unsigned r1 = fl(tid), r2 = fn(r1), r3 = fn(r2);
    if (r1 != tid / L || r2 != r1 / N || r3 != r2 / N || r3 != 5) {
      std::printf("large-grid split wrong: %u %u %u\n", r1, r2, r3);
      ++bad;
    }
  }
  if (bad) {
    std::printf("fastdiv: %d failures in %ld checks\n", bad, count);
    return 1;
  }
  std::printf("fastdiv: ok (%ld checks)\n", count);
  return 0;
}
