/* Multipliers for the 64-bit multiply-with-carry generator (rnd.txt format: one per line).
 *
 * A multiplier a gives a stream of long period when p = a*2^32 - 1 is a safe prime,
 * i.e. p and (p-1)/2 = a*2^31 - 1 are both prime (Marsaglia's construction for MWC).
 * This writes the largest such a < 2^32, in descending order.  Primality: deterministic
 * Miller-Rabin for 64-bit integers with the first twelve prime bases.
 *
 * usage: mwc_multipliers <count>
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) { return (uint64_t)((u128)a * b % m); }

static uint64_t powmod(uint64_t b, uint64_t e, uint64_t m) {
  uint64_t r = 1;
  b %= m;
  while (e) {
    if (e & 1) r = mulmod(r, b, m);
    b = mulmod(b, b, m);
    e >>= 1;
  }
  return r;
}

static const uint32_t small[] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89, 97};

static int is_prime(uint64_t n) {
  if (n < 2) return 0;
  if ((n & 1) == 0) return n == 2;
  for (unsigned i = 0; i < sizeof(small) / sizeof(small[0]); i++)
    if (n % small[i] == 0) return n == small[i];
  uint64_t d = n - 1;
  int s = 0;
  while ((d & 1) == 0) { d >>= 1; s++; }
  static const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  for (unsigned i = 0; i < 12; i++) {
    uint64_t x = powmod(bases[i], d, n);
    if (x == 1 || x == n - 1) continue;
    int ok = 0;
    for (int r = 1; r < s; r++) {
      x = mulmod(x, x, n);
      if (x == n - 1) { ok = 1; break; }
    }
    if (!ok) return 0;
  }
  return 1;
}

int main(int argc, char** argv) {
  long count = argc > 1 ? atol(argv[1]) : 131072;
  /* scan blocks of candidates in parallel, keep the descending order */
  const uint64_t B = 1u << 16;
  uint64_t top = 0xFFFFFFFFull;
  long found = 0;
  uint32_t* out = (uint32_t*)malloc(sizeof(uint32_t) * (count + 1));
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  uint32_t* buf = (uint32_t*)malloc(sizeof(uint32_t) * B * nt);
  long* nb = (long*)calloc(nt, sizeof(long));
  while (found < count && top > B * nt) {
#pragma omp parallel for schedule(static, 1)
    for (int t = 0; t < nt; t++) {
      uint64_t hi = top - (uint64_t)t * B;
      long k = 0;
      for (uint64_t a = hi; a > hi - B; a--) {
        uint64_t q = (a << 31) - 1;
        uint64_t p = (a << 32) - 1;
        if (is_prime(q) && is_prime(p)) buf[(size_t)t * B + k++] = (uint32_t)a;
      }
      nb[t] = k;
    }
    for (int t = 0; t < nt && found < count; t++)
      for (long k = 0; k < nb[t] && found < count; k++) out[found++] = buf[(size_t)t * B + k];
    top -= B * nt;
  }
  for (long i = 0; i < found; i++) printf("%u\n", out[i]);
  return found == count ? 0 : 1;
}
