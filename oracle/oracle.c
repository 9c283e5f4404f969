#include "oracle.h"
#include <xmmintrin.h>
#include <omp.h>
uint32_t te_fnv1a(const uint32_t* w, size_t n) {
  uint32_t h = 0x811c9dc5u;
  for (size_t i = 0; i < n; i++) h = (h ^ w[i]) * 0x01000193u;
  return h;
}
/* Flush-to-zero + denormals-are-zero on every OpenMP worker and the caller. */
void te_set_ftz(int on) {
  unsigned bits = 0x8000u | 0x0040u;
#pragma omp parallel
  { unsigned c = _mm_getcsr(); _mm_setcsr(on ? (c | bits) : (c & ~bits)); }
  unsigned c = _mm_getcsr(); _mm_setcsr(on ? (c | bits) : (c & ~bits));
}
