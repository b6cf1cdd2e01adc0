// Tridiagonal eigenvalue helpers shared by the eigensolvers: Sturm counts
// by the leading principal minors (multiplications only, rescaled to stay in
// range) and a seeded uniform value for inverse-iteration starts.
#pragma once

#include <cuda_runtime.h>

namespace gwb {

// Seeded uniform value in [-1, 1): SplitMix64 (Steele, Lea & Flood, OOPSLA 2014).
__device__ __forceinline__ double hash_pm1(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * 0x1.0p-52 - 1.0;
}

// Number of eigenvalues of the real tridiagonal (d, e) below x: sign changes
// of the leading principal minors,
// rescaled by 2^-+400 after every fourth step (the minors grow by at most
// |d_i - x| + e_i^2 per step).
__device__ __forceinline__ void sturm_step(double di, double e2i, double x, double& p0, double& p1, int& cnt) {
  constexpr double TINY = 0x1.0p-100;
  double p2 = fma(di - x, p1, -e2i * p0);
  if (p2 == 0.0) p2 = -TINY * p1;  // a zero minor takes the sign opposite to its predecessor
  cnt += (p2 < 0.0) != (p1 < 0.0);
  p0 = p1;
  p1 = p2;
}
__device__ __forceinline__ void sturm_rescale(double& p0, double& p1) {
  constexpr double BIG = 0x1.0p400, SMALL = 0x1.0p-400;
  const double mx = fmax(fabs(p0), fabs(p1));
  if (mx > BIG) {
    p0 *= SMALL;
    p1 *= SMALL;
  } else if (mx < SMALL) {
    p0 *= BIG;
    p1 *= BIG;
  }
}
__device__ __forceinline__ int sturm_count(const double* __restrict__ d, const double* __restrict__ e2, int m,
                                           double x) {
  constexpr double TINY = 0x1.0p-100;
  double p0 = 1.0, p1 = d[0] - x;
  if (p1 == 0.0) p1 = -TINY;
  int cnt = p1 < 0.0;
  int i = 1;
  for (; i + 3 < m; i += 4) {
    double dd[4], ee[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      dd[q] = d[i + q];
      ee[q] = e2[i + q - 1];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) sturm_step(dd[q], ee[q], x, p0, p1, cnt);
    sturm_rescale(p0, p1);
  }
  for (; i < m; ++i) sturm_step(d[i], e2[i - 1], x, p0, p1, cnt);
  return cnt;
}

}  // namespace gwb
