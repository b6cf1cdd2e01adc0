// Whole-transform DFTs in registers: one thread holds all N points of a
// transform in a local array and runs a fully unrolled mixed-radix
// decimation-in-time Cooley-Tukey recursion over it (N = R M: R interleaved
// M-point DFTs, twiddles W_N^(r k), R-point DFTs across them; Cooley & Tukey,
// Math. Comp. 19 (1965) 297; Van Loan, "Computational Frameworks for the
// FFT", 1992, sec. 2.3). The recursion works in place on strided views of the
// one array, every index and every twiddle is a compile-time constant, so the
// array lives in registers and a twiddle is an immediate operand; no shared
// memory, no barriers. Meant for the short box axes (N <= 48) where a thread
// can hold a whole pencil.
//
// The twiddle constants cos/sin(2 pi k / N) come from a constexpr evaluator
// (octant reduction on the integer ratio k/N, then Taylor series on
// [0, pi/4)); they agree with the correctly rounded values to a few ulps of
// double and are rounded to float once.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace gwb {
namespace rdft_detail {

constexpr double kPi = 3.14159265358979323846264338327950288;

constexpr double sin_series(double x) {  // |x| <= pi/4
  double term = x, sum = x;
  for (int n = 1; n < 12; ++n) {
    term *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double cos_series(double x) {
  double term = 1.0, sum = 1.0;
  for (int n = 1; n < 12; ++n) {
    term *= -x * x / ((2.0 * n - 1.0) * (2.0 * n));
    sum += term;
  }
  return sum;
}
// cos(2 pi k / n) (which = 0) or sin(2 pi k / n) (which = 1)
constexpr double cis(long k, long n, int which) {
  k %= n;
  if (k < 0) k += n;
  const long q8 = (8 * k) / n;  // octant
  const double r = 2.0 * kPi * (double)(8 * k - q8 * n) / (8.0 * (double)n);
  const double cs = cos_series(r), sn = sin_series(r);
  const double h = 0.70710678118654752440;
  double cc = 0.0, ss = 0.0;
  switch (q8) {
    case 0: cc = cs; ss = sn; break;
    case 1: cc = h * (cs - sn); ss = h * (cs + sn); break;
    case 2: cc = -sn; ss = cs; break;
    case 3: cc = -h * (cs + sn); ss = h * (cs - sn); break;
    case 4: cc = -cs; ss = -sn; break;
    case 5: cc = -h * (cs - sn); ss = -h * (cs + sn); break;
    case 6: cc = sn; ss = -cs; break;
    default: cc = h * (cs + sn); ss = -h * (cs - sn); break;
  }
  return which == 0 ? cc : ss;
}

constexpr int first_radix(int n) { return n % 4 == 0 ? 4 : (n % 3 == 0 ? 3 : (n % 2 == 0 ? 2 : n)); }

template <int I, int N>
struct StaticFor {
  template <class F>
  __host__ __device__ __forceinline__ static void run(F&& f) {
    if constexpr (I < N) {
      f(std::integral_constant<int, I>{});
      StaticFor<I + 1, N>::run(f);
    }
  }
};

// v * exp(SIGN 2 pi i K / N) with compile-time K, N
template <int N, int K, int SIGN, typename T>
__host__ __device__ __forceinline__ cplx<T> twiddle(cplx<T> v) {
  constexpr int k = ((K % N) + N) % N;
  if constexpr (k == 0) {
    return v;
  } else if constexpr (2 * k == N) {
    return mk<T>(-v.x, -v.y);
  } else if constexpr (4 * k == N) {
    return SIGN > 0 ? mk<T>(-v.y, v.x) : mk<T>(v.y, -v.x);
  } else if constexpr (4 * k == 3 * N) {
    return SIGN > 0 ? mk<T>(v.y, -v.x) : mk<T>(-v.y, v.x);
  } else {
    constexpr double cd = cis(k, N, 0), sd = SIGN * cis(k, N, 1);
    const T c = (T)cd, s = (T)sd;
    return mk<T>(v.x * c - v.y * s, v.x * s + v.y * c);
  }
}

template <int R, int SIGN, typename T>
__host__ __device__ __forceinline__ void small_dft(cplx<T> (&t)[R]) {
  if constexpr (R == 2) {
    const cplx<T> a = t[0], b = t[1];
    t[0] = a + b;
    t[1] = a - b;
  } else if constexpr (R == 3) {
    const T h = (T)0.86602540378443864676;
    const cplx<T> s1 = t[1] + t[2], d = t[1] - t[2];
    const cplx<T> m = mk<T>(t[0].x - (T)0.5 * s1.x, t[0].y - (T)0.5 * s1.y);
    // SIGN i sqrt3/2 d
    const cplx<T> q = SIGN > 0 ? mk<T>(-h * d.y, h * d.x) : mk<T>(h * d.y, -h * d.x);
    t[0] = t[0] + s1;
    t[1] = m + q;
    t[2] = m - q;
  } else if constexpr (R == 4) {
    const cplx<T> a0 = t[0] + t[2], a1 = t[0] - t[2];
    const cplx<T> b0 = t[1] + t[3], dd = t[1] - t[3];
    const cplx<T> b1 = SIGN > 0 ? mk<T>(-dd.y, dd.x) : mk<T>(dd.y, -dd.x);
    t[0] = a0 + b0;
    t[2] = a0 - b0;
    t[1] = a1 + b1;
    t[3] = a1 - b1;
  }
}

// Position, within a length-N subsequence, where the in-place recursion below
// leaves output X[k]: for N = R M, X[kk + M q] lands where sub-DFT q kept its
// output kk, i.e. at q + R pos_M(kk) (digit reversal over the radix chain).
constexpr int out_pos(int n, int k) {
  if (n <= 4) return k;
  const int r = first_radix(n), m = n / r;
  return (k / m) + r * out_pos(m, k % m);
}

// In-place DFT of the length-N subsequence x[OFF + STRIDE i], outputs in
// out_pos order.
template <int N, int SIGN, int OFF, int STRIDE, typename T, int NT>
__host__ __device__ __forceinline__ void dit_ip(cplx<T> (&x)[NT]) {
  if constexpr (N == 1) {
    return;
  } else if constexpr (N <= 4) {
    cplx<T> t[N];
    StaticFor<0, N>::run([&](auto ic) { t[decltype(ic)::value] = x[OFF + STRIDE * decltype(ic)::value]; });
    small_dft<N, SIGN>(t);
    StaticFor<0, N>::run([&](auto ic) { x[OFF + STRIDE * decltype(ic)::value] = t[decltype(ic)::value]; });
  } else {
    constexpr int R = first_radix(N);
    constexpr int M = N / R;
    static_assert(R * M == N && R <= 4, "rdft: lengths with prime factors 2 and 3 only");
    StaticFor<0, R>::run([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      dit_ip<M, SIGN, OFF + STRIDE * r, STRIDE * R>(x);
    });
    StaticFor<0, M>::run([&](auto kc) {
      constexpr int kk = decltype(kc)::value;
      constexpr int slot = STRIDE * R * out_pos(M, kk);  // where every sub-DFT keeps its output kk
      cplx<T> t[R];
      StaticFor<0, R>::run([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        t[r] = twiddle<N, r * kk, SIGN>(x[OFF + STRIDE * r + slot]);
      });
      small_dft<R, SIGN>(t);
      StaticFor<0, R>::run([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        x[OFF + STRIDE * q + slot] = t[q];
      });
    });
  }
}

}  // namespace rdft_detail

// DFT of x (natural order): X[k] = sum_n x[n] exp(SIGN 2 pi i n k / N),
// unnormalised, left in x at position out_pos(N, k).
template <int N, int SIGN, typename T>
__host__ __device__ __forceinline__ void rdft_perm(cplx<T> (&x)[N]) {
  rdft_detail::dit_ip<N, SIGN, 0, 1>(x);
}

// The same with the output in natural order (a compile-time renaming).
template <int N, int SIGN, typename T>
__host__ __device__ __forceinline__ void rdft(cplx<T> (&x)[N]) {
  using namespace rdft_detail;
  rdft_perm<N, SIGN>(x);
  cplx<T> y[N];
  StaticFor<0, N>::run([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    y[k] = x[out_pos(N, k)];
  });
  StaticFor<0, N>::run([&](auto kc) { x[decltype(kc)::value] = y[decltype(kc)::value]; });
}

}  // namespace gwb
