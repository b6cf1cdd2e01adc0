// In-shared-memory batched mixed-radix FFT passes (Stockham autosort) for box
// axes of length <= 128 with prime factors 2, 3, 5, 7.
//
// One pass of radix R over a batch of transforms held in shared memory: every
// butterfly j (0 <= j < n/R) of every transform reads R inputs at stride n/R,
// applies twiddles exp(sign 2 pi i (j mod Ns) r / (Ns R)), does a radix-R DFT
// and writes its R outputs to (j / Ns) Ns R + (j mod Ns) + r Ns. After the
// passes of a plan (Ns = product of the radices done so far) the transform is
// in natural order. The Stockham formulation is the textbook one (Van Loan,
// "Computational Frameworks for the FFT", 1992, sec. 1.7; Govindaraju et al.,
// SC'08); twiddles come from a host-built table of exp(-2 pi i t / n).
//
// In place: each thread keeps its butterflies of one row batch in registers
// across a barrier, so a batch is loaded completely before any output is
// stored. Rows (independent transforms) are processed in batches that fit the
// per-thread register budget.
#pragma once

#include "common.cuh"

namespace gwb {

// Radix plan of one axis: stage s has radix (code >> 4s) & 15 (packed so a
// dynamic stage index never forces the plan into local memory).
struct AxisPlan {
  int n;
  int nst;
  unsigned code;
};

// Transform length of a packed plan: the product of its radices.
__host__ __device__ constexpr int plan_length(unsigned code) {
  int n = 1;
  for (int s = 0; s < 8; ++s) {
    const int r = (int)((code >> (4 * s)) & 15u);
    if (r == 0) break;
    n *= r;
  }
  return n;
}

#define GWB_SQRT3_2 0.86602540378443864676
#define GWB_SQRT1_2 0.70710678118654752440

template <typename T> __device__ __forceinline__ void dft2(cplx<T>* v) {
  cplx<T> a = v[0], b = v[1];
  v[0] = a + b;
  v[1] = a - b;
}

template <typename T> __device__ __forceinline__ void dft3(cplx<T>* v, int sign) {
  cplx<T> t1 = v[1] + v[2];
  cplx<T> d = v[1] - v[2];
  cplx<T> m = v[0] - scale(t1, (T)0.5);
  cplx<T> q = mul_i(scale(d, (T)GWB_SQRT3_2), sign);
  v[0] = v[0] + t1;
  v[1] = m + q;
  v[2] = m - q;
}

template <typename T> __device__ __forceinline__ void dft4(cplx<T>* v, int sign) {
  cplx<T> a0 = v[0] + v[2], a1 = v[0] - v[2];
  cplx<T> b0 = v[1] + v[3], b1 = mul_i(v[1] - v[3], sign);
  v[0] = a0 + b0;
  v[2] = a0 - b0;
  v[1] = a1 + b1;
  v[3] = a1 - b1;
}

template <typename T> __device__ __forceinline__ void dft8(cplx<T>* v, int sign) {
  cplx<T> e[4] = {v[0], v[2], v[4], v[6]};
  cplx<T> o[4] = {v[1], v[3], v[5], v[7]};
  dft4(e, sign);
  dft4(o, sign);
  const T h = (T)GWB_SQRT1_2;
  // w8^1 = (1 + sign i)/sqrt2, w8^2 = sign i, w8^3 = (-1 + sign i)/sqrt2
  cplx<T> o1 = mk<T>(h * (o[1].x - sign * o[1].y), h * (o[1].y + sign * o[1].x));
  cplx<T> o2 = mul_i(o[2], sign);
  cplx<T> o3 = mk<T>(h * (-o[3].x - sign * o[3].y), h * (-o[3].y + sign * o[3].x));
  v[0] = e[0] + o[0];
  v[4] = e[0] - o[0];
  v[1] = e[1] + o1;
  v[5] = e[1] - o1;
  v[2] = e[2] + o2;
  v[6] = e[2] - o2;
  v[3] = e[3] + o3;
  v[7] = e[3] - o3;
}

template <typename T> __device__ __forceinline__ void dft6(cplx<T>* v, int sign) {
  cplx<T> e[3] = {v[0], v[2], v[4]};
  cplx<T> o[3] = {v[1], v[3], v[5]};
  dft3(e, sign);
  dft3(o, sign);
  // w6^1 = 1/2 + sign i sqrt3/2, w6^2 = -1/2 + sign i sqrt3/2
  const T c = (T)0.5, s = (T)GWB_SQRT3_2 * (T)sign;
  cplx<T> o1 = mk<T>(c * o[1].x - s * o[1].y, c * o[1].y + s * o[1].x);
  cplx<T> o2 = mk<T>(-c * o[2].x - s * o[2].y, -c * o[2].y + s * o[2].x);
  v[0] = e[0] + o[0];
  v[3] = e[0] - o[0];
  v[1] = e[1] + o1;
  v[4] = e[1] - o1;
  v[2] = e[2] + o2;
  v[5] = e[2] - o2;
}

// Generic radix-R DFT (R = 5, 7); the roots exp(-2 pi i j / R) are entries
// j * n / R of the axis twiddle table tw of length n.
template <typename T, int R>
__device__ __forceinline__ void dft_generic(cplx<T>* v, int sign, const cplx<T>* tw, int n) {
  cplx<T> y[R];
  const int step = n / R;
#pragma unroll
  for (int q = 0; q < R; ++q) {
    cplx<T> acc = v[0];
#pragma unroll
    for (int p = 1; p < R; ++p) {
      cplx<T> w = tw[((p * q) % R) * step];
      if (sign > 0) w = conj(w);
      acc = acc + v[p] * w;
    }
    y[q] = acc;
  }
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = y[q];
}

template <typename T, int R>
__device__ __forceinline__ void dft(cplx<T>* v, int sign, const cplx<T>* tw, int n) {
  if constexpr (R == 2) dft2(v);
  else if constexpr (R == 3) dft3(v, sign);
  else if constexpr (R == 4) dft4(v, sign);
  else if constexpr (R == 6) dft6(v, sign);
  else if constexpr (R == 8) dft8(v, sign);
  else dft_generic<T, R>(v, sign, tw, n);
}

// Row r of a pass lives at memory row rowmap(r): the first M+1 rows map to
// themselves and the rest to the top of the axis (the wrapped negative Miller
// indices of a pruned axis). With nrows == rowN the map is the identity.
__device__ __forceinline__ int rowmap(int r, int rowM, int nrows, int rowN) {
  return r <= rowM ? r : r + rowN - nrows;
}

// One radix-R Stockham pass over nrows transforms of length n in S.
// Element e of row r is at S[rowmap(r) * rs + e * es].
// ROWFAST: consecutive threads take consecutive rows (strided transforms);
// otherwise consecutive butterflies of one row (contiguous transforms).
template <typename T, int R, bool ROWFAST>
__device__ __forceinline__ void fft_pass(cplx<T>* S, int nrows, int n, int rs, int es, int rowM, int rowN, int Ns,
                         const cplx<T>* tw, int sign) {
  // butterflies held per thread across the barrier: at most 16 (fp32) or 8
  // (fp64) complex values, so the staging stays in registers
  constexpr int KMAX = ((sizeof(T) == 4 ? 16 : 8) / R) > 0 ? ((sizeof(T) == 4 ? 16 : 8) / R) : 1;
  const int nbf = n / R;
  const int cap = (int)blockDim.x * KMAX;
  int rows_per = cap / nbf;
  if (rows_per < 1) rows_per = 1;
  const int tstep = n / (Ns * R);
  for (int r0 = 0; r0 < nrows; r0 += rows_per) {
    const int nr = min(rows_per, nrows - r0);
    const int total = nr * nbf;
    cplx<T> v[KMAX][R];
    int dst[KMAX];
#pragma unroll
    for (int kk = 0; kk < KMAX; ++kk) {
      const int b = (int)threadIdx.x + kk * (int)blockDim.x;
      dst[kk] = -1;
      if (b < total) {
        int row, j;
        if (ROWFAST) {
          row = b % nr;
          j = b / nr;
        } else {
          j = b % nbf;
          row = b / nbf;
        }
        const int prow = rowmap(row + r0, rowM, nrows, rowN);
        const cplx<T>* src = S + prow * rs;
        const int kq = j % Ns;
#pragma unroll
        for (int r = 0; r < R; ++r) v[kk][r] = src[(j + r * nbf) * es];
#pragma unroll
        for (int r = 1; r < R; ++r) {
          cplx<T> w = tw[kq * r * tstep];
          if (sign > 0) w = conj(w);
          v[kk][r] = v[kk][r] * w;
        }
        dft<T, R>(v[kk], sign, tw, n);
        dst[kk] = prow * rs + ((j / Ns) * Ns * R + kq) * es;
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < KMAX; ++kk) {
      if (dst[kk] >= 0) {
#pragma unroll
        for (int r = 0; r < R; ++r) S[dst[kk] + r * Ns * es] = v[kk][r];
      }
    }
    __syncthreads();
  }
}

// All passes of a compile-time plan CODE (radix of stage s in bits 4s..4s+3):
// every radix, stride and twiddle step is a constant, which keeps the staging
// in registers. Caller syncs before; the last pass ends with a barrier.
template <typename T, bool ROWFAST, int SIGN, unsigned CODE, int STAGE = 0, int NS = 1>
__device__ __forceinline__ void fft_axis_ct(cplx<T>* S, int nrows, int rs, int es, int rowM, int rowN,
                                            const cplx<T>* tw) {
  constexpr int R = (int)((CODE >> (4 * STAGE)) & 15u);
  if constexpr (R != 0 && STAGE < 8) {
    constexpr int N = plan_length(CODE);
    fft_pass<T, R, ROWFAST>(S, nrows, N, rs, es, rowM, rowN, NS, tw, SIGN);
    fft_axis_ct<T, ROWFAST, SIGN, CODE, STAGE + 1, NS * R>(S, nrows, rs, es, rowM, rowN, tw);
  }
}

// All passes of one runtime axis plan (any supported length; slower: the
// radix switch costs registers). Caller syncs before (S filled); the last pass
// ends with a barrier.
template <typename T, bool ROWFAST>
__device__ void fft_axis(cplx<T>* S, int nrows, const AxisPlan& pl, int rs, int es, int rowM,
                         int rowN, const cplx<T>* tw, int sign) {
  int Ns = 1;
  for (int s = 0; s < pl.nst; ++s) {
    const int R = (int)((pl.code >> (4 * s)) & 15u);
    switch (R) {
      case 2: fft_pass<T, 2, ROWFAST>(S, nrows, pl.n, rs, es, rowM, rowN, Ns, tw, sign); break;
      case 3: fft_pass<T, 3, ROWFAST>(S, nrows, pl.n, rs, es, rowM, rowN, Ns, tw, sign); break;
      case 4: fft_pass<T, 4, ROWFAST>(S, nrows, pl.n, rs, es, rowM, rowN, Ns, tw, sign); break;
      case 5: fft_pass<T, 5, ROWFAST>(S, nrows, pl.n, rs, es, rowM, rowN, Ns, tw, sign); break;
      case 6: fft_pass<T, 6, ROWFAST>(S, nrows, pl.n, rs, es, rowM, rowN, Ns, tw, sign); break;
      case 7: fft_pass<T, 7, ROWFAST>(S, nrows, pl.n, rs, es, rowM, rowN, Ns, tw, sign); break;
      default: fft_pass<T, 8, ROWFAST>(S, nrows, pl.n, rs, es, rowM, rowN, Ns, tw, sign); break;
    }
    Ns *= R;
  }
}

// Compile-time plan when CODE != 0, else the runtime plan pl.
template <typename T, bool ROWFAST, int SIGN, unsigned CODE>
__device__ __forceinline__ void fft_any(cplx<T>* S, int nrows, const AxisPlan& pl, int rs, int es, int rowM,
                                        int rowN, const cplx<T>* tw) {
  if constexpr (CODE != 0u) {
    fft_axis_ct<T, ROWFAST, SIGN, CODE>(S, nrows, rs, es, rowM, rowN, tw);
  } else {
    fft_axis<T, ROWFAST>(S, nrows, pl, rs, es, rowM, rowN, tw, SIGN);
  }
}

}  // namespace gwb
