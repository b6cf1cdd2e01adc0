// Device steps of the batched block Davidson (sm_100a), float64/complex128.
//
//   gwb_residual        r = hx - eps x, |r| per band      (gradwave solvers/davidson.py:656-657)
//   gwb_conv_stats      max |r| and max_k #(|r| > tol)    (davidson.py:691-698)
//   gwb_select_worst    the n_add largest |r| per k       (davidson.py:729-730)
//   gwb_precond_teter   TPA filter + unit rows            (davidson.py:732-743,
//                                                           solvers/precond.py:20-39)
//   gwb_subspace_insert new columns/rows of s = v^H H v   (davidson.py:648-649)
//   gwb_chol_inv        Cholesky G = L L^H and L^-1       (davidson.py:195-222, CholQR)
//
// All reductions run in float64 in a fixed order (deterministic).
#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace gwb {

template <int NT> __device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = l < NT / 32 ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (l == 0) red[0] = v;
  }
  __syncthreads();
  v = red[0];
  __syncthreads();
  return v;
}

// one CTA per (k, band)
__global__ void __launch_bounds__(256) k_residual(int npw, const cplx<double>* __restrict__ x, int64_t xk,
                                                  const cplx<double>* __restrict__ hx, int64_t hk,
                                                  const double* __restrict__ eig, int64_t ek,
                                                  cplx<double>* __restrict__ r, int64_t rk,
                                                  double* __restrict__ rn, int nb) {
  __shared__ double red[8];
  const int k = blockIdx.x / nb, b = blockIdx.x % nb;
  const double e = eig[k * ek + b];
  const cplx<double>* xr = x + k * xk + (int64_t)b * npw;
  const cplx<double>* hr = hx + k * hk + (int64_t)b * npw;
  cplx<double>* rr = r + k * rk + (int64_t)b * npw;
  double acc = 0.0;
  for (int g = threadIdx.x; g < npw; g += blockDim.x) {
    const cplx<double> v = hr[g] - scale(xr[g], e);
    rr[g] = v;
    acc += norm2(v);
  }
  acc = block_sum<256>(acc, red);
  if (threadIdx.x == 0) rn[(int64_t)k * nb + b] = sqrt(acc);
}

__global__ void k_conv_stats(const double* __restrict__ rn, int nk, int nb, double tol, double* __restrict__ out) {
  __shared__ double smax[32];
  __shared__ int scnt[32];
  // thread t handles k = t (nk <= 1024 per launch chunk loop)
  double mx = 0.0;
  int best = 0;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) {
    int c = 0;
    for (int b = 0; b < nb; ++b) {
      const double v = rn[(int64_t)k * nb + b];
      if (!(v <= mx)) mx = v;  // NaN propagates as "not converged"
      c += (v > tol || v != v) ? 1 : 0;
    }
    best = max(best, c);
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double om = __shfl_xor_sync(0xffffffffu, mx, o);
    if (!(om <= mx)) mx = om;
    best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    smax[w] = mx;
    scnt[w] = best;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
      if (!(smax[i] <= mx)) mx = smax[i];
      best = max(best, scnt[i]);
    }
    out[0] = mx;
    out[1] = (double)best;
  }
}

// Stable descending order by |r|: rank = #(larger) + #(equal and earlier).
__global__ void k_select_worst(const double* __restrict__ rn, int nb, int n_add, int* __restrict__ sel) {
  const int k = blockIdx.x;
  const double* row = rn + (int64_t)k * nb;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const double v = row[b];
    int rank = 0;
    for (int c = 0; c < nb; ++c) {
      const double u = row[c];
      rank += (u > v || (u == v && c < b)) ? 1 : 0;
    }
    if (rank < n_add) sel[(int64_t)k * n_add + rank] = b;
  }
}

// TPA coefficient K(x) = p / (p + 16 x^4), p = 27 + 18x + 12x^2 + 8x^3, float64.
__device__ __forceinline__ double tpa(double tg, double tband) {
  const double x = tg / fmax(tband, 1e-12);
  const double x2 = x * x;
  const double p = 27.0 + 18.0 * x + 12.0 * x2 + 8.0 * x2 * x;
  return p / (p + 16.0 * x2 * x2);
}

// one CTA per (k, selected slot): t_band = <x|T|x>, d = K r, d /= |d|
__global__ void __launch_bounds__(256) k_precond_teter(int npw, int nb, int n_add,
                                                       const cplx<double>* __restrict__ x, int64_t xk,
                                                       const cplx<double>* __restrict__ r, int64_t rk,
                                                       const double* __restrict__ t,
                                                       const int* __restrict__ sel,
                                                       cplx<double>* __restrict__ d, int64_t dk) {
  __shared__ double red[8];
  const int k = blockIdx.x / n_add, s = blockIdx.x % n_add;
  const int b = sel[(int64_t)k * n_add + s];
  const cplx<double>* xr = x + k * xk + (int64_t)b * npw;
  const cplx<double>* rr = r + k * rk + (int64_t)b * npw;
  const double* tk = t + (int64_t)k * npw;
  cplx<double>* dr = d + k * dk + (int64_t)s * npw;
  double tb = 0.0;
  for (int g = threadIdx.x; g < npw; g += blockDim.x) tb += tk[g] * norm2(xr[g]);
  tb = block_sum<256>(tb, red);
  double nn = 0.0;
  for (int g = threadIdx.x; g < npw; g += blockDim.x) {
    const cplx<double> v = scale(rr[g], tpa(tk[g], tb));
    dr[g] = v;
    nn += norm2(v);
  }
  nn = sqrt(block_sum<256>(nn, red));
  if (nn > 1e-300) {
    const double inv = 1.0 / nn;
    for (int g = threadIdx.x; g < npw; g += blockDim.x) dr[g] = scale(dr[g], inv);
  }
}

// C (nk, m, nnew) = V[:m] . HV[m0:m]^H ; S[i][j] = <v_i|H|v_j> for the new
// columns j >= m0 and their mirrored rows; the new diagonal block is Hermitised.
__global__ void k_subspace_insert(const cplx<double>* __restrict__ C, int m, int m0, cplx<double>* __restrict__ S,
                                  int lds, int64_t sk) {
  const int k = blockIdx.y;
  const int nnew = m - m0;
  const int64_t total = (int64_t)m * nnew;
  const cplx<double>* Ck = C + (int64_t)k * m * nnew;
  cplx<double>* Sk = S + k * sk;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / nnew), jj = (int)(idx % nnew);
    const int j = m0 + jj;
    const cplx<double> c = Ck[idx];
    if (i < m0) {
      Sk[(int64_t)i * lds + j] = conj(c);
      Sk[(int64_t)j * lds + i] = c;
    } else {
      const cplx<double> c2 = Ck[(int64_t)j * nnew + (i - m0)];
      cplx<double> v = scale(conj(c) + c2, 0.5);
      if (i == j) v.y = 0.0;
      Sk[(int64_t)i * lds + j] = v;
    }
  }
}

// One CTA per k: G (n x n, leading dim ld) -> lower Cholesky factor L in place
// (Cholesky-Banachiewicz, column by column), then Linv = L^-1 (lower, upper
// part zeroed) by columnwise forward substitution. info[k] = j+1 when pivot j
// is not positive (or not finite): Linv is then not written.
__global__ void __launch_bounds__(256) k_chol_inv(cplx<double>* __restrict__ G, int n, int ld, int64_t gk,
                                                  cplx<double>* __restrict__ Linv, int64_t lk,
                                                  int* __restrict__ info, int* __restrict__ flag) {
  __shared__ double red[8];
  __shared__ int bad;
  const int k = blockIdx.x;
  cplx<double>* A = G + k * gk;
  cplx<double>* Li = Linv + k * lk;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    double s = 0.0;
    for (int q = threadIdx.x; q < j; q += blockDim.x) s += norm2(A[(int64_t)j * ld + q]);
    s = block_sum<256>(s, red);
    const double dj = A[(int64_t)j * ld + j].x - s;
    if (!(dj > 0.0) || !isfinite(dj)) {
      if (threadIdx.x == 0) bad = j + 1;
      __syncthreads();
      break;
    }
    const double ljj = sqrt(dj);
    __syncthreads();
    if (threadIdx.x == 0) A[(int64_t)j * ld + j] = mk<double>(ljj, 0.0);
    const double inv = 1.0 / ljj;
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      cplx<double> acc = A[(int64_t)i * ld + j];
      for (int q = 0; q < j; ++q) acc = acc - mul_conj(A[(int64_t)i * ld + q], A[(int64_t)j * ld + q]);
      A[(int64_t)i * ld + j] = scale(acc, inv);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    info[k] = bad;
    if (bad && flag) atomicOr(flag, 2);
  }
  if (bad) return;
  // Linv column jc by forward substitution (one thread per column)
  for (int jc = threadIdx.x; jc < n; jc += blockDim.x) {
    for (int i = 0; i < jc; ++i) Li[(int64_t)i * n + jc] = mk<double>(0.0, 0.0);
    Li[(int64_t)jc * n + jc] = mk<double>(1.0 / A[(int64_t)jc * ld + jc].x, 0.0);
    for (int i = jc + 1; i < n; ++i) {
      cplx<double> acc = mk<double>(0.0, 0.0);
      for (int q = jc; q < i; ++q) acc = acc + A[(int64_t)i * ld + q] * Li[(int64_t)q * n + jc];
      Li[(int64_t)i * n + jc] = scale(acc, -1.0 / A[(int64_t)i * ld + i].x);
    }
  }
}

// Shared-memory version for n <= CHOL_SMEM_MAX: the same column-by-column
// Cholesky and forward substitution, with L and L^-1 kept on chip (the global
// version is bound by L2 latency on these tiny dependent loops). The inverse
// runs row by row: row i of L^-1 needs rows < i only, all columns in parallel.
constexpr int CHOL_SMEM_MAX = 64;
__global__ void __launch_bounds__(256) k_chol_inv_smem(cplx<double>* __restrict__ G, int n, int ld, int64_t gk,
                                                       cplx<double>* __restrict__ Linv, int64_t lk,
                                                       int* __restrict__ info, int* __restrict__ flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<double>* A = reinterpret_cast<cplx<double>*>(smem_raw);  // n*n
  cplx<double>* Li = A + n * n;                                 // n*n
  __shared__ double red[8];
  __shared__ int bad;
  const int k = blockIdx.x;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) A[i] = G[k * gk + (int64_t)(i / n) * ld + (i % n)];
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    double s = 0.0;
    for (int q = threadIdx.x; q < j; q += blockDim.x) s += norm2(A[j * n + q]);
    s = block_sum<256>(s, red);
    const double dj = A[j * n + j].x - s;
    if (!(dj > 0.0) || !isfinite(dj)) {
      if (threadIdx.x == 0) bad = j + 1;
      __syncthreads();
      break;
    }
    const double ljj = sqrt(dj), inv = 1.0 / ljj;
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      cplx<double> acc = A[i * n + j];
      for (int q = 0; q < j; ++q) acc = acc - mul_conj(A[i * n + q], A[j * n + q]);
      A[i * n + j] = scale(acc, inv);
    }
    __syncthreads();
    if (threadIdx.x == 0) A[j * n + j] = mk<double>(ljj, 0.0);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    info[k] = bad;
    if (bad && flag) atomicOr(flag, 2);
  }
  if (bad) return;
  for (int i = 0; i < n; ++i) {
    const double dinv = 1.0 / A[i * n + i].x;
    for (int jc = threadIdx.x; jc < n; jc += blockDim.x) {
      cplx<double> v;
      if (jc > i) {
        v = mk<double>(0.0, 0.0);
      } else if (jc == i) {
        v = mk<double>(dinv, 0.0);
      } else {
        cplx<double> acc = mk<double>(0.0, 0.0);
        for (int q = jc; q < i; ++q) acc = acc + A[i * n + q] * Li[q * n + jc];
        v = scale(acc, -dinv);
      }
      Li[i * n + jc] = v;
    }
    __syncthreads();
  }
  cplx<double>* Lo = Linv + k * lk;
  cplx<double>* Gw = G + k * gk;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
    Lo[i] = Li[i];
    const int r = i / n, c = i % n;
    if (c <= r) Gw[(int64_t)r * ld + c] = A[i];  // the factor in place, as the global version
  }
}

// Deterministic pseudo-random value in [-1, 1) from an integer key
// (SplitMix64 finaliser, Steele, Lea & Flood, OOPSLA 2014).
__device__ __forceinline__ double hash_unit(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// Rank repair of the expansion block (the reference's jitter for rows that
// vanish after projection, gradwave solvers/davidson.py:450-456): a row whose
// norm is below thresh is replaced by masked deterministic noise and flag
// gets bit 0. One CTA per (k, row).
__global__ void __launch_bounds__(256) k_row_repair(int npw, int n, cplx<double>* __restrict__ D, int64_t dk,
                                                    const unsigned char* __restrict__ mask, double thresh,
                                                    int* __restrict__ flag) {
  __shared__ double red[8];
  const int k = blockIdx.x / n, s = blockIdx.x % n;
  cplx<double>* row = D + k * dk + (int64_t)s * npw;
  double nn = 0.0;
  for (int g = threadIdx.x; g < npw; g += blockDim.x) nn += norm2(row[g]);
  nn = block_sum<256>(nn, red);
  if (sqrt(nn) < thresh) {
    const unsigned long long base = ((unsigned long long)k * 4099ull + (unsigned long long)s) * 1000003ull;
    for (int g = threadIdx.x; g < npw; g += blockDim.x) {
      const unsigned long long key = (base + (unsigned long long)g) * 2ull;
      row[g] = mask[(int64_t)k * npw + g] ? mk<double>(hash_unit(key), hash_unit(key + 1)) : mk<double>(0.0, 0.0);
    }
    if (threadIdx.x == 0) atomicOr(flag, 1);
  }
}

}  // namespace gwb

using namespace gwb;

extern "C" {

int gwb_residual(int32_t nk, int32_t nb, int32_t npw, const void* x, int64_t x_kstride, const void* hx,
                 int64_t hx_kstride, const double* eig, int64_t eig_kstride, void* r, int64_t r_kstride,
                 double* rn, void* stream) {
  GWB_REQUIRE(nk >= 0 && nb >= 0 && npw > 0, "bad sizes");
  if (nk == 0 || nb == 0) return GWB_OK;
  GWB_REQUIRE(x && hx && eig && r && rn, "null pointer");
  k_residual<<<nk * nb, 256, 0, (cudaStream_t)stream>>>(npw, (const cplx<double>*)x, x_kstride,
                                                       (const cplx<double>*)hx, hx_kstride, eig, eig_kstride,
                                                       (cplx<double>*)r, r_kstride, rn, nb);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

int gwb_conv_stats(int32_t nk, int32_t nb, const double* rn, double tol, double* out, void* stream) {
  GWB_REQUIRE(nk > 0 && nb > 0 && rn && out, "bad arguments");
  k_conv_stats<<<1, 256, 0, (cudaStream_t)stream>>>(rn, nk, nb, tol, out);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

int gwb_select_worst(int32_t nk, int32_t nb, const double* rn, int32_t n_add, int32_t* sel, void* stream) {
  GWB_REQUIRE(nk > 0 && nb > 0 && n_add > 0 && n_add <= nb && rn && sel, "bad arguments");
  k_select_worst<<<nk, 256, 0, (cudaStream_t)stream>>>(rn, nb, n_add, sel);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

int gwb_precond_teter(int32_t nk, int32_t nb, int32_t n_add, int32_t npw, const void* x, int64_t x_kstride,
                      const void* r, int64_t r_kstride, const double* t, const int32_t* sel, void* d,
                      int64_t d_kstride, void* stream) {
  GWB_REQUIRE(nk > 0 && nb > 0 && n_add > 0 && n_add <= nb && npw > 0, "bad sizes");
  GWB_REQUIRE(x && r && t && sel && d, "null pointer");
  k_precond_teter<<<nk * n_add, 256, 0, (cudaStream_t)stream>>>(npw, nb, n_add, (const cplx<double>*)x, x_kstride,
                                                               (const cplx<double>*)r, r_kstride, t, sel,
                                                               (cplx<double>*)d, d_kstride);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

int gwb_subspace_insert(int32_t nk, int32_t m, int32_t m0, const void* C, void* S, int32_t lds,
                        int64_t s_kstride, void* stream) {
  GWB_REQUIRE(nk > 0 && m > 0 && m0 >= 0 && m0 < m && lds >= m, "bad sizes");
  GWB_REQUIRE(C && S, "null pointer");
  const int64_t total = (int64_t)m * (m - m0);
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 1024);
  dim3 grid(blocks, nk);
  k_subspace_insert<<<grid, 256, 0, (cudaStream_t)stream>>>((const cplx<double>*)C, m, m0, (cplx<double>*)S, lds,
                                                           s_kstride);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

int gwb_chol_inv(int32_t nk, int32_t n, void* G, int32_t ldg, int64_t g_kstride, void* Linv,
                 int64_t linv_kstride, int32_t* info, int32_t* flag, void* stream) {
  GWB_REQUIRE(nk > 0 && n > 0 && ldg >= n, "bad sizes");
  GWB_REQUIRE(G && Linv && info, "null pointer");
  if (n <= CHOL_SMEM_MAX) {
    const size_t sm = (size_t)2 * n * n * sizeof(cplx<double>);
    GWB_CUDA_TRY(allow_smem(k_chol_inv_smem));
    k_chol_inv_smem<<<nk, 256, sm, (cudaStream_t)stream>>>((cplx<double>*)G, n, ldg, g_kstride,
                                                          (cplx<double>*)Linv, linv_kstride, info, flag);
  } else {
    k_chol_inv<<<nk, 256, 0, (cudaStream_t)stream>>>((cplx<double>*)G, n, ldg, g_kstride, (cplx<double>*)Linv,
                                                    linv_kstride, info, flag);
  }
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

int gwb_row_repair(int32_t nk, int32_t n, int32_t npw, void* D, int64_t d_kstride, const uint8_t* mask,
                   double thresh, int32_t* flag, void* stream) {
  GWB_REQUIRE(nk > 0 && n > 0 && npw > 0, "bad sizes");
  GWB_REQUIRE(D && mask && flag, "null pointer");
  k_row_repair<<<nk * n, 256, 0, (cudaStream_t)stream>>>(npw, n, (cplx<double>*)D, d_kstride, mask, thresh, flag);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

}  // extern "C"
