// Batched float64 Hermitian eigensolver for the Davidson subspace matrices
// (replaces torch.linalg.eigh in gradwave solvers/davidson.py:66-75,650).
//
// One CTA per matrix, the matrix in shared memory (m <= GWB_HEEV_MMAX), three
// textbook stages:
//   1. Householder tridiagonalisation with Hermitian reflectors
//      P_j = I - w_j u_j u_j^H, A <- P_j A P_j (Golub & Van Loan, Matrix
//      Computations, 4th ed., sec. 8.3.1, complex form); the complex
//      subdiagonal is made real by a diagonal phase D (T = D T_r D^H).
//   2. Implicit QL with Wilkinson-type shifts on the real tridiagonal T_r
//      (Bowdler, Martin, Reinsch & Wilkinson, "The QR and QL algorithms for
//      symmetric matrices", Numer. Math. 11 (1968), procedure tql2). One thread
//      runs the scalar recurrence of a sweep and records its plane rotations;
//      then every thread applies them to its rows of the eigenvector matrix Z
//      (column-major in global scratch, coalesced).
//   3. The lowest nb eigenpairs, ascending: y = Q D z with Q = P_0 ... P_{m-3},
//      one warp per eigenvector, no block barriers.
// Every loop is bounded: a QL iteration cap reports info = 1 instead of
// spinning.
#include <cmath>

#include "common.cuh"

#define GWB_HEEV_MMAX 112

namespace gwb {

constexpr int HEEV_THREADS = 256;
constexpr int QL_MAX_ITER = 60;

// Bytes of the fixed shared-memory part (matrix, vectors), 8-byte aligned end.
__host__ __device__ inline size_t heev_smem_base(int m) {
  return ((size_t)m * (m + 1) * 16 + (size_t)m * (3 * 16 + 5 * 8 + 4) + 15) / 16 * 16;
}

__device__ __forceinline__ double blk_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = l < HEEV_THREADS / 32 ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (l == 0) red[0] = v;
  }
  __syncthreads();
  v = red[0];
  __syncthreads();
  return v;
}

// S (nk, lds, lds) row-major Hermitian (both triangles filled), leading m x m.
// eig (nk, nb) ascending; U (nk, m, nb) row-major eigenvector columns;
// Z scratch (nk, m, m) float64; info (nk).
template <bool ZSMEM>
__global__ void __launch_bounds__(HEEV_THREADS, 1) k_heev_lowest(const cplx<double>* __restrict__ S, int lds,
                                                              int64_t sk, int m, int nb, double* __restrict__ eig,
                                                              cplx<double>* __restrict__ U,
                                                              double* __restrict__ Zg, int* __restrict__ info) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lda = m + 1;  // padded row stride of A in shared memory
  cplx<double>* A = reinterpret_cast<cplx<double>*>(smem_raw);  // m*lda
  cplx<double>* pv = A + m * lda;                                // m  (p, then q)
  cplx<double>* ec = pv + m;                                     // m  complex subdiagonal
  cplx<double>* ph = ec + m;                                     // m  phases
  double* d = reinterpret_cast<double*>(ph + m);                 // m
  double* er = d + m;                                            // m
  double* wv = er + m;                                           // m  reflector scales
  double* rc = wv + m;                                           // m  rotation cosines
  double* rs = rc + m;                                           // m  rotation sines
  int* order = reinterpret_cast<int*>(rs + m);                   // m
  __shared__ double red[HEEV_THREADS / 32];
  __shared__ int s_ctl[4];  // 0: mm, 1: lowest rotation index, 2: converged-l flag, 3: fail
  const int k = blockIdx.x, tid = threadIdx.x;
  const cplx<double>* Sk = S + k * sk;
  // Z(row r, col i) at Z[i*m + r]: in shared memory when it fits (the global
  // scratch then holds the rotation log), else in the global scratch
  double* Zglob = Zg + (int64_t)k * m * m;
  double* Z = ZSMEM ? reinterpret_cast<double*>(smem_raw + heev_smem_base(m)) : Zglob;

  for (int i = tid; i < m * m; i += blockDim.x) A[(i / m) * lda + (i % m)] = Sk[(int64_t)(i / m) * lds + (i % m)];
  __syncthreads();

  // ---- 1. tridiagonalisation -------------------------------------------
  for (int j = 0; j + 2 < m; ++j) {
    const int r0 = j + 1, nr = m - r0;
    double s2 = 0.0;
    for (int r = r0 + tid; r < m; r += blockDim.x) s2 += norm2(A[r * lda + j]);
    s2 = blk_sum(s2, red);
    if (tid == 0) d[j] = A[j * lda + j].x;
    if (s2 == 0.0) {
      if (tid == 0) {
        wv[j] = 0.0;
        ec[j] = mk<double>(0.0, 0.0);
      }
      __syncthreads();
      continue;
    }
    const double sig = sqrt(s2);
    const cplx<double> x0 = A[r0 * lda + j];
    const double a0 = sqrt(norm2(x0));
    const cplx<double> phs = a0 > 0.0 ? scale(x0, 1.0 / a0) : mk<double>(1.0, 0.0);
    const double w = 1.0 / (sig * (sig + a0));
    __syncthreads();
    if (tid == 0) {
      A[r0 * lda + j] = x0 + scale(phs, sig);  // u_0; the rest of u is the column itself
      wv[j] = w;
      ec[j] = scale(phs, -sig);
    }
    __syncthreads();
    // p_r = w sum_c A[r][c] u_c = w sum_c conj(A[c][r]) u_c: TPR threads per row
    // split c (the padded row stride keeps their column reads on distinct banks)
    constexpr int TPR = 4;
    for (int b0 = 0; b0 < nr * TPR; b0 += blockDim.x) {
      const int bi = b0 + tid;
      const int rr = bi / TPR, part = bi % TPR;
      cplx<double> acc = mk<double>(0.0, 0.0);
      if (rr < nr) {
        const int r = r0 + rr;
        for (int c = r0 + part; c < m; c += TPR) acc = acc + conj_mul(A[c * lda + r], A[c * lda + j]);
      }
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 2);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 2);
      if (rr < nr && part == 0) pv[rr] = scale(acc, w);
    }
    __syncthreads();
    double kk = 0.0;
    for (int rr = tid; rr < nr; rr += blockDim.x) {
      const cplx<double> u = A[(r0 + rr) * lda + j];
      kk += u.x * pv[rr].x + u.y * pv[rr].y;  // Re(conj(u) p)
    }
    kk = 0.5 * w * blk_sum(kk, red);
    for (int rr = tid; rr < nr; rr += blockDim.x) pv[rr] = pv[rr] - scale(A[(r0 + rr) * lda + j], kk);
    __syncthreads();
    for (int idx = tid; idx < nr * nr; idx += blockDim.x) {
      const int rr = idx / nr, cc = idx % nr;
      const cplx<double> ur = A[(r0 + rr) * lda + j], uc = A[(r0 + cc) * lda + j];
      cplx<double>& a = A[(r0 + rr) * lda + r0 + cc];
      a = a - mul_conj(ur, pv[cc]) - mul_conj(pv[rr], uc);
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (m >= 2) {
      d[m - 2] = A[(m - 2) * lda + m - 2].x;
      ec[m - 2] = A[(m - 1) * lda + m - 2];
      if (m == 2) wv[0] = 0.0;
    }
    d[m - 1] = A[(m - 1) * lda + m - 1].x;
    // phases making the subdiagonal real: ph[j+1] = ph[j] e_j / |e_j|
    ph[0] = mk<double>(1.0, 0.0);
    for (int j = 0; j + 1 < m; ++j) {
      const double a = sqrt(norm2(ec[j]));
      er[j] = a;
      ph[j + 1] = a > 0.0 ? ph[j] * scale(ec[j], 1.0 / a) : ph[j];
    }
    er[m - 1] = 0.0;
    s_ctl[3] = 0;
  }
  for (int i = tid; i < m * m; i += blockDim.x) Z[i] = (i / m == i % m) ? 1.0 : 0.0;
  __syncthreads();

  // ---- 2. implicit QL on (d, er), rotations deferred to Z ---------------
  const double eps = 2.220446049250313e-16;
  if constexpr (ZSMEM) {
    // Thread 0 runs whole batches of QL sweeps and logs each sweep as a
    // header {-(mm+2), ilo} followed by its rotations {c, s} (i = mm-1 .. ilo);
    // then every thread replays the log on its rows of Z. The d/e recurrence
    // never reads Z, so batches need only two barriers each.
    // plain doubles: the per-matrix offset k*m*m is only 8-byte aligned for odd m
    double* lg = Zglob;
    const int cap = (m * m) / 2;  // entries of two doubles
    int l = 0, iter = 0;  // scalar QL state, used by thread 0 only
    while (true) {
      if (tid == 0) {
        int n = 0;
        bool done = false, fail = false;
        while (true) {
          if (l >= m) {
            done = true;
            break;
          }
          int mm = l;
          while (mm < m - 1) {
            const double dd = fabs(d[mm]) + fabs(d[mm + 1]);
            if (fabs(er[mm]) <= eps * dd) break;
            ++mm;
          }
          if (mm == l) {
            ++l;
            iter = 0;
            continue;
          }
          if (iter >= QL_MAX_ITER) {
            fail = done = true;
            break;
          }
          if (n + (mm - l) + 1 > cap) break;  // log full: replay, then continue
          ++iter;
          const int hpos = n++;
          double g = (d[l + 1] - d[l]) / (2.0 * er[l]);
          double r = sqrt(fma(g, g, 1.0));
          g = d[mm] - d[l] + er[l] / (g + copysign(r, g));
          double sn = 1.0, cs = 1.0, p = 0.0;
          int i = mm - 1;
          bool broke = false;
          // the next rotation's e and d are loaded one step ahead (they do not
          // depend on the recurrence); one rsqrt gives r, c and s
          double e_i = er[i], d_i = d[i], d_i1 = d[i + 1];
          for (; i >= l; --i) {
            const double e_nx = i > l ? er[i - 1] : 0.0;
            const double d_nx = i > l ? d[i - 1] : 0.0;
            const double f = sn * e_i, b = cs * e_i;
            const double r2 = fma(f, f, g * g);  // subspace spectra are O(1e3): no overflow
            if (r2 == 0.0) {
              er[i + 1] = 0.0;
              d[i + 1] = d_i1 - p;
              er[mm] = 0.0;
              broke = true;
              break;
            }
            const double rinv = rsqrt(r2);
            er[i + 1] = r2 * rinv;
            sn = f * rinv;
            cs = g * rinv;
            g = d_i1 - p;
            const double rr = (d_i - g) * sn + 2.0 * cs * b;
            p = sn * rr;
            d[i + 1] = g + p;
            g = cs * rr - b;
            lg[2 * n] = cs;
            lg[2 * n + 1] = sn;
            ++n;
            e_i = e_nx;
            d_i1 = d_i;
            d_i = d_nx;
          }
          lg[2 * hpos] = -(double)(mm + 2);
          lg[2 * hpos + 1] = (double)(broke ? i + 1 : l);
          if (!broke) {
            d[l] -= p;
            er[l] = g;
            er[mm] = 0.0;
          }
        }
        s_ctl[0] = n;
        s_ctl[2] = done;
        s_ctl[3] = fail;
      }
      __syncthreads();
      const int n = s_ctl[0];
      const bool done = s_ctl[2];
      for (int r = tid; r < m; r += blockDim.x) {
        int e = 0;
        while (e < n) {
          const int mm = -(int)lg[2 * e] - 2, ilo = (int)lg[2 * e + 1];
          ++e;
          double carry = Z[mm * m + r];
          int i = mm - 1;
          // four rotations at a time: all loads before the stores they precede
          for (; i - 3 >= ilo; i -= 4) {
            const double c0 = lg[2 * e], s0 = lg[2 * e + 1], c1 = lg[2 * e + 2], s1 = lg[2 * e + 3];
            const double c2 = lg[2 * e + 4], s2 = lg[2 * e + 5], c3 = lg[2 * e + 6], s3 = lg[2 * e + 7];
            e += 4;
            const double z0 = Z[i * m + r], z1 = Z[(i - 1) * m + r], z2 = Z[(i - 2) * m + r],
                         z3 = Z[(i - 3) * m + r];
            Z[(i + 1) * m + r] = s0 * z0 + c0 * carry;
            carry = c0 * z0 - s0 * carry;
            Z[i * m + r] = s1 * z1 + c1 * carry;
            carry = c1 * z1 - s1 * carry;
            Z[(i - 1) * m + r] = s2 * z2 + c2 * carry;
            carry = c2 * z2 - s2 * carry;
            Z[(i - 2) * m + r] = s3 * z3 + c3 * carry;
            carry = c3 * z3 - s3 * carry;
          }
          for (; i >= ilo; --i) {
            const double rc_ = lg[2 * e], rs_ = lg[2 * e + 1];
            ++e;
            const double zi = Z[i * m + r];
            Z[(i + 1) * m + r] = rs_ * zi + rc_ * carry;
            carry = rc_ * zi - rs_ * carry;
          }
          Z[ilo * m + r] = carry;
        }
      }
      __syncthreads();
      if (done) break;
    }
  } else {
  int l = 0, iter = 0;
  while (l < m) {
    if (tid == 0) {
      int mm = l;
      while (mm < m - 1) {
        const double dd = fabs(d[mm]) + fabs(d[mm + 1]);
        if (fabs(er[mm]) <= eps * dd) break;
        ++mm;
      }
      s_ctl[0] = mm;
      s_ctl[2] = (mm == l);
      if (mm != l) {
        if (iter >= QL_MAX_ITER) {
          s_ctl[3] = 1;
          s_ctl[2] = 1;
        } else {
          double g = (d[l + 1] - d[l]) / (2.0 * er[l]);
          double r = sqrt(fma(g, g, 1.0));
          g = d[mm] - d[l] + er[l] / (g + copysign(r, g));
          double s = 1.0, c = 1.0, p = 0.0;
          int i = mm - 1;
          bool broke = false;
          for (; i >= l; --i) {
            const double f = s * er[i], b = c * er[i];
            r = sqrt(fma(f, f, g * g));  // subspace spectra are O(1e3): no overflow
            er[i + 1] = r;
            if (r == 0.0) {
              d[i + 1] -= p;
              er[mm] = 0.0;
              broke = true;
              break;
            }
            const double rinv = 1.0 / r;
            s = f * rinv;
            c = g * rinv;
            g = d[i + 1] - p;
            r = (d[i] - g) * s + 2.0 * c * b;
            p = s * r;
            d[i + 1] = g + p;
            g = c * r - b;
            rc[i] = c;
            rs[i] = s;
          }
          s_ctl[1] = broke ? i + 1 : l;  // rotations mm-1 .. s_ctl[1] were recorded
          if (!broke) {
            d[l] -= p;
            er[l] = g;
            er[mm] = 0.0;
          }
        }
      }
    }
    __syncthreads();
    if (s_ctl[3]) break;
    if (s_ctl[2]) {
      ++l;
      iter = 0;
      __syncthreads();
      continue;
    }
    ++iter;
    const int mm = s_ctl[0], ilo = s_ctl[1];
    // column i+1 is final once rotation i is applied; the running column i is
    // carried in a register, so each rotation is one load and one store
    for (int r = tid; r < m; r += blockDim.x) {
      double carry = Z[(int64_t)mm * m + r];
      for (int i = mm - 1; i >= ilo; --i) {
        const double zi = Z[(int64_t)i * m + r];
        Z[(int64_t)(i + 1) * m + r] = rs[i] * zi + rc[i] * carry;
        carry = rc[i] * zi - rs[i] * carry;
      }
      Z[(int64_t)ilo * m + r] = carry;
    }
    __syncthreads();
  }
  }
  if (s_ctl[3]) {
    if (tid == 0) info[k] = 1;
    return;
  }
  // ascending order (stable)
  for (int i = tid; i < m; i += blockDim.x) {
    int rank = 0;
    for (int j = 0; j < m; ++j) rank += (d[j] < d[i] || (d[j] == d[i] && j < i)) ? 1 : 0;
    order[rank] = i;
  }
  __syncthreads();
  if (tid == 0) info[k] = 0;
  for (int a = tid; a < nb; a += blockDim.x) eig[(int64_t)k * nb + a] = d[order[a]];

  // ---- 3. back-transform y = Q D z, one warp per eigenvector -------------
  const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  constexpr int PER = (GWB_HEEV_MMAX + 31) / 32;
  cplx<double>* Uk = U + (int64_t)k * m * nb;
  for (int a = warp; a < nb; a += nw) {
    const int src = order[a];
    cplx<double> y[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      y[t] = r < m ? scale(ph[r], Z[(int64_t)src * m + r]) : mk<double>(0.0, 0.0);
    }
    for (int j = m - 3; j >= 0; --j) {
      const double w = wv[j];
      if (w == 0.0) continue;
      cplx<double> dot = mk<double>(0.0, 0.0);
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const int r = lane + 32 * t;
        if (r > j && r < m) dot = dot + conj_mul(A[r * lda + j], y[t]);
      }
      for (int o = 16; o > 0; o >>= 1) {
        dot.x += __shfl_xor_sync(0xffffffffu, dot.x, o);
        dot.y += __shfl_xor_sync(0xffffffffu, dot.y, o);
      }
      dot = scale(dot, w);
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const int r = lane + 32 * t;
        if (r > j && r < m) y[t] = y[t] - A[r * lda + j] * dot;
      }
    }
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      if (r < m) Uk[(int64_t)r * nb + a] = y[t];
    }
  }
}

// Z in shared memory when the whole working set fits the 227 KB opt-in limit.
static bool heev_zsmem(int m) { return heev_smem_base(m) + (size_t)m * m * 8 <= 232448; }
size_t heev_smem(int m) { return heev_smem_base(m) + (heev_zsmem(m) ? (size_t)m * m * 8 : 0); }

// One launch of the eigensolver with Z scratch z (nk * m * m float64).
static int launch_heev(int nk, int m, int nb, const void* S, int lds, int64_t sk, double* eig, void* U,
                       double* z, int* info, cudaStream_t st) {
  const size_t sm = heev_smem(m);
  if (heev_zsmem(m)) {
    GWB_CUDA_TRY(cudaFuncSetAttribute(k_heev_lowest<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_heev_lowest<true><<<nk, HEEV_THREADS, sm, st>>>((const cplx<double>*)S, lds, sk, m, nb, eig,
                                                      (cplx<double>*)U, z, info);
  } else {
    GWB_CUDA_TRY(cudaFuncSetAttribute(k_heev_lowest<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_heev_lowest<false><<<nk, HEEV_THREADS, sm, st>>>((const cplx<double>*)S, lds, sk, m, nb, eig,
                                                       (cplx<double>*)U, z, info);
  }
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

}  // namespace gwb

using namespace gwb;

extern "C" int gwb_heev_lowest(int32_t nk, int32_t m, int32_t nb, const void* S, int32_t lds, int64_t s_kstride,
                               double* eig, void* U, double* zscratch, int32_t* info, void* stream) {
  GWB_REQUIRE(nk > 0 && m > 0 && nb > 0 && nb <= m && lds >= m, "bad sizes");
  GWB_REQUIRE(m <= GWB_HEEV_MMAX, "m exceeds the shared-memory eigensolver limit (112)");
  GWB_REQUIRE(S && eig && U && zscratch && info, "null pointer");
  return launch_heev(nk, m, nb, S, lds, s_kstride, eig, U, zscratch, info, (cudaStream_t)stream);
}

extern "C" int gwb_heev_max_dim(void) { return GWB_HEEV_MMAX; }

// ---------------------------------------------------------------------------
// Allocation-free variant of gwb_heev_lowest.
//
// Who needs it: a caller whose device memory is owned by a pool allocator - a
// framework's caching allocator that holds most of HBM, or an application that
// runs under a fixed device-memory budget - cannot call cudaMalloc itself: the
// call fails when the pool already holds the memory, or escapes the budget the
// pool accounts for. This entry point takes only the caller's inputs and
// outputs and runs the eigenvector scratch Z in a fixed device array that is
// part of the library image.
//
// Limits and sharing:
//   * the array holds GWB_HEEV_NOALLOC_DOUBLES float64 (8 MiB); every GPU that
//     loads libgwb.so holds it until the process exits;
//   * a call needs nk * m * m float64 of it; larger problems are rejected with
//     GWB_ERR_ARG (use gwb_heev_lowest with caller-provided scratch);
//   * every call on a device uses the same array and leaves its last contents
//     there; the kernel writes every element of Z it reads (identity fill), so
//     nothing has to start at zero. Two calls whose kernels overlap on the GPU
//     (different streams without ordering) race on the array: order them.
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress with that device current); make that first call
//     before any stream capture.
#include <mutex>

#define GWB_HEEV_NOALLOC_DOUBLES (1 << 20)
#define GWB_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double g_heev_noalloc_z[GWB_HEEV_NOALLOC_DOUBLES];

namespace gwb {
static std::mutex g_noalloc_mu;
static double* g_noalloc_addr[GWB_NOALLOC_MAX_DEVICES] = {};
}  // namespace gwb

extern "C" int gwb_heev_lowest_noalloc(int32_t nk, int32_t m, int32_t nb, const void* S, int32_t lds,
                                       int64_t s_kstride, double* eig, void* U, int32_t* info, void* stream) {
  GWB_REQUIRE(nk > 0 && m > 0 && nb > 0 && nb <= m && lds >= m, "bad sizes");
  GWB_REQUIRE(m <= GWB_HEEV_MMAX, "m exceeds the shared-memory eigensolver limit (112)");
  GWB_REQUIRE(S && eig && U && info, "null pointer");
  if ((int64_t)nk * m * m > (int64_t)GWB_HEEV_NOALLOC_DOUBLES) {
    set_error("gwb_heev_lowest_noalloc: nk*m*m = " + std::to_string((int64_t)nk * m * m) +
              " float64 of scratch exceeds the fixed " + std::to_string(GWB_HEEV_NOALLOC_DOUBLES) +
              " (8 MiB); call gwb_heev_lowest with caller-provided scratch");
    return GWB_ERR_ARG;
  }
  int dev = 0;
  GWB_CUDA_TRY(cudaGetDevice(&dev));
  GWB_REQUIRE(dev >= 0 && dev < GWB_NOALLOC_MAX_DEVICES, "device index beyond the supported 64");
  double* z = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_heev_noalloc_z);
      if (e != cudaSuccess || p == nullptr) {
        set_error(std::string("cudaGetSymbolAddress(g_heev_noalloc_z): ") + cudaGetErrorString(e));
        return GWB_ERR_CUDA;
      }
      g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    z = g_noalloc_addr[dev];
  }
  return launch_heev(nk, m, nb, S, lds, s_kstride, eig, U, z, info, (cudaStream_t)stream);
}

