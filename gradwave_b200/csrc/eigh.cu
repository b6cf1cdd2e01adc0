// Batched float64 Hermitian eigensolver for the Davidson subspace matrices
// (replaces torch.linalg.eigh in gradwave solvers/davidson.py:66-75,650):
// the lowest nb eigenpairs of each m x m matrix, ascending. Two kernels, one
// CTA per matrix, everything in shared memory (m <= GWB_HEEV_MMAX):
//
// k_heev_tridiag (512 threads)
//   1. Householder tridiagonalisation with Hermitian reflectors
//      P_j = I - w_j u_j u_j^H, A <- P_j A P_j (Golub & Van Loan, Matrix
//      Computations, 4th ed., sec. 8.3.1, complex form) on the lower triangle,
//      two block barriers per column. Reflectors, diagonal, complex
//      subdiagonal and scales go to the caller's scratch.
// k_heev_lowest (256 threads)
//   The complex subdiagonal is made real by a diagonal phase D (T = D T_r D^H);
//   the packed reflectors sit at the front of the shared memory and the rest
//   is the working pool of:
//   2. Eigenvalues lambda_0..lambda_{nb+3} of T_r by multisection on Sturm
//      counts (8 lanes per eigenvalue, 9 sub-intervals per round). The count
//      is the number of sign changes of the leading principal minors
//      p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2}, rescaled by powers of two;
//      the computed count is exact for T_r with each e_i^2 perturbed by a few
//      ulps (Wilkinson, The Algebraic Eigenvalue Problem, ch. 5, secs. 37-40;
//      Barth, Martin & Wilkinson, Numer. Math. 9 (1967) 386). The wanted set
//      grows past nb while the next eigenvalue belongs to the same cluster.
//   3. Eigenvectors of T_r by three steps of inverse iteration (one thread per
//      vector; Gaussian elimination with partial pivoting of T_r - shift I,
//      factored once, zero pivots lifted to eps |T|; seeded random starts).
//      Each vector is shifted by its own eigenvalue; eigenvalues closer than
//      1e6 x the bisection width form a cluster that is Gram-Schmidt
//      orthonormalised after every step, so its vectors span its invariant
//      subspace even where the shifts coincide.
//   4. Newton-Schulz orthonormalisation Z <- Z (3I - Z^T Z)/2, then
//      Rayleigh-Ritz: H = Z^T T_r Z and a cyclic Jacobi sweep on H (Golub &
//      Van Loan sec. 8.5.2) that rotates only pairs above eps |T| / 2 (the
//      clusters); the Ritz values diag(H) are the eigenvalues.
//   5. y = Q D Z q: each warp carries four eigenvectors through the
//      reflectors and measures |T_r v - theta v|. If any step fails (non-finite
//      iterate, orthonormalisation not converging, residual above 64 eps |T|)
//      or the pool is too small for stages 3-4, the CTA redoes stages 2-5 with
//      implicit QL on T_r (Bowdler, Martin, Reinsch & Wilkinson, Numer. Math.
//      11 (1968), tql2), whose rotations one thread logs and every thread
//      replays on Z.
// Every loop is bounded: a QL iteration cap reports info = 1.
#include <cmath>

#include "common.cuh"
#include "sturm.cuh"

#define GWB_HEEV_MMAX 112

namespace gwb {

constexpr int HEEV_THREADS = 256;
constexpr int HEEV_WARPS = HEEV_THREADS / 32;
constexpr int QL_MAX_ITER = 60;
constexpr int PER = (GWB_HEEV_MMAX + 31) / 32;  // vector elements per lane
constexpr double EPS = 2.220446049250313e-16;
constexpr int HEEV_XB = 4;  // eigenvalues computed beyond nb, for a cluster straddling nb

// matrices sent down the QL path, by reason: 0 pool too small, 1 non-finite
// inverse iterate, 2 CholQR breakdown, 3 residual above bound; and the largest
// residual / |T| the bisection path measured (bits of a non-negative double)
__device__ unsigned long long g_heev_ql[4] = {0, 0, 0, 0};
__device__ unsigned long long g_heev_maxres = 0;

// Bytes of the fixed per-matrix vectors (pv, ec, ph complex; d, er, wv, e2,
// lam float64; order int), 16-byte aligned.
__host__ __device__ inline size_t heev_base_bytes(int m) { return ((size_t)m * (3 * 16 + 5 * 8 + 4) + 15) / 16 * 16; }
// float64 of the matrix storage (m rows of lda = m + 1 complex).
__host__ __device__ inline size_t heev_a_doubles(int m) { return (size_t)2 * m * (m + 1); }
// float64 taken by the packed reflectors at the front of the matrix storage.
__host__ __device__ inline size_t heev_h_doubles(int m) { return (size_t)m * (m > 0 ? m - 1 : 0); }
// float64 the bisection/inverse-iteration path wants in the pool.
__host__ __device__ inline size_t heev_fast_need(int m, int nb) {
  const size_t ldz = (size_t)(m | 1);
  const size_t a = 3 * (size_t)m * nb, b = 2 * (size_t)nb * nb;
  return nb * ldz + (a > b ? a : b);
}
// offset of reflector j in the packed layout (complex units): rows j+1..m-1
__device__ __forceinline__ int hoff(int m, int j) { return j * (m - 1) - j * (j - 1) / 2; }

__device__ __forceinline__ double blk_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = l < HEEV_WARPS ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (l == 0) red[0] = v;
  }
  __syncthreads();
  v = red[0];
  __syncthreads();
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Reflectors applied to NV eigenvectors held by a warp (interleaved, so the
// warp reductions of the NV dot products overlap): y <- Q y with
// Q = P_0 ... P_{m-3}; Hc the packed reflectors, wv their scales.
template <int NV>
__device__ __forceinline__ void apply_reflectors(cplx<double> (&y)[NV][PER], int m, int lane,
                                                 const cplx<double>* __restrict__ Hc, const double* __restrict__ wv) {
  for (int j = m - 3; j >= 0; --j) {
    const double w = wv[j];
    if (w == 0.0) continue;
    const cplx<double>* u = Hc + hoff(m, j) - (j + 1);  // u[r] for r > j
    cplx<double> uu[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      uu[t] = (r > j && r < m) ? u[r] : mk<double>(0.0, 0.0);
    }
    const int t0 = (j + 1) >> 5;  // slots below t0 hold rows <= j only (warp-uniform)
    cplx<double> dot[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      dot[v] = mk<double>(0.0, 0.0);
#pragma unroll
      for (int t = 0; t < PER; ++t)
        if (t >= t0) dot[v] = dot[v] + conj_mul(uu[t], y[v][t]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        dot[v].x += __shfl_xor_sync(0xffffffffu, dot[v].x, o);
        dot[v].y += __shfl_xor_sync(0xffffffffu, dot[v].y, o);
      }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const cplx<double> dw = scale(dot[v], w);
#pragma unroll
      for (int t = 0; t < PER; ++t)
        if (t >= t0) y[v][t] = y[v][t] - uu[t] * dw;
    }
  }
}

// Per-matrix float64 scratch of the eigensolver: packed reflectors
// (heev_h_doubles), d (m), the complex subdiagonal (2m), the reflector scales
// (m), the phases D (2m), a flag (1: the back-transform kernel builds the
// eigenvectors; 0: the QL path already wrote them) and, from m (m + 8) on,
// the wanted eigenvectors of T_r (nb columns of m). The QL rotation log
// reuses the first m*m.
__host__ __device__ inline size_t heev_scratch_doubles(int m) { return (size_t)m * (2 * m + 8); }
__host__ __device__ inline size_t heev_off_d(int m) { return (size_t)m * (m > 0 ? m - 1 : 0); }
__host__ __device__ inline size_t heev_off_ph(int m) { return heev_off_d(m) + 4 * (size_t)m; }
__host__ __device__ inline size_t heev_off_flag(int m) { return heev_off_ph(m) + 2 * (size_t)m; }
__host__ __device__ inline size_t heev_off_v(int m) { return (size_t)m * (m + 8); }

constexpr int TRI_THREADS = 512;
constexpr int TRI_WARPS = TRI_THREADS / 32;

// Stage 1 alone, 512 threads per matrix: Householder tridiagonalisation of the
// lower triangle (the rank-2 update touches c <= r only; the matrix-vector
// product reads A[r][c] for c <= r and conj(A[c][r]) above). The column the
// next reflector is built from is copied to a contiguous buffer by the update
// that finalises it. Output per matrix in Zg: reflector j (u_0 first, rows
// j+1..m-1) at complex offset hoff(j), then d, the complex subdiagonal and the
// reflector scales w_j (0 where a column needed no reflector).
__global__ void __launch_bounds__(TRI_THREADS, 1)
    k_heev_tridiag(const cplx<double>* __restrict__ S, int lds, int64_t sk, int m, double* __restrict__ Zg) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lda = m + 1;
  cplx<double>* A = reinterpret_cast<cplx<double>*>(smem_raw);  // m*lda, lower triangle
  cplx<double>* pv = A + m * lda;                                // m
  cplx<double>* ucol = pv + m;                                   // 2m: raw column j below the diagonal, by parity
  __shared__ double red[TRI_WARPS];
  __shared__ double red1[TRI_WARPS];
  __shared__ double red2[2][TRI_WARPS];
  const int k = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const cplx<double>* Sk = S + k * sk;
  double* Zk = Zg + (int64_t)k * heev_scratch_doubles(m);
  double* o_d = Zk + heev_h_doubles(m);
  double* o_ec = o_d + m;
  double* o_wv = o_ec + 2 * m;

  for (int r = warp; r < m; r += TRI_WARPS)
    for (int c = lane; c <= r; c += 32) A[r * lda + c] = Sk[(int64_t)r * lds + c];
  double v0 = 0.0;
  for (int i = tid; i + 1 < m; i += TRI_THREADS) {
    const cplx<double> a = Sk[(int64_t)(i + 1) * lds];
    ucol[i] = a;
    v0 += norm2(a);
  }
  v0 = warp_sum(v0);
  if (lane == 0) red[warp] = v0;
  __syncthreads();
  double s2 = 0.0;
#pragma unroll
  for (int q = 0; q < TRI_WARPS; ++q) s2 += red[q];

  for (int j = 0; j + 2 < m; ++j) {
    const int r0 = j + 1, nr = m - r0, par = j & 1;
    const cplx<double>* uc_ = ucol + par * m;  // uc_[i] = A[r0 + i][j], i < nr
    cplx<double>* un_ = ucol + (par ^ 1) * m;  // next: A[r0 + 1 + i][r0], i < nr - 1
    if (s2 == 0.0) {  // column already reduced: no reflector
      if (tid == 0) {
        o_d[j] = A[j * lda + j].x;
        o_wv[j] = 0.0;
        o_ec[2 * j] = 0.0;
        o_ec[2 * j + 1] = 0.0;
      }
      double v = 0.0;
      for (int i = tid; i + 1 < nr; i += TRI_THREADS) {
        const cplx<double> a = A[(r0 + 1 + i) * lda + r0];
        un_[i] = a;
        v += norm2(a);
      }
      v = warp_sum(v);
      if (lane == 0) red2[par][warp] = v;
      __syncthreads();
      s2 = 0.0;
#pragma unroll
      for (int q = 0; q < TRI_WARPS; ++q) s2 += red2[par][q];
      continue;
    }
    const double sig = sqrt(s2);
    const cplx<double> x0 = uc_[0];
    const double a0 = sqrt(norm2(x0));
    const cplx<double> phs = a0 > 0.0 ? scale(x0, 1.0 / a0) : mk<double>(1.0, 0.0);
    const double w = 1.0 / (sig * (sig + a0));
    const cplx<double> u0 = x0 + scale(phs, sig);
    // p_r = w sum_c A[r][c] u_c, eight threads per row
    constexpr int TPR = 8;
    double kpart = 0.0;
    for (int b0 = 0; b0 < nr * TPR; b0 += TRI_THREADS) {
      const int bi = b0 + tid;
      const int rr = bi / TPR, part = bi % TPR;
      cplx<double> acc = mk<double>(0.0, 0.0);
      if (rr < nr) {
        const int r = r0 + rr;
        for (int c = r0 + part; c < m; c += TPR) {
          const cplx<double> uc = c == r0 ? u0 : uc_[c - r0];
          const cplx<double> a = c <= r ? A[r * lda + c] : conj(A[c * lda + r]);
          acc = acc + a * uc;
        }
      }
#pragma unroll
      for (int o = 1; o < TPR; o <<= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
      }
      if (rr < nr && part == 0) {
        const cplx<double> p = scale(acc, w);
        pv[rr] = p;
        const cplx<double> ur = rr == 0 ? u0 : uc_[rr];
        kpart += ur.x * p.x + ur.y * p.y;
      }
    }
    kpart = warp_sum(kpart);
    if (lane == 0) red1[warp] = kpart;
    __syncthreads();  // pv, red1 complete
    double kk = 0.0;
#pragma unroll
    for (int q = 0; q < TRI_WARPS; ++q) kk += red1[q];
    kk *= 0.5 * w;
    // lower triangle: A <- A - u q^H - q u^H with q = p - kk u; warps over rows,
    // lanes over columns c <= r with u_c, q_c in registers
    double s2p = 0.0;
    {
      cplx<double> ucs[PER], qcs[PER];
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const int cc = lane + 32 * t;
        ucs[t] = cc == 0 ? u0 : (cc < nr ? uc_[cc] : mk<double>(0.0, 0.0));
        qcs[t] = cc < nr ? pv[cc] - scale(ucs[t], kk) : mk<double>(0.0, 0.0);
      }
      for (int rr = warp; rr < nr; rr += TRI_WARPS) {
        const cplx<double> ur = rr == 0 ? u0 : uc_[rr];
        const cplx<double> qr = pv[rr] - scale(ur, kk);
        cplx<double>* arow = A + (r0 + rr) * lda + r0;
#pragma unroll
        for (int t = 0; t < PER; ++t) {
          const int cc = lane + 32 * t;
          if (cc <= rr) {
            const cplx<double> an = arow[cc] - mul_conj(ur, qcs[t]) - mul_conj(qr, ucs[t]);
            arow[cc] = an;
            if (cc == 0 && rr > 0) {
              s2p += norm2(an);
              un_[rr - 1] = an;
            }
          }
        }
      }
    }
    // reflector j to the scratch (u_0 first), as doubles: the per-matrix base
    // is only 8-byte aligned
    {
      const int o = hoff(m, j);
      for (int i = tid; i < nr; i += TRI_THREADS) {
        const cplx<double> u = i == 0 ? u0 : uc_[i];
        Zk[2 * (o + i)] = u.x;
        Zk[2 * (o + i) + 1] = u.y;
      }
    }
    if (tid == 0) {
      o_d[j] = A[j * lda + j].x;
      o_wv[j] = w;
      o_ec[2 * j] = -phs.x * sig;
      o_ec[2 * j + 1] = -phs.y * sig;
    }
    s2p = warp_sum(s2p);
    if (lane == 0) red2[par][warp] = s2p;
    __syncthreads();  // update complete
    s2 = 0.0;
#pragma unroll
    for (int q = 0; q < TRI_WARPS; ++q) s2 += red2[par][q];
  }
  if (tid == 0) {
    if (m >= 2) {
      o_d[m - 2] = A[(m - 2) * lda + m - 2].x;
      const cplx<double> e = A[(m - 1) * lda + m - 2];
      o_ec[2 * (m - 2)] = e.x;
      o_ec[2 * (m - 2) + 1] = e.y;
      o_wv[m - 2] = 0.0;
    }
    o_d[m - 1] = A[(m - 1) * lda + m - 1].x;
    o_ec[2 * (m - 1)] = 0.0;
    o_ec[2 * (m - 1) + 1] = 0.0;
    o_wv[m - 1] = 0.0;
  }
}
static size_t tri_smem(int m) { return ((size_t)m * (m + 1) + 3 * (size_t)m) * 16; }

// Stages 2-5 on the output of k_heev_tridiag in Zg (nk, heev_scratch_doubles(m));
// eig (nk, nb) ascending; U (nk, m, nb) row-major eigenvector columns; info
// (nk). extra: float64 of shared memory added to the pool beyond the matrix
// storage.
__global__ void __launch_bounds__(HEEV_THREADS, 1)
    k_heev_lowest(int m, int nb, double* __restrict__ eig, cplx<double>* __restrict__ U, double* __restrict__ Zg,
                  int* __restrict__ info, int extra) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<double>* A = reinterpret_cast<cplx<double>*>(smem_raw);  // m*lda, later packed reflectors + pool
  double* Ad = reinterpret_cast<double*>(smem_raw);
  unsigned char* base = smem_raw + (heev_a_doubles(m) + (size_t)extra) * 8;
  cplx<double>* pv = reinterpret_cast<cplx<double>*>(base);  // m  (p)
  cplx<double>* ec = pv + m;                                 // m  complex subdiagonal
  cplx<double>* ph = ec + m;                                 // m  phases
  double* d = reinterpret_cast<double*>(ph + m);             // m
  double* er = d + m;                                        // m
  double* wv = er + m;                                       // m  reflector scales
  double* e2 = wv + m;                                       // m  er^2
  double* lam = e2 + m;                                      // m  eigenvalues (ascending)
  int* order = reinterpret_cast<int*>(lam + m);              // m
  __shared__ double s_rng[2][HEEV_WARPS];
  __shared__ int s_ctl[4];  // 0: QL log count, 2: QL done, 3: QL failed
  __shared__ int s_fail;  // reason + 1 of a bisection-path failure
  const int k = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double* Zglob = Zg + (int64_t)k * heev_scratch_doubles(m);

  // stage 1 output (k_heev_tridiag): packed reflectors into the front of the
  // matrix storage, d, the complex subdiagonal and the reflector scales
  cplx<double>* Hc = A;
  {
    const int hcount = m >= 3 ? hoff(m, m - 2) : 0;
    const double* o_d = Zglob + heev_h_doubles(m);
    const double* o_ec = o_d + m;
    const double* o_wv = o_ec + 2 * m;
    for (int i = tid; i < hcount; i += blockDim.x) Hc[i] = mk<double>(Zglob[2 * i], Zglob[2 * i + 1]);
    for (int i = tid; i < m; i += blockDim.x) {
      d[i] = o_d[i];
      ec[i] = mk<double>(o_ec[2 * i], o_ec[2 * i + 1]);
      wv[i] = o_wv[i];
    }
  }
  if (tid == 0) s_fail = 0;
  __syncthreads();
  if (tid == 0) {
    // phases making the subdiagonal real: ph[j+1] = ph[j] e_j / |e_j|
    ph[0] = mk<double>(1.0, 0.0);
    for (int j = 0; j + 1 < m; ++j) {
      const double a = sqrt(norm2(ec[j]));
      er[j] = a;
      ph[j + 1] = a > 0.0 ? ph[j] * scale(ec[j], 1.0 / a) : ph[j];
    }
    er[m - 1] = 0.0;
  }
  __syncthreads();
  for (int i = tid; i < m; i += blockDim.x) e2[i] = er[i] * er[i];
  __syncthreads();
  double* pool = Ad + heev_h_doubles(m);
  const int pool_n = (int)(heev_a_doubles(m) + extra - heev_h_doubles(m));

  // spectral bounds (Gershgorin) and |T|
  double glo = 1e300, ghi = -1e300;
  for (int i = tid; i < m; i += blockDim.x) {
    const double rad = er[i] + (i > 0 ? er[i - 1] : 0.0);
    glo = fmin(glo, d[i] - rad);
    ghi = fmax(ghi, d[i] + rad);
  }
  for (int o = 16; o > 0; o >>= 1) {
    glo = fmin(glo, __shfl_xor_sync(0xffffffffu, glo, o));
    ghi = fmax(ghi, __shfl_xor_sync(0xffffffffu, ghi, o));
  }
  if (lane == 0) {
    s_rng[0][warp] = glo;
    s_rng[1][warp] = ghi;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < HEEV_WARPS; ++q) {
    glo = fmin(glo, s_rng[0][q]);
    ghi = fmax(ghi, s_rng[1][q]);
  }
  const double tnorm = fmax(fmax(fabs(glo), fabs(ghi)), 1e-300);
  glo -= 4.0 * EPS * tnorm;
  ghi += 4.0 * EPS * tnorm;

  // ---- 2-4. bisection, inverse iteration, Rayleigh-Ritz --------------------
  // nbq = nb + up to HEEV_XB eigenvalues above the wanted ones: a cluster that
  // straddles index nb is carried whole (nbx vectors) into the Rayleigh-Ritz
  const int nbq = min(m, nb + HEEV_XB);
  const int ldz = m | 1;
  double* zT = pool;                  // nbq x ldz: vector a at zT[a*ldz + i]
  double* fac = pool + nbq * ldz;     // 3 m B: 1/pivot, first superdiagonal of U, multiplier
  double* Hm = fac;                   // nbq x nbq (after inverse iteration)
  double* Qm = fac + nbq * nbq;       // nbq x nbq
  double* shift = e2;                 // per-vector shift (e2 is free after the bisection)
  int* cl = order;                    // first index of each vector's cluster
  int B = (pool_n - nbq * ldz) / (3 * m);
  if (B > nbq) B = nbq;
  bool fast = B >= 1 && nbq * ldz + 2 * nbq * nbq <= pool_n;
  const double tol = 8.0 * EPS * tnorm;  // bisection interval width
  int nbx = nb;
  if (fast) {
    // eigenvalue a by its 8-lane group: 9 sub-intervals per round (one Sturm
    // chain per lane: the count is bound by float64 issue, not latency)
    const int g = lane >> 3, gl = lane & 7;
    for (int a0 = 0; a0 < nbq; a0 += 4 * HEEV_WARPS) {
      const int a = a0 + warp * 4 + g;
      const bool act = a < nbq;
      double L = glo, Uu = ghi;
      for (int round = 0; round < 40; ++round) {
        const bool done = !act || Uu - L <= tol;
        if (__all_sync(0xffffffffu, done)) break;
        const double x = fma(Uu - L, (double)(gl + 1) * (1.0 / 9.0), L);
        const int cnt = sturm_count(d, e2, m, x);
        const unsigned bal = __ballot_sync(0xffffffffu, cnt > a);
        const unsigned gb = (bal >> (8 * g)) & 0xffu;
        const int jj = gb ? __ffs(gb) - 1 : 8;  // first point with count > a
        const double xu = __shfl_sync(0xffffffffu, x, 8 * g + min(jj, 7));
        const double xl = __shfl_sync(0xffffffffu, x, 8 * g + max(jj - 1, 0));
        if (!done) {
          if (jj < 8) {
            Uu = xu;
            if (jj > 0) L = xl;
          } else {
            L = xu;
          }
        }
      }
      if (act && gl == 0) lam[a] = 0.5 * (L + Uu);
    }
    __syncthreads();
    // clusters: runs of eigenvalues less than 1e6 * tol apart (degenerate
    // bands of an unconverged subspace split by ~1e-9 |T|). Every vector is
    // shifted by its own eigenvalue, so it converges away from everything
    // outside its cluster; each cluster is Gram-Schmidt orthonormalised after
    // every step, so near-equal shifts cannot make its vectors collapse.
    if (tid == 0) {
      const double gap = 1e6 * tol;
      int n = nb;
      while (n < nbq && lam[n] - lam[n - 1] <= gap) ++n;
      s_ctl[1] = n;
      int a = 0;
      while (a < n) {
        int b = a + 1;
        while (b < n && lam[b] - lam[b - 1] <= gap) ++b;
        for (int c = a; c < b; ++c) {
          cl[c] = a;
          shift[c] = lam[c];
        }
        a = b;
      }
    }
    __syncthreads();
    nbx = s_ctl[1];

    // inverse iteration, one thread per vector, B vectors at a time; three
    // steps, each cluster orthonormalised after every step. The pivoted LU
    // of T - shift I (1/pivot, first superdiagonal, multiplier; the swaps in
    // two bit masks) is kept across the steps when every vector fits (B >= nbx).
    const double ptiny = EPS * tnorm;
    const bool keep = B >= nbx;
    unsigned long long sw0 = 0ull, sw1 = 0ull;
    for (int it = 0; it < 3; ++it) {
      for (int b0 = 0; b0 < nbx; b0 += B) {
        const int t = tid, a = b0 + t;
        if (t < B && a < nbx) {
          const double sg = shift[a];
          double* __restrict__ z = zT + a * ldz;
          double* __restrict__ iu = fac + t;              // iu[i * B]
          double* __restrict__ u1 = fac + m * B + t;      // u1[i * B]
          double* __restrict__ lm = fac + 2 * m * B + t;  // lm[i * B]
          if (it == 0)
            for (int i = 0; i < m; ++i) z[i] = hash_pm1(((unsigned long long)(k * 131 + a) << 32) + i);
          double rc = z[0];
          if (it == 0 || !keep) {  // factor and transform the right-hand side
            sw0 = sw1 = 0ull;
            double c0 = d[0] - sg, c1 = m > 1 ? er[0] : 0.0;
            double ei = 0.0, ai1 = 0.0, ei1 = 0.0, b1 = 0.0;
            if (m > 1) {
              ei = er[0];
              ai1 = d[1] - sg;
              ei1 = er[1];
              b1 = z[1];
            }
            for (int i = 0; i + 1 < m; ++i) {
              double ei_n = 0.0, ai1_n = 0.0, ei1_n = 0.0, b1_n = 0.0;
              if (i + 2 < m) {  // next step's operands, loaded ahead of this step's stores
                ei_n = er[i + 1];
                ai1_n = d[i + 2] - sg;
                ei1_n = er[i + 2];
                b1_n = z[i + 2];
              }
              if (fabs(c0) >= ei || ei < ptiny) {  // no swap; a pivot below eps |T| is lifted to it
                const double piv = fabs(c0) < ptiny ? ptiny : c0;
                const double inv = 1.0 / piv, l = ei * inv;
                iu[i * B] = inv;
                u1[i * B] = c1;
                lm[i * B] = l;
                z[i] = rc;
                c0 = fma(-l, c1, ai1);
                c1 = ei1;
                rc = fma(-l, rc, b1);
              } else {
                const double inv = 1.0 / ei, l = c0 * inv;
                iu[i * B] = inv;
                u1[i * B] = ai1;
                lm[i * B] = l;
                if (i < 64) sw0 |= 1ull << i; else sw1 |= 1ull << (i - 64);
                z[i] = b1;
                const double nc0 = fma(-l, ai1, c1);
                c1 = -l * ei1;
                c0 = nc0;
                rc = fma(-l, b1, rc);
              }
              ei = ei_n;
              ai1 = ai1_n;
              ei1 = ei1_n;
              b1 = b1_n;
            }
            const double piv = fabs(c0) < ptiny ? ptiny : c0;
            iu[(m - 1) * B] = 1.0 / piv;
          } else {  // factors kept: transform the right-hand side only
            double b1 = m > 1 ? z[1] : 0.0;
            for (int i = 0; i + 1 < m; ++i) {
              const double b1_n = i + 2 < m ? z[i + 2] : 0.0;
              const double l = lm[i * B];
              const bool sw = i < 64 ? (sw0 >> i) & 1ull : (sw1 >> (i - 64)) & 1ull;
              if (!sw) {
                z[i] = rc;
                rc = fma(-l, rc, b1);
              } else {
                z[i] = b1;
                rc = fma(-l, b1, rc);
              }
              b1 = b1_n;
            }
          }
          // back substitution with U (1/pivot, first superdiagonal, second
          // superdiagonal e_{i+1} where rows were swapped)
          double zn1 = rc * iu[(m - 1) * B], zn2 = 0.0;
          z[m - 1] = zn1;
          double nrm = zn1 * zn1;
          if (m > 1) {
            double yi = z[m - 2], u1i = u1[(m - 2) * B], iui = iu[(m - 2) * B], e_i1 = er[m - 1];
            for (int i = m - 2; i >= 0; --i) {
              double yn = 0.0, u1n = 0.0, iun = 0.0, en = 0.0;
              if (i > 0) {
                yn = z[i - 1];
                u1n = u1[(i - 1) * B];
                iun = iu[(i - 1) * B];
                en = er[i];
              }
              const bool sw = i < 64 ? (sw0 >> i) & 1ull : (sw1 >> (i - 64)) & 1ull;
              const double u2 = sw ? e_i1 : 0.0;
              const double zi = fma(-u2, zn2, fma(-u1i, zn1, yi)) * iui;
              z[i] = zi;
              nrm = fma(zi, zi, nrm);
              zn2 = zn1;
              zn1 = zi;
              yi = yn;
              u1i = u1n;
              iui = iun;
              e_i1 = en;
            }
          }
          if (!(nrm > 0.0 && nrm < 1e300)) {
            s_fail = 2;
          } else {
            const double sc = rsqrt(nrm);
            for (int i = 0; i < m; ++i) z[i] *= sc;
          }
        }
        __syncthreads();
      }
      if (s_fail) break;
      // modified Gram-Schmidt inside each cluster, one warp per cluster
      for (int a = warp; a < nbx; a += HEEV_WARPS) {
        if (cl[a] != a || a + 1 >= nbx || cl[a + 1] != a) continue;
        int b = a;
        while (b < nbx && cl[b] == a) ++b;
        for (int c = a; c < b; ++c) {
          double* zc = zT + c * ldz;
          for (int e = a; e < c; ++e) {
            const double* ze = zT + e * ldz;
            double pr = 0.0;
            for (int i = lane; i < m; i += 32) pr = fma(ze[i], zc[i], pr);
            pr = warp_sum(pr);
            for (int i = lane; i < m; i += 32) zc[i] = fma(-pr, ze[i], zc[i]);
            __syncwarp();
          }
          double nrm = 0.0;
          for (int i = lane; i < m; i += 32) nrm = fma(zc[i], zc[i], nrm);
          nrm = warp_sum(nrm);
          if (!(nrm > 1e-30)) {
            if (lane == 0) s_fail = 3;
            break;
          }
          const double sc = rsqrt(nrm);
          for (int i = lane; i < m; i += 32) zc[i] *= sc;
          __syncwarp();
        }
      }
      __syncthreads();
      if (s_fail) break;
    }
    fast = !s_fail;
  }
  if (fast) {
    // Orthonormalisation: the vectors of distinct clusters are orthogonal to
    // the inverse-iteration accuracy and each cluster is Gram-Schmidt
    // orthonormal, so G = Z^T Z = I + E with E tiny; Newton-Schulz steps
    // Z <- Z (3I - G)/2 square the deviation (|E| -> 3|E|^2/4) until it is at
    // round-off. A deviation above 1/4 means the inverse iteration failed.
    bool polish = false;
    for (int pass = 0; pass < 8; ++pass) {
      double dev = 0.0;
      for (int a = warp; a < nbx; a += HEEV_WARPS) {
        const double* za = zT + a * ldz;
        double acc[PER];
#pragma unroll
        for (int t = 0; t < PER; ++t) acc[t] = 0.0;
        for (int i = 0; i < m; ++i) {
          const double zai = za[i];
#pragma unroll
          for (int t = 0; t < PER; ++t) {
            const int b = lane + 32 * t;
            if (b >= a && b < nbx) acc[t] = fma(zai, zT[b * ldz + i], acc[t]);
          }
        }
#pragma unroll
        for (int t = 0; t < PER; ++t) {
          const int b = lane + 32 * t;
          if (b >= a && b < nbx) {
            Hm[a * nbx + b] = acc[t];
            Hm[b * nbx + a] = acc[t];
            dev = fmax(dev, fabs(acc[t] - (a == b ? 1.0 : 0.0)));
          }
        }
      }
      for (int o = 16; o > 0; o >>= 1) dev = fmax(dev, __shfl_xor_sync(0xffffffffu, dev, o));
      if (lane == 0) s_rng[pass & 1][warp] = dev;
      __syncthreads();
      dev = 0.0;
#pragma unroll
      for (int q = 0; q < HEEV_WARPS; ++q) dev = fmax(dev, s_rng[pass & 1][q]);
      if (dev <= 32.0 * EPS && polish) break;  // round-off level of an m-term dot product
      if (dev <= 32.0 * EPS) polish = true;      // one more step takes the error to round-off
      if (!(dev < 0.25) || pass == 7) {
        fast = false;
        if (tid == 0) s_fail = 3;
        break;
      }
      // Z <- Z (1.5 I - 0.5 G): warp per row i, lanes over columns b, in place
      for (int i = warp; i < m; i += HEEV_WARPS) {
        double o[PER];
#pragma unroll
        for (int t = 0; t < PER; ++t) o[t] = 0.0;
        for (int a = 0; a < nbx; ++a) {
          const double za = zT[a * ldz + i];
#pragma unroll
          for (int t = 0; t < PER; ++t) {
            const int b = lane + 32 * t;
            if (b < nbx) o[t] = fma(za, (a == b ? 1.5 : 0.0) - 0.5 * Hm[a * nbx + b], o[t]);
          }
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < PER; ++t) {
          const int b = lane + 32 * t;
          if (b < nbx) zT[b * ldz + i] = o[t];
        }
      }
      __syncthreads();
    }
  }
  if (fast) {
    // H = Z^T T Z (full): warp per row a, lanes over columns b >= a
    for (int a = warp; a < nbx; a += HEEV_WARPS) {
      const double* za = zT + a * ldz;
      double acc[PER];
#pragma unroll
      for (int t = 0; t < PER; ++t) acc[t] = 0.0;
      for (int i = 0; i < m; ++i) {
        double tz = d[i] * za[i];
        if (i > 0) tz = fma(er[i - 1], za[i - 1], tz);
        if (i + 1 < m) tz = fma(er[i], za[i + 1], tz);
#pragma unroll
        for (int t = 0; t < PER; ++t) {
          const int b = lane + 32 * t;
          if (b >= a && b < nbx) acc[t] = fma(tz, zT[b * ldz + i], acc[t]);
        }
      }
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const int b = lane + 32 * t;
        if (b >= a && b < nbx) {
          Hm[a * nbx + b] = acc[t];
          Hm[b * nbx + a] = acc[t];
        }
      }
    }
    __syncthreads();
    for (int i = tid; i < nbx * nbx; i += blockDim.x) Qm[i] = (i / nbx == i % nbx) ? 1.0 : 0.0;
    __syncthreads();
    if (warp == 0) {  // cyclic Jacobi on the pairs above threshold
      const double thr = 0.5 * EPS * tnorm;  // below this a rotation only moves round-off
      for (int sweep = 0; sweep < 12; ++sweep) {
        int nrot = 0;
        for (int p = 0; p + 1 < nbx; ++p) {
          bool any = false;
          for (int q = p + 1 + lane; q < nbx; q += 32) any |= fabs(Hm[p * nbx + q]) > thr;
          if (!__any_sync(0xffffffffu, any)) continue;
          for (int q = p + 1; q < nbx; ++q) {
            const double apq = Hm[p * nbx + q];
            if (!(fabs(apq) > thr)) continue;
            const double app = Hm[p * nbx + p], aqq = Hm[q * nbx + q];
            const double th = (aqq - app) / (2.0 * apq);
            const double tt = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(fma(th, th, 1.0)));
            const double c = rsqrt(fma(tt, tt, 1.0)), s = tt * c;
            __syncwarp();
            for (int r = lane; r < nbx; r += 32) {
              if (r != p && r != q) {
                const double arp = Hm[r * nbx + p], arq = Hm[r * nbx + q];
                const double np = c * arp - s * arq, nq = s * arp + c * arq;
                Hm[r * nbx + p] = np;
                Hm[p * nbx + r] = np;
                Hm[r * nbx + q] = nq;
                Hm[q * nbx + r] = nq;
              }
              const double qp = Qm[r * nbx + p], qq = Qm[r * nbx + q];
              Qm[r * nbx + p] = c * qp - s * qq;
              Qm[r * nbx + q] = s * qp + c * qq;
            }
            __syncwarp();
            if (lane == 0) {
              Hm[p * nbx + p] = app - tt * apq;
              Hm[q * nbx + q] = aqq + tt * apq;
              Hm[p * nbx + q] = 0.0;
              Hm[q * nbx + p] = 0.0;
            }
            __syncwarp();
            ++nrot;
          }
        }
        if (nrot == 0) break;
      }
      // ascending order of the Ritz values
      for (int i = lane; i < nbx; i += 32) {
        const double di = Hm[i * nbx + i];
        int rank = 0;
        for (int j = 0; j < nbx; ++j) {
          const double dj = Hm[j * nbx + j];
          rank += (dj < di || (dj == di && j < i)) ? 1 : 0;
        }
        order[rank] = i;
      }
    }
    __syncthreads();
    // eigenvectors of T_r: v = Z Q[:, src] into the scratch (k_heev_backtransform
    // applies D and the reflectors), with the residual |T v - theta v| checked
    double* Vk = Zglob + heev_off_v(m);
    const double rtol = 64.0 * EPS * tnorm;
    for (int ra = warp; ra < nb; ra += HEEV_WARPS) {
      const int src = order[ra];
      const double th = Hm[src * nbx + src];
      double v[PER];
#pragma unroll
      for (int t = 0; t < PER; ++t) v[t] = 0.0;
      for (int b = 0; b < nbx; ++b) {
        const double qb = Qm[b * nbx + src];
        if (qb == 0.0) continue;
#pragma unroll
        for (int t = 0; t < PER; ++t) {
          const int i = lane + 32 * t;
          if (i < m) v[t] = fma(zT[b * ldz + i], qb, v[t]);
        }
      }
      double res = 0.0;
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const int i = lane + 32 * t;
        const double up = __shfl_up_sync(0xffffffffu, v[t], 1);
        const double wrapu = __shfl_sync(0xffffffffu, t > 0 ? v[t > 0 ? t - 1 : 0] : 0.0, 31);
        const double dn = __shfl_down_sync(0xffffffffu, v[t], 1);
        const double wrapd = __shfl_sync(0xffffffffu, t + 1 < PER ? v[t + 1 < PER ? t + 1 : t] : 0.0, 0);
        const double vm = lane > 0 ? up : wrapu, vp = lane < 31 ? dn : wrapd;
        if (i < m) {
          double tv = (d[i] - th) * v[t];
          if (i > 0) tv = fma(er[i - 1], vm, tv);
          if (i + 1 < m) tv = fma(er[i], vp, tv);
          res = fma(tv, tv, res);
        }
      }
      res = warp_sum(res);
      if (lane == 0) atomicMax(&g_heev_maxres, (unsigned long long)__double_as_longlong(sqrt(res) / tnorm));
      if (!(res <= rtol * rtol)) {
        if (lane == 0) s_fail = 4;
      }
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const int i = lane + 32 * t;
        if (i < m) Vk[(int64_t)ra * m + i] = v[t];
      }
      if (lane == 0) eig[(int64_t)k * nb + ra] = th;
    }
    __syncthreads();
    if (!s_fail) {
      for (int i = tid; i < m; i += blockDim.x) {
        Zglob[heev_off_ph(m) + 2 * i] = ph[i].x;
        Zglob[heev_off_ph(m) + 2 * i + 1] = ph[i].y;
      }
      if (tid == 0) {
        Zglob[heev_off_flag(m)] = 1.0;
        info[k] = 0;
      }
      return;
    }
  }

  // ---- QL path: implicit QL on (d, er), Z in the pool -----------------------
  if (tid == 0) {
    atomicAdd(&g_heev_ql[s_fail > 0 ? s_fail - 1 : 0], 1ull);
    Zglob[heev_off_flag(m)] = 0.0;  // the eigenvectors are written here, not by the back-transform kernel
  }
  double* Z = pool;  // Z(row r, col i) at Z[i*m + r]; pool_n >= m*m
  double* dq = lam;  // the QL recurrence works on copies of d and er
  double* eq = e2;
  for (int i = tid; i < m; i += blockDim.x) {
    dq[i] = d[i];
    eq[i] = er[i];
  }
  for (int i = tid; i < m * m; i += blockDim.x) Z[i] = (i / m == i % m) ? 1.0 : 0.0;
  if (tid == 0) s_ctl[3] = 0;
  __syncthreads();
  {
    // Thread 0 runs whole batches of QL sweeps and logs each sweep as a
    // header {-(mm+2), ilo} followed by its rotations {c, s} (i = mm-1 .. ilo);
    // then every thread replays the log on its rows of Z. The d/e recurrence
    // never reads Z, so batches need only two barriers each.
    // plain doubles: the per-matrix offset k*m*(2m+8) is only 8-byte aligned for odd m
    double* lg = Zglob;
    const int cap = (m * m) / 2;  // entries of two doubles
    int l = 0, iter = 0;          // scalar QL state, used by thread 0 only
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
            const double dd = fabs(dq[mm]) + fabs(dq[mm + 1]);
            if (fabs(eq[mm]) <= EPS * dd) break;
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
          double g = (dq[l + 1] - dq[l]) / (2.0 * eq[l]);
          double r = sqrt(fma(g, g, 1.0));
          g = dq[mm] - dq[l] + eq[l] / (g + copysign(r, g));
          double sn = 1.0, cs = 1.0, p = 0.0;
          int i = mm - 1;
          bool broke = false;
          // the next rotation's e and d are loaded one step ahead (they do not
          // depend on the recurrence); one rsqrt gives r, c and s
          double e_i = eq[i], d_i = dq[i], d_i1 = dq[i + 1];
          for (; i >= l; --i) {
            const double e_nx = i > l ? eq[i - 1] : 0.0;
            const double d_nx = i > l ? dq[i - 1] : 0.0;
            const double f = sn * e_i, b = cs * e_i;
            const double r2 = fma(f, f, g * g);  // subspace spectra are O(1e3): no overflow
            if (r2 == 0.0) {
              eq[i + 1] = 0.0;
              dq[i + 1] = d_i1 - p;
              eq[mm] = 0.0;
              broke = true;
              break;
            }
            const double rinv = rsqrt(r2);
            eq[i + 1] = r2 * rinv;
            sn = f * rinv;
            cs = g * rinv;
            g = d_i1 - p;
            const double rr = (d_i - g) * sn + 2.0 * cs * b;
            p = sn * rr;
            dq[i + 1] = g + p;
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
            dq[l] -= p;
            eq[l] = g;
            eq[mm] = 0.0;
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
            const double c2 = lg[2 * e + 4], s2_ = lg[2 * e + 5], c3 = lg[2 * e + 6], s3 = lg[2 * e + 7];
            e += 4;
            const double z0 = Z[i * m + r], z1 = Z[(i - 1) * m + r], z2 = Z[(i - 2) * m + r],
                         z3 = Z[(i - 3) * m + r];
            Z[(i + 1) * m + r] = s0 * z0 + c0 * carry;
            carry = c0 * z0 - s0 * carry;
            Z[i * m + r] = s1 * z1 + c1 * carry;
            carry = c1 * z1 - s1 * carry;
            Z[(i - 1) * m + r] = s2_ * z2 + c2 * carry;
            carry = c2 * z2 - s2_ * carry;
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
  }
  if (s_ctl[3]) {
    if (tid == 0) info[k] = 1;
    return;
  }
  // ascending order (stable)
  for (int i = tid; i < m; i += blockDim.x) {
    int rank = 0;
    for (int j = 0; j < m; ++j) rank += (dq[j] < dq[i] || (dq[j] == dq[i] && j < i)) ? 1 : 0;
    order[rank] = i;
  }
  __syncthreads();
  if (tid == 0) info[k] = 0;
  for (int a = tid; a < nb; a += blockDim.x) eig[(int64_t)k * nb + a] = dq[order[a]];
  cplx<double>* Uk = U + (int64_t)k * m * nb;
  for (int a = warp; a < nb; a += HEEV_WARPS) {
    const int src = order[a];
    cplx<double> y[1][PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      y[0][t] = r < m ? scale(ph[r], Z[(int64_t)src * m + r]) : mk<double>(0.0, 0.0);
    }
    apply_reflectors<1>(y, m, lane, Hc, wv);
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      if (r < m) Uk[(int64_t)r * nb + a] = y[0][t];
    }
  }
}

// Stage 5 on many SMs: y = Q_H D v for the eigenvectors v of T_r that
// k_heev_lowest left in the scratch. Grid (k, groups of BT_WARPS * BT_NV
// vectors); the CTA stages the packed reflectors in shared memory, and each
// warp carries BT_NV vectors through them. Matrices the QL path solved (flag
// 0) are skipped: their eigenvectors are already in U.
constexpr int BT_WARPS = 4, BT_NV = 2;

__global__ void __launch_bounds__(BT_WARPS * 32) k_heev_backtransform(int m, int nb, const double* __restrict__ Zg,
                                                                      cplx<double>* __restrict__ U) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int k = blockIdx.x;
  const double* Zk = Zg + (int64_t)k * heev_scratch_doubles(m);
  if (Zk[heev_off_flag(m)] == 0.0) return;
  const int hcount = m >= 3 ? hoff(m, m - 2) : 0;
  cplx<double>* Hc = reinterpret_cast<cplx<double>*>(smem_raw);
  cplx<double>* phs = Hc + hcount;
  double* wvs = reinterpret_cast<double*>(phs + m);
  for (int i = threadIdx.x; i < hcount; i += blockDim.x) Hc[i] = mk<double>(Zk[2 * i], Zk[2 * i + 1]);
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    phs[i] = mk<double>(Zk[heev_off_ph(m) + 2 * i], Zk[heev_off_ph(m) + 2 * i + 1]);
    wvs[i] = Zk[heev_off_d(m) + 3 * (size_t)m + i];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a0 = (blockIdx.y * BT_WARPS + warp) * BT_NV;
  if (a0 >= nb) return;  // warp-uniform; no barrier follows
  const double* Vk = Zk + heev_off_v(m);
  cplx<double> y[BT_NV][PER];
#pragma unroll
  for (int sv = 0; sv < BT_NV; ++sv) {
    const int ra = a0 + sv;
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      y[sv][t] = (ra < nb && r < m) ? scale(phs[r], Vk[(int64_t)ra * m + r]) : mk<double>(0.0, 0.0);
    }
  }
  apply_reflectors<BT_NV>(y, m, lane, Hc, wvs);
  cplx<double>* Uk = U + (int64_t)k * m * nb;
#pragma unroll
  for (int sv = 0; sv < BT_NV; ++sv) {
    const int ra = a0 + sv;
    if (ra >= nb) continue;
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      if (r < m) Uk[(int64_t)r * nb + ra] = y[sv][t];
    }
  }
}
static size_t bt_smem(int m) {
  const size_t hcount = m >= 3 ? (size_t)((m - 2) * (m - 1) - (m - 2) * (m - 3) / 2) : 0;
  return hcount * 16 + (size_t)m * 16 + (size_t)m * 8;
}

// Shared memory: matrix storage + extra pool + per-matrix vectors, within the
// 227 KB opt-in limit; the extra pool lets stages 3-4 hold every vector at once.
static int heev_extra(int m, int nb) {
  const size_t fixed = (heev_a_doubles(m)) * 8 + heev_base_bytes(m);
  const size_t pool0 = heev_a_doubles(m) - heev_h_doubles(m);
  const size_t need = heev_fast_need(m, nb + HEEV_XB < m ? nb + HEEV_XB : m);
  size_t extra = need > pool0 ? need - pool0 : 0;
  const size_t limit = 232448 - 1024;  // opt-in maximum less the kernel's static shared memory
  const size_t room = fixed < limit ? (limit - fixed) / 8 : 0;
  if (extra > room) extra = room;
  return (int)(extra & ~(size_t)1);  // keep the vectors behind it 16-byte aligned
}
size_t heev_smem(int m, int nb) { return heev_a_doubles(m) * 8 + (size_t)heev_extra(m, nb) * 8 + heev_base_bytes(m); }

// The eigensolver on nk matrices with scratch z (nk * heev_scratch_doubles(m)
// float64): stage 1, then stages 2-5.
static int launch_heev(int nk, int m, int nb, const void* S, int lds, int64_t sk, double* eig, void* U,
                       double* z, int* info, cudaStream_t st) {
  const size_t sm1 = tri_smem(m);
  GWB_CUDA_TRY(allow_smem(k_heev_tridiag));
  k_heev_tridiag<<<nk, TRI_THREADS, sm1, st>>>((const cplx<double>*)S, lds, sk, m, z);
  const int extra = heev_extra(m, nb);
  const size_t sm = heev_smem(m, nb);
  GWB_CUDA_TRY(allow_smem(k_heev_lowest));
  k_heev_lowest<<<nk, HEEV_THREADS, sm, st>>>(m, nb, eig, (cplx<double>*)U, z, info, extra);
  const size_t sm3 = bt_smem(m);
  GWB_CUDA_TRY(allow_smem(k_heev_backtransform));
  dim3 g3(nk, (nb + BT_WARPS * BT_NV - 1) / (BT_WARPS * BT_NV));
  k_heev_backtransform<<<g3, BT_WARPS * 32, sm3, st>>>(m, nb, z, (cplx<double>*)U);
  GWB_LAUNCH_CHECK();
  count_launches(3);
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

extern "C" int64_t gwb_heev_scratch_doubles(int32_t m) { return m > 0 ? (int64_t)heev_scratch_doubles(m) : 0; }

// Diagnostics of the bisection path on the current device since load:
// out[0..3] matrices sent to QL by reason (pool too small, non-finite inverse
// iterate, CholQR breakdown, residual bound), out[4] the largest residual / |T|
// measured (bits of a float64).
extern "C" int gwb_heev_ql_count(unsigned long long* out) {
  GWB_REQUIRE(out, "null pointer");
  GWB_CUDA_TRY(cudaMemcpyFromSymbol(out, g_heev_ql, 4 * sizeof(unsigned long long)));
  GWB_CUDA_TRY(cudaMemcpyFromSymbol(out + 4, g_heev_maxres, sizeof(unsigned long long)));
  return GWB_OK;
}

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
//   * a call needs nk * m * (2m + 8) float64 of it; larger problems are rejected with
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
  if ((int64_t)nk * (int64_t)heev_scratch_doubles(m) > (int64_t)GWB_HEEV_NOALLOC_DOUBLES) {
    set_error("gwb_heev_lowest_noalloc: nk*m*(2m+8) = " + std::to_string((int64_t)nk * (int64_t)heev_scratch_doubles(m)) +
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

