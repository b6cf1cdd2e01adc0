// Batched float64 Hermitian eigensolver for the Davidson subspace matrices
// (replaces torch.linalg.eigh in gradwave solvers/davidson.py:66-75,650):
// the lowest nb eigenpairs of each m x m matrix, ascending.
//
// One CTA per matrix, the matrix in shared memory (m <= GWB_HEEV_MMAX):
//   1. Householder tridiagonalisation with Hermitian reflectors
//      P_j = I - w_j u_j u_j^H, A <- P_j A P_j (Golub & Van Loan, Matrix
//      Computations, 4th ed., sec. 8.3.1, complex form), two block barriers
//      per column: the u^H p reduction rides on the matrix-vector pass and the
//      next column's norm on the rank-2 update. The complex subdiagonal is
//      made real by a diagonal phase D (T = D T_r D^H); the reflectors are
//      then packed into the front of the matrix storage and the rest of it
//      becomes the working pool of the stages below.
//   2. Eigenvalues lambda_0..lambda_{nb-1} of T_r by multisection on Sturm
//      counts (8 lanes per eigenvalue, 9 sub-intervals per round). The count
//      is the number of sign changes of the leading principal minors
//      p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2}, rescaled by powers of two;
//      the computed count is exact for T_r with each e_i^2 perturbed by a few
//      ulps (Wilkinson, The Algebraic Eigenvalue Problem, ch. 5, secs. 37-40;
//      Barth, Martin & Wilkinson, Numer. Math. 9 (1967) 386).
//   3. Eigenvectors of T_r by two steps of inverse iteration per eigenvalue
//      (one thread each; Gaussian elimination with partial pivoting of the
//      tridiagonal T_r - lambda I, zero pivots lifted to eps |T|; seeded random
//      start vectors, so the vectors of a degenerate cluster span it).
//   4. CholQR2 of those vectors, then Rayleigh-Ritz: H = Z^T T_r Z, a cyclic
//      Jacobi sweep on H (Golub & Van Loan sec. 8.5.2) that only rotates
//      pairs with |H_pq| > 2 eps |T| (the clusters), eigenvalues diag(H).
//   5. y = Q D Z q, one warp per eigenvector; each warp also measures the
//      residual |T_r v - theta v|. If any step fails (non-finite iterate,
//      Cholesky breakdown, residual above 64 eps |T|) or the pool is too small
//      for stages 3-4, the CTA redoes stage 2-5 with implicit QL on T_r
//      (Bowdler, Martin, Reinsch & Wilkinson, Numer. Math. 11 (1968), tql2),
//      whose rotations one thread logs and every thread replays on Z.
// Every loop is bounded: a QL iteration cap reports info = 1.
#include <cmath>

#include "common.cuh"

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
  const size_t a = 2 * (size_t)m * nb, b = 2 * (size_t)nb * nb;
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

// Seeded uniform value in [-1, 1): SplitMix64 (Steele, Lea & Flood, OOPSLA 2014).
__device__ __forceinline__ double hash_pm1(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * 0x1.0p-52 - 1.0;
}

// Number of eigenvalues of the real tridiagonal (d, e) below x: sign changes
// of the leading principal minors, rescaled by 2^-+400 every fourth step (the
// minors grow by at most |d_i - x| + e_i^2 per step).
__device__ __forceinline__ int sturm_count(const double* __restrict__ d, const double* __restrict__ e2, int m,
                                           double x) {
  constexpr double BIG = 0x1.0p400, SMALL = 0x1.0p-400, TINY = 0x1.0p-100;
  double p0 = 1.0, p1 = d[0] - x;
  if (p1 == 0.0) p1 = -TINY;
  int cnt = p1 < 0.0;
  for (int i = 1; i < m; ++i) {
    double p2 = fma(d[i] - x, p1, -e2[i - 1] * p0);
    if (p2 == 0.0) p2 = -TINY * p1;  // a zero minor takes the sign opposite to its predecessor
    cnt += (p2 < 0.0) != (p1 < 0.0);
    p0 = p1;
    p1 = p2;
    if ((i & 3) == 0) {
      const double mx = fmax(fabs(p0), fabs(p1));
      if (mx > BIG) {
        p0 *= SMALL;
        p1 *= SMALL;
      } else if (mx < SMALL) {
        p0 *= BIG;
        p1 *= BIG;
      }
    }
  }
  return cnt;
}

// Reflectors applied to one eigenvector held by a warp: y <- Q y with
// Q = P_0 ... P_{m-3}; Hc the packed reflectors, wv their scales.
__device__ __forceinline__ void apply_reflectors(cplx<double> (&y)[PER], int m, int lane,
                                                 const cplx<double>* __restrict__ Hc, const double* __restrict__ wv) {
  for (int j = m - 3; j >= 0; --j) {
    const double w = wv[j];
    if (w == 0.0) continue;
    const cplx<double>* u = Hc + hoff(m, j) - (j + 1);  // u[r] for r > j
    cplx<double> dot = mk<double>(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      if (r > j && r < m) dot = dot + conj_mul(u[r], y[t]);
    }
    for (int o = 16; o > 0; o >>= 1) {
      dot.x += __shfl_xor_sync(0xffffffffu, dot.x, o);
      dot.y += __shfl_xor_sync(0xffffffffu, dot.y, o);
    }
    dot = scale(dot, w);
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      if (r > j && r < m) y[t] = y[t] - u[r] * dot;
    }
  }
}

// S (nk, lds, lds) row-major Hermitian (both triangles filled), leading m x m.
// eig (nk, nb) ascending; U (nk, m, nb) row-major eigenvector columns;
// Zg scratch (nk, m, m) float64 (reflector staging, QL rotation log); info (nk).
// extra: float64 of shared memory added to the pool beyond the matrix storage.
__global__ void __launch_bounds__(HEEV_THREADS, 1)
    k_heev_lowest(const cplx<double>* __restrict__ S, int lds, int64_t sk, int m, int nb, double* __restrict__ eig,
                  cplx<double>* __restrict__ U, double* __restrict__ Zg, int* __restrict__ info, int extra) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lda = m + 1;  // padded row stride of A in shared memory
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
  __shared__ double red[HEEV_WARPS];
  __shared__ double red1[HEEV_WARPS];
  __shared__ double red2[2][HEEV_WARPS];
  __shared__ double s_rng[2][HEEV_WARPS];
  __shared__ int s_ctl[4];  // 0: QL log count, 2: QL done, 3: QL failed
  __shared__ int s_fail;  // reason + 1 of a bisection-path failure
  const int k = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const cplx<double>* Sk = S + k * sk;
  double* Zglob = Zg + (int64_t)k * m * m;

  for (int i = tid; i < m * m; i += blockDim.x) A[(i / m) * lda + (i % m)] = Sk[(int64_t)(i / m) * lds + (i % m)];
  if (tid == 0) s_fail = 0;
  __syncthreads();

  // ---- 1. tridiagonalisation ---------------------------------------------
  double s2 = 0.0;
  {
    double v = 0.0;
    for (int r = 1 + tid; r < m; r += blockDim.x) v += norm2(A[r * lda]);
    s2 = blk_sum(v, red);
  }
  for (int j = 0; j + 2 < m; ++j) {
    const int r0 = j + 1, nr = m - r0;
    const int par = j & 1;
    if (s2 == 0.0) {  // column already reduced: no reflector
      if (tid == 0) {
        d[j] = A[j * lda + j].x;
        wv[j] = 0.0;
        ec[j] = mk<double>(0.0, 0.0);
      }
      double v = 0.0;
      for (int r = j + 2 + tid; r < m; r += blockDim.x) v += norm2(A[r * lda + j + 1]);
      v = warp_sum(v);
      if (lane == 0) red2[par][warp] = v;
      __syncthreads();
      s2 = 0.0;
#pragma unroll
      for (int w = 0; w < HEEV_WARPS; ++w) s2 += red2[par][w];
      continue;
    }
    const double sig = sqrt(s2);
    const cplx<double> x0 = A[r0 * lda + j];
    const double a0 = sqrt(norm2(x0));
    const cplx<double> phs = a0 > 0.0 ? scale(x0, 1.0 / a0) : mk<double>(1.0, 0.0);
    const double w = 1.0 / (sig * (sig + a0));
    const cplx<double> u0 = x0 + scale(phs, sig);  // u = column j below the diagonal, first entry u0
    // p_r = w sum_c A[r][c] u_c = w sum_c conj(A[c][r]) u_c, TPR threads per row;
    // the same pass accumulates Re(u^H p)
    constexpr int TPR = 4;
    double kpart = 0.0;
    for (int b0 = 0; b0 < nr * TPR; b0 += blockDim.x) {
      const int bi = b0 + tid;
      const int rr = bi / TPR, part = bi % TPR;
      cplx<double> acc = mk<double>(0.0, 0.0);
      if (rr < nr) {
        const int r = r0 + rr;
        for (int c = r0 + part; c < m; c += TPR) {
          const cplx<double> uc = c == r0 ? u0 : A[c * lda + j];
          acc = acc + conj_mul(A[c * lda + r], uc);
        }
      }
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 2);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 2);
      if (rr < nr && part == 0) {
        const cplx<double> p = scale(acc, w);
        pv[rr] = p;
        const cplx<double> ur = rr == 0 ? u0 : A[(r0 + rr) * lda + j];
        kpart += ur.x * p.x + ur.y * p.y;
      }
    }
    kpart = warp_sum(kpart);
    if (lane == 0) red1[warp] = kpart;
    __syncthreads();  // pv, red1 complete
    double kk = 0.0;
#pragma unroll
    for (int q = 0; q < HEEV_WARPS; ++q) kk += red1[q];
    kk *= 0.5 * w;
    // A <- A - u q^H - q u^H with q = p - kk u; the norm of the next column
    // (column r0, rows > r0) is summed from the updated entries
    double s2p = 0.0;
    for (int idx = tid; idx < nr * nr; idx += blockDim.x) {
      const int rr = idx / nr, cc = idx - rr * nr;
      const cplx<double> ur = rr == 0 ? u0 : A[(r0 + rr) * lda + j];
      const cplx<double> uc = cc == 0 ? u0 : A[(r0 + cc) * lda + j];
      const cplx<double> qr = pv[rr] - scale(ur, kk), qc = pv[cc] - scale(uc, kk);
      cplx<double>& a = A[(r0 + rr) * lda + r0 + cc];
      const cplx<double> an = a - mul_conj(ur, qc) - mul_conj(qr, uc);
      a = an;
      if (cc == 0 && rr > 0) s2p += norm2(an);
    }
    if (tid == 0) {  // nobody reads A[r0][j] in this phase (u0 is in registers)
      d[j] = A[j * lda + j].x;
      wv[j] = w;
      ec[j] = scale(phs, -sig);
      A[r0 * lda + j] = u0;
    }
    s2p = warp_sum(s2p);
    if (lane == 0) red2[par][warp] = s2p;
    __syncthreads();  // update complete
    s2 = 0.0;
#pragma unroll
    for (int q = 0; q < HEEV_WARPS; ++q) s2 += red2[par][q];
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
  }
  // pack the reflectors (column j, rows j+1..m-1, j <= m-3) at the front of
  // the matrix storage, staged through the global scratch (as plain doubles:
  // the per-matrix offset k*m*m is only 8-byte aligned for odd m)
  double* stage = Zglob;
  const int hcount = m >= 3 ? hoff(m, m - 2) : 0;
  for (int idx = tid; idx < (m - 2) * (m - 1); idx += blockDim.x) {
    const int j = idx / (m - 1), t = idx - j * (m - 1);
    if (t < m - 1 - j) {
      const cplx<double> v = A[(j + 1 + t) * lda + j];
      stage[2 * (hoff(m, j) + t)] = v.x;
      stage[2 * (hoff(m, j) + t) + 1] = v.y;
    }
  }
  __syncthreads();
  cplx<double>* Hc = A;
  for (int i = tid; i < hcount; i += blockDim.x) Hc[i] = mk<double>(stage[2 * i], stage[2 * i + 1]);
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
  double* fac = pool + nbq * ldz;     // 2 m B: 1/pivot, first superdiagonal of U
  double* Hm = fac;                   // nbq x nbq (after inverse iteration)
  double* Qm = fac + nbq * nbq;       // nbq x nbq
  double* shift = e2;                 // per-vector shift (e2 is free after the bisection)
  int* cl = order;                    // first index of each vector's cluster
  int B = (pool_n - nbq * ldz) / (2 * m);
  if (B > nbq) B = nbq;
  bool fast = B >= 1 && nbq * ldz + 2 * nbq * nbq <= pool_n;
  const double tol = 8.0 * EPS * tnorm;  // bisection interval width
  int nbx = nb;
  if (fast) {
    // eigenvalue a by its 8-lane group; 9 sub-intervals per round
    const int g = lane >> 3, gl = lane & 7;
    for (int a0 = 0; a0 < nbq; a0 += 4 * HEEV_WARPS) {
      const int a = a0 + warp * 4 + g;
      const bool act = a < nbq;
      double L = glo, Uu = ghi;
      for (int round = 0; round < 40; ++round) {
        const bool done = !act || Uu - L <= tol;
        if (__all_sync(0xffffffffu, done)) break;
        const double x = fma((Uu - L), (double)(gl + 1) * (1.0 / 9.0), L);
        const int cnt = sturm_count(d, e2, m, x);
        const unsigned bal = __ballot_sync(0xffffffffu, cnt > a);
        const unsigned gb = (bal >> (8 * g)) & 0xffu;
        const int jj = gb ? __ffs(gb) - 1 : 8;
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
    // clusters: runs of eigenvalues less than 1e4 * tol apart. An isolated
    // eigenvalue is its own shift; a cluster [lo, hi] shares the shift
    // lo - (hi - lo) - 16 tol, where every member is amplified within a factor
    // of two of the others, and its block is re-orthonormalised between steps
    if (tid == 0) {
      const double gap = 1e4 * tol;
      int n = nb;
      while (n < nbq && lam[n] - lam[n - 1] <= gap) ++n;
      s_ctl[1] = n;
      int a = 0;
      while (a < n) {
        int b = a + 1;
        while (b < n && lam[b] - lam[b - 1] <= gap) ++b;
        const double sh = b - a == 1 ? lam[a] : lam[a] - (lam[b - 1] - lam[a]) - 16.0 * tol;
        for (int c = a; c < b; ++c) {
          cl[c] = a;
          shift[c] = sh;
        }
        a = b;
      }
    }
    __syncthreads();
    nbx = s_ctl[1];

    // inverse iteration, one thread per vector, B vectors at a time; three
    // steps, the clusters orthonormalised after the first two
    const double ptiny = EPS * tnorm;
    for (int it = 0; it < 3; ++it) {
      for (int b0 = 0; b0 < nbx; b0 += B) {
        const int t = tid, a = b0 + t;
        if (t < B && a < nbx) {
          const double sg = shift[a];
          double* z = zT + a * ldz;
          double* iu = fac + t;          // iu[i * B]
          double* u1 = fac + m * B + t;  // u1[i * B]
          if (it == 0)
            for (int i = 0; i < m; ++i) z[i] = hash_pm1(((unsigned long long)(k * 131 + a) << 32) + i);
          unsigned long long sw0 = 0ull, sw1 = 0ull;
          double c0 = d[0] - sg, c1 = m > 1 ? er[0] : 0.0, rc = z[0];
          for (int i = 0; i + 1 < m; ++i) {
            const double ei = er[i], ai1 = d[i + 1] - sg, ei1 = er[i + 1], b1 = z[i + 1];
            if (fabs(c0) >= ei || ei < ptiny) {  // no swap; a pivot below eps |T| is lifted to it
              const double piv = fabs(c0) < ptiny ? ptiny : c0;
              const double inv = 1.0 / piv, l = ei * inv;
              iu[i * B] = inv;
              u1[i * B] = c1;
              z[i] = rc;
              c0 = fma(-l, c1, ai1);
              c1 = ei1;
              rc = fma(-l, rc, b1);
            } else {
              const double inv = 1.0 / ei, l = c0 * inv;
              iu[i * B] = inv;
              u1[i * B] = ai1;
              if (i < 64) sw0 |= 1ull << i; else sw1 |= 1ull << (i - 64);
              z[i] = b1;
              const double nc0 = fma(-l, ai1, c1);
              c1 = -l * ei1;
              c0 = nc0;
              rc = fma(-l, b1, rc);
            }
          }
          {
            const double piv = fabs(c0) < ptiny ? ptiny : c0;
            iu[(m - 1) * B] = 1.0 / piv;
            z[m - 1] = rc;
          }
          double zn1 = z[m - 1] * iu[(m - 1) * B], zn2 = 0.0;
          z[m - 1] = zn1;
          for (int i = m - 2; i >= 0; --i) {
            const bool s = i < 64 ? (sw0 >> i) & 1ull : (sw1 >> (i - 64)) & 1ull;
            const double u2 = s ? er[i + 1] : 0.0;
            const double zi = (z[i] - u1[i * B] * zn1 - u2 * zn2) * iu[i * B];
            z[i] = zi;
            zn2 = zn1;
            zn1 = zi;
          }
          double nrm = 0.0;
          for (int i = 0; i < m; ++i) nrm = fma(z[i], z[i], nrm);
          if (!(nrm > 0.0 && nrm < 1e300)) {
            s_fail = 2;
          } else {
            const double sc = rsqrt(nrm);
            for (int i = 0; i < m; ++i) z[i] *= sc;
          }
        }
        __syncthreads();
      }
      if (s_fail || it == 2) break;
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
    // CholQR2: Z <- Z R^{-1} with Z^T Z = R^T R, twice
    const int npair = nbx * (nbx + 1) / 2;
    for (int pass = 0; pass < 2 && fast; ++pass) {
      for (int pr = warp; pr < npair; pr += HEEV_WARPS) {
        int a = 0, rem = pr;
        while (rem >= nbx - a) {
          rem -= nbx - a;
          ++a;
        }
        const int b = a + rem;
        double s = 0.0;
        for (int i = lane; i < m; i += 32) s = fma(zT[a * ldz + i], zT[b * ldz + i], s);
        s = warp_sum(s);
        if (lane == 0) Hm[a * nbx + b] = s;
      }
      __syncthreads();
      if (warp == 0) {  // upper Cholesky factor R in place
        for (int j = 0; j < nbx; ++j) {
          const double piv = Hm[j * nbx + j];
          if (!(piv > 1e-20)) {  // columns are unit vectors: a pivot this small is a collapse
            if (lane == 0) s_fail = 3;
            break;
          }
          const double rj = sqrt(piv), ri = 1.0 / rj;
          __syncwarp();
          for (int c = j + 1 + lane; c < nbx; c += 32) Hm[j * nbx + c] *= ri;
          if (lane == 0) Hm[j * nbx + j] = rj;
          __syncwarp();
          const int rem = nbx - 1 - j;
          for (int q = lane; q < rem * rem; q += 32) {
            const int r = j + 1 + q / rem, c = j + 1 + q % rem;
            if (c >= r) Hm[r * nbx + c] -= Hm[j * nbx + r] * Hm[j * nbx + c];
          }
          __syncwarp();
        }
      }
      __syncthreads();
      if (s_fail) {
        fast = false;
        break;
      }
      // row i of Z: w R = z_i by forward substitution over the columns, one warp per row
      for (int i = warp; i < m; i += HEEV_WARPS) {
        double v[PER];
#pragma unroll
        for (int t = 0; t < PER; ++t) {
          const int b = lane + 32 * t;
          v[t] = b < nbx ? zT[b * ldz + i] : 0.0;
        }
#pragma unroll
        for (int ta = 0; ta < PER; ++ta) {
          for (int al = 0; al < 32; ++al) {
            const int a = 32 * ta + al;
            if (a >= nbx) break;
            double wa = __shfl_sync(0xffffffffu, v[ta], al) / Hm[a * nbx + a];
            if (lane == al) v[ta] = wa;
#pragma unroll
            for (int t = ta; t < PER; ++t) {
              const int b = lane + 32 * t;
              if (b > a && b < nbx) v[t] = fma(-wa, Hm[a * nbx + b], v[t]);
            }
          }
        }
#pragma unroll
        for (int t = 0; t < PER; ++t) {
          const int b = lane + 32 * t;
          if (b < nbx) zT[b * ldz + i] = v[t];
        }
      }
      __syncthreads();
    }
  }
  if (fast) {
    // H = Z^T T Z (full), Q = I
    const int npair = nbx * (nbx + 1) / 2;
    for (int pr = warp; pr < npair; pr += HEEV_WARPS) {
      int a = 0, rem = pr;
      while (rem >= nbx - a) {
        rem -= nbx - a;
        ++a;
      }
      const int b = a + rem;
      const double* za = zT + a * ldz;
      const double* zb = zT + b * ldz;
      double s = 0.0;
      for (int i = lane; i < m; i += 32) {
        double tz = d[i] * zb[i];
        if (i > 0) tz = fma(er[i - 1], zb[i - 1], tz);
        if (i + 1 < m) tz = fma(er[i], zb[i + 1], tz);
        s = fma(za[i], tz, s);
      }
      s = warp_sum(s);
      if (lane == 0) {
        Hm[a * nbx + b] = s;
        Hm[b * nbx + a] = s;
      }
    }
    for (int i = tid; i < nbx * nbx; i += blockDim.x) Qm[i] = (i / nbx == i % nbx) ? 1.0 : 0.0;
    __syncthreads();
    if (warp == 0) {  // cyclic Jacobi on the pairs above threshold
      const double thr = 2.0 * EPS * tnorm;
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
    // eigenvectors: v = Z Q[:, src], residual |T v - theta v|, y = Q_H D v
    cplx<double>* Uk = U + (int64_t)k * m * nb;
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
      cplx<double> y[PER];
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const int r = lane + 32 * t;
        y[t] = r < m ? scale(ph[r], v[t]) : mk<double>(0.0, 0.0);
      }
      apply_reflectors(y, m, lane, Hc, wv);
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const int r = lane + 32 * t;
        if (r < m) Uk[(int64_t)r * nb + ra] = y[t];
      }
      if (lane == 0) eig[(int64_t)k * nb + ra] = th;
    }
    __syncthreads();
    if (!s_fail) {
      if (tid == 0) info[k] = 0;
      return;
    }
  }

  // ---- QL path: implicit QL on (d, er), Z in the pool -----------------------
  if (tid == 0) atomicAdd(&g_heev_ql[s_fail > 0 ? s_fail - 1 : 0], 1ull);
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
    // plain doubles: the per-matrix offset k*m*m is only 8-byte aligned for odd m
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
    cplx<double> y[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      y[t] = r < m ? scale(ph[r], Z[(int64_t)src * m + r]) : mk<double>(0.0, 0.0);
    }
    apply_reflectors(y, m, lane, Hc, wv);
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int r = lane + 32 * t;
      if (r < m) Uk[(int64_t)r * nb + a] = y[t];
    }
  }
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

// One launch of the eigensolver with scratch z (nk * m * m float64).
static int launch_heev(int nk, int m, int nb, const void* S, int lds, int64_t sk, double* eig, void* U,
                       double* z, int* info, cudaStream_t st) {
  const int extra = heev_extra(m, nb);
  const size_t sm = heev_smem(m, nb);
  GWB_CUDA_TRY(cudaFuncSetAttribute(k_heev_lowest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_heev_lowest<<<nk, HEEV_THREADS, sm, st>>>((const cplx<double>*)S, lds, sk, m, nb, eig, (cplx<double>*)U, z,
                                              info, extra);
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

