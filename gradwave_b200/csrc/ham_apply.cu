// Batched plane-wave Hamiltonian apply H c = T c + V_loc c + sum p D <p|c>
// for all k-points and bands in a few launches (sm_100a).
//
// Local term (replaces gradwave core/batch.py:405-428). The sphere of each k
// occupies Miller indices |m_a| <= M_a of a box n0 x n1 x n2, so only
// L_a = 2 M_a + 1 planes/rows/columns per axis ever hold data:
//
//   K1 plane_inverse  one CTA per (axis-0 plane j0 < L0, band, k):
//                     scatter the sphere points of the plane into a shared-
//                     memory n1 x n2 plane, inverse FFT along axis 2 on the L1
//                     occupied rows, inverse FFT along axis 1 on all columns,
//                     store the plane to the scratch W (L0 planes per band).
//   K2 pencil_vloc    one CTA per (axis-1 row i1, band, k): load the L0 planes'
//                     row i1 as n2 pencils along axis 0, inverse FFT, multiply
//                     by v(r)/N, forward FFT, store back the L0 occupied planes
//                     (the V(r) psi(r) product never leaves shared memory).
//   K3 plane_forward  one CTA per (j0, band, k): forward FFT along axis 1 and
//                     along axis 2 on the occupied rows, gather the sphere,
//                     add the kinetic term t c, write out (padding zeroed).
//
// The bands are processed in chunks whose scratch W fits in L2, so W is
// written and re-read from L2 rather than HBM.
//
// Nonlocal term (replaces gradwave core/batch.py:499-500 and becp_b :590-595):
//   K4 becp_partial   becp partial sums conj(p) . c over a slice of G
//   K5 becp_reduce_d  sum of slices, times D  -> bd (nk, nb, nproj)
//   K6 nl_add         out += bd . p
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "fft.cuh"
#include "rdft.cuh"

namespace gwb {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
static std::atomic<unsigned long long> g_launches{0};
void count_launches(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

struct FftGeom {
  int n[3];
  int M[3];  // max |Miller index| per axis over all k (compact row map)
  int L[3];  // occupied extent per axis (2M+1, capped at n)
  AxisPlan plan[3];
};

}  // namespace gwb

struct gwb_ham {
  int device = 0;
  int nk = 0, npw_max = 0, nproj = 0;
  gwb::FftGeom g{};
  std::vector<int64_t> npw_host;
  // device tables
  int* d_npw = nullptr;
  int* d_plane_ptr = nullptr;  // (nk*L0 + 1)
  int* d_plane_g = nullptr;    // sphere index of each plane entry
  int* d_plane_pos = nullptr;  // i1*n2 + i2 of each plane entry
  double* d_t64 = nullptr;
  float* d_t32 = nullptr;
  double* d_v64 = nullptr;  // v(r)/N
  float* d_v32 = nullptr;
  gwb::cplx<double>* d_p64 = nullptr;
  gwb::cplx<float>* d_p32 = nullptr;
  double* d_d64 = nullptr;
  float* d_d32 = nullptr;
  double* d_q64 = nullptr;  // augmentation q_pq of the overlap S (USPP/PAW), when set
  float* d_q32 = nullptr;
  gwb::cplx<double>* d_tw64[3] = {nullptr, nullptr, nullptr};
  gwb::cplx<float>* d_tw32[3] = {nullptr, nullptr, nullptr};
  // scratch
  void* d_W = nullptr;
  size_t W_bytes = 0;
  void* d_part = nullptr;  // becp partials
  size_t part_bytes = 0;
  void* d_bd = nullptr;  // becp * D
  size_t bd_bytes = 0;
  void* d_bq = nullptr;  // becp * q (overlap apply)
  size_t bq_bytes = 0;
  // tensor-core nonlocal term (float32 applies of complex128 blocks)
  void* d_pplanes = nullptr;  // BF16 planes of P: (nk, 4, nproj, ldp)
  size_t pplanes_bytes = 0;
  bool pplanes_ok = false;
  void* d_cplanes = nullptr;  // BF16 planes of the input rows: (nk, 4, nb, ldp)
  size_t cplanes_bytes = 0;
  void* d_becp = nullptr;  // becp (nk, nb, nproj) complex128
  size_t becp_bytes = 0;
  void* d_bdplanes = nullptr;  // BF16 planes of becp D: (nk, 4, nb, ldq)
  size_t bdplanes_bytes = 0;
  void* d_tcwork = nullptr;  // split-K partial sums
  size_t tcwork_bytes = 0;
  int* d_tcstatus = nullptr;  // pipeline-wait timeouts of the tensor-core products
  double* d_rhok = nullptr;  // density accumulators, one box per k
  size_t rhok_bytes = 0;
  bool have_t = false, have_v = false, have_p = false, have_q = false;
  // tuning (gwb_ham_set_tuning; 0 = the built-in rule)
  size_t w_budget = 0;   // bytes of FFT scratch W per band chunk
  int nl_target = 0;     // CTAs the G-sliced becp contraction aims for
  int fft_nt[2] = {0, 0};  // threads of the shared-memory FFT blocks (float32, float64); 0: the built-in rule
};

namespace gwb {

static bool plan_axis(int n, AxisPlan* pl) {
  if (n < 2 || n > 128) return false;
  pl->n = n;
  pl->nst = 0;
  pl->code = 0;
  int m = n;
  const int order[7] = {8, 4, 6, 3, 2, 5, 7};
  while (m > 1) {
    bool found = false;
    for (int R : order) {
      if (m % R == 0) {
        if (pl->nst >= 8) return false;
        pl->code |= (unsigned)R << (4 * pl->nst);
        pl->nst++;
        m /= R;
        found = true;
        break;
      }
    }
    if (!found) return false;
  }
  return true;
}

static size_t w_budget_bytes() {
  const char* s = std::getenv("GWB_W_BUDGET_MB");
  long mb = s ? std::atol(s) : 48;
  if (mb < 1) mb = 1;
  return (size_t)mb << 20;
}

// ---------------------------------------------------------------------------
// K1: sphere scatter + inverse FFT along axes 2 and 1, one plane per CTA.
// Blocks per SM the shared-memory FFT kernels are compiled for: three 256-thread
// blocks (the 72^3 and 96^3 planes of float32 fit three per SM), one block of
// 512 or 1024 threads (float64 planes fill the shared memory with one).
template <typename T, int NT, bool CT> constexpr int fft_minb() {
  return !CT ? 1 : (NT == 256 ? 3 : (NT == 512 && sizeof(T) == 4 ? 2 : 1));
}

template <typename T, typename SIO, unsigned C1, unsigned C2, int NT = 256>
__global__ void __launch_bounds__(NT, (fft_minb<T, NT, (C1 && C2)>())) k_plane_inverse(FftGeom g, const int* __restrict__ plane_ptr,
                                                       const int* __restrict__ plane_g,
                                                       const int* __restrict__ plane_pos,
                                                       const SIO* __restrict__ c, cplx<T>* __restrict__ W,
                                                       const cplx<T>* __restrict__ tw1,
                                                       const cplx<T>* __restrict__ tw2, int64_t ck, int b0,
                                                       int nbc, int npw_max) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n1 = g.n[1], n2 = g.n[2], L0 = g.L[0];
  const int j0 = blockIdx.x, bl = blockIdx.y, k = blockIdx.z;
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* t1 = S + n1 * n2;
  cplx<T>* t2 = t1 + n1;
  for (int i = threadIdx.x; i < n1; i += blockDim.x) t1[i] = tw1[i];
  for (int i = threadIdx.x; i < n2; i += blockDim.x) t2[i] = tw2[i];
  for (int i = threadIdx.x; i < n1 * n2; i += blockDim.x) S[i] = mk<T>(0, 0);
  __syncthreads();
  const size_t crow = (size_t)k * ck + (size_t)(b0 + bl) * npw_max;
  const int e0 = plane_ptr[k * L0 + j0], e1 = plane_ptr[k * L0 + j0 + 1];
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) S[plane_pos[e]] = ld<T>(c, crow + plane_g[e]);
  __syncthreads();
  fft_any<T, false, +1, C2>(S, g.L[1], g.plan[2], n2, 1, g.M[1], n1, t2);
  fft_any<T, true, +1, C1>(S, n2, g.plan[1], 1, n2, n2, n2, t1);
  cplx<T>* dst = W + (((size_t)k * nbc + bl) * L0 + j0) * (size_t)(n1 * n2);
  for (int i = threadIdx.x; i < n1 * n2; i += blockDim.x) dst[i] = S[i];
}

// K2: pencils along axis 0 for one (i1, band, k): inverse FFT, x v(r)/N, forward FFT.
template <typename T, unsigned C0, int NT = 256>
__global__ void __launch_bounds__(NT, (fft_minb<T, NT, (C0 != 0)>())) k_pencil_vloc(FftGeom g, cplx<T>* __restrict__ W,
                                                     const T* __restrict__ v,
                                                     const cplx<T>* __restrict__ tw0, int nbc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2], L0 = g.L[0];
  const int i1 = blockIdx.x, bl = blockIdx.y, k = blockIdx.z;
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);  // [i0][i2]
  cplx<T>* t0 = S + n0 * n2;
  for (int i = threadIdx.x; i < n0; i += blockDim.x) t0[i] = tw0[i];
  cplx<T>* base = W + ((size_t)k * nbc + bl) * L0 * (size_t)(n1 * n2) + (size_t)i1 * n2;
  for (int i = threadIdx.x; i < n0 * n2; i += blockDim.x) {
    const int r = i / n2, i2 = i - r * n2;
    // memory row r holds compact plane j0 (or stays zero)
    int j0;
    if (r <= g.M[0]) j0 = r;
    else if (r >= n0 - (L0 - g.M[0] - 1)) j0 = r - (n0 - L0);
    else j0 = -1;
    S[i] = j0 >= 0 ? base[(size_t)j0 * n1 * n2 + i2] : mk<T>(0, 0);
  }
  __syncthreads();
  fft_any<T, true, +1, C0>(S, n2, g.plan[0], 1, n2, n2, n2, t0);
  for (int i = threadIdx.x; i < n0 * n2; i += blockDim.x) {
    const int i0 = i / n2, i2 = i - i0 * n2;
    S[i] = scale(S[i], v[((size_t)i0 * n1 + i1) * n2 + i2]);
  }
  __syncthreads();
  fft_any<T, true, -1, C0>(S, n2, g.plan[0], 1, n2, n2, n2, t0);
  for (int i = threadIdx.x; i < L0 * n2; i += blockDim.x) {
    const int j0 = i / n2, i2 = i - j0 * n2;
    const int r = rowmap(j0, g.M[0], L0, n0);
    base[(size_t)j0 * n1 * n2 + i2] = S[r * n2 + i2];
  }
}

// K2 with the whole axis-0 transform in registers (cubic box, N0 <= 48): one
// thread per pencil (i1, i2) of one (band, k); the occupied planes are loaded
// (coalesced over i2), inverse DFT, x v(r)/N, forward DFT, occupied planes
// stored back. No shared memory, no barriers; the plane stride is a constant,
// so every load and store is one base register plus an immediate offset.
template <typename T, int N0>
__global__ void __launch_bounds__(128) k_pencil_vloc_reg(FftGeom g, cplx<T>* __restrict__ W, const T* __restrict__ v,
                                                         int nbc) {
  constexpr int PLANE = N0 * N0;
  const int L0 = g.L[0], M0 = g.M[0];
  const int bl = blockIdx.y, k = blockIdx.z;
  const int pidx = blockIdx.x * blockDim.x + threadIdx.x;
  if (pidx >= PLANE) return;
  cplx<T>* base = W + ((size_t)k * nbc + bl) * L0 * (size_t)PLANE + pidx;
  // occupied rows: 0..M0 hold planes 0..M0; rows N0-(L0-M0-1)..N0-1 hold the
  // wrapped planes M0+1..L0-1, i.e. plane r - (N0 - L0)
  const int hi0 = N0 - (L0 - M0 - 1);
  cplx<T>* wrap = base - (ptrdiff_t)(N0 - L0) * PLANE;
  cplx<T> x[N0];
  rdft_detail::StaticFor<0, N0>::run([&](auto rc) {
    constexpr int r = decltype(rc)::value;
    x[r] = r <= M0 ? base[r * PLANE] : (r >= hi0 ? wrap[r * PLANE] : mk<T>(0, 0));
  });
  rdft<N0, +1>(x);
  const T* vp = v + pidx;
  rdft_detail::StaticFor<0, N0>::run([&](auto rc) {
    constexpr int r = decltype(rc)::value;
    x[r] = scale(x[r], vp[r * PLANE]);
  });
  rdft<N0, -1>(x);
  rdft_detail::StaticFor<0, N0>::run([&](auto rc) {
    constexpr int r = decltype(rc)::value;
    if (r <= M0) base[r * PLANE] = x[r];
    else if (r >= hi0) wrap[r * PLANE] = x[r];
  });
}

// Density (gradwave core/batch.py:562-587, density_b): after K1 has put a
// chunk of bands into W (inverse FFT along axes 2 and 1 over the occupied
// planes), the axis-0 inverse FFT of each pencil and rho_k[k][r] +=
// w[k][b] |psi_b(r)|^2, float64. One CTA (general box) or one thread (cubic
// box, whole pencil in registers) owns each output element of one k and loops
// over the chunk's bands, so the sums need no atomics and run in a fixed order.
template <typename T, unsigned C0>
__global__ void __launch_bounds__(256) k_pencil_density(FftGeom g, const cplx<T>* __restrict__ W,
                                                        const cplx<T>* __restrict__ tw0,
                                                        const double* __restrict__ w, int64_t wk, int b0, int nbc,
                                                        double* __restrict__ rho_k, int first) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2], L0 = g.L[0];
  const int i1 = blockIdx.x, k = blockIdx.z;
  const size_t N = (size_t)n0 * n1 * n2;
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);  // [i0][i2]
  cplx<T>* t0 = S + n0 * n2;
  for (int i = threadIdx.x; i < n0; i += blockDim.x) t0[i] = tw0[i];
  double* rk = rho_k + (size_t)k * N + (size_t)i1 * n2;
  if (first)
    for (int i = threadIdx.x; i < n0 * n2; i += blockDim.x) {
      const int i0 = i / n2, i2 = i - i0 * n2;
      rk[(size_t)i0 * n1 * n2 + i2] = 0.0;
    }
  for (int bl = 0; bl < nbc; ++bl) {
    const double wb = w[(size_t)k * wk + b0 + bl];
    if (wb == 0.0) continue;  // the same for every thread of the CTA
    const cplx<T>* base = W + ((size_t)k * nbc + bl) * L0 * (size_t)(n1 * n2) + (size_t)i1 * n2;
    __syncthreads();  // S of the previous band fully read
    for (int i = threadIdx.x; i < n0 * n2; i += blockDim.x) {
      const int r = i / n2, i2 = i - r * n2;
      int j0;
      if (r <= g.M[0]) j0 = r;
      else if (r >= n0 - (L0 - g.M[0] - 1)) j0 = r - (n0 - L0);
      else j0 = -1;
      S[i] = j0 >= 0 ? base[(size_t)j0 * n1 * n2 + i2] : mk<T>(0, 0);
    }
    __syncthreads();
    fft_any<T, true, +1, C0>(S, n2, g.plan[0], 1, n2, n2, n2, t0);
    __syncthreads();
    for (int i = threadIdx.x; i < n0 * n2; i += blockDim.x) {
      const int i0 = i / n2, i2 = i - i0 * n2;
      const cplx<T> v = S[i];
      rk[(size_t)i0 * n1 * n2 + i2] += wb * ((double)v.x * (double)v.x + (double)v.y * (double)v.y);
    }
  }
}

template <typename T, int N0>
__global__ void __launch_bounds__(128) k_pencil_density_reg(FftGeom g, const cplx<T>* __restrict__ W,
                                                            const double* __restrict__ w, int64_t wk, int b0,
                                                            int nbc, double* __restrict__ rho_k, int first) {
  constexpr int PLANE = N0 * N0;
  const int L0 = g.L[0], M0 = g.M[0];
  const int k = blockIdx.z;
  const int pidx = blockIdx.x * blockDim.x + threadIdx.x;
  if (pidx >= PLANE) return;
  double* rk = rho_k + (size_t)k * N0 * PLANE + pidx;
  if (first)
    rdft_detail::StaticFor<0, N0>::run([&](auto rc) { rk[decltype(rc)::value * PLANE] = 0.0; });
  const int hi0 = N0 - (L0 - M0 - 1);
  for (int bl = 0; bl < nbc; ++bl) {
    const double wb = w[(size_t)k * wk + b0 + bl];
    if (wb == 0.0) continue;
    const cplx<T>* base = W + ((size_t)k * nbc + bl) * L0 * (size_t)PLANE + pidx;
    const cplx<T>* wrap = base - (ptrdiff_t)(N0 - L0) * PLANE;
    cplx<T> x[N0];
    rdft_detail::StaticFor<0, N0>::run([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      x[r] = r <= M0 ? base[r * PLANE] : (r >= hi0 ? wrap[r * PLANE] : mk<T>(0, 0));
    });
    rdft<N0, +1>(x);
    rdft_detail::StaticFor<0, N0>::run([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      rk[r * PLANE] += wb * ((double)x[r].x * (double)x[r].x + (double)x[r].y * (double)x[r].y);
    });
  }
}

// rho[r] = scale sum_k rho_k[k][r], k in order.
__global__ void k_density_sum(int nk, int64_t N, const double* __restrict__ rho_k, double scale,
                              double* __restrict__ rho) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    double a = 0.0;
    for (int k = 0; k < nk; ++k) a += rho_k[(int64_t)k * N + i];
    rho[i] = scale * a;
  }
}

// K1 and K3 with whole transforms in registers (cubic box, N <= 48): a CTA
// takes PLR planes of one (band, k), N threads per plane, the planes in shared
// memory with rows padded to N + 1. K1: sphere scatter, one thread per
// occupied row runs the axis-2 inverse DFT, then one thread per column the
// axis-1 inverse DFT and writes the column (coalesced over i2) to W. K3: one
// thread per column loads it from W and runs the axis-1 forward DFT, one
// thread per occupied row the axis-2 forward DFT, then the sphere gather + t c.
// Two barriers after the staging, instead of two per radix pass.
constexpr int PLR = 4;  // planes per CTA

template <int N>
__device__ __forceinline__ int occ_row(int rr, int M, int L) {  // memory row of occupied row rr
  return rr <= M ? rr : rr + N - L;
}

template <typename T, typename SIO, int N>
__global__ void __launch_bounds__(PLR * N) k_plane_inverse_reg(FftGeom g, const int* __restrict__ plane_ptr,
                                                              const int* __restrict__ plane_g,
                                                              const int* __restrict__ plane_pos,
                                                              const SIO* __restrict__ c, cplx<T>* __restrict__ W,
                                                              int64_t ck, int b0, int nbc, int npw_max) {
  constexpr int LDS = N + 1, PS = N * LDS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);  // [PLR][N][LDS]
  const int L0 = g.L[0], L1 = g.L[1], M1 = g.M[1];
  const int jb = blockIdx.x * PLR, bl = blockIdx.y, k = blockIdx.z;
  const int np = min(PLR, L0 - jb);
  for (int i = threadIdx.x; i < PLR * PS; i += blockDim.x) S[i] = mk<T>(0, 0);
  __syncthreads();
  const size_t crow = (size_t)k * ck + (size_t)(b0 + bl) * npw_max;
  const int* pp = plane_ptr + k * L0 + jb;
  const int e0 = pp[0], e1 = pp[np];
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    int q = 0;
#pragma unroll
    for (int qq = 1; qq < PLR; ++qq) q += (qq < np && e >= pp[qq]) ? 1 : 0;
    const int pos = plane_pos[e], i1 = pos / N, i2 = pos - i1 * N;
    S[q * PS + i1 * LDS + i2] = ld<T>(c, crow + plane_g[e]);
  }
  __syncthreads();
  const int p = threadIdx.x / N, lane = threadIdx.x - p * N;
  if (p < np && lane < L1) {  // axis 2 (rows), occupied rows only
    cplx<T>* row = S + p * PS + occ_row<N>(lane, M1, L1) * LDS;
    cplx<T> x[N];
    rdft_detail::StaticFor<0, N>::run([&](auto qc) { x[decltype(qc)::value] = row[decltype(qc)::value]; });
    rdft<N, +1>(x);
    rdft_detail::StaticFor<0, N>::run([&](auto qc) { row[decltype(qc)::value] = x[decltype(qc)::value]; });
  }
  __syncthreads();
  if (p < np) {  // axis 1 (columns): the whole column out to W
    const cplx<T>* col = S + p * PS + lane;
    cplx<T> x[N];
    rdft_detail::StaticFor<0, N>::run([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      x[r] = col[r * LDS];
    });
    rdft<N, +1>(x);
    cplx<T>* dst = W + (((size_t)k * nbc + bl) * L0 + jb + p) * (size_t)(N * N) + lane;
    rdft_detail::StaticFor<0, N>::run([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      dst[r * N] = x[r];
    });
  }
}

template <typename T, typename SIO, int N>
__global__ void __launch_bounds__(PLR * N) k_plane_forward_reg(
    FftGeom g, const int* __restrict__ plane_ptr, const int* __restrict__ plane_g, const int* __restrict__ plane_pos,
    const int* __restrict__ npw, const SIO* __restrict__ c, SIO* __restrict__ out, const cplx<T>* __restrict__ W,
    const T* __restrict__ t, int64_t ck, int64_t ok, int b0, int nbc, int npw_max) {
  constexpr int LDS = N + 1, PS = N * LDS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);  // [PLR][N][LDS]
  const int L0 = g.L[0], L1 = g.L[1], M1 = g.M[1];
  const int jb = blockIdx.x * PLR, bl = blockIdx.y, k = blockIdx.z;
  const int np = min(PLR, L0 - jb);
  const int p = threadIdx.x / N, lane = threadIdx.x - p * N;
  const int hi1 = N - (L1 - M1 - 1);
  if (p < np) {  // axis 1 (columns) forward; keep the occupied rows
    const cplx<T>* src = W + (((size_t)k * nbc + bl) * L0 + jb + p) * (size_t)(N * N) + lane;
    cplx<T> x[N];
    rdft_detail::StaticFor<0, N>::run([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      x[r] = src[r * N];
    });
    rdft<N, -1>(x);
    cplx<T>* col = S + p * PS + lane;
    rdft_detail::StaticFor<0, N>::run([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      if (r <= M1 || r >= hi1) col[r * LDS] = x[r];
    });
  }
  __syncthreads();
  if (p < np && lane < L1) {  // axis 2 (rows) forward, occupied rows only
    cplx<T>* row = S + p * PS + occ_row<N>(lane, M1, L1) * LDS;
    cplx<T> x[N];
    rdft_detail::StaticFor<0, N>::run([&](auto qc) { x[decltype(qc)::value] = row[decltype(qc)::value]; });
    rdft<N, -1>(x);
    rdft_detail::StaticFor<0, N>::run([&](auto qc) { row[decltype(qc)::value] = x[decltype(qc)::value]; });
  }
  __syncthreads();
  const size_t crow = (size_t)k * ck + (size_t)(b0 + bl) * npw_max;
  const size_t orow = (size_t)k * ok + (size_t)(b0 + bl) * npw_max;
  const T* tk = t + (size_t)k * npw_max;
  const int* pp = plane_ptr + k * L0 + jb;
  const int e0 = pp[0], e1 = pp[np];
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    int q = 0;
#pragma unroll
    for (int qq = 1; qq < PLR; ++qq) q += (qq < np && e >= pp[qq]) ? 1 : 0;
    const int pos = plane_pos[e], i1 = pos / N, i2 = pos - i1 * N;
    const int gi = plane_g[e];
    const cplx<T> cv = ld<T>(c, crow + gi);
    st(out, orow + gi, S[q * PS + i1 * LDS + i2] + scale(cv, tk[gi]));
  }
  if (jb == 0) {
    for (int gi = npw[k] + threadIdx.x; gi < npw_max; gi += blockDim.x) st(out, orow + gi, mk<T>(0, 0));
  }
}

// K3: forward FFT along axes 1 and 2, sphere gather, + t c, padding zeroed.
template <typename T, typename SIO, unsigned C1, unsigned C2, int NT = 256>
__global__ void __launch_bounds__(NT, (fft_minb<T, NT, (C1 && C2)>())) k_plane_forward(
    FftGeom g, const int* __restrict__ plane_ptr, const int* __restrict__ plane_g,
    const int* __restrict__ plane_pos, const int* __restrict__ npw, const SIO* __restrict__ c,
    SIO* __restrict__ out, const cplx<T>* __restrict__ W, const T* __restrict__ t,
    const cplx<T>* __restrict__ tw1, const cplx<T>* __restrict__ tw2, int64_t ck, int64_t ok, int b0, int nbc,
    int npw_max) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n1 = g.n[1], n2 = g.n[2], L0 = g.L[0];
  const int j0 = blockIdx.x, bl = blockIdx.y, k = blockIdx.z;
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* t1 = S + n1 * n2;
  cplx<T>* t2 = t1 + n1;
  for (int i = threadIdx.x; i < n1; i += blockDim.x) t1[i] = tw1[i];
  for (int i = threadIdx.x; i < n2; i += blockDim.x) t2[i] = tw2[i];
  const cplx<T>* src = W + (((size_t)k * nbc + bl) * L0 + j0) * (size_t)(n1 * n2);
  for (int i = threadIdx.x; i < n1 * n2; i += blockDim.x) S[i] = src[i];
  __syncthreads();
  fft_any<T, true, -1, C1>(S, n2, g.plan[1], 1, n2, n2, n2, t1);
  fft_any<T, false, -1, C2>(S, g.L[1], g.plan[2], n2, 1, g.M[1], n1, t2);
  const size_t crow = (size_t)k * ck + (size_t)(b0 + bl) * npw_max;
  const size_t orow = (size_t)k * ok + (size_t)(b0 + bl) * npw_max;
  const int e0 = plane_ptr[k * L0 + j0], e1 = plane_ptr[k * L0 + j0 + 1];
  const T* tk = t + (size_t)k * npw_max;
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const int gi = plane_g[e];
    cplx<T> cv = ld<T>(c, crow + gi);
    st(out, orow + gi, S[plane_pos[e]] + scale(cv, tk[gi]));
  }
  if (j0 == 0) {
    for (int gi = npw[k] + threadIdx.x; gi < npw_max; gi += blockDim.x) st(out, orow + gi, mk<T>(0, 0));
  }
}

// ---------------------------------------------------------------------------
// Nonlocal term. Tiles: TB bands x TP projectors, G slices of TG.
constexpr int NL_TB = 16, NL_TP = 32, NL_TG = 32;

// K4: part[s][k][b][p] = sum_{g in slice s} conj(P[k][p][g]) c[k][b][g].
// The next step's tiles are loaded into registers while this step multiplies
// out of shared memory (one barrier pair per step).
template <typename T, typename SIO>
__global__ void __launch_bounds__(256) k_becp_partial(const SIO* __restrict__ c,
                                                      const cplx<T>* __restrict__ P,
                                                      cplx<T>* __restrict__ part, int nk, int nb,
                                                      int nproj, int npw_max, int gslice, int64_t ck) {
  constexpr int LC = NL_TB * NL_TG / 256, LP = NL_TP * NL_TG / 256;  // elements per thread per step
  __shared__ cplx<T> sc[NL_TB][NL_TG + 1];
  __shared__ cplx<T> sp[NL_TP][NL_TG + 1];
  const int pt = blockIdx.x, bt = blockIdx.y;
  const int k = blockIdx.z % nk, s = blockIdx.z / nk;
  const int tid = threadIdx.x;
  const int lb = tid / 16, lp = tid % 16;  // each thread: band lb, projectors lp and lp+16
  cplx<T> acc0 = mk<T>(0, 0), acc1 = mk<T>(0, 0);
  const int g_begin = s * gslice, g_end = min(npw_max, g_begin + gslice);
  cplx<T> rc[LC], rp[LP];
  auto fetch = [&](int gb) {
#pragma unroll
    for (int q = 0; q < LC; ++q) {
      const int i = tid + 256 * q, bb = i / NL_TG, gg = i % NL_TG;
      const int b = bt * NL_TB + bb, gi = gb + gg;
      rc[q] = (b < nb && gi < g_end) ? ld<T>(c, (size_t)k * ck + (size_t)b * npw_max + gi) : mk<T>(0, 0);
    }
#pragma unroll
    for (int q = 0; q < LP; ++q) {
      const int i = tid + 256 * q, pp = i / NL_TG, gg = i % NL_TG;
      const int p = pt * NL_TP + pp, gi = gb + gg;
      rp[q] = (p < nproj && gi < g_end) ? P[((size_t)k * nproj + p) * npw_max + gi] : mk<T>(0, 0);
    }
  };
  if (g_begin < g_end) fetch(g_begin);
  for (int gb = g_begin; gb < g_end; gb += NL_TG) {
#pragma unroll
    for (int q = 0; q < LC; ++q) {
      const int i = tid + 256 * q;
      sc[i / NL_TG][i % NL_TG] = rc[q];
    }
#pragma unroll
    for (int q = 0; q < LP; ++q) {
      const int i = tid + 256 * q;
      sp[i / NL_TG][i % NL_TG] = rp[q];
    }
    __syncthreads();
    if (gb + NL_TG < g_end) fetch(gb + NL_TG);
#pragma unroll 8
    for (int gg = 0; gg < NL_TG; ++gg) {
      const cplx<T> cv = sc[lb][gg];
      acc0 = acc0 + conj_mul(sp[lp][gg], cv);
      acc1 = acc1 + conj_mul(sp[lp + 16][gg], cv);
    }
    __syncthreads();
  }
  const int b = bt * NL_TB + lb;
  if (b < nb) {
    const size_t row = (((size_t)s * nk + k) * nb + b) * nproj;
    const int p0 = pt * NL_TP + lp, p1 = p0 + 16;
    if (p0 < nproj) part[row + p0] = acc0;
    if (p1 < nproj) part[row + p1] = acc1;
  }
}

// K5: bd[k][b][q] = sum_p (sum_s part[s][k][b][p]) D[p][q]. The slice sums
// are split over the threads (projector p, slice group) and combined in a
// fixed order (deterministic).
template <typename T>
__global__ void __launch_bounds__(128) k_becp_reduce_d(const cplx<T>* __restrict__ part, const T* __restrict__ D,
                                                       cplx<T>* __restrict__ bd, int nk, int nb, int nproj,
                                                       int nslice) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* becp = reinterpret_cast<cplx<T>*>(smem_raw);  // nproj
  cplx<T>* grp = becp + nproj;                            // nproj * ngrp partial sums
  const int kb = blockIdx.x;                               // k*nb + b
  const size_t stride = (size_t)nk * nb * nproj;
  const int ngrp = max(1, (int)blockDim.x / nproj);
  for (int idx = threadIdx.x; idx < nproj * ngrp; idx += blockDim.x) {
    const int p = idx % nproj, gq = idx / nproj;
    cplx<T> a = mk<T>(0, 0);
    for (int s = gq; s < nslice; s += ngrp) a = a + part[s * stride + (size_t)kb * nproj + p];
    grp[gq * nproj + p] = a;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < nproj; p += blockDim.x) {
    cplx<T> a = mk<T>(0, 0);
    for (int gq = 0; gq < ngrp; ++gq) a = a + grp[gq * nproj + p];
    becp[p] = a;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nproj; q += blockDim.x) {
    cplx<T> a = mk<T>(0, 0);
    for (int p = 0; p < nproj; ++p) a = a + scale(becp[p], D[(size_t)p * nproj + q]);
    bd[(size_t)kb * nproj + q] = a;
  }
}

// K6: out[k][b][g] += sum_q bd[k][b][q] P[k][q][g]; tiles TB bands x 64 G.
template <typename T, typename SIO>
__global__ void __launch_bounds__(256) k_nl_add(const cplx<T>* __restrict__ bd,
                                                const cplx<T>* __restrict__ P,
                                                SIO* __restrict__ out, int nk, int nb, int nproj,
                                                int npw_max, int64_t ok) {
  constexpr int TGO = 64, TQ = 16;
  __shared__ cplx<T> sb[NL_TB][TQ];
  __shared__ cplx<T> sp[TQ][TGO];
  const int gt = blockIdx.x, bt = blockIdx.y, k = blockIdx.z;
  const int tid = threadIdx.x;
  const int lg = tid % TGO, lb0 = tid / TGO;  // 4 band groups x 64 g; each thread 4 bands
  cplx<T> acc[4];
  const int gi_o = gt * TGO + lg;
#pragma unroll
  for (int i = 0; i < 4; ++i) {  // the output rows first: their loads overlap the tile staging below
    const int b = bt * NL_TB + lb0 * 4 + i;
    acc[i] = (gi_o < npw_max && b < nb) ? ld<T>(out, (size_t)k * ok + (size_t)b * npw_max + gi_o) : mk<T>(0, 0);
  }
  for (int q0 = 0; q0 < nproj; q0 += TQ) {
    for (int i = tid; i < NL_TB * TQ; i += blockDim.x) {
      const int bb = i / TQ, qq = i % TQ;
      const int b = bt * NL_TB + bb, q = q0 + qq;
      sb[bb][qq] = (b < nb && q < nproj) ? bd[((size_t)k * nb + b) * nproj + q] : mk<T>(0, 0);
    }
    for (int i = tid; i < TQ * TGO; i += blockDim.x) {
      const int qq = i / TGO, gg = i % TGO;
      const int q = q0 + qq, gi = gt * TGO + gg;
      sp[qq][gg] = (q < nproj && gi < npw_max) ? P[((size_t)k * nproj + q) * npw_max + gi] : mk<T>(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int qq = 0; qq < TQ; ++qq) {
      const cplx<T> pv = sp[qq][lg];
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] = acc[i] + sb[lb0 * 4 + i][qq] * pv;
    }
    __syncthreads();
  }
  if (gi_o < npw_max) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int b = bt * NL_TB + lb0 * 4 + i;
      if (b < nb) st(out, (size_t)k * ok + (size_t)b * npw_max + gi_o, acc[i]);
    }
  }
}

// K5 of the generalized apply: one pass over the slice partials gives both
// bd = becp D (H) and bq = becp q (S). Same fixed-order reduction as K5.
template <typename T>
__global__ void __launch_bounds__(128) k_becp_reduce_dq(const cplx<T>* __restrict__ part, const T* __restrict__ D,
                                                        const T* __restrict__ Q, cplx<T>* __restrict__ bd,
                                                        cplx<T>* __restrict__ bq, int nk, int nb, int nproj,
                                                        int nslice) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* becp = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* grp = becp + nproj;
  const int kb = blockIdx.x;
  const size_t stride = (size_t)nk * nb * nproj;
  const int ngrp = max(1, (int)blockDim.x / nproj);
  for (int idx = threadIdx.x; idx < nproj * ngrp; idx += blockDim.x) {
    const int p = idx % nproj, gq = idx / nproj;
    cplx<T> a = mk<T>(0, 0);
    for (int s = gq; s < nslice; s += ngrp) a = a + part[s * stride + (size_t)kb * nproj + p];
    grp[gq * nproj + p] = a;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < nproj; p += blockDim.x) {
    cplx<T> a = mk<T>(0, 0);
    for (int gq = 0; gq < ngrp; ++gq) a = a + grp[gq * nproj + p];
    becp[p] = a;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nproj; q += blockDim.x) {
    cplx<T> a = mk<T>(0, 0), b = mk<T>(0, 0);
    for (int p = 0; p < nproj; ++p) {
      a = a + scale(becp[p], D[(size_t)p * nproj + q]);
      b = b + scale(becp[p], Q[(size_t)p * nproj + q]);
    }
    bd[(size_t)kb * nproj + q] = a;
    bq[(size_t)kb * nproj + q] = b;
  }
}

// K6 of the generalized apply: each projector tile is read once for both
// outputs, out_h += bd P and out_s = (c + bq P) on the sphere, 0 in the
// padding (the overlap's mask).
template <typename T, typename SIO>
__global__ void __launch_bounds__(256) k_nl_add_hs(const cplx<T>* __restrict__ bd, const cplx<T>* __restrict__ bq,
                                                   const cplx<T>* __restrict__ P, const SIO* __restrict__ c,
                                                   int64_t ck, SIO* __restrict__ out_h, int64_t ohk,
                                                   SIO* __restrict__ out_s, int64_t osk,
                                                   const int* __restrict__ npw_k, int nk, int nb, int nproj,
                                                   int npw_max) {
  constexpr int TGO = 64, TQ = 16;
  __shared__ cplx<T> sb[NL_TB][TQ];
  __shared__ cplx<T> sq[NL_TB][TQ];
  __shared__ cplx<T> sp[TQ][TGO];
  const int gt = blockIdx.x, bt = blockIdx.y, k = blockIdx.z;
  const int tid = threadIdx.x;
  const int lg = tid % TGO, lb0 = tid / TGO;
  const int gi_o = gt * TGO + lg;
  const bool on_sphere = gi_o < npw_k[k];
  cplx<T> ah[4], as[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int b = bt * NL_TB + lb0 * 4 + i;
    const bool ok = gi_o < npw_max && b < nb;
    ah[i] = ok ? ld<T>(out_h, (size_t)k * ohk + (size_t)b * npw_max + gi_o) : mk<T>(0, 0);
    as[i] = (ok && on_sphere) ? ld<T>(c, (size_t)k * ck + (size_t)b * npw_max + gi_o) : mk<T>(0, 0);
  }
  for (int q0 = 0; q0 < nproj; q0 += TQ) {
    for (int i = tid; i < NL_TB * TQ; i += blockDim.x) {
      const int bb = i / TQ, qq = i % TQ;
      const int b = bt * NL_TB + bb, q = q0 + qq;
      const bool ok = b < nb && q < nproj;
      sb[bb][qq] = ok ? bd[((size_t)k * nb + b) * nproj + q] : mk<T>(0, 0);
      sq[bb][qq] = ok ? bq[((size_t)k * nb + b) * nproj + q] : mk<T>(0, 0);
    }
    for (int i = tid; i < TQ * TGO; i += blockDim.x) {
      const int qq = i / TGO, gg = i % TGO;
      const int q = q0 + qq, gi = gt * TGO + gg;
      sp[qq][gg] = (q < nproj && gi < npw_max) ? P[((size_t)k * nproj + q) * npw_max + gi] : mk<T>(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int qq = 0; qq < TQ; ++qq) {
      const cplx<T> pv = sp[qq][lg];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        ah[i] = ah[i] + sb[lb0 * 4 + i][qq] * pv;
        as[i] = as[i] + sq[lb0 * 4 + i][qq] * pv;
      }
    }
    __syncthreads();
  }
  if (gi_o < npw_max) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int b = bt * NL_TB + lb0 * 4 + i;
      if (b < nb) {
        st(out_h, (size_t)k * ohk + (size_t)b * npw_max + gi_o, ah[i]);
        st(out_s, (size_t)k * osk + (size_t)b * npw_max + gi_o, on_sphere ? as[i] : mk<T>(0, 0));
      }
    }
  }
}

template <typename T> __global__ void k_scale_copy(const double* src, T* dst, size_t n, double s) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (T)(src[i] * s);
}
__global__ void k_c128_to_c64(const cplx<double>* src, cplx<float>* dst, size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = mk<float>((float)src[i].x, (float)src[i].y);
}

static int ensure_buf(void** p, size_t* have, size_t need) {
  if (*have >= need) return GWB_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  if (cudaMalloc(p, need) != cudaSuccess) {
    cudaGetLastError();
    set_error("device allocation of " + std::to_string(need) + " bytes failed");
    return GWB_ERR_ALLOC;
  }
  *have = need;
  return GWB_OK;
}

static size_t plane_smem(const FftGeom& g, size_t es) {
  return (size_t)(g.n[1] * g.n[2] + g.n[1] + g.n[2]) * es;
}
static size_t pencil_smem(const FftGeom& g, size_t es) {
  return (size_t)(g.n[0] * g.n[2] + g.n[0]) * es;
}

// G slices of the becp reduction: enough CTAs to fill the GPU (4 per SM)
// with every slice at least 256 plane waves long.
static int nl_slices(const gwb_ham* h, int nb) {
  const int tiles = ((h->nproj + NL_TP - 1) / NL_TP) * ((nb + NL_TB - 1) / NL_TB) * h->nk;
  const int target = h->nl_target > 0 ? h->nl_target : 4 * 148;
  const int want = (target + tiles - 1) / tiles;
  const int cap = std::max(1, h->npw_max / 256);
  return std::max(1, std::min(want, cap));
}

// Compile-time FFT plans instantiated for the cubic boxes of the workloads
// (24 = 8*3, 36 = 4*3*3, 72 = 8*3*3, 96 = 8*4*3); any other box runs the
// runtime-plan kernels.
constexpr unsigned kCode24 = 0x38u, kCode36 = 0x334u, kCode72 = 0x338u, kCode96 = 0x348u;

// The shared-memory kernels of one band chunk (K1, K2, K3) with NT threads per block.
template <typename T, typename SIO, unsigned C, int NT>
static int local_shared(gwb_ham* h, const SIO* c, int64_t ck, SIO* out, int64_t ok, cplx<T>* W, const T* v,
                        const T* t, const cplx<T>* tw0, const cplx<T>* tw1, const cplx<T>* tw2, int b0, int cb,
                        cudaStream_t st, size_t smA, size_t smB) {
  const FftGeom& g = h->g;
  GWB_CUDA_TRY(allow_smem(k_plane_inverse<T, SIO, C, C, NT>));
  GWB_CUDA_TRY(allow_smem(k_plane_forward<T, SIO, C, C, NT>));
  GWB_CUDA_TRY(allow_smem(k_pencil_vloc<T, C, NT>));
  dim3 gA(g.L[0], cb, h->nk), gB(g.n[1], cb, h->nk);
  k_plane_inverse<T, SIO, C, C, NT><<<gA, NT, smA, st>>>(g, h->d_plane_ptr, h->d_plane_g, h->d_plane_pos, c, W, tw1,
                                                        tw2, ck, b0, cb, h->npw_max);
  k_pencil_vloc<T, C, NT><<<gB, NT, smB, st>>>(g, W, v, tw0, cb);
  k_plane_forward<T, SIO, C, C, NT><<<gA, NT, smA, st>>>(g, h->d_plane_ptr, h->d_plane_g, h->d_plane_pos, h->d_npw,
                                                        c, out, W, t, tw1, tw2, ck, ok, b0, cb, h->npw_max);
  return GWB_OK;
}

template <typename T, typename SIO, unsigned C>
static int local_chunks(gwb_ham* h, const SIO* c, int64_t ck, SIO* out, int64_t ok, int nb, int nbc,
                        cudaStream_t st, size_t smA, size_t smB) {
  const FftGeom& g = h->g;
  const bool dbl = sizeof(T) == 8;
  const cplx<T>* tw0 = dbl ? (const cplx<T>*)h->d_tw64[0] : (const cplx<T>*)h->d_tw32[0];
  const cplx<T>* tw1 = dbl ? (const cplx<T>*)h->d_tw64[1] : (const cplx<T>*)h->d_tw32[1];
  const cplx<T>* tw2 = dbl ? (const cplx<T>*)h->d_tw64[2] : (const cplx<T>*)h->d_tw32[2];
  const T* v = dbl ? (const T*)h->d_v64 : (const T*)h->d_v32;
  const T* t = dbl ? (const T*)h->d_t64 : (const T*)h->d_t32;
  cplx<T>* W = (cplx<T>*)h->d_W;
  const bool cubic = g.n[0] == g.n[1] && g.n[1] == g.n[2];
  const int nreg = (cubic && g.n[0] == 36 && C == kCode36) ? 36 : ((cubic && g.n[0] == 24 && C == kCode24) ? 24 : 0);
  const size_t smR = (size_t)PLR * nreg * (nreg + 1) * sizeof(cplx<T>);
  if (nreg == 36) {
    GWB_CUDA_TRY(allow_smem(k_plane_inverse_reg<T, SIO, 36>));
    GWB_CUDA_TRY(allow_smem(k_plane_forward_reg<T, SIO, 36>));
  } else if (nreg == 24) {
    GWB_CUDA_TRY(allow_smem(k_plane_inverse_reg<T, SIO, 24>));
    GWB_CUDA_TRY(allow_smem(k_plane_forward_reg<T, SIO, 24>));
  }
  for (int b0 = 0; b0 < nb; b0 += nbc) {
    const int cb = std::min(nbc, nb - b0);
    dim3 gA(g.L[0], cb, h->nk), gB(g.n[1], cb, h->nk), gP((g.L[0] + PLR - 1) / PLR, cb, h->nk);
    dim3 gR((g.n[1] * g.n[2] + 127) / 128, cb, h->nk);
    if (nreg == 36) {
      k_plane_inverse_reg<T, SIO, 36><<<gP, PLR * 36, smR, st>>>(g, h->d_plane_ptr, h->d_plane_g, h->d_plane_pos, c,
                                                                 W, ck, b0, cb, h->npw_max);
      k_pencil_vloc_reg<T, 36><<<gR, 128, 0, st>>>(g, W, v, cb);
      k_plane_forward_reg<T, SIO, 36><<<gP, PLR * 36, smR, st>>>(g, h->d_plane_ptr, h->d_plane_g, h->d_plane_pos,
                                                                 h->d_npw, c, out, W, t, ck, ok, b0, cb, h->npw_max);
    } else if (nreg == 24) {
      k_plane_inverse_reg<T, SIO, 24><<<gP, PLR * 24, smR, st>>>(g, h->d_plane_ptr, h->d_plane_g, h->d_plane_pos, c,
                                                                 W, ck, b0, cb, h->npw_max);
      k_pencil_vloc_reg<T, 24><<<gR, 128, 0, st>>>(g, W, v, cb);
      k_plane_forward_reg<T, SIO, 24><<<gP, PLR * 24, smR, st>>>(g, h->d_plane_ptr, h->d_plane_g, h->d_plane_pos,
                                                                 h->d_npw, c, out, W, t, ck, ok, b0, cb, h->npw_max);
    } else {
      // threads per block of the large compile-time boxes (72^3, 96^3):
      // gwb_ham_set_fft_threads, else 512 (float32: two 73 KB planes per SM)
      // and 1024 (float64: one 147 KB plane per SM). Measured on the 96^3
      // box of si216, 480 bands: float32 6.35 -> 6.26 ms, float64 16.7 ->
      // 12.0 ms against 256 threads.
      const int nt = h->fft_nt[dbl ? 1 : 0] ? h->fft_nt[dbl ? 1 : 0] : (dbl ? 1024 : 512);
      int rc = GWB_OK;
      if constexpr (C == kCode96 || C == kCode72) {
        if (nt == 1024) rc = local_shared<T, SIO, C, 1024>(h, c, ck, out, ok, W, v, t, tw0, tw1, tw2, b0, cb, st, smA, smB);
        else if (nt == 512) rc = local_shared<T, SIO, C, 512>(h, c, ck, out, ok, W, v, t, tw0, tw1, tw2, b0, cb, st, smA, smB);
        else rc = local_shared<T, SIO, C, 256>(h, c, ck, out, ok, W, v, t, tw0, tw1, tw2, b0, cb, st, smA, smB);
      } else {
        rc = local_shared<T, SIO, C, 256>(h, c, ck, out, ok, W, v, t, tw0, tw1, tw2, b0, cb, st, smA, smB);
      }
      if (rc != GWB_OK) return rc;
    }
    GWB_LAUNCH_CHECK();
    count_launches(3);
  }
  return GWB_OK;
}

int tc_becp_d_planes(int nk, int nb, int nproj, const cplx<double>* becp, const double* D, void* planes, int64_t ldq,
                     cudaStream_t st);

// Projector counts from which the float32 apply of complex128 blocks runs its
// nonlocal term on the tensor cores (GWB_TC_NONLOCAL=0 keeps the CUDA-core
// kernels everywhere).
constexpr int TC_NONLOCAL_MIN_NPROJ = 128;

static bool tc_nonlocal_enabled(const gwb_ham* h) {
  static const bool env_on = [] {
    const char* v = std::getenv("GWB_TC_NONLOCAL");
    return !(v && v[0] == '0');
  }();
  return env_on && h->nproj >= TC_NONLOCAL_MIN_NPROJ;
}

// out += P^T D (P^* . c) with split-BF16 tensor-core products:
// becp = c P^H (A B^H, FP32 accumulation, float64 slice sums), bd = becp D in
// float64 written as BF16 planes, out += bd P (A B, P read MN-major). The
// BF16 planes of P are built once per set of projectors.
static int nonlocal_tc(gwb_ham* h, const cplx<double>* c, int64_t ck, cplx<double>* out, int64_t ok, int nb,
                       cudaStream_t st) {
  const int nk = h->nk, np = h->nproj, npw = h->npw_max;
  const int64_t ldp = ((int64_t)npw + 7) / 8 * 8, ldq = ((int64_t)np + 7) / 8 * 8;
  int rc;
  if (!h->d_tcstatus) {
    GWB_CUDA_TRY(cudaMalloc((void**)&h->d_tcstatus, sizeof(int)));
    GWB_CUDA_TRY(cudaMemsetAsync(h->d_tcstatus, 0, sizeof(int), st));
  }
  if (!h->pplanes_ok) {
    if ((rc = ensure_buf(&h->d_pplanes, &h->pplanes_bytes, (size_t)nk * 4 * np * ldp * 2))) return rc;
    if ((rc = gwb_tc_planes(nk, np, npw, h->d_p64, npw, (int64_t)np * npw, GWB_C128, 0, h->d_pplanes, ldp, np, 0,
                            st)))
      return rc;
    h->pplanes_ok = true;
  }
  if ((rc = ensure_buf(&h->d_cplanes, &h->cplanes_bytes, (size_t)nk * 4 * nb * ldp * 2))) return rc;
  if ((rc = ensure_buf(&h->d_becp, &h->becp_bytes, (size_t)nk * nb * np * 16))) return rc;
  if ((rc = ensure_buf(&h->d_bdplanes, &h->bdplanes_bytes, (size_t)nk * 4 * nb * ldq * 2))) return rc;
  const int64_t wb = gwb_zgemm_tc_work_bytes(2, nb, np, npw, nk);
  if (wb > 0 && (rc = ensure_buf(&h->d_tcwork, &h->tcwork_bytes, (size_t)wb))) return rc;
  if ((rc = gwb_tc_planes(nk, nb, npw, c, npw, ck, GWB_C128, 0, h->d_cplanes, ldp, nb, 0, st))) return rc;
  if ((rc = gwb_zgemm_tc(2, nb, np, npw, 1.0, 0.0, h->d_cplanes, ldp, nb, h->d_pplanes, ldp, np, 0.0, 0.0, h->d_becp,
                         np, (int64_t)nb * np, nk, h->d_tcwork, h->tcwork_bytes, h->d_tcstatus, st)))
    return rc;
  if ((rc = tc_becp_d_planes(nk, nb, np, (const cplx<double>*)h->d_becp, h->d_d64, h->d_bdplanes, ldq, st))) return rc;
  return gwb_zgemm_tc(0, nb, npw, np, 1.0, 0.0, h->d_bdplanes, ldq, nb, h->d_pplanes, ldp, np, 1.0, 0.0, out, npw, ok,
                      nk, nullptr, 0, h->d_tcstatus, st);
}

// out = T c + local(c): the kinetic and FFT local terms, band chunks sized to L2.
template <typename T, typename SIO>
static int local_term(gwb_ham* h, const SIO* c, int64_t ck, SIO* out, int64_t ok, int nb, cudaStream_t st) {
  const FftGeom& g = h->g;
  const size_t es = sizeof(cplx<T>);
  const size_t plane_elems = (size_t)g.n[1] * g.n[2];
  const size_t per_band = (size_t)h->nk * g.L[0] * plane_elems * es;
  // balanced chunks: as few as the L2 budget allows, all of (nearly) equal size
  const size_t budget = std::max(h->w_budget ? h->w_budget : w_budget_bytes(), per_band);
  const size_t max_nbc = std::max<size_t>(1, budget / per_band);
  const size_t nchunks = ((size_t)nb + max_nbc - 1) / max_nbc;
  int nbc = (int)(((size_t)nb + nchunks - 1) / nchunks);
  if (nbc < 1) nbc = 1;
  int rc = ensure_buf(&h->d_W, &h->W_bytes, per_band * nbc);
  if (rc) return rc;
  const size_t smA = plane_smem(g, es), smB = pencil_smem(g, es);
  const unsigned c0 = g.plan[0].code, c1 = g.plan[1].code, c2 = g.plan[2].code;
  const bool cubic = c0 == c1 && c1 == c2;
  int rcl;
  if (cubic && c0 == kCode24) rcl = local_chunks<T, SIO, kCode24>(h, c, ck, out, ok, nb, nbc, st, smA, smB);
  else if (cubic && c0 == kCode36) rcl = local_chunks<T, SIO, kCode36>(h, c, ck, out, ok, nb, nbc, st, smA, smB);
  else if (cubic && c0 == kCode72) rcl = local_chunks<T, SIO, kCode72>(h, c, ck, out, ok, nb, nbc, st, smA, smB);
  else if (cubic && c0 == kCode96) rcl = local_chunks<T, SIO, kCode96>(h, c, ck, out, ok, nb, nbc, st, smA, smB);
  else rcl = local_chunks<T, SIO, 0u>(h, c, ck, out, ok, nb, nbc, st, smA, smB);
  return rcl;
}

// The nonlocal slices: enough G slices to fill the GPU for this band count.
template <typename T>
static int nl_geometry(gwb_ham* h, int nb, int* gslice, int* nsl) {
  const int ns = nl_slices(h, nb);
  *gslice = ((h->npw_max + ns - 1) / ns + NL_TG - 1) / NL_TG * NL_TG;
  *nsl = (h->npw_max + *gslice - 1) / *gslice;
  const size_t es = sizeof(cplx<T>);
  int rc = ensure_buf(&h->d_part, &h->part_bytes, (size_t)*nsl * h->nk * nb * h->nproj * es);
  if (rc) return rc;
  return ensure_buf(&h->d_bd, &h->bd_bytes, (size_t)h->nk * nb * h->nproj * es);
}

template <typename T, typename SIO>
static int apply_impl(gwb_ham* h, const SIO* c, int64_t ck, SIO* out, int64_t ok, int nb, cudaStream_t st) {
  const size_t es = sizeof(cplx<T>);
  const bool dbl = sizeof(T) == 8;
  int rc = local_term<T, SIO>(h, c, ck, out, ok, nb, st);
  if (rc) return rc;
  if constexpr (std::is_same<T, float>::value && std::is_same<SIO, cplx<double>>::value) {
    if (h->nproj > 0 && tc_nonlocal_enabled(h)) return nonlocal_tc(h, c, ck, out, ok, nb, st);
  }
  if (h->nproj > 0) {
    int gslice = 0, nsl = 0;
    if ((rc = nl_geometry<T>(h, nb, &gslice, &nsl))) return rc;
    const cplx<T>* P = dbl ? (const cplx<T>*)h->d_p64 : (const cplx<T>*)h->d_p32;
    const T* D = dbl ? (const T*)h->d_d64 : (const T*)h->d_d32;
    dim3 g4((h->nproj + NL_TP - 1) / NL_TP, (nb + NL_TB - 1) / NL_TB, h->nk * nsl);
    k_becp_partial<T, SIO><<<g4, 256, 0, st>>>(c, P, (cplx<T>*)h->d_part, h->nk, nb, h->nproj, h->npw_max, gslice, ck);
    const int ngrp = std::max(1, 128 / h->nproj);
    k_becp_reduce_d<T><<<h->nk * nb, 128, (size_t)h->nproj * (1 + ngrp) * es, st>>>(
        (const cplx<T>*)h->d_part, D, (cplx<T>*)h->d_bd, h->nk, nb, h->nproj, nsl);
    dim3 g6((h->npw_max + 63) / 64, (nb + NL_TB - 1) / NL_TB, h->nk);
    k_nl_add<T, SIO><<<g6, 256, 0, st>>>((const cplx<T>*)h->d_bd, P, out, h->nk, nb, h->nproj, h->npw_max, ok);
    GWB_LAUNCH_CHECK();
    count_launches(3);
  }
  return GWB_OK;
}


// Generalized apply: out_h = H c and out_s = S c = (c + sum_pq |p> q_pq <q|c>)
// masked, from one becp contraction (CUDA cores, every precision).
template <typename T, typename SIO>
static int apply_hs_impl(gwb_ham* h, const SIO* c, int64_t ck, SIO* out_h, int64_t ohk, SIO* out_s, int64_t osk,
                         int nb, cudaStream_t st) {
  const size_t es = sizeof(cplx<T>);
  const bool dbl = sizeof(T) == 8;
  int rc = local_term<T, SIO>(h, c, ck, out_h, ohk, nb, st);
  if (rc) return rc;
  const cplx<T>* P = dbl ? (const cplx<T>*)h->d_p64 : (const cplx<T>*)h->d_p32;
  if (h->nproj > 0) {
    int gslice = 0, nsl = 0;
    if ((rc = nl_geometry<T>(h, nb, &gslice, &nsl))) return rc;
    if ((rc = ensure_buf(&h->d_bq, &h->bq_bytes, (size_t)h->nk * nb * h->nproj * es))) return rc;
    const T* D = dbl ? (const T*)h->d_d64 : (const T*)h->d_d32;
    const T* Q = dbl ? (const T*)h->d_q64 : (const T*)h->d_q32;
    dim3 g4((h->nproj + NL_TP - 1) / NL_TP, (nb + NL_TB - 1) / NL_TB, h->nk * nsl);
    k_becp_partial<T, SIO><<<g4, 256, 0, st>>>(c, P, (cplx<T>*)h->d_part, h->nk, nb, h->nproj, h->npw_max, gslice, ck);
    const int ngrp = std::max(1, 128 / h->nproj);
    k_becp_reduce_dq<T><<<h->nk * nb, 128, (size_t)h->nproj * (1 + ngrp) * es, st>>>(
        (const cplx<T>*)h->d_part, D, Q, (cplx<T>*)h->d_bd, (cplx<T>*)h->d_bq, h->nk, nb, h->nproj, nsl);
    count_launches(2);
  }
  dim3 g6((h->npw_max + 63) / 64, (nb + NL_TB - 1) / NL_TB, h->nk);
  k_nl_add_hs<T, SIO><<<g6, 256, 0, st>>>((const cplx<T>*)h->d_bd, (const cplx<T>*)h->d_bq, P, c, ck, out_h, ohk,
                                          out_s, osk, h->d_npw, h->nk, nb, h->nproj, h->npw_max);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

// Density of nb bands (float64 FFTs): K1 per band chunk into W, then the
// pencil kernel accumulating w |psi|^2 into rho_k, finally the k sum.
template <typename SIO, unsigned C>
static int density_chunks(gwb_ham* h, const SIO* c, int64_t ck, int nb, int nbc, const double* w, int64_t wk,
                          cudaStream_t st, size_t smA, size_t smB) {
  using T = double;
  const FftGeom& g = h->g;
  const cplx<T>* tw0 = (const cplx<T>*)h->d_tw64[0];
  const cplx<T>* tw1 = (const cplx<T>*)h->d_tw64[1];
  const cplx<T>* tw2 = (const cplx<T>*)h->d_tw64[2];
  cplx<T>* W = (cplx<T>*)h->d_W;
  const bool cubic = g.n[0] == g.n[1] && g.n[1] == g.n[2];
  const int nreg = (cubic && g.n[0] == 36 && C == kCode36) ? 36 : ((cubic && g.n[0] == 24 && C == kCode24) ? 24 : 0);
  const size_t smR = (size_t)PLR * nreg * (nreg + 1) * sizeof(cplx<T>);
  GWB_CUDA_TRY(allow_smem(k_plane_inverse<T, SIO, C, C>));
  GWB_CUDA_TRY(allow_smem(k_pencil_density<T, C>));
  if (nreg == 36) GWB_CUDA_TRY(allow_smem(k_plane_inverse_reg<T, SIO, 36>));
  if (nreg == 24) GWB_CUDA_TRY(allow_smem(k_plane_inverse_reg<T, SIO, 24>));
  for (int b0 = 0; b0 < nb; b0 += nbc) {
    const int cb = std::min(nbc, nb - b0);
    const int first = b0 == 0;
    dim3 gA(g.L[0], cb, h->nk), gP((g.L[0] + PLR - 1) / PLR, cb, h->nk);
    dim3 gR((g.n[1] * g.n[2] + 127) / 128, 1, h->nk), gB(g.n[1], 1, h->nk);
    if (nreg == 36) {
      k_plane_inverse_reg<T, SIO, 36><<<gP, PLR * 36, smR, st>>>(g, h->d_plane_ptr, h->d_plane_g, h->d_plane_pos, c,
                                                                 W, ck, b0, cb, h->npw_max);
      k_pencil_density_reg<T, 36><<<gR, 128, 0, st>>>(g, W, w, wk, b0, cb, h->d_rhok, first);
    } else if (nreg == 24) {
      k_plane_inverse_reg<T, SIO, 24><<<gP, PLR * 24, smR, st>>>(g, h->d_plane_ptr, h->d_plane_g, h->d_plane_pos, c,
                                                                 W, ck, b0, cb, h->npw_max);
      k_pencil_density_reg<T, 24><<<gR, 128, 0, st>>>(g, W, w, wk, b0, cb, h->d_rhok, first);
    } else {
      k_plane_inverse<T, SIO, C, C><<<gA, 256, smA, st>>>(g, h->d_plane_ptr, h->d_plane_g, h->d_plane_pos, c, W,
                                                         tw1, tw2, ck, b0, cb, h->npw_max);
      k_pencil_density<T, C><<<gB, 256, smB, st>>>(g, W, tw0, w, wk, b0, cb, h->d_rhok, first);
    }
    GWB_LAUNCH_CHECK();
    count_launches(2);
  }
  return GWB_OK;
}

template <typename SIO>
static int density_impl(gwb_ham* h, const SIO* c, int64_t ck, int nb, const double* w, int64_t wk, double scale,
                        double* rho, cudaStream_t st) {
  const FftGeom& g = h->g;
  const size_t es = sizeof(cplx<double>);
  const size_t N = (size_t)g.n[0] * g.n[1] * g.n[2];
  const size_t per_band = (size_t)h->nk * g.L[0] * g.n[1] * g.n[2] * es;
  const size_t budget = std::max(h->w_budget ? h->w_budget : w_budget_bytes(), per_band);
  const size_t max_nbc = std::max<size_t>(1, budget / per_band);
  const size_t nchunks = ((size_t)nb + max_nbc - 1) / max_nbc;
  int nbc = (int)(((size_t)nb + nchunks - 1) / nchunks);
  if (nbc < 1) nbc = 1;
  int rc = ensure_buf(&h->d_W, &h->W_bytes, per_band * nbc);
  if (rc) return rc;
  rc = ensure_buf((void**)&h->d_rhok, &h->rhok_bytes, (size_t)h->nk * N * sizeof(double));
  if (rc) return rc;
  const size_t smA = plane_smem(g, es), smB = pencil_smem(g, es);
  const unsigned c0 = g.plan[0].code, c1 = g.plan[1].code, c2 = g.plan[2].code;
  const bool cubic = c0 == c1 && c1 == c2;
  if (cubic && c0 == kCode24) rc = density_chunks<SIO, kCode24>(h, c, ck, nb, nbc, w, wk, st, smA, smB);
  else if (cubic && c0 == kCode36) rc = density_chunks<SIO, kCode36>(h, c, ck, nb, nbc, w, wk, st, smA, smB);
  else if (cubic && c0 == kCode72) rc = density_chunks<SIO, kCode72>(h, c, ck, nb, nbc, w, wk, st, smA, smB);
  else if (cubic && c0 == kCode96) rc = density_chunks<SIO, kCode96>(h, c, ck, nb, nbc, w, wk, st, smA, smB);
  else rc = density_chunks<SIO, 0u>(h, c, ck, nb, nbc, w, wk, st, smA, smB);
  if (rc) return rc;
  const int blocks = (int)std::min<size_t>((N + 255) / 256, 148 * 8);
  k_density_sum<<<blocks, 256, 0, st>>>(h->nk, (int64_t)N, h->d_rhok, scale, rho);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}
}  // namespace gwb

using namespace gwb;

extern "C" {

const char* gwb_last_error(void) { return g_last_error.c_str(); }
const char* gwb_version(void) { return "gwb 0.1 sm_100a"; }
unsigned long long gwb_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int gwb_ham_create(const gwb_ham_geometry* geom, int device, gwb_ham** out) {
  GWB_REQUIRE(geom && out, "null argument");
  GWB_REQUIRE(geom->nk > 0 && geom->npw_max > 0 && geom->nproj >= 0, "bad nk/npw_max/nproj");
  GWB_REQUIRE(geom->npw && geom->flat_idx, "null npw/flat_idx");
  *out = nullptr;
  auto* h = new gwb_ham();
  h->device = device;
  h->nk = geom->nk;
  h->npw_max = geom->npw_max;
  h->nproj = geom->nproj;
  FftGeom& g = h->g;
  for (int a = 0; a < 3; ++a) {
    g.n[a] = geom->n[a];
    if (!plan_axis(g.n[a], &g.plan[a])) {
      delete h;
      set_error("FFT axis length " + std::to_string(geom->n[a]) + " unsupported (need <=128, factors 2,3,5,7)");
      return GWB_ERR_ARG;
    }
  }
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const int64_t nbox = (int64_t)n0 * n1 * n2;
  h->npw_host.assign(geom->npw, geom->npw + geom->nk);
  // Miller extents over all k
  int M[3] = {0, 0, 0};
  for (int k = 0; k < h->nk; ++k) {
    const int64_t np_k = h->npw_host[k];
    if (np_k < 0 || np_k > h->npw_max) {
      delete h;
      set_error("npw[k] out of range");
      return GWB_ERR_ARG;
    }
    for (int64_t gi = 0; gi < np_k; ++gi) {
      const int64_t f = geom->flat_idx[(size_t)k * h->npw_max + gi];
      if (f < 0 || f >= nbox) {
        delete h;
        set_error("flat_idx out of the box");
        return GWB_ERR_ARG;
      }
      const int idx[3] = {(int)(f / ((int64_t)n1 * n2)), (int)((f / n2) % n1), (int)(f % n2)};
      for (int a = 0; a < 3; ++a) {
        const int m = idx[a] <= g.n[a] / 2 ? idx[a] : idx[a] - g.n[a];
        M[a] = std::max(M[a], std::abs(m));
      }
    }
  }
  for (int a = 0; a < 3; ++a) {
    g.L[a] = std::min(2 * M[a] + 1, g.n[a]);
    g.M[a] = g.L[a] == g.n[a] ? g.n[a] : M[a];
  }
  const int L0 = g.L[0];
  // sphere points grouped by compact axis-0 plane
  std::vector<int> cnt((size_t)h->nk * L0 + 1, 0);
  auto compact0 = [&](int i0) -> int {
    if (g.L[0] == n0) return i0;
    if (i0 <= g.M[0]) return i0;
    return i0 - (n0 - L0);
  };
  for (int k = 0; k < h->nk; ++k)
    for (int64_t gi = 0; gi < h->npw_host[k]; ++gi) {
      const int64_t f = geom->flat_idx[(size_t)k * h->npw_max + gi];
      cnt[(size_t)k * L0 + compact0((int)(f / ((int64_t)n1 * n2))) + 1]++;
    }
  for (size_t i = 1; i < cnt.size(); ++i) cnt[i] += cnt[i - 1];
  const int total = cnt.back();
  std::vector<int> pg(std::max(total, 1)), pp(std::max(total, 1));
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  for (int k = 0; k < h->nk; ++k)
    for (int64_t gi = 0; gi < h->npw_host[k]; ++gi) {
      const int64_t f = geom->flat_idx[(size_t)k * h->npw_max + gi];
      const int slot = fill[(size_t)k * L0 + compact0((int)(f / ((int64_t)n1 * n2)))]++;
      pg[slot] = (int)gi;
      pp[slot] = (int)(f % ((int64_t)n1 * n2));
    }
  std::vector<int> npw32(h->npw_host.begin(), h->npw_host.end());
  // twiddles exp(-2 pi i t / n), computed in double on the host
  std::vector<cplx<double>> tw64[3];
  std::vector<cplx<float>> tw32[3];
  for (int a = 0; a < 3; ++a) {
    for (int t = 0; t < g.n[a]; ++t) {
      const double ang = -2.0 * M_PI * (double)t / (double)g.n[a];
      tw64[a].push_back(mk<double>(std::cos(ang), std::sin(ang)));
      tw32[a].push_back(mk<float>((float)std::cos(ang), (float)std::sin(ang)));
    }
  }
  auto fail = [&](cudaError_t e) {
    set_error(std::string("gwb_ham_create: ") + cudaGetErrorString(e));
    gwb_ham_destroy(h);
    return GWB_ERR_CUDA;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(e);
#define GWB_ALLOC_COPY(dst, vec)                                                            \
  do {                                                                                      \
    e = cudaMalloc((void**)&(dst), (vec).size() * sizeof((vec)[0]));                        \
    if (e != cudaSuccess) return fail(e);                                                   \
    e = cudaMemcpy((dst), (vec).data(), (vec).size() * sizeof((vec)[0]), cudaMemcpyHostToDevice); \
    if (e != cudaSuccess) return fail(e);                                                   \
  } while (0)
  GWB_ALLOC_COPY(h->d_plane_ptr, cnt);
  GWB_ALLOC_COPY(h->d_plane_g, pg);
  GWB_ALLOC_COPY(h->d_plane_pos, pp);
  GWB_ALLOC_COPY(h->d_npw, npw32);
  for (int a = 0; a < 3; ++a) {
    GWB_ALLOC_COPY(h->d_tw64[a], tw64[a]);
    GWB_ALLOC_COPY(h->d_tw32[a], tw32[a]);
  }
#undef GWB_ALLOC_COPY
  const size_t nkp = (size_t)h->nk * h->npw_max;
  if ((e = cudaMalloc((void**)&h->d_t64, nkp * 8)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc((void**)&h->d_t32, nkp * 4)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc((void**)&h->d_v64, nbox * 8)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc((void**)&h->d_v32, nbox * 4)) != cudaSuccess) return fail(e);
  if (h->nproj > 0) {
    const size_t np = (size_t)h->nk * h->nproj * h->npw_max;
    if ((e = cudaMalloc((void**)&h->d_p64, np * 16)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc((void**)&h->d_p32, np * 8)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc((void**)&h->d_d64, (size_t)h->nproj * h->nproj * 8)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc((void**)&h->d_d32, (size_t)h->nproj * h->nproj * 4)) != cudaSuccess) return fail(e);
  }
  *out = h;
  return GWB_OK;
}

int gwb_ham_destroy(gwb_ham* h) {
  if (!h) return GWB_OK;
  void* ptrs[] = {h->d_npw, h->d_plane_ptr, h->d_plane_g, h->d_plane_pos, h->d_t64, h->d_t32, h->d_v64,
                  h->d_v32, h->d_p64, h->d_p32, h->d_d64, h->d_d32, h->d_q64, h->d_q32, h->d_W, h->d_part, h->d_bd, h->d_bq,
                  h->d_pplanes, h->d_cplanes, h->d_becp, h->d_bdplanes, h->d_tcwork, h->d_tcstatus, h->d_rhok,
                  h->d_tw64[0], h->d_tw64[1], h->d_tw64[2], h->d_tw32[0], h->d_tw32[1], h->d_tw32[2]};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete h;
  return GWB_OK;
}

static unsigned blocks_for(size_t n, unsigned bs) { return (unsigned)((n + bs - 1) / bs); }

int gwb_ham_set_kinetic(gwb_ham* h, const double* t, void* stream) {
  GWB_REQUIRE(h && t, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)h->nk * h->npw_max;
  GWB_CUDA_TRY(cudaMemcpyAsync(h->d_t64, t, n * 8, cudaMemcpyDeviceToDevice, st));
  k_scale_copy<float><<<blocks_for(n, 256), 256, 0, st>>>(t, h->d_t32, n, 1.0);
  GWB_LAUNCH_CHECK();
  h->have_t = true;
  return GWB_OK;
}

int gwb_ham_set_potential(gwb_ham* h, const double* v, void* stream) {
  GWB_REQUIRE(h && v, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)h->g.n[0] * h->g.n[1] * h->g.n[2];
  const double s = 1.0 / (double)n;
  k_scale_copy<double><<<blocks_for(n, 256), 256, 0, st>>>(v, h->d_v64, n, s);
  k_scale_copy<float><<<blocks_for(n, 256), 256, 0, st>>>(v, h->d_v32, n, s);
  GWB_LAUNCH_CHECK();
  h->have_v = true;
  return GWB_OK;
}

int gwb_ham_set_projectors(gwb_ham* h, const void* p, const double* dij, void* stream) {
  GWB_REQUIRE(h, "null handle");
  if (h->nproj == 0) {
    h->have_p = true;
    return GWB_OK;
  }
  GWB_REQUIRE(p && dij, "null projector pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t np = (size_t)h->nk * h->nproj * h->npw_max;
  const size_t nd = (size_t)h->nproj * h->nproj;
  GWB_CUDA_TRY(cudaMemcpyAsync(h->d_p64, p, np * 16, cudaMemcpyDeviceToDevice, st));
  k_c128_to_c64<<<blocks_for(np, 256), 256, 0, st>>>((const cplx<double>*)p, h->d_p32, np);
  GWB_CUDA_TRY(cudaMemcpyAsync(h->d_d64, dij, nd * 8, cudaMemcpyDeviceToDevice, st));
  h->pplanes_ok = false;  // the tensor-core planes of P are rebuilt on next use
  k_scale_copy<float><<<blocks_for(nd, 256), 256, 0, st>>>(dij, h->d_d32, nd, 1.0);
  GWB_LAUNCH_CHECK();
  h->have_p = true;
  return GWB_OK;
}

int gwb_ham_apply_strided(gwb_ham* h, const void* c, int64_t c_kstride, void* out, int64_t out_kstride,
                          int32_t nb, int32_t io_dtype, int32_t prec, void* stream) {
  GWB_REQUIRE(h && c && out, "null argument");
  GWB_REQUIRE(nb >= 0, "nb < 0");
  GWB_REQUIRE(h->have_t && h->have_v && h->have_p, "kinetic, potential and projectors must be set first");
  GWB_REQUIRE(io_dtype == GWB_C64 || io_dtype == GWB_C128, "io_dtype must be GWB_C64 or GWB_C128");
  GWB_REQUIRE(prec == GWB_FP32 || prec == GWB_FP64, "prec must be GWB_FP32 or GWB_FP64");
  GWB_REQUIRE(c != out, "c and out must not overlap");
  GWB_REQUIRE(c_kstride >= (int64_t)nb * h->npw_max && out_kstride >= (int64_t)nb * h->npw_max,
              "k stride smaller than nb * npw_max");
  if (nb == 0) return GWB_OK;
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    return GWB_ERR_CUDA;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (io_dtype == GWB_C128) {
    auto* ci = (const cplx<double>*)c;
    auto* co = (cplx<double>*)out;
    return prec == GWB_FP64 ? apply_impl<double>(h, ci, c_kstride, co, out_kstride, nb, st)
                            : apply_impl<float>(h, ci, c_kstride, co, out_kstride, nb, st);
  }
  auto* ci = (const cplx<float>*)c;
  auto* co = (cplx<float>*)out;
  return prec == GWB_FP64 ? apply_impl<double>(h, ci, c_kstride, co, out_kstride, nb, st)
                          : apply_impl<float>(h, ci, c_kstride, co, out_kstride, nb, st);
}

int gwb_ham_apply(gwb_ham* h, const void* c, void* out, int32_t nb, int32_t io_dtype, int32_t prec,
                  void* stream) {
  GWB_REQUIRE(h, "null handle");
  const int64_t ks = (int64_t)nb * h->npw_max;
  return gwb_ham_apply_strided(h, c, ks, out, ks, nb, io_dtype, prec, stream);
}

int gwb_ham_set_tuning(gwb_ham* h, int64_t w_budget_bytes, int32_t nl_target_ctas) {
  GWB_REQUIRE(h, "null handle");
  GWB_REQUIRE(w_budget_bytes >= 0 && nl_target_ctas >= 0, "tuning values must be >= 0");
  h->w_budget = (size_t)w_budget_bytes;
  h->nl_target = nl_target_ctas;
  return GWB_OK;
}

int gwb_ham_set_fft_threads(gwb_ham* h, int32_t threads_fp32, int32_t threads_fp64) {
  GWB_REQUIRE(h, "null handle");
  auto ok = [](int32_t n) { return n == 0 || n == 256 || n == 512 || n == 1024; };
  GWB_REQUIRE(ok(threads_fp32) && ok(threads_fp64), "FFT block threads must be 0, 256, 512 or 1024");
  h->fft_nt[0] = threads_fp32;
  h->fft_nt[1] = threads_fp64;
  return GWB_OK;
}

int gwb_ham_set_overlap(gwb_ham* h, const double* q, void* stream) {
  GWB_REQUIRE(h, "null handle");
  GWB_REQUIRE(h->have_p, "projectors must be set before the overlap");
  if (h->nproj == 0) {
    h->have_q = true;
    return GWB_OK;
  }
  GWB_REQUIRE(q, "null overlap pointer");
  GWB_CUDA_TRY(cudaSetDevice(h->device));
  cudaStream_t st = (cudaStream_t)stream;
  const size_t nd = (size_t)h->nproj * h->nproj;
  if (!h->d_q64) {
    GWB_CUDA_TRY(cudaMalloc((void**)&h->d_q64, nd * 8));
    GWB_CUDA_TRY(cudaMalloc((void**)&h->d_q32, nd * 4));
  }
  GWB_CUDA_TRY(cudaMemcpyAsync(h->d_q64, q, nd * 8, cudaMemcpyDeviceToDevice, st));
  k_scale_copy<float><<<blocks_for(nd, 256), 256, 0, st>>>(q, h->d_q32, nd, 1.0);
  GWB_LAUNCH_CHECK();
  h->have_q = true;
  return GWB_OK;
}

int gwb_ham_apply_hs(gwb_ham* h, const void* c, int64_t c_kstride, void* out_h, int64_t oh_kstride, void* out_s,
                     int64_t os_kstride, int32_t nb, int32_t io_dtype, int32_t prec, void* stream) {
  GWB_REQUIRE(h && c && out_h && out_s, "null argument");
  GWB_REQUIRE(nb >= 0, "nb < 0");
  GWB_REQUIRE(h->have_t && h->have_v && h->have_p, "kinetic, potential and projectors must be set first");
  GWB_REQUIRE(h->have_q, "the overlap (gwb_ham_set_overlap) must be set first");
  GWB_REQUIRE(io_dtype == GWB_C64 || io_dtype == GWB_C128, "io_dtype must be GWB_C64 or GWB_C128");
  GWB_REQUIRE(prec == GWB_FP32 || prec == GWB_FP64, "prec must be GWB_FP32 or GWB_FP64");
  GWB_REQUIRE(c != out_h && c != out_s && out_h != out_s, "c, out_h and out_s must not overlap");
  const int64_t row = (int64_t)nb * h->npw_max;
  GWB_REQUIRE(c_kstride >= row && oh_kstride >= row && os_kstride >= row, "k stride smaller than nb * npw_max");
  if (nb == 0) return GWB_OK;
  GWB_CUDA_TRY(cudaSetDevice(h->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (io_dtype == GWB_C128) {
    auto* ci = (const cplx<double>*)c;
    auto* oh = (cplx<double>*)out_h;
    auto* os = (cplx<double>*)out_s;
    return prec == GWB_FP64 ? apply_hs_impl<double>(h, ci, c_kstride, oh, oh_kstride, os, os_kstride, nb, st)
                            : apply_hs_impl<float>(h, ci, c_kstride, oh, oh_kstride, os, os_kstride, nb, st);
  }
  auto* ci = (const cplx<float>*)c;
  auto* oh = (cplx<float>*)out_h;
  auto* os = (cplx<float>*)out_s;
  return prec == GWB_FP64 ? apply_hs_impl<double>(h, ci, c_kstride, oh, oh_kstride, os, os_kstride, nb, st)
                          : apply_hs_impl<float>(h, ci, c_kstride, oh, oh_kstride, os, os_kstride, nb, st);
}

int gwb_ham_density(gwb_ham* h, const void* c, int64_t c_kstride, int32_t nb, int32_t io_dtype,
                    const double* weights, int64_t w_kstride, double scale, double* rho, void* stream) {
  GWB_REQUIRE(h && c && weights && rho, "null argument");
  GWB_REQUIRE(nb > 0, "nb must be positive");
  GWB_REQUIRE(io_dtype == GWB_C64 || io_dtype == GWB_C128, "io_dtype must be GWB_C64 or GWB_C128");
  GWB_REQUIRE(c_kstride >= (int64_t)nb * h->npw_max, "k stride smaller than nb * npw_max");
  GWB_REQUIRE(w_kstride >= nb, "weight k stride smaller than nb");
  GWB_CUDA_TRY(cudaSetDevice(h->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (io_dtype == GWB_C128)
    return density_impl(h, (const cplx<double>*)c, c_kstride, nb, weights, w_kstride, scale, rho, st);
  return density_impl(h, (const cplx<float>*)c, c_kstride, nb, weights, w_kstride, scale, rho, st);
}

size_t gwb_ham_scratch_bytes(const gwb_ham* h) {
  return h ? h->W_bytes + h->part_bytes + h->bd_bytes + h->bq_bytes + h->pplanes_bytes + h->cplanes_bytes + h->becp_bytes +
                 h->bdplanes_bytes + h->tcwork_bytes + h->rhok_bytes
           : 0;
}

int gwb_ham_tc_status(gwb_ham* h, int* status) {
  GWB_REQUIRE(h && status, "null argument");
  *status = 0;
  if (!h->d_tcstatus) return GWB_OK;
  GWB_CUDA_TRY(cudaSetDevice(h->device));
  GWB_CUDA_TRY(cudaMemcpy(status, h->d_tcstatus, sizeof(int), cudaMemcpyDeviceToHost));
  if (*status) {
    GWB_CUDA_TRY(cudaMemset(h->d_tcstatus, 0, sizeof(int)));
    set_error("tensor-core nonlocal term: a bounded pipeline wait ran out");
    return GWB_ERR_TIMEOUT;
  }
  return GWB_OK;
}

}  // extern "C"
