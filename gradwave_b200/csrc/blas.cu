// Batched complex GEMM with row-major semantics over cuBLAS (the plain
// library GEMMs of the Davidson subspace steps).
//
// C[b] = alpha * op(A[b]) * op(B[b]) + beta * C[b], op in {N, T, H}, every
// matrix row-major with a leading dimension and a batch stride. A row-major
// matrix is the column-major storage of its transpose, so the call becomes
// C^T = op(B)^T op(A)^T in cuBLAS terms with the operands swapped.
#include <cublas_v2.h>

#include <algorithm>
#include <string>
#include <unordered_map>

#include "common.cuh"

namespace gwb {

// One cuBLAS handle per (host thread, device): a handle's stream is set before
// every call, so threads that drive solves on different streams at the same
// time must not share one.
static thread_local std::unordered_map<int, cublasHandle_t> g_blas;

int blas_handle(cublasHandle_t* out) {
  int dev = 0;
  GWB_CUDA_TRY(cudaGetDevice(&dev));
  auto it = g_blas.find(dev);
  if (it == g_blas.end()) {
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) {
      set_error("cublasCreate failed");
      return GWB_ERR_CUDA;
    }
    it = g_blas.emplace(dev, h).first;
  }
  *out = it->second;
  return GWB_OK;
}

static cublasOperation_t to_op(int op) {
  return op == 0 ? CUBLAS_OP_N : (op == 1 ? CUBLAS_OP_T : CUBLAS_OP_C);
}

}  // namespace gwb

using namespace gwb;

extern "C" int gwb_zgemm(int opA, int opB, int64_t M, int64_t N, int64_t K, double alpha_re, double alpha_im,
                         const void* A, int64_t lda, int64_t strideA, const void* B, int64_t ldb,
                         int64_t strideB, double beta_re, double beta_im, void* C, int64_t ldc,
                         int64_t strideC, int64_t batch, void* stream) {
  GWB_REQUIRE(opA >= 0 && opA <= 2 && opB >= 0 && opB <= 2, "op must be 0 (N), 1 (T) or 2 (H)");
  GWB_REQUIRE(M >= 0 && N >= 0 && K >= 0 && batch >= 0, "negative size");
  if (M == 0 || N == 0 || batch == 0) return GWB_OK;
  GWB_REQUIRE(A && B && C, "null matrix");
  cublasHandle_t h;
  int rc = blas_handle(&h);
  if (rc) return rc;
  if (cublasSetStream(h, (cudaStream_t)stream) != CUBLAS_STATUS_SUCCESS) {
    set_error("cublasSetStream failed");
    return GWB_ERR_CUDA;
  }
  const cuDoubleComplex alpha = make_cuDoubleComplex(alpha_re, alpha_im);
  const cuDoubleComplex beta = make_cuDoubleComplex(beta_re, beta_im);
  // row-major C (M x N) == column-major C^T (N x M) = op(B)^T op(A)^T
  cublasStatus_t s = cublasZgemmStridedBatched(
      h, to_op(opB), to_op(opA), (int)N, (int)M, (int)K, &alpha, (const cuDoubleComplex*)B, (int)ldb, strideB,
      (const cuDoubleComplex*)A, (int)lda, strideA, &beta, (cuDoubleComplex*)C, (int)ldc, strideC, (int)batch);
  if (s != CUBLAS_STATUS_SUCCESS) {
    set_error("cublasZgemmStridedBatched failed with status " + std::to_string((int)s));
    return GWB_ERR_CUDA;
  }
  return GWB_OK;
}

// ---------------------------------------------------------------------------
// Inner-product GEMM with a long reduction: C = alpha A B^H + beta C with
// A (M x K), B (N x K) row-major and M, N small (the subspace, projection and
// Gram products of the Davidson step: M, N <= a few hundred, K = npw). cuBLAS
// tiles such shapes into a few dozen CTAs; here K is split into slices so the
// grid fills the GPU, each CTA accumulates a TM x TN output tile of one slice
// (2 x 2 outputs per thread, float64; TM, TN in {8, 16, 24, 32} chosen from M
// and N so narrow blocks are not padded to 32), staging 16-column K steps of A
// and B through double-buffered shared memory with cp.async (the next step
// loads while this one multiplies), and a second kernel sums the slices in a
// fixed order (deterministic).
namespace gwb {

constexpr int NH_K = 16;

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc, bool valid) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
  const int n = valid ? 16 : 0;  // 0: zero-fill, nothing read
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(gsrc), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <int TM, int TN>
__global__ void __launch_bounds__(TM * TN / 4) k_zgemm_nh_part(int M, int N, int K, int kslice,
                                                             const cplx<double>* __restrict__ A, int64_t lda,
                                                             int64_t sA, const cplx<double>* __restrict__ B,
                                                             int64_t ldb, int64_t sB, cplx<double>* __restrict__ part,
                                                             int batch) {
  constexpr int NT = TM * TN / 4;  // threads: (TM/2) x (TN/2)
  constexpr int HM = TM / 2, HN = TN / 2;
  __shared__ __align__(16) cplx<double> sa[2][TM][NH_K + 1];
  __shared__ __align__(16) cplx<double> sb[2][TN][NH_K + 1];
  const int tilesN = (N + TN - 1) / TN;
  const int ti = blockIdx.x / tilesN, tj = blockIdx.x % tilesN;
  const int s = blockIdx.y, b = blockIdx.z;
  const int tx = threadIdx.x % HN, ty = threadIdx.x / HN;
  const cplx<double>* Ab = A + b * sA;
  const cplx<double>* Bb = B + b * sB;
  const int g0 = s * kslice, g1 = min(K, g0 + kslice);
  const int nsteps = (g1 - g0 + NH_K - 1) / NH_K;

  auto load = [&](int step, int buf) {
    const int gb = g0 + step * NH_K;
    for (int idx = threadIdx.x; idx < (TM + TN) * NH_K; idx += NT) {
      const int r = idx / NH_K, kk = idx % NH_K, g = gb + kk;
      if (r < TM) {
        const int ia = ti * TM + r;
        const bool ok = ia < M && g < g1;
        cp_async16(&sa[buf][r][kk], ok ? (const void*)(Ab + (int64_t)ia * lda + g) : (const void*)Ab, ok);
      } else {
        const int jb = tj * TN + (r - TM);
        const bool ok = jb < N && g < g1;
        cp_async16(&sb[buf][r - TM][kk], ok ? (const void*)(Bb + (int64_t)jb * ldb + g) : (const void*)Bb, ok);
      }
    }
    cp_async_commit();
  };

  cplx<double> acc[2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int c = 0; c < 2; ++c) acc[a][c] = mk<double>(0.0, 0.0);
  if (nsteps > 0) load(0, 0);
  for (int st = 0; st < nsteps; ++st) {
    const int buf = st & 1;
    if (st + 1 < nsteps) {
      load(st + 1, buf ^ 1);
      cp_async_wait<1>();  // this step's group has landed; the next may still fly
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < NH_K; ++kk) {
      const cplx<double> a0 = sa[buf][ty][kk], a1 = sa[buf][ty + HM][kk];
      const cplx<double> b0 = sb[buf][tx][kk], b1 = sb[buf][tx + HN][kk];
      acc[0][0] = acc[0][0] + mul_conj(a0, b0);
      acc[0][1] = acc[0][1] + mul_conj(a0, b1);
      acc[1][0] = acc[1][0] + mul_conj(a1, b0);
      acc[1][1] = acc[1][1] + mul_conj(a1, b1);
    }
    __syncthreads();  // buf is refilled by the load two steps on
  }
  cplx<double>* P = part + ((int64_t)s * batch + b) * M * N;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int i = ti * TM + ty + HM * a, j = tj * TN + tx + HN * c;
      if (i < M && j < N) P[(int64_t)i * N + j] = acc[a][c];
    }
}

__global__ void k_zgemm_nh_reduce(int M, int N, int nslice, int batch, const cplx<double>* __restrict__ part,
                                  cplx<double> alpha, cplx<double> beta, cplx<double>* __restrict__ C, int64_t ldc,
                                  int64_t sC) {
  const int64_t total = (int64_t)batch * M * N;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(idx / ((int64_t)M * N));
    const int64_t r = idx % ((int64_t)M * N);
    const int i = (int)(r / N), j = (int)(r % N);
    cplx<double> a = mk<double>(0.0, 0.0);
    for (int s = 0; s < nslice; ++s) a = a + part[(int64_t)s * total + idx];
    cplx<double>* c = C + b * sC + (int64_t)i * ldc + j;
    cplx<double> v = alpha * a;
    if (beta.x != 0.0 || beta.y != 0.0) v = v + beta * (*c);
    *c = v;
  }
}

}  // namespace gwb

extern "C" int gwb_zgemm_nh(int64_t M, int64_t N, int64_t K, double alpha_re, double alpha_im, const void* A,
                            int64_t lda, int64_t strideA, const void* B, int64_t ldb, int64_t strideB,
                            double beta_re, double beta_im, void* C, int64_t ldc, int64_t strideC, int64_t batch,
                            void* work, size_t work_bytes, void* stream) {
  GWB_REQUIRE(M >= 0 && N >= 0 && K >= 0 && batch >= 0, "negative size");
  if (M == 0 || N == 0 || batch == 0) return GWB_OK;
  GWB_REQUIRE(A && B && C && work, "null pointer");
  GWB_REQUIRE(M * N * batch * 16 <= (int64_t)work_bytes, "work smaller than one M*N*batch slice");
  // tile edges: multiples of 8 up to 32 covering M and N
  const int TM = (int)std::min<int64_t>(32, (M + 7) / 8 * 8), TN = (int)std::min<int64_t>(32, (N + 7) / 8 * 8);
  const int tiles = (int)(((M + TM - 1) / TM) * ((N + TN - 1) / TN));
  const int64_t slice_bytes = M * N * batch * 16;
  const int threads = TM * TN / 4;
  // enough CTAs for ~4 x 148 x (256 / threads) tiles in flight
  const int64_t target = 4 * 148 * (256 / threads);
  int64_t want = (target + (int64_t)tiles * batch - 1) / ((int64_t)tiles * batch);
  want = std::min<int64_t>(want, std::max<int64_t>(1, K / 128));
  want = std::min<int64_t>(want, (int64_t)work_bytes / slice_bytes);
  const int nslice = (int)std::max<int64_t>(1, want);
  const int kslice = (int)(((K + nslice - 1) / nslice + NH_K - 1) / NH_K * NH_K);
  const int ns = (int)((K + kslice - 1) / kslice);
  dim3 g1(tiles, ns, (unsigned)batch);
  cudaStream_t st = (cudaStream_t)stream;
  const cplx<double>* Ap = (const cplx<double>*)A;
  const cplx<double>* Bp = (const cplx<double>*)B;
  cplx<double>* Wp = (cplx<double>*)work;
#define GWB_NH_CASE(tm, tn)                                                                                      \
  if (TM == tm && TN == tn)                                                                                      \
    k_zgemm_nh_part<tm, tn><<<g1, tm * tn / 4, 0, st>>>((int)M, (int)N, (int)K, kslice, Ap, lda, strideA, Bp, ldb, \
                                                        strideB, Wp, (int)batch);
#define GWB_NH_ROW(tm) GWB_NH_CASE(tm, 8) GWB_NH_CASE(tm, 16) GWB_NH_CASE(tm, 24) GWB_NH_CASE(tm, 32)
  GWB_NH_ROW(8) GWB_NH_ROW(16) GWB_NH_ROW(24) GWB_NH_ROW(32)
#undef GWB_NH_ROW
#undef GWB_NH_CASE
  const int64_t total = M * N * batch;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 4096);
  k_zgemm_nh_reduce<<<blocks, 256, 0, st>>>((int)M, (int)N, ns, (int)batch,
                                            (const cplx<double>*)work, mk<double>(alpha_re, alpha_im),
                                                              mk<double>(beta_re, beta_im), (cplx<double>*)C, ldc,
                                                              strideC);
  GWB_LAUNCH_CHECK();
  count_launches(2);
  return GWB_OK;
}
