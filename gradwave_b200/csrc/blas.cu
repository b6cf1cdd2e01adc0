// Batched complex GEMM with row-major semantics over cuBLAS (the plain
// library GEMMs of the Davidson subspace steps).
//
// C[b] = alpha * op(A[b]) * op(B[b]) + beta * C[b], op in {N, T, H}, every
// matrix row-major with a leading dimension and a batch stride. A row-major
// matrix is the column-major storage of its transpose, so the call becomes
// C^T = op(B)^T op(A)^T in cuBLAS terms with the operands swapped.
#include <cublas_v2.h>

#include <mutex>
#include <string>
#include <unordered_map>

#include "common.cuh"

namespace gwb {

static std::mutex g_blas_mu;
static std::unordered_map<int, cublasHandle_t> g_blas;

static int blas_handle(cublasHandle_t* out) {
  int dev = 0;
  GWB_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_blas_mu);
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
