// Native block-Davidson driver: the whole band solve in one library call.
//
// Same algorithm, step order and modes as the Python driver
// (gradwave_b200/davidson.py) and the reference it mirrors (gradwave
// solvers/davidson.py:528-774): float64 subspace, incremental s = V^H H V,
// TPA (or learned) preconditioning of the worst n_add residuals, projection,
// device rank repair, CholQR2, restart at max_dim with the images transformed
// by the same triangle; mode 1 adds the float32-expansion / float64
// certification schedule of davidson.py:581-687. Everything runs on `stream`;
// the host reads four doubles per round (max |r|, n_add, eigensolver and
// orthonormalisation flags) - the reference's own two host reads.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>
#include <cmath>
#include <cstring>
#include <string>

#include "common.cuh"

extern "C" {
int gwb_zgemm(int opA, int opB, int64_t M, int64_t N, int64_t K, double alpha_re, double alpha_im,
              const void* A, int64_t lda, int64_t strideA, const void* B, int64_t ldb, int64_t strideB,
              double beta_re, double beta_im, void* C, int64_t ldc, int64_t strideC, int64_t batch, void* stream);
int gwb_zgemm_nh(int64_t M, int64_t N, int64_t K, double alpha_re, double alpha_im, const void* A, int64_t lda,
                 int64_t strideA, const void* B, int64_t ldb, int64_t strideB, double beta_re, double beta_im,
                 void* C, int64_t ldc, int64_t strideC, int64_t batch, void* work, size_t work_bytes, void* stream);
}

namespace gwb {

// Gs[k][i][j] = (conj(G[k][i][j]) + G[k][j][i]) / 2  (G = X HX^H -> s = X^* HX^T)
__global__ void k_hermitize_conj(const cplx<double>* __restrict__ G, cplx<double>* __restrict__ Gs, int n) {
  const int k = blockIdx.y;
  const cplx<double>* g = G + (int64_t)k * n * n;
  cplx<double>* o = Gs + (int64_t)k * n * n;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
    const int i = idx / n, j = idx % n;
    cplx<double> v = scale(conj(g[idx]) + g[(int64_t)j * n + i], 0.5);
    if (i == j) v.y = 0.0;
    o[idx] = v;
  }
}

// dst rows (k stride dk) = src rows (k stride sk) * mask
__global__ void k_masked_copy(const cplx<double>* __restrict__ src, int64_t sk, cplx<double>* __restrict__ dst,
                              int64_t dk, const unsigned char* __restrict__ mask, int rows, int npw) {
  const int k = blockIdx.y;
  const int64_t n = (int64_t)rows * npw;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int g = (int)(i % npw);
    dst[k * dk + i] = mask[(int64_t)k * npw + g] ? src[k * sk + i] : mk<double>(0.0, 0.0);
  }
}

// *flag |= 4 when any of the n complex values is not finite
__global__ void k_nonfinite(const cplx<double>* __restrict__ z, int64_t n, int* __restrict__ flag) {
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    bad |= !(isfinite(z[i].x) && isfinite(z[i].y));
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 4);
}

__global__ void k_fill(double* __restrict__ p, int n, double v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// stats[2] = max info (eigensolver), stats[3] = flags; flags reset.
__global__ void k_pack_flags(const int* __restrict__ heev_info, int nk, int* __restrict__ flags,
                             double* __restrict__ stats) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int mx = 0;
    for (int k = 0; k < nk; ++k) mx = max(mx, heev_info[k]);
    stats[2] = (double)mx;
    stats[3] = (double)flags[0];
    flags[0] = 0;
  }
}

}  // namespace gwb

extern "C" {
int gwb_residual(int32_t, int32_t, int32_t, const void*, int64_t, const void*, int64_t, const double*, int64_t,
                 void*, int64_t, double*, void*);
int gwb_conv_stats(int32_t, int32_t, const double*, double, double*, void*);
int gwb_select_worst(int32_t, int32_t, const double*, int32_t, int32_t*, void*);
int gwb_precond_teter(int32_t, int32_t, int32_t, int32_t, const void*, int64_t, const void*, int64_t,
                      const double*, const int32_t*, void*, int64_t, void*);
int gwb_subspace_insert(int32_t, int32_t, int32_t, const void*, void*, int32_t, int64_t, void*);
int gwb_chol_inv(int32_t, int32_t, void*, int32_t, int64_t, void*, int64_t, int32_t*, int32_t*, void*);
int gwb_row_repair(int32_t, int32_t, int32_t, void*, int64_t, const uint8_t*, double, int32_t*, void*);
int gwb_heev_lowest(int32_t, int32_t, int32_t, const void*, int32_t, int64_t, double*, void*, double*, int32_t*,
                    void*);
int gwb_heev_max_dim(void);
int64_t gwb_heev_scratch_doubles(int32_t);
int gwb_ham_apply_strided(gwb_ham*, const void*, int64_t, void*, int64_t, int32_t, int32_t, int32_t, void*);
int64_t gwb_precond_learned_work_bytes(int32_t, int32_t, int32_t);
int gwb_precond_learned(const float*, int32_t, int32_t, int32_t, int32_t, const void*, int64_t, const void*, int64_t,
                        const double*, const double*, const int32_t*, const uint8_t*, void*, int64_t, void*, size_t,
                        void*);
int gwb_stall_update(const double*, double*, uint8_t*, uint8_t*, int32_t, double, int32_t, void*);
}

namespace gwb {

struct Buf {
  size_t off = 0;
  template <typename T> T* take(unsigned char* base, size_t count) {
    off = (off + 255) / 256 * 256;
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
    return p;
  }
};

typedef cplx<double> Z16;

constexpr size_t NH_WORK_BYTES = (size_t)24 << 20;  // split-K partials of the A B^H products

struct Work {
  unsigned char* nh_work;
  Z16 *V, *HV, *S, *X, *HX, *R, *D, *D2, *C, *G, *Linv, *Gs, *U;
  double *Zs, *rn, *eig, *eig2, *stats, *rn_prev;
  int *sel, *info, *heev_info, *flags, *sync_flag;
  unsigned char *tpa_only, *stall_count;
  unsigned char* pl_work;
  size_t pl_work_bytes;
};

static size_t layout(const gwb_davidson_params& p, unsigned char* base, Work* w) {
  const size_t nk = p.nk, nb = p.nb, npw = p.npw, md = p.max_dim;
  const size_t hm = std::min<size_t>(md, (size_t)gwb_heev_max_dim());
  Buf b;
  Work t{};
  t.V = b.take<Z16>(base, nk * md * npw);
  t.HV = b.take<Z16>(base, nk * md * npw);
  t.S = b.take<Z16>(base, nk * md * md);
  t.X = b.take<Z16>(base, nk * nb * npw);
  t.HX = b.take<Z16>(base, nk * nb * npw);
  t.R = b.take<Z16>(base, nk * nb * npw);
  t.D = b.take<Z16>(base, nk * nb * npw);
  t.D2 = b.take<Z16>(base, nk * nb * npw);
  t.C = b.take<Z16>(base, nk * md * md);
  t.G = b.take<Z16>(base, nk * nb * nb);
  t.Linv = b.take<Z16>(base, nk * nb * nb);
  t.Gs = b.take<Z16>(base, nk * nb * nb);
  t.U = b.take<Z16>(base, nk * std::max(hm, nb) * nb);
  t.Zs = b.take<double>(base, nk * (size_t)gwb_heev_scratch_doubles((int32_t)hm));
  t.rn = b.take<double>(base, nk * nb);
  t.eig = b.take<double>(base, nk * nb);
  t.eig2 = b.take<double>(base, nk * nb);
  t.stats = b.take<double>(base, 4);
  t.sel = b.take<int>(base, nk * nb);
  t.info = b.take<int>(base, nk);
  t.heev_info = b.take<int>(base, nk);
  t.flags = b.take<int>(base, 1);
  t.sync_flag = b.take<int>(base, 1);
  t.nh_work = b.take<unsigned char>(base, NH_WORK_BYTES);
  t.rn_prev = b.take<double>(base, nk * nb);
  t.tpa_only = b.take<unsigned char>(base, nk * nb);
  t.stall_count = b.take<unsigned char>(base, nk * nb);
  t.pl_work_bytes = (size_t)gwb_precond_learned_work_bytes((int32_t)nk, (int32_t)nb, (int32_t)npw);
  t.pl_work = b.take<unsigned char>(base, t.pl_work_bytes);
  if (w) *w = t;
  return b.off + 256;
}

#define GWB_TRY(expr)            \
  do {                           \
    int _rc = (expr);            \
    if (_rc != GWB_OK) return _rc; \
  } while (0)

class Solver {
 public:
  Solver(gwb_ham* h, const gwb_davidson_params& p, const void* model, const double* t, const unsigned char* mask,
         const Work& w, cudaStream_t st)
      : h_(h), p_(p), model_(model), t_(t), mask_(mask), w_(w), st_(st) {
    nk_ = p.nk;
    nb_ = p.nb;
    npw_ = p.npw;
    md_ = p.max_dim;
  }

  int run(const void* x0, double* eig_out, void* vec_out, double* rn_out, gwb_davidson_stats* out) {
    const int64_t nbp = (int64_t)nb_ * npw_, mdp = (int64_t)md_ * npw_;
    fp32_exp_ = p_.mode == 1 || p_.mode == 2;
    if (p_.precond == 1) {
      k_fill<<<(nk_ * nb_ + 255) / 256, 256, 0, st_>>>(w_.rn_prev, nk_ * nb_, INFINITY);
      GWB_LAUNCH_CHECK();
      GWB_CUDA_TRY(cudaMemsetAsync(w_.tpa_only, 0, (size_t)nk_ * nb_, st_));
      GWB_CUDA_TRY(cudaMemsetAsync(w_.stall_count, 0, (size_t)nk_ * nb_, st_));
    }
    // a non-finite start block is refused before any kernel uses it
    {
      int host_flag = 0;
      GWB_CUDA_TRY(cudaMemsetAsync(w_.sync_flag, 0, sizeof(int), st_));
      k_nonfinite<<<148, 256, 0, st_>>>(static_cast<const Z16*>(x0), (int64_t)nk_ * nbp, w_.sync_flag);
      GWB_LAUNCH_CHECK();
      count_launches(1);
      GWB_CUDA_TRY(cudaMemcpyAsync(&host_flag, w_.sync_flag, sizeof(int), cudaMemcpyDeviceToHost, st_));
      GWB_CUDA_TRY(cudaStreamSynchronize(st_));
      if (host_flag & 4) {
        set_error("the start block holds a non-finite value");
        return GWB_ERR_NONFINITE;
      }
    }
    // initial block: masked copy, orthonormalised with host-checked CholQR2
    GWB_TRY(masked_copy(static_cast<const Z16*>(x0), nbp, w_.D, nbp, nb_));
    int ok = 0;
    GWB_TRY(cholqr2(w_.D, nbp, nb_, w_.D2, nullptr, nullptr, /*sync=*/true, &ok));
    if (!ok) {
      set_error("initial block is rank deficient (Cholesky breakdown)");
      return GWB_ERR_BREAKDOWN;
    }
    GWB_TRY(copy_rows(w_.V, mdp, w_.D, nbp, nb_));
    GWB_TRY(apply(w_.V, mdp, w_.HV, mdp, nb_, fp32_exp_));
    int m = nb_, m0 = 0, m_prev = nb_;
    const double eps32 = 1.1920928955078125e-07;
    const double cert_floor = fp32_exp_ ? 32.0 * eps32 * std::max(p_.t_max, 1.0) : 0.0;
    double prev = INFINITY;
    double rnmax = INFINITY;
    int n_add = 0, it = 0;
    const double* eig = w_.eig;
    while (it < p_.max_iter) {
      ++it;
      GWB_TRY(rayleigh_ritz(m, m0));
      m0 = m;
      bool breakdown = false;
      GWB_TRY(read_stats(&rnmax, &n_add, &breakdown));
      if (breakdown) {
        // the expansion is redone from the same basis with different inputs:
        // TPA in place of the network and a rank repair that replaces every
        // row keeping less than 1e-4 (then 1e-1) of its norm after the first
        // projection, since the rows that broke CholQR2 were nearly in the span
        ++n_rollback_;
        m = m0 = m_prev;
        --it;
        force_tpa_ = true;
        repair_thresh_ = repair_thresh_ < 1e-4 ? 1e-4 : 1e-1;
        if (n_rollback_ > 8) {
          set_error("repeated CholQR2 breakdown in the expansion block");
          return GWB_ERR_BREAKDOWN;
        }
        continue;
      }
      force_tpa_ = false;
      repair_thresh_ = 1e-8;
      if (fp32_exp_) {
        // mode 1 (the reference's rule) treats any round that shrinks the
        // residual by < 30 % as a float32 stall; mode 2 only once the residual
        // is within 100x of the float32 floor (early rounds often stagnate)
        const bool gated = p_.mode == 1 || rnmax < 100.0 * cert_floor;
        const bool stalled = it > 1 && rnmax > 0.7 * prev && gated;
        prev = rnmax;
        if (rnmax < std::max(p_.tol, cert_floor) || stalled) {
          GWB_TRY(certify());
          GWB_TRY(read_stats(&rnmax, &n_add, &breakdown));
          eig = w_.eig2;
          if (rnmax >= p_.tol) {
            GWB_TRY(copy_rows(w_.V, mdp, w_.X, nbp, nb_));
            GWB_TRY(copy_rows(w_.HV, mdp, w_.HX, nbp, nb_));
            m = nb_;
            m0 = 0;
            fp32_exp_ = false;
          }
        } else {
          eig = w_.eig;
        }
      } else {
        eig = last_eig_;
      }
      if (rnmax < p_.tol) return finish(it, eig, eig_out, vec_out, rn_out, out, rnmax);
      GWB_TRY(gwb_select_worst(nk_, nb_, w_.rn, n_add, w_.sel, st_));
      GWB_TRY(precondition(n_add, eig));
      if (m + n_add > md_) {
        ++n_restart_;
        GWB_TRY(cholqr2(w_.X, nbp, nb_, w_.D2, w_.HX, w_.R, /*sync=*/true, &ok));
        if (!ok) {
          set_error("Ritz block lost rank at restart");
          return GWB_ERR_BREAKDOWN;
        }
        GWB_TRY(copy_rows(w_.V, mdp, w_.X, nbp, nb_));
        GWB_TRY(copy_rows(w_.HV, mdp, w_.HX, nbp, nb_));
        m = nb_;
        m0 = 0;
      }
      GWB_TRY(orthonormalize_new(n_add, m));
      GWB_TRY(copy_rows(w_.V + (int64_t)m * npw_, mdp, w_.D, nbp, n_add));
      GWB_TRY(apply(w_.V + (int64_t)m * npw_, mdp, w_.HV + (int64_t)m * npw_, mdp, n_add, fp32_exp_));
      m_prev = m;
      m += n_add;
    }
    if (fp32_exp_) {
      GWB_TRY(certify());
      bool bd = false;
      GWB_TRY(read_stats(&rnmax, &n_add, &bd));
      eig = w_.eig2;
    }
    return finish(p_.max_iter, eig, eig_out, vec_out, rn_out, out, rnmax);
  }

 private:
  int finish(int it, const double* eig, double* eig_out, void* vec_out, double* rn_out, gwb_davidson_stats* out,
             double rnmax) {
    const int64_t nbp = (int64_t)nb_ * npw_;
    GWB_CUDA_TRY(cudaMemcpyAsync(eig_out, eig, sizeof(double) * nk_ * nb_, cudaMemcpyDeviceToDevice, st_));
    GWB_CUDA_TRY(cudaMemcpyAsync(rn_out, w_.rn, sizeof(double) * nk_ * nb_, cudaMemcpyDeviceToDevice, st_));
    GWB_CUDA_TRY(cudaMemcpyAsync(vec_out, w_.X, sizeof(Z16) * nk_ * nbp, cudaMemcpyDeviceToDevice, st_));
    if (out) {
      if (p_.flags & 1) {
        GWB_CUDA_TRY(cudaStreamSynchronize(st_));
        out->apply_ms = apply_ms();
      } else {
        out->apply_ms = 0.0;
      }
      out->n_apply_calls = n_apply_calls_;
      out->n_tpa_fallback = 0;
      if (p_.precond == 1) {
        std::vector<unsigned char> fb((size_t)nk_ * nb_);
        GWB_CUDA_TRY(cudaMemcpyAsync(fb.data(), w_.tpa_only, fb.size(), cudaMemcpyDeviceToHost, st_));
        GWB_CUDA_TRY(cudaStreamSynchronize(st_));
        for (unsigned char f : fb) out->n_tpa_fallback += f ? 1 : 0;
      }
      out->n_iter = it;
      out->hit_max_iter = it >= p_.max_iter ? 1 : 0;
      out->n_restart = n_restart_;
      out->n_cert = n_cert_;
      out->n_repair = n_repair_;
      out->n_rollback = n_rollback_;
      out->n_apply_low = n_low_;
      out->n_apply_full = n_full_;
      out->max_residual = rnmax;
    }
    return GWB_OK;
  }

  int masked_copy(const Z16* src, int64_t sk, Z16* dst, int64_t dk, int rows) {
    dim3 g((unsigned)std::min<int64_t>(((int64_t)rows * npw_ + 255) / 256, 1024), nk_);
    k_masked_copy<<<g, 256, 0, st_>>>(src, sk, dst, dk, mask_, rows, npw_);
    GWB_LAUNCH_CHECK();
    count_launches(1);
    return GWB_OK;
  }

  int copy_rows(Z16* dst, int64_t dk, const Z16* src, int64_t sk, int rows) {
    GWB_CUDA_TRY(cudaMemcpy2DAsync(dst, dk * sizeof(Z16), src, sk * sizeof(Z16), (size_t)rows * npw_ * sizeof(Z16),
                                   nk_, cudaMemcpyDeviceToDevice, st_));
    return GWB_OK;
  }

  int apply(const Z16* src, int64_t sk, Z16* dst, int64_t dk, int rows, bool low) {
    if (low) n_low_ += (int64_t)nk_ * rows;
    else n_full_ += (int64_t)nk_ * rows;
    ++n_apply_calls_;
    const bool timed = (p_.flags & 1) && n_events_ + 2 <= kMaxEvents;
    if (timed) {
      GWB_CUDA_TRY(cudaEventCreate(&ev_[n_events_]));
      GWB_CUDA_TRY(cudaEventRecord(ev_[n_events_], st_));
    }
    const int rc = gwb_ham_apply_strided(h_, src, sk, dst, dk, rows, GWB_C128, low ? GWB_FP32 : GWB_FP64, st_);
    if (timed) {
      GWB_CUDA_TRY(cudaEventCreate(&ev_[n_events_ + 1]));
      GWB_CUDA_TRY(cudaEventRecord(ev_[n_events_ + 1], st_));
      n_events_ += 2;
    }
    return rc;
  }

 public:
  ~Solver() {
    for (int i = 0; i < n_events_; ++i) cudaEventDestroy(ev_[i]);
  }

 private:
  // sum of the timed apply intervals (the stream is drained by then)
  double apply_ms() {
    double tot = 0.0;
    for (int i = 0; i + 1 < n_events_; i += 2) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev_[i], ev_[i + 1]) == cudaSuccess) tot += ms;
    }
    return tot;
  }

  // A B^H products (long reduction over plane waves) go to the split-K kernel,
  // the rest (long output rows) to cuBLAS.
  int zgemm(int oa, int ob, int64_t M, int64_t N, int64_t K, const void* A, int64_t lda, int64_t sA, const void* B,
            int64_t ldb, int64_t sB, void* C, int64_t ldc, int64_t sC, double alpha = 1.0, double beta = 0.0) {
    if (oa == 0 && ob == 2 && M * N * nk_ * 16 <= (int64_t)NH_WORK_BYTES)
      return gwb_zgemm_nh(M, N, K, alpha, 0.0, A, lda, sA, B, ldb, sB, beta, 0.0, C, ldc, sC, nk_, w_.nh_work,
                          NH_WORK_BYTES, st_);
    return gwb_zgemm(oa, ob, M, N, K, alpha, 0.0, A, lda, sA, B, ldb, sB, beta, 0.0, C, ldc, sC, nk_, st_);
  }

  int rayleigh_ritz(int m, int m0) {
    const int64_t mdp = (int64_t)md_ * npw_, nbp = (int64_t)nb_ * npw_;
    const int nnew = m - m0;
    if (nnew > 0) {
      GWB_TRY(zgemm(0, 2, m, nnew, npw_, w_.V, npw_, mdp, w_.HV + (int64_t)m0 * npw_, npw_, mdp, w_.C, nnew,
                    (int64_t)m * nnew));
      GWB_TRY(gwb_subspace_insert(nk_, m, m0, w_.C, w_.S, md_, (int64_t)md_ * md_, st_));
    }
    GWB_TRY(gwb_heev_lowest(nk_, m, nb_, w_.S, md_, (int64_t)md_ * md_, w_.eig, w_.U, w_.Zs, w_.heev_info, st_));
    last_eig_ = w_.eig;
    GWB_TRY(zgemm(1, 0, nb_, npw_, m, w_.U, nb_, (int64_t)m * nb_, w_.V, npw_, mdp, w_.X, npw_, nbp));
    GWB_TRY(zgemm(1, 0, nb_, npw_, m, w_.U, nb_, (int64_t)m * nb_, w_.HV, npw_, mdp, w_.HX, npw_, nbp));
    return gwb_residual(nk_, nb_, npw_, w_.X, nbp, w_.HX, nbp, w_.eig, nb_, w_.R, nbp, w_.rn, st_);
  }

  int certify() {
    const int64_t nbp = (int64_t)nb_ * npw_;
    ++n_cert_;
    GWB_TRY(apply(w_.X, nbp, w_.HX, nbp, nb_, false));
    GWB_TRY(zgemm(0, 2, nb_, nb_, npw_, w_.X, npw_, nbp, w_.HX, npw_, nbp, w_.G, nb_, (int64_t)nb_ * nb_));
    dim3 g((unsigned)std::min((nb_ * nb_ + 255) / 256, 64), nk_);
    k_hermitize_conj<<<g, 256, 0, st_>>>(w_.G, w_.Gs, nb_);
    GWB_LAUNCH_CHECK();
    count_launches(1);
    GWB_TRY(gwb_heev_lowest(nk_, nb_, nb_, w_.Gs, nb_, (int64_t)nb_ * nb_, w_.eig2, w_.U, w_.Zs, w_.heev_info, st_));
    GWB_TRY(zgemm(1, 0, nb_, npw_, nb_, w_.U, nb_, (int64_t)nb_ * nb_, w_.X, npw_, nbp, w_.D2, npw_, nbp));
    GWB_CUDA_TRY(cudaMemcpyAsync(w_.X, w_.D2, sizeof(Z16) * nk_ * nbp, cudaMemcpyDeviceToDevice, st_));
    GWB_TRY(zgemm(1, 0, nb_, npw_, nb_, w_.U, nb_, (int64_t)nb_ * nb_, w_.HX, npw_, nbp, w_.D2, npw_, nbp));
    GWB_CUDA_TRY(cudaMemcpyAsync(w_.HX, w_.D2, sizeof(Z16) * nk_ * nbp, cudaMemcpyDeviceToDevice, st_));
    return gwb_residual(nk_, nb_, npw_, w_.X, nbp, w_.HX, nbp, w_.eig2, nb_, w_.R, nbp, w_.rn, st_);
  }

  int read_stats(double* rnmax, int* n_add, bool* breakdown) {
    GWB_TRY(gwb_conv_stats(nk_, nb_, w_.rn, p_.tol, w_.stats, st_));
    k_pack_flags<<<1, 32, 0, st_>>>(w_.heev_info, nk_, w_.flags, w_.stats);
    GWB_LAUNCH_CHECK();
    count_launches(1);
    double hst[4];
    GWB_CUDA_TRY(cudaMemcpyAsync(hst, w_.stats, sizeof(hst), cudaMemcpyDeviceToHost, st_));
    GWB_CUDA_TRY(cudaStreamSynchronize(st_));
    if (!(hst[0] == hst[0])) {
      set_error("non-finite residual norm");
      return GWB_ERR_NONFINITE;
    }
    if (hst[2] != 0.0) {
      set_error("subspace eigensolver hit the QL iteration limit");
      return GWB_ERR_NOT_CONVERGED;
    }
    const int flags = (int)hst[3];
    if (flags & 1) ++n_repair_;
    *breakdown = (flags & 2) != 0;
    *rnmax = hst[0];
    *n_add = (int)hst[1];
    return GWB_OK;
  }

  int precondition(int n_add, const double* eig) {
    const int64_t nbp = (int64_t)nb_ * npw_;
    if (p_.precond == 1 && !force_tpa_) {
      // stall fallback: a band whose residual has not improved on its best by
      // 10 % for 3 rounds keeps TPA from then on
      GWB_TRY(gwb_stall_update(w_.rn, w_.rn_prev, w_.stall_count, w_.tpa_only, nk_ * nb_, 0.9, 3, st_));
      return gwb_precond_learned(static_cast<const float*>(model_), nk_, nb_, n_add, npw_, w_.X, nbp, w_.R, nbp, t_,
                                 eig, w_.sel, w_.tpa_only, w_.D, nbp, w_.pl_work, w_.pl_work_bytes, st_);
    }
    return gwb_precond_teter(nk_, nb_, n_add, npw_, w_.X, nbp, w_.R, nbp, t_, w_.sel, w_.D, nbp, st_);
  }

  // Two rounds of Gram -> Cholesky -> L^-1 on n rows of Y (k stride ys); the
  // companion Z (if any) gets the same transform. sync: check breakdown on the
  // host (ok = 0 on failure); else breakdown only raises bit 1 of flags.
  int cholqr2(Z16* Y, int64_t ys, int n, Z16* Ytmp, Z16* Z, Z16* Ztmp, bool sync, int* ok) {
    const int64_t nn = (int64_t)n * n;
    *ok = 1;
    for (int pass = 0; pass < 2; ++pass) {
      GWB_TRY(zgemm(0, 2, n, n, npw_, Y, npw_, ys, Y, npw_, ys, w_.G, n, nn));
      if (sync) GWB_CUDA_TRY(cudaMemsetAsync(w_.sync_flag, 0, sizeof(int), st_));
      GWB_TRY(gwb_chol_inv(nk_, n, w_.G, n, nn, w_.Linv, nn, w_.info, sync ? w_.sync_flag : w_.flags, st_));
      if (sync) {
        // bit 1 of the flag: a breakdown at any k
        int host_flag = 0;
        GWB_CUDA_TRY(cudaMemcpyAsync(&host_flag, w_.sync_flag, sizeof(int), cudaMemcpyDeviceToHost, st_));
        GWB_CUDA_TRY(cudaStreamSynchronize(st_));
        if (host_flag & 2) {
          *ok = 0;
          return GWB_OK;
        }
      }
      GWB_TRY(zgemm(0, 0, n, npw_, n, w_.Linv, n, nn, Y, npw_, ys, Ytmp, npw_, (int64_t)nb_ * npw_));
      GWB_TRY(copy_rows(Y, ys, Ytmp, (int64_t)nb_ * npw_, n));
      if (Z) {
        GWB_TRY(zgemm(0, 0, n, npw_, n, w_.Linv, n, nn, Z, npw_, ys, Ztmp, npw_, (int64_t)nb_ * npw_));
        GWB_TRY(copy_rows(Z, ys, Ztmp, (int64_t)nb_ * npw_, n));
      }
    }
    return GWB_OK;
  }

  int project_out(Z16* Dblk, int64_t ds, int n, int m) {
    const int64_t mdp = (int64_t)md_ * npw_;
    GWB_TRY(zgemm(0, 2, n, m, npw_, Dblk, npw_, ds, w_.V, npw_, mdp, w_.C, m, (int64_t)n * m));
    return zgemm(0, 0, n, npw_, m, w_.C, m, (int64_t)n * m, w_.V, npw_, mdp, Dblk, npw_, ds, -1.0, 1.0);
  }

  int orthonormalize_new(int n, int m) {
    const int64_t nbp = (int64_t)nb_ * npw_;
    GWB_TRY(masked_copy(w_.D, nbp, w_.D, nbp, n));
    if (m) GWB_TRY(project_out(w_.D, nbp, n, m));
    GWB_TRY(gwb_row_repair(nk_, n, npw_, w_.D, nbp, mask_, repair_thresh_, w_.flags, st_));
    if (m) GWB_TRY(project_out(w_.D, nbp, n, m));
    int ok = 1;
    return cholqr2(w_.D, nbp, n, w_.D2, nullptr, nullptr, false, &ok);
  }

  gwb_ham* h_;
  gwb_davidson_params p_;
  const void* model_;
  const double* t_;
  const unsigned char* mask_;
  Work w_;
  cudaStream_t st_;
  int nk_, nb_, npw_, md_;
  bool fp32_exp_ = false;
  bool force_tpa_ = false;       // the round after a rollback preconditions with TPA
  double repair_thresh_ = 1e-8;  // rank-repair threshold of the expansion rows
  const double* last_eig_ = nullptr;
  int n_restart_ = 0, n_cert_ = 0, n_repair_ = 0, n_rollback_ = 0;
  int64_t n_low_ = 0, n_full_ = 0, n_apply_calls_ = 0;
  static constexpr int kMaxEvents = 2048;
  cudaEvent_t ev_[kMaxEvents];
  int n_events_ = 0;
};

}  // namespace gwb

using namespace gwb;

extern "C" {

int gwb_davidson_workspace_bytes(const gwb_davidson_params* p, size_t* bytes) {
  GWB_REQUIRE(p && bytes, "null argument");
  GWB_REQUIRE(p->nk > 0 && p->nb > 0 && p->npw > 0 && p->max_dim >= p->nb, "bad sizes");
  *bytes = layout(*p, nullptr, nullptr);
  return GWB_OK;
}

int gwb_davidson_solve(gwb_ham* h, const gwb_davidson_params* p, const void* model, const void* x0, const double* t,
                       const uint8_t* mask, void* workspace, size_t workspace_bytes, double* eig_out, void* vec_out,
                       double* rn_out, gwb_davidson_stats* stats, void* stream) {
  GWB_REQUIRE(h && p && x0 && t && mask && workspace && eig_out && vec_out && rn_out, "null argument");
  GWB_REQUIRE(p->nk > 0 && p->nb > 0 && p->npw > 0 && p->max_dim >= p->nb && p->max_iter > 0, "bad sizes");
  GWB_REQUIRE(p->max_dim <= gwb_heev_max_dim(),
              "max_dim exceeds the batched eigensolver limit; use the host-driven solver");
  GWB_REQUIRE(p->mode >= 0 && p->mode <= 2, "mode must be 0 (float64), 1 or 2 (float32 expansion)");
  GWB_REQUIRE(p->precond == 0 || (p->precond == 1 && model), "precond must be 0 (TPA) or 1 (learned, model set)");
  Work w;
  const size_t need = layout(*p, static_cast<unsigned char*>(workspace), &w);
  GWB_REQUIRE(workspace_bytes >= need, "workspace too small (see gwb_davidson_workspace_bytes)");
  GWB_REQUIRE(((uintptr_t)workspace % 256) == 0, "workspace must be 256-byte aligned");
  GWB_CUDA_TRY(cudaMemsetAsync(w.flags, 0, sizeof(int), (cudaStream_t)stream));
  Solver s(h, *p, model, t, mask, w, (cudaStream_t)stream);
  return s.run(x0, eig_out, vec_out, rn_out, stats);
}

}  // extern "C"
