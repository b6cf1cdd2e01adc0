// Householder tridiagonalisation of a dense real symmetric matrix across the
// whole GPU, for the Davidson subspace matrices too large for the one-CTA
// eigensolver (m in the hundreds to thousands): the step of
// torch.linalg.eigh (gradwave solvers/davidson.py:66-75,650) that cuSOLVER
// runs at ~11 us per column, latency-bound.
//
// Q^T A Q = T with Q = H_0 H_1 ... H_{m-2}, H_j = I - tau_j v_j v_j^T,
// v_j = (0, ..., 0, 1, v_j[j+2..m-1]) (Golub & Van Loan, Matrix Computations,
// 4th ed., sec. 8.3.1). The output is the LAPACK lower-storage convention of
// dsytrd: d = diag(T), e = the subdiagonal, tau, and v_j[j+2..] in column j of
// A below the subdiagonal (column-major, lda).
//
// Blocked in panels of NB columns with the update of the trailing matrix
// deferred (the panel form of LAPACK's dlatrd, Dongarra, Hammarling &
// Sorensen 1989): within a panel, column j is first brought up to date with
// the panel's earlier reflectors, a = A e_j - V W^T e_j - W V^T e_j, and the
// reflector's image w = tau (A v - V (W^T v) - W (V^T v)) - (tau^2 / 2)(...) v
// is formed from one product with the not-yet-updated trailing matrix; after
// the panel, A <- A - V W^T - W V^T on the trailing square.
//
// One cooperative launch with one block per SM. Each column takes two
// grid-wide barriers: (1) after the column update (the reflector needs the
// column's norm), (2) after the product y = A v and the panel dot products
// V^T v, W^T v, y . v (w needs them). The partial sums of each block are
// reduced by every block in the same fixed order, so all blocks hold the same
// values and the result does not depend on timing. The matrix is kept in full
// (both triangles, updated alike), so row r of the trailing matrix is read as
// its column r, contiguous: one warp per row. The barrier is one atomic per
// block (the last arrival flips bit 31 of the counter) and a spin bounded by
// gwb_tc_set_wait_limit's cycle count; a spin that runs out sets
// GWB_ERR_TIMEOUT and every block leaves at its next barrier.
#include <cooperative_groups.h>
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "sturm.cuh"
#include "tcgen05.cuh"

namespace gwb {
namespace {

constexpr int TD_NB = 8;         // panel width
constexpr int TD_THREADS = 512;  // threads per block
constexpr int TD_WARPS = TD_THREADS / 32;
constexpr int TD_NCOMP = 2 * TD_NB + 1;  // panel dot products V^T v, W^T v and y . v
constexpr int TD_MMAX = 4096;

struct TdArgs {
  int m;
  int kend;  // panels start below kend (the cluster kernel reduces the rest)
  double* A;  // column-major, lda
  int64_t lda;
  double *d, *e, *tau;
  double *V, *W;   // panel vectors, m x NB each (column i at i m)
  double *acol, *ycol;  // the current column, the product A v
  double *part1, *part2;  // per-block partial sums (gridDim.x and gridDim.x * TD_NCOMP)
  unsigned* bar;
  int* status;
  long long wait_cycles;
  long long* trace;  // per-phase SM cycles of block 0 (gwb_sytrd_set_trace), or null
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier: one release-add per block (the last arrival flips bit
// 31 of the counter) and an acquire spin bounded by `limit` cycles; false
// once a spin ran out (then every caller leaves).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* status, long long limit, int* s_abort) {
  __syncthreads();
  if (threadIdx.x == 0 && !*s_abort) {
    const unsigned inc = blockIdx.x == 0 ? (0x80000000u - (gridDim.x - 1u)) : 1u;
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(bar), "r"(inc) : "memory");
    const long long t0 = clock64();
    while (((ld_acquire_u32(bar) ^ old) & 0x80000000u) == 0u) {
      if (clock64() - t0 > limit) {
        *s_abort = 1;
        atomicOr(status, GWB_ERR_TIMEOUT);
        break;
      }
    }
  }
  __syncthreads();
  return *s_abort == 0;
}

// Phase trace of block 0 (thread 0): cycles spent in phases 0-5, added up
// over all columns: 0 phase B up to the product, 1 the product y = A v,
// 2 the barrier after it, 3 phase C and the next column update, 4 the barrier
// after that, 5 the trailing updates with their barriers.
#define TD_MARK(slot)                                                 \
  do {                                                                \
    if (a.trace && gt == 0) {                                         \
      const long long _now = clock64();                              \
      a.trace[(slot)] += _now - td_t;                                 \
      td_t = _now;                                                    \
    }                                                                 \
  } while (0)

// Row ownership: thread t of the grid owns row t (m <= 4096 rows, so the
// owners sit in the first ceil(m / 512) blocks) and keeps its row of the
// panel's V and W in registers. Every block keeps the panel's own rows
// (k0 .. k0 + NB - 1) of V and W in shared tables, built redundantly from
// data every block has, so the column update reads nothing shared but its
// own column element.
__global__ void __launch_bounds__(TD_THREADS, 1) k_sytrd_coop(TdArgs a) {
  extern __shared__ __align__(16) double td_smem[];
  double* vs = td_smem;                 // v_j[j+1 ..], m doubles
  __shared__ double wpart[TD_WARPS][TD_NCOMP];
  __shared__ double comp[TD_NCOMP];
  __shared__ double tabV[TD_NB][TD_NB], tabW[TD_NB][TD_NB];  // [panel row][reflector]
  __shared__ double sc_s[4];
  __shared__ int s_abort;
  if (threadIdx.x == 0) s_abort = 0;
  __syncthreads();

  const int m = a.m;
  const int64_t lda = a.lda;
  double* A = a.A;
  const int gt = blockIdx.x * TD_THREADS + threadIdx.x;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int gw = blockIdx.x * TD_WARPS + wib, GW = gridDim.x * TD_WARPS;
  const int nbo = (m + TD_THREADS - 1) / TD_THREADS;  // blocks that own rows
  const bool owner_block = (int)blockIdx.x < nbo;
  const int r = gt;                                    // this thread's row (if < m)
  const bool own = r < m;
  double vreg[TD_NB], wreg[TD_NB];

  if (m == 1) {
    if (gt == 0) a.d[0] = A[0];
    return;
  }
  long long td_t = clock64();

  for (int k0 = 0; k0 < min(m - 1, a.kend); k0 += TD_NB) {
    const int nbk = min(TD_NB, m - 1 - k0);
#pragma unroll
    for (int i = 0; i < TD_NB; ++i) vreg[i] = wreg[i] = 0.0;
    if (threadIdx.x < TD_NB * TD_NB) {
      tabV[threadIdx.x / TD_NB][threadIdx.x % TD_NB] = 0.0;
      tabW[threadIdx.x / TD_NB][threadIdx.x % TD_NB] = 0.0;
    }
    // ---- phase A of the panel's first column (no corrections yet) ----
    {
      const int j = k0;
      double ssq = 0.0;
      if (own && r >= j) {
        const double v = A[r + (int64_t)j * lda];
        a.acol[r] = v;
        if (r == j) a.d[j] = v;
        if (r >= j + 2) ssq = v * v;
      }
      if (owner_block) {
        for (int o = 16; o > 0; o >>= 1) ssq += __shfl_xor_sync(0xffffffffu, ssq, o);
        if (lane == 0) wpart[wib][0] = ssq;
        __syncthreads();
        if (threadIdx.x == 0) {
          double s = 0.0;
          for (int w = 0; w < TD_WARPS; ++w) s += wpart[w][0];
          a.part1[blockIdx.x] = s;
        }
      }
      if (!grid_barrier(a.bar, a.status, a.wait_cycles, &s_abort)) return;
    }
    for (int jj = 0; jj < nbk; ++jj) {
      const int j = k0 + jj;
      const int n1 = m - j - 1;  // length of v from j + 1
      // ---- phase B: the reflector, y = A v, panel dot products ----
      // one round trip: the norm partials and the updated column
      double ps = 0.0;
      if (wib == 0)
        for (int b = lane; b < nbo; b += 32) ps += a.part1[b];
      for (int c = threadIdx.x; c < n1; c += TD_THREADS) vs[c] = a.acol[j + 1 + c];
      if (wib == 0) {
        for (int o = 16; o > 0; o >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, o);
        if (lane == 0) {
          const double alpha = a.acol[j + 1];
          double tau = 0.0, beta = alpha, scl = 0.0;
          if (ps > 0.0) {
            beta = -copysign(sqrt(alpha * alpha + ps), alpha);
            tau = (beta - alpha) / beta;
            scl = 1.0 / (alpha - beta);
          }
          sc_s[0] = tau;
          sc_s[1] = scl;
          if (blockIdx.x == 0) {
            a.e[j] = beta;
            a.tau[j] = tau;
            A[j + 1 + (int64_t)j * lda] = beta;
            A[j + (int64_t)j * lda] = a.d[j];
          }
        }
      }
      __syncthreads();
      const double tau = sc_s[0], scl = sc_s[1];
      for (int c = threadIdx.x; c < n1; c += TD_THREADS) vs[c] = c == 0 ? 1.0 : vs[c] * scl;
      __syncthreads();
      // the panel rows of v_j into the table; this thread's row of V
      if (threadIdx.x < TD_NB) {
        const int pr = threadIdx.x, row = k0 + pr;
        tabV[pr][jj] = row >= j + 1 && row < m ? vs[row - j - 1] : 0.0;
      }
      double acc_v = 0.0;  // this row's v_j entry
      if (own && r >= j + 1) {
        acc_v = vs[r - j - 1];
        vreg[jj] = acc_v;
        a.V[r + (int64_t)jj * m] = acc_v;
        if (r >= j + 2) A[r + (int64_t)j * lda] = acc_v;
      }
      TD_MARK(0);
      // every warp: y_r = A[r, j+1:] . v for its row, and the row's shares of
      // V^T v (lanes i < jj), W^T v (lanes NB + i) and y . v (lane 2 NB)
      double yv = 0.0, pc = 0.0;
      for (int rr = j + 1 + gw; rr < m; rr += GW) {
        const double* col = A + (int64_t)rr * lda + (j + 1);
        double vw = 0.0;  // this lane's entry of the row of V or W
        if (lane < jj) vw = a.V[rr + (int64_t)lane * m];
        else if (lane >= TD_NB && lane - TD_NB < jj) vw = a.W[rr + (int64_t)(lane - TD_NB) * m];
        double y = 0.0;
        int c = lane;
        for (; c + 15 * 32 < n1; c += 16 * 32) {
          double t[16];
#pragma unroll
          for (int u = 0; u < 16; ++u) t[u] = col[c + u * 32];
#pragma unroll
          for (int u = 0; u < 16; ++u) y += t[u] * vs[c + u * 32];
        }
        for (; c + 7 * 32 < n1; c += 8 * 32) {
          double t[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) t[u] = col[c + u * 32];
#pragma unroll
          for (int u = 0; u < 8; ++u) y += t[u] * vs[c + u * 32];
        }
        for (; c < n1; c += 32) y += col[c] * vs[c];
        for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        if (lane == 0) a.ycol[rr] = y;
        const double vr = vs[rr - j - 1];
        yv += y * vr;
        pc += vw * vr;
      }
      if (lane < 2 * TD_NB) wpart[wib][lane] = pc;
      if (lane == 0) wpart[wib][2 * TD_NB] = yv;
      __syncthreads();
      if (threadIdx.x < TD_NCOMP) {
        double s = 0.0;
        for (int w = 0; w < TD_WARPS; ++w) s += wpart[w][threadIdx.x];
        a.part2[(int64_t)blockIdx.x * TD_NCOMP + threadIdx.x] = s;
      }
      TD_MARK(1);
      if (!grid_barrier(a.bar, a.status, a.wait_cycles, &s_abort)) return;
      TD_MARK(2);

      // ---- phase C (w_j) and phase A of column j + 1 ----
      // one round trip: the dot-product partials, this row's y, the panel
      // rows' y, this row's element of column j + 1
      const bool next_in_panel = jj + 1 < nbk;
      const int j1 = j + 1;
      // this warp's product row of the next column into L1 while the
      // barriers pass (A's trailing part is not written before it is read)
      if (next_in_panel) {
        const int rr = j1 + 1 + gw;
        if (rr < m) {
          const char* base = reinterpret_cast<const char*>(A + (int64_t)rr * lda + (j1 + 1));
          const int bytes = (m - j1 - 1) * 8;
          for (int off = lane * 128; off < bytes; off += 32 * 128)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(base + off));
        }
      }
      double y_own = 0.0, a_next = 0.0;
      if (own && r >= j + 1) y_own = a.ycol[r];
      if (own && next_in_panel && r >= j1) a_next = A[r + (int64_t)j1 * lda];
      double y_tab = 0.0;
      if (threadIdx.x < TD_NB) {
        const int row = k0 + threadIdx.x;
        if (row >= j + 1 && row < m) y_tab = a.ycol[row];
      }
      for (int q = wib; q < TD_NCOMP; q += TD_WARPS) {
        double sq = 0.0;
        for (int b = lane; b < (int)gridDim.x; b += 32) sq += a.part2[(int64_t)b * TD_NCOMP + q];
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
        if (lane == 0) comp[q] = sq;
      }
      __syncthreads();
      // comp[i] = (V^T v)_i, comp[NB + i] = (W^T v)_i, comp[2 NB] = y . v
      double pvw = 0.0;
      for (int i = 0; i < jj; ++i) pvw += comp[i] * comp[TD_NB + i];
      const double wv = tau * (comp[2 * TD_NB] - 2.0 * pvw);
      const double half = 0.5 * tau * wv;
      if (own && r >= j + 1) {
        double sw = y_own;
#pragma unroll
        for (int i = 0; i < TD_NB; ++i)
          if (i < jj) sw -= vreg[i] * comp[TD_NB + i] + wreg[i] * comp[i];
        const double w = tau * sw - half * acc_v;
        wreg[jj] = w;
        a.W[r + (int64_t)jj * m] = w;
      }
      if (threadIdx.x < TD_NB) {
        const int pr = threadIdx.x, row = k0 + pr;
        double w = 0.0;
        if (row >= j + 1 && row < m) {
          double sw = y_tab;
          for (int i = 0; i < jj; ++i) sw -= tabV[pr][i] * comp[TD_NB + i] + tabW[pr][i] * comp[i];
          w = tau * sw - half * tabV[pr][jj];
        }
        tabW[pr][jj] = w;
      }
      __syncthreads();
      if (next_in_panel) {
        // column j + 1 up to date: a = A e_{j1} - V W[j1,:]^T - W V[j1,:]^T
        const int pr1 = j1 - k0;
        double ssq = 0.0;
        if (own && r >= j1) {
          double v = a_next;
#pragma unroll
          for (int i = 0; i < TD_NB; ++i)
            if (i <= jj) v -= vreg[i] * tabW[pr1][i] + wreg[i] * tabV[pr1][i];
          a.acol[r] = v;
          if (r == j1) a.d[j1] = v;
          if (r >= j1 + 2) ssq = v * v;
        }
        if (owner_block) {
          for (int o = 16; o > 0; o >>= 1) ssq += __shfl_xor_sync(0xffffffffu, ssq, o);
          if (lane == 0) wpart[wib][0] = ssq;
          __syncthreads();
          if (threadIdx.x == 0) {
            double s = 0.0;
            for (int w = 0; w < TD_WARPS; ++w) s += wpart[w][0];
            a.part1[blockIdx.x] = s;
          }
        }
        TD_MARK(3);
        if (!grid_barrier(a.bar, a.status, a.wait_cycles, &s_abort)) return;
        TD_MARK(4);
      }
    }
    // ---- trailing update A <- A - V W^T - W V^T on rows/columns >= k0 + nbk ----
    // 32 x 32 tiles spread over all warps of the grid: lane rr holds row
    // rt + rr of V and W, the tile's columns of V and W go to the warp's
    // shared slice, and the warp updates the tile column by column
    // (consecutive rows per column: coalesced).
    const int t0 = k0 + nbk;
    if (t0 < m) {
      if (!grid_barrier(a.bar, a.status, a.wait_cycles, &s_abort)) return;
      const int nt = m - t0;
      const int tiles = (nt + 31) / 32;
      double* cvw = vs + (size_t)wib * 2 * 32 * TD_NB;  // this warp's 32 columns of V then W
      const double* V = a.V;
      const double* W = a.W;
      for (int tile = gw; tile < tiles * tiles; tile += GW) {
        const int rt = t0 + (tile % tiles) * 32, ct = t0 + (tile / tiles) * 32;
        const int row = rt + lane, colr = ct + lane;
        double tv[TD_NB], tw[TD_NB];
#pragma unroll
        for (int i = 0; i < TD_NB; ++i) {
          tv[i] = (i < nbk && row < m) ? V[row + (int64_t)i * m] : 0.0;
          tw[i] = (i < nbk && row < m) ? W[row + (int64_t)i * m] : 0.0;
          cvw[lane * TD_NB + i] = (i < nbk && colr < m) ? V[colr + (int64_t)i * m] : 0.0;
          cvw[32 * TD_NB + lane * TD_NB + i] = (i < nbk && colr < m) ? W[colr + (int64_t)i * m] : 0.0;
        }
        __syncwarp();
        const int ncol = min(32, m - ct);
        if (row < m) {
          // sixteen columns' elements of this row in flight at once
          for (int c0 = 0; c0 < ncol; c0 += 16) {
            double av[16];
#pragma unroll
            for (int u = 0; u < 16; ++u)
              av[u] = c0 + u < ncol ? A[row + (int64_t)(ct + c0 + u) * lda] : 0.0;
#pragma unroll
            for (int u = 0; u < 16; ++u) {
              const int cc = c0 + u;
              double sacc = 0.0;
#pragma unroll
              for (int i = 0; i < TD_NB; ++i)
                sacc += tv[i] * cvw[32 * TD_NB + cc * TD_NB + i] + tw[i] * cvw[cc * TD_NB + i];
              if (cc < ncol) A[row + (int64_t)(ct + cc) * lda] = av[u] - sacc;
            }
          }
        }
        __syncwarp();
      }
      if (!grid_barrier(a.bar, a.status, a.wait_cycles, &s_abort)) return;
    }
    TD_MARK(5);
  }
  // d[m-1]: the last diagonal element after the final panel's update (when
  // the cluster kernel does not take over the trailing part)
  if (gt == 0 && a.kend >= m - 1) a.d[m - 1] = A[(m - 1) + (int64_t)(m - 1) * lda];
}

// ---------------------------------------------------------------------------
// The trailing part inside one thread-block cluster. Once the trailing
// matrix (n = m - t0 rows, fully updated, both triangles) fits in the
// cluster's distributed shared memory, the rest of the reduction runs there:
// CTA c of the cluster keeps rows c, c + CS, c + 2 CS, ... (full rows), and a
// column costs one cluster barrier and one pass over the local rows instead
// of two grid barriers and several L2 round trips.
//
// Unblocked form (LAPACK dsytd2: p = tau A v, w = p - (tau/2)(p.v) v,
// A <- A - v w^T - w v^T), with the rank-2 update of reflector j - 1
// deferred into the pass that forms the product of reflector j:
//   R(j), in every CTA with the same arithmetic: w_{j-1} = p - K v_{j-1}
//     from the gathered p and the partial sums of p.v; column j brought up
//     to date from its gathered entries, a_k = raw_k - v_k w_j - w_k v_j
//     (reflector j - 1); the reflector v_j, tau_j from it. Every CTA thus
//     holds identical w_{j-1}, v_j and tau_j;
//   F(j), own rows i > j, columns k > j: A_ik -= v_i w_k + w_i v_k
//     (reflector j - 1) and y_i = sum_k A_ik v_j[k] on the updated values;
//     each owner sends p_i = tau_j y_i, its row's element of column j + 1
//     (raw, updated through reflector j - 1) and the CTA's part of p.v to
//     every CTA;
//   one cluster barrier.
// The gathered vectors are double-buffered by the parity of j: a CTA still
// reading column j's values while another already sends column j + 1's uses
// the other buffer, and the barrier after j + 1 orders the next reuse. Sums
// that every CTA needs are formed in one fixed order in every CTA. The
// cluster barriers are hardware barriers that every thread of every CTA
// reaches the same number of times.
constexpr int TK_THREADS = 1024;
constexpr int TK_WARPS = TK_THREADS / 32;
static_assert(TK_WARPS == 32, "tk_block_sum reduces one warp sum per lane");
constexpr int TK_SEG = 128;    // columns per warp item of the pass (4 per lane)
constexpr int TK_NSEG = 8;     // segments per row at most (n <= 1024)

struct TkArgs {
  int m, t0;  // the trailing part A[t0:, t0:], n = m - t0 rows
  double* A;
  int64_t lda;
  double *d, *e, *tau;
  long long* trace;  // cycles of CTA 0 in R, F, the exchange, the barrier (4 slots), or null
};

// local rows (padded to an even count of doubles, so the exchange buffers
// after them are 16-byte aligned), column, v [2], w, (p, raw) pairs [2],
// row partial products
__host__ __device__ inline size_t tk_smem_doubles(int n, int cs) {
  const size_t nl = (size_t)(n + cs - 1) / cs;
  return (nl * n + 1) / 2 * 2 + 8 * (size_t)n + nl * TK_NSEG;
}

// Sum over the block: each warp's sum by shuffles, then every warp reduces
// the 32 warp sums by shuffles in the same order, so every thread gets the
// same value.
__device__ __forceinline__ double tk_block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = red[threadIdx.x & 31];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// Sum of the CS per-CTA parts, by shuffles (the same order in every warp).
template <int CS>
__device__ __forceinline__ double tk_part_sum(const double* part) {
  double s = (threadIdx.x & 31) < CS ? part[threadIdx.x & 31] : 0.0;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

#define TK_MARK(slot)                                      \
  do {                                                     \
    if (a.trace && c == 0 && tid == 0) {                   \
      const long long _now = clock64();                   \
      a.trace[(slot)] += _now - tk_t;                      \
      tk_t = _now;                                         \
    }                                                      \
  } while (0)

template <int CS>
__global__ void __launch_bounds__(TK_THREADS, 1) k_sytrd_cluster(TkArgs a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) double tk_smem[];
  __shared__ double part[2][CS];
  __shared__ double red[TK_WARPS];
  const int c = (int)cl.block_rank();
  const int n = a.m - a.t0, t0 = a.t0;
  const int nl = (n + CS - 1) / CS;
  const int64_t lda = a.lda;
  double* A = a.A + t0 + (int64_t)t0 * lda;  // the trailing block's origin
  double* Al = tk_smem;                       // local row li = trailing row c + li CS, n columns
  double* col = Al + ((size_t)nl * n + 1) / 2 * 2;  // column j, fully updated
  double* vbuf = col + n;                     // [2][n]: v_j by parity of j
  double* wbuf = vbuf + 2 * (size_t)n;        // w_{j-1}
  double2* prbuf = reinterpret_cast<double2*>(wbuf + n);  // [2][n]: gathered (p, raw) by parity
  double* ypart = reinterpret_cast<double*>(prbuf + 2 * (size_t)n);  // [nl][TK_NSEG] row partial products
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  long long tk_t = clock64();

  for (int t = tid; t < nl * n; t += TK_THREADS) {
    const int li = t / n, k = t - li * n, i = c + li * CS;
    Al[t] = i < n ? A[k + (int64_t)i * lda] : 0.0;  // column i = row i
  }
  for (int k = tid; k < n; k += TK_THREADS) col[k] = A[k];
  cl.sync();  // every CTA of the cluster runs: shared windows are valid

  double tau_prev = 0.0;
  for (int j = 0; j + 1 < n; ++j) {
    const int q = j & 1, qp = q ^ 1;
    double* vj = vbuf + (size_t)q * n;
    const double* vq = vbuf + (size_t)qp * n;  // v_{j-1}
    // ---- R(j): w_{j-1}, column j, reflector j (identical in every CTA) ----
    double s = 0.0;
    if (j > 0) {
      const double K = tk_part_sum<CS>(part[qp]) * (0.5 * tau_prev);
      const double2* pr = prbuf + (size_t)qp * n;
      const double vjj = vq[j];
      const double wj = pr[j].x - K * vjj;
      for (int k = j + tid; k < n; k += TK_THREADS) {
        const double2 x = pr[k];
        const double vk = vq[k];
        const double wk = x.x - K * vk;
        const double ck = x.y - vk * wj - wk * vjj;
        wbuf[k] = wk;
        col[k] = ck;
        if (k >= j + 2) s += ck * ck;
      }
    } else {
      for (int k = j + 2 + tid; k < n; k += TK_THREADS) s += col[k] * col[k];
    }
    s = tk_block_sum(s, red);  // its barriers also publish col and w
    const double alpha = col[j + 1];
    double tau = 0.0, beta = alpha, scl = 0.0;
    if (s > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + s), alpha);
      tau = (beta - alpha) / beta;
      scl = 1.0 / (alpha - beta);
    }
    for (int k = j + 1 + tid; k < n; k += TK_THREADS) vj[k] = k == j + 1 ? 1.0 : col[k] * scl;
    if (c == 0) {
      for (int k = j + 2 + tid; k < n; k += TK_THREADS) A[k + (int64_t)j * lda] = col[k] * scl;
      if (tid == 0) {
        a.d[t0 + j] = col[j];
        a.e[t0 + j] = beta;
        a.tau[t0 + j] = tau;
        A[j + (int64_t)j * lda] = col[j];
        A[j + 1 + (int64_t)j * lda] = beta;
      }
    }
    __syncthreads();
    TK_MARK(0);
    // ---- F(j): update with reflector j - 1, product with v_j ----
    const int kb = j + 1, ncol = n - kb;
    const int nseg = (ncol + TK_SEG - 1) / TK_SEG;
    const int wps = TK_WARPS / nseg;  // warps per segment
    const int li0 = kb > c ? (kb - c + CS - 1) / CS : 0;
    double2* pr = prbuf + (size_t)q * n;
    if (warp < nseg * wps) {
      const int sg = warp / wps, wr = warp - sg * wps;
      const int klo = kb + sg * TK_SEG, khi = min(n, klo + TK_SEG);
      double vk[4], wk[4], qk[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int k = klo + lane + 32 * u;
        const bool in = k < khi;
        vk[u] = in ? vj[k] : 0.0;
        wk[u] = (in && j > 0) ? wbuf[k] : 0.0;
        qk[u] = (in && j > 0) ? vq[k] : 0.0;
      }
      for (int li = li0 + wr; li < nl; li += wps) {
        const int i = c + li * CS;
        if (i >= n) break;
        double* row = Al + (size_t)li * n;
        const double vi = j > 0 ? vq[i] : 0.0, wi = j > 0 ? wbuf[i] : 0.0;
        double y = 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = klo + lane + 32 * u;
          if (k < khi) {
            double x = row[k];
            if (j > 0) {
              x -= vi * wk[u] + wi * qk[u];
              row[k] = x;
            }
            if (u == 0 && sg == 0 && lane == 0) pr[i].y = x;  // column j + 1's entry (k = kb)
            y += x * vk[u];
          }
        }
        for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        if (lane == 0) ypart[(size_t)li * TK_NSEG + sg] = y;
      }
    }
    __syncthreads();
    TK_MARK(1);
    // p_i = tau y_i for own rows; the CTA's part of p.v; everything to every CTA
    double pv = 0.0;
    for (int li = li0 + tid; li < nl; li += TK_THREADS) {
      const int i = c + li * CS;
      if (i < n) {
        double y = 0.0;
        for (int sg = 0; sg < nseg; ++sg) y += ypart[(size_t)li * TK_NSEG + sg];
        const double p = tau * y;
        pr[i].x = p;
        pv += p * vj[i];
      }
    }
    pv = tk_block_sum(pv, red);
    const int nown = nl - li0;
    for (int t = tid; t < nown * CS; t += TK_THREADS) {
      const int li = li0 + t / CS, r = t % CS, i = c + li * CS;
      if (i < n && r != c) *cl.map_shared_rank(pr + i, r) = pr[i];
    }
    if (tid < CS) *cl.map_shared_rank(&part[q][c], tid) = pv;
    tau_prev = tau;
    TK_MARK(2);
    cl.sync();
    TK_MARK(3);
  }
  if (c == 0) {
    // the last diagonal element: column n - 1 through the last reflector
    double dl = col[0];
    if (n >= 2) {
      const int j = n - 1, qp = (j - 1) & 1;
      const double K = tk_part_sum<CS>(part[qp]) * (0.5 * tau_prev);
      const double* vq = vbuf + (size_t)qp * n;
      const double2 x = prbuf[(size_t)qp * n + j];
      const double w = x.x - K * vq[j];
      dl = x.y - 2.0 * vq[j] * w;
    }
    if (tid == 0) {
      a.d[t0 + n - 1] = dl;
      A[(n - 1) + (int64_t)(n - 1) * lda] = dl;
    }
  }
}
// ---------------------------------------------------------------------------
// The middle part across the whole GPU with the trailing matrix in shared
// memory. Once the trailing matrix (n = m - t0 rows, fully updated, both
// triangles) fits the shared memory of all the SMs (~1790 rows with one
// 1024-thread CTA per SM), columns t0 .. t1 - 1 are reduced as in
// k_sytrd_cluster, with the exchange through global memory: CTA c keeps rows
// c, c + G, ... (G = the grid); per column every CTA forms w of the previous
// reflector, the column and the reflector from the gathered (p, raw) pairs
// (the same arithmetic everywhere), passes over its rows (the previous
// reflector's rank-2 update fused with the product of the current one),
// writes its rows' p and next-column entries and its part of p.v, and meets
// the others at one grid barrier. The pairs and parts are double-buffered by
// the parity of the column and read past L1 (ld.global.cg). When t1 < m - 1
// the trailing part at t1, brought up to date with reflector t1 - 1, is
// written back (both triangles) for the cluster kernel.
constexpr int TG_NSEG = 16;  // segments of 128 columns per row at most (n <= 2048)

struct TgArgs {
  int m, t0, t1;
  double* A;
  int64_t lda;
  double *d, *e, *tau;
  double2* pr;     // [2][n] (p, raw) by parity
  double* part;    // [2][gridDim.x] parts of p.v by parity
  unsigned* bar;
  int* status;
  long long wait_cycles;
};

__host__ __device__ inline size_t tg_smem_doubles(int n, int g) {
  const size_t nl = (size_t)(n + g - 1) / g;
  return (nl * n + 1) / 2 * 2 + 3 * (size_t)n + nl * TG_NSEG;
}

// Sum of the g parts, read past L1, in the same order in every warp.
__device__ __forceinline__ double tg_part_sum(const double* part, int g) {
  double s = 0.0;
  for (int i = (threadIdx.x & 31); i < g; i += 32) s += __ldcg(part + i);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

__global__ void __launch_bounds__(TK_THREADS, 1) k_sytrd_grid(TgArgs a) {
  extern __shared__ __align__(16) double tg_smem[];
  __shared__ double red[TK_WARPS];
  __shared__ double sc[2];
  __shared__ int s_abort;
  const int G = gridDim.x, c = blockIdx.x;
  const int n = a.m - a.t0, t0 = a.t0, ncols = a.t1 - a.t0;
  const int nl = (n + G - 1) / G;
  const int64_t lda = a.lda;
  double* A = a.A + t0 + (int64_t)t0 * lda;
  double* Al = tg_smem;                                  // local row li = trailing row c + li G
  double* vbuf = Al + ((size_t)nl * n + 1) / 2 * 2;      // [2][n]: v_j by parity
  double* wbuf = vbuf + 2 * (size_t)n;                   // w_{j-1}
  double* ypart = wbuf + n;                              // [nl][TG_NSEG]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_abort = 0;
  for (int t = tid; t < nl * n; t += TK_THREADS) {
    const int li = t / n, k = t - li * n, i = c + li * G;
    Al[t] = i < n ? A[k + (int64_t)i * lda] : 0.0;  // column i = row i
  }
  // column 0 into registers before any CTA writes reflector 0 into it
  double c0[2];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int k = tid + TK_THREADS * r;
    c0[r] = k < n ? A[k] : 0.0;
  }
  if (!grid_barrier(a.bar, a.status, a.wait_cycles, &s_abort)) return;

  double tau_prev = 0.0;
  for (int j = 0; j < ncols; ++j) {
    const int q = j & 1, qp = q ^ 1;
    double* vj = vbuf + (size_t)q * n;
    const double* vq = vbuf + (size_t)qp * n;  // v_{j-1}
    const double2* prq = a.pr + (size_t)qp * n;
    // ---- R(j): w_{j-1}, column j (two entries per thread), reflector j ----
    double ck[2] = {0.0, 0.0};
    double s = 0.0;
    double K = 0.0, wj = 0.0, vjj = 0.0;
    if (j > 0) {
      K = tg_part_sum(a.part + (size_t)qp * G, G) * (0.5 * tau_prev);
      vjj = vq[j];
      wj = __ldcg(&prq[j].x) - K * vjj;
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int k = j + tid + TK_THREADS * r;
      if (k < n) {
        double x;
        if (j > 0) {
          const double2 e2 = __ldcg(&prq[k]);
          const double vk = vq[k];
          const double wk = e2.x - K * vk;
          wbuf[k] = wk;
          x = e2.y - vk * wj - wk * vjj;
        } else {
          x = c0[r];  // column 0 (k = tid + 1024 r at j = 0)
        }
        ck[r] = x;
        if (k >= j + 2) s += x * x;
        if (k == j) sc[1] = x;
        if (k == j + 1) sc[0] = x;
      }
    }
    s = tk_block_sum(s, red);  // its barriers also publish sc and w
    const double alpha = sc[0], dj = sc[1];
    double tau = 0.0, beta = alpha, scl = 0.0;
    if (s > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + s), alpha);
      tau = (beta - alpha) / beta;
      scl = 1.0 / (alpha - beta);
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int k = j + tid + TK_THREADS * r;
      if (k >= j + 1 && k < n) {
        const double v = k == j + 1 ? 1.0 : ck[r] * scl;
        vj[k] = v;
        if (c == 0 && k >= j + 2) A[k + (int64_t)j * lda] = v;
      }
    }
    if (c == 0 && tid == 0) {
      a.d[t0 + j] = dj;
      a.e[t0 + j] = beta;
      a.tau[t0 + j] = tau;
      A[j + (int64_t)j * lda] = dj;
      A[j + 1 + (int64_t)j * lda] = beta;
    }
    __syncthreads();
    // ---- F(j): update with reflector j - 1, product with v_j ----
    const int kb = j + 1, ncol = n - kb;
    const int nseg = (ncol + TK_SEG - 1) / TK_SEG;
    const int wps = TK_WARPS / nseg;
    const int li0 = kb > c ? (kb - c + G - 1) / G : 0;
    double2* prw = a.pr + (size_t)q * n;
    if (warp < nseg * wps) {
      const int sg = warp / wps, wr = warp - sg * wps;
      const int klo = kb + sg * TK_SEG, khi = min(n, klo + TK_SEG);
      double vk[4], wk[4], qk[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int k = klo + lane + 32 * u;
        const bool in = k < khi;
        vk[u] = in ? vj[k] : 0.0;
        wk[u] = (in && j > 0) ? wbuf[k] : 0.0;
        qk[u] = (in && j > 0) ? vq[k] : 0.0;
      }
      for (int li = li0 + wr; li < nl; li += wps) {
        const int i = c + li * G;
        if (i >= n) break;
        double* row = Al + (size_t)li * n;
        const double vi = j > 0 ? vq[i] : 0.0, wi = j > 0 ? wbuf[i] : 0.0;
        double y = 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = klo + lane + 32 * u;
          if (k < khi) {
            double x = row[k];
            if (j > 0) {
              x -= vi * wk[u] + wi * qk[u];
              row[k] = x;
            }
            if (u == 0 && sg == 0 && lane == 0) prw[i].y = x;  // column j + 1's entry (k = kb)
            y += x * vk[u];
          }
        }
        for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        if (lane == 0) ypart[(size_t)li * TG_NSEG + sg] = y;
      }
    }
    __syncthreads();
    double pv = 0.0;
    for (int li = li0 + tid; li < nl; li += TK_THREADS) {
      const int i = c + li * G;
      if (i < n) {
        double y = 0.0;
        for (int sg = 0; sg < nseg; ++sg) y += ypart[(size_t)li * TG_NSEG + sg];
        const double p = tau * y;
        prw[i].x = p;
        pv += p * vj[i];
      }
    }
    pv = tk_block_sum(pv, red);
    if (tid == 0) a.part[(size_t)q * G + c] = pv;
    tau_prev = tau;
    if (!grid_barrier(a.bar, a.status, a.wait_cycles, &s_abort)) return;
  }
  const int J = ncols;  // the first column not reduced here
  if (J >= n - 1) {
    // to the end: the last diagonal element through the last reflector
    if (c == 0 && n >= 2) {
      const int qp = (J - 1) & 1;
      const double K = tg_part_sum(a.part + (size_t)qp * G, G) * (0.5 * tau_prev);
      const double* vq = vbuf + (size_t)qp * n;
      const double2 x = __ldcg(&a.pr[(size_t)qp * n + (n - 1)]);
      const double w = x.x - K * vq[n - 1];
      const double dl = x.y - 2.0 * vq[n - 1] * w;
      if (tid == 0) {
        a.d[t0 + n - 1] = dl;
        A[(n - 1) + (int64_t)(n - 1) * lda] = dl;
      }
    }
    return;
  }
  // the trailing part at J through reflector J - 1, back to global memory
  if (J > 0) {
    const int qp = (J - 1) & 1;
    const double K = tg_part_sum(a.part + (size_t)qp * G, G) * (0.5 * tau_prev);
    const double* vq = vbuf + (size_t)qp * n;
    const double2* prq = a.pr + (size_t)qp * n;
    for (int k = J + tid; k < n; k += TK_THREADS) wbuf[k] = __ldcg(&prq[k].x) - K * vq[k];
    __syncthreads();
    for (int li = 0; li < nl; ++li) {
      const int i = c + li * G;
      if (i < J || i >= n) continue;
      const double vi = vq[i], wi = wbuf[i];
      const double* row = Al + (size_t)li * n;
      for (int k = J + tid; k < n; k += TK_THREADS) A[k + (int64_t)i * lda] = row[k] - vi * wbuf[k] - wi * vq[k];
    }
  }
}

// ---------------------------------------------------------------------------
// The lowest nev eigenpairs of the tridiagonal (d, e), then of A.
//
// 1. Eigenvalues by multisection on Sturm counts: one warp per eigenvalue,
//    its 32 lanes count at 32 points of the current interval, so each round
//    narrows it 33-fold (Gershgorin start; Barth, Martin & Wilkinson,
//    Numer. Math. 9 (1967) 386).
// 2. Eigenvectors of T by three steps of inverse iteration from seeded
//    random starts: Gaussian elimination of T - lambda I with partial
//    pivoting, factored once (Wilkinson, The Algebraic Eigenvalue Problem,
//    ch. 9; LAPACK dstein). Eigenvalues within 1e-9 |T| of each other form a
//    cluster: one thread runs its members in order and orthogonalises each
//    against the earlier ones after every step, then rotates the cluster by
//    a Jacobi Rayleigh-Ritz of T on it (clusters up to 16).
// 3. Newton-Schulz orthonormalisation Z <- Z (3 I - Z^T Z) / 2, twice: the
//    vectors of separated eigenvalues are orthogonal to eps |T| / gap, and
//    the rotation that removes that moves each residual by about eps |T|.
// 4. U = Q Z with Q = H_0 ... H_{m-2} from gwb_sytrd, applied in blocks of
//    256 reflectors as I - V T V^T (compact WY; Schreiber & Van Loan, SIAM J.
//    Sci. Stat. Comput. 10 (1989) 53): two GEMMs and a triangular solve with
//    T^-1 per block.

constexpr int TE_BW = 8;      // warps per block of the multisection
constexpr int TE_CLMAX = 16;  // largest cluster rotated by the Rayleigh-Ritz step
constexpr int TE_WYB = 256;   // reflectors per back-transform block

__global__ void k_tri_bounds(int m, const double* __restrict__ d, const double* __restrict__ e,
                             double* __restrict__ bounds) {
  __shared__ double slo[8], shi[8];
  double lo = INFINITY, hi = -INFINITY;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < m - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    slo[threadIdx.x >> 5] = lo;
    shi[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      lo = fmin(lo, slo[w]);
      hi = fmax(hi, shi[w]);
    }
    lo = fmin(lo, slo[0]);
    hi = fmax(hi, shi[0]);
    const double tn = fmax(fabs(lo), fabs(hi));
    const double pad = 1e-12 * tn + 1e-300;
    bounds[0] = lo - pad;
    bounds[1] = hi + pad;
    bounds[2] = tn;
  }
}

__global__ void __launch_bounds__(TE_BW * 32) k_tri_bisect(int m, int nev, const double* __restrict__ d,
                                                          const double* __restrict__ e,
                                                          const double* __restrict__ bounds, double* __restrict__ w) {
  extern __shared__ double te_smem[];
  double* sd = te_smem;
  double* se2 = te_smem + m;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    sd[i] = d[i];
    if (i < m - 1) se2[i] = e[i] * e[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int idx = blockIdx.x * TE_BW + (threadIdx.x >> 5);
  if (idx >= nev) return;
  double lo = bounds[0], hi = bounds[1];
  for (int round = 0; round < 48; ++round) {
    if (hi - lo <= 4.4e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300) break;
    const double x = lo + (hi - lo) * (double)(lane + 1) / 33.0;
    const int cnt = sturm_count(sd, se2, m, x);
    const unsigned le = __ballot_sync(0xffffffffu, cnt <= idx);
    const double x_lo = le ? __shfl_sync(0xffffffffu, x, 31 - __clz(le)) : lo;
    const int up = le ? 32 - __clz(le) : 0;  // first lane above the eigenvalue
    const double x_hi = up < 32 ? __shfl_sync(0xffffffffu, x, up & 31) : hi;
    lo = x_lo;
    hi = x_hi;
  }
  if (lane == 0) w[idx] = 0.5 * (lo + hi);
}

// Factors of T - lam I for one vector: per row r, 1 / u0, u1, u2 (the row
// of U), l (the multiplier) and the interchange flag, at F[5 r + q] (each
// vector's factors contiguous: one thread walks them in order).
__device__ void tri_factor(int m, const double* __restrict__ d, const double* __restrict__ e, double lam,
                           double pivmin, double* __restrict__ F) {
  double c0 = d[0] - lam, c1 = m > 1 ? e[0] : 0.0, c2 = 0.0;
  for (int r = 0; r < m - 1; ++r) {
    const double er = e[r];
    const double dn = d[r + 1] - lam, en = r + 1 < m - 1 ? e[r + 1] : 0.0;
    double u0, u1, u2, l, sw;
    if (fabs(c0) >= fabs(er)) {
      if (c0 == 0.0) c0 = pivmin;
      u0 = c0;
      u1 = c1;
      u2 = c2;
      l = er / c0;
      sw = 0.0;
      c0 = dn - l * c1;
      c1 = en - l * c2;
      c2 = 0.0;
    } else {
      u0 = er;
      u1 = dn;
      u2 = en;
      l = c0 / er;
      sw = 1.0;
      const double n0 = c1 - l * dn, n1 = c2 - l * en;
      c0 = n0;
      c1 = n1;
      c2 = 0.0;
    }
    double* f = F + (int64_t)5 * r;
    f[0] = 1.0 / u0;
    f[1] = u1;
    f[2] = u2;
    f[3] = l;
    f[4] = sw;
  }
  if (fabs(c0) < pivmin) c0 = c0 < 0.0 ? -pivmin : pivmin;
  double* f = F + (int64_t)5 * (m - 1);
  f[0] = 1.0 / c0;
  f[1] = 0.0;
  f[2] = 0.0;
  f[3] = 0.0;
  f[4] = 0.0;
}

// z <- (T - lam I)^-1 z with the stored factors, in place (z contiguous).
__device__ void tri_solve(int m, const double* __restrict__ F, double* __restrict__ z) {
  double carry = z[0];
#pragma unroll 8
  for (int r = 0; r < m - 1; ++r) {
    const double* f = F + (int64_t)5 * r;
    const double l = f[3], sw = f[4];
    const double nxt = z[r + 1];
    if (sw != 0.0) {
      z[r] = nxt;
      carry = carry - l * nxt;
    } else {
      z[r] = carry;
      carry = nxt - l * carry;
    }
  }
  z[m - 1] = carry;
  double z1 = 0.0, z2 = 0.0;  // z[r + 1], z[r + 2]
#pragma unroll 8
  for (int r = m - 1; r >= 0; --r) {
    const double* f = F + (int64_t)5 * r;
    const double v = (z[r] - f[1] * z1 - f[2] * z2) * f[0];
    z[r] = v;
    z2 = z1;
    z1 = v;
  }
}

// Dot product of two contiguous vectors by a warp (lanes stride the rows,
// then a fixed-order shuffle tree; every lane gets the sum).
__device__ double warp_dot(int m, const double* __restrict__ a, const double* __restrict__ b, int lane) {
  double s = 0.0;
  for (int r = lane; r < m; r += 32) s += a[r] * b[r];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

constexpr int TE_IW = 1;  // warps per block of the inverse iteration

// Eigenvectors of T into Z (m x nev, column-major: vector k at Z + k m);
// eigenvalues into wout (the cluster Rayleigh-Ritz refines those of
// clusters). One warp (block) per eigenvalue, with the factors of T - lambda I
// and the vector being iterated in shared memory (6 m doubles): lane 0 runs
// the factor and the solves (sequential recurrences), the warp the starts,
// the orthogonalisation against earlier cluster members, the norms and the
// cluster Rayleigh-Ritz.
__global__ void __launch_bounds__(TE_IW * 32) k_tri_invit(int m, int nev, const double* __restrict__ d,
                                                          const double* __restrict__ e, const double* __restrict__ w,
                                                          const double* __restrict__ bounds, double* __restrict__ Z,
                                                          double* __restrict__ wout) {
  extern __shared__ double iv_smem[];
  double* Fs = iv_smem;          // 5 m
  double* zs = iv_smem + 5 * m;  // m
  __shared__ double Hs[TE_IW][TE_CLMAX][TE_CLMAX + 1];
  __shared__ double Rs[TE_IW][TE_CLMAX][TE_CLMAX + 1];
  __shared__ int ords[TE_IW][TE_CLMAX];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * TE_IW + wib;
  if (i >= nev) return;
  const double tn = fmax(bounds[2], 1e-300);
  const double ctol = 1e-9 * tn;
  const double pivmin = 2.2e-16 * tn;
  if (i > 0 && w[i] - w[i - 1] <= ctol) return;  // a later member of a cluster
  int end = i + 1;
  while (end < nev && w[end] - w[end - 1] <= ctol) ++end;
  for (int k = i; k < end; ++k) {
    double* z = Z + (int64_t)k * m;
    if (lane == 0) tri_factor(m, d, e, w[k], pivmin, Fs);
    for (int r = lane; r < m; r += 32) zs[r] = hash_pm1(((unsigned long long)(k + 1) << 32) ^ (unsigned long long)r);
    __syncwarp();
    for (int it = 0; it < 3; ++it) {
      if (lane == 0) tri_solve(m, Fs, zs);
      __syncwarp();
      for (int pass = 0; pass < 2; ++pass) {
        for (int c = i; c < k; ++c) {
          const double* zc = Z + (int64_t)c * m;
          const double dt = warp_dot(m, zs, zc, lane);
          for (int r = lane; r < m; r += 32) zs[r] -= dt * zc[r];
          __syncwarp();
        }
      }
      const double nrm = sqrt(warp_dot(m, zs, zs, lane));
      const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
      for (int r = lane; r < m; r += 32) zs[r] *= inv;
      __syncwarp();
    }
    for (int r = lane; r < m; r += 32) z[r] = zs[r];
    __syncwarp();
  }
  const int nc = end - i;
  if (nc < 2 || nc > TE_CLMAX) {
    for (int k = i + lane; k < end; k += 32) wout[k] = w[k];
    return;
  }
  // Rayleigh-Ritz of T on the cluster: H = Z_c^T T Z_c, cyclic Jacobi (lane 0)
  double (*H)[TE_CLMAX + 1] = Hs[wib];
  double (*R)[TE_CLMAX + 1] = Rs[wib];
  int* ord = ords[wib];
  for (int p = 0; p < nc; ++p) {
    const double* zp = Z + (int64_t)(i + p) * m;
    for (int q = p; q < nc; ++q) {
      const double* zq = Z + (int64_t)(i + q) * m;
      double s = 0.0;
      for (int r = lane; r < m; r += 32) {
        double tz = d[r] * zq[r];
        if (r > 0) tz += e[r - 1] * zq[r - 1];
        if (r < m - 1) tz += e[r] * zq[r + 1];
        s += zp[r] * tz;
      }
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) H[p][q] = H[q][p] = s;
    }
  }
  if (lane == 0) {
    for (int p = 0; p < nc; ++p)
      for (int q = 0; q < nc; ++q) R[p][q] = p == q ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 12; ++sweep) {
      double off = 0.0;
      for (int p = 0; p < nc; ++p)
        for (int q = p + 1; q < nc; ++q) off = fmax(off, fabs(H[p][q]));
      if (off <= 1e-17 * tn) break;
      for (int p = 0; p < nc; ++p)
        for (int q = p + 1; q < nc; ++q) {
          if (fabs(H[p][q]) <= 1e-18 * tn) continue;
          // rotation zeroing H[p][q] (Golub & Van Loan sec. 8.5.2)
          const double th = (H[q][q] - H[p][p]) / (2.0 * H[p][q]);
          const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
          const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
          for (int k = 0; k < nc; ++k) {
            const double hp = H[k][p], hq = H[k][q];
            H[k][p] = c * hp - sn * hq;
            H[k][q] = sn * hp + c * hq;
          }
          for (int k = 0; k < nc; ++k) {
            const double hp = H[p][k], hq = H[q][k];
            H[p][k] = c * hp - sn * hq;
            H[q][k] = sn * hp + c * hq;
          }
          for (int k = 0; k < nc; ++k) {
            const double rp = R[k][p], rq = R[k][q];
            R[k][p] = c * rp - sn * rq;
            R[k][q] = sn * rp + c * rq;
          }
        }
    }
    // ascending order of the cluster's Ritz values
    for (int p = 0; p < nc; ++p) ord[p] = p;
    for (int p = 1; p < nc; ++p)
      for (int q = p; q > 0 && H[ord[q]][ord[q]] < H[ord[q - 1]][ord[q - 1]]; --q) {
        const int t = ord[q];
        ord[q] = ord[q - 1];
        ord[q - 1] = t;
      }
    for (int p = 0; p < nc; ++p) wout[i + p] = H[ord[p]][ord[p]];
  }
  __syncwarp();
  // Z_c <- Z_c R (ordered), a row per lane
  for (int r = lane; r < m; r += 32) {
    double zr[TE_CLMAX], out[TE_CLMAX];
    for (int p = 0; p < nc; ++p) zr[p] = Z[r + (int64_t)(i + p) * m];
    for (int q = 0; q < nc; ++q) {
      double s = 0.0;
      for (int p = 0; p < nc; ++p) s += zr[p] * R[p][ord[q]];
      out[q] = s;
    }
    for (int q = 0; q < nc; ++q) Z[r + (int64_t)(i + q) * m] = out[q];
  }
}

// M = (3 I - G) / 2 for the Newton-Schulz step (n x n, column-major).
__global__ void k_ns_matrix(int n, const double* __restrict__ G, double* __restrict__ M) {
  const int64_t total = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(t % n), c = (int)(t / n);
    M[t] = (r == c ? 1.5 : 0.0) - 0.5 * G[t];
  }
}

// Vb (rows j0 + 1 .. m - 1, kb columns, column-major with leading dimension
// mb = m - j0 - 1): reflector j0 + c is 1 at row j0 + c + 1, A's stored
// vector below it, zero above.
__global__ void k_wy_build(int m, int j0, int kb, const double* __restrict__ A, int64_t lda,
                           const double* __restrict__ tau, double* __restrict__ Vb) {
  const int mb = m - j0 - 1;
  const int64_t total = (int64_t)mb * kb;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int rr = (int)(t % mb), c = (int)(t / mb);
    const int r = j0 + 1 + rr, j = j0 + c;
    double v = 0.0;
    if (tau[j] != 0.0) {  // a reflector with tau = 0 is the identity: a zero column
      if (r == j + 1) v = 1.0;
      else if (r > j + 1) v = A[r + (int64_t)j * lda];
    }
    Vb[t] = v;
  }
}

// T^-1 of the block's compact WY form, in place of its Gram G = Vb^T Vb
// (kb x kb, column-major): T^-1 = diag(1 / tau) + the strictly upper part of
// G (Puglisi, SIAM J. Matrix Anal. Appl. 13 (1992) 723; Joffrain et al.,
// ACM TOMS 32 (2006) 169). A Householder tau lies in [1, 2] or is 0; a
// reflector with tau = 0 has a zero column and a unit diagonal here.
__global__ void k_wy_tinv(int kb, const double* __restrict__ tau, double* __restrict__ G) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < kb * kb; t += gridDim.x * blockDim.x) {
    const int r = t % kb, c = t / kb;
    if (r > c) G[t] = 0.0;
    else if (r == c) G[t] = tau[c] != 0.0 ? 1.0 / tau[c] : 1.0;
  }
}

int blas_call(cublasStatus_t s, const char* what) {
  if (s != CUBLAS_STATUS_SUCCESS) {
    set_error(std::string(what) + " failed with status " + std::to_string((int)s));
    return GWB_ERR_CUDA;
  }
  return GWB_OK;
}

struct SyLayout {
  size_t trd, d, e, tau, bounds, wbis, G, M, Zt, Vb, Gb, W1, total;
};

SyLayout sy_layout(int m, int nev, size_t trd_bytes) {
  SyLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  L.trd = take(trd_bytes);
  L.d = take((size_t)m * 8);
  L.e = take((size_t)m * 8);
  L.tau = take((size_t)m * 8);
  L.bounds = take(4 * 8);
  L.wbis = take((size_t)nev * 8);
  L.G = take((size_t)nev * nev * 8);
  L.M = take((size_t)nev * nev * 8);
  L.Zt = take((size_t)m * nev * 8);
  L.Vb = take((size_t)m * TE_WYB * 8);
  L.Gb = take((size_t)TE_WYB * TE_WYB * 8);
  L.W1 = take((size_t)TE_WYB * nev * 8);
  L.total = off;
  return L;
}

}  // namespace
}  // namespace gwb

using namespace gwb;

static int g_sytrd_blocks = 0;
static long long* g_sytrd_trace = nullptr;
static int g_sytrd_cluster = -1;  // cluster size of the trailing part: -1 largest that fits, 0 none

extern "C" int gwb_sytrd_set_cluster(int32_t size) {
  GWB_REQUIRE(size == -1 || size == 0 || size == 8 || size == 16, "cluster size must be -1, 0, 8 or 16");
  g_sytrd_cluster = size;
  return GWB_OK;
}

namespace {
// The cluster kernel's size on this device: the cluster size and the largest
// trailing part that fits its distributed shared memory (0, 0: none).
struct TkChoice {
  int cs, nmax;
};

template <int CS>
int tk_try(int dev, TkChoice* out) {
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, k_sytrd_cluster<CS>) != cudaSuccess) return 0;
  int nmax = 0;
  for (int n = TK_NSEG * TK_SEG; n >= 2; --n)
    if (tk_smem_doubles(n, CS) * 8 + fa.sharedSizeBytes <= (size_t)optin) {
      nmax = n;
      break;
    }
  if (nmax < 2) return 0;
  const int bytes = (int)(tk_smem_doubles(nmax, CS) * 8);
  if (cudaFuncSetAttribute(k_sytrd_cluster<CS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
    return 0;
  if (CS > 8 && cudaFuncSetAttribute(k_sytrd_cluster<CS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                    cudaSuccess)
    return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CS);
  cfg.blockDim = dim3(TK_THREADS);
  cfg.dynamicSmemBytes = bytes;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int nc = 0;
  if (cudaOccupancyMaxActiveClusters(&nc, k_sytrd_cluster<CS>, &cfg) != cudaSuccess || nc < 1) {
    cudaGetLastError();
    return 0;
  }
  *out = TkChoice{CS, nmax};
  return 1;
}

TkChoice tk_choice(int dev, int want) {
  static std::mutex mu;
  static TkChoice cache[64][3];
  static bool done[64][3];
  const int slot = want == 8 ? 1 : (want == 16 ? 2 : 0);
  std::lock_guard<std::mutex> g(mu);
  if (dev < 0 || dev >= 64) return TkChoice{0, 0};
  if (!done[dev][slot]) {
    TkChoice ch{0, 0};
    if (want != 8 && tk_try<16>(dev, &ch)) {
    } else if (want != 16) {
      tk_try<8>(dev, &ch);
    }
    cache[dev][slot] = ch;
    done[dev][slot] = true;
  }
  return cache[dev][slot];
}
}  // namespace

// the shared-memory-resident grid part: 0 off (the default: measured no
// faster than the cooperative launch, ~11 us per column), 1 on
static int g_sytrd_grid = 0;

extern "C" int gwb_sytrd_set_grid(int32_t on) {
  GWB_REQUIRE(on == 0 || on == 1, "on must be 0 or 1");
  g_sytrd_grid = on;
  return GWB_OK;
}

namespace {
// The largest trailing part the grid kernel holds with one CTA per SM (0: none).
int tg_nmax(int dev, int sms) {
  static std::mutex mu;
  static int cache[64];
  static bool done[64];
  std::lock_guard<std::mutex> g(mu);
  if (dev < 0 || dev >= 64) return 0;
  if (!done[dev]) {
    int nmax = 0, optin = 0;
    cudaFuncAttributes fa{};
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess &&
        cudaFuncGetAttributes(&fa, k_sytrd_grid) == cudaSuccess) {
      for (int n = TG_NSEG * TK_SEG; n >= 2; --n)
        if (tg_smem_doubles(n, sms) * 8 + fa.sharedSizeBytes <= (size_t)optin) {
          nmax = n;
          break;
        }
      int per_sm = 0;
      if (nmax >= 2 &&
          (cudaFuncSetAttribute(k_sytrd_grid, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(tg_smem_doubles(nmax, sms) * 8)) != cudaSuccess ||
           cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sytrd_grid, TK_THREADS,
                                                         tg_smem_doubles(nmax, sms) * 8) != cudaSuccess ||
           per_sm < 1)) {
        cudaGetLastError();
        nmax = 0;
      }
    }
    cache[dev] = nmax;
    done[dev] = true;
  }
  return cache[dev];
}

// Where gwb_sytrd hands over: columns [0, k1) in the cooperative launch,
// [k1, k2) in the grid kernel, [k2, m - 1) in the cluster.
struct SyPlan {
  int k1, k2;
  TkChoice ch;
};

SyPlan sy_plan(int m, int dev, int sms) {
  SyPlan p{m, m, TkChoice{0, 0}};
  if (m <= 1) return p;
  p.ch = g_sytrd_cluster != 0 ? tk_choice(dev, g_sytrd_cluster) : TkChoice{0, 0};
  const int gmax = g_sytrd_grid ? tg_nmax(dev, sms) : 0;
  // the cluster's first column: the trailing part fits its shared memory
  const int kc = p.ch.cs > 0 ? std::max(0, m - p.ch.nmax) : m - 1;
  if (gmax >= 2 && kc > 0) {
    p.k1 = m <= gmax ? 0 : (m - gmax + TD_NB - 1) / TD_NB * TD_NB;
    p.k2 = std::max(p.k1, kc);
    if (p.k2 == p.k1 && p.ch.cs == 0) p.k2 = m - 1;
  } else if (p.ch.cs > 0) {
    p.k1 = p.k2 = m <= p.ch.nmax ? 0 : (m - p.ch.nmax + TD_NB - 1) / TD_NB * TD_NB;
  }
  if (p.k1 >= m - 1) p.k1 = p.k2 = m;  // all in the cooperative launch
  return p;
}
}  // namespace

extern "C" int32_t gwb_sytrd_cluster_rows(int32_t m) {
  int dev = 0;
  if (m <= 1 || g_sytrd_cluster == 0 || cudaGetDevice(&dev) != cudaSuccess) return 0;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  const SyPlan p = sy_plan(m, dev, sms);
  return p.k2 < m - 1 ? m - p.k2 : 0;
}


extern "C" int gwb_sytrd_set_trace(long long* cycles10) {
  g_sytrd_trace = cycles10;
  return GWB_OK;
}

extern "C" int gwb_sytrd_set_blocks(int32_t blocks) {
  GWB_REQUIRE(blocks >= 0, "blocks must be >= 0");
  g_sytrd_blocks = blocks;
  return GWB_OK;
}

static size_t sytrd_need(int m, int sms) {
  return (size_t)(2 * TD_NB * (size_t)m + 2 * (size_t)m + (size_t)sms * (1 + TD_NCOMP)) * 8 + 256;
}

extern "C" size_t gwb_sytrd_work_bytes(int32_t m) {
  if (m <= 0) return 0;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                cudaSuccess || sms <= 0)
    sms = 1024;  // no device: an upper bound
  return sytrd_need(m, sms);
}

extern "C" int gwb_sytrd(int32_t m, double* A, int64_t lda, double* d, double* e, double* tau, void* work,
                         size_t work_bytes, int* status, void* stream) {
  GWB_REQUIRE(m >= 1 && m <= TD_MMAX, "m must be in 1..4096");
  GWB_REQUIRE(lda >= m, "lda < m");
  GWB_REQUIRE(A && d && e && tau && work && status, "null pointer");
  int dev = 0, sms = 0, coop = 0;
  GWB_CUDA_TRY(cudaGetDevice(&dev));
  GWB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GWB_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  GWB_REQUIRE(coop, "the device does not support cooperative launches");
  const size_t need = sytrd_need(m, sms);
  GWB_REQUIRE(work_bytes >= need, "workspace smaller than gwb_sytrd_work_bytes");
  cudaStream_t st = (cudaStream_t)stream;
  auto* w = static_cast<double*>(work);
  // blocks of the cooperative launch: one per SM, or fewer (a cheaper grid
  // barrier against less bandwidth for the products; gwb_sytrd_set_blocks)
  const int nblk = std::max((m + TD_THREADS - 1) / TD_THREADS, g_sytrd_blocks > 0 ? std::min(g_sytrd_blocks, sms) : sms);
  // whole panels in the cooperative launch until the trailing part fits the
  // shared memory of all SMs, then the grid kernel until it fits one
  // cluster's, then the cluster
  const SyPlan plan = sy_plan(m, dev, sms);
  const TkChoice ch = plan.ch;
  const int kend = plan.k1;
  if (m > 1) GWB_CUDA_TRY(cudaMemsetAsync(tau + (m - 1), 0, sizeof(double), st));
  if (plan.k2 < m - 1) {
    GWB_REQUIRE(ch.cs > 0 && m - plan.k2 <= ch.nmax, "internal: trailing part larger than the cluster holds");
  }
  TdArgs args;
  args.m = m;
  args.kend = kend;
  args.A = A;
  args.lda = lda;
  args.d = d;
  args.e = e;
  args.tau = tau;
  args.V = w;
  args.W = w + (size_t)TD_NB * m;
  args.acol = w + 2 * (size_t)TD_NB * m;
  args.ycol = args.acol + m;
  args.part1 = args.ycol + m;
  args.part2 = args.part1 + sms;
  args.bar = reinterpret_cast<unsigned*>(args.part2 + (size_t)sms * TD_NCOMP);
  args.status = status;
  args.wait_cycles = tc_wait_cycles();
  args.trace = g_sytrd_trace;
  if (kend > 0) {
    // V and W start at zero (entries above a reflector's row are read as zeros)
    GWB_CUDA_TRY(cudaMemsetAsync(w, 0, need, st));
    const size_t smem = (size_t)std::max(m, TD_WARPS * 2 * 32 * TD_NB) * 8;
    GWB_CUDA_TRY(cudaFuncSetAttribute(k_sytrd_coop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    void* kargs[] = {&args};
    GWB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_sytrd_coop, dim3(nblk), dim3(TD_THREADS), kargs, smem, st));
    count_launches(1);
  }
  if (plan.k2 > plan.k1) {
    GWB_REQUIRE(m - plan.k1 <= tg_nmax(dev, sms), "internal: trailing part larger than the grid holds");
    TgArgs ga;
    ga.m = m;
    ga.t0 = plan.k1;
    ga.t1 = plan.k2;
    ga.A = A;
    ga.lda = lda;
    ga.d = d;
    ga.e = e;
    ga.tau = tau;
    ga.pr = reinterpret_cast<double2*>(w);  // the cooperative launch's panel vectors, free by now
    ga.part = w + 4 * (size_t)m;
    ga.bar = args.bar;
    ga.status = status;
    ga.wait_cycles = args.wait_cycles;
    const size_t smem = tg_smem_doubles(m - plan.k1, sms) * 8;
    // the barrier counter starts at zero (its low bits are the arrival count)
    GWB_CUDA_TRY(cudaMemsetAsync(args.bar, 0, sizeof(unsigned), st));
    void* kargs[] = {&ga};
    GWB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_sytrd_grid, dim3(sms), dim3(TK_THREADS), kargs, smem, st));
    count_launches(1);
  }
  if (plan.k2 < m - 1) {
    const int kend2 = plan.k2;
    TkArgs ta{m, kend2, A, lda, d, e, tau, g_sytrd_trace ? g_sytrd_trace + 6 : nullptr};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ch.cs);
    cfg.blockDim = dim3(TK_THREADS);
    cfg.dynamicSmemBytes = tk_smem_doubles(m - kend2, ch.cs) * 8;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = ch.cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (ch.cs == 16) GWB_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_sytrd_cluster<16>, ta));
    else GWB_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_sytrd_cluster<8>, ta));
    count_launches(1);
  }
  return GWB_OK;
}

namespace gwb {
int blas_handle(cublasHandle_t* out);
}

extern "C" size_t gwb_sy_lowest_work_bytes(int32_t m, int32_t nev) {
  if (m <= 0 || nev <= 0) return 0;
  return sy_layout(m, nev, gwb_sytrd_work_bytes(m)).total;
}

extern "C" int gwb_sy_lowest(int32_t m, int32_t nev, double* A, int64_t lda, double* w, double* U, int64_t ldu,
                             void* work, size_t work_bytes, int* status, void* stream) {
  GWB_REQUIRE(m >= 1 && m <= TD_MMAX && nev >= 1 && nev <= m, "need 1 <= nev <= m <= 4096");
  GWB_REQUIRE(lda >= m && ldu >= m, "leading dimension < m");
  GWB_REQUIRE(A && w && U && work && status, "null pointer");
  const size_t trd = gwb_sytrd_work_bytes(m);
  const SyLayout L = sy_layout(m, nev, trd);
  GWB_REQUIRE(work_bytes >= L.total, "workspace smaller than gwb_sy_lowest_work_bytes");
  cudaStream_t st = (cudaStream_t)stream;
  char* wb = static_cast<char*>(work);
  auto P = [&](size_t off) { return reinterpret_cast<double*>(wb + off); };
  double *d = P(L.d), *e = P(L.e), *tau = P(L.tau), *bounds = P(L.bounds), *wbis = P(L.wbis);
  double *G = P(L.G), *M = P(L.M), *Zt = P(L.Zt), *Vb = P(L.Vb), *Gb = P(L.Gb), *W1 = P(L.W1);
  int rc = gwb_sytrd(m, A, lda, d, e, tau, wb + L.trd, trd, status, stream);
  if (rc != GWB_OK) return rc;
  if (m == 1) {
    GWB_CUDA_TRY(cudaMemcpyAsync(w, d, 8, cudaMemcpyDeviceToDevice, st));
    const double one = 1.0;
    GWB_CUDA_TRY(cudaMemcpyAsync(U, &one, 8, cudaMemcpyHostToDevice, st));
    return GWB_OK;
  }
  k_tri_bounds<<<1, 256, 0, st>>>(m, d, e, bounds);
  const size_t smb = (size_t)2 * m * 8;
  GWB_CUDA_TRY(cudaFuncSetAttribute(k_tri_bisect, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb));
  k_tri_bisect<<<(nev + TE_BW - 1) / TE_BW, TE_BW * 32, smb, st>>>(m, nev, d, e, bounds, wbis);
  const size_t smi = (size_t)6 * m * 8;
  GWB_CUDA_TRY(cudaFuncSetAttribute(k_tri_invit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smi));
  k_tri_invit<<<(nev + TE_IW - 1) / TE_IW, TE_IW * 32, smi, st>>>(m, nev, d, e, wbis, bounds, Zt, w);
  GWB_LAUNCH_CHECK();
  count_launches(3);
  cublasHandle_t h;
  rc = blas_handle(&h);
  if (rc) return rc;
  if ((rc = blas_call(cublasSetStream(h, st), "cublasSetStream"))) return rc;
  const double one = 1.0, zero = 0.0, mone = -1.0;
  // Newton-Schulz: G = Z^T Z, M = (3 I - G) / 2, Z <- Z M (twice). The
  // first pass reads Z (column-major, ld m) and writes U; the second works
  // on U.
  const int gblk = (int)std::min<int64_t>(((int64_t)nev * nev + 255) / 256, 1024);
  if ((rc = blas_call(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, nev, nev, m, &one, Zt, m, Zt, m, &zero, G, nev),
                      "cublasDgemm")))
    return rc;
  k_ns_matrix<<<gblk, 256, 0, st>>>(nev, G, M);
  if ((rc = blas_call(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, nev, nev, &one, Zt, m, M, nev, &zero, U, (int)ldu),
                      "cublasDgemm")))
    return rc;
  if ((rc = blas_call(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, nev, nev, m, &one, U, (int)ldu, U, (int)ldu, &zero, G,
                                  nev), "cublasDgemm")))
    return rc;
  k_ns_matrix<<<gblk, 256, 0, st>>>(nev, G, M);
  if ((rc = blas_call(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, nev, nev, &one, U, (int)ldu, M, nev, &zero, Zt, m),
                      "cublasDgemm")))
    return rc;
  GWB_CUDA_TRY(cudaMemcpy2DAsync(U, ldu * 8, Zt, (size_t)m * 8, (size_t)m * 8, nev, cudaMemcpyDeviceToDevice, st));
  // U = Q Z: blocks of reflectors from the last to the first, each as
  // U <- U - Vb (T (Vb^T U)) with T applied by a triangular solve with T^-1
  for (int j1 = m - 1; j1 > 0;) {
    const int j0 = std::max(0, j1 - TE_WYB);
    const int kb = j1 - j0, mb = m - j0 - 1;
    k_wy_build<<<(int)std::min<int64_t>(((int64_t)mb * kb + 255) / 256, 2048), 256, 0, st>>>(m, j0, kb, A, lda,
                                                                                             tau, Vb);
    if ((rc = blas_call(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, kb, kb, mb, &one, Vb, mb, Vb, mb, &zero, Gb, kb),
                        "cublasDgemm")))
      return rc;
    k_wy_tinv<<<(kb * kb + 255) / 256, 256, 0, st>>>(kb, tau + j0, Gb);
    double* Us = U + (j0 + 1);
    if ((rc = blas_call(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, kb, nev, mb, &one, Vb, mb, Us, (int)ldu, &zero, W1,
                                    kb), "cublasDgemm")))
      return rc;
    if ((rc = blas_call(cublasDtrsm(h, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                                    kb, nev, &one, Gb, kb, W1, kb), "cublasDtrsm")))
      return rc;
    if ((rc = blas_call(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, mb, nev, kb, &mone, Vb, mb, W1, kb, &one, Us,
                                    (int)ldu), "cublasDgemm")))
      return rc;
    GWB_LAUNCH_CHECK();
    count_launches(3);
    j1 = j0;
  }
  return GWB_OK;
}
