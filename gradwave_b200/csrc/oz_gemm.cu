// Float64-accurate real products on the int8 tensor cores (tcgen05
// kind::i8): the Ozaki scheme, first form (Ozaki, Ogita, Oishi, Rump 2012;
// Ootomo, Ozaki, Yokota 2024 for integer tensor cores).
//
// Splitting. Every row of an operand is scaled by a power of two sigma above
// its largest magnitude, so |x / sigma| < 1, and cut into S signed slices by
// repeated rounding to nearest: t = 64 x / sigma; for p = 1..S: q_p = rint(t)
// in [-64, 64], t = 128 (t - q_p). Then x = sigma sum_p q_p 2^(1-7p) to
// within 2^-7S sigma, every step exact in float64. Rounding (not truncation)
// leaves errors of either sign, so they do not add up coherently in sums such
// as the diagonal of a Gram matrix. A slice set holds the S int8 planes of
// rows_cap x ldk (ldk a multiple of 64, columns K..ldk-1 zero), plane p at
// p rows_cap ldk, and the per-row scales.
//
// Product. C = alpha diag(sa) (sum_{i+j <= S+1} 2^(2-7(i+j)) A_i B_j^T)
// diag(sb) + beta C for slice sets A (M x K) and B (N x K): every A_i B_j^T
// is an exact int8 product with int32 accumulation, the pairs of one level
// L = i + j share an int32 accumulator in tensor memory, and the levels are
// added into float64 registers once per K chunk of 32768 (S x 32768 x 64^2 <
// 2^31 for S <= 8, so no int32 sum can overflow). The pairs with
// i + j > S + 1 lie below the error of the kept ones and are not formed:
// S(S+1)/2 int8 products per float64 product. The error of an element is
// about 2^-7S of the rows' scales times sqrt(K): with S = 8 the level of a
// float64 GEMM of the same shape.
//
// A product C = A B with B held as K x N rows (the Davidson updates
// D -= C V and the Ritz vectors X = U^T V) uses B's slices transposed
// (gwb_oz_split_cols: N rows of length K, scaled per K row of the source),
// with those per-K scales folded into A's rows before A is split
// (gwb_oz_split_rows with fold).
//
// CTA: 192 threads for a 128 x 64 tile of C. Warp 0 lane 0 loads both slice
// tiles of a 64-wide K step (all S planes, one 3-D TMA box each, 64-byte
// swizzle) into a 2-stage ring; warp 1 lane 0 issues the S(S+1) tcgen05.mma
// (M 128, N 64, K 32) of a step and commits them; warps 2-5 drain the S level
// accumulators (512 TMEM columns) into float64 after each chunk, then stage
// the tile through shared memory and write whole rows of C. Every mbarrier
// wait is bounded (gwb_tc_set_wait_limit); a wait that runs out ORs
// GWB_ERR_TIMEOUT into *status, the producer waits for the copies it issued,
// and the TMEM is always released.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "tcgen05.cuh"

namespace gwb {
namespace {

constexpr int OZ_M = 128;
constexpr int OZ_N = 64;
constexpr int OZ_KS = 64;                    // K elements (bytes) per stage: one 64-byte swizzle row
constexpr int OZ_STAGES = 2;
constexpr int OZ_CHUNK_STEPS = 32768 / OZ_KS;  // stages per int32 accumulation chunk
constexpr int OZ_THREADS = 192;
constexpr int OZ_TMEM_COLS = 512;
constexpr int OZ_SROW = OZ_N + 1;            // staging row (doubles), padded

template <int S> struct OzShape {
  static constexpr int A_BYTES = S * OZ_M * OZ_KS;
  static constexpr int B_BYTES = S * OZ_N * OZ_KS;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int SMEM = OZ_STAGES * STAGE + 1024;
  static_assert(S * OZ_N <= OZ_TMEM_COLS, "levels exceed tensor memory");
  static_assert(OZ_M * OZ_SROW * 8 <= OZ_STAGES * STAGE, "output staging exceeds the pipeline buffers");
};

// kind::i8 instruction descriptor: D s32, A and B s8, both K-major, M 128, N 64.
constexpr uint32_t OZ_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OZ_N >> 3) << 17) |
                              ((uint32_t)(OZ_M >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(OZ_IDESC), "r"(accumulate)
      : "memory");
}

struct OzOut {
  double* C;       // direct: C[i ldc + j]; split: partial slice blockIdx.y of a (splits, M, N) array
  int64_t ldc;
  double alpha, beta;
  int split;
};

template <int S>
__global__ void __launch_bounds__(OZ_THREADS, 1)
    k_oz_gemm(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int M, int N,
              int K, int a_row0, int b_row0, int steps_per_split, OzOut out, const double* __restrict__ sa,
              const double* __restrict__ sb, int* status, long long wait_cycles) {
  using Sh = OzShape<S>;
  __shared__ __align__(8) uint64_t bar_full[OZ_STAGES];
  __shared__ __align__(8) uint64_t bar_empty[OZ_STAGES];
  __shared__ __align__(8) uint64_t bar_acc;   // the MMAs of a chunk have completed
  __shared__ __align__(8) uint64_t bar_free;  // the drain of a chunk has read the accumulators
  __shared__ uint32_t tmem_base_slot;
  __shared__ int abort_flag;
  extern __shared__ uint8_t dsm_raw[];
  const uint32_t dsm = (smem_u32(dsm_raw) + 1023u) & ~1023u;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Mt = (M + OZ_M - 1) / OZ_M;
  const int mt = blockIdx.x % Mt, nt = blockIdx.x / Mt;
  const int m0 = mt * OZ_M, n0 = nt * OZ_N;
  const int nsteps_all = (K + OZ_KS - 1) / OZ_KS;
  const int ks0 = blockIdx.y * steps_per_split;
  const int nsteps = max(0, min(nsteps_all, ks0 + steps_per_split) - ks0);
  const int nchunks = (nsteps + OZ_CHUNK_STEPS - 1) / OZ_CHUNK_STEPS;

  if (tid == 0) {
    for (int s = 0; s < OZ_STAGES; ++s) {
      mbar_init(smem_u32(&bar_full[s]), 1);
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    mbar_init(smem_u32(&bar_acc), 1);
    mbar_init(smem_u32(&bar_free), 128);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                 "r"((uint32_t)OZ_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_slot;

  double acc[OZ_N];
#pragma unroll
  for (int j = 0; j < OZ_N; ++j) acc[j] = 0.0;
  bool drained_all = false;

  if (warp == 0 && lane == 0 && nsteps > 0) {
    // producer
    int last_round[OZ_STAGES];
#pragma unroll
    for (int s = 0; s < OZ_STAGES; ++s) last_round[s] = -1;
    for (int i = 0; i < nsteps; ++i) {
      const int s = i % OZ_STAGES;
      if (i >= OZ_STAGES && !mbar_wait(smem_u32(&bar_empty[s]), ((i / OZ_STAGES) - 1) & 1, wait_cycles)) {
        abort_flag = 1;
        atomicOr(status, GWB_ERR_TIMEOUT);
        break;
      }
      if (*(volatile int*)&abort_flag) break;
      last_round[s] = i / OZ_STAGES;
      const uint32_t full = smem_u32(&bar_full[s]);
      const uint32_t a_s = dsm + s * Sh::STAGE, b_s = a_s + Sh::A_BYTES;
      mbar_expect_tx(full, Sh::STAGE);
      const int k0 = (ks0 + i) * OZ_KS;
      tma_load_3d(a_s, &mapA, full, k0, a_row0 + m0, 0);
      tma_load_3d(b_s, &mapB, full, k0, b_row0 + n0, 0);
    }
    // every issued box must have landed before the CTA can leave (only this
    // thread arms the full barriers: a landed phase r keeps parity r complete)
#pragma unroll
    for (int s = 0; s < OZ_STAGES; ++s)
      if (last_round[s] >= 0 && !mbar_wait(smem_u32(&bar_full[s]), last_round[s] & 1, wait_cycles))
        atomicOr(status, GWB_ERR_TIMEOUT);
  } else if (warp == 1 && lane == 0 && nsteps > 0) {
    // MMA issuer
    bool stop = false;
    for (int c = 0; c < nchunks && !stop; ++c) {
      if (c > 0 && !mbar_wait(smem_u32(&bar_free), (c - 1) & 1, wait_cycles)) {
        abort_flag = 1;
        atomicOr(status, GWB_ERR_TIMEOUT);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int i0 = c * OZ_CHUNK_STEPS, i1 = min(nsteps, i0 + OZ_CHUNK_STEPS);
      for (int i = i0; i < i1; ++i) {
        const int s = i % OZ_STAGES;
        if (!mbar_wait(smem_u32(&bar_full[s]), (i / OZ_STAGES) & 1, wait_cycles)) {
          abort_flag = 1;
          atomicOr(status, GWB_ERR_TIMEOUT);
          stop = true;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_s = dsm + s * Sh::STAGE, b_s = a_s + Sh::A_BYTES;
#pragma unroll
        for (int kk = 0; kk < OZ_KS / 32; ++kk) {
#pragma unroll
          for (int p = 0; p < S; ++p) {
            const uint64_t da = sdesc(a_s + p * (OZ_M * OZ_KS) + kk * 32, 16, 512);
#pragma unroll
            for (int q = 0; q < S - p; ++q) {
              // level p + q: the first product of a chunk into each level
              // (p = 0 at the chunk's first K step) overwrites it
              const uint64_t db = sdesc(b_s + q * (OZ_N * OZ_KS) + kk * 32, 16, 512);
              const bool first = (i == i0 && kk == 0 && p == 0);
              mma_i8(tmem + (uint32_t)((p + q) * OZ_N), da, db, first ? 0u : 1u);
            }
          }
        }
        mma_commit(smem_u32(&bar_empty[s]));
      }
      // the chunk's accumulators are complete once its MMAs are (also after
      // an abort, so that the drain warps are released without waiting out)
      mma_commit(smem_u32(&bar_acc));
    }
  } else if (warp >= 2) {
    // drain: warp w reads TMEM lanes 32 (w % 4) .. +31, i.e. those rows of the tile
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    bool ok = nsteps > 0;
    for (int c = 0; c < nchunks; ++c) {
      const bool got = mbar_wait(smem_u32(&bar_acc), c & 1, wait_cycles);
      if (!got) atomicOr(status, GWB_ERR_TIMEOUT);
      const bool stop = __any_sync(0xffffffffu, !got || *(volatile int*)&abort_flag);
      if (stop) {
        ok = false;
        abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int l = 0; l < S; ++l) {
        const double f = ldexp(1.0, 2 - 7 * (l + 2));  // level L = l + 2: weight 2^(2 - 7L)
#pragma unroll
        for (int cb = 0; cb < OZ_N / 16; ++cb) {
          uint32_t r[16];
          tmem_ld16(tmem + lane_base + (uint32_t)(l * OZ_N + cb * 16), r);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int e = 0; e < 16; ++e) acc[cb * 16 + e] += (double)(int)r[e] * f;
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(smem_u32(&bar_free));
    }
    drained_all = ok;
  }

  // all roles done: no copy in flight, no MMA outstanding, TMEM read
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  const bool ok = !*(volatile int*)&abort_flag;
  double* stage = reinterpret_cast<double*>(dsm_raw + (dsm - smem_u32(dsm_raw)));
  if (warp >= 2 && ok) {
    const int rl = (warp & 3) * 32 + lane;
    const int row = m0 + rl;
    const double ra = (row < M && drained_all) ? sa[a_row0 + row] : 0.0;
#pragma unroll
    for (int j = 0; j < OZ_N; ++j) stage[rl * OZ_SROW + j] = acc[j] * ra;
  }
  __syncthreads();
  if (warp >= 2 && ok) {
    // warp w writes local rows (w - 2), (w - 2) + 4, ...: two columns per lane
    for (int rl = warp - 2; rl < OZ_M; rl += 4) {
      const int row = m0 + rl;
      if (row >= M) break;
#pragma unroll
      for (int h = 0; h < OZ_N / 32; ++h) {
        const int jl = lane + 32 * h, j = n0 + jl;
        if (j >= N) continue;
        double v = stage[rl * OZ_SROW + jl];
        if (sb) v *= sb[b_row0 + j];
        if (out.split) {
          out.C[((int64_t)blockIdx.y * M + row) * (int64_t)N + j] = v;
        } else {
          double* c = out.C + (int64_t)row * out.ldc + j;
          double w = out.alpha * v;
          if (out.beta != 0.0) w += out.beta * *c;
          *c = w;
        }
      }
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)OZ_TMEM_COLS)
                 : "memory");
  }
}

// C = alpha sum_s part[s] + beta C (fixed order over the splits).
__global__ void k_oz_reduce(int M, int N, int nsplit, const double* __restrict__ part, double alpha, double beta,
                            double* __restrict__ C, int64_t ldc) {
  const int64_t total = (int64_t)M * N;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / N), j = (int)(idx % N);
    double a = 0.0;
    for (int s = 0; s < nsplit; ++s) a += part[(int64_t)s * total + idx];
    double* c = C + (int64_t)i * ldc + j;
    double v = alpha * a;
    if (beta != 0.0) v += beta * *c;
    *c = v;
  }
}

// the power of two above |mx| (1 for a zero or non-finite row)
__device__ __forceinline__ double pow2_above(double mx) {
  if (!(mx > 0.0) || !isfinite(mx)) return 1.0;
  int e;
  frexp(mx, &e);
  return ldexp(1.0, e);
}

template <int NT> __device__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = l < NT / 32 ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (l == 0) red[0] = v;
  }
  __syncthreads();
  v = red[0];
  __syncthreads();
  return v;
}

// S slices of t (|t| < 1) into q[0..S-1]: q_p in [-64, 64] with weight 2^(1-7p)
template <int S> __device__ __forceinline__ void cut(double t, signed char (&q)[S]) {
  t *= 64.0;
#pragma unroll
  for (int p = 0; p < S; ++p) {
    const double w = rint(t);
    q[p] = (signed char)(int)w;
    t = (t - w) * 128.0;
  }
}

// One CTA per row r: scale[row0 + r] = 2^e above max_k |src[r][k] fold[k]|,
// slices of row r (and zeros in columns K..ldk-1) into plane rows row0 + r.
template <int S>
__global__ void __launch_bounds__(256) k_oz_split_rows(int K, const double* __restrict__ src, int64_t ld,
                                                       const double* __restrict__ fold, signed char* __restrict__ out,
                                                       int64_t ldk, int64_t plane, int64_t row0,
                                                       double* __restrict__ scale) {
  __shared__ double red[8];
  const int64_t r = blockIdx.x;
  const double* x = src + r * ld;
  double mx = 0.0;
  for (int k = threadIdx.x; k < K; k += blockDim.x) mx = fmax(mx, fabs(fold ? x[k] * fold[k] : x[k]));
  mx = block_max<256>(mx, red);
  const double sc = pow2_above(mx), inv = 1.0 / sc;
  if (threadIdx.x == 0) scale[row0 + r] = sc;
  signed char* o = out + (row0 + r) * ldk;
  // 16 columns per thread step; ldk is a multiple of 64, so every store is
  // 16 bytes, 16-byte aligned
  for (int64_t k0 = (int64_t)threadIdx.x * 16; k0 < ldk; k0 += (int64_t)blockDim.x * 16) {
    __align__(16) signed char q[S][16];
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const int64_t k = k0 + e;
      double t = 0.0;
      if (k < K) t = (fold ? x[k] * fold[k] : x[k]) * inv;
      signed char qq[S];
      cut<S>(t, qq);
#pragma unroll
      for (int p = 0; p < S; ++p) q[p][e] = qq[p];
    }
#pragma unroll
    for (int p = 0; p < S; ++p) *reinterpret_cast<uint4*>(o + p * plane + k0) = *reinterpret_cast<const uint4*>(q[p]);
  }
}

// One CTA per source row k (krows of them, R columns): kscale[k0 + k] = 2^e
// above max_r |src[k][r]|.
__global__ void __launch_bounds__(256) k_oz_row_scale(int64_t R, const double* __restrict__ src, int64_t ld,
                                                      int64_t k0, double* __restrict__ kscale) {
  __shared__ double red[8];
  const double* x = src + (int64_t)blockIdx.x * ld;
  double mx = 0.0;
  for (int64_t r = threadIdx.x; r < R; r += blockDim.x) mx = fmax(mx, fabs(x[r]));
  mx = block_max<256>(mx, red);
  if (threadIdx.x == 0) kscale[k0 + blockIdx.x] = pow2_above(mx);
}

// Transposed slices: operand row r, column k0 + k holds the slices of
// src[k][r] / kscale[k0 + k]. Tiles of 64 k x 64 r through shared memory.
template <int S>
__global__ void __launch_bounds__(256) k_oz_split_cols(int krows, int64_t R, const double* __restrict__ src,
                                                       int64_t ld, signed char* __restrict__ out, int64_t ldk,
                                                       int64_t plane, int64_t k0, const double* __restrict__ kscale) {
  __shared__ double tile[64][65];
  const int kt = blockIdx.y * 64;
  const int64_t rt = (int64_t)blockIdx.x * 64;
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
    const int kk = i / 64, rr = i % 64;
    const int k = kt + kk;
    const int64_t r = rt + rr;
    tile[kk][rr] = (k < krows && r < R) ? src[(int64_t)k * ld + r] / kscale[k0 + k] : 0.0;
  }
  __syncthreads();
  // thread: row rr, 16 consecutive k (kq * 16 ..)
  const int rr = threadIdx.x / 4, kq = threadIdx.x % 4;
  const int64_t r = rt + rr;
  if (r >= R) return;
  const int kb = kt + kq * 16;
  if (kb >= krows) return;
  const int nk = min(16, krows - kb);
  __align__(16) signed char q[S][16];
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    signed char qq[S];
    cut<S>(e < nk ? tile[kq * 16 + e][rr] : 0.0, qq);
#pragma unroll
    for (int p = 0; p < S; ++p) q[p][e] = qq[p];
  }
  signed char* o = out + r * ldk + k0 + kb;
  const bool vec = nk == 16 && (reinterpret_cast<uintptr_t>(o) % 16 == 0);
#pragma unroll
  for (int p = 0; p < S; ++p) {
    if (vec) {
      *reinterpret_cast<uint4*>(o + p * plane) = *reinterpret_cast<const uint4*>(q[p]);
    } else {
      for (int e = 0; e < nk; ++e) o[p * plane + e] = q[p][e];
    }
  }
}

// 3-D view (K bytes, rows, S planes) of a slice set; box (64, box_rows, S).
int make_slice_map(CUtensorMap* map, const void* base, int64_t ldk, int64_t rows_cap, int s, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return GWB_ERR_CUDA;
  }
  cuuint64_t dims[3] = {(cuuint64_t)ldk, (cuuint64_t)rows_cap, (cuuint64_t)s};
  cuuint64_t strides[2] = {(cuuint64_t)ldk, (cuuint64_t)(rows_cap * ldk)};
  cuuint32_t box[3] = {(cuuint32_t)OZ_KS, (cuuint32_t)box_rows, (cuuint32_t)s};
  cuuint32_t es[3] = {1u, 1u, 1u};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed with CUresult " + std::to_string((int)r));
    return GWB_ERR_CUDA;
  }
  return GWB_OK;
}

// K splits of a small tile grid: waves of 148 CTAs (one per SM), at least 16
// K steps per split, the fullest last wave, fewer splits on ties.
int64_t oz_splits(int64_t tiles, int64_t nsteps) {
  if (tiles >= 148) return 1;
  const int64_t smax = std::max<int64_t>(1, std::min<int64_t>(64, nsteps / 16));
  int64_t best = 1;
  double best_eff = -1.0;
  for (int64_t s = 1; s <= smax; ++s) {
    const int64_t ctas = tiles * s, waves = (ctas + 147) / 148;
    const double eff = (double)ctas / (double)(waves * 148) - 0.004 * (double)s;
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = s;
    }
  }
  return best;
}

template <int S>
int launch_oz(const CUtensorMap& mapA, const CUtensorMap& mapB, int64_t M, int64_t N, int64_t K, int64_t a_row0,
              int64_t b_row0, int64_t kps, int64_t splits, const OzOut& out, const double* sa, const double* sb,
              int* status, cudaStream_t st) {
  const int64_t Mt = (M + OZ_M - 1) / OZ_M, Nt = (N + OZ_N - 1) / OZ_N;
  dim3 grid((unsigned)(Mt * Nt), (unsigned)splits, 1);
  GWB_CUDA_TRY(allow_smem(k_oz_gemm<S>));
  k_oz_gemm<S><<<grid, OZ_THREADS, OzShape<S>::SMEM, st>>>(mapA, mapB, (int)M, (int)N, (int)K, (int)a_row0,
                                                           (int)b_row0, (int)kps, out, sa, sb, status,
                                                           tc_wait_cycles());
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

}  // namespace
}  // namespace gwb

using namespace gwb;

extern "C" int gwb_oz_split_rows(int32_t s, int64_t rows, int64_t K, const double* src, int64_t ld_src,
                                 const double* fold, void* slices, int64_t ldk, int64_t rows_cap, int64_t row0,
                                 double* scale, void* stream) {
  GWB_REQUIRE(s >= 6 && s <= 8, "slice count must be 6, 7 or 8");
  GWB_REQUIRE(rows >= 0 && K >= 0 && ldk % 64 == 0 && ldk >= K && ld_src >= K, "bad sizes");
  GWB_REQUIRE(row0 >= 0 && row0 + rows <= rows_cap, "rows beyond the slice set");
  if (rows == 0) return GWB_OK;
  GWB_REQUIRE(src && slices && scale, "null pointer");
  GWB_REQUIRE(reinterpret_cast<uintptr_t>(slices) % 16 == 0, "slices must be 16-byte aligned");
  GWB_REQUIRE(rows <= INT32_MAX && K <= INT32_MAX, "size beyond the grid limits");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t plane = rows_cap * ldk;
  auto* o = static_cast<signed char*>(slices);
  if (s == 6) k_oz_split_rows<6><<<(unsigned)rows, 256, 0, st>>>((int)K, src, ld_src, fold, o, ldk, plane, row0, scale);
  if (s == 7) k_oz_split_rows<7><<<(unsigned)rows, 256, 0, st>>>((int)K, src, ld_src, fold, o, ldk, plane, row0, scale);
  if (s == 8) k_oz_split_rows<8><<<(unsigned)rows, 256, 0, st>>>((int)K, src, ld_src, fold, o, ldk, plane, row0, scale);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

extern "C" int gwb_oz_split_cols(int32_t s, int64_t krows, int64_t R, const double* src, int64_t ld_src,
                                 void* slices, int64_t ldk, int64_t rows_cap, int64_t k0, double* kscale,
                                 void* stream) {
  GWB_REQUIRE(s >= 6 && s <= 8, "slice count must be 6, 7 or 8");
  GWB_REQUIRE(krows >= 0 && R >= 0 && ld_src >= R && ldk % 64 == 0, "bad sizes");
  GWB_REQUIRE(k0 >= 0 && k0 + krows <= ldk && R <= rows_cap, "columns beyond the slice set");
  if (krows == 0 || R == 0) return GWB_OK;
  GWB_REQUIRE(src && slices && kscale, "null pointer");
  GWB_REQUIRE(krows <= 65535 * 64LL && R <= INT32_MAX, "size beyond the grid limits");
  cudaStream_t st = (cudaStream_t)stream;
  k_oz_row_scale<<<(unsigned)krows, 256, 0, st>>>(R, src, ld_src, k0, kscale);
  const int64_t plane = rows_cap * ldk;
  auto* o = static_cast<signed char*>(slices);
  dim3 g((unsigned)((R + 63) / 64), (unsigned)((krows + 63) / 64));
  if (s == 6) k_oz_split_cols<6><<<g, 256, 0, st>>>((int)krows, R, src, ld_src, o, ldk, plane, k0, kscale);
  if (s == 7) k_oz_split_cols<7><<<g, 256, 0, st>>>((int)krows, R, src, ld_src, o, ldk, plane, k0, kscale);
  if (s == 8) k_oz_split_cols<8><<<g, 256, 0, st>>>((int)krows, R, src, ld_src, o, ldk, plane, k0, kscale);
  GWB_LAUNCH_CHECK();
  count_launches(2);
  return GWB_OK;
}

extern "C" int64_t gwb_oz_work_bytes(int64_t M, int64_t N, int64_t K) {
  if (M <= 0 || N <= 0 || K <= 0) return 0;
  const int64_t tiles = ((M + OZ_M - 1) / OZ_M) * ((N + OZ_N - 1) / OZ_N);
  const int64_t splits = oz_splits(tiles, (K + OZ_KS - 1) / OZ_KS);
  return splits > 1 ? splits * M * N * 8 : 0;
}

extern "C" int gwb_oz_gemm(int32_t s, int64_t M, int64_t N, int64_t K, const void* A, int64_t lda,
                           int64_t a_rows_cap, int64_t a_row0, const double* a_scale, const void* B, int64_t ldb,
                           int64_t b_rows_cap, int64_t b_row0, const double* b_scale, double alpha, double beta,
                           double* C, int64_t ldc, void* work, size_t work_bytes, int* status, void* stream) {
  GWB_REQUIRE(s >= 6 && s <= 8, "slice count must be 6, 7 or 8");
  GWB_REQUIRE(M >= 0 && N >= 0 && K >= 0, "negative size");
  if (M == 0 || N == 0) return GWB_OK;
  GWB_REQUIRE(A && B && a_scale && C && status, "null pointer");
  GWB_REQUIRE(lda % 64 == 0 && ldb % 64 == 0 && lda >= K && ldb >= K, "slice ld must be a multiple of 64, >= K");
  GWB_REQUIRE(reinterpret_cast<uintptr_t>(A) % 16 == 0 && reinterpret_cast<uintptr_t>(B) % 16 == 0,
              "slices must be 16-byte aligned");
  GWB_REQUIRE(a_row0 >= 0 && a_row0 + M <= a_rows_cap && b_row0 >= 0 && b_row0 + N <= b_rows_cap,
              "rows beyond the slice sets");
  GWB_REQUIRE(ldc >= N, "ldc < N");
  GWB_REQUIRE(a_rows_cap <= INT32_MAX && b_rows_cap <= INT32_MAX && K <= INT32_MAX, "size beyond the grid limits");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nsteps = (K + OZ_KS - 1) / OZ_KS;
  if (nsteps == 0) {
    const int blocks = (int)std::min<int64_t>((M * N + 255) / 256, 4096);
    k_oz_reduce<<<blocks, 256, 0, st>>>((int)M, (int)N, 0, nullptr, alpha, beta, C, ldc);
    GWB_LAUNCH_CHECK();
    count_launches(1);
    return GWB_OK;
  }
  CUtensorMap mapA, mapB;
  int rc = make_slice_map(&mapA, A, lda, a_rows_cap, s, OZ_M);
  if (rc != GWB_OK) return rc;
  rc = make_slice_map(&mapB, B, ldb, b_rows_cap, s, OZ_N);
  if (rc != GWB_OK) return rc;
  const int64_t tiles = ((M + OZ_M - 1) / OZ_M) * ((N + OZ_N - 1) / OZ_N);
  GWB_REQUIRE(tiles <= INT32_MAX, "too many tiles");
  int64_t splits = oz_splits(tiles, nsteps);
  while (splits > 1 && (!work || splits * M * N * 8 > (int64_t)work_bytes)) --splits;
  const int64_t kps = (nsteps + splits - 1) / splits;
  splits = (nsteps + kps - 1) / kps;
  OzOut out;
  out.ldc = ldc;
  out.alpha = alpha;
  out.beta = beta;
  out.split = splits > 1;
  out.C = splits > 1 ? static_cast<double*>(work) : C;
  if (s == 6) rc = launch_oz<6>(mapA, mapB, M, N, K, a_row0, b_row0, kps, splits, out, a_scale, b_scale, status, st);
  if (s == 7) rc = launch_oz<7>(mapA, mapB, M, N, K, a_row0, b_row0, kps, splits, out, a_scale, b_scale, status, st);
  if (s == 8) rc = launch_oz<8>(mapA, mapB, M, N, K, a_row0, b_row0, kps, splits, out, a_scale, b_scale, status, st);
  if (rc != GWB_OK) return rc;
  if (splits > 1) {
    const int blocks = (int)std::min<int64_t>((M * N + 255) / 256, 4096);
    k_oz_reduce<<<blocks, 256, 0, st>>>((int)M, (int)N, (int)splits, static_cast<const double*>(work), alpha, beta,
                                        C, ldc);
    GWB_LAUNCH_CHECK();
    count_launches(1);
  }
  return GWB_OK;
}
