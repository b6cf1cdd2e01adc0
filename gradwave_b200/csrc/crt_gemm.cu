// Float64-accurate real products on the int8 tensor cores through residues:
// the Ozaki scheme, second form (Ozaki, Uchino & Imamura, "Ozaki Scheme II:
// A GEMM-oriented emulation of floating-point matrix multiplication using an
// integer modular technique", 2025), on tcgen05 kind::i8.
//
// Conversion. Row r of an operand is scaled by 2^(p - e_r), with 2^e_r the
// power of two above the row's largest magnitude, and rounded to the nearest
// integer, so |x_int| < 2^p and x = x_int 2^(e_r - p) to within 2^(e_r-p-1).
// The integer is stored as its n centred residues modulo n pairwise coprime
// moduli m_t <= 256 (kCrtMod), one int8 plane per modulus: a residue set holds
// n planes of rows_cap x ldk bytes (ldk a multiple of 64, columns K..ldk-1
// zero) and a float64 scale 2^(e_r - p) per row.
//
// Product. For every modulus the int8 product A_t B_t^T is exact in int32
// (at most 131008 columns per split: 128^2 x 131008 < 2^31); it is reduced
// modulo m_t and multiplied by y_t = (M / m_t)^-1 mod m_t (M = prod m_t), and
// that byte is the kernel's output. With |C_int| < K 2^2p <= M / 2 (p is
// chosen from n so that this holds for K <= 2^19), the Chinese remainder
// theorem gives C_int / M = frac(sum_t (C_t y_t mod m_t) / m_t), centred into
// [-1/2, 1/2): the reduction sums the terms in double-double arithmetic
// (absolute error ~2^-100, i.e. ~2^40 on C_int, against the ~2^(2p-p) of the
// rounding in the conversion) and scales by M and the two rows' scales. So
// n int8 products make one float64 product, and only one accumulator is live
// per modulus: the kernel runs M 128 x N 256 tiles with two accumulators
// (512 TMEM columns) so that the drain of modulus t overlaps the MMAs of t+1.
// Accuracy: each element is within about 2^-p-1 of the row maxima of A and B
// times the column sums of the other operand (p = 52, 60, 67 for n = 16, 18,
// 20), against 2^-53 times |A||B| for a float64 GEMM.
//
// The product C = A B with B held as K x N rows (X = U^T V) uses B's columns
// as rows (gwb_crt_split_cols: scaled per source row k by a power of two
// kscale_k, which is folded into A's columns before A is split).
//
// CTA: 192 threads, one 128 x 256 tile of one K split. Warp 0 lane 0 streams
// (modulus, K step) boxes of 64 columns of both operands into an 8-stage ring
// (TMA, 64-byte swizzle); warp 1 lane 0 issues two tcgen05.mma (M 128, N 256,
// K 32) per step into accumulator t % 2; warps 2-5 read an accumulator when
// its modulus is done, reduce it and write one byte per element to the
// workspace (nsplit, n, M, ldw). k_crt_reduce then forms C = alpha A B^T +
// beta C. Every mbarrier wait is bounded (gwb_tc_set_wait_limit); a wait that
// runs out ORs GWB_ERR_TIMEOUT into *status, the producer waits for its copies
// in flight, and the TMEM is always released.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "common.cuh"
#include "tcgen05.cuh"

namespace gwb {
namespace {

constexpr int CRT_MAXN = 20;
// pairwise coprime (256 = 2^8, 255 = 3 5 17, 253 = 11 23, 247 = 13 19,
// 217 = 7 31, the rest prime); centred residues fit int8
constexpr int kCrtMod[CRT_MAXN] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                                   223, 217, 211, 199, 197, 193, 191, 181, 179, 173};
// the same table for device code (folded to a constant in unrolled loops)
__host__ __device__ constexpr int crt_mod(int t) {
  return t == 0 ? 256 : t == 1 ? 255 : t == 2 ? 253 : t == 3 ? 251 : t == 4 ? 247 : t == 5 ? 241 : t == 6 ? 239
       : t == 7 ? 233 : t == 8 ? 229 : t == 9 ? 227 : t == 10 ? 223 : t == 11 ? 217 : t == 12 ? 211
       : t == 13 ? 199 : t == 14 ? 197 : t == 15 ? 193 : t == 16 ? 191 : t == 17 ? 181 : t == 18 ? 179 : 173;
}
constexpr int CRT_M = 128;
constexpr int CRT_N = 256;
constexpr int CRT_KS = 64;  // K elements (bytes) per stage: one 64-byte swizzle row
constexpr int CRT_STAGES = 8;
constexpr int CRT_THREADS = 192;
constexpr int CRT_TMEM_COLS = 512;
constexpr int CRT_A_BYTES = CRT_M * CRT_KS;
constexpr int CRT_B_BYTES = CRT_N * CRT_KS;
constexpr int CRT_STAGE = CRT_A_BYTES + CRT_B_BYTES;
constexpr int CRT_SMEM = CRT_STAGES * CRT_STAGE + 1024;
constexpr int64_t CRT_SPLIT_STEPS = 131008 / CRT_KS;  // K steps per split with exact int32 sums
constexpr int64_t CRT_MAX_K = (int64_t)1 << 19;

// kind::i8 instruction descriptor: D s32, A and B s8, both K-major, M 128, N 256.
constexpr uint32_t CRT_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(CRT_N >> 3) << 17) |
                               ((uint32_t)(CRT_M >> 4) << 24);

__device__ __forceinline__ void mma_i8_n256(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(CRT_IDESC), "r"(accumulate)
      : "memory");
}

// Per-modulus constants of the drain: m, the multiplier of the division by m
// (floor(2^39 / m) + 1: for u < 2^32, (u mg) >> 39 is floor(u / m) or one
// more), 2^31 mod m, and y = (M / m)^-1 mod m.
struct CrtDrain {
  uint32_t m[CRT_MAXN];
  uint32_t mg[CRT_MAXN];
  uint32_t c31[CRT_MAXN];
  uint32_t y[CRT_MAXN];
};

// Constants of the reconstruction: 1/m_t as a double-double (ih + il) and M
// as a double-double (Mh + Ml).
struct CrtRecon {
  double ih[CRT_MAXN];
  double il[CRT_MAXN];
  double Mh, Ml;
};

// u mod m for u < 2^32
__device__ __forceinline__ uint32_t mod_u32(uint32_t u, uint32_t m, uint32_t mg) {
  const uint32_t q = (uint32_t)(((uint64_t)u * mg) >> 39);
  int r = (int)(u - q * m);
  if (r < 0) r += (int)m;
  return (uint32_t)r;
}

struct CrtArgs {
  int M, N, K;
  int a_row0, b_row0;
  int steps_per_split;
  uint8_t* work;  // (nsplit, n, M, ldw) bytes
  int64_t ldw;
  int* status;
  long long wait_cycles;
};

template <int NM>
__global__ void __launch_bounds__(CRT_THREADS, 1)
    k_crt_gemm(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, CrtArgs a,
               CrtDrain dc) {
  __shared__ __align__(8) uint64_t bar_full[CRT_STAGES];
  __shared__ __align__(8) uint64_t bar_empty[CRT_STAGES];
  __shared__ __align__(8) uint64_t bar_acc[2];   // the MMAs of a modulus have completed
  __shared__ __align__(8) uint64_t bar_free[2];  // the drain has read the accumulator
  __shared__ uint32_t tmem_base_slot;
  __shared__ int abort_flag;
  extern __shared__ uint8_t dsm_raw[];
  const uint32_t dsm = (smem_u32(dsm_raw) + 1023u) & ~1023u;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Mt = (a.M + CRT_M - 1) / CRT_M;
  const int mt = blockIdx.x % Mt, nt = blockIdx.x / Mt;
  const int m0 = mt * CRT_M, n0 = nt * CRT_N;
  const int nsteps_all = (a.K + CRT_KS - 1) / CRT_KS;
  const int ks0 = blockIdx.y * a.steps_per_split;
  const int nsteps = max(0, min(nsteps_all, ks0 + a.steps_per_split) - ks0);
  const long long wc = a.wait_cycles;

  if (tid == 0) {
    for (int s = 0; s < CRT_STAGES; ++s) {
      mbar_init(smem_u32(&bar_full[s]), 1);
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&bar_acc[b]), 1);
      mbar_init(smem_u32(&bar_free[b]), 128);
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                 "r"((uint32_t)CRT_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_slot;

  if (warp == 0 && lane == 0 && nsteps > 0) {
    // producer: (modulus t, K step i) in order
    int last_round[CRT_STAGES];
#pragma unroll
    for (int s = 0; s < CRT_STAGES; ++s) last_round[s] = -1;
    const int total = nsteps * NM;
    for (int g = 0; g < total; ++g) {
      const int s = g % CRT_STAGES;
      if (g >= CRT_STAGES && !mbar_wait(smem_u32(&bar_empty[s]), ((g / CRT_STAGES) - 1) & 1, wc)) {
        abort_flag = 1;
        atomicOr(a.status, GWB_ERR_TIMEOUT);
        break;
      }
      if (*(volatile int*)&abort_flag) break;
      last_round[s] = g / CRT_STAGES;
      const int t = g / nsteps, i = g - t * nsteps;
      const uint32_t full = smem_u32(&bar_full[s]);
      const uint32_t a_s = dsm + s * CRT_STAGE, b_s = a_s + CRT_A_BYTES;
      mbar_expect_tx(full, CRT_STAGE);
      const int k0 = (ks0 + i) * CRT_KS;
      tma_load_3d(a_s, &mapA, full, k0, a.a_row0 + m0, t);
      tma_load_3d(b_s, &mapB, full, k0, a.b_row0 + n0, t);
    }
    // every issued box must have landed before the CTA can leave
#pragma unroll
    for (int s = 0; s < CRT_STAGES; ++s)
      if (last_round[s] >= 0 && !mbar_wait(smem_u32(&bar_full[s]), last_round[s] & 1, wc))
        atomicOr(a.status, GWB_ERR_TIMEOUT);
  } else if (warp == 1 && lane == 0 && nsteps > 0) {
    // MMA issuer
    bool stop = false;
    for (int t = 0; t < NM && !stop; ++t) {
      const int b = t & 1;
      if (t >= 2 && !mbar_wait(smem_u32(&bar_free[b]), ((t >> 1) - 1) & 1, wc)) {
        abort_flag = 1;
        atomicOr(a.status, GWB_ERR_TIMEOUT);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int i = 0; i < nsteps; ++i) {
        const int g = t * nsteps + i, s = g % CRT_STAGES;
        if (!mbar_wait(smem_u32(&bar_full[s]), (g / CRT_STAGES) & 1, wc)) {
          abort_flag = 1;
          atomicOr(a.status, GWB_ERR_TIMEOUT);
          stop = true;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_s = dsm + s * CRT_STAGE, b_s = a_s + CRT_A_BYTES;
#pragma unroll
        for (int kk = 0; kk < CRT_KS / 32; ++kk) {
          const uint64_t da = sdesc(a_s + kk * 32, 16, 512);
          const uint64_t db = sdesc(b_s + kk * 32, 16, 512);
          mma_i8_n256(tmem + (uint32_t)(b * CRT_N), da, db, (i == 0 && kk == 0) ? 0u : 1u);
        }
        mma_commit(smem_u32(&bar_empty[s]));
      }
      // the modulus' accumulator is complete once its MMAs are (also after an
      // abort, so that the drain warps are released without waiting out)
      mma_commit(smem_u32(&bar_acc[b]));
    }
  } else if (warp >= 2) {
    // drain: warp w reads TMEM lanes 32 (w % 4) .. +31, i.e. those rows of the tile
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const int row = m0 + (warp & 3) * 32 + lane;
    for (int t = 0; t < NM && nsteps > 0; ++t) {
      const int b = t & 1;
      const bool got = mbar_wait(smem_u32(&bar_acc[b]), (t >> 1) & 1, wc);
      if (!got) atomicOr(a.status, GWB_ERR_TIMEOUT);
      if (__any_sync(0xffffffffu, !got || *(volatile int*)&abort_flag)) {
        abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t m = dc.m[t], mg = dc.mg[t], c31 = dc.c31[t], y = dc.y[t];
      uint8_t* dst = a.work + (((int64_t)blockIdx.y * NM + t) * a.M + row) * a.ldw + n0;
#pragma unroll 1
      for (int cb = 0; cb < CRT_N / 16; ++cb) {
        uint32_t r[16];
        tmem_ld16(tmem + lane_base + (uint32_t)(b * CRT_N + cb * 16), r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        __align__(16) uint8_t o[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          // x + 2^31 (as u32) mod m, minus 2^31 mod m: x mod m; then times y
          uint32_t v = mod_u32(r[e] + 0x80000000u, m, mg) + m - c31;
          v = mod_u32(v * y, m, mg);
          o[e] = (uint8_t)v;
        }
        if (row < a.M && n0 + cb * 16 < a.ldw)
          *reinterpret_cast<uint4*>(dst + cb * 16) = *reinterpret_cast<const uint4*>(o);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(smem_u32(&bar_free[b]));
    }
  }

  // all roles done: no copy in flight, no MMA outstanding, TMEM read
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)CRT_TMEM_COLS)
                 : "memory");
  }
}

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// C = alpha (C_int sa_i sb_j) + beta C from the residue bytes of nsplit splits.
template <int NM>
__global__ void __launch_bounds__(256) k_crt_reduce(int M, int N, int nsplit, const uint8_t* __restrict__ work,
                                                    int64_t ldw, CrtRecon rc, const double* __restrict__ sa,
                                                    const double* __restrict__ sb, double alpha, double beta,
                                                    double* __restrict__ C, int64_t ldc) {
  const int64_t total = (int64_t)M * N;
  const int64_t plane = (int64_t)M * ldw;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / N), j = (int)(idx % N);
    const uint8_t* w = work + (int64_t)i * ldw + j;
    double sh = 0.0, sl = 0.0;
#pragma unroll
    for (int t = 0; t < NM; ++t) {
      int R = 0;
      for (int sp = 0; sp < nsplit; ++sp) R += w[((int64_t)sp * NM + t) * plane];
      const double r = (double)R;
      const double ph = r * rc.ih[t];
      const double pl = fma(r, rc.il[t], fma(r, rc.ih[t], -ph));
      double s, e;
      two_sum(sh, ph, s, e);
      sh = s;
      sl += e + pl;
    }
    sh -= floor(sh);  // exact: sh < 2^52
    double f, fl;
    two_sum(sh, sl, f, fl);
    if (f >= 0.5) f -= 1.0;  // exact (Sterbenz)
    if (f < -0.5) f += 1.0;
    const double cint = fma(f, rc.Mh, fma(f, rc.Ml, fl * rc.Mh));
    const double v = cint * sa[i] * sb[j];
    double* c = C + (int64_t)i * ldc + j;
    double o = alpha * v;
    if (beta != 0.0) o += beta * *c;
    *c = o;
  }
}

// the power of two above |mx| (2^0 for a zero row; NaN for a non-finite one,
// so that the products of that row come out NaN as a float64 GEMM's would)
__device__ __forceinline__ int exp_above(double mx, bool& bad) {
  bad = !isfinite(mx);
  if (!(mx > 0.0) || bad) return 0;
  int e;
  frexp(mx, &e);
  return e;
}

template <int NT> __device__ double block_max_crt(double v, double* red) {
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

// centred residue of the integer-valued double xi (|xi| < 2^68) modulo m:
// q = rint(xi / m) is within a few hundred of the true quotient, so xi - q m
// is small and the fma forms it exactly.
__device__ __forceinline__ signed char residue(double xi, int m) {
  const double q = rint(xi * (1.0 / (double)m));
  int r = (int)fma(-q, (double)m, xi);
  r %= m;
  if (r > (m - 1) / 2) r -= m;
  else if (r < -(m / 2)) r += m;
  return (signed char)r;
}

// the NM residue planes of 16 consecutive integer-valued doubles: one 16-byte
// store per plane (o 16-byte aligned) or nk single bytes
template <int NM>
__device__ __forceinline__ void store_residues(const double (&xi)[16], signed char* o, int64_t plane, int nk,
                                               bool vec) {
#pragma unroll
  for (int t = 0; t < NM; ++t) {
    const int m = crt_mod(t);
    __align__(16) signed char q[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) q[e] = residue(xi[e], m);
    if (vec) {
      *reinterpret_cast<uint4*>(o + t * plane) = *reinterpret_cast<const uint4*>(q);
    } else {
      for (int e = 0; e < nk; ++e) o[t * plane + e] = q[e];
    }
  }
}

// One CTA per row r: scale[row0 + r] = 2^(e - p) with 2^e above
// max_k |src[r][k] fold[k]|; residues of rint(x 2^(p - e)) into plane rows row0 + r.
template <int NM>
__global__ void __launch_bounds__(256) k_crt_split_rows(int K, int p, const double* __restrict__ src, int64_t ld,
                                                        const double* __restrict__ fold,
                                                        signed char* __restrict__ out, int64_t ldk, int64_t plane,
                                                        int64_t row0, double* __restrict__ scale) {
  __shared__ double red[8];
  const int64_t r = blockIdx.x;
  const double* x = src + r * ld;
  double mx = 0.0;
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    const double v = fold ? x[k] * fold[k] : x[k];
    mx = fmax(mx, isfinite(v) ? fabs(v) : INFINITY);
  }
  mx = block_max_crt<256>(mx, red);
  bool bad;
  const int e = exp_above(mx, bad);
  const double up = ldexp(1.0, p - e);
  if (threadIdx.x == 0) scale[row0 + r] = bad ? NAN : ldexp(1.0, e - p);
  signed char* o = out + (row0 + r) * ldk;
  // 16 columns per thread step; ldk is a multiple of 64, so every store is
  // 16 bytes, 16-byte aligned
  for (int64_t k0 = (int64_t)threadIdx.x * 16; k0 < ldk; k0 += (int64_t)blockDim.x * 16) {
    double xi[16];
#pragma unroll
    for (int e2 = 0; e2 < 16; ++e2) {
      const int64_t k = k0 + e2;
      xi[e2] = (k < K && !bad) ? rint((fold ? x[k] * fold[k] : x[k]) * up) : 0.0;
    }
    store_residues<NM>(xi, o + k0, plane, 16, true);
  }
}

// One CTA per source row k: kscale[k0 + k] = the power of two above
// max_r |src[k][r]| (1 for a zero row, NaN for a non-finite one).
__global__ void __launch_bounds__(256) k_crt_row_scale(int64_t R, const double* __restrict__ src, int64_t ld,
                                                       int64_t k0, double* __restrict__ kscale) {
  __shared__ double red[8];
  const double* x = src + (int64_t)blockIdx.x * ld;
  double mx = 0.0;
  for (int64_t r = threadIdx.x; r < R; r += blockDim.x) mx = fmax(mx, isfinite(x[r]) ? fabs(x[r]) : INFINITY);
  mx = block_max_crt<256>(mx, red);
  bool bad;
  const int e = exp_above(mx, bad);
  if (threadIdx.x == 0) kscale[k0 + blockIdx.x] = bad ? NAN : ldexp(1.0, e);
}

// Transposed residues: operand row r, column k0 + k holds the residues of
// rint(2^p src[k][r] / kscale[k0 + k]); the row scale of every such row is
// 2^-p. Tiles of 64 k x 64 r through shared memory.
template <int NM>
__global__ void __launch_bounds__(256) k_crt_split_cols(int krows, int64_t R, int p, const double* __restrict__ src,
                                                        int64_t ld, signed char* __restrict__ out, int64_t ldk,
                                                        int64_t plane, int64_t k0, const double* __restrict__ kscale,
                                                        double* __restrict__ scale) {
  __shared__ double tile[64][65];
  const int kt = blockIdx.y * 64;
  const int64_t rt = (int64_t)blockIdx.x * 64;
  const double up = ldexp(1.0, p);
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
    const int kk = i / 64, rr = i % 64;
    const int k = kt + kk;
    const int64_t r = rt + rr;
    double v = 0.0;
    if (k < krows && r < R) {
      const double ks = kscale[k0 + k];
      v = isfinite(ks) ? rint(src[(int64_t)k * ld + r] / ks * up) : 0.0;
    }
    tile[kk][rr] = v;
  }
  __syncthreads();
  const int rr = threadIdx.x / 4, kq = threadIdx.x % 4;
  const int64_t r = rt + rr;
  if (r >= R) return;
  if (blockIdx.y == 0 && kq == 0) scale[r] = ldexp(1.0, -p);
  const int kb = kt + kq * 16;
  if (kb >= krows) return;
  const int nk = min(16, krows - kb);
  double xi[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) xi[e] = e < nk ? tile[kq * 16 + e][rr] : 0.0;
  signed char* o = out + r * ldk + k0 + kb;
  store_residues<NM>(xi, o, plane, nk, nk == 16 && (reinterpret_cast<uintptr_t>(o) % 16 == 0));
}

// ---- host side -------------------------------------------------------------

int64_t inv_mod(int64_t a, int64_t m) {
  int64_t t = 0, nt = 1, r = m, nr = ((a % m) + m) % m;
  while (nr != 0) {
    const int64_t q = r / nr;
    int64_t tmp = t - q * nt;
    t = nt;
    nt = tmp;
    tmp = r - q * nr;
    r = nr;
    nr = tmp;
  }
  return t < 0 ? t + m : t;
}

struct CrtTables {
  CrtDrain drain;
  CrtRecon recon;
  double log2M;
  int p;
};

CrtTables make_tables(int n) {
  CrtTables T{};
  T.log2M = 0.0;
  for (int t = 0; t < n; ++t) T.log2M += std::log2((double)kCrtMod[t]);
  // 2p + 19 <= log2 M - 1: |C_int| < 2^19 2^2p <= M / 2
  T.p = (int)std::floor((T.log2M - 1.0 - 19.0) / 2.0);
  double mh = 1.0, ml = 0.0;
  for (int t = 0; t < n; ++t) {
    const int64_t m = kCrtMod[t];
    int64_t prod = 1;
    for (int j = 0; j < n; ++j)
      if (j != t) prod = (prod * (kCrtMod[j] % m)) % m;
    T.drain.m[t] = (uint32_t)m;
    T.drain.mg[t] = (uint32_t)(((uint64_t)1 << 39) / (uint64_t)m + 1);
    T.drain.c31[t] = (uint32_t)(((uint64_t)1 << 31) % (uint64_t)m);
    T.drain.y[t] = (uint32_t)inv_mod(prod, m);
    const double ih = 1.0 / (double)m;
    T.recon.ih[t] = ih;
    T.recon.il[t] = std::fma(-ih, (double)m, 1.0) / (double)m;
    // (mh + ml) *= m, renormalised
    const double ph = mh * (double)m;
    const double pe = std::fma(mh, (double)m, -ph) + ml * (double)m;
    mh = ph + pe;
    ml = pe - (mh - ph);
  }
  T.recon.Mh = mh;
  T.recon.Ml = ml;
  return T;
}

const CrtTables& tables(int n) {
  static CrtTables tab[CRT_MAXN + 1];
  static std::once_flag once;
  std::call_once(once, [] {
    for (int k = 1; k <= CRT_MAXN; ++k) tab[k] = make_tables(k);
  });
  return tab[n];
}

bool supported(int n) { return n == 16 || n == 18 || n == 20; }

// 3-D view (K bytes, rows, n planes) of a residue set; box (64, box_rows, 1).
int make_residue_map(CUtensorMap* map, const void* base, int64_t ldk, int64_t rows_cap, int n, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return GWB_ERR_CUDA;
  }
  cuuint64_t dims[3] = {(cuuint64_t)ldk, (cuuint64_t)rows_cap, (cuuint64_t)n};
  cuuint64_t strides[2] = {(cuuint64_t)ldk, (cuuint64_t)(rows_cap * ldk)};
  cuuint32_t box[3] = {(cuuint32_t)CRT_KS, (cuuint32_t)box_rows, 1u};
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

// K splits: at least ceil(nsteps / CRT_SPLIT_STEPS) (exact int32 sums), then
// waves of 148 CTAs (one per SM), at least 16 K steps per split, the fullest
// last wave, fewer splits on ties.
int64_t crt_splits(int64_t tiles, int64_t nsteps) {
  const int64_t smin = std::max<int64_t>(1, (nsteps + CRT_SPLIT_STEPS - 1) / CRT_SPLIT_STEPS);
  if (tiles * smin >= 148) return smin;
  const int64_t smax = std::max<int64_t>(smin, std::min<int64_t>(64, nsteps / 16));
  int64_t best = smin;
  double best_eff = -1.0;
  for (int64_t s = smin; s <= smax; ++s) {
    const int64_t ctas = tiles * s, waves = (ctas + 147) / 148;
    const double eff = (double)ctas / (double)(waves * 148) - 0.004 * (double)s;
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = s;
    }
  }
  return best;
}

int64_t ldw_of(int64_t N) { return (N + 15) / 16 * 16; }

template <int NM>
int launch_crt(const CUtensorMap& mapA, const CUtensorMap& mapB, int64_t Mt, int64_t Nt, int64_t splits,
               const CrtArgs& args, cudaStream_t st) {
  dim3 grid((unsigned)(Mt * Nt), (unsigned)splits, 1);
  GWB_CUDA_TRY(allow_smem(k_crt_gemm<NM>));
  k_crt_gemm<NM><<<grid, CRT_THREADS, CRT_SMEM, st>>>(mapA, mapB, args, tables(NM).drain);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

template <int NM>
void launch_reduce(int64_t M, int64_t N, int64_t splits, const uint8_t* work, int64_t ldw, const double* sa,
                   const double* sb, double alpha, double beta, double* C, int64_t ldc, cudaStream_t st) {
  const int blocks = (int)std::min<int64_t>((M * N + 255) / 256, 148 * 16);
  k_crt_reduce<NM><<<blocks, 256, 0, st>>>((int)M, (int)N, (int)splits, work, ldw, tables(NM).recon, sa, sb, alpha,
                                           beta, C, ldc);
}

}  // namespace
}  // namespace gwb

using namespace gwb;

extern "C" int32_t gwb_crt_bits(int32_t n) { return supported(n) ? tables(n).p : -1; }

extern "C" int gwb_crt_constants(int32_t n, uint32_t* m, uint32_t* y, double* inv_hi, double* inv_lo,
                                 double* M_hl) {
  GWB_REQUIRE(supported(n), "modulus count must be 16, 18 or 20");
  GWB_REQUIRE(m && y && inv_hi && inv_lo && M_hl, "null pointer");
  const CrtTables& T = tables(n);
  for (int t = 0; t < n; ++t) {
    m[t] = T.drain.m[t];
    y[t] = T.drain.y[t];
    inv_hi[t] = T.recon.ih[t];
    inv_lo[t] = T.recon.il[t];
  }
  M_hl[0] = T.recon.Mh;
  M_hl[1] = T.recon.Ml;
  return GWB_OK;
}

extern "C" int gwb_crt_split_rows(int32_t n, int64_t rows, int64_t K, const double* src, int64_t ld_src,
                                  const double* fold, void* planes, int64_t ldk, int64_t rows_cap, int64_t row0,
                                  double* scale, void* stream) {
  GWB_REQUIRE(supported(n), "modulus count must be 16, 18 or 20");
  GWB_REQUIRE(rows >= 0 && K >= 0 && ldk % 64 == 0 && ldk >= K && ld_src >= K, "bad sizes");
  GWB_REQUIRE(row0 >= 0 && row0 + rows <= rows_cap, "rows beyond the residue set");
  if (rows == 0) return GWB_OK;
  GWB_REQUIRE(src && planes && scale, "null pointer");
  GWB_REQUIRE(reinterpret_cast<uintptr_t>(planes) % 16 == 0, "residue planes must be 16-byte aligned");
  GWB_REQUIRE(rows <= INT32_MAX && K <= INT32_MAX, "size beyond the grid limits");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t plane = rows_cap * ldk;
  const int p = tables(n).p;
  auto* o = static_cast<signed char*>(planes);
  if (n == 16) k_crt_split_rows<16><<<(unsigned)rows, 256, 0, st>>>((int)K, p, src, ld_src, fold, o, ldk, plane, row0, scale);
  if (n == 18) k_crt_split_rows<18><<<(unsigned)rows, 256, 0, st>>>((int)K, p, src, ld_src, fold, o, ldk, plane, row0, scale);
  if (n == 20) k_crt_split_rows<20><<<(unsigned)rows, 256, 0, st>>>((int)K, p, src, ld_src, fold, o, ldk, plane, row0, scale);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

extern "C" int gwb_crt_split_cols(int32_t n, int64_t krows, int64_t R, const double* src, int64_t ld_src,
                                  void* planes, int64_t ldk, int64_t rows_cap, int64_t k0, double* kscale,
                                  double* scale, void* stream) {
  GWB_REQUIRE(supported(n), "modulus count must be 16, 18 or 20");
  GWB_REQUIRE(krows >= 0 && R >= 0 && ld_src >= R && ldk % 64 == 0, "bad sizes");
  GWB_REQUIRE(k0 >= 0 && k0 + krows <= ldk && R <= rows_cap, "columns beyond the residue set");
  if (krows == 0 || R == 0) return GWB_OK;
  GWB_REQUIRE(src && planes && kscale && scale, "null pointer");
  GWB_REQUIRE(krows <= 65535 * 64LL && R <= INT32_MAX, "size beyond the grid limits");
  cudaStream_t st = (cudaStream_t)stream;
  k_crt_row_scale<<<(unsigned)krows, 256, 0, st>>>(R, src, ld_src, k0, kscale);
  const int64_t plane = rows_cap * ldk;
  const int p = tables(n).p;
  auto* o = static_cast<signed char*>(planes);
  dim3 g((unsigned)((R + 63) / 64), (unsigned)((krows + 63) / 64));
  if (n == 16) k_crt_split_cols<16><<<g, 256, 0, st>>>((int)krows, R, p, src, ld_src, o, ldk, plane, k0, kscale, scale);
  if (n == 18) k_crt_split_cols<18><<<g, 256, 0, st>>>((int)krows, R, p, src, ld_src, o, ldk, plane, k0, kscale, scale);
  if (n == 20) k_crt_split_cols<20><<<g, 256, 0, st>>>((int)krows, R, p, src, ld_src, o, ldk, plane, k0, kscale, scale);
  GWB_LAUNCH_CHECK();
  count_launches(2);
  return GWB_OK;
}

extern "C" int64_t gwb_crt_work_bytes(int32_t n, int64_t M, int64_t N, int64_t K) {
  if (!supported(n) || M <= 0 || N <= 0 || K < 0) return 0;
  const int64_t tiles = ((M + CRT_M - 1) / CRT_M) * ((N + CRT_N - 1) / CRT_N);
  const int64_t splits = crt_splits(tiles, (K + CRT_KS - 1) / CRT_KS);
  return splits * n * M * ldw_of(N);
}

extern "C" int gwb_crt_gemm(int32_t n, int64_t M, int64_t N, int64_t K, const void* A, int64_t lda,
                            int64_t a_rows_cap, int64_t a_row0, const double* a_scale, const void* B, int64_t ldb,
                            int64_t b_rows_cap, int64_t b_row0, const double* b_scale, double alpha, double beta,
                            double* C, int64_t ldc, void* work, size_t work_bytes, int* status, void* stream) {
  GWB_REQUIRE(supported(n), "modulus count must be 16, 18 or 20");
  GWB_REQUIRE(M >= 0 && N >= 0 && K >= 0, "negative size");
  if (M == 0 || N == 0) return GWB_OK;
  GWB_REQUIRE(K <= CRT_MAX_K, "K beyond 2^19: the residue product could exceed the moduli's range");
  GWB_REQUIRE(A && B && a_scale && b_scale && C && status, "null pointer");
  GWB_REQUIRE(lda % 64 == 0 && ldb % 64 == 0 && lda >= K && ldb >= K, "residue ld must be a multiple of 64, >= K");
  GWB_REQUIRE(reinterpret_cast<uintptr_t>(A) % 16 == 0 && reinterpret_cast<uintptr_t>(B) % 16 == 0,
              "residue planes must be 16-byte aligned");
  GWB_REQUIRE(a_row0 >= 0 && a_row0 + M <= a_rows_cap && b_row0 >= 0 && b_row0 + N <= b_rows_cap,
              "rows beyond the residue sets");
  GWB_REQUIRE(ldc >= N, "ldc < N");
  GWB_REQUIRE(a_rows_cap <= INT32_MAX && b_rows_cap <= INT32_MAX && M <= INT32_MAX && N <= INT32_MAX,
              "size beyond the grid limits");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nsteps = (K + CRT_KS - 1) / CRT_KS;
  const int64_t Mt = (M + CRT_M - 1) / CRT_M, Nt = (N + CRT_N - 1) / CRT_N;
  GWB_REQUIRE(Mt * Nt <= INT32_MAX, "too many tiles");
  const int64_t ldw = ldw_of(N);
  int64_t splits = 1, kps = 1;
  if (nsteps > 0) {
    splits = crt_splits(Mt * Nt, nsteps);
    kps = (nsteps + splits - 1) / splits;
    splits = (nsteps + kps - 1) / kps;
  }
  GWB_REQUIRE(splits <= 65535, "too many K splits");
  GWB_REQUIRE(work && (int64_t)work_bytes >= splits * n * M * ldw, "workspace smaller than gwb_crt_work_bytes");
  GWB_REQUIRE(reinterpret_cast<uintptr_t>(work) % 16 == 0, "workspace must be 16-byte aligned");
  auto* w = static_cast<uint8_t*>(work);
  if (nsteps == 0) {
    GWB_CUDA_TRY(cudaMemsetAsync(w, 0, (size_t)(n * M * ldw), st));
  } else {
    CUtensorMap mapA, mapB;
    int rc = make_residue_map(&mapA, A, lda, a_rows_cap, n, CRT_M);
    if (rc != GWB_OK) return rc;
    rc = make_residue_map(&mapB, B, ldb, b_rows_cap, n, CRT_N);
    if (rc != GWB_OK) return rc;
    CrtArgs args;
    args.M = (int)M;
    args.N = (int)N;
    args.K = (int)K;
    args.a_row0 = (int)a_row0;
    args.b_row0 = (int)b_row0;
    args.steps_per_split = (int)kps;
    args.work = w;
    args.ldw = ldw;
    args.status = status;
    args.wait_cycles = tc_wait_cycles();
    if (n == 16) rc = launch_crt<16>(mapA, mapB, Mt, Nt, splits, args, st);
    if (n == 18) rc = launch_crt<18>(mapA, mapB, Mt, Nt, splits, args, st);
    if (n == 20) rc = launch_crt<20>(mapA, mapB, Mt, Nt, splits, args, st);
    if (rc != GWB_OK) return rc;
  }
  if (n == 16) launch_reduce<16>(M, N, splits, w, ldw, a_scale + a_row0, b_scale + b_row0, alpha, beta, C, ldc, st);
  if (n == 18) launch_reduce<18>(M, N, splits, w, ldw, a_scale + a_row0, b_scale + b_row0, alpha, beta, C, ldc, st);
  if (n == 20) launch_reduce<20>(M, N, splits, w, ldw, a_scale + a_row0, b_scale + b_row0, alpha, beta, C, ldc, st);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}
