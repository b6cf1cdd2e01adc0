// Split-precision complex GEMMs on the sm_100a tensor cores: tcgen05.mma with
// BF16 operands staged in shared memory by TMA and FP32 accumulators in tensor
// memory (TMEM).
//
// Operand format (a "plane set"). A complex matrix X (rows x cols, stored as
// complex128 or complex64) is carried as four BF16 planes per batch entry, in
// the order re_hi, re_lo, im_hi, im_lo, with hi = bf16(x) and lo = bf16(x - hi),
// so that hi + lo represents x to about 2^-17 |x|. Each plane is rows_cap x ld
// BF16, row-major, ld a multiple of 8 with columns cols..ld-1 zero; plane q of
// batch entry b starts at element (4 b + q) rows_cap ld. gwb_tc_planes writes
// them from complex rows.
//
// Products. C = alpha A op(B) + beta C, float64 complex C, with
//   op(B) = B^H: B holds N rows of length K (K-major): the A B^H products of
//                the Davidson projection (D V^H) and of the projector
//                contraction (psi P^H);
//   op(B) = B:   B holds K rows of length N (read MN-major): the updates
//                D -= C V.
// Each complex product is four real products and each real product three BF16
// ones (hi hi + hi lo + lo hi; the lo lo term is below the representation
// error), accumulated in FP32: 12 tcgen05.mma per 16-wide K step into two
// accumulators (re, im) of 128 x 128 FP32 in TMEM. Error: about
// 2^-15 sum_k |a_ik| |b_kj| plus FP32 accumulation. The solver uses these
// products only where a float64 step follows that removes their error (the
// first of the two projection passes of the expansion block).
//
// CTA: 128 threads compute a 128 x 128 complex tile of C, stepping K by 32
// through a 3-stage ring of 64 KB stages (A: 4 planes x 128 rows x 32, B: 4
// planes x 32 x 128). Each stage is filled by one (A, B^H) or four (B)
// three-dimensional TMA boxes with 64-byte rows and the 64-byte swizzle, which
// land directly in the canonical SWIZZLE_64B layouts the MMA descriptors name
// (K-major: 8-row atoms of 64 B; MN-major: 8 K-rows of 32 MN elements).
// Thread 0 issues the loads, thread 32 the MMAs;
// the four warps then read their 32 TMEM lanes each for the epilogue. Every
// mbarrier wait is bounded (by default about two seconds of SM clock;
// gwb_tc_set_wait_limit changes it); a wait that runs out ORs
// GWB_ERR_TIMEOUT (4) into *status and the CTA goes to its clean-up: the
// producer first waits (bounded) until every TMA box it issued has landed,
// all threads wait for the committed MMAs, and the TMEM is always released.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "common.cuh"
#include "tcgen05.cuh"

namespace gwb {
namespace {

constexpr int TC_M = 128;          // rows of C per CTA (MMA M)
constexpr int TC_N = 128;          // complex columns of C per CTA (MMA N)
constexpr int TC_K = 32;           // K per pipeline stage
constexpr int TC_STAGES = 3;
constexpr int TC_THREADS = 128;
constexpr int TC_ROW = TC_K * 2;                   // 64-byte rows (the swizzle span)
constexpr int TC_PLANE_A = TC_M * TC_ROW;          // one plane of an A (or B^H) tile: 128 rows x 64 B = 8 KB
constexpr int TC_A_BYTES = 4 * TC_PLANE_A;         // 32 KB
constexpr int TC_PLANE_BN = TC_K * TC_ROW;         // one plane of a 32-column block of a B tile: 32 rows x 64 B
constexpr int TC_BLOCK_BN = 4 * TC_PLANE_BN;       // 8 KB per 32-column block (four per tile)
constexpr int TC_B_BYTES = 32768;                  // B: 4 planes x 32 x 128 BF16 in either layout
constexpr int TC_STAGE_BYTES = TC_A_BYTES + TC_B_BYTES;
constexpr int TC_SMEM = TC_STAGES * TC_STAGE_BYTES + 1024;  // + alignment slack
constexpr int TC_TMEM_COLS = 2 * TC_N;             // re and im accumulators
constexpr long long TC_WAIT_CYCLES = 4000000000LL;  // default wait limit: ~2 s at 1.9 GHz

// Instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator,
// M = 128, N = 128, A K-major, B K-major (NN = false) or MN-major (NN = true).
__host__ __device__ constexpr uint32_t idesc(bool b_mn, bool negate_a) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((negate_a ? 1u : 0u) << 13) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(TC_N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(id), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tmem_ld16f(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  tmem_ld16(taddr, r);
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Where the epilogue puts the tile.
struct TcOut {
  cplx<double>* C;  // direct: C[b sC + i ldc + j] = alpha acc + beta C; split: partial slices
  int64_t ldc, sC;
  cplx<double> alpha, beta;
  int split;  // 1: write partial slice blockIdx.y of a (splits, batch, M, N) array
};

// One CTA: C tile (mt, nt) of batch entry blockIdx.z over the K steps
// [kt0, kt1) of this split. wait_cycles bounds every mbarrier wait.
// withhold >= 0 is the failure-test hook of gwb_tc_test_withhold: the
// producer issues no load for that K step of the split, so its consumer's
// wait must run out.
template <bool NN>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_zgemm_tc(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int M, int N,
               int K, int kt_per_split, TcOut out, int* status, long long wait_cycles, int withhold) {
  __shared__ __align__(8) uint64_t bar_full[TC_STAGES];
  __shared__ __align__(8) uint64_t bar_empty[TC_STAGES];
  __shared__ __align__(8) uint64_t bar_done;
  __shared__ uint32_t tmem_base_slot;
  __shared__ int abort_flag;
  extern __shared__ uint8_t dsm_raw[];
  const uint32_t dsm = (smem_u32(dsm_raw) + 1023u) & ~1023u;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Mt = (M + TC_M - 1) / TC_M;
  const int mt = blockIdx.x % Mt, nt = blockIdx.x / Mt;
  const int m0 = mt * TC_M, n0 = nt * TC_N;
  const int b = blockIdx.z;
  const int nkt = (K + TC_K - 1) / TC_K;
  const int kt0 = blockIdx.y * kt_per_split;
  const int kt1 = min(nkt, kt0 + kt_per_split);

  if (tid == 0) {
    for (int s = 0; s < TC_STAGES; ++s) {
      mbar_init(smem_u32(&bar_full[s]), 1);
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    mbar_init(smem_u32(&bar_done), 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                 "r"((uint32_t)TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_slot;

  if (tid == 0 && kt1 > kt0) {
    // producer: TMA boxes of stage s for K step kt; last_round[s] is the
    // last round for which stage s was armed (its loads may be in flight)
    int last_round[TC_STAGES];
#pragma unroll
    for (int s = 0; s < TC_STAGES; ++s) last_round[s] = -1;
    for (int kt = kt0; kt < kt1; ++kt) {
      const int i = kt - kt0, s = i % TC_STAGES;
      if (i >= TC_STAGES && !mbar_wait(smem_u32(&bar_empty[s]), ((i / TC_STAGES) - 1) & 1, wait_cycles)) {
        abort_flag = 1;
        atomicOr(status, GWB_ERR_TIMEOUT);
        break;
      }
      if (*(volatile int*)&abort_flag) break;
      if (i == withhold) continue;
      last_round[s] = i / TC_STAGES;
      const uint32_t full = smem_u32(&bar_full[s]);
      const uint32_t sa = dsm + s * TC_STAGE_BYTES, sb = sa + TC_A_BYTES;
      mbar_expect_tx(full, TC_STAGE_BYTES);
      const int k0 = kt * TC_K;
      // A: [plane][128 rows][64 B]
      tma_load_3d(sa, &mapA, full, k0, m0, 4 * b);
      if (NN) {
        // B rows k0..k0+31, one box per block of 32 columns: [block][plane][32 rows][64 B]
#pragma unroll
        for (int g = 0; g < TC_N / 32; ++g) tma_load_3d(sb + g * TC_BLOCK_BN, &mapB, full, n0 + 32 * g, k0, 4 * b);
      } else {
        tma_load_3d(sb, &mapB, full, k0, n0, 4 * b);
      }
    }
    // no bulk copy may still be landing in shared memory when the CTA leaves:
    // wait (bounded) for the last armed phase of every stage. Only this thread
    // arms the full barriers, so a landed phase r leaves the barrier in phase
    // r + 1 and the parity test of phase r holds from then on.
#pragma unroll
    for (int s = 0; s < TC_STAGES; ++s)
      if (last_round[s] >= 0 && !mbar_wait(smem_u32(&bar_full[s]), last_round[s] & 1, wait_cycles))
        atomicOr(status, GWB_ERR_TIMEOUT);
  } else if (tid == 32) {
    // MMA issuer
    constexpr uint32_t ID_POS = idesc(NN, false), ID_NEG = idesc(NN, true);
    // terms (a plane, b plane, accumulator, negate): plane 0 = re, 2 = im
    // B^H: re += Ar Br + Ai Bi, im += Ai Br - Ar Bi;  B: re += Ar Br - Ai Bi, im += Ar Bi + Ai Br
    constexpr int TA[4] = {0, 2, NN ? 0 : 2, NN ? 2 : 0};
    constexpr int TB[4] = {0, 2, NN ? 2 : 0, NN ? 0 : 2};
    constexpr int TACC[4] = {0, 0, 1, 1};
    constexpr bool TNEG[4] = {false, NN, false, !NN};
    constexpr int SA[3] = {0, 0, 1}, SB[3] = {0, 1, 0};  // hi hi, hi lo, lo hi
    for (int kt = kt0; kt < kt1; ++kt) {
      const int i = kt - kt0, s = i % TC_STAGES;
      if (!mbar_wait(smem_u32(&bar_full[s]), (i / TC_STAGES) & 1, wait_cycles)) {
        abort_flag = 1;
        atomicOr(status, GWB_ERR_TIMEOUT);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = dsm + s * TC_STAGE_BYTES, sb = sa + TC_A_BYTES;
#pragma unroll
      for (int ks = 0; ks < TC_K / 16; ++ks) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
#pragma unroll
          for (int sp = 0; sp < 3; ++sp) {
            const int qa = TA[t] + SA[sp], qb = TB[t] + SB[sp];
            // K-major: 8-row atoms 512 B apart, the 16-wide K step 32 B into the
            // 64-byte row; MN-major: K-row groups 512 B apart, 32-column blocks
            // TC_BLOCK_BN apart, the K step 16 rows = 1024 B
            const uint64_t da = sdesc(sa + qa * TC_PLANE_A + ks * 32, 16, 512);
            const uint64_t db = NN ? sdesc(sb + qb * TC_PLANE_BN + ks * 1024, TC_BLOCK_BN, 512)
                                   : sdesc(sb + qb * TC_PLANE_A + ks * 32, 16, 512);
            // the first product into each accumulator overwrites it
            const bool first = (i == 0 && ks == 0 && (t == 0 || t == 2) && sp == 0);
            mma_bf16(tmem + TACC[t] * TC_N, da, db, TNEG[t] ? ID_NEG : ID_POS, first ? 0u : 1u);
          }
        }
      }
      mma_commit(smem_u32(&bar_empty[s]));
    }
    mma_commit(smem_u32(&bar_done));
  }
  __syncwarp();

  // epilogue: warp w holds rows m0 + 32 w + lane in TMEM lanes 32 w ..; the
  // tile goes TMEM -> shared memory (the pipeline buffers, idle once the
  // last MMA has completed; rows padded to 129 float2 so the staging stores
  // are conflict-free) -> whole rows of C, so that the global reads and writes
  // are coalesced
  const bool have = kt1 > kt0;
  bool ok = have && mbar_wait(smem_u32(&bar_done), 0, wait_cycles);
  if (have && !ok) atomicOr(status, GWB_ERR_TIMEOUT);
  if (*(volatile int*)&abort_flag) ok = false;
  ok = __syncthreads_and(ok || !have) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  constexpr int SROW = TC_N + 1;
  float2* stage = reinterpret_cast<float2*>(dsm_raw + (dsm - smem_u32(dsm_raw)));
  const int rl_own = warp * 32 + lane;
  for (int c = 0; c < TC_N; c += 16) {
    float re[16], im[16];
    __syncwarp();  // the TMEM loads are warp-collective
    if (have) {    // CTA-uniform
      tmem_ld16f(tmem + ((uint32_t)(warp * 32) << 16) + c, re);
      tmem_ld16f(tmem + ((uint32_t)(warp * 32) << 16) + TC_N + c, im);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    } else {
#pragma unroll
      for (int e = 0; e < 16; ++e) re[e] = im[e] = 0.f;
    }
    if (ok) {
#pragma unroll
      for (int e = 0; e < 16; ++e) stage[rl_own * SROW + c + e] = make_float2(re[e], im[e]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TC_TMEM_COLS)
                 : "memory");
  }
  if (!ok) return;
  // warp w writes local rows w, w + 4, ...; four rows at a time, loads first
  constexpr int RU = 4, Q = TC_N / 32;
  const bool use_beta = out.beta.x != 0.0 || out.beta.y != 0.0;
  for (int rl0 = warp; rl0 < TC_M; rl0 += 4 * RU) {
    cplx<double> old[RU][Q];
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const int rl = rl0 + 4 * u, row = m0 + rl;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int j = n0 + lane + 32 * q;
        old[u][q] = mk<double>(0.0, 0.0);
        if (!out.split && use_beta && row < M && j < N)
          old[u][q] = out.C[b * out.sC + (int64_t)row * out.ldc + j];
      }
    }
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const int rl = rl0 + 4 * u, row = m0 + rl;
      if (row >= M) continue;
      const float2* srow = stage + rl * SROW;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int jl = lane + 32 * q, j = n0 + jl;
        if (j >= N) continue;
        const float2 a = srow[jl];
        if (out.split) {
          out.C[(((int64_t)blockIdx.y * gridDim.z + b) * M + row) * (int64_t)N + j] = mk<double>(a.x, a.y);
        } else {
          cplx<double> v = out.alpha * mk<double>((double)a.x, (double)a.y);
          if (use_beta) v = v + out.beta * old[u][q];
          out.C[b * out.sC + (int64_t)row * out.ldc + j] = v;
        }
      }
    }
  }
}

__global__ void k_tc_reduce(int M, int N, int nsplit, int batch, const cplx<double>* __restrict__ part,
                            cplx<double> alpha, cplx<double> beta, cplx<double>* __restrict__ C, int64_t ldc,
                            int64_t sC) {
  const int64_t total = (int64_t)batch * M * N;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(idx / ((int64_t)M * N));
    const int64_t r = idx % ((int64_t)M * N);
    const int i = (int)(r / N), j = (int)(r % N);
    cplx<double> a = mk<double>(0.0, 0.0);
    for (int s = 0; s < nsplit; ++s) a = a + part[(int64_t)s * total + idx];
    cplx<double>* c = C + b * sC + (int64_t)i * ldc + j;
    cplx<double> v = alpha * a;
    if (beta.x != 0.0 || beta.y != 0.0) v = v + beta * (*c);
    *c = v;
  }
}

// BF16 hi/lo split of x: x ~ hi + lo.
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn((float)x);
  lo = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hi)));
}

// rows [0, rows) x cols of src -> plane rows [row0, row0 + rows), zeros in
// columns cols..ld-1; one thread per 8 columns of one row.
template <typename S>
__global__ void k_tc_planes(int nk, int rows, int cols, const S* __restrict__ src, int64_t src_ld, int64_t src_ks,
                            double conj_sign, __nv_bfloat16* __restrict__ planes, int64_t ld, int64_t rows_cap,
                            int row0) {
  const int64_t groups = ld / 8;
  const int64_t total = (int64_t)nk * rows * groups;
  const int64_t plane = rows_cap * ld;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(idx / ((int64_t)rows * groups));
    const int64_t rem = idx % ((int64_t)rows * groups);
    const int r = (int)(rem / groups);
    const int c0 = (int)(rem % groups) * 8;
    __align__(16) __nv_bfloat16 rh[8], rl[8], ih[8], il[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      double xr = 0.0, xi = 0.0;
      if (c0 + e < cols) {
        const S v = src[k * src_ks + (int64_t)r * src_ld + c0 + e];
        xr = (double)v.x;
        xi = conj_sign * (double)v.y;
      }
      split_bf16(xr, rh[e], rl[e]);
      split_bf16(xi, ih[e], il[e]);
    }
    __nv_bfloat16* dst = planes + (int64_t)4 * k * plane + (int64_t)(row0 + r) * ld + c0;
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(rh);
    *reinterpret_cast<uint4*>(dst + plane) = *reinterpret_cast<const uint4*>(rl);
    *reinterpret_cast<uint4*>(dst + 2 * plane) = *reinterpret_cast<const uint4*>(ih);
    *reinterpret_cast<uint4*>(dst + 3 * plane) = *reinterpret_cast<const uint4*>(il);
  }
}

// planes of bd = becp D for the nonlocal term: rows (k, b) of becp
// (complex128, nproj per row) times the real nproj x nproj D, split into the
// four BF16 planes of a (nk, 4, nb, ldq) set, columns nproj..ldq-1 zero; TB_R
// rows per CTA share each read of D.
constexpr int TB_R = 4;
__global__ void __launch_bounds__(256) k_becp_d_planes(int nk, int nb, int nproj, const cplx<double>* __restrict__ becp,
                                                       const double* __restrict__ D, __nv_bfloat16* __restrict__ planes,
                                                       int64_t ldq) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<double>* rows = reinterpret_cast<cplx<double>*>(smem_raw);  // TB_R x nproj
  const int64_t r0 = (int64_t)blockIdx.x * TB_R;
  const int64_t nrows = (int64_t)nk * nb;
  for (int i = threadIdx.x; i < TB_R * nproj; i += blockDim.x) {
    const int64_t r = r0 + i / nproj;
    rows[i] = r < nrows ? becp[r * nproj + i % nproj] : mk<double>(0.0, 0.0);
  }
  __syncthreads();
  const int64_t plane = (int64_t)nb * ldq;
  for (int q = threadIdx.x; q < ldq; q += blockDim.x) {
    double ar[TB_R], ai[TB_R];
#pragma unroll
    for (int r = 0; r < TB_R; ++r) ar[r] = ai[r] = 0.0;
    if (q < nproj) {
      for (int p = 0; p < nproj; ++p) {
        const double d = D[(int64_t)p * nproj + q];
#pragma unroll
        for (int r = 0; r < TB_R; ++r) {
          const cplx<double> v = rows[r * nproj + p];
          ar[r] += v.x * d;
          ai[r] += v.y * d;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < TB_R; ++r) {
      const int64_t row = r0 + r;
      if (row >= nrows) break;
      const int64_t k = row / nb, b = row % nb;
      __nv_bfloat16 h, l;
      __nv_bfloat16* base = planes + 4 * k * plane + b * ldq + q;
      split_bf16(ar[r], h, l);
      base[0] = h;
      base[plane] = l;
      split_bf16(ai[r], h, l);
      base[2 * plane] = h;
      base[3 * plane] = l;
    }
  }
}

// 3-D view of a plane set: (columns, rows, 4 x batch planes); box
// (32, box_rows, 4): 32 columns (64 B, the swizzle span) of box_rows rows of
// all four planes of one batch entry, 64-byte swizzled in shared memory.
int make_plane_map(CUtensorMap* map, const void* base, int64_t ld, int64_t rows, int64_t rows_cap, int64_t batch,
                   int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return GWB_ERR_CUDA;
  }
  cuuint64_t dims[3] = {(cuuint64_t)ld, (cuuint64_t)rows, (cuuint64_t)(4 * batch)};
  cuuint64_t strides[2] = {(cuuint64_t)(ld * 2), (cuuint64_t)(rows_cap * ld * 2)};
  cuuint32_t box[3] = {(cuuint32_t)TC_K, (cuuint32_t)box_rows, 4u};
  cuuint32_t es[3] = {1u, 1u, 1u};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed with CUresult " + std::to_string((int)r));
    return GWB_ERR_CUDA;
  }
  return GWB_OK;
}

// Split count for the A B^H form: each CTA holds a whole SM (shared memory),
// so the grid runs in waves of 148; pick the split count (at most one per 8 K
// steps) whose last wave is fullest, preferring fewer splits on ties.
int64_t pick_splits(int64_t tiles, int64_t nkt) {
  if (tiles >= 2 * 148) return 1;
  const int64_t smax = std::max<int64_t>(1, std::min<int64_t>(64, nkt / 8));
  int64_t best = 1;
  double best_eff = -1.0;
  for (int64_t s = 1; s <= smax; ++s) {
    const int64_t ctas = tiles * s, waves = (ctas + 147) / 148;
    // occupancy of the waves, less a small cost per split (partial sums)
    const double eff = (double)ctas / (double)(waves * 148) - 0.004 * (double)s;
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = s;
    }
  }
  return best;
}

}  // namespace

// bd = becp D written as BF16 planes (the A operand of the nonlocal update
// out += bd P); used by the Hamiltonian apply.
int tc_becp_d_planes(int nk, int nb, int nproj, const cplx<double>* becp, const double* D, void* planes, int64_t ldq,
                     cudaStream_t st) {
  const int64_t rows = (int64_t)nk * nb;
  const unsigned blocks = (unsigned)((rows + TB_R - 1) / TB_R);
  const size_t sm = (size_t)TB_R * nproj * sizeof(cplx<double>);
  GWB_CUDA_TRY(allow_smem(k_becp_d_planes));
  k_becp_d_planes<<<blocks, 256, sm, st>>>(nk, nb, nproj, becp, D, (__nv_bfloat16*)planes, ldq);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

// Wait limit of the pipeline barriers (SM clock cycles) and the
// failure-test hook (K step whose load is withheld; -1: none), read at launch.
static std::atomic<long long> g_wait_cycles{TC_WAIT_CYCLES};
static std::atomic<int> g_withhold{-1};
long long tc_wait_cycles() { return g_wait_cycles.load(); }
int tc_withhold() { return g_withhold.load(); }

}  // namespace gwb

using namespace gwb;

extern "C" int gwb_tc_set_wait_limit(int64_t cycles) {
  GWB_REQUIRE(cycles > 0, "the wait limit must be positive");
  g_wait_cycles.store((long long)cycles);
  return GWB_OK;
}

extern "C" int gwb_tc_test_withhold(int32_t kstep) {
  GWB_REQUIRE(kstep >= -1, "kstep must be -1 (off) or a K step index");
  g_withhold.store((int)kstep);
  return GWB_OK;
}

extern "C" int gwb_tc_planes(int64_t nk, int64_t rows, int64_t cols, const void* src, int64_t src_ld,
                             int64_t src_kstride, int dtype, int conj, void* planes, int64_t ld, int64_t rows_cap,
                             int64_t row0, void* stream) {
  GWB_REQUIRE(nk >= 0 && rows >= 0 && cols >= 0 && row0 >= 0, "negative size");
  if (nk == 0 || rows == 0) return GWB_OK;
  GWB_REQUIRE(src && planes, "null pointer");
  GWB_REQUIRE(ld % 8 == 0 && ld >= cols && ld > 0, "plane ld must be a positive multiple of 8 covering the columns");
  GWB_REQUIRE(row0 + rows <= rows_cap, "rows beyond the plane capacity");
  GWB_REQUIRE(reinterpret_cast<uintptr_t>(planes) % 16 == 0, "planes must be 16-byte aligned");
  GWB_REQUIRE(dtype == GWB_C64 || dtype == GWB_C128, "dtype must be GWB_C64 or GWB_C128");
  const int64_t total = nk * rows * (ld / 8);
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  cudaStream_t st = (cudaStream_t)stream;
  const double cs = conj ? -1.0 : 1.0;
  if (dtype == GWB_C128)
    k_tc_planes<cplx<double>><<<blocks, 256, 0, st>>>((int)nk, (int)rows, (int)cols, (const cplx<double>*)src, src_ld,
                                                      src_kstride, cs, (__nv_bfloat16*)planes, ld, rows_cap,
                                                      (int)row0);
  else
    k_tc_planes<cplx<float>><<<blocks, 256, 0, st>>>((int)nk, (int)rows, (int)cols, (const cplx<float>*)src, src_ld,
                                                     src_kstride, cs, (__nv_bfloat16*)planes, ld, rows_cap,
                                                     (int)row0);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

extern "C" int64_t gwb_zgemm_tc_work_bytes(int opB, int64_t M, int64_t N, int64_t K, int64_t batch) {
  if (opB != 2 || M <= 0 || N <= 0 || K <= 0 || batch <= 0) return 0;
  // the largest split count gwb_zgemm_tc picks for A B^H
  const int64_t tiles = ((M + TC_M - 1) / TC_M) * ((N + TC_N - 1) / TC_N) * batch;
  const int64_t nkt = (K + TC_K - 1) / TC_K;
  const int64_t splits = pick_splits(tiles, nkt);
  return splits > 1 ? splits * batch * M * N * 16 : 0;
}

extern "C" int gwb_zgemm_tc(int opB, int64_t M, int64_t N, int64_t K, double alpha_re, double alpha_im,
                            const void* A_planes, int64_t lda, int64_t a_rows_cap, const void* B_planes, int64_t ldb,
                            int64_t b_rows_cap, double beta_re, double beta_im, void* C, int64_t ldc, int64_t strideC,
                            int64_t batch, void* work, size_t work_bytes, int* status, void* stream) {
  GWB_REQUIRE(opB == 0 || opB == 2, "opB must be 0 (B) or 2 (B^H)");
  GWB_REQUIRE(M >= 0 && N >= 0 && K >= 0 && batch >= 0, "negative size");
  if (M == 0 || N == 0 || batch == 0) return GWB_OK;
  GWB_REQUIRE(A_planes && B_planes && C && status, "null pointer");
  GWB_REQUIRE(lda % 8 == 0 && ldb % 8 == 0, "plane ld must be a multiple of 8");
  GWB_REQUIRE(reinterpret_cast<uintptr_t>(A_planes) % 16 == 0 && reinterpret_cast<uintptr_t>(B_planes) % 16 == 0,
              "planes must be 16-byte aligned");
  const bool nn = opB == 0;
  GWB_REQUIRE(a_rows_cap >= M && lda >= K, "A planes smaller than M x K");
  if (nn)
    GWB_REQUIRE(b_rows_cap >= K && ldb >= N, "B planes smaller than K x N");
  else
    GWB_REQUIRE(b_rows_cap >= N && ldb >= K, "B planes smaller than N x K");
  GWB_REQUIRE(M <= INT32_MAX && N <= INT32_MAX && K <= INT32_MAX && batch <= 65535, "size beyond the grid limits");
  cudaStream_t st = (cudaStream_t)stream;
  const cplx<double> alpha = mk<double>(alpha_re, alpha_im), beta = mk<double>(beta_re, beta_im);
  if (K == 0) {
    // C = beta C
    const int64_t total = M * N * batch;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 4096);
    k_tc_reduce<<<blocks, 256, 0, st>>>((int)M, (int)N, 0, (int)batch, nullptr, alpha, beta, (cplx<double>*)C, ldc,
                                        strideC);
    GWB_LAUNCH_CHECK();
    count_launches(1);
    return GWB_OK;
  }
  CUtensorMap mapA, mapB;
  int rc = make_plane_map(&mapA, A_planes, lda, M, a_rows_cap, batch, TC_M);
  if (rc != GWB_OK) return rc;
  rc = nn ? make_plane_map(&mapB, B_planes, ldb, K, b_rows_cap, batch, TC_K)
          : make_plane_map(&mapB, B_planes, ldb, N, b_rows_cap, batch, TC_N);
  if (rc != GWB_OK) return rc;
  const int64_t Mt = (M + TC_M - 1) / TC_M, Nt = (N + TC_N - 1) / TC_N;
  GWB_REQUIRE(Mt * Nt <= INT32_MAX, "too many tiles");
  const int64_t nkt = (K + TC_K - 1) / TC_K;
  int64_t splits = 1;
  if (!nn) {
    const int64_t tiles = Mt * Nt * batch;
    splits = pick_splits(tiles, nkt);
    while (splits > 1 && (!work || splits * batch * M * N * 16 > (int64_t)work_bytes)) --splits;
  }
  const int64_t kps = (nkt + splits - 1) / splits;
  splits = (nkt + kps - 1) / kps;
  TcOut out;
  out.alpha = alpha;
  out.beta = beta;
  out.ldc = ldc;
  out.sC = strideC;
  out.split = splits > 1;
  out.C = splits > 1 ? (cplx<double>*)work : (cplx<double>*)C;
  dim3 grid((unsigned)(Mt * Nt), (unsigned)splits, (unsigned)batch);
  if (nn) {
    GWB_CUDA_TRY(allow_smem(k_zgemm_tc<true>));
    k_zgemm_tc<true><<<grid, TC_THREADS, TC_SMEM, st>>>(mapA, mapB, (int)M, (int)N, (int)K, (int)kps, out, status,
                                                       g_wait_cycles.load(), g_withhold.load());
  } else {
    GWB_CUDA_TRY(allow_smem(k_zgemm_tc<false>));
    k_zgemm_tc<false><<<grid, TC_THREADS, TC_SMEM, st>>>(mapA, mapB, (int)M, (int)N, (int)K, (int)kps, out, status,
                                                        g_wait_cycles.load(), g_withhold.load());
  }
  GWB_LAUNCH_CHECK();
  count_launches(1);
  if (splits > 1) {
    const int64_t total = M * N * batch;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 4096);
    k_tc_reduce<<<blocks, 256, 0, st>>>((int)M, (int)N, (int)splits, (int)batch, (const cplx<double>*)work, alpha,
                                        beta, (cplx<double>*)C, ldc, strideC);
    GWB_LAUNCH_CHECK();
    count_launches(1);
  }
  return GWB_OK;
}
