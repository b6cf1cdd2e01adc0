// Learned Davidson preconditioner: a per-plane-wave MLP with BF16 weights and
// activations and FP32 accumulation, trained on the GPU by these kernels.
//
//   features u (4) -> 64 -> 64 -> 64 -> 1, SiLU between layers
//   K(G) = TPA(x) * exp(clamp(o, -3, 3)),  d = K r / |K r|
//
// Features of plane wave G of band b (one shared definition for logging,
// training and inference, gwb_precond_features):
//   u0 = log(1 + x),            x = t_G / t_b        (|k+G|^2, kinetic of psi)
//   u1 = clamp(eps_b / t_b, -8, 8) / 4               (band eigenvalue)
//   u2 = log10(|r_G| / r_rms + 1e-6) / 3             (residual amplitude)
//   u3 = log10(max(t_b, 1e-3) / 10)                  (kinetic scale of psi)
// with t_b = <x_b|T|x_b> and r_rms = |r_b| / sqrt(npw).
//
// Parameters: one float32 master array of GWB_MLP_NPARAM values,
//   W1[64][4] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64] b4
// rounded to BF16 on load for the forward pass (straight-through gradients).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "tcgen05.cuh"

namespace gwb {

constexpr int HID = 64, NIN = 4;
constexpr int O_W1 = 0, O_B1 = O_W1 + HID * NIN, O_W2 = O_B1 + HID, O_B2 = O_W2 + HID * HID, O_W3 = O_B2 + HID,
              O_B3 = O_W3 + HID * HID, O_W4 = O_B3 + HID, O_B4 = O_W4 + HID, NPARAM = O_B4 + 1;

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float sigm(float z) { return 1.f / (1.f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigm(z);
  return s * (1.f + z * (1.f - s));
}

// float32 with fast intrinsics: the values feed a BF16 network
__device__ __forceinline__ void features(double tg, double tb, double eps, double rabs, double rrms, float* u) {
  const float t = (float)fmax(tb, 1e-12);
  const float x = (float)tg / t;
  const float inv_ln10 = 0.43429448190325176f;
  u[0] = __logf(1.f + x);
  u[1] = fminf(fmaxf((float)eps / t, -8.f), 8.f) * 0.25f;
  u[2] = __logf((float)(rabs / fmax(rrms, 1e-300)) + 1e-6f) * (inv_ln10 / 3.f);
  u[3] = __logf(fmaxf((float)tb, 1e-3f) * 0.1f) * inv_ln10;
}

__device__ __forceinline__ double tpa_coeff(double tg, double tb) {
  const double x = tg / fmax(tb, 1e-12);
  const double x2 = x * x;
  const double p = 27.0 + 18.0 * x + 12.0 * x2 + 8.0 * x2 * x;
  return p / (p + 16.0 * x2 * x2);
}

// BF16-rounded copy of the parameters into shared memory (floats).
__device__ void load_params(const float* __restrict__ P, float* s) {
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) s[i] = bf(P[i]);
  __syncthreads();
}

// Forward of one sample by one thread: a3 kept for nothing; returns o.
__device__ float forward_one(const float* s, const float* u) {
  float a0[NIN], h1[HID], h2[HID];
#pragma unroll
  for (int i = 0; i < NIN; ++i) a0[i] = bf(u[i]);
#pragma unroll 4
  for (int o = 0; o < HID; ++o) {
    float z = s[O_B1 + o];
#pragma unroll
    for (int i = 0; i < NIN; ++i) z = fmaf(s[O_W1 + o * NIN + i], a0[i], z);
    h1[o] = bf(silu(z));
  }
#pragma unroll 2
  for (int o = 0; o < HID; ++o) {
    float z = s[O_B2 + o];
#pragma unroll
    for (int i = 0; i < HID; ++i) z = fmaf(s[O_W2 + o * HID + i], h1[i], z);
    h2[o] = bf(silu(z));
  }
  float out = s[O_B4];
#pragma unroll 2
  for (int o = 0; o < HID; ++o) {
    float z = s[O_B3 + o];
#pragma unroll
    for (int i = 0; i < HID; ++i) z = fmaf(s[O_W3 + o * HID + i], h2[i], z);
    out = fmaf(s[O_W4 + o], bf(silu(z)), out);
  }
  return out;
}

__global__ void __launch_bounds__(256) k_mlp_forward(const float* __restrict__ P, int n, const float* __restrict__ U,
                                                     float* __restrict__ out) {
  extern __shared__ float sp[];
  load_params(P, sp);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float u[NIN];
#pragma unroll
    for (int q = 0; q < NIN; ++q) u[q] = U[(int64_t)i * NIN + q];
    out[i] = forward_one(sp, u);
  }
}

// Forward + backward over tiles of TS samples: with targets Y the loss is
// sum_i w_i (o_i - y_i)^2; with Y == NULL, Wt holds dL/do_i of any loss.
// Activations of a tile stay in shared memory; weight gradients accumulate per
// CTA in shared memory and are added to G once per CTA.
constexpr int TS = 32;
__global__ void __launch_bounds__(256) k_mlp_loss_grad(const float* __restrict__ P, int n, const float* __restrict__ U,
                                                       const float* __restrict__ Y, const float* __restrict__ Wt,
                                                       float* __restrict__ G, float* __restrict__ loss) {
  extern __shared__ float sm[];
  float* sp = sm;                      // NPARAM   bf16-rounded params
  float* sg = sp + NPARAM;             // NPARAM   gradient accumulators
  float* a0 = sg + NPARAM;             // TS*NIN
  float* z1 = a0 + TS * NIN;           // TS*HID  (pre-activations)
  float* a1 = z1 + TS * HID;
  float* z2 = a1 + TS * HID;
  float* a2 = z2 + TS * HID;
  float* z3 = a2 + TS * HID;
  float* a3 = z3 + TS * HID;
  float* dz = a3 + TS * HID;           // TS*HID  (current layer dz)
  float* dz2 = dz + TS * HID;          // TS*HID
  float* dout = dz2 + TS * HID;        // TS
  __shared__ float sloss;
  load_params(P, sp);
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) sg[i] = 0.f;
  if (threadIdx.x == 0) sloss = 0.f;
  __syncthreads();
  const int ntiles = (n + TS - 1) / TS;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int s0 = tile * TS;
    for (int i = threadIdx.x; i < TS * NIN; i += blockDim.x) {
      const int s = s0 + i / NIN;
      a0[i] = s < n ? bf(U[(int64_t)s * NIN + i % NIN]) : 0.f;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < TS * HID; i += blockDim.x) {
      const int s = i / HID, o = i % HID;
      float z = sp[O_B1 + o];
      for (int q = 0; q < NIN; ++q) z = fmaf(sp[O_W1 + o * NIN + q], a0[s * NIN + q], z);
      z1[i] = z;
      a1[i] = bf(silu(z));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < TS * HID; i += blockDim.x) {
      const int s = i / HID, o = i % HID;
      float z = sp[O_B2 + o];
      for (int q = 0; q < HID; ++q) z = fmaf(sp[O_W2 + o * HID + q], a1[s * HID + q], z);
      z2[i] = z;
      a2[i] = bf(silu(z));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < TS * HID; i += blockDim.x) {
      const int s = i / HID, o = i % HID;
      float z = sp[O_B3 + o];
      for (int q = 0; q < HID; ++q) z = fmaf(sp[O_W3 + o * HID + q], a2[s * HID + q], z);
      z3[i] = z;
      a3[i] = bf(silu(z));
    }
    __syncthreads();
    if (threadIdx.x < TS) {
      const int s = threadIdx.x, gs = s0 + s;
      float o = sp[O_B4];
      for (int q = 0; q < HID; ++q) o = fmaf(sp[O_W4 + q], a3[s * HID + q], o);
      float d = 0.f;
      if (gs < n) {
        if (Y) {
          const float e = o - Y[gs];
          d = 2.f * Wt[gs] * e;
          atomicAdd(&sloss, Wt[gs] * e * e);
        } else {
          d = Wt[gs];  // caller-supplied dL/do
        }
      }
      dout[s] = d;
    }
    __syncthreads();
    // output layer
    for (int q = threadIdx.x; q < HID; q += blockDim.x) {
      float g = 0.f;
      for (int s = 0; s < TS; ++s) g = fmaf(dout[s], a3[s * HID + q], g);
      sg[O_W4 + q] += g;
    }
    if (threadIdx.x == 0) {
      float g = 0.f;
      for (int s = 0; s < TS; ++s) g += dout[s];
      sg[O_B4] += g;
    }
    for (int i = threadIdx.x; i < TS * HID; i += blockDim.x) {
      const int s = i / HID, q = i % HID;
      dz[i] = dout[s] * sp[O_W4 + q] * dsilu(z3[i]);
    }
    __syncthreads();
    // layer 3: W3 grads, propagate to dz2
    for (int i = threadIdx.x; i < HID * HID; i += blockDim.x) {
      const int o = i / HID, q = i % HID;
      float g = 0.f;
      for (int s = 0; s < TS; ++s) g = fmaf(dz[s * HID + o], a2[s * HID + q], g);
      sg[O_W3 + i] += g;
    }
    for (int o = threadIdx.x; o < HID; o += blockDim.x) {
      float g = 0.f;
      for (int s = 0; s < TS; ++s) g += dz[s * HID + o];
      sg[O_B3 + o] += g;
    }
    for (int i = threadIdx.x; i < TS * HID; i += blockDim.x) {
      const int s = i / HID, q = i % HID;
      float g = 0.f;
      for (int o = 0; o < HID; ++o) g = fmaf(sp[O_W3 + o * HID + q], dz[s * HID + o], g);
      dz2[i] = g * dsilu(z2[i]);
    }
    __syncthreads();
    // layer 2
    for (int i = threadIdx.x; i < HID * HID; i += blockDim.x) {
      const int o = i / HID, q = i % HID;
      float g = 0.f;
      for (int s = 0; s < TS; ++s) g = fmaf(dz2[s * HID + o], a1[s * HID + q], g);
      sg[O_W2 + i] += g;
    }
    for (int o = threadIdx.x; o < HID; o += blockDim.x) {
      float g = 0.f;
      for (int s = 0; s < TS; ++s) g += dz2[s * HID + o];
      sg[O_B2 + o] += g;
    }
    for (int i = threadIdx.x; i < TS * HID; i += blockDim.x) {
      const int s = i / HID, q = i % HID;
      float g = 0.f;
      for (int o = 0; o < HID; ++o) g = fmaf(sp[O_W2 + o * HID + q], dz2[s * HID + o], g);
      dz[i] = g * dsilu(z1[i]);
    }
    __syncthreads();
    // layer 1
    for (int i = threadIdx.x; i < HID * NIN; i += blockDim.x) {
      const int o = i / NIN, q = i % NIN;
      float g = 0.f;
      for (int s = 0; s < TS; ++s) g = fmaf(dz[s * HID + o], a0[s * NIN + q], g);
      sg[O_W1 + i] += g;
    }
    for (int o = threadIdx.x; o < HID; o += blockDim.x) {
      float g = 0.f;
      for (int s = 0; s < TS; ++s) g += dz[s * HID + o];
      sg[O_B1 + o] += g;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) atomicAdd(&G[i], sg[i]);
  if (threadIdx.x == 0 && Y) atomicAdd(loss, sloss);
}

// Adam (Kingma & Ba, 2015) on the float32 master parameters.
__global__ void k_mlp_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M,
                           float* __restrict__ V, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = G[i];
    const float m = b1 * M[i] + (1.f - b1) * g;
    const float v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
  }
}

// Features of the selected rows at every plane wave: U (nk, n_add, npw, 4).
__global__ void __launch_bounds__(256) k_features(int npw, int nb, int n_add, const cplx<double>* __restrict__ x,
                                                  int64_t xk, const cplx<double>* __restrict__ r, int64_t rk,
                                                  const double* __restrict__ t, const double* __restrict__ eig,
                                                  const int* __restrict__ sel, float* __restrict__ U) {
  __shared__ double red[8];
  __shared__ double sv[2];
  const int k = blockIdx.x / n_add, s = blockIdx.x % n_add;
  const int b = sel[(int64_t)k * n_add + s];
  const cplx<double>* xr = x + k * xk + (int64_t)b * npw;
  const cplx<double>* rr = r + k * rk + (int64_t)b * npw;
  const double* tk = t + (int64_t)k * npw;
  double tb = 0.0, r2 = 0.0;
  for (int g = threadIdx.x; g < npw; g += blockDim.x) {
    tb += tk[g] * norm2(xr[g]);
    r2 += norm2(rr[g]);
  }
  // two block sums
  for (int o = 16; o > 0; o >>= 1) {
    tb += __shfl_xor_sync(0xffffffffu, tb, o);
    r2 += __shfl_xor_sync(0xffffffffu, r2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = tb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < 8; ++w) a += red[w];
    sv[0] = a;
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = r2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < 8; ++w) a += red[w];
    sv[1] = a;
  }
  __syncthreads();
  const double tbv = sv[0], rrms = sqrt(sv[1] / npw), eps = eig[(int64_t)k * nb + b];
  float* Uo = U + ((int64_t)k * n_add + s) * npw * NIN;
  for (int g = threadIdx.x; g < npw; g += blockDim.x) {
    float u[NIN];
    features(tk[g], tbv, eps, sqrt(norm2(rr[g])), rrms, u);
#pragma unroll
    for (int q = 0; q < NIN; ++q) Uo[(int64_t)g * NIN + q] = u[q];
  }
}

// ---------------------------------------------------------------------------
// Tensor-core inference (mma.sync m16n8k16, BF16 in, FP32 accumulate). A warp
// evaluates 16 plane waves at a time: layer 1 (4 -> 64) on the CUDA cores
// writes its SiLU outputs straight into the A fragments of layer 2; the FP32
// accumulators of n-tiles 2j and 2j+1 of a layer are, element for element,
// the A fragment of k-tile j of the next layer, so activations never leave
// registers; layer 4 (64 -> 1) is a quad shuffle reduction.
constexpr int WSTR = HID + 8;  // padded row stride (BF16) of W2/W3 in shared memory: conflict-free B loads

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&v);
}

__device__ __forceinline__ void mma_bf16(float* d, const unsigned* a, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// SiLU as h + h tanh(h), h = z/2: one SFU op (tanh.approx.f32, |rel. err| < 2^-10.9)
// per activation instead of an exponential and a reciprocal; well inside the
// BF16 rounding the activations get next.
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float silu_fast(float z) {
  const float h = 0.5f * z;
  return fmaf(h, tanh_approx(h), h);
}

// One hidden 64 -> 64 layer: acc[nt][4] = bias + A . W^T, then SiLU and BF16
// packing into the next A fragments an[kt][4].
__device__ __forceinline__ void tc_layer(const unsigned (&a)[4][4], const __nv_bfloat16* __restrict__ W,
                                         const float* __restrict__ bias, int g, int t, unsigned (&an)[4][4]) {
  float acc[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = bias[8 * nt + 2 * t], b1 = bias[8 * nt + 2 * t + 1];
    acc[nt][0] = b0;
    acc[nt][1] = b1;
    acc[nt][2] = b0;
    acc[nt][3] = b1;
  }
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const __nv_bfloat16* w = W + (8 * nt + g) * WSTR + 16 * kt + 2 * t;
      const unsigned b0 = *reinterpret_cast<const unsigned*>(w);
      const unsigned b1 = *reinterpret_cast<const unsigned*>(w + 8);
      mma_bf16(acc[nt], a[kt], b0, b1);
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    an[j][0] = pack_bf16(silu_fast(acc[2 * j][0]), silu_fast(acc[2 * j][1]));
    an[j][1] = pack_bf16(silu_fast(acc[2 * j][2]), silu_fast(acc[2 * j][3]));
    an[j][2] = pack_bf16(silu_fast(acc[2 * j + 1][0]), silu_fast(acc[2 * j + 1][1]));
    an[j][3] = pack_bf16(silu_fast(acc[2 * j + 1][2]), silu_fast(acc[2 * j + 1][3]));
  }
}

// Per selected row (k, s): tb = sum_G t_G |x_G|^2 (the band's kinetic energy)
// and the rms residual amplitude, float64 in a fixed order.
__global__ void __launch_bounds__(256) k_precond_row_stats(int npw, int nb, int n_add,
                                                           const cplx<double>* __restrict__ x, int64_t xk,
                                                           const cplx<double>* __restrict__ r, int64_t rk,
                                                           const double* __restrict__ t_, const int* __restrict__ sel,
                                                           double* __restrict__ stats) {
  __shared__ double red[2][8];
  const int k = blockIdx.x / n_add, s = blockIdx.x % n_add;
  const int b = sel[(int64_t)k * n_add + s];
  const cplx<double>* xr = x + k * xk + (int64_t)b * npw;
  const cplx<double>* rr = r + k * rk + (int64_t)b * npw;
  const double* tk = t_ + (int64_t)k * npw;
  double tb = 0.0, r2 = 0.0;
  for (int gi = threadIdx.x; gi < npw; gi += blockDim.x) {
    tb += tk[gi] * norm2(xr[gi]);
    r2 += norm2(rr[gi]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    tb += __shfl_xor_sync(0xffffffffu, tb, o);
    r2 += __shfl_xor_sync(0xffffffffu, r2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = tb;
    red[1][threadIdx.x >> 5] = r2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, c = 0.0;
    for (int w = 0; w < 8; ++w) {
      a += red[0][w];
      c += red[1][w];
    }
    stats[2 * blockIdx.x] = a;
    stats[2 * blockIdx.x + 1] = sqrt(c / npw);
  }
}

constexpr int PL_CHUNK = 512;   // plane waves per CTA of the inference kernel
constexpr int PL_THREADS = 128;

// Learned preconditioner on one chunk of one selected row: grid (chunks, rows),
// four warps, each evaluating 16 plane waves at a time with the network on
// the tensor cores; d = r * TPA * exp(clamp(o, +-3)) unnormalised, and the
// chunk's sum of |d|^2 into partial[row * chunks + chunk].
__global__ void __launch_bounds__(PL_THREADS) k_precond_learned_tc(
    const float* __restrict__ P, int npw, int nb, int n_add, const cplx<double>* __restrict__ r, int64_t rk,
    const double* __restrict__ t_, const double* __restrict__ eig, const int* __restrict__ sel,
    const unsigned char* __restrict__ tpa_only, const double* __restrict__ stats, cplx<double>* __restrict__ d,
    int64_t dk, double* __restrict__ partial) {
  __shared__ __align__(16) __nv_bfloat16 sW2[HID * WSTR];
  __shared__ __align__(16) __nv_bfloat16 sW3[HID * WSTR];
  __shared__ float sW1[HID * NIN], sB1[HID], sB2[HID], sB3[HID], sW4[HID], sB4;
  __shared__ double red[PL_THREADS / 32];
  const int row = blockIdx.y, k = row / n_add, s = row % n_add;
  const int b = sel[(int64_t)k * n_add + s];
  const bool plain = tpa_only && tpa_only[(int64_t)k * nb + b];
  if (!plain) {
    for (int i = threadIdx.x; i < HID * HID; i += blockDim.x) {
      const int n = i / HID, kx = i % HID;
      sW2[n * WSTR + kx] = __float2bfloat16_rn(P[O_W2 + i]);
      sW3[n * WSTR + kx] = __float2bfloat16_rn(P[O_W3 + i]);
    }
    for (int i = threadIdx.x; i < HID * NIN; i += blockDim.x) sW1[i] = bf(P[O_W1 + i]);
    for (int i = threadIdx.x; i < HID; i += blockDim.x) {
      sB1[i] = bf(P[O_B1 + i]);
      sB2[i] = bf(P[O_B2 + i]);
      sB3[i] = bf(P[O_B3 + i]);
      sW4[i] = bf(P[O_W4 + i]);
    }
    if (threadIdx.x == 0) sB4 = bf(P[O_B4]);
  }
  __syncthreads();
  const cplx<double>* rr = r + k * rk + (int64_t)b * npw;
  const double* tk = t_ + (int64_t)k * npw;
  cplx<double>* dr = d + k * dk + (int64_t)s * npw;
  const double tbv = stats[2 * row], rrms = stats[2 * row + 1], eps = eig[(int64_t)k * nb + b];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
  const int c_begin = blockIdx.x * PL_CHUNK, c_end = min(npw, c_begin + PL_CHUNK);
  double nn = 0.0;
  for (int base = c_begin + 16 * warp; base < c_end; base += 16 * (PL_THREADS / 32)) {
    // features of sample (lane & 15) by lanes 0..15
    float u[NIN] = {0.f, 0.f, 0.f, 0.f};
    cplx<double> rv = mk<double>(0.0, 0.0);
    double tg = 0.0;
    {
      const int gi = base + (lane & 15);
      if (lane < 16 && gi < c_end) {
        rv = rr[gi];
        tg = tk[gi];
        if (!plain) features(tg, tbv, eps, sqrt(norm2(rv)), rrms, u);
      }
    }
    float o_row0 = 0.f, o_row8 = 0.f;
    if (!plain) {
      float ua[NIN], ub[NIN];
#pragma unroll
      for (int q = 0; q < NIN; ++q) {
        ua[q] = bf(__shfl_sync(0xffffffffu, u[q], g));
        ub[q] = bf(__shfl_sync(0xffffffffu, u[q], g + 8));
      }
      // layer 1 straight into A fragments of layer 2
      unsigned a1[4][4];
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) {
        float h[2][4];  // [row g / g+8][col 2t, 2t+1, 2t+8, 2t+9]
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          const int col = 16 * kt + 2 * tq + (cc & 1) + 8 * (cc >> 1);
          float za = sB1[col], zb = sB1[col];
#pragma unroll
          for (int q = 0; q < NIN; ++q) {
            za = fmaf(sW1[col * NIN + q], ua[q], za);
            zb = fmaf(sW1[col * NIN + q], ub[q], zb);
          }
          h[0][cc] = silu_fast(za);
          h[1][cc] = silu_fast(zb);
        }
        a1[kt][0] = pack_bf16(h[0][0], h[0][1]);
        a1[kt][1] = pack_bf16(h[1][0], h[1][1]);
        a1[kt][2] = pack_bf16(h[0][2], h[0][3]);
        a1[kt][3] = pack_bf16(h[1][2], h[1][3]);
      }
      unsigned a2[4][4], a3[4][4];
      tc_layer(a1, sW2, sB2, g, tq, a2);
      tc_layer(a2, sW3, sB3, g, tq, a3);
      // layer 4: unpack a3 (rows g, g+8; cols 16kt + 2t + {0,1,8,9}) and dot with W4
      float pa = 0.f, pb = 0.f;
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) {
#pragma unroll
        for (int reg = 0; reg < 4; ++reg) {
          const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&a3[kt][reg]);
          const int col = 16 * kt + 2 * tq + 8 * (reg >> 1);
          const float p0 = __bfloat162float(v.x) * sW4[col] + __bfloat162float(v.y) * sW4[col + 1];
          if (reg & 1) pb += p0;
          else pa += p0;
        }
      }
      pa += __shfl_xor_sync(0xffffffffu, pa, 1);
      pa += __shfl_xor_sync(0xffffffffu, pa, 2);
      pb += __shfl_xor_sync(0xffffffffu, pb, 1);
      pb += __shfl_xor_sync(0xffffffffu, pb, 2);
      o_row0 = pa + sB4;
      o_row8 = pb + sB4;
    }
    // sample (lane & 15) needs the output of row (lane & 15): rows g come from
    // quad g (lane 4g), rows g+8 from quad g too (second value)
    const int srow = lane & 15;
    const float o_a = __shfl_sync(0xffffffffu, o_row0, 4 * (srow & 7));
    const float o_b = __shfl_sync(0xffffffffu, o_row8, 4 * (srow & 7));
    const float o = srow < 8 ? o_a : o_b;
    const int gi = base + srow;
    if (lane < 16 && gi < c_end) {
      double c = tpa_coeff(tg, tbv);
      if (!plain && (rv.x != 0.0 || rv.y != 0.0)) c *= (double)__expf(fminf(fmaxf(o, -3.f), 3.f));
      const cplx<double> v = scale(rv, c);
      dr[gi] = v;
      nn += norm2(v);
    }
  }
  for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xffffffffu, nn, o);
  if (lane == 0) red[warp] = nn;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < PL_THREADS / 32; ++w) a += red[w];
    partial[(int64_t)row * gridDim.x + blockIdx.x] = a;
  }
}

// d row <- d row / |d row|, the norm summed from the chunk partials in order.
__global__ void k_precond_normalize(int npw, int n_add, int chunks, const double* __restrict__ partial,
                                    cplx<double>* __restrict__ d, int64_t dk) {
  const int row = blockIdx.x, k = row / n_add, s = row % n_add;
  double a = 0.0;
  for (int c = 0; c < chunks; ++c) a += partial[(int64_t)row * chunks + c];
  if (!(a > 0.0)) return;
  const double inv = 1.0 / sqrt(a);
  cplx<double>* dr = d + k * dk + (int64_t)s * npw;
  for (int gi = threadIdx.x; gi < npw; gi += blockDim.x) dr[gi] = scale(dr[gi], inv);
}

// ---------------------------------------------------------------------------
// Inference on the tcgen05 tensor cores. A tile is 128 plane waves of one
// selected row, one per thread. Layers 1-3 are M = 128, N = 64 BF16 MMAs
// (kind::f16, FP32 accumulator in 64 TMEM columns): A = the tile's inputs
// (K = 16: the four features, a constant 1, zeros; K = 80: the 64 SiLU
// outputs of the layer before, a constant 1, zeros), B = the layer's weights
// with its bias as the column that meets the constant 1 (the forward pass
// rounds biases to BF16, so the product by 1 adds them exactly). Between the
// MMAs each thread reads its row of the accumulator (tcgen05.ld), applies
// SiLU and writes the BF16 row of the next A; layer 4 (64 -> 1) is a dot
// product on the CUDA cores. Operands are K-major without swizzle: 8-row x
// 16-byte core matrices, consecutive along K (leading byte offset 128), row
// groups kw * 16 bytes apart (stride byte offset).
//
// Rows come in two forms: complex rows (GAMMA = false, as
// k_precond_learned_tc), or the Gamma path's embedded real rows (GAMMA =
// true): half-sphere coefficient c_G = phi[2G-1] + i phi[2G] (c_0 = phi[0]),
// which are the sqrt(w)-scaled half rows, so sums over them are full-sphere
// sums; the output is written back in the same embedding.
constexpr int PU_THREADS = 128;
constexpr int PU_TILE = 128;
constexpr int PU_K1 = 16, PU_K = 80;
constexpr int PU_A = PU_TILE * PU_K * 2;   // 20480 B
constexpr int PU_B1 = HID * PU_K1 * 2;      // 2048 B
constexpr int PU_B = HID * PU_K * 2;        // 10240 B
constexpr int PU_SMEM = PU_A + PU_B1 + 2 * PU_B + 16;  // 43 KB: five CTAs per SM
constexpr int PU_TMEM_COLS = 64;
// kind::f16 instruction descriptor: F32 accumulator, BF16 A and B, both
// K-major, N = 64, M = 128
constexpr uint32_t PU_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(HID >> 3) << 17) |
                              ((uint32_t)(PU_TILE >> 4) << 24);

__host__ __device__ constexpr int pu_off(int row, int k, int kw) {
  return (row >> 3) * (kw * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// tcgen05 shared-memory descriptor, no swizzle (layout type 0)
__device__ __forceinline__ uint64_t pu_desc(uint32_t addr, int kw) {
  const uint32_t lbo = 128, sbo = (uint32_t)kw * 16;
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
         (1ull << 46);
}

__device__ __forceinline__ void pu_mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %4, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(accumulate), "r"(PU_IDESC)
      : "memory");
}

struct PuArgs {
  const float* P;
  int nb, n_add, npw;  // npw: plane waves per row (Gamma: half-sphere slots)
  const void* r;       // complex: (nk, nb, npw) with k stride rk; Gamma: nb embedded rows, row stride r_row
  int64_t rk, r_row;
  const double* t;     // (nk, npw) kinetic diagonal
  const double* eig;   // (nk, nb)
  const int* sel;      // (nk, n_add)
  const unsigned char* tpa_only;
  const double* stats;  // per row: t_b, r_rms
  void* d;              // complex: (nk, n_add, npw) with k stride dk; Gamma: n_add embedded rows, row stride d_row
  int64_t dk, d_row;
  double* partial;      // per (row, tile): sum of |d|^2
  int tiles, total;     // tiles per row, rows * tiles
  int* status;
  long long wait_cycles;
};

// This warp's 32 rows of the 64 accumulator columns, 16 at a time: SiLU,
// then either the BF16 chunks of the next A (hidden layers) or, for the last
// hidden layer, layer 4's dot product with w4 added to o in column order.
__device__ __forceinline__ float pu_hidden(uint32_t taddr, uint8_t* sA, int row, const float* w4, bool last,
                                           float o) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t r[16];
    tmem_ld16(taddr + 16 * q, r);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    float h[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) h[i] = silu_fast(__uint_as_float(r[i]));
    if (last) {
#pragma unroll
      for (int i = 0; i < 16; ++i) o = fmaf(bf(h[i]), w4[16 * q + i], o);
    } else {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        uint4 v;
        v.x = pack_bf16(h[8 * c + 0], h[8 * c + 1]);
        v.y = pack_bf16(h[8 * c + 2], h[8 * c + 3]);
        v.z = pack_bf16(h[8 * c + 4], h[8 * c + 5]);
        v.w = pack_bf16(h[8 * c + 6], h[8 * c + 7]);
        *reinterpret_cast<uint4*>(sA + pu_off(row, 16 * q + 8 * c, PU_K)) = v;
      }
    }
  }
  return o;
}

template <bool GAMMA>
__global__ void __launch_bounds__(PU_THREADS, 5) k_precond_learned_umma(PuArgs a) {
  extern __shared__ uint8_t pu_raw[];
  __shared__ float sW4[HID];
  __shared__ float sB4;
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  __shared__ double red[PU_THREADS / 32];
  __shared__ int abort_f;
  uint8_t* sA = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(pu_raw) + 15) & ~(uintptr_t)15);
  uint8_t* sB1 = sA + PU_A;
  uint8_t* sB2 = sB1 + PU_B1;
  uint8_t* sB3 = sB2 + PU_B;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const float* P = a.P;
  for (int i = tid; i < HID * PU_K1; i += PU_THREADS) {
    const int n = i / PU_K1, k = i % PU_K1;
    const float v = k < NIN ? P[O_W1 + n * NIN + k] : (k == NIN ? P[O_B1 + n] : 0.f);
    *reinterpret_cast<__nv_bfloat16*>(sB1 + pu_off(n, k, PU_K1)) = __float2bfloat16_rn(v);
  }
  for (int i = tid; i < HID * PU_K; i += PU_THREADS) {
    const int n = i / PU_K, k = i % PU_K;
    const float v2 = k < HID ? P[O_W2 + n * HID + k] : (k == HID ? P[O_B2 + n] : 0.f);
    const float v3 = k < HID ? P[O_W3 + n * HID + k] : (k == HID ? P[O_B3 + n] : 0.f);
    *reinterpret_cast<__nv_bfloat16*>(sB2 + pu_off(n, k, PU_K)) = __float2bfloat16_rn(v2);
    *reinterpret_cast<__nv_bfloat16*>(sB3 + pu_off(n, k, PU_K)) = __float2bfloat16_rn(v3);
  }
  for (int i = tid; i < HID; i += PU_THREADS) sW4[i] = bf(P[O_W4 + i]);
  if (tid == 0) sB4 = bf(P[O_B4]);
  // the constant columns of this thread's A row for layers 2 and 3: k = 64 holds 1
  {
    const uint32_t one = 0x3F80u;  // BF16 1.0
    *reinterpret_cast<uint4*>(sA + pu_off(tid, 64, PU_K)) = make_uint4(one, 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(sA + pu_off(tid, 72, PU_K)) = make_uint4(0u, 0u, 0u, 0u);
  }
  if (tid == 0) {
    mbar_init(smem_u32(&bar), 1);
    abort_f = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"((uint32_t)PU_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16);  // this warp's 32 lanes
  const uint32_t bar_a = smem_u32(&bar);
  // layer 1 reads the first 16 columns of A (its features, a 1 at k = 4, zeros)
  const uint64_t dA1 = pu_desc(smem_u32(sA), PU_K), dB1 = pu_desc(smem_u32(sB1), PU_K1);
  const uint32_t aA = smem_u32(sA), aB2 = smem_u32(sB2), aB3 = smem_u32(sB3);
  uint32_t parity = 0;

  // one layer's MMA (issued by thread 0 after every thread's A row is in
  // place), then every thread waits for the accumulator
  auto layer = [&](int which) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (which == 1) {
        pu_mma(tmem, dA1, dB1, 0u);
      } else {
        const uint32_t aB = which == 2 ? aB2 : aB3;
#pragma unroll
        for (int s = 0; s < PU_K / 16; ++s)
          pu_mma(tmem, pu_desc(aA + 256 * s, PU_K), pu_desc(aB + 256 * s, PU_K), s > 0 ? 1u : 0u);
      }
      mma_commit(bar_a);
    }
    if (!mbar_wait(bar_a, parity, a.wait_cycles)) {
      atomicOr(a.status, GWB_ERR_TIMEOUT);
      abort_f = 1;
    }
    parity ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  };

  for (int w = blockIdx.x; w < a.total; w += gridDim.x) {
    const int row = w / a.tiles, tile = w - row * a.tiles;
    const int k = row / a.n_add, s = row - k * a.n_add;
    const int b = a.sel[(int64_t)k * a.n_add + s];
    const bool plain = a.tpa_only && a.tpa_only[(int64_t)k * a.nb + b];
    const double tbv = a.stats[2 * row], rrms = a.stats[2 * row + 1], eps = a.eig[(int64_t)k * a.nb + b];
    const int gi = tile * PU_TILE + tid;
    const bool valid = gi < a.npw;
    cplx<double> rv = mk<double>(0.0, 0.0);
    double tg = 0.0;
    if (valid) {
      tg = a.t[(int64_t)k * a.npw + gi];
      if (GAMMA) {
        const double* rr = static_cast<const double*>(a.r) + (int64_t)b * a.r_row;
        rv = gi == 0 ? mk<double>(rr[0], 0.0) : mk<double>(rr[2 * gi - 1], rr[2 * gi]);
      } else {
        rv = static_cast<const cplx<double>*>(a.r)[k * a.rk + (int64_t)b * a.npw + gi];
      }
    }
    double c = tpa_coeff(tg, tbv);
    if (!plain) {
      float u[NIN] = {0.f, 0.f, 0.f, 0.f};
      if (valid) features(tg, tbv, eps, sqrt(norm2(rv)), rrms, u);
      // layer 1's inputs in the first two chunks of A (the second zero: the
      // previous tile left activations there)
      *reinterpret_cast<uint4*>(sA + pu_off(tid, 0, PU_K)) =
          make_uint4(pack_bf16(u[0], u[1]), pack_bf16(u[2], u[3]), pack_bf16(1.f, 0.f), 0u);
      *reinterpret_cast<uint4*>(sA + pu_off(tid, 8, PU_K)) = make_uint4(0u, 0u, 0u, 0u);
      layer(1);
      pu_hidden(taddr, sA, tid, sW4, false, 0.f);
      layer(2);
      pu_hidden(taddr, sA, tid, sW4, false, 0.f);
      layer(3);
      const float o = pu_hidden(taddr, sA, tid, sW4, true, sB4);
      if (rv.x != 0.0 || rv.y != 0.0) c *= (double)__expf(fminf(fmaxf(o, -3.f), 3.f));
    }
    double nn = 0.0;
    if (valid) {
      const cplx<double> v = scale(rv, c);
      nn = norm2(v);
      if (GAMMA) {
        double* dr = static_cast<double*>(a.d) + (int64_t)s * a.d_row;
        if (gi == 0) {
          dr[0] = v.x;
        } else {
          dr[2 * gi - 1] = v.x;
          dr[2 * gi] = v.y;
        }
      } else {
        static_cast<cplx<double>*>(a.d)[k * a.dk + (int64_t)s * a.npw + gi] = v;
      }
    }
    for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xffffffffu, nn, o);
    __syncthreads();  // red from the previous tile is read
    if (lane == 0) red[warp] = nn;
    __syncthreads();
    if (tid == 0) a.partial[(int64_t)row * a.tiles + tile] = red[0] + red[1] + red[2] + red[3];
    if (abort_f) break;
  }
  // after a wait that ran out, the MMA it waited for may still run: give it
  // one more bounded wait before the accumulator's columns are freed
  if (abort_f && tid == 0) mbar_wait(bar_a, parity ^ 1u, a.wait_cycles);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)PU_TMEM_COLS)
                 : "memory");
  }
}

// Per selected row of the Gamma path's embedded real rows: t_b = sum_G t_G
// |c_G|^2 and the rms of the residual's half-sphere coefficients (as
// k_precond_row_stats on the half rows).
__global__ void __launch_bounds__(256) k_precond_row_stats_gamma(int nhalf, int n_add, const double* __restrict__ x,
                                                                 int64_t x_row, const double* __restrict__ r,
                                                                 int64_t r_row, const double* __restrict__ t_,
                                                                 const int* __restrict__ sel,
                                                                 double* __restrict__ stats) {
  __shared__ double red[2][8];
  const int s = blockIdx.x;
  const int b = sel[s];
  const double* xr = x + (int64_t)b * x_row;
  const double* rr = r + (int64_t)b * r_row;
  double tb = 0.0, r2 = 0.0;
  for (int g = threadIdx.x; g < nhalf; g += blockDim.x) {
    double xa, xb = 0.0, ra, rb = 0.0;
    if (g == 0) {
      xa = xr[0];
      ra = rr[0];
    } else {
      xa = xr[2 * g - 1];
      xb = xr[2 * g];
      ra = rr[2 * g - 1];
      rb = rr[2 * g];
    }
    tb += t_[g] * (xa * xa + xb * xb);
    r2 += ra * ra + rb * rb;
  }
  for (int o = 16; o > 0; o >>= 1) {
    tb += __shfl_xor_sync(0xffffffffu, tb, o);
    r2 += __shfl_xor_sync(0xffffffffu, r2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = tb;
    red[1][threadIdx.x >> 5] = r2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double p = 0.0, q = 0.0;
    for (int w = 0; w < 8; ++w) {
      p += red[0][w];
      q += red[1][w];
    }
    stats[2 * s] = p;
    stats[2 * s + 1] = sqrt(q / nhalf);
  }
}

// Embedded rows: d <- d / |d| over the 2 nhalf - 1 coordinates, the norm
// summed from the tile partials in order; pad columns set to zero.
__global__ void k_precond_normalize_gamma(int nhalf, int npad, int tiles, const double* __restrict__ partial,
                                          double* __restrict__ d, int64_t d_row) {
  const int s = blockIdx.x;
  double a = 0.0;
  for (int c = 0; c < tiles; ++c) a += partial[(int64_t)s * tiles + c];
  const double inv = a > 0.0 ? 1.0 / sqrt(a) : 1.0;
  double* dr = d + (int64_t)s * d_row;
  const int nphi = 2 * nhalf - 1;
  for (int i = threadIdx.x; i < npad; i += blockDim.x) dr[i] = i < nphi ? dr[i] * inv : 0.0;
}

// Stall rule of the learned preconditioner: a band whose residual has not
// dropped below ratio * (its best so far) for `patience` consecutive rounds
// reverts to TPA for the rest of the solve (tpa_only is sticky).
__global__ void k_stall_update(const double* __restrict__ rn, double* __restrict__ rn_best,
                               unsigned char* __restrict__ count, unsigned char* __restrict__ tpa_only, int n,
                               double ratio, int patience) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = rn[i];
    if (v < ratio * rn_best[i]) {
      count[i] = 0;
    } else if (count[i] < 255) {
      count[i] = count[i] + 1;
    }
    if (count[i] >= patience) tpa_only[i] = 1;
    rn_best[i] = fmin(rn_best[i], v);
  }
}

// The tcgen05 inference kernel over all (row, tile) items: a persistent grid
// of up to five CTAs per SM (43 KB of shared memory and 64 TMEM columns each).
template <bool GAMMA>
int precond_umma(const float* params, int nb, int n_add, int npw, const void* r, int64_t rk, int64_t r_row,
                 const double* t, const double* eig, const int* sel, const uint8_t* tpa_only, const double* stats,
                 void* d, int64_t dk, int64_t d_row, double* partial, int rows, int* status, cudaStream_t st) {
  int dev = 0, sms = 0;
  GWB_CUDA_TRY(cudaGetDevice(&dev));
  GWB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  PuArgs a;
  a.P = params;
  a.nb = nb;
  a.n_add = n_add;
  a.npw = npw;
  a.r = r;
  a.rk = rk;
  a.r_row = r_row;
  a.t = t;
  a.eig = eig;
  a.sel = sel;
  a.tpa_only = tpa_only;
  a.stats = stats;
  a.d = d;
  a.dk = dk;
  a.d_row = d_row;
  a.partial = partial;
  a.tiles = (npw + PU_TILE - 1) / PU_TILE;
  a.total = rows * a.tiles;
  a.status = status;
  a.wait_cycles = tc_wait_cycles();
  GWB_CUDA_TRY(cudaFuncSetAttribute(k_precond_learned_umma<GAMMA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    PU_SMEM));
  GWB_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), st));
  const int grid = std::min(a.total, 5 * sms);
  k_precond_learned_umma<GAMMA><<<grid, PU_THREADS, PU_SMEM, st>>>(a);
  GWB_LAUNCH_CHECK();
  return GWB_OK;
}

}  // namespace gwb

using namespace gwb;

extern "C" {

int gwb_mlp_param_count(void) { return NPARAM; }

int gwb_mlp_forward(const float* params, int32_t n, const float* feats, float* out, void* stream) {
  GWB_REQUIRE(params && feats && out && n >= 0, "bad arguments");
  if (n == 0) return GWB_OK;
  const size_t sm = NPARAM * sizeof(float);
  GWB_CUDA_TRY(allow_smem(k_mlp_forward));
  const int blocks = std::min((n + 255) / 256, 4 * 148);
  k_mlp_forward<<<blocks, 256, sm, (cudaStream_t)stream>>>(params, n, feats, out);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

int gwb_mlp_loss_grad(const float* params, int32_t n, const float* feats, const float* target, const float* weight,
                      float* grad, float* loss, void* stream) {
  GWB_REQUIRE(params && feats && target && weight && grad && loss && n >= 0, "bad arguments");
  if (n == 0) return GWB_OK;
  const size_t sm = (2 * NPARAM + TS * NIN + 8 * TS * HID + TS) * sizeof(float);
  GWB_CUDA_TRY(allow_smem(k_mlp_loss_grad));
  const int tiles = (n + TS - 1) / TS;
  const int blocks = std::min(tiles, 2 * 148);
  k_mlp_loss_grad<<<blocks, 256, sm, (cudaStream_t)stream>>>(params, n, feats, target, weight, grad, loss);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

int gwb_mlp_adam(float* params, const float* grad, float* m, float* v, int32_t step, float lr, float beta1,
                 float beta2, float eps, void* stream) {
  GWB_REQUIRE(params && grad && m && v && step >= 1, "bad arguments");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_mlp_adam<<<(NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grad, m, v, NPARAM, lr, beta1, beta2,
                                                                     eps, c1, c2);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

int gwb_mlp_backward(const float* params, int32_t n, const float* feats, const float* dout, float* grad,
                     void* stream) {
  GWB_REQUIRE(params && feats && dout && grad && n >= 0, "bad arguments");
  if (n == 0) return GWB_OK;
  const size_t sm = (2 * NPARAM + TS * NIN + 8 * TS * HID + TS) * sizeof(float);
  GWB_CUDA_TRY(allow_smem(k_mlp_loss_grad));
  const int tiles = (n + TS - 1) / TS;
  const int blocks = std::min(tiles, 2 * 148);
  k_mlp_loss_grad<<<blocks, 256, sm, (cudaStream_t)stream>>>(params, n, feats, nullptr, dout, grad, nullptr);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

int gwb_precond_features(int32_t nk, int32_t nb, int32_t n_add, int32_t npw, const void* x, int64_t x_kstride,
                         const void* r, int64_t r_kstride, const double* t, const double* eig, const int32_t* sel,
                         float* feats, void* stream) {
  GWB_REQUIRE(nk > 0 && nb > 0 && n_add > 0 && npw > 0, "bad sizes");
  GWB_REQUIRE(x && r && t && eig && sel && feats, "null pointer");
  k_features<<<nk * n_add, 256, 0, (cudaStream_t)stream>>>(npw, nb, n_add, (const cplx<double>*)x, x_kstride,
                                                          (const cplx<double>*)r, r_kstride, t, eig, sel, feats);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

// inference kernel of gwb_precond_learned: 1 tcgen05 (default), 0 mma.sync
static int g_precond_kernel = 1;

int gwb_precond_set_kernel(int32_t which) {
  GWB_REQUIRE(which == 0 || which == 1, "kernel must be 0 (mma.sync) or 1 (tcgen05)");
  g_precond_kernel = which;
  return GWB_OK;
}

int64_t gwb_precond_learned_work_bytes(int32_t nk, int32_t n_add, int32_t npw) {
  if (nk <= 0 || n_add <= 0 || npw <= 0) return 0;
  const int64_t rows = (int64_t)nk * n_add, tiles = (npw + PU_TILE - 1) / PU_TILE;
  return (rows * (2 + tiles) + 1) * (int64_t)sizeof(double);
}

int gwb_precond_learned(const float* params, int32_t nk, int32_t nb, int32_t n_add, int32_t npw, const void* x,
                        int64_t x_kstride, const void* r, int64_t r_kstride, const double* t, const double* eig,
                        const int32_t* sel, const uint8_t* tpa_only, void* d, int64_t d_kstride, void* work,
                        size_t work_bytes, void* stream) {
  GWB_REQUIRE(params && nk > 0 && nb > 0 && n_add > 0 && n_add <= nb && npw > 0, "bad sizes");
  GWB_REQUIRE(x && r && t && eig && sel && d && work, "null pointer");
  GWB_REQUIRE((int64_t)work_bytes >= gwb_precond_learned_work_bytes(nk, n_add, npw),
              "work smaller than gwb_precond_learned_work_bytes");
  const int rows = nk * n_add;
  double* stats = static_cast<double*>(work);
  double* partial = stats + 2 * (int64_t)rows;
  const cudaStream_t st = (cudaStream_t)stream;
  k_precond_row_stats<<<rows, 256, 0, st>>>(npw, nb, n_add, (const cplx<double>*)x, x_kstride,
                                            (const cplx<double>*)r, r_kstride, t, sel, stats);
  if (g_precond_kernel == 0) {
    const int chunks = (npw + PL_CHUNK - 1) / PL_CHUNK;
    k_precond_learned_tc<<<dim3(chunks, rows), PL_THREADS, 0, st>>>(params, npw, nb, n_add, (const cplx<double>*)r,
                                                                    r_kstride, t, eig, sel, tpa_only, stats,
                                                                    (cplx<double>*)d, d_kstride, partial);
    k_precond_normalize<<<rows, 256, 0, st>>>(npw, n_add, chunks, partial, (cplx<double>*)d, d_kstride);
  } else {
    const int64_t tiles = (npw + PU_TILE - 1) / PU_TILE;
    int* status = reinterpret_cast<int*>(partial + (int64_t)rows * tiles);
    int rc = precond_umma<false>(params, nb, n_add, npw, r, r_kstride, 0, t, eig, sel, tpa_only, stats, d, d_kstride,
                                 0, partial, rows, status, st);
    if (rc) return rc;
    k_precond_normalize<<<rows, 256, 0, st>>>(npw, n_add, (int)tiles, partial, (cplx<double>*)d, d_kstride);
  }
  GWB_LAUNCH_CHECK();
  count_launches(3);
  return GWB_OK;
}

int64_t gwb_precond_learned_gamma_work_bytes(int32_t n_add, int32_t nhalf) {
  if (n_add <= 0 || nhalf <= 0) return 0;
  return ((int64_t)n_add * (2 + (nhalf + PU_TILE - 1) / PU_TILE) + 1) * (int64_t)sizeof(double);
}

int gwb_precond_learned_gamma(const float* params, int32_t nb, int32_t n_add, int32_t nhalf, int32_t npad,
                              const double* x, int64_t x_row, const double* r, int64_t r_row, const double* t_half,
                              const double* eig, const int32_t* sel, const uint8_t* tpa_only, double* d,
                              int64_t d_row, void* work, size_t work_bytes, void* stream) {
  GWB_REQUIRE(params && nb > 0 && n_add > 0 && n_add <= nb && nhalf > 0, "bad sizes");
  GWB_REQUIRE(npad >= 2 * nhalf - 1 && x_row >= 2 * nhalf - 1 && r_row >= 2 * nhalf - 1 && d_row >= npad,
              "rows shorter than the embedding");
  GWB_REQUIRE(x && r && t_half && eig && sel && d && work, "null pointer");
  GWB_REQUIRE((int64_t)work_bytes >= gwb_precond_learned_gamma_work_bytes(n_add, nhalf),
              "work smaller than gwb_precond_learned_gamma_work_bytes");
  double* stats = static_cast<double*>(work);
  double* partial = stats + 2 * (int64_t)n_add;
  const int tiles = (nhalf + PU_TILE - 1) / PU_TILE;
  int* status = reinterpret_cast<int*>(partial + (int64_t)n_add * tiles);
  const cudaStream_t st = (cudaStream_t)stream;
  k_precond_row_stats_gamma<<<n_add, 256, 0, st>>>(nhalf, n_add, x, x_row, r, r_row, t_half, sel, stats);
  int rc = precond_umma<true>(params, nb, n_add, nhalf, r, 0, r_row, t_half, eig, sel, tpa_only, stats, d, 0, d_row,
                              partial, n_add, status, st);
  if (rc) return rc;
  k_precond_normalize_gamma<<<n_add, 256, 0, st>>>(nhalf, npad, tiles, partial, d, d_row);
  GWB_LAUNCH_CHECK();
  count_launches(3);
  return GWB_OK;
}

int gwb_stall_update(const double* rn, double* rn_best, uint8_t* count, uint8_t* tpa_only, int32_t n, double ratio,
                     int32_t patience, void* stream) {
  GWB_REQUIRE(rn && rn_best && count && tpa_only && n > 0 && patience > 0, "bad arguments");
  k_stall_update<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(rn, rn_best, count, tpa_only, n, ratio, patience);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}

}  // extern "C"
