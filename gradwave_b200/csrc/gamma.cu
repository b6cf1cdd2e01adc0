// Gamma-point apply in the real embedding of the half sphere (gradwave
// core/gamma.py:161-250: GammaHamiltonian.apply with embed_real/unembed_real).
//
// At k = 0 the bands are real fields, c(-G) = conj(c(G)), and only the half
// sphere (G = 0 first, then one member of each {G, -G} pair) is stored, as the
// real vector phi = (Re c0, sqrt2 Re c1, sqrt2 Im c1, ...) of length
// 2 nhalf - 1 whose plain dot product is the full-sphere inner product.
//
// Two real fields share one complex transform: z = c_a + i c_b on the full
// sphere, one pass of the complex apply (FFTs, V(r), kinetic, nonlocal) gives
// Hz = H c_a + i H c_b, and since both images are again Hermitian-symmetric,
//   H c_a (G) = (Hz(G) + conj Hz(-G)) / 2,   H c_b (G) = (Hz(G) - conj Hz(-G)) / 2i.
// So nb real bands cost ceil(nb/2) complex rows of the existing apply kernels:
// half the FFT and nonlocal work of the complex path, with no real-FFT kernel.
// k_gamma_pack builds the z rows from phi, k_gamma_unpack the phi images.
#include <algorithm>

#include "common.cuh"

namespace gwb {
namespace {

constexpr double kSqrt2 = 1.41421356237309504880;
constexpr double kInvSqrt2 = 0.70710678118654752440;

// c_b at half slot j from phi row b
__device__ __forceinline__ cplx<double> half_coeff(const double* __restrict__ phi, int j) {
  if (j == 0) return mk<double>(phi[0], 0.0);
  return mk<double>(kInvSqrt2 * phi[2 * j - 1], kInvSqrt2 * phi[2 * j]);
}

// z[p][g] = c_{2p}(g) + i c_{2p+1}(g), c_b(g) = h_b[src_half[g]] (conjugated
// where conj_full[g]); the partner band of an odd last row is zero.
__global__ void k_gamma_pack(int nb, int nphi, int npw, const double* __restrict__ phi, int64_t ldphi,
                             const int* __restrict__ src_half, const unsigned char* __restrict__ conj_full,
                             cplx<double>* __restrict__ z) {
  const int npair = (nb + 1) / 2;
  const int64_t total = (int64_t)npair * npw;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(idx / npw), g = (int)(idx % npw);
    const int j = src_half[g];
    const bool cj = conj_full[g] != 0;
    cplx<double> a = half_coeff(phi + (int64_t)(2 * p) * ldphi, j);
    cplx<double> b = 2 * p + 1 < nb ? half_coeff(phi + (int64_t)(2 * p + 1) * ldphi, j) : mk<double>(0.0, 0.0);
    if (cj) {
      a.y = -a.y;
      b.y = -b.y;
    }
    z[idx] = mk<double>(a.x - b.y, a.y + b.x);  // a + i b
  }
}

// out rows 2p, 2p+1 (phi layout) from Hz row p: the Hermitian parts at the
// representative G and its partner -G.
__global__ void k_gamma_unpack(int nb, int nhalf, int npw, const cplx<double>* __restrict__ hz,
                               const int* __restrict__ rep_full, const int* __restrict__ partner_rep,
                               double* __restrict__ out, int64_t ldout) {
  const int npair = (nb + 1) / 2;
  const int64_t total = (int64_t)npair * nhalf;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(idx / nhalf), j = (int)(idx % nhalf);
    const cplx<double>* row = hz + (int64_t)p * npw;
    const cplx<double> u = row[rep_full[j]], w = row[partner_rep[j]];
    // A = (u + conj w) / 2, B = (u - conj w) / 2i
    const cplx<double> A = mk<double>(0.5 * (u.x + w.x), 0.5 * (u.y - w.y));
    const cplx<double> B = mk<double>(0.5 * (u.y + w.y), -0.5 * (u.x - w.x));
    double* oa = out + (int64_t)(2 * p) * ldout;
    if (j == 0) {
      oa[0] = A.x;
    } else {
      oa[2 * j - 1] = kSqrt2 * A.x;
      oa[2 * j] = kSqrt2 * A.y;
    }
    if (2 * p + 1 < nb) {
      double* ob = out + (int64_t)(2 * p + 1) * ldout;
      if (j == 0) {
        ob[0] = B.x;
      } else {
        ob[2 * j - 1] = kSqrt2 * B.x;
        ob[2 * j] = kSqrt2 * B.y;
      }
    }
  }
}

}  // namespace
}  // namespace gwb

using namespace gwb;

extern "C" size_t gwb_gamma_work_bytes(int32_t nb, int32_t npw) {
  if (nb <= 0 || npw <= 0) return 0;
  return (size_t)2 * ((nb + 1) / 2) * npw * sizeof(cplx<double>);
}

extern "C" int gwb_gamma_apply(gwb_ham* h, int32_t nb, int32_t nhalf, int32_t npw, const double* phi, int64_t ldphi,
                               double* out, int64_t ldout, const int32_t* src_half, const uint8_t* conj_full,
                               const int32_t* rep_full, const int32_t* partner_rep, int32_t prec, void* work,
                               size_t work_bytes, void* stream) {
  GWB_REQUIRE(h && phi && out && src_half && conj_full && rep_full && partner_rep && work, "null argument");
  GWB_REQUIRE(nb > 0 && nhalf > 0 && npw == 2 * nhalf - 1, "a Gamma sphere has npw = 2 nhalf - 1");
  const int nphi = 2 * nhalf - 1;
  GWB_REQUIRE(ldphi >= nphi && ldout >= nphi, "row stride shorter than 2 nhalf - 1");
  GWB_REQUIRE(work_bytes >= gwb_gamma_work_bytes(nb, npw), "work smaller than gwb_gamma_work_bytes");
  GWB_REQUIRE(phi != out, "phi and out must not overlap");
  const int npair = (nb + 1) / 2;
  cplx<double>* z = (cplx<double>*)work;
  cplx<double>* hz = z + (size_t)npair * npw;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t t1 = (int64_t)npair * npw, t2 = (int64_t)npair * nhalf;
  k_gamma_pack<<<(unsigned)std::min<int64_t>((t1 + 255) / 256, 148 * 16), 256, 0, st>>>(nb, nphi, npw, phi, ldphi,
                                                                                      src_half, conj_full, z);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  const int rc = gwb_ham_apply_strided(h, z, (int64_t)npair * npw, hz, (int64_t)npair * npw, npair, GWB_C128, prec,
                                       stream);
  if (rc != GWB_OK) return rc;
  k_gamma_unpack<<<(unsigned)std::min<int64_t>((t2 + 255) / 256, 148 * 16), 256, 0, st>>>(nb, nhalf, npw, hz,
                                                                                        rep_full, partner_rep, out,
                                                                                        ldout);
  GWB_LAUNCH_CHECK();
  count_launches(1);
  return GWB_OK;
}
