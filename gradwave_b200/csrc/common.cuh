// Shared helpers for the sm_100a band-solve kernels: complex arithmetic in
// float/double, status handling, launch checks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <mutex>
#include <set>
#include <string>
#include <utility>

#include "../../include/gwb.h"

namespace gwb {

template <typename T> struct cplx;
template <> struct __align__(8) cplx<float> {
  float x, y;
};
template <> struct __align__(16) cplx<double> {
  double x, y;
};

template <typename T> __host__ __device__ __forceinline__ cplx<T> mk(T a, T b) {
  cplx<T> r;
  r.x = a;
  r.y = b;
  return r;
}
template <typename T> __host__ __device__ __forceinline__ cplx<T> operator+(cplx<T> a, cplx<T> b) {
  return mk<T>(a.x + b.x, a.y + b.y);
}
template <typename T> __host__ __device__ __forceinline__ cplx<T> operator-(cplx<T> a, cplx<T> b) {
  return mk<T>(a.x - b.x, a.y - b.y);
}
template <typename T> __host__ __device__ __forceinline__ cplx<T> operator*(cplx<T> a, cplx<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __host__ __device__ __forceinline__ cplx<T> scale(cplx<T> a, T s) {
  return mk<T>(a.x * s, a.y * s);
}
template <typename T> __host__ __device__ __forceinline__ cplx<T> conj(cplx<T> a) {
  return mk<T>(a.x, -a.y);
}
// a * conj(b)
template <typename T> __host__ __device__ __forceinline__ cplx<T> mul_conj(cplx<T> a, cplx<T> b) {
  return mk<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// conj(a) * b
template <typename T> __host__ __device__ __forceinline__ cplx<T> conj_mul(cplx<T> a, cplx<T> b) {
  return mk<T>(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <typename T> __host__ __device__ __forceinline__ T norm2(cplx<T> a) {
  return a.x * a.x + a.y * a.y;
}
// multiply by -i (sign<0) or +i (sign>0)
template <typename T> __device__ __forceinline__ cplx<T> mul_i(cplx<T> a, int sign) {
  return sign > 0 ? mk<T>(-a.y, a.x) : mk<T>(a.y, -a.x);
}

// Load an element stored as complex128 or complex64 into compute precision T.
template <typename T, typename S> __device__ __forceinline__ cplx<T> ld(const S* p, size_t i);
template <> __device__ __forceinline__ cplx<float> ld<float, cplx<float>>(const cplx<float>* p, size_t i) {
  return p[i];
}
template <> __device__ __forceinline__ cplx<double> ld<double, cplx<double>>(const cplx<double>* p, size_t i) {
  return p[i];
}
template <> __device__ __forceinline__ cplx<float> ld<float, cplx<double>>(const cplx<double>* p, size_t i) {
  cplx<double> v = p[i];
  return mk<float>((float)v.x, (float)v.y);
}
template <> __device__ __forceinline__ cplx<double> ld<double, cplx<float>>(const cplx<float>* p, size_t i) {
  cplx<float> v = p[i];
  return mk<double>(v.x, v.y);
}
template <typename S, typename T> __device__ __forceinline__ void st(S* p, size_t i, cplx<T> v) {
  p[i].x = v.x;
  p[i].y = v.y;
}

void set_error(const std::string& msg);
// Tally of kernels this library launched (gwb_launch_count).
void count_launches(int n);

// Raise a kernel's dynamic shared-memory cap to the device's opt-in maximum
// (less its static shared memory), once per (kernel, device). The cap is a
// process-wide attribute of the kernel: setting it to each launch's own size
// would let a thread launching a larger size race a thread setting a smaller
// one (concurrent solves on separate streams). Every caller sets the same
// value, so there is no such race.
template <typename F>
inline cudaError_t allow_smem(F* func) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_pair(reinterpret_cast<const void*>(func), dev);
  if (done.count(key)) return cudaSuccess;
  int optin = 0;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  cudaFuncAttributes fa;
  e = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(func));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(reinterpret_cast<const void*>(func), cudaFuncAttributeMaxDynamicSharedMemorySize,
                           optin - (int)fa.sharedSizeBytes);
  if (e == cudaSuccess) done.insert(key);
  return e;
}

}  // namespace gwb

#define GWB_CUDA_TRY(expr)                                                        \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      gwb::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));         \
      return GWB_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

#define GWB_LAUNCH_CHECK()                                                        \
  do {                                                                            \
    cudaError_t _e = cudaGetLastError();                                          \
    if (_e != cudaSuccess) {                                                      \
      gwb::set_error(std::string("kernel launch: ") + cudaGetErrorString(_e));    \
      return GWB_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

#define GWB_REQUIRE(cond, msg)                                                    \
  do {                                                                            \
    if (!(cond)) {                                                                \
      gwb::set_error(msg);                                                        \
      return GWB_ERR_ARG;                                                         \
    }                                                                             \
  } while (0)
