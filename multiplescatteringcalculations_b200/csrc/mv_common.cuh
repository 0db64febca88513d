// Shared pieces of the matvec translation units.
#pragma once
#include <mutex>
#include <unordered_set>

#include "plan.cuh"

namespace msc {

// Lines per tile so that one tile row is 128 bytes: 16 (complex64) / 8 (complex128).
template <typename T> struct Tile { static constexpr int W = 128 / (int)sizeof(cx<T>); };

template <typename T> __device__ __forceinline__ T load_scale(const double* s) { return s ? (T)(*s) : (T)1; }

// Walks it = start, start + step, ... as (q, r) = (it / D, it % D) with one
// division at construction and additions afterwards.
struct QR {
  int q, r, dq, dr, D;
  __device__ __forceinline__ QR(int start, int step, int D_) : D(D_) {
    q = start / D_;
    r = start - q * D_;
    dq = step / D_;
    dr = step - dq * D_;
  }
  __device__ __forceinline__ void next() {
    q += dq;
    r += dr;
    if (r >= D) {
      r -= D;
      ++q;
    }
  }
};

// Allow the kernel the full dynamic shared memory and prefer shared memory over L1
// (these kernels stage everything in shared memory); done once per kernel.
inline cudaError_t prep_kernel(const void* fn) {
  static std::mutex mu;
  static std::unordered_set<const void*> seen;
  std::lock_guard<std::mutex> lk(mu);
  if (seen.count(fn)) return cudaSuccess;
  // dynamic limit = the device's opt-in maximum minus the kernel's static shared memory
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e == cudaSuccess) seen.insert(fn);
  return e;
}

#define MSC_POW2_DISPATCH(pow2, CALL) \
  do {                                \
    if (pow2) { CALL(true); }         \
    else { CALL(false); }             \
  } while (0)

// Kernel launchers (one translation unit each).
template <typename T>
int launch_fft_contig(msc_plan* pl, const cx<T>* in, cx<T>* out, long long nlines, long long G, long long GS,
                      long long stride, int n_in, int n_out, const FftPlan1D& f, const cx<T>* tw, int dir,
                      const int* done);
template <typename T>
int launch_t0_fft_y(msc_plan* pl, const cx<T>* x, const double* scale, cx<T>* W, const cx<T>* tw, const int* done);
template <typename T>
int launch_fft_strided(msc_plan* pl, const cx<T>* in, long long es, long long S1, long long S2, cx<T>* out,
                       long long eo, long long O1, long long O2, float2* out32, int ncol, int n1, int n2, int n_in,
                       int n_out, const FftPlan1D& f, const cx<T>* tw, int dir, const int* done);
template <typename T>
int launch_block_mul(msc_plan* pl, cx<T>* W, const int* done);
template <typename T>
int launch_fft_y_out(msc_plan* pl, const cx<T>* W, const cx<T>* x, const double* scale, cx<T>* y, const cx<T>* tw,
                     const int* done);

}  // namespace msc
