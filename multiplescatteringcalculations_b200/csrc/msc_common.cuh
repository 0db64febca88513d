// Common device helpers of the slab Foldy-Lax solver: complex arithmetic on
// float2/double2, status codes, launch helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/msc.h"

namespace msc {

// ---- complex element type per real type -----------------------------------
template <typename T> struct CxT;
template <> struct CxT<float> { using type = float2; };
template <> struct CxT<double> { using type = double2; };
template <typename T> using cx = typename CxT<T>::type;

template <typename T> __host__ __device__ __forceinline__ cx<T> mk(T a, T b) { cx<T> r; r.x = a; r.y = b; return r; }
// complex64 sums and differences as paired FP32 instructions on the device (each lane
// rounds as the scalar operation does, so results are the same bits); a - b is
// fma(b, -1, a), exact in the product
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
  return __fadd2_rn(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
__host__ __device__ __forceinline__ float2 operator*(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ float2& operator+=(float2& a, float2 b) { a = a + b; return a; }
__host__ __device__ __forceinline__ double2& operator+=(double2& a, double2 b) { a.x += b.x; a.y += b.y; return a; }
__host__ __device__ __forceinline__ float2& operator-=(float2& a, float2 b) { a = a - b; return a; }
__host__ __device__ __forceinline__ double2& operator-=(double2& a, double2 b) { a.x -= b.x; a.y -= b.y; return a; }

template <typename C> __host__ __device__ __forceinline__ C conj_(C a) { a.y = -a.y; return a; }
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C mul_conj(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
// conj(a) * b
template <typename C> __host__ __device__ __forceinline__ C conj_mul(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.x * b.y - a.y * b.x; return r;
}
// multiply by +i (s = +1) or -i (s = -1)
template <int S, typename C> __host__ __device__ __forceinline__ C mul_i(C a) {
  C r;
  if (S > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}
// fused a += b * c
template <typename C> __host__ __device__ __forceinline__ void fma_(C& a, C b, C c) {
  a.x = fma(b.x, c.x, a.x); a.x = fma(-b.y, c.y, a.x);
  a.y = fma(b.x, c.y, a.y); a.y = fma(b.y, c.x, a.y);
}
__device__ __forceinline__ void fma_(float2& a, float2 b, float2 c) {
  a.x = fmaf(b.x, c.x, a.x); a.x = fmaf(-b.y, c.y, a.x);
  a.y = fmaf(b.x, c.y, a.y); a.y = fmaf(b.y, c.x, a.y);
}

template <typename C> __device__ __forceinline__ C czero() { C r; r.x = 0; r.y = 0; return r; }

__device__ __forceinline__ float2 to_c(double2 a, float2*) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 to_c(double2 a, double2*) { return a; }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
template <typename C> __device__ __forceinline__ C from_d(double2 a) { return to_c(a, (C*)nullptr); }

// Streaming loads (ld.global.cs: evict-first) for data read exactly once per
// matvec, such as the kernel spectrum, so it does not displace reusable lines.
__device__ __forceinline__ float2 ld_stream(const float2* p) { return __ldcs(p); }
__device__ __forceinline__ double2 ld_stream(const double2* p) { return __ldcs(p); }

// Programmatic dependent launch. A kernel launched by launch_pdl may be scheduled while
// its predecessor in the stream is still draining; it calls pdl_wait() (griddepcontrol.
// wait: blocks until the predecessor grid has completed and its writes are visible; a
// no-op for an ordinary launch) before it reads anything, and pdl_trigger() to let its
// own successor's blocks be scheduled once every block of this grid has issued it. The
// successor's blocks then wait in hardware, not in a spin loop.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

inline cudaError_t launch_pdl(const void* f, dim3 grid, dim3 block, void** args, size_t smem, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, f, args);
}

// Asynchronous global -> shared copies (cp.async): one complex element per call,
// zero-filled without a read when ok is false (src must still be a valid address).
// Many copies stay in flight per thread; cp_async_wait_all() then a barrier
// makes them visible to the block.
__device__ __forceinline__ void cp_async_elem(float2* dst, const float2* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_elem(double2* dst, const double2* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 16 : 0) : "memory");
}
// 16 bytes, both addresses 16-byte aligned
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace msc
