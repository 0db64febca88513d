// Generated by gen_radix_constants.py: cos/sin(2*pi*q/R), q = 0..R-1, for the odd
// FFT radices. Correctly rounded from 50-digit values.
#pragma once
namespace msc {
template <int R> struct RadixTrig;
template <> struct RadixTrig<3> {
  static __host__ __device__ constexpr double c(int q) { constexpr double t[3] = {1.0, -0.5, -0.5}; return t[q]; }
  static __host__ __device__ constexpr double s(int q) { constexpr double t[3] = {0.0, 0.8660254037844386, -0.8660254037844386}; return t[q]; }
};
template <> struct RadixTrig<5> {
  static __host__ __device__ constexpr double c(int q) { constexpr double t[5] = {1.0, 0.30901699437494745, -0.8090169943749475, -0.8090169943749475, 0.30901699437494745}; return t[q]; }
  static __host__ __device__ constexpr double s(int q) { constexpr double t[5] = {0.0, 0.9510565162951535, 0.5877852522924731, -0.5877852522924731, -0.9510565162951535}; return t[q]; }
};
template <> struct RadixTrig<7> {
  static __host__ __device__ constexpr double c(int q) { constexpr double t[7] = {1.0, 0.6234898018587335, -0.2225209339563144, -0.9009688679024191, -0.9009688679024191, -0.2225209339563144, 0.6234898018587335}; return t[q]; }
  static __host__ __device__ constexpr double s(int q) { constexpr double t[7] = {0.0, 0.7818314824680298, 0.9749279121818236, 0.4338837391175581, -0.4338837391175581, -0.9749279121818236, -0.7818314824680298}; return t[q]; }
};
template <> struct RadixTrig<11> {
  static __host__ __device__ constexpr double c(int q) { constexpr double t[11] = {1.0, 0.8412535328311812, 0.41541501300188644, -0.14231483827328514, -0.6548607339452851, -0.9594929736144974, -0.9594929736144974, -0.6548607339452851, -0.14231483827328514, 0.41541501300188644, 0.8412535328311812}; return t[q]; }
  static __host__ __device__ constexpr double s(int q) { constexpr double t[11] = {0.0, 0.5406408174555976, 0.9096319953545183, 0.9898214418809327, 0.7557495743542583, 0.28173255684142967, -0.28173255684142967, -0.7557495743542583, -0.9898214418809327, -0.9096319953545183, -0.5406408174555976}; return t[q]; }
};
}  // namespace msc
