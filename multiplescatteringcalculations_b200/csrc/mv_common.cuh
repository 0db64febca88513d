// Shared pieces of the matvec translation units.
#pragma once
#include "plan.cuh"

namespace msc {

template <typename T> struct Tile { static constexpr int W = 128 / (int)sizeof(cx<T>); };  // 16 (c64) / 8 (c128)

template <typename T> __device__ __forceinline__ T load_scale(const double* s) { return s ? (T)(*s) : (T)1; }

#define MSC_KMAX_DISPATCH(kmax, CALL) \
  do {                                \
    if ((kmax) <= 1) { CALL(1); }     \
    else if ((kmax) <= 2) { CALL(2); } \
    else if ((kmax) <= 4) { CALL(4); } \
    else if ((kmax) <= 8) { CALL(8); } \
    else { set_error("FFT tile needs KMAX=%d > 8", (int)(kmax)); return MSC_ERR_UNSUPPORTED; } \
  } while (0)


// Kernel launchers (one translation unit each).
template <typename T>
int launch_fft_contig(msc_plan* pl, const cx<T>* in, cx<T>* out, long long nlines, long long in_stride,
                      long long out_stride, int n_in, int n_out, const FftPlan1D& f, const cx<T>* tw, int dir,
                      const int* done);
template <typename T>
int launch_t0_fft_y(msc_plan* pl, const cx<T>* x, const double* scale, cx<T>* W, const cx<T>* tw, const int* done);
template <typename T>
int launch_zfft_block(msc_plan* pl, cx<T>* W, const cx<T>* tw, const int* done);
template <typename T>
int launch_fft_y_out(msc_plan* pl, const cx<T>* W, const cx<T>* x, const double* scale, cx<T>* y, const cx<T>* tw,
                     const int* done);

}  // namespace msc
