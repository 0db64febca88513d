// Line FFT along the contiguous axis (the x passes of the matvec and of the G0 build).
#include "mv_common.cuh"

namespace msc {

// ---- generic line FFT along the contiguous axis (X and X') ---------------------------
// Lines l in [0, nlines) at in + l*in_stride; the first n_in inputs are used (rest zero);
// the first n_out outputs are written to out + l*out_stride.
template <typename T, int DIR, int KMAX>
__global__ void __launch_bounds__(256) k_fft_contig(const cx<T>* in, cx<T>* out, long long nlines, long long in_stride,
                                                    long long out_stride, int n_in, int n_out, FftPlan1D pl,
                                                    const cx<T>* __restrict__ twg, const int* done) {
  if (done && *done) return;
  constexpr int TL = Tile<T>::W;
  constexpr int P = TL + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* tile = tw + pl.L;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const long long line0 = (long long)blockIdx.x * TL;
  const int nl = (int)min((long long)TL, nlines - line0);
  for (int t = tid; t < pl.L; t += nthr) tw[t] = twg[t];
  for (int it = tid; it < TL * n_in; it += nthr) {
    const int l = it / n_in, xx = it % n_in;
    tile[xx * P + l] = (l < nl) ? in[(line0 + l) * in_stride + xx] : czero<cx<T>>();
  }
  for (int it = tid; it < TL * (pl.L - n_in); it += nthr) {
    const int l = it % TL, xx = n_in + it / TL;
    tile[xx * P + l] = czero<cx<T>>();
  }
  __syncthreads();
  fft_tile<DIR, KMAX>(tile, P, TL, pl, tw, tid, nthr);
  for (int it = tid; it < TL * n_out; it += nthr) {
    const int l = it / n_out, xx = it % n_out;
    if (l < nl) out[(line0 + l) * out_stride + xx] = tile[xx * P + l];
  }
}

template <typename T>
int launch_fft_contig(msc_plan* pl, const cx<T>* in, cx<T>* out, long long nlines, long long in_stride,
                      long long out_stride, int n_in, int n_out, const FftPlan1D& f, const cx<T>* tw, int dir,
                      const int* done) {
  constexpr int TL = Tile<T>::W;
  const int nthr = 256;
  const size_t sm = sizeof(cx<T>) * ((size_t)f.L + (size_t)f.L * (TL + 1));
  const int kmax = fft_kmax_needed(f, TL, nthr);
  const unsigned nb = (unsigned)((nlines + TL - 1) / TL);
#define CALL(K)                                                                                          \
  {                                                                                                      \
    auto kern = (dir < 0) ? k_fft_contig<T, -1, K> : k_fft_contig<T, +1, K>;                             \
    MSC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));          \
    kern<<<nb, nthr, sm, pl->stream>>>(in, out, nlines, in_stride, out_stride, n_in, n_out, f, tw, done); \
  }
  MSC_KMAX_DISPATCH(kmax, CALL);
#undef CALL
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}
template int launch_fft_contig<float>(msc_plan*, const float2*, float2*, long long, long long, long long, int, int,
                                      const FftPlan1D&, const float2*, int, const int*);
template int launch_fft_contig<double>(msc_plan*, const double2*, double2*, long long, long long, long long, int, int,
                                       const FftPlan1D&, const double2*, int, const int*);

}  // namespace msc
