// Line FFT along the contiguous axis (the x passes of the matvec and of the G0 build).
#include "mv_common.cuh"

namespace msc {

// Lines l in [0, nlines) start at off(l) = (l / G) * GS + (l % G) * stride in both
// in and out (groups of G equally spaced lines, groups GS apart); the first n_in
// inputs are used (rest zero), the first n_out outputs are written.
template <typename T, int DIR, bool POW2>
__global__ void __launch_bounds__(256, 4) k_fft_contig(const cx<T>* in, cx<T>* out, long long nlines, long long G,
                                                       long long GS, long long stride, int n_in, int n_out,
                                                       FftPlan1D pl, const cx<T>* __restrict__ twg, const int* done) {
  if (done && *done) return;
  using C = cx<T>;
  constexpr int TL = Tile<T>::W;
  constexpr int P = TL + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* ta = tw + pl.L;
  C* tb = ta + (size_t)pl.L * P;
  __shared__ long long loff[TL];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const long long line0 = (long long)blockIdx.x * TL;
  if (tid < TL) {
    const long long ln = line0 + tid;
    loff[tid] = ln < nlines ? (ln / G) * GS + (ln % G) * stride : -1;
  }
  for (int t = tid; t < pl.L; t += nthr) tw[t] = twg[t];
  __syncthreads();
  {
    QR w(tid, nthr, pl.L);  // (line, x)
    for (int it = tid; it < TL * pl.L; it += nthr, w.next()) {
      const long long o = loff[w.q];
      ta[w.r * P + w.q] = (o >= 0 && w.r < n_in) ? in[o + w.r] : czero<C>();
    }
  }
  __syncthreads();
  const C* res = fft_tile<DIR, POW2>(ta, tb, P, TL, pl, tw, tid, nthr);
  {
    QR w(tid, nthr, n_out);
    for (int it = tid; it < TL * n_out; it += nthr, w.next()) {
      const long long o = loff[w.q];
      if (o >= 0) out[o + w.r] = res[w.r * P + w.q];
    }
  }
}

template <typename T>
int launch_fft_contig(msc_plan* pl, const cx<T>* in, cx<T>* out, long long nlines, long long G, long long GS,
                      long long stride, int n_in, int n_out, const FftPlan1D& f, const cx<T>* tw, int dir,
                      const int* done) {
  constexpr int TL = Tile<T>::W;
  const int nthr = 256;
  const size_t sm = sizeof(cx<T>) * ((size_t)f.L + 2 * (size_t)f.L * (TL + 1));
  const unsigned nb = (unsigned)((nlines + TL - 1) / TL);
#define CALL(P2)                                                                                                 \
  {                                                                                                              \
    auto kern = (dir < 0) ? k_fft_contig<T, -1, P2> : k_fft_contig<T, +1, P2>;                                   \
    MSC_CUDA(prep_kernel((const void*)kern));                                                                    \
    kern<<<nb, nthr, sm, pl->stream>>>(in, out, nlines, G, GS, stride, n_in, n_out, f, tw, done);         \
    ::msc::note_launch();                                                                                        \
  }
  MSC_POW2_DISPATCH(f.pow2, CALL);
#undef CALL
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}
template int launch_fft_contig<float>(msc_plan*, const float2*, float2*, long long, long long, long long, long long,
                                      int, int, const FftPlan1D&, const float2*, int, const int*);
template int launch_fft_contig<double>(msc_plan*, const double2*, double2*, long long, long long, long long,
                                       long long, int, int, const FftPlan1D&, const double2*, int, const int*);

}  // namespace msc
