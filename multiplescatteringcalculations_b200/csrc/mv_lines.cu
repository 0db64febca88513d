// Line FFT along the contiguous axis (the x passes of the matvec and of the G0 build).
#include "mv_common.cuh"

namespace msc {

// Lines l in [0, nlines) start at off(l) = (l / G) * GS + (l % G) * stride in both
// in and out (groups of G equally spaced lines, groups GS apart); the first n_in
// inputs are used (rest zero), the first n_out outputs are written. A block takes
// TL lines; its gather is a set of cp.async copies awaited once. LC > 0: the
// length is the compile-time power of two LC (<= the block size), so a thread
// keeps one element index x = tid % LC in the gather and the store. PR (with LC):
// the forward transform has n_in <= LC/2 (its first stage reads only x < LC/2),
// the inverse n_out <= LC/2 (its last stage computes only x < LC/2).
template <typename T, int DIR, bool POW2, int LC, bool PR>
__global__ void __launch_bounds__(256, 4) k_fft_contig(const cx<T>* in, cx<T>* out, long long nlines, long long G,
                                                       long long GS, long long stride, int n_in, int n_out,
                                                       FftPlan1D pl, const cx<T>* __restrict__ twg, const int* done) {
  if (done && *done) return;
  using C = cx<T>;
  constexpr int TL = Tile<T>::W;
  constexpr int P = TL + 1;
  constexpr int NT = 256;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L = LC > 0 ? LC : pl.L;
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* ta = tw + L;
  C* tb = ta + (size_t)L * P;
  __shared__ long long loff[TL];
  const int tid = threadIdx.x;
  const long long line0 = (long long)blockIdx.x * TL;
  if (tid < TL) {
    const long long ln = line0 + tid;
    loff[tid] = ln < nlines ? (ln / G) * GS + (ln % G) * stride : -1;
  }
  for (int t = tid; t < L; t += NT) tw[t] = twg[t];
  __syncthreads();
  const C* res;
  if constexpr (LC > 0) {
    static_assert(NT % LC == 0, "length divides the block");
    constexpr int QS = NT / LC;  // lines per sweep
    const int x = tid % LC, q0 = tid / LC;
    constexpr bool HIN = PR && DIR < 0, HOUT = PR && DIR > 0;
    if (!HIN || x < LC / 2) {
#pragma unroll
      for (int k = 0; k < (TL + QS - 1) / QS; ++k) {
        const int q = q0 + k * QS;
        if (QS > TL && q >= TL) break;
        const long long o = loff[q];
        const bool ok = o >= 0 && x < n_in;
        cp_async_elem(ta + x * P + q, ok ? in + o + x : in, ok);
      }
    }
    cp_async_wait_all();
    __syncthreads();
    res = fft_tile_ct<LC, DIR, P, TL, NT, HIN, HOUT>(ta, tb, tw, tid);
    if (x < n_out) {
#pragma unroll
      for (int k = 0; k < (TL + QS - 1) / QS; ++k) {
        const int q = q0 + k * QS;
        if (QS > TL && q >= TL) break;
        const long long o = loff[q];
        if (o >= 0) out[o + x] = res[x * P + q];
      }
    }
  } else {
    {
      QR w(tid, NT, L);  // (line, x)
      for (int it = tid; it < TL * L; it += NT, w.next()) {
        const long long o = loff[w.q];
        const bool ok = o >= 0 && w.r < n_in;
        cp_async_elem(ta + w.r * P + w.q, ok ? in + o + w.r : in, ok);
      }
    }
    cp_async_wait_all();
    __syncthreads();
    res = fft_tile<DIR, POW2>(ta, tb, P, TL, pl, tw, tid, NT);
    QR w(tid, NT, n_out);
    for (int it = tid; it < TL * n_out; it += NT, w.next()) {
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
  const void* kern = nullptr;
  const bool pr = 2 * (dir < 0 ? n_in : n_out) <= f.L;
#define LEN(D, LL) \
  kern = pr ? (const void*)k_fft_contig<T, D, true, LL, true> : (const void*)k_fft_contig<T, D, true, LL, false>;
#define PICK(D)                                                                                                  \
  switch (f.L) {                                                                                                 \
    case 16: LEN(D, 16) break;                                                                                   \
    case 32: LEN(D, 32) break;                                                                                   \
    case 64: LEN(D, 64) break;                                                                                   \
    case 128: LEN(D, 128) break;                                                                                 \
    case 256: LEN(D, 256) break;                                                                                 \
    default:                                                                                                     \
      kern = f.pow2 ? (const void*)k_fft_contig<T, D, true, 0, false> : (const void*)k_fft_contig<T, D, false, 0, false>; \
  }
  if (dir < 0) { PICK(-1) } else { PICK(+1) }
#undef PICK
#undef LEN
  MSC_CUDA(prep_kernel(kern));
  FftPlan1D ff = f;
  void* args[] = {(void*)&in, (void*)&out, (void*)&nlines, (void*)&G, (void*)&GS, (void*)&stride,
                  (void*)&n_in, (void*)&n_out, (void*)&ff, (void*)&tw, (void*)&done};
  MSC_CUDA(cudaLaunchKernel(kern, dim3(nb), dim3(nthr), args, sm, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}
template int launch_fft_contig<float>(msc_plan*, const float2*, float2*, long long, long long, long long, long long,
                                      int, int, const FftPlan1D&, const float2*, int, const int*);
template int launch_fft_contig<double>(msc_plan*, const double2*, double2*, long long, long long, long long,
                                       long long, int, int, const FftPlan1D&, const double2*, int, const int*);

}  // namespace msc
