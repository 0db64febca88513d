// Line FFT along a strided axis (the z passes of the matvec, the y and z passes
// of the G0 build).
//
// Element idx of column col in slab (s1, s2) is read at
//   in + s1*S1 + s2*S2 + idx*es + col      (idx < n_in; zero beyond)
// and written at
//   out + s1*O1 + s2*O2 + idx*eo + col     (idx < n_out)
// with an optional complex64 copy at the same offsets of out32. A block takes TC
// consecutive columns of one slab.
#include "mv_common.cuh"

namespace msc {

template <typename T, int DIR, bool POW2, bool MIRROR>
__global__ void __launch_bounds__(256, 3) k_fft_strided(const cx<T>* in, long long es, long long S1, long long S2,
                                                        cx<T>* out, long long eo, long long O1, long long O2,
                                                        float2* out32, int ncol, int TC, int n_in, int n_out,
                                                        FftPlan1D pl, const cx<T>* __restrict__ twg, const int* done,
                                                        unsigned long long odd_lo, unsigned long long odd_hi) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  using C = cx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int P = TC + 1;
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* ta = tw + pl.L;
  C* tb = ta + (size_t)pl.L * P;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int col0 = blockIdx.x * TC;
  const int nc = min(TC, ncol - col0);
  const long long ib = (long long)blockIdx.y * S1 + (long long)blockIdx.z * S2 + col0;
  const long long ob = (long long)blockIdx.y * O1 + (long long)blockIdx.z * O2 + col0;
  for (int t = tid; t < pl.L; t += nthr) tw[t] = twg[t];
  {
    // MIRROR: idx >= n_in is the sign-flipped (odd entry) or plain mirror L - idx
    const int sl = blockIdx.z;
    const bool odd = MIRROR && ((sl < 64 ? (odd_lo >> sl) : (odd_hi >> (sl - 64))) & 1ull);
    QR w(tid, nthr, TC);  // (idx, column)
    for (int it = tid; it < TC * pl.L; it += nthr, w.next()) {
      C v = czero<C>();
      if (w.r < nc) {
        if (w.q < n_in) {
          v = in[ib + (long long)w.q * es + w.r];
        } else if (MIRROR) {
          v = in[ib + (long long)(pl.L - w.q) * es + w.r];
          if (odd) {
            v.x = -v.x;
            v.y = -v.y;
          }
        }
      }
      ta[w.q * P + w.r] = v;
    }
  }
  __syncthreads();
  const C* res = fft_tile<DIR, POW2>(ta, tb, P, TC, pl, tw, tid, nthr);
  {
    QR w(tid, nthr, TC);
    for (int it = tid; it < TC * n_out; it += nthr, w.next()) {
      if (w.r < nc) {
        const C v = res[w.q * P + w.r];
        const long long o = ob + (long long)w.q * eo + w.r;
        out[o] = v;
        if (out32) out32[o] = make_float2((float)v.x, (float)v.y);
      }
    }
  }
}

// Columns per block: up to 128 (and at most ncol), shared memory <= 72 KB.
template <typename T> static int strided_columns(int L, int ncol) {
  int tc = 128;
  while (tc > 8 && (tc > ncol * 2 || sizeof(cx<T>) * ((size_t)L + 2 * (size_t)L * (tc + 1)) > 72 * 1024)) tc /= 2;
  return tc;
}

template <typename T>
int launch_fft_strided(msc_plan* pl, const cx<T>* in, long long es, long long S1, long long S2, cx<T>* out,
                       long long eo, long long O1, long long O2, float2* out32, int ncol, int n1, int n2, int n_in,
                       int n_out, const FftPlan1D& f, const cx<T>* tw, int dir, const int* done,
                       const unsigned long long* odd) {
  const int TC = strided_columns<T>(f.L, ncol);
  if (odd && (n_in != f.L / 2 + 1 || n2 > 128)) {
    set_error("mirrored strided FFT: %d stored inputs of %d, %d slabs", n_in, f.L, n2);
    return MSC_ERR_UNSUPPORTED;
  }
  const unsigned long long olo = odd ? odd[0] : 0ull, ohi = odd ? odd[1] : 0ull;
  const int nthr = 256;
  if (TC > nthr) {
    set_error("strided FFT tile of %d columns exceeds the block", TC);
    return MSC_ERR_UNSUPPORTED;
  }
  const size_t sm = sizeof(cx<T>) * ((size_t)f.L + 2 * (size_t)f.L * (TC + 1));
  dim3 grid((unsigned)((ncol + TC - 1) / TC), (unsigned)n1, (unsigned)n2);
#define CALL(P2)                                                                                              \
  {                                                                                                           \
    auto kern = odd ? ((dir < 0) ? k_fft_strided<T, -1, P2, true> : k_fft_strided<T, +1, P2, true>)            \
                    : ((dir < 0) ? k_fft_strided<T, -1, P2, false> : k_fft_strided<T, +1, P2, false>);         \
    MSC_CUDA(prep_kernel((const void*)kern));                                                                 \
    kern<<<grid, nthr, sm, pl->stream>>>(in, es, S1, S2, out, eo, O1, O2, out32, ncol, TC, n_in, n_out, f, tw, \
                                         done, olo, ohi);                                                     \
    ::msc::note_launch();                                                                                     \
  }
  MSC_POW2_DISPATCH(f.pow2, CALL);
#undef CALL
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}
template int launch_fft_strided<float>(msc_plan*, const float2*, long long, long long, long long, float2*, long long,
                                       long long, long long, float2*, int, int, int, int, int, const FftPlan1D&,
                                       const float2*, int, const int*, const unsigned long long*);
template int launch_fft_strided<double>(msc_plan*, const double2*, long long, long long, long long, double2*,
                                        long long, long long, long long, float2*, int, int, int, int, int,
                                        const FftPlan1D&, const double2*, int, const int*,
                                        const unsigned long long*);

}  // namespace msc
