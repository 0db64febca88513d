// Matvec kernel C: inverse FFT along y and y = s x - acc on the M x M window.
#include "mv_common.cuh"

namespace msc {

template <typename T, bool POW2>
__global__ void __launch_bounds__(256, 4) k_fft_y_out(const cx<T>* __restrict__ W, const cx<T>* __restrict__ x,
                                                      const double* scale, cx<T>* __restrict__ y, Geo g,
                                                      FftPlan1D pl, const cx<T>* __restrict__ twg, const int* done) {
  if (done && *done) return;
  using C = cx<T>;
  constexpr int TR = Tile<T>::W;
  constexpr int P = TR + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* ta = tw + g.Ly;
  C* tb = ta + (size_t)g.Ly * P;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int c = blockIdx.z, m = blockIdx.y, x0 = blockIdx.x * TR;
  const int nr = min(TR, g.M - x0);
  for (int t = tid; t < g.Ly; t += nthr) tw[t] = twg[t];
  const C* Wl = W + ((size_t)(c * g.Nz + m) * g.Ly) * g.Lx + x0;
  for (int it = tid; it < TR * g.Ly; it += nthr) {
    const int r = it & (TR - 1), ky = it / TR;  // TR is a power of two
    ta[ky * P + r] = (r < nr) ? Wl[(size_t)ky * g.Lx + r] : czero<C>();
  }
  __syncthreads();
  const C* res = fft_tile<+1, POW2>(ta, tb, P, TR, pl, tw, tid, nthr);
  const T s = load_scale<T>(scale);
  {
    QR w(tid, nthr, g.M);  // (row, j)
    const size_t base = (size_t)c * g.nsite + (size_t)(m * g.M + x0) * g.M;
    for (int it = tid; it < TR * g.M; it += nthr, w.next()) {
      if (w.q < nr) {
        const size_t idx = base + (size_t)w.q * g.M + w.r;
        y[idx] = s * x[idx] - res[w.r * P + w.q];
      }
    }
  }
}

template <typename T>
int launch_fft_y_out(msc_plan* pl, const cx<T>* W, const cx<T>* x, const double* scale, cx<T>* y, const cx<T>* tw,
                     const int* done) {
  const Geo& g = pl->g;
  constexpr int TR = Tile<T>::W;
  const int nthr = 256;
  const size_t sm = sizeof(cx<T>) * ((size_t)g.Ly + 2 * (size_t)g.Ly * (TR + 1));
  dim3 grid((unsigned)((g.M + TR - 1) / TR), (unsigned)g.Nz, 9);
#define CALL(P2)                                                                                   \
  {                                                                                                \
    MSC_CUDA(prep_kernel((const void*)k_fft_y_out<T, P2>));                                        \
    k_fft_y_out<T, P2><<<grid, nthr, sm, pl->stream>>>(W, x, scale, y, g, pl->fxy, tw, done);      \
    ::msc::note_launch();                                                                          \
  }
  MSC_POW2_DISPATCH(pl->fxy.pow2, CALL);
#undef CALL
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}
template int launch_fft_y_out<float>(msc_plan*, const float2*, const float2*, const double*, float2*, const float2*,
                                     const int*);
template int launch_fft_y_out<double>(msc_plan*, const double2*, const double2*, const double*, double2*,
                                      const double2*, const int*);

}  // namespace msc
