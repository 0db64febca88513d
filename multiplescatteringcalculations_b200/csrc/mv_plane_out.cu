// Matvec kernel C: inverse FFT along y and y = s x - acc on the M x M window.
#include "mv_common.cuh"

namespace msc {

// ---- C: inverse FFT along y + y = s*x - acc -----------------------------------------
template <typename T, int KMAX>
__global__ void __launch_bounds__(256) k_fft_y_out(const cx<T>* __restrict__ W, const cx<T>* __restrict__ x,
                                                   const double* scale, cx<T>* __restrict__ y, Geo g, FftPlan1D pl,
                                                   const cx<T>* __restrict__ twg, const int* done) {
  if (done && *done) return;
  constexpr int TR = Tile<T>::W;
  constexpr int P = TR + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* tw = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* tile = tw + g.Ly;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int c = blockIdx.z, m = blockIdx.y, x0 = blockIdx.x * TR;
  const int nr = min(TR, g.M - x0);
  for (int t = tid; t < g.Ly; t += nthr) tw[t] = twg[t];
  const cx<T>* Wl = W + ((size_t)(c * g.Nz + m) * g.Ly) * g.Lx + x0;
  for (int it = tid; it < TR * g.Ly; it += nthr) {
    const int r = it % TR, ky = it / TR;
    tile[ky * P + r] = (r < nr) ? Wl[(size_t)ky * g.Lx + r] : czero<cx<T>>();
  }
  __syncthreads();
  fft_tile<+1, KMAX>(tile, P, TR, pl, tw, tid, nthr);
  const T s = load_scale<T>(scale);
  for (int it = tid; it < TR * g.M; it += nthr) {
    const int j = it % g.M, r = it / g.M;
    if (r < nr) {
      const size_t idx = (size_t)c * g.nsite + (size_t)(m * g.M + x0 + r) * g.M + j;
      y[idx] = s * x[idx] - tile[j * P + r];
    }
  }
}

template <typename T>
int launch_fft_y_out(msc_plan* pl, const cx<T>* W, const cx<T>* x, const double* scale, cx<T>* y, const cx<T>* tw,
                     const int* done) {
  const Geo& g = pl->g;
  constexpr int TR = Tile<T>::W;
  const int nthr = 256;
  const size_t sm = sizeof(cx<T>) * ((size_t)g.Ly + (size_t)g.Ly * (TR + 1));
  const int kmax = fft_kmax_needed(pl->fxy, TR, nthr);
  dim3 grid((unsigned)((g.M + TR - 1) / TR), (unsigned)g.Nz, 9);
#define CALL(K)                                                                                               \
  {                                                                                                           \
    MSC_CUDA(cudaFuncSetAttribute(k_fft_y_out<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));  \
    k_fft_y_out<T, K><<<grid, nthr, sm, pl->stream>>>(W, x, scale, y, g, pl->fxy, tw, done);                  \
  }
  MSC_KMAX_DISPATCH(kmax, CALL);
#undef CALL
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}
template int launch_fft_y_out<float>(msc_plan*, const float2*, const float2*, const double*, float2*, const float2*,
                                     const int*);
template int launch_fft_y_out<double>(msc_plan*, const double2*, const double2*, const double*, double2*,
                                      const double2*, const int*);
}  // namespace msc
