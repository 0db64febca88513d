// Matvec kernel A: T0 apply, zero padding and the forward FFT along y.
#include "mv_common.cuh"

namespace msc {

// tau_c = (T0 x)_c at a site: c<3 t_u x_c; 3..5 t_l (x3+x4+x5) + t_d x_c; 6..8 t_s x_c
template <typename T>
__device__ __forceinline__ cx<T> tau_component(const cx<T>* __restrict__ x, const cx<T>* __restrict__ t4, int nsite,
                                               int site, int c) {
  const cx<T> xc = x[(size_t)c * nsite + site];
  if (c < 3) return t4[site] * xc;
  if (c >= 6) return t4[(size_t)3 * nsite + site] * xc;
  const cx<T> tr = x[(size_t)3 * nsite + site] + x[(size_t)4 * nsite + site] + x[(size_t)5 * nsite + site];
  return t4[(size_t)1 * nsite + site] * tr + t4[(size_t)2 * nsite + site] * xc;
}

// Block (i-tile of TR rows, layer n, component c): tau rows along y into a tile
// [y][row] (zero for y >= M), FFT along y, store W[c][n][ky][i0 + row].
template <typename T, bool POW2>
__global__ void __launch_bounds__(256, 4) k_t0_fft_y(const cx<T>* __restrict__ x, const double* scale,
                                                     const cx<T>* __restrict__ t4, cx<T>* __restrict__ W, Geo g,
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
  const int c = blockIdx.z, n = blockIdx.y, i0 = blockIdx.x * TR;
  const int nr = min(TR, g.M - i0);
  const T s = load_scale<T>(scale);
  for (int t = tid; t < g.Ly; t += nthr) tw[t] = twg[t];
  // rows r < nr hold tau; y >= M and rows >= nr are zero
  {
    QR w(tid, nthr, g.Ly);  // (row, y)
    const int base = (n * g.M + i0) * g.M;
    for (int it = tid; it < TR * g.Ly; it += nthr, w.next()) {
      C v = czero<C>();
      if (w.r < g.M && w.q < nr) v = s * tau_component<T>(x, t4, g.nsite, base + w.q * g.M + w.r, c);
      ta[w.r * P + w.q] = v;
    }
  }
  __syncthreads();
  const C* res = fft_tile<-1, POW2>(ta, tb, P, TR, pl, tw, tid, nthr);
  C* Wl = W + ((size_t)(c * g.Nz + n) * g.Ly) * g.Lx + i0;
  for (int it = tid; it < TR * g.Ly; it += nthr) {
    const int r = it & (TR - 1), ky = it / TR;  // TR is a power of two
    if (r < nr) Wl[(size_t)ky * g.Lx + r] = res[ky * P + r];
  }
}

template <typename T>
int launch_t0_fft_y(msc_plan* pl, const cx<T>* x, const double* scale, cx<T>* W, const cx<T>* tw, const int* done) {
  const Geo& g = pl->g;
  constexpr int TR = Tile<T>::W;
  const cx<T>* t4 = (const cx<T>*)(sizeof(T) == 8 ? pl->t4_64.p : pl->t4_32.p);
  const int nthr = 256;
  const size_t sm = sizeof(cx<T>) * ((size_t)g.Ly + 2 * (size_t)g.Ly * (TR + 1));
  dim3 grid((unsigned)((g.M + TR - 1) / TR), (unsigned)g.Nz, 9);
#define CALL(P2)                                                                                   \
  {                                                                                                \
    MSC_CUDA(prep_kernel((const void*)k_t0_fft_y<T, P2>));                                         \
    k_t0_fft_y<T, P2><<<grid, nthr, sm, pl->stream>>>(x, scale, t4, W, g, pl->fxy, tw, done);      \
    ::msc::note_launch();                                                                          \
  }
  MSC_POW2_DISPATCH(pl->fxy.pow2, CALL);
#undef CALL
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}
template int launch_t0_fft_y<float>(msc_plan*, const float2*, const double*, float2*, const float2*, const int*);
template int launch_t0_fft_y<double>(msc_plan*, const double2*, const double*, double2*, const double2*, const int*);

}  // namespace msc
