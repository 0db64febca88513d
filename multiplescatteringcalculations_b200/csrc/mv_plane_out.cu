// Matvec kernel C: inverse FFT along y and y = s x - acc on the M x M window.
#include "mv_common.cuh"

namespace msc {

// Block (x-tile of TR rows, layer m, component c): W rows [ky][row] (cp.async),
// inverse FFT along y, y = s x - acc for the rows of the tile. LC > 0:
// compile-time power-of-two Ly = LC. PR (with LC): M <= LC/2, the last FFT stage
// computes only y < LC/2.
template <typename T, bool POW2, int LC, bool PR>
__global__ void __launch_bounds__(256, 4) k_fft_y_out(const cx<T>* __restrict__ W, const cx<T>* __restrict__ x,
                                                      const double* scale, cx<T>* __restrict__ y, Geo g,
                                                      FftPlan1D pl, const cx<T>* __restrict__ twg, const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  using C = cx<T>;
  constexpr int TR = Tile<T>::W;
  constexpr int P = TR + 1;
  constexpr int NT = 256;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Ly = LC > 0 ? LC : g.Ly;
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* ta = tw + Ly;
  C* tb = ta + (size_t)Ly * P;
  const int tid = threadIdx.x;
  // blockIdx.z = 9 rh + c: component c of right-hand side rh
  const int c = blockIdx.z % 9, m = blockIdx.y, x0 = blockIdx.x * TR;
  {
    const size_t rh = blockIdx.z / 9;
    W += rh * 9 * (size_t)g.Nz * g.Ly * g.Lx;
    x += rh * 9 * (size_t)g.nsite;
    y += rh * 9 * (size_t)g.nsite;
  }
  const int nr = min(TR, g.M - x0);
  for (int t = tid; t < Ly; t += NT) tw[t] = twg[t];
  const C* Wl = W + ((size_t)(c * g.Nz + m) * g.Ly) * g.Lx + x0;
  {
    const int r = tid & (TR - 1);  // TR is a power of two dividing NT
    const bool ok = r < nr;
    const int nky = LC > 0 ? (LC + NT / TR - 1) / (NT / TR) : (Ly - tid / TR + NT / TR - 1) / (NT / TR);
#pragma unroll 4
    for (int k = 0; k < nky; ++k) {
      const int ky = tid / TR + k * (NT / TR);
      if (ky >= Ly) break;
      cp_async_elem(ta + ky * P + r, ok ? Wl + (size_t)ky * g.Lx + r : Wl, ok);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  const C* res;
  if constexpr (LC > 0) res = fft_tile_ct<LC, +1, P, TR, NT, false, PR>(ta, tb, tw, tid);
  else res = fft_tile<+1, POW2>(ta, tb, P, TR, pl, tw, tid, NT);
  const T s = load_scale<T>(scale);
  {
    QR w(tid, NT, g.M);  // (row, j)
    const size_t base = (size_t)c * g.nsite + (size_t)(m * g.M + x0) * g.M;
    for (int it = tid; it < TR * g.M; it += NT, w.next()) {
      if (w.q < nr) {
        const size_t idx = base + (size_t)w.q * g.M + w.r;
        y[idx] = s * x[idx] - res[w.r * P + w.q];
      }
    }
  }
}

template <typename T>
int launch_fft_y_out(msc_plan* pl, const cx<T>* W, const cx<T>* x, const double* scale, cx<T>* y, const cx<T>* tw,
                     const int* done, int nrhs) {
  const Geo& g = pl->g;
  constexpr int TR = Tile<T>::W;
  const int nthr = 256;
  const size_t sm = sizeof(cx<T>) * ((size_t)g.Ly + 2 * (size_t)g.Ly * (TR + 1));
  dim3 grid((unsigned)((g.M + TR - 1) / TR), (unsigned)g.Nz, 9u * (unsigned)nrhs);
  const void* kern;
  const bool pr = 2 * g.M <= g.Ly;
#define LEN(LL) kern = pr ? (const void*)k_fft_y_out<T, true, LL, true> : (const void*)k_fft_y_out<T, true, LL, false>;
  switch (g.Ly) {
    case 16: LEN(16) break;
    case 32: LEN(32) break;
    case 64: LEN(64) break;
    case 128: LEN(128) break;
    case 256: LEN(256) break;
    default:
      kern = pl->fxy.pow2 ? (const void*)k_fft_y_out<T, true, 0, false> : (const void*)k_fft_y_out<T, false, 0, false>;
  }
#undef LEN
  MSC_CUDA(prep_kernel(kern));
  Geo gg = g;
  FftPlan1D ff = pl->fxy;
  void* args[] = {(void*)&W, (void*)&x, (void*)&scale, (void*)&y, (void*)&gg, (void*)&ff, (void*)&tw, (void*)&done};
  MSC_CUDA(launch_pdl(kern, grid, dim3(nthr), args, sm, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}
template int launch_fft_y_out<float>(msc_plan*, const float2*, const float2*, const double*, float2*, const float2*,
                                     const int*, int);
template int launch_fft_y_out<double>(msc_plan*, const double2*, const double2*, const double*, double2*,
                                      const double2*, const int*, int);

}  // namespace msc
