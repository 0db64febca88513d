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
// [y][row] (zero for y >= M), FFT along y, store W[c][n][ky][i0 + row]. LC > 0:
// compile-time power-of-two Ly = LC; a thread keeps y = tid % LC. PR (with LC):
// M <= LC/2, the first FFT stage reads only y < LC/2.
template <typename T, bool POW2, int LC, bool PR>
__global__ void __launch_bounds__(256, 4) k_t0_fft_y(const cx<T>* __restrict__ x, const double* scale,
                                                     const cx<T>* __restrict__ t4, cx<T>* __restrict__ W, Geo g,
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
  // blockIdx.z = 9 rh + c: component c of right-hand side rh (fields and workspaces
  // of the right-hand sides follow each other)
  const int c = blockIdx.z % 9, n = blockIdx.y, i0 = blockIdx.x * TR;
  {
    const size_t rh = blockIdx.z / 9;
    x += rh * 9 * (size_t)g.nsite;
    W += rh * 9 * (size_t)g.Nz * g.Ly * g.Lx;
  }
  const int nr = min(TR, g.M - i0);
  const T s = load_scale<T>(scale);
  for (int t = tid; t < Ly; t += NT) tw[t] = twg[t];
  const int base = (n * g.M + i0) * g.M;
  const C* res;
  // rows r < nr hold tau; y >= M and rows >= nr are zero
  if constexpr (LC > 0) {
    constexpr int QS = NT / LC;
    const int y = tid % LC, q0 = tid / LC;
    if (!PR || y < LC / 2) {
#pragma unroll
      for (int k = 0; k < (TR + QS - 1) / QS; ++k) {
        const int q = q0 + k * QS;
        if (QS > TR && q >= TR) break;
        C v = czero<C>();
        if (y < g.M && q < nr) v = s * tau_component<T>(x, t4, g.nsite, base + q * g.M + y, c);
        ta[y * P + q] = v;
      }
    }
    __syncthreads();
    res = fft_tile_ct<LC, -1, P, TR, NT, PR, false>(ta, tb, tw, tid);
  } else {
    QR w(tid, NT, Ly);  // (row, y)
    for (int it = tid; it < TR * Ly; it += NT, w.next()) {
      C v = czero<C>();
      if (w.r < g.M && w.q < nr) v = s * tau_component<T>(x, t4, g.nsite, base + w.q * g.M + w.r, c);
      ta[w.r * P + w.q] = v;
    }
    __syncthreads();
    res = fft_tile<-1, POW2>(ta, tb, P, TR, pl, tw, tid, NT);
  }
  C* Wl = W + ((size_t)(c * g.Nz + n) * g.Ly) * g.Lx + i0;
  const int r = tid & (TR - 1);  // TR is a power of two dividing NT
  if (r < nr) {
#pragma unroll 4
    for (int ky = tid / TR; ky < Ly; ky += NT / TR) Wl[(size_t)ky * g.Lx + r] = res[ky * P + r];
  }
}

template <typename T>
int launch_t0_fft_y(msc_plan* pl, const cx<T>* x, const double* scale, cx<T>* W, const cx<T>* tw, const int* done,
                    int nrhs) {
  const Geo& g = pl->g;
  constexpr int TR = Tile<T>::W;
  const cx<T>* t4 = (const cx<T>*)(sizeof(T) == 8 ? pl->t4_64.p : pl->t4_32.p);
  const int nthr = 256;
  const size_t sm = sizeof(cx<T>) * ((size_t)g.Ly + 2 * (size_t)g.Ly * (TR + 1));
  dim3 grid((unsigned)((g.M + TR - 1) / TR), (unsigned)g.Nz, 9u * (unsigned)nrhs);
  const void* kern;
  const bool pr = 2 * g.M <= g.Ly;
#define LEN(LL) kern = pr ? (const void*)k_t0_fft_y<T, true, LL, true> : (const void*)k_t0_fft_y<T, true, LL, false>;
  switch (g.Ly) {
    case 16: LEN(16) break;
    case 32: LEN(32) break;
    case 64: LEN(64) break;
    case 128: LEN(128) break;
    case 256: LEN(256) break;
    default:
      kern = pl->fxy.pow2 ? (const void*)k_t0_fft_y<T, true, 0, false> : (const void*)k_t0_fft_y<T, false, 0, false>;
  }
#undef LEN
  MSC_CUDA(prep_kernel(kern));
  Geo gg = g;
  FftPlan1D ff = pl->fxy;
  void* args[] = {(void*)&x, (void*)&scale, (void*)&t4, (void*)&W, (void*)&gg, (void*)&ff, (void*)&tw, (void*)&done};
  MSC_CUDA(launch_pdl(kern, grid, dim3(nthr), args, sm, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}
template int launch_t0_fft_y<float>(msc_plan*, const float2*, const double*, float2*, const float2*, const int*, int);
template int launch_t0_fft_y<double>(msc_plan*, const double2*, const double*, double2*, const double2*, const int*,
                                     int);

}  // namespace msc
