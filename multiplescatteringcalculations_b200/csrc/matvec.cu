// The slab operator y = (I - G0 T0) x as a 3D FFT convolution over the padded
// (Lz, Lx, Ly) grid, the B200 replacement of _slab_matvec_gpu
// (tmnestor/MultipleScatteringCalculations cubic_scattering/slab_scattering_gpu.py:95-155).
//
// Five launches, every one a shared-memory line-FFT pass:
//   A  tau = T0 x (4 scalars per site), zero padded, FFT along y  -> W[c][n][ky][x]
//   X  FFT along x (only x < M nonzero)                           -> W[c][n][ky][kx]
//   B  per (kx, ky) column pair {k, -k}: zero pad z, FFT along z, 9x9 block multiply
//      by the stored half-space spectrum (K(-k) = S K(k) S, S = diag(1,1,1,-1 x6)),
//      inverse FFT along z, keep the N_z output planes                 -> W
//   X' inverse FFT along kx, keep x < M                            -> W[c][m][ky][x]
//   C  inverse FFT along ky, y = scale*x - acc on the M x M window  -> y
// The kernel spectrum carries the 1/(Lz Lx Ly) normalisation. W is 9*N_z*Ly*Lx
// complex and stays L2-resident at the benchmark sizes; the spectrum is streamed
// once per matvec with evict-first loads.
#include "mv_common.cuh"

namespace msc {

template <typename T>
int launch_matvec(msc_plan* pl, const cx<T>* x, const double* scale, cx<T>* y, const int* done) {
  const Geo& g = pl->g;
  if (!pl->has_t0 || !pl->has_g0) {
    set_error("matvec needs build_t0 and build_g0 first");
    return MSC_ERR_STATE;
  }
  cx<T>* W = (cx<T>*)(sizeof(T) == 8 ? pl->W64.p : pl->W32.p);
  const cx<T>* twz = (const cx<T>*)(sizeof(T) == 8 ? pl->tw64_z.p : pl->tw32_z.p);
  const cx<T>* twxy = (const cx<T>*)(sizeof(T) == 8 ? pl->tw64_xy.p : pl->tw32_xy.p);
  MSC_TRY(launch_t0_fft_y<T>(pl, x, scale, W, twxy, done));                                                  // A
  MSC_TRY(launch_fft_contig<T>(pl, W, W, (long long)9 * g.Nz * g.Ly, g.Lx, g.Lx, g.M, g.Lx, pl->fxy, twxy, -1, done));  // X
  MSC_TRY(launch_zfft_block<T>(pl, W, twz, done));                                                           // B
  MSC_TRY(launch_fft_contig<T>(pl, W, W, (long long)9 * g.Nz * g.Ly, g.Lx, g.Lx, g.Lx, g.M, pl->fxy, twxy, +1, done));  // X'
  MSC_TRY(launch_fft_y_out<T>(pl, W, x, scale, y, twxy, done));                                              // C
  return MSC_OK;
}

template int launch_matvec<float>(msc_plan*, const float2*, const double*, float2*, const int*);
template int launch_matvec<double>(msc_plan*, const double2*, const double*, double2*, const int*);

}  // namespace msc
