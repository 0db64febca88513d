// The slab operator y = (I - G0 T0) x as a 3D FFT convolution over the padded
// (Lz, Lx, Ly) grid, the B200 replacement of _slab_matvec_gpu
// (tmnestor/MultipleScatteringCalculations cubic_scattering/slab_scattering_gpu.py:95-155).
//
// Five launches over the workspace W[c][n][ky][kx] (9 x N_z x Ly x Lx):
//   A    tau = T0 (s x) (4 scalars per site), zero padded, FFT along y
//   X    FFT along x (only x < M nonzero)
//   ZBZ' per column (ky, kx), all 9 components in shared memory: FFT along z
//        (zero padded to Lz), 9x9 block multiply by the kernel spectrum, inverse
//        FFT along z, keep the N_z layers
//   X'   inverse FFT along kx, keep x < M
//   C    inverse FFT along ky, y = s x - acc on the M x M window
// The x and y passes are shared-memory line FFTs on data that stays in L2 at the
// benchmark sizes; the z-padded spectrum exists only inside ZBZ'. The kernel
// spectrum carries the 1/(Lz Lx Ly) normalisation.
//
// Several right-hand sides (msc_solve_multi, msc_matvec_multi): the fields and
// workspaces of R vectors follow each other; the plane passes take the right-hand
// side from the grid (blockIdx.z), the x passes run over all R workspaces' rows in
// one launch, and each ZBZ' block stages its slice of the spectrum once and applies
// it to the same columns of all R vectors in turn.
#include "mv_common.cuh"

namespace msc {

template <typename T>
int launch_matvec_ws(msc_plan* pl, const cx<T>* x, const double* scale, cx<T>* y, cx<T>* W, const int* done,
                     int nrhs) {
  const Geo& g = pl->g;
  if (!pl->has_t0 || !pl->has_g0) {
    set_error("matvec needs build_t0 and build_g0 first");
    return MSC_ERR_STATE;
  }
  if constexpr (sizeof(T) == 4) {
    // aperiodic, Lx = Ly in {64, 128}: the y and x passes of each direction fused per plane
    if (plane_fused_ok(pl)) {
      MSC_TRY(launch_plane_fwd(pl, x, scale, W, done, nrhs));    // A + X
      MSC_TRY(launch_zbz<T>(pl, W, done, nrhs));                 // ZBZ'
      MSC_TRY(launch_plane_inv(pl, W, x, scale, y, done, nrhs)); // X' + C
      return MSC_OK;
    }
  }
  const cx<T>* twxy = (const cx<T>*)(sizeof(T) == 8 ? pl->tw64_xy.p : pl->tw32_xy.p);
  // x lines: the contiguous rows of the nrhs workspaces
  const long long G = (long long)nrhs * 9 * g.Nz * g.Ly;
  bool yreg = false;
  if constexpr (sizeof(T) == 4) yreg = y_reg_ok(pl);
  MSC_TRY(launch_t0_fft_y<T>(pl, x, scale, W, twxy, done, nrhs));                                 // A
  MSC_TRY(launch_fft_contig<T>(pl, W, W, G, G, 0, g.Lx, g.M, g.Lx, pl->fxy, twxy, -1, done));      // X
  MSC_TRY(launch_zbz<T>(pl, W, done, nrhs));                                                      // ZBZ'
  MSC_TRY(launch_fft_contig<T>(pl, W, W, G, G, 0, g.Lx, g.Lx, g.M, pl->fxy, twxy, +1, done));      // X'
  if constexpr (sizeof(T) == 4) {
    if (yreg) MSC_TRY(launch_fft_y_out_reg(pl, W, x, scale, y, done, nrhs));                     // C
  }
  if (!yreg) MSC_TRY(launch_fft_y_out<T>(pl, W, x, scale, y, twxy, done, nrhs));                  // C
  return MSC_OK;
}

template <typename T>
int launch_matvec(msc_plan* pl, const cx<T>* x, const double* scale, cx<T>* y, const int* done) {
  if (pl->nrhs > 1)
    return launch_matvec_ws<T>(pl, x, scale, y, (cx<T>*)(sizeof(T) == 8 ? pl->Wm64.p : pl->Wm32.p), done, pl->nrhs);
  return launch_matvec_ws<T>(pl, x, scale, y, (cx<T>*)(sizeof(T) == 8 ? pl->W64.p : pl->W32.p), done, 1);
}

template int launch_matvec_ws<float>(msc_plan*, const float2*, const double*, float2*, float2*, const int*, int);
template int launch_matvec_ws<double>(msc_plan*, const double2*, const double*, double2*, double2*, const int*, int);
template int launch_matvec<float>(msc_plan*, const float2*, const double*, float2*, const int*);
template int launch_matvec<double>(msc_plan*, const double2*, const double*, double2*, const int*);

}  // namespace msc
