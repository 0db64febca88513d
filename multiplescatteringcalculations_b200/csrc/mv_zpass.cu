// Fused z pass, register form (k_zpass, mv_zpass.cuh): launcher for the octant
// spectrum. complex64: Lz in {8, 16, 32, 64}, one thread per z line up to Lz = 32, two at
// Lz = 64 (whose line would not fit one thread's registers); complex128: Lz in {8, 16, 32},
// two threads per line at Lz = 32.
#include "mv_zpass.cuh"

namespace msc {

namespace {

template <typename T, int LZ, int KX, int S, bool SYM>
int run(msc_plan* pl, cx<T>* W, const int* done, int nrhs, int nxc) {
  using Cf = ZpCfg<T, LZ, KX, S, SYM>;
  const Geo& g = pl->g;
  const void* kern = (const void*)k_zpass<T, LZ, KX, S, SYM>;
  MSC_CUDA(prep_kernel(kern));
  const cx<T>* kh = (const cx<T>*)(sizeof(T) == 8 ? pl->khat64.p : pl->khat32.p);
  const cx<T>* tw = (const cx<T>*)(sizeof(T) == 8 ? pl->tw64_z.p : pl->tw32_z.p);
  Geo gg = g;
  int nx = nxc;
  int* status = (int*)pl->status.p;
  long long lim = pl->wait_limit > 0 ? pl->wait_limit : ZP_WAIT_LIMIT;
  void* args[] = {(void*)&W,    (void*)&kh,   (void*)&gg,     (void*)&nx, (void*)&tw,
                  (void*)&done, (void*)&nrhs, (void*)&status, (void*)&lim};
  MSC_CUDA(launch_pdl(kern, dim3((unsigned)nxc, (unsigned)g.Hy), dim3(Cf::NT), args, Cf::SMEM, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}

}  // namespace

// Runs the z pass with k_zpass when the plan's shape has a compile-time form;
// returns 1 (nothing launched) otherwise.
template <typename T>
int launch_zpass(msc_plan* pl, cx<T>* W, const int* done, int nrhs) {
  const Geo& g = pl->g;
  if (!g.oct || 2 * g.Nz > g.Lz) return 1;
  const bool sym = pl->E == 45;
  const ZbzLayout lay = zbz_layout<T>(g, pl->E);
  // the spectrum slices are blocked with the layout's KX; the kernel's must match
#define ZP_CASE(LZ, S)                                                                                 \
  case LZ:                                                                                             \
    if (sym && lay.KX == zbz_kx_ct<T>(LZ, 45))                                                         \
      return run<T, LZ, zbz_kx_ct<T>(LZ, 45), S, true>(pl, W, done, nrhs, lay.NXC);                    \
    if (!sym && lay.KX == zbz_kx_ct<T>(LZ, 81))                                                        \
      return run<T, LZ, zbz_kx_ct<T>(LZ, 81), S, false>(pl, W, done, nrhs, lay.NXC);                   \
    return 1;
  if constexpr (sizeof(T) == 4) {
    switch (g.Lz) {
      ZP_CASE(8, 1)
      ZP_CASE(16, 1)
      ZP_CASE(32, 1)
      ZP_CASE(64, 2)
      default: return 1;
    }
  } else {
    switch (g.Lz) {
      ZP_CASE(8, 1)
      ZP_CASE(16, 1)
      ZP_CASE(32, 2)
      default: return 1;
    }
  }
#undef ZP_CASE
}
template int launch_zpass<float>(msc_plan*, float2*, const int*, int);
template int launch_zpass<double>(msc_plan*, double2*, const int*, int);

}  // namespace msc
