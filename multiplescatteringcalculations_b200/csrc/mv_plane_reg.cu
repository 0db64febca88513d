// The inverse y pass of the complex64 matvec on the register four-step engine, for the
// planes that the fused plane kernels do not hold (periodic lattices, and the 256 x 256
// planes of the large lattices, 512 KB each): Ly in {64, 128, 256}.
//
//   C (k_fft_y_out_reg): the LPB columns x of W[c][n][ky][.], the inverse FFT along ky,
//                        y = s x - acc on the rows' y < M.
//
// A line of L points is held by NTL threads (L / NTL points each): an (L / NTL)-point
// DFT in registers, the twiddle, a transpose within the line's threads through shared
// memory, an NTL-point DFT in registers (the engine of the x passes, RowReg in
// mv_lines.cu). The columns of W ([ky][x], x fastest) come in through a shared tile
// [ky][x] of the block's LPB columns, so W is read in rows of LPB consecutive x (128
// bytes for LPB = 16), and the rows along y are written 128 bytes at a time. At
// 256 x 256 x 32 this pass takes 128 us against 153 us for the shared-memory Stockham
// tiles (three barrier-separated passes over shared memory per transform). The forward
// pass keeps the shared-memory kernel: a register form of it (100 registers, 2 blocks
// per SM) measured slower, 213 against 157 us, its T0 gathers exposed at the lower
// occupancy.
#include "mv_common.cuh"

namespace msc {

namespace {

template <int L> struct YReg {
  static constexpr int NTL = L >= 256 ? 16 : 8;  // threads per line
  static constexpr int R1 = L / NTL;             // points per thread
  static constexpr int KPT = R1 / NTL;           // outputs k1 per thread after the transpose
  static constexpr int LPB = 256 / NTL;          // lines (rows x) per block of 256 threads
  static constexpr int RS = NTL + 1;             // transpose row pitch
  static constexpr int LS0 = R1 * RS;
  static constexpr int LS = ((LS0 * 8 / 4) % 32 == 16) ? LS0 : LS0 + 8;  // line pitch
  static constexpr int TP = LPB + 1;             // pitch of the [ky][x] tile
  static constexpr int SM = (LPB * LS > L * TP) ? LPB * LS : L * TP;   // float2 entries
};

// One line's four-step transform, v in (thread t holds points t + NTL m), u out
// (u[c][k2] = output t KPT + c + R1 k2).
template <int L, int DIR>
__device__ __forceinline__ void four_step(float2 (&v)[YReg<L>::R1], float2 (&u)[YReg<L>::KPT][YReg<L>::NTL],
                                          float2* ls, int t, const float2* __restrict__ twg) {
  using Y = YReg<L>;
  constexpr int NTL = Y::NTL, R1 = Y::R1, KPT = Y::KPT, RS = Y::RS;
  fft_reg_c<R1, DIR>(v);
#pragma unroll
  for (int k1 = 1; k1 < R1; ++k1) {
    float2 w = __ldg(twg + ((t * k1) & (L - 1)));
    if (DIR > 0) w.y = -w.y;
    v[k1] = v[k1] * w;
  }
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) ls[k1 * RS + t] = v[k1];
  __syncwarp();
#pragma unroll
  for (int c = 0; c < KPT; ++c)
#pragma unroll
    for (int s = 0; s < NTL; ++s) u[c][s] = ls[(t * KPT + c) * RS + s];
#pragma unroll
  for (int c = 0; c < KPT; ++c) fft_reg_c<NTL, DIR>(u[c]);
}

// C: blockIdx.x = chunk of LPB rows x, blockIdx.y = layer n, blockIdx.z = 9 rh + c.
template <int L>
__global__ void __launch_bounds__(256) k_fft_y_out_reg(const float2* __restrict__ W, const float2* __restrict__ x,
                                                       const double* scale, float2* __restrict__ y, Geo g,
                                                       const float2* __restrict__ twg, const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  using Y = YReg<L>;
  constexpr int NTL = Y::NTL, R1 = Y::R1, KPT = Y::KPT, LPB = Y::LPB, LS = Y::LS, TP = Y::TP;
  __shared__ __align__(16) float2 sm[Y::SM];
  const int c = blockIdx.z % 9, n = blockIdx.y, i0 = blockIdx.x * LPB;
  {
    const size_t rh = blockIdx.z / 9;
    W += rh * 9 * (size_t)g.Nz * g.Ly * g.Lx;
    x += rh * 9 * (size_t)g.nsite;
    y += rh * 9 * (size_t)g.nsite;
  }
  const float2* Wp = W + (size_t)(c * g.Nz + n) * g.Ly * g.Lx + i0;
  {
    const int xq = threadIdx.x % LPB;
    const bool ok = i0 + xq < g.M;
#pragma unroll 4
    for (int ky = threadIdx.x / LPB; ky < L; ky += 256 / LPB)
      sm[ky * TP + xq] = ok ? Wp[(size_t)ky * g.Lx + xq] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const int q = threadIdx.x / NTL, t = threadIdx.x % NTL;
  const int xr = i0 + q;
  float2 v[R1];
#pragma unroll
  for (int m = 0; m < R1; ++m) v[m] = sm[(t + NTL * m) * TP + q];
  __syncthreads();  // the tile is reused as the line slots
  float2 u[KPT][NTL];
  four_step<L, +1>(v, u, sm + q * LS, t, twg);
  if (xr >= g.M) return;
  const float s = scale ? (float)(*scale) : 1.f;
  const size_t row = (size_t)c * g.nsite + (size_t)(n * g.M + xr) * g.M;
#pragma unroll
  for (int k2 = 0; k2 < NTL; ++k2)
#pragma unroll
    for (int cc = 0; cc < KPT; ++cc) {
      const int yy = t * KPT + cc + R1 * k2;
      if (yy < g.M) y[row + yy] = s * x[row + yy] - u[cc][k2];
    }
}

template <int L> const void* c_kernel() { return (const void*)k_fft_y_out_reg<L>; }

}  // namespace

bool y_reg_ok(const msc_plan* pl) {
  const int L = pl->g.Ly;
  return L == 64 || L == 128 || L == 256;
}

int launch_fft_y_out_reg(msc_plan* pl, const float2* W, const float2* x, const double* scale, float2* y,
                         const int* done, int nrhs) {
  const Geo& g = pl->g;
  const float2* tw = (const float2*)pl->tw32_xy.p;
  int lpb = 0;
  const void* kern = nullptr;
  if (g.Ly == 64) { kern = c_kernel<64>(); lpb = YReg<64>::LPB; }
  else if (g.Ly == 128) { kern = c_kernel<128>(); lpb = YReg<128>::LPB; }
  else if (g.Ly == 256) { kern = c_kernel<256>(); lpb = YReg<256>::LPB; }
  else { set_error("internal: register y pass for Ly = %d", g.Ly); return MSC_ERR_STATE; }
  Geo gg = g;
  void* args[] = {(void*)&W, (void*)&x, (void*)&scale, (void*)&y, (void*)&gg, (void*)&tw, (void*)&done};
  dim3 grid((unsigned)((g.M + lpb - 1) / lpb), (unsigned)g.Nz, 9u * (unsigned)nrhs);
  MSC_CUDA(launch_pdl(kern, grid, dim3(256), args, 0, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}

}  // namespace msc
