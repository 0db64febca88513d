// Fused plane passes of the complex64 matvec for aperiodic lattices with L = Lx = Ly in
// {64, 128} (so M <= L/2): one block per (component, layer) plane.
//
//   forward  (A+X): tau = T0 (s x) on the M x M plane, FFT along y of its M rows, then
//                   FFT along x of the L rows ky, written to W[c][n][ky][kx] once;
//   inverse (X'+C): inverse FFT along kx of the L rows of W (keeping x < M), inverse FFT
//                   along y of the M rows x, y = s x - acc on the M x M window.
//
// The intermediate [ky][x] plane (L x M complex) stays in shared memory between the two
// transforms, so W is read or written once per direction instead of twice, and one
// launch replaces two. Each 1-D transform is the register four-step engine: a line of L
// points is held by 8 threads of a warp, L/8 points each (an L/8-point DFT in registers,
// the twiddle W_L^(t k1), a transpose through shared memory within the warp, an 8-point
// DFT in registers); thread t then holds outputs k1 + (L/8) k2 for its L/64 values of k1.
#include "mv_common.cuh"

namespace msc {

namespace {

template <int L> struct PlaneCfg {
  static constexpr int NTL = 8;               // threads per line
  static constexpr int R1 = L / NTL;          // points per thread
  static constexpr int KPT = R1 / NTL;        // k1 values per thread after the transpose
  static constexpr int LINES = L / 2;         // lines per pass (M <= L/2 rows, L/2 rows of ky)
  static constexpr int NT = LINES * NTL;      // threads per block
  static constexpr int RS = NTL + 1;          // transpose row pitch
  static constexpr int LS0 = R1 * RS;
  static constexpr int LS = (LS0 % 2) ? LS0 : LS0 + 1;  // line pitch, odd
  static constexpr int TP = L / 2 + 1;        // pitch of the [ky][x] plane (x < L/2)
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)LINES * LS + (size_t)L * TP);
};

// One four-step transform of the line held in v (thread t of the line's 8): on return
// u[c][k2] holds the output k1 + R1 k2, k1 = t KPT + c. ls: the line's transpose slots.
template <int L, int DIR>
__device__ __forceinline__ void line_fft(float2 (&v)[PlaneCfg<L>::R1], float2 (&u)[PlaneCfg<L>::KPT][8],
                                         float2* ls, int t, const float2* __restrict__ twg) {
  using PC = PlaneCfg<L>;
  constexpr int R1 = PC::R1, KPT = PC::KPT, RS = PC::RS;
  fft_reg_c<R1, DIR>(v);
#pragma unroll
  for (int k1 = 1; k1 < R1; ++k1) {
    float2 w = __ldg(twg + ((t * k1) & (L - 1)));
    if (DIR > 0) w.y = -w.y;
    v[k1] = v[k1] * w;
  }
  __syncwarp();  // earlier readers of these slots (the previous transform) are done
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) ls[k1 * RS + t] = v[k1];
  __syncwarp();
#pragma unroll
  for (int c = 0; c < KPT; ++c)
#pragma unroll
    for (int s = 0; s < 8; ++s) u[c][s] = ls[(t * KPT + c) * RS + s];
#pragma unroll
  for (int c = 0; c < KPT; ++c) fft_reg_c<8, DIR>(u[c]);
}

__device__ __forceinline__ float2 tau_c(const float2* __restrict__ x, const float2* __restrict__ t4, int nsite,
                                        int site, int c) {
  const float2 xc = x[(size_t)c * nsite + site];
  if (c < 3) return t4[site] * xc;
  if (c >= 6) return t4[(size_t)3 * nsite + site] * xc;
  const float2 tr = x[(size_t)3 * nsite + site] + x[(size_t)4 * nsite + site] + x[(size_t)5 * nsite + site];
  return t4[(size_t)1 * nsite + site] * tr + t4[(size_t)2 * nsite + site] * xc;
}

// A + X: blockIdx.x = n, blockIdx.y = c.
template <int L>
__global__ void __launch_bounds__(PlaneCfg<L>::NT) k_plane_fwd(const float2* __restrict__ x, const double* scale,
                                                               const float2* __restrict__ t4, float2* __restrict__ W,
                                                               Geo g, const float2* __restrict__ twg, const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  using PC = PlaneCfg<L>;
  constexpr int R1 = PC::R1, KPT = PC::KPT, LINES = PC::LINES, LS = PC::LS, TP = PC::TP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tb = reinterpret_cast<float2*>(smem_raw);  // [LINES][LS] transpose slots
  float2* T = tb + LINES * LS;                        // [L][TP]: [ky][x], x < L/2
  const int n = blockIdx.x, c = blockIdx.y;
  // blockIdx.z: the right-hand side (fields and workspaces follow each other)
  x += (size_t)blockIdx.z * 9 * g.nsite;
  W += (size_t)blockIdx.z * 9 * g.Nz * L * L;
  const int q = threadIdx.x / 8, t = threadIdx.x % 8;
  const float s = scale ? (float)(*scale) : 1.f;
  float2* ls = tb + q * LS;
  // y transform of row x = q (rows q >= M are zero: the x transform's zero padding)
  {
    float2 v[R1];
#pragma unroll
    for (int m = 0; m < R1; ++m) {
      const int y = t + 8 * m;
      v[m] = (m < R1 / 2 && q < g.M && y < g.M) ? s * tau_c(x, t4, g.nsite, (n * g.M + q) * g.M + y, c)
                                                : make_float2(0.f, 0.f);
    }
    float2 u[KPT][8];
    line_fft<L, -1>(v, u, ls, t, twg);
#pragma unroll
    for (int cc = 0; cc < KPT; ++cc)
#pragma unroll
      for (int k2 = 0; k2 < 8; ++k2) T[(t * KPT + cc + R1 * k2) * TP + q] = u[cc][k2];
  }
  __syncthreads();
  // x transforms of the L rows ky, LINES at a time
  float2* Wp = W + (size_t)(c * g.Nz + n) * L * L;
#pragma unroll
  for (int pass = 0; pass < L / LINES; ++pass) {
    const int ky = pass * LINES + q;
    float2 v[R1];
#pragma unroll
    for (int m = 0; m < R1; ++m) v[m] = m < R1 / 2 ? T[ky * TP + t + 8 * m] : make_float2(0.f, 0.f);
    float2 u[KPT][8];
    line_fft<L, -1>(v, u, ls, t, twg);
    float2* o = Wp + (size_t)ky * L;
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) {
      const int k = t * KPT + R1 * k2;
      if constexpr (KPT == 2)
        *reinterpret_cast<float4*>(o + k) = make_float4(u[0][k2].x, u[0][k2].y, u[1][k2].x, u[1][k2].y);
      else
        o[k] = u[0][k2];
    }
  }
}

// X' + C: blockIdx.x = n, blockIdx.y = c. y = s x - acc.
template <int L>
__global__ void __launch_bounds__(PlaneCfg<L>::NT) k_plane_inv(const float2* __restrict__ W,
                                                               const float2* __restrict__ x, const double* scale,
                                                               float2* __restrict__ y, Geo g,
                                                               const float2* __restrict__ twg, const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  using PC = PlaneCfg<L>;
  constexpr int R1 = PC::R1, KPT = PC::KPT, LINES = PC::LINES, LS = PC::LS, TP = PC::TP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tb = reinterpret_cast<float2*>(smem_raw);
  float2* T = tb + LINES * LS;  // [ky][x], x < L/2
  const int n = blockIdx.x, c = blockIdx.y;
  // blockIdx.z: the right-hand side
  W += (size_t)blockIdx.z * 9 * g.Nz * L * L;
  x += (size_t)blockIdx.z * 9 * g.nsite;
  y += (size_t)blockIdx.z * 9 * g.nsite;
  const int q = threadIdx.x / 8, t = threadIdx.x % 8;
  float2* ls = tb + q * LS;
  const float2* Wp = W + (size_t)(c * g.Nz + n) * L * L;
  // inverse x transforms of the L rows ky; keep x < L/2 (x >= M is never read)
#pragma unroll
  for (int pass = 0; pass < L / LINES; ++pass) {
    const int ky = pass * LINES + q;
    float2 v[R1];
    const float2* r = Wp + (size_t)ky * L;
#pragma unroll
    for (int m = 0; m < R1; ++m) v[m] = r[t + 8 * m];
    float2 u[KPT][8];
    line_fft<L, +1>(v, u, ls, t, twg);
#pragma unroll
    for (int cc = 0; cc < KPT; ++cc)
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) T[ky * TP + t * KPT + cc + R1 * k2] = u[cc][k2];  // x < L/2
  }
  __syncthreads();
  // inverse y transform of row x = q (every line runs it: line_fft synchronises the
  // warp; only rows q < M are stored), then y = s x - acc for y < M
  float2 v[R1];
#pragma unroll
  for (int m = 0; m < R1; ++m) v[m] = T[(t + 8 * m) * TP + q];
  float2 u[KPT][8];
  line_fft<L, +1>(v, u, ls, t, twg);
  const float s = scale ? (float)(*scale) : 1.f;
  const size_t row = (size_t)c * g.nsite + (size_t)(n * g.M + q) * g.M;
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) {
#pragma unroll
    for (int cc = 0; cc < KPT; ++cc) {
      const int yy = t * KPT + cc + R1 * k2;
      if (q < g.M && yy < g.M) y[row + yy] = s * x[row + yy] - u[cc][k2];
    }
  }
}

}  // namespace

// True when the fused plane passes serve this plan's complex64 matvec.
bool plane_fused_ok(const msc_plan* pl) {
  const Geo& g = pl->g;
  return !pl->desc.periodic && g.Lx == g.Ly && (g.Lx == 64 || g.Lx == 128) && 2 * g.M <= g.Lx;
}

int launch_plane_fwd(msc_plan* pl, const float2* x, const double* scale, float2* W, const int* done, int nrhs) {
  const Geo& g = pl->g;
  const float2* t4 = (const float2*)pl->t4_32.p;
  const float2* tw = (const float2*)pl->tw32_xy.p;
  const void* kern = g.Lx == 64 ? (const void*)k_plane_fwd<64> : (const void*)k_plane_fwd<128>;
  const size_t sm = g.Lx == 64 ? PlaneCfg<64>::SMEM : PlaneCfg<128>::SMEM;
  const int nt = g.Lx == 64 ? PlaneCfg<64>::NT : PlaneCfg<128>::NT;
  MSC_CUDA(prep_kernel(kern));
  Geo gg = g;
  void* args[] = {(void*)&x, (void*)&scale, (void*)&t4, (void*)&W, (void*)&gg, (void*)&tw, (void*)&done};
  MSC_CUDA(launch_pdl(kern, dim3((unsigned)g.Nz, 9, (unsigned)nrhs), dim3(nt), args, sm, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}

int launch_plane_inv(msc_plan* pl, const float2* W, const float2* x, const double* scale, float2* y,
                     const int* done, int nrhs) {
  const Geo& g = pl->g;
  const float2* tw = (const float2*)pl->tw32_xy.p;
  const void* kern = g.Lx == 64 ? (const void*)k_plane_inv<64> : (const void*)k_plane_inv<128>;
  const size_t sm = g.Lx == 64 ? PlaneCfg<64>::SMEM : PlaneCfg<128>::SMEM;
  const int nt = g.Lx == 64 ? PlaneCfg<64>::NT : PlaneCfg<128>::NT;
  MSC_CUDA(prep_kernel(kern));
  Geo gg = g;
  void* args[] = {(void*)&W, (void*)&x, (void*)&scale, (void*)&y, (void*)&gg, (void*)&tw, (void*)&done};
  MSC_CUDA(launch_pdl(kern, dim3((unsigned)g.Nz, 9, (unsigned)nrhs), dim3(nt), args, sm, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}

}  // namespace msc
