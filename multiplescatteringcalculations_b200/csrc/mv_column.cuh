// Matvec kernel B: per (kx, ky) column pair, z FFT, 9x9 block multiply by the
// half-space kernel spectrum, inverse z FFT.
#pragma once
#include "mv_common.cuh"

namespace msc {

// ---- B: z FFT + 9x9 block multiply + inverse z FFT on column pairs ------------------
// Spectrum layout khat[e][ky][kx][kz], ky in [0, Hy). SYM (E = 45): entry e enumerates
// i <= j row-major and holds (K D)_ij with D = diag(1 x6, 2 x3), which is symmetric
// for the point propagator; K_ij = (K D)_ij / D_j. FULL (E = 81): K_ij row-major.
template <bool SYM> struct BlockMul;

template <> struct BlockMul<true> {
  static constexpr int E = 45;
  template <typename C, typename LD>
  static __device__ __forceinline__ void run(LD ld, const C* t, const C* tp, C* acc, C* accp, bool paired) {
    C u[9], up[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      u[j] = t[j];
      up[j] = tp[j];
      if (j >= 6) {
        u[j].x *= 0.5f; u[j].y *= 0.5f;
        up[j].x *= 0.5f; up[j].y *= 0.5f;
      }
      acc[j] = czero<C>();
      accp[j] = czero<C>();
    }
    int e = 0;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
#pragma unroll
      for (int j = i; j < 9; ++j, ++e) {
        const C m = ld(e);
        fma_(acc[i], m, u[j]);
        if (i != j) fma_(acc[j], m, u[i]);
        if (paired) {
          // partner block S M S: sign s_i s_j, s = (+,+,+,-,...)
          const bool neg = (i < 3) != (j < 3);
          C mm = m;
          if (neg) { mm.x = -mm.x; mm.y = -mm.y; }
          fma_(accp[i], mm, up[j]);
          if (i != j) fma_(accp[j], mm, up[i]);
        }
      }
    }
  }
};

template <> struct BlockMul<false> {
  static constexpr int E = 81;
  template <typename C, typename LD>
  static __device__ __forceinline__ void run(LD ld, const C* t, const C* tp, C* acc, C* accp, bool paired) {
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      acc[j] = czero<C>();
      accp[j] = czero<C>();
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) {
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        const C m = ld(i * 9 + j);
        fma_(acc[i], m, t[j]);
        if (paired) {
          C mm = m;
          if ((i < 3) != (j < 3)) { mm.x = -mm.x; mm.y = -mm.y; }
          fma_(accp[i], mm, tp[j]);
        }
      }
    }
  }
};

constexpr int ZB_TC = 8;  // columns per side in kernel B

template <typename T, bool SYM, int KMAX>
__global__ void __launch_bounds__(288) k_zfft_block(cx<T>* __restrict__ W, const cx<T>* __restrict__ khat, Geo g,
                                                    FftPlan1D pl, const cx<T>* __restrict__ twg, const int* done) {
  if (done && *done) return;
  using C = cx<T>;
  constexpr int TC = ZB_TC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* tile = tw + g.Lz;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int ky = blockIdx.y, kx0 = blockIdx.x * TC;
  const bool paired = g.half && !(ky == 0 || ((g.Ly & 1) == 0 && ky == g.Ly / 2));
  const int nside = paired ? 2 : 1;
  const int nlines = nside * 9 * TC;
  const int P = nlines + 1;
  const int pky = (g.Ly - ky) % g.Ly;
  for (int t = tid; t < g.Lz; t += nthr) tw[t] = twg[t];
  // load the N_z planes of both column groups; zero the padding planes
  const int nload = nlines * g.Nz;
  for (int it = tid; it < nload; it += nthr) {
    const int t = it % TC;
    const int rest = it / TC;
    const int c9 = rest % (nside * 9);
    const int z = rest / (nside * 9);
    const int side = c9 >= 9, c = c9 - 9 * side;
    const int kx = kx0 + t;
    C v = czero<C>();
    if (kx < g.Lx) {
      const int col = side ? (g.Lx - kx) % g.Lx : kx;
      const int line = side ? pky : ky;
      v = W[((size_t)(c * g.Nz + z) * g.Ly + line) * g.Lx + col];
    }
    tile[z * P + c9 * TC + t] = v;
  }
  for (int it = tid; it < nlines * (g.Lz - g.Nz); it += nthr) {
    const int l = it % nlines, z = g.Nz + it / nlines;
    tile[z * P + l] = czero<C>();
  }
  __syncthreads();
  fft_tile<-1, KMAX>(tile, P, nlines, pl, tw, tid, nthr);
  // block multiply at (kz, t) and its partner (-kz, t)
  const size_t estride = (size_t)g.Hy * g.Lx * g.Lz;
  for (int it = tid; it < g.Lz * TC; it += nthr) {
    const int kz = it % g.Lz, t = it / g.Lz;
    const int kx = kx0 + t;
    if (kx >= g.Lx) continue;
    const int pkz = (g.Lz - kz) % g.Lz;
    C tv[9], tp[9], acc[9], accp[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      tv[c] = tile[kz * P + c * TC + t];
      tp[c] = paired ? tile[pkz * P + (9 + c) * TC + t] : czero<C>();
    }
    const C* kb = khat + ((size_t)ky * g.Lx + kx) * g.Lz + kz;
    auto ld = [&](int e) { return ld_stream(kb + (size_t)e * estride); };
    BlockMul<SYM>::run(ld, tv, tp, acc, accp, paired);
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      tile[kz * P + c * TC + t] = acc[c];
      if (paired) tile[pkz * P + (9 + c) * TC + t] = accp[c];
    }
  }
  __syncthreads();
  fft_tile<+1, KMAX>(tile, P, nlines, pl, tw, tid, nthr);
  for (int it = tid; it < nload; it += nthr) {
    const int t = it % TC;
    const int rest = it / TC;
    const int c9 = rest % (nside * 9);
    const int z = rest / (nside * 9);
    const int side = c9 >= 9, c = c9 - 9 * side;
    const int kx = kx0 + t;
    if (kx < g.Lx) {
      const int col = side ? (g.Lx - kx) % g.Lx : kx;
      const int line = side ? pky : ky;
      W[((size_t)(c * g.Nz + z) * g.Ly + line) * g.Lx + col] = tile[z * P + c9 * TC + t];
    }
  }
}

template <typename T>
int launch_zfft_block(msc_plan* pl, cx<T>* W, const cx<T>* tw, const int* done) {
  const Geo& g = pl->g;
  const cx<T>* kh = (const cx<T>*)(sizeof(T) == 8 ? pl->khat64.p : pl->khat32.p);
  const int nlines = 2 * 9 * ZB_TC;
  // threads: a multiple of the paired line count, enough for KMAX <= 8
  int nthr = 288;
  while (fft_kmax_needed(pl->fz, nlines, nthr) > 4 && nthr + nlines <= 1024) nthr += nlines;
  const size_t sm = sizeof(cx<T>) * ((size_t)g.Lz + (size_t)g.Lz * (nlines + 1));
  const int kmax = std::max(fft_kmax_needed(pl->fz, nlines, nthr), fft_kmax_needed(pl->fz, 9 * ZB_TC, nthr));
  dim3 grid((unsigned)((g.Lx + ZB_TC - 1) / ZB_TC), (unsigned)g.Hy);
#define CALL(K)                                                                                                      \
  {                                                                                                                  \
    if (pl->E == 45) {                                                                                               \
      MSC_CUDA(cudaFuncSetAttribute(k_zfft_block<T, true, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));  \
      k_zfft_block<T, true, K><<<grid, nthr, sm, pl->stream>>>(W, kh, g, pl->fz, tw, done);                          \
    } else {                                                                                                         \
      MSC_CUDA(cudaFuncSetAttribute(k_zfft_block<T, false, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); \
      k_zfft_block<T, false, K><<<grid, nthr, sm, pl->stream>>>(W, kh, g, pl->fz, tw, done);                         \
    }                                                                                                                \
  }
  MSC_KMAX_DISPATCH(kmax, CALL);
#undef CALL
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}
}  // namespace msc
