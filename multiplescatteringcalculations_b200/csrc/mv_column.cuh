// Matvec kernel B: the per-wavevector 9x9 block multiply acc(k) = K(k) tau(k) on
// the 3D spectrum W[c][kz][ky][kx] (in place), reading the kernel spectrum
// khat[e][kz][ky][kx] for ky in [0, Hy) exactly once.
//
// Half-space storage: for 0 < ky < Ly/2 the thread of point k also updates the
// partner point -k with K(-k) = S K(k) S, S = diag(1,1,1,-1 x6) (parity of the
// propagator). The lines ky = 0 and ky = Ly/2, and every line of a full-plane
// spectrum (Bloch-phased kernels), hold K at each point and are not paired.
// Consecutive threads take consecutive kx, so the spectrum and both field
// points are read with coalesced (the partner in descending) addresses.
#pragma once
#include "mv_common.cuh"

namespace msc {

// SYM (E = 45): entry e enumerates i <= j row-major and holds (K D)_ij with
// D = diag(1 x6, 2 x3), symmetric for the point propagator; K_ij = (K D)_ij / D_j.
// FULL (E = 81): K_ij row-major.
template <bool SYM> struct BlockMul;

template <> struct BlockMul<true> {
  static constexpr int E = 45;
  template <typename C, typename LD>
  static __device__ __forceinline__ void run(LD ld, C* t, C* tp, bool paired) {
    C acc[9], accp[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      if (j >= 6) {
        t[j].x *= 0.5f; t[j].y *= 0.5f;
        tp[j].x *= 0.5f; tp[j].y *= 0.5f;
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
        fma_(acc[i], m, t[j]);
        if (i != j) fma_(acc[j], m, t[i]);
        if (paired) {
          C mm = m;
          if ((i < 3) != (j < 3)) { mm.x = -mm.x; mm.y = -mm.y; }
          fma_(accp[i], mm, tp[j]);
          if (i != j) fma_(accp[j], mm, tp[i]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      t[j] = acc[j];
      tp[j] = accp[j];
    }
  }
};

template <> struct BlockMul<false> {
  static constexpr int E = 81;
  template <typename C, typename LD>
  static __device__ __forceinline__ void run(LD ld, C* t, C* tp, bool paired) {
    C acc[9], accp[9];
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
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      t[j] = acc[j];
      tp[j] = accp[j];
    }
  }
};

template <typename T, bool SYM>
__global__ void __launch_bounds__(128, 4) k_block_mul(cx<T>* __restrict__ W, const cx<T>* __restrict__ khat, Geo g,
                                                   const int* done) {
  if (done && *done) return;
  using C = cx<T>;
  const long long npt = (long long)g.Lz * g.Hy * g.Lx;
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npt) return;
  const int kx = (int)(p % g.Lx);
  const int ky = (int)((p / g.Lx) % g.Hy);
  const int kz = (int)(p / ((long long)g.Lx * g.Hy));
  const bool paired = g.half && !(ky == 0 || ((g.Ly & 1) == 0 && ky == g.Ly / 2));
  const size_t cstride = (size_t)g.Lz * g.Ly * g.Lx;
  const size_t own = ((size_t)kz * g.Ly + ky) * g.Lx + kx;
  const size_t par = paired ? ((size_t)((g.Lz - kz) % g.Lz) * g.Ly + (g.Ly - ky)) * g.Lx + (g.Lx - kx) % g.Lx : own;
  C t[9], tp[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    t[c] = W[c * cstride + own];
    tp[c] = paired ? W[c * cstride + par] : czero<C>();
  }
  const size_t estride = (size_t)npt;
  const C* kb = khat + p;
  auto ld = [&](int e) { return ld_stream(kb + (size_t)e * estride); };
  BlockMul<SYM>::run(ld, t, tp, paired);
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    W[c * cstride + own] = t[c];
    if (paired) W[c * cstride + par] = tp[c];
  }
}

template <typename T>
int launch_block_mul(msc_plan* pl, cx<T>* W, const int* done) {
  const Geo& g = pl->g;
  const cx<T>* kh = (const cx<T>*)(sizeof(T) == 8 ? pl->khat64.p : pl->khat32.p);
  const long long npt = (long long)g.Lz * g.Hy * g.Lx;
  const int nthr = 128;
  const unsigned nb = (unsigned)((npt + nthr - 1) / nthr);
  if (pl->E == 45) k_block_mul<T, true><<<nb, nthr, 0, pl->stream>>>(W, kh, g, done);
  else k_block_mul<T, false><<<nb, nthr, 0, pl->stream>>>(W, kh, g, done);
  ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}

}  // namespace msc
