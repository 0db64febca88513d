// Mixed-radix Stockham FFT on shared-memory tiles.
//
// A tile holds `nlines` independent lines of length L, interleaved: element
// (idx, line) sits at buf[idx * pitch + line], pitch >= nlines. With pitch =
// nlines + 1 and 128-byte rows the butterfly loads/stores of a warp touch
// consecutive words (conflict free), and the transposing global loads/stores
// done by the callers are conflict free as well.
//
// Stage s with radix R and Ns = product of the earlier radices combines Ns-point
// transforms into (Ns*R)-point ones (self-sorting Stockham, decimation in time):
//   j in [0, L/R): k = j mod Ns, v_r = x[j + r L/R] * w_{Ns R}^{r k},
//   v <- DFT_R(v), out[(j / Ns) Ns R + k + r Ns] = v_r.
// Each stage runs in place: every thread loads its butterfly inputs into
// registers, the block synchronises, then all threads store.
#pragma once
#include "msc_common.cuh"
#include "radix_constants.cuh"

namespace msc {

constexpr int FFT_MAX_STAGES = 12;

struct FftPlan1D {
  int L;
  int nstages;
  int min_radix;
  int radix[FFT_MAX_STAGES];
  int ns[FFT_MAX_STAGES];
};

// Factorise L into radices {8,4,2,3,5,7,11}; false if L has another prime factor.
inline bool make_fft_plan(int L, FftPlan1D* p) {
  if (L < 1 || L > 4096) return false;
  int rad[FFT_MAX_STAGES];
  int n = 0, rest = L, e2 = 0;
  while (rest % 2 == 0) { rest /= 2; ++e2; }
  // powers of two: prefer radix 8, then 4 (no radix-2 stage unless L = 2^1)
  if (e2 == 1) rad[n++] = 2;
  else if (e2 > 0) {
    int r3 = e2 % 3;
    int n8 = e2 / 3;
    if (r3 == 1) { n8 -= 1; rad[n++] = 4; rad[n++] = 4; }
    else if (r3 == 2) rad[n++] = 4;
    for (int i = 0; i < n8; ++i) rad[n++] = 8;
  }
  const int odd[] = {3, 5, 7, 11};
  for (int r : odd) {
    while (rest % r == 0) {
      if (n >= FFT_MAX_STAGES) return false;
      rad[n++] = r;
      rest /= r;
    }
  }
  if (rest != 1) return false;
  // order: largest radix first (fewest butterflies in the early stages does not
  // matter for Stockham; any order is exact)
  p->L = L;
  p->nstages = n;
  int ns = 1, mr = 64;
  for (int s = 0; s < n; ++s) {
    p->radix[s] = rad[s];
    p->ns[s] = ns;
    ns *= rad[s];
    if (rad[s] < mr) mr = rad[s];
  }
  p->min_radix = (n == 0) ? 1 : mr;
  if (L == 1) { p->nstages = 0; p->min_radix = 1; }
  return true;
}

// ---- radix-R DFT on registers: X_k = sum_n v_n exp(DIR 2 pi i n k / R) ----------
template <int R, int DIR, typename C> struct Dft;

template <int DIR, typename C> struct Dft<2, DIR, C> {
  static __device__ __forceinline__ void run(C* v) {
    C t = v[0];
    v[0] = t + v[1];
    v[1] = t - v[1];
  }
};

template <int DIR, typename C> struct Dft<4, DIR, C> {
  static __device__ __forceinline__ void run(C* v) {
    C a0 = v[0] + v[2], a1 = v[0] - v[2], a2 = v[1] + v[3], a3 = mul_i<DIR>(v[1] - v[3]);
    v[0] = a0 + a2;
    v[2] = a0 - a2;
    v[1] = a1 + a3;
    v[3] = a1 - a3;
  }
};

template <int DIR, typename C> struct Dft<8, DIR, C> {
  static __device__ __forceinline__ void run(C* v) {
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, DIR, C>::run(e);
    Dft<4, DIR, C>::run(o);
    using T = decltype(v[0].x);
    const T h = (T)0.70710678118654752440;
    // w^1 = (1 + DIR i)/sqrt2, w^2 = DIR i, w^3 = (-1 + DIR i)/sqrt2
    C o1, o2, o3;
    o1.x = h * (o[1].x - (T)DIR * o[1].y);
    o1.y = h * (o[1].y + (T)DIR * o[1].x);
    o2 = mul_i<DIR>(o[2]);
    o3.x = h * (-o[3].x - (T)DIR * o[3].y);
    o3.y = h * (-o[3].y + (T)DIR * o[3].x);
    v[0] = e[0] + o[0];
    v[4] = e[0] - o[0];
    v[1] = e[1] + o1;
    v[5] = e[1] - o1;
    v[2] = e[2] + o2;
    v[6] = e[2] - o2;
    v[3] = e[3] + o3;
    v[7] = e[3] - o3;
  }
};

// Odd radix by the symmetric cosine/sine form.
template <int R, int DIR, typename C> struct Dft {
  static __device__ __forceinline__ void run(C* v) {
    using T = decltype(v[0].x);
    constexpr int H = (R - 1) / 2;
    C s[H], d[H];
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      s[q - 1] = v[q] + v[R - q];
      d[q - 1] = v[q] - v[R - q];
    }
    C y0 = v[0];
#pragma unroll
    for (int q = 0; q < H; ++q) y0 += s[q];
    C out[R];
    out[0] = y0;
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      C A = v[0], B;
      B.x = 0;
      B.y = 0;
#pragma unroll
      for (int q = 1; q <= H; ++q) {
        const T c = (T)RadixTrig<R>::c((q * k) % R);
        const T sn = (T)RadixTrig<R>::s((q * k) % R);
        A.x += c * s[q - 1].x;
        A.y += c * s[q - 1].y;
        B.x += sn * d[q - 1].x;
        B.y += sn * d[q - 1].y;
      }
      C iB = mul_i<DIR>(B);  // DIR * i * B
      out[k] = A + iB;
      out[R - k] = A - iB;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = out[k];
  }
};

// One Stockham stage over the tile. Thread `tid` owns line l = tid % nlines and
// butterflies j = tid / nlines + k * jstride, k < KMAX.
template <int R, int DIR, int KMAX, typename C>
__device__ __forceinline__ void fft_stage(C* buf, int pitch, int L, int Ns, const C* tw, int l, int j0, int jstride,
                                          bool active) {
  const int nb = L / R;
  C v[KMAX][R];
  if (active) {
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      const int j = j0 + k * jstride;
      if (j < nb) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[k][r] = buf[(j + r * nb) * pitch + l];
      }
    }
  }
  __syncthreads();
  if (active) {
    const int tstep = L / (Ns * R);
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      const int j = j0 + k * jstride;
      if (j < nb) {
        const int kk = j % Ns;
        if (Ns > 1) {
#pragma unroll
          for (int r = 1; r < R; ++r) {
            C w = tw[r * kk * tstep];
            if (DIR > 0) w.y = -w.y;
            v[k][r] = v[k][r] * w;
          }
        }
        Dft<R, DIR, C>::run(v[k]);
        const int idxD = (j - kk) * R + kk;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[(idxD + r * Ns) * pitch + l] = v[k][r];
      }
    }
  }
  __syncthreads();
}

// Full transform of every line in the tile. Requirements (checked by the host):
// nlines <= nthr and ceil((L / min_radix) / (nthr / nlines)) <= KMAX.
template <int DIR, int KMAX, typename C>
__device__ void fft_tile(C* buf, int pitch, int nlines, const FftPlan1D& pl, const C* tw, int tid, int nthr) {
  const int jstride = nthr / nlines;
  const bool active = tid < jstride * nlines;
  const int l = tid % nlines;
  const int j0 = tid / nlines;
  for (int s = 0; s < pl.nstages; ++s) {
    const int Ns = pl.ns[s];
    switch (pl.radix[s]) {
      case 8: fft_stage<8, DIR, KMAX>(buf, pitch, pl.L, Ns, tw, l, j0, jstride, active); break;
      case 4: fft_stage<4, DIR, KMAX>(buf, pitch, pl.L, Ns, tw, l, j0, jstride, active); break;
      case 2: fft_stage<2, DIR, KMAX>(buf, pitch, pl.L, Ns, tw, l, j0, jstride, active); break;
      case 3: fft_stage<3, DIR, KMAX>(buf, pitch, pl.L, Ns, tw, l, j0, jstride, active); break;
      case 5: fft_stage<5, DIR, KMAX>(buf, pitch, pl.L, Ns, tw, l, j0, jstride, active); break;
      case 7: fft_stage<7, DIR, KMAX>(buf, pitch, pl.L, Ns, tw, l, j0, jstride, active); break;
      case 11: fft_stage<11, DIR, KMAX>(buf, pitch, pl.L, Ns, tw, l, j0, jstride, active); break;
      default: break;
    }
  }
}

// Host helper: the KMAX a tile transform needs for the given thread count.
inline int fft_kmax_needed(const FftPlan1D& pl, int nlines, int nthr) {
  if (pl.nstages == 0) return 1;
  const int jstride = nthr / nlines;
  if (jstride < 1) return 1 << 30;
  const int nb = pl.L / pl.min_radix;
  return (nb + jstride - 1) / jstride;
}

}  // namespace msc
