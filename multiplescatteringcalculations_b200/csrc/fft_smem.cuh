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
// Stages alternate between two tiles (ping-pong), so a thread streams one
// butterfly at a time through registers and a stage costs one barrier.
#pragma once
#include "msc_common.cuh"
#include "radix_constants.cuh"

namespace msc {

constexpr int FFT_MAX_STAGES = 12;

struct FftPlan1D {
  int L;
  int nstages;
  int pow2;  // 1 if L is a power of two (radices 2, 4, 8 only)
  int radix[FFT_MAX_STAGES];
  int ns[FFT_MAX_STAGES];
};

// Factorise L into radices {8,4,2,3,5,7,11}; false if L has another prime factor.
inline bool make_fft_plan(int L, FftPlan1D* p) {
  if (L < 1 || L > 4096) return false;
  int rad[FFT_MAX_STAGES];
  int n = 0, rest = L, e2 = 0;
  while (rest % 2 == 0) { rest /= 2; ++e2; }
  // powers of two: radix 8 stages, completed by one radix 4 or 2 stage
  int n8 = e2 / 3, r3 = e2 % 3;
  for (int i = 0; i < n8; ++i) rad[n++] = 8;
  if (r3 == 2) rad[n++] = 4;
  if (r3 == 1) rad[n++] = 2;
  const int odd[] = {3, 5, 7, 11};
  for (int r : odd) {
    while (rest % r == 0) {
      if (n >= FFT_MAX_STAGES) return false;
      rad[n++] = r;
      rest /= r;
    }
  }
  if (rest != 1) return false;
  p->L = L;
  p->nstages = n;
  p->pow2 = (rest == 1 && (L & (L - 1)) == 0) ? 1 : 0;
  int ns = 1;
  for (int s = 0; s < n; ++s) {
    p->radix[s] = rad[s];
    p->ns[s] = ns;
    ns *= rad[s];
  }
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
    const C v0 = v[0];
    v[0] = y0;
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      C A = v0, B;
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
      v[k] = A + iB;
      v[R - k] = A - iB;
    }
  }
};

// One Stockham stage src -> dst. Element idx of line l sits at idx*is + l*ls.
// Thread owns line l and butterflies j0, j0 + jstride, ...
template <int R, int DIR, bool POW2, typename C>
__device__ __forceinline__ void fft_stage(const C* __restrict__ src, C* __restrict__ dst, int is, int ls, int L,
                                          int Ns, const C* __restrict__ tw, int l, int j0, int jstride) {
  const int nb = L / R;
  const int tstep = L / (Ns * R);
  const int lo = l * ls;
  for (int j = j0; j < nb; j += jstride) {
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[(j + r * nb) * is + lo];
    const int kk = POW2 ? (j & (Ns - 1)) : (j % Ns);
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = tw[r * kk * tstep];
        if (DIR > 0) w.y = -w.y;
        v[r] = v[r] * w;
      }
    }
    Dft<R, DIR, C>::run(v);
    const int idxD = (j - kk) * R + kk;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(idxD + r * Ns) * is + lo] = v[r];
  }
}

// Full transform of every line of the tile in `a`, using `b` as the second tile;
// element idx of line l at idx*is + l*ls. Returns the tile holding the result (a
// or b). Needs nthr >= nlines; threads tid >= (nthr / nlines) * nlines idle during
// the stages. Ends with a barrier.
template <int DIR, bool POW2, typename C>
__device__ __forceinline__ C* fft_tile2(C* a, C* b, int is, int ls, int nlines, const FftPlan1D& pl, const C* tw,
                                        int tid, int nthr) {
  const int jstride = nthr / nlines;
  const bool active = tid < jstride * nlines;
  const int l = tid % nlines;
  const int j0 = active ? tid / nlines : (1 << 30);
  C* src = a;
  C* dst = b;
  for (int s = 0; s < pl.nstages; ++s) {
    const int Ns = pl.ns[s];
    switch (pl.radix[s]) {
      case 8: fft_stage<8, DIR, POW2>(src, dst, is, ls, pl.L, Ns, tw, l, j0, jstride); break;
      case 4: fft_stage<4, DIR, POW2>(src, dst, is, ls, pl.L, Ns, tw, l, j0, jstride); break;
      case 2: fft_stage<2, DIR, POW2>(src, dst, is, ls, pl.L, Ns, tw, l, j0, jstride); break;
      default:
        if (!POW2) {
          switch (pl.radix[s]) {
            case 3: fft_stage<3, DIR, false>(src, dst, is, ls, pl.L, Ns, tw, l, j0, jstride); break;
            case 5: fft_stage<5, DIR, false>(src, dst, is, ls, pl.L, Ns, tw, l, j0, jstride); break;
            case 7: fft_stage<7, DIR, false>(src, dst, is, ls, pl.L, Ns, tw, l, j0, jstride); break;
            case 11: fft_stage<11, DIR, false>(src, dst, is, ls, pl.L, Ns, tw, l, j0, jstride); break;
            default: break;
          }
        }
        break;
    }
    __syncthreads();
    C* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

// Lines interleaved: element idx of line l at idx*pitch + l.
template <int DIR, bool POW2, typename C>
__device__ C* fft_tile(C* a, C* b, int pitch, int nlines, const FftPlan1D& pl, const C* tw, int tid, int nthr) {
  return fft_tile2<DIR, POW2>(a, b, pitch, 1, nlines, pl, tw, tid, nthr);
}

// ---- compile-time engine for power-of-two lengths ---------------------------
// The same Stockham stages with the length, the radix sequence, the tile pitch,
// the line count and the block size known at compile time: every stride and
// loop bound is a constant, the loops unroll and the address arithmetic folds
// into the shared-memory offsets.
constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }

template <int L> struct Pow2Plan {
  static_assert(L >= 2 && (L & (L - 1)) == 0, "power-of-two length");
  static constexpr int LG = ilog2(L);
  static constexpr int N8 = LG / 3;
  static constexpr int NSTAGES = N8 + (LG % 3 != 0 ? 1 : 0);
  static constexpr int radix(int s) { return s < N8 ? 8 : (LG % 3 == 2 ? 4 : 2); }
  static constexpr int ns(int s) { return s == 0 ? 1 : ns(s - 1) * radix(s - 1); }
};

// Stage (R, NS) for line l, butterflies j0, j0 + JS, ...; element idx of line l at
// idx * P + l. HIN (first stage only): inputs idx >= L/2 are zero and not read.
// HOUT (last stage only): outputs idx >= L/2 are not needed and not computed.
template <int R, int NS, int L, int DIR, int P, int JS, bool HIN, bool HOUT, typename C>
__device__ __forceinline__ void fft_stage_ct(const C* __restrict__ src, C* __restrict__ dst, const C* __restrict__ tw,
                                             int l, int j0) {
  constexpr int NB = L / R;
  constexpr int TSTEP = L / (NS * R);
  constexpr int ITER = (NB + JS - 1) / JS;
  static_assert(!HIN || NS == 1, "pruned inputs on the first stage");
  static_assert(!HOUT || NS * R == L, "pruned outputs on the last stage");
#pragma unroll
  for (int it = 0; it < ITER; ++it) {
    const int j = j0 + it * JS;
    if (NB % JS != 0 && j >= NB) break;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = (HIN && r * NB >= L / 2) ? czero<C>() : src[(j + r * NB) * P + l];
    const int kk = j & (NS - 1);
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = tw[r * kk * TSTEP];
        if (DIR > 0) w.y = -w.y;
        v[r] = v[r] * w;
      }
    }
    Dft<R, DIR, C>::run(v);
    const int idxD = (j - kk) * R + kk;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (!HOUT || r * NS < L / 2) dst[(idxD + r * NS) * P + l] = v[r];
  }
}

template <int S, int L, int DIR, int P, int JS, bool HIN, bool HOUT, typename C>
__device__ __forceinline__ void fft_stages_ct(C* src, C* dst, const C* tw, int l, int j0, bool active) {
  using PL = Pow2Plan<L>;
  if constexpr (S < PL::NSTAGES) {
    constexpr bool hin = HIN && S == 0;
    constexpr bool hout = HOUT && S == PL::NSTAGES - 1;
    if (active) fft_stage_ct<PL::radix(S), PL::ns(S), L, DIR, P, JS, hin, hout>(src, dst, tw, l, j0);
    __syncthreads();
    fft_stages_ct<S + 1, L, DIR, P, JS, HIN, HOUT>(dst, src, tw, l, j0, active);
  }
}

// Full transform of the NLINES lines of tile a (pitch P), b the second tile; the
// block has NTHR threads. Returns the tile holding the result. Ends with a barrier.
// HIN: the inputs idx >= L/2 are zero (zero padding to L >= 2n); they need not be
// set in the tile. HOUT: only the outputs idx < L/2 are used; the others are left
// undefined.
template <int L, int DIR, int P, int NLINES, int NTHR, bool HIN = false, bool HOUT = false, typename C>
__device__ __forceinline__ C* fft_tile_ct(C* a, C* b, const C* tw, int tid) {
  constexpr int JS = NTHR / NLINES;
  static_assert(JS >= 1, "at least one thread per line");
  const bool active = tid < JS * NLINES;
  const int l = tid % NLINES;
  const int j0 = tid / NLINES;
  fft_stages_ct<0, L, DIR, P, JS, HIN, HOUT>(a, b, tw, l, j0, active);
  return (Pow2Plan<L>::NSTAGES % 2 == 0) ? a : b;
}

// ---- register-resident engine ------------------------------------------------------
// One thread transforms one line of L points held in registers (the same Stockham
// stages as above, every index a compile-time constant, so the stages are register
// renamings); twiddles come from the block's shared table tw[t] = exp(-2 pi i t / L).
// An output the caller never reads is not computed (dead code).
template <int L, int S, int DIR, int TS = 1, typename C>
__device__ __forceinline__ void fft_reg_stages(C* v, const C* __restrict__ tw) {
  using PL = Pow2Plan<L>;
  if constexpr (S < PL::NSTAGES) {
    constexpr int R = PL::radix(S), NS = PL::ns(S), NB = L / R, TSTEP = L / (NS * R);
    C out[L];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const int kk = j % NS;
      C u[R];
#pragma unroll
      for (int r = 0; r < R; ++r) u[r] = v[j + r * NB];
      if (kk != 0) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = tw[r * kk * TSTEP * TS];
          if (DIR > 0) w.y = -w.y;
          u[r] = u[r] * w;
        }
      }
      Dft<R, DIR, C>::run(u);
      const int idxD = (j - kk) * R + kk;
#pragma unroll
      for (int r = 0; r < R; ++r) out[idxD + r * NS] = u[r];
    }
#pragma unroll
    for (int i = 0; i < L; ++i) v[i] = out[i];
    fft_reg_stages<L, S + 1, DIR, TS>(v, tw);
  }
}

// TS: the table's entries are TS apart (tw[t TS] = exp(-2 pi i t / L)), so a table of
// a longer length L TS serves.
template <int L, int DIR, int TS = 1, typename C>
__device__ __forceinline__ void fft_reg(C* v, const C* __restrict__ tw) {
  fft_reg_stages<L, 0, DIR, TS>(v, tw);
}

// exp(-2 pi i t / 256), t < 256, complex64, in constant memory (the same values as the
// plans' twiddle tables; filled once per device, ensure_const_twiddles). In a register
// transform every twiddle index is a compile-time constant, so each twiddle is a
// constant-bank operand of the arithmetic instead of a load.
extern __constant__ float2 c_tw256[256];
extern __constant__ double2 c_tw256d[256];
template <int L> __device__ __forceinline__ float2 ctw(int t) {
  static_assert(L >= 1 && L <= 256 && 256 % L == 0, "a power-of-two length up to 256");
  return c_tw256[t * (256 / L)];
}
template <int L> __device__ __forceinline__ double2 ctwd(int t) {
  static_assert(L >= 1 && L <= 256 && 256 % L == 0, "a power-of-two length up to 256");
  return c_tw256d[t * (256 / L)];
}
// the constant-table twiddle of the element type
template <int L, typename C> __device__ __forceinline__ C ctw_t(int t) {
  if constexpr (sizeof(C) == 8) return ctw<L>(t);
  else return ctwd<L>(t);
}

template <int L, int S, int DIR, typename C>
__device__ __forceinline__ void fft_reg_c_stages(C* v) {
  using PL = Pow2Plan<L>;
  if constexpr (S < PL::NSTAGES) {
    constexpr int R = PL::radix(S), NS = PL::ns(S), NB = L / R, TSTEP = L / (NS * R);
    C out[L];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const int kk = j % NS;
      C u[R];
#pragma unroll
      for (int r = 0; r < R; ++r) u[r] = v[j + r * NB];
      if (kk != 0) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = ctw_t<L, C>(r * kk * TSTEP);
          if (DIR > 0) w.y = -w.y;
          u[r] = u[r] * w;
        }
      }
      Dft<R, DIR, C>::run(u);
      const int idxD = (j - kk) * R + kk;
#pragma unroll
      for (int r = 0; r < R; ++r) out[idxD + r * NS] = u[r];
    }
#pragma unroll
    for (int i = 0; i < L; ++i) v[i] = out[i];
    fft_reg_c_stages<L, S + 1, DIR, C>(v);
  }
}

// fft_reg with the twiddles from the constant tables (L a power of two <= 256)
template <int L, int DIR> __device__ __forceinline__ void fft_reg_c(float2* v) { fft_reg_c_stages<L, 0, DIR>(v); }
template <int L, int DIR> __device__ __forceinline__ void fft_reg_c(double2* v) { fft_reg_c_stages<L, 0, DIR>(v); }

}  // namespace msc
