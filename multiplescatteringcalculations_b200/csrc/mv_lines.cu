// Line FFT along the contiguous axis (the x passes of the matvec and of the G0 build).
#include <cstdint>

#include "mv_common.cuh"

namespace msc {

// Lines l in [0, nlines) start at off(l) = (l / G) * GS + (l % G) * stride in both
// in and out (groups of G equally spaced lines, groups GS apart); the first n_in
// inputs are used (rest zero), the first n_out outputs are written. A block takes
// TL lines; its gather is a set of cp.async copies awaited once. LC > 0: the
// length is the compile-time power of two LC (<= the block size), so a thread
// keeps one element index x = tid % LC in the gather and the store. PR (with LC):
// the forward transform has n_in <= LC/2 (its first stage reads only x < LC/2),
// the inverse n_out <= LC/2 (its last stage computes only x < LC/2).
template <typename T, int DIR, bool POW2, int LC, bool PR>
__global__ void __launch_bounds__(256, 4) k_fft_contig(const cx<T>* in, cx<T>* out, long long nlines, long long G,
                                                       long long GS, long long stride, int n_in, int n_out,
                                                       FftPlan1D pl, const cx<T>* __restrict__ twg, const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  using C = cx<T>;
  constexpr int TL = Tile<T>::W;
  constexpr int P = TL + 1;
  constexpr int NT = 256;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L = LC > 0 ? LC : pl.L;
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* ta = tw + L;
  C* tb = ta + (size_t)L * P;
  __shared__ long long loff[TL];
  const int tid = threadIdx.x;
  const long long line0 = (long long)blockIdx.x * TL;
  if (tid < TL) {
    const long long ln = line0 + tid;
    loff[tid] = ln < nlines ? (ln / G) * GS + (ln % G) * stride : -1;
  }
  for (int t = tid; t < L; t += NT) tw[t] = twg[t];
  __syncthreads();
  const C* res;
  if constexpr (LC > 0) {
    static_assert(NT % LC == 0, "length divides the block");
    constexpr int QS = NT / LC;  // lines per sweep
    const int x = tid % LC, q0 = tid / LC;
    constexpr bool HIN = PR && DIR < 0, HOUT = PR && DIR > 0;
    if (!HIN || x < LC / 2) {
#pragma unroll
      for (int k = 0; k < (TL + QS - 1) / QS; ++k) {
        const int q = q0 + k * QS;
        if (QS > TL && q >= TL) break;
        const long long o = loff[q];
        const bool ok = o >= 0 && x < n_in;
        cp_async_elem(ta + x * P + q, ok ? in + o + x : in, ok);
      }
    }
    cp_async_wait_all();
    __syncthreads();
    res = fft_tile_ct<LC, DIR, P, TL, NT, HIN, HOUT>(ta, tb, tw, tid);
    if (x < n_out) {
#pragma unroll
      for (int k = 0; k < (TL + QS - 1) / QS; ++k) {
        const int q = q0 + k * QS;
        if (QS > TL && q >= TL) break;
        const long long o = loff[q];
        if (o >= 0) out[o + x] = res[x * P + q];
      }
    }
  } else {
    {
      QR w(tid, NT, L);  // (line, x)
      for (int it = tid; it < TL * L; it += NT, w.next()) {
        const long long o = loff[w.q];
        const bool ok = o >= 0 && w.r < n_in;
        cp_async_elem(ta + w.r * P + w.q, ok ? in + o + w.r : in, ok);
      }
    }
    cp_async_wait_all();
    __syncthreads();
    res = fft_tile<DIR, POW2>(ta, tb, P, TL, pl, tw, tid, NT);
    QR w(tid, NT, n_out);
    for (int it = tid; it < TL * n_out; it += NT, w.next()) {
      const long long o = loff[w.q];
      if (o >= 0) out[o + w.r] = res[w.r * P + w.q];
    }
  }
}

// ---- register four-step engine (complex64, L = 64, 128, 256) -------------------------
// A line of L = R1 * NTL points is held by NTL consecutive threads of a warp, R1 points
// each: thread t holds x[t + NTL m], m < R1. Four steps: an R1-point DFT over m in
// registers, the twiddle W_L^(t k1), a transpose through shared memory within the warp
// (__syncwarp only; no block barrier), an NTL-point DFT over t in registers. Thread t
// then holds X[k1 + R1 k2] for its KPT = R1 / NTL values of k1 and every k2. Shared
// memory per line: R1 rows of NTL + 1 entries (the odd row pitch spreads a reader's
// rows over the banks), lines padded to alternate bank halves.
template <int L> struct RowReg {
  static constexpr int NTL = L >= 256 ? 16 : 8;
  static constexpr int R1 = L / NTL;
  static constexpr int KPT = R1 / NTL;
  static constexpr int LPB = 256 / NTL;  // lines per block
  static constexpr int RS = NTL + 1;     // row pitch
  static constexpr int LS0 = R1 * RS;
  static constexpr int LS = ((LS0 * 8 / 4) % 32 == 16) ? LS0 : LS0 + 8;  // line pitch (complex)
};

template <int DIR, int L>
__global__ void __launch_bounds__(256) k_fft_rows_reg(const float2* __restrict__ in, float2* __restrict__ out,
                                                      long long nlines, long long G, long long GS, long long stride,
                                                      int n_in, int n_out, const float2* __restrict__ twg,
                                                      const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  using RR = RowReg<L>;
  constexpr int NTL = RR::NTL, R1 = RR::R1, KPT = RR::KPT, LPB = RR::LPB, RS = RR::RS, LS = RR::LS;
  static_assert(R1 % NTL == 0, "R1 a multiple of NTL");
  __shared__ __align__(16) float2 sm[LPB * LS];
  const int q = threadIdx.x / NTL, t = threadIdx.x % NTL;
  const long long line = (long long)blockIdx.x * LPB + q;
  const long long off = line < nlines ? (line / G) * GS + (line % G) * stride : -1;
  float2 v[R1];
#pragma unroll
  for (int m = 0; m < R1; ++m) {
    const int n = t + NTL * m;
    v[m] = (off >= 0 && n < n_in) ? in[off + n] : make_float2(0.f, 0.f);
  }
  fft_reg_c<R1, DIR>(v);
#pragma unroll
  for (int k1 = 1; k1 < R1; ++k1) {
    float2 w = __ldg(twg + ((t * k1) & (L - 1)));
    if (DIR > 0) w.y = -w.y;
    v[k1] = v[k1] * w;
  }
  float2* ls = sm + q * LS;
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) ls[k1 * RS + t] = v[k1];
  __syncwarp();
  float2 u[KPT][NTL];
#pragma unroll
  for (int c = 0; c < KPT; ++c)
#pragma unroll
    for (int s = 0; s < NTL; ++s) u[c][s] = ls[(t * KPT + c) * RS + s];
#pragma unroll
  for (int c = 0; c < KPT; ++c) fft_reg_c<NTL, DIR>(u[c]);
  if (off < 0) return;
  float2* o = out + off;
#pragma unroll
  for (int k2 = 0; k2 < NTL; ++k2) {
    const int k = t * KPT + R1 * k2;
    if constexpr (KPT == 2) {
      if (k + 1 < n_out)
        *reinterpret_cast<float4*>(o + k) = make_float4(u[0][k2].x, u[0][k2].y, u[1][k2].x, u[1][k2].y);
      else if (k < n_out)
        o[k] = u[0][k2];
    } else {
#pragma unroll
      for (int c = 0; c < KPT; ++c)
        if (k + c < n_out) o[k + c] = u[c][k2];
    }
  }
}

template <typename T>
int launch_fft_contig(msc_plan* pl, const cx<T>* in, cx<T>* out, long long nlines, long long G, long long GS,
                      long long stride, int n_in, int n_out, const FftPlan1D& f, const cx<T>* tw, int dir,
                      const int* done) {
  constexpr int TL = Tile<T>::W;
  const int nthr = 256;
  const size_t sm = sizeof(cx<T>) * ((size_t)f.L + 2 * (size_t)f.L * (TL + 1));
  const unsigned nb = (unsigned)((nlines + TL - 1) / TL);
  const void* kern = nullptr;
  const bool pr = 2 * (dir < 0 ? n_in : n_out) <= f.L;
#define LEN(D, LL) \
  kern = pr ? (const void*)k_fft_contig<T, D, true, LL, true> : (const void*)k_fft_contig<T, D, true, LL, false>;
#define PICK(D)                                                                                                  \
  switch (f.L) {                                                                                                 \
    case 16: LEN(D, 16) break;                                                                                   \
    case 32: LEN(D, 32) break;                                                                                   \
    case 64: LEN(D, 64) break;                                                                                   \
    case 128: LEN(D, 128) break;                                                                                 \
    case 256: LEN(D, 256) break;                                                                                 \
    default:                                                                                                     \
      kern = f.pow2 ? (const void*)k_fft_contig<T, D, true, 0, false> : (const void*)k_fft_contig<T, D, false, 0, false>; \
  }
  if (dir < 0) { PICK(-1) } else { PICK(+1) }
#undef PICK
#undef LEN
  if constexpr (sizeof(T) == 4) {
    // register four-step engine: complex64, L = 64, 128, 256, even line offsets (16-byte stores)
    const bool even = (GS % 2 == 0) && (stride % 2 == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
    const void* rk = nullptr;
    int lpb = 0;
#define RR(D, LL) rk = (const void*)k_fft_rows_reg<D, LL>; lpb = RowReg<LL>::LPB;
    if (even && f.pow2) {
      if (dir < 0) {
        if (f.L == 64) { RR(-1, 64) } else if (f.L == 128) { RR(-1, 128) } else if (f.L == 256) { RR(-1, 256) }
      } else {
        if (f.L == 64) { RR(+1, 64) } else if (f.L == 128) { RR(+1, 128) } else if (f.L == 256) { RR(+1, 256) }
      }
    }
#undef RR
    if (rk) {
      const unsigned nbr = (unsigned)((nlines + lpb - 1) / lpb);
      void* args[] = {(void*)&in, (void*)&out, (void*)&nlines, (void*)&G, (void*)&GS, (void*)&stride,
                      (void*)&n_in, (void*)&n_out, (void*)&tw, (void*)&done};
      MSC_CUDA(launch_pdl(rk, dim3(nbr), dim3(256), args, 0, pl->stream));
      ::msc::note_launch();
      return MSC_OK;
    }
  }
  MSC_CUDA(prep_kernel(kern));
  FftPlan1D ff = f;
  void* args[] = {(void*)&in, (void*)&out, (void*)&nlines, (void*)&G, (void*)&GS, (void*)&stride,
                  (void*)&n_in, (void*)&n_out, (void*)&ff, (void*)&tw, (void*)&done};
  MSC_CUDA(launch_pdl(kern, dim3(nb), dim3(nthr), args, sm, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}
template int launch_fft_contig<float>(msc_plan*, const float2*, float2*, long long, long long, long long, long long,
                                      int, int, const FftPlan1D&, const float2*, int, const int*);
template int launch_fft_contig<double>(msc_plan*, const double2*, double2*, long long, long long, long long,
                                       long long, int, int, const FftPlan1D&, const double2*, int, const int*);

}  // namespace msc
