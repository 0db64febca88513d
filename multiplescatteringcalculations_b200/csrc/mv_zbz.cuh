// Matvec kernel ZBZ': forward FFT along z, the per-wavevector 9x9 block multiply
// acc(k) = K(k) tau(k), and the inverse FFT along z, fused over columns (ky, kx).
//
// The workspace W[c][n][ky][kx] holds tau transformed along y and x with the
// N_z layers in space. A block loads, for all 9 components, a set of columns
// (n < N_z, zero padded to Lz) into one shared-memory tile, transforms along z,
// multiplies every wavevector of the tile by its 9x9 kernel block, transforms
// back and stores the N_z layers in place. The zero-padded z spectrum never
// leaves shared memory.
//
// Octant spectrum (mirror-symmetric kernel): the block of (ky_o, kx chunk) takes
// the four columns (+-ky_o, +-kx_o) of each kx_o in the chunk; the point k reads
// K at its octant image |k| = (min(kz, Lz-kz), ky_o, kx_o) and uses
// K(k) = S_f K(|k|) S_f, S_f the product of the reflection sign matrices of the
// axes on which k is the negative frequency. Columns that coincide (kx_o = 0 or
// Lx/2, ky_o = 0 or Ly/2) are taken once. Full spectrum (Bloch-phased kernels):
// 4 KX consecutive kx of one ky, each point reading its own K.
#pragma once
#include "mv_common.cuh"

namespace msc {

// v <- S_f v: the sign flips as XORs of the sign bits (no compare and select per
// component). sign_mask(f) holds bit c when component c is odd under the reflections
// f (bit 0 x, bit 1 y, bit 2 z).
__device__ __forceinline__ unsigned sign_mask(int f) {
  unsigned m = 0;
#pragma unroll
  for (int c = 0; c < 9; ++c) m |= (unsigned)(__popc(dof_parity(c) & f) & 1) << c;
  return m;
}
__device__ __forceinline__ void reflect_mask(float2* v, unsigned m) {
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    if (dof_parity(c) == 0) continue;  // even under every reflection
    const unsigned s = ((m >> c) & 1u) << 31;
    v[c].x = __uint_as_float(__float_as_uint(v[c].x) ^ s);
    v[c].y = __uint_as_float(__float_as_uint(v[c].y) ^ s);
  }
}
__device__ __forceinline__ void reflect_mask(double2* v, unsigned m) {
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    if (dof_parity(c) == 0) continue;
    const unsigned long long s = (unsigned long long)((m >> c) & 1u) << 63;
    v[c].x = __longlong_as_double((long long)((unsigned long long)__double_as_longlong(v[c].x) ^ s));
    v[c].y = __longlong_as_double((long long)((unsigned long long)__double_as_longlong(v[c].y) ^ s));
  }
}
template <typename C> __device__ __forceinline__ void reflect(C* v, int f) { reflect_mask(v, sign_mask(f)); }

// One field vector t multiplied by one kernel block, in place; ld(e) returns the
// stored entry e. SYM (E = 45): entry e enumerates i <= j row-major and holds
// (K D)_ij with D = diag(1 x6, 2 x3), symmetric for the point propagator;
// K_ij = (K D)_ij / D_j. FULL (E = 81): K_ij row-major.
//
// complex128: plain complex FMAs.
template <bool SYM, typename LD> __device__ __forceinline__ void block_mul(LD ld, double2* t) {
  double2 acc[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    if (SYM && j >= 6) {
      t[j].x *= 0.5;
      t[j].y *= 0.5;
    }
    acc[j] = czero<double2>();
  }
  if constexpr (SYM) {
    int e = 0;
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
      for (int j = i; j < 9; ++j, ++e) {
        const double2 m = ld(e);
        fma_(acc[i], m, t[j]);
        if (i != j) fma_(acc[j], m, t[i]);
      }
  } else {
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
      for (int j = 0; j < 9; ++j) fma_(acc[i], ld(i * 9 + j), t[j]);
  }
#pragma unroll
  for (int j = 0; j < 9; ++j) t[j] = acc[j];
}

// complex64: m t = m.x (t.x, t.y) + m.y (-t.y, t.x), two paired FP32 FMAs per
// complex FMA; (-t.y, t.x) is formed once per vector.
template <bool SYM, typename LD> __device__ __forceinline__ void block_mul(LD ld, float2* t) {
  float2 tr[9], acc[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    if (SYM && j >= 6) t[j] = __fmul2_rn(t[j], make_float2(0.5f, 0.5f));
    tr[j] = make_float2(-t[j].y, t[j].x);
    acc[j] = make_float2(0.f, 0.f);
  }
  auto cfma = [&](float2& a, const float2& m, int j) {
    a = __ffma2_rn(make_float2(m.x, m.x), t[j], a);
    a = __ffma2_rn(make_float2(m.y, m.y), tr[j], a);
  };
  if constexpr (SYM) {
    int e = 0;
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
      for (int j = i; j < 9; ++j, ++e) {
        const float2 m = ld(e);
        cfma(acc[i], m, j);
        if (i != j) cfma(acc[j], m, i);
      }
  } else {
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
      for (int j = 0; j < 9; ++j) cfma(acc[i], ld(i * 9 + j), j);
  }
#pragma unroll
  for (int j = 0; j < 9; ++j) t[j] = acc[j];
}

// Block (blockIdx.x = kx chunk, blockIdx.y = ky_o), ZBZ_THREADS threads. Lines of
// the tile: line c * NC + s for component c and column slot s < NC = 4 KX; element
// kz of a line at kz * (NL + 1) + line. Shared memory: [spectrum slice (octant,
// staged)] [twiddles Lz] [tile a] [tile b]. All global reads are cp.async copies
// issued together and awaited once.
//
// LC > 0: compile-time Lz = LC (a power of two, so N_z <= Lz/2: the forward
// transform reads only kz < Lz/2 and the inverse computes only kz < Lz/2) and
// KX = KXC; LC = 0: both from the plan and the layout at run time. The block size is a multiple of NL and of
// 8 KX, so a thread keeps one line in the load and store loops and one slot in
// the multiply.
//
// nrhs > 1: the block applies its slice of the spectrum (staged once) to the same
// columns of nrhs vectors in turn, vector r's workspace at W + r * 9 N_z Ly Lx.
template <typename T, int LC, int KXC, bool SYM, bool OCT, bool POW2>
__global__ void __launch_bounds__(ZBZ_THREADS, 2) k_zbz(cx<T>* __restrict__ W, const kent<T>* __restrict__ khat, Geo g,
                                                        ZbzLayout lay, FftPlan1D pl, const cx<T>* __restrict__ twg,
                                                        const int* done, int nrhs) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  using C = cx<T>;
  using KE = kent<T>;
  constexpr bool CT = LC > 0;
  constexpr int NT = ZBZ_THREADS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long loff[ZBZ_MAX_LINES];  // W offset of each line, -1: slot unused
  __shared__ int sflag[ZBZ_MAX_LINES / 9];   // slot reflections: bit 0 kx mirrored, bit 1 ky mirrored
  const int KX = CT ? KXC : lay.KX;
  const int NC = 4 * KX, NL = 9 * NC, P = NL + 1;
  const int Lz = CT ? LC : pl.L;
  const bool ksm = OCT && lay.ksm;
  KE* ks = reinterpret_cast<KE*>(smem_raw);
  C* tw = reinterpret_cast<C*>(ks + (ksm ? lay.CS : 0));
  C* ta = tw + Lz;
  C* tb = ta + (size_t)Lz * P;
  const int tid = threadIdx.x;
  const long long plane = (long long)g.Ly * g.Lx;
  const long long cstride = (long long)g.Nz * plane;
  const int kyo = blockIdx.y;
  const int x0 = blockIdx.x * (OCT ? KX : NC);
  const KE* kblk = OCT ? khat + ((long long)kyo * lay.NXC + blockIdx.x) * lay.CS : khat;
  if (ksm) {
    const int n16 = (int)(lay.CS * sizeof(KE) / 16);
    for (int i = tid; i < n16; i += NT)
      cp_async16(reinterpret_cast<unsigned char*>(ks) + 16 * i, reinterpret_cast<const unsigned char*>(kblk) + 16 * i);
  }
  if (tid < NC) {
    const int s = tid;
    long long col = -1;
    int f = 0;
    if (OCT) {
      const int q = s / KX, kxo = x0 + s % KX;
      bool ok = kxo < g.Hx;
      if (q & 1) ok = ok && kxo != 0 && 2 * kxo != g.Lx;  // kx_o has a distinct mirror
      if (q & 2) ok = ok && kyo != 0 && 2 * kyo != g.Ly;
      const int kx = (q & 1) ? g.Lx - kxo : kxo;
      const int ky = (q & 2) ? g.Ly - kyo : kyo;
      if (ok) col = (long long)ky * g.Lx + kx;
      f = q;
    } else {
      const int kx = x0 + s;
      if (kx < g.Lx) col = (long long)kyo * g.Lx + kx;
    }
#pragma unroll
    for (int c = 0; c < 9; ++c) loff[c * NC + s] = col >= 0 ? c * cstride + col : -1;
    sflag[s] = f;
  }
  for (int t = tid; t < Lz; t += NT) tw[t] = twg[t];
  __syncthreads();
  // this thread's line and rows kz = r0, r0 + RS, ...
  const int line = tid % NL, r0 = tid / NL, RS = NT / NL;
  const long long o0 = loff[line];
  for (int rh = 0; rh < nrhs; ++rh) {
  const long long o = o0 >= 0 ? o0 + (long long)rh * 9 * cstride : -1;
  {
    // compile time: only rows kz < Lz/2 are read by the pruned first FFT stage (N_z <= Lz/2)
    const int nrow = (CT && (LC / 2) % (NT / (36 * (CT ? KXC : 1))) == 0) ? (LC / 2) / (NT / (36 * (CT ? KXC : 1)))
                                                                        : (Lz - r0 + RS - 1) / RS;
#pragma unroll 4
    for (int k = 0; k < nrow; ++k) {
      const int kz = r0 + k * RS;
      const bool ok = o >= 0 && kz < g.Nz;
      cp_async_elem(ta + kz * P + line, ok ? W + o + kz * plane : W, ok);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  C* res;
  if constexpr (CT) res = fft_tile_ct<LC, -1, 36 * KXC + 1, 36 * KXC, NT, true, false>(ta, tb, tw, tid);
  else res = fft_tile<-1, POW2>(ta, tb, P, NL, pl, tw, tid, NT);
  C* oth = (res == ta) ? tb : ta;
  if (OCT) {
    // item (j, q, side, kp), j fastest: the point kz = kp (side 0) or Lz - kp (side 1)
    // of slot q KX + j. The up to 8 points of one octant entry share a warp. A
    // thread keeps (j, q, side) and walks kp = kp0, kp0 + NT / (8 KX), ...
    const int j = tid % KX, q = (tid / KX) & 3, side = (tid / (4 * KX)) & 1;
    const int kstep = NT / (8 * KX);
    const int s = q * KX + j;
    const int estr = g.Hz * KX;
    const int f0 = sflag[s] | (side ? 4 : 0);
    if (loff[s] >= 0) {
      for (int kp = tid / (8 * KX); kp < g.Hz; kp += kstep) {
        if (side && (kp == 0 || 2 * kp == Lz)) continue;
        const int kz = side ? Lz - kp : kp;
        const int ko = kp * KX + j;
        C* ra = res + kz * P + s;
        C t[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) t[c] = ra[c * NC];
        reflect(t, f0);
        if (ksm) {
          auto ld = [&](int e) { return ks[e * estr + ko]; };
          block_mul<SYM>(ld, t);
        } else {
          auto ld = [&](int e) { return __ldg(kblk + e * estr + ko); };
          block_mul<SYM>(ld, t);
        }
        reflect(t, f0);
#pragma unroll
        for (int c = 0; c < 9; ++c) ra[c * NC] = t[c];
      }
    }
  } else {
    const long long estride = (long long)g.Hz * g.Hy * g.Hx;
    const int nitem = Lz * NC;
    for (int it = tid; it < nitem; it += NT) {
      const int s = it % NC, kz = it / NC;
      if (loff[s] < 0) continue;
      const KE* kb = khat + ((long long)kz * g.Hy + kyo) * g.Hx + (x0 + s);
      auto ld = [&](int e) { return __ldg(kb + (long long)e * estride); };
      C* ra = res + kz * P + s;
      C t[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) t[c] = ra[c * NC];
      block_mul<SYM>(ld, t);
#pragma unroll
      for (int c = 0; c < 9; ++c) ra[c * NC] = t[c];
    }
  }
  __syncthreads();
  const C* out;
  if constexpr (CT) out = fft_tile_ct<LC, +1, 36 * KXC + 1, 36 * KXC, NT, false, true>(res, oth, tw, tid);
  else out = fft_tile<+1, POW2>(res, oth, P, NL, pl, tw, tid, NT);
  if (o >= 0) {
    const int nrow = (g.Nz - r0 + RS - 1) / RS;
#pragma unroll 4
    for (int k = 0; k < nrow; ++k) {
      const int kz = r0 + k * RS;
      W[o + kz * plane] = out[kz * P + line];
    }
  }
  // the next vector's gather writes the tiles this vector's store reads
  if (rh + 1 < nrhs) __syncthreads();
  }
}

// Compile-time KX of a power-of-two Lz (the layout's choice for an octant spectrum).
template <typename T> constexpr int zbz_kx_ct(int L, int E) { return zbz_layout<T>(L, L / 2 + 1, 1, E, true).KX; }

template <typename T>
int launch_zbz(msc_plan* pl, cx<T>* W, const int* done, int nrhs) {
  const Geo& g = pl->g;
  const kent<T>* kh = (const kent<T>*)(sizeof(T) == 8 ? pl->khat64.p : pl->khat32.p);
  const cx<T>* tw = (const cx<T>*)(sizeof(T) == 8 ? pl->tw64_z.p : pl->tw32_z.p);
  const ZbzLayout lay = zbz_layout<T>(g, pl->E);
  if (lay.smem > (size_t)ZBZ_SMEM_LIMIT) {
    set_error("Lz=%d exceeds the shared memory of the fused z pass", g.Lz);
    return MSC_ERR_UNSUPPORTED;
  }
  {
    const int r = launch_zpass<T>(pl, W, done, nrhs);
    if (r != 1) return r;
  }
  const bool sym = pl->E == 45;
  dim3 grid(g.oct ? (unsigned)lay.NXC : (unsigned)((g.Lx + 4 * lay.KX - 1) / (4 * lay.KX)),
            (unsigned)(g.oct ? g.Hy : g.Ly));
  const void* kern = nullptr;
  // compile-time kernels: octant spectrum, Lz in {8, 16, 32, 64, 128}
#define CT_CASE(LZ)                                                                                  \
  case LZ:                                                                                           \
    if (sym && lay.KX == zbz_kx_ct<T>(LZ, 45))                                                       \
      kern = (const void*)k_zbz<T, LZ, zbz_kx_ct<T>(LZ, 45), true, true, true>;                       \
    else if (!sym && lay.KX == zbz_kx_ct<T>(LZ, 81))                                                 \
      kern = (const void*)k_zbz<T, LZ, zbz_kx_ct<T>(LZ, 81), false, true, true>;                      \
    break;
  if (g.oct) switch (g.Lz) {
      CT_CASE(8)
      CT_CASE(16)
      CT_CASE(32)
      CT_CASE(64)
      CT_CASE(128)
      default: break;
    }
#undef CT_CASE
  if (!kern) {
#define RT(P2)                                                                                        \
  kern = sym ? (g.oct ? (const void*)k_zbz<T, 0, 0, true, true, P2> : (const void*)k_zbz<T, 0, 0, true, false, P2>) \
             : (g.oct ? (const void*)k_zbz<T, 0, 0, false, true, P2> : (const void*)k_zbz<T, 0, 0, false, false, P2>);
    if (pl->fz.pow2) { RT(true) } else { RT(false) }
#undef RT
  }
  MSC_CUDA(prep_kernel(kern));
  Geo gg = g;
  ZbzLayout ll = lay;
  FftPlan1D ff = pl->fz;
  void* args[] = {(void*)&W, (void*)&kh, (void*)&gg, (void*)&ll, (void*)&ff, (void*)&tw, (void*)&done,
                  (void*)&nrhs};
  MSC_CUDA(launch_pdl(kern, grid, dim3(ZBZ_THREADS), args, lay.smem, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}

}  // namespace msc
