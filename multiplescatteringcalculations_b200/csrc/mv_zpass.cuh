// Matvec kernel ZBZ', register form for the octant spectrum at power-of-two Lz (complex64
// up to 64, complex128 up to 32): forward FFT along z, the 9x9 block multiply, inverse FFT
// along z, one block per (ky_o, kx chunk) as in k_zbz (the four mirror columns of
// KX octant columns, all 9 components: 36 KX lines of Lz points).
//
// Each line is transformed in registers by S = 1 or 2 threads. With S = 2 thread b
// of a line computes the outputs X[2m + b]: since the line holds data only at
// n < N_z <= Lz/2, X[2m + b] = sum_{n < Lz/2} (x[n] W^{n b}) W_{Lz/2}^{n m}, one
// Lz/2-point transform of the twiddled input (W = exp(-2 pi i / Lz)). The inverse
// x[2n + b] = sum_{k < Lz/2} W_{Lz/2}^{-n k} [W^{-b k} (X[k] + (-1)^b X[k + Lz/2])]
// is again one Lz/2-point transform per thread. Neither direction exchanges data
// between the two threads, and a line of Lz = 64 needs 32 complex registers.
//
// Phases: (1) each thread loads its line's N_z layers from W straight into
// registers (the two threads of a line are adjacent lanes, so their loads coalesce
// into one request) while one bulk copy (cp.async.bulk, completing on an mbarrier)
// brings the block's contiguous slice of the spectrum into shared memory; (2) transform,
// spectrum rows to the tile; (3) once the slice has landed, the block multiply, one
// wavevector per item, every offset into the staged slice a compile-time constant;
// (4) the inverse transform from the tile, the N_z layers back to W. The wait for the
// slice is bounded (the plan's wait limit): when it runs out the kernel records a
// timeout in the plan's status word and finishes without the slice; before the block
// exits its first thread waits, with a fixed limit, for the copy to land.
//
// Measured alternatives that lost (B200, 64x64x16 and 256x256x32): the slice staged
// pre-broadcast (re, re, im, im) to save the operand moves (two blocks per SM instead
// of three: 50 against 36 us), the slice read from L2 in the multiply instead of
// staged (six blocks per SM, exposed L2 latency: 42 against 36 us; 331 against
// 297 us), two threads per line at Lz = 32 (39 us), the lightest blocks (the kx = Lx/2
// chunk, the ky_o = 0 and Ly/2 rows) dispatched last (matvec 55.5 against 55.4 us).
#pragma once
#include "mv_zbz.cuh"

namespace msc {

template <typename T, int LZ, int KX, int S, bool SYM> struct ZpCfg {
  using C = cx<T>;
  static_assert(S == 1 || S == 2, "one or two threads per line");
  static_assert(LZ >= 8 && LZ <= 64 && (LZ & (LZ - 1)) == 0, "power-of-two Lz");
  static_assert(sizeof(T) == 4 || LZ / S <= 16, "complex128 lines of at most 16 points per thread");
  static constexpr int NC = 4 * KX;                   // column slots: 4 mirrors x KX
  static constexpr int NL = 9 * NC;                   // lines
  static constexpr int NT = ((S * NL + 31) / 32) * 32;
  static constexpr int LH = LZ / S;                   // points of a thread's transform
  static constexpr int HZ = LZ / 2 + 1;               // stored kz rows (octant)
  static constexpr int E = SYM ? 45 : 81;
  static constexpr int KE = E * HZ * KX;              // entries of a block's slice
  // the slice's stride in khat (zbz_layout: complex64 slices padded to 16 bytes)
  static constexpr int CS = sizeof(T) == 4 ? (KE + 1) / 2 * 2 : KE;
  // tile pitch: the complex64 S = 2 forward stores of a half warp cover rows k and k + 1
  // of 8 lines; a pitch of 8 mod 16 elements puts them in disjoint banks (a complex128
  // row of 8 lines already fills the 32 banks)
  static constexpr int P = (S == 1 || sizeof(T) == 8) ? NL : NL + (8 - NL % 16 + 16) % 16;
  static constexpr size_t ES = sizeof(C);
  static constexpr size_t KBYTES = ES * CS;
  static constexpr size_t TW_OFF = (KBYTES + 15) / 16 * 16;
  static constexpr size_t SMEM = TW_OFF + ES * (size_t)LZ + ES * (size_t)LZ * P;
  static_assert(SMEM <= 227 * 1024 - 1024, "shared memory of one block");
  static constexpr int BLK_SMEM = (int)((228 * 1024) / (SMEM + 1024 + 16 * NC));
  static constexpr int BLK_REG = 65536 / (NT * (sizeof(T) == 4 ? 96 : 128));
  static constexpr int AUTO = BLK_SMEM < BLK_REG ? BLK_SMEM : BLK_REG;
  static constexpr int MINB = AUTO < 1 ? 1 : AUTO;
};

constexpr long long ZP_WAIT_LIMIT = 1ll << 22;  // mbarrier polls before a timeout is recorded

__device__ __forceinline__ bool zp_try_wait(uint32_t addr, uint32_t phase) {
  uint32_t ok = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(addr), "r"(phase)
      : "memory");
  return ok != 0;
}

template <typename T, int LZ, int KX, int S, bool SYM>
__global__ void __launch_bounds__(ZpCfg<T, LZ, KX, S, SYM>::NT, ZpCfg<T, LZ, KX, S, SYM>::MINB)
    k_zpass(cx<T>* __restrict__ W, const cx<T>* __restrict__ khat, Geo g, int nxc, const cx<T>* __restrict__ twg,
            const int* done, int nrhs, int* status, long long wait_limit) {
  using Cf = ZpCfg<T, LZ, KX, S, SYM>;
  using C = cx<T>;
  constexpr int NC = Cf::NC, NL = Cf::NL, NT = Cf::NT, LH = Cf::LH, HZ = Cf::HZ, P = Cf::P;
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int sq[NC];  // mirror flags of slot s (bit 0 kx, bit 1 ky), -1: slot unused
  __shared__ __align__(8) unsigned long long kbar;  // completion of the slice's bulk copy
  C* tw = reinterpret_cast<C*>(smem_raw + Cf::TW_OFF);
  C* tile = tw + LZ;
  const int tid = threadIdx.x;
  const long long plane = (long long)g.Ly * g.Lx;
  const long long cstride = (long long)g.Nz * plane;
  const int kyo = blockIdx.y;
  const int x0 = blockIdx.x * KX;
  const C* kblk = khat + ((long long)kyo * nxc + blockIdx.x) * Cf::CS;
  // the column of slot s: q = s / KX (mirror flags), kx_o = x0 + s % KX; -1 when the
  // mirror coincides with another slot's column or kx_o lies beyond the octant
  auto slot_col = [&](int s) -> long long {
    const int q = s / KX, kxo = x0 + s % KX;
    bool ok = kxo < g.Hx;
    if (q & 1) ok = ok && kxo != 0 && 2 * kxo != g.Lx;
    if (q & 2) ok = ok && kyo != 0 && 2 * kyo != g.Ly;
    const int kx = (q & 1) ? g.Lx - kxo : kxo;
    const int ky = (q & 2) ? g.Ly - kyo : kyo;
    return ok ? (long long)ky * g.Lx + kx : -1;
  };
  const int b = S == 1 ? 0 : (tid & (S - 1));
  const int l = tid / S;
  const bool lact = l < NL;
  long long o0 = -1;
  if (lact) {
    const long long col = slot_col(l % NC);
    if (col >= 0) o0 = (l / NC) * cstride + col;
  }
  if (tid < NC) sq[tid] = slot_col(tid) >= 0 ? tid / KX : -1;
  const uint32_t kbar_a = (uint32_t)__cvta_generic_to_shared(&kbar);
  if (tid == 0) {
    // the slice: CS entries, 16-byte aligned at both ends (zbz_layout pads CS to even)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(kbar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(kbar_a), "r"((int)Cf::KBYTES)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem_raw)),
                 "l"(kblk), "r"((int)Cf::KBYTES), "r"(kbar_a)
                 : "memory");
  }
  bool kready = false;
  for (int rh = 0; rh < nrhs; ++rh) {
    const long long o = o0 >= 0 ? o0 + (long long)rh * 9 * cstride : -1;
    C v[LH];
    // (1) the line's layers n < N_z <= Lz/2; the upper half of an S = 1 line is zero
#pragma unroll
    for (int n = 0; n < LH; ++n) v[n] = (n < LZ / 2 && o >= 0 && n < g.Nz) ? W[o + n * plane] : czero<C>();
    // the previous vector's inverse reads of the tile are done; the barrier's init visible
    __syncthreads();
    // (2) forward transform, rows kz = S m + b of the tile
    if (S == 2 && b) {
#pragma unroll
      for (int n = 0; n < LH; ++n) v[n] = v[n] * ctw_t<LZ, C>(n);
    }
    fft_reg_c<LH, -1>(v);
    if (lact) {
#pragma unroll
      for (int m = 0; m < LH; ++m) tile[(S * m + b) * P + l] = v[m];
    }
    if (rh == 0) {
      for (long long it = 0; it < wait_limit && !kready; ++it) kready = zp_try_wait(kbar_a, 0u);
      if (!kready && status) atomicExch(status, 1);
    }
    __syncthreads();
    // (3) block multiply. Item (j, q, kpa, side, kph), j fastest: the point kz = kp
    // (side 0) or Lz - kp (side 1), kp = kph A + kpa, of slot q KX + j. A half warp
    // holds one side and A x KX = 4 octant entries (each a shared-memory broadcast),
    // its 16 tile reads consecutive or P apart.
    {
      constexpr int A = 4 / KX;
      constexpr int NITEM = 32 * ((HZ + A - 1) / A);
      for (int it = tid; it < NITEM; it += NT) {
        const int j = it % KX, q = (it / KX) & 3, kpa = (it / (4 * KX)) % A, side = (it >> 4) & 1;
        const int kp = (it >> 5) * A + kpa;
        if (kp >= HZ) continue;
        if (side && (kp == 0 || 2 * kp == LZ)) continue;
        const int s = q * KX + j;
        if (sq[s] < 0) continue;
        const int f = q | (side << 2);
        const int kz = side ? LZ - kp : kp;
        const int ko = kp * KX + j;
        C* ra = tile + kz * P + s;
        C t[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) t[c] = ra[c * NC];
        const unsigned sm = sign_mask(f);
        reflect_mask(t, sm);
        const C* k2 = reinterpret_cast<const C*>(smem_raw) + ko;
        block_mul<SYM>([&](int e) { return k2[e * HZ * KX]; }, t);
        reflect_mask(t, sm);
#pragma unroll
        for (int c = 0; c < 9; ++c) ra[c * NC] = t[c];
      }
    }
    __syncthreads();
    // (4) inverse transform; thread b keeps the layers n = S m + b < N_z
    if (lact && o >= 0) {
      if constexpr (S == 1) {
#pragma unroll
        for (int k = 0; k < LZ; ++k) v[k] = tile[k * P + l];
      } else {
        // b = 0: X[k] + X[k + Lz/2]; b = 1: W^{-k} (X[k] - X[k + Lz/2]) (branch free:
        // the two threads of a line are adjacent lanes)
        const T sg = b ? (T)-1 : (T)1;
#pragma unroll
        for (int k = 0; k < LH; ++k) {
          const C a = tile[k * P + l], c = tile[(k + LH) * P + l];
          const C w = b ? ctw_t<LZ, C>(k) : mk<T>((T)1, (T)0);
          v[k] = conj_mul(w, mk<T>(fma(sg, c.x, a.x), fma(sg, c.y, a.y)));
        }
      }
      fft_reg_c<LH, +1>(v);
#pragma unroll
      for (int m = 0; m < LH; ++m) {
        const int n = S * m + b;
        if ((S == 2 || m < LZ / 2) && n < g.Nz) W[o + n * plane] = v[m];
      }
    }
  }
  // a wait that ran out: the bulk copy still lands before the block's shared memory is
  // given back
  if (tid == 0 && !kready) {
    for (long long it = 0; it < ZP_WAIT_LIMIT && !kready; ++it) kready = zp_try_wait(kbar_a, 0u);
    if (!kready && status) atomicExch(status, 1);
  }
}

}  // namespace msc
