// Near-field stencil on the 5th-generation tensor cores (tcgen05): the complex64
// preconditioner layer with BF16 weights (the form the learned network is trained in).
//
// One layer y_a(v) = sum_o sum_b G[o][a][b] tau_b(v - o), tau = T0 (s x), is a dense
// contraction once written as a real GEMM over a tile of 128 voxels:
//   Y (128 x 32) = A (128 x 496) B^T (496 x 32),
//   A[v][k]  = tau_b(v - o).re / .im            k = 2 (9 o + b) + {0, 1}   (486 used, 496 padded)
//   B[n][k]  rows n = 2 a + {0: re, 1: im} of the complex product   (18 used, 32 padded)
//            (re, re) = G.re, (re, im) = -G.im, (im, re) = G.im, (im, im) = G.re,
// with the entries the lattice's mirror symmetry sets to zero masked out of B. The block
// stages tau on the tile plus a one-voxel halo in shared memory (FP32), writes A and B
// as BF16 in the K-major no-swizzle layout of the tensor core (core matrices of 8 rows x
// 16 bytes; 8-row groups 128 bytes apart; the two 8-element K chunks of one MMA step
// LBO bytes apart), and one thread issues the 31 MMA steps (M 128, N 32, K 16) into a
// 32-column FP32 accumulator in tensor memory. A commit to an mbarrier signals their
// completion; every thread then reads its voxel's row from tensor memory (tcgen05.ld)
// and applies the layer's epilogue (h = y; acc = c0 s x + ch y or acc += ch y), as the
// CUDA-core kernel (pc.cu) does. Accumulation is FP32; tau enters as BF16.
//
// The wait on the mbarrier is bounded: when it runs out the kernel records a timeout
// in the plan's status word, waits once more (bounded) and frees its tensor memory.
#include <cuda_bf16.h>

#include <cstdint>

#include "mv_common.cuh"
#include "pc.cuh"

namespace msc {

namespace {

constexpr int TC_TZ = 2, TC_TX = 4, TC_TY = 16, TC_M = TC_TZ * TC_TX * TC_TY;  // 128 voxels
constexpr int TC_HZ = TC_TZ + 2, TC_HX = TC_TX + 2, TC_HY = TC_TY + 2, TC_HALO = TC_HZ * TC_HX * TC_HY;
constexpr int TC_K = 496, TC_KC = TC_K / 8, TC_KUSED = 2 * NF_OFFS * 9;  // 486
constexpr int TC_N = 32, TC_NUSED = 18;
constexpr int TC_STEPS = TC_K / 16;
constexpr int TC_A_BYTES = TC_M * TC_K * 2;   // 126976
constexpr int TC_B_BYTES = TC_N * TC_K * 2;   // 31744
constexpr int TC_LBO_A = (TC_M / 8) * 128;    // bytes between K chunks of A
constexpr int TC_LBO_B = (TC_N / 8) * 128;
constexpr size_t TC_TAU_BYTES = sizeof(float2) * 9 * TC_HALO;
constexpr size_t TC_ALIGN = 1024;  // operand base alignment in the shared window
constexpr size_t TC_SMEM = TC_ALIGN + (size_t)TC_A_BYTES + TC_B_BYTES + TC_TAU_BYTES + 16;
constexpr long long TC_WAIT_LIMIT = 1ll << 22;  // mbarrier polls before a timeout is recorded

__device__ __forceinline__ bool tc_allowed(int o, int a, int b) {
  const int dz = o / 9 - 1, dx = (o / 3) % 3 - 1, dy = o % 3 - 1;
  const int zm = (dx == 0 ? 1 : 0) | (dy == 0 ? 2 : 0) | (dz == 0 ? 4 : 0);
  return ((dof_parity(a) ^ dof_parity(b)) & zm) == 0;
}

// byte offset of element (row r, k) in a K-major no-swizzle operand with R rows
template <int R>
__device__ __forceinline__ uint32_t umma_off(int r, int kc) {
  return (uint32_t)((kc * (R / 8) + r / 8) * 8 + r % 8) * 16u;
}

// shared-memory matrix descriptor (K-major, no swizzle): start >> 4 in bits 0-13, LBO >> 4
// in bits 16-29, SBO >> 4 in bits 32-45, version 1 in bits 46-47, layout type 0
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1),
// both K-major, N >> 3 in bits 17-22, M >> 4 in bits 24-28
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t phase) {
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

__global__ void __launch_bounds__(TC_M, 1)
    k_nf_tc(const float2* __restrict__ x, const double* scale, const float2* __restrict__ t4, float2* __restrict__ h,
            float2* __restrict__ acc, float2 ch, float2 c0, int init, const __nv_bfloat162* __restrict__ G16, Geo g,
            const int* done, int* status) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  // The operands start on a 1024-byte boundary of the shared address space (with a 128-byte
  // static block ahead of the dynamic window, the MMA read both operands 16 bytes before
  // their start), and the mbarrier and the tensor-memory slot follow tau.
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t raw_a = (uint32_t)__cvta_generic_to_shared(smem_raw);
  unsigned char* As = smem_raw + (((raw_a + (uint32_t)TC_ALIGN - 1) & ~((uint32_t)TC_ALIGN - 1)) - raw_a);
  unsigned char* Bs = As + TC_A_BYTES;
  float2* tau = reinterpret_cast<float2*>(Bs + TC_B_BYTES);  // [9][TC_HALO]
  uint64_t& mbar = *reinterpret_cast<uint64_t*>(Bs + TC_B_BYTES + TC_TAU_BYTES);
  uint32_t& tmem_slot = *reinterpret_cast<uint32_t*>(Bs + TC_B_BYTES + TC_TAU_BYTES + 8);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t mbar_a = (uint32_t)__cvta_generic_to_shared(&mbar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(&tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot), "r"(TC_N)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  // tile origin
  const int nby = (g.M + TC_TY - 1) / TC_TY, nbx = (g.M + TC_TX - 1) / TC_TX;
  const int by = blockIdx.x % nby, bx = (blockIdx.x / nby) % nbx, bz = blockIdx.x / (nby * nbx);
  const int y0 = by * TC_TY, x0 = bx * TC_TX, z0 = bz * TC_TZ;
  const float s = scale ? (float)(*scale) : 1.f;
  // tau = T0 (s x) on the tile and its halo (zero outside the slab)
  for (int i = tid; i < TC_HALO; i += TC_M) {
    const int hy = i % TC_HY, hx = (i / TC_HY) % TC_HX, hz = i / (TC_HY * TC_HX);
    const int z = z0 + hz - 1, xx = x0 + hx - 1, y = y0 + hy - 1;
    float2 v[9];
    if (z >= 0 && z < g.Nz && xx >= 0 && xx < g.M && y >= 0 && y < g.M) {
      const int site = (z * g.M + xx) * g.M + y;
      float2 xv[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) xv[c] = x[(size_t)c * g.nsite + site];
      const float2 tu = t4[site], tl = t4[(size_t)g.nsite + site], td = t4[(size_t)2 * g.nsite + site],
                   ts = t4[(size_t)3 * g.nsite + site];
      const float2 tr = xv[3] + xv[4] + xv[5];
#pragma unroll
      for (int c = 0; c < 3; ++c) v[c] = s * (tu * xv[c]);
#pragma unroll
      for (int c = 3; c < 6; ++c) v[c] = s * (tl * tr + td * xv[c]);
#pragma unroll
      for (int c = 6; c < 9; ++c) v[c] = s * (ts * xv[c]);
    } else {
#pragma unroll
      for (int c = 0; c < 9; ++c) v[c] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int c = 0; c < 9; ++c) tau[c * TC_HALO + i] = v[c];
  }
  // B (weights): TC_N rows x TC_KC chunks of 8
  for (int u = tid; u < TC_N * TC_KC; u += TC_M) {
    const int n = u % TC_N, kc = u / TC_N;
    const int a = n >> 1, rout = n & 1;
    uint32_t w[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      float f[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int k = kc * 8 + 2 * p + q;  // q = rin (k even: re input, odd: im input)
        float val = 0.f;
        if (n < TC_NUSED && k < TC_KUSED) {
          const int pair = k >> 1, o = pair / 9, b = pair % 9;
          if (tc_allowed(o, a, b)) {
            const float2 gv = __bfloat1622float2(G16[o * 81 + a * 9 + b]);
            val = rout == 0 ? (q == 0 ? gv.x : -gv.y) : (q == 0 ? gv.y : gv.x);
          }
        }
        f[q] = val;
      }
      w[p] = pack_bf16(f[0], f[1]);
    }
    *reinterpret_cast<uint4*>(Bs + umma_off<TC_N>(n, kc)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  __syncthreads();
  // A (activations): row m = voxel of the tile, TC_KC chunks of 8
  for (int u = tid; u < TC_M * TC_KC; u += TC_M) {
    const int m = u % TC_M, kc = u / TC_M;
    const int vy = m % TC_TY, vx = (m / TC_TY) % TC_TX, vz = m / (TC_TY * TC_TX);
    uint32_t w[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int pair = kc * 4 + p;  // (o, b): one complex value = two consecutive k
      float2 tv = make_float2(0.f, 0.f);
      if (pair < NF_OFFS * 9) {
        const int o = pair / 9, b = pair % 9;
        const int dz = o / 9 - 1, dx = (o / 3) % 3 - 1, dy = o % 3 - 1;
        const int hi = ((vz + 1 - dz) * TC_HX + (vx + 1 - dx)) * TC_HY + (vy + 1 - dy);
        tv = tau[b * TC_HALO + hi];
      }
      w[p] = pack_bf16(tv.x, tv.y);
    }
    *reinterpret_cast<uint4*>(As + umma_off<TC_M>(m, kc)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  // the generic-proxy writes of A and B become visible to the tensor core's async proxy
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;
  if (tid == 0) {
    const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(As), b0 = (uint32_t)__cvta_generic_to_shared(Bs);
    for (int st = 0; st < TC_STEPS; ++st) {
      const uint64_t ad = umma_desc(a0 + (uint32_t)st * 2u * TC_LBO_A, TC_LBO_A, 128);
      const uint64_t bd = umma_desc(b0 + (uint32_t)st * 2u * TC_LBO_B, TC_LBO_B, 128);
      const uint32_t accum = st > 0 ? 1u : 0u;
      const uint32_t z = 0;  // disable-output-lane mask: all lanes written
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "setp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
          "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(accum), "r"(z), "r"(z), "r"(z), "r"(z)
          : "memory");
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar_a)
                 : "memory");
  }
  // bounded wait for the MMAs
  bool ok = false;
  for (long long it = 0; it < TC_WAIT_LIMIT && !ok; ++it) ok = mbar_try_wait(mbar_a, 0);
  if (!ok) {
    if (status) atomicExch(status, 1);
    for (long long it = 0; it < TC_WAIT_LIMIT && !ok; ++it) ok = mbar_try_wait(mbar_a, 0);
  }
  ok = __syncthreads_and(ok) != 0;  // one decision for the block: the loads below are warp-collective
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  uint32_t r[32];
  if (ok) {
    const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(ta));
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(ta + 16u));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_N) : "memory");
  if (!ok) return;
  // epilogue: row m = tid is voxel (vz, vx, vy) of the tile
  const int vy = tid % TC_TY, vx = (tid / TC_TY) % TC_TX, vz = tid / (TC_TY * TC_TX);
  const int z = z0 + vz, xx = x0 + vx, y = y0 + vy;
  if (z >= g.Nz || xx >= g.M || y >= g.M) return;
  const int site = (z * g.M + xx) * g.M + y;
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    const float2 out = make_float2(__uint_as_float(r[2 * a]), __uint_as_float(r[2 * a + 1]));
    const size_t e = (size_t)a * g.nsite + site;
    if (h) h[e] = out;
    if (init) acc[e] = c0 * (s * x[e]) + ch * out;
    else acc[e] = acc[e] + ch * out;
  }
}

}  // namespace

int launch_nf_tc(msc_plan* pl, const float2* x, const double* scale, const float2* t4, float2* h, float2* acc,
                 float2 ch, float2 c0, int init, const __nv_bfloat162* G16, const int* done) {
  const Geo& g = pl->g;
  const int nb = ((g.M + TC_TY - 1) / TC_TY) * ((g.M + TC_TX - 1) / TC_TX) * ((g.Nz + TC_TZ - 1) / TC_TZ);
  MSC_CUDA(prep_kernel((const void*)k_nf_tc));
  int* status = (int*)pl->status.p;
  k_nf_tc<<<nb, TC_M, TC_SMEM, pl->stream>>>(x, scale, t4, h, acc, ch, c0, init, G16, g, done, status);
  ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}

}  // namespace msc
