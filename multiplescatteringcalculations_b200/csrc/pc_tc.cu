// Near-field stencil on the 5th-generation tensor cores (tcgen05): the complex64
// preconditioner layer with BF16 weights and activations, FP32 accumulation.
//
// One layer y_a(v) = sum_o sum_b G[o][a][b] tau_b(v - o), tau = T0 (s x), is computed
// per tile of 128 voxels as real GEMMs accumulated in tensor memory, Y (128 x 32) +=
// A B^T, with the complex products in real form: B rows n = 2 a + {0: re, 1: im},
// (re, re) = G.re, (re, im) = -G.im, (im, re) = G.im, (im, im) = G.re, and the entries
// the mirror symmetry of the lattice sets to zero left at zero (18 of 32 rows used).
//
// The operands are not materialised per offset. The tile is 16 x-lines of 8 voxels along
// y in one layer z; tau of a halo plane (18 x 10 voxels) is stored in shared memory as
// BF16 in the K-major no-swizzle layout (core matrices of 8 rows x 16 bytes, row = halo
// voxel, y fastest, 160 bytes = one halo line between 8-row groups), so an operand that
// reads the tile's voxels shifted by (dx, dy) is the plane's descriptor started
// (1 - dx) 10 + (1 - dy) rows later. Each row holds 4 K chunks of 8 BF16:
//   chunks 0-1: tau_0..tau_7 of the row                (one MMA per offset: 27 MMAs)
//   chunk 2:    tau_8 of the rows r, r + 1, r + 2       (y neighbours)
//   chunk 3:    tau_8 of the rows r + 10, r + 11, r + 12 (the next x-line)
// so two MMAs per dz (started at shifts 0 and 20 rows) cover the 9 (dx, dy) taps of
// DOF 8: 33 MMAs (M 128, N 32, K 16) per layer instead of 54.
//
// A block walks a column of tiles through zc consecutive layers; its halo planes live in
// a ring of 4 slots, each plane staged once and read by three layers. Warp 8 allocates
// the tensor memory, copies the layer's packed weights (33 tiles of 1 KB, built on the
// host when the blocks change) into shared memory with one bulk copy, and issues the MMAs
// of layer j into accumulator j & 1 once the plane j + 1 is staged and the epilogue of
// layer j - 2 has drained that accumulator (mbarrier staged[j & 1], 256 arrivals). Warps
// 0-7 stage planes and run the epilogue: for layer j - 1 they prefetch acc (or x), wait
// for its MMAs (mbarrier done[(j - 1) & 1], committed by the MMA warp), read the
// accumulator (tcgen05.ld; warps w and w + 4 share the lane quadrant w & 3 and split the
// 9 DOFs) and write h = y and acc = c0 s x + ch y or acc += ch y; then they stage plane
// j + 2 into the slot the MMAs of layer j - 1 released.
//
// Every wait on an mbarrier is bounded (the plan's wait limit, msc_plan_set_wait_limit):
// when one runs out the kernel records a timeout in the plan's status word and sets the
// block's abort flag, after which no warp issues or waits for further work; the MMA warp
// then drains the weights' bulk copy and its last commits (with the fixed limit) before
// the tensor memory is freed and the block exits.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "mv_common.cuh"
#include "pc.cuh"

namespace msc {

namespace {

constexpr int TV_TX = 16, TV_TY = 8, TV_M = TV_TX * TV_TY;                  // 128 voxel rows
constexpr int TV_HX = TV_TX + 2, TV_HY = TV_TY + 2, TV_PROWS = TV_HX * TV_HY;  // 180 halo rows
constexpr int TV_STAGE = 256;                 // warps 0-7: staging and epilogue
constexpr int TV_THREADS = TV_STAGE + 32;     // warp 8: tensor memory, weights, MMA issue
constexpr int TV_LBO_A = TV_PROWS * 16;       // bytes between the K chunks of a plane
constexpr int TV_SBO_A = TV_HY * 16;          // bytes between 8-row groups (x-lines)
constexpr int TV_PLANE = 4 * TV_LBO_A;        // one staged plane: 4 K chunks of 8 BF16
constexpr int TV_RING = 4;
constexpr int TV_N = 32;
constexpr int TV_BTILE = TV_N * 16 * 2;       // one weight tile: 32 rows x 16 BF16
constexpr int TV_LBO_B = (TV_N / 8) * 128;
constexpr int TV_TILES = NF_OFFS + 6;         // 27 offsets (DOF 0-7) + 2 per dz (DOF 8)
constexpr int TV_B_BYTES = TV_TILES * TV_BTILE;
static_assert(TV_B_BYTES == NF_TC_LAYER_BYTES, "packed layer size");
static_assert(TV_M == 128, "one accumulator lane per voxel row");
constexpr int TV_ALIGN = 1024;                // operand base alignment in the shared window
constexpr int TV_T8_BYTES = TV_RING * TV_PROWS * 8;
// + 64: mbarriers done[2], weights, staged[2] (40 bytes), the tensor-memory address and
// the abort flag (8 bytes), the never-completed mbarrier (8 bytes)
constexpr size_t TV_SMEM = TV_ALIGN + (size_t)TV_B_BYTES + (size_t)TV_RING * TV_PLANE + TV_T8_BYTES + 64;
constexpr long long TV_WAIT_LIMIT = 1ll << 22;  // mbarrier polls before a timeout is recorded

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
constexpr uint32_t TV_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TV_N >> 3) << 17) |
                              ((uint32_t)(TV_M >> 4) << 24);

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

// bounded wait of the pipeline (`limit` polls, the plan's setting); on a timeout the
// status word is set and the wait is tried once more
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t addr, uint32_t phase, int* status, long long limit) {
  bool ok = false;
  for (long long it = 0; it < limit && !ok; ++it) ok = mbar_try_wait(addr, phase);
  if (!ok) {
    if (status) atomicExch(status, 1);
    for (long long it = 0; it < limit && !ok; ++it) ok = mbar_try_wait(addr, phase);
  }
  return ok;
}

// the drain before the block releases its tensor memory and exits: wait, with the fixed
// limit TV_WAIT_LIMIT whatever the pipeline's limit, for an asynchronous operation of this
// block (the weights' bulk copy, the MMAs of a commit) to complete
__device__ __forceinline__ void mbar_drain(uint32_t addr, uint32_t phase, int* status) {
  bool ok = false;
  for (long long it = 0; it < TV_WAIT_LIMIT && !ok; ++it) ok = mbar_try_wait(addr, phase);
  if (!ok && status) atomicExch(status, 1);
}

struct TvTile {
  int x0, y0, z0, zc;
};

// One halo row of a plane: the 9 components of x and the 4 T0 scalars at its voxel.
struct HaloRow {
  float2 xv[9], t[4];
  bool in;
};

__device__ __forceinline__ void load_row(HaloRow& hr, int r, int z, const TvTile& tl, const float2* __restrict__ x,
                                         const float2* __restrict__ t4, const Geo& g) {
  const int hy = r % TV_HY, hx = r / TV_HY;
  const int xx = tl.x0 + hx - 1, y = tl.y0 + hy - 1;
  hr.in = z >= 0 && z < g.Nz && xx >= 0 && xx < g.M && y >= 0 && y < g.M;
  if (hr.in) {
    const int site = (z * g.M + xx) * g.M + y;
#pragma unroll
    for (int c = 0; c < 9; ++c) hr.xv[c] = x[(size_t)c * g.nsite + site];
#pragma unroll
    for (int c = 0; c < 4; ++c) hr.t[c] = t4[(size_t)c * g.nsite + site];
  }
}

// tau = T0 (s x) of the row: tau_0..tau_7 as BF16 into chunks 0-1 of its slot, tau_8
// into the slot's tau_8 line t8
__device__ __forceinline__ void store_row01(const HaloRow& hr, unsigned char* ring, int slot, int r, float s,
                                            float2* t8) {
  float2 v[9];
  if (hr.in) {
    const float2 tr = hr.xv[3] + hr.xv[4] + hr.xv[5];
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = s * (hr.t[0] * hr.xv[c]);
#pragma unroll
    for (int c = 3; c < 6; ++c) v[c] = s * (hr.t[1] * tr + hr.t[2] * hr.xv[c]);
#pragma unroll
    for (int c = 6; c < 9; ++c) v[c] = s * (hr.t[3] * hr.xv[c]);
  } else {
#pragma unroll
    for (int c = 0; c < 9; ++c) v[c] = make_float2(0.f, 0.f);
  }
  uint4* q = reinterpret_cast<uint4*>(ring + slot * TV_PLANE + r * 16);
  q[0] = make_uint4(pack_bf16(v[0].x, v[0].y), pack_bf16(v[1].x, v[1].y), pack_bf16(v[2].x, v[2].y),
                    pack_bf16(v[3].x, v[3].y));
  q[TV_LBO_A / 16] = make_uint4(pack_bf16(v[4].x, v[4].y), pack_bf16(v[5].x, v[5].y), pack_bf16(v[6].x, v[6].y),
                                pack_bf16(v[7].x, v[7].y));
  t8[r] = v[8];
}

__device__ __forceinline__ uint32_t t8_at(const float2* t8, int r) {
  const float2 v = r < TV_PROWS ? t8[r] : make_float2(0.f, 0.f);
  return pack_bf16(v.x, v.y);
}

// chunks 2-3 of row r: tau_8 of the rows r, r + 1, r + 2 and r + 10, r + 11, r + 12
__device__ __forceinline__ void store_row23(unsigned char* ring, int slot, int r, const float2* t8) {
  uint4* q = reinterpret_cast<uint4*>(ring + slot * TV_PLANE + r * 16);
  q[2 * TV_LBO_A / 16] = make_uint4(t8_at(t8, r), t8_at(t8, r + 1), t8_at(t8, r + 2), 0u);
  q[3 * TV_LBO_A / 16] = make_uint4(t8_at(t8, r + TV_HY), t8_at(t8, r + TV_HY + 1), t8_at(t8, r + TV_HY + 2), 0u);
}

// barrier of the 8 staging warps only (the MMA warp does not take part)
__device__ __forceinline__ void stage_bar() { asm volatile("bar.sync 1, %0;\n" ::"n"(TV_STAGE) : "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t ad, uint64_t bd, uint32_t accum) {
  const uint32_t zm = 0;  // disable-output-lane mask: all lanes written
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
      "l"(ad), "l"(bd), "r"(TV_IDESC), "r"(accum), "r"(zm), "r"(zm), "r"(zm), "r"(zm)
      : "memory");
}

// The 33 MMAs of one layer into accumulator d. dA[dz + 1]: descriptor of chunk 0 of the
// plane of layer z - dz. The start address field is the low 14 bits of a descriptor
// (address >> 4) and stays below 2^14 here, so byte offsets >> 4 are added to it.
__device__ __forceinline__ void issue_layer(uint32_t d, const uint64_t (&dA)[3], uint64_t dB) {
#pragma unroll
  for (int o = 0; o < NF_OFFS; ++o) {
    const int dz = o / 9 - 1, dx = (o / 3) % 3 - 1, dy = o % 3 - 1;
    mma_bf16(d, dA[dz + 1] + (uint64_t)((((1 - dx) * TV_HY + (1 - dy)) * 16) >> 4),
             dB + (uint64_t)((o * TV_BTILE) >> 4), o > 0 ? 1u : 0u);
  }
#pragma unroll
  for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
    for (int part = 0; part < 2; ++part)
      mma_bf16(d, dA[dz + 1] + (uint64_t)(((part ? 2 * TV_HY * 16 : 0) + 2 * TV_LBO_A) >> 4),
               dB + (uint64_t)(((NF_OFFS + 2 * (dz + 1) + part) * TV_BTILE) >> 4), 1u);
}

__device__ __forceinline__ void mbar_arrive(uint32_t addr) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(addr) : "memory");
}

__global__ void __launch_bounds__(TV_THREADS, 2)
    k_nf_tc(const float2* __restrict__ x, const double* scale, const float2* __restrict__ t4, float2* __restrict__ h,
            float2* __restrict__ acc, float2 ch, float2 c0, int init, const uint4* __restrict__ Bg, Geo g, int zc,
            const int* done, int* status, long long wait_limit, int inject_wait) {
  // Launched as a programmatic dependent of the previous layer: everything up to
  // pdl_wait() (barrier set-up, tensor-memory allocation, the bulk copy of this layer's
  // weights, which no kernel writes) overlaps the previous kernel's tail; the halo
  // planes, x, acc, the scale and the done flag are read only after it.
  // The operands start on a 1024-byte boundary of the shared address space (with a 128-byte
  // static block ahead of the dynamic window, the MMA read its operands 16 bytes before
  // their start).
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t raw_a = (uint32_t)__cvta_generic_to_shared(smem_raw);
  unsigned char* Bs = smem_raw + (((raw_a + (uint32_t)TV_ALIGN - 1) & ~((uint32_t)TV_ALIGN - 1)) - raw_a);
  unsigned char* ring = Bs + TV_B_BYTES;
  float2* t8 = reinterpret_cast<float2*>(ring + TV_RING * TV_PLANE);  // [4][180]
  // mbarriers: done[2] (MMAs of a layer), weights, staged[2] (256 arrivals)
  uint64_t* mbar = reinterpret_cast<uint64_t*>(ring + TV_RING * TV_PLANE + TV_T8_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(mbar + 5) + 1;
  // an mbarrier that nothing arrives at: the wait on it that inject_wait asks for runs
  // out (the plan's failure-path test)
  const uint32_t mb_never = (uint32_t)__cvta_generic_to_shared(mbar + 6);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t mb = (uint32_t)__cvta_generic_to_shared(mbar);
  const uint32_t mb_done = mb, mb_w = mb + 16u, mb_staged = mb + 24u;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb_done) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb_done + 8u) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb_w) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mb_staged), "n"(TV_STAGE) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mb_staged + 8u), "n"(TV_STAGE) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb_never) : "memory");
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 8) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot), "r"(2 * TV_N)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  __syncthreads();
  const uint32_t b_a = (uint32_t)__cvta_generic_to_shared(Bs), ring_a = (uint32_t)__cvta_generic_to_shared(ring);
  // tile column and chunk of layers
  const int nty = (g.M + TV_TY - 1) / TV_TY, ntx = (g.M + TV_TX - 1) / TV_TX;
  const int col = blockIdx.x % (nty * ntx), chunk = blockIdx.x / (nty * ntx);
  TvTile tl;
  tl.y0 = (col % nty) * TV_TY;
  tl.x0 = (col / nty) * TV_TX;
  tl.z0 = chunk * zc;
  tl.zc = min(zc, g.Nz - tl.z0);
  if (warp == 8 && lane == 0) {
    // the layer's packed weights: one bulk copy into shared memory, completed on mb_w
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mb_w), "r"(TV_B_BYTES)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(b_a),
        "l"(Bg), "r"(TV_B_BYTES), "r"(mb_w)
        : "memory");
  }
  pdl_wait();
  pdl_trigger();
  if (done && *done) {
    // nothing to compute: the weights' copy lands before the shared memory and the
    // tensor memory are given back
    if (warp == 8 && lane == 0) mbar_drain(mb_w, 0u, status);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp == 8)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(*tmem_slot), "r"(2 * TV_N)
                   : "memory");
    return;
  }
  const float s = scale ? (float)(*scale) : 1.f;
  // planes of the layers z0 - 1, z0, z0 + 1 (plane p of the chunk, layer z0 + p, lives in
  // slot (p + 1) & 3), staged by all 288 threads (the MMA warp has nothing to issue yet),
  // each thread's rows' loads in flight at once
  constexpr int NR = (3 * TV_PROWS + TV_THREADS - 1) / TV_THREADS;
  {
    HaloRow hr[NR];
#pragma unroll
    for (int i = 0; i < NR; ++i) {
      const int q = tid + i * TV_THREADS;
      if (q < 3 * TV_PROWS) load_row(hr[i], q % TV_PROWS, tl.z0 + q / TV_PROWS - 1, tl, x, t4, g);
    }
#pragma unroll
    for (int i = 0; i < NR; ++i) {
      const int q = tid + i * TV_THREADS;
      if (q < 3 * TV_PROWS) store_row01(hr[i], ring, q / TV_PROWS, q % TV_PROWS, s, t8 + (q / TV_PROWS) * TV_PROWS);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    const int q = tid + i * TV_THREADS;
    if (q < 3 * TV_PROWS) store_row23(ring, q / TV_PROWS, q % TV_PROWS, t8 + (q / TV_PROWS) * TV_PROWS);
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (warp == 8) {
    if (lane == 0) {
      bool ok = mbar_wait_bounded(mb_w, 0u, status, wait_limit);  // the weights have landed
      if (ok && inject_wait) ok = mbar_wait_bounded(mb_never, 0u, status, wait_limit);
      const uint64_t dB = umma_desc(b_a, TV_LBO_B, 128);
      int issued = 0;
      for (int j = 0; j < tl.zc && ok && !*abort_flag; ++j) {
        // plane j + 1 staged and accumulator j & 1 drained: the staging warps' pass j - 1
        if (j >= 1)
          ok = mbar_wait_bounded(mb_staged + (uint32_t)(((j - 1) & 1) * 8), (uint32_t)(((j - 1) >> 1) & 1), status,
                                 wait_limit);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        uint64_t dA[3];
#pragma unroll
        for (int i = 0; i < 3; ++i)  // plane of layer z0 + j - (i - 1) in slot (j - i + 2) & 3
          dA[i] = umma_desc(ring_a + (uint32_t)(((j - i + 2) & 3) * TV_PLANE), TV_LBO_A, TV_SBO_A);
        issue_layer(tmem + (uint32_t)((j & 1) * TV_N), dA, dB);
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         mb_done + (uint32_t)((j & 1) * 8))
                     : "memory");
        issued = j + 1;
      }
      if (!ok) *abort_flag = 1;
      // Drain (a no-op unless a wait ran out): the weights' bulk copy has landed and the
      // MMAs of the last commit on each accumulator have completed before the tensor
      // memory is released and the block's shared memory is given back. Layer j's commit
      // is phase j >> 1 of done[j & 1], the newest on that barrier for the last two layers.
      mbar_drain(mb_w, 0u, status);
      for (int j = std::max(0, issued - 2); j < issued; ++j)
        mbar_drain(mb_done + (uint32_t)((j & 1) * 8), (uint32_t)((j >> 1) & 1), status);
    }
    __syncwarp();
  } else {
    // warps w and w + 4 read the lane quadrant w & 3: voxel row m, DOFs 0-4 (columns 0-9)
    // or 5-8 (columns 10-17)
    const int m = (warp & 3) * 32 + lane, half = warp >> 2;
    const int xx = tl.x0 + (m >> 3), yy = tl.y0 + (m & 7);
    const bool mine = xx < g.M && yy < g.M;
    const int a0 = half ? 5 : 0, na = half ? 4 : 5;
    for (int j = 0; j <= tl.zc; ++j) {
      const bool stage = j + 2 <= tl.zc;
      HaloRow hr;
      if (stage && tid < TV_PROWS) load_row(hr, tid, tl.z0 + j + 2, tl, x, t4, g);
      if (j >= 1) {
        const int jp = j - 1;
        const int site = ((tl.z0 + jp) * g.M + xx) * g.M + yy;
        float2 pre[5];
#pragma unroll
        for (int i = 0; i < 5; ++i) {
          pre[i] = make_float2(0.f, 0.f);
          if (mine && i < na) {
            const size_t e = (size_t)(a0 + i) * g.nsite + site;
            pre[i] = init ? x[e] : acc[e];
          }
        }
        bool ok = !*abort_flag;
        if (ok)
          ok = mbar_wait_bounded(mb_done + (uint32_t)((jp & 1) * 8), (uint32_t)((jp >> 1) & 1), status, wait_limit);
        if (!ok) *abort_flag = 1;
        if (__all_sync(0xffffffffu, ok)) {
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          uint32_t r[10];
          const uint32_t ta = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((jp & 1) * TV_N);
          if (half == 0) {
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(ta));
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];\n" : "=r"(r[8]), "=r"(r[9]) : "r"(ta + 8u));
          } else {
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(ta + 10u));
            r[8] = r[9] = 0u;
          }
          asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
          if (mine) {
#pragma unroll
            for (int i = 0; i < 5; ++i) {
              if (i >= na) break;
              const float2 out = make_float2(__uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1]));
              const size_t e = (size_t)(a0 + i) * g.nsite + site;
              if (h) h[e] = out;
              acc[e] = init ? c0 * (s * pre[i]) + ch * out : pre[i] + ch * out;
            }
          }
        }
      }
      if (stage) {
        // plane j + 2 (read by the MMAs of layer z0 + j + 1) into the slot the MMAs of
        // layer z0 + j - 1 released (slot 3 is free at j = 0)
        const int slot = (j + 3) & 3;
        if (tid < TV_PROWS) store_row01(hr, ring, slot, tid, s, t8 + slot * TV_PROWS);
        stage_bar();
        if (tid < TV_PROWS) store_row23(ring, slot, tid, t8 + slot * TV_PROWS);
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      mbar_arrive(mb_staged + (uint32_t)((j & 1) * 8));
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 8)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(2 * TV_N) : "memory");
}

inline uint16_t bf16_bits(__nv_bfloat16 v) {
  uint16_t u;
  std::memcpy(&u, &v, 2);
  return u;
}

inline void put_b(uint16_t* out, int t, int n, int kl, uint16_t v) {
  const int kc = kl / 8;
  out[((size_t)t * TV_BTILE + (size_t)(kc * (TV_N / 8) + n / 8) * 128 + (size_t)(n % 8) * 16 + (size_t)(kl % 8) * 2) /
      2] = v;
}

// real form of G[o][a][b] into rows 2 a, 2 a + 1 of tile t at K columns kre (re input)
// and kre + 1 (im input)
inline void put_block(uint16_t* out, int t, const __nv_bfloat162* G16, int o, int a, int b, int kre) {
  const int dz = o / 9 - 1, dx = (o / 3) % 3 - 1, dy = o % 3 - 1;
  const int zm = (dx == 0 ? 1 : 0) | (dy == 0 ? 2 : 0) | (dz == 0 ? 4 : 0);
  if ((dof_parity(a) ^ dof_parity(b)) & zm) return;  // zero by symmetry
  const __nv_bfloat162 gv = G16[o * 81 + a * 9 + b];
  const uint16_t re = bf16_bits(gv.x), im = bf16_bits(gv.y);
  put_b(out, t, 2 * a, kre, re);
  put_b(out, t, 2 * a, kre + 1, (uint16_t)(im ^ 0x8000u));
  put_b(out, t, 2 * a + 1, kre, im);
  put_b(out, t, 2 * a + 1, kre + 1, re);
}

}  // namespace

void nf_tc_pack_layer(const __nv_bfloat162* G16, uint16_t* out) {
  std::memset(out, 0, NF_TC_LAYER_BYTES);
  // tile o: DOFs 0-7 of offset o, K column 2 b + {re, im}
  for (int o = 0; o < NF_OFFS; ++o)
    for (int a = 0; a < 9; ++a)
      for (int b = 0; b < 8; ++b) put_block(out, o, G16, o, a, b, 2 * b);
  // tiles 27 + 2 (dz + 1) + part: DOF 8 of the taps (dx, dy = 1 - e), e = 0..2, read from
  // K chunk c (0: chunk 2 of the row, 1: chunk 3) at K column 8 c + 2 e + {re, im};
  // part 0: dx = +1 (c = 0) and dx = 0 (c = 1); part 1 (20 rows on): dx = -1 (c = 0)
  for (int dz = -1; dz <= 1; ++dz)
    for (int part = 0; part < 2; ++part)
      for (int c = 0; c < 2; ++c) {
        if (part == 1 && c == 1) continue;
        const int dx = part == 0 ? (c == 0 ? 1 : 0) : -1;
        for (int e = 0; e < 3; ++e) {
          const int o = ((dz + 1) * 3 + dx + 1) * 3 + (1 - e) + 1;
          for (int a = 0; a < 9; ++a) put_block(out, NF_OFFS + 2 * (dz + 1) + part, G16, o, a, 8, 8 * c + 2 * e);
        }
      }
}

int launch_nf_tc(msc_plan* pl, const float2* x, const double* scale, const float2* t4, float2* h, float2* acc,
                 float2 ch, float2 c0, int init, const void* Bpacked, const int* done) {
  const Geo& g = pl->g;
  const int ncol = ((g.M + TV_TY - 1) / TV_TY) * ((g.M + TV_TX - 1) / TV_TX);
  // layers per block: at most two blocks per SM, one wave (a partial second wave of
  // shorter blocks measured slower: 128 x 128 x 16, 384 blocks 173 us against 256 blocks
  // 147 us per degree-4 application)
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    MSC_CUDA(cudaGetDevice(&dev));
    MSC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  const int nzc = std::min(g.Nz, std::max(1, (2 * sms) / ncol));
  const int zc = (g.Nz + nzc - 1) / nzc;
  const int nb = ncol * ((g.Nz + zc - 1) / zc);
  MSC_CUDA(prep_kernel((const void*)k_nf_tc));
  int* status = (int*)pl->status.p;
  const long long limit = pl->wait_limit > 0 ? pl->wait_limit : TV_WAIT_LIMIT;
  const uint4* Bg = (const uint4*)Bpacked;
  Geo gg = g;
  int zcc = zc, inj = pl->inject_wait;
  long long lim = limit;
  void* args[] = {(void*)&x,  (void*)&scale, (void*)&t4,     (void*)&h,      (void*)&acc, (void*)&ch, (void*)&c0,
                  (void*)&init, (void*)&Bg,  (void*)&gg,     (void*)&zcc,    (void*)&done, (void*)&status,
                  (void*)&lim, (void*)&inj};
  MSC_CUDA(launch_pdl((const void*)k_nf_tc, dim3((unsigned)nb), dim3(TV_THREADS), args, TV_SMEM, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}

}  // namespace msc
