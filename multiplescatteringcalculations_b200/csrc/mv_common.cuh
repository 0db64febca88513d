// Shared pieces of the matvec translation units.
#pragma once
#include <mutex>
#include <unordered_set>

#include "plan.cuh"

namespace msc {

// Reflection parity of the 9 DOF [u_z, u_x, u_y, e_zz, e_xx, e_yy, 2e_xy, 2e_zy,
// 2e_zx]: bit 0 odd under x -> -x, bit 1 under y -> -y, bit 2 under z -> -z.
__host__ __device__ constexpr int dof_parity(int c) {
  return c == 0 ? 4 : c == 1 ? 1 : c == 2 ? 2 : c < 6 ? 0 : c == 6 ? 3 : c == 7 ? 6 : 5;
}

// Lines per tile so that one tile row is 128 bytes: 16 (complex64) / 8 (complex128).
template <typename T> struct Tile { static constexpr int W = 128 / (int)sizeof(cx<T>); };

template <typename T> __device__ __forceinline__ T load_scale(const double* s) { return s ? (T)(*s) : (T)1; }

// Walks it = start, start + step, ... as (q, r) = (it / D, it % D) with one
// division at construction and additions afterwards.
struct QR {
  int q, r, dq, dr, D;
  __device__ __forceinline__ QR(int start, int step, int D_) : D(D_) {
    q = start / D_;
    r = start - q * D_;
    dq = step / D_;
    dr = step - dq * D_;
  }
  __device__ __forceinline__ void next() {
    q += dq;
    r += dr;
    if (r >= D) {
      r -= D;
      ++q;
    }
  }
};

// Allow the kernel the full dynamic shared memory and prefer shared memory over L1
// (these kernels stage everything in shared memory); done once per kernel.
inline cudaError_t prep_kernel(const void* fn) {
  static std::mutex mu;
  static std::unordered_set<const void*> seen;
  std::lock_guard<std::mutex> lk(mu);
  if (seen.count(fn)) return cudaSuccess;
  // dynamic limit = the device's opt-in maximum minus the kernel's static shared memory
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e == cudaSuccess) seen.insert(fn);
  return e;
}

// Fused z pass (mv_zbz.cuh). A block holds 9 components x 4 KX column slots
// (lines) of Lz points twice (ping-pong) plus the twiddles and, for an octant
// spectrum, the block's contiguous slice of the kernel spectrum.
constexpr int ZBZ_THREADS = 288;
constexpr int ZBZ_MAX_LINES = 144;
constexpr int ZBZ_SMEM_LIMIT = 227 * 1024 - 2048;  // opt-in maximum less the static tables

// Stored kernel-spectrum entry of element type T (complex, 8 or 16 bytes).
template <typename T> struct KEnt;
template <> struct KEnt<float> { using type = float2; };
template <> struct KEnt<double> { using type = double2; };
template <typename T> using kent = typename KEnt<T>::type;
__host__ __device__ inline float2 kent_pack(double2 v, float2*) { return make_float2((float)v.x, (float)v.y); }
__host__ __device__ inline double2 kent_pack(double2 v, double2*) { return v; }

struct ZbzLayout {
  int KX;       // kx per quadrant; 4 KX column slots per block, KX in {4, 2, 1}
  int NXC;      // kx chunks of the octant, ceil(Hx / KX)
  int CS;       // entries of one block's spectrum slice [e][kz][j]
  int ksm;      // 1: the slice is staged in shared memory
  size_t smem;  // dynamic shared memory of a block
};

// Layout for element type T. Preference: two blocks per SM with the slice in
// shared memory, then two blocks per SM reading the slice from global memory,
// then one block per SM. The octant spectrum of type T is stored blocked with
// this layout: slice (ky_o, xc) at ((ky_o * NXC + xc) * CS), entry (e, kz, j) at
// (e * Hz + kz) * KX + j, kx = xc * KX + j (zero beyond Hx).
template <typename T> constexpr ZbzLayout zbz_layout(int Lz, int Hz, int Hx, int E, bool oct) {
  const size_t es = sizeof(cx<T>);
  const size_t ek = sizeof(kent<T>);
  const int al = (int)(16 / ek);  // slices start 16-byte aligned
  auto tiles = [&](int kx) { return es * ((size_t)Lz + 2 * (size_t)Lz * (36 * kx + 1)); };
  auto make = [&](int kx, int ksm) {
    ZbzLayout L{};
    L.KX = kx;
    L.NXC = oct ? (Hx + kx - 1) / kx : 0;
    L.CS = oct ? (E * Hz * kx + al - 1) / al * al : 0;
    L.ksm = ksm;
    L.smem = tiles(kx) + (ksm ? ek * (size_t)L.CS : 0);
    return L;
  };
  const size_t two = (size_t)(ZBZ_SMEM_LIMIT / 2);
  if (oct)
    for (int kx = 4; kx >= 1; kx /= 2)
      if (make(kx, 1).smem <= two) return make(kx, 1);
  for (int kx = 4; kx >= 1; kx /= 2)
    if (make(kx, 0).smem <= two) return make(kx, 0);
  if (oct && make(1, 1).smem <= (size_t)ZBZ_SMEM_LIMIT) return make(1, 1);
  return make(1, 0);
}
template <typename T> inline ZbzLayout zbz_layout(const Geo& g, int E) {
  return zbz_layout<T>(g.Lz, g.Hz, g.Hx, E, g.oct != 0);
}
// entries (kent<T>) of the stored kernel spectrum of type T
template <typename T> inline size_t khat_elems_t(const Geo& g, int E) {
  if (!g.oct) return (size_t)E * g.Hz * g.Hy * g.Hx;
  const ZbzLayout L = zbz_layout<T>(g, E);
  return (size_t)g.Hy * L.NXC * L.CS;
}
// smallest shared memory of the fused z pass for complex128 (one block per SM)
inline size_t zbz_min_smem64(int Lz) { return sizeof(double2) * ((size_t)Lz + 2 * (size_t)Lz * 37); }

#define MSC_POW2_DISPATCH(pow2, CALL) \
  do {                                \
    if (pow2) { CALL(true); }         \
    else { CALL(false); }             \
  } while (0)

// Kernel launchers (one translation unit each).
template <typename T>
int launch_fft_contig(msc_plan* pl, const cx<T>* in, cx<T>* out, long long nlines, long long G, long long GS,
                      long long stride, int n_in, int n_out, const FftPlan1D& f, const cx<T>* tw, int dir,
                      const int* done);
template <typename T>
int launch_t0_fft_y(msc_plan* pl, const cx<T>* x, const double* scale, cx<T>* W, const cx<T>* tw, const int* done,
                    int nrhs);
// odd (two words, optional): mirror-symmetric input lines of length f.L stored for
// idx < n_in = f.L/2 + 1 only; idx >= n_in is read as s in[f.L - idx], s = -1 when bit
// blockIdx.z (the slab index s2, an entry of the G0 build) of the 128-bit mask is set.
template <typename T>
int launch_fft_strided(msc_plan* pl, const cx<T>* in, long long es, long long S1, long long S2, cx<T>* out,
                       long long eo, long long O1, long long O2, float2* out32, int ncol, int n1, int n2, int n_in,
                       int n_out, const FftPlan1D& f, const cx<T>* tw, int dir, const int* done,
                       const unsigned long long* odd = nullptr);
template <typename T>
int launch_zbz(msc_plan* pl, cx<T>* W, const int* done, int nrhs);
// the register form of the z pass (mv_zpass.cu); 1 = not applicable to the
// plan's shape (nothing launched), else a status
template <typename T>
int launch_zpass(msc_plan* pl, cx<T>* W, const int* done, int nrhs);
template <typename T>
int launch_fft_y_out(msc_plan* pl, const cx<T>* W, const cx<T>* x, const double* scale, cx<T>* y, const cx<T>* tw,
                     const int* done, int nrhs);

}  // namespace msc
