// Restarted GMRES(m) with CGS2 Arnoldi on the device, and the mixed-precision
// driver: complex64 inner solves inside FP64 iterative refinement.
//
// Replaces torch_gmres (tmnestor/MultipleScatteringCalculations
// cubic_scattering/torch_gmres.py:83-205) and the scipy.sparse.linalg.gmres call of
// compute_slab_scattering (slab_scattering.py:539-552). Differences by design:
//  * the Givens rotation is the unitary complex one, G = [[c, s], [-conj(s), c]],
//    c = |a|/r, s = (a/|a|) conj(b)/r (the reference's torch_gmres drops the
//    conjugates, which is not unitary for complex Hessenberg entries);
//  * restarted with a fixed basis of m+1 vectors; Hessenberg, rotations and the
//    least-squares solve are FP64 on the device;
//  * Krylov vectors are stored unnormalised with a per-vector FP64 scale
//    (V_i = s_i v_i), so normalisation costs no pass over memory;
//  * the host checks convergence one Arnoldi step behind the GPU: the kernels of
//    a step enqueued after convergence see the device `done` flag and return.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "pc.cuh"
#include "plan.cuh"

namespace msc {

template <typename T>
int launch_fft_contig(msc_plan* pl, const cx<T>* in, cx<T>* out, long long nlines, long long G, long long GS,
                      long long stride, int n_in, int n_out, const FftPlan1D& f, const cx<T>* tw, int dir,
                      const int* done);

struct GState {
  int done;       // cycle finished
  int converged;  // |g_{j+1}| <= tol_abs
  int status;     // msc_status of the cycle
  int k;          // columns in the least-squares solution
  int steps;      // Arnoldi steps run in the cycle (operator applications)
  double tol_abs; // target on |g_{j+1}|
  double beta;    // initial residual norm of the cycle
  double res;     // current residual estimate
  int counter[4]; // last-block reduction counters
};

struct GmresWork {
  int m = 0;
  size_t n = 0;
  DBuf V32, V64;          // (m+1) x n Krylov basis
  DBuf Z32, Z64;          // m x n preconditioned directions (flexible GMRES)
  DBuf x64, r64, ax64;    // FP64 iterate, residual, A x
  DBuf d32, r32;          // inner correction and right-hand side (complex64)
  DBuf state;             // GState
  DBuf hess;              // H[(m+1) x m], cs[m], sn[m], g[m+1], y[m], scale[m+1], h1[m+1], h2[m+1], nrm[2]
  DBuf part;              // partial sums [NB][33]
  GState* hstate = nullptr;  // pinned host mirror
  double* hd = nullptr;      // pinned scalar readback
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaEvent_t tev[2] = {nullptr, nullptr};  // timing of a cycle (preconditioner policy)
  // captured Arnoldi cycles, [precision][preconditioned]
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    int m = 0;
    bool cgs2 = false;
    int nrhs = 1;  // right-hand sides of the matvec the graph holds
    uint64_t gen = 0;
    int warm = 0;  // cycles of this kind run uncaptured (kernel attributes set, buffers allocated)
  } graph[2][2];
};

constexpr int NB = 592;     // blocks of the multi-vector kernels (4 per SM)
constexpr int NTH = 256;
constexpr int PLD = 33;     // partials leading dimension (<= 32 vectors + norm)

struct HessPtr {
  double2* H;
  double* cs;
  double2* sn;
  double2* g;
  double2* y;
  double* scale;
  double2* h1;
  double2* h2;
  double2* nrm;   // [4]: 0 = GMRES cycle norms, 1 = outer residual
};

static HessPtr hess_ptrs(GmresWork* gw) {
  const int m = gw->m;
  char* p = (char*)gw->hess.p;
  HessPtr h;
  h.nrm = (double2*)p; p += sizeof(double2) * 4;
  h.H = (double2*)p; p += sizeof(double2) * (size_t)(m + 1) * m;
  h.sn = (double2*)p; p += sizeof(double2) * m;
  h.g = (double2*)p; p += sizeof(double2) * (m + 1);
  h.y = (double2*)p; p += sizeof(double2) * m;
  h.h1 = (double2*)p; p += sizeof(double2) * (m + 1);
  h.h2 = (double2*)p; p += sizeof(double2) * (m + 1);
  h.cs = (double*)p; p += sizeof(double) * m;
  h.scale = (double*)p; p += sizeof(double) * (m + 1);
  return h;
}
static size_t hess_bytes(int m) {
  return sizeof(double2) * ((size_t)(m + 1) * m + m + (m + 1) + m + 2 * (m + 1) + 4) + sizeof(double) * (m + m + 1);
}

// Row i of the per-block partials summed over the nb blocks in a fixed order: lane l
// takes blocks l, l + 32, ... and the warp adds the lanes by shuffles. All of a lane's
// loads (through L2, ld.global.cg, which sees the other blocks' fenced stores) are in
// flight before the first add, so the last block pays one L2 round trip per row instead
// of one per partial.
__device__ __forceinline__ double2 sum_partials(const double2* __restrict__ part, int i, int nb, int l) {
  constexpr int MAXQ = (NB + 31) / 32;
  double2 t[MAXQ];
#pragma unroll
  for (int q = 0; q < MAXQ; ++q) {
    const int b = l + 32 * q;
    t[q] = b < nb ? __ldcg(part + (size_t)b * PLD + i) : make_double2(0, 0);
  }
  double2 v = make_double2(0, 0);
#pragma unroll
  for (int q = 0; q < MAXQ; ++q) v += t[q];
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// ---- block reduction of NV complex partials; last block reduces over blocks -----------
// sums[i] (i < nv) are this thread's partials. The final values land in out[i].
template <int NV>
__device__ bool reduce_to(double2* sums, int nv, double2* __restrict__ part, int* counter, double2* out) {
  __shared__ double2 sh[NTH / 32][NV];
  __shared__ bool last;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    if (i < nv) {
      double2 v = sums[i];
      for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
      }
      if (l == 0) sh[w][i] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < nv) {
    double2 v = make_double2(0, 0);
    for (int k = 0; k < NTH / 32; ++k) v += sh[k][threadIdx.x];
    part[(size_t)blockIdx.x * PLD + threadIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1) == (int)gridDim.x - 1);
  __syncthreads();
  if (!last) return false;
  __threadfence();
  for (int i = w; i < nv; i += NTH / 32) {
    const double2 v = sum_partials(part, i, (int)gridDim.x, l);
    if (l == 0) out[i] = v;
  }
  if (threadIdx.x == 0) *counter = 0;
  return true;
}

// Chunked multi-vector kernels. A block of NTH threads covers chunks of NTH*EPT
// consecutive elements; thread t loads the CPL consecutive elements at
// base + (u NTH + t) CPL + c (u < EPT/CPL), so each warp access is coalesced. CPL = 2
// for complex64 vectors of even length (16-byte loads), else 1. Blocks stride over
// the chunks.
constexpr int EPT = 8;
// vectors per load group in k_mdot / k_maxpy (memory-level parallelism: VG x EPT
// independent loads per thread)
constexpr int VG = 4;

// Basis vectors i >= keep are read with the L2 evict-first policy. Every later step
// of a cycle reads the first vectors again, and the matvec between two steps needs
// its spectrum and workspace in L2: streaming the rest as evict-first keeps both
// resident instead of cycling the whole basis through L2.
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
template <typename T, int CPL> struct LdV;
template <> struct LdV<float, 1> {
  static __device__ __forceinline__ void run(const float2* p, float2* o, bool ef, uint64_t pol) {
    if (ef)
      asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0,%1}, [%2], %3;"
                   : "=f"(o[0].x), "=f"(o[0].y) : "l"(p), "l"(pol));
    else
      o[0] = __ldg(p);
  }
};
template <> struct LdV<float, 2> {
  static __device__ __forceinline__ void run(const float2* p, float2* o, bool ef, uint64_t pol) {
    if (ef) {
      asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
                   : "=f"(o[0].x), "=f"(o[0].y), "=f"(o[1].x), "=f"(o[1].y) : "l"(p), "l"(pol));
    } else {
      const float4 v = __ldg((const float4*)p);
      o[0] = make_float2(v.x, v.y);
      o[1] = make_float2(v.z, v.w);
    }
  }
};
template <> struct LdV<double, 1> {
  static __device__ __forceinline__ void run(const double2* p, double2* o, bool ef, uint64_t pol) {
    if (ef)
      asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;"
                   : "=d"(o[0].x), "=d"(o[0].y) : "l"(p), "l"(pol));
    else
      o[0] = __ldg(p);
  }
};

// a thread's EPT elements of one vector's chunk (zeros past n; n is a multiple of CPL)
template <typename T, int CPL>
__device__ __forceinline__ void ld_chunk(const cx<T>* p, size_t base, size_t n, cx<T>* o, bool ef, uint64_t pol) {
#pragma unroll
  for (int u = 0; u < EPT / CPL; ++u) {
    const size_t k = base + ((size_t)u * NTH + threadIdx.x) * CPL;
    if (k < n) {
      LdV<T, CPL>::run(p + k, o + u * CPL, ef, pol);
    } else {
#pragma unroll
      for (int c = 0; c < CPL; ++c) o[u * CPL + c] = czero<cx<T>>();
    }
  }
}
template <typename T, int CPL>
__device__ __forceinline__ void st_chunk(cx<T>* p, size_t base, size_t n, const cx<T>* v) {
#pragma unroll
  for (int u = 0; u < EPT / CPL; ++u) {
    const size_t k = base + ((size_t)u * NTH + threadIdx.x) * CPL;
    if (k < n) {
      if constexpr (CPL == 2)
        *(float4*)(p + k) = make_float4((float)v[2 * u].x, (float)v[2 * u].y, (float)v[2 * u + 1].x,
                                        (float)v[2 * u + 1].y);
      else
        p[k] = v[u];
    }
  }
}

// Thread i < nv of every block holds the block's total of row i; the last block
// to finish sums the rows over blocks in a fixed order into out[i].
__device__ void reduce_rows(double2 mine, int nv, double2* __restrict__ part, int* counter, double2* out) {
  __shared__ bool last;
  if (threadIdx.x < nv) part[(size_t)blockIdx.x * PLD + threadIdx.x] = mine;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1) == (int)gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int i = w; i < nv; i += NTH / 32) {
    const double2 v = sum_partials(part, i, (int)gridDim.x, l);
    if (l == 0) out[i] = v;
  }
  if (threadIdx.x == 0) *counter = 0;
}

// out[i] = sum_k conj(s_i V_i[k]) w[k], i < nv. Per chunk and vector the
// products of a warp are summed (FP32 within a thread's 8 elements, warp
// shuffles), and lane 0 accumulates into the block's FP64 shared totals.
template <typename T, int CPL>
__global__ void __launch_bounds__(NTH, sizeof(T) == 4 ? 2 : 1) k_mdot(const cx<T>* __restrict__ V, size_t n, int nv, const double* scale,
                                              const cx<T>* __restrict__ w, double2* part, int* counter, double2* out,
                                              const int* done, int keep) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  __shared__ double2 sh[NTH / 32][33];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  for (int i = lane; i < nv; i += 32) sh[wp][i] = make_double2(0, 0);
  __syncwarp();
  const uint64_t pol = l2_evict_first();
  const size_t chunk = (size_t)NTH * EPT;
  for (size_t base = (size_t)blockIdx.x * chunk; base < n; base += (size_t)gridDim.x * chunk) {
    cx<T> wr[EPT];
    ld_chunk<T, CPL>(w, base, n, wr, false, pol);
    int i = 0;
    // groups of VG vectors: all VG x EPT loads are in flight before the first product
    for (; i + VG <= nv; i += VG) {
      cx<T> v[VG][EPT];
#pragma unroll
      for (int q = 0; q < VG; ++q) ld_chunk<T, CPL>(V + (size_t)(i + q) * n, base, n, v[q], i + q >= keep, pol);
      double ax[VG], ay[VG];
#pragma unroll
      for (int q = 0; q < VG; ++q) {
        cx<T> a = czero<cx<T>>();
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
          a.x += v[q][u].x * wr[u].x + v[q][u].y * wr[u].y;
          a.y += v[q][u].x * wr[u].y - v[q][u].y * wr[u].x;
        }
        ax[q] = a.x;
        ay[q] = a.y;
      }
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < VG; ++q) {
          ax[q] += __shfl_xor_sync(0xffffffffu, ax[q], o);
          ay[q] += __shfl_xor_sync(0xffffffffu, ay[q], o);
        }
      if (lane == 0)
#pragma unroll
        for (int q = 0; q < VG; ++q) {
          sh[wp][i + q].x += ax[q];
          sh[wp][i + q].y += ay[q];
        }
    }
    for (; i < nv; ++i) {
      cx<T> v[EPT];
      ld_chunk<T, CPL>(V + (size_t)i * n, base, n, v, i >= keep, pol);
      cx<T> a = czero<cx<T>>();
#pragma unroll
      for (int u = 0; u < EPT; ++u) {
        a.x += v[u].x * wr[u].x + v[u].y * wr[u].y;
        a.y += v[u].x * wr[u].y - v[u].y * wr[u].x;
      }
      double ax = a.x, ay = a.y;
      for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
      }
      if (lane == 0) {
        sh[wp][i].x += ax;
        sh[wp][i].y += ay;
      }
    }
  }
  __syncthreads();
  double2 mine[1] = {make_double2(0, 0)};
  // thread i < nv owns vector i's block total
  if (threadIdx.x < nv) {
    double2 v = make_double2(0, 0);
    for (int q = 0; q < NTH / 32; ++q) v += sh[q][threadIdx.x];
    const double sc = scale ? scale[threadIdx.x] : 1.0;
    mine[0] = make_double2(sc * v.x, sc * v.y);
  }
  reduce_rows(mine[0], nv, part, counter, out);
}

// Column j of H from the CGS passes (h1, plus h2 for CGS2), rotations, residual
// estimate, and (when the cycle ends) the back substitution. Run by one warp (the
// last block of the normalising k_maxpy) right after ||w|| is known; the warp stages
// the data in shared memory and lane 0 runs the sequential FP64 recurrences.
__device__ __forceinline__ double cabs_(double2 a) { return hypot(a.x, a.y); }
__device__ void givens_step(GState* st, HessPtr h, int m, int j, bool cgs2) {
  __shared__ double2 col[33], sn[32];
  __shared__ double cs[32];
  __shared__ int stop;
  const int l = threadIdx.x & 31;
  if (l == 0) stop = st->done;
  __syncwarp();
  if (stop) return;
  double2* Hc = h.H + (size_t)j * (m + 1);
  for (int i = l; i <= j; i += 32) col[i] = cgs2 ? h.h1[i] + h.h2[i] : h.h1[i];
  for (int i = l; i < j; i += 32) {
    cs[i] = h.cs[i];
    sn[i] = h.sn[i];
  }
  __syncwarp();
  if (l == 0) {
    st->steps = j + 1;
    const double hn = sqrt(h.nrm[0].x);
    col[j + 1] = make_double2(hn, 0);
    h.scale[j + 1] = hn > 0 ? 1.0 / hn : 0.0;
    for (int i = 0; i < j; ++i) {
      const double c = cs[i];
      const double2 s = sn[i];
      const double2 a = col[i], b = col[i + 1];
      col[i] = c * a + s * b;
      col[i + 1] = c * b - conj_(s) * a;
    }
    const double2 a = col[j];
    const double bb = hn;
    const double aa = cabs_(a);
    double c;
    double2 s;
    if (aa == 0.0 && bb == 0.0) {
      // A v_j (or A P v_j) = 0: the column adds nothing; the cycle ends on the previous
      // columns with the residual estimate unchanged
      h.cs[j] = 1.0;
      h.sn[j] = make_double2(0, 0);
      st->res = cabs_(h.g[j]);
      st->status = MSC_BREAKDOWN;
      stop = 2;
    } else if (bb == 0.0) {
      c = 1.0;
      s = make_double2(0, 0);
    } else if (aa == 0.0) {
      c = 0.0;
      s = make_double2(1, 0);
      col[j] = make_double2(bb, 0);
    } else {
      const double r = hypot(aa, bb);
      c = aa / r;
      const double2 ph = make_double2(a.x / aa, a.y / aa);
      s = make_double2(ph.x * bb / r, ph.y * bb / r);  // (a/|a|) conj(b)/r with b real
      col[j] = make_double2(ph.x * r, ph.y * r);
    }
    if (stop != 2) {
    col[j + 1] = make_double2(0, 0);
    h.cs[j] = c;
    h.sn[j] = s;
    const double2 gj = h.g[j];
    h.g[j] = c * gj;
    h.g[j + 1] = make_double2(0, 0) - conj_(s) * gj;
    const double res = cabs_(h.g[j + 1]);
    st->res = res;
    bool end = false;
    if (!(res == res) || isinf(res)) {
      st->status = MSC_ERR_NONFINITE;
      end = true;
    } else if (res <= st->tol_abs) {
      st->converged = 1;
      end = true;
    } else if (hn <= 1e-300 * (st->beta > 0 ? st->beta : 1.0)) {
      st->status = MSC_BREAKDOWN;  // invariant subspace: the solution is exact in it
      end = true;
    } else if (j + 1 == m) {
      end = true;
    }
    stop = end ? 1 : 0;
    }
  }
  __syncwarp();
  for (int i = l; i <= j + 1; i += 32) Hc[i] = col[i];
  if (stop) {
    __syncwarp();
    if (l == 0) {
      const int k = stop == 2 ? j : j + 1;
      st->k = k;
      for (int i = k - 1; i >= 0; --i) {
        double2 v = h.g[i];
        for (int q = i + 1; q < k; ++q) v -= h.H[(size_t)q * (m + 1) + i] * h.y[q];
        const double2 d = h.H[(size_t)i * (m + 1) + i];
        const double dd = d.x * d.x + d.y * d.y;
        h.y[i] = dd > 0 ? make_double2((v.x * d.x + v.y * d.y) / dd, (v.y * d.x - v.x * d.y) / dd)
                        : make_double2(0, 0);
      }
      __threadfence();
      st->done = 1;
    }
  }
}

// w -= sum_i coef_i s_i V_i (i < nv); optionally out_norm.x = ||w||^2
template <typename T, bool NORM, int CPL>
__global__ void __launch_bounds__(NTH, sizeof(T) == 4 ? 2 : 1) k_maxpy(const cx<T>* __restrict__ V, size_t n, int nv, const double* scale,
                                               const double2* coef, cx<T>* __restrict__ w, double2* part, int* counter,
                                               double2* out_norm, const int* done, GState* st, HessPtr hp, int m,
                                               int j, int cgs2, int keep) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  __shared__ cx<T> cf[32];
  if (threadIdx.x < 32) {
    const int i = threadIdx.x;
    const double s = (scale && i < nv) ? scale[i] : 1.0;
    cf[i] = i < nv ? mk<T>((T)(s * coef[i].x), (T)(s * coef[i].y)) : czero<cx<T>>();
  }
  __syncthreads();
  const uint64_t pol = l2_evict_first();
  const size_t chunk = (size_t)NTH * EPT;
  double nrm = 0.0;
  // The reverse of k_mdot's order, chunks and vectors alike: what k_mdot read last is
  // still in L2 when this kernel reads it first.
  const size_t nchunk = (n + chunk - 1) / chunk;
  for (size_t c0 = blockIdx.x; c0 < nchunk; c0 += gridDim.x) {
    const size_t rounds = (nchunk - 1 - blockIdx.x) / gridDim.x;  // this block's last round
    const size_t base = ((size_t)blockIdx.x + (rounds - (c0 - blockIdx.x) / gridDim.x) * gridDim.x) * chunk;
    cx<T> wr[EPT];
    ld_chunk<T, CPL>(w, base, n, wr, false, pol);
    int i = 0;
    for (; i + VG <= nv; i += VG) {
      cx<T> v[VG][EPT];
#pragma unroll
      for (int q = 0; q < VG; ++q) {
        const int vi = nv - 1 - (i + q);
        ld_chunk<T, CPL>(V + (size_t)vi * n, base, n, v[q], vi >= keep, pol);
      }
#pragma unroll
      for (int q = 0; q < VG; ++q) {
        const cx<T> c = cf[nv - 1 - (i + q)];
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
          wr[u].x -= c.x * v[q][u].x - c.y * v[q][u].y;
          wr[u].y -= c.x * v[q][u].y + c.y * v[q][u].x;
        }
      }
    }
    for (; i < nv; ++i) {
      cx<T> v[EPT];
      const int vi = nv - 1 - i;
      ld_chunk<T, CPL>(V + (size_t)vi * n, base, n, v, vi >= keep, pol);
      const cx<T> c = cf[vi];
#pragma unroll
      for (int u = 0; u < EPT; ++u) {
        wr[u].x -= c.x * v[u].x - c.y * v[u].y;
        wr[u].y -= c.x * v[u].y + c.y * v[u].x;
      }
    }
    st_chunk<T, CPL>(w, base, n, wr);
    if (NORM)
#pragma unroll
      for (int u = 0; u < EPT / CPL; ++u) {
        const size_t k = base + ((size_t)u * NTH + threadIdx.x) * CPL;
        if (k < n)
#pragma unroll
          for (int c = 0; c < CPL; ++c)
            nrm += (double)wr[u * CPL + c].x * wr[u * CPL + c].x + (double)wr[u * CPL + c].y * wr[u * CPL + c].y;
      }
  }
  if (NORM) {
    double2 a[1] = {make_double2(nrm, 0.0)};
    const bool last = reduce_to<1>(a, 1, part, counter, out_norm);
    // the last block holds the final ||w||^2: it runs the step's Givens update
    if (last && st && threadIdx.x < 32) {
      __syncwarp();
      givens_step(st, hp, m, j, cgs2 != 0);
    }
  }
}

// ||v||^2 -> out.x ; optionally also r = b - ax written first (when b != null)
template <typename T>
__global__ void __launch_bounds__(NTH) k_resid_norm(const cx<T>* __restrict__ b, const cx<T>* __restrict__ ax,
                                                    cx<T>* __restrict__ r, size_t n, double2* part, int* counter,
                                                    double2* out) {
  double2 nrm = make_double2(0, 0);
  for (size_t k = (size_t)blockIdx.x * NTH + threadIdx.x; k < n; k += (size_t)gridDim.x * NTH) {
    cx<T> v;
    if (ax) {
      v = b[k] - ax[k];
      r[k] = v;
    } else {
      v = b[k];
    }
    const double2 d = to_d(v);
    nrm.x += d.x * d.x + d.y * d.y;
  }
  double2 a[1] = {nrm};
  reduce_to<1>(a, 1, part, counter, out);
}

// cycle start: beta = sqrt(nrm), scale[0] = 1/beta, g = (beta, 0, ...)
__global__ void k_cycle_init(GState* st, HessPtr h, int m, double tol_abs) {
  if (threadIdx.x != 0) return;
  const double beta = sqrt(h.nrm[0].x);
  st->beta = beta;
  st->res = beta;
  st->tol_abs = tol_abs;
  st->k = 0;
  st->steps = 0;
  st->status = MSC_OK;
  st->converged = 0;
  st->done = 0;
  for (int i = 0; i <= m; ++i) h.g[i] = make_double2(0, 0);
  h.g[0] = make_double2(beta, 0);
  h.scale[0] = beta > 0 ? 1.0 / beta : 0.0;
  if (!(beta == beta) || isinf(beta)) {
    st->status = MSC_ERR_NONFINITE;
    st->done = 1;
  } else if (beta <= tol_abs || beta == 0.0) {
    st->converged = 1;
    st->done = 1;
  }
}


// x += sum_{i<k} y_i s_i V_i, with k from the state (s_i = 1 when scale is null); the
// chunked loads of the Arnoldi kernels, FP64 sums
template <typename T, int CPL>
__global__ void __launch_bounds__(NTH, sizeof(T) == 4 ? 2 : 1)
    k_update_x(cx<T>* __restrict__ x, const cx<T>* __restrict__ V, size_t n, const double* scale,
               const double2* y, const GState* st) {
  __shared__ double2 cf[32];
  const int k = st->k;
  if (threadIdx.x < 32)
    cf[threadIdx.x] = threadIdx.x < k ? (scale ? scale[threadIdx.x] : 1.0) * y[threadIdx.x] : make_double2(0, 0);
  __syncthreads();
  if (k == 0) return;
  const size_t chunk = (size_t)NTH * EPT;
  for (size_t base = (size_t)blockIdx.x * chunk; base < n; base += (size_t)gridDim.x * chunk) {
    double2 acc[EPT];
#pragma unroll
    for (int u = 0; u < EPT; ++u) acc[u] = make_double2(0, 0);
    int i = 0;
    for (; i + VG <= k; i += VG) {
      cx<T> v[VG][EPT];
#pragma unroll
      for (int q = 0; q < VG; ++q) ld_chunk<T, CPL>(V + (size_t)(i + q) * n, base, n, v[q], false, 0);
#pragma unroll
      for (int q = 0; q < VG; ++q) {
        const double2 c = cf[i + q];
#pragma unroll
        for (int u = 0; u < EPT; ++u) acc[u] += c * to_d(v[q][u]);
      }
    }
    for (; i < k; ++i) {
      cx<T> v[EPT];
      ld_chunk<T, CPL>(V + (size_t)i * n, base, n, v, false, 0);
      const double2 c = cf[i];
#pragma unroll
      for (int u = 0; u < EPT; ++u) acc[u] += c * to_d(v[u]);
    }
    cx<T> xv[EPT];
    ld_chunk<T, CPL>(x, base, n, xv, false, 0);
#pragma unroll
    for (int u = 0; u < EPT; ++u) xv[u] = from_d<cx<T>>(to_d(xv[u]) + acc[u]);
    st_chunk<T, CPL>(x, base, n, xv);
  }
}

// x64 += c * d32 ; out32 = (complex64)(r64 * inv)
__global__ void k_axpy_mixed(double2* __restrict__ x, const float2* __restrict__ d, size_t n, const double* c) {
  const double cc = *c;
  for (size_t e = (size_t)blockIdx.x * NTH + threadIdx.x; e < n; e += (size_t)gridDim.x * NTH) {
    const float2 v = d[e];
    x[e].x += cc * v.x;
    x[e].y += cc * v.y;
  }
}
__global__ void k_to32_scaled(const double2* __restrict__ r, float2* __restrict__ o, size_t n, const double* nrm2) {
  const double inv = 1.0 / sqrt(*nrm2);
  for (size_t e = (size_t)blockIdx.x * NTH + threadIdx.x; e < n; e += (size_t)gridDim.x * NTH)
    o[e] = make_float2((float)(r[e].x * inv), (float)(r[e].y * inv));
}
__global__ void k_sqrt(const double* a, double* b) {
  if (threadIdx.x == 0) *b = sqrt(*a);
}

// ---- host side ---------------------------------------------------------------------------

// Basis vectors kept in L2 by the Arnoldi kernels: as many as fit in KEEP_BYTES
// (64x64x16, complex64, 4.7 MB per vector: the first 8).
constexpr double KEEP_BYTES = 40e6;
template <typename T>
static int keep_vectors(size_t n) {
  const double k = KEEP_BYTES / ((double)n * sizeof(cx<T>));
  return k < 1.0 ? 1 : (k > 32.0 ? 32 : (int)k);
}
// 16-byte loads of complex64 pairs when every vector starts on a 16-byte boundary
template <typename T>
static bool paired(const void* V, size_t n) {
  return sizeof(T) == 4 && n % 2 == 0 && ((uintptr_t)V & 15) == 0;
}

template <typename T>
static int mdot(msc_plan* pl, GmresWork* gw, const cx<T>* V, int nv, const double* scale, const cx<T>* w, double2* out,
                const int* done) {
  GState* st = (GState*)gw->state.p;
  double2* part = (double2*)gw->part.p;
  const int nb = std::min<long long>(NB, ceil_div((long long)gw->n, (long long)NTH * EPT));
  size_t n = gw->n;
  int* counter = &st->counter[0];
  int keep = keep_vectors<T>(n);
  void* args[] = {(void*)&V,    (void*)&n,       (void*)&nv,  (void*)&scale, (void*)&w,   (void*)&part,
                  (void*)&counter, (void*)&out, (void*)&done, (void*)&keep};
  const void* kern = (const void*)k_mdot<T, 1>;
  if constexpr (sizeof(T) == 4)
    if (paired<T>(V, n)) kern = (const void*)k_mdot<T, 2>;
  // an ordinary launch: with programmatic dependent launch the Arnoldi kernels made the
  // cfg2 solve 8% slower (the matvec kernels, which gain from it, keep it)
  MSC_CUDA(cudaLaunchKernel(kern, dim3(nb), dim3(NTH), args, 0, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}

// With giv_j >= 0 (NORM only) the last block also runs the Givens update of step giv_j.
template <typename T, bool NORM>
static int maxpy(msc_plan* pl, GmresWork* gw, const cx<T>* V, int nv, const double* scale, const double2* coef,
                 cx<T>* w, double2* out_norm, const int* done, int giv_j = -1, int m = 0, bool cgs2 = false) {
  GState* st = (GState*)gw->state.p;
  double2* part = (double2*)gw->part.p;
  const int nb = std::min<long long>(NB, ceil_div((long long)gw->n, (long long)NTH * EPT));
  size_t n = gw->n;
  int* counter = &st->counter[1];
  GState* gst = giv_j >= 0 ? st : nullptr;
  HessPtr hp = hess_ptrs(gw);
  int c2 = cgs2 ? 1 : 0;
  int keep = keep_vectors<T>(n);
  void* args[] = {(void*)&V,       (void*)&n,        (void*)&nv,   (void*)&scale, (void*)&coef, (void*)&w,
                  (void*)&part,    (void*)&counter,  (void*)&out_norm, (void*)&done, (void*)&gst, (void*)&hp,
                  (void*)&m,       (void*)&giv_j,    (void*)&c2,   (void*)&keep};
  const void* kern = (const void*)k_maxpy<T, NORM, 1>;
  if constexpr (sizeof(T) == 4)
    if (paired<T>(V, n)) kern = (const void*)k_maxpy<T, NORM, 2>;
  MSC_CUDA(cudaLaunchKernel(kern, dim3(nb), dim3(NTH), args, 0, pl->stream));
  ::msc::note_launch();
  return MSC_OK;
}

// One FP64 scalar to the host through page-locked memory: into a pageable destination the
// copy waits for the host's staging path with the device idle.
static int read_scalar(msc_plan* pl, GmresWork* gw, const double* d, double* out) {
  MSC_CUDA(cudaMemcpyAsync(gw->hd, d, sizeof(double), cudaMemcpyDeviceToHost, pl->stream));
  MSC_CUDA(cudaStreamSynchronize(pl->stream));
  *out = *gw->hd;
  return MSC_OK;
}

template <typename T>
static int resid_norm(msc_plan* pl, GmresWork* gw, const cx<T>* b, const cx<T>* ax, cx<T>* r, double* out_nrm2) {
  GState* st = (GState*)gw->state.p;
  const int nb = std::min<long long>(NB, ceil_div((long long)gw->n, NTH));
  k_resid_norm<T><<<nb, NTH, 0, pl->stream>>>(b, ax, r, gw->n, (double2*)gw->part.p, &st->counter[2],
                                             (double2*)out_nrm2); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}

// ||v||^2 of n elements into out (device, FP64, deterministic)
static int norm2_n(msc_plan* pl, GmresWork* gw, const double2* v, size_t n, double* out) {
  GState* st = (GState*)gw->state.p;
  const int nb = std::min<long long>(NB, ceil_div((long long)n, NTH));
  k_resid_norm<double><<<nb, NTH, 0, pl->stream>>>(v, nullptr, nullptr, n, (double2*)gw->part.p, &st->counter[2],
                                                   (double2*)out); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}

static int ensure_work(msc_plan* pl, int m) {
  if (!pl->gw) pl->gw = new GmresWork();
  GmresWork* gw = pl->gw;
  const size_t n = field_elems(pl->g) * (size_t)pl->nrhs;
  if (gw->m >= m && gw->n == n) return MSC_OK;
  gw->m = std::max(m, gw->m);
  gw->n = n;
  const size_t vb = (size_t)(gw->m + 1) * n;
  MSC_TRY(dalloc(pl, gw->V32, sizeof(float2) * vb));
  MSC_TRY(dalloc(pl, gw->V64, sizeof(double2) * vb));
  MSC_TRY(dalloc(pl, gw->x64, sizeof(double2) * n));
  MSC_TRY(dalloc(pl, gw->r64, sizeof(double2) * n));
  MSC_TRY(dalloc(pl, gw->ax64, sizeof(double2) * n));
  MSC_TRY(dalloc(pl, gw->d32, sizeof(float2) * n));
  MSC_TRY(dalloc(pl, gw->r32, sizeof(float2) * n));
  MSC_TRY(dalloc(pl, gw->hess, hess_bytes(gw->m)));
  MSC_TRY(dalloc(pl, gw->part, sizeof(double2) * (size_t)NB * PLD));
  if (!gw->state.p) {
    MSC_TRY(dalloc(pl, gw->state, sizeof(GState)));
    MSC_CUDA(cudaMemsetAsync(gw->state.p, 0, sizeof(GState), pl->stream));
    MSC_CUDA(cudaMallocHost((void**)&gw->hstate, sizeof(GState) * 2));
    MSC_CUDA(cudaMallocHost((void**)&gw->hd, sizeof(double) * 4));
    MSC_CUDA(cudaEventCreateWithFlags(&gw->ev[0], cudaEventDisableTiming));
    MSC_CUDA(cudaEventCreateWithFlags(&gw->ev[1], cudaEventDisableTiming));
    MSC_CUDA(cudaEventCreate(&gw->tev[0]));
    MSC_CUDA(cudaEventCreate(&gw->tev[1]));
  }
  return MSC_OK;
}

void gmres_free(msc_plan* pl) {
  GmresWork* gw = pl->gw;
  if (!gw) return;
  dfree(pl, gw->V32); dfree(pl, gw->V64); dfree(pl, gw->Z32); dfree(pl, gw->Z64); dfree(pl, gw->x64); dfree(pl, gw->r64); dfree(pl, gw->ax64);
  dfree(pl, gw->d32); dfree(pl, gw->r32); dfree(pl, gw->state); dfree(pl, gw->hess); dfree(pl, gw->part);
  if (gw->hstate) cudaFreeHost(gw->hstate);
  if (gw->hd) cudaFreeHost(gw->hd);
  for (auto& row : gw->graph)
    for (auto& gr : row)
      if (gr.exec) cudaGraphExecDestroy(gr.exec);
  for (auto& e : gw->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : gw->tev)
    if (e) cudaEventDestroy(e);
  delete gw;
  pl->gw = nullptr;
}

// Which cycles of flexible GMRES run with the preconditioner (MSC_PC_NEARFIELD): it has
// to earn its cost. Every cycle's residual reduction per millisecond of device time,
// -ln(res / beta) / t, is kept for the preconditioned and for the plain form (the mean
// with the previous value of that form). The solve starts preconditioned; after
// PROBE_AFTER preconditioned cycles one plain cycle measures the other form (restarted
// GMRES converges fastest in its first cycles, plain or not, so an early comparison
// favours the plain form), and from then on the faster form runs. A preconditioned
// form at least twice as fast keeps running; a closer race is measured again after
// 8, 32, 128, ... cycles of the faster form. MSC_PC_NEARFIELD_ALWAYS runs every cycle
// preconditioned. Under both, a preconditioned cycle that makes no progress at all (a
// breakdown of A P included) turns the preconditioner off for the rest of the solve.
// Cycles during which a graph was captured are not measured (the capture is host
// time). The policy lives for one solve, across its refinement sweeps.
struct PcPolicy {
  static constexpr int PROBE_AFTER = 4;
  bool allowed = false;       // a preconditioner is asked for and has not failed
  bool adaptive = true;       // false: every cycle preconditioned (MSC_PC_NEARFIELD_ALWAYS)
  bool on = true;             // form of the next cycle
  double eff[2] = {-1, -1};   // [plain, preconditioned] log-reduction per ms; -1 unknown
  int run = 0;                // cycles of the faster form since the last probe
  int interval = 8;           // cycles between probes of the slower form
  int cycles[2] = {0, 0};     // cycles run per form
  bool failed = false;        // the no-progress fallback happened

  void measure(bool pc, double beta, double res, float ms) {
    if (!(beta > 0) || !(res > 0) || !(ms > 0)) return;
    const double e = -std::log(res / beta) / (double)ms;
    double& v = eff[pc ? 1 : 0];
    v = v < 0 ? e : 0.5 * (v + e);
  }
  bool next() {
    if (!allowed) return on = false;
    if (!adaptive) return on = true;
    if (eff[0] < 0) return on = cycles[1] < PROBE_AFTER;  // the first plain measurement
    if (eff[1] < 0) return on = true;
    const bool pc_faster = eff[1] >= eff[0];
    if (eff[1] >= 2.0 * eff[0]) return on = true;
    if (++run >= interval) {
      run = 0;
      interval *= 4;
      return on = !pc_faster;
    }
    return on = pc_faster;
  }
};

// One restarted GMRES(m) solve of A x = rhs in precision T (x in/out, same precision).
// Stops when the residual estimate <= tol_abs or after max_mv operator applications.
// Returns the number of matvecs used in *n_mv and the final estimate in *res.
//
// With a policy `pol` that allows it the solve is flexible GMRES with the near-field
// preconditioner on the right, z_j = P(v_j), w = A z_j, x += Z y, in the cycles the
// policy chooses; plain GMRES runs the others.
template <typename T>
static int gmres_core(msc_plan* pl, int m, const cx<T>* rhs, cx<T>* x, bool x_zero, double tol_abs, int max_mv,
                      int* n_mv, double* res, int* status, bool cgs2, PcPolicy* pol, int* n_pc) {
  GmresWork* gw = pl->gw;
  GState* st = (GState*)gw->state.p;
  HessPtr h = hess_ptrs(gw);
  const size_t n = gw->n;
  cx<T>* V = (cx<T>*)(sizeof(T) == 8 ? gw->V64.p : gw->V32.p);
  bool use_pc = pol && pol->allowed && pol->on;
  cx<T>* Z = nullptr;
  if (pol && pol->allowed) {
    DBuf& zb = sizeof(T) == 8 ? gw->Z64 : gw->Z32;
    MSC_TRY(dalloc(pl, zb, sizeof(cx<T>) * (size_t)gw->m * n));
    Z = (cx<T>*)zb.p;
  }
  const int* done = &st->done;
  int used = 0;
  *status = MSC_NOT_CONVERGED;
  bool first = true;
  while (true) {
    const bool timed = pol && pol->allowed;
    if (timed) MSC_CUDA(cudaEventRecord(gw->tev[0], pl->stream));
    bool captured_now = false;
    // V0 = rhs - A x  (or rhs when x == 0 on the first cycle)
    if (first && x_zero) {
      MSC_CUDA(cudaMemcpyAsync(V, rhs, sizeof(cx<T>) * n, cudaMemcpyDeviceToDevice, pl->stream));
      MSC_TRY(resid_norm<T>(pl, gw, V, nullptr, nullptr, &h.nrm[0].x));
    } else {
      if (used >= max_mv) break;
      MSC_TRY(launch_matvec<T>(pl, x, nullptr, V + n, nullptr));  // A x into V[1] as scratch
      ++used;
      MSC_TRY(resid_norm<T>(pl, gw, rhs, V + n, V, &h.nrm[0].x));
    }
    first = false;
    k_cycle_init<<<1, 32, 0, pl->stream>>>(st, h, m, tol_abs); ::msc::note_launch();
    MSC_CUDA(cudaGetLastError());
    int enq = 0;  // steps enqueued in this cycle
    auto step = [&](int j) -> int {
      // Arnoldi step j: w = A v_j (or A P v_j) into V[j+1]
      if (use_pc) {
        cx<T>* zj = Z + (size_t)j * n;
        MSC_TRY(nearfield_apply<T>(pl, V + (size_t)j * n, h.scale + j, zj, done));
        MSC_TRY(launch_matvec<T>(pl, zj, nullptr, V + (size_t)(j + 1) * n, done));
      } else {
        MSC_TRY(launch_matvec<T>(pl, V + (size_t)j * n, h.scale + j, V + (size_t)(j + 1) * n, done));
      }
      cx<T>* w = V + (size_t)(j + 1) * n;
      MSC_TRY(mdot<T>(pl, gw, V, j + 1, h.scale, w, h.h1, done));
      if (cgs2) {
        MSC_TRY((maxpy<T, false>(pl, gw, V, j + 1, h.scale, h.h1, w, nullptr, done)));
        MSC_TRY(mdot<T>(pl, gw, V, j + 1, h.scale, w, h.h2, done));
        MSC_TRY((maxpy<T, true>(pl, gw, V, j + 1, h.scale, h.h2, w, &h.nrm[0], done, j, m, true)));
      } else {
        // one projection: the Hessenberg column is h1
        MSC_TRY((maxpy<T, true>(pl, gw, V, j + 1, h.scale, h.h1, w, &h.nrm[0], done, j, m, false)));
      }
      return MSC_OK;
    };
    GState cur;
    auto& gr = gw->graph[sizeof(T) == 8 ? 1 : 0][use_pc ? 1 : 0];
    // A whole cycle as one captured graph: m steps whose kernels return at once
    // after the device flag `done` is set. Captured after two uncaptured cycles of the
    // kind (buffers allocated, kernel attributes set; a solve of one or two cycles on a
    // short-lived plan does not repay the capture and instantiation) when the budget
    // covers m steps, and replayed while the plan generation holds. Plans with graphs
    // off (the batch's) always run uncaptured.
    const bool graph_ok = gr.exec && gr.m == m && gr.cgs2 == cgs2 && gr.nrhs == pl->nrhs && gr.gen == pl->gen;
    if (pl->graphs && (graph_ok || gr.warm >= 2) && used + m <= max_mv) {
      if (!graph_ok) {
        if (use_pc) MSC_TRY(nearfield_refresh(pl));
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
        gr.exec = nullptr;
        cudaGraph_t graph = nullptr;
        int cs = MSC_OK;
        MSC_CUDA(cudaStreamBeginCapture(pl->stream, cudaStreamCaptureModeThreadLocal));
        for (int j = 0; j < m && cs == MSC_OK; ++j) cs = step(j);
        const cudaError_t ce = cudaStreamEndCapture(pl->stream, &graph);
        if (cs != MSC_OK) {
          if (graph) cudaGraphDestroy(graph);
          return cs;
        }
        MSC_CUDA(ce);
        const cudaError_t ie = cudaGraphInstantiate(&gr.exec, graph, 0);
        cudaGraphDestroy(graph);
        MSC_CUDA(ie);
        gr.m = m;
        gr.cgs2 = cgs2;
        gr.nrhs = pl->nrhs;
        gr.gen = pl->gen;
        captured_now = true;
      }
      if (use_pc) MSC_TRY(nearfield_refresh(pl));  // new blocks (a new frequency) into the same buffers
      MSC_CUDA(cudaGraphLaunch(gr.exec, pl->stream));
      ::msc::note_launch();
      if (timed) MSC_CUDA(cudaEventRecord(gw->tev[1], pl->stream));
      MSC_CUDA(cudaMemcpyAsync(&gw->hstate[0], st, sizeof(GState), cudaMemcpyDeviceToHost, pl->stream));
      MSC_CUDA(cudaStreamSynchronize(pl->stream));
      cur = gw->hstate[0];
      used += cur.steps;
      enq = cur.steps;
      if (use_pc) *n_pc += cur.steps;
    } else {
      bool cycle_over = false;
      // state after cycle init
      MSC_CUDA(cudaMemcpyAsync(&gw->hstate[0], st, sizeof(GState), cudaMemcpyDeviceToHost, pl->stream));
      MSC_CUDA(cudaEventRecord(gw->ev[0], pl->stream));
      int pending = 0;  // index of the event holding the newest state
      for (int j = 0; j < m && !cycle_over; ++j) {
        if (used + 1 > max_mv) break;
        MSC_TRY(step(j));
        ++used;
        ++enq;
        if (use_pc) ++*n_pc;
        const int slot = (pending + 1) & 1;
        MSC_CUDA(cudaMemcpyAsync(&gw->hstate[slot], st, sizeof(GState), cudaMemcpyDeviceToHost, pl->stream));
        MSC_CUDA(cudaEventRecord(gw->ev[slot], pl->stream));
        // check the state of the previous step (lagged by one step)
        MSC_CUDA(cudaEventSynchronize(gw->ev[pending]));
        if (gw->hstate[pending].done) {
          cycle_over = true;  // step j early-exits on the device
          --used;             // ... and applies no operator
          if (use_pc) --*n_pc;
        }
        pending = slot;
      }
      // cycles that ended at step j (and not before) are visible in the newest state
      if (timed) MSC_CUDA(cudaEventRecord(gw->tev[1], pl->stream));
      MSC_CUDA(cudaMemcpyAsync(&gw->hstate[0], st, sizeof(GState), cudaMemcpyDeviceToHost, pl->stream));
      MSC_CUDA(cudaStreamSynchronize(pl->stream));
      cur = gw->hstate[0];
      gr.warm += 1;
    }
    if (pol && enq > 0) ++pol->cycles[use_pc ? 1 : 0];
    // x += V y (k columns), or Z y with the preconditioner
    if (cur.k > 0) {
      const int nb = std::min<long long>(NB, ceil_div((long long)n, (long long)NTH * EPT));
      const cx<T>* B = use_pc ? Z : V;
      const double* sc = use_pc ? nullptr : h.scale;
      bool pair = false;
      if constexpr (sizeof(T) == 4) {
        pair = paired<T>(B, n) && paired<T>(x, n);
        if (pair) k_update_x<T, 2><<<nb, NTH, 0, pl->stream>>>(x, B, n, sc, h.y, st);
      }
      if (!pair) k_update_x<T, 1><<<nb, NTH, 0, pl->stream>>>(x, B, n, sc, h.y, st);
      ::msc::note_launch();
      MSC_CUDA(cudaGetLastError());
    }
    *res = cur.res;
    if (cur.status == MSC_ERR_NONFINITE) {
      *status = MSC_ERR_NONFINITE;
      break;
    }
    if (cur.converged) {
      *status = MSC_OK;
      break;
    }
    // The policy measures this cycle and picks the next cycle's form. A preconditioned
    // cycle that fails to reduce the residual estimate at all (a breakdown of A P
    // included) turns the preconditioner off for the rest of the solve.
    if (pol && pol->allowed) {
      float ms = 0.f;
      if (!captured_now && cur.steps > 0) MSC_CUDA(cudaEventElapsedTime(&ms, gw->tev[0], gw->tev[1]));
      pol->measure(use_pc, cur.beta, cur.res, captured_now ? 0.f : ms);
      const bool stalled = use_pc && cur.res >= (1.0 - 1e-6) * cur.beta;
      if (stalled) {
        pol->allowed = false;
        pol->failed = true;
      }
      use_pc = pol->next();
      if (stalled) continue;
    }
    if (cur.status == MSC_BREAKDOWN) {
      *status = MSC_OK;
      break;
    }
    if (used >= max_mv) break;
    if (enq == 0) break;
  }
  *n_mv = used;
  return MSC_OK;
}

// The FP64 or mixed-precision solve of A x = b on the plan's component-major vectors
// (gw->n elements: pl->nrhs fields one after the other). x holds the initial guess on
// entry and the solution on return; b has the FP64 norm bnorm; the target is the
// relative residual tol. On return gw->r64 holds b - A x of the final x and s the
// counters, the status and the relative residual.
static int solve_core(msc_plan* pl, const double2* b, double2* x, double bnorm, double tol, const msc_solve_opts* o,
                      msc_solve_stats& s) {
  GmresWork* gw = pl->gw;
  HessPtr h = hess_ptrs(gw);
  const size_t n = gw->n;
  const int m = std::max(1, std::min(o->restart > 0 ? o->restart : 30, 32));
  double2* r = (double2*)gw->r64.p;
  double2* ax = (double2*)gw->ax64.p;
  double* dn = &h.nrm[1].x;  // outer ||.||^2 (h.nrm[1].y is scratch of the reduction)
  s.status = MSC_NOT_CONVERGED;
  const int max_mv = o->max_iter > 0 ? o->max_iter : 500;
  PcPolicy pol;
  pol.allowed = o->preconditioner == MSC_PC_NEARFIELD || o->preconditioner == MSC_PC_NEARFIELD_ALWAYS;
  pol.adaptive = o->preconditioner == MSC_PC_NEARFIELD;
  PcPolicy* pp = pol.allowed ? &pol : nullptr;
  if (bnorm == 0.0) {
    MSC_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * n, pl->stream));
    MSC_CUDA(cudaMemsetAsync(r, 0, sizeof(double2) * n, pl->stream));
    s.status = MSC_OK;
    s.residual = 0.0;
  } else if (o->precision == MSC_SOLVE_FP64) {
    int used = 0, st = 0;
    double est = 0;
    MSC_TRY(gmres_core<double>(pl, m, b, x, o->initial_guess != 0, tol * bnorm, max_mv, &used, &est, &st,
                               o->ortho != 1, pp, &s.n_precond));
    s.n_matvec = used;
    s.n_matvec64 = used;
    s.status = st;
    // true residual
    MSC_TRY(launch_matvec<double>(pl, x, nullptr, ax, nullptr));
    s.n_matvec += 1;
    s.n_matvec64 += 1;
    MSC_TRY(resid_norm<double>(pl, gw, b, ax, r, dn));
    double rn2 = 0;
    MSC_TRY(read_scalar(pl, gw, dn, &rn2));
    s.residual = std::sqrt(rn2) / bnorm;
    if (s.status != MSC_ERR_NONFINITE) s.status = s.residual <= tol ? MSC_OK : MSC_NOT_CONVERGED;
  } else {
    // mixed: FP64 refinement around complex64 GMRES
    const double inner = o->inner_tol > 0 ? o->inner_tol : 1e-5;
    float2* d = (float2*)gw->d32.p;
    float2* r32 = (float2*)gw->r32.p;
    int used = 0;  // complex64 Krylov matvecs (the budget); FP64 residuals count apart
    double res = 0;
    int outer = 0;
    while (true) {
      MSC_TRY(launch_matvec<double>(pl, x, nullptr, ax, nullptr));
      ++s.n_matvec64;
      MSC_TRY(resid_norm<double>(pl, gw, b, ax, r, dn));
      double rn2 = 0;
      MSC_TRY(read_scalar(pl, gw, dn, &rn2));
      res = std::sqrt(rn2) / bnorm;
      if (!(res == res)) {
        s.status = MSC_ERR_NONFINITE;
        break;
      }
      if (res <= tol) {
        s.status = MSC_OK;
        break;
      }
      if (used >= max_mv) break;
      // inner: A d = r / ||r|| in complex64, relative target `inner` (or what is left to reach tol)
      k_to32_scaled<<<std::min<long long>(NB, ceil_div((long long)n, NTH)), NTH, 0, pl->stream>>>(r, r32, n, dn); ::msc::note_launch();
      MSC_CUDA(cudaMemsetAsync(d, 0, sizeof(float2) * n, pl->stream));
      const double target = std::max(inner, 0.5 * tol / res);
      int iu = 0, ist = 0;
      double est = 0;
      MSC_TRY(gmres_core<float>(pl, m, r32, d, true, target, max_mv - used, &iu, &est, &ist, o->ortho == 2, pp,
                                &s.n_precond));
      used += iu;
      ++outer;
      if (ist == MSC_ERR_NONFINITE) {
        s.status = MSC_ERR_NONFINITE;
        break;
      }
      // x += ||r|| d (d = 0 when the inner solve made no step: x and r stay as they are)
      k_sqrt<<<1, 32, 0, pl->stream>>>(dn, dn); ::msc::note_launch();
      k_axpy_mixed<<<std::min<long long>(NB, ceil_div((long long)n, NTH)), NTH, 0, pl->stream>>>(x, d, n, dn); ::msc::note_launch();
      MSC_CUDA(cudaGetLastError());
      if (iu == 0) break;
    }
    s.n_matvec = used + s.n_matvec64;
    s.n_outer = outer;
    s.residual = res;
  }
  s.pc_fallback = pol.failed ? 1 : 0;
  s.pc_cycles = pol.cycles[1];
  s.plain_cycles = pol.cycles[0];
  return MSC_OK;
}

static int check_solve_opts(msc_plan* pl, const msc_solve_opts* o) {
  if (!pl->has_t0 || !pl->has_g0) {
    set_error("solve needs build_t0 and build_g0 first");
    return MSC_ERR_STATE;
  }
  if (o->preconditioner < 0 || o->preconditioner > 2) {
    set_error("unknown preconditioner %d", o->preconditioner);
    return MSC_ERR_INVALID;
  }
  if (o->preconditioner != MSC_PC_NONE && (!pl->nf || !pl->nf->ready)) {
    set_error("the near-field preconditioner needs build_g0 first");
    return MSC_ERR_STATE;
  }
  return MSC_OK;
}

// The plan's bounded-wait status after a solve: a timeout invalidates the result.
static int solve_timeout_status(msc_plan* pl) {
  int kerr = 0;
  MSC_TRY(read_status(pl, &kerr));
  if (kerr) {
    set_error("a kernel's bounded wait on its asynchronous copies or tensor-core work ran out; the result is invalid");
    return MSC_ERR_TIMEOUT;
  }
  return MSC_OK;
}

int solve(msc_plan* pl, const double2* b_ref, double2* x_ref, const msc_solve_opts* o, msc_solve_stats* stats) {
  MSC_TRY(check_solve_opts(pl, o));
  const int m = std::max(1, std::min(o->restart > 0 ? o->restart : 30, 32));
  MSC_TRY(ensure_work(pl, m));
  GmresWork* gw = pl->gw;
  HessPtr h = hess_ptrs(gw);
  const size_t n = gw->n;
  double2* x = (double2*)gw->x64.p;
  MSC_TRY(dalloc(pl, pl->f64a, sizeof(double2) * n));
  double2* b = (double2*)pl->f64a.p;
  MSC_TRY(launch_ref_to_soa<double, double>(pl, b_ref, b));
  if (pl->bloch) {
    // the solve runs in the demodulated frame; b arrives physical
    MSC_TRY(bloch_modulate(pl, b, -1));
  }
  if (o->initial_guess == 0)
    MSC_CUDA(cudaMemcpyAsync(x, b, sizeof(double2) * n, cudaMemcpyDeviceToDevice, pl->stream));
  else
    MSC_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * n, pl->stream));
  // ||b||
  double* dn = &h.nrm[1].x;
  MSC_TRY(resid_norm<double>(pl, gw, b, nullptr, nullptr, dn));
  double bn2 = 0;
  MSC_TRY(read_scalar(pl, gw, dn, &bn2));
  msc_solve_stats s{};
  MSC_TRY(solve_core(pl, b, x, std::sqrt(bn2), o->tol > 0 ? o->tol : 1e-6, o, s));
  // x back to the caller's layout (and physical frame)
  if (pl->bloch) {
    MSC_TRY(bloch_modulate(pl, x, +1));
  }
  MSC_TRY(launch_soa_to_ref<double, double>(pl, x, x_ref));
  const int ts = solve_timeout_status(pl);
  if (stats) *stats = s;
  if (ts != MSC_OK) return ts;
  if (s.status == MSC_ERR_NONFINITE)
    set_error("the solve met a non-finite (NaN or Inf) residual: check the contrasts, T0 and the frequency");
  return s.status;
}

// Scales the field v (n elements) by f on the device.
__global__ void k_scale_field(double2* __restrict__ v, size_t n, double f) {
  for (size_t k = (size_t)blockIdx.x * NTH + threadIdx.x; k < n; k += (size_t)gridDim.x * NTH) {
    v[k].x *= f;
    v[k].y *= f;
  }
}

// Sets the plan's right-hand-side count for the duration of a multi-RHS solve (a
// captured solver graph records the count it was captured with and serves only that).
struct NrhsScope {
  msc_plan* pl;
  NrhsScope(msc_plan* p, int r) : pl(p) { pl->nrhs = r; }
  ~NrhsScope() { pl->nrhs = 1; }
};

int solve_multi(msc_plan* pl, int R, const double2* b_ref, double2* x_ref, const msc_solve_opts* o,
                msc_solve_stats* stats) {
  MSC_TRY(check_solve_opts(pl, o));
  const Geo& g = pl->g;
  const size_t nf = field_elems(g);
  // workspaces of R right-hand sides, kept by the plan for its next multi-RHS solve
  MSC_TRY(dalloc(pl, pl->Wm64, sizeof(double2) * ws_elems(g) * R));
  MSC_TRY(dalloc(pl, pl->Wm32, sizeof(float2) * ws_elems(g) * R));
  NrhsScope scope(pl, R);
  const int m = std::max(1, std::min(o->restart > 0 ? o->restart : 30, 32));
  MSC_TRY(ensure_work(pl, m));
  GmresWork* gw = pl->gw;
  HessPtr h = hess_ptrs(gw);
  const size_t n = gw->n;  // R nf
  double2* x = (double2*)gw->x64.p;
  MSC_TRY(dalloc(pl, pl->f64a, sizeof(double2) * n));
  double2* b = (double2*)pl->f64a.p;
  const int nbk = (int)std::min<long long>(NB, ceil_div((long long)nf, NTH));
  double* dn = &h.nrm[1].x;
  // each right-hand side in the solver's layout (and frame), scaled to unit norm
  std::vector<double> bn(R, 0.0);
  for (int r = 0; r < R; ++r) {
    double2* br = b + (size_t)r * nf;
    MSC_TRY(launch_ref_to_soa<double, double>(pl, b_ref + (size_t)r * nf, br));
    if (pl->bloch) MSC_TRY(bloch_modulate(pl, br, -1));
    MSC_TRY(norm2_n(pl, gw, br, nf, dn));
    double v = 0;
    MSC_TRY(read_scalar(pl, gw, dn, &v));
    bn[r] = std::sqrt(v);
    if (bn[r] > 0) {
      k_scale_field<<<nbk, NTH, 0, pl->stream>>>(br, nf, 1.0 / bn[r]);
      ::msc::note_launch();
    }
  }
  int nz = 0;
  for (int r = 0; r < R; ++r) nz += bn[r] > 0 ? 1 : 0;
  if (o->initial_guess == 0)
    MSC_CUDA(cudaMemcpyAsync(x, b, sizeof(double2) * n, cudaMemcpyDeviceToDevice, pl->stream));
  else
    MSC_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * n, pl->stream));
  // One Krylov space of the stacked system: every right-hand side has unit norm, so a
  // stacked relative residual of tol / sqrt(R) bounds each one's by tol.
  const double tol = o->tol > 0 ? o->tol : 1e-6;
  msc_solve_stats s{};
  MSC_TRY(solve_core(pl, b, x, std::sqrt((double)nz), tol / std::sqrt((double)std::max(1, nz)), o, s));
  // per right-hand side: the FP64 residual of the final x (gw->r64 = b - A x), the
  // field unscaled, back to the caller's frame and layout
  const double2* res = (const double2*)gw->r64.p;
  std::vector<double> rr(R, 0.0);
  for (int r = 0; r < R; ++r) {
    MSC_TRY(norm2_n(pl, gw, res + (size_t)r * nf, nf, dn));
    double v = 0;
    MSC_TRY(read_scalar(pl, gw, dn, &v));
    rr[r] = bn[r] > 0 ? std::sqrt(v) : 0.0;
    double2* xr = x + (size_t)r * nf;
    k_scale_field<<<nbk, NTH, 0, pl->stream>>>(xr, nf, bn[r]);
    ::msc::note_launch();
    if (pl->bloch) MSC_TRY(bloch_modulate(pl, xr, +1));
    MSC_TRY(launch_soa_to_ref<double, double>(pl, xr, x_ref + (size_t)r * nf));
  }
  MSC_CUDA(cudaGetLastError());
  const int ts = solve_timeout_status(pl);
  int worst = MSC_OK;
  for (int r = 0; r < R; ++r) {
    msc_solve_stats sr = s;
    sr.residual = rr[r];
    if (s.status == MSC_ERR_NONFINITE || !(rr[r] == rr[r]))
      sr.status = MSC_ERR_NONFINITE;
    else
      sr.status = rr[r] <= tol ? MSC_OK : MSC_NOT_CONVERGED;
    if (stats) stats[r] = sr;
    if (sr.status < 0 || (worst >= 0 && sr.status > worst)) worst = sr.status;
  }
  if (ts != MSC_OK) return ts;
  if (worst == MSC_ERR_NONFINITE)
    set_error("the solve met a non-finite (NaN or Inf) residual: check the contrasts, T0 and the frequency");
  return worst;
}

}  // namespace msc
