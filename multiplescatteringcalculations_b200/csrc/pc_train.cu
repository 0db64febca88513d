// Training of the learned near-field preconditioner on the GPU: forward and
// backward kernels, the adjoint slab operator and Adam.
//
// Model (the preconditioner of pc.cu with learned parameters): for a residual r,
//   h_0 = r,  h_l = S_l h_{l-1},  S_l x = (G_nn + dG_l)(T0 x)   (27-point stencil, l = 1..L),
//   z = P r = sum_{l=0..L} c_l h_l,
// stencil entries restricted to the lattice's mirror-symmetry pattern. Parameters:
// c_l (complex) and w_l = dG_l / s (27 x 9 x 9 complex per layer), s = max |G_nn|, so
// the weights are dimensionless and carry over between frequencies.
//
// Objective: the residual of one GMRES step on the preconditioned operator,
//   loss(r) = min_alpha || alpha A P r^ - r^ ||^2 = 1 - |<y, r^>|^2 / <y, y>,
//   y = A P r^,  r^ = r / ||r||,  A = I - G0 T0 the slab operator,
// invariant to the scale of P as GMRES is (an objective without the optimal alpha,
// || A P r^ - r^ ||^2, trains the polynomial towards damped coefficients that lower
// it while they slow GMRES on the hard slabs).
// Backward, in Wirtinger derivatives d/dconj of the real loss (the envelope theorem
// removes alpha's own dependence):
//   alpha = <y, r^> / <y, y>,  q = alpha y - r^,  d = A^H (conj(alpha) q)
//   g(c_l) = <h_l, d>
//   delta_L = conj(c_L) d,  delta_{l-1} = conj(c_{l-1}) d + S_l^H delta_l
//   g(w_l)[o][a][b] = s sum_v delta_{l,a}(v) conj(tau_{l-1,b}(v - o)),  tau_{l-1} = T0 h_{l-1}
//   S_l^H y = T0^H (sum_o G_{l,o}^H y(. + o))
// The adjoint operator comes from the kernel's symmetries: reciprocity makes K D
// symmetric (D = diag(1 x 6, 2 x 3), the Voigt factors) and the mirror symmetry gives
// K(-r) = P K(r) P with P = diag(-1 x 3, 1 x 6) (displacements odd, strains even), so
// G0^T = P D^-1 G0 D P and
//   A^H q = q - conj(T0) P D^-1 conj(G0 (D P conj(q))),
// where G0 u = s (u - A_tau u) with A_tau the slab operator run with T0 = tau I,
// tau = 1/s: G0 tau u is of the order of u, so the difference does not cancel (|G0| is
// about 1e-11 in physical units; u - A_I u would lose all FP32 digits). Bloch-phased kernels
// lose the mirror symmetry and the volume-averaged kernel is not D-symmetric, so
// training takes the point-propagator kernel without a Bloch phase.
//
// Precision: the complex64 path trains with BF16 layer weights (G_nn + s w_l rounded
// to BF16, the form inference uses) and FP32 accumulation in the stencils, FP32
// master weights and Adam moments; gradient sums are reduced in FP64. The complex128
// path (FP64 weights) serves the gradient check against the oracle.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "mv_common.cuh"
#include "pc.cuh"

namespace msc {

namespace {

__device__ __forceinline__ bool nf_allowed(int o, int a, int b) {
  const int dz = o / 9 - 1, dx = (o / 3) % 3 - 1, dy = o % 3 - 1;
  const int zm = (dx == 0 ? 1 : 0) | (dy == 0 ? 2 : 0) | (dz == 0 ? 4 : 0);
  return ((dof_parity(a) ^ dof_parity(b)) & zm) == 0;
}

__device__ __forceinline__ float2 wload(__nv_bfloat162 w) { return __bfloat1622float2(w); }
__device__ __forceinline__ double2 wload(double2 w) { return w; }

// y = T0 x (conj = 0) or T0^H x (conj = 1) on SoA fields; T0 is complex symmetric per
// voxel, so T0^H = conj(T0)
template <typename T>
__global__ void k_tr_tapply(const cx<T>* __restrict__ x, const cx<T>* __restrict__ t4, cx<T>* __restrict__ y,
                            int nsite, int conj) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsite) return;
  cx<T> tq[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) tq[q] = conj ? conj_(t4[(size_t)q * nsite + s]) : t4[(size_t)q * nsite + s];
  cx<T> xv[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) xv[c] = x[(size_t)c * nsite + s];
  const cx<T> tr = xv[3] + xv[4] + xv[5];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    cx<T> v;
    if (c < 3) v = tq[0] * xv[c];
    else if (c < 6) v = tq[1] * tr + tq[2] * xv[c];
    else v = tq[3] * xv[c];
    y[(size_t)c * nsite + s] = v;
  }
}

// forward: y_a(v) = sum_o sum_b G[o][a][b] x_b(v - o)
// adjoint: y_b(u) = sum_o sum_a conj(G[o][a][b]) x_a(u + o)
template <typename T, typename WT>
__global__ void k_tr_stencil(const cx<T>* __restrict__ x, const WT* __restrict__ G, cx<T>* __restrict__ y, Geo g,
                             int adjoint) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.nsite) return;
  const int j = s % g.M, i = (s / g.M) % g.M, n = s / (g.M * g.M);
  cx<T> acc[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) acc[c] = czero<cx<T>>();
  const int sg = adjoint ? 1 : -1;
  for (int o = 0; o < NF_OFFS; ++o) {
    const int dz = o / 9 - 1, dx = (o / 3) % 3 - 1, dy = o % 3 - 1;
    const int zn = n + sg * dz, xi = i + sg * dx, yj = j + sg * dy;
    if (zn < 0 || zn >= g.Nz || xi < 0 || xi >= g.M || yj < 0 || yj >= g.M) continue;
    const int src = (zn * g.M + xi) * g.M + yj;
    cx<T> xv[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) xv[c] = x[(size_t)c * g.nsite + src];
#pragma unroll
    for (int a = 0; a < 9; ++a)
#pragma unroll
      for (int b = 0; b < 9; ++b) {
        if (!nf_allowed(o, a, b)) continue;
        const cx<T> m = wload(G[o * 81 + a * 9 + b]);
        if (!adjoint) fma_(acc[a], m, xv[b]);
        else fma_(acc[b], conj_(m), xv[a]);
      }
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) y[(size_t)c * g.nsite + s] = acc[c];
}

// Block-sum of a double2 over blockDim.x (a power of two <= 256) threads.
__device__ double2 block_sum(double2 v) {
  __shared__ double2 sh[256];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + w];
    __syncthreads();
  }
  const double2 r = sh[0];
  __syncthreads();
  return r;
}

// Weight gradient, tiled: a block stages delta on its tile of 2 x 8 x 16 sites and tau on
// the tile with a one-voxel halo (zero outside the slab) in shared memory, and each thread
// accumulates sum_v delta_a(v) conj(tau_b(v - o)) over the tile for its entries (o, a, b)
// of the mirror-symmetry pattern; part[block][entry] holds the block's sums, which
// k_tr_wgrad_reduce adds over the blocks in a fixed order. Row pitches 257 and 721 put
// the rows of different components in different banks.
constexpr int WG_TZ = 2, WG_TX = 8, WG_TY = 16, WG_NT = WG_TZ * WG_TX * WG_TY;
constexpr int WG_HZ = WG_TZ + 2, WG_HX = WG_TX + 2, WG_HY = WG_TY + 2, WG_HALO = WG_HZ * WG_HX * WG_HY;
constexpr int WG_DP = WG_NT + 1, WG_TP = WG_HALO + 1;

template <typename T>
__global__ void __launch_bounds__(WG_NT) k_tr_wgrad_tile(const cx<T>* __restrict__ delta, const cx<T>* __restrict__ tau,
                                                         double2* __restrict__ part, Geo g) {
  using C = cx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* dl = reinterpret_cast<C*>(smem_raw);  // [9][WG_DP]
  C* tu = dl + 9 * WG_DP;                   // [9][WG_TP]
  const int nby = (g.M + WG_TY - 1) / WG_TY, nbx = (g.M + WG_TX - 1) / WG_TX;
  const int by = blockIdx.x % nby, bx = (blockIdx.x / nby) % nbx, bz = blockIdx.x / (nby * nbx);
  const int y0 = by * WG_TY, x0 = bx * WG_TX, z0 = bz * WG_TZ;
  const int tid = threadIdx.x;
  {
    const int vy = tid % WG_TY, vx = (tid / WG_TY) % WG_TX, vz = tid / (WG_TY * WG_TX);
    const int z = z0 + vz, x = x0 + vx, y = y0 + vy;
    const bool in = z < g.Nz && x < g.M && y < g.M;
    const int site = (z * g.M + x) * g.M + y;
#pragma unroll
    for (int c = 0; c < 9; ++c) dl[c * WG_DP + tid] = in ? delta[(size_t)c * g.nsite + site] : czero<C>();
  }
  for (int i = tid; i < WG_HALO; i += WG_NT) {
    const int hy = i % WG_HY, hx = (i / WG_HY) % WG_HX, hz = i / (WG_HY * WG_HX);
    const int z = z0 + hz - 1, x = x0 + hx - 1, y = y0 + hy - 1;
    const bool in = z >= 0 && z < g.Nz && x >= 0 && x < g.M && y >= 0 && y < g.M;
    const int site = (z * g.M + x) * g.M + y;
#pragma unroll
    for (int c = 0; c < 9; ++c) tu[c * WG_TP + i] = in ? tau[(size_t)c * g.nsite + site] : czero<C>();
  }
  __syncthreads();
  double2* pb = part + (size_t)blockIdx.x * NF_OFFS * 81;
  for (int e = tid; e < NF_OFFS * 81; e += WG_NT) {
    const int o = e / 81, a = (e / 9) % 9, b = e % 9;
    C sum = czero<C>();
    if (nf_allowed(o, a, b)) {
      const int dz = o / 9 - 1, dx = (o / 3) % 3 - 1, dy = o % 3 - 1;
      const C* da = dl + a * WG_DP;
      const C* tb = tu + b * WG_TP;
      for (int vz = 0; vz < WG_TZ; ++vz)
        for (int vx = 0; vx < WG_TX; ++vx) {
          const int v0 = (vz * WG_TX + vx) * WG_TY;
          const int h0 = ((vz + 1 - dz) * WG_HX + (vx + 1 - dx)) * WG_HY + 1 - dy;
#pragma unroll
          for (int vy = 0; vy < WG_TY; ++vy) sum += mul_conj(da[v0 + vy], tb[h0 + vy]);
        }
    }
    pb[e] = to_d(sum);
  }
}

// gG[e] += scale sum over blocks of part[block][e] (fixed order)
__global__ void k_tr_wgrad_reduce(const double2* __restrict__ part, int nblocks, double2* gG, double scale) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NF_OFFS * 81) return;
  double2 s = make_double2(0, 0);
  for (int b = 0; b < nblocks; ++b) s = s + part[(size_t)b * NF_OFFS * 81 + e];
  gG[e] = gG[e] + scale * s;
}

inline int wgrad_blocks(const Geo& g) {
  return ((g.M + WG_TY - 1) / WG_TY) * ((g.M + WG_TX - 1) / WG_TX) * ((g.Nz + WG_TZ - 1) / WG_TZ);
}

// out[k] += sum conj(a_k) b over n elements for the vectors a_k = A + k n: blockIdx.y = k,
// the blocks along x split the elements; each adds its FP64 block sum atomically (out
// zeroed by the caller)
template <typename T>
__global__ void k_tr_dots(const cx<T>* __restrict__ A, size_t n, const cx<T>* __restrict__ b, double2* out) {
  const cx<T>* a = A + (size_t)blockIdx.y * n;
  double2 sum = make_double2(0, 0);
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    sum = sum + to_d(conj_mul(a[k], b[k]));
  const double2 r = block_sum(sum);
  if (threadIdx.x == 0) {
    atomicAdd(&out[blockIdx.y].x, r.x);
    atomicAdd(&out[blockIdx.y].y, r.y);
  }
}

// out[k] = sum conj(a_k) b, k < nv
template <typename T>
int tr_dots(cudaStream_t st, const cx<T>* A, size_t n, const cx<T>* b, double2* out, int nv) {
  MSC_CUDA(cudaMemsetAsync(out, 0, sizeof(double2) * nv, st));
  const unsigned nbx = (unsigned)std::min<size_t>(592, (n + 255) / 256);
  k_tr_dots<T><<<dim3(nbx, (unsigned)nv), 256, 0, st>>>(A, n, b, out);
  return MSC_OK;
}

// z = sum_l c_l H_l (nv vectors)
template <typename T>
__global__ void k_tr_combine(const cx<T>* __restrict__ H, int nv, const double2* __restrict__ c, size_t n,
                             cx<T>* __restrict__ z) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double2 s = make_double2(0, 0);
  for (int l = 0; l < nv; ++l) s = s + c[l] * to_d(H[(size_t)l * n + k]);
  z[k] = from_d<cx<T>>(s);
}

// y = alpha x + beta y (alpha, beta complex)
template <typename T>
__global__ void k_tr_axpby(const cx<T>* __restrict__ x, double2 alpha, double2 beta, cx<T>* __restrict__ y,
                           size_t n) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) y[k] = from_d<cx<T>>(alpha * to_d(x[k]) + beta * to_d(y[k]));
}

// y = s x (s real)
template <typename T>
__global__ void k_tr_scale(const cx<T>* __restrict__ x, double s, cx<T>* __restrict__ y, size_t n) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) y[k] = from_d<cx<T>>(s * to_d(x[k]));
}

__host__ __device__ __forceinline__ double adj_p(int c) { return c < 3 ? -1.0 : 1.0; }
__host__ __device__ __forceinline__ double adj_d(int c) { return c < 6 ? 1.0 : 2.0; }

// u = D P conj(q)
template <typename T>
__global__ void k_tr_adj_pre(const cx<T>* __restrict__ q, cx<T>* __restrict__ u, int nsite) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (size_t)9 * nsite) return;
  const int c = (int)(k / nsite);
  u[k] = from_d<cx<T>>((adj_d(c) * adj_p(c)) * to_d(conj_(q[k])));
}

// d = q - conj(T0) P D^-1 conj(s (u - y)),  y = A_tau u (so s (u - y) = G0 u)
template <typename T>
__global__ void k_tr_adj_post(const cx<T>* __restrict__ q, const cx<T>* __restrict__ u, const cx<T>* __restrict__ y,
                              const cx<T>* __restrict__ t4, cx<T>* __restrict__ d, int nsite, double s_g) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsite) return;
  cx<T> w[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    const size_t e = (size_t)c * nsite + s;
    w[c] = from_d<cx<T>>((s_g * adj_p(c) / adj_d(c)) * to_d(conj_(u[e] - y[e])));
  }
  cx<T> tq[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) tq[i] = conj_(t4[(size_t)i * nsite + s]);
  const cx<T> tr = w[3] + w[4] + w[5];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    cx<T> v;
    if (c < 3) v = tq[0] * w[c];
    else if (c < 6) v = tq[1] * tr + tq[2] * w[c];
    else v = tq[3] * w[c];
    const size_t e = (size_t)c * nsite + s;
    d[e] = q[e] - v;
  }
}

// T0 = tau I in the 4-scalar form: t_u = tau, t_l = 0, t_d = tau, t_s = tau
template <typename T>
__global__ void k_tr_ident_t4(cx<T>* t4, int nsite, double tau) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsite) return;
  t4[s] = mk<T>((T)tau, 0);
  t4[(size_t)nsite + s] = mk<T>(0, 0);
  t4[(size_t)2 * nsite + s] = mk<T>((T)tau, 0);
  t4[(size_t)3 * nsite + s] = mk<T>((T)tau, 0);
}

// Adam on the real parameters (re/im parts as separate reals). g holds dL/dconj(theta)
// as (re, im) pairs; its real and imaginary parts are half the partial derivatives
// along the real and imaginary parts of theta, which Adam's normalisation absorbs.
__global__ void k_tr_adam(float* p, const double* __restrict__ gr, float* m, float* v, int n, float lr, float b1,
                          float b2, float eps, float bc1, float bc2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float gk = (float)gr[k];
  const float mk_ = b1 * m[k] + (1.f - b1) * gk;
  const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
  m[k] = mk_;
  v[k] = vk;
  p[k] -= lr * (mk_ / bc1) / (sqrtf(vk / bc2) + eps);
}

inline int nblk(size_t n, int t = 256) { return (int)((n + t - 1) / t); }

template <typename T> struct WType { using type = double2; };
template <> struct WType<float> { using type = __nv_bfloat162; };

// Training state on the device for one plan and degree.
struct Trainer {
  msc_plan* pl;
  int L;
  size_t n;
  double s = 1;  // max |G_nn|
  std::vector<DBuf> bufs;

  Trainer(msc_plan* p, int deg) : pl(p), L(deg), n(field_elems(p->g)) { bufs.reserve(32); }
  ~Trainer() {
    for (auto& b : bufs) dfree(pl, b);
  }
  template <typename X>
  int get(X** out, size_t elems) {
    bufs.emplace_back();
    MSC_TRY(dalloc(pl, bufs.back(), sizeof(X) * std::max<size_t>(elems, 1)));
    *out = (X*)bufs.back().p;
    return MSC_OK;
  }

  int scale_from_blocks() {
    MSC_TRY(nf_host_sync(pl));
    s = 0;
    for (const double2& v : pl->nf->g64) s = std::max(s, std::hypot(v.x, v.y));
    if (!(s > 0)) {
      set_error("the near-field blocks are zero (a single voxel?)");
      return MSC_ERR_STATE;
    }
    return MSC_OK;
  }

  // layer blocks G_nn + s w_l on the device ([L][27][81]; BF16 for the complex64 path)
  template <typename T, typename P>
  int layers(const P* w, typename WType<T>::type* dst) {
    using WT = typename WType<T>::type;
    MSC_TRY(nf_host_sync(pl));
    std::vector<WT> h((size_t)L * NF_OFFS * 81);
    for (int l = 0; l < L; ++l)
      for (int i = 0; i < NF_OFFS * 81; ++i) {
        const size_t k = (size_t)l * NF_OFFS * 81 + i;
        const double2 v = make_double2(pl->nf->g64[i].x + s * (double)w[2 * k],
                                       pl->nf->g64[i].y + s * (double)w[2 * k + 1]);
        if constexpr (sizeof(T) == 8) h[k] = v;
        else h[k] = __floats2bfloat162_rn((float)v.x, (float)v.y);
      }
    MSC_CUDA(cudaMemcpyAsync(dst, h.data(), sizeof(WT) * h.size(), cudaMemcpyHostToDevice, pl->stream));
    // the staging vector goes out of scope: wait for the copy
    MSC_CUDA(cudaStreamSynchronize(pl->stream));
    return MSC_OK;
  }

  // y = x - G0 (tau x) (the slab operator with T0 = tau I); those scalars in t4id
  template <typename T>
  int matvec_identity(const cx<T>* x, cx<T>* y, const cx<T>* t4id) {
    DBuf& t4 = sizeof(T) == 8 ? pl->t4_64 : pl->t4_32;
    void* saved = t4.p;
    t4.p = (void*)t4id;
    const int st = launch_matvec<T>(pl, x, nullptr, y, nullptr);
    t4.p = saved;
    return st;
  }

  // Loss of one residual r (SoA, device) and the gradients: gc_dev (L+1) and gw
  // (accumulated, [L][27][81]), both with respect to the conjugate parameters.
  template <typename T>
  int loss_grad(const cx<T>* r, const double2* coef_dev, const std::vector<double2>& coef,
                const typename WType<T>::type* Gl, const cx<T>* t4id, double* loss, double2* gw, double2* gc_dev,
                cx<T>* H, cx<T>* tau, cx<T>* z, cx<T>* q, cx<T>* u, cx<T>* y, cx<T>* d, cx<T>* del, double2* red,
                double2* part) {
    const Geo& g = pl->g;
    cudaStream_t st = pl->stream;
    const cx<T>* t4 = (const cx<T>*)(sizeof(T) == 8 ? pl->t4_64.p : pl->t4_32.p);
    MSC_TRY(tr_dots<T>(st, r, n, r, red, 1));
    double2 rn2;
    MSC_CUDA(cudaMemcpyAsync(&rn2, red, sizeof(rn2), cudaMemcpyDeviceToHost, st));
    MSC_CUDA(cudaStreamSynchronize(st));
    if (!(rn2.x > 0) || !std::isfinite(rn2.x)) {
      set_error("training residual is zero or not finite");
      return MSC_ERR_INVALID;
    }
    // forward
    k_tr_scale<T><<<nblk(n), 256, 0, st>>>(r, 1.0 / std::sqrt(rn2.x), H, n);
    for (int l = 1; l <= L; ++l) {
      k_tr_tapply<T><<<nblk(g.nsite), 256, 0, st>>>(H + (l - 1) * n, t4, tau + (l - 1) * n, g.nsite, 0);
      k_tr_stencil<T><<<nblk(g.nsite, 128), 128, 0, st>>>(tau + (l - 1) * n, Gl + (size_t)(l - 1) * NF_OFFS * 81,
                                                          H + l * n, g, 0);
    }
    k_tr_combine<T><<<nblk(n), 256, 0, st>>>(H, L + 1, coef_dev, n, z);
    MSC_TRY(launch_matvec<T>(pl, z, nullptr, q, nullptr));  // y = A z (in q)
    // the optimal scale alpha = <y, r^> / <y, y>
    MSC_TRY(tr_dots<T>(st, q, n, H, red + 2, 1));
    MSC_TRY(tr_dots<T>(st, q, n, q, red + 3, 1));
    double2 ab[2];
    MSC_CUDA(cudaMemcpyAsync(ab, red + 2, sizeof(ab), cudaMemcpyDeviceToHost, st));
    MSC_CUDA(cudaStreamSynchronize(st));
    if (!(ab[1].x > 0) || !std::isfinite(ab[1].x)) {
      set_error("the preconditioned residual A P r vanishes or is not finite");
      return MSC_ERR_NONFINITE;
    }
    const double2 alpha = make_double2(ab[0].x / ab[1].x, ab[0].y / ab[1].x);
    k_tr_axpby<T><<<nblk(n), 256, 0, st>>>(H, make_double2(-1, 0), alpha, q, n);  // q = alpha y - r^
    MSC_TRY(tr_dots<T>(st, q, n, q, red + 1, 1));
    k_tr_axpby<T><<<nblk(n), 256, 0, st>>>(q, conj_(alpha), make_double2(0, 0), q, n);  // q *= conj(alpha)
    // d = A^H q
    k_tr_adj_pre<T><<<nblk(n), 256, 0, st>>>(q, u, g.nsite);
    MSC_TRY(matvec_identity<T>(u, y, t4id));
    k_tr_adj_post<T><<<nblk(g.nsite), 256, 0, st>>>(q, u, y, t4, d, g.nsite, s);
    // coefficient gradients
    MSC_TRY(tr_dots<T>(st, H, n, d, gc_dev, L + 1));
    // backward through the layers
    MSC_CUDA(cudaMemsetAsync(del, 0, sizeof(cx<T>) * n, st));
    k_tr_axpby<T><<<nblk(n), 256, 0, st>>>(d, conj_(coef[L]), make_double2(0, 0), del, n);
    for (int l = L; l >= 1; --l) {
      {
        const int nbw = wgrad_blocks(g);
        const size_t smw = sizeof(cx<T>) * 9 * (size_t)(WG_DP + WG_TP);
        MSC_CUDA(prep_kernel((const void*)k_tr_wgrad_tile<T>));
        k_tr_wgrad_tile<T><<<nbw, WG_NT, smw, st>>>(del, tau + (l - 1) * n, part, g);
        k_tr_wgrad_reduce<<<(NF_OFFS * 81 + 255) / 256, 256, 0, st>>>(part, nbw,
                                                                      gw + (size_t)(l - 1) * NF_OFFS * 81, s);
      }
      if (l > 1) {
        k_tr_stencil<T><<<nblk(g.nsite, 128), 128, 0, st>>>(del, Gl + (size_t)(l - 1) * NF_OFFS * 81, u, g, 1);
        k_tr_tapply<T><<<nblk(g.nsite), 256, 0, st>>>(u, t4, del, g.nsite, 1);
        k_tr_axpby<T><<<nblk(n), 256, 0, st>>>(d, conj_(coef[l - 1]), make_double2(1, 0), del, n);
      }
    }
    MSC_CUDA(cudaGetLastError());
    for (int k = 0; k < 12 + 5 * L; ++k) ::msc::note_launch();
    double2 ln;
    MSC_CUDA(cudaMemcpyAsync(&ln, red + 1, sizeof(ln), cudaMemcpyDeviceToHost, st));
    MSC_CUDA(cudaStreamSynchronize(st));
    *loss = ln.x;
    return MSC_OK;
  }
};

int check_plan(msc_plan* pl, int degree) {
  if (degree < 1 || degree > NF_MAXL) {
    set_error("degree must be in [1, %d], got %d", NF_MAXL, degree);
    return MSC_ERR_INVALID;
  }
  if (!pl->has_t0 || !pl->has_g0 || !pl->nf || !pl->nf->ready) {
    set_error("preconditioner training needs build_t0 and build_g0 first");
    return MSC_ERR_STATE;
  }
  if (pl->bloch || pl->E != 45) {
    set_error("preconditioner training needs the point-propagator kernel without a Bloch phase");
    return MSC_ERR_UNSUPPORTED;
  }
  return MSC_OK;
}

// field buffers of one loss/gradient evaluation
template <typename T>
struct Fields {
  cx<T> *r, *H, *tau, *z, *q, *u, *y, *d, *del, *t4id;
  double2 *gw, *gc, *cd, *red, *part;
  typename WType<T>::type* Gl;
  int alloc(Trainer& tr) {
    const size_t n = tr.n;
    const int L = tr.L, nb = L * NF_OFFS * 81;
    MSC_TRY(tr.get(&r, n));
    MSC_TRY(tr.get(&H, n * (L + 1)));
    MSC_TRY(tr.get(&tau, n * L));
    MSC_TRY(tr.get(&z, n));
    MSC_TRY(tr.get(&q, n));
    MSC_TRY(tr.get(&u, n));
    MSC_TRY(tr.get(&y, n));
    MSC_TRY(tr.get(&d, n));
    MSC_TRY(tr.get(&del, n));
    MSC_TRY(tr.get(&t4id, (size_t)4 * tr.pl->g.nsite));
    MSC_TRY(tr.get(&gw, nb));
    MSC_TRY(tr.get(&gc, L + 1));
    MSC_TRY(tr.get(&cd, L + 1));
    MSC_TRY(tr.get(&red, 4));
    MSC_TRY(tr.get(&part, (size_t)wgrad_blocks(tr.pl->g) * NF_OFFS * 81));
    MSC_TRY(tr.get(&Gl, nb));
    k_tr_ident_t4<T><<<nblk(tr.pl->g.nsite), 256, 0, tr.pl->stream>>>(t4id, tr.pl->g.nsite, 1.0 / tr.s);
    ::msc::note_launch();
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
  }
  int run(Trainer& tr, const std::vector<double2>& c, double* loss) {
    MSC_CUDA(cudaMemcpyAsync(cd, c.data(), sizeof(double2) * c.size(), cudaMemcpyHostToDevice, tr.pl->stream));
    MSC_CUDA(cudaMemsetAsync(gw, 0, sizeof(double2) * (size_t)tr.L * NF_OFFS * 81, tr.pl->stream));
    return tr.loss_grad<T>(r, cd, c, Gl, t4id, loss, gw, gc, H, tau, z, q, u, y, d, del, red, part);
  }
};

template <typename T>
int run_loss_grad(msc_plan* pl, const void* r_ref, int L, const double* coef, const double* w, double* loss,
                  double* gcoef, double* gw) {
  Trainer tr(pl, L);
  MSC_TRY(tr.scale_from_blocks());
  Fields<T> f;
  MSC_TRY(f.alloc(tr));
  const int nb = L * NF_OFFS * 81;
  MSC_TRY((tr.layers<T, double>(w, f.Gl)));
  std::vector<double2> c(L + 1);
  for (int l = 0; l <= L; ++l) c[l] = make_double2(coef[2 * l], coef[2 * l + 1]);
  MSC_TRY((launch_ref_to_soa<T, T>(pl, (const cx<T>*)r_ref, f.r)));
  MSC_TRY(f.run(tr, c, loss));
  MSC_CUDA(cudaMemcpyAsync(gcoef, f.gc, sizeof(double2) * (L + 1), cudaMemcpyDeviceToHost, pl->stream));
  MSC_CUDA(cudaMemcpyAsync(gw, f.gw, sizeof(double2) * nb, cudaMemcpyDeviceToHost, pl->stream));
  MSC_CUDA(cudaStreamSynchronize(pl->stream));
  return MSC_OK;
}

}  // namespace
}  // namespace msc

using namespace msc;

extern "C" {

double msc_nearfield_scale(const msc_plan* pl) {
  if (!pl || !pl->nf || !pl->nf->ready) return 0.0;
  if (nf_host_sync(pl) != MSC_OK) return 0.0;
  double s = 0;
  for (const double2& v : pl->nf->g64) s = std::max(s, std::hypot(v.x, v.y));
  return s;
}

int msc_nf_loss_grad(msc_plan* pl, const void* r, int precision, int degree, const double* coef, const double* w,
                     double* loss, double* gcoef, double* gw) {
  if (!pl || !r || !coef || !w || !loss || !gcoef || !gw) {
    set_error("null argument");
    return MSC_ERR_INVALID;
  }
  MSC_TRY(check_plan(pl, degree));
  StreamFence fence(pl);
  if (precision == MSC_COMPLEX128) return run_loss_grad<double>(pl, r, degree, coef, w, loss, gcoef, gw);
  if (precision == MSC_COMPLEX64) return run_loss_grad<float>(pl, r, degree, coef, w, loss, gcoef, gw);
  set_error("precision must be 0 (complex64) or 1 (complex128)");
  return MSC_ERR_INVALID;
}

int msc_nf_train(msc_plan* pl, const void* r, int n_res, int degree, int steps, double lr, double* coef, double* w,
                 double* adam, double* losses) {
  if (!pl || !r || !coef || !w || !adam || n_res < 1 || steps < 0) {
    set_error("null argument or no residuals");
    return MSC_ERR_INVALID;
  }
  if (!(lr > 0) || !std::isfinite(lr)) {
    set_error("learning rate must be positive, got %g", lr);
    return MSC_ERR_INVALID;
  }
  MSC_TRY(check_plan(pl, degree));
  StreamFence fence(pl);
  const int L = degree;
  Trainer tr(pl, L);
  MSC_TRY(tr.scale_from_blocks());
  Fields<float> f;
  MSC_TRY(f.alloc(tr));
  const size_t n = tr.n;
  const int nb = L * NF_OFFS * 81;
  const int nc = 2 * (L + 1);
  const int np = nc + 2 * nb;  // real parameters: coefficients, then weights
  double* gall;
  float *pd, *md, *vd;
  MSC_TRY(tr.get(&gall, np));
  MSC_TRY(tr.get(&pd, np));
  MSC_TRY(tr.get(&md, np));
  MSC_TRY(tr.get(&vd, np));
  // host state: parameters, moments, step count (adam = [m (np)] [v (np)] [t])
  std::vector<float> p(np), m(np), v(np);
  for (int i = 0; i < nc; ++i) p[i] = (float)coef[i];
  for (int i = 0; i < 2 * nb; ++i) p[nc + i] = (float)w[i];
  for (int i = 0; i < np; ++i) {
    m[i] = (float)adam[i];
    v[i] = (float)adam[np + i];
  }
  long long t = (long long)adam[2 * np];
  cudaStream_t st = pl->stream;
  MSC_CUDA(cudaMemcpyAsync(pd, p.data(), sizeof(float) * np, cudaMemcpyHostToDevice, st));
  MSC_CUDA(cudaMemcpyAsync(md, m.data(), sizeof(float) * np, cudaMemcpyHostToDevice, st));
  MSC_CUDA(cudaMemcpyAsync(vd, v.data(), sizeof(float) * np, cudaMemcpyHostToDevice, st));
  std::vector<double2> c(L + 1);
  for (int it = 0; it < steps; ++it) {
    // the current FP32 master weights -> BF16 layer blocks and coefficients
    MSC_CUDA(cudaMemcpyAsync(p.data(), pd, sizeof(float) * np, cudaMemcpyDeviceToHost, st));
    MSC_CUDA(cudaStreamSynchronize(st));
    for (int l = 0; l <= L; ++l) c[l] = make_double2(p[2 * l], p[2 * l + 1]);
    MSC_TRY((tr.layers<float, float>(p.data() + nc, f.Gl)));
    MSC_TRY((launch_ref_to_soa<float, float>(pl, (const float2*)r + (size_t)(it % n_res) * n, f.r)));
    double loss = 0;
    MSC_TRY(f.run(tr, c, &loss));
    if (losses) losses[it] = loss;
    // gradient vector [gc | gw] and the Adam step on the device
    MSC_CUDA(cudaMemcpyAsync(gall, f.gc, sizeof(double2) * (L + 1), cudaMemcpyDeviceToDevice, st));
    MSC_CUDA(cudaMemcpyAsync(gall + nc, f.gw, sizeof(double2) * nb, cudaMemcpyDeviceToDevice, st));
    ++t;
    const float bc1 = 1.f - std::pow(0.9f, (float)t), bc2 = 1.f - std::pow(0.999f, (float)t);
    k_tr_adam<<<nblk(np), 256, 0, st>>>(pd, gall, md, vd, np, (float)lr, 0.9f, 0.999f, 1e-8f, bc1, bc2);
    ::msc::note_launch();
    MSC_CUDA(cudaGetLastError());
  }
  MSC_CUDA(cudaMemcpyAsync(p.data(), pd, sizeof(float) * np, cudaMemcpyDeviceToHost, st));
  MSC_CUDA(cudaMemcpyAsync(m.data(), md, sizeof(float) * np, cudaMemcpyDeviceToHost, st));
  MSC_CUDA(cudaMemcpyAsync(v.data(), vd, sizeof(float) * np, cudaMemcpyDeviceToHost, st));
  MSC_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < nc; ++i) coef[i] = p[i];
  for (int i = 0; i < 2 * nb; ++i) w[i] = p[nc + i];
  for (int i = 0; i < np; ++i) {
    adam[i] = m[i];
    adam[np + i] = v[i];
  }
  adam[2 * np] = (double)t;
  return MSC_OK;
}

}  // extern "C"
