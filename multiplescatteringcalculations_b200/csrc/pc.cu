// Near-field polynomial preconditioner (pc.cuh): extraction of the 27 stencil
// blocks from the spatial kernel of the G0 build, and the stencil kernels.
//
// One stencil launch computes, for a field x (SoA, scaled by *scale when given),
//   h = S x = G_nn (T0 x)                       (written when h != null)
//   acc = c0 x + ch h  (init)   or   acc += ch h
// A block stages tau = T0 x on its tile plus a one-voxel halo in shared memory
// (zero outside the slab) and each thread accumulates the 27 x 81 complex
// products of its voxels (the self offset holds zero for G_nn and a learned
// pointwise block for a corrected layer). In complex64 the blocks are a __grid_constant__ kernel
// parameter, so every FMA takes its block entry from the constant bank.
#include <vector>

#include "mv_common.cuh"
#include "pc.cuh"

namespace msc {

// index of entry (i, j), i <= j, in the 45-entry symmetric form (row-major upper triangle)
__host__ __device__ inline int sym_index(int i, int j) { return i * 9 - i * (i - 1) / 2 + (j - i); }

// out[o][a][b] = K_ab at offset o, read from the spatial kernel K[e][z][y][x] (values
// times `scale`, (K D)_ij for the 45-entry form), in physical units.
__global__ void k_nf_extract(const double2* __restrict__ K, Geo g, int E, double inv_scale, double2* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NF_OFFS * 81) return;
  const int o = t / 81, a = (t / 9) % 9, b = t % 9;
  const int dz = o / 9 - 1, dx = (o / 3) % 3 - 1, dy = o % 3 - 1;
  if ((dz == 0 && dx == 0 && dy == 0) || (dz != 0 && g.Nz < 2) || (dx != 0 && g.M < 2) || (dy != 0 && g.M < 2)) {
    out[t] = make_double2(0.0, 0.0);
    return;
  }
  const long long npts = (long long)g.Lz * g.Ly * g.Lx;
  const long long gid =
      ((long long)((dz + g.Lz) % g.Lz) * g.Ly + (dy + g.Ly) % g.Ly) * g.Lx + (dx + g.Lx) % g.Lx;
  double2 v;
  if (E == 81) {
    v = K[(size_t)(a * 9 + b) * npts + gid];
  } else {
    v = K[(size_t)sym_index(min(a, b), max(a, b)) * npts + gid];
    if (b >= 6) v = 0.5 * v;  // K_ab = (K D)_ab / D_b
  }
  out[t] = inv_scale * v;
}

int nearfield_extract(msc_plan* pl, const double2* Ks, double scale) {
  if (!pl->nf) pl->nf = new NearField();
  NearField* nf = pl->nf;
  MSC_TRY(dalloc(pl, nf->g64_dev, sizeof(double2) * (size_t)(NF_MAXL + 1) * NF_OFFS * 81));
  double2* dst = (double2*)nf->g64_dev.p;
  k_nf_extract<<<ceil_div(NF_OFFS * 81, 256), 256, 0, pl->stream>>>(Ks, pl->g, pl->E, 1.0 / scale, dst);
  ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  nf->g64.resize((size_t)NF_OFFS * 81);
  MSC_CUDA(cudaMemcpyAsync(nf->g64.data(), dst, sizeof(double2) * NF_OFFS * 81, cudaMemcpyDeviceToHost, pl->stream));
  MSC_CUDA(cudaStreamSynchronize(pl->stream));
  nf->ready = true;
  nf->dirty = true;
  return MSC_OK;
}

// ---- stencil ------------------------------------------------------------------------------
template <typename T> struct NFTile;
template <> struct NFTile<float> {  // 256 threads, two voxels each along z
  static constexpr int TZ = 4, TX = 8, TY = 16, VPT = 2;
};
template <> struct NFTile<double> {
  static constexpr int TZ = 2, TX = 8, TY = 16, VPT = 1;
};

template <typename T, typename GF>
__device__ __forceinline__ void nf_body(const cx<T>* __restrict__ x, const double* scale, const cx<T>* __restrict__ t4,
                                        cx<T>* __restrict__ h, cx<T>* __restrict__ acc, cx<T> ch, cx<T> c0, int init,
                                        GF gf, const Geo& g) {
  using C = cx<T>;
  using TL = NFTile<T>;
  constexpr int TZ = TL::TZ, TX = TL::TX, TY = TL::TY, VPT = TL::VPT;
  constexpr int HZ = TZ + 2, HX = TX + 2, HY = TY + 2, HALO = HZ * HX * HY;
  constexpr int NT = (TZ / VPT) * TX * TY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tau = reinterpret_cast<C*>(smem_raw);  // [9][HALO]
  const int tid = threadIdx.x;
  const int nxb = (g.M + TX - 1) / TX;
  const int y0 = blockIdx.x * TY, x0 = (blockIdx.y % nxb) * TX, z0 = (blockIdx.y / nxb) * TZ;
  const T s = scale ? (T)(*scale) : (T)1;
  const int nsite = g.nsite;
  for (int i = tid; i < HALO; i += NT) {
    const int hy = i % HY, hx = (i / HY) % HX, hz = i / (HY * HX);
    const int z = z0 + hz - 1, xx = x0 + hx - 1, y = y0 + hy - 1;
    C v[9];
    if (z >= 0 && z < g.Nz && xx >= 0 && xx < g.M && y >= 0 && y < g.M) {
      const int site = (z * g.M + xx) * g.M + y;
      C xv[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) xv[c] = x[(size_t)c * nsite + site];
      const C tu = t4[site], tl = t4[(size_t)nsite + site], td = t4[(size_t)2 * nsite + site],
              ts = t4[(size_t)3 * nsite + site];
      const C tr = xv[3] + xv[4] + xv[5];
#pragma unroll
      for (int c = 0; c < 3; ++c) v[c] = s * (tu * xv[c]);
#pragma unroll
      for (int c = 3; c < 6; ++c) v[c] = s * (tl * tr + td * xv[c]);
#pragma unroll
      for (int c = 6; c < 9; ++c) v[c] = s * (ts * xv[c]);
    } else {
#pragma unroll
      for (int c = 0; c < 9; ++c) v[c] = czero<C>();
    }
#pragma unroll
    for (int c = 0; c < 9; ++c) tau[c * HALO + i] = v[c];
  }
  __syncthreads();
  const int vy = tid % TY, vx = (tid / TY) % TX, vz0 = (tid / (TY * TX)) * VPT;
  C out[VPT][9];
#pragma unroll
  for (int p = 0; p < VPT; ++p)
#pragma unroll
    for (int a = 0; a < 9; ++a) out[p][a] = czero<C>();
#pragma unroll
  for (int o = 0; o < NF_OFFS; ++o) {
    const int dz = o / 9 - 1, dx = (o / 3) % 3 - 1, dy = o % 3 - 1;
#pragma unroll
    for (int p = 0; p < VPT; ++p) {
      // source voxel v - o in halo coordinates
      const int hi = ((vz0 + p + 1 - dz) * HX + (vx + 1 - dx)) * HY + (vy + 1 - dy);
      C tb[9];
#pragma unroll
      for (int b = 0; b < 9; ++b) tb[b] = tau[b * HALO + hi];
#pragma unroll
      for (int a = 0; a < 9; ++a)
#pragma unroll
        for (int b = 0; b < 9; ++b) fma_(out[p][a], gf(o * 81 + a * 9 + b), tb[b]);
    }
  }
  const int yy = y0 + vy, xx = x0 + vx;
  if (yy >= g.M || xx >= g.M) return;
#pragma unroll
  for (int p = 0; p < VPT; ++p) {
    const int z = z0 + vz0 + p;
    if (z >= g.Nz) continue;
    const int site = (z * g.M + xx) * g.M + yy;
#pragma unroll
    for (int a = 0; a < 9; ++a) {
      const size_t e = (size_t)a * nsite + site;
      if (h) h[e] = out[p][a];
      if (init) {
        const C xv = s * x[e];
        acc[e] = c0 * xv + ch * out[p][a];
      } else {
        acc[e] = acc[e] + ch * out[p][a];
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_nf32(const float2* __restrict__ x, const double* scale,
                                              const float2* __restrict__ t4, float2* __restrict__ h,
                                              float2* __restrict__ acc, float2 ch, float2 c0, int init,
                                              const __grid_constant__ NFStencil32 S, Geo g, const int* done) {
  if (done && *done) return;
  nf_body<float>(x, scale, t4, h, acc, ch, c0, init, [&](int i) { return S.g[i]; }, g);
}

__global__ void __launch_bounds__(256) k_nf64(const double2* __restrict__ x, const double* scale,
                                              const double2* __restrict__ t4, double2* __restrict__ h,
                                              double2* __restrict__ acc, double2 ch, double2 c0, int init,
                                              const double2* __restrict__ G, Geo g, const int* done) {
  if (done && *done) return;
  nf_body<double>(x, scale, t4, h, acc, ch, c0, init, [&](int i) { return __ldg(G + i); }, g);
}

// Rebuild the per-layer blocks g64 + dg[l] (complex64 parameters, complex128 device copy).
int nearfield_refresh(msc_plan* pl) {
  NearField* nf = pl->nf;
  if (!nf->dirty) return MSC_OK;
  const int L = std::max(1, std::min(nf->L, NF_MAXL));
  std::vector<double2> all((size_t)L * NF_OFFS * 81);
  nf->s32.resize(L);
  for (int l = 0; l < L; ++l) {
    for (int i = 0; i < NF_OFFS * 81; ++i) {
      double2 v = nf->g64[i];
      if (!nf->dg.empty()) v = v + nf->dg[(size_t)l * NF_OFFS * 81 + i];
      all[(size_t)l * NF_OFFS * 81 + i] = v;
      nf->s32[l].g[i] = make_float2((float)v.x, (float)v.y);
    }
  }
  MSC_CUDA(cudaMemcpyAsync(nf->g64_dev.p, all.data(), sizeof(double2) * all.size(), cudaMemcpyHostToDevice,
                           pl->stream));
  MSC_CUDA(cudaStreamSynchronize(pl->stream));
  nf->dirty = false;
  ++pl->gen;
  return MSC_OK;
}

template <typename T>
int nearfield_apply(msc_plan* pl, const cx<T>* v, const double* scale, cx<T>* z, const int* done) {
  NearField* nf = pl->nf;
  if (!nf || !nf->ready) {
    set_error("the near-field preconditioner needs build_g0 first");
    return MSC_ERR_STATE;
  }
  MSC_TRY(nearfield_refresh(pl));
  const Geo& g = pl->g;
  using TL = NFTile<T>;
  const size_t n = field_elems(g);
  DBuf& tb = sizeof(T) == 8 ? nf->tmp64 : nf->tmp32;
  MSC_TRY(dalloc(pl, tb, 2 * sizeof(cx<T>) * n));
  cx<T>* hbuf[2] = {(cx<T>*)tb.p, (cx<T>*)tb.p + n};
  const cx<T>* t4 = (const cx<T>*)(sizeof(T) == 8 ? pl->t4_64.p : pl->t4_32.p);
  const int nxb = (g.M + TL::TX - 1) / TL::TX;
  dim3 grid((unsigned)((g.M + TL::TY - 1) / TL::TY), (unsigned)(nxb * ((g.Nz + TL::TZ - 1) / TL::TZ)));
  const size_t sm = sizeof(cx<T>) * 9 * (TL::TZ + 2) * (TL::TX + 2) * (TL::TY + 2);
  const int L = std::max(1, std::min(nf->L, NF_MAXL));
  const void* kern = sizeof(T) == 8 ? (const void*)k_nf64 : (const void*)k_nf32;
  MSC_CUDA(prep_kernel(kern));
  const cx<T> c0 = mk<T>((T)nf->coef[0].x, (T)nf->coef[0].y);
  const cx<T>* in = v;
  const double* sc = scale;
  for (int l = 1; l <= L; ++l) {
    cx<T>* h = l < L ? hbuf[l & 1] : nullptr;
    const cx<T> ch = mk<T>((T)nf->coef[l].x, (T)nf->coef[l].y);
    const int init = l == 1 ? 1 : 0;
    if constexpr (sizeof(T) == 4) {
      k_nf32<<<grid, 256, sm, pl->stream>>>((const float2*)in, sc, (const float2*)t4, (float2*)h, (float2*)z,
                                             make_float2((float)ch.x, (float)ch.y),
                                             make_float2((float)c0.x, (float)c0.y), init, nf->s32[l - 1], g, done);
    } else {
      k_nf64<<<grid, 256, sm, pl->stream>>>((const double2*)in, sc, (const double2*)t4, (double2*)h, (double2*)z,
                                             make_double2((double)ch.x, (double)ch.y),
                                             make_double2((double)c0.x, (double)c0.y), init,
                                             (const double2*)nf->g64_dev.p + (size_t)(l - 1) * NF_OFFS * 81, g, done);
    }
    ::msc::note_launch();
    MSC_CUDA(cudaGetLastError());
    in = h;
    sc = nullptr;
  }
  return MSC_OK;
}

template int nearfield_apply<float>(msc_plan*, const float2*, const double*, float2*, const int*);
template int nearfield_apply<double>(msc_plan*, const double2*, const double*, double2*, const int*);

}  // namespace msc
