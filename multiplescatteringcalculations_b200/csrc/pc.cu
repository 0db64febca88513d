// Near-field polynomial preconditioner (pc.cuh): extraction of the 27 stencil
// blocks from the spatial kernel of the G0 build, and the stencil kernels.
//
// One stencil launch computes, for a field x (SoA, scaled by *scale when given),
//   h = S x = G_nn (T0 x)                       (written when h != null)
//   acc = c0 x + ch h  (init)   or   acc += ch h
// A block stages tau = T0 x on its tile plus a one-voxel halo in shared memory
// (zero outside the slab) and each thread accumulates the 27 x 81 complex
// products of its voxels (the self offset holds zero for G_nn and a learned
// pointwise block for a corrected layer). The block's 27 x 81 blocks are staged in
// shared memory next to the halo tile and read as broadcasts.
//
// Mirror symmetry: where the offset has a zero component along an axis, the block is
// invariant under that axis' reflection, so its entries odd under it vanish
// (K_ab = 0 when dof_parity(a) ^ dof_parity(b) has the axis' bit). The kernel skips
// those entries at compile time (1338 of the 2187 products remain); block corrections
// are applied within the same pattern.
#include <type_traits>
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

int nearfield_extract(msc_plan* pl, const double2* Ks, double scale, const Geo* box) {
  if (!pl->nf) pl->nf = new NearField();
  NearField* nf = pl->nf;
  MSC_TRY(dalloc(pl, nf->g64_dev, sizeof(double2) * (size_t)(NF_MAXL + 1) * NF_OFFS * 81));
  MSC_TRY(dalloc(pl, nf->g32_dev, sizeof(float2) * (size_t)(NF_MAXL + 1) * NF_OFFS * 81));
  MSC_TRY(dalloc(pl, nf->g16_dev, sizeof(__nv_bfloat162) * (size_t)(NF_MAXL + 1) * NF_OFFS * 81));
  MSC_TRY(dalloc(pl, nf->gtc_dev, (size_t)NF_MAXL * NF_TC_LAYER_BYTES));
  double2* dst = (double2*)nf->g64_dev.p;
  k_nf_extract<<<ceil_div(NF_OFFS * 81, 256), 256, 0, pl->stream>>>(Ks, box ? *box : pl->g, pl->E, 1.0 / scale, dst);
  ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  if (!nf->pin) MSC_CUDA(cudaMallocHost((void**)&nf->pin, sizeof(double2) * NF_OFFS * 81));
  if (!nf->ev) MSC_CUDA(cudaEventCreateWithFlags(&nf->ev, cudaEventDisableTiming));
  MSC_CUDA(cudaMemcpyAsync(nf->pin, dst, sizeof(double2) * NF_OFFS * 81, cudaMemcpyDeviceToHost, pl->stream));
  MSC_CUDA(cudaEventRecord(nf->ev, pl->stream));
  nf->host_pending = true;
  nf->ready = true;
  nf->dirty = true;
  return MSC_OK;
}

int nf_host_sync(const msc_plan* pl) {
  NearField* nf = pl->nf;
  if (!nf || !nf->host_pending) return MSC_OK;
  MSC_CUDA(cudaEventSynchronize(nf->ev));
  nf->g64.assign(nf->pin, nf->pin + (size_t)NF_OFFS * 81);
  nf->host_pending = false;
  return MSC_OK;
}

// ---- stencil ------------------------------------------------------------------------------
// Tile of 2 layers x 8 x 16 voxels, one voxel per thread: 256 threads; a 64 x 64 x 16
// slab gives 256 blocks, one wave at two blocks per SM (halo tile 4 x 10 x 18 voxels).
template <typename T> struct NFTile {
  static constexpr int TZ = 2, TX = 8, TY = 16, VPT = 1;
  static constexpr int NT = (TZ / VPT) * TX * TY;
};

template <typename T>
__device__ __forceinline__ void nf_body(const cx<T>* __restrict__ x, const double* scale, const cx<T>* __restrict__ t4,
                                        cx<T>* __restrict__ h, cx<T>* __restrict__ acc, cx<T> ch, cx<T> c0, int init,
                                        const cx<T>* __restrict__ G, const __nv_bfloat162* __restrict__ G16,
                                        const Geo& g) {
  using C = cx<T>;
  using TL = NFTile<T>;
  constexpr int TZ = TL::TZ, TX = TL::TX, TY = TL::TY, VPT = TL::VPT;
  constexpr int HZ = TZ + 2, HX = TX + 2, HY = TY + 2, HALO = HZ * HX * HY;
  constexpr int NT = (TZ / VPT) * TX * TY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // blocks: complex128 as they are; complex64 as pairs (g.x, g.x, g.y, g.y) for the
  // paired FP32 FMAs
  using GE = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  GE* Gs = reinterpret_cast<GE*>(smem_raw);                  // [27][81]
  C* tau = reinterpret_cast<C*>(Gs + NF_OFFS * 81);          // [9][HALO]
  const int tid = threadIdx.x;
  for (int i = tid; i < NF_OFFS * 81; i += NT) {
    if constexpr (sizeof(T) == 4) {
      const float2 v = G16 ? __bfloat1622float2(G16[i]) : __ldg(G + i);  // BF16 or FP32 weights
      Gs[i] = make_float4(v.x, v.x, v.y, v.y);
    } else {
      Gs[i] = __ldg(G + i);
    }
  }
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
    const int zmask = (dx == 0 ? 1 : 0) | (dy == 0 ? 2 : 0) | (dz == 0 ? 4 : 0);
#pragma unroll
    for (int p = 0; p < VPT; ++p) {
      // source voxel v - o in halo coordinates
      const int hi = ((vz0 + p + 1 - dz) * HX + (vx + 1 - dx)) * HY + (vy + 1 - dy);
      C tb[9];
#pragma unroll
      for (int b = 0; b < 9; ++b) tb[b] = tau[b * HALO + hi];
      if constexpr (sizeof(T) == 4) {
        float2 tr[9];
#pragma unroll
        for (int b = 0; b < 9; ++b) tr[b] = make_float2(-tb[b].y, tb[b].x);
#pragma unroll
        for (int a = 0; a < 9; ++a)
#pragma unroll
          for (int b = 0; b < 9; ++b) {
            if ((dof_parity(a) ^ dof_parity(b)) & zmask) continue;  // zero by symmetry
            const float4 m = Gs[o * 81 + a * 9 + b];
            out[p][a] = __ffma2_rn(make_float2(m.x, m.y), tb[b], out[p][a]);
            out[p][a] = __ffma2_rn(make_float2(m.z, m.w), tr[b], out[p][a]);
          }
      } else {
#pragma unroll
        for (int a = 0; a < 9; ++a)
#pragma unroll
          for (int b = 0; b < 9; ++b) {
            if ((dof_parity(a) ^ dof_parity(b)) & zmask) continue;  // zero by symmetry
            fma_(out[p][a], Gs[o * 81 + a * 9 + b], tb[b]);
          }
      }
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

__global__ void __launch_bounds__(256, 2) k_nf32(const float2* __restrict__ x, const double* scale,
                                              const float2* __restrict__ t4, float2* __restrict__ h,
                                              float2* __restrict__ acc, float2 ch, float2 c0, int init,
                                              const float2* __restrict__ G, const __nv_bfloat162* __restrict__ G16,
                                              Geo g, const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  nf_body<float>(x, scale, t4, h, acc, ch, c0, init, G, G16, g);
}

__global__ void __launch_bounds__(256) k_nf64(const double2* __restrict__ x, const double* scale,
                                              const double2* __restrict__ t4, double2* __restrict__ h,
                                              double2* __restrict__ acc, double2 ch, double2 c0, int init,
                                              const double2* __restrict__ G, Geo g, const int* done) {
  pdl_wait();
  pdl_trigger();
  if (done && *done) return;
  nf_body<double>(x, scale, t4, h, acc, ch, c0, init, G, nullptr, g);
}

// Upload the per-layer blocks g64 + dg[l] (complex128 and complex64) to the device.
int nearfield_refresh(msc_plan* pl) {
  NearField* nf = pl->nf;
  if (!nf->dirty) return MSC_OK;
  MSC_TRY(nf_host_sync(pl));
  const int L = std::max(1, std::min(nf->L, NF_MAXL));
  const size_t nb = (size_t)L * NF_OFFS * 81;
  nf->h64.resize(nb);
  nf->h32.resize(nb);
  nf->h16.resize(nb);
  for (int l = 0; l < L; ++l)
    for (int i = 0; i < NF_OFFS * 81; ++i) {
      double2 v = nf->g64[i];
      if (!nf->dg.empty()) v = v + nf->dg[(size_t)l * NF_OFFS * 81 + i];
      nf->h64[(size_t)l * NF_OFFS * 81 + i] = v;
      nf->h32[(size_t)l * NF_OFFS * 81 + i] = make_float2((float)v.x, (float)v.y);
      nf->h16[(size_t)l * NF_OFFS * 81 + i] = __floats2bfloat162_rn((float)v.x, (float)v.y);
    }
  MSC_CUDA(cudaMemcpyAsync(nf->g64_dev.p, nf->h64.data(), sizeof(double2) * nb, cudaMemcpyHostToDevice, pl->stream));
  MSC_CUDA(cudaMemcpyAsync(nf->g32_dev.p, nf->h32.data(), sizeof(float2) * nb, cudaMemcpyHostToDevice, pl->stream));
  MSC_CUDA(cudaMemcpyAsync(nf->g16_dev.p, nf->h16.data(), sizeof(__nv_bfloat162) * nb, cudaMemcpyHostToDevice,
                           pl->stream));
  nf->htc.resize((size_t)L * NF_TC_LAYER_BYTES / 2);
  for (int l = 0; l < L; ++l)
    nf_tc_pack_layer(nf->h16.data() + (size_t)l * NF_OFFS * 81, nf->htc.data() + (size_t)l * NF_TC_LAYER_BYTES / 2);
  MSC_CUDA(cudaMemcpyAsync(nf->gtc_dev.p, nf->htc.data(), (size_t)L * NF_TC_LAYER_BYTES, cudaMemcpyHostToDevice,
                           pl->stream));
  MSC_CUDA(cudaStreamSynchronize(pl->stream));
  nf->dirty = false;
  return MSC_OK;
}

template <typename T>
static int nearfield_apply_one(msc_plan* pl, const cx<T>* v, const double* scale, cx<T>* z, const int* done) {
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
  const size_t sm = (size_t)NF_OFFS * 81 * (sizeof(T) == 4 ? 16 : 16) +
                    sizeof(cx<T>) * 9 * (TL::TZ + 2) * (TL::TX + 2) * (TL::TY + 2);
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
      if (nf->wbf16 == MSC_NF_WEIGHTS_BF16_TC) {
        // the layer on the tensor cores
        MSC_TRY(launch_nf_tc(pl, (const float2*)in, sc, (const float2*)t4, (float2*)h, (float2*)z,
                             make_float2((float)ch.x, (float)ch.y), make_float2((float)c0.x, (float)c0.y), init,
                             (const unsigned char*)nf->gtc_dev.p + (size_t)(l - 1) * NF_TC_LAYER_BYTES, done));
        in = h;
        sc = nullptr;
        continue;
      }
      k_nf32<<<grid, TL::NT, sm, pl->stream>>>((const float2*)in, sc, (const float2*)t4, (float2*)h, (float2*)z,
                                             make_float2((float)ch.x, (float)ch.y),
                                             make_float2((float)c0.x, (float)c0.y), init,
                                             (const float2*)nf->g32_dev.p + (size_t)(l - 1) * NF_OFFS * 81,
                                             nf->wbf16 ? (const __nv_bfloat162*)nf->g16_dev.p + (size_t)(l - 1) * NF_OFFS * 81
                                                       : nullptr,
                                             g, done);
    } else {
      k_nf64<<<grid, TL::NT, sm, pl->stream>>>((const double2*)in, sc, (const double2*)t4, (double2*)h, (double2*)z,
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

// z = P v for each of the plan's pl->nrhs fields (one after the other)
template <typename T>
int nearfield_apply(msc_plan* pl, const cx<T>* v, const double* scale, cx<T>* z, const int* done) {
  const size_t nf = field_elems(pl->g);
  for (int r = 0; r < pl->nrhs; ++r)
    MSC_TRY(nearfield_apply_one<T>(pl, v + (size_t)r * nf, scale, z + (size_t)r * nf, done));
  return MSC_OK;
}

template int nearfield_apply<float>(msc_plan*, const float2*, const double*, float2*, const int*);
template int nearfield_apply<double>(msc_plan*, const double2*, const double*, double2*, const int*);

}  // namespace msc
