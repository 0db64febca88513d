// Per-frequency setup on the device: twiddle tables, T0 (4 scalars per voxel),
// the incident plane wave, layout conversions, and the G0 spectrum build.
#include <mutex>
#include <algorithm>
#include <cstring>
#include <cstdlib>

#include "physics.cuh"
#include "mv_common.cuh"
#include "pc.cuh"
#include "plan.cuh"

namespace msc {

template <typename T>
int launch_fft_contig(msc_plan* pl, const cx<T>* in, cx<T>* out, long long nlines, long long G, long long GS,
                      long long stride, int n_in, int n_out, const FftPlan1D& f, const cx<T>* tw, int dir,
                      const int* done);

// ---- twiddles ------------------------------------------------------------------------
__global__ void k_twiddles(double2* t64, float2* t32, int L) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L) return;
  double s, c;
  sincospi(2.0 * (double)t / (double)L, &s, &c);
  t64[t] = make_double2(c, -s);
  t32[t] = make_float2((float)c, (float)-s);
}

__constant__ float2 c_tw256[256];
__constant__ double2 c_tw256d[256];

// Fill the constant twiddle tables (complex64 and complex128) of the current device once
// (k_twiddles at L = 256 into scratch buffers, then device-to-device copies to the symbols).
static int ensure_const_twiddles(msc_plan* pl) {
  static std::mutex mu;
  static bool ready[64] = {};
  int dev = 0;
  MSC_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64) {
    set_error("device index %d out of range", dev);
    return MSC_ERR_INVALID;
  }
  if (ready[dev]) return MSC_OK;
  DBuf t64, t32;
  int s = dalloc(pl, t64, sizeof(double2) * 256);
  if (s == MSC_OK) s = dalloc(pl, t32, sizeof(float2) * 256);
  if (s == MSC_OK) {
    k_twiddles<<<2, 128, 0, pl->stream>>>((double2*)t64.p, (float2*)t32.p, 256);
    ::msc::note_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyToSymbolAsync(c_tw256, t32.p, sizeof(float2) * 256, 0, cudaMemcpyDeviceToDevice, pl->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyToSymbolAsync(c_tw256d, t64.p, sizeof(double2) * 256, 0, cudaMemcpyDeviceToDevice, pl->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(pl->stream);
    if (e != cudaSuccess) {
      set_error("constant twiddle table: %s", cudaGetErrorString(e));
      s = MSC_ERR_CUDA;
    }
  }
  dfree(pl, t64);
  dfree(pl, t32);
  if (s == MSC_OK) ready[dev] = true;
  return s;
}

int build_twiddles(msc_plan* pl) {
  MSC_TRY(ensure_const_twiddles(pl));
  const int Lz = pl->g.Lz, Lxy = pl->g.Lx;
  MSC_TRY(dalloc(pl, pl->tw64_z, sizeof(double2) * Lz));
  MSC_TRY(dalloc(pl, pl->tw32_z, sizeof(float2) * Lz));
  MSC_TRY(dalloc(pl, pl->tw64_xy, sizeof(double2) * Lxy));
  MSC_TRY(dalloc(pl, pl->tw32_xy, sizeof(float2) * Lxy));
  k_twiddles<<<ceil_div(Lz, 128), 128, 0, pl->stream>>>((double2*)pl->tw64_z.p, (float2*)pl->tw32_z.p, Lz); ::msc::note_launch();
  k_twiddles<<<ceil_div(Lxy, 128), 128, 0, pl->stream>>>((double2*)pl->tw64_xy.p, (float2*)pl->tw32_xy.p, Lxy); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}

// ---- T0 --------------------------------------------------------------------------------
__global__ void k_t0(const double* __restrict__ dl, const double* __restrict__ dm, const double* __restrict__ dr,
                     double2* __restrict__ t64, float2* __restrict__ t32, int nsite, double omega, double a,
                     CubeConst cc) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsite) return;
  double2 t[4];
  t0_voxel(cc, omega, a, dl[s], dm[s], dr[s], t);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    t64[(size_t)q * nsite + s] = t[q];
    t32[(size_t)q * nsite + s] = make_float2((float)t[q].x, (float)t[q].y);
  }
}

int launch_t0(msc_plan* pl, const double* dlam, const double* dmu, const double* drho, double omega) {
  const Geo& g = pl->g;
  MSC_TRY(dalloc(pl, pl->t4_64, sizeof(double2) * 4 * g.nsite));
  MSC_TRY(dalloc(pl, pl->t4_32, sizeof(float2) * 4 * g.nsite));
  const CubeConst cc = cube_constants(omega, pl->desc.a, pl->desc.alpha, pl->desc.beta, pl->desc.rho);
  k_t0<<<ceil_div(g.nsite, 256), 256, 0, pl->stream>>>(dlam, dmu, drho, (double2*)pl->t4_64.p, (float2*)pl->t4_32.p,
                                                       g.nsite, omega, pl->desc.a, cc); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}

// ---- incident plane wave (slab_scattering.py:426-478) ---------------------------------
struct IncVec {
  double kh[3], pol[3], k;
};

__global__ void k_incident(double2* ref_out, double2* soa_out, int M, int Nz, double a, IncVec iv, int demod,
                           double kx, double ky) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int nsite = Nz * M * M;
  if (s >= nsite) return;
  const int j = s % M, i = (s / M) % M, n = s / (M * M);
  const double d = 2.0 * a;
  const double z = (n + 0.5) * d, x = (i - (M - 1) / 2.0) * d, y = (j - (M - 1) / 2.0) * d;
  double ph = iv.k * (iv.kh[0] * z + iv.kh[1] * x + iv.kh[2] * y);
  if (demod) ph -= kx * x + ky * y;
  double sp, cp;
  sincos(ph, &sp, &cp);
  const double2 e = make_double2(cp, sp);
  double2 v[9];
  for (int q = 0; q < 3; ++q) v[q] = make_double2(iv.pol[q], 0.0);
  // eps_pq = (i k / 2)(kh_p pol_q + pol_p kh_q); Voigt with engineering shear
  for (int al = 0; al < 6; ++al) {
    const int p = voigt_p(al), q = voigt_q(al);
    double re = 0.5 * iv.k * (iv.kh[p] * iv.pol[q] + iv.pol[p] * iv.kh[q]);
    if (p != q) re *= 2.0;
    v[3 + al] = make_double2(0.0, re);
  }
  for (int c = 0; c < 9; ++c) {
    const double2 w = v[c] * e;
    if (ref_out) ref_out[(size_t)s * 9 + c] = w;
    if (soa_out) soa_out[(size_t)c * nsite + s] = w;
  }
}

int launch_incident(msc_plan* pl, double omega, const double* k_hat, int wave, double2* ref_out, double2* soa_out,
                    bool demod) {
  const double nrm = sqrt(k_hat[0] * k_hat[0] + k_hat[1] * k_hat[1] + k_hat[2] * k_hat[2]);
  if (!(nrm > 0)) {
    set_error("k_hat must be a nonzero 3-vector");
    return MSC_ERR_INVALID;
  }
  IncVec iv;
  for (int q = 0; q < 3; ++q) iv.kh[q] = k_hat[q] / nrm;
  if (wave == MSC_WAVE_P) {
    iv.k = omega / pl->desc.alpha;
    for (int q = 0; q < 3; ++q) iv.pol[q] = iv.kh[q];
  } else if (wave == MSC_WAVE_S) {
    iv.k = omega / pl->desc.beta;
    // SV: cross = k_hat x z_hat; pol = cross x k_hat normalised; vertical incidence -> x
    const double zh[3] = {1, 0, 0};
    double cr[3] = {iv.kh[1] * zh[2] - iv.kh[2] * zh[1], iv.kh[2] * zh[0] - iv.kh[0] * zh[2],
                    iv.kh[0] * zh[1] - iv.kh[1] * zh[0]};
    const double cn = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    if (cn < 1e-10) {
      iv.pol[0] = 0; iv.pol[1] = 1; iv.pol[2] = 0;
    } else {
      double p[3] = {cr[1] * iv.kh[2] - cr[2] * iv.kh[1], cr[2] * iv.kh[0] - cr[0] * iv.kh[2],
                     cr[0] * iv.kh[1] - cr[1] * iv.kh[0]};
      const double pn = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
      for (int q = 0; q < 3; ++q) iv.pol[q] = p[q] / pn;
    }
  } else {
    set_error("wave_type must be 'P' or 'S', got code %d", wave);
    return MSC_ERR_INVALID;
  }
  const Geo& g = pl->g;
  k_incident<<<ceil_div(g.nsite, 256), 256, 0, pl->stream>>>(ref_out, soa_out, g.M, g.Nz, pl->desc.a, iv, demod ? 1 : 0,
                                                            pl->kpar[0], pl->kpar[1]); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}

// ---- layout conversion (reference [site][9] <-> SoA [9][site]) -------------------------
template <typename Tin, typename Tout>
__global__ void k_ref_to_soa(const cx<Tin>* __restrict__ in, cx<Tout>* __restrict__ out, int nsite) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 9LL * nsite) return;
  const int s = (int)(e / 9), c = (int)(e % 9);
  const cx<Tin> v = in[e];
  out[(size_t)c * nsite + s] = mk<Tout>((Tout)v.x, (Tout)v.y);
}
template <typename Tin, typename Tout>
__global__ void k_soa_to_ref(const cx<Tin>* __restrict__ in, cx<Tout>* __restrict__ out, int nsite) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 9LL * nsite) return;
  const int s = (int)(e / 9), c = (int)(e % 9);
  const cx<Tin> v = in[(size_t)c * nsite + s];
  out[e] = mk<Tout>((Tout)v.x, (Tout)v.y);
}
template <typename Tin, typename Tout>
int launch_ref_to_soa(msc_plan* pl, const cx<Tin>* in, cx<Tout>* out) {
  const long long n = 9LL * pl->g.nsite;
  k_ref_to_soa<Tin, Tout><<<ceil_div(n, 256), 256, 0, pl->stream>>>(in, out, pl->g.nsite); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}
template <typename Tin, typename Tout>
int launch_soa_to_ref(msc_plan* pl, const cx<Tin>* in, cx<Tout>* out) {
  const long long n = 9LL * pl->g.nsite;
  k_soa_to_ref<Tin, Tout><<<ceil_div(n, 256), 256, 0, pl->stream>>>(in, out, pl->g.nsite); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}
template int launch_ref_to_soa<double, double>(msc_plan*, const double2*, double2*);
template int launch_ref_to_soa<double, float>(msc_plan*, const double2*, float2*);
template int launch_ref_to_soa<float, float>(msc_plan*, const float2*, float2*);
template int launch_soa_to_ref<double, double>(msc_plan*, const double2*, double2*);
template int launch_soa_to_ref<float, float>(msc_plan*, const float2*, float2*);
template int launch_soa_to_ref<float, double>(msc_plan*, const float2*, double2*);

// ---- G0 spectrum -----------------------------------------------------------------------
__global__ void k_va_blocks(double* out, double alpha, double beta, double rho, double omega, int n_orders) {
  const int t = threadIdx.x;
  if (t >= 27 || t == 13) return;
  const int R[3] = {t / 9 - 1, (t / 3) % 3 - 1, t % 3 - 1};
  const int slot = t < 13 ? t : t - 1;
  va_block(R, alpha, beta, rho, omega, n_orders, out + slot * 81);
}

__device__ __forceinline__ int va_slot(int dz, int dx, int dy) {
  const int t = (dz + 1) * 9 + (dx + 1) * 3 + (dy + 1);
  return t < 13 ? t : t - 1;
}

// Lattice offsets of padded index u along an axis of length L for a lattice of n:
// aperiodic: u < n -> u; u > L - n -> u - L; periodic (L == n): u and u - n (u > 0).
__device__ __forceinline__ int axis_offsets(int u, int L, int n, bool periodic, int* o) {
  if (periodic) {
    o[0] = u;
    if (u > 0) { o[1] = u - n; return 2; }
    return 1;
  }
  if (u < n) { o[0] = u; return 1; }
  if (u > L - n) { o[0] = u - L; return 1; }
  return 0;
}

struct G0Params {
  Geo g;
  double d, omega, alpha, beta, rho;
  int periodic, va, E;
  int bloch;
  double kx, ky;   // Bloch wavevector (rad/m)
  double scale;    // 1/(Lz Lx Ly)
};

// Spatial kernel at padded point (z, y, x), all E entries: the sum over the images
// of the point (or volume-averaged) propagator; SYM stores (K D)_ij for i <= j.
// One thread per point; Ks[e][point].
__global__ void __launch_bounds__(128) k_g0_spatial(double2* __restrict__ Ks, const double* __restrict__ vab,
                                                    G0Params p) {
  const Geo& g = p.g;
  const long long npts = (long long)g.Lz * g.Ly * g.Lx;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= npts) return;
  const int x = (int)(gid % g.Lx);
  const int y = (int)((gid / g.Lx) % g.Ly);
  const int z = (int)(gid / ((long long)g.Lx * g.Ly));
  int oz[2], ox[2], oy[2];
  const int nz = axis_offsets(z, g.Lz, g.Nz, false, oz);
  const int nx = axis_offsets(x, g.Lx, g.M, p.periodic, ox);
  const int ny = axis_offsets(y, g.Ly, g.M, p.periodic, oy);
  bool first = true;
  for (int iz = 0; iz < nz; ++iz)
    for (int ix = 0; ix < nx; ++ix)
      for (int iy = 0; iy < ny; ++iy) {
        const int dz = oz[iz], dx = ox[ix], dy = oy[iy];
        if (dz == 0 && dx == 0 && dy == 0) continue;  // self term
        double2 ph = make_double2(p.scale, 0.0);
        if (p.bloch) {
          double s, c;
          sincos(-(p.kx * dx + p.ky * dy) * p.d, &s, &c);
          ph = make_double2(p.scale * c, p.scale * s);
        }
        const bool va = p.va && abs(dz) <= 1 && abs(dx) <= 1 && abs(dy) <= 1;
        const double* vb = va ? vab + va_slot(dz, dx, dy) * 81 : nullptr;
        PointProp pp;
        if (!va) pp.init(dz * p.d, dx * p.d, dy * p.d, p.omega, p.alpha, p.beta, p.rho);
        int e = 0;
        for (int a = 0; a < 9; ++a)
          for (int b = (p.E == 45 ? a : 0); b < 9; ++b, ++e) {
            double2 v = va ? make_double2(vb[a * 9 + b], 0.0) : pp.entry(a, b);
            if (p.E == 45 && b >= 6) v = 2.0 * v;  // (K D)_ij = K_ij D_j
            v = v * ph;
            double2* dst = Ks + (size_t)e * npts + gid;
            if (first) *dst = v;
            else *dst = *dst + v;
          }
        first = false;
      }
  if (first) {  // no offset maps here: zero
    for (int e = 0; e < p.E; ++e) Ks[(size_t)e * npts + gid] = make_double2(0, 0);
  }
}

// The same kernel for a mirror-symmetric spectrum (octant storage): one thread per
// point of the octant z <= Lz/2, y <= Ly/2, x <= Lx/2, evaluated as above and written
// to its mirror images too. Reflecting the axes in f (bit 0 x, 1 y, 2 z) negates the
// image offsets and multiplies entry (a, b) by (-1)^popc((par_a ^ par_b) & f), par the
// DOF parities; the mirror of index u is (L - u) mod L.
__global__ void __launch_bounds__(128) k_g0_spatial_oct(double2* __restrict__ Ks, const double* __restrict__ vab,
                                                        G0Params p) {
  const Geo& g = p.g;
  const long long npts = (long long)g.Lz * g.Ly * g.Lx;
  const int qx = g.Lx / 2 + 1, qy = g.Ly / 2 + 1, qz = g.Lz / 2 + 1;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)qz * qy * qx) return;
  const int x = (int)(gid % qx);
  const int y = (int)((gid / qx) % qy);
  const int z = (int)(gid / ((long long)qx * qy));
  const long long pt = ((long long)z * g.Ly + y) * g.Lx + x;
  int oz[2], ox[2], oy[2];
  const int nz = axis_offsets(z, g.Lz, g.Nz, false, oz);
  const int nx = axis_offsets(x, g.Lx, g.M, p.periodic, ox);
  const int ny = axis_offsets(y, g.Ly, g.M, p.periodic, oy);
  bool first = true;
  for (int iz = 0; iz < nz; ++iz)
    for (int ix = 0; ix < nx; ++ix)
      for (int iy = 0; iy < ny; ++iy) {
        const int dz = oz[iz], dx = ox[ix], dy = oy[iy];
        if (dz == 0 && dx == 0 && dy == 0) continue;  // self term
        const bool va = p.va && abs(dz) <= 1 && abs(dx) <= 1 && abs(dy) <= 1;
        const double* vb = va ? vab + va_slot(dz, dx, dy) * 81 : nullptr;
        PointProp pp;
        if (!va) pp.init(dz * p.d, dx * p.d, dy * p.d, p.omega, p.alpha, p.beta, p.rho);
        int e = 0;
        for (int a = 0; a < 9; ++a)
          for (int b = (p.E == 45 ? a : 0); b < 9; ++b, ++e) {
            double2 v = va ? make_double2(vb[a * 9 + b], 0.0) : pp.entry(a, b);
            if (p.E == 45 && b >= 6) v = 2.0 * v;  // (K D)_ij = K_ij D_j
            v = p.scale * v;
            double2* dst = Ks + (size_t)e * npts + pt;
            if (first) *dst = v;
            else *dst = *dst + v;
          }
        first = false;
      }
  // the mirror images: distinct indices per axis, and the reflections that reach them
  const int mz = z == 0 || 2 * z == g.Lz ? 1 : 2;
  const int my = y == 0 || 2 * y == g.Ly ? 1 : 2;
  const int mx = x == 0 || 2 * x == g.Lx ? 1 : 2;
  int e = 0;
  for (int a = 0; a < 9; ++a)
    for (int b = (p.E == 45 ? a : 0); b < 9; ++b, ++e) {
      double2* base = Ks + (size_t)e * npts;
      const double2 v = first ? make_double2(0, 0) : base[pt];
      if (first) base[pt] = v;
      const int par = dof_parity(a) ^ dof_parity(b);
      for (int rz = 0; rz < mz; ++rz)
        for (int ry = 0; ry < my; ++ry)
          for (int rx = 0; rx < mx; ++rx) {
            const int f = rx | (ry << 1) | (rz << 2);
            if (f == 0) continue;
            const int zz = rz ? g.Lz - z : z, yy = ry ? g.Ly - y : y, xx = rx ? g.Lx - x : x;
            const double sg = (__popc(par & f) & 1) ? -1.0 : 1.0;
            base[((long long)zz * g.Ly + yy) * g.Lx + xx] = make_double2(sg * v.x, sg * v.y);
          }
    }
}

// Aperiodic, mirror-symmetric kernels: the spatial evaluation fused with the x
// transform, so the spatial box (377 MB at 64x64x16) is neither stored nor read back.
// One block per row (z <= Lz/2, y <= Ly/2) of the octant; the E entries in groups of
// G0X_EG lines. Thread x <= Lx/2 evaluates the row's point x (aperiodic: at most one
// image) into a shared tile of Lx points and fills the mirror point Lx - x with the
// entry's x-parity sign; the tile is transformed along x and kx < Hx is stored. Points
// within one cell of the origin also go, with all their mirror images, to the 3x3x3 box
// Kn[e][27] ((d + 3) % 3 per axis) from which the near-field blocks are taken. Only the
// octant rows are stored: the y and z passes read the mirror rows' values through the
// entries' parity signs (launch_fft_strided with a parity mask).
constexpr int G0X_EG = 16;
constexpr int G0X_NT = 256;

// A row point of k_g0_x: the propagator's per-point state (or the VA table slot), shared by
// the threads that evaluate its entries. Padded to an odd number of 16-byte units (the
// struct's alignment), which spreads consecutive points over the shared-memory banks.
struct G0Pt {
  PointProp pp;
  int slot;  // VA table block (-1: the point propagator)
  int has;   // the point has an image (aperiodic: at most one)
  double pad[2];
};
static_assert(sizeof(G0Pt) % 16 == 0 && (sizeof(G0Pt) / 16) % 2 == 1, "odd stride in 16-byte units");

template <bool POW2>
__global__ void __launch_bounds__(G0X_NT, 2) k_g0_x(double2* __restrict__ K, double2* __restrict__ Kn,
                                                 const double* __restrict__ vab, G0Params p, FftPlan1D f,
                                                 const double2* __restrict__ twg) {
  const Geo& g = p.g;
  constexpr int P = G0X_EG + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L = g.Lx;
  double2* tw = reinterpret_cast<double2*>(smem_raw);
  double2* ta = tw + L;
  double2* tb = ta + (size_t)L * P;
  G0Pt* pts = reinterpret_cast<G0Pt*>(tb + (size_t)L * P);
  __shared__ unsigned char ea[81], eb[81], epar[81];
  const int tid = threadIdx.x;
  const int y = blockIdx.x, z = blockIdx.y;
  const int qx = L / 2 + 1;
  for (int t = tid; t < L; t += G0X_NT) tw[t] = twg[t];
  if (tid < p.E) {
    int a = tid / 9, b = tid % 9;
    if (p.E == 45) {  // upper triangle, row by row
      int e = tid;
      a = 0;
      while (e >= 9 - a) {
        e -= 9 - a;
        ++a;
      }
      b = a + e;
    }
    ea[tid] = (unsigned char)a;
    eb[tid] = (unsigned char)b;
    epar[tid] = (unsigned char)(dof_parity(a) ^ dof_parity(b));
  }
  // the row's points x <= Lx/2: one thread each sets up the point's propagator
  {
    int oz[2], oy[2];
    const int nz = axis_offsets(z, g.Lz, g.Nz, false, oz);
    const int ny = axis_offsets(y, g.Ly, g.M, false, oy);
    for (int x = tid; x < qx; x += G0X_NT) {
      int ox[2];
      const int nx = axis_offsets(x, L, g.M, false, ox);
      const bool has = nz == 1 && ny == 1 && nx == 1 && !(oz[0] == 0 && oy[0] == 0 && ox[0] == 0);
      G0Pt& pt = pts[x];
      pt.has = has ? 1 : 0;
      pt.slot = -1;
      if (has) {
        const int dz = oz[0], dy = oy[0], dx = ox[0];
        if (p.va && abs(dz) <= 1 && abs(dx) <= 1 && abs(dy) <= 1) pt.slot = va_slot(dz, dx, dy);
        else pt.pp.init(dz * p.d, dx * p.d, dy * p.d, p.omega, p.alpha, p.beta, p.rho);
      }
    }
  }
  __syncthreads();
  for (int e0 = 0; e0 < p.E; e0 += G0X_EG) {
    const int ne = min(G0X_EG, p.E - e0);
    // every thread: (point, entry) items of the group, points fastest
    for (int it = tid; it < qx * ne; it += G0X_NT) {
      const int q = it / qx, x = it - q * qx;
      const int e = e0 + q;
      const G0Pt& pt = pts[x];
      double2 v = make_double2(0.0, 0.0);
      if (pt.has) {
        const int a = ea[e], b = eb[e];
        v = pt.slot >= 0 ? make_double2(vab[pt.slot * 81 + a * 9 + b], 0.0) : pt.pp.entry(a, b);
        if (p.E == 45 && b >= 6) v = 2.0 * v;  // (K D)_ij = K_ij D_j
        v = p.scale * v;
      }
      const int par = epar[e];
      ta[x * P + q] = v;
      if (x != 0 && 2 * x != L) {
        const double sx = (par & 1) ? -1.0 : 1.0;
        ta[(L - x) * P + q] = make_double2(sx * v.x, sx * v.y);
      }
      if (x <= 1 && y <= 1 && z <= 1)
        for (int rz = 0; rz < (z ? 2 : 1); ++rz)
          for (int ry = 0; ry < (y ? 2 : 1); ++ry)
            for (int rx = 0; rx < (x ? 2 : 1); ++rx) {
              const int fl = rx | (ry << 1) | (rz << 2);
              const double sg = (__popc(par & fl) & 1) ? -1.0 : 1.0;
              const int iz = rz ? 3 - z : z, iy = ry ? 3 - y : y, ix = rx ? 3 - x : x;  // (d + 3) % 3
              Kn[(size_t)e * 27 + (iz % 3 * 3 + iy % 3) * 3 + ix % 3] = make_double2(sg * v.x, sg * v.y);
            }
    }
    __syncthreads();
    const double2* res = fft_tile<-1, POW2>(ta, tb, P, ne, f, tw, tid, G0X_NT);
    for (int it = tid; it < ne * g.Hx; it += G0X_NT) {
      const int q = it / g.Hx, k = it - q * g.Hx;
      K[(((size_t)(e0 + q) * g.Lz + z) * g.Ly + y) * L + k] = res[k * P + q];
    }
    __syncthreads();
  }
}

// The G0 build fuses the spatial evaluation with the x pass where it applies, unless
// MSC_G0_FUSED=0 (the unfused passes, kept for the kernels it does not cover).
static bool g0_fused() {
  const char* e = getenv("MSC_G0_FUSED");
  return !(e && e[0] == '0');
}

static size_t g0x_smem(int L) {
  return sizeof(double2) * ((size_t)L + 2 * (size_t)L * (G0X_EG + 1)) + sizeof(G0Pt) * (size_t)(L / 2 + 1);
}

// Copy the spectrum box kz < Hz, ky < Hy, kx < Hx of the transformed work array
// K[e][z][y][x] into the stored layout of element type T (entries kent<T>): blocked slices of the
// fused z pass for an octant spectrum (zero in the padding and beyond Hx), plain
// [e][kz][ky][kx] for a full one.
template <typename T>
__global__ void k_khat_pack(const double2* __restrict__ K, kent<T>* __restrict__ out, Geo g, int E, ZbzLayout lay,
                            long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int e, kz, ky, kx;
  bool ok = true;
  if (g.oct) {
    const long long blk = i / lay.CS;
    const int r = (int)(i - blk * lay.CS);
    const int xc = (int)(blk % lay.NXC);
    ky = (int)(blk / lay.NXC);
    const int j = r % lay.KX, ekz = r / lay.KX;
    e = ekz / g.Hz;
    kz = ekz % g.Hz;
    kx = xc * lay.KX + j;
    ok = e < E && kx < g.Hx;
  } else {
    long long t = i;
    kx = (int)(t % g.Hx);
    t /= g.Hx;
    ky = (int)(t % g.Hy);
    t /= g.Hy;
    kz = (int)(t % g.Hz);
    e = (int)(t / g.Hz);
  }
  const double2 v = ok ? K[(((long long)e * g.Lz + kz) * g.Ly + ky) * g.Lx + kx] : make_double2(0.0, 0.0);
  out[i] = kent_pack(v, (kent<T>*)nullptr);
}

template <typename T> static int launch_khat_pack(msc_plan* pl, const double2* K, kent<T>* out, int E) {
  const Geo& g = pl->g;
  const long long n = (long long)khat_elems_t<T>(g, E);
  k_khat_pack<T><<<ceil_div(n, 256), 256, 0, pl->stream>>>(K, out, g, E, zbz_layout<T>(g, E), n);
  ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  return MSC_OK;
}

int launch_g0(msc_plan* pl, double omega, const double* kpar, int va, int n_orders) {
  // The kernel is mirror symmetric in each axis, K(R_a r) = S_a K(r) S_a, and its
  // spectrum is stored on the octant kz <= Lz/2, ky <= Ly/2, kx <= Lx/2. The
  // Bloch-phased kernel loses the symmetry in x and y and is stored in full.
  const Geo before = pl->g;
  set_spectrum_box(pl->g, kpar == nullptr);
  if (memcmp(&before, &pl->g, sizeof(Geo)) != 0) ++pl->gen;  // kernels take the geometry by value
  const Geo& g = pl->g;
  const int E = va ? 81 : 45;
  if (pl->khat64.p && pl->E != E) {
    dfree(pl, pl->khat64);
    dfree(pl, pl->khat32);
  }
  pl->E = E;
  MSC_TRY(dalloc(pl, pl->khat64, sizeof(double2) * khat_elems_t<double>(g, E)));
  MSC_TRY(dalloc(pl, pl->khat32, sizeof(float2) * khat_elems_t<float>(g, E)));
  MSC_TRY(dalloc(pl, pl->va_blocks, sizeof(double) * 26 * 81));
  const long long npts = (long long)g.Lz * g.Ly * g.Lx;
  // FP64 spatial kernel and its partial transforms; kept by the plan for the next frequency
  MSC_TRY(dalloc(pl, pl->g0_scratch, sizeof(double2) * (size_t)E * npts));
  DBuf& ks = pl->g0_scratch;
  if (va) {
    k_va_blocks<<<1, 32, 0, pl->stream>>>((double*)pl->va_blocks.p, pl->desc.alpha, pl->desc.beta, pl->desc.rho, omega,
                                          n_orders); ::msc::note_launch();
    MSC_CUDA(cudaGetLastError());
  }
  G0Params p;
  p.g = g;
  p.d = 2.0 * pl->desc.a;
  p.omega = omega;
  p.alpha = pl->desc.alpha;
  p.beta = pl->desc.beta;
  p.rho = pl->desc.rho;
  p.periodic = pl->desc.periodic;
  p.va = va;
  p.E = E;
  p.bloch = kpar != nullptr;
  p.kx = kpar ? kpar[0] : 0.0;
  p.ky = kpar ? kpar[1] : 0.0;
  p.scale = 1.0 / ((double)g.Lz * g.Lx * g.Ly);
  double2* K = (double2*)ks.p;
  const double2* twxy = (const double2*)pl->tw64_xy.p;
  const double2* twz = (const double2*)pl->tw64_z.p;
  const long long plane = (long long)g.Ly * g.Lx, vol = (long long)g.Lz * plane;
  int s = MSC_OK;
  // aperiodic mirror-symmetric kernel: spatial evaluation fused with the x pass
  const bool fused = g.oct && !p.periodic && g0_fused() && g.Lx >= 8 && g.Lx / 2 + 1 <= G0X_NT &&
                     g0x_smem(g.Lx) <= 200 * 1024;
  if (fused) {
    MSC_TRY(dalloc(pl, pl->g0_near, sizeof(double2) * 81 * 27));
    double2* Kn = (double2*)pl->g0_near.p;
    const size_t sm = g0x_smem(g.Lx);
    const dim3 grid((unsigned)(g.Ly / 2 + 1), (unsigned)(g.Lz / 2 + 1));
    const double* vab = (const double*)pl->va_blocks.p;
    const FftPlan1D& f = pl->fxy;
#define CALL(P2)                                                                                 \
  {                                                                                              \
    MSC_CUDA(prep_kernel((const void*)k_g0_x<P2>));                                              \
    k_g0_x<P2><<<grid, G0X_NT, sm, pl->stream>>>(K, Kn, vab, p, f, twxy);                        \
  }
    MSC_POW2_DISPATCH(f.pow2, CALL);
#undef CALL
    ::msc::note_launch();
    MSC_CUDA(cudaGetLastError());
    // near-field blocks from the 3x3x3 box
    Geo box = g;
    box.Lz = box.Ly = box.Lx = 3;
    MSC_TRY(nearfield_extract(pl, Kn, p.scale, &box));
  } else {
    if (g.oct) {
      const long long noct = (long long)(g.Lz / 2 + 1) * (g.Ly / 2 + 1) * (g.Lx / 2 + 1);
      k_g0_spatial_oct<<<(unsigned)ceil_div(noct, 128), 128, 0, pl->stream>>>(K, (const double*)pl->va_blocks.p, p);
    } else {
      k_g0_spatial<<<(unsigned)ceil_div(npts, 128), 128, 0, pl->stream>>>(K, (const double*)pl->va_blocks.p, p);
    }
    ::msc::note_launch();
    MSC_CUDA(cudaGetLastError());
    // near-field blocks for the preconditioner, before the transforms overwrite K
    MSC_TRY(nearfield_extract(pl, K, p.scale));
    // x pass (contiguous lines), in place; keep kx < Hx
    s = launch_fft_contig<double>(pl, K, K, (long long)E * g.Lz * g.Ly, (long long)E * g.Lz * g.Ly, 0, g.Lx, g.Lx,
                                  g.Hx, pl->fxy, twxy, -1, nullptr);
  }
  // y pass: axis stride Lx, columns kx < Hx, slabs (z, e); keep ky < Hy. After k_g0_x
  // only the octant rows are stored: slabs z <= Lz/2, inputs y <= Ly/2, the rest mirrored.
  unsigned long long odd_y[2] = {0, 0}, odd_z[2] = {0, 0};
  for (int a = 0, e = 0; a < 9; ++a)
    for (int b = (E == 45 ? a : 0); b < 9; ++b, ++e) {
      const int par = dof_parity(a) ^ dof_parity(b);
      if (par & 2) odd_y[e >> 6] |= 1ull << (e & 63);
      if (par & 4) odd_z[e >> 6] |= 1ull << (e & 63);
    }
  if (s == MSC_OK)
    s = launch_fft_strided<double>(pl, K, g.Lx, plane, vol, K, g.Lx, plane, vol, nullptr, g.Hx,
                                   fused ? g.Lz / 2 + 1 : g.Lz, E, fused ? g.Ly / 2 + 1 : g.Ly, g.Hy, pl->fxy, twxy,
                                   -1, nullptr, fused ? odd_y : nullptr);
  // z pass: axis stride Ly*Lx, columns kx < Hx, slabs (ky < Hy, e); keep kz < Hz, in place
  if (s == MSC_OK)
    s = launch_fft_strided<double>(pl, K, plane, g.Lx, vol, K, plane, g.Lx, vol, nullptr, g.Hx, g.Hy, E,
                                   fused ? g.Lz / 2 + 1 : g.Lz, g.Hz, pl->fz, twz, -1, nullptr,
                                   fused ? odd_z : nullptr);
  // stored layouts of the fused z pass, complex128 and complex64
  if (s == MSC_OK) s = launch_khat_pack<double>(pl, K, (double2*)pl->khat64.p, E);
  if (s == MSC_OK) s = launch_khat_pack<float>(pl, K, (float2*)pl->khat32.p, E);
  return s;
}

}  // namespace msc
