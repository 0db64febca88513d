// Observables of a solved slab as device reductions in FP64:
//  * periodic specular R_PP (slab_rpp_periodic, slab_scattering.py:672-735),
//  * reflected far-field amplitudes (slab_reflected_field, slab_scattering.py:589-669).
#include "plan.cuh"

namespace msc {

// tau = T0 psi at one site from the 4 scalars; psi in reference layout [site][9].
__device__ __forceinline__ void tau_site(const double2* __restrict__ psi, const double2* __restrict__ t4, int nsite,
                                         int s, double2* tau) {
  double2 v[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) v[c] = psi[(size_t)s * 9 + c];
  const double2 tu = t4[s], tl = t4[(size_t)nsite + s], td = t4[(size_t)2 * nsite + s], ts = t4[(size_t)3 * nsite + s];
  const double2 tr = v[3] + v[4] + v[5];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    tau[c] = tu * v[c];
    tau[3 + c] = tl * tr + td * v[3 + c];
    tau[6 + c] = ts * v[6 + c];
  }
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x < 32) {
    r = (threadIdx.x < NT / 32) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  return r;  // valid in thread 0
}

// One block per layer: mean of tau (9 complex) over the M x M sites, optionally
// demodulated by exp(-i (kx x + ky y)).
template <int NT>
__global__ void __launch_bounds__(NT) k_layer_means(const double2* __restrict__ psi, const double2* __restrict__ t4,
                                                    int M, int nsite, double a, int demod, double kx, double ky,
                                                    double2* __restrict__ means) {
  __shared__ double sh[NT / 32];
  const int l = blockIdx.x;
  double acc[18];
#pragma unroll
  for (int q = 0; q < 18; ++q) acc[q] = 0.0;
  const double d = 2.0 * a;
  for (int k = threadIdx.x; k < M * M; k += NT) {
    const int s = l * M * M + k;
    double2 tau[9];
    tau_site(psi, t4, nsite, s, tau);
    if (demod) {
      const int i = k / M, j = k % M;
      const double x = (i - (M - 1) / 2.0) * d, y = (j - (M - 1) / 2.0) * d;
      double sn, cs;
      sincos(-(kx * x + ky * y), &sn, &cs);
#pragma unroll
      for (int c = 0; c < 9; ++c) tau[c] = tau[c] * make_double2(cs, sn);
    }
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      acc[2 * c] += tau[c].x;
      acc[2 * c + 1] += tau[c].y;
    }
  }
  for (int q = 0; q < 18; ++q) {
    const double r = block_sum<NT>(acc[q], sh);
    if (threadIdx.x == 0) (q & 1 ? means[(size_t)l * 9 + q / 2].y : means[(size_t)l * 9 + q / 2].x) = r / (M * M);
  }
}

// R_PP = -i/(2 kz d^2 rho alpha^2) sum_l Q_l exp(i kz z_l),
// Q_l = -rh.f - i km rh.sigma.rh, rh = (-eta alpha, p alpha, 0), kz = omega eta.
// km = kz is the reference's moment factor; plane_wave = 1 takes km = omega/alpha,
// the magnitude of the gradient of the reflected plane wave (equal at p = 0).
__global__ void k_rpp_combine(const double2* __restrict__ means, int Nz, double a, double omega, double alpha,
                              double rho, double p, int plane_wave, double2* out) {
  if (threadIdx.x != 0) return;
  // eta = sqrt(1/alpha^2 - p^2) on the Im >= 0 (then Re >= 0) branch (kennett_layers.py:273-284)
  const double s = 1.0 / alpha;
  const double T = (s + p) * (s - p);
  double2 eta = T >= 0 ? make_double2(sqrt(T), 0.0) : make_double2(0.0, sqrt(-T));
  const double2 kz = make_double2(omega * eta.x, omega * eta.y);
  const double2 km = plane_wave ? make_double2(omega / alpha, 0.0) : kz;
  const double2 rh0 = make_double2(-eta.x * alpha, -eta.y * alpha);
  const double rh1 = p * alpha;
  const double d = 2.0 * a;
  double2 tot = make_double2(0, 0);
  for (int l = 0; l < Nz; ++l) {
    const double2* m = means + (size_t)l * 9;
    // sigma tensor from Voigt (zz, xx, yy, 2xy, 2zy, 2zx); rh = (rh0, rh1, 0)
    const double2 s00 = m[3], s11 = m[4], s01 = 0.5 * m[8];
    // rh.sigma.rh = rh0^2 s00 + 2 rh0 rh1 s01 + rh1^2 s11
    const double2 srr = rh0 * rh0 * s00 + 2.0 * rh1 * (rh0 * s01) + (rh1 * rh1) * s11;
    const double2 rf = rh0 * m[0] + rh1 * m[1];
    const double2 q = make_double2(-rf.x, -rf.y) - mul_i<1>(km * srr);
    const double zl = (l + 0.5) * d;
    const double2 ph = make_double2(-kz.y * zl, kz.x * zl);  // i kz z
    const double mag = exp(ph.x);
    double sn, cs;
    sincos(ph.y, &sn, &cs);
    tot += q * make_double2(mag * cs, mag * sn);
  }
  // -i / (2 kz d^2 rho alpha^2)
  const double2 den = (2.0 * d * d * rho * alpha * alpha) * kz;
  const double dd = den.x * den.x + den.y * den.y;
  const double2 inv = make_double2(den.x / dd, -den.y / dd);
  *out = mul_i<-1>(inv) * tot;
}

int rpp_periodic(msc_plan* pl, const double2* psi, double omega, double p, int flags, double* out) {
  const int bloch = flags & MSC_RPP_BLOCH;
  if (!pl->has_t0) {
    set_error("rpp_periodic needs build_t0 first");
    return MSC_ERR_STATE;
  }
  const Geo& g = pl->g;
  MSC_TRY(dalloc(pl, pl->red, sizeof(double2) * ((size_t)9 * g.Nz + 8 + 4 * 1184)));
  double2* means = (double2*)pl->red.p;
  double2* res = means + (size_t)9 * g.Nz;
  k_layer_means<256><<<g.Nz, 256, 0, pl->stream>>>(psi, (const double2*)pl->t4_64.p, g.M, g.nsite, pl->desc.a,
                                                   bloch ? 1 : 0, pl->kpar[0], pl->kpar[1], means); ::msc::note_launch();
  k_rpp_combine<<<1, 32, 0, pl->stream>>>(means, g.Nz, pl->desc.a, omega, pl->desc.alpha, pl->desc.rho, p,
                                  (flags & MSC_RPP_PLANE_WAVE_MOMENT) ? 1 : 0, res); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  double2 h;
  MSC_TRY(read_small(pl, res, &h, sizeof(double2)));
  out[0] = h.x;
  out[1] = h.y;
  return MSC_OK;
}

// ---- reflected field: per-block partial sums of (phP QP) and (phS QS_perp) -----------
struct ReflP {
  double kP, kS, rh[3], a;
  int M, nsite;
};

template <int NT>
__global__ void __launch_bounds__(NT) k_refl_partial(const double2* __restrict__ psi, const double2* __restrict__ t4,
                                                     ReflP r, double2* __restrict__ part) {
  __shared__ double sh[NT / 32];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // QP (re, im), QSp[3] (re, im)
  const double d = 2.0 * r.a;
  for (int s = blockIdx.x * NT + threadIdx.x; s < r.nsite; s += gridDim.x * NT) {
    double2 tau[9];
    tau_site(psi, t4, r.nsite, s, tau);
    const int j = s % r.M, i = (s / r.M) % r.M, n = s / (r.M * r.M);
    const double c[3] = {(n + 0.5) * d, (i - (r.M - 1) / 2.0) * d, (j - (r.M - 1) / 2.0) * d};
    const double cr = c[0] * r.rh[0] + c[1] * r.rh[1] + c[2] * r.rh[2];
    double sn, cs;
    sincos(-r.kP * cr, &sn, &cs);
    const double2 phP = make_double2(cs, sn);
    sincos(-r.kS * cr, &sn, &cs);
    const double2 phS = make_double2(cs, sn);
    // sigma (symmetric) from Voigt
    double2 sg[3][3];
    sg[0][0] = tau[3]; sg[1][1] = tau[4]; sg[2][2] = tau[5];
    sg[1][2] = sg[2][1] = 0.5 * tau[6];
    sg[0][2] = sg[2][0] = 0.5 * tau[7];
    sg[0][1] = sg[1][0] = 0.5 * tau[8];
    double2 sr[3];
    for (int q = 0; q < 3; ++q) sr[q] = r.rh[0] * sg[q][0] + r.rh[1] * sg[q][1] + r.rh[2] * sg[q][2];
    const double2 srr = r.rh[0] * sr[0] + r.rh[1] * sr[1] + r.rh[2] * sr[2];
    const double2 fr = r.rh[0] * tau[0] + r.rh[1] * tau[1] + r.rh[2] * tau[2];
    const double2 QP = fr - mul_i<1>(r.kP * srr);
    const double2 a0 = phP * QP;
    acc[0] += a0.x;
    acc[1] += a0.y;
    double2 QS[3];
    for (int q = 0; q < 3; ++q) QS[q] = tau[q] - mul_i<1>(r.kS * sr[q]);
    const double2 qr = r.rh[0] * QS[0] + r.rh[1] * QS[1] + r.rh[2] * QS[2];
    for (int q = 0; q < 3; ++q) {
      const double2 v = phS * (QS[q] - r.rh[q] * qr);
      acc[2 + 2 * q] += v.x;
      acc[3 + 2 * q] += v.y;
    }
  }
  for (int q = 0; q < 8; ++q) {
    const double v = block_sum<NT>(acc[q], sh);
    if (threadIdx.x == 0) (q & 1 ? part[(size_t)blockIdx.x * 4 + q / 2].y : part[(size_t)blockIdx.x * 4 + q / 2].x) = v;
  }
}

int reflected_field(msc_plan* pl, const double2* psi, double omega, const double* k_hat, double* out) {
  if (!pl->has_t0) {
    set_error("reflected_field needs build_t0 first");
    return MSC_ERR_STATE;
  }
  const Geo& g = pl->g;
  const int nb = std::min(ceil_div(g.nsite, 256), 1184);
  MSC_TRY(dalloc(pl, pl->red, sizeof(double2) * ((size_t)9 * g.Nz + 8 + 4 * 1184)));
  double2* part = (double2*)pl->red.p;
  ReflP r;
  const double nrm = sqrt(k_hat[0] * k_hat[0] + k_hat[1] * k_hat[1] + k_hat[2] * k_hat[2]);
  for (int q = 0; q < 3; ++q) r.rh[q] = -k_hat[q] / nrm;
  r.kP = omega / pl->desc.alpha;
  r.kS = omega / pl->desc.beta;
  r.a = pl->desc.a;
  r.M = g.M;
  r.nsite = g.nsite;
  k_refl_partial<256><<<nb, 256, 0, pl->stream>>>(psi, (const double2*)pl->t4_64.p, r, part); ::msc::note_launch();
  MSC_CUDA(cudaGetLastError());
  std::vector<double2> h((size_t)nb * 4);
  MSC_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double2) * nb * 4, cudaMemcpyDeviceToHost, pl->stream));
  MSC_CUDA(cudaStreamSynchronize(pl->stream));
  // fixed-order sum of the block partials, then the scalar prefactors
  double2 s[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  for (int b = 0; b < nb; ++b)
    for (int q = 0; q < 4; ++q) s[q] = s[q] + h[(size_t)b * 4 + q];
  const double al = pl->desc.alpha, be = pl->desc.beta, rho = pl->desc.rho;
  const double gP = 1.0 / (4.0 * M_PI * rho * al * al), gS = 1.0 / (4.0 * M_PI * rho * be * be);
  const double area = (g.M * 2.0 * pl->desc.a) * (g.M * 2.0 * pl->desc.a);
  // R_PP = rh . uP = -gP * sum(phP QP) (rh.rh = 1) / area
  const double2 Rpp = make_double2(-gP * s[0].x / area, -gP * s[0].y / area);
  double2 uS[3];
  for (int q = 0; q < 3; ++q) uS[q] = make_double2(-gS * s[1 + q].x / area, -gS * s[1 + q].y / area);
  // SV direction of the reflected ray
  const double* rh = r.rh;
  const double cr[3] = {rh[1] * 0 - rh[2] * 0, rh[2] * 1 - rh[0] * 0, rh[0] * 0 - rh[1] * 1};
  const double cn = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  double sv[3];
  if (cn < 1e-10) {
    sv[0] = 0; sv[1] = 1; sv[2] = 0;
  } else {
    double p[3] = {cr[1] * rh[2] - cr[2] * rh[1], cr[2] * rh[0] - cr[0] * rh[2], cr[0] * rh[1] - cr[1] * rh[0]};
    const double pn = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    for (int q = 0; q < 3; ++q) sv[q] = p[q] / pn;
  }
  const double2 Rps = sv[0] * uS[0] + sv[1] * uS[1] + sv[2] * uS[2];
  out[0] = Rpp.x; out[1] = Rpp.y;
  out[2] = Rps.x; out[3] = Rps.y;
  out[4] = Rpp.x; out[5] = Rpp.y;
  return MSC_OK;
}

}  // namespace msc
