// FP64 physics of the slab operator, evaluated on the device:
//  * the 9x9 point propagator [[G, C], [H, S]] entry by entry
//    (tmnestor/MultipleScatteringCalculations cubic_scattering/resonance_tmatrix.py:214-428),
//  * the volume-averaged nearest-neighbour 9x9 (inter_voxel_propagator.py:1295-1355),
//  * the contrast-independent cube constants Gamma0, A, B, C
//    (effective_contrasts.py:112-330) and the per-voxel T0 scalars (:338-451,
//    resonance_tmatrix.py:461-487, voigt_tmatrix.py:131-169).
// Index conventions: Cartesian (z=0, x=1, y=2); 9 DOF = [u(3), Voigt strain (zz, xx,
// yy, 2xy, 2zy, 2zx)].
#pragma once
#include "msc_common.cuh"
#include "va_tables.cuh"

namespace msc {

__host__ __device__ constexpr int voigt_p(int a) { return a < 3 ? a : (a == 3 ? 1 : 0); }
__host__ __device__ constexpr int voigt_q(int a) { return a < 3 ? a : (a == 3 ? 2 : (a == 4 ? 2 : 1)); }

__host__ __device__ __forceinline__ double2 cmulr(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double kd(int i, int j) { return i == j ? 1.0 : 0.0; }

// ---------------------------------------------------------------------------
// Point propagator. G_ij = P [phi d_ij + psi g_i g_j] with P = 1/(4 pi rho w^2);
// the radial functions are sums of c e^{ikr} r^p, p in {-1,-2,-3}.
// ---------------------------------------------------------------------------
struct PointProp {
  double g[3];
  double P;
  bool zero;
  double2 c1, c2, c3;                  // G_{ij,k} coefficients
  double2 t1, t2, t3, t4, t7;          // G_{ij,kl} coefficients
  double2 phi, psi;

  __device__ void init(double rz, double rx, double ry, double omega, double alpha, double beta, double rho) {
    const double r = sqrt(rz * rz + rx * rx + ry * ry);
    zero = !(r >= 1.0e-14);
    if (zero) return;
    g[0] = rz / r;
    g[1] = rx / r;
    g[2] = ry / r;
    const double kP = omega / alpha, kS = omega / beta;
    P = 1.0 / (4.0 * M_PI * rho * omega * omega);
    double sP, cP, sS, cS;
    sincos(kP * r, &sP, &cP);
    sincos(kS * r, &sS, &cS);
    const double2 eP = make_double2(cP, sP), eS = make_double2(cS, sS);
    // term lists (coefficient, wave, power): resonance_tmatrix.py:238-252
    double2 f[2] = {make_double2(0, 0), make_double2(0, 0)};
    double2 fp[2] = {make_double2(0, 0), make_double2(0, 0)};
    double2 fpp[2] = {make_double2(0, 0), make_double2(0, 0)};
    const double2 coef[11] = {make_double2(kS * kS, 0), make_double2(0, kS), make_double2(-1, 0), make_double2(0, -kP),
                              make_double2(1, 0),
                              make_double2(-kS * kS, 0), make_double2(0, -3 * kS), make_double2(3, 0),
                              make_double2(kP * kP, 0), make_double2(0, 3 * kP), make_double2(-3, 0)};
    const int wave[11] = {1, 1, 1, 0, 0, 1, 1, 1, 0, 0, 0};   // 0 = P, 1 = S
    const int pw[11] = {-1, -2, -3, -2, -3, -1, -2, -3, -1, -2, -3};
    const double ir = 1.0 / r;
#pragma unroll
    for (int t = 0; t < 11; ++t) {
      const int which = t < 5 ? 0 : 1;
      const double k = wave[t] ? kS : kP;
      const double2 e = wave[t] ? eS : eP;
      const int p = pw[t];
      const double rp = (p == -1) ? ir : (p == -2 ? ir * ir : ir * ir * ir);
      const double2 ce = coef[t] * e;
      // ikr + p ; (ikr)^2 + 2 p ikr + p(p-1)
      const double2 d1 = make_double2((double)p, k * r);
      const double2 d2 = make_double2(-(k * r) * (k * r) + p * (p - 1.0), 2.0 * p * k * r);
      f[which] += rp * ce;
      fp[which] += (rp * ir) * (ce * d1);
      fpp[which] += (rp * ir * ir) * (ce * d2);
    }
    phi = f[0];
    psi = f[1];
    const double2 phi_p = fp[0], psi_p = fp[1], phi_pp = fpp[0], psi_pp = fpp[1];
    c1 = phi_p;
    c2 = psi_p - cmulr(2.0 * ir, psi);
    c3 = cmulr(ir, psi);
    t1 = cmulr(ir, phi_p);
    t2 = phi_pp - cmulr(ir, phi_p);
    t3 = cmulr(ir, psi_p) - cmulr(2.0 * ir * ir, psi);
    t4 = cmulr(ir * ir, psi);
    t7 = psi_pp - cmulr(5.0 * ir, psi_p) + cmulr(8.0 * ir * ir, psi);
  }
  __device__ double2 G(int i, int j) const { return cmulr(P, cmulr(kd(i, j), phi) + cmulr(g[i] * g[j], psi)); }
  __device__ double2 Gd(int i, int j, int k) const {
    return cmulr(P, cmulr(g[k] * kd(i, j), c1) + cmulr(g[i] * g[j] * g[k], c2) +
                        cmulr(kd(i, k) * g[j] + kd(j, k) * g[i], c3));
  }
  __device__ double2 Gdd(int i, int j, int k, int l) const {
    const double s3 = g[i] * g[j] * kd(k, l) + kd(i, l) * g[j] * g[k] + kd(j, l) * g[i] * g[k] +
                      kd(i, k) * g[j] * g[l] + kd(j, k) * g[i] * g[l];
    return cmulr(P, cmulr(kd(i, j) * kd(k, l), t1) + cmulr(kd(i, j) * g[k] * g[l], t2) + cmulr(s3, t3) +
                        cmulr(kd(i, k) * kd(j, l) + kd(j, k) * kd(i, l), t4) + cmulr(g[i] * g[j] * g[k] * g[l], t7));
  }
  // Entry (a, b) of the 9x9 block with the engineering-shear column halving
  // (resonance_tmatrix.py:353-428).
  __device__ double2 entry(int a, int b) const {
    if (zero) return make_double2(0, 0);
    if (a < 3 && b < 3) return G(a, b);
    if (a < 3) {
      const int al = b - 3, p = voigt_p(al), q = voigt_q(al);
      if (p == q) return Gd(a, p, p);
      return cmulr(0.5, Gd(a, p, q) + Gd(a, q, p));
    }
    const int al = a - 3, p = voigt_p(al), q = voigt_q(al);
    if (b < 3) {
      if (p == q) return Gd(p, b, p);
      return Gd(p, b, q) + Gd(q, b, p);
    }
    const int be = b - 3, m = voigt_p(be), n = voigt_q(be);
    double2 v;
    if (p == q && m == n) v = Gdd(p, m, m, p);
    else if (p == q) v = Gdd(p, m, n, p) + Gdd(p, n, m, p);
    else if (m == n) v = Gdd(p, m, m, q) + Gdd(q, m, m, p);
    else v = Gdd(p, m, n, q) + Gdd(p, n, m, q) + Gdd(q, m, n, p) + Gdd(q, n, m, p);
    return be >= 3 ? cmulr(0.5, v) : v;
  }
};

// ---------------------------------------------------------------------------
// Volume-averaged NN block (real), written to out[81] (row major).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int va_idx4(int n0, int n1) {
  const int off[5] = {0, 5, 9, 12, 14};
  return off[n0] + n1;
}
__device__ __forceinline__ int va_idx3(int n0, int n1) {
  const int off[4] = {0, 4, 7, 9};
  return off[n0] + n1;
}
__device__ __forceinline__ double va_B(int t, int n, int a, int b, int c, int d) {
  int cnt[3] = {0, 0, 0};
  cnt[a]++; cnt[b]++; cnt[c]++; cnt[d]++;
  return VA_B[t][n][va_idx4(cnt[0], cnt[1])];
}
__device__ __forceinline__ double va_D3(int t, int n, int a, int b, int c) {
  int cnt[3] = {0, 0, 0};
  cnt[a]++; cnt[b]++; cnt[c]++;
  return VA_D3[t][n][va_idx3(cnt[0], cnt[1])];
}
__device__ __forceinline__ double sym3(const double* v6, int i, int j) {
  if (i == j) return v6[i];
  const int s = i + j;  // (0,1)->1, (0,2)->2, (1,2)->3
  return v6[2 + s];
}

// Signed permutation P with P @ canon = R (greedy as inter_voxel_propagator.py:734-760):
// row i has its nonzero in column sig[i] with sign sgn[i].
__device__ inline void va_perm(const int* canon, const int* R, int* sig, double* sgn) {
  bool used[3] = {false, false, false};
  for (int i = 0; i < 3; ++i) {
    sig[i] = 0;
    sgn[i] = 0.0;
    for (int j = 0; j < 3; ++j) {
      if (!used[j] && abs(R[i]) == abs(canon[j]) && canon[j] != 0) {
        sig[i] = j;
        sgn[i] = (double)((R[i] > 0) - (R[i] < 0)) * (double)((canon[j] > 0) - (canon[j] < 0));
        used[j] = true;
        break;
      }
      if (!used[j] && canon[j] == 0 && R[i] == 0) {
        sig[i] = j;
        sgn[i] = 1.0;
        used[j] = true;
        break;
      }
    }
  }
}

// R = (dz, dx, dy), one of the 26 neighbours. out[a*9+b].
__device__ inline void va_block(const int* R, double alpha, double beta, double rho, double omega, int n_orders,
                                double* out) {
  int na[3] = {abs(R[0]), abs(R[1]), abs(R[2])};
  const int nnz = (na[0] != 0) + (na[1] != 0) + (na[2] != 0);
  const int t = nnz - 1;  // 0 face, 1 edge, 2 corner
  int canon[3] = {1, nnz >= 2 ? 1 : 0, nnz >= 3 ? 1 : 0};
  int sig[3];
  double sgn[3];
  va_perm(canon, R, sig, sgn);
  const int no = n_orders < 3 ? n_orders : 3;
  const double cs = beta, cp = alpha;
  const double mu = rho * beta * beta;
  const double nu = (alpha * alpha - 2.0 * beta * beta) / (2.0 * (alpha * alpha - beta * beta));
  // order-n material factors: S block -1/(2 mu_n), eta_n; G/dG coefficient and Laplacian
  double sfac[4], seta[4], gco[4], glap[4], geta[4];
  sfac[0] = -1.0 / (2.0 * mu);
  seta[0] = 1.0 / (2.0 * (1.0 - nu));
  const double gc[4] = {0.0, -(omega * omega) / (8.0 * M_PI * rho * pow(cs, 4)),
                        pow(omega, 4) / (96.0 * M_PI * rho * pow(cs, 6)),
                        -pow(omega, 6) / (2880.0 * M_PI * rho * pow(cs, 8))};
  const double lp[4] = {0.0, 12.0, 30.0, 56.0};
  for (int n = 1; n <= 3; ++n) {
    sfac[n] = -1.0 / (2.0 * rho * pow(cs, 2 * n + 2));
    seta[n] = 1.0 - pow(cs / cp, 2 * n + 2);
    gco[n] = gc[n];
    glap[n] = lp[n];
    geta[n] = 1.0 - pow(cs / cp, 2 * n + 2);
  }
  // canonical P_abcd (summed over orders with omega^{2n}) evaluated at permuted indices
  auto Pc = [&](int a, int b, int c, int d) {
    double v = 0.0;
    for (int n = 0; n <= no; ++n) {
      const double* A = VA_A[t][n];
      const double pn = sfac[n] * (kd(a, c) * sym3(A, b, d) + kd(b, c) * sym3(A, a, d) -
                                   2.0 * seta[n] * va_B(t, n, a, b, c, d));
      v += (n == 0 ? 1.0 : pow(omega, 2 * n)) * pn;
    }
    return v;
  };
  auto Prot = [&](int i, int j, int k, int l) {
    return sgn[i] * sgn[j] * sgn[k] * sgn[l] * Pc(sig[i], sig[j], sig[k], sig[l]);
  };
  // canonical G_ab (inter_voxel_propagator.py:985-1057)
  auto Gc = [&](int a, int b) {
    const double* D = VA_D2W[t][0];
    const double tr = D[0] + D[1] + D[2];
    double v = (1.0 / (4.0 * M_PI * mu)) * (kd(a, b) * 0.5 * tr - sym3(D, a, b) / (4.0 * (1.0 - nu)));
    for (int n = 1; n <= no; ++n) {
      const double* Dn = VA_D2W[t][n];
      const double trn = Dn[0] + Dn[1] + Dn[2];
      v += gco[n] * (kd(a, b) * trn / glap[n] - (geta[n] / glap[n]) * sym3(Dn, a, b));
    }
    return v;
  };
  // canonical dG_abc (:1192-1269); omega terms skipped at omega == 0
  auto dGc = [&](int a, int b, int c) {
    double v = (1.0 / (4.0 * M_PI * mu)) * (kd(a, b) * VA_DW[t][0][c] - va_D3(t, 0, a, b, c) / (4.0 * (1.0 - nu)));
    if (omega != 0.0) {
      for (int n = 1; n <= no; ++n)
        v += gco[n] * (kd(a, b) * VA_DW[t][n][c] - (geta[n] / glap[n]) * va_D3(t, n, a, b, c));
    }
    return v;
  };
  auto dG = [&](int i, int j, int k) { return sgn[i] * sgn[j] * sgn[k] * dGc(sig[i], sig[j], sig[k]); };
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out[i * 9 + j] = sgn[i] * sgn[j] * Gc(sig[i], sig[j]);
  for (int al = 0; al < 6; ++al) {
    const int m = voigt_p(al), n = voigt_q(al);
    for (int i = 0; i < 3; ++i) {
      const double c = (m == n) ? dG(i, m, m) : 0.5 * (dG(i, m, n) + dG(i, n, m));
      out[i * 9 + 3 + al] = c;
      out[(3 + al) * 9 + i] = c;  // H = C^T
    }
  }
  for (int al = 0; al < 6; ++al) {
    const int p = voigt_p(al), q = voigt_q(al);
    const double mult = (p != q) ? 2.0 : 1.0;
    for (int be = 0; be < 6; ++be) {
      const int m = voigt_p(be), n = voigt_q(be);
      double v = mult * Prot(p, q, m, n);
      if (m != n) v += mult * Prot(p, q, n, m);
      if (be >= 3) v *= 0.5;
      out[(3 + al) * 9 + 3 + be] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Cube constants (contrast independent): Gamma0, A^c, B^c, C^c.
// ---------------------------------------------------------------------------
struct CubeConst {
  double2 gamma0, A, B, C;
};

__host__ __device__ inline double fact(int n) {
  double f = 1.0;
  for (int i = 2; i <= n; ++i) f *= (double)i;
  return f;
}
__host__ __device__ inline double2 cpow_i(double k, int m) {
  // (i k)^m
  double mag = 1.0;
  for (int i = 0; i < m; ++i) mag *= k;
  switch (m & 3) {
    case 0: return make_double2(mag, 0);
    case 1: return make_double2(0, mag);
    case 2: return make_double2(-mag, 0);
    default: return make_double2(0, -mag);
  }
}

// Evaluated on the host once per T0 build (a serial FP64 recurrence that, run by one thread
// per block, had dominated the T0 kernel) and passed to it by value.
__host__ __device__ inline CubeConst cube_constants(double omega, double a, double alpha, double beta, double rho) {
  constexpr int N = 8;
  const double a0 = (alpha * alpha + beta * beta) / (8.0 * M_PI * rho * alpha * alpha * beta * beta);
  const double b0 = (alpha * alpha - beta * beta) / (8.0 * M_PI * rho * alpha * alpha * beta * beta);
  const double G0_CUBE = (4.0 / 3.0) * log(70226.0 + 40545.0 * sqrt(3.0)) - 2.0 * M_PI;
  double2 phi[N], psi[N];
  const double cf = 1.0 / (4.0 * M_PI * rho * beta * beta);
  const double cg = 1.0 / (4.0 * M_PI * rho);
  for (int n = 0; n < N; ++n) {
    phi[n] = cmulr(cf / fact(2 * n + 1), cpow_i(omega / beta, 2 * n + 1));
    const double2 pa = cpow_i(omega / alpha, 2 * n + 3), pb = cpow_i(omega / beta, 2 * n + 3);
    psi[n] = cmulr(cg / fact(2 * n + 3), cmulr(1.0 / (alpha * alpha), pa) - cmulr(1.0 / (beta * beta), pb));
  }
  double mu1[N + 3];
  for (int k = 0; k < N + 3; ++k) mu1[k] = 2.0 * pow(a, 2 * k + 1) / (2 * k + 1);
  double S0[N], S1[N], S2[N], S11[N];
  for (int m = 0; m < N; ++m) {
    S0[m] = S1[m] = S2[m] = S11[m] = 0.0;
    for (int p = 0; p <= m; ++p)
      for (int q = 0; q <= m - p; ++q) {
        const int r = m - p - q;
        const double c = fact(m) / (fact(p) * fact(q) * fact(r));
        S0[m] += c * mu1[p] * mu1[q] * mu1[r];
        S1[m] += c * mu1[p + 1] * mu1[q] * mu1[r];
        S2[m] += c * mu1[p + 2] * mu1[q] * mu1[r];
        S11[m] += c * mu1[p + 1] * mu1[q + 1] * mu1[r];
      }
  }
  CubeConst cc;
  double2 gs = make_double2(0, 0);
  for (int n = 0; n < N; ++n) gs += cmulr(S0[n], phi[n]) + cmulr(S1[n], psi[n]);
  cc.gamma0 = make_double2(a * a * (a0 + b0 / 3.0) * G0_CUBE, 0) + gs;
  const double s3 = sqrt(3.0);
  const double j1 = 2.0 * M_PI / 3.0, j2 = -2.0 * (s3 - M_PI) / 9.0, k1 = 2.0 * (2.0 * s3 + M_PI) / 9.0;
  double2 As = make_double2(2.0 * (-a0 * j1 - 3.0 * b0 * j2), 0);
  double2 Bs = make_double2(2.0 * b0 * (j1 - 3.0 * j2), 0);
  double2 Cs = make_double2(6.0 * b0 * (3.0 * j2 - k1), 0);
  for (int n = 2; n < N; ++n) {
    const double f = 4.0 * n * (n - 1);
    As += cmulr(f * S1[n - 2], phi[n]) + cmulr(f * S11[n - 2], psi[n]);
    Bs += cmulr(f * S11[n - 2], psi[n]);
    Cs += cmulr(f * (S2[n - 2] - 3.0 * S11[n - 2]), psi[n]);
  }
  for (int n = 1; n < N; ++n) {
    As += cmulr(2.0 * n * S0[n - 1], phi[n]) + cmulr(2.0 * n * S1[n - 1], psi[n]);
    Bs += cmulr(4.0 * n * S1[n - 1], psi[n]);
  }
  for (int n = 0; n < N; ++n) Bs += cmulr(S0[n], psi[n]);
  cc.A = As;
  cc.B = Bs;
  cc.C = Cs;
  return cc;
}

__device__ __forceinline__ double2 cdiv1(double2 z) {  // 1 / z
  const double d = z.x * z.x + z.y * z.y;
  return make_double2(z.x / d, -z.y / d);
}

// The four T0 scalars (t_u, t_l, t_d, t_s) of one voxel:
// T0 = diag(t_u I3, [t_l + t_d delta_ij] on the normal strains, t_s I3 on the shears).
__device__ inline void t0_voxel(const CubeConst& cc, double omega, double a, double dl, double dm, double dr,
                                double2* t) {
  const double2 T1 = cmulr(dl, cc.A + cmulr(4.0, cc.B) + cc.C) + cmulr(2.0 * dm, cc.B);
  const double2 T2 = cmulr(dm, cc.A + cc.B);
  const double2 T3 = cmulr(2.0 * dm, cc.C);
  const double2 one = make_double2(1.0, 0.0);
  const double2 amp_u = cdiv1(one - cmulr(omega * omega * dr, cc.gamma0));
  const double2 amp_th = cdiv1(one - cmulr(3.0, T1) - cmulr(2.0, T2) - T3);
  const double2 amp_off = cdiv1(one - cmulr(2.0, T2));
  const double2 amp_diag = cdiv1(one - cmulr(2.0, T2) - T3);
  const double V = 8.0 * a * a * a;
  const double2 drho_s = cmulr(dr, amp_u);
  const double2 dmu_off = cmulr(dm, amp_off);
  const double2 dmu_diag = cmulr(dm, amp_diag);
  const double2 dlam_s = cmulr(dl + 2.0 / 3.0 * dm, amp_th) - cmulr(2.0 / 3.0 * dm, amp_diag);
  t[0] = cmulr(omega * omega * V, drho_s);
  t[1] = cmulr(V, dlam_s);
  t[2] = cmulr(2.0 * V, dmu_diag);
  t[3] = cmulr(2.0 * V, dmu_off);
}

}  // namespace msc
