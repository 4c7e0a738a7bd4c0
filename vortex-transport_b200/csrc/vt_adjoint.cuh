// Derivatives of the pointwise pieces of the right-hand side, for the
// discrete adjoint and the tangent-linear model:
//
//   roe_flux_vjp         reverse sweep of roe_flux (vt_device.cuh): given the
//                        adjoint of the flux, the adjoints of both states,
//                        through the Roe averages, the c2^2 "sound speed" and
//                        the entropy fix (Numericalflux.cpp:99-156);
//   contravariant_vjp    reverse sweep of contravariant_flux (the nodal Euler
//                        flux of Timestepping.cpp:141-158 contracted with J^-1);
//   Dual<N>, roe_flux_t,
//   contravariant_flux_t forward-mode versions of the same formulas on dual
//                        numbers, for the tangent-linear model and as the
//                        independent check of the reverse sweeps.
//
// All functions are __host__ __device__ so the reverse sweeps can be checked
// against the dual-number Jacobians on the CPU.
#pragma once

#include <cmath>

#include "vt_device.cuh"

namespace vt {

// 1/x: recip_nr (vt_device.cuh) in device code, IEEE division on the host, where
// the reverse sweeps are checked against the dual-number Jacobians.
__host__ __device__ inline double rcp(double x) {
#ifdef __CUDA_ARCH__
  return recip_nr(x);
#else
  return 1.0 / x;
#endif
}

// ---- dual numbers -------------------------------------------------------------
template <int N>
struct Dual {
  double v;
  double d[N];
  __host__ __device__ Dual() : v(0.0) {
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
  __host__ __device__ Dual(double x) : v(x) {  // NOLINT: constants promote
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
};

template <int N>
__host__ __device__ inline Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  const double ib = 1.0 / b.v;
  r.v = a.v * ib;
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N>
__host__ __device__ inline Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N>
__host__ __device__ inline Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a) { return Dual<N>(0.0) - a; }
template <int N>
__host__ __device__ inline Dual<N> operator*(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v * b;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N>
__host__ __device__ inline Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }
template <int N>
__host__ __device__ inline Dual<N> dsqrt(const Dual<N>& a) {
  Dual<N> r;
  r.v = sqrt(a.v);
  const double h = 0.5 / r.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * h;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> dabs(const Dual<N>& a) { return a.v < 0 ? -a : a; }
template <int N>
__host__ __device__ inline double val(const Dual<N>& a) { return a.v; }
__host__ __device__ inline double val(double a) { return a; }
__host__ __device__ inline double dsqrt(double a) { return sqrt(a); }
__host__ __device__ inline double dabs(double a) { return fabs(a); }

// ---- forward formulas on any scalar type (the algebra of roe_flux) --------------
template <typename T>
__host__ __device__ inline int roe_flux_t(const T* uL, const T* uR, double nx, double ny, T* f) {
  const T rL = uL[0], rR = uR[0];
  const T irLR = 1.0 / (rL * rR);
  const T irL = rR * irLR, irR = rL * irLR;
  const T vxL = uL[1] * irL, vyL = uL[2] * irL;
  const T unL = vxL * nx + vyL * ny;
  const T pL = kGm1 * (uL[3] - 0.5 * (uL[1] * vxL + uL[2] * vyL));
  int code = 0;
  if ((val(pL) <= 0) || (val(rL) <= 0)) code = 1;
  const T rHL = uL[3] + pL;
  const T HL = rHL * irL;
  const T vxR = uR[1] * irR, vyR = uR[2] * irR;
  const T unR = vxR * nx + vyR * ny;
  const T pR = kGm1 * (uR[3] - 0.5 * (uR[1] * vxR + uR[2] * vyR));
  if (code == 0 && ((val(pR) <= 0) || (val(rR) <= 0))) code = 2;
  const T rHR = uR[3] + pR;
  const T HR = rHR * irR;
  const T du0 = uR[0] - uL[0], du1 = uR[1] - uL[1], du2 = uR[2] - uL[2], du3 = uR[3] - uL[3];
  const T di = dsqrt(rR * irL);
  const T d1 = 1.0 / (1.0 + di);
  const T ui = (di * vxR + vxL) * d1;
  const T vi = (di * vyR + vyL) * d1;
  const T Hi = (di * HR + HL) * d1;
  const T af = 0.5 * (ui * ui + vi * vi);
  const T ucp = ui * nx + vi * ny;
  const T c2 = kGm1 * (Hi - af);
  if (code == 0 && val(c2) <= 0) code = 3;
  const T ci = c2 * c2;
  const T ci1 = 1.0 / ci;
  const T eps = 0.1 * ci;
  const T ieps = 10.0 * ci1;
  T l0 = ucp + ci, l1 = ucp - ci, l3 = ucp;
  l0 = val(dabs(l0)) < val(eps) ? 0.5 * (eps + l0 * l0 * ieps) : dabs(l0);
  l1 = val(dabs(l1)) < val(eps) ? 0.5 * (eps + l1 * l1 * ieps) : dabs(l1);
  l3 = val(dabs(l3)) < val(eps) ? 0.5 * (eps + l3 * l3 * ieps) : dabs(l3);
  const T s1 = 0.5 * (l0 + l1);
  const T s2 = 0.5 * (l0 - l1);
  const T G1 = kGm1 * (af * du0 - ui * du1 - vi * du2 + du3);
  const T G2 = -ucp * du0 + du1 * nx + du2 * ny;
  const T C1 = (G1 * (s1 - l3) * ci1 + G2 * s2) * ci1;
  const T C2 = G1 * s2 * ci1 + G2 * (s1 - l3);
  f[0] = 0.5 * ((uL[1] * nx + uL[2] * ny) + (uR[1] * nx + uR[2] * ny)) - 0.5 * (l3 * du0 + C1);
  f[1] = 0.5 * ((uL[1] * unL + pL * nx) + (uR[1] * unR + pR * nx)) - 0.5 * (l3 * du1 + C1 * ui + C2 * nx);
  f[2] = 0.5 * ((uL[2] * unL + pL * ny) + (uR[2] * unR + pR * ny)) - 0.5 * (l3 * du2 + C1 * vi + C2 * ny);
  f[3] = 0.5 * (rHL * unL + rHR * unR) - 0.5 * (l3 * du3 + C1 * Hi + C2 * ucp);
  return code;
}

template <typename T>
__host__ __device__ inline void contravariant_flux_t(const T* s, double j00, double j01, double j10,
                                                     double j11, T* gxi, T* geta) {
  const T ir = 1.0 / s[0];
  const T vx = s[1] * ir, vy = s[2] * ir;
  const T p = kGm1 * (s[3] - 0.5 * (s[1] * vx + s[2] * vy));
  const T rH = s[3] + p;
  const T fx[4] = {s[1], s[1] * vx + p, s[2] * vx, rH * vx};
  const T fy[4] = {s[2], s[1] * vy, s[2] * vy + p, rH * vy};
  for (int c = 0; c < 4; ++c) {
    gxi[c] = j00 * fx[c] + j01 * fy[c];
    geta[c] = j10 * fx[c] + j11 * fy[c];
  }
}

// ---- reverse sweeps ------------------------------------------------------------------
// bf: adjoint of the flux (4). Adds the adjoints of uL and uR to buL, buR.
__host__ __device__ inline void roe_flux_vjp(const double* uL, const double* uR, double nx, double ny,
                                             const double* bf, double* buL, double* buR) {
  // forward recomputation of the intermediates
  const double rL = uL[0], rR = uR[0];
  const double irLR = rcp(rL * rR);
  const double irL = rR * irLR, irR = rL * irLR;
  const double vxL = uL[1] * irL, vyL = uL[2] * irL;
  const double unL = vxL * nx + vyL * ny;
  const double pL = kGm1 * (uL[3] - 0.5 * (uL[1] * vxL + uL[2] * vyL));
  const double rHL = uL[3] + pL;
  const double HL = rHL * irL;
  const double vxR = uR[1] * irR, vyR = uR[2] * irR;
  const double unR = vxR * nx + vyR * ny;
  const double pR = kGm1 * (uR[3] - 0.5 * (uR[1] * vxR + uR[2] * vyR));
  const double rHR = uR[3] + pR;
  const double HR = rHR * irR;
  const double du0 = uR[0] - uL[0], du1 = uR[1] - uL[1], du2 = uR[2] - uL[2], du3 = uR[3] - uL[3];
  const double di = sqrt(rR * irL);
  const double d1 = rcp(1.0 + di);
  const double ui = (di * vxR + vxL) * d1;
  const double vi = (di * vyR + vyL) * d1;
  const double Hi = (di * HR + HL) * d1;
  const double af = 0.5 * (ui * ui + vi * vi);
  const double ucp = ui * nx + vi * ny;
  const double c2 = kGm1 * (Hi - af);
  const double ci = c2 * c2;
  const double ci1 = rcp(ci);
  const double eps = 0.1 * ci;
  const double ieps = 10.0 * ci1;
  const double l0r = ucp + ci, l1r = ucp - ci, l3r = ucp;
  const bool fx0 = fabs(l0r) < eps, fx1 = fabs(l1r) < eps, fx3 = fabs(l3r) < eps;
  const double L0 = fx0 ? 0.5 * (eps + l0r * l0r * ieps) : fabs(l0r);
  const double L1 = fx1 ? 0.5 * (eps + l1r * l1r * ieps) : fabs(l1r);
  const double L3 = fx3 ? 0.5 * (eps + l3r * l3r * ieps) : fabs(l3r);
  const double s1 = 0.5 * (L0 + L1);
  const double s2 = 0.5 * (L0 - L1);
  const double G1 = kGm1 * (af * du0 - ui * du1 - vi * du2 + du3);
  const double G2 = -ucp * du0 + du1 * nx + du2 * ny;
  const double A = G1 * (s1 - L3) * ci1 + G2 * s2;
  const double C1 = A * ci1;
  const double C2 = G1 * s2 * ci1 + G2 * (s1 - L3);

  // flux assembly
  double b_uL1 = 0.5 * bf[0] * nx + 0.5 * bf[1] * unL;
  double b_uL2 = 0.5 * bf[0] * ny + 0.5 * bf[2] * unL;
  double b_uR1 = 0.5 * bf[0] * nx + 0.5 * bf[1] * unR;
  double b_uR2 = 0.5 * bf[0] * ny + 0.5 * bf[2] * unR;
  double b_unL = 0.5 * (bf[1] * uL[1] + bf[2] * uL[2] + bf[3] * rHL);
  double b_unR = 0.5 * (bf[1] * uR[1] + bf[2] * uR[2] + bf[3] * rHR);
  double b_pL = 0.5 * (bf[1] * nx + bf[2] * ny);
  double b_pR = b_pL;
  double b_rHL = 0.5 * bf[3] * unL;
  double b_rHR = 0.5 * bf[3] * unR;
  double b_L3 = -0.5 * (bf[0] * du0 + bf[1] * du1 + bf[2] * du2 + bf[3] * du3);
  double b_du0 = -0.5 * L3 * bf[0], b_du1 = -0.5 * L3 * bf[1];
  double b_du2 = -0.5 * L3 * bf[2], b_du3 = -0.5 * L3 * bf[3];
  const double b_C1 = -0.5 * (bf[0] + bf[1] * ui + bf[2] * vi + bf[3] * Hi);
  const double b_C2 = -0.5 * (bf[1] * nx + bf[2] * ny + bf[3] * ucp);
  double b_ui = -0.5 * bf[1] * C1;
  double b_vi = -0.5 * bf[2] * C1;
  double b_Hi = -0.5 * bf[3] * C1;
  double b_ucp = -0.5 * bf[3] * C2;
  // C2 = G1 s2 ci1 + G2 (s1 - L3)
  double b_G1 = b_C2 * s2 * ci1;
  double b_s2 = b_C2 * G1 * ci1;
  double b_ci1 = b_C2 * G1 * s2;
  double b_G2 = b_C2 * (s1 - L3);
  double b_s1 = b_C2 * G2;
  b_L3 -= b_C2 * G2;
  // C1 = A ci1, A = G1 (s1 - L3) ci1 + G2 s2
  const double b_A = b_C1 * ci1;
  b_ci1 += b_C1 * A;
  b_G1 += b_A * (s1 - L3) * ci1;
  b_s1 += b_A * G1 * ci1;
  b_L3 -= b_A * G1 * ci1;
  b_ci1 += b_A * G1 * (s1 - L3);
  b_G2 += b_A * s2;
  b_s2 += b_A * G2;
  // G2 = -ucp du0 + du1 nx + du2 ny
  b_ucp -= b_G2 * du0;
  b_du0 -= b_G2 * ucp;
  b_du1 += b_G2 * nx;
  b_du2 += b_G2 * ny;
  // G1 = (gamma-1) (af du0 - ui du1 - vi du2 + du3)
  const double tg = kGm1 * b_G1;
  double b_af = tg * du0;
  b_du0 += tg * af;
  b_ui -= tg * du1;
  b_du1 -= tg * ui;
  b_vi -= tg * du2;
  b_du2 -= tg * vi;
  b_du3 += tg;
  // s1 = (L0 + L1) / 2, s2 = (L0 - L1) / 2
  const double b_L0 = 0.5 * (b_s1 + b_s2);
  const double b_L1 = 0.5 * (b_s1 - b_s2);
  // entropy fix: L = |l| < eps ? (eps + l^2 ieps) / 2 : |l|
  double b_eps = 0.0, b_ieps = 0.0;
  double b_l0, b_l1, b_l3;
  if (fx0) {
    b_l0 = b_L0 * l0r * ieps;
    b_eps += 0.5 * b_L0;
    b_ieps += 0.5 * b_L0 * l0r * l0r;
  } else {
    b_l0 = l0r < 0 ? -b_L0 : b_L0;
  }
  if (fx1) {
    b_l1 = b_L1 * l1r * ieps;
    b_eps += 0.5 * b_L1;
    b_ieps += 0.5 * b_L1 * l1r * l1r;
  } else {
    b_l1 = l1r < 0 ? -b_L1 : b_L1;
  }
  if (fx3) {
    b_l3 = b_L3 * l3r * ieps;
    b_eps += 0.5 * b_L3;
    b_ieps += 0.5 * b_L3 * l3r * l3r;
  } else {
    b_l3 = l3r < 0 ? -b_L3 : b_L3;
  }
  // l0 = ucp + ci, l1 = ucp - ci, l3 = ucp; eps = ci / 10, ieps = 10 ci1
  b_ucp += b_l0 + b_l1 + b_l3;
  double b_ci = b_l0 - b_l1 + 0.1 * b_eps;
  b_ci1 += 10.0 * b_ieps;
  // ci1 = 1 / ci, ci = c2^2, c2 = (gamma-1) (Hi - af)
  b_ci -= b_ci1 * ci1 * ci1;
  const double b_c2 = 2.0 * c2 * b_ci;
  b_Hi += kGm1 * b_c2;
  b_af -= kGm1 * b_c2;
  // ucp = ui nx + vi ny; af = (ui^2 + vi^2) / 2
  b_ui += b_ucp * nx + b_af * ui;
  b_vi += b_ucp * ny + b_af * vi;
  // ui = (di vxR + vxL) d1 and likewise vi, Hi
  const double b_d1 = b_ui * (di * vxR + vxL) + b_vi * (di * vyR + vyL) + b_Hi * (di * HR + HL);
  double b_di = d1 * (b_ui * vxR + b_vi * vyR + b_Hi * HR);
  double b_vxR = b_ui * di * d1, b_vxL = b_ui * d1;
  double b_vyR = b_vi * di * d1, b_vyL = b_vi * d1;
  const double b_HR = b_Hi * di * d1, b_HL = b_Hi * d1;
  // d1 = 1 / (1 + di); di = sqrt(rR irL)
  b_di -= b_d1 * d1 * d1;
  const double b_q = b_di * 0.5 * rcp(di);
  double b_rR = b_q * irL;
  double b_irL = b_q * rR;
  // du = uR - uL
  double b_uR0 = b_du0, b_uL0 = -b_du0;
  b_uR1 += b_du1;
  b_uL1 -= b_du1;
  b_uR2 += b_du2;
  b_uL2 -= b_du2;
  double b_uR3 = b_du3, b_uL3 = -b_du3;
  // right state: HR = rHR irR, rHR = uR3 + pR, pR, unR, vxR, vyR
  b_rHR += b_HR * irR;
  double b_irR = b_HR * rHR;
  b_uR3 += b_rHR;
  b_pR += b_rHR;
  const double tR = kGm1 * b_pR;
  b_uR3 += tR;
  b_uR1 -= 0.5 * tR * vxR;
  b_vxR -= 0.5 * tR * uR[1];
  b_uR2 -= 0.5 * tR * vyR;
  b_vyR -= 0.5 * tR * uR[2];
  b_vxR += b_unR * nx;
  b_vyR += b_unR * ny;
  b_uR1 += b_vxR * irR;
  b_irR += b_vxR * uR[1];
  b_uR2 += b_vyR * irR;
  b_irR += b_vyR * uR[2];
  // left state, the same
  b_rHL += b_HL * irL;
  b_irL += b_HL * rHL;
  b_uL3 += b_rHL;
  b_pL += b_rHL;
  const double tL = kGm1 * b_pL;
  b_uL3 += tL;
  b_uL1 -= 0.5 * tL * vxL;
  b_vxL -= 0.5 * tL * uL[1];
  b_uL2 -= 0.5 * tL * vyL;
  b_vyL -= 0.5 * tL * uL[2];
  b_vxL += b_unL * nx;
  b_vyL += b_unL * ny;
  b_uL1 += b_vxL * irL;
  b_irL += b_vxL * uL[1];
  b_uL2 += b_vyL * irL;
  b_irL += b_vyL * uL[2];
  // irL = rR irLR, irR = rL irLR, irLR = 1 / (rL rR)
  b_rR += b_irL * irLR;
  const double b_irLR = b_irL * rR + b_irR * rL;
  double b_rL = b_irR * irLR;
  const double b_prod = -b_irLR * irLR * irLR;
  b_rL += b_prod * rR;
  b_rR += b_prod * rL;
  b_uL0 += b_rL;
  b_uR0 += b_rR;
  buL[0] += b_uL0;
  buL[1] += b_uL1;
  buL[2] += b_uL2;
  buL[3] += b_uL3;
  buR[0] += b_uR0;
  buR[1] += b_uR1;
  buR[2] += b_uR2;
  buR[3] += b_uR3;
}

// bgxi, bgeta: adjoints of the contravariant flux (4 each); adds the state's adjoint to bs.
__host__ __device__ inline void contravariant_vjp(const double* s, double j00, double j01, double j10, double j11,
                                                  const double* bgxi, const double* bgeta, double* bs) {
  const double ir = rcp(s[0]);
  const double vx = s[1] * ir, vy = s[2] * ir;
  const double p = kGm1 * (s[3] - 0.5 * (s[1] * vx + s[2] * vy));
  const double rH = s[3] + p;
  double bfx[4], bfy[4];
  for (int c = 0; c < 4; ++c) {
    bfx[c] = j00 * bgxi[c] + j10 * bgeta[c];
    bfy[c] = j01 * bgxi[c] + j11 * bgeta[c];
  }
  // fx = (s1, s1 vx + p, s2 vx, rH vx), fy = (s2, s1 vy, s2 vy + p, rH vy)
  double b_s1 = bfx[0] + bfx[1] * vx + bfy[1] * vy;
  double b_s2 = bfx[2] * vx + bfy[0] + bfy[2] * vy;
  double b_vx = bfx[1] * s[1] + bfx[2] * s[2] + bfx[3] * rH;
  double b_vy = bfy[1] * s[1] + bfy[2] * s[2] + bfy[3] * rH;
  double b_p = bfx[1] + bfy[2];
  const double b_rH = bfx[3] * vx + bfy[3] * vy;
  double b_s3 = b_rH;
  b_p += b_rH;
  const double t = kGm1 * b_p;
  b_s3 += t;
  b_s1 -= 0.5 * t * vx;
  b_vx -= 0.5 * t * s[1];
  b_s2 -= 0.5 * t * vy;
  b_vy -= 0.5 * t * s[2];
  b_s1 += b_vx * ir;
  b_s2 += b_vy * ir;
  const double b_ir = b_vx * s[1] + b_vy * s[2];
  bs[0] += -b_ir * ir * ir;
  bs[1] += b_s1;
  bs[2] += b_s2;
  bs[3] += b_s3;
}

}  // namespace vt
