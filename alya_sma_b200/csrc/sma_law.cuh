// sma_law.cuh -- device math of the explicit SMA step: HEX08 reference
// element, the law-160 Kirchhoff stress and its return map.
//
// Law 160 (Alya solidz, sld_stress_model_160.f90:212-500) computes the
// Kirchhoff stress from the logarithmic principal stretches of b = F F^T:
//   tau = K (theta - 3 alpha eL xS) I + sum_i 2G (e_i - eL xS e_i/|e|) n_i n_i^T
// which is an isotropic function of b:
//   tau = pv I + kappa dev(ln V),  ln V = 1/2 log(b),
//   pv = K (theta - 3 alpha eL xS),  kappa = 2G (1 - eL xS / |e|).
// Only the matrix logarithm log(b) = log1p(A), A = b - I = H + H^T + H H^T
// (H = F - I), and the eigenvalues of A are needed; no eigenvectors.  The
// device evaluates log1p(A) by Newton-form interpolation of log1p at the
// eigenvalues of A (primary matrix function; Higham, Functions of Matrices,
// SIAM 2008, sect. 1.2), with the eigenvalues from the trigonometric
// closed form for 3x3 symmetric matrices (Smith, CACM 4(4) 1961) and the
// divided differences written so that clustered eigenvalues cancel
// nothing.  Working on A rather than b keeps the small strains of an
// explicit step at full relative precision, which is what lets the FP32 form
// meet its error target.  The reference sorts eigenpairs (eigsrt.f90); the
// interpolation is symmetric in the eigenvalues, so no sort is needed.
//
// The return map (martensite fraction, sld_stress_model_160.f90:335-484) is
// scalar work and always runs in FP64, restating the reference's
// Newton-Raphson loop step for step (65 iterations, tolerance 1e-8 with the
// squared first residual).  With the linear flow rule its residual is linear
// in xS, so it converges in one iteration.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sma {

// NR flags (match the CPU oracle)
constexpr int NR_NONE = 0, NR_CONVERGED = 1, NR_FAILED = 2, NR_BOTH = 4;

// Per-material constants, precomputed on the host as the reference computes
// them (sld_stress_model_160.f90:282-289).
struct MatC {
  double K, G, G1, eL;          // bulk, shear, (2G + 9 a^2 K) eL, eL
  double alfa, C_AS, C_SA;      // alpha, Clausius-Clapeyron slopes
  double Rs_AS, Rf_AS, Rs_SA, Rf_SA;
  double EA, EM, nu;            // extension: Reuss modulus E(xS0) when EM != EA
  double densi;
  int ext_E;                    // 1: E depends on xS0
  int pad;
};

// ---------------------------------------------------------------------------
// scalar helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float  dlog1p(float x)  { return log1pf(x); }
__device__ __forceinline__ double dlog1p(double x) { return log1p(x); }
__device__ __forceinline__ float  dsqrt(float x)   { return sqrtf(x); }
__device__ __forceinline__ double dsqrt(double x)  { return sqrt(x); }
__device__ __forceinline__ float  dacos(float x)   { return acosf(x); }
__device__ __forceinline__ double dacos(double x)  { return acos(x); }
__device__ __forceinline__ void dsincos(float x, float* s, float* c)    { sincosf(x, s, c); }
__device__ __forceinline__ void dsincos(double x, double* s, double* c) { sincos(x, s, c); }

template <typename T> struct Eps;
template <> struct Eps<float>  {
  static __device__ __forceinline__ float series() { return 1e-3f; }   // |w| below: series
  static __device__ __forceinline__ float dd2()    { return 1e-4f; }   // clustered spread
};
template <> struct Eps<double> {
  static __device__ __forceinline__ double series() { return 1e-3; }
  static __device__ __forceinline__ double dd2()    { return 1e-8; }
};

// log1p(w)/w, accurate for all w > -1 (series below |w| < 1e-3: the
// truncation error w^7/8 < 1.3e-22).
template <typename T>
__device__ __forceinline__ T log1p_ratio(T w) {
  if (fabs(w) < Eps<T>::series()) {
    return T(1) + w * (T(-0.5) + w * (T(1) / T(3) + w * (T(-0.25) + w * (T(0.2) +
           w * (T(-1) / T(6) + w * (T(1) / T(7)))))));
  }
  return dlog1p(w) / w;
}

// ---------------------------------------------------------------------------
// log1p of a symmetric 3x3 matrix.  A, L stored as (xx, yy, zz, xy, yz, xz).
// f[3] receives log1p of the three eigenvalues of A (any order).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void sym_log1p(const T* A, T* L, T* f) {
  const T m = (A[0] + A[1] + A[2]) * (T(1) / T(3));
  const T a0 = A[0] - m, a1 = A[1] - m, a2 = A[2] - m;
  const T off = A[3] * A[3] + A[4] * A[4] + A[5] * A[5];
  const T p2 = (a0 * a0 + a1 * a1 + a2 * a2 + T(2) * off) * (T(1) / T(6));
  const T p = dsqrt(p2);
  // det(A - m I)
  const T det = a0 * (a1 * a2 - A[4] * A[4]) - A[3] * (A[3] * a2 - A[4] * A[5])
              + A[5] * (A[3] * A[4] - a1 * A[5]);
  T r = (p2 > T(1e-30)) ? det / (T(2) * p2 * p) : T(0);
  r = fmin(fmax(r, T(-1)), T(1));
  const T phi = dacos(r) * (T(1) / T(3));
  T sn, cs;
  dsincos(phi, &sn, &cs);
  const T d0 = m + T(2) * p * cs;                                          // largest
  const T d2 = m + T(2) * p * (T(-0.5) * cs - T(0.86602540378443864676) * sn);  // smallest
  const T d1 = T(3) * m - d0 - d2;
  // (u, v): the closest pair, s: the remaining eigenvalue
  const bool lo = (d0 - d1) <= (d1 - d2);
  const T u = lo ? d0 : d1;
  const T v = lo ? d1 : d2;
  const T s = lo ? d2 : d0;
  const T fu = dlog1p(u), fv = dlog1p(v), fs = dlog1p(s);
  f[0] = fs; f[1] = fu; f[2] = fv;
  const T iv = T(1) / (T(1) + v);
  const T fuv = log1p_ratio((u - v) * iv) * iv;              // f[u,v]
  const T fsv = log1p_ratio((s - v) * iv) * iv;              // f[s,v]
  const T dsu = s - u;
  T fsuv;                                                    // f[s,u,v]
  if (fabs(dsu) > Eps<T>::dd2()) fsuv = (fsv - fuv) / dsu;
  else { const T q = T(1) / (T(1) + m); fsuv = T(-0.5) * q * q; }
  // L = fv I + f[u,v] (A - v I) + f[s,u,v] (A - u I)(A - v I)
  //   = c0 I + c1 A + c2 A^2
  const T c2 = fsuv;
  const T c1 = fuv - fsuv * (u + v);
  const T c0 = fv - fuv * v + fsuv * u * v;
  const T s00 = A[0] * A[0] + A[3] * A[3] + A[5] * A[5];
  const T s11 = A[3] * A[3] + A[1] * A[1] + A[4] * A[4];
  const T s22 = A[5] * A[5] + A[4] * A[4] + A[2] * A[2];
  const T s01 = A[0] * A[3] + A[3] * A[1] + A[5] * A[4];
  const T s12 = A[3] * A[5] + A[1] * A[4] + A[4] * A[2];
  const T s02 = A[0] * A[5] + A[3] * A[4] + A[5] * A[2];
  L[0] = c0 + c1 * A[0] + c2 * s00;
  L[1] = c0 + c1 * A[1] + c2 * s11;
  L[2] = c0 + c1 * A[2] + c2 * s22;
  L[3] = c1 * A[3] + c2 * s01;
  L[4] = c1 * A[4] + c2 * s12;
  L[5] = c1 * A[5] + c2 * s02;
}

// ---------------------------------------------------------------------------
// Return map of law 160 in FP64: eval_loading_function (:513-537, beta = 1),
// activation (:342-374), Newton-Raphson (:389-465), clamp (:484).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double loading(double K, double G, double alfa, double C,
                                          double eL, double theta, double enor,
                                          double tmp, double xS) {
  double pres = K * (theta - 3.0 * alfa * eL * xS);
  double trac = 2.0 * G * (enor - eL * xS);
  return trac * 1.0 + 3.0 * alfa * pres - C * tmp;
}

struct RMOut { double xS, F_AS, F_SA; int flag; };

__device__ __forceinline__ RMOut return_map(const MatC& m, double K, double G, double G_1,
                                            double theta, double e_n, double tmp,
                                            double xS_0, double F_AS_0, double F_SA_0) {
  RMOut o;
  o.flag = NR_NONE;
  double F_AS = loading(K, G, m.alfa, m.C_AS, m.eL, theta, e_n, tmp, xS_0);
  double F_AS_dot = F_AS - F_AS_0;
  const bool kf_AS = (F_AS > F_AS_0) && (F_AS - m.Rs_AS > 0.0) && (xS_0 < 1.0);
  double F_SA = loading(K, G, m.alfa, m.C_SA, m.eL, theta, e_n, tmp, xS_0);
  double F_SA_dot = F_SA - F_SA_0;
  const bool kf_SA = (F_SA < F_SA_0) && (F_SA - m.Rs_SA < 0.0) && (xS_0 > 0.0);
  if (kf_AS && kf_SA) o.flag |= NR_BOTH;
  double xS = xS_0;
  if (kf_AS || kf_SA) {
    const double H_AS = kf_AS ? 1.0 : 0.0, H_SA = kf_SA ? 1.0 : 0.0;
    double dh_SA = 0.0, dh_AS = 0.0;
    int iter = 0;
    double RHS_AS = (F_AS - m.Rf_AS) * dh_AS + H_AS * F_AS_dot * (1.0 - xS);
    double RHS_SA = (F_SA - m.Rf_SA) * dh_SA - H_SA * F_SA_dot * xS;
    double resi = RHS_AS * RHS_AS + RHS_SA * RHS_SA;
    while (iter < 65 && resi > 1.0e-8) {
      ++iter;
      const double m11 = -G_1 * dh_AS - (H_AS * F_AS_dot + H_AS * (1.0 - xS) * G_1) + (F_AS - m.Rf_AS);
      const double m12 = -G_1 * dh_AS - (H_AS * F_AS_dot + H_AS * (1.0 - xS) * G_1);
      const double m21 = -G_1 * dh_SA - (H_SA * F_SA_dot - H_SA * xS * G_1);
      const double m22 = -G_1 * dh_SA - (H_SA * F_SA_dot - H_SA * xS * G_1) + (F_SA - m.Rf_SA);
      const double det = m11 * m22 - m12 * m21;
      const double sol1 = (m22 / det) * RHS_AS + (-m12 / det) * RHS_SA;
      const double sol2 = (-m21 / det) * RHS_AS + (m11 / det) * RHS_SA;
      dh_AS = dh_AS - sol1;
      dh_SA = dh_SA - sol2;
      xS = xS + dh_SA + dh_AS;
      F_AS = loading(K, G, m.alfa, m.C_AS, m.eL, theta, e_n, tmp, xS);
      F_AS_dot = F_AS - F_AS_0;
      F_SA = loading(K, G, m.alfa, m.C_SA, m.eL, theta, e_n, tmp, xS);
      F_SA_dot = F_SA - F_SA_0;
      RHS_AS = (F_AS - m.Rf_AS) * dh_AS + H_AS * F_AS_dot * (1.0 - xS);
      RHS_SA = (F_SA - m.Rf_SA) * dh_SA - H_SA * F_SA_dot * xS;
      resi = sqrt(RHS_AS * RHS_AS + RHS_SA * RHS_SA);
    }
    if (iter >= 65) {
      o.flag |= NR_FAILED;
      F_AS = F_AS_0;
      F_SA = F_SA_0;
      xS = xS_0;
    } else {
      o.flag |= NR_CONVERGED;
    }
  }
  xS = fmin(xS, 1.0);
  xS = fmax(xS, 0.0);
  o.xS = xS;
  o.F_AS = F_AS;
  o.F_SA = F_SA;
  return o;
}

// ---------------------------------------------------------------------------
// Kirchhoff stress of law 160 from H = F - I.  state = (xS, F_AS, F_SA) of
// the previous step; on return the new state.  tau as (xx,yy,zz,xy,yz,xz).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ int law160_tau(const MatC& m, const T* H, double tmp,
                                          double& xS, double& F_AS, double& F_SA, T* tau) {
  // A = b - I = H + H^T + H H^T, H row-major (H[3i+j] = du_i/dX_j)
  T A[6];
  A[0] = T(2) * H[0] + (H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
  A[1] = T(2) * H[4] + (H[3] * H[3] + H[4] * H[4] + H[5] * H[5]);
  A[2] = T(2) * H[8] + (H[6] * H[6] + H[7] * H[7] + H[8] * H[8]);
  A[3] = H[1] + H[3] + (H[0] * H[3] + H[1] * H[4] + H[2] * H[5]);   // (0,1)
  A[4] = H[5] + H[7] + (H[3] * H[6] + H[4] * H[7] + H[5] * H[8]);   // (1,2)
  A[5] = H[2] + H[6] + (H[0] * H[6] + H[1] * H[7] + H[2] * H[8]);   // (0,2)
  T L[6], f[3];
  sym_log1p(A, L, f);
  // logarithmic strains (:313-332): ln(lambda_i) = f_i/2
  const T theta_t = T(0.5) * (f[0] + f[1] + f[2]);
  const T t3 = theta_t * (T(1) / T(3));
  const T e0 = T(0.5) * f[0] - t3, e1 = T(0.5) * f[1] - t3, e2 = T(0.5) * f[2] - t3;
  const T en_t = dsqrt(e0 * e0 + e1 * e1 + e2 * e2);
  // moduli (extension: Reuss E at the start-of-step fraction)
  double K = m.K, G = m.G, G_1 = m.G1;
  if (m.ext_E) {
    const double E = 1.0 / ((1.0 - xS) / m.EA + xS / m.EM);
    K = E / (3.0 - 6.0 * m.nu);
    G = E / (2.0 + 2.0 * m.nu);
    G_1 = (2.0 * G + 9.0 * (m.alfa * m.alfa) * K) * m.eL;
  }
  const double theta = (double)theta_t, e_n = (double)en_t;
  RMOut r = return_map(m, K, G, G_1, theta, e_n, tmp, xS, F_AS, F_SA);
  xS = r.xS;
  F_AS = r.F_AS;
  F_SA = r.F_SA;
  // tau = pv I + kappa (L/2 - theta/3 I)   (:487-491)
  const double pv = K * (theta - 3.0 * m.alfa * m.eL * xS);
  const double kap = (e_n > 2.220446049250313e-16) ? 2.0 * G * (1.0 - m.eL * xS / e_n) : 2.0 * G;
  const T kp = (T)kap;
  const T dg = (T)pv - kp * t3;
  tau[0] = dg + kp * T(0.5) * L[0];
  tau[1] = dg + kp * T(0.5) * L[1];
  tau[2] = dg + kp * T(0.5) * L[2];
  tau[3] = kp * T(0.5) * L[3];
  tau[4] = kp * T(0.5) * L[4];
  tau[5] = kp * T(0.5) * L[5];
  return r.flag;
}

// inverse and determinant of a general 3x3 (row-major M[3*i+j])
template <typename T>
__device__ __forceinline__ T inv3(const T* M, T* Mi) {
  const T c00 = M[4] * M[8] - M[5] * M[7];
  const T c01 = M[5] * M[6] - M[3] * M[8];
  const T c02 = M[3] * M[7] - M[4] * M[6];
  const T det = M[0] * c00 + M[1] * c01 + M[2] * c02;
  const T id = T(1) / det;
  Mi[0] = c00 * id;
  Mi[3] = c01 * id;
  Mi[6] = c02 * id;
  Mi[1] = (M[2] * M[7] - M[1] * M[8]) * id;
  Mi[4] = (M[0] * M[8] - M[2] * M[6]) * id;
  Mi[7] = (M[1] * M[6] - M[0] * M[7]) * id;
  Mi[2] = (M[1] * M[5] - M[2] * M[4]) * id;
  Mi[5] = (M[2] * M[3] - M[0] * M[5]) * id;
  Mi[8] = (M[0] * M[4] - M[1] * M[3]) * id;
  return det;
}

// ---------------------------------------------------------------------------
// HEX08 at Gauss point g: shape functions and derivatives
// (mod_lagrange.f90:935-977; point order of mod_quadrature_gauss.f90:2373-2385
// with the reference's 15-digit abscissa).  dN[3*a + j] = dN_a/dxi_j.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void hex8_gp(int g, T* N, T* dN) {
  const T p = T(0.577350269189626);
  const T s = (g & 4) ? p : -p;
  const T t = (g & 2) ? p : -p;
  const T z = (g & 1) ? p : -p;
  const T sm = T(0.5) * (T(1) - s), sq = T(0.5) * (T(1) + s);
  const T tm = T(0.5) * (T(1) - t), tp = T(0.5) * (T(1) + t);
  const T zm = T(0.5) * (T(1) - z), zp = T(0.5) * (T(1) + z);
  const T h = T(0.5);
  if (N) {
    N[0] = sm * tm * zm; N[1] = sq * tm * zm; N[2] = sq * tp * zm; N[3] = sm * tp * zm;
    N[4] = sm * tm * zp; N[5] = sq * tm * zp; N[6] = sq * tp * zp; N[7] = sm * tp * zp;
  }
  dN[0]  = -h * tm * zm; dN[1]  = -h * sm * zm; dN[2]  = -h * sm * tm;
  dN[3]  =  h * tm * zm; dN[4]  = -h * sq * zm; dN[5]  = -h * sq * tm;
  dN[6]  =  h * tp * zm; dN[7]  =  h * sq * zm; dN[8]  = -h * sq * tp;
  dN[9]  = -h * tp * zm; dN[10] =  h * sm * zm; dN[11] = -h * sm * tp;
  dN[12] = -h * tm * zp; dN[13] = -h * sm * zp; dN[14] =  h * sm * tm;
  dN[15] =  h * tm * zp; dN[16] = -h * sq * zp; dN[17] =  h * sq * tm;
  dN[18] =  h * tp * zp; dN[19] =  h * sq * zp; dN[20] =  h * sq * tp;
  dN[21] = -h * tp * zp; dN[22] =  h * sm * zp; dN[23] =  h * sm * tp;
}

}  // namespace sma
