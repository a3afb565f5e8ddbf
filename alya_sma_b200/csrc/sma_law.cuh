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
  double iEA, iEM;              // 1/EA, 1/EM
  double kK, kG;                // 1/(3 - 6 nu), 1/(2 + 2 nu)
  double densi;
  int ext_E;                    // 1: E depends on xS0
  int pad;
  double ray_a;                 // Rayleigh alpha (mass-proportional damping), 0: none
  double T0;                    // base temperature of compact per-element records
};

// ---------------------------------------------------------------------------
// scalar helpers.  Fm<double> calls the accurate library functions; Fm<float>
// (the precision form) uses fast reciprocals and short series whose error
// stays at a few FP32 ulp on the ranges they are used on.
// ---------------------------------------------------------------------------
template <typename T> struct Fm;

template <> struct Fm<double> {
  static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
  static __device__ __forceinline__ double div(double a, double b) { return a / b; }
  static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
  static __device__ __forceinline__ double acos_(double x) { return acos(x); }
  static __device__ __forceinline__ double log1p_(double x) { return log1p(x); }
  // log1p(w)/w; series below |w| < 1e-3 (truncation w^7/8 < 1.3e-22)
  static __device__ __forceinline__ double log1p_ratio(double w) {
    if (fabs(w) < 1e-3)
      return 1.0 + w * (-0.5 + w * (1.0 / 3.0 + w * (-0.25 + w * (0.2 + w * (-1.0 / 6.0 + w * (1.0 / 7.0))))));
    return log1p(w) / w;
  }
  // cos and sin of phi in [0, pi/3] by Taylor series (truncation < 1e-18)
  static __device__ __forceinline__ void sincos_third(double x, double* s, double* c) {
    const double x2 = x * x;
    *c = 1.0 + x2 * (-1.0 / 2 + x2 * (1.0 / 24 + x2 * (-1.0 / 720 + x2 * (1.0 / 40320 + x2 * (-1.0 / 3628800 +
         x2 * (1.0 / 479001600 + x2 * (-1.0 / 87178291200.0 + x2 * (1.0 / 20922789888000.0 +
         x2 * (-1.0 / 6402373705728000.0)))))))));
    *s = x * (1.0 + x2 * (-1.0 / 6 + x2 * (1.0 / 120 + x2 * (-1.0 / 5040 + x2 * (1.0 / 362880 +
         x2 * (-1.0 / 39916800 + x2 * (1.0 / 6227020800.0 + x2 * (-1.0 / 1307674368000.0 +
         x2 * (1.0 / 355687428096000.0 + x2 * (-1.0 / 121645100408832000.0))))))))));
  }
  static __device__ __forceinline__ double clustered() { return 1e-8; }
  // first divided difference f[u,v] of log1p, given fu = log1p(u), fv =
  // log1p(v) and iv = 1/(1+v): the series of log1p(w)/w for near-equal
  // arguments (|w| < 1e-3, w = (u-v)/(1+v)), else the difference quotient of
  // the values already computed (cancellation below 1e-13 relative there)
  static __device__ __forceinline__ double ddiff(double u, double v, double fu, double fv, double iv) {
    const double w = (u - v) * iv;
    if (fabs(w) < 1e-3) return log1p_ratio(w) * iv;
    return (fu - fv) / (u - v);
  }
};

template <> struct Fm<float> {
  static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
  static __device__ __forceinline__ float sqrt_(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }
  static __device__ __forceinline__ float acos_(float x) { return acosf(x); }
  // log1p(x) = 2 atanh(s), s = x/(2+x): series to s^9 for |x| <= 0.25
  // (|s| <= 1/7, truncation 2 s^11/11 < 6e-11 relative)
  static __device__ __forceinline__ float log1p_(float x) {
    if (fabsf(x) > 0.25f) return log1pf(x);
    const float s = __fdividef(x, 2.0f + x);
    const float s2 = s * s;
    return 2.0f * s * (1.0f + s2 * (1.0f / 3 + s2 * (1.0f / 5 + s2 * (1.0f / 7 + s2 * (1.0f / 9)))));
  }
  // log1p(w)/w = 2/(2+w) * (1 + s^2/3 + s^4/5 + ...), stable through w = 0
  static __device__ __forceinline__ float log1p_ratio(float w) {
    if (fabsf(w) > 0.25f) return __fdividef(log1pf(w), w);
    const float r = __fdividef(1.0f, 2.0f + w);
    const float s = w * r;
    const float s2 = s * s;
    return 2.0f * r * (1.0f + s2 * (1.0f / 3 + s2 * (1.0f / 5 + s2 * (1.0f / 7 + s2 * (1.0f / 9)))));
  }
  // cos and sin of phi in [0, pi/3] (truncation < 1e-9)
  static __device__ __forceinline__ void sincos_third(float x, float* s, float* c) {
    const float x2 = x * x;
    *c = 1.0f + x2 * (-1.0f / 2 + x2 * (1.0f / 24 + x2 * (-1.0f / 720 + x2 * (1.0f / 40320 +
         x2 * (-1.0f / 3628800 + x2 * (1.0f / 479001600))))));
    *s = x * (1.0f + x2 * (-1.0f / 6 + x2 * (1.0f / 120 + x2 * (-1.0f / 5040 + x2 * (1.0f / 362880 +
         x2 * (-1.0f / 39916800))))));
  }
  static __device__ __forceinline__ float clustered() { return 1e-4f; }
  // f[u,v] of log1p: the series of log1p(w)/w covers |w| <= 0.25, the
  // strains of an explicit step (fu, fv unused)
  static __device__ __forceinline__ float ddiff(float u, float v, float, float, float iv) {
    return log1p_ratio((u - v) * iv) * iv;
  }
};

// ---------------------------------------------------------------------------
// log1p of a symmetric 3x3 matrix.  A, L stored as (xx, yy, zz, xy, yz, xz).
// f[3] receives log1p of the three eigenvalues of A (any order).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void sym_log1p(const T* A, T* L, T* f) {
  using M = Fm<T>;
  const T m = (A[0] + A[1] + A[2]) * (T(1) / T(3));
  const T a0 = A[0] - m, a1 = A[1] - m, a2 = A[2] - m;
  const T off = A[3] * A[3] + A[4] * A[4] + A[5] * A[5];
  const T p2 = (a0 * a0 + a1 * a1 + a2 * a2 + T(2) * off) * (T(1) / T(6));
  const T p = M::sqrt_(p2);
  // det(A - m I)
  const T det = a0 * (a1 * a2 - A[4] * A[4]) - A[3] * (A[3] * a2 - A[4] * A[5])
              + A[5] * (A[3] * A[4] - a1 * A[5]);
  T r = (p2 > T(1e-30)) ? M::div(det, T(2) * p2 * p) : T(0);
  r = fmin(fmax(r, T(-1)), T(1));
  const T phi = M::acos_(r) * (T(1) / T(3));
  T sn, cs;
  M::sincos_third(phi, &sn, &cs);
  const T d0 = m + T(2) * p * cs;                                               // largest
  const T d2 = m + T(2) * p * (T(-0.5) * cs - T(0.86602540378443864676) * sn);  // smallest
  const T d1 = T(3) * m - d0 - d2;
  // (u, v): the closest pair, s: the remaining eigenvalue
  const bool lo = (d0 - d1) <= (d1 - d2);
  const T u = lo ? d0 : d1;
  const T v = lo ? d1 : d2;
  const T s = lo ? d2 : d0;
  const T fu = M::log1p_(u), fv = M::log1p_(v), fs = M::log1p_(s);
  f[0] = fs; f[1] = fu; f[2] = fv;
  const T iv = M::rcp(T(1) + v);
  const T fuv = M::ddiff(u, v, fu, fv, iv);                     // f[u,v]
  const T fsv = M::ddiff(s, v, fs, fv, iv);                     // f[s,v]
  const T dsu = s - u;
  T fsuv;                                                       // f[s,u,v]
  if (fabs(dsu) > M::clustered()) fsuv = M::div(fsv - fuv, dsu);
  else { const T q = M::rcp(T(1) + m); fsuv = T(-0.5) * q * q; }
  // L = fv I + f[u,v] (A - v I) + f[s,u,v] (A - u I)(A - v I) = c0 I + c1 A + c2 A^2
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
    // the reference tests the squared residual on entry (:403) and the norm
    // in the loop (:454); norm > 1e-8 is tested as squared norm > 1e-16
    double r2 = RHS_AS * RHS_AS + RHS_SA * RHS_SA;
    bool go = r2 > 1.0e-8;
    while (iter < 65 && go) {
      ++iter;
      const double m11 = -G_1 * dh_AS - (H_AS * F_AS_dot + H_AS * (1.0 - xS) * G_1) + (F_AS - m.Rf_AS);
      const double m12 = -G_1 * dh_AS - (H_AS * F_AS_dot + H_AS * (1.0 - xS) * G_1);
      const double m21 = -G_1 * dh_SA - (H_SA * F_SA_dot - H_SA * xS * G_1);
      const double m22 = -G_1 * dh_SA - (H_SA * F_SA_dot - H_SA * xS * G_1) + (F_SA - m.Rf_SA);
      const double rdet = 1.0 / (m11 * m22 - m12 * m21);
      const double sol1 = (m22 * RHS_AS - m12 * RHS_SA) * rdet;
      const double sol2 = (m11 * RHS_SA - m21 * RHS_AS) * rdet;
      dh_AS = dh_AS - sol1;
      dh_SA = dh_SA - sol2;
      xS = xS + dh_SA + dh_AS;
      F_AS = loading(K, G, m.alfa, m.C_AS, m.eL, theta, e_n, tmp, xS);
      F_AS_dot = F_AS - F_AS_0;
      F_SA = loading(K, G, m.alfa, m.C_SA, m.eL, theta, e_n, tmp, xS);
      F_SA_dot = F_SA - F_SA_0;
      RHS_AS = (F_AS - m.Rf_AS) * dh_AS + H_AS * F_AS_dot * (1.0 - xS);
      RHS_SA = (F_SA - m.Rf_SA) * dh_SA - H_SA * F_SA_dot * xS;
      r2 = RHS_AS * RHS_AS + RHS_SA * RHS_SA;
      go = r2 > 1.0e-16;
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

// The return map where at most one transformation is active, in closed
// form.  With the linear flow rule the reference's residual (:403-459) is
// linear in xS, so its Newton iteration lands on the solution in one step:
// from dh = 0 the step of :427-448 is, forward (A->S),
//   dh = -F_AS_dot (1 - xS0) / ((F_AS - Rf_AS) - F_AS_dot - (1 - xS0) G1),
// and reverse (S->A),
//   dh =  F_SA_dot xS0 / ((F_SA - Rf_SA) - F_SA_dot + xS0 G1),
// the other row's pivot (F - Rf of the inactive transformation) only
// scaling the determinant; the loading functions re-evaluated there leave a
// residual at rounding level, which ends the reference's loop.  As the
// reference: the activation tests (:351, :368), no step when the squared
// first residual is at most 1e-8 (:403), the loading functions evaluated at
// the unclamped xS, then the clamp (:484).  FP64, so the result is the
// reference's to rounding.  Returns false, with nothing written, for both
// transformations active and for a zero pivot; those take the iteration.
__device__ __forceinline__ bool return_map_closed(const MatC& m, double K, double G, double G_1, double theta,
                                                  double e_n, double tmp, double& xS, double& F_AS,
                                                  double& F_SA, int& flag) {
  const double x0 = xS, fas0 = F_AS, fsa0 = F_SA;
  const double fas = loading(K, G, m.alfa, m.C_AS, m.eL, theta, e_n, tmp, x0);
  const double fsa = loading(K, G, m.alfa, m.C_SA, m.eL, theta, e_n, tmp, x0);
  const bool kAS = (fas > fas0) && (fas - m.Rs_AS > 0.0) && (x0 < 1.0);
  const bool kSA = (fsa < fsa0) && (fsa - m.Rs_SA < 0.0) && (x0 > 0.0);
  if (kAS && kSA) return false;
  if (!kAS && !kSA) {
    F_AS = fas;
    F_SA = fsa;
    flag = NR_NONE;
    return true;
  }
  double rhs, piv, other;
  if (kAS) {
    const double dot = fas - fas0;
    rhs = dot * (1.0 - x0);
    piv = (fas - m.Rf_AS) - dot - (1.0 - x0) * G_1;
    other = fsa - m.Rf_SA;
  } else {
    const double dot = fsa - fsa0;
    rhs = -dot * x0;
    piv = (fsa - m.Rf_SA) - dot + x0 * G_1;
    other = fas - m.Rf_AS;
  }
  if (piv == 0.0 || other == 0.0) return false;
  if (rhs * rhs > 1.0e-8) {
    const double x = x0 - rhs / piv;
    F_AS = loading(K, G, m.alfa, m.C_AS, m.eL, theta, e_n, tmp, x);
    F_SA = loading(K, G, m.alfa, m.C_SA, m.eL, theta, e_n, tmp, x);
    xS = fmin(fmax(x, 0.0), 1.0);
  } else {
    F_AS = fas;
    F_SA = fsa;
  }
  flag = NR_CONVERGED;
  return true;
}

// ---------------------------------------------------------------------------
// Law 160 from A = b - I (spatial frame: tau, the Kirchhoff stress) or from
// A = C - I = 2E (material frame: the rotated-back Kirchhoff stress
// R^T tau R, whose pull-back C^-1 (R^T tau R) is the second Piola-Kirchhoff
// stress, since it is coaxial with C).  b and C share their eigenvalues, so
// the return map is the same.  state = (xS, F_AS, F_SA) of the previous
// step; on return the new state.  Tensors as (xx, yy, zz, xy, yz, xz).
// dir, if not null, receives the unit deviatoric direction e / |e| of the
// logarithmic strain in the same frame (zero when |e| is below FP64 epsilon).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ int law160_from_A(const MatC& m, const T* A, double tmp,
                                             double& xS, double& F_AS, double& F_SA, T* tau,
                                             T* dir = nullptr) {
  using M = Fm<T>;
  T L[6], f[3];
  sym_log1p(A, L, f);
  // logarithmic strains (:313-332): ln(lambda_i) = f_i/2
  const T theta_t = T(0.5) * (f[0] + f[1] + f[2]);
  const T t3 = theta_t * (T(1) / T(3));
  const T e0 = T(0.5) * f[0] - t3, e1 = T(0.5) * f[1] - t3, e2 = T(0.5) * f[2] - t3;
  const T en_t = M::sqrt_(e0 * e0 + e1 * e1 + e2 * e2);
  // moduli (extension: Reuss E at the start-of-step fraction)
  double K = m.K, G = m.G, G_1 = m.G1;
  if (m.ext_E) {
    const double E = 1.0 / ((1.0 - xS) * m.iEA + xS * m.iEM);
    K = E * m.kK;
    G = E * m.kG;
    G_1 = (2.0 * G + 9.0 * (m.alfa * m.alfa) * K) * m.eL;
  }
  const double theta = (double)theta_t, e_n = (double)en_t;
  int flag = NR_NONE;
  bool done = false;
  // the FP32 form takes the closed form (element loop -1.3 % on the 2.0 M
  // cylinder, -4 % on the cantilever); the FP64 form keeps the reference's
  // iteration, where the closed form's extra code cost it 3 % in spills
  if constexpr (sizeof(T) == 4) done = return_map_closed(m, K, G, G_1, theta, e_n, tmp, xS, F_AS, F_SA, flag);
  if (!done) {
    RMOut r = return_map(m, K, G, G_1, theta, e_n, tmp, xS, F_AS, F_SA);
    xS = r.xS;
    F_AS = r.F_AS;
    F_SA = r.F_SA;
    flag = r.flag;
  }
  // tau = pv I + kappa (L/2 - theta/3 I)   (:487-491)
  const T pv = (T)(K * (theta - 3.0 * m.alfa * m.eL * xS));
  const T twoG = (T)(2.0 * G);
  const T kp = (en_t > T(2.220446049250313e-16)) ? twoG * (T(1) - (T)(m.eL * xS) * M::rcp(en_t)) : twoG;
  const T kh = T(0.5) * kp;
  const T dg = pv - kp * t3;
  tau[0] = dg + kh * L[0];
  tau[1] = dg + kh * L[1];
  tau[2] = dg + kh * L[2];
  tau[3] = kh * L[3];
  tau[4] = kh * L[4];
  tau[5] = kh * L[5];
  if (dir) {
    // e = L/2 - theta/3 I
    const T ie = (en_t > T(2.220446049250313e-16)) ? M::rcp(en_t) : T(0);
    const T h = T(0.5) * ie, d0 = t3 * ie;
    dir[0] = h * L[0] - d0;
    dir[1] = h * L[1] - d0;
    dir[2] = h * L[2] - d0;
    dir[3] = h * L[3];
    dir[4] = h * L[4];
    dir[5] = h * L[5];
  }
  return flag;
}

// Kirchhoff stress of law 160 from H = F - I (row-major, H[3i+j] =
// du_i/dX_j): the spatial frame, A = b - I = H + H^T + H H^T
template <typename T>
__device__ __forceinline__ int law160_tau(const MatC& m, const T* H, double tmp,
                                          double& xS, double& F_AS, double& F_SA, T* tau) {
  T A[6];
  A[0] = T(2) * H[0] + (H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
  A[1] = T(2) * H[4] + (H[3] * H[3] + H[4] * H[4] + H[5] * H[5]);
  A[2] = T(2) * H[8] + (H[6] * H[6] + H[7] * H[7] + H[8] * H[8]);
  A[3] = H[1] + H[3] + (H[0] * H[3] + H[1] * H[4] + H[2] * H[5]);   // (0,1)
  A[4] = H[5] + H[7] + (H[3] * H[6] + H[4] * H[7] + H[5] * H[8]);   // (1,2)
  A[5] = H[2] + H[6] + (H[0] * H[6] + H[1] * H[7] + H[2] * H[8]);   // (0,2)
  return law160_from_A<T>(m, A, tmp, xS, F_AS, F_SA, tau);
}

// A = C - I = 2E = H + H^T + H^T H (the material frame)
template <typename T>
__device__ __forceinline__ void green_2E(const T* H, T* A) {
  A[0] = T(2) * H[0] + (H[0] * H[0] + H[3] * H[3] + H[6] * H[6]);
  A[1] = T(2) * H[4] + (H[1] * H[1] + H[4] * H[4] + H[7] * H[7]);
  A[2] = T(2) * H[8] + (H[2] * H[2] + H[5] * H[5] + H[8] * H[8]);
  A[3] = H[1] + H[3] + (H[0] * H[1] + H[3] * H[4] + H[6] * H[7]);   // (0,1)
  A[4] = H[5] + H[7] + (H[1] * H[2] + H[4] * H[5] + H[7] * H[8]);   // (1,2)
  A[5] = H[2] + H[6] + (H[0] * H[2] + H[3] * H[5] + H[6] * H[8]);   // (0,2)
}

// inverse of a symmetric 3x3 (xx, yy, zz, xy, yz, xz)
template <typename T>
__device__ __forceinline__ void sym_inv3(const T* S, T* Si) {
  const T c00 = S[1] * S[2] - S[4] * S[4];
  const T c01 = S[4] * S[5] - S[3] * S[2];
  const T c02 = S[3] * S[4] - S[1] * S[5];
  const T id = Fm<T>::rcp(S[0] * c00 + S[3] * c01 + S[5] * c02);
  Si[0] = c00 * id;
  Si[1] = (S[0] * S[2] - S[5] * S[5]) * id;
  Si[2] = (S[0] * S[1] - S[3] * S[3]) * id;
  Si[3] = c01 * id;
  Si[4] = (S[3] * S[5] - S[0] * S[4]) * id;
  Si[5] = c02 * id;
}

// product of two commuting symmetric 3x3 (the result is symmetric)
template <typename T>
__device__ __forceinline__ void sym_mul_commuting(const T* A, const T* B, T* P) {
  P[0] = A[0] * B[0] + A[3] * B[3] + A[5] * B[5];
  P[1] = A[3] * B[3] + A[1] * B[1] + A[4] * B[4];
  P[2] = A[5] * B[5] + A[4] * B[4] + A[2] * B[2];
  P[3] = A[0] * B[3] + A[3] * B[1] + A[5] * B[4];
  P[4] = A[3] * B[5] + A[1] * B[4] + A[4] * B[2];
  P[5] = A[0] * B[5] + A[3] * B[4] + A[5] * B[2];
}

// inverse and determinant of a general 3x3 (row-major M[3*i+j])
template <typename T>
__device__ __forceinline__ T inv3(const T* M, T* Mi) {
  const T c00 = M[4] * M[8] - M[5] * M[7];
  const T c01 = M[5] * M[6] - M[3] * M[8];
  const T c02 = M[3] * M[7] - M[4] * M[6];
  const T det = M[0] * c00 + M[1] * c01 + M[2] * c02;
  const T id = Fm<T>::rcp(det);
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
