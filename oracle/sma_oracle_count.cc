/*
 * sma_oracle_count.cc -- the oracle (sma_oracle_impl.h) instantiated on a
 * counting number type: every floating-point add/subtract, multiply, divide,
 * compare, sqrt, log and pow that the double oracle performs is tallied.
 *
 * TEST INFRASTRUCTURE ONLY.  It gives the per-Gauss-point operation counts
 * of the reference path (the law, compute_kirchoff_stress with its eigen-
 * solver, and the element loop of sld_elmope) that the kernels' rooflines
 * quote.  Nothing in the product links this file.
 */
#include "sma_oracle.h"

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>

namespace {

enum { OP_ADD, OP_MUL, OP_DIV, OP_CMP, OP_SQRT, OP_LOG, OP_POW, OP_N };
thread_local uint64_t g_ops[OP_N];

// a double that counts the arithmetic done on it
struct CD {
  double v;
  CD() = default;
  constexpr CD(double x) : v(x) {}
  explicit operator double() const { return v; }
};
inline CD operator+(CD a, CD b) { ++g_ops[OP_ADD]; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { ++g_ops[OP_ADD]; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { ++g_ops[OP_MUL]; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { ++g_ops[OP_DIV]; return CD(a.v / b.v); }
inline CD operator-(CD a) { return CD(-a.v); }                      // sign change: free
inline CD operator+(CD a) { return a; }
inline CD& operator+=(CD& a, CD b) { a = a + b; return a; }
inline CD& operator-=(CD& a, CD b) { a = a - b; return a; }
inline CD& operator*=(CD& a, CD b) { a = a * b; return a; }
inline CD& operator/=(CD& a, CD b) { a = a / b; return a; }
inline bool operator<(CD a, CD b) { ++g_ops[OP_CMP]; return a.v < b.v; }
inline bool operator>(CD a, CD b) { ++g_ops[OP_CMP]; return a.v > b.v; }
inline bool operator<=(CD a, CD b) { ++g_ops[OP_CMP]; return a.v <= b.v; }
inline bool operator>=(CD a, CD b) { ++g_ops[OP_CMP]; return a.v >= b.v; }
inline bool operator==(CD a, CD b) { ++g_ops[OP_CMP]; return a.v == b.v; }
inline bool operator!=(CD a, CD b) { ++g_ops[OP_CMP]; return a.v != b.v; }
inline CD sqrt_c(CD a) { ++g_ops[OP_SQRT]; return CD(std::sqrt(a.v)); }
inline CD log_c(CD a) { ++g_ops[OP_LOG]; return CD(std::log(a.v)); }
inline CD pow_c(CD a, CD b) { ++g_ops[OP_POW]; return CD(std::pow(a.v, b.v)); }
inline CD fabs_c(CD a) { return CD(std::fabs(a.v)); }                // sign mask: free

}  // namespace

#define REAL CD
#define SUFFIX _cnt
#define SQRT sqrt_c
#define FABS fabs_c
#define LOG log_c
#define POW pow_c
#define REAL_EPS DBL_EPSILON
#include "sma_oracle_impl.h"

namespace {
void take(uint64_t* ops) {
  for (int k = 0; k < OP_N; ++k) ops[k] = g_ops[k];
}
}  // namespace

extern "C" {

/* One law evaluation (compute_kirchoff_stress): ops[7] = add/sub, mul, div,
 * compare, sqrt, log, pow.  Returns the Newton-Raphson flag; sdv in/out. */
int orc_count_law160(const double props[18], double e_mart, const double F[9], double tmp, double sdv[3],
                     uint64_t ops[7]) {
  CD p[18], f[9], s[3], tau[9];
  for (int i = 0; i < 18; ++i) p[i] = props[i];
  for (int i = 0; i < 9; ++i) f[i] = F[i];
  for (int i = 0; i < 3; ++i) s[i] = sdv[i];
  std::memset(g_ops, 0, sizeof g_ops);
  const int fl = orc_law160_kirchhoff_cnt(p, CD(e_mart), f, CD(tmp), s, tau);
  take(ops);
  for (int i = 0; i < 3; ++i) sdv[i] = s[i].v;
  return fl;
}

/* One HEX08 element of the explicit element loop (orc_element: geometry,
 * F, the law at its 8 Gauss points, P, forces and the lumped mass the
 * reference rebuilds every step): ops[7] as above; nr_active receives the
 * Gauss points that ran the return map. */
int orc_count_element(const double elcod[24], const double eldis[24], const double props[18], double e_mart,
                      double densi, const double sdv_old[24], uint64_t ops[7], int* nr_active) {
  CD c[24], u[24], p[18], so[24], sn[24], fint[24], fext[24], muu[8], ppio[72];
  for (int i = 0; i < 24; ++i) { c[i] = elcod[i]; u[i] = eldis[i]; so[i] = sdv_old[i]; }
  for (int i = 0; i < 18; ++i) p[i] = props[i];
  const CD grav[3] = {CD(0.0), CD(0.0), CD(0.0)};
  CD detmin(1e300);
  int nr[5] = {0, 0, 0, 0, 0};
  std::memset(g_ops, 0, sizeof g_ops);
  const int rc = orc_element_cnt(c, u, p, CD(e_mart), CD(densi), CD(0.0), grav, so, sn, fint, fext, muu, ppio,
                                 &detmin, nr, nullptr, CD(0.0), nullptr);
  take(ops);
  if (nr_active) *nr_active = nr[0];
  return rc;
}

}  // extern "C"
