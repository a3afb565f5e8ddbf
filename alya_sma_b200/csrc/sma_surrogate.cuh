// sma_surrogate.cuh -- the learned constitutive surrogate of law 160 on the
// B200: its network, the plain-law data generator, the BF16 tensor-core
// training kernel, the optimiser, and the tcgen05 inference.
//
// The reference has no surrogate (its adjacent hook is the ANN framework's
// libtorch forward pass, src/alya-ann/mod_ann_framework.f90:421-446); the
// law it stands in for is compute_kirchoff_stress,
// sld_stress_model_160.f90:212-500.
//
// Network: 14 inputs -> 64 -> 64 -> 64 -> 64 -> 13 outputs, SiLU after the
// hidden layers.  Per Gauss point, in the material frame (tensors as
// xx, yy, zz, xy, yz, xz):
//   inputs   E (Green-Lagrange strain, 6), eps_tr_p = eL xS0 dev h / |dev h|
//            (the previous step's transformation strain on the current
//            deviatoric direction, h ~ ln U; 6), temperature, xS0 (the
//            previous step's martensite fraction)
//   outputs  (S - S_p) / E(xS0) (6): the second Piola-Kirchhoff stress less
//            its analytic part S_p (analytic_part: the law's elastic
//            response on a third-order logarithmic strain with eps_tr_p),
//            over the Reuss modulus, so the network carries only the
//            remainder; xS - xS0; eps_tr - eps_tr_p (6)
// Inputs and outputs are normalised per feature by the training set's mean
// and standard deviation (SurStats).  Weights are BF16 with FP32
// accumulation on the tensor cores; biases and the epilogue are FP32.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "sma_law.cuh"

namespace sma {
namespace sur {

constexpr int NIN = 14, NOUT = 13, HID = 64, KIN = 16, KOUT = 16;

// padded flat parameter layout (FP32 master weights, their BF16 copy, the
// gradient): W[o][i] is the weight from input i to output o
enum : int {
  OW1 = 0, OB1 = OW1 + HID * KIN, OW2 = OB1 + HID, OB2 = OW2 + HID * HID, OW3 = OB2 + HID,
  OB3 = OW3 + HID * HID, OW4 = OB3 + HID, OB4 = OW4 + HID * HID, OW5 = OB4 + HID,
  OB5 = OW5 + KOUT * HID, NPARAM = OB5 + KOUT
};
static_assert(NPARAM == 14608, "parameter layout");

// normalisation and the out-of-envelope gate.  Linv: the inverse of the
// Cholesky factor of the covariance of the normalised training inputs
// (lower triangular, row-major); score = |Linv xh| / sqrt(14) is the
// Mahalanobis distance per input dimension.
struct SurStats {
  float mu_x[NIN], sd_x[NIN], mu_y[NOUT], sd_y[NOUT];
  float Linv[NIN * NIN];
  float lo_x[NIN], hi_x[NIN];   // the training inputs' range: outside it is out of the envelope
};

// ---------------------------------------------------------------------------
// SiLU on the MUFU tanh: silu(z) = z sigmoid(z) = h (1 + tanh h), h = z/2
// (max relative error of tanh.approx.f32 about 2^-11, below the BF16
// rounding the activations take next)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float silu(float z) {
  const float h = 0.5f * z;
  return fmaf(h, tanh_fast(h), h);
}
// d silu / dz = s (1 + z (1 - s)), s = sigmoid(z) = (1 + tanh(z/2)) / 2
__device__ __forceinline__ float dsilu(float z) {
  const float s = 0.5f + 0.5f * tanh_fast(0.5f * z);
  return s * fmaf(z, 1.0f - s, 1.0f);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float2 unpack_bf16(uint32_t u) {
  const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&u);
  return __bfloat1622float2(v);
}

// The analytic part of the response.  h = E - E^2 + 4/3 E^3 is ln U to
// O(E^4) (E the Green-Lagrange strain, C = I + 2E).  The law's transformation
// strain always lies along the current deviatoric direction with length
// eL xS (eps_tr = eL xS D, sld_stress_model_160.f90:487-491), so it is no
// state of its own: eps_tr = ntr dev h / |dev h| with ntr = eL xS0.  Then
// T_p = kK (tr h - 3 alpha ntr) I + 2 kG (dev h - eps_tr) and
// S_p = sym(C^-1 T_p) -- the law's elastic response over E(xS0), so the
// network carries only the O(E^4) remainder.
template <typename T>
__device__ __forceinline__ void analytic_part(double kK, double kG, double alfa, const T* E, T ntr, T* Sp,
                                              T* etr) {
  // E^2 and E^3 (symmetric products, xx yy zz xy yz xz)
  T q[6];
  q[0] = E[0] * E[0] + E[3] * E[3] + E[5] * E[5];
  q[1] = E[3] * E[3] + E[1] * E[1] + E[4] * E[4];
  q[2] = E[5] * E[5] + E[4] * E[4] + E[2] * E[2];
  q[3] = E[0] * E[3] + E[3] * E[1] + E[5] * E[4];
  q[4] = E[3] * E[5] + E[1] * E[4] + E[4] * E[2];
  q[5] = E[0] * E[5] + E[3] * E[4] + E[5] * E[2];
  T c[6];
  c[0] = q[0] * E[0] + q[3] * E[3] + q[5] * E[5];
  c[1] = q[3] * E[3] + q[1] * E[1] + q[4] * E[4];
  c[2] = q[5] * E[5] + q[4] * E[4] + q[2] * E[2];
  c[3] = q[0] * E[3] + q[3] * E[1] + q[5] * E[4];
  c[4] = q[3] * E[5] + q[1] * E[4] + q[4] * E[2];
  c[5] = q[0] * E[5] + q[3] * E[4] + q[5] * E[2];
  const T f3 = T(4) / T(3);
  T h[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) h[k] = E[k] - q[k] + f3 * c[k];
  const T tr = h[0] + h[1] + h[2], t3 = tr * (T(1) / T(3));
  const T dh[6] = {h[0] - t3, h[1] - t3, h[2] - t3, h[3], h[4], h[5]};
  const T ndh = sqrt(dh[0] * dh[0] + dh[1] * dh[1] + dh[2] * dh[2] + T(2) * (dh[3] * dh[3] + dh[4] * dh[4] + dh[5] * dh[5]));
  const T sc = ndh > T(1e-12) ? ntr / ndh : T(0);              // no direction: no deviatoric strain
#pragma unroll
  for (int k = 0; k < 6; ++k) etr[k] = sc * dh[k];
  const T pv = (T)kK * (tr - T(3) * (T)alfa * ntr), g2 = T(2) * (T)kG;
  const T Tp[6] = {pv + g2 * (dh[0] - etr[0]), pv + g2 * (dh[1] - etr[1]), pv + g2 * (dh[2] - etr[2]),
                   g2 * (dh[3] - etr[3]), g2 * (dh[4] - etr[4]), g2 * (dh[5] - etr[5])};
  const T Cm[6] = {T(1) + T(2) * E[0], T(1) + T(2) * E[1], T(1) + T(2) * E[2], T(2) * E[3], T(2) * E[4],
                   T(2) * E[5]};
  T Ci[6];
  sym_inv3<T>(Cm, Ci);
  // sym(Ci Tp)
  const T p00 = Ci[0] * Tp[0] + Ci[3] * Tp[3] + Ci[5] * Tp[5];
  const T p11 = Ci[3] * Tp[3] + Ci[1] * Tp[1] + Ci[4] * Tp[4];
  const T p22 = Ci[5] * Tp[5] + Ci[4] * Tp[4] + Ci[2] * Tp[2];
  const T p01 = Ci[0] * Tp[3] + Ci[3] * Tp[1] + Ci[5] * Tp[4], p10 = Ci[3] * Tp[0] + Ci[1] * Tp[3] + Ci[4] * Tp[5];
  const T p12 = Ci[3] * Tp[5] + Ci[1] * Tp[4] + Ci[4] * Tp[2], p21 = Ci[5] * Tp[3] + Ci[4] * Tp[1] + Ci[2] * Tp[4];
  const T p02 = Ci[0] * Tp[5] + Ci[3] * Tp[4] + Ci[5] * Tp[2], p20 = Ci[5] * Tp[0] + Ci[4] * Tp[3] + Ci[2] * Tp[5];
  Sp[0] = p00;
  Sp[1] = p11;
  Sp[2] = p22;
  Sp[3] = T(0.5) * (p01 + p10);
  Sp[4] = T(0.5) * (p12 + p21);
  Sp[5] = T(0.5) * (p02 + p20);
}

// Reuss modulus at the start-of-step fraction (the law's extension rule)
__device__ __forceinline__ double reuss_E(const MatC& m, double xS0) {
  return 1.0 / ((1.0 - xS0) * m.iEA + xS0 * m.iEM);
}
// its inverse in FP32 (the stress scale of the FP32 element loop)
__device__ __forceinline__ float reuss_iE_f(const MatC& m, double xS0) {
  const float x = (float)xS0;
  return (1.f - x) * (float)m.iEA + x * (float)m.iEM;
}

// ---------------------------------------------------------------------------
// counter-based random numbers (SplitMix64, Steele, Lea & Flood, OOPSLA
// 2014): one stream per path, no state in memory
// ---------------------------------------------------------------------------
struct Rng {
  uint64_t s;
  __device__ __forceinline__ uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  __device__ __forceinline__ double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  __device__ __forceinline__ double uni(double a, double b) { return a + (b - a) * uni(); }
  // standard normal by Box-Muller
  __device__ __forceinline__ double normal() {
    const double u1 = fmax(uni(), 1e-300), u2 = uni();
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
};

// Path generator parameters (host-filled)
struct GenArgs {
  MatC base;              // the material every path scales (C_AS, C_SA, alpha, nu shared)
  double EA, EM, eL;      // base E_A, E_M, eL
  double Ss_AS, Sf_AS, Ss_SA, Sf_SA, Ts_AS, Tf_AS, Ts_SA, Tf_SA;  // base stresses and temperatures
  double spread;          // materials scaled by U(1 - spread, 1 + spread)
  double t_lo, t_hi;      // temperature range
  double e_lo, e_hi;      // axial strain targets of the load segments
  double shear;           // standard deviation of the shear strain targets
  int nseg;               // load segments per path
  int nstep;              // steps per path (samples written per path)
  int64_t npath;
  uint64_t seed;
  float* x;               // (npath * nstep, 14)
  float* y;               // (npath * nstep, 13)
};

// One thread per randomized load path of the plain law in FP64 (the material
// frame, law160_from_A on A = C - I): a random material around the base, a
// random temperature and frame, and nseg linear segments between random
// strain states (uniaxial-like with lateral contraction plus shear), nstep
// steps in all; each step writes one training sample, the law's answer to a
// small strain increment from the path's state at that step.
static __global__ void k_sur_generate(GenArgs g) {
  const int64_t path = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (path >= g.npath) return;
  Rng rng{g.seed * 0x2545F4914F6CDD1Dull + (uint64_t)path * 0x9E3779B97F4A7C15ull};
  // material
  const double fE = rng.uni(1 - g.spread, 1 + g.spread), fM = rng.uni(1 - g.spread, 1 + g.spread);
  const double fL = rng.uni(1 - g.spread, 1 + g.spread);
  const double f1 = rng.uni(1 - g.spread, 1 + g.spread), f2 = rng.uni(1 - g.spread, 1 + g.spread);
  const double f3 = rng.uni(1 - g.spread, 1 + g.spread), f4 = rng.uni(1 - g.spread, 1 + g.spread);
  MatC m = g.base;
  m.EA = g.EA * fE;
  m.EM = g.EM * fM;
  m.iEA = 1.0 / m.EA;
  m.iEM = 1.0 / m.EM;
  m.ext_E = 1;
  m.eL = g.eL * fL;
  const double aux = 0.816496580927726 + m.alfa;                 // sqrt(2/3) + alpha
  m.Rs_AS = g.Ss_AS * f1 * aux + m.C_AS * g.Ts_AS;
  m.Rf_AS = g.Sf_AS * f2 * aux + m.C_AS * g.Tf_AS;
  m.Rs_SA = g.Ss_SA * f3 * aux + m.C_SA * g.Ts_SA;
  m.Rf_SA = g.Sf_SA * f4 * aux + m.C_SA * g.Tf_SA;
  const double tmp = rng.uni(g.t_lo, g.t_hi);
  // frame: a random rotation from a unit quaternion
  double q0 = rng.normal(), q1 = rng.normal(), q2 = rng.normal(), q3 = rng.normal();
  const double qn = 1.0 / sqrt(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
  q0 *= qn; q1 *= qn; q2 *= qn; q3 *= qn;
  const double R[9] = {1 - 2 * (q2 * q2 + q3 * q3), 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2),
                       2 * (q1 * q2 + q0 * q3), 1 - 2 * (q1 * q1 + q3 * q3), 2 * (q2 * q3 - q0 * q1),
                       2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 1 - 2 * (q1 * q1 + q2 * q2)};
  // segment end states: U - I in the rotated frame (symmetric)
  auto target = [&](double* Hs) {
    const double ea = rng.uni(g.e_lo, g.e_hi), nu = rng.uni(0.30, 0.50);
    double D[6] = {ea, -nu * ea, -nu * ea, g.shear * rng.normal(), g.shear * rng.normal(),
                   g.shear * rng.normal()};
    // Hs = R D R^T
    const double Dm[9] = {D[0], D[3], D[5], D[3], D[1], D[4], D[5], D[4], D[2]};
    double RD[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) RD[3 * i + j] = R[3 * i] * Dm[j] + R[3 * i + 1] * Dm[3 + j] + R[3 * i + 2] * Dm[6 + j];
    double M[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) M[3 * i + j] = RD[3 * i] * R[3 * j] + RD[3 * i + 1] * R[3 * j + 1] + RD[3 * i + 2] * R[3 * j + 2];
    Hs[0] = M[0]; Hs[1] = M[4]; Hs[2] = M[8]; Hs[3] = M[1]; Hs[4] = M[5]; Hs[5] = M[2];
  };
  double H0[6] = {0, 0, 0, 0, 0, 0}, H1[6];
  target(H1);
  const int per = (g.nstep + g.nseg - 1) / g.nseg;
  double xS = 0.0, F_AS = 0.0, F_SA = 0.0;
  double Hp[6] = {0, 0, 0, 0, 0, 0};                             // the path's last stretch
  for (int s = 0; s < g.nstep; ++s) {
    const int k = s % per;
    if (k == 0 && s > 0) {
      for (int c = 0; c < 6; ++c) H0[c] = H1[c];
      target(H1);
    }
    const double w = (double)(k + 1) / per;
    double Hn[6];
    for (int c = 0; c < 6; ++c) Hn[c] = H0[c] + w * (H1[c] - H0[c]);
    // The sample is one explicit-sized step from the path's state: a strain
    // increment of up to 5 % of the path's own step (an explicit step moves
    // the strain by 1e-6..1e-5; a path step here by ~1e-3), so the direction
    // of ln U, and with it the transformation strain, turns as little as it
    // does in the element loop.  The path itself then advances a full step.
    const double mu = 0.05 * rng.uni();
    for (int pass = 0; pass < 2; ++pass) {
    double Hs[6];
    for (int c = 0; c < 6; ++c) Hs[c] = (pass == 0) ? Hp[c] + mu * (Hn[c] - Hp[c]) : Hn[c];
    // U = I + Hs: C - I = 2 Hs + Hs^2, E = (C - I)/2
    const double Hm[9] = {Hs[0], Hs[3], Hs[5], Hs[3], Hs[1], Hs[4], Hs[5], Hs[4], Hs[2]};
    double A[6];
    A[0] = 2 * Hs[0] + (Hm[0] * Hm[0] + Hm[1] * Hm[1] + Hm[2] * Hm[2]);
    A[1] = 2 * Hs[1] + (Hm[3] * Hm[3] + Hm[4] * Hm[4] + Hm[5] * Hm[5]);
    A[2] = 2 * Hs[2] + (Hm[6] * Hm[6] + Hm[7] * Hm[7] + Hm[8] * Hm[8]);
    A[3] = 2 * Hs[3] + (Hm[0] * Hm[3] + Hm[1] * Hm[4] + Hm[2] * Hm[5]);
    A[4] = 2 * Hs[4] + (Hm[3] * Hm[6] + Hm[4] * Hm[7] + Hm[5] * Hm[8]);
    A[5] = 2 * Hs[5] + (Hm[0] * Hm[6] + Hm[1] * Hm[7] + Hm[2] * Hm[8]);
    if (pass == 1) {                                             // the path's step: state only
      double Tm[6], D[6];
      law160_from_A<double>(m, A, tmp, xS, F_AS, F_SA, Tm, D);
      for (int c = 0; c < 6; ++c) Hp[c] = Hn[c];
      continue;
    }
    const double xS0 = xS;
    const double Ex = reuss_E(m, xS0);
    double Tm[6], D[6];
    double xSm = xS, FASm = F_AS, FSAm = F_SA;
    law160_from_A<double>(m, A, tmp, xSm, FASm, FSAm, Tm, D);
    // S = C^-1 T (coaxial)
    const double Cm[6] = {1 + A[0], 1 + A[1], 1 + A[2], A[3], A[4], A[5]};
    double Ci[6], S[6];
    sym_inv3<double>(Cm, Ci);
    sym_mul_commuting<double>(Ci, Tm, S);
    // sample
    float* xo = g.x + (path * g.nstep + s) * NIN;
    float* yo = g.y + (path * g.nstep + s) * NOUT;
    double E[6], sl[6], er[6];
    for (int c = 0; c < 6; ++c) E[c] = 0.5 * A[c];
    analytic_part<double>(m.kK, m.kG, m.alfa, E, m.eL * xS0, sl, er);
    for (int c = 0; c < 6; ++c) {
      xo[c] = (float)E[c];
      xo[6 + c] = (float)er[c];
      yo[c] = (float)(S[c] / Ex - sl[c]);
    }
    xo[12] = (float)tmp;
    xo[13] = (float)xS0;
    yo[6] = (float)(xSm - xS0);
    for (int c = 0; c < 6; ++c) yo[7 + c] = (float)(m.eL * xSm * D[c] - er[c]);
    }
  }
}

// ---------------------------------------------------------------------------
// Training: one warp per 32 samples, BF16 mma.sync m16n8k16 with FP32
// accumulation for the forward pass, the backward pass and the weight
// gradients (ldmatrix.trans gives the transposed operands); the block's
// gradient is summed in shared memory and added to the global FP32 gradient
// once per block.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma16816(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ void ldsm_x4(uint32_t* r, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"((uint32_t)__cvta_generic_to_shared(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t* r, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"((uint32_t)__cvta_generic_to_shared(p)));
}
__device__ __forceinline__ void red_smem(float* p, float v) { atomicAdd(p, v); }

// shared-memory pitches (bf16 elements): rows of 16 and 64 padded by 8 so
// the 8 row addresses of an ldmatrix fall in different banks
constexpr int P16 = 24, P64 = 72;
struct TrainSmem {
  alignas(16) __nv_bfloat16 w1[HID * P16];
  alignas(16) __nv_bfloat16 w2[HID * P64];
  alignas(16) __nv_bfloat16 w3[HID * P64];
  alignas(16) __nv_bfloat16 w4[HID * P64];
  alignas(16) __nv_bfloat16 w5[KOUT * P64];
  alignas(16) float bias[4 * HID + KOUT];
  alignas(16) float grad[NPARAM];
  alignas(16) float stats[2 * NIN + 2 * NOUT];
  float loss;
  struct alignas(16) Warp {
    alignas(16) __nv_bfloat16 xh[32 * P16];         // normalised inputs (a_0)
    alignas(16) __nv_bfloat16 z[4][32 * P64];       // pre-activations of the hidden layers
    alignas(16) __nv_bfloat16 d[32 * P64];          // the layer's delta, for the transposed loads
  } warp[4];
};

struct TrainArgs {
  const __nv_bfloat16* wb;   // BF16 weights, padded flat layout
  const float* w;            // FP32 master (biases read from it)
  const SurStats* stats;
  const float* x;            // (n, 14)
  const float* y;            // (n, 13) targets, raw
  int64_t n;                 // samples in the batch
  float* grad;               // (NPARAM) += d loss / d params
  float* loss;               // += loss (mean over n x 13)
};

// forward layer: C[mt][nt] = bias + A (2 m-tiles x KB k-blocks) W^T
template <int KB, int NT>
__device__ __forceinline__ void fwd_layer(float (*C)[NT][4], const uint32_t (*A)[KB][4], const __nv_bfloat16* W,
                                          int pitch, const float* bias, int lane) {
  const int t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const float b0 = bias[8 * nt + 2 * t], b1 = bias[8 * nt + 2 * t + 1];
      C[mt][nt][0] = b0; C[mt][nt][1] = b1; C[mt][nt][2] = b0; C[mt][nt][3] = b1;
    }
  const int j = lane >> 3, r = lane & 7;
#pragma unroll
  for (int kb = 0; kb < KB; ++kb)
#pragma unroll
    for (int nt = 0; nt < NT; nt += 2) {
      // B fragments of n-tiles nt, nt+1 (rows = outputs, K contiguous)
      uint32_t bq[4];
      ldsm_x4(bq, W + (8 * (nt + (j >> 1)) + r) * pitch + 16 * kb + 8 * (j & 1));
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        mma16816(C[mt][nt], A[mt][kb], bq);
        mma16816(C[mt][nt + 1], A[mt][kb], bq + 2);
      }
    }
}

// backward through a layer: D[mt][nt] (over the layer's inputs, NT n-tiles)
// = delta (2 m-tiles x KB k-blocks over the outputs) W, W row-major [out][in]
template <int KB, int NT>
__device__ __forceinline__ void bwd_layer(float (*D)[NT][4], const uint32_t (*A)[KB][4], const __nv_bfloat16* W,
                                          int pitch, int lane) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) D[mt][nt][0] = D[mt][nt][1] = D[mt][nt][2] = D[mt][nt][3] = 0.f;
  const int j = lane >> 3, r = lane & 7;
#pragma unroll
  for (int kb = 0; kb < KB; ++kb)
#pragma unroll
    for (int nt = 0; nt < NT; nt += 2) {
      uint32_t bq[4];
      ldsm_x4_t(bq, W + (16 * kb + 8 * (j & 1) + r) * pitch + 8 * (nt + (j >> 1)));
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        mma16816(D[mt][nt], A[mt][kb], bq);
        mma16816(D[mt][nt + 1], A[mt][kb], bq + 2);
      }
    }
}

// C fragments (2 m-tiles x NT n-tiles) -> A fragments of the next product
template <int NT>
__device__ __forceinline__ void c_to_a(uint32_t (*A)[NT / 2][4], const float (*C)[NT][4]) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int kb = 0; kb < NT / 2; ++kb) {
      A[mt][kb][0] = pack_bf16(C[mt][2 * kb][0], C[mt][2 * kb][1]);
      A[mt][kb][1] = pack_bf16(C[mt][2 * kb][2], C[mt][2 * kb][3]);
      A[mt][kb][2] = pack_bf16(C[mt][2 * kb + 1][0], C[mt][2 * kb + 1][1]);
      A[mt][kb][3] = pack_bf16(C[mt][2 * kb + 1][2], C[mt][2 * kb + 1][3]);
    }
}

// C fragments -> shared memory rows (bf16), pitch p
template <int NT>
__device__ __forceinline__ void c_to_smem(__nv_bfloat16* s, int p, const float (*C)[NT][4], int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      *reinterpret_cast<uint32_t*>(s + (16 * mt + g) * p + 8 * nt + 2 * t) = pack_bf16(C[mt][nt][0], C[mt][nt][1]);
      *reinterpret_cast<uint32_t*>(s + (16 * mt + g + 8) * p + 8 * nt + 2 * t) = pack_bf16(C[mt][nt][2], C[mt][nt][3]);
    }
}

// weight gradient of one layer from this warp's 32 samples:
// dW[o][i] += sum_b delta[b][o] a[b][i]; delta rows in `ds` (pitch pd,
// MT m-tiles of outputs), a rows in `as` (pitch pa, NT n-tiles of inputs),
// SILU: a = silu(stored pre-activation)
template <int MT, int NT, bool SILU>
__device__ __forceinline__ void wgrad(float* dW, int nin, const __nv_bfloat16* ds, int pd, const __nv_bfloat16* as,
                                      int pa, int lane) {
  const int g = lane >> 2, t = lane & 3, j = lane >> 3, r = lane & 7;
#pragma unroll
  for (int mt = 0; mt < MT; ++mt) {
    float C[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) C[nt][0] = C[nt][1] = C[nt][2] = C[nt][3] = 0.f;
#pragma unroll
    for (int kb = 0; kb < 2; ++kb) {
      uint32_t a[4];
      // A = delta^T: matrices (b lo, o lo), (b lo, o hi), (b hi, o lo), (b hi, o hi)
      ldsm_x4_t(a, ds + (16 * kb + 8 * (j >> 1) + r) * pd + 16 * mt + 8 * (j & 1));
#pragma unroll
      for (int nt = 0; nt < NT; nt += 2) {
        uint32_t bq[4];
        ldsm_x4_t(bq, as + (16 * kb + 8 * (j & 1) + r) * pa + 8 * (nt + (j >> 1)));
        if (SILU) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const float2 v = unpack_bf16(bq[q]);
            bq[q] = pack_bf16(silu(v.x), silu(v.y));
          }
        }
        mma16816(C[nt], a, bq);
        if (nt + 1 < NT) mma16816(C[nt + 1], a, bq + 2);
      }
    }
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      red_smem(dW + (16 * mt + g) * nin + 8 * nt + 2 * t, C[nt][0]);
      red_smem(dW + (16 * mt + g) * nin + 8 * nt + 2 * t + 1, C[nt][1]);
      red_smem(dW + (16 * mt + g + 8) * nin + 8 * nt + 2 * t, C[nt][2]);
      red_smem(dW + (16 * mt + g + 8) * nin + 8 * nt + 2 * t + 1, C[nt][3]);
    }
  }
}

// bias gradient: column sums of the delta C fragments over the warp's rows
template <int NT>
__device__ __forceinline__ void bgrad(float* db, const float (*D)[NT][4], int lane) {
  const int t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    float s0 = D[0][nt][0] + D[0][nt][2] + D[1][nt][0] + D[1][nt][2];
    float s1 = D[0][nt][1] + D[0][nt][3] + D[1][nt][1] + D[1][nt][3];
#pragma unroll
    for (int o = 4; o < 32; o <<= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    if (lane < 4) {
      red_smem(db + 8 * nt + 2 * t, s0);
      red_smem(db + 8 * nt + 2 * t + 1, s1);
    }
  }
}

// delta_{l-1} = D * silu'(z_{l-1}) at the C positions
template <int NT>
__device__ __forceinline__ void mul_dsilu(float (*D)[NT][4], const __nv_bfloat16* z, int p, int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const float2 a = unpack_bf16(*reinterpret_cast<const uint32_t*>(z + (16 * mt + g) * p + 8 * nt + 2 * t));
      const float2 b = unpack_bf16(*reinterpret_cast<const uint32_t*>(z + (16 * mt + g + 8) * p + 8 * nt + 2 * t));
      D[mt][nt][0] *= dsilu(a.x);
      D[mt][nt][1] *= dsilu(a.y);
      D[mt][nt][2] *= dsilu(b.x);
      D[mt][nt][3] *= dsilu(b.y);
    }
}

static __global__ void __launch_bounds__(128, 1) k_sur_train(TrainArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainSmem& sm = *reinterpret_cast<TrainSmem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  // weights into padded rows, biases, stats; gradient and loss zeroed
  for (int k = tid; k < HID * KIN; k += 128) sm.w1[(k / KIN) * P16 + k % KIN] = a.wb[OW1 + k];
  for (int k = tid; k < HID * HID; k += 128) {
    const int o = k / HID, i = k % HID;
    sm.w2[o * P64 + i] = a.wb[OW2 + k];
    sm.w3[o * P64 + i] = a.wb[OW3 + k];
    sm.w4[o * P64 + i] = a.wb[OW4 + k];
  }
  for (int k = tid; k < KOUT * HID; k += 128) sm.w5[(k / HID) * P64 + k % HID] = a.wb[OW5 + k];
  for (int k = tid; k < HID; k += 128) {
    sm.bias[k] = a.w[OB1 + k];
    sm.bias[HID + k] = a.w[OB2 + k];
    sm.bias[2 * HID + k] = a.w[OB3 + k];
    sm.bias[3 * HID + k] = a.w[OB4 + k];
  }
  if (tid < KOUT) sm.bias[4 * HID + tid] = a.w[OB5 + tid];
  for (int k = tid; k < NPARAM; k += 128) sm.grad[k] = 0.f;
  const float* st = reinterpret_cast<const float*>(a.stats);
  for (int k = tid; k < 2 * NIN + 2 * NOUT; k += 128) sm.stats[k] = st[k];
  if (tid == 0) sm.loss = 0.f;
  __syncthreads();
  const float *mu_x = sm.stats, *sd_x = sm.stats + NIN, *mu_y = sm.stats + 2 * NIN,
              *sd_y = sm.stats + 2 * NIN + NOUT;
  TrainSmem::Warp& w = sm.warp[wid];
  const int g = lane >> 2, t = lane & 3, j = lane >> 3, r = lane & 7;
  const float scale = 1.0f / ((float)a.n * (float)NOUT);
  float loss = 0.f;
  for (int64_t s0 = ((int64_t)blockIdx.x * 4 + wid) * 32; s0 < a.n; s0 += (int64_t)gridDim.x * 128) {
    // normalised inputs of row `lane` (zero past the batch and in the padding)
    {
      const int64_t s = s0 + lane;
      float xr[KIN];
#pragma unroll
      for (int c = 0; c < KIN; ++c) xr[c] = 0.f;
      if (s < a.n)
#pragma unroll
        for (int c = 0; c < NIN; ++c) xr[c] = (a.x[s * NIN + c] - mu_x[c]) / sd_x[c];
#pragma unroll
      for (int c = 0; c < KIN; c += 2)
        *reinterpret_cast<uint32_t*>(w.xh + lane * P16 + c) = pack_bf16(xr[c], xr[c + 1]);
    }
    __syncwarp();
    uint32_t A1[2][1][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) ldsm_x4(A1[mt][0], w.xh + (16 * mt + 8 * (j & 1) + r) * P16 + 8 * (j >> 1));
    // forward
    float C[2][8][4];
    uint32_t A[2][4][4];
    fwd_layer<1, 8>(C, A1, sm.w1, P16, sm.bias, lane);
    c_to_smem<8>(w.z[0], P64, C, lane);
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) C[mt][nt][q] = silu(C[mt][nt][q]);
    c_to_a<8>(A, C);
    const __nv_bfloat16* Ws[3] = {sm.w2, sm.w3, sm.w4};
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      fwd_layer<4, 8>(C, A, Ws[l], P64, sm.bias + (l + 1) * HID, lane);
      c_to_smem<8>(w.z[l + 1], P64, C, lane);
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
#pragma unroll
          for (int q = 0; q < 4; ++q) C[mt][nt][q] = silu(C[mt][nt][q]);
      c_to_a<8>(A, C);
    }
    float C5[2][2][4];
    fwd_layer<4, 2>(C5, A, sm.w5, P64, sm.bias + 4 * HID, lane);
    // loss and output delta (normalised targets; padding and rows past n: 0)
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int row = 16 * mt + g + ((q & 2) ? 8 : 0), col = 8 * nt + 2 * t + (q & 1);
          const int64_t s = s0 + row;
          float d = 0.f;
          if (s < a.n && col < NOUT) {
            const float tgt = (a.y[s * NOUT + col] - mu_y[col]) / sd_y[col];
            d = C5[mt][nt][q] - tgt;
            loss += d * d;
          }
          C5[mt][nt][q] = 2.f * d * scale;
        }
    // backward: output layer
    c_to_smem<2>(w.d, P16, C5, lane);
    __syncwarp();
    wgrad<1, 8, true>(sm.grad + OW5, HID, w.d, P16, w.z[3], P64, lane);
    bgrad<2>(sm.grad + OB5, C5, lane);
    uint32_t Ad5[2][1][4];
    c_to_a<2>(Ad5, C5);
    bwd_layer<1, 8>(C, Ad5, sm.w5, P64, lane);
    mul_dsilu<8>(C, w.z[3], P64, lane);
    // hidden layers 4, 3, 2
#pragma unroll
    for (int l = 3; l >= 1; --l) {
      __syncwarp();
      c_to_smem<8>(w.d, P64, C, lane);
      __syncwarp();
      const int ow = (l == 3) ? OW4 : (l == 2) ? OW3 : OW2;
      const int ob = (l == 3) ? OB4 : (l == 2) ? OB3 : OB2;
      wgrad<4, 8, true>(sm.grad + ow, HID, w.d, P64, w.z[l - 1], P64, lane);
      bgrad<8>(sm.grad + ob, C, lane);
      c_to_a<8>(A, C);
      bwd_layer<4, 8>(C, A, Ws[l - 1], P64, lane);
      mul_dsilu<8>(C, w.z[l - 1], P64, lane);
    }
    // first layer
    __syncwarp();
    c_to_smem<8>(w.d, P64, C, lane);
    __syncwarp();
    wgrad<4, 2, false>(sm.grad + OW1, KIN, w.d, P64, w.xh, P16, lane);
    bgrad<8>(sm.grad + OB1, C, lane);
    __syncwarp();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  if (lane == 0) atomicAdd(&sm.loss, loss * scale);
  __syncthreads();
  for (int k = tid; k < NPARAM; k += 128) {
    const float v = sm.grad[k];
    if (v != 0.f) atomicAdd(a.grad + k, v);
  }
  if (tid == 0) atomicAdd(a.loss, sm.loss);
}

// Adam (Kingma & Ba, ICLR 2015) on the FP32 master weights, then their BF16
// copy; step t >= 1; the padding keeps zero gradients and stays zero
static __global__ void k_sur_adam(float* w, float* m, float* v, const float* grad, __nv_bfloat16* wb, float lr,
                           float b1, float b2, float eps, int t) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= NPARAM) return;
  const float gk = grad[k];
  const float mk = b1 * m[k] + (1.f - b1) * gk;
  const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
  m[k] = mk;
  v[k] = vk;
  const float mh = mk / (1.f - powf(b1, (float)t)), vh = vk / (1.f - powf(b2, (float)t));
  const float wk = w[k] - lr * mh / (sqrtf(vh) + eps);
  w[k] = wk;
  wb[k] = __float2bfloat16_rn(wk);
}

static __global__ void k_sur_to_bf16(const float* w, __nv_bfloat16* wb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < NPARAM) wb[k] = __float2bfloat16_rn(w[k]);
}

// ---------------------------------------------------------------------------
// Inference on the 5th-generation tensor cores.  A tile is 128 Gauss points
// (thread r of the 128-thread block owns row r: TMEM lane r holds its
// accumulators).  Operands sit in shared memory in the canonical K-major
// layout with the 128-byte swizzle: rows of 64 BF16 (128 B), groups of 8
// rows 1024 B apart, the 16-byte chunk c of row r stored at c ^ (r mod 8).
// One thread issues tcgen05.mma (M = 128, N = 64 or 16, K = 16 per
// instruction) into a 64-column TMEM accumulator and commits to an
// mbarrier; every thread then reads its row with tcgen05.ld, applies bias
// and SiLU in FP32, and writes the next layer's operand row.
// ---------------------------------------------------------------------------
constexpr int TILE_BYTES_64 = 64 * 128;       // 64 rows
constexpr int TILE_BYTES_16 = 16 * 128;       // 16 rows (the output layer's weights)
constexpr int A_TILE_BYTES = 128 * 128;       // 128 rows
// weight image: W1..W4 (64 rows each), W5 (16 rows), then the FP32 biases
constexpr int IMG_W1 = 0, IMG_W2 = IMG_W1 + TILE_BYTES_64, IMG_W3 = IMG_W2 + TILE_BYTES_64,
              IMG_W4 = IMG_W3 + TILE_BYTES_64, IMG_W5 = IMG_W4 + TILE_BYTES_64, IMG_B = IMG_W5 + TILE_BYTES_16,
              IMG_BYTES = IMG_B + (4 * HID + KOUT) * 4;
static_assert(IMG_BYTES % 16 == 0, "weight image");

// byte offset of element (row, k) in a swizzled K-major tile
__host__ __device__ __forceinline__ int sw128_off(int row, int k) {
  return (row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 3) ^ (row & 7)) & 7) << 4) + ((k & 7) << 1);
}

// the weight image from the FP32 master weights (one thread per element)
static __global__ void k_sur_pack_image(const float* w, unsigned char* img) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  // zero-filled tiles first (the host clears img), then the weights
  if (k < HID * KIN) {
    const int o = k / KIN, i = k % KIN;
    *reinterpret_cast<__nv_bfloat16*>(img + IMG_W1 + sw128_off(o, i)) = __float2bfloat16_rn(w[OW1 + k]);
  }
  if (k < HID * HID) {
    const int o = k / HID, i = k % HID;
    *reinterpret_cast<__nv_bfloat16*>(img + IMG_W2 + sw128_off(o, i)) = __float2bfloat16_rn(w[OW2 + k]);
    *reinterpret_cast<__nv_bfloat16*>(img + IMG_W3 + sw128_off(o, i)) = __float2bfloat16_rn(w[OW3 + k]);
    *reinterpret_cast<__nv_bfloat16*>(img + IMG_W4 + sw128_off(o, i)) = __float2bfloat16_rn(w[OW4 + k]);
  }
  if (k < KOUT * HID) {
    const int o = k / HID, i = k % HID;
    *reinterpret_cast<__nv_bfloat16*>(img + IMG_W5 + sw128_off(o, i)) = __float2bfloat16_rn(w[OW5 + k]);
  }
  float* b = reinterpret_cast<float*>(img + IMG_B);
  if (k < HID) {
    b[k] = w[OB1 + k];
    b[HID + k] = w[OB2 + k];
    b[2 * HID + k] = w[OB3 + k];
    b[3 * HID + k] = w[OB4 + k];
  }
  if (k < KOUT) b[4 * HID + k] = w[OB5 + k];
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// smem matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B
// apart (SBO), leading offset unused for this layout (1), version 1
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
// instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, dense, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* mbar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}
// bounded wait for the phase with the given parity; false after `limit` tries
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, int limit) {
  const uint32_t a = smem_u32(mbar);
  for (int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// The bounded wait on its own: thread 0 initialises an mbarrier that
// nothing arrives at and waits for its first phase, `tries` tries -- the path
// a network kernel takes if its tensor-core work never completes.
// status = 1 if the wait gave up (the expected answer), 0 if it saw the phase
// complete.
static __global__ void k_sur_wait_check(int tries, int* status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *status = mbar_wait(&bar, 0u, tries) ? 0 : 1;
  }
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 16 consecutive FP32 columns of this thread's TMEM lane, waited for
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

constexpr int MBAR_LIMIT = 1 << 22;    // tries before a wait is given up (an error, never expected)
constexpr int TMEM_COLS = 64;

// Shared state of a tcgen05 MLP block: 1024-aligned weight image and
// operand tile, the mbarrier, the TMEM base address and a status word.
struct MlpSmem {
  unsigned char img[IMG_BYTES];          // at a 1024-byte boundary (IMG_W* are multiples of 1024)
  unsigned char pad[(1024 - IMG_BYTES % 1024) % 1024];
  unsigned char a[A_TILE_BYTES];         // activation tile (1024-aligned)
  uint64_t mbar;
  uint32_t tmem;
  uint32_t phase;
  int status;                            // 0 ok, 1 a wait ran out
};
static_assert(offsetof(MlpSmem, a) % 1024 == 0, "operand tile alignment");

// block set-up: weight image in (16-byte copies), mbarrier, TMEM (warp 0).
// Needs all 128 threads; ends with a block barrier.
__device__ __forceinline__ void mlp_setup(MlpSmem& s, const unsigned char* img) {
  const int tid = threadIdx.x;
  const uint4* src = reinterpret_cast<const uint4*>(img);
  uint4* dst = reinterpret_cast<uint4*>(s.img);
  for (int k = tid; k < IMG_BYTES / 16; k += blockDim.x) dst[k] = __ldg(src + k);
  if (tid == 0) {
    mbar_init(&s.mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s.phase = 0;
    s.status = 0;
  }
  if (tid < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

// block tear-down: TMEM back (warp 0), after every thread's last TMEM access
__device__ __forceinline__ void mlp_teardown(MlpSmem& s) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem), "r"(TMEM_COLS));
}

// one layer: thread 0 issues the MMAs (K = 16 per instruction) and waits
// (bounded) for them; the block then reads the accumulators.  Returns false
// (block-uniform) if the wait ran out.
__device__ __forceinline__ bool mlp_mma(MlpSmem& s, int w_off, int nk, int n) {
  if (threadIdx.x == 0) {
    tc_fence_after();
    const uint32_t a0 = smem_u32(s.a), b0 = smem_u32(s.img + w_off);
    const uint32_t id = idesc_bf16(128, n);
    for (int k = 0; k < nk; ++k)
      umma_bf16(s.tmem, desc_sw128(a0 + 32 * k), desc_sw128(b0 + 32 * k), id, k > 0 ? 1u : 0u);
    umma_commit(&s.mbar);
    if (!mbar_wait(&s.mbar, s.phase, MBAR_LIMIT)) s.status = 1;
    s.phase ^= 1u;
  }
  __syncthreads();
  tc_fence_after();
  return s.status == 0;
}

// this thread's row of the operand tile from 16 or 64 floats (bf16)
template <int K>
__device__ __forceinline__ void mlp_put_row(MlpSmem& s, int row, const float* v) {
#pragma unroll
  for (int c = 0; c < K / 8; ++c) {
    uint4 q;
    q.x = pack_bf16(v[8 * c], v[8 * c + 1]);
    q.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
    q.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
    q.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4*>(s.a + sw128_off(row, 8 * c)) = q;
  }
}

// The network on the block's 128 rows: row r's normalised inputs xh[16]
// (thread r), the normalised outputs yh[16] back.  Returns false if a wait
// ran out (block-uniform).  Every thread of the 128-thread block calls it.
__device__ __forceinline__ bool mlp_tile(MlpSmem& s, const float* xh, float* yh) {
  const int row = threadIdx.x, warp = row >> 5;
  const uint32_t trow = s.tmem + ((uint32_t)(32 * warp) << 16);
  const float* bias = reinterpret_cast<const float*>(s.img + IMG_B);
  mlp_put_row<KIN>(s, row, xh);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  const int woff[4] = {IMG_W1, IMG_W2, IMG_W3, IMG_W4};
#pragma unroll 1
  for (int l = 0; l < 4; ++l) {
    if (!mlp_mma(s, woff[l], l == 0 ? 1 : 4, HID)) return false;
    float v[HID];
#pragma unroll
    for (int c = 0; c < HID; c += 16) tmem_ld16(trow + c, v + c);
#pragma unroll
    for (int c = 0; c < HID; ++c) v[c] = silu(v[c] + bias[l * HID + c]);
    mlp_put_row<HID>(s, row, v);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
  }
  if (!mlp_mma(s, IMG_W5, 4, KOUT)) return false;
  tmem_ld16(trow, yh);
#pragma unroll
  for (int c = 0; c < KOUT; ++c) yh[c] += bias[4 * HID + c];
  tc_fence_before();
  return true;
}

// normalised inputs and the out-of-envelope score of one raw input row:
// the Mahalanobis distance per dimension, or +inf if an input lies outside
// the training inputs' range (a single feature's excursion, which the
// distance averages over 14 dimensions)
__device__ __forceinline__ float normalise(const SurStats& st, const float* x, float* xh) {
  bool out = false;
#pragma unroll
  for (int c = 0; c < NIN; ++c) {
    xh[c] = (x[c] - st.mu_x[c]) / st.sd_x[c];
    out |= !(x[c] >= st.lo_x[c] && x[c] <= st.hi_x[c]);
  }
  xh[14] = xh[15] = 0.f;
  float d2 = out ? __int_as_float(0x7f800000) : 0.f;
#pragma unroll
  for (int i = 0; i < NIN; ++i) {
    float u = 0.f;
#pragma unroll
    for (int j = 0; j <= i; ++j) u = fmaf(st.Linv[i * NIN + j], xh[j], u);
    d2 = fmaf(u, u, d2);
  }
  return sqrtf(d2 * (1.0f / NIN));
}

// Batched inference (the network alone): raw inputs x (n, 14) -> raw outputs
// y (n, 13) and, if score is not null, the out-of-envelope score per row.
// Persistent blocks of 128 threads; status[0] set to 1 if a wait ran out.
static __global__ void __launch_bounds__(128) k_sur_forward(const unsigned char* img, const SurStats* stats, int64_t n,
                                                     const float* x, float* y, float* score, int* status) {
  extern __shared__ __align__(1024) unsigned char mlp_smem_raw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(mlp_smem_raw + ((1024 - (smem_u32(mlp_smem_raw) & 1023)) & 1023));
  mlp_setup(s, img);
  const SurStats& st = *stats;
  const int64_t ntiles = (n + 127) / 128;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t r = tile * 128 + threadIdx.x;
    float xr[NIN], xh[KIN], yh[KOUT];
#pragma unroll
    for (int c = 0; c < NIN; ++c) xr[c] = (r < n) ? x[r * NIN + c] : st.mu_x[c];
    const float sc = normalise(st, xr, xh);
    if (!mlp_tile(s, xh, yh)) {
      if (threadIdx.x == 0) atomicExch(status, 1);
      break;
    }
    if (r < n) {
#pragma unroll
      for (int c = 0; c < NOUT; ++c) y[r * NOUT + c] = yh[c] * st.sd_y[c] + st.mu_y[c];
      if (score) score[r] = sc;
    }
  }
  mlp_teardown(s);
}

inline size_t mlp_smem_bytes() { return sizeof(MlpSmem) + 1024; }

}  // namespace sur
}  // namespace sma
