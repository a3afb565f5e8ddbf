// sma_surrogate_elem.cuh -- the element loop with the learned surrogate in
// place of law 160's evaluation (the FP32 precision form): the network on
// the tcgen05 tensor cores for every Gauss point, the plain law for the
// points the gates send back.
//
// Per Gauss point (lane = Gauss point, 8 lanes per element, 16 elements =
// 128 Gauss points = one M = 128 tile per block):
//   1. gather, kinematics (as k_element), E = (C - I)/2;
//   2. the network on the block's 128 points (tcgen05.mma into TMEM) every
//      `period` steps per tile (staggered) or when a point has no residual
//      yet, the residual held in between (FP16 per Gauss point; a point
//      the plain law handled holds the law's residual);
//   3. S = E(xS0) (y_S + S_p) (analytic_part: eps_tr turned onto the current
//      strain direction, as the law keeps it), the rotated-back Kirchhoff stress
//      T = sym(C S) and from it the law's loading functions
//      F = +-|dev T| + 3 alpha tr(T)/3 - C T_K (sld_stress_model_160.f90:
//      513-537 with beta = 1: +-|dev T| = 2G (|e| - eL xS0), negative below
//      the transformation strain);
//   4. gates: the out-of-envelope score above its limit, loading functions
//      within f_margin of a transformation start (F_AS > Rs_AS - margin with
//      xS0 < 1, F_SA < Rs_SA + margin with xS0 > 0: the law's activation test,
//      :351-374, needs the exact F there), or a network xS increment above
//      its tolerance on a point the law leaves inactive (its residual
//      (F - Rf) dh + H (F - F0)(1 - xS) is then not zero) -> the plain law
//      (material frame, FP32 kinematics, FP64 return map) for that point;
//   5. tau = F S F^T and the element forces as k_element (tile_forces).
// Accepted points keep xS0, turn eps_tr onto the current direction and
// store the loading functions of the predicted stress as (F_AS, F_SA);
// fallback points store the law's (xS, F_AS, F_SA) and eps_tr = eL xS D.
#pragma once

#include "sma_kernels.cuh"
#include "sma_surrogate.cuh"

namespace sma {
namespace sur {

struct SurElemArgs {
  const unsigned char* img;   // weight image (IMG_BYTES, 16-byte aligned)
  const SurStats* stats;
  const float* etr_old;       // eps_tr at TIME_N, SoA [6][sst]
  float* etr_new;             // eps_tr at ITER_K
  __half* rcache;             // the held stress residual per Gauss point, SoA [6][sst] (NaN: none yet)
  const StepTime* clock;      // the step's time (its index picks the tiles that refresh)
  int* tile_ctr;              // next tile (zeroed before the launch)
  int* status;                // set to 1 if a wait for the tensor cores ran out
  float gate;                 // out-of-envelope score limit
  float xs_tol;               // network xS increment allowed on an inactive point
  float f_margin;             // distance from the transformation surfaces (loading-function units)
  int period;                 // steps between two evaluations of the network on a tile
};

constexpr int SUR_BLOCK = 128, SUR_EPB = SUR_BLOCK / 8;
constexpr int CNT_SUR_FALLBACK = CNT_RESERVED5;   // points sent to the plain law
constexpr int CNT_SUR_OOD = 7;                    // of those, out of the envelope

// the element rows start at a 128-byte boundary after the MLP state (the
// element code reads them with 128-bit shared-memory loads)
constexpr size_t SUR_ELEM_OFF = (sizeof(MlpSmem) + 127) / 128 * 128;
inline size_t sur_elem_smem_bytes() {
  return 1024 + SUR_ELEM_OFF + (size_t)SUR_EPB * ElemSmem<float>::PER_ELEM * sizeof(float) + 16;
}

template <bool CMP>
__global__ void __launch_bounds__(SUR_BLOCK, 3) k_element_sur(ElemArgs<float> a, SurElemArgs s) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
  MlpSmem& ms = *reinterpret_cast<MlpSmem*>(base);
  float* elem_sm = reinterpret_cast<float*>(base + SUR_ELEM_OFF);
  int* tile_sm = reinterpret_cast<int*>(elem_sm + SUR_EPB * ElemSmem<float>::PER_ELEM);
  if (a.ts && blockIdx.x == 0 && threadIdx.x == 0) advance_time(a.ts, a.ft);
  mlp_setup(ms, s.img);
  const SurStats& st = *s.stats;
  const int lane8 = threadIdx.x & 7, le = threadIdx.x >> 3;
  float* nsm = elem_sm + le * ElemSmem<float>::PER_ELEM;
  float* qsm = nsm + ElemSmem<float>::NODE_STRIDE;
  const int64_t ntiles = ((int64_t)a.end - a.beg + SUR_EPB - 1) / SUR_EPB;
  const int src = (threadIdx.x & 31) & ~7;
  for (;;) {
    if (threadIdx.x == 0) *tile_sm = atomicAdd(s.tile_ctr, 1);
    __syncthreads();
    const int64_t tile = *tile_sm;
    if (tile >= ntiles) break;                                   // block-uniform
    const int64_t e = (int64_t)a.beg + tile * SUR_EPB + le;
    const bool valid = e < a.end;
    const int64_t ec = valid ? e : (int64_t)a.end - 1;
    // ---- gather and kinematics (as k_element) --------------------------
    const int nid = a.lnods[8 * ec + lane8];
    double X[3], U[3], dX[3], dU[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      X[c] = __ldg(a.coord + c * a.npad + nid);
      U[c] = __ldg(a.u + c * a.npad + nid);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      dX[c] = X[c] - __shfl_sync(0xffffffffu, X[c], src);
      dU[c] = U[c] - __shfl_sync(0xffffffffu, U[c], src);
    }
    {
      const float v[6] = {(float)dX[0], (float)dX[1], (float)dX[2], (float)dU[0], (float)dU[1], (float)dU[2]};
      stage_node_rows<float>(nsm, lane8, v);
    }
    __syncwarp();
    float Ji[9], H[9], Jc[9];
    const float detJ = gp_kinematics<float>(nsm, lane8, Ji, H, Jc);
    const int64_t gp = 8 * ec + lane8;
    const double xS0 = (double)a.sold[gp], F_AS0 = (double)a.sold[a.sst + gp];
    const double F_SA0 = (double)a.sold[2 * a.sst + gp];
    float etr0[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) etr0[c] = s.etr_old[c * a.sst + gp];
    double tmp = 0.0;
    if constexpr (CMP) tmp = a.mat0.T0 + (double)__ldg(a.matx + MATX * ec + MX_TEMP);
    else tmp = a.tempe ? __ldg(a.tempe + ec) : 0.0;
    float A2[6];                                                 // C - I = 2E
    green_2E<float>(H, A2);
    // ---- the network's stress residual: held between evaluations -------
    // A BF16 network's output moves in quantisation steps while an explicit
    // step moves the strain by ~1e-6: evaluated every step, those steps act
    // as a local stiffness several times the elastic one and the explicit
    // scheme drifts.  So a tile evaluates the network every `period` steps
    // (tiles staggered) or when one of its points has no residual yet (NaN,
    // the first step), and holds the residual in between; a point the plain
    // law handled holds the law's residual; the analytic part S_p follows
    // the strain every step.
    float x[NIN];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      x[c] = 0.5f * A2[c];
      x[6 + c] = etr0[c];
    }
    x[12] = (float)tmp;
    x[13] = (float)xS0;
    bool inbox = true;
#pragma unroll
    for (int c = 0; c < NIN; ++c) inbox &= (x[c] >= st.lo_x[c] && x[c] <= st.hi_x[c]);
    float r[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) r[c] = __half2float(s.rcache[c * a.sst + gp]);
    const int64_t kstep = s.clock ? (int64_t)(s.clock->cutim / s.clock->dtime + 0.5) : 0;
    const bool due = ((tile + kstep) % s.period) == 0;
    const bool refresh = __syncthreads_or(due || isnan(r[0]));   // block-uniform
    float score = inbox ? 0.f : __int_as_float(0x7f800000), xs_inc = 0.f;
    if (refresh) {
      float xh[KIN], yh[KOUT];
      score = normalise(st, x, xh);
      if (!mlp_tile(ms, xh, yh)) {
        if (threadIdx.x == 0) atomicExch(s.status, 1);
        break;                                                   // block-uniform
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) r[c] = yh[c] * st.sd_y[c] + st.mu_y[c];
      xs_inc = yh[6] * st.sd_y[6] + st.mu_y[6];
    }
    double tmp2;
    const MatC m = CMP ? compact_mat<float>(a, ec, &tmp2) : a.mat0;
    // ---- stress of the network, loading functions, gates ---------------
    const float Ex = (float)reuss_E(m, xS0);
    float S[6], etr_p[6];
    {
      float E[6], sp[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) E[c] = 0.5f * A2[c];
      analytic_part<float>(m.kK, m.kG, m.alfa, E, etr0, sp, etr_p);
#pragma unroll
      for (int c = 0; c < 6; ++c) S[c] = (r[c] + sp[c]) * Ex;
    }
    double F_AS, F_SA;
    {
      // T = sym(C S), C = I + A2 (xx, yy, zz, xy, yz, xz)
      const float C00 = 1.f + A2[0], C11 = 1.f + A2[1], C22 = 1.f + A2[2];
      const float C01 = A2[3], C12 = A2[4], C02 = A2[5];
      const float t00 = C00 * S[0] + C01 * S[3] + C02 * S[5];
      const float t11 = C01 * S[3] + C11 * S[1] + C12 * S[4];
      const float t22 = C02 * S[5] + C12 * S[4] + C22 * S[2];
      const float t01 = 0.5f * ((C00 * S[3] + C01 * S[1] + C02 * S[4]) + (C01 * S[0] + C11 * S[3] + C12 * S[5]));
      const float t12 = 0.5f * ((C01 * S[5] + C11 * S[4] + C12 * S[2]) + (C02 * S[3] + C12 * S[1] + C22 * S[4]));
      const float t02 = 0.5f * ((C00 * S[5] + C01 * S[4] + C02 * S[2]) + (C02 * S[0] + C12 * S[3] + C22 * S[5]));
      const float p = (t00 + t11 + t22) * (1.f / 3.f);
      const float d0 = t00 - p, d1 = t11 - p, d2 = t22 - p;
      // the law's deviatoric term 2G (|e| - eL xS0) is signed: dev T points
      // against the strain deviator once the strain is below the
      // transformation strain, so |dev T| takes the sign of the projection
      // of dev T on dev E (whose direction is e's to first order)
      const float em = (A2[0] + A2[1] + A2[2]) * (1.f / 6.f);
      const float proj = d0 * (0.5f * A2[0] - em) + d1 * (0.5f * A2[1] - em) + d2 * (0.5f * A2[2] - em) +
                         (t01 * A2[3] + t12 * A2[4] + t02 * A2[5]);
      const double dn = sqrt((double)(d0 * d0 + d1 * d1 + d2 * d2 + 2.f * (t01 * t01 + t12 * t12 + t02 * t02)));
      const double trac = proj < 0.f ? -dn : dn;
      const double pr = 3.0 * m.alfa * (double)p;
      F_AS = trac + pr - m.C_AS * tmp;
      F_SA = trac + pr - m.C_SA * tmp;
    }
    // A point on or near a transformation surface goes to the law, which
    // alone decides its activation: the test F > F0 (:351, :368) compares
    // two loading values one explicit step apart (~0.05 MPa), far below the
    // network's stress error (~0.5 MPa), so only points at least f_margin
    // inside the elastic band -- where neither transformation can start
    // this step -- keep the network's stress.
    const bool near_AS = (F_AS - m.Rs_AS > -(double)s.f_margin) && (xS0 < 1.0);
    const bool near_SA = (F_SA - m.Rs_SA < (double)s.f_margin) && (xS0 > 0.0);
    const bool ood = !(score <= s.gate);
    const bool fallback = ood || near_AS || near_SA || !(fabsf(xs_inc) <= s.xs_tol);
    double xS = xS0;
    float etr[6];
    int flag = NR_NONE;
    if (fallback) {
      // the plain law in the material frame: T, then S = C^-1 T (coaxial)
      float Tm[6], D[6], Cm[6], Ci[6];
      double fas = F_AS0, fsa = F_SA0;
      flag = law160_from_A<float>(m, A2, tmp, xS, fas, fsa, Tm, D);
      F_AS = fas;
      F_SA = fsa;
#pragma unroll
      for (int c = 0; c < 6; ++c) Cm[c] = (c < 3 ? 1.f : 0.f) + A2[c];
      sym_inv3<float>(Cm, Ci);
      sym_mul_commuting<float>(Ci, Tm, S);
      const float ex = (float)(m.eL * xS);
#pragma unroll
      for (int c = 0; c < 6; ++c) etr[c] = ex * D[c];
      // the law's own residual against the state the next step starts from
      // (xS, eps_tr): held like the network's, so a tile with points back
      // from the law needs no extra evaluation of the network
      float E[6], sp[6], ep[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) E[c] = 0.5f * A2[c];
      analytic_part<float>(m.kK, m.kG, m.alfa, E, etr, sp, ep);
      const float rE = (float)(1.0 / reuss_E(m, xS));
#pragma unroll
      for (int c = 0; c < 6; ++c) r[c] = S[c] * rE - sp[c];
    } else {
      // the transformation strain of an inactive point: its length eL xS0
      // turned onto the current direction (analytic_part); the network's
      // remainder on it (O(E^3) of eps_tr) is below its BF16 resolution and
      // is not integrated, so its noise cannot random-walk the state
#pragma unroll
      for (int c = 0; c < 6; ++c) etr[c] = etr_p[c];
    }
    if (valid) {
      a.snew[gp] = (float)xS;
      a.snew[a.sst + gp] = (float)F_AS;
      a.snew[2 * a.sst + gp] = (float)F_SA;
#pragma unroll
      for (int c = 0; c < 6; ++c) s.etr_new[c * a.sst + gp] = etr[c];
      // the residual held for the next steps: the network's after an
      // evaluation, the law's after a fallback
      if (refresh || fallback)
#pragma unroll
        for (int c = 0; c < 6; ++c) s.rcache[c * a.sst + gp] = __float2half_rn(r[c]);
    }
    // ---- tau = F S F^T (F = I + H, row-major) and the element forces ----
    float tau[6];
    {
      float FS[9];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const float f0 = (i == 0 ? 1.f : 0.f) + H[3 * i], f1 = (i == 1 ? 1.f : 0.f) + H[3 * i + 1],
                    f2 = (i == 2 ? 1.f : 0.f) + H[3 * i + 2];
        FS[3 * i + 0] = f0 * S[0] + f1 * S[3] + f2 * S[5];
        FS[3 * i + 1] = f0 * S[3] + f1 * S[1] + f2 * S[4];
        FS[3 * i + 2] = f0 * S[5] + f1 * S[4] + f2 * S[2];
      }
      // tau_ij = (F S)_ik F_jk; (i, j) = (0,0) (1,1) (2,2) (0,1) (1,2) (0,2)
      const int ii[6] = {0, 1, 2, 0, 1, 0}, jj[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const int i = ii[q], j = jj[q];
        tau[q] = FS[3 * i + 0] * ((j == 0 ? 1.f : 0.f) + H[3 * j]) +
                 FS[3 * i + 1] * ((j == 1 ? 1.f : 0.f) + H[3 * j + 1]) +
                 FS[3 * i + 2] * ((j == 2 ? 1.f : 0.f) + H[3 * j + 2]);
      }
    }
    const float Vn[3] = {0.f, 0.f, 0.f};
    const float detFJ = tile_forces<float, true, false>(a, hex8_tab<float>(), qsm, lane8, valid, nid, tau, Jc, detJ,
                                                         m, Vn);
    count_warp(a.cnt, CNT_NR_ACTIVE, valid && (flag & (NR_CONVERGED | NR_FAILED)));
    count_warp(a.cnt, CNT_SUR_FALLBACK, valid && fallback);
    count_warp(a.cnt, CNT_SUR_OOD, valid && ood);
    const bool negdet = !(detFJ * detJ > 0.f);
    if (__any_sync(0xffffffffu, valid && ((flag & (NR_FAILED | NR_BOTH)) || negdet))) {
      count_warp(a.cnt, CNT_NR_FAILED, valid && (flag & NR_FAILED));
      count_warp(a.cnt, CNT_NR_BOTH, valid && (flag & NR_BOTH));
      count_warp(a.cnt, CNT_NEG_DET, valid && negdet);
      if (valid && negdet) atomicMin(a.cnt + CNT_DETMIN, detmin_key(detFJ / (512.f * detJ), ec));
    }
    __syncthreads();                                             // tile_sm and the element rows are reused
  }
  mlp_teardown(ms);
}

// eps_tr = eL xS D of the TIME_N state at the current displacement (D the
// unit deviatoric direction of ln U): the surrogate's extra state, derived
// when the surrogate is switched on.  Lane = Gauss point, 8 per element.
template <bool CMP>
__global__ void __launch_bounds__(128) k_sur_etr_init(ElemArgs<float> a, float* etr) {
  __shared__ __align__(16) float elem_sm[16 * ElemSmem<float>::PER_ELEM];
  const int lane8 = threadIdx.x & 7, le = threadIdx.x >> 3;
  float* nsm = elem_sm + le * ElemSmem<float>::PER_ELEM;
  const int64_t e = (int64_t)blockIdx.x * 16 + le;
  const bool valid = e < a.end;
  const int64_t ec = valid ? e : (int64_t)a.end - 1;
  const int nid = a.lnods[8 * ec + lane8];
  const int src = (threadIdx.x & 31) & ~7;
  double X[3], U[3];
  float v[6];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    X[c] = __ldg(a.coord + c * a.npad + nid);
    U[c] = __ldg(a.u + c * a.npad + nid);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    v[c] = (float)(X[c] - __shfl_sync(0xffffffffu, X[c], src));
    v[3 + c] = (float)(U[c] - __shfl_sync(0xffffffffu, U[c], src));
  }
  stage_node_rows<float>(nsm, lane8, v);
  __syncwarp();
  float Ji[9], H[9];
  gp_kinematics<float>(nsm, lane8, Ji, H);
  float A2[6], Tm[6], D[6];
  green_2E<float>(H, A2);
  const int64_t gp = 8 * ec + lane8;
  double xS = (double)a.sold[gp], fas = (double)a.sold[a.sst + gp], fsa = (double)a.sold[2 * a.sst + gp];
  const double xS0 = xS;
  double tmp = 0.0;
  const MatC m = CMP ? compact_mat<float>(a, ec, &tmp) : a.mat0;
  if (!CMP) tmp = a.tempe ? __ldg(a.tempe + ec) : 0.0;
  law160_from_A<float>(m, A2, tmp, xS, fas, fsa, Tm, D);        // for D only
  if (valid)
#pragma unroll
    for (int c = 0; c < 6; ++c) etr[c * a.sst + gp] = (float)(m.eL * xS0) * D[c];
}

}  // namespace sur
}  // namespace sma
