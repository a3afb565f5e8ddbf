// sma_surrogate_elem.cuh -- the element loop with the learned surrogate in
// place of law 160's evaluation (the FP32 precision form).  Two kernels per
// step:
//
// k_element_sur, one block per tile of 16 elements (lane = Gauss point, 8
// lanes per element, 128 Gauss points per tile; tiles numbered over the
// whole mesh):
//   1. gather, kinematics (as k_element), E = (C - I)/2;
//   2. S = E(xS0) (r + S_p): r the stress residual held for the point
//      (FP16; the network's from its last evaluation on the tile, or the
//      plain law's if the law handled the point since), S_p the analytic
//      part (analytic_part: the law's elastic response with its
//      transformation strain eL xS0 on the current strain direction, as the
//      law keeps it);
//   3. the rotated-back Kirchhoff stress T = sym(C S) and from it the law's
//      loading functions F = +-|dev T| + 3 alpha tr(T)/3 - C T_K
//      (sld_stress_model_160.f90:513-537 with beta = 1: +-|dev T| =
//      2G (|e| - eL xS0), negative below the transformation strain);
//   4. gates -> the plain law (material frame, FP32 kinematics, FP64 return
//      map) for the point: no residual held (NaN: the network's gates
//      refused its last evaluation), an input outside the training inputs'
//      box, or loading functions within f_margin of a transformation start
//      (F_AS > Rs_AS - margin with xS0 < 1, F_SA < Rs_SA + margin with
//      xS0 > 0: the law's activation test, :351-374, needs the exact F
//      there).  The law's point then holds the law's own residual;
//   5. tau = F S F^T and the element forces as k_element (tile_forces);
//   6. on the step's due tiles ((tile + k) % period == 0, k the step index)
//      the network's inputs of each point into the staging rows (a point
//      the law handled is marked NaN there and keeps the law's residual).
// k_sur_refresh: the network on the staged tiles (tcgen05.mma into TMEM,
// 128 points per tile): each point's residual into the held residuals, or
// NaN where its out-of-envelope score is above `gate` or its predicted
// martensite increment above `xs_tol` (a point the law would transform):
// that point goes to the plain law on the next step.
//
// Why the residual is held: a BF16 network's output moves in quantisation
// steps while an explicit step moves the strain by ~1e-6; evaluated every
// step, those steps act as a local stiffness several times the elastic one
// and the explicit trajectory drifts.  Held for `period` steps, with the
// analytic part following the strain every step, it does not.
//
// Accepted points keep xS0 and store the loading functions of the predicted
// stress as (F_AS, F_SA); the law's points store the law's (xS, F_AS, F_SA).
#pragma once

#include "sma_kernels.cuh"
#include "sma_surrogate.cuh"

namespace sma {
namespace sur {

struct SurElemArgs {
  const SurStats* stats;      // the training inputs' box (lo_x, hi_x)
  __half* rcache;             // held stress residual per Gauss point, SoA [6][sst] (NaN: none, plain law)
  float* xstage;              // network inputs of the due tiles, [slot][NIN][128], slot = tile / period
  const StepTime* clock;      // the step's time (its index picks the due tiles)
  float f_margin;             // distance from the transformation surfaces (loading-function units)
  int period;                 // steps between two evaluations of the network on a tile
};

constexpr int SUR_BLOCK = 128, SUR_EPB = SUR_BLOCK / 8;
constexpr int CNT_SUR_FALLBACK = CNT_RESERVED5;   // points the plain law handled
constexpr int CNT_SUR_OOD = 7;                    // network evaluations its gates refused

// residue class of the tiles due in the running step: tile t is due when
// (t + k) % period == 0, k = t_k / dt the step index
__device__ __forceinline__ int due_class(const StepTime* clock, int period) {
  const int64_t k = clock ? (int64_t)(clock->cutim / clock->dtime + 0.5) : 0;
  return (int)((period - k % period) % period);
}

// node lane8 of element ec relative to the element's first node (formed in
// FP64, then FP32) into the element's shared-memory rows; returns its id
__device__ __forceinline__ int sur_gather(const ElemArgs<float>& a, float* nsm, int lane8, int64_t ec) {
  const int nid = a.lnods[8 * ec + lane8];
  const int src = (threadIdx.x & 31) & ~7;
  double X[3], U[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    X[c] = __ldg(a.coord + c * a.npad + nid);
    U[c] = __ldg(a.u + c * a.npad + nid);
  }
  float v[6];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    v[c] = (float)(X[c] - __shfl_sync(0xffffffffu, X[c], src));
    v[3 + c] = (float)(U[c] - __shfl_sync(0xffffffffu, U[c], src));
  }
  stage_node_rows<float>(nsm, lane8, v);
  __syncwarp();
  return nid;
}

// the network's inputs of one point into its staging row (x[0] = NaN: none)
__device__ __forceinline__ void sur_stage(float* row, const float* E, const float* etr_p, double tmp, double xS0,
                                          bool none) {
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    row[c * SUR_BLOCK] = (c == 0 && none) ? __int_as_float(0x7fc00000) : E[c];
    row[(6 + c) * SUR_BLOCK] = etr_p[c];
  }
  row[12 * SUR_BLOCK] = (float)tmp;
  row[13 * SUR_BLOCK] = (float)xS0;
}

template <bool CMP>
__global__ void __launch_bounds__(SUR_BLOCK, 6) k_element_sur(ElemArgs<float> a, SurElemArgs s) {
  __shared__ __align__(16) float elem_sm[SUR_EPB * ElemSmem<float>::PER_ELEM];
  if (a.ts && blockIdx.x == 0 && threadIdx.x == 0) advance_time(a.ts, a.ft);
  const int lane8 = threadIdx.x & 7, le = threadIdx.x >> 3;
  float* nsm = elem_sm + le * ElemSmem<float>::PER_ELEM;
  float* qsm = nsm + ElemSmem<float>::NODE_STRIDE;
  const int64_t tile = (int64_t)a.beg / SUR_EPB + blockIdx.x;
  const int64_t e = tile * SUR_EPB + le;
  const bool valid = e >= a.beg && e < a.end;
  const int64_t ec = e < a.beg ? (int64_t)a.beg : (e < a.end ? e : (int64_t)a.end - 1);
  // ---- gather and kinematics (as k_element) ----------------------------
  const int nid = sur_gather(a, nsm, lane8, ec);
  float Ji[9], H[9], Jc[9];
  const float detJ = gp_kinematics<float>(nsm, lane8, Ji, H, Jc);
  const int64_t gp = 8 * ec + lane8;
  const double xS0 = (double)a.sold[gp], F_AS0 = (double)a.sold[a.sst + gp];
  const double F_SA0 = (double)a.sold[2 * a.sst + gp];
  double tmp = 0.0;
  const MatC m = CMP ? compact_mat<float>(a, ec, &tmp) : a.mat0;
  if (!CMP) tmp = a.tempe ? __ldg(a.tempe + ec) : 0.0;
  float A2[6], E[6];                                             // C - I = 2E
  green_2E<float>(H, A2);
#pragma unroll
  for (int c = 0; c < 6; ++c) E[c] = 0.5f * A2[c];
  // ---- stress from the held residual and the analytic part ------------
  float r[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) r[c] = __half2float(s.rcache[c * a.sst + gp]);
  const float Ex = 1.f / reuss_iE_f(m, xS0);
  float S[6], etr_p[6];
  {
    float sp[6];
    analytic_part<float>(m.kK, m.kG, m.alfa, E, (float)(m.eL * xS0), sp, etr_p);
#pragma unroll
    for (int c = 0; c < 6; ++c) S[c] = (r[c] + sp[c]) * Ex;
  }
  bool inbox = (float)tmp >= s.stats->lo_x[12] && (float)tmp <= s.stats->hi_x[12] &&
               (float)xS0 >= s.stats->lo_x[13] && (float)xS0 <= s.stats->hi_x[13];
#pragma unroll
  for (int c = 0; c < 6; ++c)
    inbox &= E[c] >= s.stats->lo_x[c] && E[c] <= s.stats->hi_x[c] && etr_p[c] >= s.stats->lo_x[6 + c] &&
             etr_p[c] <= s.stats->hi_x[6 + c];
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
    const float proj = d0 * (E[0] - em) + d1 * (E[1] - em) + d2 * (E[2] - em) +
                       (t01 * A2[3] + t12 * A2[4] + t02 * A2[5]);
    // FP32: the loading functions feed the margin test and are stored as
    // FP32 state
    const float dn = sqrtf(d0 * d0 + d1 * d1 + d2 * d2 + 2.f * (t01 * t01 + t12 * t12 + t02 * t02));
    const float tp = (proj < 0.f ? -dn : dn) + 3.f * (float)m.alfa * p;
    F_AS = (double)(tp - (float)(m.C_AS * tmp));
    F_SA = (double)(tp - (float)(m.C_SA * tmp));
  }
  // A point on or near a transformation surface goes to the law, which
  // alone decides its activation: the test F > F0 (:351, :368) compares two
  // loading values one explicit step apart (~0.05 MPa), far below the
  // surrogate's stress error, so only points at least f_margin inside the
  // elastic band -- where neither transformation can start this step --
  // keep the surrogate's stress.
  const bool near_AS = (F_AS - m.Rs_AS > -(double)s.f_margin) && (xS0 < 1.0);
  const bool near_SA = (F_SA - m.Rs_SA < (double)s.f_margin) && (xS0 > 0.0);
  const bool fallback = isnan(r[0]) || !inbox || near_AS || near_SA;
  double xS = xS0;
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
    // the law's own residual against the state the next step starts from
    // (xS): held like the network's until the tile's next evaluation
    float sp[6], ep[6];
    analytic_part<float>(m.kK, m.kG, m.alfa, E, (float)(m.eL * xS), sp, ep);
    const float rE = reuss_iE_f(m, xS);
#pragma unroll
    for (int c = 0; c < 6; ++c) r[c] = S[c] * rE - sp[c];
  }
  if (valid) {
    a.snew[gp] = (float)xS;
    a.snew[a.sst + gp] = (float)F_AS;
    a.snew[2 * a.sst + gp] = (float)F_SA;
    if (fallback)
#pragma unroll
      for (int c = 0; c < 6; ++c) s.rcache[c * a.sst + gp] = __float2half_rn(r[c]);
    if (tile % s.period == due_class(s.clock, s.period))
      sur_stage(s.xstage + (tile / s.period) * (NIN * SUR_BLOCK) + threadIdx.x, E, etr_p, tmp, xS0, fallback);
  }
  // ---- tau = F S F^T (F = I + H, row-major) and the element forces ------
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
  const bool negdet = !(detFJ * detJ > 0.f);
  if (__any_sync(0xffffffffu, valid && ((flag & (NR_FAILED | NR_BOTH)) || negdet))) {
    count_warp(a.cnt, CNT_NR_FAILED, valid && (flag & NR_FAILED));
    count_warp(a.cnt, CNT_NR_BOTH, valid && (flag & NR_BOTH));
    count_warp(a.cnt, CNT_NEG_DET, valid && negdet);
    if (valid && negdet) atomicMin(a.cnt + CNT_DETMIN, detmin_key(detFJ / (512.f * detJ), ec));
  }
}

// The network's inputs of every point of the tiles in residue class `cls`
// (tile = slot * period + cls) at the TIME_N state and the current
// displacement: with k_sur_refresh, the first residual of each point when
// the surrogate is switched on.  One block per tile, lane = Gauss point.
template <bool CMP>
__global__ void __launch_bounds__(SUR_BLOCK) k_sur_stage(ElemArgs<float> a, SurElemArgs s, int cls) {
  __shared__ __align__(16) float elem_sm[SUR_EPB * ElemSmem<float>::PER_ELEM];
  const int lane8 = threadIdx.x & 7, le = threadIdx.x >> 3;
  float* nsm = elem_sm + le * ElemSmem<float>::PER_ELEM;
  const int64_t tile = (int64_t)blockIdx.x * s.period + cls;
  const int64_t e = tile * SUR_EPB + le;
  const bool valid = e < a.end;
  const int64_t ec = valid ? e : (int64_t)a.end - 1;
  sur_gather(a, nsm, lane8, ec);
  float Ji[9], H[9];
  gp_kinematics<float>(nsm, lane8, Ji, H);
  float A2[6], E[6], sp[6], etr_p[6];
  green_2E<float>(H, A2);
#pragma unroll
  for (int c = 0; c < 6; ++c) E[c] = 0.5f * A2[c];
  const int64_t gp = 8 * ec + lane8;
  const double xS0 = (double)a.sold[gp];
  double tmp = 0.0;
  const MatC m = CMP ? compact_mat<float>(a, ec, &tmp) : a.mat0;
  if (!CMP) tmp = a.tempe ? __ldg(a.tempe + ec) : 0.0;
  analytic_part<float>(m.kK, m.kG, m.alfa, E, (float)(m.eL * xS0), sp, etr_p);
  if (valid) sur_stage(s.xstage + (int64_t)blockIdx.x * (NIN * SUR_BLOCK) + threadIdx.x, E, etr_p, tmp, xS0, false);
}

struct RefreshArgs {
  const unsigned char* img;   // weight image (IMG_BYTES, 16-byte aligned)
  const SurStats* stats;
  const float* xstage;        // staged inputs, [slot][NIN][128]
  __half* rcache;             // held residuals, SoA [6][sst]
  const StepTime* clock;      // picks the residue class when cls < 0
  unsigned long long* cnt;    // counters (CNT_SUR_OOD), or NULL: not counted
  int* status;                // set to 1 if a wait for the tensor cores ran out
  int64_t sst, nelem;
  int cls;                    // residue class of the staged tiles; < 0: the running step's
  int period;
  float gate;                 // out-of-envelope score limit
  float xs_tol;               // predicted martensite increment allowed
};

// The network on the staged tiles: persistent blocks of 128 threads, the
// weight image in shared memory once per block, one tile (M = 128) per MMA
// chain.  Rows marked NaN (the plain law's points) and rows past the mesh
// keep what they hold.
static __global__ void __launch_bounds__(SUR_BLOCK) k_sur_refresh(RefreshArgs r) {
  extern __shared__ __align__(1024) unsigned char mlp_smem_raw[];
  MlpSmem& ms = *reinterpret_cast<MlpSmem*>(mlp_smem_raw + ((1024 - (smem_u32(mlp_smem_raw) & 1023)) & 1023));
  mlp_setup(ms, r.img);
  const SurStats& st = *r.stats;
  const int cls = r.cls >= 0 ? r.cls : due_class(r.clock, r.period);
  const int64_t ntiles = (r.nelem + SUR_EPB - 1) / SUR_EPB;
  const int64_t nslots = cls < ntiles ? (ntiles - cls + r.period - 1) / r.period : 0;
  for (int64_t slot = blockIdx.x; slot < nslots; slot += gridDim.x) {
    const int64_t gp = (slot * r.period + cls) * SUR_BLOCK + threadIdx.x;
    const bool live = gp < 8 * r.nelem;
    const float* row = r.xstage + slot * (NIN * SUR_BLOCK) + threadIdx.x;
    float x[NIN], xh[KIN], yh[KOUT];
#pragma unroll
    for (int c = 0; c < NIN; ++c) x[c] = live ? row[c * SUR_BLOCK] : st.mu_x[c];
    const bool skip = !live || isnan(x[0]);
    if (skip)
#pragma unroll
      for (int c = 0; c < NIN; ++c) x[c] = st.mu_x[c];
    const float score = normalise(st, x, xh);
    if (!mlp_tile(ms, xh, yh)) {                                 // block-uniform
      if (threadIdx.x == 0) atomicExch(r.status, 1);
      break;
    }
    bool refused = false;
    if (!skip) {
      const float xs_inc = yh[6] * st.sd_y[6] + st.mu_y[6];
      refused = !(score <= r.gate) || !(fabsf(xs_inc) <= r.xs_tol);
#pragma unroll
      for (int c = 0; c < 6; ++c)
        r.rcache[c * r.sst + gp] = refused ? __ushort_as_half((unsigned short)0x7fff)
                                           : __float2half_rn(yh[c] * st.sd_y[c] + st.mu_y[c]);
    }
    if (r.cnt) count_warp(r.cnt, CNT_SUR_OOD, refused);           // r.cnt is uniform
  }
  mlp_teardown(ms);
}

}  // namespace sur
}  // namespace sma
