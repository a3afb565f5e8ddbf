// sma_kernels.cuh -- sm_100a kernels of the explicit SMA step.
//
//   k_element   one thread per Gauss point, 8 lanes per HEX08 element:
//               gather (sld_elmgat.f90:53-63) of the 8 nodes into shared
//               memory relative to node 1, geometry (jacobi.f90:172-219),
//               F = I + du/dX (sld_elmpre.f90:149-221), law 160, P = tau F^-T
//               (= F S, sld_builtin_materials.f90:362-371), element forces
//               (sld_elmmat.f90:137-166), an 8-lane butterfly reduce-scatter
//               that leaves lane a with the force on node a, and the FP64
//               scatter-add into the nodal residual (mod_matrix.f90:2327-2431)
//               by atomics or colour-by-colour read-modify-write.
//   k_nodal     the central-difference node loops
//               (mod_sld_solution_methods.f90:122-145 and 192-210) with the
//               lumped-mass solve a = r * (1/m) (solric.f90:305-320) fused in;
//               FP64 always.
//   k_law_batch the material plugin on a batch of Gauss points.
#pragma once

#include "sma_law.cuh"

namespace sma {

constexpr int MAXFUN = 16;
constexpr int MAXPTS = 32;

enum Cnt { CNT_NR_ACTIVE = 0, CNT_NR_FAILED, CNT_NR_BOTH, CNT_NEG_DET, CNT_NONFINITE,
           CNT_FALLBACK64, NCNT = 8 };

// DISCRETE time functions (tload_sld tables), rows (t, vx, vy, vz)
struct FunTab {
  int nfun;
  int npts[MAXFUN];
  int smooth[MAXFUN];
  double tab[MAXFUN][MAXPTS][4];
};

// Time bookkeeping of the running step k, advanced on the device so the
// step loop needs no host round trip (setgts.f90:98, sld_updbcs.f90:85-114).
struct StepTime {
  double cutim;       // t_k
  double dtime;
  double c_corr;      // t_end - t_mid of step k  (corrector)
  double nx_cutim;    // t_{k+1}
  double nx_c_pred;   // t_mid - t of step k+1    (predictor)
  double nx_load;     // load factor at t_{k+1}
  double nx_fval[MAXFUN][3];
  int load_fun;
  int pad;
};

// sld_funbou.f90:99-140 for one dof
__device__ __forceinline__ double funbou(const FunTab* ft, int f, int idime, double cutim) {
  const int n = ft->npts[f];
  double xretu = 0.0;
  for (int k = 0; k < n - 1; ++k) {
    const double t1 = ft->tab[f][k][0], t2 = ft->tab[f][k + 1][0];
    if (cutim >= t1 && cutim <= t2) {
      const double p1 = ft->tab[f][k][1 + idime], p2 = ft->tab[f][k + 1][1 + idime];
      if (ft->smooth[f]) {
        const double m = (cutim - t1) / (t2 - t1);
        xretu = p1 + (p2 - p1) * pow(m, 3.0) * (10.0 - 15.0 * m + 6.0 * pow(m, 2.0));
      } else {
        const double m = (p2 - p1) / (t2 - t1);
        xretu = p1 + m * (cutim - t1);
      }
      break;
    }
  }
  const double tlast = ft->tab[f][n - 1][0];
  if (cutim > tlast) xretu = ft->tab[f][n - 1][1 + idime] * cutim / tlast;
  return xretu;
}

// corrector constant of step k and predictor data of step k+1
__device__ __forceinline__ void advance_time(StepTime* ts, const FunTab* ft) {
  const double cutim = ts->cutim, dt = ts->dtime;
  const double t_end = cutim + dt;
  const double t_mid = 0.5 * (cutim + t_end);
  ts->c_corr = t_end - t_mid;
  const double nc = cutim + dt;
  const double nte = nc + dt;
  const double ntm = 0.5 * (nc + nte);
  ts->nx_cutim = nc;
  ts->nx_c_pred = ntm - nc;
  for (int f = 0; f < ft->nfun; ++f)
    for (int i = 0; i < 3; ++i) ts->nx_fval[f][i] = funbou(ft, f, i, nc);
  ts->nx_load = (ts->load_fun >= 0) ? funbou(ft, ts->load_fun, 0, nc) : 0.0;
}

__global__ void k_advance_time(StepTime* ts, const FunTab* ft) {
  if (threadIdx.x == 0 && blockIdx.x == 0) advance_time(ts, ft);
}

// ---------------------------------------------------------------------------
// element kernel
// ---------------------------------------------------------------------------
template <typename T>
struct ElemArgs {
  const int32_t* lnods;        // (8, nelem), internal element order
  const double* coord;         // SoA [3][npad]
  const double* u;             // SoA [3][npad]
  double* f;                   // SoA [3][npad] residual accumulator
  const int32_t* lmate;        // (nelem) or null
  const MatC* mats;
  const double* tempe;         // (nelem) or null
  const T* sold;               // state TIME_N, SoA [3][sst]
  T* snew;                     // state ITER_K
  unsigned long long* cnt;
  StepTime* ts;                // non-null: advance the step time (block 0)
  const FunTab* ft;
  int64_t npad, sst;
  int32_t beg, end;            // element range of this launch
  double grav[3];              // rho-scaled body force per unit mass (elfext)
  int has_grav;
};

template <typename T>
struct ElemSmem { T v[6]; };

// 8-lane butterfly reduce-scatter: f[24] (node-major, 3 comps) summed over
// the 8 lanes of the element; lane a keeps node a.
template <typename T>
__device__ __forceinline__ void reduce_scatter8(const T* f, int lane8, T* out) {
  const unsigned FULL = 0xffffffffu;
  const bool b2 = lane8 & 4, b1 = lane8 & 2, b0 = lane8 & 1;
  T r12[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const T send = b2 ? f[k] : f[12 + k];
    const T keep = b2 ? f[12 + k] : f[k];
    r12[k] = keep + __shfl_xor_sync(FULL, send, 4);
  }
  T r6[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const T send = b1 ? r12[k] : r12[6 + k];
    const T keep = b1 ? r12[6 + k] : r12[k];
    r6[k] = keep + __shfl_xor_sync(FULL, send, 2);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const T send = b0 ? r6[k] : r6[3 + k];
    const T keep = b0 ? r6[3 + k] : r6[k];
    out[k] = keep + __shfl_xor_sync(FULL, send, 1);
  }
}

__device__ __forceinline__ void count_warp(unsigned long long* cnt, int idx, bool pred) {
  const unsigned b = __ballot_sync(0xffffffffu, pred);
  if (b && (threadIdx.x & 31) == 0) atomicAdd(cnt + idx, (unsigned long long)__popc(b));
}

template <typename T, bool ATOMIC>
__global__ void __launch_bounds__(256) k_element(ElemArgs<T> a) {
  extern __shared__ unsigned char smem_raw[];
  ElemSmem<T>* sm = reinterpret_cast<ElemSmem<T>*>(smem_raw);
  const int lane8 = threadIdx.x & 7;
  const int le = threadIdx.x >> 3;
  const int epb = blockDim.x >> 3;
  const int64_t e = (int64_t)a.beg + (int64_t)blockIdx.x * epb + le;
  const bool valid = e < a.end;
  const int64_t ec = valid ? e : (int64_t)a.end - 1;

  if (a.ts && blockIdx.x == 0 && threadIdx.x == 0) advance_time(a.ts, a.ft);

  // gather: lane a loads node a of its element
  const int nid = a.lnods[8 * ec + lane8];
  double X[3], U[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    X[c] = __ldg(a.coord + c * a.npad + nid);
    U[c] = __ldg(a.u + c * a.npad + nid);
  }
  // 9 slots per element (one pad slot) keep the 4 elements of a warp in
  // different shared-memory banks
  const int src = (threadIdx.x & 31) & ~7;
  ElemSmem<T>& mine = sm[le * 9 + lane8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double x0 = __shfl_sync(0xffffffffu, X[c], src);
    const double u0 = __shfl_sync(0xffffffffu, U[c], src);
    mine.v[c] = (T)(X[c] - x0);
    mine.v[3 + c] = (T)(U[c] - u0);
  }
  __syncwarp();
  const ElemSmem<T>* en = sm + le * 9;

  // geometry and displacement gradient at Gauss point g = lane8
  T N[8], dN[24];
  hex8_gp<T>(lane8, N, dN);
  T J[9], Gu[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) { J[k] = T(0); Gu[k] = T(0); }
#pragma unroll
  for (int n = 1; n < 8; ++n) {
    const ElemSmem<T> nd = en[n];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        J[3 * i + j] += nd.v[i] * dN[3 * n + j];
        Gu[3 * i + j] += nd.v[3 + i] * dN[3 * n + j];
      }
  }
  T Ji[9];
  const T detJ = inv3(J, Ji);         // Ji[3j+k] = dxi_j/dX_k
  T H[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      H[3 * i + k] = Gu[3 * i + 0] * Ji[0 + k] + Gu[3 * i + 1] * Ji[3 + k] + Gu[3 * i + 2] * Ji[6 + k];

  // constitutive update
  const int im = a.lmate ? a.lmate[ec] : 0;
  const MatC& mat = a.mats[im];
  const double tmp = a.tempe ? a.tempe[ec] : 0.0;
  const int64_t gp = 8 * ec + lane8;
  double xS = (double)a.sold[gp], F_AS = (double)a.sold[a.sst + gp], F_SA = (double)a.sold[2 * a.sst + gp];
  T tau[6];
  const int flag = law160_tau<T>(mat, H, tmp, xS, F_AS, F_SA, tau);
  if (valid) {
    a.snew[gp] = (T)xS;
    a.snew[a.sst + gp] = (T)F_AS;
    a.snew[2 * a.sst + gp] = (T)F_SA;
  }

  // P = tau F^-T; element force f_a = P gpcar_a vol = vol tau (F J)^-T dN_a
  T Fm[9], Fi[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) Fm[k] = H[k];
  Fm[0] += T(1); Fm[4] += T(1); Fm[8] += T(1);
  const T detF = inv3(Fm, Fi);
  T B[9];                              // B = Ji Fi = (F J)^-1
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      B[3 * m + k] = Ji[3 * m + 0] * Fi[0 + k] + Ji[3 * m + 1] * Fi[3 + k] + Ji[3 * m + 2] * Fi[6 + k];
  const T vol = detJ;                  // Gauss weight 1
  const T t00 = tau[0] * vol, t11 = tau[1] * vol, t22 = tau[2] * vol;
  const T t01 = tau[3] * vol, t12 = tau[4] * vol, t02 = tau[5] * vol;
  T Q[9];                              // Q[3i+m] = vol sum_k tau(i,k) B[3m+k]
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    Q[0 + m] = t00 * B[3 * m + 0] + t01 * B[3 * m + 1] + t02 * B[3 * m + 2];
    Q[3 + m] = t01 * B[3 * m + 0] + t11 * B[3 * m + 1] + t12 * B[3 * m + 2];
    Q[6 + m] = t02 * B[3 * m + 0] + t12 * B[3 * m + 1] + t22 * B[3 * m + 2];
  }
  T fe[24];                            // element residual contribution: -f_int (+ f_ext)
#pragma unroll
  for (int n = 0; n < 8; ++n)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      fe[3 * n + i] = -(Q[3 * i + 0] * dN[3 * n + 0] + Q[3 * i + 1] * dN[3 * n + 1] + Q[3 * i + 2] * dN[3 * n + 2]);
  if (a.has_grav) {
    const T rv = (T)mat.densi * vol;
#pragma unroll
    for (int n = 0; n < 8; ++n)
#pragma unroll
      for (int i = 0; i < 3; ++i) fe[3 * n + i] += (N[n] * rv) * (T)a.grav[i];
  }
  T out[3];
  reduce_scatter8<T>(fe, lane8, out);
  if (valid) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double* dst = a.f + c * a.npad + nid;
      if (ATOMIC) atomicAdd(dst, (double)out[c]);
      else *dst += (double)out[c];
    }
  }
  count_warp(a.cnt, CNT_NR_ACTIVE, valid && (flag & (NR_CONVERGED | NR_FAILED)));
  count_warp(a.cnt, CNT_NR_FAILED, valid && (flag & NR_FAILED));
  count_warp(a.cnt, CNT_NR_BOTH, valid && (flag & NR_BOTH));
  count_warp(a.cnt, CNT_NEG_DET, valid && !(detF > T(0)));
}

// ---------------------------------------------------------------------------
// nodal kernels (FP64): MODE 0 predictor, 1 corrector + next predictor,
// 2 corrector
// ---------------------------------------------------------------------------
struct NodalArgs {
  double* u;          // displacement
  double* vt;         // velocity at the half step (veloctmp_sld)
  double* v;          // velocity at the step boundary
  double* acc;        // acceleration at the step boundary
  double* f;          // residual accumulator
  const double* invm; // 1 / lumped mass
  const uint8_t* flags;   // bit c: dof c prescribed; bit 3: loaded
  const int8_t* bcfun;    // time function of the prescribed dofs, -1: value 0
  const double* fext;     // SoA [3][npad] nodal load at factor 1
  StepTime* ts;
  unsigned long long* cnt;
  int64_t npoin, npad;
};

template <int MODE>
__global__ void __launch_bounds__(256) k_nodal(NodalArgs a) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = p < a.npoin;
  bool bad = false;
  if (valid) {
    const StepTime& ts = *a.ts;
    const uint8_t fl = a.flags[p];
    const double dt = ts.dtime;
    double invm = 0.0;
    if (MODE >= 1) invm = a.invm[p];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t k = c * a.npad + p;
      double vv, aa;
      if (MODE == 0) {
        vv = a.v[k];
        aa = a.acc[k];
      } else {
        aa = 0.0 + a.f[k] * invm;           // lumped-mass solve
        vv = a.vt[k] + ts.c_corr * aa;      // corrector
        bad |= !isfinite(aa);
      }
      if (MODE == 2) {
        a.acc[k] = aa;
        a.v[k] = vv;
      } else {
        const double vt = vv + ts.nx_c_pred * aa;   // predictor of step k+1
        double un = a.u[k] + dt * vt;
        if (fl & (1u << c)) {
          const int fn = a.bcfun[p];
          un = (fn >= 0) ? ts.nx_fval[fn][c] : 0.0;
        }
        a.vt[k] = vt;
        a.u[k] = un;
        a.f[k] = (fl & 8u) ? a.fext[k] * ts.nx_load : 0.0;
      }
    }
  }
  if (MODE >= 1) count_warp(a.cnt, CNT_NONFINITE, valid && bad);
  if (MODE != 2 && blockIdx.x == 0 && threadIdx.x == 0) a.ts->cutim = a.ts->nx_cutim;
}

// witness: displacement of selected dofs after a step
__global__ void k_witness(const double* u, int64_t npad, const int32_t* wdof, int nwit,
                          double* hist, int* row, int max_rows) {
  const int r = *row;
  for (int w = threadIdx.x; w < nwit; w += blockDim.x) {
    const int d = wdof[w];
    if (r < max_rows) hist[(int64_t)r * nwit + w] = u[(int64_t)(d % 3) * npad + d / 3];
  }
  __syncthreads();
  if (threadIdx.x == 0) *row = r + 1;
}

// ---------------------------------------------------------------------------
// layout conversion between the reference's (3, npoin) and SoA [3][npad]
// ---------------------------------------------------------------------------
__global__ void k_aos_to_soa(const double* aos, double* soa, int64_t npoin, int64_t npad) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < npoin)
    for (int c = 0; c < 3; ++c) soa[c * npad + p] = aos[3 * p + c];
}
__global__ void k_soa_to_aos(const double* soa, double* aos, int64_t npoin, int64_t npad) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < npoin)
    for (int c = 0; c < 3; ++c) aos[3 * p + c] = soa[c * npad + p];
}
__global__ void k_fill_f(double* f, const double* fext, const uint8_t* flags, double scale,
                         int64_t npoin, int64_t npad) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < npoin)
    for (int c = 0; c < 3; ++c) {
      const int64_t k = c * npad + p;
      f[k] = (fext && (flags[p] & 8u)) ? fext[k] * scale : 0.0;
    }
}
// assemble outputs (3, npoin): rhsid, finte = fexte - rhsid, fexte (nodal
// loads), frxid = element part of rhsid on prescribed dofs
__global__ void k_outputs(const double* f, const double* fext, const uint8_t* flags,
                          double scale, int64_t npoin, int64_t npad, double* rhsid,
                          double* finte, double* fexte, double* frxid) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoin) return;
  const uint8_t fl = flags[p];
  for (int c = 0; c < 3; ++c) {
    const int64_t k = c * npad + p;
    const double r = f[k];
    const double fx = (fext && (fl & 8u)) ? fext[k] * scale : 0.0;
    rhsid[3 * p + c] = r;
    if (fexte) fexte[3 * p + c] = fx;
    if (finte) finte[3 * p + c] = fx - r;
    if (frxid) frxid[3 * p + c] = (fl & (1u << c)) ? r - fx : 0.0;
  }
}

// state layout: reference (3, 8, 2, nelem) <-> SoA [3][sst] per slot
template <typename T>
__global__ void k_state_in(const double* host_layout, const int32_t* perm, T* s_iterk,
                           T* s_timen, int64_t nelem, int64_t sst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;   // internal gp id
  if (i >= 8 * nelem) return;
  const int64_t e = i >> 3, g = i & 7;
  const int64_t ue = perm ? perm[e] : e;
  const double* src = host_layout + 48 * ue;
  for (int c = 0; c < 3; ++c) {
    s_iterk[c * sst + i] = (T)src[c + 3 * g];
    s_timen[c * sst + i] = (T)src[24 + c + 3 * g];
  }
}
template <typename T>
__global__ void k_state_out(double* host_layout, const int32_t* perm, const T* s_iterk,
                            const T* s_timen, int64_t nelem, int64_t sst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 8 * nelem) return;
  const int64_t e = i >> 3, g = i & 7;
  const int64_t ue = perm ? perm[e] : e;
  double* dst = host_layout + 48 * ue;
  for (int c = 0; c < 3; ++c) {
    dst[c + 3 * g] = (double)s_iterk[c * sst + i];
    dst[24 + c + 3 * g] = (double)s_timen[c * sst + i];
  }
}

// ---------------------------------------------------------------------------
// batched law (material-plugin boundary): F column-major (9n) -> PK2 (9n)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_law_batch(int64_t n, MatC mat, const double* F, const double* tmp,
                            const double* sdv_old, double* sdv_new, double* pk2,
                            int32_t* nr_flag) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const double* Fg = F + 9 * g;
  T H[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) H[3 * i + j] = (T)(Fg[i + 3 * j] - (i == j ? 1.0 : 0.0));
  double xS = sdv_old[3 * g], F_AS = sdv_old[3 * g + 1], F_SA = sdv_old[3 * g + 2];
  T tau[6];
  const int fl = law160_tau<T>(mat, H, tmp ? tmp[g] : 0.0, xS, F_AS, F_SA, tau);
  sdv_new[3 * g] = xS;
  sdv_new[3 * g + 1] = F_AS;
  sdv_new[3 * g + 2] = F_SA;
  // S = F^-1 tau F^-T (eval_sld_stress_model_160, :159-168)
  T Fm[9], Fi[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) Fm[k] = H[k];
  Fm[0] += T(1); Fm[4] += T(1); Fm[8] += T(1);
  inv3(Fm, Fi);
  const T tf[9] = {tau[0], tau[3], tau[5], tau[3], tau[1], tau[4], tau[5], tau[4], tau[2]};
  T Wt[9];                                   // Fi tau
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int l = 0; l < 3; ++l)
      Wt[3 * i + l] = Fi[3 * i + 0] * tf[0 + l] + Fi[3 * i + 1] * tf[3 + l] + Fi[3 * i + 2] * tf[6 + l];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      pk2[9 * g + i + 3 * j] = (double)(Wt[3 * i + 0] * Fi[3 * j + 0] + Wt[3 * i + 1] * Fi[3 * j + 1] +
                                        Wt[3 * i + 2] * Fi[3 * j + 2]);
  if (nr_flag) nr_flag[g] = fl;
}

}  // namespace sma
