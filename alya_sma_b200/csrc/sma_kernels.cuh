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
           CNT_RESERVED5, CNT_DETMIN, NCNT = 8 };

// CNT_DETMIN holds min over Gauss points with det F <= 0 of (det F, element)
// packed for one 64-bit atomicMin: the float's bits mapped to an unsigned
// key in the same order, then the internal element index; all ones = none
// (sld_elmpre.f90:229-238, gpdet_min / ielem_min).
__device__ __forceinline__ unsigned long long detmin_key(float det, int64_t e) {
  const unsigned b = __float_as_uint(det);
  const unsigned k = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  return ((unsigned long long)k << 32) | (unsigned long long)(unsigned)e;
}

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
  double load;        // load factor at t_k
  double phi;         // Tchamwa-Wielgosz parameter (tifac_sld(4))
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
        xretu = p1 + (p2 - p1) * (m * m * m) * (10.0 - 15.0 * m + 6.0 * (m * m));
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
__device__ __noinline__ void advance_time(StepTime* ts, const FunTab* ft) {
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
  const double* vel;           // SoA [3][npad] velocity for Rayleigh alpha, or null
  MatC mat0;                   // the material when lmate is null (kernel-parameter space);
                               // with compact records the values every element shares
  int64_t pf_ahead;            // elements ahead whose connectivity is prefetched to L2 (0: none)
  const T* matx;               // compact per-element records [nelem][MATX] (internal order), or null
};

// Compact per-element material record: the values a mesh whose elements
// differ only in their moduli,
// transformation strain and thresholds needs per element (the ensemble's and
// the cylinder's sampled materials), and the element's temperature.  The
// shared values (nu-derived factors, alpha, Clausius-Clapeyron slopes,
// density, Rayleigh alpha) stay in ElemArgs::mat0.  The Young's modulus
// enters through the Reuss rule E(xS0) = 1 / ((1 - xS0)/E_A + xS0/E_M),
// which is E_A when E_M = E_A.  FP64 forms store the values; FP32 forms store
// their offsets from mat0's (temperature: from mat0.T0) in FP32, 32 bytes
// per element, whose rounding (relative 6e-8 of an offset of ~10 %) stays
// an order below FP32 rounding of the values themselves: with the values
// rounded to FP32 the thresholds and temperature moved the step at which
// Gauss points start transforming, and the 2.0 M-element cylinder's 300-step
// FP32 trajectory parted from the FP64 oracle by 2e-5 instead of 2.5e-6.
enum MatX { MX_IEA = 0, MX_IEM, MX_EL, MX_RS_AS, MX_RF_AS, MX_RS_SA, MX_RF_SA, MX_TEMP, MATX };

// the element's material from its compact record: mat0's shared values,
// the record's own (8 lanes of an element read the same 8 words)
template <typename T>
__device__ __forceinline__ MatC compact_mat(const ElemArgs<T>& a, int64_t ec, double* tmp) {
  double r[MATX];
  const T* src = a.matx + MATX * ec;
  MatC m = a.mat0;
  if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int k = 0; k < MATX; k += 2) {
      const double2 v = __ldg(reinterpret_cast<const double2*>(src + k));
      r[k] = v.x;
      r[k + 1] = v.y;
    }
  } else {
    const float4 v0 = __ldg(reinterpret_cast<const float4*>(src));
    const float4 v1 = __ldg(reinterpret_cast<const float4*>(src + 4));
    r[MX_IEA] = m.iEA + (double)v0.x;
    r[MX_IEM] = m.iEM + (double)v0.y;
    r[MX_EL] = m.eL + (double)v0.z;
    r[MX_RS_AS] = m.Rs_AS + (double)v0.w;
    r[MX_RF_AS] = m.Rf_AS + (double)v1.x;
    r[MX_RS_SA] = m.Rs_SA + (double)v1.y;
    r[MX_RF_SA] = m.Rf_SA + (double)v1.z;
    r[MX_TEMP] = m.T0 + (double)v1.w;
  }
  m.iEA = r[MX_IEA];
  m.iEM = r[MX_IEM];
  m.eL = r[MX_EL];
  m.Rs_AS = r[MX_RS_AS];
  m.Rf_AS = r[MX_RF_AS];
  m.Rs_SA = r[MX_RS_SA];
  m.Rf_SA = r[MX_RF_SA];
  m.ext_E = 1;
  *tmp = r[MX_TEMP];
  return m;
}

// Shared memory of one element (8 lanes): node data as structure of arrays
// (phase 1 reads all 8 nodes of one component with 128-bit loads), and the
// 8 Gauss points' force operators Q (phase 2).  The strides carry a 16-byte
// pad so the 4 elements of a warp start in different banks.
template <typename T>
struct ElemSmem {
  static constexpr int NODE_STRIDE = 6 * 8 + 16 / sizeof(T);    // elements of T
  static constexpr int Q_STRIDE = 8 * 12 + 16 / sizeof(T);
  static constexpr int PER_ELEM = NODE_STRIDE + Q_STRIDE;
};

// reference-element table: dN_a/dxi_j and N_a at Gauss point g, stored
// [g][a][4] = (dN/ds, dN/dt, dN/dz, N).  Node a of the brick sits at s = +1
// for a in {1,2,5,6}, t = +1 for a in {2,3,6,7}, z = +1 for a >= 4
// (mod_lagrange.f90:935-977), so its factors and derivative signs follow
// from the bits of a.  Row k = 8 g + a:
template <typename T>
struct Hex8Row {
  T v[4];
};
template <typename T>
__host__ __device__ constexpr Hex8Row<T> hex8_tab_row(int k) {
  const T p = T(0.577350269189626);
  const int g = k >> 3, a = k & 7;
  const T s = (g & 4) ? p : -p, t = (g & 2) ? p : -p, z = (g & 1) ? p : -p;
  const int sa = (a ^ (a >> 1)) & 1, ta = (a >> 1) & 1, za = (a >> 2) & 1;
  const T S = T(0.5) * (sa ? T(1) + s : T(1) - s);
  const T Tt = T(0.5) * (ta ? T(1) + t : T(1) - t);
  const T Z = T(0.5) * (za ? T(1) + z : T(1) - z);
  return Hex8Row<T>{{(sa ? T(0.5) : T(-0.5)) * Tt * Z, (ta ? T(0.5) : T(-0.5)) * S * Z,
                     (za ? T(0.5) : T(-0.5)) * S * Tt, S * Tt * Z}};
}

// the table in shared memory, filled by the block (behind its barrier)
template <typename T>
__device__ __forceinline__ void fill_hex8_table(T* tab) {
  for (int k = threadIdx.x; k < 64; k += blockDim.x) {
    const Hex8Row<T> r = hex8_tab_row<T>(k);
#pragma unroll
    for (int c = 0; c < 4; ++c) tab[4 * k + c] = r.v[c];
  }
}

// the same table as a constant device array built at compile time, read
// through the read-only cache with no fill and no block barrier
template <typename T>
struct alignas(16) Hex8Tab {
  T v[256];
};
template <typename T>
constexpr Hex8Tab<T> make_hex8_tab() {
  Hex8Tab<T> r{};
  for (int k = 0; k < 64; ++k) {
    const Hex8Row<T> row = hex8_tab_row<T>(k);
    for (int c = 0; c < 4; ++c) r.v[4 * k + c] = row.v[c];
  }
  return r;
}
__device__ const Hex8Tab<float> g_hex8_tab_f = make_hex8_tab<float>();
__device__ const Hex8Tab<double> g_hex8_tab_d = make_hex8_tab<double>();
template <typename T>
__device__ __forceinline__ const T* hex8_tab();
template <>
__device__ __forceinline__ const float* hex8_tab<float>() { return g_hex8_tab_f.v; }
template <>
__device__ __forceinline__ const double* hex8_tab<double>() { return g_hex8_tab_d.v; }

__device__ __forceinline__ void count_warp(unsigned long long* cnt, int idx, bool pred) {
  const unsigned b = __ballot_sync(0xffffffffu, pred);
  if (b && (threadIdx.x & 31) == 0) atomicAdd(cnt + idx, (unsigned long long)__popc(b));
}

// vector loads of 4 consecutive T from shared memory (16-byte aligned)
__device__ __forceinline__ void lds4(const float* p, float* v) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void lds4(const double* p, double* v) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// vector loads of 8 consecutive T from shared memory
__device__ __forceinline__ void lds8(const float* p, float* v) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  const float4 b = *reinterpret_cast<const float4*>(p + 4);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void lds8(const double* p, double* v) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double2 a = *reinterpret_cast<const double2*>(p + 2 * k);
    v[2 * k] = a.x;
    v[2 * k + 1] = a.y;
  }
}

// The element's node rows in shared memory, [6][8] (x, y, z, ux, uy, uz of
// its 8 nodes relative to node 1), as their Walsh-Hadamard transform across
// the element's 8 lanes: lane k stores W_k = sum_a v_a (-1)^popc(a & k).
// A trilinear field sum_a v_a N_a(s,t,z) has, with the brick's node signs
// (s = +1 where bit0 ^ bit1 of a, t = +1 where bit1, z = +1 where bit2,
// mod_lagrange.f90:935-977),
//   8 d/ds = -W3 + W1 t + W7 z - W5 t z
//   8 d/dt = -W2 + W1 s + W6 z - W5 s z
//   8 d/dz = -W4 + W7 s + W6 t - W5 s t,
// so a Gauss point's 18 derivatives take 54 FMAs instead of 126, after three
// shuffle butterfly stages shared by the element's lanes.
template <typename T>
__device__ __forceinline__ void stage_node_rows(T* nsm, int lane8, const T* v) {
  T w[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) w[c] = v[c];
#pragma unroll
  for (int m = 1; m < 8; m <<= 1) {
    const T sg = (lane8 & m) ? T(-1) : T(1);                     // low lane w + p, high lane p - w
#pragma unroll
    for (int c = 0; c < 6; ++c) w[c] = fma(sg, w[c], __shfl_xor_sync(0xffffffffu, w[c], m));
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) nsm[8 * c + lane8] = w[c];
}

// Phase 1 of a tile, lane = Gauss point g (s, t, z from bits 2, 1, 0 of g,
// as hex8_gp): J8 = 8 dX/dxi and Gu8 = 8 du/dxi from the transformed node
// rows (stage_node_rows), Ji = J8^-1 and H = dU/dX = Gu8 J8^-1 (jacobi.f90:
// 172-219, sld_elmpre.f90:149-162), Jc8 = 8 F J = J8 + Gu8 if asked.
// Returns det J.
template <typename T>
__device__ __forceinline__ T gp_kinematics(const T* nsm, int g, T* Ji, T* H, T* Jc8 = nullptr) {
  const T p = T(0.577350269189626);
  const T s = (g & 4) ? p : -p, t = (g & 2) ? p : -p, z = (g & 1) ? p : -p;
  const T st = s * t, tz = t * z, sz = s * z;
  T J[9], Gu[9];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    T w[8];
    lds8(nsm + 8 * c, w);
    T* d = (c < 3) ? J + 3 * c : Gu + 3 * (c - 3);
    d[0] = w[1] * t + w[7] * z - w[5] * tz - w[3];
    d[1] = w[1] * s + w[6] * z - w[5] * sz - w[2];
    d[2] = w[7] * s + w[6] * t - w[5] * st - w[4];
  }
  const T det8 = inv3(J, Ji);                                    // det(8 J) = 512 det J
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      H[3 * i + k] = Gu[3 * i + 0] * Ji[0 + k] + Gu[3 * i + 1] * Ji[3 + k] + Gu[3 * i + 2] * Ji[6 + k];
  if (Jc8)
#pragma unroll
    for (int k = 0; k < 9; ++k) Jc8[k] = J[k] + Gu[k];
  return det8 * T(1.0 / 512.0);
}

// Phase 2 of a tile once the Kirchhoff stress tau of this lane's Gauss point
// is known: the force operator Q = vol tau (F J)^-T in shared memory, then
// lane = node a sums f_a = -sum_g Q_g dN_a(g) (+ the body force) and
// scatters it (FP64 atomics or read-modify-write).  Jc = 8 F J.  Returns
// det(8 F J).
template <typename T, bool ATOMIC, bool DAMP>
__device__ __forceinline__ T tile_forces(const ElemArgs<T>& a, const T* tab, T* qsm, int lane8, bool valid, int nid,
                                         const T* tau, const T* Jc, T detJ, const MatC& mat, const T* Vn) {
  // ---- force operator Q = vol tau (F J)^-T, f_a = -Q dN_a ---------------
  T B[9];                                                        // B = (8 F J)^-1 = dxi/dx / 8
  const T detFJ = inv3(Jc, B);                                   // det F = det(8 F J) / (512 det J)
  const T vol = detJ;                                            // Gauss weight 1
  const T vol8 = T(8) * detJ;                                    // vol (F J)^-1 = vol8 B
  const T t00 = tau[0] * vol8, t11 = tau[1] * vol8, t22 = tau[2] * vol8;
  const T t01 = tau[3] * vol8, t12 = tau[4] * vol8, t02 = tau[5] * vol8;
  T* q = qsm + 12 * lane8;
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    q[0 + m] = t00 * B[3 * m + 0] + t01 * B[3 * m + 1] + t02 * B[3 * m + 2];
    q[3 + m] = t01 * B[3 * m + 0] + t11 * B[3 * m + 1] + t12 * B[3 * m + 2];
    q[6 + m] = t02 * B[3 * m + 0] + t12 * B[3 * m + 1] + t22 * B[3 * m + 2];
  }
  // body force of the Gauss point, dV rho (g - alpha v(g)): gravity
  // (elfext) and the Rayleigh alpha term (elrayl_alpha, sld_elmmat.f90:159-
  // 164) with v(g) = sum_b N_b(g) v_b from the element's lanes by shuffle
  const bool body = DAMP || a.has_grav;
  if (body) {
    const T rho = (T)mat.densi;
    T b0 = rho * (T)a.grav[0], b1 = rho * (T)a.grav[1], b2 = rho * (T)a.grav[2];
    if constexpr (DAMP) {
      T N[8], dN[24];
      hex8_gp<T>(lane8, N, dN);
      const int src = (threadIdx.x & 31) & ~7;
      T v0 = T(0), v1 = T(0), v2 = T(0);
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        v0 += N[b] * __shfl_sync(0xffffffffu, Vn[0], src + b);
        v1 += N[b] * __shfl_sync(0xffffffffu, Vn[1], src + b);
        v2 += N[b] * __shfl_sync(0xffffffffu, Vn[2], src + b);
      }
      const T ra = rho * (T)mat.ray_a;
      b0 -= ra * v0;
      b1 -= ra * v1;
      b2 -= ra * v2;
    }
    q[9] = vol * b0;
    q[10] = vol * b1;
    q[11] = vol * b2;
  }
  __syncwarp();

  // ---- phase 2, lane = node a: sum the 8 Gauss points ---------------------
  T f0 = T(0), f1 = T(0), f2 = T(0);
#pragma unroll
  for (int g = 0; g < 8; ++g) {
    T qg[12], dn[4];
    lds4(qsm + 12 * g, qg);                                      // rows shared by the element
    lds4(qsm + 12 * g + 4, qg + 4);
    lds4(qsm + 12 * g + 8, qg + 8);
    lds4(tab + 32 * g + 4 * lane8, dn);                          // consecutive across lanes
    f0 -= qg[0] * dn[0] + qg[1] * dn[1] + qg[2] * dn[2];
    f1 -= qg[3] * dn[0] + qg[4] * dn[1] + qg[5] * dn[2];
    f2 -= qg[6] * dn[0] + qg[7] * dn[1] + qg[8] * dn[2];
    if (body) {
      f0 += dn[3] * qg[9];
      f1 += dn[3] * qg[10];
      f2 += dn[3] * qg[11];
    }
  }
  if (valid) {
    double* dst = a.f + nid;
    if (ATOMIC) {
      atomicAdd(dst, (double)f0);
      atomicAdd(dst + a.npad, (double)f1);
      atomicAdd(dst + 2 * a.npad, (double)f2);
    } else {
      dst[0] += (double)f0;
      dst[a.npad] += (double)f1;
      dst[2 * a.npad] += (double)f2;
    }
  }
  return detFJ;
}

// Work of one lane (element le, lane a) on one tile once its node is
// gathered: dX, dU are node a's coordinates and displacement relative to the
// element's first node (formed in FP64), (xS, F_AS, F_SA) the TIME_N state of
// Gauss point a, `mat` the element's material (the kernel parameter for a
// one-material mesh, so its constants are instruction operands; a shared-
// memory copy otherwise), `tmp` its temperature and Vn node a's velocity
// (read only in the DAMP instance, which adds the Rayleigh alpha force; the
// others keep the register budget of the undamped step).  Stages the node
// rows, then phase 1 (lane = Gauss point), the law, phase 2 (lane = node) and
// the scatter-add.  Needs the block's reference table in `tab`.
template <typename T, bool ATOMIC, bool DAMP = false>
__device__ __forceinline__ void element_tile(const ElemArgs<T>& a, const T* tab, T* nsm, T* qsm,
                                             int lane8, bool valid, int64_t ec, int nid,
                                             const double* dX, const double* dU,
                                             double xS, double F_AS, double F_SA,
                                             const MatC& mat, double tmp, const T* Vn) {
  {
    const T v[6] = {(T)dX[0], (T)dX[1], (T)dX[2], (T)dU[0], (T)dU[1], (T)dU[2]};
    stage_node_rows<T>(nsm, lane8, v);
  }
  const int64_t gp = 8 * ec + lane8;
  __syncwarp();                                                  // node rows of the element

  // ---- phase 1, lane = Gauss point g ------------------------------------
  T Ji[9], H[9], Jc[9];                                          // Jc = 8 F J, live across the law
  const T detJ = gp_kinematics<T>(nsm, lane8, Ji, H, Jc);

  // ---- constitutive update ----------------------------------------------
  T tau[6];
  const int flag = law160_tau<T>(mat, H, tmp, xS, F_AS, F_SA, tau);
  if (valid) {
    a.snew[gp] = (T)xS;
    a.snew[a.sst + gp] = (T)F_AS;
    a.snew[2 * a.sst + gp] = (T)F_SA;
  }

  const T detFJ = tile_forces<T, ATOMIC, DAMP>(a, tab, qsm, lane8, valid, nid, tau, Jc, detJ, mat, Vn);
  count_warp(a.cnt, CNT_NR_ACTIVE, valid && (flag & (NR_CONVERGED | NR_FAILED)));
  // the rare events behind one vote: failed return map, both transformations,
  // det F <= 0 (det F = det(8 F J) / (512 det J))
  const bool negdet = !(detFJ * detJ > T(0));
  if (__any_sync(0xffffffffu, valid && ((flag & (NR_FAILED | NR_BOTH)) || negdet))) {
    count_warp(a.cnt, CNT_NR_FAILED, valid && (flag & NR_FAILED));
    count_warp(a.cnt, CNT_NR_BOTH, valid && (flag & NR_BOTH));
    count_warp(a.cnt, CNT_NEG_DET, valid && negdet);
    if (valid && negdet)
      atomicMin(a.cnt + CNT_DETMIN, detmin_key((float)(detFJ / (T(512) * detJ)), ec));
  }
}


// a material is copied as MAT_CHUNKS 16-byte chunks by the 8 lanes of its element
constexpr int MAT_CHUNKS = (int)(sizeof(MatC) / 16);
static_assert(sizeof(MatC) % 16 == 0 && MAT_CHUNKS <= 16, "MatC copy layout");

// The element's material: the kernel parameter (one material) or the copy
// in shared memory (per-element materials).
template <bool MATS, typename T>
__device__ __forceinline__ const MatC& elem_mat(const ElemArgs<T>& a, const MatC* msm) {
  if constexpr (MATS) return *msm;
  else return a.mat0;
}

// Launch bounds of the element kernels: the largest block (NARROW: 128
// threads, the one-tile default; else 256) and the minimum resident blocks,
// which cap registers at 65536 / (threads x blocks).  Measured on B200 over
// fixed step windows of the one-tile kernel:
//   FP32, one material: 72 registers narrow (7 x 128: 28 warps per SM at
//     64-thread blocks, 32 B of spills), which beat 80 (24 warps) by 2.3 %
//     and 64 (32 warps, 56 B of spills) by 0.7 % on the 640 k-element
//     cantilever once the connectivity prefetch was in; 80 wide (3 x 256);
//   FP64, one material: 80 registers narrow (6 x 128, 24 warps, 80 B of
//     spills): -4.7 % against 96 on the cantilever;
//   FP32 with per-element materials, and FP64 with per-element materials:
//     96 registers at 5 x 128 (20 warps; FP32 92 without spills) beat 128
//     registers at 16 warps by 2-8 % (FP32 ensemble 1.643 -> 1.611 ms);
//     80 registers lost 18 % on the FP32 ensemble and were even in FP64,
//     168 registers at 12 warps lost 17 % on the FP64 cantilever;
//   256-thread blocks with per-element materials or FP64, and the pipelined
//     kernel: 2 x 256 (128 registers).
//   compact per-element records (CMP): no shared-memory material, no block
//     barrier: the one-material caps.
template <typename T, bool PIPE, bool MATS, bool NARROW = false, bool CMP = false>
constexpr int elem_min_blocks() {
  if (PIPE) return 2;
  if (NARROW) return (MATS && !CMP) ? 5 : (sizeof(T) == 4 ? 7 : 6);
  return (sizeof(T) == 4 && (!MATS || CMP)) ? 3 : 2;
}
constexpr int ELEM_NARROW_BLOCK = 128;

// One tile of elements per block: each lane gathers its node with __ldg,
// takes node 1's values from lane 0 of its element by shuffle.  MATS: the
// mesh has per-element materials (lmate), copied into shared memory per
// element.  DAMP: Rayleigh alpha damping with the velocity a.vel.  NARROW:
// compiled for blocks of at most ELEM_NARROW_BLOCK threads.  The reference
// table comes from the constant device array with one material (no block
// barrier: 2 % faster on the 640 k-element cantilever) and from a shared-
// memory copy with per-element materials (the constant array was 1.6 %
// slower on the 2.0 M-element cylinder).  With one material each lane also
// prefetches the connectivity one wave ahead: 4.9 % faster on the
// cantilever (4.1 % of it with the prefetch compiled in but not taken, from
// the instruction schedule around it); with per-element materials it was
// -1.2 % on the cylinder and +1.3 % on the 256-specimen ensemble, so off.
// CMP (with MATS): the element's material from its compact record in
// registers (compact_mat), the reference table from the constant array, no
// shared-memory material and no block barrier.
template <typename T, bool ATOMIC, bool MATS, bool DAMP = false, bool NARROW = false, bool CMP = false>
__global__ void __launch_bounds__(NARROW ? ELEM_NARROW_BLOCK : 256,
                                  (elem_min_blocks<T, false, MATS, NARROW, CMP>())) k_element(ElemArgs<T> a) {
  constexpr bool STAGE = MATS && !CMP;                           // material and table through shared memory
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tab_sm = reinterpret_cast<T*>(smem_raw);                    // [8][8][4]
  T* elem_sm = tab_sm + 256;
  const int lane8 = threadIdx.x & 7;
  const int le = threadIdx.x >> 3;
  const int epb = blockDim.x >> 3;
  const int64_t e = (int64_t)a.beg + (int64_t)blockIdx.x * epb + le;
  const bool valid = e < a.end;
  const int64_t ec = valid ? e : (int64_t)a.end - 1;
  T* nsm = elem_sm + le * ElemSmem<T>::PER_ELEM;                 // node rows [6][8]
  T* qsm = nsm + ElemSmem<T>::NODE_STRIDE;                       // Q rows [8][12]
  MatC* msm = reinterpret_cast<MatC*>(elem_sm + epb * ElemSmem<T>::PER_ELEM) + le;

  if (a.ts && blockIdx.x == 0 && threadIdx.x == 0) advance_time(a.ts, a.ft);
  if constexpr (STAGE) fill_hex8_table<T>(tab_sm);
  if constexpr (!STAGE) {
    // the connectivity of the element one resident wave ahead, into L2, so
    // the block that gathers it there starts from an L2 hit
    if (a.pf_ahead) {
      const int64_t ep = e + a.pf_ahead;
      if (ep < a.end) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.lnods + 8 * ep + lane8));
    }
  }

  const int nid = a.lnods[8 * ec + lane8];
  double tmp = 0.0;
  MatC mx;
  if constexpr (CMP) mx = compact_mat<T>(a, ec, &tmp);
  else tmp = a.tempe ? __ldg(a.tempe + ec) : 0.0;
  if constexpr (STAGE) {
    const uint4* src = reinterpret_cast<const uint4*>(a.mats + __ldg(a.lmate + ec));
    uint4* dst = reinterpret_cast<uint4*>(msm);
    dst[lane8] = __ldg(src + lane8);
    if (lane8 + 8 < MAT_CHUNKS) dst[8 + lane8] = __ldg(src + 8 + lane8);
  }
  double X[3], U[3], dX[3], dU[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    X[c] = __ldg(a.coord + c * a.npad + nid);
    U[c] = __ldg(a.u + c * a.npad + nid);
  }
  const int src = (threadIdx.x & 31) & ~7;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    dX[c] = X[c] - __shfl_sync(0xffffffffu, X[c], src);
    dU[c] = U[c] - __shfl_sync(0xffffffffu, U[c], src);
  }
  const int64_t gp = 8 * ec + lane8;
  const double xS = (double)a.sold[gp], F_AS = (double)a.sold[a.sst + gp];
  const double F_SA = (double)a.sold[2 * a.sst + gp];
  T Vn[3] = {T(0), T(0), T(0)};
  if constexpr (DAMP) {
#pragma unroll
    for (int c = 0; c < 3; ++c) Vn[c] = (T)__ldg(a.vel + c * a.npad + nid);
  }
  if constexpr (STAGE) __syncthreads();                          // reference table, materials
  if constexpr (CMP)
    element_tile<T, ATOMIC, DAMP>(a, hex8_tab<T>(), nsm, qsm, lane8, valid, ec, nid, dX, dU, xS, F_AS, F_SA,
                                  mx, tmp, Vn);
  else
    element_tile<T, ATOMIC, DAMP>(a, STAGE ? tab_sm : hex8_tab<T>(), nsm, qsm, lane8, valid, ec, nid, dX, dU,
                                  xS, F_AS, F_SA, elem_mat<MATS>(a, msm), tmp, Vn);
}

// ---------------------------------------------------------------------------
// Persistent element kernel: each block walks tiles blockIdx.x, +gridDim.x,
// ...; while it computes tile t, cp.async copies the node data and state of
// tile t+1 into a second shared-memory stage and the connectivity of tile t+2
// is already in a register, so the dependent gather (lnods -> coord, displ)
// is off the critical path.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
  else if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }

// one stage per element: 8 lanes x (X[3], U[3]) doubles, 8 x 3 state T
// (padded to 4), the material (MATS) and the temperature (+ 8 bytes pad);
// every part starts on a 16-byte boundary
template <typename T, bool MATS>
struct PipeStage {
  static constexpr int NODE_DOUBLES = 8 * 6;
  static constexpr int MAT_OFF = NODE_DOUBLES * 8 + 8 * 4 * (int)sizeof(T);
  static constexpr int TEMP_OFF = MAT_OFF + (MATS ? (int)sizeof(MatC) : 0);
  static constexpr int BYTES = TEMP_OFF + 16;
};

template <typename T, bool ATOMIC, bool MATS>
__global__ void __launch_bounds__(256, (elem_min_blocks<T, true, MATS>())) k_element_pipe(ElemArgs<T> a) {
  using PS = PipeStage<T, MATS>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tab = reinterpret_cast<T*>(smem_raw);
  T* elem_sm = tab + 256;
  const int lane8 = threadIdx.x & 7;
  const int le = threadIdx.x >> 3;
  const int epb = blockDim.x >> 3;
  T* nsm = elem_sm + le * ElemSmem<T>::PER_ELEM;
  T* qsm = nsm + ElemSmem<T>::NODE_STRIDE;
  unsigned char* stages = reinterpret_cast<unsigned char*>(elem_sm + epb * ElemSmem<T>::PER_ELEM);
  const int64_t n = (int64_t)a.end - a.beg;
  const int64_t ntiles = (n + epb - 1) / epb;

  if (a.ts && blockIdx.x == 0 && threadIdx.x == 0) advance_time(a.ts, a.ft);
  fill_hex8_table<T>(tab);
  __syncthreads();
  int64_t t = blockIdx.x;
  if (t >= ntiles) return;                                       // uniform across the block

  auto elem = [&](int64_t tile, bool& v) -> int64_t {
    const int64_t e = (int64_t)a.beg + tile * epb + le;
    v = e < a.end;
    return v ? e : (int64_t)a.end - 1;
  };
  auto stage_ptr = [&](int s) -> unsigned char* {
    return stages + ((size_t)s * epb + le) * PS::BYTES;
  };
  auto issue = [&](int s, int nid, int im, int64_t ec) {
    unsigned char* st = stage_ptr(s);
    double* nd = reinterpret_cast<double*>(st) + 6 * lane8;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      cp_async(nd + c, a.coord + c * a.npad + nid, 8);
      cp_async(nd + 3 + c, a.u + c * a.npad + nid, 8);
    }
    T* ss = reinterpret_cast<T*>(st + PS::NODE_DOUBLES * 8) + 4 * lane8;
    const int64_t gp = 8 * ec + lane8;
#pragma unroll
    for (int c = 0; c < 3; ++c) cp_async(ss + c, a.sold + c * a.sst + gp, (int)sizeof(T));
    if constexpr (MATS) {
      const unsigned char* src = reinterpret_cast<const unsigned char*>(a.mats + im);
      cp_async(st + PS::MAT_OFF + 16 * lane8, src + 16 * lane8, 16);
      if (lane8 + 8 < MAT_CHUNKS)
        cp_async(st + PS::MAT_OFF + 16 * (8 + lane8), src + 16 * (8 + lane8), 16);
    }
    if (a.tempe && lane8 == 0) cp_async(st + PS::TEMP_OFF, a.tempe + ec, 8);
  };
  auto mate = [&](int64_t ec) -> int { return MATS ? a.lmate[ec] : 0; };

  bool v0, v1;
  int64_t ec0 = elem(t, v0);
  int nid0 = a.lnods[8 * ec0 + lane8];
  issue(0, nid0, mate(ec0), ec0);
  cp_async_commit();
  int64_t t1 = t + gridDim.x;
  int64_t ec1 = elem(t1 < ntiles ? t1 : t, v1);
  int nid1 = a.lnods[8 * ec1 + lane8];
  int im1 = mate(ec1);
  int s = 0;
  for (; t < ntiles; t += gridDim.x) {
    const int64_t tn = t + gridDim.x;
    if (tn < ntiles) issue(s ^ 1, nid1, im1, ec1);
    cp_async_commit();
    const int64_t tn2 = tn + gridDim.x;
    bool v2;
    const int64_t ec2 = elem(tn2 < ntiles ? tn2 : t, v2);
    const int nid2 = a.lnods[8 * ec2 + lane8];
    const int im2 = mate(ec2);
    cp_async_wait1();                                            // this tile's copies landed
    __syncwarp();
    const unsigned char* st = stage_ptr(s);
    const double* nd = reinterpret_cast<const double*>(st);
    const T* ss = reinterpret_cast<const T*>(st + PS::NODE_DOUBLES * 8) + 4 * lane8;
    double dX[3], dU[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      dX[c] = nd[6 * lane8 + c] - nd[c];                         // relative to node 1 (lane 0)
      dU[c] = nd[6 * lane8 + 3 + c] - nd[3 + c];
    }
    const double tmp = a.tempe ? *reinterpret_cast<const double*>(st + PS::TEMP_OFF) : 0.0;
    const T Vn[3] = {T(0), T(0), T(0)};                         // undamped runs only
    element_tile<T, ATOMIC>(a, tab, nsm, qsm, lane8, v0, ec0, nid0, dX, dU, (double)ss[0],
                            (double)ss[1], (double)ss[2],
                            elem_mat<MATS>(a, reinterpret_cast<const MatC*>(st + PS::MAT_OFF)), tmp, Vn);
    __syncwarp();                                                // stage s is reused next-but-one
    nid0 = nid1; ec0 = ec1; v0 = v1;
    nid1 = nid2; ec1 = ec2; v1 = v2; im1 = im2;
    s ^= 1;
  }
  cp_async_wait0();
}

// dynamic shared memory of the element kernels for a block of `block` threads
// (k_element: table, element rows, then one material per element if mats)
template <typename T>
inline size_t element_smem_bytes(int block, bool mats) {
  return (256 + (size_t)(block / 8) * ElemSmem<T>::PER_ELEM) * sizeof(T) +
         (mats ? (size_t)(block / 8) * sizeof(MatC) : 0);
}
template <typename T>
inline size_t element_pipe_smem_bytes(int block, bool mats) {
  const size_t stage = mats ? PipeStage<T, true>::BYTES : PipeStage<T, false>::BYTES;
  return element_smem_bytes<T>(block, false) + 2 * (size_t)(block / 8) * stage;
}

// ---------------------------------------------------------------------------
// Stress/strain post-processing (sld_calculate_pp_tensors_ielem.f90:110-150,
// 186-218; itask 3 of the element loop).  Lane = Gauss point: the law is
// evaluated from the state in a.sold (its new state is discarded), then
//   sigma = tau / det F                  (= F P^T / det F of the reference)
//   E     = (H + H^T + H^T H) / 2        (Green strain, = (F^T F - I) / 2)
//   lnV   = log1p(H + H^T + H H^T) / 2   (logarithmic strain)
// and row g = dV_g (sigma, E, lnV, 1) in Voigt order xx yy zz yz xz xy
// (nvgij_sld, sld_inivar.f90:568-579).  Lane = node a then adds
// sum_g N_a(g) row_g into acc[19][npad] with FP64 atomics (the last column is
// the volume-lumped mass of mod_mass_matrix.f90:150-215).  gp_sig, if not
// null, receives sigma per Gauss point as (6, 8, nelem) in the caller's
// element order (perm maps the internal order to it).
// ---------------------------------------------------------------------------
constexpr int PP_COLS = 19;
constexpr int PP_ROW = 20;                 // doubles per Gauss-point row (16-byte multiple)

struct PostArgs {
  double* acc;                             // [PP_COLS][npad], or null: no nodal sums
  double* gp_sig;                          // (6, 8, nelem) or null
  double* gp_F;                            // gpgdi (3, 3, 8, nelem) column-major, or null
  double* gp_P;                            // gppio (3, 3, 8, nelem) column-major, or null
  double* gp_det;                          // det F (8, nelem), or null
  double* volum;                           // [2] += (dV, dV det F) (volum_sld), or null
  const int32_t* perm;                     // internal element -> caller's element
};

// shared memory: table, Gauss-point rows, node rows, materials
template <typename T>
inline size_t postproc_smem_bytes(int block, bool mats) {
  const size_t epb = (size_t)(block / 8);
  return 256 * sizeof(T) + epb * (8 * PP_ROW * sizeof(double) + ElemSmem<T>::NODE_STRIDE * sizeof(T)) +
         (mats ? epb * sizeof(MatC) : 0);
}

template <typename T, bool MATS>
__global__ void __launch_bounds__(128) k_postproc(ElemArgs<T> a, PostArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane8 = threadIdx.x & 7;
  const int le = threadIdx.x >> 3;
  const int epb = blockDim.x >> 3;
  T* tab = reinterpret_cast<T*>(smem_raw);                       // [8][8][4]
  double* rows_all = reinterpret_cast<double*>(tab + 256);       // [epb][8][PP_ROW]
  T* nsm_all = reinterpret_cast<T*>(rows_all + epb * 8 * PP_ROW); // [epb][NODE_STRIDE]
  MatC* msm = reinterpret_cast<MatC*>(nsm_all + epb * ElemSmem<T>::NODE_STRIDE) + le;
  double* rows = rows_all + le * 8 * PP_ROW;
  T* nsm = nsm_all + le * ElemSmem<T>::NODE_STRIDE;
  const int64_t e = (int64_t)a.beg + (int64_t)blockIdx.x * epb + le;
  const bool valid = e < a.end;
  const int64_t ec = valid ? e : (int64_t)a.end - 1;
  fill_hex8_table<T>(tab);

  const int nid = a.lnods[8 * ec + lane8];
  const double tmp = a.tempe ? __ldg(a.tempe + ec) : 0.0;
  if constexpr (MATS) {
    const uint4* src = reinterpret_cast<const uint4*>(a.mats + __ldg(a.lmate + ec));
    uint4* dst = reinterpret_cast<uint4*>(msm);
    dst[lane8] = __ldg(src + lane8);
    if (lane8 + 8 < MAT_CHUNKS) dst[8 + lane8] = __ldg(src + 8 + lane8);
  }
  double X[3], U[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    X[c] = __ldg(a.coord + c * a.npad + nid);
    U[c] = __ldg(a.u + c * a.npad + nid);
  }
  const int src = (threadIdx.x & 31) & ~7;
  {
    T v[6];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v[c] = (T)(X[c] - __shfl_sync(0xffffffffu, X[c], src));
      v[3 + c] = (T)(U[c] - __shfl_sync(0xffffffffu, U[c], src));
    }
    stage_node_rows<T>(nsm, lane8, v);
  }
  const int64_t gp = 8 * ec + lane8;
  double xS = (double)a.sold[gp], F_AS = (double)a.sold[a.sst + gp];
  double F_SA = (double)a.sold[2 * a.sst + gp];
  __syncthreads();                                               // table, node rows, materials

  T Ji[9], H[9];
  const T vol = gp_kinematics<T>(nsm, lane8, Ji, H);            // Gauss weight 1
  T tau[6];
  law160_tau<T>(elem_mat<MATS>(a, msm), H, tmp, xS, F_AS, F_SA, tau);
  const T detF = (T(1) + H[0]) * ((T(1) + H[4]) * (T(1) + H[8]) - H[5] * H[7])
               - H[1] * (H[3] * (T(1) + H[8]) - H[5] * H[6])
               + H[2] * (H[3] * H[7] - (T(1) + H[4]) * H[6]);
  const T iJ = Fm<T>::rcp(detF);
  // Voigt (xx yy zz yz xz xy); tau and L come as (xx yy zz xy yz xz)
  const double sig[6] = {(double)(tau[0] * iJ), (double)(tau[1] * iJ), (double)(tau[2] * iJ),
                         (double)(tau[4] * iJ), (double)(tau[5] * iJ), (double)(tau[3] * iJ)};
  T A[6], L[6], f[3];
  A[0] = T(2) * H[0] + (H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
  A[1] = T(2) * H[4] + (H[3] * H[3] + H[4] * H[4] + H[5] * H[5]);
  A[2] = T(2) * H[8] + (H[6] * H[6] + H[7] * H[7] + H[8] * H[8]);
  A[3] = H[1] + H[3] + (H[0] * H[3] + H[1] * H[4] + H[2] * H[5]);
  A[4] = H[5] + H[7] + (H[3] * H[6] + H[4] * H[7] + H[5] * H[8]);
  A[5] = H[2] + H[6] + (H[0] * H[6] + H[1] * H[7] + H[2] * H[8]);
  sym_log1p(A, L, f);
  // Green strain E_ij = (H_ij + H_ji + sum_k H_ki H_kj) / 2
  auto gre = [&](int i, int j) -> double {
    return 0.5 * ((double)H[3 * i + j] + (double)H[3 * j + i] + (double)H[i] * H[j] +
                  (double)H[3 + i] * H[3 + j] + (double)H[6 + i] * H[6 + j]);
  };
  const double dv = (double)vol;
  double* r = rows + lane8 * PP_ROW;
#pragma unroll
  for (int v = 0; v < 6; ++v) r[v] = dv * sig[v];
  r[6] = dv * gre(0, 0);
  r[7] = dv * gre(1, 1);
  r[8] = dv * gre(2, 2);
  r[9] = dv * gre(1, 2);
  r[10] = dv * gre(0, 2);
  r[11] = dv * gre(0, 1);
  r[12] = dv * 0.5 * (double)L[0];
  r[13] = dv * 0.5 * (double)L[1];
  r[14] = dv * 0.5 * (double)L[2];
  r[15] = dv * 0.5 * (double)L[4];
  r[16] = dv * 0.5 * (double)L[5];
  r[17] = dv * 0.5 * (double)L[3];
  r[18] = dv;
  if (p.gp_sig && valid) {
    double* o = p.gp_sig + 6 * (8 * (int64_t)p.perm[ec] + lane8);
#pragma unroll
    for (int v = 0; v < 6; ++v) o[v] = sig[v];
  }
  // element-loop fields: F, P = tau F^-T (sld_builtin_materials.f90:362-371),
  // det F (sld_elmpre.f90:217-226), column-major per Gauss point
  if ((p.gp_F || p.gp_P || p.gp_det) && valid) {
    const int64_t o9 = 9 * (8 * (int64_t)p.perm[ec] + lane8);
    T Fm[9], Fi[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) Fm[k] = H[k];
    Fm[0] += T(1); Fm[4] += T(1); Fm[8] += T(1);
    inv3(Fm, Fi);
    const T tf[9] = {tau[0], tau[3], tau[5], tau[3], tau[1], tau[4], tau[5], tau[4], tau[2]};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        if (p.gp_F) p.gp_F[o9 + i + 3 * j] = (double)Fm[3 * i + j];
        if (p.gp_P)
          p.gp_P[o9 + i + 3 * j] = (double)(tf[3 * i + 0] * Fi[3 * j + 0] + tf[3 * i + 1] * Fi[3 * j + 1] +
                                            tf[3 * i + 2] * Fi[3 * j + 2]);
      }
    if (p.gp_det) p.gp_det[8 * (int64_t)p.perm[ec] + lane8] = (double)detF;
  }
  if (p.volum) {                                                 // warp sums, one atomic per warp
    double v0 = valid ? dv : 0.0, v1 = valid ? dv * (double)detF : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      v0 += __shfl_xor_sync(0xffffffffu, v0, o);
      v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(p.volum, v0);
      atomicAdd(p.volum + 1, v1);
    }
  }
  __syncwarp();

  // lane = node a: sum over the element's Gauss points
  if (valid && p.acc) {
#pragma unroll 1
    for (int k = 0; k < PP_COLS; ++k) {
      double s = 0.0;
#pragma unroll
      for (int g = 0; g < 8; ++g) s += (double)tab[32 * g + 4 * lane8 + 3] * rows[g * PP_ROW + k];
      atomicAdd(p.acc + (int64_t)k * a.npad + nid, s);
    }
  }
}

// nodal values: X / vmass for the three tensors, von Mises of the Cauchy
// stress (sld_calculate_pp_tensors.f90:98-142); out = [caust | green | lepsi]
// each (6, npoin), then seqvm (npoin)
__global__ void k_postproc_nodal(const double* acc, int64_t npad, int64_t npoin, double* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npoin) return;
  const double inv = 1.0 / acc[(PP_COLS - 1) * npad + i];
  double c[6];
#pragma unroll
  for (int t = 0; t < 3; ++t)
#pragma unroll
    for (int v = 0; v < 6; ++v) {
      const double x = inv * acc[(6 * t + v) * npad + i];
      out[t * 6 * npoin + 6 * i + v] = x;
      if (t == 0) c[v] = x;
    }
  out[18 * npoin + i] = sqrt(0.5 * ((c[0] - c[1]) * (c[0] - c[1]) + (c[1] - c[2]) * (c[1] - c[2]) +
                                    (c[2] - c[0]) * (c[2] - c[0]) +
                                    6.0 * (c[3] * c[3] + c[4] * c[4] + c[5] * c[5])));
}

// ---------------------------------------------------------------------------
// nodal kernels (FP64): MODE 0 predictor, 1 corrector + next predictor,
// 2 corrector
// ---------------------------------------------------------------------------
struct NodalArgs {
  double* u;          // displacement
  double* vt;         // CD: velocity at the half step (veloctmp_sld); TW: predicted velocity
  double* v;          // velocity at the step boundary
  double* acc;        // acceleration at the step boundary
  double* f;          // residual accumulator
  const double* invm; // 1 / lumped mass
  const uint8_t* flags;   // bit c: dof c prescribed; bit 3: loaded
  const int8_t* bcfun;    // time function of the prescribed dofs, -1: value 0
  const double* fext;     // SoA [3][npad] nodal load at factor 1
  StepTime* ts;
  unsigned long long* cnt;
  // energy balance (ENERGY only): previous displacement and forces, and the
  // step's partial sums (ALLIE, ALLWK increments, 2*ALLKE, EENER)
  double* uprev;
  double* fint_prev;
  double* fext_prev;
  double* en_step;
  const double* fray;     // Rayleigh alpha nodal force of the step (kept out of fint), or null
  int store_v;            // MODE 1 also stores the step-boundary velocity (damped CD runs)
  int64_t npoin, npad;
};

constexpr int SCHEME_CD = 0, SCHEME_TW = 1;

// MODE 0: predictor of step k+1 from the step-boundary state
// MODE 1: corrector of step k fused with the predictor of step k+1
// MODE 2: corrector of step k (leaves the step-boundary state)
// CD: mod_sld_solution_methods.f90:122-145 (predictor), 192-210 (corrector)
// TW: mod_sld_solution_methods.f90:406-429 (predictor), 504-527 (corrector)
template <int MODE, int SCHEME, bool ENERGY>
__global__ void __launch_bounds__(256) k_nodal(NodalArgs a) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = p < a.npoin;
  bool bad = false;
  double e_ie = 0.0, e_wk = 0.0, e_ke = 0.0, e_ee = 0.0;
  if (valid) {
    const StepTime& ts = *a.ts;
    const uint8_t fl = a.flags[p];
    const double dt = ts.dtime;
    double invm = 0.0;
    if (MODE >= 1) invm = a.invm[p];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t k = c * a.npad + p;
      const bool fixed = fl & (1u << c);
      double vv, aa;
      if (MODE == 0) {
        vv = a.v[k];
        aa = a.acc[k];
      } else {
        const double r = a.f[k];
        aa = 0.0 + r * invm;                              // lumped-mass solve
        bad |= !isfinite(aa);
        if (SCHEME == SCHEME_CD) {
          vv = a.vt[k] + ts.c_corr * aa;                  // CD corrector
        } else {
          vv = fixed ? 0.0 : a.vt[k];                     // TW: fixed dofs at rest
          if (fixed) aa = 0.0;
        }
        if (ENERGY) {                                     // mod_sld_energy.f90:71-193
          const double uk = a.u[k];
          const double fx = (fl & 8u) ? a.fext[k] * ts.load : 0.0;
          // r = fext - fint - f_rayleigh (sld_elmmat.f90:170)
          const double fi = fx - r - (a.fray ? a.fray[k] : 0.0);
          const double dd = uk - a.uprev[k];
          e_ie += (fi + a.fint_prev[k]) * dd;
          e_wk += (fx + a.fext_prev[k]) * dd;
          e_ke += vv * vv / invm;
          e_ee += r * dd;
          a.uprev[k] = uk;
          a.fint_prev[k] = fi;
          a.fext_prev[k] = fx;
        }
      }
      if (MODE == 2) {
        a.acc[k] = aa;
        a.v[k] = vv;
      } else {
        if (MODE == 1 && a.store_v) a.v[k] = vv;                  // v_n for the next damping term
        double vn, un;
        if (SCHEME == SCHEME_CD) {
          vn = vv + ts.nx_c_pred * aa;                    // v at the half step k+1/2
          un = a.u[k] + dt * vn;
        } else {
          vn = vv + dt * aa;                              // TW predictor
          un = a.u[k] + dt * vv + ts.phi * (dt * dt) * aa;
        }
        if (fixed) {
          const int fn = a.bcfun[p];
          un = (fn >= 0) ? ts.nx_fval[fn][c] : 0.0;
        }
        a.vt[k] = vn;
        a.u[k] = un;
        a.f[k] = (fl & 8u) ? a.fext[k] * ts.nx_load : 0.0;
      }
    }
  }
  if (MODE >= 1) count_warp(a.cnt, CNT_NONFINITE, valid && bad);
  if (ENERGY && MODE >= 1) {
    // fixed-order sums (warp butterfly, then the block's 8 warps in order)
    // into one partial per block, so the balance is bitwise reproducible
    __shared__ double wsum[8][4];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      e_ie += __shfl_xor_sync(0xffffffffu, e_ie, o);
      e_wk += __shfl_xor_sync(0xffffffffu, e_wk, o);
      e_ke += __shfl_xor_sync(0xffffffffu, e_ke, o);
      e_ee += __shfl_xor_sync(0xffffffffu, e_ee, o);
    }
    if ((threadIdx.x & 31) == 0) {
      const int w = threadIdx.x >> 5;
      wsum[w][0] = e_ie; wsum[w][1] = e_wk; wsum[w][2] = e_ke; wsum[w][3] = e_ee;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += wsum[w][threadIdx.x];
      a.en_step[4 * (int64_t)blockIdx.x + threadIdx.x] = s;
    }
  }
  if (MODE != 2 && blockIdx.x == 0 && threadIdx.x == 0) {
    a.ts->cutim = a.ts->nx_cutim;
    a.ts->load = a.ts->nx_load;
  }
}

// energy totals after a step (mod_sld_energy.f90:130-157): increments are
// taken in absolute value, halved except on the first step; one history row
// (ALLIE, ALLWK, ALLKE, ETOTA, EENER) per step
// one block of 256 threads: the nodal kernel's per-block partials summed in
// a fixed order (strided per thread, then a tree), then the totals
__global__ void __launch_bounds__(256) k_energy_finalize(const double* part, int nblocks,
                                                         double* en_tot, double* hist, int* row,
                                                         int max_rows) {
  __shared__ double red[256][4];
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += 256)
    for (int q = 0; q < 4; ++q) s[q] += part[4 * (int64_t)b + q];
  for (int q = 0; q < 4; ++q) red[threadIdx.x][q] = s[q];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int q = 0; q < 4; ++q) red[threadIdx.x][q] += red[threadIdx.x + w][q];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const bool first = en_tot[4] == 0.0;
  const double w = first ? 1.0 : 0.5;
  en_tot[0] += w * fabs(red[0][0]);
  en_tot[1] += w * fabs(red[0][1]);
  en_tot[2] = 0.5 * red[0][2];
  en_tot[3] = fabs(red[0][3]);
  en_tot[4] += 1.0;
  const int r = *row;
  if (hist && r < max_rows) {
    double* h = hist + 5 * (int64_t)r;
    h[0] = en_tot[0];
    h[1] = en_tot[1];
    h[2] = en_tot[2];
    h[3] = en_tot[0] + en_tot[2] - en_tot[1];
    h[4] = en_tot[3];
  }
  *row = r + 1;
}

// witness: after the element loop of a step, record displacement (ids in
// [0, 3 npoin)) or residual (ids in [3 npoin, 6 npoin)) of selected dofs
__global__ void k_witness(const double* u, const double* f, int64_t npoin, int64_t npad,
                          const int32_t* wdof, int nwit, double* hist, int* row, int max_rows) {
  const int r = *row;
  for (int w = threadIdx.x; w < nwit; w += blockDim.x) {
    int d = wdof[w];
    const double* src = u;
    if (d >= 3 * npoin) { d -= (int)(3 * npoin); src = f; }
    if (r < max_rows) hist[(int64_t)r * nwit + w] = src[(int64_t)(d % 3) * npad + d / 3];
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
// pipelined element-loop boundary, nodes [p0, p1): displacement (3, npoin)
// -> SoA, and the residual initialised with the scaled nodal load
__global__ void k_assemble_in(const double* aos, double* u, double* f, const double* fext,
                              const uint8_t* flags, double scale, int64_t p0, int64_t p1,
                              int64_t npad) {
  const int64_t p = p0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= p1) return;
  const bool loaded = fext && (flags[p] & 8u);
  for (int c = 0; c < 3; ++c) {
    const int64_t k = c * npad + p;
    u[k] = aos[3 * p + c];
    f[k] = loaded ? fext[k] * scale : 0.0;
  }
}
// ... and the residual of nodes [p0, p1) back to (3, npoin)
__global__ void k_rhsid_out(const double* f, double* aos, int64_t p0, int64_t p1, int64_t npad) {
  const int64_t p = p0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < p1)
    for (int c = 0; c < 3; ++c) aos[3 * p + c] = f[c * npad + p];
}

// assemble outputs (3, npoin): rhsid, finte = fexte - rhsid, fexte (nodal
// loads), frxid = element part of rhsid on prescribed dofs
__global__ void k_outputs(const double* f, const double* fext, const uint8_t* flags,
                          double scale, int64_t npoin, int64_t npad, double* rhsid,
                          double* finte, double* fexte, double* frxid, const double* fray) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npoin) return;
  const uint8_t fl = flags[p];
  for (int c = 0; c < 3; ++c) {
    const int64_t k = c * npad + p;
    const double r = f[k];
    const double fx = (fext && (fl & 8u)) ? fext[k] * scale : 0.0;
    rhsid[3 * p + c] = r;
    if (fexte) fexte[3 * p + c] = fx;
    if (finte) finte[3 * p + c] = fx - r - (fray ? fray[k] : 0.0);   // damping kept out
    if (frxid) frxid[3 * p + c] = (fl & (1u << c)) ? r - fx : 0.0;
  }
}

// The Rayleigh alpha nodal force alone, sum_e sum_g N_a(g) dV rho alpha v(g)
// (elrayl_alpha of sld_elmmat.f90:159-164), FP64, one thread per element,
// added into fray (SoA [3][npad], zeroed by the caller).  The element kernel
// already folds this force into the residual; this pass exists so that the
// internal force of the energy balance and of sma_assemble's finte leaves it
// out, as the reference does.
__global__ void k_rayleigh(const int32_t* lnods, const double* coord, const double* vel,
                           const int32_t* lmate, const MatC* mats, MatC mat0, int64_t nelem,
                           int64_t npad, double* fray) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nelem) return;
  const MatC& m = lmate ? mats[lmate[e]] : mat0;
  if (!(m.ray_a > 0.0)) return;
  int nd[8];
  double X[8][3], V[8][3];
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    nd[b] = lnods[8 * e + b];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      X[b][c] = coord[c * npad + nd[b]];
      V[b][c] = vel[c * npad + nd[b]];
    }
  }
  double f[8][3];
#pragma unroll
  for (int b = 0; b < 8; ++b) f[b][0] = f[b][1] = f[b][2] = 0.0;
  const double ra = m.ray_a * m.densi;
  for (int g = 0; g < 8; ++g) {
    double N[8], dN[24];
    hex8_gp<double>(g, N, dN);
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, v[3] = {0, 0, 0};
    for (int b = 0; b < 8; ++b)
      for (int c = 0; c < 3; ++c) {
        J[3 * c + 0] += X[b][c] * dN[3 * b + 0];
        J[3 * c + 1] += X[b][c] * dN[3 * b + 1];
        J[3 * c + 2] += X[b][c] * dN[3 * b + 2];
        v[c] += N[b] * V[b][c];
      }
    const double detJ = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                        J[2] * (J[3] * J[7] - J[4] * J[6]);
    const double w = ra * detJ;                                  // Gauss weight 1
    for (int b = 0; b < 8; ++b)
      for (int c = 0; c < 3; ++c) f[b][c] += w * N[b] * v[c];
  }
  for (int b = 0; b < 8; ++b)
    for (int c = 0; c < 3; ++c) atomicAdd(fray + c * npad + nd[b], f[b][c]);
}

// state layout: reference (3, 8, 2, nelem) <-> SoA [3][sst] per slot; a
// null slot pointer leaves that slot alone (not read, not written)
template <typename T>
__global__ void k_state_in(const double* host_layout, const int32_t* perm, T* s_iterk,
                           T* s_timen, int64_t nelem, int64_t sst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;   // internal gp id
  if (i >= 8 * nelem) return;
  const int64_t e = i >> 3, g = i & 7;
  const int64_t ue = perm ? perm[e] : e;
  const double* src = host_layout + 48 * ue;
  for (int c = 0; c < 3; ++c) {
    if (s_iterk) s_iterk[c * sst + i] = (T)src[c + 3 * g];
    if (s_timen) s_timen[c * sst + i] = (T)src[24 + c + 3 * g];
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
    if (s_iterk) dst[c + 3 * g] = (double)s_iterk[c * sst + i];
    if (s_timen) dst[24 + c + 3 * g] = (double)s_timen[c * sst + i];
  }
}

// residual rows of selected nodes (interface nodes of a partitioned mesh):
// rows[3i + c] = f[c][nodes[i]]; ids outside [0, npoin) read as zero and are
// never written
__global__ void k_gather_rows(const double* f, int64_t npad, int64_t npoin, int32_t n,
                              const int32_t* nodes, double* rows) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t p = nodes[i];
  const bool ok = p >= 0 && p < npoin;
  for (int c = 0; c < 3; ++c) rows[3 * i + c] = ok ? f[c * npad + p] : 0.0;
}
__global__ void k_scatter_rows(double* f, int64_t npad, int64_t npoin, int32_t n, const int32_t* nodes,
                               const double* rows) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t p = nodes[i];
  if (p < 0 || p >= npoin) return;
  for (int c = 0; c < 3; ++c) f[c * npad + p] = rows[3 * i + c];
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

// ---------------------------------------------------------------------------
// batched law with the algorithmic tangent (flagt = 1,
// sld_stress_model_160.f90:118-155 and 170-191), FP64.  The Kirchhoff stress
// at F + eps/2 (e_i e_j^T + e_j e_i^T) F, eps = 1e-5 (:61), from the TIME_N
// state, for the six distinct pairs i <= j (the reference's nine evaluate
// each off-diagonal pair twice, with identical results); forward
// differences, the correction of its Eq. 68 with the unperturbed Kirchhoff
// stress, and the pull-back with F^-1 on all four indices.  Both index pairs
// are symmetric, so the tangent is carried as a 6 x 6 matrix on
// (xx yy zz xy yz xz) and expanded to the reference's (3,3,3,3) on output:
// dds[i + 3j + 9k + 27l + 81g].
// ---------------------------------------------------------------------------
__device__ __forceinline__ int voigt6(int i, int j) {
  return i == j ? i : (i + j == 1 ? 3 : (i + j == 3 ? 4 : 5));
}
__device__ __forceinline__ void voigt6_pair(int v, int& i, int& j) {
  i = v < 3 ? v : (v == 4 ? 1 : 0);
  j = v < 3 ? v : (v == 3 ? 1 : 2);
}

__global__ void __launch_bounds__(128) k_law_tangent(int64_t n, MatC mat, const double* F,
                                                     const double* tmp, const double* sdv_old,
                                                     double* sdv_new, double* pk2, double* dds,
                                                     int32_t* nr_flag) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const double eps = 1.0e-5;
  const double* Fg = F + 9 * g;
  double Fm[9], H[9];                                        // Fm[3i+j] = F(i, j)
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      Fm[3 * i + j] = Fg[i + 3 * j];
      H[3 * i + j] = Fm[3 * i + j] - (i == j ? 1.0 : 0.0);
    }
  const double tg = tmp ? tmp[g] : 0.0;
  const double xs0 = sdv_old[3 * g], fas0 = sdv_old[3 * g + 1], fsa0 = sdv_old[3 * g + 2];
  double xS = xs0, F_AS = fas0, F_SA = fsa0, tau[6];
  const int fl = law160_tau<double>(mat, H, tg, xS, F_AS, F_SA, tau);
  sdv_new[3 * g] = xS;
  sdv_new[3 * g + 1] = F_AS;
  sdv_new[3 * g + 2] = F_SA;
  if (nr_flag) nr_flag[g] = fl;

  // X[p][v]: d tau_v for the perturbation pair p, minus the Eq. 68 term
  double X[6][6];
  for (int p = 0; p < 6; ++p) {
    int i, j;
    voigt6_pair(p, i, j);
    double Hp[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        const double a = (r == i ? Fm[3 * j + c] : 0.0) + (r == j ? Fm[3 * i + c] : 0.0);
        Hp[3 * r + c] = H[3 * r + c] + 0.5 * eps * a;
      }
    double xs = xs0, fas = fas0, fsa = fsa0, tp[6];
    law160_tau<double>(mat, Hp, tg, xs, fas, fsa, tp);
    for (int v = 0; v < 6; ++v) {
      int c, d;
      voigt6_pair(v, c, d);
      const double corr = (i == c ? tau[voigt6(d, j)] : 0.0) + (c == j ? tau[voigt6(i, d)] : 0.0) +
                          (i == d ? tau[voigt6(c, j)] : 0.0) + (d == j ? tau[voigt6(i, c)] : 0.0);
      X[p][v] = (tp[v] - tau[v]) / eps - 0.5 * corr;
    }
  }

  // pull-back: G = Q X Q^T with Q[s][w] = sum over (m, n) of pair w of
  // F^-1(i, m) F^-1(j, n), (i, j) the pair s
  double Fi[9];
  inv3(Fm, Fi);
  double Q[6][6];
  for (int s = 0; s < 6; ++s) {
    int i, j;
    voigt6_pair(s, i, j);
    for (int w = 0; w < 6; ++w) {
      int m, nn;
      voigt6_pair(w, m, nn);
      Q[s][w] = Fi[3 * i + m] * Fi[3 * j + nn] + (m != nn ? Fi[3 * i + nn] * Fi[3 * j + m] : 0.0);
    }
  }
  double Y[6][6];                                            // Y = X Q^T
  for (int w = 0; w < 6; ++w)
    for (int t = 0; t < 6; ++t) {
      double acc = 0.0;
      for (int u = 0; u < 6; ++u) acc += X[w][u] * Q[t][u];
      Y[w][t] = acc;
    }
  double* out = dds + 81 * g;
  for (int s = 0; s < 6; ++s)
    for (int t = 0; t < 6; ++t) {
      double acc = 0.0;
      for (int w = 0; w < 6; ++w) acc += Q[s][w] * Y[w][t];
      int i, j, k, l;
      voigt6_pair(s, i, j);
      voigt6_pair(t, k, l);
      out[i + 3 * j + 9 * k + 27 * l] = acc;
      out[j + 3 * i + 9 * k + 27 * l] = acc;
      out[i + 3 * j + 9 * l + 27 * k] = acc;
      out[j + 3 * i + 9 * l + 27 * k] = acc;
    }

  // S = F^-1 tau F^-T (eval_sld_stress_model_160, :159-168)
  const double tf[9] = {tau[0], tau[3], tau[5], tau[3], tau[1], tau[4], tau[5], tau[4], tau[2]};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) acc += Fi[3 * i + k] * Fi[3 * j + l] * tf[3 * k + l];
      pk2[9 * g + i + 3 * j] = acc;
    }
}

}  // namespace sma
