/*
 * sma_oracle_impl.h -- body of the CPU oracle, instantiated twice by
 * sma_oracle.c with REAL = double (suffix _f64) and REAL = float (_f32).
 *
 * TEST INFRASTRUCTURE ONLY (see sma_oracle.h).
 *
 * Reference files restated here (paths relative to the reference's src/):
 *   modules/solidz/sld_stress_model_160.f90       law 160 (NITINOL)
 *   alya-kernel/mathru/dsytrd3.f90, dsyevq3.f90   Householder + implicit QL
 *                                                 (Kopp, "Efficient numerical
 *                                                 diagonalization of hermitian
 *                                                 3x3 matrices", IJMPC 19 (2008))
 *   alya-kernel/mathru/eigsrt.f90                 eigenpair sort (descending)
 *   alya-fem/mod_lagrange.f90:935-977             HEX08 shape functions
 *   alya-fem/mod_quadrature_gauss.f90:2320-2386   2x2x2 Gauss rule
 *   alya-kernel/domain/jacobi.f90:172-219         Jacobian, gpcar, det
 *   alya-kernel/domain/elmlen.f90:75-146          element lengths
 *   modules/solidz/sld_elmpre.f90:149-226         deformation gradient
 *   modules/solidz/sld_builtin_materials.f90:355-372  PK2 -> PK1
 *   modules/solidz/sld_elmmat.f90:115-244         explicit element forces + mass
 *   modules/solidz/sld_element_operations.f90:239-256  assembly
 *   modules/solidz/sld_elmope.f90:53-99           colour-parallel element loop
 *   modules/solidz/mod_sld_solution_methods.f90:101-223  central difference
 *   alya-kernel/solite/solric.f90:305-320         lumped-mass Richardson solve
 *   modules/solidz/sld_funbou.f90:99-140          tabulated smooth-step BCs
 *   modules/solidz/sld_velsnd.f90:117-124         sound speed for law 160
 *   modules/solidz/mod_sld_minle_time_step.f90:262-268  critical time step
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SUFFIX)
#define M3(A, i, j) (A)[(i) + 3 * (j)]

/* ------------------------------------------------------------------------ */
/* 3x3 symmetric eigen-decomposition: Householder tridiagonalisation followed
 * by the QL method with implicit shifts, as in dsytrd3.f90:22-108 and
 * dsyevq3.f90:22-136.  Only the diagonal and upper triangle of A are read. */
/* ------------------------------------------------------------------------ */
static void FN(tridiag3)(const REAL* A, REAL* Q, REAL* d, REAL* e)
{
  REAL u[3], p[3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) M3(Q, i, j) = (i == j) ? (REAL)1 : (REAL)0;

  /* first row/column to tridiagonal form: dsytrd3.f90:198-238 */
  REAL h = M3(A, 0, 1) * M3(A, 0, 1) + M3(A, 0, 2) * M3(A, 0, 2);
  REAL g = (M3(A, 0, 1) > 0) ? -SQRT(h) : SQRT(h);
  e[0] = g;
  REAL f = g * M3(A, 0, 1);
  u[1] = M3(A, 0, 1) - g;
  u[2] = M3(A, 0, 2);
  REAL omega = h - f;
  if (omega > 0) {
    omega = (REAL)1 / omega;
    REAL K = 0;
    /* p = omega * A' u restricted to rows/cols 2..3 (upper triangle access) */
    f = M3(A, 1, 1) * u[1] + M3(A, 1, 2) * u[2];
    p[1] = omega * f;
    K = K + u[1] * f;
    f = M3(A, 1, 2) * u[1] + M3(A, 2, 2) * u[2];
    p[2] = omega * f;
    K = K + u[2] * f;
    K = (REAL)0.5 * K * omega * omega;
    p[1] = p[1] - K * u[1];
    p[2] = p[2] - K * u[2];
    d[0] = M3(A, 0, 0);
    d[1] = M3(A, 1, 1) - (REAL)2 * p[1] * u[1];
    d[2] = M3(A, 2, 2) - (REAL)2 * p[2] * u[2];
    for (int j = 1; j < 3; ++j) {
      f = omega * u[j];
      for (int i = 1; i < 3; ++i) M3(Q, i, j) = M3(Q, i, j) - f * u[i];
    }
    e[1] = M3(A, 1, 2) - p[1] * u[2] - u[1] * p[2];
  } else {
    for (int i = 0; i < 3; ++i) d[i] = M3(A, i, i);
    e[1] = M3(A, 1, 2);
  }
}

void FN(orc_dsyevq3)(const REAL A[9], REAL Q[9], REAL w[3], int* fail)
{
  REAL e[3];
  *fail = 0;
  FN(tridiag3)(A, Q, w, e);
  e[2] = 0;
  /* QL with implicit shifts: dsyevq3.f90:64-134 */
  for (int l = 0; l < 2; ++l) {
    int niter = 0;
    for (int it = 0; it < 50; ++it) {
      int m;
      for (m = l; m < 2; ++m) {
        REAL g = FABS(w[m]) + FABS(w[m + 1]);
        if (FABS(e[m]) + g == g) break;
      }
      if (m == l) break;
      if (++niter >= 30) { *fail = 1; return; }
      REAL g = (w[l + 1] - w[l]) / ((REAL)2 * e[l]);
      REAL r = SQRT((REAL)1 + g * g);
      if (g >= 0) g = w[m] - w[l] + e[l] / (g + r);
      else        g = w[m] - w[l] + e[l] / (g - r);
      REAL s = 1, c = 1, p = 0;
      for (int j = m - 1; j >= l; --j) {
        REAL f = s * e[j];
        REAL b = c * e[j];
        if (FABS(f) > FABS(g)) {
          c = g / f;
          r = SQRT((REAL)1 + c * c);
          e[j + 1] = f * r;
          s = (REAL)1 / r;
          c = c * s;
        } else {
          s = f / g;
          r = SQRT((REAL)1 + s * s);
          e[j + 1] = g * r;
          c = (REAL)1 / r;
          s = s * c;
        }
        g = w[j + 1] - p;
        r = (w[j] - g) * s + (REAL)2 * c * b;
        p = s * r;
        w[j + 1] = g + p;
        g = c * r - b;
        for (int k = 0; k < 3; ++k) {
          REAL t = M3(Q, k, j + 1);
          M3(Q, k, j + 1) = s * M3(Q, k, j) + c * t;
          M3(Q, k, j) = c * M3(Q, k, j) - s * t;
        }
      }
      w[l] = w[l] - p;
      e[l] = g;
      e[m] = 0;
    }
  }
}

/* eigsrt.f90:19-48: selection sort, largest eigenvalue first (ties move). */
void FN(orc_eigsrt)(REAL d[3], REAL V[9])
{
  for (int i = 0; i < 2; ++i) {
    int k = i;
    REAL p = d[i];
    for (int j = i + 1; j < 3; ++j)
      if (d[j] >= p) { k = j; p = d[j]; }
    if (k != i) {
      d[k] = d[i];
      d[i] = p;
      for (int r = 0; r < 3; ++r) {
        REAL t = M3(V, r, i);
        M3(V, r, i) = M3(V, r, k);
        M3(V, r, k) = t;
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Law 160 (sld_stress_model_160.f90)                                        */
/* ------------------------------------------------------------------------ */

/* eval_loading_function, :513-537, with eval_beta forced to 1 (:554) */
static inline REAL FN(loading)(REAL K, REAL G, REAL alfa, REAL C, REAL eL,
                                REAL theta, REAL enor, REAL tmp, REAL xS)
{
  REAL pres = K * (theta - (REAL)3 * alfa * eL * xS);
  REAL trac = (REAL)2 * G * (enor - eL * xS);
  REAL beta = 1;
  return trac * beta + (REAL)3 * alfa * pres - C * tmp;
}

/* INV3x3, :575-599 */
static void FN(inv3x3)(const REAL* M, REAL* Mi)
{
  REAL det = M3(M,0,0)*M3(M,1,1)*M3(M,2,2) + M3(M,0,2)*M3(M,1,0)*M3(M,2,1)
           + M3(M,2,0)*M3(M,0,1)*M3(M,1,2) - M3(M,2,0)*M3(M,1,1)*M3(M,0,2)
           - M3(M,2,2)*M3(M,0,1)*M3(M,1,0) - M3(M,0,0)*M3(M,1,2)*M3(M,2,1);
  M3(Mi,0,0) =  (M3(M,1,1)*M3(M,2,2) - M3(M,2,1)*M3(M,1,2)) / det;
  M3(Mi,0,1) = -(M3(M,0,1)*M3(M,2,2) - M3(M,0,2)*M3(M,2,1)) / det;
  M3(Mi,0,2) =  (M3(M,0,1)*M3(M,1,2) - M3(M,1,1)*M3(M,0,2)) / det;
  M3(Mi,1,0) = -(M3(M,1,0)*M3(M,2,2) - M3(M,2,0)*M3(M,1,2)) / det;
  M3(Mi,1,1) =  (M3(M,0,0)*M3(M,2,2) - M3(M,0,2)*M3(M,2,0)) / det;
  M3(Mi,1,2) = -(M3(M,0,0)*M3(M,1,2) - M3(M,1,0)*M3(M,0,2)) / det;
  M3(Mi,2,0) =  (M3(M,1,0)*M3(M,2,1) - M3(M,2,0)*M3(M,1,1)) / det;
  M3(Mi,2,1) = -(M3(M,0,0)*M3(M,2,1) - M3(M,2,0)*M3(M,0,1)) / det;
  M3(Mi,2,2) =  (M3(M,0,0)*M3(M,1,1) - M3(M,0,1)*M3(M,1,0)) / det;
}

/* Young's modulus at the start-of-step martensite fraction.  Extension with
 * no reference counterpart: Reuss mix of austenite (props[0]) and martensite
 * moduli.  e_mart <= 0 or e_mart == props[0] returns props[0] unchanged, which
 * is the reference law. */
static inline REAL FN(young)(REAL E_A, REAL e_mart, REAL xS0)
{
  if (!(e_mart > 0) || e_mart == E_A) return E_A;
  return (REAL)1 / (((REAL)1 - xS0) / E_A + xS0 / e_mart);
}

/* compute_kirchoff_stress, :212-500 (linear flow rule, beta = 1).
 * sdv = (xS, F_AS, F_SA) in: previous step, out: this step.
 * tmp is the temperature; the reference hard-wires 0 (:105). */
int FN(orc_law160_kirchhoff)(const REAL props[18], REAL e_mart, const REAL F[9],
                             REAL tmp, REAL sdv[3], REAL tau[9])
{
  const int iter_NR = 65;
  const REAL tole_NR = (REAL)1.0e-8;
  int flag = ORC_NR_NONE;

  REAL xS_0 = sdv[0], F_AS_0 = sdv[1], F_SA_0 = sdv[2];

  REAL E = FN(young)(props[0], e_mart, xS_0);
  REAL v = props[1], eL = props[2];
  REAL Ss_AS = props[3], Sf_AS = props[4], C_AS = props[5];
  REAL Tf_AS = props[6], Ts_AS = props[7];
  REAL Ss_SA = props[9], Sf_SA = props[10], C_SA = props[11];
  REAL Tf_SA = props[12], Ts_SA = props[13], alfa = props[14];

  REAL K = E / ((REAL)3 - (REAL)6 * v);
  REAL G = E / ((REAL)2 + (REAL)2 * v);
  REAL aux = SQRT((REAL)2 / (REAL)3) + alfa;
  REAL Rf_AS = Sf_AS * aux + C_AS * Tf_AS;
  REAL Rs_AS = Ss_AS * aux + C_AS * Ts_AS;
  REAL Rf_SA = Sf_SA * aux + C_SA * Tf_SA;
  REAL Rs_SA = Ss_SA * aux + C_SA * Ts_SA;
  REAL G_1 = ((REAL)2 * G + (REAL)9 * (alfa * alfa) * K) * eL;

  /* b = F F^T, :293 */
  REAL b[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      REAL s = 0;
      for (int k = 0; k < 3; ++k) s = s + M3(F, i, k) * M3(F, j, k);
      M3(b, i, j) = s;
    }

  /* spectral decomposition, :298-308 */
  REAL n_A[9], h_A[3];
  int eigfail;
  FN(orc_dsyevq3)(b, n_A, h_A, &eigfail);
  FN(orc_eigsrt)(h_A, n_A);
  REAL h1 = SQRT(h_A[0]), h2 = SQRT(h_A[1]), h3 = SQRT(h_A[2]);

  /* logarithmic strains, :313-332 */
  REAL J_vol = h1 * h2 * h3;
  REAL theta = LOG(J_vol);
  REAL J_dev = POW(J_vol, (REAL)-1 / (REAL)3);
  REAL e1 = LOG(J_dev * h1), e2 = LOG(J_dev * h2), e3 = LOG(J_dev * h3);
  REAL e_n = SQRT(e1 * e1 + e2 * e2 + e3 * e3);
  REAL d1, d2, d3;
  if (e_n > REAL_EPS) { d1 = e1 / e_n; d2 = e2 / e_n; d3 = e3 / e_n; }
  else { d1 = 0; d2 = 0; d3 = 0; }

  /* activation, :342-374 */
  REAL F_AS = FN(loading)(K, G, alfa, C_AS, eL, theta, e_n, tmp, xS_0);
  REAL Fs_AS = F_AS - Rs_AS;
  REAL F_AS_dot = F_AS - F_AS_0;
  int kf_AS = (F_AS > F_AS_0 && Fs_AS > 0 && xS_0 < 1);
  REAL H_AS = kf_AS ? (REAL)1 : (REAL)0;

  REAL F_SA = FN(loading)(K, G, alfa, C_SA, eL, theta, e_n, tmp, xS_0);
  REAL Fs_SA = F_SA - Rs_SA;
  REAL F_SA_dot = F_SA - F_SA_0;
  int kf_SA = (F_SA < F_SA_0 && Fs_SA < 0 && xS_0 > 0);
  REAL H_SA = kf_SA ? (REAL)1 : (REAL)0;
  if (kf_SA && kf_AS) flag |= ORC_NR_BOTH;

  REAL xS;
  if (kf_SA || kf_AS) {
    /* return map by Newton-Raphson on (dh_AS, dh_SA), :389-465 */
    xS = xS_0;
    REAL dh_SA = 0, dh_AS = 0;
    int iter = 0;
    REAL RHS_AS = (F_AS - Rf_AS) * dh_AS + H_AS * F_AS_dot * ((REAL)1 - xS);
    REAL RHS_SA = (F_SA - Rf_SA) * dh_SA - H_SA * F_SA_dot * xS;
    REAL resi = RHS_AS * RHS_AS + RHS_SA * RHS_SA;  /* squared on entry, :403 */
    while (iter < iter_NR && resi > tole_NR) {
      iter = iter + 1;
      REAL m11 = -G_1 * dh_AS - (H_AS * F_AS_dot + H_AS * ((REAL)1 - xS) * G_1) + (F_AS - Rf_AS);
      REAL m12 = -G_1 * dh_AS - (H_AS * F_AS_dot + H_AS * ((REAL)1 - xS) * G_1);
      REAL m21 = -G_1 * dh_SA - (H_SA * F_SA_dot - H_SA * xS * G_1);
      REAL m22 = -G_1 * dh_SA - (H_SA * F_SA_dot - H_SA * xS * G_1) + (F_SA - Rf_SA);
      /* INV2x2 (:558-573) then matmul with the RHS */
      REAL det = m11 * m22 - m12 * m21;
      REAL r11 = m22 / det, r12 = -m12 / det, r21 = -m21 / det, r22 = m11 / det;
      REAL sol1 = r11 * RHS_AS + r12 * RHS_SA;
      REAL sol2 = r21 * RHS_AS + r22 * RHS_SA;
      dh_AS = dh_AS - sol1;
      dh_SA = dh_SA - sol2;
      xS = xS + dh_SA + dh_AS;
      F_AS = FN(loading)(K, G, alfa, C_AS, eL, theta, e_n, tmp, xS);
      F_AS_dot = F_AS - F_AS_0;
      F_SA = FN(loading)(K, G, alfa, C_SA, eL, theta, e_n, tmp, xS);
      F_SA_dot = F_SA - F_SA_0;
      RHS_AS = (F_AS - Rf_AS) * dh_AS + H_AS * F_AS_dot * ((REAL)1 - xS);
      RHS_SA = (F_SA - Rf_SA) * dh_SA - H_SA * F_SA_dot * xS;
      resi = SQRT(RHS_AS * RHS_AS + RHS_SA * RHS_SA);
    }
    if (iter >= iter_NR) {
      /* WARNING 2: reset to the previous state, :459-465 */
      flag |= ORC_NR_FAILED;
      F_AS = sdv[1];
      F_SA = sdv[2];
      xS = xS_0;
    } else {
      flag |= ORC_NR_CONVERGED;
    }
  } else {
    xS = xS_0;
  }

  /* clamp, :484 */
  xS = (xS < (REAL)1) ? xS : (REAL)1;
  xS = (xS > (REAL)0) ? xS : (REAL)0;

  /* Kirchhoff stress, :487-491 */
  REAL pv = K * (theta - (REAL)3 * alfa * eL * xS);
  REAL c1 = (REAL)2 * G * (e1 - eL * xS * d1);
  REAL c2 = (REAL)2 * G * (e2 - eL * xS * d2);
  REAL c3 = (REAL)2 * G * (e3 - eL * xS * d3);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      M3(tau, i, j) = pv * ((i == j) ? (REAL)1 : (REAL)0)
                    + c1 * (M3(n_A, j, 0) * M3(n_A, i, 0))
                    + c2 * (M3(n_A, j, 1) * M3(n_A, i, 1))
                    + c3 * (M3(n_A, j, 2) * M3(n_A, i, 2));

  sdv[0] = xS;
  sdv[1] = F_AS;
  sdv[2] = F_SA;
  if (eigfail) flag |= 8;
  return flag;
}

/* eval_sld_stress_model_160, :99-192 with flagt = 0: per Gauss point read
 * state slot 2 (TIME_N), evaluate, write slot 1 (ITER_K), S = F^-1 tau F^-T.
 * gpsdv is (3, pgaus, 2) column-major; returns OR of NR flags. */
int FN(orc_eval_law160)(int pgaus, const REAL props[18], REAL e_mart,
                        const REAL* gpgdi, const REAL* gptmp, REAL* gpsdv, REAL* gpstr)
{
  int flags = 0;
  (void)gptmp; /* the reference ignores the temperature (:105) */
  for (int g = 0; g < pgaus; ++g) {
    const REAL* F = gpgdi + 9 * g;
    REAL Finv[9], tau[9], sdv[3];
    FN(inv3x3)(F, Finv);
    for (int c = 0; c < 3; ++c) sdv[c] = gpsdv[c + 3 * g + 3 * pgaus];
    flags |= FN(orc_law160_kirchhoff)(props, e_mart, F, (REAL)0, sdv, tau);
    for (int c = 0; c < 3; ++c) gpsdv[c + 3 * g] = sdv[c];
    REAL* S = gpstr + 9 * g;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        REAL s = 0;
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l)
            s = s + M3(Finv, i, k) * M3(Finv, j, l) * M3(tau, k, l);
        M3(S, i, j) = s;
      }
  }
  return flags;
}

/* Batched law: n independent Gauss points, returns the second Piola stress
 * (as eval_sld_stress_model_160) and the new state. */
void FN(orc_law160_batch)(int64_t n, const REAL props[18], REAL e_mart, const REAL* F,
                          const REAL* tmp, const REAL* sdv_old, REAL* sdv_new,
                          REAL* pk2, int32_t* nr_flag)
{
  for (int64_t g = 0; g < n; ++g) {
    REAL Finv[9], tau[9], sdv[3];
    const REAL* Fg = F + 9 * g;
    FN(inv3x3)(Fg, Finv);
    for (int c = 0; c < 3; ++c) sdv[c] = sdv_old[3 * g + c];
    int fl = FN(orc_law160_kirchhoff)(props, e_mart, Fg, tmp ? tmp[g] : (REAL)0, sdv, tau);
    for (int c = 0; c < 3; ++c) sdv_new[3 * g + c] = sdv[c];
    REAL* S = pk2 + 9 * g;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        REAL s = 0;
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l)
            s = s + M3(Finv, i, k) * M3(Finv, j, l) * M3(tau, k, l);
        M3(S, i, j) = s;
      }
    if (nr_flag) nr_flag[g] = fl;
  }
}

/* Batched law with the algorithmic tangent (flagt = 1), following
 * eval_sld_stress_model_160 (sld_stress_model_160.f90:118-155, 170-191):
 * for every (i, j) the Kirchhoff stress at F + eps/2 (e_i e_j^T F +
 * e_j e_i^T F), eps = 1e-5 (:61), each from the TIME_N state (:130-131);
 * forward differences (:137); the correction of its Ref_D Eq. 68 with the
 * unperturbed Kirchhoff stress (:140-153, car_basis = identity); the pull-
 * back with F^-1 on all four indices (:170-191).  Outputs as
 * orc_law160_batch plus dds[i + 3j + 9k + 27l + 81g] = gpdds(i,j,k,l,g). */
void FN(orc_law160_tangent_batch)(int64_t n, const REAL props[18], REAL e_mart,
                                  const REAL* F, const REAL* tmp, const REAL* sdv_old,
                                  REAL* sdv_new, REAL* pk2, REAL* dds, int32_t* nr_flag)
{
  const REAL eps = (REAL)1.0e-5;
  for (int64_t g = 0; g < n; ++g) {
    const REAL* Fg = F + 9 * g;
    const REAL tg = tmp ? tmp[g] : (REAL)0;
    REAL Finv[9], tau[9], sdv[3], D[81];
    FN(inv3x3)(Fg, Finv);
    for (int c = 0; c < 3; ++c) sdv[c] = sdv_old[3 * g + c];
    const int fl = FN(orc_law160_kirchhoff)(props, e_mart, Fg, tg, sdv, tau);
    for (int c = 0; c < 3; ++c) sdv_new[3 * g + c] = sdv[c];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        REAL Fp[9], tp[9], sp[3];
        /* (e_i e_j^T F)(r, c) = delta_ri F(j, c) */
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) {
            const REAL a = (r == i ? M3(Fg, j, c) : (REAL)0) + (r == j ? M3(Fg, i, c) : (REAL)0);
            M3(Fp, r, c) = M3(Fg, r, c) + (REAL)0.5 * eps * a;
          }
        for (int c = 0; c < 3; ++c) sp[c] = sdv_old[3 * g + c];
        FN(orc_law160_kirchhoff)(props, e_mart, Fp, tg, sp, tp);
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l)
            D[i + 3 * j + 9 * k + 27 * l] = (M3(tp, k, l) - M3(tau, k, l)) / eps;
      }
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d)
            D[a + 3 * b + 9 * c + 27 * d] -= (REAL)0.5 *
                ((a == c ? M3(tau, d, b) : (REAL)0) + (c == b ? M3(tau, a, d) : (REAL)0) +
                 (a == d ? M3(tau, c, b) : (REAL)0) + (d == b ? M3(tau, a, c) : (REAL)0));
    REAL* out = dds + 81 * g;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) {
            REAL s = 0;
            for (int m = 0; m < 3; ++m)
              for (int nn = 0; nn < 3; ++nn)
                for (int p = 0; p < 3; ++p)
                  for (int q = 0; q < 3; ++q)
                    s = s + M3(Finv, i, m) * M3(Finv, j, nn) * M3(Finv, k, p) * M3(Finv, l, q) *
                                D[m + 3 * nn + 9 * p + 27 * q];
            out[i + 3 * j + 9 * k + 27 * l] = s;
          }
    REAL* S = pk2 + 9 * g;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        REAL s = 0;
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l)
            s = s + M3(Finv, i, k) * M3(Finv, j, l) * M3(tau, k, l);
        M3(S, i, j) = s;
      }
    if (nr_flag) nr_flag[g] = fl;
  }
}

/* ------------------------------------------------------------------------ */
/* HEX08 reference element                                                   */
/* ------------------------------------------------------------------------ */

/* gauss_qua, mod_quadrature_gauss.f90:2320-2386: nlocs = 2, points in the
 * order i (s) outer, j (t), k (z) inner; the abscissa is the 15-digit literal
 * the reference uses, weights 1. */
void FN(orc_hex8_gauss)(REAL posgp[24], REAL weigp[8])
{
  const REAL posgl[2] = {(REAL)-0.577350269189626, (REAL)0.577350269189626};
  int g = 0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k) {
        weigp[g] = (REAL)1 * (REAL)1 * (REAL)1;
        posgp[0 + 3 * g] = posgl[i];
        posgp[1 + 3 * g] = posgl[j];
        posgp[2 + 3 * g] = posgl[k];
        ++g;
      }
}

/* shape3 trilinear brick, mod_lagrange.f90:935-977.  deriv is (3,8). */
void FN(orc_hex8_shape)(REAL s, REAL t, REAL z, REAL shapf[8], REAL deriv[24])
{
  REAL sm = (REAL)0.5 * ((REAL)1 - s), tm = (REAL)0.5 * ((REAL)1 - t), zm = (REAL)0.5 * ((REAL)1 - z);
  REAL sq = (REAL)0.5 * ((REAL)1 + s), tp = (REAL)0.5 * ((REAL)1 + t), zp = (REAL)0.5 * ((REAL)1 + z);
  shapf[0] = sm * tm * zm; shapf[1] = sq * tm * zm; shapf[2] = sq * tp * zm; shapf[3] = sm * tp * zm;
  shapf[4] = sm * tm * zp; shapf[5] = sq * tm * zp; shapf[6] = sq * tp * zp; shapf[7] = sm * tp * zp;
  const REAL h = (REAL)0.5;
  REAL* d = deriv;
  d[0]  = -h * tm * zm; d[1]  = -h * sm * zm; d[2]  = -h * sm * tm;
  d[3]  =  h * tm * zm; d[4]  = -h * sq * zm; d[5]  = -h * sq * tm;
  d[6]  =  h * tp * zm; d[7]  =  h * sq * zm; d[8]  = -h * sq * tp;
  d[9]  = -h * tp * zm; d[10] =  h * sm * zm; d[11] = -h * sm * tp;
  d[12] = -h * tm * zp; d[13] = -h * sm * zp; d[14] =  h * sm * tm;
  d[15] =  h * tm * zp; d[16] = -h * sq * zp; d[17] =  h * sq * tm;
  d[18] =  h * tp * zp; d[19] =  h * sq * zp; d[20] =  h * sq * tp;
  d[21] = -h * tp * zp; d[22] =  h * sm * zp; d[23] =  h * sm * tp;
}

/* Jacobian, its inverse and gpcar = J^-T dN, jacobi.f90:172-219 (3D branch).
 * Returns det J. */
static REAL FN(jacobi3)(const REAL* elcod, const REAL* deriv, REAL* xjaci, REAL* gpcar)
{
  REAL xj[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < 8; ++k)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        M3(xj, i, j) = M3(xj, i, j) + elcod[i + 3 * k] * deriv[j + 3 * k];
  REAL t1 = M3(xj,1,1) * M3(xj,2,2) - M3(xj,2,1) * M3(xj,1,2);
  REAL t2 = -M3(xj,1,0) * M3(xj,2,2) + M3(xj,2,0) * M3(xj,1,2);
  REAL t3 = M3(xj,1,0) * M3(xj,2,1) - M3(xj,2,0) * M3(xj,1,1);
  REAL det = M3(xj,0,0) * t1 + M3(xj,0,1) * t2 + M3(xj,0,2) * t3;
  if (det == 0) return det;
  REAL den = (REAL)1 / det;
  M3(xjaci,0,0) = t1 * den;
  M3(xjaci,1,0) = t2 * den;
  M3(xjaci,2,0) = t3 * den;
  M3(xjaci,1,1) = ( M3(xj,0,0) * M3(xj,2,2) - M3(xj,2,0) * M3(xj,0,2)) * den;
  M3(xjaci,2,1) = (-M3(xj,0,0) * M3(xj,2,1) + M3(xj,0,1) * M3(xj,2,0)) * den;
  M3(xjaci,2,2) = ( M3(xj,0,0) * M3(xj,1,1) - M3(xj,1,0) * M3(xj,0,1)) * den;
  M3(xjaci,0,1) = (-M3(xj,0,1) * M3(xj,2,2) + M3(xj,2,1) * M3(xj,0,2)) * den;
  M3(xjaci,0,2) = ( M3(xj,0,1) * M3(xj,1,2) - M3(xj,1,1) * M3(xj,0,2)) * den;
  M3(xjaci,1,2) = (-M3(xj,0,0) * M3(xj,1,2) + M3(xj,1,0) * M3(xj,0,2)) * den;
  if (gpcar)
    for (int a = 0; a < 8; ++a)
      for (int i = 0; i < 3; ++i)
        gpcar[i + 3 * a] = M3(xjaci, 0, i) * deriv[0 + 3 * a]
                         + M3(xjaci, 1, i) * deriv[1 + 3 * a]
                         + M3(xjaci, 2, i) * deriv[2 + 3 * a];
  return det;
}

/* Minimum element length for the critical time step: elmlen.f90:75-146 at the
 * element centre (dercg), natural length 2 for the [-1,1]^3 brick, divided by
 * the element order 1 (sld_element_operations.f90:145). */
REAL FN(orc_hex8_celen)(const REAL elcod[24])
{
  REAL shapf[8], dercg[24], tragl[9];
  FN(orc_hex8_shape)((REAL)0, (REAL)0, (REAL)0, shapf, dercg);
  FN(jacobi3)(elcod, dercg, tragl, NULL);
  const REAL hnatu = 2;
  REAL hl[3];
  for (int i = 0; i < 3; ++i) {
    REAL enor0 = M3(tragl, i, 0) * M3(tragl, i, 0) + M3(tragl, i, 1) * M3(tragl, i, 1)
               + M3(tragl, i, 2) * M3(tragl, i, 2);
    hl[i] = hnatu / SQRT(enor0);
  }
  REAL tmp;
  if (hl[1] > hl[0]) { tmp = hl[1]; hl[1] = hl[0]; hl[0] = tmp; }
  if (hl[2] > hl[0]) { tmp = hl[2]; hl[2] = hl[0]; hl[0] = tmp; }
  if (hl[2] > hl[1]) { tmp = hl[2]; hl[2] = hl[1]; hl[1] = tmp; }
  return hl[2] / (REAL)1;
}

/* ------------------------------------------------------------------------ */
/* One element of the explicit scheme: sld_element_operations.f90:109-276    */
/* (gather done by the caller), sld_elmpre, law 160, PK1, sld_elmmat.       */
/* sdv_old/sdv_new are (3,8) slices of svegm (TIME_N / ITER_K slots).       */
/* nr_counts: [0] active, [1] failed, [2] both, [3] det<=0, [4] eig failures */
/* ------------------------------------------------------------------------ */
int FN(orc_element)(const REAL elcod[24], const REAL eldis[24], const REAL props[18],
                    REAL e_mart, REAL densi, REAL tmp, const REAL gravi[3],
                    const REAL* sdv_old, REAL* sdv_new, REAL elfint[24], REAL elfext[24],
                    REAL elmuu[8], REAL gppio[72], REAL* gpdet_min, int* nr_counts,
                    const REAL* elvel, REAL ray_alpha, REAL elrayl[24])
{
  REAL posgp[24], weigp[8];
  FN(orc_hex8_gauss)(posgp, weigp);
  for (int i = 0; i < 24; ++i) { elfint[i] = 0; elfext[i] = 0; }
  if (elrayl)
    for (int i = 0; i < 24; ++i) elrayl[i] = 0;
  for (int a = 0; a < 8; ++a) elmuu[a] = 0;

  for (int g = 0; g < 8; ++g) {
    REAL shapf[8], deriv[24], xjaci[9], gpcar[24];
    FN(orc_hex8_shape)(posgp[3 * g], posgp[3 * g + 1], posgp[3 * g + 2], shapf, deriv);
    REAL gpdet_ref = FN(jacobi3)(elcod, deriv, xjaci, gpcar);
    REAL volux = weigp[g] * gpdet_ref;

    /* F = I + sum_a u_a (x) gpcar_a, sld_elmpre.f90:149-162, 217-221 */
    REAL F[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        REAL s = 0;
        for (int a = 0; a < 8; ++a) s = s + eldis[i + 3 * a] * gpcar[j + 3 * a];
        M3(F, i, j) = s;
      }
    M3(F, 0, 0) = M3(F, 0, 0) + (REAL)1;
    M3(F, 1, 1) = M3(F, 1, 1) + (REAL)1;
    M3(F, 2, 2) = M3(F, 2, 2) + (REAL)1;
    /* det F as invmtx.f90 (3x3 branch); tracked for the J<=0 check */
    REAL t1 = M3(F,1,1) * M3(F,2,2) - M3(F,2,1) * M3(F,1,2);
    REAL t2 = -M3(F,1,0) * M3(F,2,2) + M3(F,2,0) * M3(F,1,2);
    REAL t3 = M3(F,1,0) * M3(F,2,1) - M3(F,2,0) * M3(F,1,1);
    REAL detF = M3(F,0,0) * t1 + M3(F,0,1) * t2 + M3(F,0,2) * t3;
    if (detF < *gpdet_min) *gpdet_min = detF;
    if (detF <= 0) nr_counts[3]++;

    /* law 160 with the PK2 pull-back (eval_sld_stress_model_160, :103-168) */
    REAL Finv[9], tau[9], S[9], sdv[3];
    FN(inv3x3)(F, Finv);
    for (int c = 0; c < 3; ++c) sdv[c] = sdv_old[c + 3 * g];
    int fl = FN(orc_law160_kirchhoff)(props, e_mart, F, tmp, sdv, tau);
    for (int c = 0; c < 3; ++c) sdv_new[c + 3 * g] = sdv[c];
    if (fl & (ORC_NR_CONVERGED | ORC_NR_FAILED)) nr_counts[0]++;
    if (fl & ORC_NR_FAILED) nr_counts[1]++;
    if (fl & ORC_NR_BOTH) nr_counts[2]++;
    if (fl & 8) nr_counts[4]++;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        REAL s = 0;
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l)
            s = s + M3(Finv, i, k) * M3(Finv, j, l) * M3(tau, k, l);
        M3(S, i, j) = s;
      }
    /* P = F S, sld_builtin_materials.f90:362-371 */
    REAL* P = gppio + 9 * g;
    for (int k = 0; k < 3; ++k)
      for (int j = 0; j < 3; ++j) {
        REAL s = 0;
        for (int i = 0; i < 3; ++i) s = s + M3(F, j, i) * M3(S, i, k);
        M3(P, j, k) = s;
      }

    /* internal/external forces, sld_elmmat.f90:137-166 (no prestress), and
     * the Rayleigh alpha force alpha v(g) N_a rho dV with the Gauss-point
     * velocity v(g) = sum_b N_b elvel_b (sld_elmpre.f90:114), sld_elmmat.f90:159-164 */
    REAL gpvel[3] = {0, 0, 0};
    if (elvel && ray_alpha > 0)
      for (int i = 0; i < 3; ++i)
        for (int b = 0; b < 8; ++b) gpvel[i] = gpvel[i] + elvel[i + 3 * b] * shapf[b];
    for (int a = 0; a < 8; ++a)
      for (int i = 0; i < 3; ++i) {
        REAL s = elfint[i + 3 * a];
        for (int j = 0; j < 3; ++j) s = s + M3(P, i, j) * gpcar[j + 3 * a] * volux;
        elfint[i + 3 * a] = s;
        elfext[i + 3 * a] = elfext[i + 3 * a] + (shapf[a] * densi * volux) * gravi[i];
        if (elrayl && elvel && ray_alpha > 0)
          elrayl[i + 3 * a] = elrayl[i + 3 * a] + ray_alpha * gpvel[i] * shapf[a] * densi * volux;
      }
    /* lumped mass, sld_elmmat.f90:199-209 */
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b)
        elmuu[a] = elmuu[a] + densi * volux * shapf[a] * shapf[b];
  }
  return 0;
}

/* sld_matrix explicit branch: zero the nodal arrays, colour-parallel element
 * loop (sld_elmope.f90:53-99), scatter-add (mod_matrix.f90:2327-2431 via
 * sld_element_operations.f90:239-256), Neumann nodal loads.  State is read
 * from slot TIME_N and written to slot ITER_K of sdv.  Any output pointer
 * may be NULL except rhsid and vmass.  dampi (2, nmate) holds the Rayleigh
 * coefficients (alpha, beta) of sld_reaphy.f90:1048-1055 (NULL: none); the
 * alpha force uses the nodal velocity veloc (the ITER_K velocity the element
 * loop gathers, sld_elmgat.f90:60) and enters rhsid and frxid only, not
 * finte or fexte (sld_elmmat.f90:170).  beta is not restated (see
 * orc_run_cd). */
int FN(orc_assemble)(int nelem, int npoin, const int32_t* lnods, const REAL* coord,
                     const REAL* displ, const int32_t* lmate, const REAL* props,
                     const REAL* e_mart, const REAL* densi, const REAL* tempe,
                     const REAL gravi[3], const REAL* fext_nodal, REAL fext_scale,
                     const int32_t* fixno, REAL* sdv, int ncolor,
                     const int32_t* color_ptr, const int32_t* color_elem,
                     int nthreads, REAL* rhsid, REAL* finte, REAL* fexte, REAL* frxid,
                     REAL* vmass, REAL* gpdet_min, int32_t* counters,
                     const REAL* veloc, const REAL* dampi)
{
  const REAL zero3[3] = {0, 0, 0};
  const REAL* grav = gravi ? gravi : zero3;
  for (int64_t i = 0; i < 3 * (int64_t)npoin; ++i) {
    rhsid[i] = 0;
    if (finte) finte[i] = 0;
    if (fexte) fexte[i] = 0;
    if (frxid) frxid[i] = 0;
  }
  for (int i = 0; i < npoin; ++i) vmass[i] = 0;
  int cnt[5] = {0, 0, 0, 0, 0};
  REAL dmin = (REAL)1e30;
  if (nthreads < 1) nthreads = 1;

  for (int ic = 0; ic < ncolor; ++ic) {
    int beg = color_ptr[ic], end = color_ptr[ic + 1];
#pragma omp parallel num_threads(nthreads)
    {
      int lcnt[5] = {0, 0, 0, 0, 0};
      REAL ldmin = (REAL)1e30;
#pragma omp for schedule(dynamic, 64)
      for (int kk = beg; kk < end; ++kk) {
        int e = color_elem[kk];
        const int32_t* ln = lnods + 8 * (int64_t)e;
        REAL elcod[24], eldis[24], elvel[24], elfint[24], elfext[24], elmuu[8], gppio[72];
        REAL elrayl[24];
        for (int a = 0; a < 8; ++a)
          for (int i = 0; i < 3; ++i) {     /* sld_elmgat.f90:53-63 */
            elcod[i + 3 * a] = coord[i + 3 * (int64_t)ln[a]];
            eldis[i + 3 * a] = displ[i + 3 * (int64_t)ln[a]];
            elvel[i + 3 * a] = veloc ? veloc[i + 3 * (int64_t)ln[a]] : (REAL)0;
          }
        int im = lmate ? lmate[e] : 0;
        REAL em = e_mart ? e_mart[im] : (REAL)0;
        REAL tmp = tempe ? tempe[e] : (REAL)0;
        REAL alpha = dampi ? dampi[2 * im] : (REAL)0;
        REAL* sd = sdv + 48 * (int64_t)e;
        FN(orc_element)(elcod, eldis, props + 18 * im, em, densi[im], tmp, grav,
                        sd + 24, sd, elfint, elfext, elmuu, gppio, &ldmin, lcnt,
                        veloc ? elvel : NULL, alpha, elrayl);
        for (int a = 0; a < 8; ++a) {
          int64_t p = ln[a];
          for (int i = 0; i < 3; ++i) {
            /* elrhs = elfext - elfint - elrayl_alpha, sld_elmmat.f90:170 */
            REAL elrhs = elfext[i + 3 * a] - elfint[i + 3 * a] - elrayl[i + 3 * a];
            rhsid[i + 3 * p] += elrhs;
            if (finte) finte[i + 3 * p] += elfint[i + 3 * a];
            if (fexte) fexte[i + 3 * p] += elfext[i + 3 * a];
            if (frxid && fixno && fixno[i + 3 * p] > 0) frxid[i + 3 * p] += elrhs;
          }
          vmass[p] += elmuu[a];
        }
      }
#pragma omp critical
      {
        for (int q = 0; q < 5; ++q) cnt[q] += lcnt[q];
        if (ldmin < dmin) dmin = ldmin;
      }
    }
  }
  if (fext_nodal)
    for (int64_t i = 0; i < 3 * (int64_t)npoin; ++i) {
      REAL f = fext_scale * fext_nodal[i];
      rhsid[i] += f;
      if (fexte) fexte[i] += f;
    }
  if (gpdet_min) *gpdet_min = dmin;
  if (counters) {
    counters[ORC_CNT_NR_ACTIVE] += cnt[0];
    counters[ORC_CNT_NR_FAILED] += cnt[1];
    counters[ORC_CNT_NR_BOTH] += cnt[2];
    counters[ORC_CNT_NEG_DET] += cnt[3];
    counters[ORC_CNT_EIG_FAIL] += cnt[4];
  }
  return 0;
}

/* sld_funbou.f90:99-140 for one degree of freedom.  tab is (4, npts):
 * column 0 the time, columns 1..3 the value per direction. */
REAL FN(orc_funbou)(int npts, const REAL* tab, int smooth, int idime, REAL cutim)
{
  REAL xretu = 0;
  for (int k = 0; k < npts - 1; ++k) {
    REAL t1 = tab[4 * k], t2 = tab[4 * (k + 1)];
    if (cutim >= t1 && cutim <= t2) {
      REAL p1 = tab[4 * k + 1 + idime], p2 = tab[4 * (k + 1) + 1 + idime];
      if (smooth) {
        REAL m = (cutim - t1) / (t2 - t1);
        xretu = p1 + (p2 - p1) * POW(m, (REAL)3) * ((REAL)10 - (REAL)15 * m + (REAL)6 * POW(m, (REAL)2));
      } else {
        REAL m = (p2 - p1) / (t2 - t1);
        xretu = p1 + m * (cutim - t1);
      }
      break;
    }
  }
  REAL tlast = tab[4 * (npts - 1)];
  if (cutim > tlast) xretu = tab[4 * (npts - 1) + 1 + idime] * cutim / tlast;
  return xretu;
}

/* Critical time step: min over elements of celen / c, with the law-160 sound
 * speed c = sqrt((lambda + 2 mu) / rho) (sld_velsnd.f90:117-124,
 * mod_sld_minle_time_step.f90:262-268). */
REAL FN(orc_critical_dt)(int nelem, const int32_t* lnods, const REAL* coord,
                         const int32_t* lmate, const REAL* props, const REAL* densi)
{
  REAL dtcri = (REAL)1e30;
  for (int e = 0; e < nelem; ++e) {
    REAL elcod[24];
    for (int a = 0; a < 8; ++a)
      for (int i = 0; i < 3; ++i) elcod[i + 3 * a] = coord[i + 3 * (int64_t)lnods[8 * (int64_t)e + a]];
    int im = lmate ? lmate[e] : 0;
    REAL young = props[18 * im], poiss = props[18 * im + 1];
    REAL lame1 = poiss * young / (((REAL)1 + poiss) * ((REAL)1 - (REAL)2 * poiss));
    REAL lame2 = young / ((REAL)2 * ((REAL)1 + poiss));
    REAL velas = SQRT((lame1 + (REAL)2 * lame2) / densi[im]);
    REAL dt = FN(orc_hex8_celen)(elcod) / velas;
    if (dt < dtcri) dtcri = dt;
  }
  return dtcri;
}

/* Time loop of the explicit central-difference scheme:
 *   Timste (setgts.f90:98)        cutim <- cutim + dtime
 *   Begste (sld_updbcs.f90:85-114) Dirichlet values at cutim
 *   sld_explicit (mod_sld_solution_methods.f90:101-223): predictor, element
 *     loop, a = r * (1/m) (solric.f90:305-320), corrector
 *   Endste (sld_updunk.f90:149-185) state slot TIME_N <- ITER_K.
 * bcfun[ipoin] selects the table of a node's fixed dofs (-1: value 0);
 * fext_nodal is scaled by column 1 of table load_fun (-1: not applied).
 * wit_hist receives displ at the nwit witness dofs after every step.
 * dampi (2, nmate, NULL: none): Rayleigh alpha damping with the velocity the
 * reference holds in veloc(ITER_K) during the element loop -- the step-
 * boundary velocity v_n in the central-difference scheme (written by the
 * previous corrector, :202), the predicted v_n + dt a_n in Tchamwa-Wielgosz
 * (:413).  The stiffness-proportional beta term (sld_elmmat.f90:172-190) is
 * not restated: no reference deck sets RAYBETA and its term is marked for
 * revision there; the CUDA library rejects beta > 0. */
int FN(orc_run_cd)(int nelem, int npoin, const int32_t* lnods, const REAL* coord,
                   const int32_t* lmate, const REAL* props, const REAL* e_mart,
                   const REAL* densi, const REAL* tempe, const int32_t* fixno,
                   const int32_t* bcfun, int nfun, const int32_t* fun_npts,
                   const int32_t* fun_smooth, const REAL* fun_tab,
                   const REAL* fext_nodal, int load_fun, int ncolor,
                   const int32_t* color_ptr, const int32_t* color_elem,
                   int nthreads, REAL dtime, int nsteps, REAL* cutim, REAL* displ,
                   REAL* veloc, REAL* accel, REAL* sdv, REAL* rhsid, int nwit,
                   const int32_t* wit_dof, REAL* wit_hist, int32_t* counters,
                   int scheme, REAL phi, const REAL* dampi)
{
  int64_t ndof = 3 * (int64_t)npoin;
  REAL* vtmp = (REAL*)malloc(sizeof(REAL) * ndof);
  REAL* vmass = (REAL*)malloc(sizeof(REAL) * npoin);
  int64_t* fun_off = (int64_t*)malloc(sizeof(int64_t) * (nfun > 0 ? nfun : 1));
  int64_t off = 0;
  for (int f = 0; f < nfun; ++f) { fun_off[f] = off; off += 4 * (int64_t)fun_npts[f]; }

  for (int step = 0; step < nsteps; ++step) {
    *cutim = *cutim + dtime;
    REAL t_end = *cutim + dtime;
    REAL t_mid = (REAL)0.5 * (*cutim + t_end);
    REAL c_pred = t_mid - *cutim, c_corr = t_end - t_mid;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int p = 0; p < npoin; ++p)
      for (int i = 0; i < 3; ++i) {
        int64_t k = i + 3 * (int64_t)p;
        REAL u;
        if (scheme == 1) {
          /* Tchamwa-Wielgosz predictor, mod_sld_solution_methods.f90:406-417 */
          vtmp[k] = veloc[k] + dtime * accel[k];
          u = displ[k] + dtime * veloc[k] + phi * (dtime * dtime) * accel[k];
        } else {
          vtmp[k] = veloc[k] + c_pred * accel[k];
          u = displ[k] + dtime * vtmp[k];
        }
        if (fixno[k] == 1) {
          int f = bcfun ? bcfun[p] : -1;
          u = (f >= 0) ? FN(orc_funbou)(fun_npts[f], fun_tab + fun_off[f], fun_smooth[f], i, *cutim)
                       : (REAL)0;
        }
        displ[k] = u;
      }
    REAL scale = 0;
    if (fext_nodal && load_fun >= 0)
      scale = FN(orc_funbou)(fun_npts[load_fun], fun_tab + fun_off[load_fun],
                             fun_smooth[load_fun], 0, *cutim);
    REAL dmin;
    FN(orc_assemble)(nelem, npoin, lnods, coord, displ, lmate, props, e_mart, densi, tempe,
                     NULL, (fext_nodal && load_fun >= 0) ? fext_nodal : NULL, scale, fixno,
                     sdv, ncolor, color_ptr, color_elem, nthreads, rhsid, NULL, NULL, NULL,
                     vmass, &dmin, counters, dampi ? (scheme == 1 ? vtmp : veloc) : NULL, dampi);
    int nonfin = 0;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(+ : nonfin)
    for (int p = 0; p < npoin; ++p) {
      REAL fact1 = (REAL)1 / vmass[p];
      for (int i = 0; i < 3; ++i) {
        int64_t k = i + 3 * (int64_t)p;
        REAL a = (REAL)0 + rhsid[k] * fact1;
        if (scheme == 1) {
          /* TW corrector, :504-515: prescribed dofs at rest */
          if (fixno[k] == 1) { accel[k] = 0; veloc[k] = 0; }
          else { accel[k] = a; veloc[k] = vtmp[k]; }
        } else {
          accel[k] = a;
          veloc[k] = vtmp[k] + c_corr * a;
        }
        if (!(a == a) || a - a != 0) nonfin++;
      }
    }
    if (counters) counters[ORC_CNT_NONFINITE] += nonfin;
    /* sld_updunk ITASK_ENDSTE: svegm(:,:,TIME_N) <- svegm(:,:,ITER_K) */
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < nelem; ++e)
      for (int q = 0; q < 24; ++q) sdv[48 * (int64_t)e + 24 + q] = sdv[48 * (int64_t)e + q];
    for (int w = 0; w < nwit; ++w) wit_hist[(int64_t)step * nwit + w] = displ[wit_dof[w]];
  }
  free(vtmp);
  free(vmass);
  free(fun_off);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Stress and strain post-processing: sld_calculate_pp_tensors.f90:40-145    */
/* with sld_calculate_pp_tensors_ielem.f90:110-150 (itask 3: Cauchy stress,  */
/* Green strain) and :186-218 (logarithmic strain).  Per Gauss point          */
/*   sigma(i,j) = sum_k F(i,k) P(j,k) / det F                                 */
/*   E(i,j)     = sum_k F(k,i) F(k,j) / 2 - delta_ij / 2                      */
/*   lnV(i,j)   = sum_k log(sqrt(|w_k|)) n_k(i) n_k(j),  (w, n) eig(F F^T)     */
/* projected to the nodes as sum_e sum_g N_a(g) dV(g) X / vmass_a, vmass the  */
/* volume-lumped mass of the kernel (mod_mass_matrix.f90:150-215, no          */
/* density); von Mises of the nodal Cauchy stress (3-D branch, :135-142).     */
/* The reference diagonalises b with maths_eigen_symmetric_matrix; the oracle */
/* uses the Householder + QL solver above.  P comes from the law evaluated    */
/* on the state slot `slot` of sdv (its new state is discarded), as the       */
/* element loop that produced gppio.  Voigt order xx yy zz yz xz xy           */
/* (nvgij_sld, sld_inivar.f90:568-579).  Outputs are (6, npoin) except seqvm  */
/* (npoin) and gp_sigma (6, 8, nelem); any output may be NULL.  The element-  */
/* loop fields of the same evaluation: gp_F = gpgdi and gp_P = gppio          */
/* (3, 3, 8, nelem) column-major, gp_det = det F (8, nelem), and volum[2] =   */
/* (sum dV, sum dV det F) as volum_sld (sld_elmpre.f90:242-264).             */
/* ------------------------------------------------------------------------ */
int FN(orc_postprocess)(int nelem, int npoin, const int32_t* lnods, const REAL* coord,
                        const REAL* displ, const int32_t* lmate, const REAL* props,
                        const REAL* e_mart, const REAL* tempe, const REAL* sdv, int slot,
                        REAL* caust, REAL* green, REAL* lepsi, REAL* seqvm, REAL* gp_sigma,
                        REAL* gp_F, REAL* gp_P, REAL* gp_det, REAL* volum)
{
  if (volum) { volum[0] = 0; volum[1] = 0; }
  static const int vi[6] = {0, 1, 2, 1, 0, 0}, vj[6] = {0, 1, 2, 2, 2, 1};
  REAL posgp[24], weigp[8];
  FN(orc_hex8_gauss)(posgp, weigp);
  REAL* acc = (REAL*)calloc(19 * (size_t)npoin, sizeof(REAL));   /* 6 + 6 + 6 + vmass */
  if (!acc) return -1;
  for (int e = 0; e < nelem; ++e) {
    const int32_t* ln = lnods + 8 * (int64_t)e;
    REAL elcod[24], eldis[24];
    for (int a = 0; a < 8; ++a)
      for (int i = 0; i < 3; ++i) {
        elcod[i + 3 * a] = coord[i + 3 * (int64_t)ln[a]];
        eldis[i + 3 * a] = displ[i + 3 * (int64_t)ln[a]];
      }
    const int im = lmate ? lmate[e] : 0;
    const REAL em = e_mart ? e_mart[im] : (REAL)0;
    const REAL tmp = tempe ? tempe[e] : (REAL)0;
    for (int g = 0; g < 8; ++g) {
      REAL shapf[8], deriv[24], xjaci[9], gpcar[24];
      FN(orc_hex8_shape)(posgp[3 * g], posgp[3 * g + 1], posgp[3 * g + 2], shapf, deriv);
      const REAL volux = weigp[g] * FN(jacobi3)(elcod, deriv, xjaci, gpcar);
      REAL F[9];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          REAL s = 0;
          for (int a = 0; a < 8; ++a) s = s + eldis[i + 3 * a] * gpcar[j + 3 * a];
          M3(F, i, j) = s + (i == j ? (REAL)1 : (REAL)0);
        }
      REAL t1 = M3(F,1,1) * M3(F,2,2) - M3(F,2,1) * M3(F,1,2);
      REAL t2 = -M3(F,1,0) * M3(F,2,2) + M3(F,2,0) * M3(F,1,2);
      REAL t3 = M3(F,1,0) * M3(F,2,1) - M3(F,2,0) * M3(F,1,1);
      const REAL detF = M3(F,0,0) * t1 + M3(F,0,1) * t2 + M3(F,0,2) * t3;
      /* P as the element loop forms it (law 160, PK2 pull-back, PK1) */
      REAL Finv[9], tau[9], S[9], P[9], st[3];
      FN(inv3x3)(F, Finv);
      for (int c = 0; c < 3; ++c) st[c] = sdv[48 * (int64_t)e + 24 * slot + 3 * g + c];
      FN(orc_law160_kirchhoff)(props + 18 * im, em, F, tmp, st, tau);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          REAL s = 0;
          for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) s = s + M3(Finv, i, k) * M3(Finv, j, l) * M3(tau, k, l);
          M3(S, i, j) = s;
        }
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) {
          REAL s = 0;
          for (int i = 0; i < 3; ++i) s = s + M3(F, j, i) * M3(S, i, k);
          M3(P, j, k) = s;
        }
      REAL sig[9], gre[9], b[9], Q[9], w[3], lep[9];
      const REAL gpinv = (REAL)1 / detF;
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
          REAL s = 0, r = 0, q = 0;
          for (int k = 0; k < 3; ++k) {
            s = s + gpinv * M3(F, i, k) * M3(P, j, k);
            r = r + (REAL)0.5 * (M3(F, k, i) * M3(F, k, j));
            q = q + M3(F, i, k) * M3(F, j, k);
          }
          M3(sig, i, j) = s;
          M3(gre, i, j) = r - (i == j ? (REAL)0.5 : (REAL)0);
          M3(b, i, j) = q;
        }
      int fail = 0;
      FN(orc_dsyevq3)(b, Q, w, &fail);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          REAL s = 0;
          for (int k = 0; k < 3; ++k) s = s + LOG(SQRT(FABS(w[k]))) * M3(Q, i, k) * M3(Q, j, k);
          M3(lep, i, j) = s;
        }
      for (int a = 0; a < 8; ++a) {
        REAL* ac = acc + 19 * (int64_t)ln[a];
        const REAL xmean = shapf[a] * volux;
        for (int v = 0; v < 6; ++v) {
          ac[v] += xmean * M3(sig, vi[v], vj[v]);
          ac[6 + v] += xmean * M3(gre, vi[v], vj[v]);
          ac[12 + v] += xmean * M3(lep, vi[v], vj[v]);
        }
        ac[18] += xmean;
      }
      if (gp_sigma)
        for (int v = 0; v < 6; ++v) gp_sigma[v + 6 * (g + 8 * (int64_t)e)] = M3(sig, vi[v], vj[v]);
      for (int k = 0; k < 9; ++k) {
        if (gp_F) gp_F[k + 9 * (g + 8 * (int64_t)e)] = F[k];
        if (gp_P) gp_P[k + 9 * (g + 8 * (int64_t)e)] = P[k];
      }
      if (gp_det) gp_det[g + 8 * (int64_t)e] = detF;
      if (volum) { volum[0] += volux; volum[1] += volux * detF; }
    }
  }
  for (int p = 0; p < npoin; ++p) {
    const REAL* ac = acc + 19 * (int64_t)p;
    const REAL dummr = (REAL)1 / ac[18];
    for (int v = 0; v < 6; ++v) {
      if (caust) caust[v + 6 * (int64_t)p] = dummr * ac[v];
      if (green) green[v + 6 * (int64_t)p] = dummr * ac[6 + v];
      if (lepsi) lepsi[v + 6 * (int64_t)p] = dummr * ac[12 + v];
    }
    if (seqvm) {
      REAL c[6];
      for (int v = 0; v < 6; ++v) c[v] = dummr * ac[v];
      seqvm[p] = SQRT((REAL)0.5 * ((c[0] - c[1]) * (c[0] - c[1]) + (c[1] - c[2]) * (c[1] - c[2]) +
                                   (c[2] - c[0]) * (c[2] - c[0]) +
                                   (REAL)6 * (c[3] * c[3] + c[4] * c[4] + c[5] * c[5])));
    }
  }
  free(acc);
  return 0;
}

#undef FN
#undef M3
