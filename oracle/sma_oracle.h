/*
 * sma_oracle.h -- CPU oracle for the explicit SMA (law 160) solid-mechanics step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path and
 * the timed CPU baseline; the product library never links or calls it.
 *
 * It restates, in plain C, the reference CPU path of Alya's solidz module for
 * HEX08 elements with constitutive law 160 (NITINOL).  Every routine cites the
 * reference file:line it follows (paths relative to the reference's src/).
 *
 * Parity pin: the law (compute_kirchoff_stress) is pinned against the
 * reference's own Gauss-point trace tests/sma_explicit/data1.dat: every one of
 * its 2300 martensite-transformation rows is reproduced to < 1e-9 from the
 * row's predecessor state (fixture tests/golden/data1_transitions.npz).  The
 * element loop, lumped mass and central-difference integrator have no
 * reference-computed golden output (the reference cannot be compiled without a
 * Fortran compiler); they are checked by analytic known answers: the constant-
 * strain patch test on a jittered mesh, zero force under a finite rigid
 * motion, lumped mass = rho V, and dt_crit = h / c on a regular mesh
 * (tests/test_oracle_element.py).
 *
 * Every entry point exists twice: *_f64 (double, the oracle) and *_f32
 * (float, used only for precision studies of an all-FP32 CPU run).
 *
 * Array conventions (Fortran column-major, as in the reference):
 *   3x3 tensors        T[i + 3*j]
 *   coord, displ, ...  x[idime + 3*ipoin]
 *   lnods              lnods[inode + 8*ielem]   (0-based node ids)
 *   state (svegm)      sdv[icomp + 3*igaus + 24*islot + 48*ielem]
 *                      slot 0 = ITER_K (new), slot 1 = TIME_N (old)
 */
#ifndef SMA_ORACLE_H
#define SMA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Newton-Raphson outcome of one law evaluation */
#define ORC_NR_NONE      0   /* elastic: no transformation active            */
#define ORC_NR_CONVERGED 1   /* return map converged                          */
#define ORC_NR_FAILED    2   /* 65 iterations reached: state reset (WARNING 2) */
#define ORC_NR_BOTH      4   /* both AS and SA active (WARNING 1), OR-ed in    */

/* Extended material record shared by all entry points.
 *   props[18*imate .. +17]  reference parameter vector parco_sld(1:18)
 *   e_mart[imate]           martensite Young's modulus (extension); <= 0 or
 *                           equal to props[0] means the reference law
 *   densi[imate]            density (mass scaling already applied)           */

#define ORC_DECL(T, S)                                                              \
  void orc_dsyevq3##S(const T A[9], T Q[9], T w[3], int* fail);                     \
  void orc_eigsrt##S(T d[3], T V[9]);                                               \
  int  orc_law160_kirchhoff##S(const T props[18], T e_mart, const T F[9], T tmp,    \
                               T sdv[3], T tau[9]);                                 \
  int  orc_eval_law160##S(int pgaus, const T props[18], T e_mart, const T* gpgdi,   \
                          const T* gptmp, T* gpsdv, T* gpstr);                      \
  void orc_law160_batch##S(int64_t n, const T props[18], T e_mart, const T* F,      \
                           const T* tmp, const T* sdv_old, T* sdv_new, T* pk2,      \
                           int32_t* nr_flag);                                       \
  void orc_law160_tangent_batch##S(int64_t n, const T props[18], T e_mart,          \
                                   const T* F, const T* tmp, const T* sdv_old,      \
                                   T* sdv_new, T* pk2, T* dds, int32_t* nr_flag);   \
  void orc_hex8_gauss##S(T posgp[24], T weigp[8]);                                  \
  void orc_hex8_shape##S(T s, T t, T z, T shapf[8], T deriv[24]);                   \
  T    orc_hex8_celen##S(const T elcod[24]);                                        \
  int  orc_element##S(const T elcod[24], const T eldis[24], const T props[18],      \
                      T e_mart, T densi, T tmp, const T gravi[3],                   \
                      const T* sdv_old, T* sdv_new, T elfint[24], T elfext[24],     \
                      T elmuu[8], T gppio[72], T* gpdet_min, int* nr_counts,        \
                      const T* elvel, T ray_alpha, T elrayl[24]);                   \
  int  orc_assemble##S(int nelem, int npoin, const int32_t* lnods, const T* coord,  \
                       const T* displ, const int32_t* lmate, const T* props,        \
                       const T* e_mart, const T* densi, const T* tempe,             \
                       const T gravi[3], const T* fext_nodal, T fext_scale,         \
                       const int32_t* fixno, T* sdv, int ncolor,                    \
                       const int32_t* color_ptr, const int32_t* color_elem,         \
                       int nthreads, T* rhsid, T* finte, T* fexte, T* frxid,        \
                       T* vmass, T* gpdet_min, int32_t* counters,                   \
                       const T* veloc, const T* dampi);                             \
  T    orc_funbou##S(int npts, const T* tab, int smooth, int idime, T cutim);       \
  T    orc_critical_dt##S(int nelem, const int32_t* lnods, const T* coord,          \
                          const int32_t* lmate, const T* props, const T* densi);    \
  int  orc_run_cd##S(int nelem, int npoin, const int32_t* lnods, const T* coord,    \
                     const int32_t* lmate, const T* props, const T* e_mart,         \
                     const T* densi, const T* tempe, const int32_t* fixno,          \
                     const int32_t* bcfun, int nfun, const int32_t* fun_npts,       \
                     const int32_t* fun_smooth, const T* fun_tab,                   \
                     const T* fext_nodal, int load_fun, int ncolor,                 \
                     const int32_t* color_ptr, const int32_t* color_elem,           \
                     int nthreads, T dtime, int nsteps, T* cutim, T* displ,         \
                     T* veloc, T* accel, T* sdv, T* rhsid, int nwit,                \
                     const int32_t* wit_dof, T* wit_hist, int32_t* counters,        \
                     int scheme, T phi, const T* dampi);                            \
  int  orc_postprocess##S(int nelem, int npoin, const int32_t* lnods, const T* coord,\
                          const T* displ, const int32_t* lmate, const T* props,     \
                          const T* e_mart, const T* tempe, const T* sdv, int slot,  \
                          T* caust, T* green, T* lepsi, T* seqvm, T* gp_sigma,      \
                          T* gp_F, T* gp_P, T* gp_det, T* volum);

ORC_DECL(double, _f64)
ORC_DECL(float, _f32)

/* Greedy first-fit element colouring: no two elements of one colour share a
 * node.  Returns the number of colours; color_ptr has ncolor+1 entries and
 * color_elem lists the elements of each colour in ascending order. */
int orc_color_elements(int nelem, int npoin, const int32_t* lnods,
                       int32_t* color_of, int32_t* color_ptr, int32_t* color_elem);

/* Counters written by orc_assemble / orc_run_cd (int32 slots) */
#define ORC_CNT_NR_ACTIVE   0   /* law evaluations with a transformation active  */
#define ORC_CNT_NR_FAILED   1   /* NR reached 65 iterations (state reset)         */
#define ORC_CNT_NR_BOTH     2   /* AS and SA active together (WARNING 1)          */
#define ORC_CNT_NEG_DET     3   /* Gauss points with det F <= 0                    */
#define ORC_CNT_EIG_FAIL    4   /* eigen solver reached 30 QL iterations          */
#define ORC_CNT_NONFINITE   5   /* non-finite nodal accelerations                 */
#define ORC_NCOUNTERS       8

#ifdef __cplusplus
}
#endif
#endif
