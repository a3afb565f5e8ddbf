/*
 * alya_sma.h -- C ABI of the B200 (sm_100a) explicit solid-mechanics step for
 * superelastic shape-memory alloys (Alya solidz, constitutive law 160).
 *
 * Plain pointers, sizes and int32 status codes only, so a Fortran caller binds
 * it with ISO_C_BINDING (bind(C)) and Python with ctypes.  Every entry point
 * returns SMA_OK (0) or a negative SMA_ERR_* code; sma_last_error() gives the
 * message.  Nothing aborts, nothing throws across the boundary.
 *
 * Array conventions are the reference's (Fortran column-major):
 *   lnods  (8, nelem)  int32, 0-based node ids          lnods[a + 8*e]
 *   coord, displ, veloc, accel, rhsid ... (3, npoin)     x[i + 3*p]
 *   fixno  (3, npoin)  int32 kfl_fixno_sld codes (1 = prescribed value)
 *   props  (18, nmate) parco_sld(1:18, imate), order of
 *          sld_stress_model_160.f90:263-279
 *   state  (3, 8, 2, nelem) svegm_sld(ielem)%a(1:3,1:8,1:2):
 *          slot 1 = ITER_K (new), slot 2 = TIME_N (old)
 *   3x3 tensors: 9 doubles column-major, T(i,j) at [i + 3*j]
 *
 * Threading: one host thread per context; calls are ordered on the
 * context's CUDA stream; a context is not thread-safe.
 */
#ifndef ALYA_SMA_H
#define ALYA_SMA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SMA_OK              0
#define SMA_ERR_ARG        -1   /* invalid argument or size                  */
#define SMA_ERR_CUDA       -2   /* CUDA runtime error                         */
#define SMA_ERR_NOMEM      -3   /* device allocation failed                   */
#define SMA_ERR_NODEVICE   -4   /* no sm_100 device                           */
#define SMA_ERR_STATE      -5   /* call out of sequence                       */

/* arithmetic of the element kinematics and the constitutive update */
#define SMA_PREC_FP64       0   /* all FP64 (the reference's arithmetic)       */
#define SMA_PREC_FP32       1   /* FP32 kinematics/law, FP64 return map,       */
                                /* FP64 force accumulation and integration    */

/* scatter-add of element forces into nodal arrays */
#define SMA_SCATTER_AUTO    0
#define SMA_SCATTER_ATOMIC  1   /* 8-lane reduce-scatter + FP64 atomics        */
#define SMA_SCATTER_COLOR   2   /* colour-by-colour plain read-modify-write    */
                                /* (deterministic; reference sld_elmope.f90:53-99) */

/* nodal fields for sma_set_nodal / sma_get_nodal */
#define SMA_FIELD_DISPL     0
#define SMA_FIELD_VELOC     1
#define SMA_FIELD_ACCEL     2
#define SMA_FIELD_RHSID     3   /* last assembled residual f_ext - f_int       */
#define SMA_FIELD_VMASS     4   /* lumped mass, (npoin) only; settable (> 0)   */

/* counters (sma_counters.c[k]) accumulated since creation / reset */
#define SMA_CNT_NR_ACTIVE   0   /* law evaluations with a transformation active */
#define SMA_CNT_NR_FAILED   1   /* return map hit 65 iterations (state reset)   */
#define SMA_CNT_NR_BOTH     2   /* AS and SA active together                    */
#define SMA_CNT_NEG_DET     3   /* Gauss points with det F <= 0                 */
#define SMA_CNT_NONFINITE   4   /* non-finite nodal accelerations               */
                            /* 5, 7: surrogate counters (sma_set_surrogate);
                             * 6: reserved, read as 0                        */
#define SMA_NCOUNTERS       8

typedef struct sma_ctx sma_ctx;

typedef struct {
  int32_t nelem, npoin;
  const int32_t* lnods;     /* (8, nelem)                                      */
  const double*  coord;     /* (3, npoin) reference coordinates                */
  const int32_t* lmate;     /* (nelem) material ids, or NULL (all material 0)  */
} sma_mesh_desc;

typedef struct {
  int32_t nmate;
  const double* props;      /* (18, nmate)                                     */
  const double* e_mart;     /* (nmate) martensite modulus (extension) or NULL  */
  const double* densi;      /* (nmate) density after mass scaling              */
  const double* tempe;      /* (nelem) temperature (extension) or NULL         */
  const double* dampi;      /* (2, nmate) Rayleigh (alpha, beta) or NULL:       */
                            /* RAYLEIGH_DAMPING of sld_reaphy.f90:1048-1055;    */
                            /* alpha (mass-proportional, sld_elmmat.f90:159-164) */
                            /* is applied; beta > 0 is rejected (SMA_ERR_ARG)   */
} sma_material_desc;

typedef struct {
  int32_t precision;        /* SMA_PREC_*                                      */
  int32_t scatter;          /* SMA_SCATTER_*                                   */
  int32_t device;           /* CUDA device ordinal                             */
  int32_t nfun;             /* number of DISCRETE time functions (<= 16)       */
  double  dtime;            /* time step                                       */
  const int32_t* fixno;     /* (3, npoin) or NULL                              */
  const int32_t* bcfun;     /* (npoin) time function of the fixed dofs or -1   */
  const int32_t* fun_npts;  /* (nfun) rows per table (<= 32)                   */
  const int32_t* fun_smooth;/* (nfun) 1 = SMOOTH step, 0 = linear              */
  const double*  fun_tab;   /* concatenated (4, npts) tables (t, vx, vy, vz)   */
  const double*  fext;      /* (3, npoin) nodal load at load factor 1, or NULL */
  int32_t load_fun;         /* table whose vx column scales fext, or -1        */
  int32_t block;            /* threads per element-kernel block, a multiple of  *
                             * 32 in [32, 256]; 0: one tile per block at 32    *
                             * (one material) or 128 (per-element materials),  *
                             * the pipelined variant at 256                    */
  int32_t scheme;           /* SMA_SCHEME_CD or SMA_SCHEME_TW                   */
  double  phitw;            /* Tchamwa-Wielgosz phi (0: the reference's 1.033) */
  int32_t variant;          /* element kernel: SMA_VARIANT_*                   */
} sma_run_desc;

/* element-loop kernels */
#define SMA_VARIANT_AUTO    0   /* PLAIN in both precisions (measured on B200)                */
#define SMA_VARIANT_PIPE    1   /* persistent blocks, next tile's gather in flight (cp.async) */
#define SMA_VARIANT_PLAIN   2   /* one tile per block; per-element materials that differ only */
                                /* in E_A, E_M, eL and thresholds as compact 8-word records   */
#define SMA_VARIANT_TABLE   3   /* one tile per block, per-element materials staged from the  */
                                /* full material table through shared memory                  */

/* explicit schemes (TIME_INTEGRATION of sld_reanut.f90:118-184) */
#define SMA_SCHEME_CD       0   /* central difference, mod_sld_solution_methods.f90:101-223 */
#define SMA_SCHEME_TW       1   /* Tchamwa-Wielgosz, mod_sld_solution_methods.f90:385-574   */

/* gpdet_min / ielem_min: the smallest det F <= 0 met by an element loop since
 * creation or reset (single precision) and its element in the caller's
 * numbering; 0.0 / -1 when none (sld_elmpre.f90:229-238) */
typedef struct {
  int64_t c[SMA_NCOUNTERS];
  double gpdet_min;
  int64_t ielem_min;
} sma_counters;

/* Context: copies the host arrays to the device and owns every device buffer.
 * Replaces the reference's Begrun-time set-up of solidz (sld_inivar, mass) */
int32_t sma_ctx_create(const sma_mesh_desc* mesh, const sma_material_desc* mat,
                       const sma_run_desc* run, sma_ctx** out);
int32_t sma_ctx_destroy(sma_ctx* ctx);

/* Step boundary: nsteps explicit central-difference steps, device resident,
 * replayed as CUDA graphs.  Replaces one pass of Timste/Begste/sld_explicit/
 * Endste per step (mod_sld_solution_methods.f90:101-223,
 * sld_updbcs.f90:85-114, sld_updunk.f90:149-185). */
int32_t sma_explicit_step(sma_ctx* ctx, int32_t nsteps);

/* Element-loop boundary with HOST buffers: displ (3,npoin) in; rhsid, finte,
 * fexte, frxid (3,npoin) and vmass (npoin) out (any output may be NULL
 * except rhsid).  Reads state slot TIME_N, writes slot ITER_K.  Replaces
 * sld_matrix(SLD_EXPLICIT_SCHEME) -> sld_elmope (sld_matrix.f90:161-171). */
int32_t sma_assemble(sma_ctx* ctx, const double* displ, double fext_scale,
                     double* rhsid, double* finte, double* fexte, double* frxid,
                     double* vmass);
/* Page-lock a caller-owned host array (e.g. Alya's displ and rhsid) once, so
 * sma_assemble's copies run asynchronously and overlap its element slabs;
 * unregister before freeing the array.  No counterpart in the reference
 * (its arrays never leave the host). */
int32_t sma_host_register(void* ptr, size_t bytes);
int32_t sma_host_unregister(void* ptr);
/* same with device pointers (no host copies), ordered on the context stream */
int32_t sma_assemble_device(sma_ctx* ctx, const double* d_displ, double fext_scale,
                            double* d_rhsid);
/* sld_updunk(ITASK_ENDSTE) for the state: slot TIME_N <- slot ITER_K */
int32_t sma_end_step(sma_ctx* ctx);

/* Stress and strain post-processing, HOST buffers, any of them NULL:
 * caust, green, lepsi (6,npoin): nodal Cauchy stress, Green-Lagrange strain
 * and logarithmic strain in Voigt order xx yy zz yz xz xy, each the
 * N_a dV-weighted average over the Gauss points around node a; seqvm (npoin)
 * the von Mises stress of the nodal Cauchy stress; gp_sigma (6,8,nelem) the
 * Cauchy stress per Gauss point.  The law is evaluated at the current
 * displacement from the state the last element loop started from (TIME_N if
 * none ran since the state was set), so after sma_explicit_step or
 * sma_assemble it reproduces that loop's stresses; the state is not changed.
 * Replaces sld_calculate_pp_tensors (sld_calculate_pp_tensors.f90:40-145)
 * with sld_calculate_pp_tensors_ielem (sld_calculate_pp_tensors_ielem.f90:
 * 110-150 and 186-218, itask 3 of sld_elmope). */
int32_t sma_postprocess(sma_ctx* ctx, double* caust, double* green, double* lepsi,
                        double* seqvm, double* gp_sigma);

/* Material-plugin boundary, batched: n independent Gauss points with device
 * pointers F (9n), tmp (n or NULL), sdv_old/sdv_new (3n), pk2 (9n),
 * nr_flag (n or NULL).  Replaces eval_sld_stress_model_160 with flagt = 0
 * (sld_stress_model_160.f90:36-195).  precision: SMA_PREC_*.
 * stream: a cudaStream_t or NULL for the default stream. */
int32_t sma_eval_law160(int64_t n, const double* props, double e_mart,
                        const double* d_F, const double* d_tmp,
                        const double* d_sdv_old, double* d_sdv_new, double* d_pk2,
                        int32_t* d_nr_flag, int32_t precision, void* stream);

/* The same plugin with flagt = 1 (FP64): also the algorithmic tangent
 * d_dds (81n), dds[i + 3j + 9k + 27l + 81g] = gpdds(i,j,k,l,igaus), from
 * eps = 1e-5 forward differences of the Kirchhoff stress, corrected and
 * pulled back with F^-1 (sld_stress_model_160.f90:118-155, 170-191). */
int32_t sma_eval_law160_tangent(int64_t n, const double* props, double e_mart,
                                const double* d_F, const double* d_tmp,
                                const double* d_sdv_old, double* d_sdv_new, double* d_pk2,
                                double* d_dds, int32_t* d_nr_flag, void* stream);

/* Element loop that allocates nothing.  No counterpart in the reference:
 * it exists for callers that cannot allocate device memory themselves
 * through the CUDA runtime (a Fortran host whose device arrays belong to an
 * OpenACC data region or a caller-side pool, code where a cudaMalloc would
 * synchronise the device or exceed the caller's memory budget).  Inputs and
 * outputs are caller-owned device pointers: lnods (8,nelem) with node ids in
 * [0,npoin), coord and displ (3,npoin), sdv (3,8,2,nelem) read at slot
 * TIME_N and written at slot ITER_K only (slot TIME_N is left bit for bit
 * as it was), rhsid (3,npoin) = f_ext - f_int of the element loop (no nodal
 * loads); props is a host array of 18 doubles.
 * The working set lives in one fixed device array compiled into the
 * library (about 7.5 MB, held by every GPU that loads the library until the
 * process exits), so meshes are limited to SMA_NOALLOC_MAX_ELEMS elements and
 * SMA_NOALLOC_MAX_NODES nodes; larger ones return SMA_ERR_ARG.  The first
 * call on a device does the set-up: it looks up that array's device address
 * and, since CUDA loads a library's device code on first use (lazy module
 * loading), it may load the module, which allocates and synchronises -- make
 * that first call during initialisation, before any stream capture on the
 * device.  Every call then validates lnods with one host synchronisation on
 * `stream`, so no call may be made while `stream` is being captured into a
 * CUDA graph.  All calls share the array, which keeps the previous call's
 * contents (the accumulators and counters are cleared by each call): calls
 * that overlap on the GPU (other streams, other host threads) race and must
 * be serialised by the caller.  Ordered on `stream` (NULL: default stream).
 * The return-map and det F <= 0 counters of the last call are read with
 * sma_noalloc_counters. */
#define SMA_NOALLOC_MAX_NODES 16384
#define SMA_NOALLOC_MAX_ELEMS 16384
int32_t sma_assemble_noalloc(int32_t nelem, int32_t npoin, const int32_t* d_lnods,
                             const double* d_coord, const double* d_displ,
                             const double* props, double e_mart, double* d_sdv,
                             double* d_rhsid, int32_t precision, void* stream);
/* Counters of the last sma_assemble_noalloc call on the current device (the
 * sld_detjac report of the reference, sld_elmpre.f90:229-238, and its
 * return-map warnings, sld_stress_model_160.f90:377-379, 459-465), read on
 * `stream` with one host synchronisation; ielem_min in the caller's element
 * numbering.  SMA_ERR_STATE before the first call on the device. */
int32_t sma_noalloc_counters(sma_counters* out, void* stream);

/* ---------------------------------------------------------------------------
 * Learned constitutive surrogate of law 160.  No counterpart in the
 * reference (its adjacent hook is the ANN framework's libtorch forward pass,
 * src/alya-ann/mod_ann_framework.f90:421-446, eval_r1); the law it stands in
 * for is compute_kirchoff_stress, sld_stress_model_160.f90:212-500.
 * Network 14 -> 64 -> 64 -> 64 -> 64 -> 13 (SiLU), BF16 weights with FP32
 * accumulation on the tensor cores, per Gauss point in the material frame
 * (tensors xx, yy, zz, xy, yz, xz):
 *   x: Green-Lagrange strain E (6), eps_tr_p = eL xS0 dev h / |dev h| (the
 *      previous step's transformation strain on the current deviatoric
 *      direction; h = E - E^2 + 4/3 E^3, ln U to O(E^4); 6), temperature,
 *      previous martensite fraction xS0
 *   y: (S - S_p) / E(xS0) (6), xS - xS0, eps_tr - eps_tr_p (6), where S is
 *      the second Piola-Kirchhoff stress, E(xS0) the Reuss modulus and S_p
 *      the law's elastic response on h and eps_tr_p:
 *      T_p = K (tr h - 3 alpha eL xS0) I + 2G (dev h - eps_tr_p),
 *      S_p = sym(C^-1 T_p), over E(xS0).
 * Parameters: SMA_SUR_NPARAM FP32 values, padded flat layout W1 [64][16],
 * b1 [64], W2, W3, W4 [64][64], b2, b3, b4 [64], W5 [16][64], b5 [16]
 * (W[o][i]: input i to output o; padding zero).  All pointers d_* are
 * device pointers the caller owns; calls are ordered on `stream`. */
#define SMA_SUR_NIN          14
#define SMA_SUR_NOUT         13
#define SMA_SUR_NPARAM       14608
#define SMA_SUR_IMAGE_BYTES  35904   /* tcgen05 weight image (swizzled BF16 + FP32 biases) */
typedef struct {
  float mu_x[SMA_SUR_NIN], sd_x[SMA_SUR_NIN];    /* input normalisation            */
  float mu_y[SMA_SUR_NOUT], sd_y[SMA_SUR_NOUT];  /* output normalisation           */
  float linv[SMA_SUR_NIN * SMA_SUR_NIN];         /* inverse Cholesky factor of the  *
                                                  * normalised inputs' covariance   *
                                                  * (lower, row-major): the         *
                                                  * out-of-envelope score is        *
                                                  * |linv xh| / sqrt(14)            */
  float lo_x[SMA_SUR_NIN], hi_x[SMA_SUR_NIN];    /* the training inputs' range: an  *
                                                  * input outside it scores +inf    */
} sma_sur_stats;

/* Training data: npath randomised load paths of the plain law (FP64,
 * material frame), nstep samples each, into d_x (npath*nstep, 14) and d_y
 * (npath*nstep, 13).  Per path: the material props (18) with e_mart, its
 * E_A, E_M, eL and four transformation stresses scaled by U(1-spread,
 * 1+spread); a temperature U(t_lo, t_hi); a random frame; nseg linear
 * segments between strain states with axial strain U(e_lo, e_hi), lateral
 * contraction U(0.3, 0.5) and shear N(0, shear). */
int32_t sma_sur_generate(int64_t npath, int32_t nstep, uint64_t seed, const double* props, double e_mart,
                         double spread, double t_lo, double t_hi, double e_lo, double e_hi, double shear,
                         int32_t nseg, float* d_x, float* d_y, void* stream);
/* One training pass over a batch of n samples on the tensor cores (BF16
 * mma.sync, FP32 accumulation): forward, backward and weight gradients of
 * the loss mean((yh_pred - yh)^2) over samples and outputs (normalised
 * outputs).  d_wb: BF16 weights (SMA_SUR_NPARAM, uint16 storage), d_w the
 * FP32 master (biases are read from it); d_grad (SMA_SUR_NPARAM) and
 * d_loss (1) are ADDED to (clear them first). */
int32_t sma_sur_train_step(const uint16_t* d_wb, const float* d_w, const sma_sur_stats* d_stats, int64_t n,
                           const float* d_x, const float* d_y, float* d_grad, float* d_loss, void* stream);
/* Adam (step t >= 1) on the FP32 master weights d_w with moments d_m, d_v;
 * writes the BF16 copy d_wb. */
int32_t sma_sur_adam(float* d_w, float* d_m, float* d_v, const float* d_grad, uint16_t* d_wb, float lr,
                     float b1, float b2, float eps, int32_t t, void* stream);
/* From the FP32 master: the BF16 copy (d_wb, or NULL) and the tcgen05
 * weight image (d_img, SMA_SUR_IMAGE_BYTES, 16-byte aligned, or NULL). */
int32_t sma_sur_pack(const float* d_w, uint16_t* d_wb, unsigned char* d_img, void* stream);
/* The network alone on the 5th-generation tensor cores (tcgen05.mma into
 * tensor memory, 128 points per tile): raw d_x (n, 14) -> raw d_y (n, 13)
 * and, if d_score is not NULL, the out-of-envelope score per point.
 * *d_status is set to 1 if a wait for the tensor cores ran out (never
 * expected; the results are then incomplete). */
int32_t sma_sur_forward(const unsigned char* d_img, const sma_sur_stats* d_stats, int64_t n, const float* d_x,
                        float* d_y, float* d_score, int32_t* d_status, void* stream);
/* The surrogate in a context's element loop (FP32 precision form, atomic
 * scatter, undamped; per-element materials as compact records), in place
 * of law 160's evaluation in sld_builtin_materials.f90:316-336.  Per Gauss
 * point the stress is E(xS0) (r + S_p): S_p the analytic part above,
 * following the strain every step, r a residual held per point (FP16).
 * The network (tcgen05 tensor cores) evaluates r on each tile of 16
 * elements every `period` steps (tiles staggered: one tile in `period` per
 * step) from the inputs the element loop stages for it; held between
 * evaluations, because a BF16 network evaluated every step moves in
 * quantisation steps the explicit scheme cannot carry.  The plain law
 * handles, and then holds its own residual for, a point with no residual
 * (the network's evaluation was refused: out-of-envelope score above
 * `gate`, or a predicted martensite increment above `xs_tol`, i.e. a point
 * the law would transform), an input outside the training inputs' range,
 * or loading functions of the surrogate's stress within `f_margin` (MPa,
 * the law's deviatoric units) of a transformation start (the law's
 * activation test, sld_stress_model_160.f90:351-374, compares loading
 * values one step apart and needs the exact stress there).  Accepted points
 * keep xS; the transformation strain is eL xS on the current strain
 * direction, as the law keeps it.  params: SMA_SUR_NPARAM host FP32
 * values, stats: host.  Switching on evaluates the network once on every
 * point at the TIME_N state and the current displacement, and so does
 * replacing either while it is on (sma_set_state, sma_checkpoint_load,
 * sma_set_nodal of the displacement); enable = 0 returns to the plain law.  A step with the surrogate launches the element
 * kernel and the network kernel.  Counters: slot 5 (SMA_CNT_SUR_FALLBACK)
 * Gauss points the plain law handled, slot 7 (SMA_CNT_SUR_OOD) network
 * evaluations its gates refused. */
#define SMA_CNT_SUR_FALLBACK 5
#define SMA_CNT_SUR_OOD      7
int32_t sma_set_surrogate(sma_ctx* ctx, const float* params, const sma_sur_stats* stats, double gate,
                          double xs_tol, double f_margin, int32_t period, int32_t enable);
/* 1 in *status if a wait of the surrogate's network kernel for the tensor
 * cores ran out since it was switched on (never expected), else 0. */
int32_t sma_surrogate_status(sma_ctx* ctx, int32_t* status);
/* Check of the bounded wait the network kernels use for their tensor-core
 * work (no counterpart in the reference): one kernel waits, `tries` tries
 * (1..2^20), for an mbarrier phase that nothing completes.  *status = 1
 * when the wait gave up, as it must; 0 would mean it saw a phase complete.
 * Synchronises the device. */
int32_t sma_sur_wait_check(int32_t tries, int32_t* status);

/* host <-> context data */
int32_t sma_set_nodal(sma_ctx* ctx, int32_t field, const double* host);

/* Partitioned meshes: one sub-mesh per GPU, nodes on the cut shared by the
 * sub-meshes.  sma_explicit_step in its parts, so the caller can sum the
 * residual of shared nodes between the element loop and the nodal update --
 * the reference's rhsmod -> pararr('SLX') exchange (sld_matrix.f90:274-281)
 * -- after summing their lumped mass once (sma_set_nodal SMA_FIELD_VMASS).
 * n steps: sma_step_prologue, then n times sma_step_elements, the exchange,
 * sma_step_nodes(last = final step).  The same kernels as sma_explicit_step,
 * without its graphs; witness and energy records stay per sub-mesh.
 * sma_gather/scatter_residual copy the residual rows of n nodes (device ids,
 * 0-based) to/from a device buffer (3, n) on the context stream. */
int32_t sma_step_prologue(sma_ctx* ctx);
int32_t sma_step_elements(sma_ctx* ctx);
/* sma_step_elements in element ranges [beg, end) (atomic scatter only):
 * first = 1 on a step's first range, last = 1 on its last, so the
 * interface elements can run first and their shared rows cross to the
 * neighbouring sub-meshes while the interior elements compute (the
 * reference sums the interface after the whole loop, pararr.f90:75-162). */
int32_t sma_step_elements_range(sma_ctx* ctx, int32_t beg, int32_t end, int32_t first, int32_t last);
int32_t sma_step_nodes(sma_ctx* ctx, int32_t last);
int32_t sma_gather_residual(sma_ctx* ctx, int32_t n, const int32_t* d_nodes, double* d_rows);
int32_t sma_scatter_residual(sma_ctx* ctx, int32_t n, const int32_t* d_nodes, const double* d_rows);
int32_t sma_get_nodal(sma_ctx* ctx, int32_t field, double* host);
int32_t sma_set_state(sma_ctx* ctx, const double* host_sdv);   /* (3,8,2,nelem) */
int32_t sma_get_state(sma_ctx* ctx, double* host_sdv);
int32_t sma_get_time(sma_ctx* ctx, double* cutim);
int32_t sma_set_time(sma_ctx* ctx, double cutim);
int32_t sma_get_counters(sma_ctx* ctx, sma_counters* out);
int32_t sma_reset_counters(sma_ctx* ctx);
/* Element-loop fields per Gauss point, HOST buffers, any of them NULL, from
 * the same evaluation as sma_postprocess: gpgdi = F and gppio = P = F S
 * (3,3,8,nelem) column-major, gpdet = det F (8,nelem), volum[2] = (reference
 * volume, deformed volume) summed over the mesh.  Replaces gpgdi_sld,
 * gppio_sld, dedef_sld and volum_sld(1:2) (sld_elmpre.f90:217-264,
 * sld_builtin_materials.f90:362-371). */
int32_t sma_gauss_fields(sma_ctx* ctx, double* gpgdi, double* gppio, double* gpdet, double* volum);
/* witness dofs: flat ids 3*p+i record the displacement of dof i of node p
 * after each step of the next sma_explicit_step call, ids 3*npoin + 3*p+i
 * its residual (f_ext - f_int; on prescribed dofs the reaction, as
 * frxid_sld); sma_get_witness copies (nsteps, nwit) values of the last call. */
int32_t sma_set_witness(sma_ctx* ctx, int32_t nwit, const int32_t* dofs, int32_t max_steps);
int32_t sma_get_witness(sma_ctx* ctx, double* host, int32_t* nsteps_out);

/* Energy balance of sld_energy (mod_sld_energy.f90:71-193), accumulated on
 * the device after every step while enabled: totals[5] = ALLIE (internal
 * work), ALLWK (external work), ALLKE (kinetic energy), ETOTA = ALLIE + ALLKE
 * - ALLWK, EENER.  Enabling records one row of the five per step of the next
 * sma_explicit_step calls (up to max_steps rows; sma_get_energy returns them
 * and the current totals).  Body forces are not part of the balance. */
int32_t sma_set_energy(sma_ctx* ctx, int32_t enable, int32_t max_steps);
int32_t sma_get_energy(sma_ctx* ctx, double* totals, double* hist, int32_t* nrows);

/* Checkpoint of the step-boundary state (the restart data of
 * mod_sld_arrays.f90:61-73: displacement, velocity, acceleration, svegm, and
 * the time), in a binary file; loading it into a context of the same mesh
 * and precision resumes bit for bit. */
int32_t sma_checkpoint_save(sma_ctx* ctx, const char* path);
int32_t sma_checkpoint_load(sma_ctx* ctx, const char* path);

/* critical time step of the mesh (mod_sld_minle_time_step.f90:262-268) */
int32_t sma_critical_dt(sma_ctx* ctx, double* dtcri);

/* the CUDA stream of the context (cudaStream_t) for callers that overlap */
void* sma_stream(sma_ctx* ctx);

/* Per-phase device timers (the reference's times(k)%ini/%add brackets,
 * sld_element_operations.f90:125-266 and sld_matrix.f90:159-173): while
 * enabled, sma_explicit_step launches kernels directly (no graph) with CUDA
 * events around each phase.  ms[0] element loop, ms[1] nodal update,
 * ms[2] whole steps; counts[] the launches timed in each. */
#define SMA_NTIMERS 3
int32_t sma_set_timing(sma_ctx* ctx, int32_t enable);
int32_t sma_get_timers(sma_ctx* ctx, double* ms, int64_t* counts);

/* Launch plan of the element loop: nrange element ranges [end[r-1], end[r])
 * (end[nrange-1] = nelem) each launched with block[r] threads per block (a
 * multiple of 32 in [32, 256]); nrange = 0 returns to one launch.  For
 * meshes concatenating specimens of different sizes (the ensemble), sorted
 * by size bucket, so each bucket gets the block its autotuning picked --
 * the counterpart of the pack/chunk choice of sld_elmope.f90:66-90
 * (par_omp_nelem_chunk, VECTOR_SIZE).  Atomic scatter, one-tile kernel. */
int32_t sma_set_launch_plan(sma_ctx* ctx, int32_t nrange, const int32_t* end, const int32_t* block);

/* kernel launches issued by this context since creation (all kernels) */
int64_t sma_kernel_launches(sma_ctx* ctx);

/* The element kernel's launch shape the context chose (no counterpart in the
 * reference, whose element loop has no launch): threads per block, the
 * SMA_VARIANT_* it runs, and 1 in *compact if per-element materials are read
 * as compact records. */
int32_t sma_launch_info(sma_ctx* ctx, int32_t* block, int32_t* variant, int32_t* compact);

const char* sma_last_error(void);
const char* sma_version(void);

#ifdef __cplusplus
}
#endif
#endif
