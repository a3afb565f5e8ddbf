// sma_capi.cu -- C ABI (include/alya_sma.h) of the B200 explicit SMA step:
// context set-up, device buffers, CUDA-graph step loop, host I/O.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "alya_sma.h"
#include "sma_kernels.cuh"
#include "sma_surrogate_elem.cuh"

using namespace sma;

namespace {

thread_local std::string g_err;

int32_t fail(int32_t code, const std::string& msg) {
  g_err = msg;
  return code;
}

// A failing runtime call also leaves its error as the thread's "last error";
// it is cleared here (non-sticky errors) so that a later launch check in
// another entry point does not report it a second time.
#define CU(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      cudaGetLastError();                                                          \
      return fail(SMA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    }                                                                              \
  } while (0)

template <typename P>
int32_t dalloc(P** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return SMA_OK;
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(SMA_ERR_NOMEM, std::string("cudaMalloc ") + std::to_string(bytes) + " bytes: " +
                                   cudaGetErrorString(e));
  }
  return SMA_OK;
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// per-element materials use compact records when a material is shared by at
// most this many elements on average (more sharing: the material table,
// which the caches hold)
constexpr int COMPACT_MAX_SHARING = 4;

// host restatement of sld_elmmat.f90:199-209 summed per node in element
// order (deterministic); FP64 geometry as jacobi.f90:172-219
void host_lumped_mass(int nelem, const int32_t* lnods, const double* coord,
                      const int32_t* lmate, const double* densi, std::vector<double>& vmass) {
  const double p = 0.577350269189626;
  double shp[8][8], der[8][24];
  for (int g = 0; g < 8; ++g) {
    const double s = (g & 4) ? p : -p, t = (g & 2) ? p : -p, z = (g & 1) ? p : -p;
    const double sm = 0.5 * (1 - s), sq = 0.5 * (1 + s), tm = 0.5 * (1 - t), tp = 0.5 * (1 + t);
    const double zm = 0.5 * (1 - z), zp = 0.5 * (1 + z), h = 0.5;
    const double N[8] = {sm * tm * zm, sq * tm * zm, sq * tp * zm, sm * tp * zm,
                         sm * tm * zp, sq * tm * zp, sq * tp * zp, sm * tp * zp};
    const double d[24] = {-h * tm * zm, -h * sm * zm, -h * sm * tm, h * tm * zm, -h * sq * zm, -h * sq * tm,
                          h * tp * zm,  h * sq * zm,  -h * sq * tp, -h * tp * zm, h * sm * zm, -h * sm * tp,
                          -h * tm * zp, -h * sm * zp, h * sm * tm,  h * tm * zp, -h * sq * zp, h * sq * tm,
                          h * tp * zp,  h * sq * zp,  h * sq * tp,  -h * tp * zp, h * sm * zp, h * sm * tp};
    std::memcpy(shp[g], N, sizeof N);
    std::memcpy(der[g], d, sizeof d);
  }
  for (int e = 0; e < nelem; ++e) {
    const int32_t* ln = lnods + 8 * (int64_t)e;
    const double rho = densi[lmate ? lmate[e] : 0];
    for (int g = 0; g < 8; ++g) {
      double xj[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int k = 0; k < 8; ++k)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) xj[i + 3 * j] += coord[i + 3 * (int64_t)ln[k]] * der[g][j + 3 * k];
      const double t1 = xj[4] * xj[8] - xj[5] * xj[7];
      const double t2 = -xj[1] * xj[8] + xj[2] * xj[7];
      const double t3 = xj[1] * xj[5] - xj[2] * xj[4];
      const double vol = 1.0 * (xj[0] * t1 + xj[3] * t2 + xj[6] * t3);
      for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) vmass[ln[a]] += rho * vol * shp[g][a] * shp[g][b];
    }
  }
}

// critical time step (elmlen.f90 at the centre, natural length 2;
// sld_velsnd.f90:117-124; mod_sld_minle_time_step.f90:262-268)
double host_critical_dt(int nelem, const int32_t* lnods, const double* coord,
                        const int32_t* lmate, const double* props, const double* e_mart,
                        const double* densi) {
  double dtcri = 1e300;
  const double sg[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                           {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  for (int e = 0; e < nelem; ++e) {
    const int32_t* ln = lnods + 8 * (int64_t)e;
    double xj[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 8; ++k)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) xj[i + 3 * j] += coord[i + 3 * (int64_t)ln[k]] * 0.125 * sg[k][j];
    const double t1 = xj[4] * xj[8] - xj[5] * xj[7];
    const double t2 = -xj[1] * xj[8] + xj[2] * xj[7];
    const double t3 = xj[1] * xj[5] - xj[2] * xj[4];
    const double det = xj[0] * t1 + xj[3] * t2 + xj[6] * t3;
    const double den = 1.0 / det;
    double tr[9];
    tr[0] = t1 * den; tr[1] = t2 * den; tr[2] = t3 * den;
    tr[4] = (xj[0] * xj[8] - xj[2] * xj[6]) * den;
    tr[5] = (-xj[0] * xj[5] + xj[3] * xj[2]) * den;
    tr[8] = (xj[0] * xj[4] - xj[1] * xj[3]) * den;
    tr[3] = (-xj[3] * xj[8] + xj[5] * xj[6]) * den;
    tr[6] = (xj[3] * xj[7] - xj[4] * xj[6]) * den;
    tr[7] = (-xj[0] * xj[7] + xj[1] * xj[6]) * den;
    double hmin = 1e300;
    for (int i = 0; i < 3; ++i) {
      const double en = tr[i] * tr[i] + tr[i + 3] * tr[i + 3] + tr[i + 6] * tr[i + 6];
      hmin = std::min(hmin, 2.0 / std::sqrt(en));
    }
    const int im = lmate ? lmate[e] : 0;
    double young = props[18 * im];
    if (e_mart && e_mart[im] > young) young = e_mart[im];
    const double poiss = props[18 * im + 1];
    const double lame1 = poiss * young / ((1.0 + poiss) * (1.0 - 2.0 * poiss));
    const double lame2 = young / (2.0 * (1.0 + poiss));
    const double velas = std::sqrt((lame1 + 2.0 * lame2) / densi[im]);
    dtcri = std::min(dtcri, hmin / velas);
  }
  return dtcri;
}

// first-fit greedy colouring of elements sharing a node (the reference
// colours the same graph, mod_parall_openmp.f90:557-708)
int host_color(int nelem, int npoin, const int32_t* lnods, std::vector<int32_t>& order,
               std::vector<int32_t>& cptr) {
  std::vector<int32_t> cnt(npoin + 1, 0), adj(8 * (size_t)nelem), col(nelem, -1);
  for (int64_t k = 0; k < 8 * (int64_t)nelem; ++k) cnt[lnods[k] + 1]++;
  for (int p = 0; p < npoin; ++p) cnt[p + 1] += cnt[p];
  std::vector<int32_t> pos(cnt.begin(), cnt.end());
  for (int e = 0; e < nelem; ++e)
    for (int a = 0; a < 8; ++a) adj[pos[lnods[8 * (int64_t)e + a]]++] = e;
  int ncol = 0;
  for (int e = 0; e < nelem; ++e) {
    uint64_t used = 0;
    for (int a = 0; a < 8; ++a) {
      const int p = lnods[8 * (int64_t)e + a];
      for (int k = cnt[p]; k < cnt[p + 1]; ++k) {
        const int c = col[adj[k]];
        if (c >= 0 && c < 64) used |= 1ull << c;
      }
    }
    int c = 0;
    while (c < 64 && ((used >> c) & 1)) ++c;
    if (c >= 64) return -1;
    col[e] = c;
    ncol = std::max(ncol, c + 1);
  }
  cptr.assign(ncol + 1, 0);
  for (int e = 0; e < nelem; ++e) cptr[col[e] + 1]++;
  for (int c = 0; c < ncol; ++c) cptr[c + 1] += cptr[c];
  std::vector<int32_t> fill(cptr.begin(), cptr.end() - 1);
  order.resize(nelem);
  for (int e = 0; e < nelem; ++e) order[fill[col[e]]++] = e;
  return ncol;
}

MatC make_mat(const double* pr, double e_mart, double densi) {
  MatC m;
  std::memset(&m, 0, sizeof m);
  const double E = pr[0], v = pr[1];
  m.eL = pr[2];
  m.alfa = pr[14];
  m.C_AS = pr[5];
  m.C_SA = pr[11];
  m.K = E / (3.0 - 6.0 * v);
  m.G = E / (2.0 + 2.0 * v);
  const double aux = std::sqrt(2.0 / 3.0) + m.alfa;
  m.Rf_AS = pr[4] * aux + m.C_AS * pr[6];
  m.Rs_AS = pr[3] * aux + m.C_AS * pr[7];
  m.Rf_SA = pr[10] * aux + m.C_SA * pr[12];
  m.Rs_SA = pr[9] * aux + m.C_SA * pr[13];
  m.G1 = (2.0 * m.G + 9.0 * (m.alfa * m.alfa) * m.K) * m.eL;
  m.EA = E;
  m.EM = (e_mart > 0.0) ? e_mart : E;
  m.nu = v;
  m.iEA = 1.0 / m.EA;
  m.iEM = 1.0 / m.EM;
  m.kK = 1.0 / (3.0 - 6.0 * v);
  m.kG = 1.0 / (2.0 + 2.0 * v);
  m.densi = densi;
  m.ext_E = (e_mart > 0.0 && e_mart != E) ? 1 : 0;
  return m;
}

}  // namespace

// the error text of the other translation units of the library (not exported)
extern "C" __attribute__((visibility("hidden"))) int32_t sma_set_error_(int32_t code, const char* msg) {
  return fail(code, msg ? msg : "");
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct sma_ctx {
  int dev = 0;
  cudaStream_t stream = nullptr;
  int prec = SMA_PREC_FP64;
  int scatter = SMA_SCATTER_ATOMIC;
  int block = 256;
  int variant = SMA_VARIANT_PIPE;
  int nsm = 148;                           // multiprocessors of the device
  int resident = 0;                        // resident pipelined blocks per SM (lazy)
  int nelem = 0, npoin = 0;
  int64_t npad = 0, sst = 0;
  int nmate = 0;
  // element order: internal position -> user element id (colour-sorted for
  // SMA_SCATTER_COLOR, identity otherwise)
  std::vector<int32_t> perm;
  std::vector<int32_t> cptr;   // colour ranges (one range if ATOMIC)
  // device
  int32_t* d_lnods = nullptr;
  int32_t* d_perm = nullptr;
  int32_t* d_lmate = nullptr;
  double* d_coord = nullptr;
  double* d_u = nullptr;
  double* d_vt = nullptr;
  double* d_v = nullptr;
  double* d_a = nullptr;
  double* d_f = nullptr;
  double* d_invm = nullptr;
  double* d_fext = nullptr;
  double* d_tempe = nullptr;
  uint8_t* d_flags = nullptr;
  int8_t* d_bcfun = nullptr;
  MatC* d_mats = nullptr;
  MatC mat0;                               // material 0, passed by value when nmate == 1
  void* d_matx = nullptr;                  // compact per-element records (T [nelem][MATX]) or null
  bool compact = false;                    // element kernel reads d_matx instead of d_mats
  // learned surrogate (FP32 form): weight image, statistics, eps_tr ping-pong
  // per-range element blocks (sma_set_launch_plan): plan_end[r] ends range r
  std::vector<int32_t> plan_end, plan_block;
  bool sur = false;
  unsigned char* d_sur_img = nullptr;
  sur::SurStats* d_sur_stats = nullptr;
  __half* d_rcache = nullptr;              // held stress residual, [6][sst] FP16 (NaN: none)
  float* d_xstage = nullptr;               // network inputs of the due tiles, [slot][14][128]
  int64_t xstage_slots = 0;
  int sur_period = 64;
  int* d_sur_ctr = nullptr;                // [1] status of the tensor-core waits
  float sur_gate = 3.0f, sur_xs_tol = 1e-3f, sur_margin = 10.0f;
  int sur_grid = 0;                        // persistent grid of the network kernel
  void* d_state[2] = {nullptr, nullptr};   // T [3][sst]
  int cur = 0;                             // state buffer holding TIME_N
  int last_in = -1;                        // state buffer the last element loop read (-1: none)
  double* d_pp_acc = nullptr;              // post-processing: [19][npad] nodal sums
  double* d_pp_out = nullptr;              //   (19, npoin) nodal results
  double* d_pp_gp = nullptr;               //   (6, 8, nelem) Gauss-point Cauchy stress
  double* d_gp_F = nullptr;                // sma_gauss_fields: gpgdi, gppio (72 nelem),
  double* d_gp_P = nullptr;                //   det F (8 nelem), volumes (2)
  double* d_gp_det = nullptr;
  double* d_gp_vol = nullptr;
  unsigned long long* d_cnt = nullptr;
  StepTime* d_ts = nullptr;
  FunTab* d_ft = nullptr;
  double* d_stage = nullptr;               // (3, npoin) staging for host I/O
  double* d_stage2 = nullptr;
  // witnesses
  int nwit = 0, wit_max = 0;
  int32_t* d_wdof = nullptr;
  double* d_whist = nullptr;
  int* d_wrow = nullptr;
  // scheme and energy balance
  int scheme = SMA_SCHEME_CD;
  bool energy = false;
  bool damp = false;                       // some material has Rayleigh alpha > 0
  int ehist_max = 0;
  double* d_uprev = nullptr;
  double* d_fintp = nullptr;
  double* d_fextp = nullptr;
  double* d_en = nullptr;                  // [4..8] totals (ALLIE, ALLWK, ALLKE, EENER, steps)
  double* d_epart = nullptr;               // per-block partial sums of the nodal kernel
  double* d_fray = nullptr;                // Rayleigh alpha nodal force (damped runs), SoA
  double* d_nodal = nullptr;               // one block: coord, u, f | vt, v, a (each SoA [3][npad])
  bool l2_window = false;                  // persisting-L2 window set on the stream
  // pipelined sma_assemble (atomic scatter, >= 2 slabs): slab bounds, node
  // prefixes needed / finished per slab, copy streams and their events
  std::vector<int> pl_e, pl_need, pl_final;
  cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
  std::vector<cudaEvent_t> pl_ev;          // 2 K + 1
  double* d_ehist = nullptr;
  int* d_erow = nullptr;
  // host copies
  std::vector<double> vmass;
  double dtcri = 0.0;
  double dtime = 0.0;
  bool has_load = false;
  double grav[3] = {0, 0, 0};
  // graphs: chunk of steps starting at state parity 0 / 1
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  int gchunk = 0;
  int64_t launches = 0;
  // phase timers
  bool timing = false;
  double tms[3] = {0, 0, 0};
  int64_t tcnt[3] = {0, 0, 0};
  std::vector<cudaEvent_t> evpool;
  std::vector<std::pair<int, std::pair<int, int>>> evmarks;  // (timer, (ev_begin, ev_end))
  size_t evnext = 0;
};

namespace {

// Persisting-L2 access window over [base, base + bytes) for the kernels of
// the context stream (and the graphs captured from it).  The carve-out is a
// limit of this process's context, sized to the window within the device's
// maxima; a device that refuses it (MIG, older parts) just runs without.
void set_l2_window(sma_ctx* c, void* base, size_t bytes, const cudaDeviceProp& prop) {
  if (prop.persistingL2CacheMaxSize <= 0 || prop.accessPolicyMaxWindowSize <= 0) return;
  // only when the arrays fit the carve-out whole: a larger window (2.0 M-element
  // cylinder, 146 MB) thrashed it and made both kernels ~2x slower on B200
  if (bytes > (size_t)prop.persistingL2CacheMaxSize || bytes > (size_t)prop.accessPolicyMaxWindowSize) return;
  const size_t win = std::min<size_t>(bytes, (size_t)prop.accessPolicyMaxWindowSize);
  size_t lim = std::min<size_t>(win, (size_t)prop.persistingL2CacheMaxSize);
  size_t cur = 0;
  if (cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize) == cudaSuccess && cur > lim) lim = cur;
  if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, lim) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  cudaStreamAttrValue at = {};
  at.accessPolicyWindow.base_ptr = base;
  at.accessPolicyWindow.num_bytes = win;
  at.accessPolicyWindow.hitRatio = std::min(1.0f, (float)lim / (float)win);
  at.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  at.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  if (cudaStreamSetAttribute(c->stream, cudaStreamAttributeAccessPolicyWindow, &at) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  c->l2_window = true;
}

// Rayleigh alpha velocity: what the reference's element loop gathers from
// veloc(ITER_K) -- inside a step the boundary velocity v_n (central
// difference) or the predicted v_n + dt a_n (Tchamwa-Wielgosz); outside a
// step (sma_assemble) the velocity field as set
const double* damp_velocity(const sma_ctx* c, bool stepping) {
  if (!c->damp) return nullptr;
  return (stepping && c->scheme == SMA_SCHEME_TW) ? c->d_vt : c->d_v;
}

template <typename T>
ElemArgs<T> elem_args(sma_ctx* c, int beg, int end, bool advance, bool stepping = false) {
  ElemArgs<T> a;
  a.vel = damp_velocity(c, stepping);
  a.lnods = c->d_lnods;
  a.coord = c->d_coord;
  a.u = c->d_u;
  a.f = c->d_f;
  a.lmate = c->d_lmate;
  a.mats = c->d_mats;
  a.tempe = c->d_tempe;
  a.sold = (const T*)c->d_state[c->cur];
  a.snew = (T*)c->d_state[c->cur ^ 1];
  a.cnt = c->d_cnt;
  a.ts = advance ? c->d_ts : nullptr;
  a.ft = c->d_ft;
  a.npad = c->npad;
  a.sst = c->sst;
  a.beg = beg;
  a.end = end;
  a.mat0 = c->mat0;
  a.matx = (const T*)c->d_matx;
  // one wave of the one-tile kernel: every SM's resident blocks of block / 8 elements
  a.pf_ahead = (c->variant == SMA_VARIANT_PIPE) ? 0 : (int64_t)c->nsm * c->resident * (c->block / 8);
  a.grav[0] = c->grav[0];
  a.grav[1] = c->grav[1];
  a.grav[2] = c->grav[2];
  a.has_grav = (c->grav[0] != 0.0 || c->grav[1] != 0.0 || c->grav[2] != 0.0);
  return a;
}

// kernel attributes and the persistent grid, fixed at context creation (not
// inside a stream capture)
// the element kernel of a variant, scatter and material layout
template <typename T>
using ElemKernel = void (*)(ElemArgs<T>);

// one-tile kernels: the narrow instance (tighter register cap, more warps)
// for blocks of up to ELEM_NARROW_BLOCK threads, the wide one above
template <typename T, bool ATOMIC, bool MATS>
ElemKernel<T> elem_kernel_v(bool pipe, int block) {
  if (pipe) return k_element_pipe<T, ATOMIC, MATS>;
  return block <= ELEM_NARROW_BLOCK ? k_element<T, ATOMIC, MATS, false, true> : k_element<T, ATOMIC, MATS>;
}

template <typename T>
ElemKernel<T> elem_kernel(const sma_ctx* c) {
  const bool pipe = c->variant == SMA_VARIANT_PIPE;
  const bool atomic = c->scatter != SMA_SCATTER_COLOR;
  const bool mats = c->d_lmate != nullptr;
  const int b = c->block;
  if (c->compact) {                                              // one-tile, undamped
    const bool narrow = b <= ELEM_NARROW_BLOCK;
    if (atomic) return narrow ? k_element<T, true, true, false, true, true> : k_element<T, true, true, false, false, true>;
    return narrow ? k_element<T, false, true, false, true, true> : k_element<T, false, true, false, false, true>;
  }
  if (c->damp) {                                                 // one-tile kernel only
    if (atomic) return mats ? k_element<T, true, true, true> : k_element<T, true, false, true>;
    return mats ? k_element<T, false, true, true> : k_element<T, false, false, true>;
  }
  if (atomic) return mats ? elem_kernel_v<T, true, true>(pipe, b) : elem_kernel_v<T, true, false>(pipe, b);
  return mats ? elem_kernel_v<T, false, true>(pipe, b) : elem_kernel_v<T, false, false>(pipe, b);
}

template <typename T>
size_t elem_smem(const sma_ctx* c) {
  const bool mats = c->d_lmate != nullptr && !c->compact;
  return c->variant == SMA_VARIANT_PIPE ? element_pipe_smem_bytes<T>(c->block, mats)
                                        : element_smem_bytes<T>(c->block, mats);
}

// The kernel's dynamic shared-memory limit is a per-process attribute shared
// by every context (and the no-alloc entry point): it is raised to what a
// 256-thread block needs and never lowered.
template <typename T>
int32_t init_element_launch_t(sma_ctx* c) {
  const int block = c->block;
  c->block = 256;
  const size_t smem256 = elem_smem<T>(c);
  c->block = block;
  const size_t smem = elem_smem<T>(c);
  const ElemKernel<T> k = elem_kernel<T>(c);
  CU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)std::max<size_t>(smem256, 48 * 1024)));
  CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->resident, k, block, smem));
  if (c->resident < 1) return fail(SMA_ERR_ARG, "element kernel does not fit on an SM at this block size");
  return SMA_OK;
}

sur::SurElemArgs sur_args(const sma_ctx* c) {
  sur::SurElemArgs s;
  s.stats = c->d_sur_stats;
  s.rcache = c->d_rcache;
  s.xstage = c->d_xstage;
  s.clock = c->d_ts;
  s.f_margin = c->sur_margin;
  s.period = c->sur_period;
  return s;
}

// the surrogate element kernel on elements [beg, end): one block per tile of
// 16 elements, tiles numbered over the whole mesh (a range that starts or
// ends inside a tile leaves the tile's other lanes idle)
int32_t launch_sur_range(sma_ctx* c, int beg, int end, bool advance, bool stepping) {
  if (end <= beg) return SMA_OK;
  ElemArgs<float> a = elem_args<float>(c, beg, end, advance, stepping);
  const sur::SurElemArgs s = sur_args(c);
  const unsigned grid = (unsigned)((end - 1) / sur::SUR_EPB - beg / sur::SUR_EPB + 1);
  if (c->compact) sur::k_element_sur<true><<<grid, sur::SUR_BLOCK, 0, c->stream>>>(a, s);
  else sur::k_element_sur<false><<<grid, sur::SUR_BLOCK, 0, c->stream>>>(a, s);
  c->launches++;
  CU(cudaGetLastError());
  return SMA_OK;
}

// the network on the tiles staged in residue class cls (< 0: the running
// step's due tiles, after the step's element ranges and before its nodal
// update, which moves the step time)
int32_t launch_sur_refresh(sma_ctx* c, int cls) {
  sur::RefreshArgs r;
  r.img = c->d_sur_img;
  r.stats = c->d_sur_stats;
  r.xstage = c->d_xstage;
  r.rcache = c->d_rcache;
  r.clock = c->d_ts;
  r.cnt = cls < 0 ? c->d_cnt : nullptr;                         // the switch-on passes count nothing
  r.status = c->d_sur_ctr + 1;
  r.sst = c->sst;
  r.nelem = c->nelem;
  r.cls = cls;
  r.period = c->sur_period;
  r.gate = c->sur_gate;
  r.xs_tol = c->sur_xs_tol;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(c->xstage_slots, c->sur_grid));
  sur::k_sur_refresh<<<grid, sur::SUR_BLOCK, sur::mlp_smem_bytes(), c->stream>>>(r);
  c->launches++;
  CU(cudaGetLastError());
  return SMA_OK;
}

// the held residual of every point from the network at the TIME_N state and
// the current displacement, one residue class of tiles at a time: at
// switch-on, and when the caller replaces the state or the displacement
int32_t sur_init_residuals(sma_ctx* c) {
  CU(cudaMemsetAsync(c->d_rcache, 0xff, 6 * (size_t)c->sst * sizeof(__half), c->stream));   // NaN: none held
  ElemArgs<float> a = elem_args<float>(c, 0, c->nelem, false, false);
  const sur::SurElemArgs sa = sur_args(c);
  const int64_t ntiles = ceil_div(c->nelem, sur::SUR_EPB);
  for (int cls = 0; cls < c->sur_period && cls < ntiles; ++cls) {
    const unsigned grid = (unsigned)ceil_div(ntiles - cls, c->sur_period);
    if (c->compact) sur::k_sur_stage<true><<<grid, sur::SUR_BLOCK, 0, c->stream>>>(a, sa, cls);
    else sur::k_sur_stage<false><<<grid, sur::SUR_BLOCK, 0, c->stream>>>(a, sa, cls);
    c->launches++;
    CU(cudaGetLastError());
    int32_t rc = launch_sur_refresh(c, cls);
    if (rc) return rc;
  }
  return SMA_OK;
}

// the element loop by the launch plan: range r with its own block size (the
// one-tile kernel, narrow or wide instance by block)
template <typename T>
int32_t launch_plan_t(sma_ctx* c, bool advance) {
  int beg = 0;
  const int saved = c->block;
  for (size_t r = 0; r < c->plan_end.size(); ++r) {
    const int end = c->plan_end[r];
    if (end > beg) {
      c->block = c->plan_block[r];
      ElemArgs<T> a = elem_args<T>(c, beg, end, advance && beg == 0, advance);
      const unsigned grid = (unsigned)ceil_div(end - beg, c->block / 8);
      elem_kernel<T>(c)<<<grid, c->block, elem_smem<T>(c), c->stream>>>(a);
      c->launches++;
    }
    beg = end;
  }
  c->block = saved;
  CU(cudaGetLastError());
  return SMA_OK;
}

template <typename T>
int32_t launch_elements_t(sma_ctx* c, bool advance) {
  const int nrange = (int)c->cptr.size() - 1;
  const int epb = c->block / 8;
  if (c->resident == 0) return fail(SMA_ERR_STATE, "element launch not initialised");
  if constexpr (sizeof(T) == 4) {
    if (c->sur) {
      c->last_in = c->cur;
      const int32_t rc = launch_sur_range(c, 0, c->nelem, advance, advance);
      return (rc || !advance) ? rc : launch_sur_refresh(c, -1);
    }
  }
  if (!c->plan_end.empty()) {
    c->last_in = c->cur;
    return launch_plan_t<T>(c, advance);
  }
  c->last_in = c->cur;
  const ElemKernel<T> kern = elem_kernel<T>(c);
  const size_t smem = elem_smem<T>(c);
  for (int r = 0; r < nrange; ++r) {
    const int beg = c->cptr[r], end = c->cptr[r + 1];
    if (end <= beg) continue;
    ElemArgs<T> a = elem_args<T>(c, beg, end, advance && r == 0, advance);
    const int64_t ntiles = ceil_div(end - beg, epb);
    const unsigned grid = c->variant == SMA_VARIANT_PIPE
                              ? (unsigned)std::min<int64_t>(ntiles, (int64_t)c->nsm * c->resident)
                              : (unsigned)ntiles;
    kern<<<grid, c->block, smem, c->stream>>>(a);
    c->launches++;
  }
  CU(cudaGetLastError());
  return SMA_OK;
}

int32_t launch_elements(sma_ctx* c, bool advance) {
  return c->prec == SMA_PREC_FP32 ? launch_elements_t<float>(c, advance)
                                  : launch_elements_t<double>(c, advance);
}

// one element range [beg, end) of an atomic-scatter context outside a step
template <typename T>
int32_t launch_element_range_t(sma_ctx* c, int beg, int end) {
  if (end <= beg) return SMA_OK;
  if constexpr (sizeof(T) == 4)
    if (c->sur) return launch_sur_range(c, beg, end, false, false);
  const int epb = c->block / 8;
  ElemArgs<T> a = elem_args<T>(c, beg, end, false, false);
  const int64_t ntiles = ceil_div(end - beg, epb);
  const unsigned grid = c->variant == SMA_VARIANT_PIPE
                            ? (unsigned)std::min<int64_t>(ntiles, (int64_t)c->nsm * c->resident)
                            : (unsigned)ntiles;
  elem_kernel<T>(c)<<<grid, c->block, elem_smem<T>(c), c->stream>>>(a);
  c->launches++;
  CU(cudaGetLastError());
  return SMA_OK;
}

// Slab plan of the pipelined element-loop boundary (atomic scatter): K
// element slabs; before slab s runs, nodes [0, need[s]) must be on the
// device; after it, the residual of nodes [0, final[s]) is complete (no later
// slab touches them).  Meshes numbered with locality (structured, O-grid,
// concatenated specimens) give growing prefixes, so the copies in and out
// overlap the element work; a mesh without it degrades to need = npoin.
void plan_pipeline(sma_ctx* c, const int32_t* ln) {
  const int K = (int)std::min<int64_t>(8, std::max<int64_t>(1, c->nelem / 16384));
  c->pl_e.assign(K + 1, 0);
  c->pl_need.assign(K, 0);
  c->pl_final.assign(K, 0);
  if (K < 2) return;
  for (int s = 0; s <= K; ++s) c->pl_e[s] = (int)((int64_t)c->nelem * s / K);
  std::vector<int8_t> last(c->npoin, -1);
  int hi = 0;
  for (int s = 0; s < K; ++s) {
    for (int64_t k = 8 * (int64_t)c->pl_e[s]; k < 8 * (int64_t)c->pl_e[s + 1]; ++k) {
      hi = std::max(hi, ln[k] + 1);
      last[ln[k]] = (int8_t)s;
    }
    c->pl_need[s] = hi;
  }
  c->pl_need[K - 1] = c->npoin;                 // every node converted by the last slab
  std::vector<int> first_bad(K, c->npoin);      // first node a later slab still touches
  for (int p = c->npoin - 1; p >= 0; --p)
    for (int s = 0; s < last[p]; ++s) first_bad[s] = p;
  for (int s = 0; s < K; ++s) c->pl_final[s] = std::min(first_bad[s], c->pl_need[s]);
  c->pl_final[K - 1] = c->npoin;
}

// sma_assemble's residual path, pipelined over the slab plan: H2D of the
// node prefix a slab needs on one copy stream, conversion + element slab +
// finished-node output on the context stream, D2H of finished nodes on a
// second copy stream
template <typename T>
int32_t assemble_pipelined_t(sma_ctx* c, const double* displ, double scale, double* rhsid) {
  const int K = (int)c->pl_need.size();
  cudaEvent_t* ev_in = c->pl_ev.data();
  cudaEvent_t* ev_out = c->pl_ev.data() + K;
  cudaEvent_t ev_start = c->pl_ev[2 * K];
  c->last_in = c->cur;
  CU(cudaEventRecord(ev_start, c->stream));            // after all earlier work on the stream
  CU(cudaStreamWaitEvent(c->s_h2d, ev_start, 0));
  int64_t copied = 0, sent = 0;
  const size_t row = 3 * sizeof(double);
  for (int s = 0; s < K; ++s) {
    const int64_t need = c->pl_need[s];
    if (need > copied) {
      CU(cudaMemcpyAsync(c->d_stage + 3 * copied, displ + 3 * copied, (need - copied) * row,
                         cudaMemcpyHostToDevice, c->s_h2d));
      CU(cudaEventRecord(ev_in[s], c->s_h2d));
      CU(cudaStreamWaitEvent(c->stream, ev_in[s], 0));
      k_assemble_in<<<(unsigned)ceil_div(need - copied, 256), 256, 0, c->stream>>>(
          c->d_stage, c->d_u, c->d_f, c->d_fext, c->d_flags, scale, copied, need, c->npad);
      c->launches++;
      copied = need;
    }
    int32_t rc = launch_element_range_t<T>(c, c->pl_e[s], c->pl_e[s + 1]);
    if (rc) return rc;
    const int64_t fin = c->pl_final[s];
    if (fin > sent) {
      k_rhsid_out<<<(unsigned)ceil_div(fin - sent, 256), 256, 0, c->stream>>>(c->d_f, c->d_stage2, sent,
                                                                              fin, c->npad);
      c->launches++;
      CU(cudaEventRecord(ev_out[s], c->stream));
      CU(cudaStreamWaitEvent(c->s_d2h, ev_out[s], 0));
      CU(cudaMemcpyAsync(rhsid + 3 * sent, c->d_stage2 + 3 * sent, (fin - sent) * row,
                         cudaMemcpyDeviceToHost, c->s_d2h));
      sent = fin;
    }
  }
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(c->s_d2h));
  CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

// post-processing element pass: the law from the state the last element
// loop read (TIME_N if none ran since the state was set), outputs in p
template <typename T>
int32_t launch_postproc_t(sma_ctx* c, PostArgs p) {
  const int slot = c->last_in >= 0 ? c->last_in : c->cur;
  ElemArgs<T> a = elem_args<T>(c, 0, c->nelem, false);
  a.sold = (const T*)c->d_state[slot];
  a.snew = nullptr;
  p.perm = c->d_perm;
  const int block = 128;
  const bool mats = c->d_lmate != nullptr;
  const size_t smem = postproc_smem_bytes<T>(block, mats);      // below the 48 KB default
  const unsigned grid = (unsigned)ceil_div(c->nelem, block / 8);
  if (mats) k_postproc<T, true><<<grid, block, smem, c->stream>>>(a, p);
  else k_postproc<T, false><<<grid, block, smem, c->stream>>>(a, p);
  c->launches++;
  CU(cudaGetLastError());
  return SMA_OK;
}

NodalArgs nodal_args(sma_ctx* c) {
  NodalArgs a;
  a.u = c->d_u;
  a.vt = c->d_vt;
  a.v = c->d_v;
  a.acc = c->d_a;
  a.f = c->d_f;
  a.invm = c->d_invm;
  a.flags = c->d_flags;
  a.bcfun = c->d_bcfun;
  a.fext = c->d_fext;
  a.ts = c->d_ts;
  a.cnt = c->d_cnt;
  a.uprev = c->d_uprev;
  a.fint_prev = c->d_fintp;
  a.fext_prev = c->d_fextp;
  a.en_step = c->d_epart;
  a.fray = (c->damp && c->energy) ? c->d_fray : nullptr;
  a.store_v = (c->damp && c->scheme == SMA_SCHEME_CD) ? 1 : 0;
  a.npoin = c->npoin;
  a.npad = c->npad;
  return a;
}

// the Rayleigh alpha force alone into d_fray (energy balance, finte)
int32_t launch_rayleigh(sma_ctx* c, const double* vel) {
  CU(cudaMemsetAsync(c->d_fray, 0, 3 * (size_t)c->npad * sizeof(double), c->stream));
  k_rayleigh<<<(unsigned)ceil_div(c->nelem, 128), 128, 0, c->stream>>>(
      c->d_lnods, c->d_coord, vel, c->d_lmate, c->d_mats, c->mat0, c->nelem, c->npad, c->d_fray);
  c->launches++;
  CU(cudaGetLastError());
  return SMA_OK;
}

template <int MODE>
void launch_nodal_mode(sma_ctx* c, unsigned grid, const NodalArgs& a) {
  const bool en = c->energy && MODE >= 1;
  if (c->scheme == SMA_SCHEME_TW) {
    if (en) k_nodal<MODE, SCHEME_TW, true><<<grid, 256, 0, c->stream>>>(a);
    else k_nodal<MODE, SCHEME_TW, false><<<grid, 256, 0, c->stream>>>(a);
  } else {
    if (en) k_nodal<MODE, SCHEME_CD, true><<<grid, 256, 0, c->stream>>>(a);
    else k_nodal<MODE, SCHEME_CD, false><<<grid, 256, 0, c->stream>>>(a);
  }
}

int32_t launch_nodal(sma_ctx* c, int mode) {
  const unsigned grid = (unsigned)ceil_div(c->npoin, 256);
  NodalArgs a = nodal_args(c);
  if (mode == 0) launch_nodal_mode<0>(c, grid, a);
  else if (mode == 1) launch_nodal_mode<1>(c, grid, a);
  else launch_nodal_mode<2>(c, grid, a);
  c->launches++;
  CU(cudaGetLastError());
  if (c->energy && mode >= 1) {
    k_energy_finalize<<<1, 256, 0, c->stream>>>(c->d_epart, (int)ceil_div(c->npoin, 256), c->d_en + 4,
                                                 c->d_ehist, c->d_erow,
                                               c->ehist_max);
    c->launches++;
    CU(cudaGetLastError());
  }
  return SMA_OK;
}

int32_t launch_witness(sma_ctx* c) {
  if (c->nwit <= 0) return SMA_OK;
  k_witness<<<1, 128, 0, c->stream>>>(c->d_u, c->d_f, c->npoin, c->npad, c->d_wdof, c->nwit,
                                      c->d_whist, c->d_wrow, c->wit_max);
  c->launches++;
  CU(cudaGetLastError());
  return SMA_OK;
}

// one interior step: element loop (advancing time) + fused nodal update
int32_t issue_step(sma_ctx* c, int nodal_mode) {
  int32_t rc = launch_elements(c, true);
  if (rc) return rc;
  c->cur ^= 1;   // the state written by this step is TIME_N of the next
  // u holds u_k until the nodal kernel predicts u_{k+1}
  if ((rc = launch_witness(c))) return rc;
  if (c->damp && c->energy && (rc = launch_rayleigh(c, damp_velocity(c, true)))) return rc;
  return launch_nodal(c, nodal_mode);
}

int32_t next_event(sma_ctx* c, int* idx) {
  if (c->evnext == c->evpool.size()) {
    cudaEvent_t e;
    CU(cudaEventCreate(&e));
    c->evpool.push_back(e);
  }
  *idx = (int)c->evnext++;
  CU(cudaEventRecord(c->evpool[*idx], c->stream));
  return SMA_OK;
}

// timed variant of issue_step: events around the element loop, the nodal
// update and the whole step
int32_t issue_step_timed(sma_ctx* c, int nodal_mode) {
  int e0, e1, e2, rc;
  if ((rc = next_event(c, &e0))) return rc;
  if ((rc = launch_elements(c, true))) return rc;
  c->cur ^= 1;
  if ((rc = next_event(c, &e1))) return rc;
  if ((rc = launch_witness(c))) return rc;
  if (c->damp && c->energy && (rc = launch_rayleigh(c, damp_velocity(c, true)))) return rc;
  if ((rc = launch_nodal(c, nodal_mode))) return rc;
  if ((rc = next_event(c, &e2))) return rc;
  c->evmarks.push_back({0, {e0, e1}});
  c->evmarks.push_back({1, {e1, e2}});
  c->evmarks.push_back({2, {e0, e2}});
  return SMA_OK;
}

int32_t collect_timers(sma_ctx* c) {
  CU(cudaStreamSynchronize(c->stream));
  for (auto& m : c->evmarks) {
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, c->evpool[m.second.first], c->evpool[m.second.second]));
    c->tms[m.first] += ms;
    c->tcnt[m.first] += (m.first == 0) ? (int64_t)(c->cptr.size() - 1) : 1;
  }
  c->evmarks.clear();
  c->evnext = 0;
  return SMA_OK;
}

void destroy_graphs(sma_ctx* c) {
  for (int p = 0; p < 2; ++p)
    if (c->gexec[p]) {
      cudaGraphExecDestroy(c->gexec[p]);
      c->gexec[p] = nullptr;
    }
  c->gchunk = 0;
}

// capture `chunk` interior steps for both starting parities
int32_t build_graphs(sma_ctx* c, int chunk) {
  destroy_graphs(c);
  const int saved = c->cur;
  const int64_t saved_l = c->launches;
  for (int p = 0; p < 2; ++p) {
    c->cur = p;
    cudaGraph_t g = nullptr;
    CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int32_t rc = SMA_OK;
    for (int s = 0; s < chunk && rc == SMA_OK; ++s) rc = issue_step(c, 1);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); c->cur = saved; return rc; }
    if (e != cudaSuccess) { c->cur = saved; return fail(SMA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e)); }
    e = cudaGraphInstantiate(&c->gexec[p], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { c->cur = saved; return fail(SMA_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)); }
  }
  c->cur = saved;
  c->launches = saved_l;
  c->gchunk = chunk;
  return SMA_OK;
}

int64_t kernels_per_step(const sma_ctx* c) {
  int64_t elem = (int64_t)(c->cptr.size() - 1);
  if (!c->sur && !c->plan_end.empty()) {
    elem = 0;
    for (size_t r = 0; r < c->plan_end.size(); ++r)
      elem += c->plan_end[r] > (r ? c->plan_end[r - 1] : 0);
  }
  return elem + 1 + (c->sur ? 1 : 0) + (c->nwit > 0 ? 1 : 0) + (c->energy ? 1 : 0) +
         (c->energy && c->damp ? 1 : 0);
}

template <typename T>
int32_t alloc_state(sma_ctx* c) {
  for (int s = 0; s < 2; ++s) {
    int32_t rc = dalloc(&c->d_state[s], 3 * (size_t)c->sst * sizeof(T));
    if (rc) return rc;
    CU(cudaMemset(c->d_state[s], 0, 3 * (size_t)c->sst * sizeof(T)));
  }
  return SMA_OK;
}

}  // namespace

extern "C" {

const char* sma_last_error(void) { return g_err.c_str(); }
const char* sma_version(void) { return "alya_sma_b200 0.1 (sm_100a)"; }

int32_t sma_ctx_destroy(sma_ctx* c) {
  if (!c) return SMA_OK;
  cudaSetDevice(c->dev);
  if (c->stream) cudaStreamSynchronize(c->stream);
  destroy_graphs(c);
  for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
  if (c->l2_window) cudaCtxResetPersistingL2Cache();   // release the lines this context pinned
  void* bufs[] = {c->d_lnods, c->d_perm, c->d_lmate, c->d_nodal, c->d_matx, c->d_sur_img, c->d_sur_stats,
                  c->d_xstage, c->d_sur_ctr, c->d_rcache,
                  c->d_invm, c->d_fext, c->d_tempe, c->d_flags, c->d_bcfun, c->d_mats,
                  c->d_state[0], c->d_state[1], c->d_cnt, c->d_ts, c->d_ft, c->d_stage,
                  c->d_stage2, c->d_wdof, c->d_whist, c->d_wrow, c->d_uprev, c->d_fintp,
                  c->d_fextp, c->d_en, c->d_ehist, c->d_erow, c->d_epart, c->d_pp_acc,
                  c->d_pp_out, c->d_pp_gp, c->d_fray, c->d_gp_F, c->d_gp_P, c->d_gp_det,
                  c->d_gp_vol};
  for (void* b : bufs)
    if (b) cudaFree(b);
  for (cudaEvent_t e : c->pl_ev) cudaEventDestroy(e);
  if (c->s_h2d) cudaStreamDestroy(c->s_h2d);
  if (c->s_d2h) cudaStreamDestroy(c->s_d2h);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return SMA_OK;
}

int32_t sma_ctx_create(const sma_mesh_desc* mesh, const sma_material_desc* mat,
                       const sma_run_desc* run, sma_ctx** out) {
  if (!out) return fail(SMA_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!mesh || !mat || !run) return fail(SMA_ERR_ARG, "NULL descriptor");
  if (mesh->nelem <= 0 || mesh->npoin <= 0 || !mesh->lnods || !mesh->coord)
    return fail(SMA_ERR_ARG, "empty mesh");
  if (mat->nmate <= 0 || !mat->props || !mat->densi) return fail(SMA_ERR_ARG, "no material");
  if (run->precision != SMA_PREC_FP64 && run->precision != SMA_PREC_FP32)
    return fail(SMA_ERR_ARG, "precision must be SMA_PREC_FP64 or SMA_PREC_FP32");
  if (run->nfun < 0 || run->nfun > MAXFUN) return fail(SMA_ERR_ARG, "at most 16 time functions");
  if (run->block != 0 && (run->block % 32 != 0 || run->block < 32 || run->block > 256))
    return fail(SMA_ERR_ARG, "block must be a multiple of 32 in [32, 256]");
  if (run->scheme != SMA_SCHEME_CD && run->scheme != SMA_SCHEME_TW)
    return fail(SMA_ERR_ARG, "scheme must be SMA_SCHEME_CD or SMA_SCHEME_TW");
  if (mat->dampi)
    for (int im = 0; im < mat->nmate; ++im) {
      if (!(mat->dampi[2 * im] >= 0.0))
        return fail(SMA_ERR_ARG, "Rayleigh alpha of material " + std::to_string(im) + " must be >= 0");
      if (mat->dampi[2 * im + 1] != 0.0)
        return fail(SMA_ERR_ARG, "Rayleigh beta (stiffness-proportional damping) of material " +
                                     std::to_string(im) + " is not supported; use alpha only");
    }
  for (int64_t k = 0; k < 8 * (int64_t)mesh->nelem; ++k)
    if (mesh->lnods[k] < 0 || mesh->lnods[k] >= mesh->npoin)
      return fail(SMA_ERR_ARG, "lnods entry out of range at " + std::to_string(k));
  if (mesh->lmate)
    for (int e = 0; e < mesh->nelem; ++e)
      if (mesh->lmate[e] < 0 || mesh->lmate[e] >= mat->nmate)
        return fail(SMA_ERR_ARG, "lmate entry out of range at " + std::to_string(e));
  int nfun = run->nfun;
  for (int f = 0; f < nfun; ++f)
    if (run->fun_npts[f] < 1 || run->fun_npts[f] > MAXPTS)
      return fail(SMA_ERR_ARG, "time function tables hold 1..32 rows");
  if (run->bcfun)
    for (int p = 0; p < mesh->npoin; ++p)
      if (run->bcfun[p] >= nfun) return fail(SMA_ERR_ARG, "bcfun beyond nfun");
  if (run->load_fun >= nfun) return fail(SMA_ERR_ARG, "load_fun beyond nfun");
  for (int im = 0; im < mat->nmate; ++im) {
    const double* pr = mat->props + 18 * im;
    if (!(pr[0] > 0.0) || !(pr[1] > -1.0 && pr[1] < 0.5) || !(mat->densi[im] > 0.0))
      return fail(SMA_ERR_ARG, "material " + std::to_string(im) + ": need E > 0, -1 < nu < 0.5, rho > 0");
  }

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
    return fail(SMA_ERR_NODEVICE, "no CUDA device");
  if (run->device < 0 || run->device >= ndev) return fail(SMA_ERR_ARG, "device ordinal");
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, run->device));
  if (prop.major != 10) return fail(SMA_ERR_NODEVICE, "this build targets sm_100a (B200)");

  sma_ctx* c = new sma_ctx();
  int32_t rc = SMA_OK;
#define TRY(x)                  \
  do {                          \
    rc = (x);                   \
    if (rc) {                   \
      sma_ctx_destroy(c);       \
      return rc;                \
    }                           \
  } while (0)
#define TRYCU(call)                                                                  \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      cudaGetLastError();                                                            \
      sma_ctx_destroy(c);                                                            \
      return fail(SMA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    }                                                                                \
  } while (0)

  c->dev = run->device;
  TRYCU(cudaSetDevice(c->dev));
  TRYCU(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  c->prec = run->precision;
  c->scatter = (run->scatter == SMA_SCATTER_COLOR) ? SMA_SCATTER_COLOR : SMA_SCATTER_ATOMIC;
  // default variant, measured on B200 (cantilever 640k and cylinder 2.0M
  // elements, fixed step windows): the one-tile kernel in both precisions;
  // with the register caps of the element kernels the pipelined variant
  // spills and is 10-50 % slower
  if (run->variant < SMA_VARIANT_AUTO || run->variant > SMA_VARIANT_TABLE)
    { sma_ctx_destroy(c); return fail(SMA_ERR_ARG, "variant must be one of SMA_VARIANT_*"); }
  if (run->variant == SMA_VARIANT_AUTO || run->variant == SMA_VARIANT_TABLE)
    c->variant = SMA_VARIANT_PLAIN;
  else
    c->variant = run->variant;
  // default block, measured on B200 over fixed step windows: the one-tile
  // kernel at 32 threads (one warp, 4 elements) with one material (finer
  // scheduling at the same warps per SM, no block barrier: against 128,
  // -2.1 % FP32 and -1.9 % FP64 element time on the 640 k-element
  // cantilever), at 128 with per-element materials (their table fill and
  // barrier amortise over more elements: against 64, -0.7 % FP32 / -2.5 %
  // FP64 on the 3.73 M-element ensemble, -3.1 % FP64 on the 2.0 M-element
  // cylinder); 256 for the pipelined kernel
  const bool per_element_mats = mesh->lmate && mat->nmate > 1;
  c->block = run->block ? run->block
                        : (c->variant == SMA_VARIANT_PIPE ? 256 : (per_element_mats ? 128 : 32));
  c->nsm = prop.multiProcessorCount;
  c->nelem = mesh->nelem;
  c->npoin = mesh->npoin;
  c->npad = ceil_div(c->npoin, 32) * 32;
  c->sst = ceil_div(8 * (int64_t)c->nelem, 32) * 32;
  c->nmate = mat->nmate;
  c->dtime = run->dtime;
  c->scheme = run->scheme;

  // element order
  c->perm.resize(c->nelem);
  if (c->scatter == SMA_SCATTER_COLOR) {
    int nc = host_color(c->nelem, c->npoin, mesh->lnods, c->perm, c->cptr);
    if (nc < 0) { sma_ctx_destroy(c); return fail(SMA_ERR_ARG, "mesh needs more than 64 colours"); }
  } else {
    for (int e = 0; e < c->nelem; ++e) c->perm[e] = e;
    c->cptr = {0, c->nelem};
  }
  std::vector<int32_t> lnods_i(8 * (size_t)c->nelem);
  for (int e = 0; e < c->nelem; ++e)
    std::memcpy(&lnods_i[8 * (size_t)e], mesh->lnods + 8 * (int64_t)c->perm[e], 8 * sizeof(int32_t));
  TRY(dalloc(&c->d_lnods, lnods_i.size() * sizeof(int32_t)));
  TRYCU(cudaMemcpy(c->d_lnods, lnods_i.data(), lnods_i.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  if (c->scatter == SMA_SCATTER_ATOMIC) {
    plan_pipeline(c, lnods_i.data());
    if (c->pl_need.size() >= 2) {
      TRYCU(cudaStreamCreateWithFlags(&c->s_h2d, cudaStreamNonBlocking));
      TRYCU(cudaStreamCreateWithFlags(&c->s_d2h, cudaStreamNonBlocking));
      c->pl_ev.resize(2 * c->pl_need.size() + 1, nullptr);
      for (cudaEvent_t& e : c->pl_ev) TRYCU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    } else {
      c->pl_need.clear();                  // one slab: the serial path
    }
  }
  TRY(dalloc(&c->d_perm, c->perm.size() * sizeof(int32_t)));
  TRYCU(cudaMemcpy(c->d_perm, c->perm.data(), c->perm.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  if (mesh->lmate && c->nmate > 1) {
    std::vector<int32_t> lm(c->nelem);
    for (int e = 0; e < c->nelem; ++e) lm[e] = mesh->lmate[c->perm[e]];
    TRY(dalloc(&c->d_lmate, lm.size() * sizeof(int32_t)));
    TRYCU(cudaMemcpy(c->d_lmate, lm.data(), lm.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (mat->tempe) {
    std::vector<double> tp(c->nelem);
    for (int e = 0; e < c->nelem; ++e) tp[e] = mat->tempe[c->perm[e]];
    TRY(dalloc(&c->d_tempe, tp.size() * sizeof(double)));
    TRYCU(cudaMemcpy(c->d_tempe, tp.data(), tp.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  std::vector<MatC> mats(c->nmate);
  for (int im = 0; im < c->nmate; ++im) {
    mats[im] = make_mat(mat->props + 18 * im, mat->e_mart ? mat->e_mart[im] : 0.0, mat->densi[im]);
    mats[im].ray_a = mat->dampi ? mat->dampi[2 * im] : 0.0;
    c->damp |= mats[im].ray_a > 0.0;
  }
  if (c->damp) c->variant = SMA_VARIANT_PLAIN;                  // the damped kernel is one-tile
  TRY(dalloc(&c->d_mats, mats.size() * sizeof(MatC)));
  TRYCU(cudaMemcpy(c->d_mats, mats.data(), mats.size() * sizeof(MatC), cudaMemcpyHostToDevice));
  c->mat0 = mats[0];
  // Compact per-element records when the materials differ only in what the
  // record holds (moduli, eL, thresholds; the temperature rides along) and
  // are many: 64 bytes per element read into registers instead of the
  // 176-byte material staged through shared memory behind a block barrier.
  // Measured on B200: the 2.0 M-element cylinder (a material per element)
  // -15 % FP32 / -6 % FP64 element time; the 256-specimen ensemble (256
  // materials, a table the caches hold) +16 % FP32, so a few materials keep
  // the table.  The one-tile undamped kernel reads them; SMA_VARIANT_TABLE
  // keeps the table.
  if (c->d_lmate && (int64_t)c->nmate * COMPACT_MAX_SHARING >= c->nelem && c->variant == SMA_VARIANT_PLAIN &&
      !c->damp &&
      run->variant != SMA_VARIANT_TABLE) {
    bool shared = true;
    for (const MatC& m : mats)
      shared = shared && m.kK == c->mat0.kK && m.kG == c->mat0.kG && m.alfa == c->mat0.alfa &&
               m.C_AS == c->mat0.C_AS && m.C_SA == c->mat0.C_SA && m.densi == c->mat0.densi &&
               m.ray_a == c->mat0.ray_a;
    if (shared) {
      std::vector<double> rec((size_t)c->nelem * MATX);
      for (int e = 0; e < c->nelem; ++e) {
        const MatC& m = mats[mesh->lmate[c->perm[e]]];
        double* r = rec.data() + (size_t)e * MATX;
        r[MX_IEA] = m.iEA;
        r[MX_IEM] = m.iEM;
        r[MX_EL] = m.eL;
        r[MX_RS_AS] = m.Rs_AS;
        r[MX_RF_AS] = m.Rf_AS;
        r[MX_RS_SA] = m.Rs_SA;
        r[MX_RF_SA] = m.Rf_SA;
        r[MX_TEMP] = mat->tempe ? mat->tempe[c->perm[e]] : 0.0;
      }
      if (c->prec == SMA_PREC_FP32) {
        // offsets from material 0 (temperature: from the first element's)
        c->mat0.T0 = rec[MX_TEMP];
        const double base[MATX] = {c->mat0.iEA, c->mat0.iEM, c->mat0.eL, c->mat0.Rs_AS, c->mat0.Rf_AS,
                                   c->mat0.Rs_SA, c->mat0.Rf_SA, c->mat0.T0};
        std::vector<float> rf(rec.size());
        for (size_t q = 0; q < rec.size(); ++q) rf[q] = (float)(rec[q] - base[q % MATX]);
        TRY(dalloc(&c->d_matx, rf.size() * sizeof(float)));
        TRYCU(cudaMemcpy(c->d_matx, rf.data(), rf.size() * sizeof(float), cudaMemcpyHostToDevice));
      } else {
        TRY(dalloc(&c->d_matx, rec.size() * sizeof(double)));
        TRYCU(cudaMemcpy(c->d_matx, rec.data(), rec.size() * sizeof(double), cudaMemcpyHostToDevice));
      }
      c->compact = true;
      // no block barrier: one-warp blocks, as with one material
      if (!run->block) c->block = 32;
    }
  }

  // nodal arrays (SoA [3][npad])
  const size_t nb = 3 * (size_t)c->npad * sizeof(double);
  // One block, gathered/scattered arrays first: coordinates, displacement and
  // residual are read by every element of a node, so they are kept in L2 with
  // a persisting access window on the context stream (the state streams
  // through once per step and would otherwise evict them; measured 7 % on
  // the FP32 element loop of a 640 k-element mesh).
  {
    TRY(dalloc(&c->d_nodal, 6 * nb));
    TRYCU(cudaMemset(c->d_nodal, 0, 6 * nb));
    const size_t nd = nb / sizeof(double);
    c->d_coord = c->d_nodal;
    c->d_u = c->d_nodal + nd;
    c->d_f = c->d_nodal + 2 * nd;
    c->d_vt = c->d_nodal + 3 * nd;
    c->d_v = c->d_nodal + 4 * nd;
    c->d_a = c->d_nodal + 5 * nd;
    set_l2_window(c, c->d_nodal, 3 * nb, prop);
  }
  if (c->damp) {
    TRY(dalloc(&c->d_fray, nb));
    TRYCU(cudaMemset(c->d_fray, 0, nb));
  }
  TRY(dalloc(&c->d_stage, 3 * (size_t)c->npoin * sizeof(double)));
  TRY(dalloc(&c->d_stage2, 3 * (size_t)c->npoin * sizeof(double)));
  const unsigned ngrid = (unsigned)ceil_div(c->npoin, 256);
  // staged uploads are ordered on the context stream: the staging buffer is
  // reused, and a blocking copy does not wait for kernels on a non-blocking
  // stream that still read the previous contents
  TRYCU(cudaMemcpyAsync(c->d_stage, mesh->coord, 3 * (size_t)c->npoin * sizeof(double),
                        cudaMemcpyHostToDevice, c->stream));
  k_aos_to_soa<<<ngrid, 256, 0, c->stream>>>(c->d_stage, c->d_coord, c->npoin, c->npad);
  TRYCU(cudaGetLastError());

  // flags, boundary functions, loads
  std::vector<uint8_t> flags(c->npoin, 0);
  std::vector<int8_t> bcf(c->npoin, -1);
  for (int p = 0; p < c->npoin; ++p) {
    for (int i = 0; i < 3; ++i)
      if (run->fixno && run->fixno[3 * (int64_t)p + i] == 1) flags[p] |= (uint8_t)(1u << i);
    if (run->bcfun) bcf[p] = (int8_t)run->bcfun[p];
  }
  if (run->fext && run->load_fun >= 0) {
    c->has_load = true;
    for (int p = 0; p < c->npoin; ++p)
      if (run->fext[3 * (int64_t)p] != 0.0 || run->fext[3 * (int64_t)p + 1] != 0.0 ||
          run->fext[3 * (int64_t)p + 2] != 0.0)
        flags[p] |= 8u;
    TRY(dalloc(&c->d_fext, nb));
    TRYCU(cudaMemset(c->d_fext, 0, nb));
    TRYCU(cudaMemcpyAsync(c->d_stage, run->fext, 3 * (size_t)c->npoin * sizeof(double),
                          cudaMemcpyHostToDevice, c->stream));
    k_aos_to_soa<<<ngrid, 256, 0, c->stream>>>(c->d_stage, c->d_fext, c->npoin, c->npad);
    TRYCU(cudaGetLastError());
  }
  TRY(dalloc(&c->d_flags, flags.size()));
  TRYCU(cudaMemcpy(c->d_flags, flags.data(), flags.size(), cudaMemcpyHostToDevice));
  TRY(dalloc(&c->d_bcfun, bcf.size()));
  TRYCU(cudaMemcpy(c->d_bcfun, bcf.data(), bcf.size(), cudaMemcpyHostToDevice));

  // lumped mass (constant: geometry and density do not change)
  c->vmass.assign(c->npoin, 0.0);
  host_lumped_mass(c->nelem, mesh->lnods, mesh->coord, mesh->lmate, mat->densi, c->vmass);
  std::vector<double> invm(c->npad, 0.0);
  for (int p = 0; p < c->npoin; ++p) invm[p] = 1.0 / c->vmass[p];
  TRY(dalloc(&c->d_invm, invm.size() * sizeof(double)));
  TRYCU(cudaMemcpy(c->d_invm, invm.data(), invm.size() * sizeof(double), cudaMemcpyHostToDevice));
  c->dtcri = host_critical_dt(c->nelem, mesh->lnods, mesh->coord, mesh->lmate, mat->props,
                              mat->e_mart, mat->densi);

  // state
  TRY(c->prec == SMA_PREC_FP32 ? alloc_state<float>(c) : alloc_state<double>(c));
  TRY(c->prec == SMA_PREC_FP32 ? init_element_launch_t<float>(c) : init_element_launch_t<double>(c));
  TRY(dalloc(&c->d_cnt, NCNT * sizeof(unsigned long long)));
  TRYCU(cudaMemset(c->d_cnt, 0, NCNT * sizeof(unsigned long long)));
  TRYCU(cudaMemset(c->d_cnt + CNT_DETMIN, 0xff, sizeof(unsigned long long)));   // none seen

  // time functions and step time
  FunTab ft;
  std::memset(&ft, 0, sizeof ft);
  ft.nfun = nfun;
  int64_t off = 0;
  for (int f = 0; f < nfun; ++f) {
    ft.npts[f] = run->fun_npts[f];
    ft.smooth[f] = run->fun_smooth ? run->fun_smooth[f] : 0;
    for (int r = 0; r < ft.npts[f]; ++r)
      for (int q = 0; q < 4; ++q) ft.tab[f][r][q] = run->fun_tab[off + 4 * r + q];
    off += 4 * ft.npts[f];
  }
  TRY(dalloc(&c->d_ft, sizeof(FunTab)));
  TRYCU(cudaMemcpy(c->d_ft, &ft, sizeof ft, cudaMemcpyHostToDevice));
  StepTime ts;
  std::memset(&ts, 0, sizeof ts);
  ts.dtime = run->dtime;
  ts.load_fun = c->has_load ? run->load_fun : -1;
  ts.phi = (run->phitw != 0.0) ? run->phitw : 1.033;   // sld_reanut.f90:176 default
  TRY(dalloc(&c->d_ts, sizeof(StepTime)));
  TRYCU(cudaMemcpy(c->d_ts, &ts, sizeof ts, cudaMemcpyHostToDevice));
  TRYCU(cudaStreamSynchronize(c->stream));
#undef TRY
#undef TRYCU
  *out = c;
  return SMA_OK;
}

// the explicit step in parts, for partitioned meshes (the caller sums the
// interface residual between sma_step_elements and sma_step_nodes)
int32_t sma_step_prologue(sma_ctx* c) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  if (!(c->dtime > 0.0)) return fail(SMA_ERR_STATE, "dtime not set");
  CU(cudaSetDevice(c->dev));
  if (c->nwit > 0) CU(cudaMemsetAsync(c->d_wrow, 0, sizeof(int), c->stream));
  k_advance_time<<<1, 1, 0, c->stream>>>(c->d_ts, c->d_ft);
  c->launches++;
  return launch_nodal(c, 0);
}

int32_t sma_step_elements(sma_ctx* c) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  CU(cudaSetDevice(c->dev));
  int32_t rc = launch_elements(c, true);
  if (rc) return rc;
  c->cur ^= 1;
  if ((rc = launch_witness(c))) return rc;
  if (c->damp && c->energy && (rc = launch_rayleigh(c, damp_velocity(c, true)))) return rc;
  return SMA_OK;
}

// the element loop of a step in ranges, so a partitioned caller can send
// the interface rows while the interior elements compute: first = 1 on the
// step's first range (advances the time), last = 1 on its last (the state
// of this step becomes TIME_N of the next)
int32_t sma_step_elements_range(sma_ctx* c, int32_t beg, int32_t end, int32_t first, int32_t last) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  if (c->scatter == SMA_SCATTER_COLOR) return fail(SMA_ERR_ARG, "element ranges need the atomic scatter");
  if (beg < 0 || end > c->nelem || beg > end) return fail(SMA_ERR_ARG, "element range outside [0, nelem)");
  CU(cudaSetDevice(c->dev));
  int32_t rc = SMA_OK;
  if (first) c->last_in = c->cur;
  if (end > beg) {
    if (c->prec == SMA_PREC_FP32 && c->sur) {
      rc = launch_sur_range(c, beg, end, first != 0, true);
    } else {
      const int epb = c->block / 8;
      const int64_t ntiles = ceil_div(end - beg, epb);
      const unsigned grid = c->variant == SMA_VARIANT_PIPE
                                ? (unsigned)std::min<int64_t>(ntiles, (int64_t)c->nsm * c->resident)
                                : (unsigned)ntiles;
      if (c->prec == SMA_PREC_FP32) {
        ElemArgs<float> a = elem_args<float>(c, beg, end, first != 0, true);
        elem_kernel<float>(c)<<<grid, c->block, elem_smem<float>(c), c->stream>>>(a);
      } else {
        ElemArgs<double> a = elem_args<double>(c, beg, end, first != 0, true);
        elem_kernel<double>(c)<<<grid, c->block, elem_smem<double>(c), c->stream>>>(a);
      }
      c->launches++;
      CU(cudaGetLastError());
    }
  } else if (first) {
    k_advance_time<<<1, 1, 0, c->stream>>>(c->d_ts, c->d_ft);
    c->launches++;
    CU(cudaGetLastError());
  }
  if (rc) return rc;
  if (last && c->prec == SMA_PREC_FP32 && c->sur && (rc = launch_sur_refresh(c, -1))) return rc;
  if (last) {
    c->cur ^= 1;
    if ((rc = launch_witness(c))) return rc;
    if (c->damp && c->energy && (rc = launch_rayleigh(c, damp_velocity(c, true)))) return rc;
  }
  return SMA_OK;
}

int32_t sma_step_nodes(sma_ctx* c, int32_t last) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  CU(cudaSetDevice(c->dev));
  int32_t rc = launch_nodal(c, last ? 2 : 1);
  if (rc) return rc;
  if (last) CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

int32_t sma_gather_residual(sma_ctx* c, int32_t n, const int32_t* d_nodes, double* d_rows) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  if (n < 0) return fail(SMA_ERR_ARG, "n < 0");
  if (n == 0) return SMA_OK;
  if (!d_nodes || !d_rows) return fail(SMA_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(c->dev));
  k_gather_rows<<<(unsigned)ceil_div(n, 256), 256, 0, c->stream>>>(c->d_f, c->npad, c->npoin, n, d_nodes,
                                                                    d_rows);
  c->launches++;
  CU(cudaGetLastError());
  return SMA_OK;
}

int32_t sma_scatter_residual(sma_ctx* c, int32_t n, const int32_t* d_nodes, const double* d_rows) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  if (n < 0) return fail(SMA_ERR_ARG, "n < 0");
  if (n == 0) return SMA_OK;
  if (!d_nodes || !d_rows) return fail(SMA_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(c->dev));
  k_scatter_rows<<<(unsigned)ceil_div(n, 256), 256, 0, c->stream>>>(c->d_f, c->npad, c->npoin, n, d_nodes,
                                                                     d_rows);
  c->launches++;
  CU(cudaGetLastError());
  return SMA_OK;
}

int32_t sma_explicit_step(sma_ctx* c, int32_t nsteps) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  if (nsteps < 0) return fail(SMA_ERR_ARG, "nsteps < 0");
  if (nsteps == 0) return SMA_OK;
  if (!(c->dtime > 0.0)) return fail(SMA_ERR_STATE, "dtime not set");
  CU(cudaSetDevice(c->dev));
  int32_t rc;
  if (c->nwit > 0) CU(cudaMemsetAsync(c->d_wrow, 0, sizeof(int), c->stream));
  // prologue: time of step 1 and its predictor from the boundary state
  k_advance_time<<<1, 1, 0, c->stream>>>(c->d_ts, c->d_ft);
  c->launches++;
  if ((rc = launch_nodal(c, 0))) return rc;
  if (c->timing) {
    for (int s = 0; s < nsteps; ++s)
      if ((rc = issue_step_timed(c, s + 1 < nsteps ? 1 : 2))) return rc;
    return collect_timers(c);
  }
  // interior steps (element loop + fused corrector/predictor) as graphs
  int interior = nsteps - 1;
  const int chunk = 8;
  if (interior >= chunk) {
    if (c->gchunk != chunk && (rc = build_graphs(c, chunk))) return rc;
    while (interior >= chunk) {
      CU(cudaGraphLaunch(c->gexec[c->cur], c->stream));
      c->launches += chunk * kernels_per_step(c);
      if (chunk & 1) c->cur ^= 1;
      interior -= chunk;
    }
  }
  for (; interior > 0; --interior)
    if ((rc = issue_step(c, 1))) return rc;
  // last step: element loop + corrector only
  if ((rc = issue_step(c, 2))) return rc;
  CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

int32_t sma_assemble_device(sma_ctx* c, const double* d_displ, double fext_scale, double* d_rhsid) {
  if (!c || !d_displ || !d_rhsid) return fail(SMA_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(c->dev));
  const unsigned ngrid = (unsigned)ceil_div(c->npoin, 256);
  k_aos_to_soa<<<ngrid, 256, 0, c->stream>>>(d_displ, c->d_u, c->npoin, c->npad);
  k_fill_f<<<ngrid, 256, 0, c->stream>>>(c->d_f, c->d_fext, c->d_flags, fext_scale, c->npoin, c->npad);
  c->launches += 2;
  CU(cudaGetLastError());
  int32_t rc = launch_elements(c, false);
  if (rc) return rc;
  k_outputs<<<ngrid, 256, 0, c->stream>>>(c->d_f, c->d_fext, c->d_flags, fext_scale, c->npoin,
                                          c->npad, d_rhsid, nullptr, nullptr, nullptr, nullptr);
  c->launches++;
  CU(cudaGetLastError());
  return SMA_OK;
}

int32_t sma_assemble(sma_ctx* c, const double* displ, double fext_scale, double* rhsid,
                     double* finte, double* fexte, double* frxid, double* vmass) {
  if (!c || !displ || !rhsid) return fail(SMA_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(c->dev));
  const size_t bytes = 3 * (size_t)c->npoin * sizeof(double);
  const unsigned ngrid = (unsigned)ceil_div(c->npoin, 256);
  int32_t rc;
  const bool piped = !c->pl_need.empty();
  if (piped) {
    // displacement in, element slabs and residual out overlapped
    rc = c->prec == SMA_PREC_FP32 ? assemble_pipelined_t<float>(c, displ, fext_scale, rhsid)
                                  : assemble_pipelined_t<double>(c, displ, fext_scale, rhsid);
    if (rc) return rc;
  } else {
    CU(cudaMemcpyAsync(c->d_stage, displ, bytes, cudaMemcpyHostToDevice, c->stream));
    k_aos_to_soa<<<ngrid, 256, 0, c->stream>>>(c->d_stage, c->d_u, c->npoin, c->npad);
    k_fill_f<<<ngrid, 256, 0, c->stream>>>(c->d_f, c->d_fext, c->d_flags, fext_scale, c->npoin, c->npad);
    c->launches += 2;
    CU(cudaGetLastError());
    if ((rc = launch_elements(c, false))) return rc;
  }
  double* outs[4] = {rhsid, finte, fexte, frxid};
  // with damping, finte leaves the Rayleigh force out (it is in rhsid only)
  const double* fray = nullptr;
  if (c->damp && finte) {
    if ((rc = launch_rayleigh(c, damp_velocity(c, false)))) return rc;
    fray = c->d_fray;
  }
  for (int q = piped ? 1 : 0; q < 4; ++q) {
    if (!outs[q]) continue;
    double* dr = c->d_stage;
    k_outputs<<<ngrid, 256, 0, c->stream>>>(c->d_f, c->d_fext, c->d_flags, fext_scale, c->npoin,
                                            c->npad, q == 0 ? dr : c->d_stage2,
                                            q == 1 ? dr : nullptr, q == 2 ? dr : nullptr,
                                            q == 3 ? dr : nullptr, fray);
    c->launches++;
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(outs[q], dr, bytes, cudaMemcpyDeviceToHost, c->stream));
  }
  CU(cudaStreamSynchronize(c->stream));
  if (vmass) std::memcpy(vmass, c->vmass.data(), c->npoin * sizeof(double));
  return SMA_OK;
}

int32_t sma_host_register(void* ptr, size_t bytes) {
  if (!ptr || bytes == 0) return fail(SMA_ERR_ARG, "NULL or empty host array");
  CU(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
  return SMA_OK;
}

int32_t sma_host_unregister(void* ptr) {
  if (!ptr) return fail(SMA_ERR_ARG, "NULL host array");
  CU(cudaHostUnregister(ptr));
  return SMA_OK;
}

int32_t sma_end_step(sma_ctx* c) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  c->cur ^= 1;
  return SMA_OK;
}

int32_t sma_postprocess(sma_ctx* c, double* caust, double* green, double* lepsi, double* seqvm,
                        double* gp_sigma) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  CU(cudaSetDevice(c->dev));
  int32_t rc;
  if (!c->d_pp_acc && (rc = dalloc(&c->d_pp_acc, PP_COLS * (size_t)c->npad * sizeof(double)))) return rc;
  if (!c->d_pp_out && (rc = dalloc(&c->d_pp_out, PP_COLS * (size_t)c->npoin * sizeof(double)))) return rc;
  if (gp_sigma && !c->d_pp_gp && (rc = dalloc(&c->d_pp_gp, 48 * (size_t)c->nelem * sizeof(double))))
    return rc;
  PostArgs p{};
  p.acc = c->d_pp_acc;
  p.gp_sig = gp_sigma ? c->d_pp_gp : nullptr;                  // the kernel skips what is null
  CU(cudaMemsetAsync(c->d_pp_acc, 0, PP_COLS * (size_t)c->npad * sizeof(double), c->stream));
  rc = c->prec == SMA_PREC_FP32 ? launch_postproc_t<float>(c, p) : launch_postproc_t<double>(c, p);
  if (rc) return rc;
  k_postproc_nodal<<<(unsigned)ceil_div(c->npoin, 256), 256, 0, c->stream>>>(c->d_pp_acc, c->npad,
                                                                             c->npoin, c->d_pp_out);
  c->launches++;
  CU(cudaGetLastError());
  const size_t n6 = 6 * (size_t)c->npoin;
  double* outs[3] = {caust, green, lepsi};
  for (int t = 0; t < 3; ++t)
    if (outs[t])
      CU(cudaMemcpyAsync(outs[t], c->d_pp_out + t * n6, n6 * sizeof(double), cudaMemcpyDeviceToHost,
                         c->stream));
  if (seqvm)
    CU(cudaMemcpyAsync(seqvm, c->d_pp_out + 3 * n6, c->npoin * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
  if (gp_sigma)
    CU(cudaMemcpyAsync(gp_sigma, c->d_pp_gp, 48 * (size_t)c->nelem * sizeof(double),
                       cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

int32_t sma_gauss_fields(sma_ctx* c, double* gpgdi, double* gppio, double* gpdet, double* volum) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  CU(cudaSetDevice(c->dev));
  int32_t rc;
  const size_t n72 = 72 * (size_t)c->nelem, n8 = 8 * (size_t)c->nelem;
  // device buffers only for what is asked, kept for the next call
  if (gpgdi && !c->d_gp_F && (rc = dalloc(&c->d_gp_F, n72 * sizeof(double)))) return rc;
  if (gppio && !c->d_gp_P && (rc = dalloc(&c->d_gp_P, n72 * sizeof(double)))) return rc;
  if (gpdet && !c->d_gp_det && (rc = dalloc(&c->d_gp_det, n8 * sizeof(double)))) return rc;
  if (volum && !c->d_gp_vol && (rc = dalloc(&c->d_gp_vol, 2 * sizeof(double)))) return rc;
  PostArgs p{};
  p.gp_F = gpgdi ? c->d_gp_F : nullptr;
  p.gp_P = gppio ? c->d_gp_P : nullptr;
  p.gp_det = gpdet ? c->d_gp_det : nullptr;
  p.volum = volum ? c->d_gp_vol : nullptr;
  if (volum) CU(cudaMemsetAsync(c->d_gp_vol, 0, 2 * sizeof(double), c->stream));
  rc = c->prec == SMA_PREC_FP32 ? launch_postproc_t<float>(c, p) : launch_postproc_t<double>(c, p);
  if (rc) return rc;
  if (gpgdi) CU(cudaMemcpyAsync(gpgdi, c->d_gp_F, n72 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (gppio) CU(cudaMemcpyAsync(gppio, c->d_gp_P, n72 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (gpdet) CU(cudaMemcpyAsync(gpdet, c->d_gp_det, n8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (volum) CU(cudaMemcpyAsync(volum, c->d_gp_vol, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

int32_t sma_set_nodal(sma_ctx* c, int32_t field, const double* host) {
  if (!c || !host) return fail(SMA_ERR_ARG, "NULL argument");
  if (field == SMA_FIELD_VMASS) {
    // a partitioned mesh's interface nodes take the mass summed over the
    // sub-meshes that share them
    for (int p = 0; p < c->npoin; ++p)
      if (!(host[p] > 0.0)) return fail(SMA_ERR_ARG, "lumped mass must be positive");
    std::vector<double> invm(c->npad, 0.0);
    for (int p = 0; p < c->npoin; ++p) {
      c->vmass[p] = host[p];
      invm[p] = 1.0 / host[p];
    }
    CU(cudaSetDevice(c->dev));
    CU(cudaStreamSynchronize(c->stream));
    CU(cudaMemcpy(c->d_invm, invm.data(), invm.size() * sizeof(double), cudaMemcpyHostToDevice));
    return SMA_OK;
  }
  double* dst = nullptr;
  switch (field) {
    case SMA_FIELD_DISPL: dst = c->d_u; break;
    case SMA_FIELD_VELOC: dst = c->d_v; break;
    case SMA_FIELD_ACCEL: dst = c->d_a; break;
    case SMA_FIELD_RHSID: dst = c->d_f; break;
    default: return fail(SMA_ERR_ARG, "field not settable");
  }
  CU(cudaSetDevice(c->dev));
  CU(cudaMemcpyAsync(c->d_stage, host, 3 * (size_t)c->npoin * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  k_aos_to_soa<<<(unsigned)ceil_div(c->npoin, 256), 256, 0, c->stream>>>(c->d_stage, dst, c->npoin, c->npad);
  c->launches++;
  CU(cudaGetLastError());
  // the surrogate's held residuals belong to the displacement they were taken at
  int32_t rc;
  if (field == SMA_FIELD_DISPL && c->sur && (rc = sur_init_residuals(c))) return rc;
  CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

int32_t sma_get_nodal(sma_ctx* c, int32_t field, double* host) {
  if (!c || !host) return fail(SMA_ERR_ARG, "NULL argument");
  if (field == SMA_FIELD_VMASS) {
    std::memcpy(host, c->vmass.data(), c->npoin * sizeof(double));
    return SMA_OK;
  }
  const double* src = nullptr;
  switch (field) {
    case SMA_FIELD_DISPL: src = c->d_u; break;
    case SMA_FIELD_VELOC: src = c->d_v; break;
    case SMA_FIELD_ACCEL: src = c->d_a; break;
    case SMA_FIELD_RHSID: src = c->d_f; break;
    default: return fail(SMA_ERR_ARG, "unknown field");
  }
  CU(cudaSetDevice(c->dev));
  k_soa_to_aos<<<(unsigned)ceil_div(c->npoin, 256), 256, 0, c->stream>>>(src, c->d_stage, c->npoin, c->npad);
  c->launches++;
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(host, c->d_stage, 3 * (size_t)c->npoin * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

static int32_t state_io(sma_ctx* c, double* host, bool in) {
  if (!c || !host) return fail(SMA_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(c->dev));
  const size_t bytes = 48 * (size_t)c->nelem * sizeof(double);
  double* d = nullptr;
  int32_t rc = dalloc(&d, bytes);
  if (rc) return rc;
  const unsigned grid = (unsigned)ceil_div(8 * (int64_t)c->nelem, 256);
  // slot ITER_K is the buffer the next element loop writes (cur ^ 1),
  // slot TIME_N the one it reads (cur)
  void* sk = c->d_state[c->cur ^ 1];
  void* sn = c->d_state[c->cur];
  cudaError_t e = cudaSuccess;
  if (in) {
    c->last_in = -1;                       // post-processing reads TIME_N until the next loop
    e = cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
      if (c->prec == SMA_PREC_FP32)
        k_state_in<float><<<grid, 256, 0, c->stream>>>(d, c->d_perm, (float*)sk, (float*)sn, c->nelem, c->sst);
      else
        k_state_in<double><<<grid, 256, 0, c->stream>>>(d, c->d_perm, (double*)sk, (double*)sn, c->nelem, c->sst);
      e = cudaGetLastError();
    }
  } else {
    if (c->prec == SMA_PREC_FP32)
      k_state_out<float><<<grid, 256, 0, c->stream>>>(d, c->d_perm, (const float*)sk, (const float*)sn, c->nelem, c->sst);
    else
      k_state_out<double><<<grid, 256, 0, c->stream>>>(d, c->d_perm, (const double*)sk, (const double*)sn, c->nelem, c->sst);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, c->stream);
  }
  c->launches++;
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(SMA_ERR_CUDA, std::string("state I/O: ") + cudaGetErrorString(e));
  return SMA_OK;
}

int32_t sma_set_state(sma_ctx* c, const double* host) {
  int32_t rc = state_io(c, const_cast<double*>(host), true);
  // the surrogate's held residuals belong to the state they were taken at
  if (!rc && c->sur) {
    if ((rc = sur_init_residuals(c))) return rc;
    CU(cudaStreamSynchronize(c->stream));
  }
  return rc;
}
int32_t sma_get_state(sma_ctx* c, double* host) { return state_io(c, host, false); }

int32_t sma_get_time(sma_ctx* c, double* cutim) {
  if (!c || !cutim) return fail(SMA_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(c->dev));
  CU(cudaMemcpyAsync(cutim, &c->d_ts->cutim, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

int32_t sma_set_time(sma_ctx* c, double cutim) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  CU(cudaSetDevice(c->dev));
  CU(cudaMemcpyAsync(&c->d_ts->cutim, &cutim, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

int32_t sma_get_counters(sma_ctx* c, sma_counters* out) {
  if (!c || !out) return fail(SMA_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(c->dev));
  unsigned long long h[NCNT];
  CU(cudaMemcpyAsync(h, c->d_cnt, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < SMA_NCOUNTERS; ++k) out->c[k] = (k != CNT_DETMIN) ? (int64_t)h[k] : 0;
  // the smallest det F <= 0 seen and its element (caller's numbering)
  const unsigned long long dm = h[CNT_DETMIN];
  if (dm == ~0ull) {
    out->gpdet_min = 0.0;
    out->ielem_min = -1;
  } else {
    const unsigned key = (unsigned)(dm >> 32);
    const unsigned bits = (key & 0x80000000u) ? (key & 0x7fffffffu) : ~key;
    float det;
    std::memcpy(&det, &bits, sizeof det);
    out->gpdet_min = det;
    const int64_t e = (int64_t)(dm & 0xffffffffull);
    out->ielem_min = (e >= 0 && e < c->nelem) ? c->perm[e] : -1;
  }
  return SMA_OK;
}

int32_t sma_reset_counters(sma_ctx* c) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  CU(cudaSetDevice(c->dev));
  CU(cudaMemsetAsync(c->d_cnt, 0, NCNT * sizeof(unsigned long long), c->stream));
  CU(cudaMemsetAsync(c->d_cnt + CNT_DETMIN, 0xff, sizeof(unsigned long long), c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

int32_t sma_set_witness(sma_ctx* c, int32_t nwit, const int32_t* dofs, int32_t max_steps) {
  if (!c || nwit < 0 || (nwit > 0 && (!dofs || max_steps <= 0))) return fail(SMA_ERR_ARG, "bad witness arguments");
  for (int w = 0; w < nwit; ++w)
    if (dofs[w] < 0 || dofs[w] >= 6 * c->npoin) return fail(SMA_ERR_ARG, "witness id out of range");
  CU(cudaSetDevice(c->dev));
  cudaFree(c->d_wdof); cudaFree(c->d_whist); cudaFree(c->d_wrow);
  c->d_wdof = nullptr; c->d_whist = nullptr; c->d_wrow = nullptr;
  c->nwit = 0;
  destroy_graphs(c);
  if (nwit == 0) return SMA_OK;
  int32_t rc;
  if ((rc = dalloc(&c->d_wdof, nwit * sizeof(int32_t)))) return rc;
  if ((rc = dalloc(&c->d_whist, (size_t)nwit * max_steps * sizeof(double)))) return rc;
  if ((rc = dalloc(&c->d_wrow, sizeof(int)))) return rc;
  CU(cudaMemcpy(c->d_wdof, dofs, nwit * sizeof(int32_t), cudaMemcpyHostToDevice));
  CU(cudaMemset(c->d_wrow, 0, sizeof(int)));
  c->nwit = nwit;
  c->wit_max = max_steps;
  return SMA_OK;
}

int32_t sma_get_witness(sma_ctx* c, double* host, int32_t* nsteps_out) {
  if (!c || !host) return fail(SMA_ERR_ARG, "NULL argument");
  if (c->nwit <= 0) return fail(SMA_ERR_STATE, "no witnesses set");
  CU(cudaSetDevice(c->dev));
  CU(cudaStreamSynchronize(c->stream));    // the witness kernels run on the context stream
  int rows = 0;
  CU(cudaMemcpy(&rows, c->d_wrow, sizeof(int), cudaMemcpyDeviceToHost));
  rows = std::min(rows, c->wit_max);
  CU(cudaMemcpy(host, c->d_whist, (size_t)rows * c->nwit * sizeof(double), cudaMemcpyDeviceToHost));
  if (nsteps_out) *nsteps_out = rows;
  return SMA_OK;
}

int32_t sma_set_energy(sma_ctx* c, int32_t enable, int32_t max_steps) {
  if (!c || (enable && max_steps < 0)) return fail(SMA_ERR_ARG, "bad energy arguments");
  CU(cudaSetDevice(c->dev));
  destroy_graphs(c);
  c->energy = false;
  if (!enable) return SMA_OK;
  const size_t nb = 3 * (size_t)c->npad * sizeof(double);
  int32_t rc;
  if (!c->d_uprev) {
    if ((rc = dalloc(&c->d_uprev, nb)) || (rc = dalloc(&c->d_fintp, nb)) || (rc = dalloc(&c->d_fextp, nb)) ||
        (rc = dalloc(&c->d_en, 16 * sizeof(double))) || (rc = dalloc(&c->d_erow, sizeof(int))) ||
        (rc = dalloc(&c->d_epart, 4 * (size_t)ceil_div(c->npoin, 256) * sizeof(double))))
      return rc;
  }
  if (c->d_ehist) { cudaFree(c->d_ehist); c->d_ehist = nullptr; }
  if (max_steps > 0 && (rc = dalloc(&c->d_ehist, 5 * (size_t)max_steps * sizeof(double)))) return rc;
  c->ehist_max = max_steps;
  // the first balance step measures from the current displacement, with
  // zero previous forces (fintt/fextt(TIME_N) start at zero)
  CU(cudaMemcpyAsync(c->d_uprev, c->d_u, nb, cudaMemcpyDeviceToDevice, c->stream));
  CU(cudaMemsetAsync(c->d_fintp, 0, nb, c->stream));
  CU(cudaMemsetAsync(c->d_fextp, 0, nb, c->stream));
  CU(cudaMemsetAsync(c->d_en, 0, 16 * sizeof(double), c->stream));
  CU(cudaMemsetAsync(c->d_erow, 0, sizeof(int), c->stream));
  CU(cudaStreamSynchronize(c->stream));
  c->energy = true;
  return SMA_OK;
}

int32_t sma_get_energy(sma_ctx* c, double* totals, double* hist, int32_t* nrows) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  if (!c->d_en) return fail(SMA_ERR_STATE, "energy balance not enabled");
  CU(cudaSetDevice(c->dev));
  double h[9];
  int rows = 0;
  CU(cudaMemcpyAsync(h, c->d_en, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  CU(cudaMemcpyAsync(&rows, c->d_erow, sizeof rows, cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  if (totals) {
    totals[0] = h[4];
    totals[1] = h[5];
    totals[2] = h[6];
    totals[3] = h[4] + h[6] - h[5];
    totals[4] = h[7];
  }
  rows = std::min(rows, c->ehist_max);
  if (hist && rows > 0 && c->d_ehist)
    CU(cudaMemcpy(hist, c->d_ehist, 5 * (size_t)rows * sizeof(double), cudaMemcpyDeviceToHost));
  if (nrows) *nrows = rows;
  return SMA_OK;
}

namespace {
struct CkptHeader {
  char magic[8];
  int32_t version, precision, scheme, has_energy;
  int64_t nelem, npoin;
  double cutim;
};
}  // namespace

int32_t sma_checkpoint_save(sma_ctx* c, const char* path) {
  if (!c || !path) return fail(SMA_ERR_ARG, "NULL argument");
  const size_t n3 = 3 * (size_t)c->npoin;
  std::vector<double> buf(std::max(n3, 48 * (size_t)c->nelem));
  CkptHeader hd;
  std::memset(&hd, 0, sizeof hd);
  std::memcpy(hd.magic, "SMAB200", 8);
  hd.version = 1;
  hd.precision = c->prec;
  hd.scheme = c->scheme;
  hd.has_energy = c->energy ? 1 : 0;
  hd.nelem = c->nelem;
  hd.npoin = c->npoin;
  int32_t rc = sma_get_time(c, &hd.cutim);
  if (rc) return rc;
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return fail(SMA_ERR_ARG, std::string("cannot write ") + path);
  bool ok = std::fwrite(&hd, sizeof hd, 1, fp) == 1;
  const int fields[3] = {SMA_FIELD_DISPL, SMA_FIELD_VELOC, SMA_FIELD_ACCEL};
  for (int q = 0; q < 3 && ok; ++q) {
    if ((rc = sma_get_nodal(c, fields[q], buf.data()))) { std::fclose(fp); return rc; }
    ok = std::fwrite(buf.data(), sizeof(double), n3, fp) == n3;
  }
  if (ok) {
    if ((rc = sma_get_state(c, buf.data()))) { std::fclose(fp); return rc; }
    ok = std::fwrite(buf.data(), sizeof(double), 48 * (size_t)c->nelem, fp) == 48 * (size_t)c->nelem;
  }
  if (ok && c->energy) {
    double* arrs[3] = {c->d_uprev, c->d_fintp, c->d_fextp};
    for (int q = 0; q < 3 && ok; ++q) {
      k_soa_to_aos<<<(unsigned)ceil_div(c->npoin, 256), 256, 0, c->stream>>>(arrs[q], c->d_stage, c->npoin, c->npad);
      c->launches++;
      if (cudaMemcpyAsync(buf.data(), c->d_stage, n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
          cudaStreamSynchronize(c->stream) != cudaSuccess) { std::fclose(fp); return fail(SMA_ERR_CUDA, "checkpoint copy"); }
      ok = std::fwrite(buf.data(), sizeof(double), n3, fp) == n3;
    }
    double en[16];
    if (ok && (cudaMemcpy(en, c->d_en, sizeof en, cudaMemcpyDeviceToHost) != cudaSuccess)) { std::fclose(fp); return fail(SMA_ERR_CUDA, "checkpoint copy"); }
    if (ok) ok = std::fwrite(en, sizeof(double), 16, fp) == 16;
  }
  if (std::fclose(fp) != 0) ok = false;
  if (!ok) return fail(SMA_ERR_ARG, std::string("short write to ") + path);
  return SMA_OK;
}

int32_t sma_checkpoint_load(sma_ctx* c, const char* path) {
  if (!c || !path) return fail(SMA_ERR_ARG, "NULL argument");
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(SMA_ERR_ARG, std::string("cannot read ") + path);
  CkptHeader hd;
  if (std::fread(&hd, sizeof hd, 1, fp) != 1 || std::memcmp(hd.magic, "SMAB200", 8) != 0 || hd.version != 1) {
    std::fclose(fp);
    return fail(SMA_ERR_ARG, "not an alya_sma_b200 checkpoint");
  }
  if (hd.nelem != c->nelem || hd.npoin != c->npoin || hd.precision != c->prec || hd.scheme != c->scheme) {
    std::fclose(fp);
    return fail(SMA_ERR_ARG, "checkpoint of another mesh, precision or scheme");
  }
  const size_t n3 = 3 * (size_t)c->npoin;
  std::vector<double> buf(std::max(n3, 48 * (size_t)c->nelem));
  const int fields[3] = {SMA_FIELD_DISPL, SMA_FIELD_VELOC, SMA_FIELD_ACCEL};
  int32_t rc;
  for (int q = 0; q < 3; ++q) {
    if (std::fread(buf.data(), sizeof(double), n3, fp) != n3) { std::fclose(fp); return fail(SMA_ERR_ARG, "truncated checkpoint"); }
    if ((rc = sma_set_nodal(c, fields[q], buf.data()))) { std::fclose(fp); return rc; }
  }
  if (std::fread(buf.data(), sizeof(double), 48 * (size_t)c->nelem, fp) != 48 * (size_t)c->nelem) {
    std::fclose(fp);
    return fail(SMA_ERR_ARG, "truncated checkpoint");
  }
  if ((rc = sma_set_state(c, buf.data()))) { std::fclose(fp); return rc; }
  if (hd.has_energy) {
    if ((rc = sma_set_energy(c, 1, c->ehist_max))) { std::fclose(fp); return rc; }
    double* arrs[3] = {c->d_uprev, c->d_fintp, c->d_fextp};
    for (int q = 0; q < 3; ++q) {
      if (std::fread(buf.data(), sizeof(double), n3, fp) != n3) { std::fclose(fp); return fail(SMA_ERR_ARG, "truncated checkpoint"); }
      CU(cudaMemcpyAsync(c->d_stage, buf.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      k_aos_to_soa<<<(unsigned)ceil_div(c->npoin, 256), 256, 0, c->stream>>>(c->d_stage, arrs[q], c->npoin, c->npad);
      c->launches++;
      CU(cudaStreamSynchronize(c->stream));
    }
    double en[16];
    if (std::fread(en, sizeof(double), 16, fp) != 16) { std::fclose(fp); return fail(SMA_ERR_ARG, "truncated checkpoint"); }
    CU(cudaMemcpy(c->d_en, en, sizeof en, cudaMemcpyHostToDevice));
  }
  std::fclose(fp);
  return sma_set_time(c, hd.cutim);
}

int32_t sma_critical_dt(sma_ctx* c, double* dtcri) {
  if (!c || !dtcri) return fail(SMA_ERR_ARG, "NULL argument");
  *dtcri = c->dtcri;
  return SMA_OK;
}

int32_t sma_set_timing(sma_ctx* c, int32_t enable) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  c->timing = enable != 0;
  for (int k = 0; k < 3; ++k) { c->tms[k] = 0.0; c->tcnt[k] = 0; }
  return SMA_OK;
}

int32_t sma_get_timers(sma_ctx* c, double* ms, int64_t* counts) {
  if (!c || !ms) return fail(SMA_ERR_ARG, "NULL argument");
  for (int k = 0; k < 3; ++k) {
    ms[k] = c->tms[k];
    if (counts) counts[k] = c->tcnt[k];
  }
  return SMA_OK;
}

void* sma_stream(sma_ctx* c) { return c ? (void*)c->stream : nullptr; }

int64_t sma_kernel_launches(sma_ctx* c) { return c ? c->launches : 0; }

// the element kernel's launch shape this context chose
int32_t sma_launch_info(sma_ctx* c, int32_t* block, int32_t* variant, int32_t* compact) {
  if (!c || !block || !variant || !compact) return fail(SMA_ERR_ARG, "NULL argument");
  *block = c->block;
  *variant = c->variant;
  *compact = c->compact ? 1 : 0;
  return SMA_OK;
}

int32_t sma_eval_law160(int64_t n, const double* props, double e_mart, const double* d_F,
                        const double* d_tmp, const double* d_sdv_old, double* d_sdv_new,
                        double* d_pk2, int32_t* d_nr_flag, int32_t precision, void* stream) {
  if (n < 0) return fail(SMA_ERR_ARG, "n < 0");
  if (n == 0) return SMA_OK;
  if (!props || !d_F || !d_sdv_old || !d_sdv_new || !d_pk2) return fail(SMA_ERR_ARG, "NULL argument");
  if (precision != SMA_PREC_FP64 && precision != SMA_PREC_FP32) return fail(SMA_ERR_ARG, "precision");
  const MatC m = make_mat(props, e_mart, 1.0);
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned grid = (unsigned)ceil_div(n, 128);
  if (precision == SMA_PREC_FP32)
    k_law_batch<float><<<grid, 128, 0, s>>>(n, m, d_F, d_tmp, d_sdv_old, d_sdv_new, d_pk2, d_nr_flag);
  else
    k_law_batch<double><<<grid, 128, 0, s>>>(n, m, d_F, d_tmp, d_sdv_old, d_sdv_new, d_pk2, d_nr_flag);
  CU(cudaGetLastError());
  return SMA_OK;
}

int32_t sma_eval_law160_tangent(int64_t n, const double* props, double e_mart, const double* d_F,
                                const double* d_tmp, const double* d_sdv_old, double* d_sdv_new,
                                double* d_pk2, double* d_dds, int32_t* d_nr_flag, void* stream) {
  if (n < 0) return fail(SMA_ERR_ARG, "n < 0");
  if (n == 0) return SMA_OK;
  if (!props || !d_F || !d_sdv_old || !d_sdv_new || !d_pk2 || !d_dds) return fail(SMA_ERR_ARG, "NULL argument");
  const MatC m = make_mat(props, e_mart, 1.0);
  k_law_tangent<<<(unsigned)ceil_div(n, 128), 128, 0, (cudaStream_t)stream>>>(
      n, m, d_F, d_tmp, d_sdv_old, d_sdv_new, d_pk2, d_dds, d_nr_flag);
  CU(cudaGetLastError());
  return SMA_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Element loop that allocates nothing.
//
// For callers that must not (or cannot) allocate device memory through the
// CUDA runtime: a Fortran host whose device arrays are owned by an OpenACC
// data region or a caller-side memory pool, or code running where a
// cudaMalloc would synchronise the device or break a caller's allocation
// budget.  The caller passes every input and output as a device pointer; the
// working set the element kernel needs beyond them (structure-of-arrays
// copies of coordinates and displacements, the FP64 force accumulator, the
// state in the kernel's layout, the material constants and the counters)
// lives in one file-scope device array of fixed size, reserved when the
// library is loaded and held by every GPU that loads it until the process
// exits.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t NA_NPAD = SMA_NOALLOC_MAX_NODES;          // multiple of 32
constexpr int64_t NA_SST = 8 * (int64_t)SMA_NOALLOC_MAX_ELEMS;
constexpr size_t NA_NODAL = 3 * (size_t)NA_NPAD * sizeof(double);
constexpr size_t NA_STATE = 3 * (size_t)NA_SST * sizeof(double);
constexpr size_t NA_OFF_COORD = 0;
constexpr size_t NA_OFF_U = NA_OFF_COORD + NA_NODAL;
constexpr size_t NA_OFF_F = NA_OFF_U + NA_NODAL;
constexpr size_t NA_OFF_S0 = NA_OFF_F + NA_NODAL;
constexpr size_t NA_OFF_S1 = NA_OFF_S0 + NA_STATE;
constexpr size_t NA_OFF_MAT = NA_OFF_S1 + NA_STATE;
constexpr size_t NA_OFF_CNT = NA_OFF_MAT + 256;
constexpr size_t NA_OFF_FLAG = NA_OFF_CNT + 256;
constexpr size_t NA_BYTES = NA_OFF_FLAG + 256;
static_assert(NA_NPAD % 32 == 0, "node capacity must be a multiple of 32");
static_assert(sizeof(MatC) <= 256, "material block");

__device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// device address of g_noalloc_scratch per device ordinal (host code cannot
// use the symbol's name as an address)
unsigned char* g_noalloc_ptr[64] = {nullptr};

__global__ void k_put_mat(MatC m, MatC* dst) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = m;
}

// flag = 1 if any node id of lnods lies outside [0, npoin)
__global__ void k_check_lnods(const int32_t* lnods, int64_t n, int32_t npoin, int32_t* flag) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    const int32_t v = lnods[k];
    if (v < 0 || v >= npoin) atomicOr(flag, 1);
  }
}

template <typename T>
int32_t noalloc_run(unsigned char* base, int32_t nelem, int32_t npoin, const int32_t* d_lnods,
                    double* d_sdv, const MatC& mat, cudaStream_t s) {
  const int64_t sst = ceil_div(8 * (int64_t)nelem, 32) * 32;
  T* s_iterk = (T*)(base + NA_OFF_S0);
  T* s_timen = (T*)(base + NA_OFF_S1);
  const unsigned sgrid = (unsigned)ceil_div(8 * (int64_t)nelem, 256);
  // the caller's slot TIME_N in, slot ITER_K out: the other slot is left as it is
  k_state_in<T><<<sgrid, 256, 0, s>>>(d_sdv, nullptr, nullptr, s_timen, nelem, sst);
  ElemArgs<T> a;
  std::memset(&a, 0, sizeof a);
  a.lnods = d_lnods;
  a.coord = (const double*)(base + NA_OFF_COORD);
  a.u = (const double*)(base + NA_OFF_U);
  a.f = (double*)(base + NA_OFF_F);
  a.lmate = nullptr;
  a.mats = (const MatC*)(base + NA_OFF_MAT);
  a.mat0 = mat;
  a.tempe = nullptr;
  a.sold = s_timen;
  a.snew = s_iterk;
  a.cnt = (unsigned long long*)(base + NA_OFF_CNT);
  a.ts = nullptr;
  a.ft = nullptr;
  a.npad = NA_NPAD;
  a.sst = sst;
  a.beg = 0;
  a.end = nelem;
  a.has_grav = 0;
  a.vel = nullptr;
  // the one-material narrow instance at one-warp blocks, as a context
  // with one material runs it by default
  const int block = 32, epb = block / 8;
  const size_t smem = element_smem_bytes<T>(block, false);      // below the 48 KB default
  k_element<T, true, false, false, true><<<(unsigned)ceil_div(nelem, epb), block, smem, s>>>(a);
  k_state_out<T><<<sgrid, 256, 0, s>>>(d_sdv, nullptr, s_iterk, nullptr, nelem, sst);
  CU(cudaGetLastError());
  return SMA_OK;
}

}  // namespace

extern "C" int32_t sma_assemble_noalloc(int32_t nelem, int32_t npoin, const int32_t* d_lnods,
                                        const double* d_coord, const double* d_displ,
                                        const double* props, double e_mart, double* d_sdv,
                                        double* d_rhsid, int32_t precision, void* stream) {
  if (nelem <= 0 || npoin <= 0) return fail(SMA_ERR_ARG, "nelem and npoin must be positive");
  if (npoin > SMA_NOALLOC_MAX_NODES || nelem > SMA_NOALLOC_MAX_ELEMS)
    return fail(SMA_ERR_ARG, "sma_assemble_noalloc: mesh of " + std::to_string(nelem) + " elements, " +
                                 std::to_string(npoin) + " nodes exceeds the fixed scratch capacity of " +
                                 std::to_string(SMA_NOALLOC_MAX_ELEMS) + " elements and " +
                                 std::to_string(SMA_NOALLOC_MAX_NODES) + " nodes");
  if (!d_lnods || !d_coord || !d_displ || !props || !d_sdv || !d_rhsid)
    return fail(SMA_ERR_ARG, "NULL argument");
  if (precision != SMA_PREC_FP64 && precision != SMA_PREC_FP32) return fail(SMA_ERR_ARG, "precision");
  if (!(props[0] > 0.0) || !(props[1] > -1.0 && props[1] < 0.5))
    return fail(SMA_ERR_ARG, "material: need E > 0, -1 < nu < 0.5");
  int dev = 0;
  CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SMA_ERR_ARG, "device ordinal beyond 63");
  if (!g_noalloc_ptr[dev]) {
    // set-up, once per device, with that device current
    void* p = nullptr;
    CU(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    CU(cudaFuncSetAttribute(k_element<double, true, false, false, true>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, 48 * 1024));
    CU(cudaFuncSetAttribute(k_element<float, true, false, false, true>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, 48 * 1024));
    g_noalloc_ptr[dev] = (unsigned char*)p;
  }
  unsigned char* base = g_noalloc_ptr[dev];
  cudaStream_t s = (cudaStream_t)stream;
  // reject node ids outside [0, npoin) before any kernel dereferences them
  int32_t* d_flag = (int32_t*)(base + NA_OFF_FLAG);
  CU(cudaMemsetAsync(d_flag, 0, sizeof(int32_t), s));
  k_check_lnods<<<(unsigned)ceil_div(8 * (int64_t)nelem, 256), 256, 0, s>>>(d_lnods, 8 * (int64_t)nelem,
                                                                           npoin, d_flag);
  CU(cudaGetLastError());
  int32_t bad = 0;
  CU(cudaMemcpyAsync(&bad, d_flag, sizeof bad, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (bad) return fail(SMA_ERR_ARG, "lnods holds node ids outside [0, npoin)");
  // the scratch keeps the previous call's contents: clear what accumulates,
  // and mark "no det F <= 0 seen" as the context does (all ones)
  CU(cudaMemsetAsync(base + NA_OFF_F, 0, NA_NODAL, s));
  CU(cudaMemsetAsync(base + NA_OFF_CNT, 0, 256, s));
  CU(cudaMemsetAsync(base + NA_OFF_CNT + CNT_DETMIN * sizeof(unsigned long long), 0xff,
                     sizeof(unsigned long long), s));
  const unsigned ngrid = (unsigned)ceil_div(npoin, 256);
  k_aos_to_soa<<<ngrid, 256, 0, s>>>(d_coord, (double*)(base + NA_OFF_COORD), npoin, NA_NPAD);
  k_aos_to_soa<<<ngrid, 256, 0, s>>>(d_displ, (double*)(base + NA_OFF_U), npoin, NA_NPAD);
  const MatC mat = make_mat(props, e_mart, 1.0);
  k_put_mat<<<1, 1, 0, s>>>(mat, (MatC*)(base + NA_OFF_MAT));
  CU(cudaGetLastError());
  int32_t rc = (precision == SMA_PREC_FP32)
                   ? noalloc_run<float>(base, nelem, npoin, d_lnods, d_sdv, mat, s)
                   : noalloc_run<double>(base, nelem, npoin, d_lnods, d_sdv, mat, s);
  if (rc) return rc;
  k_soa_to_aos<<<ngrid, 256, 0, s>>>((const double*)(base + NA_OFF_F), d_rhsid, npoin, NA_NPAD);
  CU(cudaGetLastError());
  return SMA_OK;
}

// The counters of the last sma_assemble_noalloc call on the current device,
// read from the fixed array on `stream` (synchronised): return-map
// activations and failures, both transformations active, Gauss points with
// det F <= 0 with the smallest such det F and its element, in the numbering
// the caller passed (the no-alloc path keeps it).
extern "C" int32_t sma_noalloc_counters(sma_counters* out, void* stream) {
  if (!out) return fail(SMA_ERR_ARG, "NULL argument");
  int dev = 0;
  CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || !g_noalloc_ptr[dev])
    return fail(SMA_ERR_STATE, "no sma_assemble_noalloc call on this device yet");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned long long h[NCNT];
  CU(cudaMemcpyAsync(h, g_noalloc_ptr[dev] + NA_OFF_CNT, sizeof h, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  for (int k = 0; k < SMA_NCOUNTERS; ++k) out->c[k] = (k < CNT_DETMIN) ? (int64_t)h[k] : 0;
  const unsigned long long dm = h[CNT_DETMIN];
  if (dm == ~0ull) {
    out->gpdet_min = 0.0;
    out->ielem_min = -1;
  } else {
    const unsigned key = (unsigned)(dm >> 32);
    const unsigned bits = (key & 0x80000000u) ? (key & 0x7fffffffu) : ~key;
    float det;
    std::memcpy(&det, &bits, sizeof det);
    out->gpdet_min = det;
    out->ielem_min = (int64_t)(dm & 0xffffffffull);
  }
  return SMA_OK;
}

// ---------------------------------------------------------------------------
// the learned surrogate in the element loop
// ---------------------------------------------------------------------------
extern "C" int32_t sma_set_surrogate(sma_ctx* c, const float* params, const sma_sur_stats* stats, double gate,
                                     double xs_tol, double f_margin, int32_t period, int32_t enable) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  CU(cudaSetDevice(c->dev));
  if (!enable) {
    if (c->sur) destroy_graphs(c);
    c->sur = false;
    return SMA_OK;
  }
  if (!params || !stats) return fail(SMA_ERR_ARG, "NULL argument");
  if (c->prec != SMA_PREC_FP32) return fail(SMA_ERR_ARG, "the surrogate runs in the FP32 precision form");
  if (c->scatter != SMA_SCATTER_ATOMIC) return fail(SMA_ERR_ARG, "the surrogate element loop scatters by atomics");
  if (c->damp) return fail(SMA_ERR_ARG, "the surrogate element loop has no Rayleigh damping");
  if (c->d_lmate && !c->compact)
    return fail(SMA_ERR_ARG, "per-element materials need compact records for the surrogate");
  if (!(gate > 0.0) || !(xs_tol >= 0.0) || !(f_margin >= 0.0) || period < 1)
    return fail(SMA_ERR_ARG, "gate > 0, xs_tol >= 0, f_margin >= 0, period >= 1");
  for (int k = 0; k < SMA_SUR_NPARAM; ++k)
    if (!std::isfinite(params[k])) return fail(SMA_ERR_ARG, "non-finite surrogate parameter");
  int32_t rc;
  if (!c->d_sur_img) {
    if ((rc = dalloc(&c->d_sur_img, sur::IMG_BYTES))) return rc;
    if ((rc = dalloc(&c->d_sur_stats, sizeof(sur::SurStats)))) return rc;
    if ((rc = dalloc(&c->d_sur_ctr, 2 * sizeof(int)))) return rc;
    if ((rc = dalloc(&c->d_rcache, 6 * (size_t)c->sst * sizeof(__half)))) return rc;
    CU(cudaFuncSetAttribute(sur::k_sur_refresh, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)sur::mlp_smem_bytes()));
  }
  // staging rows: the due tiles of one step, ceil(tiles / period)
  const int64_t ntiles = ceil_div(c->nelem, sur::SUR_EPB);
  const int64_t slots = ceil_div(ntiles, period);
  if (slots > c->xstage_slots) {
    if (c->d_xstage) cudaFree(c->d_xstage);
    c->d_xstage = nullptr;
    c->xstage_slots = 0;
    if ((rc = dalloc(&c->d_xstage, (size_t)slots * sur::NIN * sur::SUR_BLOCK * sizeof(float)))) return rc;
    c->xstage_slots = slots;
  }
  // the network kernel's persistent grid: blocks per SM by the occupancy
  // query, or by its register and shared-memory needs against the SM's
  // limits where that allows more (no block waits for another)
  int per_sm = 0;
  CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sur::k_sur_refresh, sur::SUR_BLOCK,
                                                   sur::mlp_smem_bytes()));
  {
    cudaFuncAttributes fa;
    int regs_sm = 0, smem_sm = 0, smem_res = 0;
    CU(cudaFuncGetAttributes(&fa, sur::k_sur_refresh));
    CU(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, c->dev));
    CU(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->dev));
    CU(cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, c->dev));
    const int warp_regs = (fa.numRegs * 32 + 255) / 256 * 256;         // allocated per warp in 256s
    const int by_regs = regs_sm / (warp_regs * (sur::SUR_BLOCK / 32));
    const int by_smem = (int)((size_t)smem_sm / (sur::mlp_smem_bytes() + fa.sharedSizeBytes + smem_res));
    per_sm = std::max(per_sm, std::min(by_regs, by_smem));
  }
  if (per_sm < 1) return fail(SMA_ERR_ARG, "surrogate network kernel does not fit on an SM");
  c->sur_grid = c->nsm * per_sm;
  c->sur_gate = (float)gate;
  c->sur_xs_tol = (float)xs_tol;
  c->sur_margin = (float)f_margin;
  c->sur_period = period;
  // parameters through the staging buffer (>= 14,608 floats for any mesh of
  // at least 1,218 nodes; else a temporary), packed into the weight image
  float* d_w = nullptr;
  const bool stage = 3 * (size_t)c->npoin * sizeof(double) >= SMA_SUR_NPARAM * sizeof(float);
  if (stage) d_w = reinterpret_cast<float*>(c->d_stage);
  else if ((rc = dalloc(&d_w, SMA_SUR_NPARAM * sizeof(float)))) return rc;
  CU(cudaMemcpyAsync(d_w, params, SMA_SUR_NPARAM * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CU(cudaMemsetAsync(c->d_sur_img, 0, sur::IMG_BYTES, c->stream));
  sur::k_sur_pack_image<<<(sur::HID * sur::HID + 255) / 256, 256, 0, c->stream>>>(d_w, c->d_sur_img);
  CU(cudaMemcpyAsync(c->d_sur_stats, stats, sizeof(sur::SurStats), cudaMemcpyHostToDevice, c->stream));
  CU(cudaMemsetAsync(c->d_sur_ctr, 0, 2 * sizeof(int), c->stream));
  if ((rc = sur_init_residuals(c))) return rc;
  CU(cudaStreamSynchronize(c->stream));
  if (!stage) cudaFree(d_w);
  destroy_graphs(c);
  c->sur = true;
  return SMA_OK;
}

// status of the surrogate element loop since it was switched on: 1 if a wait
// for the tensor cores ran out (the results of that launch are incomplete)
extern "C" int32_t sma_surrogate_status(sma_ctx* c, int32_t* status) {
  if (!c || !status) return fail(SMA_ERR_ARG, "NULL argument");
  if (!c->d_sur_ctr) {
    *status = 0;
    return SMA_OK;
  }
  CU(cudaSetDevice(c->dev));
  CU(cudaMemcpyAsync(status, c->d_sur_ctr + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return SMA_OK;
}

// Launch plan of the element loop: nrange element ranges [end[r-1], end[r])
// (end increasing, the last = nelem) each launched with its own threads per
// block -- the ensemble's specimen-size buckets, tuned one by one.  One-tile
// kernel with the atomic scatter only; nrange = 0 returns to one launch.
extern "C" int32_t sma_set_launch_plan(sma_ctx* c, int32_t nrange, const int32_t* end, const int32_t* block) {
  if (!c) return fail(SMA_ERR_ARG, "NULL context");
  if (nrange < 0) return fail(SMA_ERR_ARG, "nrange < 0");
  if (nrange == 0) {
    c->plan_end.clear();
    c->plan_block.clear();
    destroy_graphs(c);
    return SMA_OK;
  }
  if (!end || !block) return fail(SMA_ERR_ARG, "NULL argument");
  if (c->scatter != SMA_SCATTER_ATOMIC || c->variant != SMA_VARIANT_PLAIN)
    return fail(SMA_ERR_ARG, "launch plans need the atomic scatter and the one-tile kernel");
  int prev = 0;
  for (int r = 0; r < nrange; ++r) {
    if (end[r] < prev || end[r] > c->nelem) return fail(SMA_ERR_ARG, "plan ends must increase within nelem");
    if (block[r] % 32 != 0 || block[r] < 32 || block[r] > 256)
      return fail(SMA_ERR_ARG, "plan blocks must be multiples of 32 in [32, 256]");
    prev = end[r];
  }
  if (end[nrange - 1] != c->nelem) return fail(SMA_ERR_ARG, "the last plan range must end at nelem");
  CU(cudaSetDevice(c->dev));
  c->plan_end.assign(end, end + nrange);
  c->plan_block.assign(block, block + nrange);
  destroy_graphs(c);
  return SMA_OK;
}
