// sma_surrogate.cu -- C ABI of the learned constitutive surrogate's
// standalone kernels: plain-law data generation, BF16 tensor-core training
// (forward + backward + weight gradients), Adam, weight packing and the
// tcgen05 batched inference.  Every pointer named d_* is a device pointer
// the caller owns; calls are ordered on `stream` (NULL: default stream).
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "alya_sma.h"
#include "sma_surrogate.cuh"

using namespace sma;

namespace {

thread_local std::string g_err_sur;

int32_t sfail(int32_t code, const std::string& msg);

#define SCU(call)                                                                   \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      cudaGetLastError();                                                           \
      return sfail(SMA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    }                                                                               \
  } while (0)

}  // namespace

// the library's error text (sma_capi.cu)
extern "C" int32_t sma_set_error_(int32_t code, const char* msg);

namespace {
int32_t sfail(int32_t code, const std::string& msg) { return sma_set_error_(code, msg.c_str()); }

MatC base_material(const double* pr, double e_mart) {
  MatC m;
  std::memset(&m, 0, sizeof m);
  const double E = pr[0], v = pr[1];
  m.eL = pr[2];
  m.alfa = pr[14];
  m.C_AS = pr[5];
  m.C_SA = pr[11];
  m.K = E / (3.0 - 6.0 * v);
  m.G = E / (2.0 + 2.0 * v);
  m.G1 = (2.0 * m.G + 9.0 * (m.alfa * m.alfa) * m.K) * m.eL;
  m.EA = E;
  m.EM = (e_mart > 0.0) ? e_mart : E;
  m.nu = v;
  m.iEA = 1.0 / m.EA;
  m.iEM = 1.0 / m.EM;
  m.kK = 1.0 / (3.0 - 6.0 * v);
  m.kG = 1.0 / (2.0 + 2.0 * v);
  m.ext_E = 1;
  return m;
}
}  // namespace

static_assert(sizeof(sma_sur_stats) == sizeof(sur::SurStats), "stats layout");

extern "C" {

int32_t sma_sur_generate(int64_t npath, int32_t nstep, uint64_t seed, const double* props, double e_mart,
                         double spread, double t_lo, double t_hi, double e_lo, double e_hi, double shear,
                         int32_t nseg, float* d_x, float* d_y, void* stream) {
  if (npath <= 0 || nstep <= 0 || nseg <= 0 || nseg > nstep) return sfail(SMA_ERR_ARG, "npath, nstep, nseg");
  if (!props || !d_x || !d_y) return sfail(SMA_ERR_ARG, "NULL argument");
  if (!(props[0] > 0.0) || !(props[1] > -1.0 && props[1] < 0.5)) return sfail(SMA_ERR_ARG, "material");
  if (!(spread >= 0.0 && spread < 1.0) || !(t_hi >= t_lo) || !(e_hi >= e_lo) || !(shear >= 0.0))
    return sfail(SMA_ERR_ARG, "sampling ranges");
  sur::GenArgs g;
  std::memset(&g, 0, sizeof g);
  g.base = base_material(props, e_mart);
  g.EA = g.base.EA;
  g.EM = g.base.EM;
  g.eL = props[2];
  g.Ss_AS = props[3];
  g.Sf_AS = props[4];
  g.Tf_AS = props[6];
  g.Ts_AS = props[7];
  g.Ss_SA = props[9];
  g.Sf_SA = props[10];
  g.Tf_SA = props[12];
  g.Ts_SA = props[13];
  g.spread = spread;
  g.t_lo = t_lo;
  g.t_hi = t_hi;
  g.e_lo = e_lo;
  g.e_hi = e_hi;
  g.shear = shear;
  g.nseg = nseg;
  g.nstep = nstep;
  g.npath = npath;
  g.seed = seed;
  g.x = d_x;
  g.y = d_y;
  sur::k_sur_generate<<<(unsigned)((npath + 127) / 128), 128, 0, (cudaStream_t)stream>>>(g);
  SCU(cudaGetLastError());
  return SMA_OK;
}

int32_t sma_sur_train_step(const uint16_t* d_wb, const float* d_w, const sma_sur_stats* d_stats, int64_t n,
                           const float* d_x, const float* d_y, float* d_grad, float* d_loss, void* stream) {
  if (n <= 0) return sfail(SMA_ERR_ARG, "empty batch");
  if (!d_wb || !d_w || !d_stats || !d_x || !d_y || !d_grad || !d_loss) return sfail(SMA_ERR_ARG, "NULL argument");
  static bool attr = false;
  const size_t smem = sizeof(sur::TrainSmem);
  if (!attr) {
    SCU(cudaFuncSetAttribute(sur::k_sur_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  int dev = 0, nsm = 148;
  SCU(cudaGetDevice(&dev));
  SCU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int64_t tiles = (n + 127) / 128;
  const unsigned grid = (unsigned)(tiles < nsm ? tiles : nsm);
  sur::TrainArgs a;
  a.wb = reinterpret_cast<const __nv_bfloat16*>(d_wb);
  a.w = d_w;
  a.stats = reinterpret_cast<const sur::SurStats*>(d_stats);
  a.x = d_x;
  a.y = d_y;
  a.n = n;
  a.grad = d_grad;
  a.loss = d_loss;
  sur::k_sur_train<<<grid, 128, smem, (cudaStream_t)stream>>>(a);
  SCU(cudaGetLastError());
  return SMA_OK;
}

int32_t sma_sur_adam(float* d_w, float* d_m, float* d_v, const float* d_grad, uint16_t* d_wb, float lr, float b1,
                     float b2, float eps, int32_t t, void* stream) {
  if (!d_w || !d_m || !d_v || !d_grad || !d_wb) return sfail(SMA_ERR_ARG, "NULL argument");
  if (t < 1 || !(lr > 0.f) || !(b1 >= 0.f && b1 < 1.f) || !(b2 >= 0.f && b2 < 1.f) || !(eps > 0.f))
    return sfail(SMA_ERR_ARG, "Adam hyper-parameters");
  sur::k_sur_adam<<<(sur::NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      d_w, d_m, d_v, d_grad, reinterpret_cast<__nv_bfloat16*>(d_wb), lr, b1, b2, eps, t);
  SCU(cudaGetLastError());
  return SMA_OK;
}

int32_t sma_sur_pack(const float* d_w, uint16_t* d_wb, unsigned char* d_img, void* stream) {
  if (!d_w) return sfail(SMA_ERR_ARG, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (d_wb) sur::k_sur_to_bf16<<<(sur::NPARAM + 255) / 256, 256, 0, s>>>(d_w, reinterpret_cast<__nv_bfloat16*>(d_wb));
  if (d_img) {
    SCU(cudaMemsetAsync(d_img, 0, sur::IMG_BYTES, s));
    sur::k_sur_pack_image<<<(sur::HID * sur::HID + 255) / 256, 256, 0, s>>>(d_w, d_img);
  }
  SCU(cudaGetLastError());
  return SMA_OK;
}

int32_t sma_sur_forward(const unsigned char* d_img, const sma_sur_stats* d_stats, int64_t n, const float* d_x,
                        float* d_y, float* d_score, int32_t* d_status, void* stream) {
  if (n <= 0) return sfail(SMA_ERR_ARG, "empty batch");
  if (!d_img || !d_stats || !d_x || !d_y || !d_status) return sfail(SMA_ERR_ARG, "NULL argument");
  if (((uintptr_t)d_img & 15) != 0) return sfail(SMA_ERR_ARG, "weight image must be 16-byte aligned");
  static bool attr = false;
  const size_t smem = sur::mlp_smem_bytes();
  if (!attr) {
    SCU(cudaFuncSetAttribute(sur::k_sur_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  int dev = 0, nsm = 148;
  SCU(cudaGetDevice(&dev));
  SCU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int64_t tiles = (n + 127) / 128;
  const int64_t cap = (int64_t)nsm * 3;
  const unsigned grid = (unsigned)(tiles < cap ? tiles : cap);
  sur::k_sur_forward<<<grid, 128, smem, (cudaStream_t)stream>>>(
      d_img, reinterpret_cast<const sur::SurStats*>(d_stats), n, d_x, d_y, d_score, d_status);
  SCU(cudaGetLastError());
  return SMA_OK;
}

int32_t sma_sur_wait_check(int32_t tries, int32_t* status) {
  if (!status) return sfail(SMA_ERR_ARG, "NULL argument");
  if (tries < 1 || tries > (1 << 20)) return sfail(SMA_ERR_ARG, "tries in [1, 2^20]");
  int* d = nullptr;
  SCU(cudaMalloc(&d, sizeof(int)));
  SCU(cudaMemset(d, 0xff, sizeof(int)));
  sur::k_sur_wait_check<<<1, 32>>>(tries, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(status, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return sfail(SMA_ERR_CUDA, cudaGetErrorString(e));
  return SMA_OK;
}

}  // extern "C"
