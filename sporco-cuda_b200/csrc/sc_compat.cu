// Reference-compatible C ABI: the entry points the reference's Cython layer
// binds (sporco_cuda/cbpdn.pyx:47-53, sporco_cuda/util.pyx:3-7), with the
// same names, argument meaning and AlgOpt layout, implemented on top of the
// native sc_* solver.  Host buffers in and out, as in the reference; device
// memory comes from the CUDA stream-ordered pool (cudaMallocAsync), which
// keeps freed blocks cached so repeated calls do not pay for allocation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/sporco_b200.h"

extern "C" {

// utils.cu:66-98: -1 marks a field as unset.  Unlike the reference this
// allocates nothing (the reference's two calloc'd pointers leak).
void clear_opts(void* data) {
  AlgOpt* opt = (AlgOpt*)data;
  memset(opt, 0, sizeof(*opt));
  opt->device = -1;
  opt->rho = -1;
  opt->Verbose = -1;
  opt->AutoRho = -1;
  opt->L1Weight = nullptr;
  opt->Weight = nullptr;
  opt->nWeight = -1;
  opt->AuxVarObj = -1;
  opt->AbsStopTol = -1;
  opt->NonNegCoef = -1;
  opt->RelaxParam = -1;
  opt->RhoScaling = -1;
  opt->RelStopTol = -1;
  opt->MaxMainIter = -1;
  opt->NoBndryCross = -1;
  opt->HighMemSolve = -1;
  opt->StdResiduals = -1;
  opt->RhoRsdlRatio = -1;
  opt->RhoRsdlTarget = -1;
  opt->AutoRhoPeriod = -1;
  opt->AutoRhoScaling = -1;
  opt->L1_WEIGHT_M_SIZE = opt->L1_WEIGHT_ROW_SIZE = opt->L1_WEIGHT_COL_SIZE = 1;
  opt->WEIGHT_SIZE = 1;
}

// utils.cu:12-64: defaults for fields still at -1.
void default_opts(void* data) {
  AlgOpt* opt = (AlgOpt*)data;
  if (opt->device == -1) opt->device = 0;
  if (opt->rho == -1) opt->rho = 0;
  if (opt->Verbose == -1) opt->Verbose = 0;
  if (opt->AutoRho == -1) opt->AutoRho = 1;
  if (opt->nWeight == -1) opt->nWeight = 1;
  if (opt->AuxVarObj == -1) opt->AuxVarObj = 0;
  if (opt->AbsStopTol == -1) opt->AbsStopTol = 0;
  if (opt->NonNegCoef == -1) opt->NonNegCoef = 0;
  if (opt->RelaxParam == -1) opt->RelaxParam = 1.8f;
  if (opt->RhoScaling == -1) opt->RhoScaling = 100;
  if (opt->RelStopTol == -1) opt->RelStopTol = 1e-4f;
  if (opt->MaxMainIter == -1) opt->MaxMainIter = 250;
  if (opt->NoBndryCross == -1) opt->NoBndryCross = 0;
  if (opt->HighMemSolve == -1) opt->HighMemSolve = 0;
  if (opt->StdResiduals == -1) opt->StdResiduals = 0;
  if (opt->RhoRsdlRatio == -1) opt->RhoRsdlRatio = 1.2f;
  if (opt->AutoRhoPeriod == -1) opt->AutoRhoPeriod = 1;
  if (opt->AutoRhoScaling == -1) opt->AutoRhoScaling = 1;
}

// utils.cu:100-144, returning -1 instead of exiting the process.
int check_cuda_req(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return -1;
  if (device < 0 || device >= n) return -1;
  int major = 0;  // (one attribute: the full property query is slow per call)
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess)
    return -1;
  if (major < 10) return -1;  // this build carries sm_100a code only
  return device;
}

int get_device_count(void) {
  int n = 0;
  return cudaGetDeviceCount(&n) == cudaSuccess ? n : 0;
}
int get_current_device(int* dev) { return (int)cudaGetDevice(dev); }
int set_current_device(int dev) { return (int)cudaSetDevice(dev); }
int get_memory_info(size_t* free_bytes, size_t* total_bytes) {
  return (int)cudaMemGetInfo(free_bytes, total_bytes);
}
const char* get_device_name(int dev) {
  static thread_local cudaDeviceProp cdp;
  return cudaGetDeviceProperties(&cdp, dev) == cudaSuccess ? cdp.name : nullptr;
}

}  // extern "C"

// Defined in sc_solver.cu: records a status on the calling thread.
int sc_set_status_external(int st, const char* msg);

namespace {

struct DevBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  ~DevBuf() {
    if (p) cudaFreeAsync(p, s);
  }
};

bool g_pool_ready[64] = {false};

void keep_pool_cached(int dev) {
  if (dev < 0 || dev >= 64 || g_pool_ready[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  g_pool_ready[dev] = true;
}

int record(int st, const char* msg) { return sc_set_status_external(st, msg); }

#define COMPAT_TRY(call)                                                   \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      char b_[256];                                                        \
      snprintf(b_, sizeof(b_), "%s: %s", #call, cudaGetErrorString(e_));   \
      record(e_ == cudaErrorMemoryAllocation ? SC_ERR_OOM : SC_ERR_CUDA, b_); \
      return;                                                              \
    }                                                                      \
  } while (0)

void print_itstat(const std::vector<double>& it, int iters, int grd) {
  // The reference's Verbose table (cbpdn.cu:309-312, 438-517): iteration,
  // functional, data fidelity, L1 term, r, s, rho; here all recorded on the
  // device during the solve (the functional at Y).
  const char* sep =
      "-------------------------------------------------------------------";
  printf("Itn   Fnc       DFid      Regl1     r         s         %s\n%s\n",
         grd ? "rho (grd) " : "rho", sep);
  for (int k = 0; k < iters; ++k) {
    const double* v = &it[(size_t)k * SC_ITSTAT_FIELDS];
    printf("%4d %9.2e %9.2e %9.2e %9.2e %9.2e %9.2e\n", k, v[5], v[6], v[7], v[0], v[1], v[2]);
  }
  printf("%s\n", sep);
}

// Device-to-host copy into a pageable buffer (the caller's numpy array).
// A plain cudaMemcpy to pageable memory goes through the driver's staging at
// a few GB/s, and a fresh array also pays one page fault per 4 KB on first
// touch.  Here the data comes over in chunks by DMA into two page-locked
// staging buffers (allocated once per process, 2 x 64 MB) while host
// threads copy the previous chunk into the destination in parallel, taking
// its page faults in parallel too.
constexpr size_t kStageBytes = (size_t)64 << 20;
std::mutex g_stage_mu;
void* g_stage[2] = {nullptr, nullptr};

cudaError_t d2h_pageable(void* dst, const void* src, size_t n, cudaStream_t s) {
  if (n < ((size_t)8 << 20)) return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, s);
  std::lock_guard<std::mutex> lock(g_stage_mu);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && e == cudaSuccess; ++i)
    if (!g_stage[i]) e = cudaHostAlloc(&g_stage[i], kStageBytes, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, s);
  }
  cudaEvent_t ev[2];
  for (int i = 0; i < 2; ++i)
    if ((e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming)) != cudaSuccess) return e;
  const size_t nch = (n + kStageBytes - 1) / kStageBytes;
  const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  auto issue = [&](size_t k) -> cudaError_t {
    const size_t off = k * kStageBytes, len = std::min(kStageBytes, n - off);
    cudaError_t r = cudaMemcpyAsync(g_stage[k & 1], (const char*)src + off, len,
                                    cudaMemcpyDeviceToHost, s);
    return r == cudaSuccess ? cudaEventRecord(ev[k & 1], s) : r;
  };
  e = issue(0);
  for (size_t k = 0; k < nch && e == cudaSuccess; ++k) {
    if (k + 1 < nch && (e = issue(k + 1)) != cudaSuccess) break;
    if ((e = cudaEventSynchronize(ev[k & 1])) != cudaSuccess) break;
    const size_t off = k * kStageBytes, len = std::min(kStageBytes, n - off);
    const size_t part = (len + hw - 1) / hw;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < hw; ++t) {
      const size_t a0 = t * part;
      if (a0 >= len) break;
      const size_t l = std::min(part, len - a0);
      th.emplace_back([=] { memcpy((char*)dst + off + a0, (const char*)g_stage[k & 1] + a0, l); });
    }
    for (auto& x : th) x.join();
  }
  for (int i = 0; i < 2; ++i) cudaEventDestroy(ev[i]);
  return e;
}

void run_compat(float* D, float* S, float lambda, float mu, void* vopt, float* Yout, int grd) {
  AlgOpt* opt = (AlgOpt*)vopt;
  record(SC_OK, "");
  if (!opt || !D || !S || !Yout) {
    record(SC_ERR_INVALID, "null argument");
    return;
  }
  default_opts(opt);
  if (check_cuda_req(opt->device) < 0) {
    record(SC_ERR_CUDA, "no usable CUDA device (sm_100 required)");
    return;
  }
  COMPAT_TRY(cudaSetDevice(opt->device));
  keep_pool_cached(opt->device);
  const int H = opt->IMG_ROW_SIZE, W = opt->IMG_COL_SIZE, M = opt->DICT_M_SIZE;
  const int Kr = opt->DICT_ROW_SIZE, Kc = opt->DICT_COL_SIZE;
  if (H < 1 || W < 1 || M < 1 || Kr < 1 || Kc < 1) {
    record(SC_ERR_INVALID, "invalid sizes in AlgOpt");
    return;
  }
  cudaStream_t s = nullptr;  // legacy default stream, as the reference

  sc_problem p = {};
  p.B = 1; p.H = H; p.W = W; p.M = M; p.Kr = Kr; p.Kc = Kc;
  p.grd = grd; p.mu = mu;
  sc_options o;
  sc_options_from_algopt(opt, &o);

  // L1 weight: scalar, per map, or an (M, Hw, Ww) array broadcast to
  // (M, H, W) (cbpdn.pyx:181-193 passes (M, Hw, Ww) after rollaxis).
  const int wm = std::max(1, opt->L1_WEIGHT_M_SIZE), wh = std::max(1, opt->L1_WEIGHT_ROW_SIZE),
            ww = std::max(1, opt->L1_WEIGHT_COL_SIZE);
  std::vector<float> l1host;
  if (!opt->L1Weight) {
    p.l1_kind = SC_L1_SCALAR;
    p.l1_scalar = 1.f;
  } else if ((long)wm * wh * ww == 1) {
    p.l1_kind = SC_L1_SCALAR;
    p.l1_scalar = opt->L1Weight[0];
  } else if (wh == 1 && ww == 1 && wm == M) {
    p.l1_kind = SC_L1_PER_MAP;
    l1host.assign(opt->L1Weight, opt->L1Weight + M);
  } else {
    if ((wm != 1 && wm != M) || (wh != 1 && wh != H) || (ww != 1 && ww != W)) {
      record(SC_ERR_INVALID, "L1Weight shape does not broadcast to the coefficient maps");
      return;
    }
    p.l1_kind = SC_L1_FULL;
    l1host.resize((size_t)M * H * W);
    for (int m = 0; m < M; ++m)
      for (int h = 0; h < H; ++h)
        for (int w = 0; w < W; ++w)
          l1host[((size_t)m * H + h) * W + w] =
              opt->L1Weight[((size_t)(wm == 1 ? 0 : m) * wh + (wh == 1 ? 0 : h)) * ww + (ww == 1 ? 0 : w)];
  }
  std::vector<float> gwhost;
  if (grd) {
    const int nw = std::max(1, opt->WEIGHT_SIZE);
    if (nw != 1 && nw != M) {
      record(SC_ERR_INVALID, "GradWeight must have 1 or M entries");
      return;
    }
    gwhost.resize(M);
    for (int m = 0; m < M; ++m) gwhost[m] = opt->GrdWeight ? opt->GrdWeight[nw == 1 ? 0 : m] : 1.f;
    p.wgrd_uniform = 1;
    for (int m = 1; m < M; ++m)
      if (gwhost[m] != gwhost[0]) p.wgrd_uniform = 0;
  }
  const bool masked = opt->nWeight > 1 && opt->Weight;
  if (masked && opt->nWeight != H * W) {
    record(SC_ERR_INVALID, "mask size differs from the image size");
    return;
  }
  const float rho0 = opt->rho;

  // one device block: D, S, lam, rho0, l1w, gw, mask, Y, workspace
  size_t sz_D = sizeof(float) * (size_t)M * Kr * Kc, sz_S = sizeof(float) * (size_t)H * W;
  size_t sz_Y = sizeof(float) * (size_t)M * H * W;
  size_t sz_l1 = sizeof(float) * l1host.size(), sz_gw = sizeof(float) * gwhost.size();
  size_t sz_mask = masked ? sizeof(int32_t) * (size_t)H * W : 0;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  // workspace size needs pointers only for validation: plan with dummies
  p.D = (const float*)1; p.S = (const float*)1; p.lmbda = (const float*)1; p.rho0 = (const float*)1;
  p.Y = (float*)1; p.wgrd = grd ? (const float*)1 : nullptr; p.l1w = (const float*)1;
  size_t ws = sc_workspace_size(&p, &o);
  if (ws == 0) return;  // status already recorded
  size_t off_D = 0, off_S = off_D + al(sz_D), off_sc = off_S + al(sz_S), off_l1 = off_sc + 256,
         off_gw = off_l1 + al(sz_l1), off_mask = off_gw + al(sz_gw), off_Y = off_mask + al(sz_mask),
         off_ws = off_Y + al(sz_Y), total = off_ws + al(ws);
  DevBuf buf;
  buf.s = s;
  COMPAT_TRY(cudaMallocAsync(&buf.p, total, s));
  unsigned char* base = (unsigned char*)buf.p;
  float scal[2] = {lambda, rho0};
  COMPAT_TRY(cudaMemcpyAsync(base + off_D, D, sz_D, cudaMemcpyHostToDevice, s));
  COMPAT_TRY(cudaMemcpyAsync(base + off_S, S, sz_S, cudaMemcpyHostToDevice, s));
  COMPAT_TRY(cudaMemcpyAsync(base + off_sc, scal, sizeof(scal), cudaMemcpyHostToDevice, s));
  if (sz_l1) COMPAT_TRY(cudaMemcpyAsync(base + off_l1, l1host.data(), sz_l1, cudaMemcpyHostToDevice, s));
  if (sz_gw) COMPAT_TRY(cudaMemcpyAsync(base + off_gw, gwhost.data(), sz_gw, cudaMemcpyHostToDevice, s));
  if (sz_mask) COMPAT_TRY(cudaMemcpyAsync(base + off_mask, opt->Weight, sz_mask, cudaMemcpyHostToDevice, s));
  p.D = (const float*)(base + off_D);
  p.S = (const float*)(base + off_S);
  p.lmbda = (const float*)(base + off_sc);
  p.rho0 = (const float*)(base + off_sc) + 1;
  p.l1w = sz_l1 ? (const float*)(base + off_l1) : nullptr;
  p.wgrd = grd ? (const float*)(base + off_gw) : nullptr;
  p.mask = masked ? (const int32_t*)(base + off_mask) : nullptr;
  p.Y = (float*)(base + off_Y);
  sc_result res;
  int st = sc_cbpdn_solve(&p, &o, base + off_ws, ws, &res, s);
  if (st != SC_OK) return;
  COMPAT_TRY(d2h_pageable(Yout, p.Y, sz_Y, s));
  if (opt->Verbose == 1) {
    std::vector<double> it(SC_ITSTAT_FIELDS * (size_t)std::max(1, o.max_iter));
    int iters = 0;
    double rho = 0;
    sc_read_state(&p, &o, base + off_ws, &iters, &rho, it.data(), s);
    print_itstat(it, iters, grd);
  }
  COMPAT_TRY(cudaStreamSynchronize(s));
}

}  // namespace

extern "C" void cuda_wrapper_CBPDN(float* D, float* S, float lambda, void* opt, float* Y) {
  run_compat(D, S, lambda, 0.f, opt, Y, 0);
}

extern "C" void cuda_wrapper_CBPDN_GR(float* D, float* S, float lambda, float mu, void* opt,
                                      float* Y) {
  run_compat(D, S, lambda, mu, opt, Y, 1);
}
