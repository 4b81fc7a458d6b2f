// Adjoint of the unrolled CBPDN ADMM iterations (plain cbpdn, fixed rho).
//
// No counterpart in the reference (sporco_cuda solves only).  Forward
// iteration k, with A = D^T D + rho I (per frequency: rho I + conj(Df) Df^T):
//   X = A^{-1} (D^T S + rho (Y - U)),  V = a X + (1 - a) Y + U,
//   Y' = soft(V, lambda w / rho),      U' = V - Y'.
// Backward, given gY', gU':
//   mask = |V| > lambda w / rho,  gV = mask gY' + (1 - mask) gU',
//   gX = a gV,  Q = A^{-1} gX   (A is symmetric: the same solve),
//   gY = (1 - a) gV + rho Q,    gU = gV - rho Q,
//   gS^ += sum_m Df_m Q^_m,
//   gD^_m += S^ conj(Q^_m) - (sum_j Df_j X^_j) conj(Q^_m) - (sum_j Df_j Q^_j) conj(X^_m)
// (products of half spectra of real signals; one inverse FFT and a crop to
// the filter support turn gD^ into the gradient of the filters).
//
// Spectra here are dense (count, H, W/2+1) complex64 arrays, transformed by
// sc_rfft2 / sc_irfft2 (this library's FFT kernels).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>

#include "../../include/sporco_b200.h"

int sc_set_status_external(int st, const char* msg);

namespace {

int fail(cudaError_t e, const char* what) {
  char b[256];
  snprintf(b, sizeof(b), "%s: %s", what, cudaGetErrorString(e));
  return sc_set_status_external(e == cudaErrorMemoryAllocation ? SC_ERR_OOM : SC_ERR_CUDA, b);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// One thread per (frequency f of the (H, W/2+1) grid, image b), all maps.
//  mode 0: io holds Z^ = rfft2(Y - U); replaced by X^ = A^{-1}(conj(Df) S^ + rho Z^)
//  mode 1: io holds gX^; replaced by Q^ = A^{-1} gX^; the image's part of gD^
//          accumulates in gDh[b] (B, M, H, W/2+1), gS^ in gSh[b]
__global__ void adj_freq_kernel(int mode, int B, int M, int Fn, float rho,
                                const float2* __restrict__ Dh, const float2* __restrict__ Sh,
                                float2* io, const float2* __restrict__ Xh, float2* gDh,
                                float2* gSh) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (f >= Fn) return;
  const size_t plane = (size_t)Fn;
  const size_t ib = (size_t)b * M * plane + f;
  const float2 Sv = __ldg(&Sh[(size_t)b * plane + f]);
  float sden = 0.f;
  // dot = sum_m Df_m v_m, v = conj(Df) S + rho Z (mode 0) or gX (mode 1)
  float2 dot = make_float2(0.f, 0.f), DX = make_float2(0.f, 0.f);
  for (int m = 0; m < M; ++m) {
    const float2 d = __ldg(&Dh[m * plane + f]);
    sden += d.x * d.x + d.y * d.y;
    float2 vm = io[ib + m * plane];
    if (mode == 0) {
      const float2 ds = cmulc(Sv, d);  // conj(Df) S
      vm = make_float2(ds.x + rho * vm.x, ds.y + rho * vm.y);
    } else {
      const float2 dx = cmul(d, __ldg(&Xh[ib + m * plane]));
      DX.x += dx.x;
      DX.y += dx.y;
    }
    const float2 p = cmul(d, vm);
    dot.x += p.x;
    dot.y += p.y;
  }
  const float inv = 1.f / (rho + sden), irho = 1.f / rho;
  const float2 c = make_float2(dot.x * inv, dot.y * inv);
  float2 DQ = make_float2(0.f, 0.f);
  for (int m = 0; m < M; ++m) {
    const float2 d = __ldg(&Dh[m * plane + f]);
    float2 vm = io[ib + m * plane];
    if (mode == 0) {
      const float2 ds = cmulc(Sv, d);
      vm = make_float2(ds.x + rho * vm.x, ds.y + rho * vm.y);
    }
    const float2 dc = cmulc(c, d);  // conj(Df) c
    const float2 out = make_float2((vm.x - dc.x) * irho, (vm.y - dc.y) * irho);
    io[ib + m * plane] = out;
    if (mode == 1) {
      const float2 dq = cmul(d, out);
      DQ.x += dq.x;
      DQ.y += dq.y;
    }
  }
  if (mode == 1) {
    float2* gs = gSh + (size_t)b * plane + f;
    *gs = make_float2(gs->x + DQ.x, gs->y + DQ.y);
    for (int m = 0; m < M; ++m) {
      const float2 q = io[ib + m * plane];
      const float2 x = __ldg(&Xh[ib + m * plane]);
      const float2 t1 = cmulc(Sv, q), t2 = cmulc(DX, q), t3 = cmulc(DQ, x);
      float2* g = gDh + ib + m * plane;
      *g = make_float2(g->x + t1.x - t2.x - t3.x, g->y + t1.y - t2.y - t3.y);
    }
  }
}

enum { EL_ZDIFF = 0, EL_FWD = 1, EL_BWD = 2, EL_COMB = 3 };

// Elementwise steps over (B, M, H, W) real arrays.
//  EL_ZDIFF: out = Y - U
//  EL_FWD:   (Y, U) <- ADMM y/u-step from X (relaxation, soft threshold)
//  EL_BWD:   from gY', gU' (in gY, gU) and X, Y, U of the step: gX (out),
//            gY <- (1 - a) gV, gU <- gV
//  EL_COMB:  gY += rho Q, gU -= rho Q (Q in X)
__global__ void adj_elem_kernel(int mode, size_t n, int M, size_t HW, float rho, float alpha,
                                const float* __restrict__ lam, int l1_kind, float l1_scalar,
                                const float* __restrict__ l1w, const float* X, float* Y, float* U,
                                float* gY, float* gU, float* out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    if (mode == EL_ZDIFF) {
      out[i] = Y[i] - U[i];
      continue;
    }
    if (mode == EL_COMB) {
      const float q = X[i];
      gY[i] += rho * q;
      gU[i] -= rho * q;
      continue;
    }
    const size_t img = i / ((size_t)M * HW);
    const int m = (int)((i / HW) % M);
    float w = l1_scalar;
    if (l1_kind == SC_L1_PER_MAP) w = l1w[m];
    else if (l1_kind == SC_L1_FULL) w = l1w[i % ((size_t)M * HW)];
    const float t = lam[img] / rho * w;
    const float v = alpha * X[i] + (1.f - alpha) * Y[i] + U[i];
    if (mode == EL_FWD) {
      const float a = fabsf(v) - t;
      const float y = a > 0.f ? copysignf(a, v) : 0.f;
      Y[i] = y;
      U[i] = v - y;
    } else {
      const bool on = fabsf(v) > t;
      const float gv = on ? gY[i] : gU[i];
      out[i] = alpha * gv;
      gY[i] = (1.f - alpha) * gv;
      gU[i] = gv;
    }
  }
}

}  // namespace

extern "C" int sc_adj_freq(int mode, int B, int M, int H, int W, float rho, const void* Dh,
                           const void* Sh, void* io, const void* Xh, void* gDh, void* gSh,
                           void* stream) {
  sc_set_status_external(SC_OK, "");
  (void)cudaGetLastError();
  if ((mode != 0 && mode != 1) || B < 1 || M < 1 || H < 1 || W < 1 || !(rho > 0.f) || !Dh ||
      !Sh || !io || (mode == 1 && (!Xh || !gDh || !gSh)))
    return sc_set_status_external(SC_ERR_INVALID, "sc_adj_freq: invalid arguments");
  const int Fn = H * (W / 2 + 1);
  adj_freq_kernel<<<dim3((Fn + 127) / 128, B), 128, 0, (cudaStream_t)stream>>>(
      mode, B, M, Fn, rho, (const float2*)Dh, (const float2*)Sh, (float2*)io, (const float2*)Xh,
      (float2*)gDh, (float2*)gSh);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SC_OK : fail(e, "adj_freq_kernel");
}

extern "C" int sc_adj_elem(int mode, int B, int M, int H, int W, float rho, float alpha,
                           const float* lam, int l1_kind, float l1_scalar, const float* l1w,
                           const float* X, float* Y, float* U, float* gY, float* gU, float* out,
                           void* stream) {
  sc_set_status_external(SC_OK, "");
  (void)cudaGetLastError();
  if (mode < EL_ZDIFF || mode > EL_COMB || B < 1 || M < 1 || H < 1 || W < 1)
    return sc_set_status_external(SC_ERR_INVALID, "sc_adj_elem: invalid arguments");
  const size_t HW = (size_t)H * W;
  const size_t n = (size_t)B * M * HW;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  adj_elem_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(mode, n, M, HW, rho, alpha, lam,
                                                            l1_kind, l1_scalar, l1w, X, Y, U,
                                                            gY, gU, out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SC_OK : fail(e, "adj_elem_kernel");
}
