// Small kernels of the solver driver: set-up (dictionary power spectrum,
// twiddles, state initialisation), the FP64 finalize step of every
// iteration (residuals, stopping test, adaptive rho), the final Y / U export
// and the functional of the Verbose statistics.  Included by sc_solver.cu
// only (the row and column pass templates are in sc_kernels.cuh).
#pragma once

#include "sc_kernels.cuh"

// Sum over the maps of |Df_m|^2 for every frequency (setup of COL_SOLVE).
__global__ void psum_kernel(const float2* __restrict__ Dh, float* __restrict__ Psum, int M,
                            size_t plane) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= plane) return;
  // summed in double precision: the solves' 1 / (rho + Psum) passes Psum's
  // relative error on to X almost undiminished (Psum >> rho for many maps)
  double s = 0.0;
  for (int m = 0; m < M; ++m) {
    const float2 d = __ldg(&Dh[(size_t)m * plane + i]);
    s += (double)d.x * d.x + (double)d.y * d.y;
  }
  Psum[i] = (float)s;
}

// ============================================================== finalize ==
// One CTA per image: FP64 reduction of the row-pass partials, residuals,
// stopping test and adaptive rho (cbpdn.cu:405-436, 519-559; Boyd et al.
// 2010 3.3-3.4; Wohlberg 2015).
__global__ void finalize_kernel(const double* __restrict__ partials, int nblk,
                                ImgState* st, FinParams F) {
  pdl_enter();
  __shared__ double scratch[(256 / 32) * 5];
  const int b = blockIdx.x;
  ImgState& S = st[b];
  if (S.done) return;
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const double* p = partials + (size_t)b * nblk * 5;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
#pragma unroll
    for (int j = 0; j < 5; ++j) v[j] += p[(size_t)i * 5 + j];
  }
  block_sum<5>(v, scratch);
  if (threadIdx.x != 0) return;
  const double rho = S.rho;
  const double nX = sqrt(v[0]), nY = sqrt(v[1]), nU = sqrt(v[2]);
  double r = sqrt(v[3]);
  double s = rho * sqrt(v[4]);
  const double sq = sqrt(F.nelem);
  double epri = sq * F.abs_tol + fmax(nX, nY) * F.rel_tol;
  double edua = sq * F.abs_tol + rho * nU * F.rel_tol;
  if (!F.std_residuals) {
    double rn = fmax(nX, nY);
    if (rn == 0.0) rn = 1.0;
    const double sn = rho * (nU == 0.0 ? 1.0 : nU);
    r /= rn;
    s /= sn;
    epri /= rn;
    edua /= sn;
  }
  const int k = S.k + 1;
  const int kc = k - S.k0;  // iterations of this solve call
  if (F.itstat) {
    double* it = F.itstat + ((size_t)b * F.max_iter + (kc - 1)) * SC_ITSTAT_FIELDS;
    it[0] = r; it[1] = s; it[2] = rho; it[3] = epri; it[4] = edua;
  }
  double rsf = 1.0;
  if (F.auto_rho && k > 1 && (k % F.period) == 0) {
    const double xi = F.xi[b];
    double rhomlt;
    if (F.auto_scaling) {
      rhomlt = (s * xi > 0.0) ? sqrt(r / (s * xi)) : INFINITY;
      if (rhomlt < 1.0) rhomlt = rhomlt > 0.0 ? 1.0 / rhomlt : INFINITY;
      if (rhomlt > F.rho_scaling) rhomlt = F.rho_scaling;
    } else {
      rhomlt = F.rho_scaling;
    }
    if (r > xi * F.rsdl_ratio * s) rsf = rhomlt;
    if (s > (F.rsdl_ratio / xi) * r) rsf = 1.0 / rhomlt;
  }
  S.nX = nX; S.nY = nY; S.nU = nU;
  S.r = r; S.s = s; S.epri = epri; S.edua = edua;
  S.rho_prev = rho;
  S.rho = rsf * rho;
  S.rsf = rsf;
  // U as stored is the U of this iteration; the next row pass reads it scaled
  // by 1/rsf (U <- U / rsf, cbpdn.cu:543-549)
  S.uscale = 1.0 / rsf;
  S.k = k;
  bool done = (r <= epri && s <= edua) || kc >= F.max_iter;
  if (!isfinite(r) || !isfinite(s)) {
    S.status = 5;  // SC_ERR_NONFINITE
    done = true;
  }
  if (done) {
    S.done = 1;
    if (F.ndone) atomicAdd(F.ndone, 1);
  }
}

__global__ void init_state_kernel(ImgState* st, const float* rho0, int B, int* ndone) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b == 0 && ndone) *ndone = 0;
  if (b >= B) return;
  ImgState s;
  s.rho = (double)rho0[b];
  s.rho_prev = s.rho;
  s.rsf = 1.0;
  s.uscale = 1.0;
  s.r = s.s = s.epri = s.edua = 0.0;
  s.nX = s.nY = s.nU = 0.0;
  s.k = 0;
  s.done = 0;
  s.status = 0;
  s.k0 = 0;
  st[b] = s;
}

// A warm-started solve call continues the state of the previous one: rho,
// the iterates and the iteration count carry over; the call's own cap counts
// from the current count, and the finished flags start afresh.
__global__ void warm_state_kernel(ImgState* st, int B, int* ndone) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b == 0 && ndone) *ndone = 0;
  if (b >= B) return;
  st[b].k0 = st[b].k;
  st[b].done = 0;
  st[b].status = 0;
}

// The convolution column solves' filter-row entries: for the row spectra e
// of the first Kr rows of every filter (Dh, before the column transform),
// (Re e, Im e, Re e + Im e, Im e - Re e), the sums the solves' three-multiply
// complex products take.
__global__ void filter_rows_kernel(const float2* __restrict__ Dh, float4* __restrict__ E, int M,
                                   int Kr, int H, int Wp) {
  const size_t n = (size_t)M * Kr * Wp;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t c = i % Wp, mr = i / Wp;
    const size_t m = mr / Kr, r = mr - m * Kr;
    const float2 e = Dh[(m * H + r) * Wp + c];
    E[i] = make_float4(e.x, e.y, e.x + e.y, e.y - e.x);
  }
}

// The unrolled solve's trace steps run the iteration's row pass from a
// given V without the finalize step: count the state as past its first
// iteration, so that the row pass recomputes Y from V at lambda / rho (at
// V = 0 that is 0, as before the first iteration).
__global__ void trace_state_kernel(ImgState* st, int B) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  if (st[b].k == 0) st[b].k = 1;
}

// tw[j] = exp(-2 pi i j / n), evaluated in double precision.
__global__ void twiddle_kernel(float2* tw, int n) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double s, c;
  sincospi(-2.0 * (double)j / (double)n, &s, &c);
  tw[j] = make_float2((float)c, (float)s);
}

// out = U scaled to the value the next iteration would read (U * uscale).
// Y and U from the state V = Y + U (row_kernel<ROW_ITER>), at the end of a
// solve or at a checkpoint: Y = shrinkage of V at lambda / rho_prev (what the
// last iteration computed), U = (V - Y) scaled by uscale; both zero before
// the first iteration.  Grid (blocks, B); U may be NULL.
__global__ void state_yu_kernel(const float* __restrict__ V, float* __restrict__ Y,
                                float* __restrict__ U, const ImgState* __restrict__ st,
                                const float* __restrict__ lam, int M, int H, int W, int l1_kind,
                                float l1_scalar, const float* __restrict__ l1w,
                                const int32_t* __restrict__ mask, int nonneg, int bnd_r,
                                int bnd_c) {
  const int b = blockIdx.y;
  const ImgState& S = st[b];
  const bool first = S.k == 0;
  const float thr = (float)((double)lam[b] / S.rho_prev);
  const float us = (float)S.uscale;
  const size_t plane = (size_t)H * W, n = (size_t)M * plane;
  const size_t off = (size_t)b * n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(i / plane);
    const size_t hw = i - (size_t)m * plane;
    const float v = V[off + i];
    float y = 0.f, u = 0.f;
    if (!first) {
      if (mask && m == 0) {
        y = (float)(1 - mask[(size_t)b * plane + hw]) * v;
      } else {
        const float w = l1_kind == 1 ? l1w[m] : l1_kind == 2 ? l1w[i] : l1_scalar;
        y = soft_threshold(v, thr * w);
        if (nonneg) y = fmaxf(y, 0.f);
        const int h = (int)(hw / W), c = (int)(hw - (size_t)h * W);
        if (h >= bnd_r || c >= bnd_c) y = 0.f;
      }
      u = (v - y) * us;
    }
    Y[off + i] = y;
    if (U) U[off + i] = u;
  }
}

// ============================================================= functional ==
// The functional at Y (Verbose statistics, cbpdn.cu:438-517): data fidelity
// 0.5 ||sum_m d_m * y_m - s||^2 and, with the gradient term,
// mu/2 sum_m w_m ||grad y_m||^2, both by Parseval over the half spectrum
// (columns 0 and W/2 once, the others twice; divided by H W), from the
// spectra Yh (B, M, H, Wp), Dh (M, H, Wp) and Sh (B, H, Wp).  Grid (nblk,
// B); part (B, nblk, 2): fidelity and gradient sums.
__global__ void objective_spec_kernel(const float2* __restrict__ Yh,
                                      const float2* __restrict__ Dh,
                                      const float2* __restrict__ Sh, Geom g, int grd,
                                      const float* __restrict__ wgrd,
                                      const float2* __restrict__ twH,
                                      const float2* __restrict__ twW, double* part) {
  __shared__ double scratch[(256 / 32) * 2];
  const int b = blockIdx.y;
  const size_t plane = (size_t)g.H * g.Wp;
  const float2* Yb = Yh + (size_t)b * g.M * plane;
  double v[2] = {0.0, 0.0};
  const size_t nf = (size_t)g.H * g.Wf;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nf;
       i += (size_t)gridDim.x * blockDim.x) {
    const int kr = (int)(i / g.Wf), kc = (int)(i - (size_t)kr * g.Wf);
    const size_t f = (size_t)kr * g.Wp + kc;
    const double w = (kc == 0 || 2 * kc == g.W) ? 1.0 : 2.0;
    double rx = -(double)Sh[(size_t)b * plane + f].x, ry = -(double)Sh[(size_t)b * plane + f].y;
    double gs = 0.0;
    for (int m = 0; m < g.M; ++m) {
      const float2 d = Dh[(size_t)m * plane + f], y = Yb[(size_t)m * plane + f];
      rx += (double)d.x * y.x - (double)d.y * y.y;
      ry += (double)d.x * y.y + (double)d.y * y.x;
      if (grd) gs += (double)wgrd[m] * ((double)y.x * y.x + (double)y.y * y.y);
    }
    v[0] += w * (rx * rx + ry * ry);
    if (grd) {
      const double gk = (2.0 - 2.0 * (double)twW[kc].x) + (2.0 - 2.0 * (double)twH[kr].x);
      v[1] += w * gk * gs;
    }
  }
  block_sum<2>(v, scratch);
  if (threadIdx.x == 0) {
    double* o = part + ((size_t)b * gridDim.x + blockIdx.x) * 2;
    o[0] = v[0];
    o[1] = v[1];
  }
}

// sum |w y| per (image, block): the L1 term at Y.  Grid (nblk, B);
// part (B, nblk).
__global__ void objective_l1_kernel(const float* __restrict__ Y, Geom g, int l1_kind,
                                    float l1_scalar, const float* __restrict__ l1w,
                                    double* part) {
  __shared__ double scratch[256 / 32];
  const int b = blockIdx.y;
  const size_t plane = (size_t)g.H * g.W, n = (size_t)g.M * plane;
  const float* Yb = Y + (size_t)b * n;
  double v[1] = {0.0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float w = l1_kind == 1 ? l1w[i / plane] : l1_kind == 2 ? l1w[i] : l1_scalar;
    v[0] += fabs((double)w * (double)Yb[i]);
  }
  block_sum<1>(v, scratch);
  if (threadIdx.x == 0) part[(size_t)b * gridDim.x + blockIdx.x] = v[0];
}

// Functional, fidelity and L1 terms into the statistics row of the iteration
// just completed (ImgState::k).  One thread per image.
__global__ void objective_final_kernel(const double* __restrict__ pspec,
                                       const double* __restrict__ pl1, int nblk,
                                       const ImgState* __restrict__ st,
                                       const float* __restrict__ lam, double invN, float mu,
                                       double* itstat, int max_iter, int B) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const int k = st[b].k - st[b].k0;  // iteration of this solve call
  if (k < 1 || k > max_iter) return;
  double df = 0.0, gr = 0.0, l1 = 0.0;
  for (int i = 0; i < nblk; ++i) {
    df += pspec[((size_t)b * nblk + i) * 2];
    gr += pspec[((size_t)b * nblk + i) * 2 + 1];
    l1 += pl1[(size_t)b * nblk + i];
  }
  df *= 0.5 * invN;
  double* it = itstat + ((size_t)b * max_iter + (k - 1)) * SC_ITSTAT_FIELDS;
  it[5] = df + (double)lam[b] * l1 + 0.5 * (double)mu * gr * invN;
  it[6] = df;
  it[7] = l1;
}

__global__ void export_u_kernel(const float* __restrict__ U, float* __restrict__ out,
                                const ImgState* __restrict__ st, size_t per_img, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = U[i] * (float)st[i / per_img].uscale;
}
