// Fused ADMM kernels of the CBPDN solvers.
//
// One ADMM iteration (sporco_cuda/src/cbpdn.cu:319-567, cbpdn_grd.cu:358-606)
// is three kernels and a conditional fourth:
//
//   col_kernel<COL_SOLVE>  spectrum columns: forward column FFT of the row
//                          spectra of Y - U, b = conj(Df) Sf + rho (Y-U)^,
//                          Sherman-Morrison solve across the M maps
//                          (cluster-wide reduction of sum_m Df_m b_m / d_m),
//                          inverse column FFT.  Replaces CalYU's consumer,
//                          cufftExecR2C (column half), cuda_solvedbi_sm*,
//                          cuda_solvedbd_sm*, cufftExecC2R (column half).
//   row_kernel<ROW_ITER>   image rows: inverse row FFT, over-relaxation,
//                          soft threshold / AMS mask step, dual update,
//                          residual partial sums (FP64), then the forward row
//                          FFT of the new Y - U.  Replaces cufftExecC2R (row
//                          half), cuda_OverRelax_vec4, cuda_Shrink_CalU_*,
//                          cuda_Cal_X_minus_U_W, cuda_Cal_residuals_norms_vec4,
//                          the Yprv copy, cuda_CalYU_vec4 and cufftExecR2C
//                          (row half).
//   finalize_kernel        FP64 reduction of the partials, residuals, stopping
//                          test, adaptive rho (host code at cbpdn.cu:405-559).
//   row_kernel<ROW_FIXUP>  only when rho changed: the row spectra of
//                          Y - U / rsf, transformed afresh from the state V;
//                          the next row pass reads U scaled by 1/rsf
//                          (replaces cublasSgeam at cbpdn.cu:546-549).
//
// HBM layout: real maps (B, M, H, W) float32; spectra (B, M, H, Wp) complex64
// with Wp = W/2+1 rounded up to a multiple of 4 (storage padding only).
//
// Both hot kernels keep copies in flight while they compute: the column pass
// double-buffers its (H x 4) tiles with cp.async and transforms them in place
// in the interleaved layout they have in HBM; the row pass double-buffers the
// spectrum rows of the next row pair and stages the pair's Y and U rows
// before its inverse FFT.
#pragma once

#include <cooperative_groups.h>

#include "sc_internal.cuh"

namespace cg = cooperative_groups;

// ------------------------------------------------------------ async copies --
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Programmatic dependent launch: the iteration's kernels are launched with
// programmatic stream serialisation, so a kernel's CTAs can be scheduled
// while the kernel before it in the stream drains.  Each waits here for that
// kernel to complete (its writes visible) before touching global memory,
// then lets the next kernel be scheduled.  Launched without the attribute,
// both instructions return at once.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// Soft threshold as the reference's shrink kernels compute it
// (cbpdn_kernels.cu:129-311): sign(v) max(|v| - t, 0), t may be negative.
__device__ __forceinline__ float soft_threshold(float v, float t) {
  const float a = fabsf(v) - t;
  return a > 0.f ? copysignf(a, v) : 0.f;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic CTA-wide sum of NV doubles; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = warp_sum(v[i]);
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) scratch[wid * NV + i] = v[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += scratch[w * NV + i];
      v[i] = s;
    }
  }
  __syncthreads();
}

// Hermitian-extend two half spectra (rows a, b of an rfft2 row pass) and pack
// them as conj(A + iB) for an inverse transform taken as conj(FFT(conj .)).
// The imaginary parts of the DC and (even W) Nyquist bins are ignored, as a
// C2R transform does.
__device__ __forceinline__ float2 pack_inverse(const float2* a, const float2* bb, bool has1,
                                               int k, int W, int Wf) {
  float2 A, Bv;
  if (k < Wf) {
    A = a[k];
    Bv = has1 ? bb[k] : make_float2(0.f, 0.f);
    if (k == 0 || 2 * k == W) { A.y = 0.f; Bv.y = 0.f; }
    return make_float2(A.x - Bv.y, -(A.y + Bv.x));
  }
  const int kk = W - k;
  A = a[kk];
  Bv = has1 ? bb[kk] : make_float2(0.f, 0.f);
  return make_float2(A.x + Bv.y, -(Bv.x - A.y));
}

// Threshold weight of one image row: scalar w, or the row wr of a full
// weight array; mrow: the AMS mask row when the row belongs to map 0 of a
// masked problem; nonneg and kcut: the projections of NonNegCoef (Y >= 0)
// and NoBndryCross (elements k >= kcut are zero: the last Kc - 1 columns,
// the whole row in the last Kr - 1 rows; SC_NO_CUT: none).
#define SC_NO_CUT 0x40000000
struct RowW {
  float w;
  const float* wr;
  const int32_t* mrow;
  int kcut;
  bool nonneg;
  // scalar threshold, no AMS row, no projection: the fast element path
  __device__ __forceinline__ bool plain() const {
    return !mrow && !wr && !nonneg && kcut == SC_NO_CUT;
  }
};

// Y of the shrinkage step at element k of a row: the AMS step (1 - mask) v
// on map 0 of masked problems, else the soft threshold at th times the
// row's weight (cbpdn_kernels.cu:129-311, 1137-1155), followed by the
// projections the reference parses but never applies (cbpdn.pyx:70-71;
// sporco's ConvBPDN y-step): NonNegCoef sets negative values to zero,
// NoBndryCross zeroes the coefficients whose filter would cross the bottom
// or right image boundary.
__device__ __forceinline__ float shrink_y(float v, float th, const RowW& r, int k) {
  if (r.mrow) return (float)(1 - r.mrow[k]) * v;
  float y = soft_threshold(v, th * (r.wr ? r.wr[k] : r.w));
  if (r.nonneg) y = fmaxf(y, 0.f);
  return k >= r.kcut ? 0.f : y;
}

// A compile-time int passed to generic lambdas.
template <int V>
struct IntC {
  static constexpr int value = V;
};

// Per-launch constants of the iteration's element-wise step.
struct IterC {
  float a, a1;   // RelaxParam, 1 - RelaxParam
  bool relax;    // RelaxParam != 1
  float uscale;  // the stored U is read scaled by this (1/rsf after a rho change)
  bool delta;    // x is the column pass's correction to Y - U (RowParams::delta)
};

// One element of the iteration's element-wise step: over-relaxation,
// shrinkage, dual update, residual partial sums (single precision within a
// row pair).  VS: the stored state is V = Y + U of the previous iteration
// (s0), whose Y is recomputed as its shrinkage at the previous threshold
// tq; else s0, s1 are Y and U.  FAST: scalar thresholds tc, tq (weights
// applied), no AMS row.  x: X, or with c.delta (DL = 1; DL < 0: as c.delta
// says) the column pass's correction to Y - U.  Writes V (VS) or Y and U;
// returns y - u.
template <bool VS, bool FAST, int DL = -1>
__device__ __forceinline__ float iter_elem(float x, float s0, float s1, const RowW& r, int k,
                                           float tc, float tq, const IterC& c, float* f,
                                           float* o0, float* o1) {
  float yo, uo;
  if constexpr (VS) {
    // before the first iteration V = 0 and tq = 0, so yo = uo = 0
    yo = FAST ? soft_threshold(s0, tq) : shrink_y(s0, tq, r, k);
    uo = (s0 - yo) * c.uscale;
  } else {
    yo = s0;
    uo = s1 * c.uscale;
  }
  // X = IFFT2(Z^ + conj(Df) SC / rho) = (Y - U) + IFFT2(conj(Df) SC / rho)
  if (DL == 1 || (DL < 0 && c.delta)) x += yo - uo;
  const float xr = c.relax ? c.a * x + c.a1 * yo : x;
  const float v = xr + uo;
  const float y = FAST ? soft_threshold(v, tc) : shrink_y(v, tc, r, k);
  const float u = v - y;
  if constexpr (VS) {
    *o0 = v;
  } else {
    *o0 = y;
    *o1 = u;
  }
  const float dxy = x - y, dyy = yo - y;
  f[0] += x * x;
  f[1] += y * y;
  f[2] += u * u;
  f[3] += dxy * dxy;
  f[4] += dyy * dyy;
  return y - u;
}

// ============================================================== row pass ==
// NW > 0: row length W known at compile time (specialised FFT plan);
// NW == 0: any W (runtime FFT plan).
template <int MODE, int NW>
__global__ void __launch_bounds__(SC_ROW_THREADS, row_min_blocks(NW))
row_kernel(RowParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red_scratch[(SC_ROW_THREADS / 32) * 5];
  pdl_enter();

  const Geom& G = P.g;
  const int b = blockIdx.y;
  const int W = G.W, Wf = G.Wf, Wp = G.Wp, H = G.H;
  constexpr int RM = row_radix(NW);
  const int g = NW > 0 ? ct_threads(NW, RM) : P.gsz;
  const int S = blockDim.x / g;
  const int s = threadIdx.x / g;
  const int t = threadIdx.x - s * g;
  const int zlen = NW > 0 ? ct_len(NW, RM, 1) : W;
  unsigned char* slot = smem_raw + (size_t)s * row_slot_bytes(MODE, zlen, W, Wp);
  float2* z = reinterpret_cast<float2*>(slot);
  auto zs = [](int k) { return fft_slot<NW, RM, 1>(k); };

  // thr: lambda / rho of this iteration; thr_prev: of the iteration that
  // produced the stored state (the same float value that iteration used)
  float thr = 0.f, thr_prev = 0.f, rsf_c = 0.f, uscale = 1.f, rho = 0.f;
  if constexpr (MODE == ROW_ITER || MODE == ROW_ITER_YU || MODE == ROW_FIXUP ||
                MODE == ROW_ADJ) {
    const ImgState& st = P.st[b];
    if (st.done) return;
    if constexpr (MODE == ROW_ITER || MODE == ROW_ITER_YU) {
      thr = (float)((double)P.lam[b] / st.rho);
      // no iteration yet: V = 0 and a zero threshold give Y = U = 0
      thr_prev = st.k == 0 ? 0.f : (float)((double)P.lam[b] / st.rho_prev);
      uscale = (float)st.uscale;
    } else if constexpr (MODE == ROW_ADJ) {
      rho = (float)st.rho;
      thr = (float)((double)P.lam[b] / st.rho);  // as the step's ROW_ITER had it
    } else {
      if (st.rsf == 1.0) return;
      rsf_c = (float)(1.0 - 1.0 / st.rsf);
      thr_prev = (float)((double)P.lam[b] / st.rho_prev);
      uscale = (float)st.uscale;
    }
  }

  const long rows = (long)G.M * H;  // rows per image
  const long npairs = (rows + 1) / 2;
  const size_t img_real = (size_t)rows * W;
  const size_t img_spec = (size_t)rows * Wp;
  float2* Fi = P.F + (size_t)b * img_spec;
  const long pstride = (long)gridDim.x * S;

  if constexpr (MODE == ROW_ITER || MODE == ROW_ITER_YU || MODE == ROW_ADJ ||
                MODE == ROW_FIXUP) {
    // ------------------------------- iteration / adjoint step / rho fix-up
    constexpr bool ADJ = MODE == ROW_ADJ;
    // ROW_ITER keeps the ADMM state as V = Y + U (one array, P.U): Y of an
    // iteration is the shrinkage of V, U = V - Y.  ROW_ITER_YU keeps Y and U.
    constexpr bool VS = MODE == ROW_ITER;
    constexpr bool TWO = MODE == ROW_ITER_YU || ADJ;  // two staged real arrays
    float2* fst = reinterpret_cast<float2*>(slot + sc_align16((size_t)zlen * 8));
    float* ysm = reinterpret_cast<float*>(fst + 2 * (size_t)Wp);
    // one staged real row pair in the iteration from V (ysm) and the fix-up
    // (usm = ysm), two otherwise
    float* usm = TWO ? ysm + sc_align16((size_t)(2 * W) * 4) / 4 : ysm;
    // staged per row pair: V (iteration), Y and U (iteration from Y, U), gV
    // and the mask source (adjoint), the state array (fix-up, into usm)
    const float* Yi = (ADJ ? P.gV : VS ? P.U : P.Y) + (size_t)b * img_real;
    const float* Ui = (ADJ ? P.Ymask : P.U) + (size_t)b * img_real;
    const bool vec = (W & 3) == 0;
    const int32_t* mk = P.mask ? P.mask + (size_t)b * H * W : nullptr;
    // threshold weights and AMS mask row of image row r of this image
    auto roww = [&](long r, bool ok) -> RowW {
      RowW o{P.l1_scalar, nullptr, nullptr, SC_NO_CUT, false};
      if (!ok) return o;
      const int m = (int)(r / H), h = (int)(r - (long)m * H);
      if (P.l1_kind == 1) o.w = P.l1w[m];
      if (P.l1_kind == 2) o.wr = P.l1w + ((size_t)m * H + h) * W;
      if (mk && m == 0) o.mrow = mk + (size_t)h * W;
      o.nonneg = P.nonneg != 0;
      if (P.bnd_r > 0 && h >= P.bnd_r) o.kcut = 0;
      else if (P.bnd_c > 0 && P.bnd_c < W) o.kcut = P.bnd_c;
      return o;
    };

    auto issue_F = [&](long p) {
      if (p < npairs) {
        const int nrow = (2 * p + 1 < rows) ? 2 : 1;
        const float2* src = Fi + 2 * p * Wp;
        const int nch = nrow * Wp / 2;
        for (int q = t; q < nch; q += g) cp_async16(fst + 2 * q, src + 2 * q);
      }
    };
    auto issue_YU = [&](long p) {
      if (p < npairs) {
        const int n = ((2 * p + 1 < rows) ? 2 : 1) * W;
        const float* ys = Yi + 2 * p * W;
        const float* us = Ui + 2 * p * W;
        if (vec) {
          for (int q = t; q < n / 4; q += g) {
            cp_async16(ysm + 4 * q, ys + 4 * q);
            if constexpr (TWO) cp_async16(usm + 4 * q, us + 4 * q);
          }
        } else {
          for (int q = t; q < n; q += g) {
            cp_async4(ysm + q, ys + q);
            if constexpr (TWO) cp_async4(usm + q, us + q);
          }
        }
      }
    };

    if constexpr (MODE == ROW_FIXUP) {
      // After a change of rho the next row pass reads U scaled by 1/rsf, so
      // the column pass needs the row spectra of Y - U / rsf.  From the state
      // V (Y = shrinkage of V at the previous threshold, U = V - Y) they are
      // transformed afresh (reads V, writes F); with Y and U kept apart,
      // F += (1 - 1/rsf) rowFFT(U) (reads U and F, writes F).  The state
      // rows are staged one pair ahead (during the transform), F rows during
      // the next pair's packing.
      const bool vstate = P.vstate != 0;
      auto issue_U = [&](long p) {
        if (p < npairs) {
          const int n = ((2 * p + 1 < rows) ? 2 : 1) * W;
          const float* us = Ui + 2 * p * W;
          if (vec) {
            for (int q = t; q < n / 4; q += g) cp_async16(usm + 4 * q, us + 4 * q);
          } else {
            for (int q = t; q < n; q += g) cp_async4(usm + q, us + q);
          }
        }
      };
      // y - u / rsf from v
      auto ymu = [&](float v, float y) { return y - (v - y) * uscale; };
      const long p0 = (long)blockIdx.x * S + s;
      issue_U(p0);
      if (!vstate) issue_F(p0);
      cp_async_commit();
      if constexpr (NW > 0 && ct_reg_edges(NW, RM)) {
        if (vstate) {
          // Register hand-over: thread t computes the elements t + g m of the
          // pair's transform input and runs the first pass on registers.
          constexpr int EM = NW / ct_threads(NW, RM);
          constexpr int NP = ct_plan(NW, RM).np;
          for (long pb = (long)blockIdx.x * S; pb < npairs; pb += pstride) {
            const long p = pb + s;
            const bool valid = p < npairs;
            const bool has1 = valid && (2 * p + 1 < rows);
            cp_async_wait<0>();  // V(p)
            __syncthreads();
            float2 v[EM];
            if (valid) {
              const RowW w0 = roww(2 * p, true), w1 = roww(2 * p + 1, has1);
              if (w0.plain() && w1.plain()) {
                const float t0 = thr_prev * w0.w, t1 = thr_prev * w1.w;
#pragma unroll
                for (int m = 0; m < EM; ++m) {
                  const int k = t + g * m;
                  const float v0 = usm[k], v1 = has1 ? usm[W + k] : 0.f;
                  v[m] = make_float2(ymu(v0, soft_threshold(v0, t0)),
                                     ymu(v1, soft_threshold(v1, t1)));
                }
              } else {
#pragma unroll
                for (int m = 0; m < EM; ++m) {
                  const int k = t + g * m;
                  const float v0 = usm[k], v1 = has1 ? usm[W + k] : 0.f;
                  v[m] = make_float2(ymu(v0, shrink_y(v0, thr_prev, w0, k)),
                                     has1 ? ymu(v1, shrink_y(v1, thr_prev, w1, k)) : 0.f);
                }
              }
            } else {
#pragma unroll
              for (int m = 0; m < EM; ++m) v[m] = make_float2(0.f, 0.f);
            }
            ct_first_from_regs<NW, RM, 1>(z, v, t);  // the staged rows are consumed
            issue_U(p + pstride);
            cp_async_commit();
            fft_ct_passes<NW, RM, ct_threads(NW, RM), 1, 1, NP>(z, P.twW, t);
            if (valid) {
              float2* fa = Fi + 2 * p * Wp;
              for (int k = t; k < Wf; k += g) {
                const float2 Zk = z[zs(k)];
                const float2 Zm = z[zs(k == 0 ? 0 : W - k)];
                fa[k] = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
                if (has1) fa[Wp + k] = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
              }
            }
            __syncthreads();
          }
          cp_async_wait<0>();
          return;
        }
      }
      for (long pb = (long)blockIdx.x * S; pb < npairs; pb += pstride) {
        const long p = pb + s;
        const bool valid = p < npairs;
        const bool has1 = valid && (2 * p + 1 < rows);
        cp_async_wait<0>();  // U(p) (or V(p)), F(p)
        __syncthreads();
        if (valid) {
          if (vstate) {
            const RowW w0 = roww(2 * p, true), w1 = roww(2 * p + 1, has1);
            if (w0.plain() && w1.plain()) {
              const float t0 = thr_prev * w0.w, t1 = thr_prev * w1.w;
              for (int k = t; k < W; k += g) {
                const float v0 = usm[k], v1 = has1 ? usm[W + k] : 0.f;
                z[zs(k)] = make_float2(ymu(v0, soft_threshold(v0, t0)),
                                       ymu(v1, soft_threshold(v1, t1)));
              }
            } else {
              for (int k = t; k < W; k += g) {
                const float v0 = usm[k], v1 = has1 ? usm[W + k] : 0.f;
                z[zs(k)] = make_float2(ymu(v0, shrink_y(v0, thr_prev, w0, k)),
                                       has1 ? ymu(v1, shrink_y(v1, thr_prev, w1, k)) : 0.f);
              }
            }
          } else {
            for (int k = t; k < W; k += g)
              z[zs(k)] = make_float2(usm[k], has1 ? usm[W + k] : 0.f);
          }
        }
        __syncthreads();
        issue_U(p + pstride);
        cp_async_commit();
        fft_any<NW, 1, RM>(z, P.pw, P.twW, t, g);
        if (valid) {
          float2* fa = Fi + 2 * p * Wp;
          for (int k = t; k < Wf; k += g) {
            const float2 Zk = z[zs(k)];
            const float2 Zm = z[zs(k == 0 ? 0 : W - k)];
            const float2 A = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
            const float2 Bv = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
            if (vstate) {
              fa[k] = A;
              if (has1) fa[Wp + k] = Bv;
            } else {
              const float2 f0 = fst[k];
              fa[k] = make_float2(f0.x + rsf_c * A.x, f0.y + rsf_c * A.y);
              if (has1) {
                const float2 f1 = fst[Wp + k];
                fa[Wp + k] = make_float2(f1.x + rsf_c * Bv.x, f1.y + rsf_c * Bv.y);
              }
            }
          }
        }
        __syncthreads();  // F staging consumed
        if (!vstate) issue_F(p + pstride);
        cp_async_commit();
      }
      cp_async_wait<0>();
      return;
    }

    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    IterC ic;
    ic.a = P.relax;
    ic.a1 = 1.f - P.relax;
    ic.relax = P.relax != 1.f;
    ic.uscale = uscale;
    ic.delta = P.delta != 0;
    // State rows of the pair (V, or Y and U) are written here.
    auto out0 = [&](long r0) -> float* {
      return (VS ? (P.Vo ? P.Vo : P.U) : P.Yo) + (size_t)b * img_real + (size_t)r0 * W;
    };
    // ROW_ADJ: the shrinkage of the step was active at element k of a row
    // (Y != 0; from V with vmask, as the step computed Y)
    auto active = [&](float src, const RowW& w, int k) -> bool {
      return P.vmask ? shrink_y(src, thr, w, k) != 0.f : src != 0.f;
    };
    auto outu = [&](long r0) -> float* { return P.U + (size_t)b * img_real + (size_t)r0 * W; };
    // The element-wise step of the iteration on the pair element k (both
    // rows): x from the inverse transform zz; returns the packed y - u.
    // fast: both rows present, scalar thresholds, no AMS row.
    // fast: both rows present, scalar thresholds (tc*, tq*), no AMS row
    // (dl: IntC<1> when F holds the column pass's correction, else IntC<0>)
    auto elem_fast = [&](auto dl, float tc0, float tc1, float tq0, float tq1, int k, float2 zz,
                         float* O0, float* Q0, float* f) -> float2 {
      constexpr int DL = decltype(dl)::value;
      const RowW w{};
      // (DL: the column pass has applied 1 / (H W) already)
      const float x0 = DL == 1 ? zz.x : zz.x * P.invN;
      const float x1 = DL == 1 ? -zz.y : -zz.y * P.invN;
      const float yu0 = iter_elem<VS, true, DL>(x0, ysm[k], TWO ? usm[k] : 0.f, w,
                                                k, tc0, tq0, ic, f, O0 + k, Q0 + k);
      const float yu1 = iter_elem<VS, true, DL>(x1, ysm[W + k],
                                                TWO ? usm[W + k] : 0.f, w, k, tc1, tq1, ic, f,
                                                O0 + W + k, Q0 + W + k);
      return make_float2(yu0, yu1);
    };
    auto elem_gen = [&](const RowW& w0, const RowW& w1, bool has1, int k, float2 zz, float* O0,
                        float* Q0, float* f) -> float2 {
      float yu1 = 0.f;
      const float xn = P.delta ? 1.f : P.invN;  // see elem_fast
      const float yu0 = iter_elem<VS, false>(zz.x * xn, ysm[k], TWO ? usm[k] : 0.f, w0, k,
                                             thr, thr_prev, ic, f, O0 + k, Q0 + k);
      if (has1)
        yu1 = iter_elem<VS, false>(-zz.y * xn, ysm[W + k], TWO ? usm[W + k] : 0.f, w1, k,
                                   thr, thr_prev, ic, f, O0 + W + k, Q0 + W + k);
      return make_float2(yu0, yu1);
    };

    long p0 = (long)blockIdx.x * S + s;
    issue_F(p0);
    cp_async_commit();
    issue_YU(p0);
    cp_async_commit();
    if constexpr (NW > 0 && ct_reg_edges(NW, RM)) {
      // Register hand-over: thread t holds the elements t + g m of the row
      // pair's transform both at the end of the inverse transform and at the
      // start of the forward one, so the unpacking of the spectrum rows, the
      // element-wise step and the first forward pass run on registers.
      constexpr int EM = NW / ct_threads(NW, RM);  // elements per thread
      constexpr int NP = ct_plan(NW, RM).np;
      for (long pb = (long)blockIdx.x * S; pb < npairs; pb += pstride) {
        const long p = pb + s;
        const bool valid = p < npairs;
        const long r0 = 2 * p, r1 = 2 * p + 1;
        const bool has1 = valid && (r1 < rows);
        float2 v[EM];
        cp_async_wait<1>();  // F(p)
        __syncthreads();
#pragma unroll
        for (int m = 0; m < EM; ++m)
          v[m] = valid ? pack_inverse(fst, fst + Wp, has1, t + g * m, W, Wf) : make_float2(0.f, 0.f);
        ct_first_from_regs<NW, RM, 1>(z, v, t);
        issue_F(p + pstride);  // the staged rows are consumed
        cp_async_commit();
        fft_ct_passes<NW, RM, ct_threads(NW, RM), 1, 1, NP - 1>(z, P.twW, t);
        cp_async_wait<1>();  // the pair's state rows
        __syncthreads();
        ct_last_to_regs<NW, RM, 1>(z, P.twW, v, t);
        if (ADJ && valid) {
          float* gv = P.gV + (size_t)b * img_real + (size_t)r0 * W;
          const bool firstq = P.first != 0;
          const RowW aw0 = roww(r0, true), aw1 = roww(r1, has1);
#pragma unroll
          for (int m = 0; m < EM; ++m) {
            const int k = t + g * m;
            const float q0 = firstq ? 0.f : v[m].x * P.invN;
            const float q1 = firstq ? 0.f : -v[m].y * P.invN;
            const float v0 = ysm[k];
            const float gy0 = firstq ? v0 : ic.a1 * v0 + rho * q0;
            const float gu0 = firstq ? 0.f : v0 - rho * q0;
            const float n0 = active(usm[k], aw0, k) ? gy0 : gu0;
            gv[k] = n0;
            float n1 = 0.f;
            if (has1) {
              const float v1 = ysm[W + k];
              const float gy1 = firstq ? v1 : ic.a1 * v1 + rho * q1;
              const float gu1 = firstq ? 0.f : v1 - rho * q1;
              n1 = active(usm[W + k], aw1, k) ? gy1 : gu1;
              gv[W + k] = n1;
            }
            v[m] = make_float2(ic.a * n0, ic.a * n1);
          }
        } else if (!ADJ && valid) {
          const RowW w0 = roww(r0, true), w1 = roww(r1, has1);
          const bool fast = has1 && w0.plain() && w1.plain();
          const float tc0 = thr * w0.w, tc1 = thr * w1.w;
          const float tq0 = thr_prev * w0.w, tq1 = thr_prev * w1.w;
          float* O0 = out0(r0);
          float* Q0 = outu(r0);
          float f[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
          if (fast && ic.delta) {
#pragma unroll
            for (int m = 0; m < EM; ++m)
              v[m] = elem_fast(IntC<1>{}, tc0, tc1, tq0, tq1, t + g * m, v[m], O0, Q0, f);
          } else if (fast) {
#pragma unroll
            for (int m = 0; m < EM; ++m)
              v[m] = elem_fast(IntC<0>{}, tc0, tc1, tq0, tq1, t + g * m, v[m], O0, Q0, f);
          } else {
#pragma unroll
            for (int m = 0; m < EM; ++m) v[m] = elem_gen(w0, w1, has1, t + g * m, v[m], O0, Q0, f);
          }
#pragma unroll
          for (int i = 0; i < 5; ++i) acc[i] += (double)f[i];
        } else {
#pragma unroll
          for (int m = 0; m < EM; ++m) v[m] = make_float2(0.f, 0.f);
        }
        ct_first_from_regs<NW, RM, 1>(z, v, t);
        issue_YU(p + pstride);  // the state staging is free again
        cp_async_commit();
        fft_ct_passes<NW, RM, ct_threads(NW, RM), 1, 1, NP>(z, P.twW, t);
        if (valid) {
          float2* fa = Fi + r0 * Wp;
          for (int k = t; k < Wf; k += g) {
            const float2 Zk = z[zs(k)];
            const float2 Zm = z[zs(k == 0 ? 0 : W - k)];
            fa[k] = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
            if (has1) fa[Wp + k] = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
          }
        }
        __syncthreads();
      }
    } else {
      for (long pb = (long)blockIdx.x * S; pb < npairs; pb += pstride) {
        const long p = pb + s;
        const bool valid = p < npairs;
        const long r0 = 2 * p, r1 = 2 * p + 1;
        const bool has1 = valid && (r1 < rows);
        cp_async_wait<1>();  // F(p)
        __syncthreads();
        if (valid) {
          for (int k = t; k < W; k += g) z[zs(k)] = pack_inverse(fst, fst + Wp, has1, k, W, Wf);
        }
        __syncthreads();
        issue_F(p + pstride);  // lands during this pair's transforms
        cp_async_commit();
        fft_any<NW, 1, RM>(z, P.pw, P.twW, t, g);
        cp_async_wait<1>();  // the pair's state rows
        __syncthreads();
        if (ADJ && valid) {
          // Q = IFFT(Q^) (zero before the first step); gradients w.r.t. Y and U
          // of this step, gY = (1 - a) gV + rho Q, gU = gV - rho Q; gV of the
          // step before: gY where its shrinkage was active (Y != 0), else gU.
          float* gv = P.gV + (size_t)b * img_real + (size_t)r0 * W;
          const bool firstq = P.first != 0;
          const RowW aw0 = roww(r0, true), aw1 = roww(r1, has1);
          for (int k = t; k < W; k += g) {
            const float2 zz = z[zs(k)];
            const float q0 = firstq ? 0.f : zz.x * P.invN;
            const float q1 = firstq ? 0.f : -zz.y * P.invN;
            const float v0 = ysm[k];
            const float gy0 = firstq ? v0 : ic.a1 * v0 + rho * q0;
            const float gu0 = firstq ? 0.f : v0 - rho * q0;
            const float n0 = active(usm[k], aw0, k) ? gy0 : gu0;
            gv[k] = n0;
            float n1 = 0.f;
            if (has1) {
              const float v1 = ysm[W + k];
              const float gy1 = firstq ? v1 : ic.a1 * v1 + rho * q1;
              const float gu1 = firstq ? 0.f : v1 - rho * q1;
              n1 = active(usm[W + k], aw1, k) ? gy1 : gu1;
              gv[W + k] = n1;
            }
            z[zs(k)] = make_float2(ic.a * n0, ic.a * n1);
          }
        } else if (!ADJ && valid) {
          const RowW w0 = roww(r0, true), w1 = roww(r1, has1);
          const bool fast = has1 && w0.plain() && w1.plain();
          const float tc0 = thr * w0.w, tc1 = thr * w1.w;
          const float tq0 = thr_prev * w0.w, tq1 = thr_prev * w1.w;
          float* O0 = out0(r0);
          float* Q0 = outu(r0);
          float f[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
          if (fast && ic.delta) {
            for (int k = t; k < W; k += g)
              z[zs(k)] = elem_fast(IntC<1>{}, tc0, tc1, tq0, tq1, k, z[zs(k)], O0, Q0, f);
          } else if (fast) {
            for (int k = t; k < W; k += g)
              z[zs(k)] = elem_fast(IntC<0>{}, tc0, tc1, tq0, tq1, k, z[zs(k)], O0, Q0, f);
          } else {
            for (int k = t; k < W; k += g) z[zs(k)] = elem_gen(w0, w1, has1, k, z[zs(k)], O0, Q0, f);
          }
#pragma unroll
          for (int i = 0; i < 5; ++i) acc[i] += (double)f[i];
        }
        __syncthreads();
        issue_YU(p + pstride);  // the state staging is free again
        cp_async_commit();
        fft_any<NW, 1, RM>(z, P.pw, P.twW, t, g);
        if (valid) {
          float2* fa = Fi + r0 * Wp;
          for (int k = t; k < Wf; k += g) {
            const float2 Zk = z[zs(k)];
            const float2 Zm = z[zs(k == 0 ? 0 : W - k)];
            // A = (Z_k + conj Z_{-k}) / 2 ;  B = (Z_k - conj Z_{-k}) / (2i)
            fa[k] = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
            if (has1) fa[Wp + k] = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
          }
        }
        __syncthreads();
      }
    }
    cp_async_wait<0>();
    if constexpr (ADJ) return;
    block_sum<5>(acc, red_scratch);
    if (threadIdx.x == 0) {
      double* out = P.partials + ((size_t)b * P.nblk + blockIdx.x) * 5;
#pragma unroll
      for (int i = 0; i < 5; ++i) out[i] = acc[i];
    }
    return;
  } else {
    // ---------------------------------------------- setup and tool modes
    for (long pb = (long)blockIdx.x * S; pb < npairs; pb += pstride) {
      const long p = pb + s;
      const bool valid = p < npairs;
      const long r0 = 2 * p, r1 = 2 * p + 1;
      const bool has1 = valid && (r1 < rows);
      if constexpr (MODE == ROW_INV_REAL) {
        if (valid) {
          const float2* a = Fi + r0 * Wp;
          for (int k = t; k < W; k += g) z[zs(k)] = pack_inverse(a, a + Wp, has1, k, W, Wf);
        }
        __syncthreads();
        fft_any<NW, 1, RM>(z, P.pw, P.twW, t, g);
        if (valid) {
          float* d0 = P.dst + (size_t)b * img_real + (size_t)r0 * W;
          for (int k = t; k < W; k += g) {
            const float2 zz = z[zs(k)];
            d0[k] = zz.x * P.invN;
            if (has1) d0[W + k] = -zz.y * P.invN;
          }
        }
        __syncthreads();
        continue;
      }
      if (valid) {
        if constexpr (MODE == ROW_FWD_REAL) {
          const float* s0 = P.src + (size_t)b * img_real + (size_t)r0 * W;
          for (int k = t; k < W; k += g) z[zs(k)] = make_float2(s0[k], has1 ? s0[W + k] : 0.f);
        } else if constexpr (MODE == ROW_FWD_DICT) {
          const int m0 = (int)(r0 / H), h0 = (int)(r0 - (long)m0 * H);
          const int m1 = (int)(r1 / H), h1 = (int)(r1 - (long)m1 * H);
          for (int k = t; k < W; k += g) {
            float v0 = 0.f, v1 = 0.f;
            if (h0 < P.Kr && k < P.Kc) v0 = P.D[((size_t)m0 * P.Kr + h0) * P.Kc + k];
            if (has1 && h1 < P.Kr && k < P.Kc) v1 = P.D[((size_t)m1 * P.Kr + h1) * P.Kc + k];
            z[zs(k)] = make_float2(v0, v1);
          }
        } else if constexpr (MODE == ROW_FWD_YU) {
          const float* Y0 = P.Y + (size_t)b * img_real + (size_t)r0 * W;
          const float* U0 = P.U + (size_t)b * img_real + (size_t)r0 * W;
          for (int k = t; k < W; k += g)
            z[zs(k)] = make_float2(Y0[k] - U0[k], has1 ? Y0[W + k] - U0[W + k] : 0.f);
        }
      }
      __syncthreads();
      fft_any<NW, 1, RM>(z, P.pw, P.twW, t, g);
      if (valid) {
        float2* a = Fi + r0 * Wp;
        float2* bb = Fi + r1 * Wp;
        for (int k = t; k < Wf; k += g) {
          const float2 Zk = z[zs(k)];
          const float2 Zm = z[zs(k == 0 ? 0 : W - k)];
          const float2 A = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
          const float2 Bv = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
          a[k] = A;
          if (has1) bb[k] = Bv;
        }
      }
      __syncthreads();
    }
  }
}

// =========================================================== column pass ==
// Grid (G, ntiles, B).  For COL_SOLVE the G CTAs of one column tile form a
// thread-block cluster; each handles a contiguous chunk of the maps.  Tiles
// keep their HBM layout in shared memory: element (kr, c) of the tile at
// [slot(kr) * T + c]; thread tid works on column c = tid % T and, in the
// element loops, on rows kr = tid / T + i g.
// RADIX: the radix of the column transform plan (0: col_radix(NH)); it sets
// the threads per column (NH / RADIX) and the rows per thread.  TW: columns
// per tile (4, or 2 for the convolution solves: half the shared memory and
// threads per CTA, twice the tiles).
template <int MODE, int NH, int RADIX = 0, int TW = SC_COL_TILE>
__global__ void __launch_bounds__(SC_COL_MAX_THREADS)
col_kernel(ColParams P) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int T = TW;
  static_assert(T == 2 || T == 4, "tiles of 2 or 4 columns");
  constexpr int RM = RADIX > 0 ? RADIX : col_radix(NH);
  // elements of the tile per thread (compile-time bound)
  constexpr int EPT = NH > 0 ? (NH + ct_threads(NH, RM) - 1) / ct_threads(NH, RM) : SC_MAXE;
  const Geom& G = P.g;
  const int H = G.H, Wf = G.Wf, Wp = G.Wp, M = G.M;
  const int hlen = NH > 0 ? ct_len(NH, RM, T) : H;
  const int TL = T * hlen;  // shared-memory slots of one tile
  float2* stg = reinterpret_cast<float2*>(smem_raw);  // [F0][F1][D]

  const int b = blockIdx.z;
  const int tile = P.tile0 + blockIdx.y;
  const int rank = blockIdx.x;
  const int c0 = tile * T;
  const int g = NH > 0 ? ct_threads(NH, RM) : P.gsz;
  const int NT = blockDim.x;
  const int tid = threadIdx.x;
  const int cc = tid % T;   // column of this thread (T divides NT)
  const int t = tid / T;    // index within the column's thread group
  auto slot = [](int kr) { return fft_slot<NH, RM, T>(kr); };

  float rho = 0.f;
  if constexpr (col_clustered(MODE)) {
    const ImgState& st = P.st[b];
    if (st.done) return;  // uniform over the cluster (same image)
    rho = (float)st.rho;
  }

  const int chunk = (M + P.G - 1) / P.G;
  const int m0 = rank * chunk;
  const int m1 = min(M, m0 + chunk);
  float2* Fi = P.F + (size_t)b * M * H * Wp;

  if constexpr (MODE == COL_FWD || MODE == COL_INV) {
    // setup / tool: plain loads (the spectrum pitch may be unaligned here)
    const bool inv = MODE == COL_INV;
    for (int m = m0; m < m1; ++m) {
      float2* src = Fi + (size_t)m * H * Wp + c0;
      for (int e = tid; e < T * H; e += NT) {
        const int kr = e / T, c = e - kr * T;
        float2 v = make_float2(0.f, 0.f);
        if (c0 + c < Wf) v = src[(size_t)kr * Wp + c];
        if (inv) v.y = -v.y;
        stg[slot(kr) * T + c] = v;
      }
      __syncthreads();
      fft_any<NH, T, RM>(stg + cc, P.ph, P.twH, t, g);
      for (int e = tid; e < T * H; e += NT) {
        const int kr = e / T, c = e - kr * T;
        if (c0 + c < Wf) {
          float2 v = stg[slot(kr) * T + c];
          if (inv) v.y = -v.y;
          src[(size_t)kr * Wp + c] = v;
        }
      }
      __syncthreads();
    }
    return;
  } else if constexpr (col_taps(MODE) > 0) {
    // Plain solve (d = rho) with the column direction done by direct
    // convolution.  In the row-spectral domain (F = row spectra P_m of
    // (Y - U)_m) filter m is E_m(t, kc), t < Kr (the row spectra of its rows),
    // and its column spectrum is Df_m(kr) = sum_t E_m(t) w^(t kr).  Hence
    //   sum_m Df_m Z^_m = FFTcol(a),   a(r) = sum_m sum_t E_m(t) P_m(r - t)
    //   IFFTcol(conj(Df_m) SC)(r) = sum_t conj(E_m(t)) sc(r + t),  sc = IFFTcol(SC)
    // (circular in r, unnormalised transforms), so
    //   IFFTcol(x^_m) = H P_m + sum_t conj(E_m(t)) sc(r + t) / rho:
    // pass 1 accumulates a over the maps (Kr complex multiply-adds per
    // element), one column FFT pair per tile gives SC = S^ - cb and sc, and
    // pass 2 writes every map's result.  Each thread owns L consecutive rows
    // of one column and slides a window of L values along the column.
    //
    // COL_SOLVE_G16: the gradient term, one d(kr, kc) = rho + mu w |G|^2 for
    // every map.  Pass 1 is the same (sum_m Df_m Z^_m, then SC with d); the
    // solution x^_m = (rho Z^_m + conj(Df_m) SC) / d splits into
    //   IFFTcol(x^_m)(r) = IFFTcol(rho Z^_m / d)(r) + sum_t conj(E_m(t)) sc'(r + t),
    //   sc' = IFFTcol(SC / d):
    // pass 2 transforms each map's tile forward and back (1/d varies along
    // the column) and adds the convolution term.  The column spectra are
    // neither written back nor the dictionary spectra read.
    //
    // COL_SOLVE_C8T / C16T (the adjoint's recomputation) also keep the pass's
    // output (the row spectra of X) in Xtr and sc / rho in SCtr.
    //
    // COL_ADJ_C8 / C16: the adjoint of the plain solve, A = rho I + conj(Df)
    // Df^T per frequency, in the same form.  F holds g_m, the row spectra of
    // a gV; with G^_m = FFTcol(g_m):
    //   cb = sum_m Df_m G^_m / (rho + Psum)     (pass 1 as above; gS^ += cb)
    //   IFFTcol(Q^_m)(r) = (H g_m(r) - sum_t conj(E_m(t)) cb'(r + t)) / rho,
    //   cb' = IFFTcol(cb)                        (pass 2, written to F)
    // and the dictionary gradient (S^ - sum_j Df_j X^_j) conj(Q^_m) -
    // cb conj(X^_m), needed only at the Kr filter rows after the inverse
    // column transform, is a circular correlation there:
    //   gE_m(t) += sum_s rho sc'(s + t) conj(q_m(s)) - cb'(s + t) conj(x_m(s)),
    // sc' = SCtr and x_m = Xtr of the step (unnormalised; the caller scales),
    // q_m the pass-2 output.  Each thread sums over its L rows, the column's
    // threads are summed by shuffles and per-warp partials, in a fixed order.
    if constexpr (NH > 0) {
      constexpr bool GRD = MODE == COL_SOLVE_G16;
      constexpr bool TRACE = MODE == COL_SOLVE_C8T || MODE == COL_SOLVE_C16T;
      constexpr bool ADJ = col_adj_conv(MODE);
      constexpr int KMAX = col_taps(MODE);
      constexpr int L = EPT;  // rows per thread; g L = H for every compiled length
      constexpr int NW = L + KMAX - 1;  // window of the L outputs
      const int Kr = P.Kr;
      float2* A = stg;            // cluster sum, its spectrum, then sc / rho
      float2* Bt = stg + TL;      // spectrum tiles (pass 1: with A; pass 2: with Ct)
      float2* Ct = stg + 2 * TL;  // partial sums of this CTA
      // [3][KMAX][T] filter rows, one float4 (two float2 slots) an entry
      constexpr int ES = 2 * KMAX * T;  // float2 slots of one staged filter tile
      float2* Es = stg + 3 * TL;
      // ADJ: the forward's sc / rho tile, then per-warp correlation partials
      float2* W4 = Es + 3 * ES;
      float2* X5 = W4 + TL;       // ADJ: the forward's row spectra of X of the map
      float2* red = X5 + TL;      // [2][NT / 32][KMAX][T]
      // 16-byte copies: T / 2 per tile row
      constexpr int CPR = T / 2;
      auto issue_tile = [&](const float2* base, float2* dst) {
        for (int q = tid; q < CPR * H; q += NT) {
          const int kr = q / CPR, h = q % CPR;
          cp_async16(dst + slot(kr) * T + 2 * h, base + (size_t)kr * Wp + c0 + 2 * h);
        }
      };
      auto issue_E = [&](int m, float2* dst) {
        float4* d4 = reinterpret_cast<float4*>(dst);
        for (int q = tid; q < T * Kr; q += NT) {
          const int r = q / T, h = q - r * T;
          cp_async16(d4 + r * T + h, P.E + ((size_t)m * Kr + r) * Wp + c0 + h);
        }
      };
      // filter-row entry of tap tp of this thread's column: (Re e, Im e,
      // Re e + Im e, Im e - Re e)
      auto ent = [&](const float2* ecur, int tp) -> float4 {
        return reinterpret_cast<const float4*>(ecur)[tp * T + cc];
      };
      const size_t plane = (size_t)H * Wp;
      const float2* Sh = P.Sh + (size_t)b * plane + c0;
      const bool colok = c0 + cc < Wf;
      const float irho = 1.f / rho;
      const int r0 = t * L;
      // Slot of row r0 + d, d a compile-time offset.  When a thread's L rows
      // are exactly one padded block of the layout (L == RM, the pad period),
      // row r0 + d lies in block t + floor(d / L) (mod the H / L blocks) at
      // offset d mod L, so every window access is a per-thread block base
      // plus a constant.
      constexpr bool BLK = L == RM;
      int bbase[5];  // slot of the first row of block t + delta, delta = -2..2
#pragma unroll
      for (int dl = -2; dl <= 2; ++dl) {
        const int nb = H / L;
        int bi = t + dl;
        if (bi < 0) bi += nb;
        if (bi >= nb) bi -= nb;
        bbase[dl + 2] = bi * (L + 1);
      }
      auto rslot = [&](int d) -> int {  // d in (-2L, 2L); compile-time after unrolling
        if constexpr (BLK) {
          const int dl = d >= 0 ? d / L : -((-d + L - 1) / L);
          return bbase[dl + 2] + (d - dl * L);
        } else {
          int rr = r0 + d;
          if (rr < 0) rr += H;
          if (rr >= H) rr -= H;
          return slot(rr);
        }
      };

      // ------------------------------------------------------------ pass 1
      // The three tile buffers rotate: map m's tiles are copied two maps
      // ahead.  One barrier per map: after it, map m's tiles are visible and
      // every thread is done with map m - 1's buffers, which then take map
      // m + 2.
      auto buf = [&](int i) -> float2* { return i == 0 ? A : i == 1 ? Bt : Ct; };
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (m0 + q < m1) {
          issue_tile(Fi + (size_t)(m0 + q) * plane, buf(q));
          issue_E(m0 + q, Es + q * ES);
        }
        cp_async_commit();
      }
      // The map loop; body(cur, ecur) consumes map m's tile and filter rows.
      auto pass1_maps = [&](auto&& body) {
        int bi = 0;  // (m - m0) mod 3
        for (int m = m0; m < m1; ++m, bi = bi == 2 ? 0 : bi + 1) {
          cp_async_wait<1>();  // P(m), E(m) (those of m + 1 may still be in flight)
          __syncthreads();
          if (m + 2 < m1) {
            const int bn = bi == 0 ? 2 : bi - 1;  // (m - m0 + 2) mod 3
            issue_tile(Fi + (size_t)(m + 2) * plane, buf(bn));
            issue_E(m + 2, Es + bn * ES);
          }
          cp_async_commit();
          body(buf(bi), Es + bi * ES);
        }
      };
      // Filter-row counts with compile-time tap loops in Gauss's form below:
      // KMAX, and 12 and 11 for the 16-tap modes (11 x 11 and 12 x 12
      // filters) at up to 8 rows per thread (with 16, the extra variants
      // cost the 16-tap one about 2 %).  f(IntC<KR>) runs for such a count;
      // false otherwise.
      auto with_taps = [&](auto&& f) -> bool {
        if (Kr == KMAX) {
          f(IntC<KMAX>{});
          return true;
        }
        if constexpr (KMAX == 16 && L <= 8) {
          if (Kr == 12) {
            f(IntC<12>{});
            return true;
          }
          if (Kr == 11) {
            f(IntC<11>{});
            return true;
          }
        }
        return false;
      };
      float2 acc[L];
      const bool gauss1 = with_taps([&](auto kc) {
        // Three real multiply-adds per complex one (Gauss): with e = c + i d
        // and P = a + i b,
        //   Re(e P) = c (a + b) - b (c + d),  Im(e P) = c (a + b) + a (d - c),
        // the sums of c (a + b), b (c + d) and a (d - c) kept apart over the
        // maps and taps; c + d and d - c are formed once per map and tap,
        // a + b once per map and window element.
        constexpr int KR = decltype(kc)::value;
        float k1[L], k3[L], k2[L];
#pragma unroll
        for (int i = 0; i < L; ++i) k1[i] = k2[i] = k3[i] = 0.f;
        pass1_maps([&](const float2* cur, const float2* ecur) {
          float ec[KR], ep[KR], em[KR];
#pragma unroll
          for (int tp = 0; tp < KR; ++tp) {
            const float4 e = ent(ecur, tp);
            ec[tp] = e.x;
            ep[tp] = e.z;  // c + d
            em[tp] = e.w;  // d - c
          }
          // window element j = P(r0 - (KR - 1) + j) meets output i at tap
          // KR - 1 + i - j (the last tap first, as in the general form)
#pragma unroll
          for (int j = 0; j < L + KR - 1; ++j) {
            const float2 v = cur[rslot(j - (KR - 1)) * T + cc];
            const float sab = v.x + v.y;
#pragma unroll
            for (int i = 0; i < L; ++i) {
              const int tp = KR - 1 + i - j;
              if (tp >= 0 && tp < KR) {
                k1[i] = fmaf(ec[tp], sab, k1[i]);
                k3[i] = fmaf(ep[tp], v.y, k3[i]);
                k2[i] = fmaf(em[tp], v.x, k2[i]);
              }
            }
          }
        });
#pragma unroll
        for (int i = 0; i < L; ++i) acc[i] = make_float2(k1[i] - k3[i], k1[i] + k2[i]);
      });
      if (!gauss1) {
#pragma unroll
        for (int i = 0; i < L; ++i) acc[i] = make_float2(0.f, 0.f);
        pass1_maps([&](const float2* cur, const float2* ecur) {
          // w[j] = P(r0 - (KMAX - 1) + j): the window of all L outputs
          float2 w[NW];
#pragma unroll
          for (int j = 0; j < NW; ++j)
            w[j] = (j < KMAX - Kr) ? make_float2(0.f, 0.f) : cur[rslot(j - (KMAX - 1)) * T + cc];
          // last tap first: it uses the window values that were loaded first
#pragma unroll
          for (int tp = KMAX - 1; tp >= 0; --tp) {
            if (tp < Kr) {
              const float4 e = ent(ecur, tp);
#pragma unroll
              for (int i = 0; i < L; ++i) {
                const float2 v = w[i - tp + KMAX - 1];
                // four fused multiply-adds per complex multiply-add
                acc[i].x = fmaf(e.x, v.x, acc[i].x);
                acc[i].x = fmaf(-e.y, v.y, acc[i].x);
                acc[i].y = fmaf(e.x, v.y, acc[i].y);
                acc[i].y = fmaf(e.y, v.x, acc[i].y);
              }
            }
          }
        });
      }
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
      // DL: the plain solves with ColParams::delta write only the
      // correction sum_t conj(E_m(t)) sc(r + t) / rho (the row pass adds
      // Y - U, whose row spectra P_m are), so pass 2 reads no P tiles
      const bool DL = !GRD && !ADJ && !TRACE && P.delta;
      const float irho_s = DL ? (float)(1.0 / ((double)rho * H * G.W)) : irho;
      // pass 2's first tile lands during the reduction and the transforms
      if (m0 < m1) {
        if (!DL) issue_tile(Fi + (size_t)m0 * plane, Bt);
        issue_E(m0, Es);
        if constexpr (ADJ) {
          issue_tile(P.SCtr + (size_t)b * plane, W4);
          issue_tile(P.Xh + ((size_t)b * M + m0) * plane, X5);
        }
      }
      cp_async_commit();

      // ------------------------------------------- sum over the cluster
      if (P.G > 1) {
#pragma unroll
        for (int i = 0; i < L; ++i) Ct[rslot(i) * T + cc] = acc[i];
        cg::cluster_group cluster = cg::this_cluster();
        cluster.sync();
        for (int e = tid; e < T * H; e += NT) {
          const int kr = e / T, c = e - (e / T) * T;
          const int sl = slot(kr) * T + c;
          float2 v = make_float2(0.f, 0.f);
          for (int r = 0; r < P.G; ++r) {
            const float2 u = cluster.map_shared_rank(Ct, r)[sl];
            v.x += u.x;
            v.y += u.y;
          }
          A[sl] = v;
        }
        cluster.sync();
      } else {
#pragma unroll
        for (int i = 0; i < L; ++i) A[rslot(i) * T + cc] = acc[i];
        __syncthreads();
      }
      // The plain solves (and their trace twins) copy pass 2's tiles two
      // maps ahead as well, over the three tile buffers (A is free once the
      // window is in registers): the second tile lands in Ct, free now.  With
      // a tap count in Gauss's form (GAUSS2) pass 2 streams the window from A
      // instead and alternates Bt and Ct.
      constexpr bool PIPE3 = !GRD && !ADJ;
      const bool GAUSS2 =
          PIPE3 && (Kr == KMAX || (KMAX == 16 && L <= 8 && (Kr == 12 || Kr == 11)));
      if constexpr (PIPE3) {
        if (m0 + 1 < m1 && !GAUSS2) {
          if (!DL) issue_tile(Fi + (size_t)(m0 + 1) * plane, Ct);
          issue_E(m0 + 1, Es + ES);
        }
        cp_async_commit();
      }
      // ------------ SC = S^ - cb, sc = IFFTcol(SC) / rho (GRD: IFFTcol(SC / d))
      // 1 / d at row kr of this thread's column (GRD)
      const float wg = GRD ? P.mu * P.wgrd[0] : 0.f;
      const float gw_col = GRD && colok ? 2.f - 2.f * __ldg(&P.twW[c0 + cc]).x : 0.f;
      auto inv_d = [&](int kr) -> float {
        return 1.f / (wg * (gw_col + 2.f - 2.f * __ldg(&P.twH[kr]).x) + rho);
      };
      fft_any<NH, T, RM>(A + cc, P.ph, P.twH, t, g);
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) {
          const int sl = slot(kr) * T + cc;
          float2 v = make_float2(0.f, 0.f);
          if (colok) {
            const float2 q = A[sl];  // sum_m Df_m Z^_m (ADJ: sum_m Df_m G^_m)
            if constexpr (ADJ) {
              const float id = 1.f / (rho + __ldg(&P.Psum[(size_t)kr * Wp + c0 + cc]));
              const float2 cb = make_float2(q.x * id, q.y * id);
              if (rank == 0) {
                float2* gs = P.gSh + (size_t)b * plane + (size_t)kr * Wp + c0 + cc;
                const float2 o = *gs;
                *gs = make_float2(o.x + cb.x, o.y + cb.y);
              }
              v = make_float2(cb.x, -cb.y);  // conj(cb)
            } else {
            const float2 Sv = __ldg(&Sh[(size_t)kr * Wp + cc]);
            // SC = S^ - cb with cb = (S^ Psum / d + rho q / d) / (1 + Psum / d),
            // computed as SC = (S^ - rho q / d) / (1 + Psum / d): the same
            // value without subtracting cb, which is close to S^ when
            // Psum >> d (many maps), from S^ (that cancellation multiplied
            // the rounding error of SC by about 1 + Psum / d)
            if constexpr (GRD) {
              const float id = inv_d(kr);
              const float sd = __ldg(&P.Psum[(size_t)kr * Wp + c0 + cc]) * id;
              const float f = id / (1.f + sd);
              const float rid = rho * id;
              v = make_float2((Sv.x - rid * q.x) * f, -(Sv.y - rid * q.y) * f);  // conj(SC) / d
            } else {
              const float sd = __ldg(&P.Psum[(size_t)kr * Wp + c0 + cc]) * irho;
              // conj(SC) / rho (DL: also times 1 / (H W), the row pass's
              // normalisation of its inverse transform, which then skips it)
              const float f = irho_s / (1.f + sd);
              v = make_float2((Sv.x - q.x) * f, -(Sv.y - q.y) * f);
            }
            }
          }
          A[sl] = v;
        }
      }
      __syncthreads();
      fft_any<NH, T, RM>(A + cc, P.ph, P.twH, t, g);
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) {
          const int sl = slot(kr) * T + cc;
          A[sl].y = -A[sl].y;
          // the forward's sc / rho of this step, for the adjoint
          if (TRACE && rank == 0 && colok)
            P.SCtr[(size_t)b * plane + (size_t)kr * Wp + c0 + cc] = A[sl];
        }
      }
      // ------------------------------------------------------------ pass 2
      const float hs = (float)H;
      float2* Fo = Fi + c0 + cc;
      __syncthreads();  // sc complete before the windows are read
      auto store_out = [&](int m, const float2* o) {
        if (colok) {
          float2* dst = Fo + (size_t)m * plane + (size_t)r0 * Wp;
#pragma unroll
          for (int i = 0; i < L; ++i) dst[(size_t)i * Wp] = o[i];
          if constexpr (TRACE) {
            float2* xt = P.Xtr + (size_t)b * M * plane + c0 + cc + (size_t)m * plane +
                         (size_t)r0 * Wp;
#pragma unroll
            for (int i = 0; i < L; ++i) xt[(size_t)i * Wp] = o[i];
          }
        }
      };
      // o[i] += sum_t conj(E_m(t)) w(r0 + i + t) over KR taps in Gauss's form
      // (as in pass 1, for conj(E) = c + i d, c = Re E, d = -Im E), the
      // window w = sc / rho (GRD: sc'; ADJ: -cb', from cb' in A) streamed
      // from A.
      auto conv2 = [&](auto kc, const float2* ecur, float2* o) {
        constexpr int KR = decltype(kc)::value;
        float ec[KR], ep[KR], em[KR];
#pragma unroll
        for (int tp = 0; tp < KR; ++tp) {
          const float4 e = ent(ecur, tp);
          if constexpr (ADJ) {  // -conj(E)
            ec[tp] = -e.x;
            ep[tp] = e.w;   // d - c
            em[tp] = e.z;   // c + d
          } else {
            ec[tp] = e.x;
            ep[tp] = -e.w;  // c - d
            em[tp] = -e.z;  // -(c + d)
          }
        }
        float k1[L], k3[L], k2[L];
#pragma unroll
        for (int i = 0; i < L; ++i) {
          k1[i] = 0.f;
          k3[i] = -o[i].x;
          k2[i] = o[i].y;
        }
        // window element j meets output i at tap j - i
#pragma unroll
        for (int j = 0; j < L + KR - 1; ++j) {
          const float2 v = A[rslot(j) * T + cc];
          const float sab = v.x + v.y;
#pragma unroll
          for (int i = 0; i < L; ++i) {
            const int tp = j - i;
            if (tp >= 0 && tp < KR) {
              k1[i] = fmaf(ec[tp], sab, k1[i]);
              k3[i] = fmaf(ep[tp], v.y, k3[i]);
              k2[i] = fmaf(em[tp], v.x, k2[i]);
            }
          }
        }
#pragma unroll
        for (int i = 0; i < L; ++i) o[i] = make_float2(k1[i] - k3[i], k1[i] + k2[i]);
      };
      // Tap counts with compile-time loops in the adjoint (12 and 11 in the
      // 16-tap modes, 8 in the 8-tap ones; with 16 the correlation's
      // accumulators would spill registers): f(IntC<KR>) runs for such a
      // count; false otherwise.
      auto with_taps_adj = [&](auto&& f) -> bool {
        if constexpr (KMAX == 16 && L <= 8) {
          if (Kr == 12) {
            f(IntC<12>{});
            return true;
          }
          if (Kr == 11) {
            f(IntC<11>{});
            return true;
          }
        } else if constexpr (KMAX == 8) {
          if (Kr == 8) {
            f(IntC<8>{});
            return true;
          }
        }
        return false;
      };
      // ADJ with such a tap count: the convolution in Gauss's form and the
      // correlation read cb' from A (no window in registers)
      const bool ADJG = ADJ && (KMAX == 16 ? (L <= 8 && (Kr == 12 || Kr == 11)) : Kr == 8);
      if constexpr (PIPE3) {
        if (GAUSS2) {
          int it = 0;
          for (int m = m0; m < m1; ++m, ++it) {
            const float2* cur = (it & 1) ? Ct : Bt;
            const float2* ecur = Es + (it & 1) * ES;
            cp_async_wait<0>();  // P(m), E(m): the only copies in flight
            __syncthreads();
            if (m + 1 < m1) {
              if (!DL) issue_tile(Fi + (size_t)(m + 1) * plane, (it & 1) ? Bt : Ct);
              issue_E(m + 1, Es + ((it + 1) & 1) * ES);
            }
            cp_async_commit();
            float2 o[L];
#pragma unroll
            for (int i = 0; i < L; ++i) {
              const float2 pv = DL ? make_float2(0.f, 0.f) : cur[rslot(i) * T + cc];
              o[i] = make_float2(hs * pv.x, hs * pv.y);
            }
            with_taps([&](auto kc) { conv2(kc, ecur, o); });
            store_out(m, o);
          }
          cp_async_commit();
          cp_async_wait<0>();
          return;
        }
      }
      // w[j] = sc(r0 + j) / rho (GRD: sc'(r0 + j)): the window of all L
      // outputs, the same for every map (GRD: re-read per map, so that it is
      // not held across the transforms)
      float2 w[NW];
      auto load_window = [&]() {
#pragma unroll
        for (int j = 0; j < NW; ++j) {
          w[j] = (j < L + Kr - 1) ? A[rslot(j) * T + cc] : make_float2(0.f, 0.f);
          if constexpr (ADJ) w[j] = make_float2(-w[j].x, -w[j].y);  // -cb'
        }
      };
      if constexpr (!GRD) {
        if (!ADJG) load_window();
      }
      // rho / d at this thread's rows (GRD)
      const float rho_c = rho;
      // One barrier per map as in pass 1, except in the adjoint, whose
      // per-warp partial sums need a barrier after the map as well.  PIPE3:
      // buffers Bt, Ct, A in rotation, copies two maps ahead; otherwise Bt
      // and Ct alternate, copies one map ahead.
      int it = 0;
      int bi = 0;
      for (int m = m0; m < m1; ++m, ++it, bi = bi == 2 ? 0 : bi + 1) {
        float2* cur = PIPE3 ? (bi == 0 ? Bt : bi == 1 ? Ct : A) : (it & 1) ? Ct : Bt;
        const float2* ecur = Es + (PIPE3 ? bi : (it & 1)) * ES;
        if constexpr (PIPE3) {
          cp_async_wait<1>();  // P(m), E(m) (those of m + 1 may still be in flight)
          __syncthreads();
          if (m + 2 < m1) {
            const int bn = bi == 0 ? 2 : bi - 1;  // (it + 2) mod 3
            if (!DL) issue_tile(Fi + (size_t)(m + 2) * plane, bn == 0 ? Bt : bn == 1 ? Ct : A);
            issue_E(m + 2, Es + bn * ES);
          }
          cp_async_commit();
        } else if constexpr (ADJ) {
          if (m + 1 < m1) {
            issue_tile(Fi + (size_t)(m + 1) * plane, (it & 1) ? Bt : Ct);
            issue_E(m + 1, Es + ((it + 1) & 1) * ES);
          }
          cp_async_commit();
          cp_async_wait<1>();  // P(m), E(m)
          __syncthreads();
        } else {
          cp_async_wait<0>();  // P(m), E(m): the only copies in flight
          __syncthreads();
          if (m + 1 < m1) {
            issue_tile(Fi + (size_t)(m + 1) * plane, (it & 1) ? Bt : Ct);
            issue_E(m + 1, Es + ((it + 1) & 1) * ES);
          }
          cp_async_commit();
        }
        float2 o[L];
        bool convd = false;  // the convolution term is added (GRD, Gauss's form)
        if constexpr (GRD) {
          // IFFTcol(rho Z^_m / d) as conj(FFT(conj(rho FFT(P_m) / d)))
          fft_any<NH, T, RM>(cur + cc, P.ph, P.twH, t, g);
#pragma unroll
          for (int i = 0; i < L; ++i) {
            const int sl = rslot(i) * T + cc;
            const float f = rho_c * inv_d(r0 + i);
            const float2 z = cur[sl];
            cur[sl] = make_float2(f * z.x, -f * z.y);
          }
          __syncthreads();
          fft_any<NH, T, RM>(cur + cc, P.ph, P.twH, t, g);
#pragma unroll
          for (int i = 0; i < L; ++i) {
            const float2 v = cur[rslot(i) * T + cc];
            o[i] = make_float2(v.x, -v.y);
          }
          // (Gauss's form only at up to 8 rows per thread: with 16, its
          // registers next to the transforms' would spill)
          if constexpr (L <= 8) convd = with_taps([&](auto kc) { conv2(kc, ecur, o); });
          if (!convd) load_window();
        } else {
#pragma unroll
          for (int i = 0; i < L; ++i) {
            const float2 pv = DL ? make_float2(0.f, 0.f) : cur[rslot(i) * T + cc];
            o[i] = make_float2(hs * pv.x, hs * pv.y);
          }
          if constexpr (ADJ) {
            if (ADJG) convd = with_taps_adj([&](auto kc) { conv2(kc, ecur, o); });
          }
        }
#pragma unroll
        for (int tp = 0; tp < KMAX; ++tp) {
          if (tp < Kr && !convd) {
            const float4 e = ent(ecur, tp);
#pragma unroll
            for (int i = 0; i < L; ++i) {
              const float2 v = w[i + tp];
              o[i].x = fmaf(e.x, v.x, o[i].x);
              o[i].x = fmaf(e.y, v.y, o[i].x);
              o[i].y = fmaf(e.x, v.y, o[i].y);
              o[i].y = fmaf(-e.y, v.x, o[i].y);
            }
          }
        }
        if constexpr (ADJ) {
          // gE_m(t) partial sums over this thread's rows, taken before o is
          // scaled to q_m = o / rho: rho sc'(s + t) conj(q_m(s)) =
          // W4(s + t) conj(o(s)) with W4 = sc' (the SCtr tile); the window w
          // is -cb' (-A), xv the forward's row spectra of X at this step (its
          // tile staged in X5)
          float2 xv[L];
#pragma unroll
          for (int i = 0; i < L; ++i) xv[i] = X5[rslot(i) * T + cc];
          const int lane = tid & 31, wid = tid >> 5;
          float2* rp = red + (size_t)(it & 1) * (NT / 32) * KMAX * T;
          // With a compile-time tap count: window element j = s + t outer,
          // one accumulator per tap (independent chains; every tap still sums
          // over the rows in ascending order), each sc' and cb' value read
          // once
          const bool corr = with_taps_adj([&](auto kc) {
            constexpr int KR = decltype(kc)::value;
            float2 a[KR];
#pragma unroll
            for (int tp = 0; tp < KR; ++tp) a[tp] = make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 0; j < L + KR - 1; ++j) {
              const float2 sv = W4[rslot(j) * T + cc];  // sc'(s + t)
              const float2 cbv = A[rslot(j) * T + cc];
              const float2 c = make_float2(-cbv.x, -cbv.y);  // -cb'(s + t)
#pragma unroll
              for (int i = 0; i < L; ++i) {
                const int tp = j - i;
                if (tp >= 0 && tp < KR) {
                  // a += sv conj(o) + c conj(x)
                  a[tp].x = fmaf(sv.x, o[i].x, a[tp].x);
                  a[tp].x = fmaf(sv.y, o[i].y, a[tp].x);
                  a[tp].y = fmaf(sv.y, o[i].x, a[tp].y);
                  a[tp].y = fmaf(-sv.x, o[i].y, a[tp].y);
                  a[tp].x = fmaf(c.x, xv[i].x, a[tp].x);
                  a[tp].x = fmaf(c.y, xv[i].y, a[tp].x);
                  a[tp].y = fmaf(c.y, xv[i].x, a[tp].y);
                  a[tp].y = fmaf(-c.x, xv[i].y, a[tp].y);
                }
              }
            }
            // sum over the lanes of this column in the warp (same tid % T)
#pragma unroll
            for (int off = T; off < 32; off <<= 1) {
#pragma unroll
              for (int tp = 0; tp < KR; ++tp) {
                a[tp].x += __shfl_xor_sync(0xffffffffu, a[tp].x, off);
                a[tp].y += __shfl_xor_sync(0xffffffffu, a[tp].y, off);
              }
            }
            if (lane < T) {
#pragma unroll
              for (int tp = 0; tp < KR; ++tp) rp[((size_t)wid * KMAX + tp) * T + lane] = a[tp];
            }
          });
#pragma unroll
          for (int tp = 0; tp < KMAX; ++tp) {
            if (corr) break;
            if (tp >= Kr) break;  // uniform over the CTA
            float2 a = make_float2(0.f, 0.f);
#pragma unroll
            for (int i = 0; i < L; ++i) {
              const float2 c = w[i + tp];                    // -cb'(s + t)
              const float2 sv = W4[rslot(i + tp) * T + cc];  // sc'(s + t)
              // a += sv conj(o) + c conj(x)
              a.x = fmaf(sv.x, o[i].x, a.x);
              a.x = fmaf(sv.y, o[i].y, a.x);
              a.y = fmaf(sv.y, o[i].x, a.y);
              a.y = fmaf(-sv.x, o[i].y, a.y);
              a.x = fmaf(c.x, xv[i].x, a.x);
              a.x = fmaf(c.y, xv[i].y, a.x);
              a.y = fmaf(c.y, xv[i].x, a.y);
              a.y = fmaf(-c.x, xv[i].y, a.y);
            }
            // sum over the lanes of this column in the warp (same tid % T)
#pragma unroll
            for (int off = T; off < 32; off <<= 1) {
              a.x += __shfl_xor_sync(0xffffffffu, a.x, off);
              a.y += __shfl_xor_sync(0xffffffffu, a.y, off);
            }
            if (lane < T) rp[((size_t)wid * KMAX + tp) * T + lane] = a;
          }
#pragma unroll
          for (int i = 0; i < L; ++i) o[i] = make_float2(o[i].x * irho, o[i].y * irho);  // q_m
        }
        store_out(m, o);
        if constexpr (ADJ) {
          __syncthreads();  // the partial sums, and before the buffers are refilled
          if (m + 1 < m1) issue_tile(P.Xh + ((size_t)b * M + m + 1) * plane, X5);
          cp_async_commit();
          // gE += the column sums, warps in a fixed order (one thread per
          // filter row and column)
          const float2* rp = red + (size_t)(it & 1) * (NT / 32) * KMAX * T;
          for (int e = tid; e < Kr * T; e += NT) {
            const int tp = e / T, c = e - tp * T;
            if (c0 + c < Wf) {
              float2 sum = make_float2(0.f, 0.f);
              for (int wv = 0; wv < NT / 32; ++wv) {
                const float2 v = rp[((size_t)wv * KMAX + tp) * T + c];
                sum.x += v.x;
                sum.y += v.y;
              }
              float2* ge = P.gE + (((size_t)b * M + m) * Kr + tp) * Wp + c0 + c;
              const float2 o2 = *ge;
              *ge = make_float2(o2.x + sum.x, o2.y + sum.y);
            }
          }
        }
      }
      cp_async_commit();
      cp_async_wait<0>();
    }
  } else if constexpr (MODE == COL_SOLVE_P) {
    // Plain solve, d = rho for every map and frequency (cbpdn, cbpdnmsk).
    // With P_m the row spectra of (Y - U)_m held in F, Z^_m = FFTcol(P_m) and
    // x^_m = Z^_m + conj(Df_m) SC / rho, so the inverse column transform is
    //   IFFTcol(x^_m) = H P_m + IFFTcol(conj(Df_m) SC) / rho
    // (unnormalised transforms): pass 1 transforms P_m only to accumulate
    // sum_m Df_m Z^_m and writes nothing back; pass 2 transforms the
    // correction and adds H P_m, re-read from F.
    float2* fbuf[2] = {stg, stg + TL};
    float2* dbuf = stg + 2 * TL;
    auto issue_tile = [&](const float2* base, float2* dst) {
      for (int q = tid; q < 2 * H; q += NT) {
        const int kr = q >> 1, h = q & 1;
        cp_async16(dst + slot(kr) * T + 2 * h, base + (size_t)kr * Wp + c0 + 2 * h);
      }
    };
    const size_t plane = (size_t)H * Wp;
    const float2* Sh = P.Sh + (size_t)b * plane + c0;
    const bool colok = c0 + cc < Wf;
    const float irho = 1.f / rho;
    // pass 1: acc = sum_m Df_m Z^_m
    float2 num[EPT];
#pragma unroll
    for (int i = 0; i < EPT; ++i) num[i] = make_float2(0.f, 0.f);
    if (m0 < m1) {
      issue_tile(Fi + (size_t)m0 * plane, fbuf[0]);
      issue_tile(P.Dh + (size_t)m0 * plane, dbuf);
    }
    cp_async_commit();
    int it = 0;
    for (int m = m0; m < m1; ++m, ++it) {
      float2* cur = fbuf[it & 1];
      if (m + 1 < m1) issue_tile(Fi + (size_t)(m + 1) * plane, fbuf[(it + 1) & 1]);
      cp_async_commit();
      cp_async_wait<1>();  // F(m) and D(m)
      __syncthreads();
      fft_any<NH, T, RM>(cur + cc, P.ph, P.twH, t, g);
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) {
          const int sl = slot(kr) * T + cc;
          const float2 Dv = dbuf[sl];
          const float2 z = cur[sl];
          num[i].x += Dv.x * z.x - Dv.y * z.y;
          num[i].y += Dv.x * z.y + Dv.y * z.x;
        }
      }
      __syncthreads();
      if (m + 1 < m1) issue_tile(P.Dh + (size_t)(m + 1) * plane, dbuf);
      cp_async_commit();
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    // the dictionary tile of pass 2's first map lands during the reduction
    // (which uses [F1] only)
    const int E = T * H;
    float2* xn = fbuf[1];  // [E] complex, reduction scratch
    // SC = S^ - cb,  cb = sum_m Df_m b_m / (rho + Psum) = (S^ Psum / rho + acc) / (1 + Psum / rho)
    auto s_minus_cb = [&](int kr, int c, float2 acc) -> float2 {
      const int k = c0 + c;
      if (k >= Wf) return make_float2(0.f, 0.f);
      const float2 Sv = __ldg(&Sh[(size_t)kr * Wp + c]);
      const float sd = __ldg(&P.Psum[(size_t)kr * Wp + k]) * irho;
      // (S^ - acc) / (1 + Psum / rho): S^ - cb without the cancellation
      const float q = 1.f / (1.f + sd);
      return make_float2((Sv.x - acc.x) * q, (Sv.y - acc.y) * q);
    };
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int kr = t + i * g;
      if (kr < H) xn[kr * T + cc] = num[i];
    }
    if (m0 < m1) issue_tile(P.Dh + (size_t)m0 * plane, dbuf);
    cp_async_commit();
    if (P.G > 1) {
      cg::cluster_group cluster = cg::this_cluster();
      cluster.sync();
      const int sl = (E + P.G - 1) / P.G;
      const int e0 = rank * sl, e1 = min(E, e0 + sl);
      for (int e = e0 + tid; e < e1; e += NT) {
        float2 ns = make_float2(0.f, 0.f);
        for (int r = 0; r < P.G; ++r) {
          const float2 v = cluster.map_shared_rank(xn, r)[e];
          ns.x += v.x;
          ns.y += v.y;
        }
        xn[e] = s_minus_cb(e / T, e % T, ns);
      }
      cluster.sync();
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) {
          const int e = kr * T + cc;
          const int owner = e / sl;
          num[i] = owner == rank ? xn[e] : cluster.map_shared_rank(xn, owner)[e];
        }
      }
      cluster.sync();
    } else {
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) num[i] = s_minus_cb(kr, cc, num[i]);
      }
      __syncthreads();
    }
    // num[i] = SC / rho; pass 2
#pragma unroll
    for (int i = 0; i < EPT; ++i) num[i] = make_float2(num[i].x * irho, num[i].y * irho);
    const float hs = (float)H;
    float2* work = fbuf[0];
    float2* ptile = fbuf[1];
    for (int m = m0; m < m1; ++m) {
      cp_async_wait<0>();  // D(m)
      __syncthreads();
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) {
          const int sl = slot(kr) * T + cc;
          float2 v = make_float2(0.f, 0.f);
          if (colok) {
            const float2 Dv = dbuf[sl];
            const float2 sc = num[i];
            // conj(conj(Df) SC / rho): the inverse via the forward FFT
            v = make_float2(Dv.x * sc.x + Dv.y * sc.y, -(Dv.x * sc.y - Dv.y * sc.x));
          }
          work[sl] = v;
        }
      }
      __syncthreads();
      // P(m) lands during the transform, D(m+1) after it
      issue_tile(Fi + (size_t)m * plane, ptile);
      cp_async_commit();
      if (m + 1 < m1) issue_tile(P.Dh + (size_t)(m + 1) * plane, dbuf);
      cp_async_commit();
      fft_any<NH, T, RM>(work + cc, P.ph, P.twH, t, g);
      cp_async_wait<1>();  // P(m)
      __syncthreads();
      float2* dst = Fi + (size_t)m * plane + c0;
      if (colok) {
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
          const int kr = t + i * g;
          if (kr < H) {
            const int sl = slot(kr) * T + cc;
            const float2 v = work[sl], pv = ptile[sl];
            dst[(size_t)kr * Wp + cc] = make_float2(v.x + hs * pv.x, hs * pv.y - v.y);
          }
        }
      }
    }
    cp_async_wait<0>();
  } else if constexpr (MODE == COL_ADJ) {
    // Adjoint of the plain cbpdn solve, A = rho I + conj(Df) Df^T per
    // frequency (one d = rho for every map).  F holds the row spectra of
    // a gV; G^ is their column FFT and
    //   cb = sum_m Df_m G^_m / (rho + Psum),   Q^_m = (G^_m - conj(Df_m) cb) / rho,
    //   sum_m Df_m Q^_m = cb,                  gS^ += cb,
    //   gD^_m += (S^ - sum_j Df_j X^_j) conj(Q^_m) - cb conj(X^_m);
    // F receives the inverse column FFT of Q^.
    float2* fbuf[2] = {stg, stg + TL};
    float2* dbuf = stg + 2 * TL;
    auto issue_tile = [&](const float2* base, float2* dst) {
      for (int q = tid; q < 2 * H; q += NT) {
        const int kr = q >> 1, h = q & 1;
        cp_async16(dst + slot(kr) * T + 2 * h, base + (size_t)kr * Wp + c0 + 2 * h);
      }
    };
    const size_t plane = (size_t)H * Wp;
    const float2* Xb = P.Xh + (size_t)b * M * plane + c0;
    float2* gDb = P.gDh + (size_t)b * M * plane + c0;
    const float2* Sh = P.Sh + (size_t)b * plane + c0;
    float2* gSb = P.gSh + (size_t)b * plane + c0;
    const bool colok = c0 + cc < Wf;
    const float irho = 1.f / rho;

    // pass 1: G^, sum_m Df_m G^_m and sum_m Df_m X^_m; G^ written back in place
    float2 dg[EPT], dx[EPT];
#pragma unroll
    for (int i = 0; i < EPT; ++i) dg[i] = dx[i] = make_float2(0.f, 0.f);
    if (m0 < m1) {
      issue_tile(Fi + (size_t)m0 * plane, fbuf[0]);
      issue_tile(P.Dh + (size_t)m0 * plane, dbuf);
    }
    cp_async_commit();
    int it = 0;
    for (int m = m0; m < m1; ++m, ++it) {
      float2* cur = fbuf[it & 1];
      if (m + 1 < m1) issue_tile(Fi + (size_t)(m + 1) * plane, fbuf[(it + 1) & 1]);
      cp_async_commit();
      cp_async_wait<1>();  // F(m) and D(m)
      __syncthreads();
      fft_any<NH, T, RM>(cur + cc, P.ph, P.twH, t, g);
      float2* fout = Fi + (size_t)m * plane + c0;
      const float2* xin = Xb + (size_t)m * plane;
      if (colok) {
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
          const int kr = t + i * g;
          if (kr < H) {
            const int sl = slot(kr) * T + cc;
            const float2 Dv = dbuf[sl];
            const float2 gv = cur[sl];
            const float2 xv = __ldg(&xin[(size_t)kr * Wp + cc]);
            fout[(size_t)kr * Wp + cc] = gv;
            dg[i].x += Dv.x * gv.x - Dv.y * gv.y;
            dg[i].y += Dv.x * gv.y + Dv.y * gv.x;
            dx[i].x += Dv.x * xv.x - Dv.y * xv.y;
            dx[i].y += Dv.x * xv.y + Dv.y * xv.x;
          }
        }
      }
      __syncthreads();
      if (m + 1 < m1) issue_tile(P.Dh + (size_t)(m + 1) * plane, dbuf);
      cp_async_commit();
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    if (m0 < m1) issue_tile(Fi + (size_t)m0 * plane, fbuf[0]);
    cp_async_commit();
    // reduce over the maps: dg -> cb, dx -> S^ - sum Df X^; the owner of an
    // element also accumulates gS^ there
    const int E = T * H;
    float2* xn = fbuf[1];  // [E] complex
    float2* xx = xn + E;   // [E] complex
    auto finish = [&](int e, float2 sdg, float2 sdx, float2* cb_out, float2* a_out) {
      const int kr = e / T, c = e - (e / T) * T;
      float2 cbv = make_float2(0.f, 0.f), av = make_float2(0.f, 0.f);
      if (c0 + c < Wf) {
        const float q = 1.f / (rho + __ldg(&P.Psum[(size_t)kr * Wp + c0 + c]));
        cbv = make_float2(sdg.x * q, sdg.y * q);
        const float2 Sv = __ldg(&Sh[(size_t)kr * Wp + c]);
        av = make_float2(Sv.x - sdx.x, Sv.y - sdx.y);
        float2* gs = gSb + (size_t)kr * Wp + c;
        const float2 o = *gs;
        *gs = make_float2(o.x + cbv.x, o.y + cbv.y);
      }
      *cb_out = cbv;
      *a_out = av;
    };
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int kr = t + i * g;
      if (kr < H) {
        xn[kr * T + cc] = dg[i];
        xx[kr * T + cc] = dx[i];
      }
    }
    if (P.G > 1) {
      cg::cluster_group cluster = cg::this_cluster();
      cluster.sync();
      const int sl = (E + P.G - 1) / P.G;
      const int e0 = rank * sl, e1 = min(E, e0 + sl);
      for (int e = e0 + tid; e < e1; e += NT) {
        float2 s1 = make_float2(0.f, 0.f), s2 = make_float2(0.f, 0.f);
        for (int r = 0; r < P.G; ++r) {
          const float2 v = cluster.map_shared_rank(xn, r)[e];
          const float2 w = cluster.map_shared_rank(xx, r)[e];
          s1.x += v.x;
          s1.y += v.y;
          s2.x += w.x;
          s2.y += w.y;
        }
        finish(e, s1, s2, &s1, &s2);
        xn[e] = s1;
        xx[e] = s2;
      }
      cluster.sync();
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) {
          const int e = kr * T + cc;
          const int owner = e / sl;
          dg[i] = owner == rank ? xn[e] : cluster.map_shared_rank(xn, owner)[e];
          dx[i] = owner == rank ? xx[e] : cluster.map_shared_rank(xx, owner)[e];
        }
      }
      cluster.sync();
    } else {
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) finish(kr * T + cc, dg[i], dx[i], &dg[i], &dx[i]);
      }
      __syncthreads();
    }
    // dg[i] = cb, dx[i] = S^ - sum_j Df_j X^_j for this thread's elements
    if (m0 < m1) issue_tile(P.Dh + (size_t)m0 * plane, dbuf);
    cp_async_commit();
    // pass 2: Q^, the dictionary gradient, inverse column FFT of Q^
    it = 0;
    for (int m = m0; m < m1; ++m, ++it) {
      float2* cur = fbuf[it & 1];
      if (m + 1 < m1) issue_tile(Fi + (size_t)(m + 1) * plane, fbuf[(it + 1) & 1]);
      cp_async_commit();
      cp_async_wait<1>();  // F(m) and D(m)
      __syncthreads();
      const float2* xin = Xb + (size_t)m * plane;
      float2* gd = gDb + (size_t)m * plane;
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) {
          const int sl = slot(kr) * T + cc;
          float2 qv = make_float2(0.f, 0.f);
          if (colok) {
            const float2 Dv = dbuf[sl];
            const float2 gv = cur[sl];
            const float2 cb = dg[i], av = dx[i];
            qv.x = (gv.x - (Dv.x * cb.x + Dv.y * cb.y)) * irho;
            qv.y = (gv.y - (Dv.x * cb.y - Dv.y * cb.x)) * irho;
            const float2 xv = __ldg(&xin[(size_t)kr * Wp + cc]);
            float2* gp = gd + (size_t)kr * Wp + cc;
            const float2 o = *gp;
            *gp = make_float2(o.x + av.x * qv.x + av.y * qv.y - (cb.x * xv.x + cb.y * xv.y),
                              o.y + av.y * qv.x - av.x * qv.y - (cb.y * xv.x - cb.x * xv.y));
          }
          cur[sl] = make_float2(qv.x, -qv.y);  // conj: inverse via forward FFT
        }
      }
      __syncthreads();
      if (m + 1 < m1) issue_tile(P.Dh + (size_t)(m + 1) * plane, dbuf);
      cp_async_commit();
      fft_any<NH, T, RM>(cur + cc, P.ph, P.twH, t, g);
      float2* dst = Fi + (size_t)m * plane + c0;
      if (colok) {
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
          const int kr = t + i * g;
          if (kr < H) {
            const float2 v = cur[slot(kr) * T + cc];
            dst[(size_t)kr * Wp + cc] = make_float2(v.x, -v.y);
          }
        }
      }
      __syncthreads();
    }
    cp_async_commit();
    cp_async_wait<0>();
  } else {
    constexpr bool SDEN = MODE == COL_SOLVE_W;  // accumulate sum |Df|^2 / d_m
    float2* fbuf[2] = {stg, stg + TL};
    float2* dbuf = stg + 2 * TL;
    // tile row kr (4 complex = 32 contiguous bytes): two 16-byte async copies
    auto issue_tile = [&](const float2* base, float2* dst) {
      for (int q = tid; q < 2 * H; q += NT) {
        const int kr = q >> 1, h = q & 1;
        cp_async16(dst + slot(kr) * T + 2 * h, base + (size_t)kr * Wp + c0 + 2 * h);
      }
    };
    const float2* Sh = P.Sh + (size_t)b * H * Wp + c0;
    const float mu = P.mu;
    const bool grd = P.grd != 0;
    const int kc = c0 + cc;
    const bool colok = kc < Wf;
    const float gw_col = grd && colok ? 2.f - 2.f * __ldg(&P.twW[kc]).x : 0.f;
    const float irho = 1.f / rho;
    // 1/d for map m, row kr (d = rho, or mu w_m |G(kr, kc)|^2 + rho)
    auto inv_d = [&](float wg, int kr) -> float {
      if (!grd) return irho;
      return 1.f / (wg * (gw_col + 2.f - 2.f * __ldg(&P.twH[kr]).x) + rho);
    };

    // ---------------------------------------------------------------- pass 1
    // Forward column FFT of the row spectra of Y - U; accumulate
    //   acc = sum_m Df_m (Y-U)^_m / d_m   (and sden = sum_m |Df_m|^2 / d_m for
    // per-map d), so that sum_m Df_m b_m / d_m = S^ sden + rho acc; write the
    // column-transformed (Y - U)^ back in place for pass 2.
    float2 num[EPT];
    float sden[SDEN ? EPT : 1];
#pragma unroll
    for (int i = 0; i < EPT; ++i) num[i] = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < (SDEN ? EPT : 1); ++i) sden[i] = 0.f;
    if (m0 < m1) {
      issue_tile(Fi + (size_t)m0 * H * Wp, fbuf[0]);
      issue_tile(P.Dh + (size_t)m0 * H * Wp, dbuf);
    }
    cp_async_commit();
    int it = 0;
    for (int m = m0; m < m1; ++m, ++it) {
      float2* cur = fbuf[it & 1];
      if (m + 1 < m1) issue_tile(Fi + (size_t)(m + 1) * H * Wp, fbuf[(it + 1) & 1]);
      cp_async_commit();
      cp_async_wait<1>();  // F(m) and D(m)
      __syncthreads();
      fft_any<NH, T, RM>(cur + cc, P.ph, P.twH, t, g);
      const float wg = grd ? mu * P.wgrd[m] : 0.f;
      float2* fout = Fi + (size_t)m * H * Wp + c0;
      if (colok) {
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
          const int kr = t + i * g;
          if (kr < H) {
            const int sl = slot(kr) * T + cc;
            const float2 Dv = dbuf[sl];
            const float2 yu = cur[sl];
            fout[(size_t)kr * Wp + cc] = yu;
            const float id = inv_d(wg, kr);
            num[i].x += (Dv.x * yu.x - Dv.y * yu.y) * id;
            num[i].y += (Dv.x * yu.y + Dv.y * yu.x) * id;
            if constexpr (SDEN) sden[i] += (Dv.x * Dv.x + Dv.y * Dv.y) * id;
          }
        }
      }
      __syncthreads();
      // the dictionary tile of the next map lands during its FFT
      if (m + 1 < m1) issue_tile(P.Dh + (size_t)(m + 1) * H * Wp, dbuf);
      cp_async_commit();
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    // prefetch the first spectrum tile of pass 2 into F0 while [F1][D] hosts
    // the reduction over the maps
    if (m0 < m1) issue_tile(Fi + (size_t)m0 * H * Wp, fbuf[0]);
    cp_async_commit();
    // ------------------------------------------------- reduce over the maps
    // cb = (S^ sden + rho acc) / (1 + sden); pass 2 keeps SC = S^ - cb
    const int E = T * H;
    float2* xn = fbuf[1];                                  // [E] complex
    float* xd = reinterpret_cast<float*>(xn + E);          // [E] real
    // sum_m |Df_m|^2 / d_m at tile element (kr, c): accumulated (per-map d)
    // or, with one d for all maps, Psum / d
    auto denom = [&](int kr, int c, float ds) -> float {
      if constexpr (SDEN) {
        return ds;
      } else {
        const int k = c0 + c;
        if (k >= Wf) return 0.f;
        float id = irho;
        if (grd) {
          const float gwc = 2.f - 2.f * __ldg(&P.twW[k]).x;
          id = 1.f / (mu * P.wgrd[0] * (gwc + 2.f - 2.f * __ldg(&P.twH[kr]).x) + rho);
        }
        return __ldg(&P.Psum[(size_t)kr * Wp + k]) * id;
      }
    };
    auto s_minus_cb = [&](int kr, int c, float2 acc, float ds) -> float2 {
      const int k = c0 + c;
      if (k >= Wf) return make_float2(0.f, 0.f);
      const float2 Sv = __ldg(&Sh[(size_t)kr * Wp + c]);
      const float sd = denom(kr, c, ds);
      // (S^ - rho acc) / (1 + sd): S^ - cb without the cancellation
      const float q = 1.f / (1.f + sd);
      return make_float2((Sv.x - rho * acc.x) * q, (Sv.y - rho * acc.y) * q);
    };
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int kr = t + i * g;
      if (kr < H) {
        xn[kr * T + cc] = num[i];
        if constexpr (SDEN) xd[kr * T + cc] = sden[i];
      }
    }
    if (P.G > 1) {
      cg::cluster_group cluster = cg::this_cluster();
      cluster.sync();
      const int sl = (E + P.G - 1) / P.G;
      const int e0 = rank * sl, e1 = min(E, e0 + sl);
      for (int e = e0 + tid; e < e1; e += NT) {
        float2 ns = make_float2(0.f, 0.f);
        float ds = 0.f;
        for (int r = 0; r < P.G; ++r) {
          const float2 v = cluster.map_shared_rank(xn, r)[e];
          ns.x += v.x;
          ns.y += v.y;
          if constexpr (SDEN) ds += cluster.map_shared_rank(xd, r)[e];
        }
        xn[e] = s_minus_cb(e / T, e % T, ns, ds);
      }
      cluster.sync();
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) {
          const int e = kr * T + cc;
          const int owner = e / sl;
          num[i] = owner == rank ? xn[e] : cluster.map_shared_rank(xn, owner)[e];
        }
      }
      cluster.sync();
    } else {
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) num[i] = s_minus_cb(kr, cc, num[i], SDEN ? sden[SDEN ? i : 0] : 0.f);
      }
      __syncthreads();
    }
    // num[i] now holds SC = S^ - cb for this thread's elements
    if (m0 < m1) issue_tile(P.Dh + (size_t)m0 * H * Wp, dbuf);
    cp_async_commit();
    // ---------------------------------------------------------------- pass 2
    // x = (conj(Df) SC + rho (Y - U)^) / d (kept in P.Xtr by COL_SOLVE_X),
    // inverse column FFT
    float2* xtr = MODE == COL_SOLVE_X ? P.Xtr + (size_t)b * M * H * Wp + c0 : nullptr;
    it = 0;
    for (int m = m0; m < m1; ++m, ++it) {
      float2* cur = fbuf[it & 1];
      if (m + 1 < m1) issue_tile(Fi + (size_t)(m + 1) * H * Wp, fbuf[(it + 1) & 1]);
      cp_async_commit();
      cp_async_wait<1>();  // F(m) and D(m)
      __syncthreads();
      const float wg = grd ? mu * P.wgrd[m] : 0.f;
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int kr = t + i * g;
        if (kr < H) {
          const int sl = slot(kr) * T + cc;
          float2 xo = make_float2(0.f, 0.f);
          if (colok) {
            const float2 Dv = dbuf[sl];
            const float2 yu = cur[sl];
            const float2 sc = num[i];
            const float id = inv_d(wg, kr);
            xo.x = (Dv.x * sc.x + Dv.y * sc.y + rho * yu.x) * id;
            xo.y = (Dv.x * sc.y - Dv.y * sc.x + rho * yu.y) * id;
            if constexpr (MODE == COL_SOLVE_X) xtr[(size_t)m * H * Wp + (size_t)kr * Wp + cc] = xo;
          }
          cur[sl] = make_float2(xo.x, -xo.y);  // conj: inverse via forward FFT
        }
      }
      __syncthreads();
      // the dictionary tile of the next map lands during this inverse FFT
      if (m + 1 < m1) issue_tile(P.Dh + (size_t)(m + 1) * H * Wp, dbuf);
      cp_async_commit();
      fft_any<NH, T, RM>(cur + cc, P.ph, P.twH, t, g);
      float2* dst = Fi + (size_t)m * H * Wp + c0;
      if (colok) {
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
          const int kr = t + i * g;
          if (kr < H) {
            const float2 v = cur[slot(kr) * T + cc];
            dst[(size_t)kr * Wp + cc] = make_float2(v.x, -v.y);
          }
        }
      }
      __syncthreads();
    }
    cp_async_commit();
    cp_async_wait<0>();
  }
}
