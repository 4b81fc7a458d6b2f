// Internal structures shared by the solver kernels and the host driver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sporco_b200.h"
#include "sc_fft.cuh"

// Elements one thread holds during an FFT pass (see sc_fft.cuh).
#define SC_MAXE 16
// Threads per CTA of the row-pass kernels.
#define SC_ROW_THREADS 256
// Image columns (spectrum columns) per column-pass CTA.
#define SC_COL_TILE 4
// Largest column-pass CTA (SC_COL_TILE transforms of length <= 2048).
#define SC_COL_MAX_THREADS 512
// Row pass: radix-16 plans (16 elements per thread, 3 passes) for rows of
// 1024 and 2048, radix-8 plans for the other compile-time lengths.
__host__ __device__ constexpr int row_radix(int W) { return W == 1024 || W == 2048 ? 16 : 8; }
// Resident row-pass CTAs per SM the kernel is compiled for (register cap).
__host__ __device__ constexpr int row_min_blocks(int W) { return row_radix(W) == 16 ? 2 : 3; }
// Column pass: radix-16 plans (16 elements per thread) for long columns,
// radix-8 plans (8 per thread, twice the threads) for short ones.
__host__ __device__ constexpr int col_radix(int H) { return H >= 512 ? 16 : 8; }
// Largest transform length this build supports along a row or a column.
#define SC_MAX_N 4096

// Per-image ADMM scalar state, kept on the device for the whole solve.
struct ImgState {
  double rho;      // rho used by the next iteration
  double rho_prev; // rho of the last iteration (its Y: shrinkage of V at lambda / rho_prev)
  double rsf;    // scale factor chosen by the last adaptive-rho step (1: none)
  double uscale; // the next row pass reads U scaled by this (1 / rsf)
  double r, s;   // last residuals (normalised unless StdResiduals)
  double epri, edua;
  double nX, nY, nU;
  int k;         // iterations completed (over all solves of a warm-started state)
  int done;      // 1: converged, iteration cap reached, or failed
  int status;    // sc_status of this image
  int k0;        // k at the start of the current solve call (its cap counts from here)
};

// Scalar options the finalize kernel needs.
struct FinParams {
  int max_iter;
  int auto_rho, period, auto_scaling, std_residuals;
  double rho_scaling, rsdl_ratio, abs_tol, rel_tol;
  double nelem;          // coefficients per image (M H W)
  const double* xi;      // (B,) residual ratio target per image
  double* itstat;        // (B, max_iter, SC_ITSTAT_FIELDS) or NULL
  int* ndone;            // images finished
};

// Geometry of one batch of equal-sized images.
struct Geom {
  int B;       // images
  int M;       // coefficient maps per image
  int H, W;
  int Wf;      // W/2 + 1 spectrum columns
  int Wp;      // spectrum row pitch (elements)
};

struct RowParams {
  Geom g;
  FftPlan pw;
  const float2* twW;
  int gsz;                 // threads per transform
  int nblk;                // CTAs per image (grid.x)
  float2* F;               // (B, M, H, Wp) spectra
  float* Y;                // (B, M, H, W)
  float* U;                // (B, M, H, W): U, or V = Y + U for ROW_ITER
  int vstate;              // ROW_FIXUP: P.U holds V (1) or U (0)
  float* Yo;               // ROW_ITER writes Y here (== Y unless a trace is kept)
  // epilogue
  const float* lam;        // (B,)
  int l1_kind;
  float l1_scalar;
  const float* l1w;
  const int32_t* mask;     // (B, H, W) or NULL
  int nonneg;              // NonNegCoef: Y >= 0
  int bnd_r, bnd_c;        // NoBndryCross: rows >= bnd_r and columns >= bnd_c
                           // of every map are zero (H, W: none)
  float relax;
  float invN;              // 1 / (H W)
  int delta;               // ROW_ITER*: F holds the column pass's correction only,
                           // X = (Y - U) + IFFTrow(F) / (H W) (ColParams::delta)
  double* partials;        // (B, nblk, 5)
  ImgState* st;            // (B,)
  // setup / tool modes
  const float* src;        // real rows (B, M, H, W) for ROW_FWD_REAL
  const float* D;          // (M, Kr, Kc) for ROW_FWD_DICT
  int Kr, Kc;
  float* dst;              // real rows out for ROW_INV_REAL
  // adjoint (ROW_ADJ)
  float* gV;               // (B, M, H, W) gradient w.r.t. V of the step, in place
  const float* Ymask;      // (B, M, H, W) Y the step produced (nonzero: shrinkage active),
                           // or with vmask its V (active: the shrinkage of V is nonzero)
  int vmask;
  float* Vo;               // ROW_ITER: V written here (NULL: in place, into U)
  int first;               // 1: gV holds dLoss/dY of the last iterate, no Q yet
};

struct ColParams {
  Geom g;
  FftPlan ph;
  const float2* twH;
  const float2* twW;
  int gsz;                 // threads per transform (column)
  int G;                   // CTAs (cluster ranks) sharing one column tile
  int Hs;                  // shared-memory column stride (elements)
  int tile0;               // column tile of blockIdx.y = 0 (a launch over part of the tiles)
  float2* F;               // (B, M, H, Wp)
  const float2* Dh;        // (M, H, Wp)
  const float2* Sh;        // (B, H, Wp)
  int grd;
  int delta;               // the plain convolution solves (COL_SOLVE_C8 / C16) write
                           // only sum_t conj(E_m(t)) sc(r + t) / rho, not H P_m plus it
  float mu;
  const float* wgrd;       // (M,)
  const float* Psum;       // (H, Wp) sum_m |Df_m|^2 (solve with one d for all maps)
  const float4* E;         // (M, Kr, Wp) row spectra e of the filter rows (COL_SOLVE_C*),
                           // as (Re e, Im e, Re e + Im e, Im e - Re e)
  int Kr;                  // filter rows
  ImgState* st;
  float2* Xtr;             // COL_SOLVE_X: x^ also written here (B, M, H, Wp)
  // adjoint (COL_ADJ)
  const float2* Xh;        // (B, M, H, Wp) x^ of the step (COL_ADJ_C*: the row spectra of X)
  float2* gDh;             // (B, M, H, Wp) dictionary-gradient spectra, accumulated
  float2* gSh;             // (B, H, Wp) signal-gradient spectra, accumulated
  // convolution-form adjoint
  float2* SCtr;            // (B, H, Wp) IFFTcol(S^ - cb) / rho of the step (written by
                           // COL_SOLVE_C*T, read by COL_ADJ_C*)
  float2* gE;              // (B, M, Kr, Wp) dictionary gradient as filter-row spectra
};

enum RowMode {
  ROW_ITER = 0, ROW_FWD_REAL = 1, ROW_FWD_DICT = 2, ROW_INV_REAL = 3, ROW_FIXUP = 4,
  ROW_FWD_YU = 5, // row spectra of Y - U (start from given iterates)
  ROW_ADJ = 6,    // adjoint step: Q = row IFFT, gV update, row FFT of relax * gV
  ROW_ITER_YU = 7 // ROW_ITER with Y and U stored separately (warm starts, the
                  // adjoint's recomputation, which keeps Y of every step)
};
// COL_SOLVE: all maps share d (cbpdn, or cbpdngrd with one GradWeight), so
// sum_m |Df_m|^2 / d comes from the precomputed Psum; COL_SOLVE_W: per-map
// d_m = mu w_m |G|^2 + rho, the sum is accumulated over the maps.
// COL_SOLVE_P: the solve with d = rho for every map and frequency (cbpdn,
// cbpdnmsk), without the write-back of the column spectra between its two
// passes.  COL_SOLVE_C8 / COL_SOLVE_C16: the same plain solve with the column
// direction done by direct convolution with the filters' Kr <= 8 / 16 rows
// (no per-map column transforms, no dictionary spectra).  COL_SOLVE_X:
// COL_SOLVE that also writes x^ to ColParams::Xtr (the recomputation inside
// the adjoint).  COL_ADJ: adjoint of the plain cbpdn
// solve (one d = rho): column FFT, Q^ = A^{-1} G^, gradient accumulation,
// inverse column FFT.
// COL_SOLVE_C8T / COL_SOLVE_C16T: COL_SOLVE_C8 / C16 that also keep, for the
// adjoint, the column pass's output (the row spectra of X) in ColParams::Xtr
// and the tile's IFFTcol(S^ - cb) / rho in ColParams::SCtr.  COL_ADJ_C8 /
// COL_ADJ_C16: the adjoint of the plain solve in the same convolution form
// (the dictionary gradient accumulated as correlations over the Kr filter
// rows, ColParams::gE).
enum ColMode {
  COL_SOLVE = 0, COL_FWD = 1, COL_INV = 2, COL_SOLVE_W = 3, COL_ADJ = 4, COL_SOLVE_X = 5,
  COL_SOLVE_P = 6, COL_SOLVE_C8 = 7, COL_SOLVE_C16 = 8, COL_SOLVE_G16 = 9,
  COL_SOLVE_C8T = 10, COL_SOLVE_C16T = 11, COL_ADJ_C8 = 12, COL_ADJ_C16 = 13
};
// Filter rows (taps) of the convolution column solves.
__host__ __device__ constexpr int col_taps(int mode) {
  return (mode == COL_SOLVE_C8 || mode == COL_SOLVE_C8T || mode == COL_ADJ_C8) ? 8
         : (mode == COL_SOLVE_C16 || mode == COL_SOLVE_G16 || mode == COL_SOLVE_C16T ||
            mode == COL_ADJ_C16)
             ? 16
             : 0;
}
// The convolution-form adjoint.
__host__ __device__ constexpr bool col_adj_conv(int mode) {
  return mode == COL_ADJ_C8 || mode == COL_ADJ_C16;
}
// Modes that launch as a cluster over the maps of one column tile.
__host__ __device__ constexpr bool col_clustered(int mode) {
  return mode == COL_SOLVE || mode == COL_SOLVE_W || mode == COL_SOLVE_X || mode == COL_ADJ ||
         mode == COL_SOLVE_P || col_taps(mode) > 0;
}

__host__ __device__ inline size_t sc_align16(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared memory of one row-pass slot (one row pair in flight); zlen is the
// (padded) number of shared-memory slots of one row transform.  The
// iteration mode stages the next pair's two spectrum rows and the pair's Y
// and U rows: [z: zlen complex][F: 2Wp complex][Y: 2W][U: 2W]; the adjoint
// step stages gV and the shrinkage mask source in the Y and U places, the
// rho fix-up the pair's U rows and spectrum rows.
__host__ __device__ inline size_t row_slot_bytes(int mode, int zlen, int W, int Wp) {
  size_t z = sc_align16((size_t)zlen * 8);
  if (mode != ROW_ITER && mode != ROW_ITER_YU && mode != ROW_ADJ && mode != ROW_FIXUP) return z;
  // staged spectrum rows, then one staged real row pair (V for ROW_ITER, the
  // state for ROW_FIXUP) or two (Y and U, gV and the mask source)
  const int nreal = mode == ROW_ITER || mode == ROW_FIXUP ? 1 : 2;
  return z + (size_t)(2 * Wp) * 8 + nreal * sc_align16((size_t)(2 * W) * 4);
}

// Shared memory of one column-pass CTA; hlen is the (padded) number of
// shared-memory slots of one column transform.  A tile is tw (default
// SC_COL_TILE) interleaved columns.  The solve double-buffers the spectrum
// tile and stages the dictionary tile: [F0][F1][D]; the cluster reduction
// reuses [F1][D].  The convolution solves use three tiles and three staged
// filter-row tiles (16 bytes an entry); the convolution adjoint two more tiles (the forward's
// SC trace and row spectra of X) and per-warp partial sums of the
// dictionary gradient for its nt threads (two maps).
__host__ __device__ inline size_t col_smem_bytes(int mode, int hlen, int tw = SC_COL_TILE,
                                                 int nt = SC_COL_MAX_THREADS) {
  const size_t tile = (size_t)tw * hlen * 8;
  return (col_clustered(mode) ? (col_adj_conv(mode) ? 5 : 3) * tile : tile) +
         (size_t)3 * col_taps(mode) * tw * 16 +
         (col_adj_conv(mode) ? (size_t)2 * (nt / 32) * col_taps(mode) * tw * 8 : 0);
}
