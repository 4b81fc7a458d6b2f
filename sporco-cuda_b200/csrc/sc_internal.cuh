// Internal structures shared by the solver kernels and the host driver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sc_fft.cuh"

// Elements one thread holds during an FFT pass (see sc_fft.cuh).
#define SC_MAXE 16
// Threads per CTA of the row-pass kernels.
#define SC_ROW_THREADS 256
// Image columns (spectrum columns) per column-pass CTA.
#define SC_COL_TILE 4
// Largest column-pass CTA (SC_COL_TILE transforms of length <= 2048).
#define SC_COL_MAX_THREADS 1024
// Largest transform length this build supports along a row or a column.
#define SC_MAX_N 4096

// Per-image ADMM scalar state, kept on the device for the whole solve.
struct ImgState {
  double rho;    // rho used by the next iteration
  double rsf;    // scale factor chosen by the last adaptive-rho step (1: none)
  double uscale; // the next row pass reads U scaled by this (1 / rsf)
  double r, s;   // last residuals (normalised unless StdResiduals)
  double epri, edua;
  double nX, nY, nU;
  int k;         // iterations completed
  int done;      // 1: converged, iteration cap reached, or failed
  int status;    // sc_status of this image
  int pad;
};

// Scalar options the finalize kernel needs.
struct FinParams {
  int max_iter;
  int auto_rho, period, auto_scaling, std_residuals;
  double rho_scaling, rsdl_ratio, abs_tol, rel_tol;
  double nelem;          // coefficients per image (M H W)
  const double* xi;      // (B,) residual ratio target per image
  double* itstat;        // (B, max_iter, 5) or NULL
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
  float* U;                // (B, M, H, W)
  // epilogue
  const float* lam;        // (B,)
  int l1_kind;
  float l1_scalar;
  const float* l1w;
  const int32_t* mask;     // (B, H, W) or NULL
  float relax;
  float invN;              // 1 / (H W)
  double* partials;        // (B, nblk, 5)
  ImgState* st;            // (B,)
  // setup / tool modes
  const float* src;        // real rows (B, M, H, W) for ROW_FWD_REAL
  const float* D;          // (M, Kr, Kc) for ROW_FWD_DICT
  int Kr, Kc;
  float* dst;              // real rows out for ROW_INV_REAL
};

struct ColParams {
  Geom g;
  FftPlan ph;
  const float2* twH;
  const float2* twW;
  int gsz;                 // threads per transform (column)
  int G;                   // CTAs (cluster ranks) sharing one column tile
  int Hs;                  // shared-memory column stride (elements)
  float2* F;               // (B, M, H, Wp)
  const float2* Dh;        // (M, H, Wp)
  const float2* Sh;        // (B, H, Wp)
  int grd;
  float mu;
  const float* wgrd;       // (M,)
  ImgState* st;
};

enum RowMode { ROW_ITER = 0, ROW_FWD_REAL = 1, ROW_FWD_DICT = 2, ROW_INV_REAL = 3, ROW_FIXUP = 4 };
enum ColMode { COL_SOLVE = 0, COL_FWD = 1, COL_INV = 2 };

__host__ __device__ inline size_t sc_align16(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared memory of one row-pass slot (one row pair in flight).  The
// iteration mode double-buffers the pair's two spectrum rows and stages the
// pair's Y and U rows: [z: W complex][F: 2 x 2Wp complex][Y: 2W][U: 2W].
__host__ __device__ inline size_t row_slot_bytes(int mode, int W, int Wp) {
  size_t z = sc_align16((size_t)W * 8);
  if (mode != ROW_ITER) return z;
  return z + 2 * (size_t)(2 * Wp) * 8 + 2 * sc_align16((size_t)(2 * W) * 4);
}

// Shared memory of one column-pass CTA: the solve double-buffers the tile
// (SC_COL_TILE interleaved columns of H complex) and accumulates
// sum_m Df b / d (complex) and sum_m |Df|^2 / d (real) per tile element.
__host__ __device__ inline size_t col_smem_bytes(int mode, int H) {
  const size_t tile = (size_t)SC_COL_TILE * H * 8;
  if (mode != COL_SOLVE) return tile;
  return 2 * tile + (size_t)SC_COL_TILE * H * 12;
}
