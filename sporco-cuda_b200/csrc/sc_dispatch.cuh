// Kernel function tables of the row and column passes.
//
// row_kernel<MODE, N> and col_kernel<MODE, N> are instantiated for every
// mode and every transform length with a compile-time FFT plan (N) plus the
// runtime-plan fallback (N = 0).  The instantiations live in several
// translation units (sc_inst_*.cu, one group of modes each) so that they
// compile in parallel; the driver (sc_solver.cu) obtains the kernel it
// launches from these getters.  Each getter returns the instantiation for
// the length n when it has one, the runtime-plan instantiation otherwise
// (or always, for n <= 0).
#pragma once

#include "sc_internal.cuh"

typedef void (*RowFn)(RowParams);
typedef void (*ColFn)(ColParams);

// Transform lengths with compile-time FFT plans (all benchmark sizes).
#define SC_SPEC_ROW(X) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) \
  X(48) X(96) X(192) X(384) X(768) X(1536)
#define SC_SPEC_COL(X) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) \
  X(48) X(96) X(192) X(384) X(768) X(1536)

// Row modes with compile-time FFT plans: the iteration, the rho fix-up, the
// adjoint step, the 2-D FFT tools and the row spectra of Y - U from given
// iterates (the adjoint's restart from a checkpoint must transform exactly
// as the iteration does, so that its recomputation reproduces the forward
// iterates bit for bit); the dictionary set-up uses the runtime plan.
__host__ __device__ constexpr bool row_specialised(int mode) {
  return mode == ROW_ITER || mode == ROW_ITER_YU || mode == ROW_FIXUP || mode == ROW_FWD_REAL ||
         mode == ROW_INV_REAL || mode == ROW_ADJ || mode == ROW_FWD_YU;
}

// sc_inst_row_iter.cu: ROW_ITER, ROW_ITER_YU
RowFn sc_row_fn_iter(int mode, int n);
// sc_inst_row_aux.cu: ROW_FIXUP, ROW_ADJ, ROW_FWD_REAL, ROW_INV_REAL,
// ROW_FWD_DICT, ROW_FWD_YU
RowFn sc_row_fn_aux(int mode, int n);
// sc_inst_col_conv.cu: COL_SOLVE_C8, COL_SOLVE_C16, COL_SOLVE_G16
ColFn sc_col_fn_conv(int mode, int n);
// sc_inst_col_solve.cu: COL_SOLVE_P, COL_SOLVE, COL_SOLVE_W
ColFn sc_col_fn_solve(int mode, int n);
// sc_inst_col_aux.cu: COL_SOLVE_X, COL_ADJ, COL_FWD, COL_INV, and, for
// compiled lengths below 512 only, COL_SOLVE_C8T, COL_SOLVE_C16T, COL_ADJ_C8,
// COL_ADJ_C16
ColFn sc_col_fn_aux(int mode, int n);

// Radix-8 column plans at lengths 512, 768, 1024 (nullptr elsewhere):
// sc_inst_col_conv.cu (C8, C16, G16), sc_inst_col_solve.cu (P, SOLVE,
// SOLVE_W).
ColFn sc_col_fn_conv_r8(int mode, int n);
ColFn sc_col_fn_solve_r8(int mode, int n);
// Two-column tiles of the convolution solves (C8, C16, G16) at the compiled
// lengths from 512, with the default radix (rm 16) or the radix-8 plan (rm 8,
// lengths 512, 768, 1024): sc_inst_col_conv_t2.cu; nullptr elsewhere.
ColFn sc_col_fn_conv_t2(int mode, int n, int rm);
__host__ __device__ constexpr bool col_has_t2(int mode) {
  return mode == COL_SOLVE_C8 || mode == COL_SOLVE_C16 || mode == COL_SOLVE_G16;
}
// The column-pass modes with a radix-8 alternative.
__host__ __device__ constexpr bool col_has_r8(int mode) {
  return mode == COL_SOLVE_C8 || mode == COL_SOLVE_C16 || mode == COL_SOLVE_G16 ||
         mode == COL_SOLVE_P || mode == COL_SOLVE || mode == COL_SOLVE_W;
}
__host__ __device__ constexpr bool col_len_r8(int n) { return n == 512 || n == 768 || n == 1024; }

// The table entry of MODE for length n.
template <int MODE>
inline RowFn row_fn(int n) {
  if constexpr (MODE == ROW_ITER || MODE == ROW_ITER_YU) return sc_row_fn_iter(MODE, n);
  else return sc_row_fn_aux(MODE, n);
}
template <int MODE>
inline ColFn col_fn(int n) {
  if constexpr (MODE == COL_SOLVE_C8 || MODE == COL_SOLVE_C16 || MODE == COL_SOLVE_G16)
    return sc_col_fn_conv(MODE, n);
  else if constexpr (MODE == COL_SOLVE_P || MODE == COL_SOLVE || MODE == COL_SOLVE_W)
    return sc_col_fn_solve(MODE, n);
  else
    return sc_col_fn_aux(MODE, n);
}

// MODE at length n with column radix rm and tiles of tw columns (nullptr
// when that variant is not compiled).
template <int MODE>
inline ColFn col_fn_variant(int n, int rm, int tw);
// The radix-8 alternative of MODE at length n (nullptr when there is none).
template <int MODE>
inline ColFn col_fn_r8(int n) {
  if constexpr (MODE == COL_SOLVE_C8 || MODE == COL_SOLVE_C16 || MODE == COL_SOLVE_G16)
    return sc_col_fn_conv_r8(MODE, n);
  else if constexpr (MODE == COL_SOLVE_P || MODE == COL_SOLVE || MODE == COL_SOLVE_W)
    return sc_col_fn_solve_r8(MODE, n);
  else
    return nullptr;
}

template <int MODE>
inline ColFn col_fn_variant(int n, int rm, int tw) {
  if (tw == SC_COL_TILE) return rm == col_radix(n) ? col_fn<MODE>(n) : col_fn_r8<MODE>(n);
  if constexpr (col_has_t2(MODE)) {
    if (tw == 2) return sc_col_fn_conv_t2(MODE, n, rm);
  }
  return nullptr;
}
