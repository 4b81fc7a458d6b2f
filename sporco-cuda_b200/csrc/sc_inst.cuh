// Helpers of the kernel instantiation units (sc_inst_*.cu): the table of
// one row or column mode over the compile-time lengths.
#pragma once

#include "sc_dispatch.cuh"
#include "sc_kernels.cuh"

template <int MODE>
RowFn row_table(int n) {
#define SC_ROW_CASE(k) case k: return row_kernel<MODE, k>;
  if constexpr (row_specialised(MODE)) {
    switch (n) { SC_SPEC_ROW(SC_ROW_CASE) default: break; }
  }
#undef SC_ROW_CASE
  return row_kernel<MODE, 0>;
}

template <int MODE>
ColFn col_table(int n) {
#define SC_COL_CASE(k) case k: return col_kernel<MODE, k>;
  switch (n) { SC_SPEC_COL(SC_COL_CASE) default: break; }
#undef SC_COL_CASE
  return col_kernel<MODE, 0>;
}

// The same over the compiled lengths below 512 only (radix-8 column plans,
// at most 8 rows per thread), for modes used only there; nullptr otherwise.
#define SC_SPEC_COL_SMALL(X) X(16) X(32) X(64) X(128) X(256) X(48) X(96) X(192) X(384)
template <int MODE>
ColFn col_table_small(int n) {
#define SC_COL_CASE(k) case k: return col_kernel<MODE, k>;
  switch (n) { SC_SPEC_COL_SMALL(SC_COL_CASE) default: break; }
#undef SC_COL_CASE
  return nullptr;
}

// Radix-8 column plans at the compiled lengths 512, 768 and 1024 (whose
// default plans are radix 16): twice the threads per column, half the rows
// per thread; the autotuner chooses between the two.  nullptr otherwise.
#define SC_SPEC_COL_R8(X) X(512) X(768) X(1024)
template <int MODE>
ColFn col_table_r8(int n) {
#define SC_COL_CASE(k) case k: return col_kernel<MODE, k, 8>;
  switch (n) { SC_SPEC_COL_R8(SC_COL_CASE) default: break; }
#undef SC_COL_CASE
  return nullptr;
}

// Two-column tiles at the compiled lengths from 512 (rm 16: the default
// plans; rm 8: the radix-8 plans at 512, 768, 1024).  nullptr otherwise.
#define SC_SPEC_COL_T2(X) X(512) X(768) X(1024) X(1536) X(2048)
template <int MODE>
ColFn col_table_t2(int n, int rm) {
  if (rm == 8) {
#define SC_COL_CASE(k) case k: return col_kernel<MODE, k, 8, 2>;
    switch (n) { SC_SPEC_COL_R8(SC_COL_CASE) default: break; }
#undef SC_COL_CASE
    return nullptr;
  }
#define SC_COL_CASE(k) case k: return col_kernel<MODE, k, 0, 2>;
  switch (n) { SC_SPEC_COL_T2(SC_COL_CASE) default: break; }
#undef SC_COL_CASE
  return nullptr;
}
