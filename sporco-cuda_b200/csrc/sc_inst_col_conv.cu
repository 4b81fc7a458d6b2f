// Instantiations of the column pass: the convolution solves.
#include "sc_inst.cuh"

ColFn sc_col_fn_conv(int mode, int n) {
  switch (mode) {
    case COL_SOLVE_C8: return col_table<COL_SOLVE_C8>(n);
    case COL_SOLVE_C16: return col_table<COL_SOLVE_C16>(n);
    case COL_SOLVE_G16: return col_table<COL_SOLVE_G16>(n);
    default: return nullptr;
  }
}

ColFn sc_col_fn_conv_r8(int mode, int n) {
  switch (mode) {
    case COL_SOLVE_C8: return col_table_r8<COL_SOLVE_C8>(n);
    case COL_SOLVE_C16: return col_table_r8<COL_SOLVE_C16>(n);
    case COL_SOLVE_G16: return col_table_r8<COL_SOLVE_G16>(n);
    default: return nullptr;
  }
}
