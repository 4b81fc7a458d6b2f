// Instantiations of the column pass: the convolution solves with tiles of
// two columns (lengths from 512).
#include "sc_inst.cuh"

ColFn sc_col_fn_conv_t2(int mode, int n, int rm) {
  switch (mode) {
    case COL_SOLVE_C8: return col_table_t2<COL_SOLVE_C8>(n, rm);
    case COL_SOLVE_C16: return col_table_t2<COL_SOLVE_C16>(n, rm);
    case COL_SOLVE_G16: return col_table_t2<COL_SOLVE_G16>(n, rm);
    default: return nullptr;
  }
}
