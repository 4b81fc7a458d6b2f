// Instantiations of the column pass: the adjoint's solves (transform and
// convolution forms) and the set-up and transform tools.
#include "sc_inst.cuh"

ColFn sc_col_fn_aux(int mode, int n) {
  switch (mode) {
    case COL_SOLVE_X: return col_table<COL_SOLVE_X>(n);
    case COL_ADJ: return col_table<COL_ADJ>(n);
    case COL_FWD: return col_table<COL_FWD>(n);
    case COL_INV: return col_table<COL_INV>(n);
    // the convolution-form adjoint and its forward traces (columns < 512)
    case COL_SOLVE_C8T: return col_table_small<COL_SOLVE_C8T>(n);
    case COL_SOLVE_C16T: return col_table_small<COL_SOLVE_C16T>(n);
    case COL_ADJ_C8: return col_table_small<COL_ADJ_C8>(n);
    case COL_ADJ_C16: return col_table_small<COL_ADJ_C16>(n);
    default: return nullptr;
  }
}
