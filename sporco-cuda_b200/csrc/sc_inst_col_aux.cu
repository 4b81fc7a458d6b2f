// Instantiations of the column pass: the adjoint's solves and the set-up
// and transform tools.
#include "sc_inst.cuh"

ColFn sc_col_fn_aux(int mode, int n) {
  switch (mode) {
    case COL_SOLVE_X: return col_table<COL_SOLVE_X>(n);
    case COL_ADJ: return col_table<COL_ADJ>(n);
    case COL_FWD: return col_table<COL_FWD>(n);
    case COL_INV: return col_table<COL_INV>(n);
    default: return nullptr;
  }
}
