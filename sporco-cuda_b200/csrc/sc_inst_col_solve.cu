// Instantiations of the column pass: the transform solves.
#include "sc_inst.cuh"

ColFn sc_col_fn_solve(int mode, int n) {
  switch (mode) {
    case COL_SOLVE_P: return col_table<COL_SOLVE_P>(n);
    case COL_SOLVE: return col_table<COL_SOLVE>(n);
    case COL_SOLVE_W: return col_table<COL_SOLVE_W>(n);
    default: return nullptr;
  }
}

ColFn sc_col_fn_solve_r8(int mode, int n) {
  switch (mode) {
    case COL_SOLVE_P: return col_table_r8<COL_SOLVE_P>(n);
    case COL_SOLVE: return col_table_r8<COL_SOLVE>(n);
    case COL_SOLVE_W: return col_table_r8<COL_SOLVE_W>(n);
    default: return nullptr;
  }
}
