// Instantiations of the row pass: the ADMM iteration (state V, or Y and U).
#include "sc_inst.cuh"

RowFn sc_row_fn_iter(int mode, int n) {
  switch (mode) {
    case ROW_ITER: return row_table<ROW_ITER>(n);
    case ROW_ITER_YU: return row_table<ROW_ITER_YU>(n);
    default: return nullptr;
  }
}
