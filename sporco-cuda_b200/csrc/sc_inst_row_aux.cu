// Instantiations of the row pass: rho fix-up, adjoint step, set-up and
// transform tools.
#include "sc_inst.cuh"

RowFn sc_row_fn_aux(int mode, int n) {
  switch (mode) {
    case ROW_FIXUP: return row_table<ROW_FIXUP>(n);
    case ROW_ADJ: return row_table<ROW_ADJ>(n);
    case ROW_FWD_REAL: return row_table<ROW_FWD_REAL>(n);
    case ROW_INV_REAL: return row_table<ROW_INV_REAL>(n);
    case ROW_FWD_DICT: return row_table<ROW_FWD_DICT>(n);
    case ROW_FWD_YU: return row_table<ROW_FWD_YU>(n);
    default: return nullptr;
  }
}
