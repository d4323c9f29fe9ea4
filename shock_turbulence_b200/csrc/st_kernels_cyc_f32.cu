// st_kernels_cyc_f32.cu - FP32-field instantiations of the periodic-line
// operators.
#include "st_linekern.cuh"

namespace st {

int launch_line_cyc_f32(st_ctx *c, OpKind op, const LineArgsF &a) { return launch_line_t<true, float>(c, op, a); }

}  // namespace st
