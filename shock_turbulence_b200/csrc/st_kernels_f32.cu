// st_kernels_f32.cu - FP32-field instantiations of the bounded-line
// operators (the FP32 mode stores derivative inputs and outputs in float;
// the stencils and solves run in double).
#include "st_linekern.cuh"

namespace st {

int launch_line_f32(st_ctx *c, OpKind op, const LineArgsF &a) { return launch_line_t<false, float>(c, op, a); }
int launch_pair_f32(st_ctx *c, const D1PairT<float> &g, double bytes) { return launch_pair_t<float>(c, g, bytes); }

}  // namespace st
