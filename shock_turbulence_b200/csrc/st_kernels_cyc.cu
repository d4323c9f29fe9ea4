// st_kernels_cyc.cu - periodic-line instantiations of the line operators
// (src/derivCDopt6_periodic.f, src/filters_periodic.f).
#include "st_linekern.cuh"

namespace st {

int launch_line_cyc(st_ctx *c, OpKind op, const LineArgs &a) { return launch_line_t<true, double>(c, op, a); }

}  // namespace st
