// row_inst.cu -- the mixed-precision row kernels for one row length M.
//
// The build compiles this file once per row length (PFC_ROW_M = 8 ... 2048) so that the
// FP64 row kernels of the different lengths compile in parallel; step_mixed.cu
// dispatches to launch_mrow_M<M>.
#include "mrow_kernel.cuh"

#ifndef PFC_ROW_M
#error "row_inst.cu is compiled with -DPFC_ROW_M=<row length>"
#endif

namespace pfc {
template cudaError_t launch_mrow_M<PFC_ROW_M>(int, const RunDesc *, int, int, const TwiddleSet &, cudaStream_t);
}  // namespace pfc
