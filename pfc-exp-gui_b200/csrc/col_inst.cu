// col_inst.cu -- the column kernels of both fused paths for one row length L.
//
// The build compiles this file once per supported L (PFC_COL_L = 32 ... 2048) and path, so the
// many (tile width, staging, mode) instantiations of each L compile in parallel;
// step_fp32.cu and step_mixed.cu dispatch to launch_col_f32_L<L> / launch_col_mixed_L<L>.
#include "col_kernel.cuh"
#include "mcol_kernel.cuh"

#if !defined(PFC_COL_L) || !defined(PFC_COL_PATH)
#error "col_inst.cu is compiled with -DPFC_COL_L=<row length> -DPFC_COL_PATH=<0: FP32, 1: mixed>"
#endif

// PFC_COL_PATH selects the path: 0 = FP32, 1 = mixed precision (one unit each).
namespace pfc {
#if PFC_COL_PATH == 0
template cudaError_t launch_col_f32_L<PFC_COL_L>(const RunDesc *, int, int, int, int, int, const TwiddleSet &,
                                                 cudaStream_t);
#else
template cudaError_t launch_col_mixed_L<PFC_COL_L>(const RunDesc *, int, int, int, int, int, const TwiddleSet &,
                                                   cudaStream_t);
#endif
}  // namespace pfc
