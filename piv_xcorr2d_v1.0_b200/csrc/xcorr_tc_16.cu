// Tensor-core correlation kernel, 16 x 16 windows (both precisions).
#include "xcorr_tc.cuh"

namespace piv {
template cudaError_t launch_tc_shape<16, 3>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_tc_shape<16, 1>(const XcorrArgs &, bool, int, cudaStream_t);
}  // namespace piv
