// Tensor-core correlation kernel, 64 x 64 windows (both precisions).
#include "xcorr_tc.cuh"

namespace piv {
template cudaError_t launch_tc_shape<64, 3>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_tc_shape<64, 1>(const XcorrArgs &, bool, int, cudaStream_t);
}  // namespace piv
