// Tensor-core correlation kernel, 32 x 32 windows (both precisions).
#include "xcorr_tc.cuh"

namespace piv {
template cudaError_t launch_tc_shape<32, 3>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_tc_shape<32, 1>(const XcorrArgs &, bool, int, cudaStream_t);
}  // namespace piv
