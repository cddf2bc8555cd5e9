// Tensor-core correlation kernel, 16 x 16 windows (split and single products, BF16 and FP16 operands).
#include "xcorr_tc.cuh"

namespace piv {
template cudaError_t launch_tc_shape<16, 3, false>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
template cudaError_t launch_tc_shape<16, 3, true>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
template cudaError_t launch_tc_shape<16, 1, false>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
template cudaError_t launch_tc_shape<16, 1, true>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
}  // namespace piv
