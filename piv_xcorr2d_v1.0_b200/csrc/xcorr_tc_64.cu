// Tensor-core correlation kernel, 64 x 64 windows (split and single products, BF16 and FP16 operands).
#include "xcorr_tc.cuh"

namespace piv {
template cudaError_t launch_tc_shape<64, 3, false>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
template cudaError_t launch_tc_shape<64, 3, true>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
template cudaError_t launch_tc_shape<64, 1, false>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
template cudaError_t launch_tc_shape<64, 1, true>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
}  // namespace piv
