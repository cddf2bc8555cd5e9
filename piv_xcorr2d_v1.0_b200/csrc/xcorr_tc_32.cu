// Tensor-core correlation kernel, 32 x 32 windows (split and single products, BF16 and FP16 operands).
#include "xcorr_tc.cuh"

namespace piv {
template cudaError_t launch_tc_shape<32, 3, false>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
template cudaError_t launch_tc_shape<32, 3, true>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
template cudaError_t launch_tc_shape<32, 1, false>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
template cudaError_t launch_tc_shape<32, 1, true>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
}  // namespace piv
