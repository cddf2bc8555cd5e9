// Tensor-core correlation kernel for the non-square windows 48x24 and 24x48 (split and single
// products, BF16 and FP16 operands).
#include "xcorr_tc_rect.cuh"

namespace piv {
template cudaError_t launch_tc_rect_shape<48, 24, 3, false>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_tc_rect_shape<48, 24, 1, false>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_tc_rect_shape<48, 24, 3, true>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_tc_rect_shape<48, 24, 1, true>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_tc_rect_shape<24, 48, 3, false>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_tc_rect_shape<24, 48, 1, false>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_tc_rect_shape<24, 48, 3, true>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_tc_rect_shape<24, 48, 1, true>(const XcorrArgs &, bool, int, cudaStream_t);
}  // namespace piv
