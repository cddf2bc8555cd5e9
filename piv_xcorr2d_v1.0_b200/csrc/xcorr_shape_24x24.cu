// Fused correlation kernel, 24x24 windows: the (windows per CTA, threads per CTA)
// variants the autotuner chooses from, and the batch-launch variants.
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<24, 24, 8, 96>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<24, 24, 4, 96>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<24, 24, 8, 192>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<24, 24, 2, 64>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<24, 24, 8, 96>(const XcorrBatch &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<24, 24, 4, 96>(const XcorrBatch &, bool, int, cudaStream_t);
}
