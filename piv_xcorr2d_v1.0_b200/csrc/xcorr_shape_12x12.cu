// Fused correlation kernel, 12x12 windows: the (windows per CTA, threads per CTA)
// variants the autotuner chooses from, and the batch-launch variants.
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<12, 12, 16, 96>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<12, 12, 8, 96>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<12, 12, 16, 192>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<12, 12, 16, 96>(const XcorrBatch &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<12, 12, 8, 96>(const XcorrBatch &, bool, int, cudaStream_t);
}
