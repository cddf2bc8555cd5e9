// Fused correlation kernel, 48x48 windows: the (windows per CTA, threads per CTA)
// variants the autotuner chooses from, and the batch-launch variants.
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<48, 48, 4, 96>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<48, 48, 2, 96>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<48, 48, 2, 64>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<48, 48, 4, 192>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<48, 48, 4, 96>(const XcorrBatch &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<48, 48, 2, 96>(const XcorrBatch &, bool, int, cudaStream_t);
}
