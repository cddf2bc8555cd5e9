// Fused correlation kernel, 64x32 windows: the (windows per CTA, threads per CTA)
// variants the autotuner chooses from, and the batch-launch variants.
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<64, 32, 4, 128>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<64, 32, 2, 64>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<64, 32, 2, 128>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<64, 32, 4, 128>(const XcorrBatch &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<64, 32, 2, 64>(const XcorrBatch &, bool, int, cudaStream_t);
}
