// Fused correlation kernel, 8x8 windows: the (windows per CTA, threads per CTA)
// variants the autotuner chooses from, and the batch-launch variants.
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<8, 8, 32, 128>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<8, 8, 16, 128>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<8, 8, 32, 256>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<8, 8, 32, 128>(const XcorrBatch &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<8, 8, 16, 128>(const XcorrBatch &, bool, int, cudaStream_t);
}
