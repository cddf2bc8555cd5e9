// Fused correlation kernel, 32x32 windows: the (windows per CTA, threads per CTA)
// variants the autotuner chooses from, and the batch-launch variants.
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<32, 32, 8, 128>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<32, 32, 4, 128>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<32, 32, 2, 64>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<32, 32, 8, 256>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<32, 32, 4, 64>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape_block<32, 32, 128>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<32, 32, 4, 128>(const XcorrBatch &, bool, int, cudaStream_t);
template cudaError_t launch_shape_batch<32, 32, 8, 128>(const XcorrBatch &, bool, int, cudaStream_t);
}
