// Fused correlation kernel, 64x32 windows: the (windows per CTA, threads per CTA)
// variants the autotuner chooses from.
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<64, 32, 4, 128>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<64, 32, 2, 64>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<64, 32, 2, 128>(const XcorrArgs &, bool, int, cudaStream_t);
}
