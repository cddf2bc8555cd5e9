// Fused correlation kernel, 32x32 windows: the (windows per CTA, threads per CTA)
// variants the autotuner chooses from.
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<32, 32, 8, 128>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<32, 32, 4, 128>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<32, 32, 2, 64>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<32, 32, 8, 256>(const XcorrArgs &, bool, int, cudaStream_t);
template cudaError_t launch_shape<32, 32, 4, 64>(const XcorrArgs &, bool, int, cudaStream_t);
}
