// Fused correlation kernel, 24x24 windows (8 windows and 96 threads per CTA).
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<24, 24, 8, 96>(const XcorrArgs &, bool, int, cudaStream_t);
}
