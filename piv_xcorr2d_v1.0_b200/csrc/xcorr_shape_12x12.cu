// Fused correlation kernel, 12x12 windows (16 windows and 96 threads per CTA).
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<12, 12, 16, 96>(const XcorrArgs &, bool, int, cudaStream_t);
}
