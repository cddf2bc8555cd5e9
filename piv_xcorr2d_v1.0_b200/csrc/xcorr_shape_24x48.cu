// Fused correlation kernel, 24x48 windows (4 windows and 96 threads per CTA).
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<24, 48, 4, 96>(const XcorrArgs &, bool, int, cudaStream_t);
}
