// Fused correlation kernel, 48x48 windows (4 windows and 96 threads per CTA).
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<48, 48, 4, 96>(const XcorrArgs &, bool, int, cudaStream_t);
}
