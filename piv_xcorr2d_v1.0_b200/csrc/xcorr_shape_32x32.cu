// Fused correlation kernel, 32x32 windows (8 windows and 128 threads per CTA).
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<32, 32, 8, 128>(const XcorrArgs &, bool, int, cudaStream_t);
}
