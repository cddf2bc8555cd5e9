// Fused correlation kernel, 8x8 windows (32 windows and 128 threads per CTA).
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<8, 8, 32, 128>(const XcorrArgs &, bool, int, cudaStream_t);
}
