// Fused correlation kernel, 16x16 windows (16 windows and 128 threads per CTA).
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<16, 16, 16, 128>(const XcorrArgs &, bool, int, cudaStream_t);
}
