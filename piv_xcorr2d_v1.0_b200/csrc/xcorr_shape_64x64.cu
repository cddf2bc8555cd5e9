// Fused correlation kernel, 64x64 windows (4 windows and 128 threads per CTA).
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<64, 64, 4, 128>(const XcorrArgs &, bool, int, cudaStream_t);
}
