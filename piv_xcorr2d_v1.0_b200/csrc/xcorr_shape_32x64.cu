// Fused correlation kernel, 32x64 windows (4 windows and 128 threads per CTA).
#include "xcorr_kernel.cuh"

namespace piv {
template cudaError_t launch_shape<32, 64, 4, 128>(const XcorrArgs &, bool, int, cudaStream_t);
}
