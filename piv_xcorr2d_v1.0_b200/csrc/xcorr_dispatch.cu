// xcorr_dispatch.cu -- window shape -> instantiated fused correlation kernel.
// Each shape (WSX, WSY) is compiled in its own translation unit (xcorr_shape_*.cu)
// with B windows per CTA and NT threads per CTA.
#include "piv_common.cuh"

namespace piv {

template <int WSX, int WSY, int B, int NT>
cudaError_t launch_shape(const XcorrArgs &a, bool deformed, int K, cudaStream_t s);

#define PIV_XCORR_SHAPES(X) \
    X(8, 8, 32, 128) \
    X(12, 12, 16, 96) \
    X(16, 16, 16, 128) \
    X(24, 24, 8, 96) \
    X(32, 32, 8, 128) \
    X(48, 48, 4, 96) \
    X(64, 64, 4, 128) \
    X(48, 24, 4, 96) \
    X(24, 48, 4, 96) \
    X(32, 16, 8, 128) \
    X(16, 32, 8, 128) \
    X(64, 32, 4, 128) \
    X(32, 64, 4, 128)

#define PIV_X(WX, WY, B, NT) extern template cudaError_t launch_shape<WX, WY, B, NT>(const XcorrArgs &, bool, int, cudaStream_t);
PIV_XCORR_SHAPES(PIV_X)
#undef PIV_X

bool xcorr_supported(int wsx, int wsy)
{
#define PIV_X(WX, WY, B, NT) \
    if (wsx == WX && wsy == WY) return true;
    PIV_XCORR_SHAPES(PIV_X)
#undef PIV_X
    return false;
}

cudaError_t launch_xcorr(const XcorrArgs &a, bool deformed, cudaStream_t s, const char **why)
{
    if (a.g.Nps > 8) {
        if (why) *why = "Npeak_save > 8 is not built into this engine";
        return cudaErrorInvalidValue;
    }
    const int K = a.g.Nps <= 4 ? 4 : 8;
#define PIV_X(WX, WY, B, NT) \
    if (a.g.ws_x == WX && a.g.ws_y == WY) return launch_shape<WX, WY, B, NT>(a, deformed, K, s);
    PIV_XCORR_SHAPES(PIV_X)
#undef PIV_X
    if (why) *why = "window shape not built into this engine";
    return cudaErrorInvalidValue;
}

}  // namespace piv
