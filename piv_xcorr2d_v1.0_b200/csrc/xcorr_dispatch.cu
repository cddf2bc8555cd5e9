// xcorr_dispatch.cu -- window shape and variant -> instantiated fused correlation kernel.
// Every shape (WSX, WSY) is compiled in its own translation unit (xcorr_shape_*.cu) in
// several variants (B windows per CTA, NT threads per CTA); the first listed variant of a
// shape is its default, the engine's autotuner may pick another one per grid.
#include <cstring>
#include <type_traits>

#include "piv_common.cuh"

namespace piv {

template <int WSX, int WSY, int B, int NT>
cudaError_t launch_shape(const XcorrArgs &a, bool deformed, int K, cudaStream_t s);

#define PIV_XCORR_VARIANTS(X) \
    X(8, 8, 32, 128) \
    X(8, 8, 16, 128) \
    X(8, 8, 32, 256) \
    X(12, 12, 16, 96) \
    X(12, 12, 8, 96) \
    X(12, 12, 16, 192) \
    X(16, 16, 16, 128) \
    X(16, 16, 8, 128) \
    X(16, 16, 16, 256) \
    X(16, 16, 4, 64) \
    X(24, 24, 8, 96) \
    X(24, 24, 4, 96) \
    X(24, 24, 8, 192) \
    X(24, 24, 2, 64) \
    X(32, 32, 8, 128) \
    X(32, 32, 4, 128) \
    X(32, 32, 2, 64) \
    X(32, 32, 8, 256) \
    X(32, 32, 4, 64) \
    X(48, 48, 4, 96) \
    X(48, 48, 2, 96) \
    X(48, 48, 2, 64) \
    X(48, 48, 4, 192) \
    X(64, 64, 2, 128) \
    X(64, 64, 4, 128) \
    X(64, 64, 2, 64) \
    X(64, 64, 4, 256) \
    X(48, 24, 4, 96) \
    X(48, 24, 2, 64) \
    X(48, 24, 2, 96) \
    X(48, 24, 8, 192) \
    X(24, 48, 4, 96) \
    X(24, 48, 2, 64) \
    X(24, 48, 4, 64) \
    X(24, 48, 8, 96) \
    X(32, 16, 8, 128) \
    X(32, 16, 4, 64) \
    X(32, 16, 8, 256) \
    X(16, 32, 8, 128) \
    X(16, 32, 4, 64) \
    X(16, 32, 8, 256) \
    X(64, 32, 4, 128) \
    X(64, 32, 2, 64) \
    X(64, 32, 2, 128) \
    X(32, 64, 4, 128) \
    X(32, 64, 2, 64) \
    X(32, 64, 2, 128)

#define PIV_X(WX, WY, B, NT) extern template cudaError_t launch_shape<WX, WY, B, NT>(const XcorrArgs &, bool, int, cudaStream_t);
PIV_XCORR_VARIANTS(PIV_X)
#undef PIV_X
// the 2x2-block form (four windows of two window rows per CTA), listed after the shape's
// row-major variants
template <int WSX, int WSY, int NT>
cudaError_t launch_shape_block(const XcorrArgs &a, bool deformed, int K, cudaStream_t s);
extern template cudaError_t launch_shape_block<32, 32, 128>(const XcorrArgs &, bool, int, cudaStream_t);

// Variants of the persistent batch launch (two per shape; the batch autotuner picks one
// per shape group).
template <int WSX, int WSY, int B, int NT>
cudaError_t launch_shape_batch(const XcorrBatch &b, bool deformed, int K, cudaStream_t s);
#define PIV_XCORR_BATCH_VARIANTS(X) \
    X(8, 8, 32, 128) \
    X(8, 8, 16, 128) \
    X(12, 12, 16, 96) \
    X(12, 12, 8, 96) \
    X(16, 16, 16, 128) \
    X(16, 16, 8, 128) \
    X(24, 24, 8, 96) \
    X(24, 24, 4, 96) \
    X(32, 32, 4, 128) \
    X(32, 32, 8, 128) \
    X(48, 48, 4, 96) \
    X(48, 48, 2, 96) \
    X(64, 64, 2, 128) \
    X(64, 64, 4, 128) \
    X(48, 24, 4, 96) \
    X(48, 24, 2, 64) \
    X(24, 48, 4, 96) \
    X(24, 48, 2, 64) \
    X(32, 16, 8, 128) \
    X(32, 16, 4, 64) \
    X(16, 32, 8, 128) \
    X(16, 32, 4, 64) \
    X(64, 32, 4, 128) \
    X(64, 32, 2, 64) \
    X(32, 64, 4, 128) \
    X(32, 64, 2, 64)
#define PIV_X(WX, WY, B, NT) extern template cudaError_t launch_shape_batch<WX, WY, B, NT>(const XcorrBatch &, bool, int, cudaStream_t);
PIV_XCORR_BATCH_VARIANTS(PIV_X)
#undef PIV_X

namespace {
struct Variant {
    int wsx, wsy, B, NT;
    cudaError_t (*fn)(const XcorrArgs &, bool, int, cudaStream_t);
};
const Variant kVariants[] = {
#define PIV_X(WX, WY, B, NT) {WX, WY, B, NT, &launch_shape<WX, WY, B, NT>},
    PIV_XCORR_VARIANTS(PIV_X)
#undef PIV_X
    {32, 32, 4, 128, &launch_shape_block<32, 32, 128>},
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

const Variant *find(int wsx, int wsy, int v)
{
    int seen = 0;
    for (int i = 0; i < kNumVariants; ++i)
        if (kVariants[i].wsx == wsx && kVariants[i].wsy == wsy) {
            if (seen == v) return &kVariants[i];
            ++seen;
        }
    return nullptr;
}
}  // namespace

int xcorr_variants(int wsx, int wsy)
{
    int n = 0;
    for (int i = 0; i < kNumVariants; ++i) n += (kVariants[i].wsx == wsx && kVariants[i].wsy == wsy);
    return n;
}

bool xcorr_supported(int wsx, int wsy) { return xcorr_variants(wsx, wsy) > 0; }

bool xcorr_variant_shape(int wsx, int wsy, int variant, int *B, int *NT)
{
    const Variant *v = find(wsx, wsy, variant);
    if (!v) return false;
    if (B) *B = v->B;
    if (NT) *NT = v->NT;
    return true;
}

namespace {
struct BatchVariant {
    int wsx, wsy, B, NT;
    cudaError_t (*fn)(const XcorrBatch &, bool, int, cudaStream_t);
};
const BatchVariant kBatchVariants[] = {
#define PIV_X(WX, WY, B, NT) {WX, WY, B, NT, &launch_shape_batch<WX, WY, B, NT>},
    PIV_XCORR_BATCH_VARIANTS(PIV_X)
#undef PIV_X
};

const BatchVariant *find_batch(int wsx, int wsy, int v)
{
    int seen = 0;
    for (const BatchVariant &b : kBatchVariants)
        if (b.wsx == wsx && b.wsy == wsy) {
            if (seen == v) return &b;
            ++seen;
        }
    return nullptr;
}
}  // namespace

int xcorr_batch_variants(int wsx, int wsy)
{
    int n = 0;
    for (const BatchVariant &b : kBatchVariants) n += (b.wsx == wsx && b.wsy == wsy);
    return n;
}

int xcorr_batch_windows_per_cta(int wsx, int wsy, int variant)
{
    const BatchVariant *v = find_batch(wsx, wsy, variant);
    return v ? v->B : 0;
}

cudaError_t launch_xcorr_batch(int wsx, int wsy, int variant, const XcorrBatch &b, bool deformed, int K,
                               cudaStream_t s, const char **why)
{
    const BatchVariant *v = find_batch(wsx, wsy, variant);
    if (!v) {
        if (why) *why = "window shape has no batch launch";
        return cudaErrorInvalidValue;
    }
    return v->fn(b, deformed, K, s);
}

cudaError_t launch_xcorr(const XcorrArgs &a, bool deformed, cudaStream_t s, const char **why, int variant)
{
    if (a.g.Nps > 8) {
        if (why) *why = "Npeak_save > 8 is not built into this engine";
        return cudaErrorInvalidValue;
    }
    const Variant *v = find(a.g.ws_x, a.g.ws_y, variant);
    if (!v) v = find(a.g.ws_x, a.g.ws_y, 0);
    if (!v) {
        if (why) *why = "window shape not built into this engine";
        return cudaErrorInvalidValue;
    }
    return v->fn(a, deformed, a.g.Nps <= 4 ? 4 : 8, s);
}

}  // namespace piv

namespace piv {

template <int WS, int NPROD, bool F16>
cudaError_t launch_tc_shape(const XcorrArgs &a, bool deformed, int K, cudaStream_t s, const TcStaging *stage);
#define PIV_TC(WS) \
    extern template cudaError_t launch_tc_shape<WS, 3, false>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *); \
    extern template cudaError_t launch_tc_shape<WS, 1, false>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *); \
    extern template cudaError_t launch_tc_shape<WS, 3, true>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *); \
    extern template cudaError_t launch_tc_shape<WS, 1, true>(const XcorrArgs &, bool, int, cudaStream_t, const TcStaging *);
PIV_TC(16)
PIV_TC(32)
PIV_TC(64)
#undef PIV_TC

template <int WX, int WY, int NPROD, bool F16>
cudaError_t launch_tc_rect_shape(const XcorrArgs &a, bool deformed, int K, cudaStream_t s);
#define PIV_TCR(WX, WY) \
    extern template cudaError_t launch_tc_rect_shape<WX, WY, 3, false>(const XcorrArgs &, bool, int, cudaStream_t); \
    extern template cudaError_t launch_tc_rect_shape<WX, WY, 1, false>(const XcorrArgs &, bool, int, cudaStream_t); \
    extern template cudaError_t launch_tc_rect_shape<WX, WY, 3, true>(const XcorrArgs &, bool, int, cudaStream_t); \
    extern template cudaError_t launch_tc_rect_shape<WX, WY, 1, true>(const XcorrArgs &, bool, int, cudaStream_t);
PIV_TCR(48, 24)
PIV_TCR(24, 48)
#undef PIV_TCR

bool xcorr_tc_supported(int wsx, int wsy)
{
    return (wsx == wsy && (wsx == 16 || wsx == 32 || wsx == 64)) || (wsx == 48 && wsy == 24) || (wsx == 24 && wsy == 48);
}

namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// the driver's tensor-map encoder, looked up once per process (a function-local static:
// engines created on several host threads initialise it once)
EncodeTiledFn encode_tiled()
{
    static const EncodeTiledFn fn = []() -> EncodeTiledFn {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<EncodeTiledFn>(f);
        return nullptr;
    }();
    return fn;
}

// a 2D map of a [rows][width] buffer (row stride `stride` bytes), box {bx, by}, zero fill
bool encode_2d(CUtensorMap &m, CUtensorMapDataType type, const void *base, int width, int rows, size_t stride, int bx,
               int by)
{
    EncodeTiledFn fn = encode_tiled();
    if (!fn || !base || (reinterpret_cast<uintptr_t>(base) & 15) || (stride & 15)) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)width, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)stride};
    const cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)by};
    const cuuint32_t estr[2] = {1, 1};
    return fn(&m, type, 2, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

cudaError_t tc_staging_build(TcStaging &st, int ws, int sp_x, const uint8_t *f1, const uint8_t *f2, int pitch,
                             int rows, const float *def, int def_pitch, int def_rows)
{
    memset(&st, 0, sizeof(st));
    if (ws != 16 && ws != 32) return cudaSuccess;  // 64 px windows load their rows directly
    const int nwin = 128 / ws, span = (nwin - 1) * sp_x + ws;
    st.bx1 = (span + 15 + 15) / 16 * 16;  // + up to 15 bytes of rounding the box start down
    st.bx2 = (span + 3 + 3) / 4 * 4;      // + up to 3 floats
    if (st.bx1 > 128 || st.bx2 > 128) return cudaSuccess;  // the kernel's staging buffers
    if (!encode_2d(st.f1, CU_TENSOR_MAP_DATA_TYPE_UINT8, f1, pitch, rows, (size_t)pitch, st.bx1, ws))
        return cudaSuccess;
    const bool ok = def ? encode_2d(st.f2, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, def, def_pitch, def_rows,
                                    (size_t)def_pitch * sizeof(float), st.bx2, ws)
                        : encode_2d(st.f2, CU_TENSOR_MAP_DATA_TYPE_UINT8, f2, pitch, rows, (size_t)pitch, st.bx1, ws);
    st.use = ok ? 1 : 0;
    return cudaSuccess;
}

cudaError_t launch_xcorr_tc(const XcorrArgs &a, bool deformed, cudaStream_t s, const char **why, int nprod, bool f16,
                            const TcStaging *stage)
{
    if (a.g.Nps > 8) {
        if (why) *why = "Npeak_save > 8 is not built into this engine";
        return cudaErrorInvalidValue;
    }
    if (!xcorr_tc_supported(a.g.ws_x, a.g.ws_y) || (nprod != 1 && nprod != 3)) {
        if (why) *why = "window shape not built into the tensor-core path";
        return cudaErrorInvalidValue;
    }
    const int K = a.g.Nps <= 4 ? 4 : 8;
    auto pick = [&](auto ws) -> cudaError_t {
        constexpr int WS = decltype(ws)::value;
        if (f16) return nprod == 3 ? launch_tc_shape<WS, 3, true>(a, deformed, K, s, stage)
                                   : launch_tc_shape<WS, 1, true>(a, deformed, K, s, stage);
        return nprod == 3 ? launch_tc_shape<WS, 3, false>(a, deformed, K, s, stage)
                          : launch_tc_shape<WS, 1, false>(a, deformed, K, s, stage);
    };
    if (a.g.ws_x != a.g.ws_y) {
        auto rect = [&](auto wx, auto wy) -> cudaError_t {
            constexpr int WX = decltype(wx)::value, WY = decltype(wy)::value;
            if (f16) return nprod == 3 ? launch_tc_rect_shape<WX, WY, 3, true>(a, deformed, K, s)
                                       : launch_tc_rect_shape<WX, WY, 1, true>(a, deformed, K, s);
            return nprod == 3 ? launch_tc_rect_shape<WX, WY, 3, false>(a, deformed, K, s)
                              : launch_tc_rect_shape<WX, WY, 1, false>(a, deformed, K, s);
        };
        if (a.g.ws_x == 48) return rect(std::integral_constant<int, 48>{}, std::integral_constant<int, 24>{});
        return rect(std::integral_constant<int, 24>{}, std::integral_constant<int, 48>{});
    }
    if (a.g.ws_x == 16) return pick(std::integral_constant<int, 16>{});
    if (a.g.ws_x == 32) return pick(std::integral_constant<int, 32>{});
    return pick(std::integral_constant<int, 64>{});
}

}  // namespace piv
