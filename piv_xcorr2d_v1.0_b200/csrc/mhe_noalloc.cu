// mhe_noalloc.cu -- MHE contrast enhancement that allocates nothing.
//
// Some callers cannot call cudaMalloc at the point where they want to enhance a frame:
// code running while a CUDA graph is being captured (an allocation synchronises the
// device and breaks the capture), real-time acquisition callbacks that must not wait
// on the allocator, and host applications that hand all device memory to their own
// pool and forbid plugins from allocating after start-up.  For them this entry point
// runs the same two MHE kernels as piv_mhe_process, with the per-tile histogram grid
// (the kernels' only scratch) in a fixed device array that the library owns.
//
// The array is a file-scope __device__ variable: every GPU that loads this library
// holds it (24 MiB) until the process exits.  In host code the symbol g_mhe_scratch
// is a host-side stand-in, not a device address, so the host asks the runtime for the
// device address once per device and passes that pointer to the kernels.
#include <cstdio>
#include <mutex>

#include "piv_common.cuh"

namespace {

constexpr long kMaxLevels = (long)PIV_MHE_NOALLOC_MAX_TILES * 256;  // ints

static __device__ __align__(256) int g_mhe_scratch[kMaxLevels];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
int *g_dev_ptr[kMaxDevices] = {};

// Device address of g_mhe_scratch on the current device (set up on first use).
int scratch_ptr(int **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PIV_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_dev_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_mhe_scratch);
        if (e != cudaSuccess || !p) return PIV_ERR_CUDA;
        g_dev_ptr[dev] = static_cast<int *>(p);
    }
    *out = g_dev_ptr[dev];
    return PIV_OK;
}

}  // namespace

extern "C" int piv_mhe_process_noalloc(const uint8_t *d_in, uint8_t *d_out, int Nx, int Ny, int ws, float thresh,
                                       void *stream)
{
    if (!d_in || !d_out) return PIV_ERR_ARG;
    piv::MheGeom m;
    if (!piv::mhe_geometry(Nx, Ny, ws, thresh, m)) return PIV_ERR_ARG;
    const long tiles = (long)(m.maxI + 2) * (m.maxJ + 2);
    if (tiles > PIV_MHE_NOALLOC_MAX_TILES) {
        fprintf(stderr,
                "piv_mhe_process_noalloc: %dx%d image with %d px tiles needs %ld histogram tiles (with the border "
                "ring), more than the fixed scratch holds (%d); use piv_mhe_process instead\n",
                Nx, Ny, ws, tiles, PIV_MHE_NOALLOC_MAX_TILES);
        return PIV_ERR_ARG;
    }
    int *levels = nullptr;
    int rc = scratch_ptr(&levels);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the array keeps the previous call's histograms; this call's zero ring must be zero
    if (cudaMemsetAsync(levels, 0, (size_t)tiles * 256 * sizeof(int), s) != cudaSuccess) return PIV_ERR_CUDA;
    if (m.width != Nx || m.height != Ny) {
        // pixels outside the centred crop are defined as 0 (the reference's zeroed d_enhanced)
        if (cudaMemsetAsync(d_out, 0, (size_t)Nx * Ny, s) != cudaSuccess) return PIV_ERR_CUDA;
    }
    if (piv::launch_mhe(m, d_in, Nx, levels, d_out, Nx, 0, 0, s) != cudaSuccess) return PIV_ERR_CUDA;
    return PIV_OK;
}
