// mhe_noalloc.cu -- MHE contrast enhancement that allocates nothing.
//
// Some callers cannot call cudaMalloc at the point where they want to enhance a frame:
// real-time acquisition callbacks that must not wait on the allocator (an allocation can
// synchronise the device), and host applications that hand all device memory to their
// own pool at start-up and forbid plugins from allocating afterwards.  For them this
// entry point runs the same two MHE kernels as piv_mhe_process, with the per-tile
// histogram grid (the kernels' only scratch) in a fixed device array that the library
// owns.
//
// The array is a file-scope __device__ variable: every GPU that loads this library
// holds it (24 MiB) until the process exits.  In host code the symbol g_mhe_scratch
// is a host-side stand-in, not a device address, so the host asks the runtime for the
// device address and passes that pointer to the kernels.  The address is looked up
// once per device context: on the first call on a device, and again when that device's
// context has been re-created (after cudaDeviceReset the module is loaded anew and the
// array may sit elsewhere).  Contexts are told apart by their unique ID (cuCtxGetId),
// not by their handle, which a new context may reuse.
#include <cuda.h>
#include <cstdio>
#include <mutex>

#include "piv_common.cuh"

namespace {

constexpr long kMaxLevels = (long)PIV_MHE_NOALLOC_MAX_TILES * 256;  // ints

static __device__ __align__(256) int g_mhe_scratch[kMaxLevels];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct Cached {
    unsigned long long ctx = 0;  // unique ID of the context the address belongs to
    int *ptr = nullptr;
};
Cached g_cache[kMaxDevices];

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_get_current = nullptr;
CtxGetIdFn g_get_id = nullptr;
bool g_resolved = false;

// Unique ID of the calling thread's current context, 0 if there is none (or the driver
// offers no context IDs).  Called with g_mu held.
unsigned long long current_context_id()
{
    if (!g_resolved) {
        g_resolved = true;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_get_id = reinterpret_cast<CtxGetIdFn>(f);
    }
    if (!g_get_current || !g_get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (g_get_current(&c) != CUDA_SUCCESS || !c) return 0;
    if (g_get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of g_mhe_scratch in the current device's current context.
int scratch_ptr(int **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PIV_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    Cached &c = g_cache[dev];
    const unsigned long long ctx = current_context_id();
    if (!c.ptr || ctx == 0 || ctx != c.ctx) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_mhe_scratch);
        if (e != cudaSuccess || !p) {
            c = Cached{};
            return PIV_ERR_CUDA;
        }
        c.ptr = static_cast<int *>(p);
        c.ctx = current_context_id();  // the lookup made the device's context current
    }
    *out = c.ptr;
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
