// learned.cuh -- the learned grid-1 predictor (no counterpart in the reference): internal
// interface between the network (learned.cu) and the engine (engine.cu).
//
// The predictor maps the 4x-downsampled frame pair to the grid-1 displacement field:
//   features  each frame is box-averaged over 4x4 pixels (grey / 255) and its global mean
//             removed; at every grid-1 vector a (ws/4)^2 window of frame 1 is correlated
//             with frame 2 at the (2R+1)^2 integer shifts |dx|, |dy| <= R of the
//             downsampled grid and normalised by the windows' energies: an 81-channel
//             cost volume on the grid-1 vector grid (fixed, no parameters);
//   network   a 4-level U-Net on that grid (levels 1, 1/2, 1/4, 1/8), 3x3 convolutions
//             with LeakyReLU(0.1), stride-2 convolutions down, nearest upsampling and
//             skip concatenation up, a linear 2-channel head in downsampled pixels
//             (x4 = image pixels).  BF16 weights, FP32 activations and accumulation.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "piv_common.cuh"

struct piv_net;

namespace piv {
namespace learned {

constexpr int kRadius = 4;                       // cost-volume shifts, downsampled px
constexpr int kShifts = 2 * kRadius + 1;
constexpr int kInChannels = kShifts * kShifts;   // 81
constexpr int kDown = 4;                         // downsampling factor
constexpr float kOutScale = (float)kDown;        // head unit -> image px

// Features of one frame pair: the padded u8 frames of the engine and its grid-1 geometry.
struct FeatArgs {
    const uint8_t *f1, *f2;  // image pixel (0, 0) of each frame
    int pitch;               // bytes per frame row
    int Nx, Ny;              // image size
    GridGeom g;              // grid-1 geometry (vector grid, spacing, left padding, window)
    float *down;             // scratch: 2 * (Nx/4) * (Ny/4) floats
    double *sums;            // scratch: 2 doubles (zeroed by the launch)
    float *out;              // [81][Ny_vec][Nx_vec]
};
size_t feature_scratch_floats(int Nx, int Ny);
cudaError_t launch_features(const FeatArgs &a, cudaStream_t s);

// Network forward on [N][81][H][W] -> [N][2][H][W] (downsampled px).  Buffers of the net
// are (re)allocated for (N, H, W) by net_reserve, which must precede a graph capture.
int net_reserve(piv_net *n, int N, int H, int W);
float *net_input(piv_net *n);
const float *net_output(piv_net *n);  // [N][2][H][W] of the last forward
cudaError_t net_forward(piv_net *n, const float *in, int N, int H, int W, float *out, cudaStream_t s);
// grid-1 field from the network output [2][Nt] (downsampled px): fx = 4*out, all valid
cudaError_t launch_field_from_net(const float *out, int Nt, float *fx, float *fy, uint8_t *fv, cudaStream_t s);
// judge[0] = sum over the Nt vectors of |pred - final|^2, judge[1] = *list_n (the last
// median test's rejects)
cudaError_t launch_judge(const float *px, const float *py, const float *fx, const float *fy, int Nt,
                         const int *list_n, float *judge, cudaStream_t s);
// changes whenever net_reserve / net_reserve_features move or re-lay-out a buffer: a
// graph captured with the net's buffers is stale once it differs
unsigned net_generation(const piv_net *n);
// PIV_ERR_DEVICE (and clears it) if a tensor-core convolution reported a timed-out wait;
// synchronous (reads one word)
int net_check_status(piv_net *n);
// feature scratch owned by the net (sized for the largest frame seen)
int net_reserve_features(piv_net *n, int Nx, int Ny);
float *net_feature_down(piv_net *n);
double *net_feature_sums(piv_net *n);

}  // namespace learned
}  // namespace piv
