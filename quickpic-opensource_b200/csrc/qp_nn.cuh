// qp_nn.cuh -- the learned predictor of the transverse-B start: a 5-layer 3x3
// convolutional network on Fourier-space images, with BF16 tcgen05 kernels.
//
// The predictor maps, for slice j, the Fourier-space B_perp iterates of the
// three previous slices (epw(j-1), epw(j-2), epw(j-3)), the current handed to slice j
// (cu_k after the xi extrapolation) and the mode coordinates to a correction
// of the quadratic extrapolation 3 epw(j-1) - 3 epw(j-2) + epw(j-3), in the
// low-mode window kx, ky < 128 it is trained on: the start of slice j's
// predictor-corrector passes (the hook at simulation_class.f03:676, where the
// reference starts from epw(j-1)).  The passes still run to the tolerance.
//
// Images are BF16 in a channel-group-planar layout [G][NB][H][W][8] (G =
// channels / 8): 8 channels of one pixel are 16 contiguous bytes, which is one
// row of a tcgen05 core matrix, so a 3x3 tap of the convolution is the same
// shared-memory tile addressed from another start (an implicit GEMM with no
// im2col copy).  H runs over kx, W over ky, from mode 0.
#pragma once

#include <cuda_bf16.h>

#include "qp_common.cuh"

namespace qp {

constexpr int NN_LAYERS = 5;
constexpr int NN_CIN0 = 16;     // input channels of layer 1 (NN_FEATURES used, the rest zero)
constexpr int NN_CH = 32;       // hidden channels
constexpr int NN_NLAST = 16;    // output channels of layer 5 as computed (NN_OUT used)
constexpr int NN_OUT = 2;       // the correction of epw_x, epw_y
// e1, e1 - e0, e0 - e(-1) (x and y each, over the epw scale), cu.x, cu.y, cu.z
// (over their scales), kx/nx, ky/ny, the slice width dxi / (10/256): the
// history enters as differences, so that the network sees slopes and
// curvatures without the cancellation of nearly equal bfloat16 values, and
// the slice width sets how far the fields move from one slice to the next
constexpr int NN_FEATURES = 12;
constexpr int NN_CROP = 128;    // side of the training crop (the low-mode corner)
constexpr int NN_NORM_BLOCKS = 148;

inline int nn_cin(int l) { return l == 0 ? NN_CIN0 : NN_CH; }
inline int nn_cout(int l) { return l == NN_LAYERS - 1 ? NN_NLAST : NN_CH; }
// fp32 parameters of layer l: W[9][cin][cout] then bias[cout]
inline int nn_layer_params(int l) { return 9 * nn_cin(l) * nn_cout(l) + nn_cout(l); }
int nn_total_params();

// The k-space planes the predictor reads and writes for one slice.
struct NNSlicePlanes {
  float* epw_x;          // in: epw(j-1); out: the start of slice j
  float* epw_y;
  float* prev_x;         // in: epw(j-2); out: epw(j-1)
  float* prev_y;
  float* prev2_x;        // in: epw(j-3); out: epw(j-2)
  float* prev2_y;
  const float* cu_x;     // the current handed to slice j
  const float* cu_y;
  const float* cu_z;
  float dxi;             // slice width (c/wp)
};

struct NNRuntime;  // per-simulation buffers and tensor maps (qp_nn.cu)

// Per-simulation inference set-up on an nx x ny grid (ny a multiple of 128).
int nn_runtime_create(const GridDims& g, NNRuntime** out);
void nn_runtime_destroy(NNRuntime* r);
// The start of slice j from the network (norms, features, 5 conv layers).
// Returns the number of launches; st->error set on a device-side failure.
int nn_predict(NNRuntime* r, const void* net, const NNSlicePlanes& p, const GridDims& g,
               DevStatus* st, cudaStream_t s);
// Recording of training pairs: at the start of slice j (features of the crop,
// minus the quadratic extrapolation into the target slot; the history moves on),
// and at its end (plus the converged epw).  Both skip once the set is full.
int nn_record_start(NNRuntime* r, void* data, const NNSlicePlanes& p, const GridDims& g,
                    DevStatus* st, cudaStream_t s);
int nn_record_end(NNRuntime* r, void* data, const NNSlicePlanes& p, const GridDims& g,
                  DevStatus* st, cudaStream_t s);

}  // namespace qp
