// qp_common.cuh -- shared definitions of the B200 quasi-static slice engine.
//
// Device data layout (all FP32, one plane per field component):
//   real-space plane  R[y][x], y = 0..ny (row ny is the guard row), x = 0..nx+1,
//                     row pitch rp = nx + 4 floats (16-byte aligned rows)
//   k-space plane     K[kx][ky], kx = 0..nx, ky = 0..ny, pitch kp = ny + 4;
//                     the same array holds the half-transformed data between
//                     the x pass and the y pass ([kx][y])
//   particles         structure of arrays: 8 planes (x, y, px, py, pz, p6, p7, q)
//                     of ntiles * cap floats; tile t owns [t*cap, t*cap+count[t])
// Grid nodes, tile size and the particle slots follow QuickPIC's part2d/ufield2d
// (16 x 16 cell tiles, positions in cell units, node j at x = j).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>

#define QP_MAX_IND 11  // largest supported log2 of a transverse grid size

namespace qp {

struct GridDims {
  int indx, indy, nx, ny;
  int rp;        // real-space row pitch (floats)
  int kp;        // k-space column pitch (floats)
  long long rplane;  // floats per real-space plane: (ny + 1) * rp
  long long kplane;  // floats per k-space plane: (nx + 1) * kp
};

inline GridDims make_dims(int indx, int indy) {
  GridDims d;
  d.indx = indx;
  d.indy = indy;
  d.nx = 1 << indx;
  d.ny = 1 << indy;
  d.rp = d.nx + 4;
  d.kp = d.ny + 4;
  d.rplane = (long long)(d.ny + 1) * d.rp;
  d.kplane = (long long)(d.nx + 1) * d.kp;
  return d;
}

// Twiddle tables for one line length n (host-computed in double, stored FP32).
struct LineTables {
  const float* sn;   // sin(pi j / n), j = 0..n
  const float* cs;   // cos(pi j / n), j = 0..n
  const float2* tw;  // exp(-2 pi i m / (n/2)), m = 0..n/2-1  (complex FFT of n/2)
  const float2* uw;  // exp(-2 pi i k / n),     k = 0..n/2    (real-FFT unscramble)
  // n >= 64: the same values rearranged as the register transform reads them,
  // one row of 32 per register slot (qp_line.cuh, LT_*), lane_floats floats
  const float* lane;
  int lane_floats;
};

// Layout of LineTables::lane for P = n / 64 (offsets in floats).
__host__ __device__ constexpr int lt_sn0(int P) { return 0; }
__host__ __device__ constexpr int lt_sn1(int P) { return 32 * P; }
__host__ __device__ constexpr int lt_cs0(int P) { return 64 * P; }
__host__ __device__ constexpr int lt_cs1(int P) { return 96 * P; }
__host__ __device__ constexpr int lt_tw4(int P) { return 128 * P; }   // float2 [P][32]
__host__ __device__ constexpr int lt_uw(int P) { return 192 * P; }    // float2 [P][32]
__host__ __device__ constexpr int lt_tw5(int P) { return 256 * P; }   // float2 [4][32]
__host__ __device__ constexpr int lt_tw3(int P) { return 256 * P + 256; }  // float2 [16]
__host__ __device__ constexpr int lt_w32(int P) { return 256 * P + 288; }  // float2 [4][8]
__host__ __device__ constexpr int lt_floats(int P) { return P > 0 ? 256 * P + 352 : 0; }
// Lines of 64 P points whose 32-point lane stage goes through shared memory
// (reg_line_tail_xs) instead of shuffles; their unscramble table is in lane
// order, the others' in bit-reversed lane order.
__host__ __device__ constexpr bool line_xs(int P) { return P == 8; }

// Sticky device status shared by every kernel of a context.
struct __align__(16) DevStatus {
  int error;          // 0 = ok; >0 = capacity overflow (see need); <0 = fatal
  int fail_slice;     // slice index at which the first error was raised
  int need_cap;       // particles a tile must hold
  int need_inbox;     // movers a tile must accept
  int cursor;         // slice cursor of the fused 3D step
  int pass_done;      // convergence-controlled B loop: the pass of this slice
                      // whose residual met the tolerance (0 = none yet)
  int store_ctas;     // CTA completion counter of the 3D store kernel
  int beam_drops;     // beam particles dropped at the conducting boundary
  float resid_num;    // residual of the current pass: sum |epw - epw_old|^2
  float resid_den;    //                               sum |epw|^2
  int pass_ctas;      // CTA completion counter of the residual decision
  int passes;         // predictor-corrector passes run in this 3D step
  int unconverged;    // slices of this step that stopped without meeting the tolerance
  float resid_hist[2];  // this slice's squared relative residuals, one and two passes back
};

// Convergence control of the B passes of a slice (k_slice_b and the oracle):
// with r the squared relative change of B_perp after pass `pass`, the slice
// has converged once r <= tol^2; from pass QP_STALL_PASS on it has stalled
// (the FP32 iteration can settle into a cycle above the tolerance) once r is
// no longer below 0.81 times the smaller of the two previous values, i.e. the
// relative change stopped dropping by 10 %.
#define QP_STALL_PASS 8
__host__ __device__ inline bool pass_stalled(int pass, float r, float r1, float r2) {
  return pass >= QP_STALL_PASS && r >= 0.81f * fminf(r1, r2);
}

// A kernel of pass `pass` (1-based; 0 = not part of a convergence-controlled
// loop) has nothing to do once an earlier pass of the slice has converged.
__device__ __forceinline__ bool pass_skipped(const DevStatus* st, int pass) {
  if (pass <= 1) return false;
  const int done = st->pass_done;
  return done > 0 && done < pass;
}

// The words of the device status a slice kernel checks before its work, read
// with two 16-byte loads (error .. need_inbox, cursor .. beam_drops) that a
// kernel issues together with its first data loads.
struct StatusSnap {
  int error, cursor, pass_done;
};
__device__ __forceinline__ StatusSnap status_snap(const DevStatus* st) {
  const int4* p = reinterpret_cast<const int4*>(st);
  const int4 a = p[0], b = p[1];
  return StatusSnap{a.x, b.x, b.y};
}
// pass_skipped on a snapshot
__device__ __forceinline__ bool snap_skipped(const StatusSnap& s, int pass) {
  return pass > 1 && s.pass_done > 0 && s.pass_done < pass;
}

enum { QP_OK = 0, QP_OVERFLOW = 1 };

// Programmatic dependent launch.  The slice kernels are launched with
// launch_pdl, which lets a grid's CTAs start on the SMs that the grid before
// it in the stream no longer fills.  Every kernel therefore opens with
// grid_dep_sync() before it touches device data: griddepcontrol.wait returns
// once the preceding grid has completed and its writes are visible (at once
// for a kernel launched without the attribute), and launch_dependents then
// allows the next grid to be scheduled behind this one.  Data that no kernel
// writes (the twiddle tables) may be read before the wait.
__device__ __forceinline__ void grid_dep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void grid_dep_launch() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void grid_dep_sync() {
  grid_dep_wait();
  grid_dep_launch();
}

template <typename... KP, typename... A>
inline cudaError_t launch_pdl(void (*k)(KP...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t s, A... a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, a...);
}

}  // namespace qp

#define QP_CUDA_CHECK(call)                                                         \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      qp_set_error(__FILE__, __LINE__, cudaGetErrorString(e_));                     \
      return -2;                                                                    \
    }                                                                               \
  } while (0)

void qp_set_error(const char* file, int line, const char* msg);
