// qp_slice.cuh -- fused Fourier-space column kernels of the slice loop.
#pragma once

#include "qp_common.cuh"
#include "qp_solve.cuh"

namespace qp {

// Slice start.  qe, qb: x-transformed columns ([kx][y]); cu_*: the extrapolated
// Fourier-space current of the previous slice; epw_*: B_perp of the previous
// slice; epwb_*: out, beam E_perp; out_*: y-inverse columns for the x pass.
struct SliceA {
  const float* qe;
  const float* qb;  // null without beams
  const float *cu_x, *cu_y, *cu_z;
  float *epw_x, *epw_y;
  // optional predictor: B_perp two (and three) slices back; epw becomes
  // 2 epw - epw_prev, or 3 epw - 3 epw_prev + epw_prev2 (written back), and the
  // history shifts by one slice
  float *epw_prev_x, *epw_prev_y;
  float *epw_prev2_x, *epw_prev2_y;  // quadratic predictor only
  float *epwb_x, *epwb_y;
  float *out_psi, *out_fx, *out_fy, *out_psit, *out_bx, *out_by, *out_bz;
  float norm, dex;
};

// One predictor-corrector pass.  in[0..7]: x-transformed cu(3), dcu(2),
// amu(3); the Fourier-space cu is written back extrapolated to cu_*; epw_* is
// read and updated; out[0..3]: y-inverse columns of psit, bx, by, bz.
struct SliceB {
  const float* in[8];
  float *cu_x, *cu_y, *cu_z;
  float *epw_x, *epw_y;
  const float *epwb_x, *epwb_y;
  float* out[4];
  const float* q_in;  // optional x-transformed q + cu_z (species2d%cbq)
  float* q_out;
  float* vpot_out[3];  // optional: the vector potential of the pass's current (Fourier space)
  float* zero[8];     // real-space planes to clear for the next pass
  int nzero;
  // convergence-controlled loop: accumulate the relative change of B_perp,
  // and let the last CTA mark the slice converged (DevStatus.pass_done = pass)
  // when sum |epw - epw_old|^2 <= tol2 * sum |epw|^2
  int track_residual;
  int pass;           // 1-based pass of this launch; later passes skip once converged
  int max_pass;       // the last pass a slice may take
  int* slice_passes;  // optional, per slice cursor: the converging pass, or -max_pass
  int max_slice;      // last valid index of slice_passes
  float tol2;
  float norm, dex, idex, aa, dxi;
};

int slice_kernels_init();
size_t slice_a_smem(const GridDims& g);
size_t slice_b_smem(const GridDims& g);
void launch_slice_a(const SliceA& a, const GridDims& g, const KCoef& K, const LineTables& ty,
                    const DevStatus* st, cudaStream_t s);
void launch_slice_b(const SliceB& b, const GridDims& g, const KCoef& K, const LineTables& ty,
                    DevStatus* st, cudaStream_t s);

}  // namespace qp
