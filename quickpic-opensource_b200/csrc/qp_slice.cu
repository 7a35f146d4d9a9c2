// qp_slice.cu -- fused Fourier-space column kernels of the slice loop.
//
// After the x pass, column kx of every transformed component is contiguous
// ([kx][y]).  One CTA owns one column: its warps transform the column's lines
// along y (one warp per line), all threads then apply the Fourier-space
// solves of the slice mode by mode, and the warps transform the results back
// along y for the inverse x pass.  This fuses the reference's chain of
// fftrk / pot / grad / div / elf / bf / bfqp / mult / add / fftkr calls of one
// slice phase (simulation_class.f03:655-709, 717-726) into one launch per phase,
// with the per-mode arithmetic of qp_solve.cuh (bit-identical to the reference).
//
// Kernel A, slice start (simulation_class.f03:655-675 and the first 677-680):
//   qe, qb -> forward y; epwb = elf(qb); psi = pot(qe); fxy = grad(psi);
//   psit = -dex * pot(div(cu)); bxyz = bf(cu); bxyz <- assembly(epw, epwb);
//   inverse y of psi, fxy, psit, bxyz.
// Kernel B, one predictor-corrector pass (683-709 with the next 677-680, and
// the current extrapolation 725-726 applied to the stored cu):
//   cu, dcu, amu -> forward y; epw = bfqp(cu, dcu, amu, epw); cu_k <- cu - dxi*dcu
//   (x, y components); psit = -dex * pot(div(cu)); bxyz = bf(cu) + assembly;
//   inverse y of psit, bxyz; optionally the species2d%cbq smoothing of one
//   more line (q + cu_z) and the zeroing of the real-space accumulators.
#include "qp_line.cuh"
#include "qp_slice.cuh"
#include "qp_solve.cuh"

namespace qp {

namespace {

// Shared lines of pitch n + 4 floats; lines shorter than 64 points also need
// one scratch line per warp (line_transform's shared-memory form).
__host__ __device__ int col_pitch(int n) { return n + 4; }

template <int P>
__global__ void __launch_bounds__(256) k_slice_a(SliceA a, GridDims g, KCoef K, LineTables ty,
                                                 const DevStatus* st) {
  extern __shared__ __align__(16) float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = g.ny, pitch = col_pitch(n);
  const int kx = blockIdx.x;
  const long long co = (long long)kx * g.kp;
  float* line[8];
#pragma unroll
  for (int w = 0; w < 8; ++w) line[w] = smem + w * pitch;
  float* L = smem + warp * pitch;
  float* S = smem + (8 + warp) * pitch;
  float* T = smem + (P > 0 ? 8 : 16) * pitch;
  if (P > 0) stage_lane_table(T, ty);  // constant tables: staged before the wait
  grid_dep_sync();
  // the columns of qe and qb are read with the status: one L2 round trip
  LineRegs<(P > 0 ? P : 1)> r;
  if (P > 0 && (warp == 0 || (warp == 1 && a.qb)))
    reg_line_load<(P > 0 ? P : 1)>((warp == 0 ? a.qe : a.qb) + co, nullptr, a.norm, r, lane);
  const StatusSnap sn = status_snap(st);
  if (sn.error) return;
  // a new slice: no pass of it has converged yet (the passes follow this kernel)
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    DevStatus* ws = const_cast<DevStatus*>(st);
    ws->pass_done = 0;
    ws->resid_hist[0] = ws->resid_hist[1] = 1e30f;
  }
  if (P > 0) __syncthreads();
  // phase 1: forward y of qe (warp 0) and qb (warp 1)
  if (warp == 0 || (warp == 1 && a.qb)) {
    if constexpr (P > 0)
      reg_line_core<P>(r, L, 0, T, lane);
    else
      line_transform<P>((warp == 0 ? a.qe : a.qb) + co, nullptr, a.norm, L, S, g.indy, 0, ty, T,
                        lane);
  } else if (warp == 1) {
    for (int j = lane; j <= n; j += 32) L[j] = 0.f;
  }
  __syncthreads();
  // phase 2: the solves of the slice start, mode by mode
  for (int ky = threadIdx.x; ky <= n; ky += blockDim.x) {
    const long long o = co + ky;
    // every global read of the mode first, so they wait for L2 together
    const float cx = a.cu_x[o], cy = a.cu_y[o], cz = a.cu_z[o];
    float ex = a.epw_x[o], ey = a.epw_y[o];
    float ex0 = 0.f, ey0 = 0.f, ex00 = 0.f, ey00 = 0.f;
    if (a.epw_prev_x) {
      ex0 = a.epw_prev_x[o];
      ey0 = a.epw_prev_y[o];
      if (a.epw_prev2_x) {
        ex00 = a.epw_prev2_x[o];
        ey00 = a.epw_prev2_y[o];
      }
    }
    const float q = line[0][ky], qb = line[1][ky];
    float ebx, eby;
    k_elf(K, kx, ky, qb, &ebx, &eby);
    a.epwb_x[o] = ebx;
    a.epwb_y[o] = eby;
    const float psi = k_pot(K, kx, ky, q);
    float fx, fy;
    k_grad(K, kx, ky, psi, &fx, &fy);
    const float psit = QM(k_pot(K, kx, ky, k_div(K, kx, ky, cx, cy)), -a.dex);
    float bx, by, bz;
    k_bf(K, kx, ky, cx, cy, cz, &bx, &by, &bz);
    if (a.epw_prev_x) {
      const float ex1 = ex, ey1 = ey;
      if (a.epw_prev2_x) {
        ex = QA(QM(3.f, QS(ex1, ex0)), ex00);
        ey = QA(QM(3.f, QS(ey1, ey0)), ey00);
        a.epw_prev2_x[o] = ex0;
        a.epw_prev2_y[o] = ey0;
      } else {
        ex = QS(QM(2.f, ex1), ex0);
        ey = QS(QM(2.f, ey1), ey0);
      }
      a.epw_x[o] = ex;
      a.epw_y[o] = ey;
      a.epw_prev_x[o] = ex1;
      a.epw_prev_y[o] = ey1;
    }
    k_assemble_mode(ex, ey, ebx, eby, a.dex, &bx, &by, &bz);
    line[0][ky] = bz;
    line[2][ky] = psi;
    line[3][ky] = fx;
    line[4][ky] = fy;
    line[5][ky] = psit;
    line[6][ky] = bx;
    line[7][ky] = by;
  }
  __syncthreads();
  // phase 3: inverse y; y parities: psi S, fx S, fy C, psit S, bx C, by S, bz C
  if (warp != 1) {
    float* dst;
    int par;
    switch (warp) {
      case 0: dst = a.out_bz; par = 1; break;
      case 2: dst = a.out_psi; par = 0; break;
      case 3: dst = a.out_fx; par = 0; break;
      case 4: dst = a.out_fy; par = 1; break;
      case 5: dst = a.out_psit; par = 0; break;
      case 6: dst = a.out_bx; par = 1; break;
      default: dst = a.out_by; par = 0; break;
    }
    line_transform<P>(L, nullptr, 1.f, L, S, g.indy, par, ty, T, lane);
    line_store(dst + co, L, n, 1.f, lane);
  }
}

// 9 warps: warps 0-7 carry the 8 transformed components, warp 8 the optional
// cbq line (q + cu_z).
template <int P>
__global__ void __launch_bounds__(288) k_slice_b(SliceB b, GridDims g, KCoef K, LineTables ty,
                                                 DevStatus* st) {
  extern __shared__ __align__(16) float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = g.ny, pitch = col_pitch(n);
  const int kx = blockIdx.x;
  const long long co = (long long)kx * g.kp;
  float* line[9];
#pragma unroll
  for (int w = 0; w < 9; ++w) line[w] = smem + w * pitch;
  float* L = smem + warp * pitch;
  float* S = smem + (9 + warp) * pitch;
  float* T = smem + (P > 0 ? 9 : 18) * pitch;
  if (P > 0) stage_lane_table(T, ty);  // constant tables: staged before the wait
  grid_dep_sync();
  if (st->error) return;
  if (pass_skipped(st, b.pass)) return;
  if (P > 0) __syncthreads();
  // phase 1: forward y of cu(3), dcu(2), amu(3): y parities S C S, S C, S S C
  if (warp < 8) {
    const int par = (warp == 1 || warp == 4 || warp == 7) ? 1 : 0;
    line_transform<P>(b.in[warp] + co, nullptr, b.norm, L, S, g.indy, par, ty, T, lane);
  } else if (b.q_in) {
    line_transform<P>(b.q_in + co, nullptr, b.norm, L, S, g.indy, 0, ty, T, lane);
  }
  __syncthreads();
  // phase 2: corrector, extrapolated current, psit and bxyz of the next pass
  float r_num = 0.f, r_den = 0.f;
  for (int ky = threadIdx.x; ky <= n; ky += blockDim.x) {
    const long long o = co + ky;
    const float cx = line[0][ky], cy = line[1][ky], cz = line[2][ky];
    float dcx = line[3][ky], dcy = line[4][ky];
    const float axx = line[5][ky], ayy = line[6][ky], axy = line[7][ky];
    // every global read of the mode first, so they wait for L2 together
    const float ex0 = b.epw_x[o], ey0 = b.epw_y[o];
    const float ebx = b.epwb_x[o], eby = b.epwb_y[o];
    float ex = ex0, ey = ey0;
    k_bfqp(K, kx, ky, b.aa, b.idex, cz, &dcx, &dcy, axx, ayy, axy, &ex, &ey);
    b.epw_x[o] = ex;
    b.epw_y[o] = ey;
    r_num += (ex - ex0) * (ex - ex0) + (ey - ey0) * (ey - ey0);
    r_den += ex * ex + ey * ey;
    // dcu = dcu * dxi; cu(1:2) = cu(1:2) - dcu(1:2)  (kept for the next slice)
    b.cu_x[o] = QS(cx, QM(dcx, b.dxi));
    b.cu_y[o] = QS(cy, QM(dcy, b.dxi));
    b.cu_z[o] = cz;
    const float psit = QM(k_pot(K, kx, ky, k_div(K, kx, ky, cx, cy)), -b.dex);
    float bx, by, bz;
    k_bf(K, kx, ky, cx, cy, cz, &bx, &by, &bz);
    k_assemble_mode(ex, ey, ebx, eby, b.dex, &bx, &by, &bz);
    line[0][ky] = psit;
    line[1][ky] = bx;
    line[2][ky] = by;
    line[3][ky] = bz;
    if (b.q_in) line[8][ky] = k_smooth(K, kx, ky, line[8][ky]);
    if (b.vpot_out[0]) {
      float ax, ay, az;
      k_vpot(K, kx, ky, cx, cy, cz, &ax, &ay, &az);
      b.vpot_out[0][o] = ax;
      b.vpot_out[1][o] = ay;
      b.vpot_out[2][o] = az;
    }
  }
  // relative change of B_perp for the convergence-controlled iteration: the
  // CTA's sums are formed in shared memory and added with one reduction each
  // (every CTA's reductions go to the same two words, and a reduction per
  // warp made those words an L2 bottleneck)
  __shared__ float rsum[2][9];
  r_num = warp_sum(r_num);
  r_den = warp_sum(r_den);
  if (lane == 0) {
    rsum[0][warp] = r_num;
    rsum[1][warp] = r_den;
  }
  __syncthreads();
  if (b.track_residual && threadIdx.x == 0) {
    float sn = 0.f, sd = 0.f;
#pragma unroll
    for (int w = 0; w < 9; ++w) {
      sn += rsum[0][w];
      sd += rsum[1][w];
    }
    atomicAdd(&st->resid_num, sn);
    atomicAdd(&st->resid_den, sd);
    // the last CTA to finish has the complete sums: decide, and reset them for
    // the next pass (which starts only after this kernel)
    __threadfence();
    if (atomicAdd(&st->pass_ctas, 1) == (int)gridDim.x - 1) {
      __threadfence();
      const float num = atomicAdd(&st->resid_num, 0.f), den = atomicAdd(&st->resid_den, 0.f);
      const int cur = st->cursor;
      const float r = den > 0.f ? num / den : (num > 0.f ? 1.f : 0.f);
      const bool stalled = pass_stalled(b.pass, r, st->resid_hist[0], st->resid_hist[1]);
      if (r <= b.tol2) {
        st->pass_done = b.pass;
        if (b.slice_passes && cur >= 0 && cur <= b.max_slice) b.slice_passes[cur] = b.pass;
      } else if (stalled || b.pass >= b.max_pass) {
        if (stalled) st->pass_done = b.pass;
        st->unconverged = st->unconverged + 1;
        if (b.slice_passes && cur >= 0 && cur <= b.max_slice) b.slice_passes[cur] = -b.pass;
      }
      st->resid_hist[1] = st->resid_hist[0];
      st->resid_hist[0] = r;
      st->passes = st->passes + 1;
      st->resid_num = 0.f;
      st->resid_den = 0.f;
      st->pass_ctas = 0;
      __threadfence();
    }
  }
  // phase 3: inverse y of psit (S), bx (C), by (S), bz (C) and the smoothed q (S)
  if (warp < 4) {
    const int par = (warp == 1 || warp == 3) ? 1 : 0;
    line_transform<P>(L, nullptr, 1.f, L, S, g.indy, par, ty, T, lane);
    line_store(b.out[warp] + co, L, n, 1.f, lane);
  } else if (warp == 8) {
    if (b.q_in) {
      line_transform<P>(L, nullptr, 1.f, L, S, g.indy, 0, ty, T, lane);
      line_store(b.q_out + co, L, n, 1.f, lane);
    }
  } else if (b.nzero) {
    // zero the real-space accumulators for the next pass (their values were
    // consumed by the x pass that precedes this kernel)
    const long long per = (g.rplane + gridDim.x - 1) / gridDim.x;
    const long long lo = per * kx, hi = min(g.rplane, lo + per);
    for (int z = 0; z < b.nzero; ++z)
      for (long long i = lo + (threadIdx.x - 128); i < hi; i += 128) b.zero[z][i] = 0.f;
  }
}

}  // namespace

size_t slice_a_smem(const GridDims& g) {
  return sizeof(float) *
         ((g.indy < 6 ? 16 : 8) * (size_t)col_pitch(g.ny) + lt_floats(line_p(g.indy)));
}
size_t slice_b_smem(const GridDims& g) {
  return sizeof(float) *
         ((g.indy < 6 ? 18 : 9) * (size_t)col_pitch(g.ny) + lt_floats(line_p(g.indy)));
}

template <int P>
static int set_slice_smem(int big) {
  if (cudaFuncSetAttribute(k_slice_a<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, big) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_slice_b<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, big) !=
          cudaSuccess)
    return -2;
  return 0;
}

int slice_kernels_init() {
  const int big =
      (int)(sizeof(float) * (9 * col_pitch(1 << QP_MAX_IND) + lt_floats(line_p(QP_MAX_IND))));
  for (int logn = 4; logn <= QP_MAX_IND; ++logn) {
    int rc = 0;
    QP_LINE_SWITCH(logn, rc = set_slice_smem<P_>(big));
    if (rc) return rc;
  }
  return 0;
}

void launch_slice_a(const SliceA& a, const GridDims& g, const KCoef& K, const LineTables& ty,
                    const DevStatus* st, cudaStream_t s) {
  QP_LINE_SWITCH(g.indy,
                 (launch_pdl(k_slice_a<P_>, g.nx + 1, 256, slice_a_smem(g), s, a, g, K, ty, st)));
}

void launch_slice_b(const SliceB& b, const GridDims& g, const KCoef& K, const LineTables& ty,
                    DevStatus* st, cudaStream_t s) {
  QP_LINE_SWITCH(g.indy,
                 (launch_pdl(k_slice_b<P_>, g.nx + 1, 288, slice_b_smem(g), s, b, g, K, ty, st)));
}

}  // namespace qp
