// qp_part.cu -- plasma particle kernels on tile-binned structure-of-arrays.
//
// One CTA owns one 16 x 16 cell tile (the reference's tile, part2d_class.f03:99)
// and stages the 17 x 17 field nodes it interpolates from in shared memory.
// The particles of a tile are kept in cell order (k_push), so the deposits sum
// runs of same-cell particles in registers and add each run's corner sums to
// the zeroed global planes with L2 reductions (red.global.add.f32, native for
// FP32, where shared-memory float atomics are compare-and-swap loops).  The
// top edge of the top tile row is folded onto row 0 as it is added -- the
// single-rank guard add PPNACGUARD2L (ufield2d_lib.f03:90-97) done in-kernel.
// Per-particle arithmetic follows the reference routines line by line:
//   deposit_rho  PPGPPOST2L         part2d_lib77.f:194-309
//   extpsi       WPGPSIPOST2L_QP    part2d_lib77.f:2207-2284
//   amjdp        PPGRDCJPPOST2L_QP  part2d_lib77.f:311-768
//   push         PPGRBPPUSHF23L_QP  part2d_lib77.f:1066-1408
//   re-binning   PPPORDERF2LA/PPPORDER2LB part2d_lib77.f:1659-2028 (periodic
//                wrap at re-insertion, part2d_lib77.f:1936-1973)
// Every particle's cell is checked against its tile before it indexes shared
// memory or a plane; a particle outside its tile raises a status error instead.
#include "qp_part.cuh"

namespace qp {

namespace {

__device__ __forceinline__ void raise_error(DevStatus* st, int code) {
  if (st) atomicCAS(&st->error, 0, code);
}

__device__ __forceinline__ void tile_origin(const TileGeom& tg, int t, int* noffp, int* moffp) {
  const int ty = t / tg.mx1;
  *noffp = TILE * (t - tg.mx1 * ty);
  *moffp = TILE * ty;
}

// Stage the same 17 x 17 nodes of np planes (np <= NP; all kernels here run
// 256 threads): every thread issues all its loads from L2 before its first
// store to shared memory, so the planes cost one wait instead of one per load.
template <int NP>
__device__ __forceinline__ void stage_planes(float (*s)[TN * TN], const float* const (&pl)[NP],
                                             int np, const TileGeom& tg, int noffp, int moffp) {
  constexpr int PER = (TN * TN + 255) / 256;
  float v[NP][PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int i = threadIdx.x + 256 * k;
    const int a = i % TN, b = i / TN;
    const long long o = (long long)(moffp + b) * tg.rp + noffp + a;
#pragma unroll
    for (int p = 0; p < NP; ++p) v[p][k] = (i < TN * TN && p < np) ? pl[p][o] : 0.f;
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int i = threadIdx.x + 256 * k;
#pragma unroll
    for (int p = 0; p < NP; ++p)
      if (i < TN * TN && p < np) s[p][i] = v[p][k];
  }
}

// Add a run's 4 corner charges to the global plane q with L2 reductions
// (red.global.add.f32), folding the top edge of the top tile row onto row 0.
__device__ __forceinline__ void deposit_q(float* q, const TileGeom& tg, int noffp, int moffp,
                                          int cell, const float* acc) {
  const int nn = cell % TN, mm = cell / TN;
  const long long o0 = (long long)(moffp + mm) * tg.rp + noffp + nn;
  const int y1 = moffp + mm + 1;
  const long long o2 = (long long)(y1 == tg.ny ? 0 : y1) * tg.rp + noffp + nn;
  atomicAdd(q + o0, acc[0]);
  atomicAdd(q + o0 + 1, acc[1]);
  atomicAdd(q + o2, acc[2]);
  atomicAdd(q + o2 + 1, acc[3]);
}

// Charge deposit with the run scheme of k_amjdp: 4 consecutive particles per
// thread, corner weights of a run of particles in one cell summed in
// registers, then added to q (which must be zero on entry) by deposit_q.
// The n particles of tile t (all the CTA's threads take part).
__device__ __forceinline__ void deposit_tile(const PartBuf& P, const TileGeom& tg, int t, int n,
                                             float* q, DevStatus* st) {
  int noffp, moffp;
  tile_origin(tg, t, &noffp, &moffp);
  const long long base = (long long)t * P.cap;
  for (int k0 = 4 * threadIdx.x; k0 < n; k0 += 4 * blockDim.x) {
    const float4 X = *reinterpret_cast<const float4*>(P.c[0] + base + k0);
    const float4 Y = *reinterpret_cast<const float4*>(P.c[1] + base + k0);
    const float4 QM = *reinterpret_cast<const float4*>(P.c[7] + base + k0);
    const float xs[4] = {X.x, X.y, X.z, X.w}, ys[4] = {Y.x, Y.y, Y.z, Y.w};
    const float qs[4] = {QM.x, QM.y, QM.z, QM.w};
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    int cell = -1;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (k0 + j < n) {
        const float x = xs[j], y = ys[j], qm = qs[j];
        int nn = (int)x, mm = (int)y;
        const float dxp = qm * (x - (float)nn);
        const float dyp = y - (float)mm;
        nn -= noffp;
        mm -= moffp;
        if (nn < 0 || nn >= TILE || mm < 0 || mm >= TILE) {
          raise_error(st, -3);
          continue;
        }
        const float amx = qm - dxp, amy = 1.f - dyp;
        const float w0 = amx * amy, w1 = dxp * amy, w2 = amx * dyp, w3 = dxp * dyp;
        const int c = mm * TN + nn;
        if (c != cell) {
          if (cell >= 0) deposit_q(q, tg, noffp, moffp, cell, acc);
          cell = c;
          acc[0] = w0;
          acc[1] = w1;
          acc[2] = w2;
          acc[3] = w3;
        } else {
          acc[0] += w0;
          acc[1] += w1;
          acc[2] += w2;
          acc[3] += w3;
        }
      }
    }
    if (cell >= 0) deposit_q(q, tg, noffp, moffp, cell, acc);
  }
}

__global__ void __launch_bounds__(256) k_deposit_rho(PartBuf P, TileGeom tg, float* q,
                                                     DevStatus* st) {
  grid_dep_sync();
  if (st && st->error) return;
  const int t = blockIdx.x;
  const int n = P.count[t];
  if (n < 0 || n > P.cap) {  // a count beyond the tile's slots: never read past them
    if (threadIdx.x == 0) raise_error(st, -6);
    return;
  }
  deposit_tile(P, tg, t, n, q, st);
}

__global__ void __launch_bounds__(256) k_extpsi(PartBuf P, TileGeom tg, const float* psi,
                                                float qbm, float dex, DevStatus* st) {
  grid_dep_sync();
  __shared__ float sp[TN * TN];
  if (st && st->error) return;
  const int t = blockIdx.x;
  int noffp, moffp;
  tile_origin(tg, t, &noffp, &moffp);
  {
    const float* const planes[1] = {psi};
    stage_planes<1>(reinterpret_cast<float(*)[TN * TN]>(sp), planes, 1, tg, noffp, moffp);
  }
  __syncthreads();
  const float dx2 = dex * dex;
  const int n = P.count[t];
  if (n < 0 || n > P.cap) {  // a count beyond the tile's slots: never read past them
    if (threadIdx.x == 0) raise_error(st, -6);
    return;
  }
  const long long base = (long long)t * P.cap;
  for (int k0 = 4 * threadIdx.x; k0 < n; k0 += 4 * blockDim.x) {
    const float4 X = *reinterpret_cast<const float4*>(P.c[0] + base + k0);
    const float4 Y = *reinterpret_cast<const float4*>(P.c[1] + base + k0);
    const float4 VX = *reinterpret_cast<const float4*>(P.c[2] + base + k0);
    const float4 VY = *reinterpret_cast<const float4*>(P.c[3] + base + k0);
    float4 P6 = *reinterpret_cast<const float4*>(P.c[5] + base + k0);
    float4 P7 = *reinterpret_cast<const float4*>(P.c[6] + base + k0);
    const float xs[4] = {X.x, X.y, X.z, X.w}, ys[4] = {Y.x, Y.y, Y.z, Y.w};
    const float vxs[4] = {VX.x, VX.y, VX.z, VX.w}, vys[4] = {VY.x, VY.y, VY.z, VY.w};
    float p6[4] = {P6.x, P6.y, P6.z, P6.w}, p7[4] = {P7.x, P7.y, P7.z, P7.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (k0 + j < n) {
        const float x = xs[j], y = ys[j], vx = vxs[j], vy = vys[j];
        int nn = (int)x, mm = (int)y;
        const float dxp = x - (float)nn, dyp = y - (float)mm;
        nn -= noffp;
        mm -= moffp;
        if (nn < 0 || nn >= TILE || mm < 0 || mm >= TILE) {
          raise_error(st, -3);
          continue;
        }
        const float amx = 1.f - dxp, amy = 1.f - dyp;
        const float* s = sp + mm * TN + nn;
        float dx = amx * s[0];
        dx = amy * (dxp * s[1] + dx);
        const float acx = amx * s[TN];
        dx = dx + dyp * (dxp * s[TN + 1] + acx);
        dx = -dx * dx2 * qbm;
        p7[j] = 1.f + dx;
        p6[j] = dx + (dx2 * (vx * vx + vy * vy) - dx * dx - 2.f * dx) / (2.f * (1.f + dx)) + 1.f;
      }
    }
    *reinterpret_cast<float4*>(P.c[5] + base + k0) = make_float4(p6[0], p6[1], p6[2], p6[3]);
    *reinterpret_cast<float4*>(P.c[6] + base + k0) = make_float4(p7[0], p7[1], p7[2], p7[3]);
  }
}

// bilinear gather at (nn, mm) of a 17 x 17 staged plane, in the reference's order
__device__ __forceinline__ float gather(const float* s, int nn, int mm, float amx, float amy,
                                        float dxp, float dyp) {
  const float* p = s + mm * TN + nn;
  float d = amx * p[0];
  d = amy * (dxp * p[1] + d);
  const float ac = amx * p[TN];
  return d + dyp * (dxp * p[TN + 1] + ac);
}

// One particle of PPGRDCJPPOST2L_QP: the half push and the 8 deposited
// quantities (cu x/y/z, dcu x/y, amu xx/yy/xy) and 4 corner weights.
struct AmjOut {
  float v[8];
  float w[4];
  float p6;
};

__device__ __forceinline__ void amjdp_one(float (*sf)[TN * TN], int nn, int mm, float dxp,
                                          float dyp, float vx, float vy, float p6, float p7,
                                          float qm, float qbm, float qtmh, float dti, float dex,
                                          float idex, AmjOut* o) {
  float amx = 1.f - dxp;
  const float amy = 1.f - dyp;
  // __frcp_rn is the correctly rounded 1/x: the same bits as 1.f / x
  const float inv_part_7 = __frcp_rn(p7);
  const float qtmh1 = qtmh * inv_part_7;
  const float qtmh2 = qtmh1 * p6;
  float dx = gather(sf[0], nn, mm, amx, amy, dxp, dyp);
  float dy = gather(sf[1], nn, mm, amx, amy, dxp, dyp);
  float dz = gather(sf[5], nn, mm, amx, amy, dxp, dyp);
  float ox = gather(sf[2], nn, mm, amx, amy, dxp, dyp);
  float oy = gather(sf[3], nn, mm, amx, amy, dxp, dyp);
  float oz = gather(sf[4], nn, mm, amx, amy, dxp, dyp);
  const float ddx = -1.f * qtmh2 * dx + qtmh * oy;
  const float ddy = -1.f * qtmh2 * dy - qtmh * ox;
  const float acx = vx + ddx, acy = vy + ddy;
  const float omzt = qtmh1 * oz;
  const float omt = omzt * omzt;
  const float anorm = 2.f * __frcp_rn(1.f + omt);  // = 2.f / (1.f + omt): 2 x is exact
  const float rot1 = 0.5f * (1.f - omt);
  const float rot2 = omzt;
  float v1 = (rot1 * acx + rot2 * acy) * anorm + ddx;
  float v2 = (rot1 * acy - rot2 * acx) * anorm + ddy;
  const float qm1 = qm * inv_part_7;
  amx = qm1 * amx;
  dxp = qm1 * dxp;
  ox = 0.5f * (v1 + vx);
  oy = 0.5f * (v2 + vy);
  oz = 0.5f * (1.f + dex * dex * (ox * ox + oy * oy)) * inv_part_7 - 0.5f * p7;
  o->p6 = p7 + oz;
  oz = oz * idex;
  vx = (v1 - vx) * dti;
  vy = (v2 - vy) * dti;
  dz = qbm * (dz + (dx * ox + dy * oy) * dex * dex * inv_part_7);
  o->w[0] = amx * amy;
  o->w[1] = dxp * amy;
  o->w[2] = amx * dyp;
  o->w[3] = dxp * dyp;
  v1 = ox * ox * inv_part_7;
  v2 = oy * oy * inv_part_7;
  const float v3 = ox * oy * inv_part_7;
  vx = vx + ox * dz * inv_part_7;
  vy = vy + oy * dz * inv_part_7;
  o->v[0] = ox;
  o->v[1] = oy;
  o->v[2] = oz;
  o->v[3] = vx;
  o->v[4] = vy;
  o->v[5] = v1;
  o->v[6] = v2;
  o->v[7] = v3;
}

// Add a run's 8 x 4 corner sums to the global planes: fire-and-forget
// reductions in L2 (red.global.add.f32), native for FP32, where a
// shared-memory float atomic is a compare-and-swap loop.  The top edge of the
// top tile row folds onto row 0 (the single-rank guard add, PPNACGUARD2L).
__device__ __forceinline__ void deposit_run(float* const* pl, const TileGeom& tg, int noffp,
                                            int moffp, int cell, const float (*acc)[4]) {
  const int nn = cell % TN, mm = cell / TN;
  const long long o0 = (long long)(moffp + mm) * tg.rp + noffp + nn;
  const int y1 = moffp + mm + 1;
  const long long o2 = (long long)(y1 == tg.ny ? 0 : y1) * tg.rp + noffp + nn;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    atomicAdd(pl[q] + o0, acc[q][0]);
    atomicAdd(pl[q] + o0 + 1, acc[q][1]);
    atomicAdd(pl[q] + o2, acc[q][2]);
    atomicAdd(pl[q] + o2 + 1, acc[q][3]);
  }
}

// deposit_run for a lane's last run, merged across lanes: the right corners
// of the previous lane's last run are added to this run's left corners when
// take is set, and this run's right corners are left to the next lane when
// give is set.  Every lane of the warp must call it (the shuffles); a lane
// with no run (cell < 0) only passes values on.
__device__ __forceinline__ void deposit_last(float* const* pl, const TileGeom& tg, int noffp,
                                             int moffp, int cell, const float (*acc)[4],
                                             bool take, bool give) {
  const unsigned full = 0xffffffffu;
  const int c = cell < 0 ? 0 : cell;
  const int nn = c % TN, mm = c / TN;
  const long long o0 = (long long)(moffp + mm) * tg.rp + noffp + nn;
  const int y1 = moffp + mm + 1;
  const long long o2 = (long long)(y1 == tg.ny ? 0 : y1) * tg.rp + noffp + nn;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const float r1 = __shfl_up_sync(full, acc[q][1], 1);
    const float r3 = __shfl_up_sync(full, acc[q][3], 1);
    if (cell >= 0) {
      atomicAdd(pl[q] + o0, take ? acc[q][0] + r1 : acc[q][0]);
      atomicAdd(pl[q] + o2, take ? acc[q][2] + r3 : acc[q][2]);
      if (!give) {
        atomicAdd(pl[q] + o0 + 1, acc[q][1]);
        atomicAdd(pl[q] + o2 + 1, acc[q][3]);
      }
    }
  }
}

// Each thread takes 4 consecutive particles (float4 loads of each component)
// and keeps the deposits of a run of particles in one cell in registers,
// adding them to the global planes when the cell changes (deposit_run).  With
// the particles of a tile stored cell by cell, runs are long and a warp's
// reductions spread over neighbouring nodes.  The per-particle products are
// those of the reference; only the order in which a node's contributions are
// summed differs.  The planes must be zero on entry.
__global__ void __launch_bounds__(256, 3) k_amjdp(PartBuf P, TileGeom tg, GatherPlanes f,
                                               float* cux, float* cuy, float* cuz, float* dcx,
                                               float* dcy, float* amxx, float* amyy,
                                               float* amxy, float qbm, float dt, float dex,
                                               float scale, DevStatus* st) {
  grid_dep_sync();
  __shared__ float sf[7][TN * TN];
  if (st && st->error) return;
  if (pass_skipped(st, f.pass)) return;
  float* const pl[8] = {cux, cuy, cuz, dcx, dcy, amxx, amyy, amxy};
  const int t = blockIdx.x;
  int noffp, moffp;
  tile_origin(tg, t, &noffp, &moffp);
  const bool ext = f.psi != nullptr;
  // the count is read with the field planes, so the two waits overlap
  const int n = P.count[t];
  {
    const float* const planes[7] = {f.fx, f.fy, f.bx, f.by, f.bz, f.psit, f.psi};
    stage_planes<7>(sf, planes, ext ? 7 : 6, tg, noffp, moffp);
  }
  __syncthreads();
  const float qtmh = 0.5f * qbm * dt;
  const float dti = 1.f / dt;
  const float idex = 1.f / dex;
  const float dx2 = dex * dex;
  if (n < 0 || n > P.cap) {  // a count beyond the tile's slots: never read past them
    if (threadIdx.x == 0) raise_error(st, -6);
    return;
  }
  const long long base = (long long)t * P.cap;
  const int lane = threadIdx.x & 31;
  // the whole warp loops while one of its lanes has particles (the shuffles
  // of the last runs); a lane past the count reads the tile's first slots and
  // neither deposits nor writes them
  for (int k0 = 4 * threadIdx.x; k0 - 4 * lane < n; k0 += 4 * blockDim.x) {
    const bool live = k0 < n;
    const long long kb = base + (live ? k0 : 0);
    const float4 X = *reinterpret_cast<const float4*>(P.c[0] + kb);
    const float4 Y = *reinterpret_cast<const float4*>(P.c[1] + kb);
    const float4 VX = *reinterpret_cast<const float4*>(P.c[2] + kb);
    const float4 VY = *reinterpret_cast<const float4*>(P.c[3] + kb);
    // with ext, p6 and p7 are formed here from psi (k_extpsi) instead of read
    float4 P6 = make_float4(0.f, 0.f, 0.f, 0.f), P7 = P6;
    if (!ext) {
      P6 = *reinterpret_cast<const float4*>(P.c[5] + kb);
      P7 = *reinterpret_cast<const float4*>(P.c[6] + kb);
    }
    const float4 QM = *reinterpret_cast<const float4*>(P.c[7] + kb);
    const float xs[4] = {X.x, X.y, X.z, X.w}, ys[4] = {Y.x, Y.y, Y.z, Y.w};
    const float vxs[4] = {VX.x, VX.y, VX.z, VX.w}, vys[4] = {VY.x, VY.y, VY.z, VY.w};
    float p6s[4] = {P6.x, P6.y, P6.z, P6.w}, p7s[4] = {P7.x, P7.y, P7.z, P7.w};
    const float qms[4] = {QM.x, QM.y, QM.z, QM.w};
    float p6o[4] = {P6.x, P6.y, P6.z, P6.w};
    float acc[8][4];
    int cell = -1;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (k0 + j < n) {
        int nn = (int)xs[j], mm = (int)ys[j];
        const float dxp = xs[j] - (float)nn, dyp = ys[j] - (float)mm;
        nn -= noffp;
        mm -= moffp;
        if (nn < 0 || nn >= TILE || mm < 0 || mm >= TILE) {
          raise_error(st, -3);
          continue;
        }
        if (ext) {
          // WPGPSIPOST2L_QP for this particle, the same arithmetic as k_extpsi
          float d = gather(sf[6], nn, mm, 1.f - dxp, 1.f - dyp, dxp, dyp);
          d = -d * dx2 * qbm;
          p7s[j] = 1.f + d;
          p6s[j] = d + (dx2 * (vxs[j] * vxs[j] + vys[j] * vys[j]) - d * d - 2.f * d) /
                           (2.f * (1.f + d)) +
                   1.f;
        }
        AmjOut o;
        amjdp_one(sf, nn, mm, dxp, dyp, vxs[j], vys[j], p6s[j], p7s[j], qms[j], qbm, qtmh, dti,
                  dex, idex, &o);
        p6o[j] = o.p6;
        // the moments only feed the deposit: the scale goes on the corner
        // weights and the run sums use fused multiply-adds (FP32 roundoff of
        // the sums, like the order of the reductions)
        float ws[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) ws[r] = o.w[r] * scale;
        const int c = mm * TN + nn;
        if (c != cell) {
          if (cell >= 0) deposit_run(pl, tg, noffp, moffp, cell, acc);
          cell = c;
#pragma unroll
          for (int q = 0; q < 8; ++q)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[q][r] = o.v[q] * ws[r];
        } else {
#pragma unroll
          for (int q = 0; q < 8; ++q)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[q][r] = __fmaf_rn(o.v[q], ws[r], acc[q][r]);
        }
      }
    }
    // the last run's right corners go to the next lane when its last run is
    // in the next cell in x (cell + 1 is never a cell at a tile row's end)
    const unsigned full = 0xffffffffu;
    int cprev = __shfl_up_sync(full, cell, 1);
    int cnext = __shfl_down_sync(full, cell, 1);
    if (lane == 0) cprev = -1;
    if (lane == 31) cnext = -1;
    deposit_last(pl, tg, noffp, moffp, cell, acc, cprev >= 0 && cell == cprev + 1,
                 cell >= 0 && cnext == cell + 1);
    if (live) {
      P6 = make_float4(p6o[0], p6o[1], p6o[2], p6o[3]);
      *reinterpret_cast<float4*>(P.c[5] + base + k0) = P6;
      if (ext)
        *reinterpret_cast<float4*>(P.c[6] + base + k0) =
            make_float4(p7s[0], p7s[1], p7s[2], p7s[3]);
    }
  }
}

// Push (mode 0, 1) and/or re-bin (mode 1, 2).  Mode 0 writes the pushed
// particles back in place.  In modes 1 and 2 the particles that stay are
// written to B's tile sorted by cell: the tile is taken in chunks of 1024
// slots, the stayers of a chunk are held in shared memory and written out in
// the order of a stable counting sort on their cell, so that the deposits see
// runs of same-cell particles (k_deposit_rho, k_amjdp).  Warp w takes the
// slots w * 128 .. w * 128 + 127 of a chunk, 32 per round, so a particle's
// rank among the earlier same-cell stayers needs only its own warp's running
// counts, and the chunk needs four CTA barriers.  Movers go to the
// destination tile's inbox with a (cell, source tile, source slot) key, which
// the insert kernel sorts, so they too arrive in cell order.
constexpr int PUSH_CHUNK = 1024;

template <int MODE>
__global__ void __launch_bounds__(256) k_push(PartBuf A, PartBuf B, Inbox ib, TileGeom tg,
                                              GatherPlanes f, float qbm, float dt, float dex,
                                              DevStatus* st) {
  grid_dep_sync();
  constexpr int CH = MODE != 0 ? PUSH_CHUNK : 1;
  constexpr int NC = MODE != 0 ? 256 : 1;
  constexpr int NR = MODE != 0 ? CH / 256 : 1;  // rounds of 256 slots per chunk
  __shared__ float sf[6][TN * TN];
  __shared__ float stg[NCOMP][CH];      // the chunk's stayers, by chunk slot
  __shared__ short perm[CH];            // output order -> chunk slot
  __shared__ unsigned char wcnt[8][NC];  // per warp: its stayers of each cell so far
  __shared__ short woff[8][NC];         // per warp: first output position of each cell
  __shared__ int wtot[8];
  if (st && st->error) return;
  const int t = blockIdx.x;
  int noffp, moffp;
  tile_origin(tg, t, &noffp, &moffp);
  const int n = A.count[t];  // read with the field planes: the waits overlap
  if (f.zero_q) {
    // the tile's 16 x 16 nodes of the charge plane, and on the last tile
    // column / row the rest of the row pitch / the guard row: every node of
    // the plane is cleared by exactly one tile
    const int x1 = (noffp + TILE >= tg.nx) ? tg.rp : noffp + TILE;
    const int y1 = (moffp + TILE >= tg.ny) ? tg.ny + 1 : moffp + TILE;
    const int w = x1 - noffp, h = y1 - moffp;
    for (int i = threadIdx.x; i < w * h; i += blockDim.x)
      f.zero_q[(long long)(moffp + i / w) * tg.rp + noffp + i % w] = 0.f;
  }
  if (MODE != 2) {
    const float* const planes[6] = {f.fx, f.fy, f.bx, f.by, f.bz, f.psit};
    stage_planes<6>(sf, planes, 6, tg, noffp, moffp);
    __syncthreads();
    if (f.combine) {
      // the slice's final force: fxy = -fxy + (bxyz(2), -bxyz(1)), simulation_class.f03:722-724
      for (int i = threadIdx.x; i < TN * TN; i += blockDim.x) {
        const float fx = -1.f * sf[0][i], fy = -1.f * sf[1][i];
        sf[0][i] = fx + sf[3][i];
        sf[1][i] = fy - sf[2][i];
      }
    }
  }
  if (MODE != 0)
    for (int i = threadIdx.x; i < 8 * NC; i += blockDim.x) (&wcnt[0][0])[i] = 0;
  __syncthreads();
  const float idex = 1.f / dex;
  const float qtmh = 0.5f * qbm * dt;
  const float anx = (float)tg.nx, any = (float)tg.ny;
  const float edgelx = (float)noffp, edgerx = (float)(noffp + TILE);
  const float edgely = (float)moffp, edgery = (float)(moffp + TILE);
  if (n < 0 || n > A.cap) {  // a count beyond the tile's slots: never read past them
    if (threadIdx.x == 0) raise_error(st, -6);
    return;
  }
  const long long base = (long long)t * A.cap;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  int written = 0;  // stayers written to B so far (the same in every thread)
  for (int c0 = 0; c0 < n; c0 += (MODE != 0 ? CH : (int)blockDim.x)) {
    int cellr[NR];
    // with re-binning the kernel never writes A: its particles are read with
    // read-only loads, and each round's are requested one round ahead, so
    // the wait for L2 overlaps the previous round's push
    float pn[NCOMP];
    {
      const int k = c0 + (MODE != 0 ? warp * (CH / 8) + lane : (int)threadIdx.x);
      if (MODE != 0 && k < n) {
#pragma unroll
        for (int c = 0; c < NCOMP; ++c) pn[c] = __ldg(A.c[c] + base + k);
      }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const int slot = MODE != 0 ? warp * (CH / 8) + r * 32 + lane : threadIdx.x;
      const int k = c0 + slot;
      cellr[r] = -1;
      float pc[NCOMP];
      if (MODE != 0) {
#pragma unroll
        for (int c = 0; c < NCOMP; ++c) pc[c] = pn[c];
        const int kn = k + 32;  // the next round's slot
        if (r + 1 < NR && kn < n) {
#pragma unroll
          for (int c = 0; c < NCOMP; ++c) pn[c] = __ldg(A.c[c] + base + kn);
        }
      }
      if (k >= n) continue;
      if (MODE == 0) {
#pragma unroll
        for (int c = 0; c < NCOMP; ++c) pc[c] = A.c[c][base + k];
      }
      if (MODE != 2) {
        const float x = pc[0], y = pc[1];
        int nn = (int)x, mm = (int)y;
        const float p6 = pc[5], p7 = pc[6];
        const float qtmh1 = qtmh / p7;
        const float qtmh2 = qtmh1 * p6;
        const float dxp = x - (float)nn, dyp = y - (float)mm;
        nn -= noffp;
        mm -= moffp;
        if (nn < 0 || nn >= TILE || mm < 0 || mm >= TILE) {
          raise_error(st, -3);
          nn = 0;
          mm = 0;
        }
        const float amx = 1.f - dxp, amy = 1.f - dyp;
        float dx = gather(sf[0], nn, mm, amx, amy, dxp, dyp);
        float dy = gather(sf[1], nn, mm, amx, amy, dxp, dyp);
        float dz = gather(sf[5], nn, mm, amx, amy, dxp, dyp);
        dz = dz * idex;
        float ox = gather(sf[2], nn, mm, amx, amy, dxp, dyp);
        float oy = gather(sf[3], nn, mm, amx, amy, dxp, dyp);
        const float oz = gather(sf[4], nn, mm, amx, amy, dxp, dyp);
        ox = ox * dex;
        oy = oy * dex;
        dx = qtmh2 * dx;
        dy = qtmh2 * dy;
        dz = qtmh2 * dz;
        const float acx = pc[2] + dx, acy = pc[3] + dy, acz = pc[4] + dz;
        const float omxt = qtmh1 * ox, omyt = qtmh1 * oy, omzt = qtmh1 * oz;
        float omt = omxt * omxt + omyt * omyt + omzt * omzt;
        const float anorm = 2.f * __frcp_rn(1.f + omt);  // = 2.f / (1.f + omt)
        omt = 0.5f * (1.f - omt);
        float rot4 = omxt * omyt, rot7 = omxt * omzt, rot8 = omyt * omzt;
        const float rot1 = omt + omxt * omxt, rot5 = omt + omyt * omyt, rot9 = omt + omzt * omzt;
        const float rot2 = omzt + rot4;
        rot4 = -omzt + rot4;
        const float rot3 = -omyt + rot7;
        rot7 = omyt + rot7;
        const float rot6 = omxt + rot8;
        rot8 = -omxt + rot8;
        dx = (rot1 * acx + rot2 * acy + rot3 * acz) * anorm + dx;
        dy = (rot4 * acx + rot5 * acy + rot6 * acz) * anorm + dy;
        dz = (rot7 * acx + rot8 * acy + rot9 * acz) * anorm + dz;
        pc[2] = dx;
        pc[3] = dy;
        pc[4] = dz;
        const float dtc1 = dt / (sqrtf(1.f + (dx * dx + dy * dy + dz * dz) * dex * dex) - dz * dex);
        dx = x + dx * dtc1;
        dy = y + dy * dtc1;
        pc[0] = dx;
        pc[1] = dy;
        // the push's own boundary handling (part2d_lib77.f:1350-1378)
        if (!(dx >= edgerx) && dx < edgelx && dx < 0.f) {
          if (dx + anx >= anx) pc[0] = 0.f;
        }
        if (!(dy >= edgery) && dy < edgely && dy < 0.f) {
          if (dy + any >= any) pc[1] = 0.f;
        }
      }
      if (MODE == 0) {
#pragma unroll
        for (int c = 0; c < 5; ++c) A.c[c][base + k] = pc[c];
        continue;
      }
      // re-insertion wrap of PPPORDER2LB (part2d_lib77.f:1936-1973)
      float xw = pc[0], yw = pc[1];
      if (xw < 0.f) xw = xw + anx;
      if (xw >= anx) xw = xw - anx;
      if (yw < 0.f) yw = yw + any;
      if (yw >= any) yw = yw - any;
      pc[0] = xw;
      pc[1] = yw;
      const int ix = (int)xw, iy = (int)yw;
      int tx = ix / TILE, ty = iy / TILE;
      if (tx < 0 || tx >= tg.mx1 || ty < 0 || ty >= tg.myp1 || !(xw == xw) || !(yw == yw)) {
        raise_error(st, -4);
        tx = 0;
        ty = 0;
      }
      const int dest = tx + tg.mx1 * ty;
      const int cell = (iy & (TILE - 1)) * TILE + (ix & (TILE - 1));
      if (dest == t) {
        cellr[r] = cell;
#pragma unroll
        for (int c = 0; c < NCOMP; ++c) stg[c][slot] = pc[c];
      } else {
        const int islot = atomicAdd(&ib.count[dest], 1);
        if (islot < ib.cap) {
          const long long o = (long long)dest * ib.cap + islot;
#pragma unroll
          for (int c = 0; c < NCOMP; ++c) ib.c[c][o] = pc[c];
          ib.key[o] = ((unsigned long long)cell << 48) | ((unsigned long long)t << 24) |
                      (unsigned long long)(k & 0xffffff);
        } else {
          raise_error(st, QP_OVERFLOW);
          atomicMax(&st->need_inbox, islot + 1);
        }
      }
    }
    if constexpr (MODE != 0) {
      // rank of each stayer among the same-cell stayers of lower slots in its
      // warp: the warp's running count of the cell plus the lower lanes of this
      // round that share the cell (warp-local, so __syncwarp suffices)
      int rank[NR];
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const int cl = cellr[r];
        const unsigned same = __match_any_sync(0xffffffffu, cl >= 0 ? cl : 256 + lane);
        rank[r] = cl >= 0 ? wcnt[warp][cl] + __popc(same & lt) : 0;
        __syncwarp();
        if (cl >= 0 && lane == __ffs(same) - 1) wcnt[warp][cl] += (unsigned char)__popc(same);
        __syncwarp();
      }
      __syncthreads();
      // thread c: the chunk's stayers of cell c, an exclusive scan over the cells,
      // and the first position of each warp's stayers of cell c
      int nst;
      {
        const int c = threadIdx.x;
        int v = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) v += wcnt[w][c];
        int inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int u = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= o) inc += u;
        }
        if (lane == 31) wtot[warp] = inc;
        __syncthreads();
        int off = 0;
        nst = 0;
        for (int w = 0; w < 8; ++w) {
          if (w < warp) off += wtot[w];
          nst += wtot[w];
        }
        int pos = off + inc - v;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
          woff[w][c] = (short)pos;
          pos += wcnt[w][c];
          wcnt[w][c] = 0;  // ready for the next chunk (read again only after a barrier)
        }
      }
      __syncthreads();
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const int cl = cellr[r];
        if (cl >= 0) {
          const int pos = woff[warp][cl] + rank[r];
          if (pos >= 0 && pos < CH)
            perm[pos] = (short)(warp * (CH / 8) + r * 32 + lane);
          else
            raise_error(st, -8);
        }
      }
      __syncthreads();
      // write the chunk's stayers in cell order
      for (int j = threadIdx.x; j < nst; j += blockDim.x) {
        const int slot = perm[j];
        const int pos = written + j;
        if (slot < 0 || slot >= CH) {
          raise_error(st, -8);
        } else if (pos < B.cap) {
          const long long o = (long long)t * B.cap + pos;
#pragma unroll
          for (int c = 0; c < NCOMP; ++c) B.c[c][o] = stg[c][slot];
        } else {
          raise_error(st, QP_OVERFLOW);
          atomicMax(&st->need_cap, pos + 1);
        }
      }
      written += nst;
      __syncthreads();
    }
  }
  if (MODE != 0 && threadIdx.x == 0) B.count[t] = written;
}

// Insert the movers of tile t after its stayers, sorted by their key so that
// the particle order does not depend on the order in which the atomics of the
// push handed out inbox slots.
__global__ void __launch_bounds__(256) k_insert(PartBuf B, Inbox ib, TileGeom tg, int p2max,
                                                DevStatus* st, float* dq) {
  grid_dep_sync();
  extern __shared__ unsigned long long skey[];
  int* sidx = reinterpret_cast<int*>(skey + p2max);
  if (st && st->error) return;
  const int t = blockIdx.x;
  int nin = ib.count[t];
  if (nin > ib.cap) {
    raise_error(st, QP_OVERFLOW);
    atomicMax(&st->need_inbox, nin);
    return;
  }
  const int stay = B.count[t];
  if (stay < 0 || stay > B.cap) {
    if (threadIdx.x == 0) raise_error(st, -6);
    return;
  }
  if (stay + nin > B.cap) {
    raise_error(st, QP_OVERFLOW);
    atomicMax(&st->need_cap, stay + nin);
    return;
  }
  int p2 = 1;
  while (p2 < nin) p2 <<= 1;
  const long long ib0 = (long long)t * ib.cap;
  for (int i = threadIdx.x; i < p2; i += blockDim.x) {
    skey[i] = (i < nin) ? ib.key[ib0 + i] : ~0ull;
    sidx[i] = i;
  }
  __syncthreads();
  for (int k = 2; k <= p2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < p2; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const bool up = (i & k) == 0;
          const unsigned long long a = skey[i], b = skey[ixj];
          if ((a > b) == up) {
            skey[i] = b;
            skey[ixj] = a;
            const int ti = sidx[i];
            sidx[i] = sidx[ixj];
            sidx[ixj] = ti;
          }
        }
      }
      __syncthreads();
    }
  }
  const long long ob = (long long)t * B.cap + stay;
  for (int i = threadIdx.x; i < nin; i += blockDim.x) {
    const int si = sidx[i];
    if (si < 0 || si >= nin) {  // the sort must map the first nin keys onto filled slots
      raise_error(st, -8);
      continue;
    }
    const long long src = ib0 + si;
    // all loads before the stores, so the mover waits for L2 once
    float v[NCOMP];
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) v[c] = ib.c[c][src];
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) B.c[c][ob + i] = v[c];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    B.count[t] = stay + nin;
    ib.count[t] = 0;
  }
  // the next slice's charge: every particle of the re-binned tile (the
  // movers were written above; the barrier makes them visible to the CTA)
  if (dq) deposit_tile(B, tg, t, stay + nin, dq, st);
}

}  // namespace

int part_kernels_init() {
  const int big = 16384 * (int)(sizeof(unsigned long long) + sizeof(int));
  if (cudaFuncSetAttribute(k_insert, cudaFuncAttributeMaxDynamicSharedMemorySize, big) !=
      cudaSuccess)
    return -2;
  return 0;
}

void launch_insert(const PartBuf& B, const Inbox& ib, const TileGeom& tg, DevStatus* st,
                   cudaStream_t s, float* deposit_q) {
  int p2 = 1;
  while (p2 < ib.cap) p2 <<= 1;
  const size_t smem = (size_t)p2 * (sizeof(unsigned long long) + sizeof(int));
  launch_pdl(k_insert, tg.ntiles, 256, smem, s, B, ib, tg, p2, st, deposit_q);
}

void launch_deposit_rho(const PartBuf& P, const TileGeom& tg, float* q, const DevStatus* st,
                        cudaStream_t s) {
  launch_pdl(k_deposit_rho, tg.ntiles, 256, 0, s, P, tg, q, const_cast<DevStatus*>(st));
}

void launch_extpsi(const PartBuf& P, const TileGeom& tg, const float* psi, float qbm, float dex,
                   const DevStatus* st, cudaStream_t s) {
  launch_pdl(k_extpsi, tg.ntiles, 256, 0, s, P, tg, psi, qbm, dex, const_cast<DevStatus*>(st));
}

void launch_amjdp(const PartBuf& P, const TileGeom& tg, const GatherPlanes& f, float* const* acc,
                  float qbm, float dt, float dex, float scale, const DevStatus* st,
                  cudaStream_t s) {
  launch_pdl(k_amjdp, tg.ntiles, 256, 0, s, P, tg, f, acc[0], acc[1], acc[2], acc[3], acc[4],
             acc[5], acc[6], acc[7], qbm, dt, dex, scale, const_cast<DevStatus*>(st));
}

void launch_push(int mode, const PartBuf& A, const PartBuf& B, const Inbox& ib,
                 const TileGeom& tg, const GatherPlanes& f, float qbm, float dt, float dex,
                 DevStatus* st, cudaStream_t s) {
  if (mode == 0)
    launch_pdl(k_push<0>, tg.ntiles, 256, 0, s, A, B, ib, tg, f, qbm, dt, dex, st);
  else if (mode == 1)
    launch_pdl(k_push<1>, tg.ntiles, 256, 0, s, A, B, ib, tg, f, qbm, dt, dex, st);
  else
    launch_pdl(k_push<2>, tg.ntiles, 256, 0, s, A, B, ib, tg, f, qbm, dt, dex, st);
}

}  // namespace qp
