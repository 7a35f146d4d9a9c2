// qp_part.cu -- plasma particle kernels on tile-binned structure-of-arrays.
//
// One CTA owns one 16 x 16 cell tile (the reference's tile, part2d_class.f03:99):
// it stages the 17 x 17 field nodes it interpolates from in shared memory,
// accumulates deposits in shared memory, and flushes them to the global
// planes once: nodes strictly inside the tile are written with plain stores
// (no other tile touches them), shared edge nodes with atomics, and the top
// edge of the top tile row is folded onto row 0 in the same flush -- the
// single-rank guard add PPNACGUARD2L (ufield2d_lib.f03:90-97) done in-kernel.
// Per-particle arithmetic follows the reference routines line by line:
//   deposit_rho  PPGPPOST2L         part2d_lib77.f:194-309
//   extpsi       WPGPSIPOST2L_QP    part2d_lib77.f:2207-2284
//   amjdp        PPGRDCJPPOST2L_QP  part2d_lib77.f:311-768
//   push         PPGRBPPUSHF23L_QP  part2d_lib77.f:1066-1408
//   re-binning   PPPORDERF2LA/PPPORDER2LB part2d_lib77.f:1659-2028 (periodic
//                wrap at re-insertion, part2d_lib77.f:1936-1973)
// Every particle's cell is checked against its tile before shared memory is
// indexed; a particle outside its tile raises a status error instead.
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

// stage nodes [noffp, noffp+16] x [moffp, moffp+16] of a plane
__device__ __forceinline__ void stage(float* s, const float* plane, const TileGeom& tg, int noffp,
                                      int moffp) {
  for (int i = threadIdx.x; i < TN * TN; i += blockDim.x) {
    const int a = i % TN, b = i / TN;
    s[i] = plane[(long long)(moffp + b) * tg.rp + noffp + a];
  }
}

// flush a tile accumulator to a zeroed global plane (see file comment)
__device__ __forceinline__ void flush(const float* s, float* plane, const TileGeom& tg, int noffp,
                                      int moffp, float scale) {
  for (int i = threadIdx.x; i < TN * TN; i += blockDim.x) {
    const int a = i % TN, b = i / TN;
    int gy = moffp + b;
    const int gx = noffp + a;
    if (gy == tg.ny) gy = 0;
    const float v = s[i] * scale;
    float* dst = plane + (long long)gy * tg.rp + gx;
    if (a > 0 && a < TILE && b > 0 && b < TILE)
      *dst = v;
    else
      atomicAdd(dst, v);
  }
}

__global__ void __launch_bounds__(256) k_deposit_rho(PartBuf P, TileGeom tg, float* q,
                                                     DevStatus* st) {
  __shared__ float sq[TN * TN];
  if (st && st->error) return;
  const int t = blockIdx.x;
  for (int i = threadIdx.x; i < TN * TN; i += blockDim.x) sq[i] = 0.f;
  int noffp, moffp;
  tile_origin(tg, t, &noffp, &moffp);
  __syncthreads();
  const int n = P.count[t];
  const long long base = (long long)t * P.cap;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const float x = P.c[0][base + k], y = P.c[1][base + k], qm = P.c[7][base + k];
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
    float* s = sq + mm * TN + nn;
    atomicAdd(s, amx * amy);
    atomicAdd(s + 1, dxp * amy);
    atomicAdd(s + TN, amx * dyp);
    atomicAdd(s + TN + 1, dxp * dyp);
  }
  __syncthreads();
  flush(sq, q, tg, noffp, moffp, 1.f);
}

__global__ void __launch_bounds__(256) k_extpsi(PartBuf P, TileGeom tg, const float* psi,
                                                float qbm, float dex, DevStatus* st) {
  __shared__ float sp[TN * TN];
  if (st && st->error) return;
  const int t = blockIdx.x;
  int noffp, moffp;
  tile_origin(tg, t, &noffp, &moffp);
  stage(sp, psi, tg, noffp, moffp);
  __syncthreads();
  const float dx2 = dex * dex;
  const int n = P.count[t];
  const long long base = (long long)t * P.cap;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const float x = P.c[0][base + k], y = P.c[1][base + k];
    const float vx = P.c[2][base + k], vy = P.c[3][base + k];
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
    P.c[6][base + k] = 1.f + dx;
    P.c[5][base + k] =
        dx + (dx2 * (vx * vx + vy * vy) - dx * dx - 2.f * dx) / (2.f * (1.f + dx)) + 1.f;
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

__global__ void __launch_bounds__(256) k_amjdp(PartBuf P, TileGeom tg, GatherPlanes f,
                                               float* cux, float* cuy, float* cuz, float* dcx,
                                               float* dcy, float* amxx, float* amyy,
                                               float* amxy, float qbm, float dt, float dex,
                                               float scale, DevStatus* st) {
  __shared__ float sf[6][TN * TN];
  __shared__ float sa[8][TN * TN];
  if (st && st->error) return;
  const int t = blockIdx.x;
  int noffp, moffp;
  tile_origin(tg, t, &noffp, &moffp);
  stage(sf[0], f.fx, tg, noffp, moffp);
  stage(sf[1], f.fy, tg, noffp, moffp);
  stage(sf[2], f.bx, tg, noffp, moffp);
  stage(sf[3], f.by, tg, noffp, moffp);
  stage(sf[4], f.bz, tg, noffp, moffp);
  stage(sf[5], f.psit, tg, noffp, moffp);
  for (int i = threadIdx.x; i < 8 * TN * TN; i += blockDim.x) (&sa[0][0])[i] = 0.f;
  __syncthreads();
  const float qtmh = 0.5f * qbm * dt;
  const float dti = 1.f / dt;
  const float idex = 1.f / dex;
  const int n = P.count[t];
  const long long base = (long long)t * P.cap;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const float x = P.c[0][base + k], y = P.c[1][base + k];
    const float p6 = P.c[5][base + k], p7 = P.c[6][base + k], qm = P.c[7][base + k];
    int nn = (int)x, mm = (int)y;
    float dxp = x - (float)nn, dyp = y - (float)mm;
    nn -= noffp;
    mm -= moffp;
    if (nn < 0 || nn >= TILE || mm < 0 || mm >= TILE) {
      raise_error(st, -3);
      continue;
    }
    float amx = 1.f - dxp;
    const float amy = 1.f - dyp;
    const float inv_part_7 = 1.f / p7;
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
    float vx = P.c[2][base + k], vy = P.c[3][base + k];
    const float acx = vx + ddx, acy = vy + ddy;
    const float omzt = qtmh1 * oz;
    const float omt = omzt * omzt;
    const float anorm = 2.f / (1.f + omt);
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
    P.c[5][base + k] = p7 + oz;
    oz = oz * idex;
    vx = (v1 - vx) * dti;
    vy = (v2 - vy) * dti;
    dz = qbm * (dz + (dx * ox + dy * oy) * dex * dex * inv_part_7);
    const float w00 = amx * amy, w10 = dxp * amy, w01 = amx * dyp, w11 = dxp * dyp;
    v1 = ox * ox * inv_part_7;
    v2 = oy * oy * inv_part_7;
    const float v3 = ox * oy * inv_part_7;
    vx = vx + ox * dz * inv_part_7;
    vy = vy + oy * dz * inv_part_7;
    const int o = mm * TN + nn;
    const int off[4] = {o, o + 1, o + TN, o + TN + 1};
    const float w[4] = {w00, w10, w01, w11};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      atomicAdd(&sa[0][off[c]], ox * w[c]);
      atomicAdd(&sa[1][off[c]], oy * w[c]);
      atomicAdd(&sa[2][off[c]], oz * w[c]);
      atomicAdd(&sa[3][off[c]], vx * w[c]);
      atomicAdd(&sa[4][off[c]], vy * w[c]);
      atomicAdd(&sa[5][off[c]], v1 * w[c]);
      atomicAdd(&sa[6][off[c]], v2 * w[c]);
      atomicAdd(&sa[7][off[c]], v3 * w[c]);
    }
  }
  __syncthreads();
  flush(sa[0], cux, tg, noffp, moffp, scale);
  flush(sa[1], cuy, tg, noffp, moffp, scale);
  flush(sa[2], cuz, tg, noffp, moffp, scale);
  flush(sa[3], dcx, tg, noffp, moffp, scale);
  flush(sa[4], dcy, tg, noffp, moffp, scale);
  flush(sa[5], amxx, tg, noffp, moffp, scale);
  flush(sa[6], amyy, tg, noffp, moffp, scale);
  flush(sa[7], amxy, tg, noffp, moffp, scale);
}

// Push (mode 0, 1) and/or re-bin (mode 1, 2).  In modes 1 and 2 particles that
// stay are compacted, in order, into B's tile; movers go to the destination
// tile's inbox with a (source tile, source slot) key.
template <int MODE>
__global__ void __launch_bounds__(256) k_push(PartBuf A, PartBuf B, Inbox ib, TileGeom tg,
                                              GatherPlanes f, float qbm, float dt, float dex,
                                              DevStatus* st) {
  __shared__ float sf[6][TN * TN];
  __shared__ int wsum[8];
  __shared__ int sbase;
  if (st && st->error) return;
  const int t = blockIdx.x;
  int noffp, moffp;
  tile_origin(tg, t, &noffp, &moffp);
  if (MODE != 2) {
    stage(sf[0], f.fx, tg, noffp, moffp);
    stage(sf[1], f.fy, tg, noffp, moffp);
    stage(sf[2], f.bx, tg, noffp, moffp);
    stage(sf[3], f.by, tg, noffp, moffp);
    stage(sf[4], f.bz, tg, noffp, moffp);
    stage(sf[5], f.psit, tg, noffp, moffp);
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
  if (threadIdx.x == 0) sbase = 0;
  __syncthreads();
  const float idex = 1.f / dex;
  const float qtmh = 0.5f * qbm * dt;
  const float anx = (float)tg.nx, any = (float)tg.ny;
  const float edgelx = (float)noffp, edgerx = (float)(noffp + TILE);
  const float edgely = (float)moffp, edgery = (float)(moffp + TILE);
  const int n = A.count[t];
  const long long base = (long long)t * A.cap;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r0 = 0; r0 < n; r0 += blockDim.x) {
    const int k = r0 + threadIdx.x;
    const bool live = k < n;
    float pc[NCOMP];
    int dest = t;
    if (live) {
#pragma unroll
      for (int c = 0; c < NCOMP; ++c) pc[c] = A.c[c][base + k];
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
        const float anorm = 2.f / (1.f + omt);
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
      if (MODE != 0) {
        // re-insertion wrap of PPPORDER2LB (part2d_lib77.f:1936-1973)
        float xw = pc[0], yw = pc[1];
        if (xw < 0.f) xw = xw + anx;
        if (xw >= anx) xw = xw - anx;
        if (yw < 0.f) yw = yw + any;
        if (yw >= any) yw = yw - any;
        pc[0] = xw;
        pc[1] = yw;
        int tx = (int)xw / TILE, ty = (int)yw / TILE;
        if (tx < 0 || tx >= tg.mx1 || ty < 0 || ty >= tg.myp1 || !(xw == xw) || !(yw == yw)) {
          raise_error(st, -4);
          tx = 0;
          ty = 0;
        }
        dest = tx + tg.mx1 * ty;
      } else {
#pragma unroll
        for (int c = 0; c < 5; ++c) A.c[c][base + k] = pc[c];
      }
    }
    if (MODE != 0) {
      const bool stay = live && dest == t;
      const unsigned bal = __ballot_sync(0xffffffffu, stay);
      if (lane == 0) wsum[warp] = __popc(bal);
      __syncthreads();
      int woff = 0;
      for (int w = 0; w < warp; ++w) woff += wsum[w];
      const int pos = sbase + woff + __popc(bal & ((1u << lane) - 1u));
      if (stay) {
        if (pos < B.cap) {
          const long long o = (long long)t * B.cap + pos;
#pragma unroll
          for (int c = 0; c < NCOMP; ++c) B.c[c][o] = pc[c];
        } else {
          raise_error(st, QP_OVERFLOW);
          atomicMax(&st->need_cap, pos + 1);
        }
      } else if (live) {
        const int slot = atomicAdd(&ib.count[dest], 1);
        if (slot < ib.cap) {
          const long long o = (long long)dest * ib.cap + slot;
#pragma unroll
          for (int c = 0; c < NCOMP; ++c) ib.c[c][o] = pc[c];
          ib.key[o] = ((unsigned long long)t << 32) | (unsigned)k;
        } else {
          raise_error(st, QP_OVERFLOW);
          atomicMax(&st->need_inbox, slot + 1);
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < 8; ++w) tot += wsum[w];
        sbase += tot;
      }
      __syncthreads();
    }
  }
  if (MODE != 0 && threadIdx.x == 0) B.count[t] = sbase;
}

// Insert the movers of tile t after its stayers, sorted by their
// (source tile, source slot) key so the particle order does not depend on the
// order in which the atomics of the push handed out inbox slots.
__global__ void __launch_bounds__(256) k_insert(PartBuf B, Inbox ib, TileGeom tg, int p2max,
                                                DevStatus* st) {
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
    const long long src = ib0 + sidx[i];
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) B.c[c][ob + i] = ib.c[c][src];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    B.count[t] = stay + nin;
    ib.count[t] = 0;
  }
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
                   cudaStream_t s) {
  int p2 = 1;
  while (p2 < ib.cap) p2 <<= 1;
  const size_t smem = (size_t)p2 * (sizeof(unsigned long long) + sizeof(int));
  k_insert<<<tg.ntiles, 256, smem, s>>>(B, ib, tg, p2, st);
}

void launch_deposit_rho(const PartBuf& P, const TileGeom& tg, float* q, const DevStatus* st,
                        cudaStream_t s) {
  k_deposit_rho<<<tg.ntiles, 256, 0, s>>>(P, tg, q, const_cast<DevStatus*>(st));
}

void launch_extpsi(const PartBuf& P, const TileGeom& tg, const float* psi, float qbm, float dex,
                   const DevStatus* st, cudaStream_t s) {
  k_extpsi<<<tg.ntiles, 256, 0, s>>>(P, tg, psi, qbm, dex, const_cast<DevStatus*>(st));
}

void launch_amjdp(const PartBuf& P, const TileGeom& tg, const GatherPlanes& f, float* const* acc,
                  float qbm, float dt, float dex, float scale, const DevStatus* st,
                  cudaStream_t s) {
  k_amjdp<<<tg.ntiles, 256, 0, s>>>(P, tg, f, acc[0], acc[1], acc[2], acc[3], acc[4], acc[5],
                                    acc[6], acc[7], qbm, dt, dex, scale,
                                    const_cast<DevStatus*>(st));
}

void launch_push(int mode, const PartBuf& A, const PartBuf& B, const Inbox& ib,
                 const TileGeom& tg, const GatherPlanes& f, float qbm, float dt, float dex,
                 DevStatus* st, cudaStream_t s) {
  if (mode == 0)
    k_push<0><<<tg.ntiles, 256, 0, s>>>(A, B, ib, tg, f, qbm, dt, dex, st);
  else if (mode == 1)
    k_push<1><<<tg.ntiles, 256, 0, s>>>(A, B, ib, tg, f, qbm, dt, dex, st);
  else
    k_push<2><<<tg.ntiles, 256, 0, s>>>(A, B, ib, tg, f, qbm, dt, dex, st);
}

}  // namespace qp
