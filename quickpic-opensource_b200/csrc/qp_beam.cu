// qp_beam.cu -- drive-beam charge deposit on the 3D grid.
//
// PGPOST32L (part3d_lib77.f:554-628): first-order (CIC) charge deposit of the
// beam macro-particles, weight part(7), into q(nx+2, ny+1, nz+1).  On one GPU
// with one pipeline stage the guard operations that follow it
// (PAGUARD32L / PCGUARD32L, ufield3d_lib77.f:2-323) do nothing.
// Device layout: nz+1 planes of the real-space layout (row pitch rp, ny+1
// rows); plane l holds xi node l.  Beam particles are 7 SoA planes
// (x, y, z, px, py, pz, q) in cell units.
#include "qp_beam.cuh"

namespace qp {

namespace {

__global__ void __launch_bounds__(256) k_beam_deposit(BeamBuf b, GridDims g, int nz, float* q3,
                                                      DevStatus* st) {
  const long long np = b.np;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < np;
       j += (long long)gridDim.x * blockDim.x) {
    const float px = b.c[0][j], py = b.c[1][j], pz = b.c[2][j], qm = b.c[6][j];
    int nn = (int)px, mm = (int)py, ll = (int)pz;
    const float dxp0 = qm * (px - (float)nn);
    float dyp = py - (float)mm;
    const float dzp = pz - (float)ll;
    if (nn < 0 || nn > g.nx || mm < 0 || mm >= g.ny || ll < 0 || ll >= nz) {
      if (st) atomicCAS(&st->error, 0, -5);
      continue;
    }
    float amx = qm - dxp0;
    float amy = 1.f - dyp;
    const float dx1 = dxp0 * dyp;
    dyp = amx * dyp;
    amx = amx * amy;
    const float amz = 1.f - dzp;
    amy = dxp0 * amy;
    float* p = q3 + (long long)ll * g.rplane + (long long)mm * g.rp + nn;
    float* pz1 = p + g.rplane;
    atomicAdd(p, amx * amz);
    atomicAdd(p + 1, amy * amz);
    atomicAdd(p + g.rp, dyp * amz);
    atomicAdd(p + g.rp + 1, dx1 * amz);
    atomicAdd(pz1, amx * dzp);
    atomicAdd(pz1 + 1, amy * dzp);
    atomicAdd(pz1 + g.rp, dyp * dzp);
    atomicAdd(pz1 + g.rp + 1, dx1 * dzp);
  }
}

// PGBPUSH32L_QP (part3d_lib77.f:630-786) for one partition: trilinear gather
// of E = bexyz(1:3) and B = bbxyz(1:2) at the particle, the transverse force
// (Ex - By, Ey + Bx), the momentum update, gamma, and the position update in
// x, y (dt / dex / gamma) and z (the quasi-static 1 - v_z term, dt / dxi).
// Every product and sum is in the reference's order; the file is built
// without contracted multiply-adds, so each particle is bit-identical to the
// reference's FP32 push.  A particle that leaves [1, n-1) in any direction is
// marked in keep[] instead of being moved (the host compacts afterwards).
__global__ void __launch_bounds__(256) k_beam_push(BeamBuf b, GridDims g, int nz, Fields3 f,
                                                   float qtmh, float dtcx, float dtcz,
                                                   float cofd1, int* keep, DevStatus* st) {
  if (st->error) return;
  const float edgerx = (float)(g.nx - 1), edgery = (float)(g.ny - 1), edgerz = (float)(nz - 1);
  const long long rp = g.rp, pl = g.rplane;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < b.np;
       j += (long long)gridDim.x * blockDim.x) {
    const float x = b.c[0][j], y = b.c[1][j], z = b.c[2][j];
    int nn = (int)x, mm = (int)y, ll = (int)z;
    if (nn < 0 || nn > g.nx || mm < 0 || mm >= g.ny || ll < 0 || ll >= nz) {
      atomicCAS(&st->error, 0, -5);  // outside the 3D arrays: gather nothing
      keep[j] = 1;
      continue;
    }
    float dxp = x - (float)nn, dyp = y - (float)mm;
    const float dzp = z - (float)ll;
    float amx = 1.f - dxp, amy = 1.f - dyp;
    const float dx1 = dxp * dyp;
    dyp = amx * dyp;
    amx = amx * amy;
    const float amz = 1.f - dzp;
    amy = dxp * amy;
    const long long o = (long long)ll * pl + (long long)mm * rp + nn;
    const long long oz = o + pl;
    auto tri = [&](const float* a) {
      const float lo = amx * a[o] + amy * a[o + 1] + dyp * a[o + rp] + dx1 * a[o + rp + 1];
      const float hi = amx * a[oz] + amy * a[oz + 1] + dyp * a[oz + rp] + dx1 * a[oz + rp + 1];
      return amz * lo + dzp * hi;
    };
    float dx = tri(f.e[0]), dy = tri(f.e[1]), dz = tri(f.e[2]);
    const float ox = tri(f.b[0]), oy = tri(f.b[1]);
    dx = dx - oy;
    dy = dy + ox;
    const float delx = qtmh * dx, dely = qtmh * dy, delz = qtmh * dz;
    dx = b.c[3][j] + delx;
    dy = b.c[4][j] + dely;
    dz = b.c[5][j] + delz;
    const float p2t = dx * dx + dy * dy;
    const float p2l = dz * dz;
    const float p2 = p2t + p2l;
    const float ngamma = sqrtf(1.f + p2);
    const float dtgx = dtcx / ngamma;
    const float dtgy = dtcx / ngamma;
    const float omvz = (1.f + p2t) / (dz * (dz + ngamma));
    dz = dz - cofd1 * ngamma * ((delx * delx + dely * dely) * dz - delz * (delx * dx + dely * dy));
    const float xn = x + dx * dtgx, yn = y + dy * dtgy, zn = z + omvz * dtcz;
    if (xn < 1.f || xn >= edgerx || yn < 1.f || yn >= edgery || zn < 1.f || zn >= edgerz) {
      keep[j] = 0;
      atomicAdd(&st->beam_drops, 1);
      continue;
    }
    keep[j] = 1;
    b.c[0][j] = xn;
    b.c[1][j] = yn;
    b.c[2][j] = zn;
    b.c[3][j] = dx;
    b.c[4][j] = dy;
    b.c[5][j] = dz;
  }
}

__device__ __forceinline__ int block_sum(int v, int* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  int t = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

// kept particles of each chunk of BEAM_CHUNK
__global__ void __launch_bounds__(256) k_beam_keep_count(const int* keep, long long np,
                                                         int* counts) {
  __shared__ int red[8];
  const long long c0 = (long long)blockIdx.x * BEAM_CHUNK;
  int n = 0;
  for (int i = threadIdx.x; i < BEAM_CHUNK; i += blockDim.x)
    if (c0 + i < np) n += keep[c0 + i];
  n = block_sum(n, red);
  if (threadIdx.x == 0) counts[blockIdx.x] = n;
}

// stable scatter of the kept particles of each chunk to dst at offsets[chunk]
__global__ void __launch_bounds__(256) k_beam_scatter(BeamBuf src, const int* keep,
                                                      const int* offsets, BeamBuf dst) {
  __shared__ int wsum[8];
  __shared__ int base;
  if (threadIdx.x == 0) base = offsets[blockIdx.x];
  __syncthreads();
  const long long c0 = (long long)blockIdx.x * BEAM_CHUNK;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = 0; r < BEAM_CHUNK; r += blockDim.x) {
    const long long j = c0 + r + threadIdx.x;
    const bool k = j < src.np && keep[j] != 0;
    const unsigned bal = __ballot_sync(0xffffffffu, k);
    if (lane == 0) wsum[warp] = __popc(bal);
    __syncthreads();
    int woff = 0, tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      if (w < warp) woff += wsum[w];
      tot += wsum[w];
    }
    if (k) {
      const long long pos = base + woff + __popc(bal & ((1u << lane) - 1u));
#pragma unroll
      for (int c = 0; c < BCOMP; ++c) dst.c[c][pos] = src.c[c][j];
    }
    __syncthreads();
    if (threadIdx.x == 0) base += tot;
    __syncthreads();
  }
}

// part(7, np) (AoS, the reference layout) -> 7 SoA planes
__global__ void k_beam_aos_to_soa(const float* aos, BeamBuf b) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < b.np;
       j += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < BCOMP; ++c) b.c[c][j] = aos[7 * j + c];
  }
}

// on-axis line of a stack of 3D planes: out[l] = p[l][y][x]
__global__ void k_lineout(const float* p, long long plane, long long off, int n, float* out) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l < n) out[l] = p[(long long)l * plane + off];
}

}  // namespace

void launch_beam_aos_to_soa(const float* aos, const BeamBuf& b, cudaStream_t s) {
  if (b.np == 0) return;
  k_beam_aos_to_soa<<<148 * 8, 256, 0, s>>>(aos, b);
}

void launch_lineout(const float* p, long long plane, long long off, int n, float* out,
                    cudaStream_t s) {
  k_lineout<<<(n + 255) / 256, 256, 0, s>>>(p, plane, off, n, out);
}

void launch_beam_push(const BeamBuf& b, const GridDims& g, int nz, const Fields3& f, float qtmh,
                      float dtcx, float dtcz, float cofd1, int* keep, DevStatus* st,
                      cudaStream_t s) {
  if (b.np == 0) return;
  // one particle per thread: the gathers of a particle wait for memory once,
  // and the many resident CTAs overlap those waits (a grid-stride loop would
  // wait once per particle of a thread)
  long long blocks = (b.np + 255) / 256;
  if (blocks > (1LL << 30)) blocks = 1LL << 30;
  k_beam_push<<<(int)blocks, 256, 0, s>>>(b, g, nz, f, qtmh, dtcx, dtcz, cofd1, keep, st);
}

void launch_beam_keep_count(const int* keep, long long np, int* counts, cudaStream_t s) {
  const long long chunks = (np + BEAM_CHUNK - 1) / BEAM_CHUNK;
  if (chunks > 0) k_beam_keep_count<<<(int)chunks, 256, 0, s>>>(keep, np, counts);
}

void launch_beam_scatter(const BeamBuf& src, const int* keep, const int* offsets,
                         const BeamBuf& dst, cudaStream_t s) {
  const long long chunks = (src.np + BEAM_CHUNK - 1) / BEAM_CHUNK;
  if (chunks > 0) k_beam_scatter<<<(int)chunks, 256, 0, s>>>(src, keep, offsets, dst);
}

void launch_beam_deposit(const BeamBuf& b, const GridDims& g, int nz, float* q3, DevStatus* st,
                         cudaStream_t s) {
  if (b.np == 0) return;
  long long blocks = (b.np + 255) / 256;  // one particle per thread, as the push
  if (blocks > (1LL << 30)) blocks = 1LL << 30;
  k_beam_deposit<<<(int)blocks, 256, 0, s>>>(b, g, nz, q3, st);
}

}  // namespace qp
