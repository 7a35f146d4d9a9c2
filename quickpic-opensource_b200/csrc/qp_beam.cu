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

void launch_beam_deposit(const BeamBuf& b, const GridDims& g, int nz, float* q3, DevStatus* st,
                         cudaStream_t s) {
  if (b.np == 0) return;
  long long blocks = (b.np + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_beam_deposit<<<(int)blocks, 256, 0, s>>>(b, g, nz, q3, st);
}

}  // namespace qp
