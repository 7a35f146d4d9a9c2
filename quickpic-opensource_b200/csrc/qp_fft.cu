// qp_fft.cu -- 2D real sine/cosine transforms of field planes (x pass with an
// on-chip transpose, y pass on contiguous columns) and their twiddle tables.
//
// fftrk of a field (field2d_class.f03:157-191) = x pass over rows y = 0..ny
// writing the transposed [kx][y] array, then y pass over columns kx = 0..nx;
// the two passes together carry the reference's normalisation 0.25/(nx*ny).
// fftkr (field2d_class.f03:193-227) = the unnormalised y pass, then the x pass
// reading [kx][y] and writing rows, then the guard copy row ny = row 0
// (ufield2d copyguard, ufield2d_lib.f03:37-42) done by the CTA owning row 0.
#include <cmath>
#include <vector>

#include "qp_fft.cuh"
#include "qp_line.cuh"

namespace qp {

int line_tables_build(LineTablesHost* t, int logn) {
  const int n = 1 << logn, h = n >> 1;
  std::vector<float> sn(n + 1), cs(n + 1);
  std::vector<float2> tw(h), uw(h + 1);
  const double pi = 3.14159265358979323846;
  for (int j = 0; j <= n; ++j) {
    sn[j] = (float)std::sin(pi * j / n);
    cs[j] = (float)std::cos(pi * j / n);
  }
  for (int m = 0; m < h; ++m)
    tw[m] = make_float2((float)std::cos(-2.0 * pi * m / h), (float)std::sin(-2.0 * pi * m / h));
  for (int k = 0; k <= h; ++k)
    uw[k] = make_float2((float)std::cos(-2.0 * pi * k / n), (float)std::sin(-2.0 * pi * k / n));
  size_t bytes = sizeof(float) * 2 * (n + 1) + sizeof(float2) * (2 * h + 1) + 64;
  char* d = nullptr;
  if (cudaMalloc(&d, bytes) != cudaSuccess) return -2;
  float* dsn = reinterpret_cast<float*>(d);
  float* dcs = dsn + (n + 1);
  size_t off = (sizeof(float) * 2 * (n + 1) + 15) & ~size_t(15);
  float2* dtw = reinterpret_cast<float2*>(d + off);
  float2* duw = dtw + h;
  cudaMemcpy(dsn, sn.data(), sizeof(float) * (n + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(dcs, cs.data(), sizeof(float) * (n + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(dtw, tw.data(), sizeof(float2) * h, cudaMemcpyHostToDevice);
  if (cudaMemcpy(duw, uw.data(), sizeof(float2) * (h + 1), cudaMemcpyHostToDevice) != cudaSuccess)
    return -2;
  t->base = d;
  t->t.sn = dsn;
  t->t.cs = dcs;
  t->t.tw = dtw;
  t->t.uw = duw;
  t->logn = logn;
  return 0;
}

void line_tables_free(LineTablesHost* t) {
  if (t->base) cudaFree(t->base);
  t->base = nullptr;
}

// ------------------------------------------------------------------ x pass
// Forward x pass: for every component c and row y, the line
//   x[j] = scale_c * (src_c[y][j] + src2_c[y][j]),  j = 0..nx
// is transformed with parity_c and stored transposed into dst_c[kx][y].
__global__ void __launch_bounds__(256) k_xfwd(XJob job, GridDims g, LineTables tx,
                                              const DevStatus* st) {
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = g.nx, npad = n + 6;
  float* L = smem + (2 * warp) * npad;
  float* S = L + npad;
  if (st && st->error) return;
  const XComp c = job.c[blockIdx.y];
  const int y0 = blockIdx.x * 8;
  const int y = y0 + warp;
  long long cur = 0;
  if (c.cursor_stride) cur = (long long)st->cursor * c.cursor_stride;
  if (y <= g.ny) {
    const float* s1 = c.src + cur + (long long)y * g.rp;
    const float* s2 = c.src2 ? c.src2 + (long long)y * g.rp : nullptr;
    for (int j = lane; j <= n; j += 32) {
      float v = s1[j];
      if (s2) v += s2[j];
      L[j] = v * c.scale;
    }
    __syncwarp();
    warp_line_transform(L, S, g.indx, c.parity, tx, lane);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < (n + 1) * 8; idx += 256) {
    const int r = idx & 7, kx = idx >> 3;
    const int yy = y0 + r;
    if (yy <= g.ny) c.dst[(long long)kx * g.kp + yy] = smem[(2 * r) * npad + kx];
  }
}

// Inverse x pass: rows y of the [kx][y] array are gathered, transformed with
// parity_c, scaled and written as real-space rows; row 0 is also written to the
// guard row ny (copyguard), and the line computed for row ny is discarded.
__global__ void __launch_bounds__(256) k_xinv(XJob job, GridDims g, LineTables tx,
                                              const DevStatus* st) {
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = g.nx, npad = n + 6;
  if (st && st->error) return;
  const XComp c = job.c[blockIdx.y];
  const int y0 = blockIdx.x * 8;
  for (int idx = threadIdx.x; idx < (n + 1) * 8; idx += 256) {
    const int r = idx & 7, kx = idx >> 3;
    const int yy = y0 + r;
    smem[(2 * r) * npad + kx] = (yy <= g.ny) ? c.src[(long long)kx * g.kp + yy] : 0.f;
  }
  __syncthreads();
  float* L = smem + (2 * warp) * npad;
  float* S = L + npad;
  const int y = y0 + warp;
  if (y < g.ny) {
    warp_line_transform(L, S, g.indx, c.parity, tx, lane);
    long long cur = 0;
    if (c.cursor_stride) cur = (long long)st->cursor * c.cursor_stride;
    float* d = c.dst + cur + (long long)y * g.rp;
    for (int j = lane; j <= n; j += 32) d[j] = L[j] * c.scale;
    if (y == 0) {
      float* dg = c.dst + cur + (long long)g.ny * g.rp;
      for (int j = lane; j <= n; j += 32) dg[j] = L[j] * c.scale;
      if (lane == 0) dg[n + 1] = d[n + 1];
    }
  }
  for (int z = blockIdx.y; z < job.nzero; z += job.ncomp) {
    float* p = job.zero[z] + (long long)y0 * g.rp;
    const int rows = min(8, g.ny + 1 - y0);
    for (int i = threadIdx.x; i < rows * g.rp; i += 256) p[i] = 0.f;
  }
}

// ------------------------------------------------------------------ y pass
// In-place y transform of the columns kx of every component, times scale_c.
__global__ void __launch_bounds__(256) k_ycol(YJob job, GridDims g, LineTables ty,
                                              const DevStatus* st) {
  extern __shared__ float smem[];
  if (st && st->error) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = g.ny, npad = n + 6;
  float* L = smem + (2 * warp) * npad;
  float* S = L + npad;
  const int kx = blockIdx.x * 8 + warp;
  if (kx > g.nx) return;
  for (int ci = 0; ci < job.ncomp; ++ci) {
    float* col = job.c[ci].plane + (long long)kx * g.kp;
    for (int j = lane; j <= n; j += 32) L[j] = col[j];
    __syncwarp();
    warp_line_transform(L, S, g.indy, job.c[ci].parity, ty, lane);
    const float sc = job.c[ci].scale;
    for (int j = lane; j <= n; j += 32) col[j] = L[j] * sc;
    __syncwarp();
  }
}

size_t xpass_smem(const GridDims& g) { return sizeof(float) * 16 * (size_t)(g.nx + 6); }
size_t ypass_smem(const GridDims& g) { return sizeof(float) * 16 * (size_t)(g.ny + 6); }

int fft_kernels_init() {
  const int big = (int)(sizeof(float) * 16 * ((1 << QP_MAX_IND) + 6));
  if (cudaFuncSetAttribute(k_xfwd, cudaFuncAttributeMaxDynamicSharedMemorySize, big) !=
      cudaSuccess)
    return -2;
  if (cudaFuncSetAttribute(k_xinv, cudaFuncAttributeMaxDynamicSharedMemorySize, big) !=
      cudaSuccess)
    return -2;
  if (cudaFuncSetAttribute(k_ycol, cudaFuncAttributeMaxDynamicSharedMemorySize, big) !=
      cudaSuccess)
    return -2;
  return 0;
}

void launch_xfwd(const XJob& job, const GridDims& g, const LineTables& tx, const DevStatus* st,
                 cudaStream_t s) {
  dim3 grid((g.ny + 1 + 7) / 8, job.ncomp);
  k_xfwd<<<grid, 256, xpass_smem(g), s>>>(job, g, tx, st);
}

void launch_xinv(const XJob& job, const GridDims& g, const LineTables& tx, const DevStatus* st,
                 cudaStream_t s) {
  dim3 grid((g.ny + 1 + 7) / 8, job.ncomp);
  k_xinv<<<grid, 256, xpass_smem(g), s>>>(job, g, tx, st);
}

void launch_ycol(const YJob& job, const GridDims& g, const LineTables& ty, const DevStatus* st,
                 cudaStream_t s) {
  dim3 grid((g.nx + 1 + 7) / 8);
  k_ycol<<<grid, 256, ypass_smem(g), s>>>(job, g, ty, st);
}

}  // namespace qp
