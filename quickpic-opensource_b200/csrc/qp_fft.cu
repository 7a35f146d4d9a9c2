// qp_fft.cu -- 2D real sine/cosine transforms of field planes (x pass with an
// on-chip transpose, y pass on contiguous columns) and their twiddle tables.
//
// fftrk of a field (field2d_class.f03:157-191) = x pass over rows y = 0..ny
// writing the transposed [kx][y] array, then y pass over columns kx = 0..nx;
// the two passes together carry the reference's normalisation 0.25/(nx*ny).
// fftkr (field2d_class.f03:193-227) = the unnormalised y pass, then the x pass
// reading [kx][y] and writing rows, then the guard copy row ny = row 0
// (ufield2d copyguard, ufield2d_lib.f03:37-42) done by the CTA owning row 0.
#include <algorithm>
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
  // the per-lane rearrangement for the register transform (n >= 64)
  const int P = n >= 64 ? n / 64 : 0;
  std::vector<float> lt(lt_floats(P), 0.f);
  if (P > 0) {
    auto f2 = [&](int off, int i, float2 v) {
      lt[off + 2 * i] = v.x;
      lt[off + 2 * i + 1] = v.y;
    };
    auto brev5 = [](int v) {
      int r = 0;
      for (int b = 0; b < 5; ++b)
        if (v >> b & 1) r |= 1 << (4 - b);
      return r;
    };
    for (int a = 0; a < P; ++a)
      for (int l = 0; l < 32; ++l) {
        const int m = l + 32 * a, j0 = 2 * m, j1 = 2 * m + 1;
        lt[lt_sn0(P) + 32 * a + l] = sn[std::min(j0, n - j0)];
        lt[lt_sn1(P) + 32 * a + l] = sn[std::min(j1, n - j1)];
        lt[lt_cs0(P) + 32 * a + l] = cs[j0];
        lt[lt_cs1(P) + 32 * a + l] = cs[j1];
      }
    for (int k2 = 0; k2 < P; ++k2)
      for (int l = 0; l < 32; ++l) {
        f2(lt_tw4(P), 32 * k2 + l, tw[l * k2]);
        f2(lt_uw(P), 32 * k2 + l, uw[k2 + P * (line_xs(P) ? l : brev5(l))]);
      }
    for (int si = 0; si < 4; ++si) {
      const int st = 16 >> si;
      for (int l = 0; l < 32; ++l)
        f2(lt_tw5(P), 32 * si + l,
           (l & st) ? tw[(l & (st - 1)) * (16 / st) * P] : make_float2(1.f, 0.f));
    }
    for (int k = 0; k < 16; ++k) f2(lt_tw3(P), k, tw[k * P]);
    // exp(-2 pi i q c / 32) = tw[q c P] for the exchange form's 8 x 4 split
    for (int q = 0; q < 4; ++q)
      for (int c = 0; c < 8; ++c) f2(lt_w32(P), 8 * q + c, tw[q * c * P]);
  }
  size_t bytes = sizeof(float) * 2 * (n + 1) + sizeof(float2) * (2 * h + 1) + 64 +
                 sizeof(float) * lt.size() + 16;
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
  float* dlt = nullptr;
  if (P > 0) {
    const size_t lo = ((size_t)(reinterpret_cast<char*>(duw + h + 1) - d) + 15) & ~size_t(15);
    dlt = reinterpret_cast<float*>(d + lo);
    if (cudaMemcpy(dlt, lt.data(), sizeof(float) * lt.size(), cudaMemcpyHostToDevice) !=
        cudaSuccess)
      return -2;
  }
  t->t.lane = dlt;
  t->t.lane_floats = (int)lt.size();
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
// The slice cursor must name one of the planes of the 3D array a component
// reads or writes; otherwise the launch raises an error and does nothing.
__device__ __forceinline__ bool cursor_ok(const XComp& c, const DevStatus* st) {
  const int cur = st->cursor;
  if (cur >= 0 && cur < c.cursor_planes) return true;
  if (threadIdx.x == 0) atomicCAS(const_cast<int*>(&st->error), 0, -7);
  return false;
}

// Shared memory of the line kernels: 8 lines of pitch n + 4 floats (16-byte
// aligned rows; the transposed accesses below hit 32 distinct banks), plus 8
// scratch lines for lines shorter than 64 points.
static __host__ __device__ int line_pitch(int n) { return n + 4; }
static __host__ __device__ int line_count(int logn) { return logn < 6 ? 16 : 8; }

// Forward x pass: for every component c and row y, the line
//   x[j] = scale_c * (src_c[y][j] + src2_c[y][j]),  j = 0..nx
// is transformed with parity_c and stored transposed into dst_c[kx][y].
template <int P>
__global__ void __launch_bounds__(256) k_xfwd(XJob job, GridDims g, LineTables tx,
                                              const DevStatus* st) {
  extern __shared__ __align__(16) float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = g.nx, pitch = line_pitch(n);
  float* L = smem + warp * pitch;
  float* S = smem + (8 + warp) * pitch;
  float* T = smem + line_count(g.indx) * pitch;
  if (P > 0) stage_lane_table(T, tx);  // constant tables: staged before the wait
  grid_dep_sync();
  if (st && st->error) return;
  if (pass_skipped(st, job.pass)) return;
  const XComp c = job.c[blockIdx.y];
  const int y0 = blockIdx.x * 8;
  const int y = y0 + warp;
  long long cur = 0;
  if (c.cursor_stride) {
    if (!cursor_ok(c, st)) return;
    cur = (long long)st->cursor * c.cursor_stride;
  }
  if (P > 0) __syncthreads();
  if (y <= g.ny) {
    const float* s1 = c.src + cur + (long long)y * g.rp;
    const float* s2 = c.src2 ? c.src2 + (long long)y * g.rp : nullptr;
    line_transform<P>(s1, s2, c.scale, L, S, g.indx, c.parity, tx, T, lane);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < (n + 1) * 8; idx += 256) {
    const int r = idx & 7, kx = idx >> 3;
    const int yy = y0 + r;
    if (yy <= g.ny) c.dst[(long long)kx * g.kp + yy] = smem[r * pitch + kx];
  }
}

// Inverse x pass: rows y of the [kx][y] array are gathered, transformed with
// parity_c, scaled and written as real-space rows; row 0 is also written to the
// guard row ny (copyguard), and the line computed for row ny is discarded.
template <int P>
__global__ void __launch_bounds__(256) k_xinv(XJob job, GridDims g, LineTables tx,
                                              const DevStatus* st) {
  extern __shared__ __align__(16) float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = g.nx, pitch = line_pitch(n);
  float* T = smem + line_count(g.indx) * pitch;
  // constant tables, staged before the wait; the barrier after the gather covers them
  if (P > 0) stage_lane_table(T, tx);
  grid_dep_sync();
  if (st && st->error) return;
  if (pass_skipped(st, job.pass)) return;
  const XComp c = job.c[blockIdx.y];
  if (c.cursor_stride && !cursor_ok(c, st)) return;
  const int y0 = blockIdx.x * 8;
  // the 8 rows' [kx][y] entries, 32 bytes per kx: batches of 8 loads per
  // thread are all issued before their shared-memory stores, so a thread waits
  // for L2 twice per 16 loads instead of once per load
  const int total = (n + 1) * 8;
  for (int b0 = threadIdx.x; b0 < total; b0 += 8 * 256) {
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int idx = b0 + u * 256;
      const int yy = y0 + (idx & 7);
      v[u] = (idx < total && yy <= g.ny) ? c.src[(long long)(idx >> 3) * g.kp + yy] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int idx = b0 + u * 256;
      if (idx < total) smem[(idx & 7) * pitch + (idx >> 3)] = v[u];
    }
  }
  __syncthreads();
  float* L = smem + warp * pitch;
  float* S = smem + (8 + warp) * pitch;
  const int y = y0 + warp;
  if (y < g.ny) {
    line_transform<P>(L, nullptr, 1.f, L, S, g.indx, c.parity, tx, T, lane);
    long long cur = 0;
    if (c.cursor_stride) cur = (long long)st->cursor * c.cursor_stride;
    float* d = c.dst + cur + (long long)y * g.rp;
    line_store(d, L, n, c.scale, lane);
    if (y == 0) {
      float* dg = c.dst + cur + (long long)g.ny * g.rp;
      line_store(dg, L, n, c.scale, lane);
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
template <int P>
__global__ void __launch_bounds__(256) k_ycol(YJob job, GridDims g, LineTables ty,
                                              const DevStatus* st) {
  grid_dep_sync();
  extern __shared__ __align__(16) float smem[];
  if (st && st->error) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = g.ny, pitch = line_pitch(n);
  float* L = smem + warp * pitch;
  float* S = smem + (8 + warp) * pitch;
  float* T = smem + line_count(g.indy) * pitch;
  if (P > 0) {
    stage_lane_table(T, ty);
    __syncthreads();
  }
  const int kx = blockIdx.x * 8 + warp;
  if (kx > g.nx) return;
  for (int ci = 0; ci < job.ncomp; ++ci) {
    float* col = job.c[ci].plane + (long long)kx * g.kp;
    line_transform<P>(col, nullptr, 1.f, L, S, g.indy, job.c[ci].parity, ty, T, lane);
    line_store(col, L, n, job.c[ci].scale, lane);
    __syncwarp();
  }
}

size_t xpass_smem(const GridDims& g) {
  return sizeof(float) * ((size_t)line_count(g.indx) * line_pitch(g.nx) + lt_floats(line_p(g.indx)));
}
size_t ypass_smem(const GridDims& g) {
  return sizeof(float) * ((size_t)line_count(g.indy) * line_pitch(g.ny) + lt_floats(line_p(g.indy)));
}

template <int P>
static int set_smem_limits(int big) {
  if (cudaFuncSetAttribute(k_xfwd<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, big) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_xinv<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, big) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_ycol<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, big) !=
          cudaSuccess)
    return -2;
  return 0;
}

int fft_kernels_init() {
  const int big = (int)(sizeof(float) * (8 * line_pitch(1 << QP_MAX_IND) +
                                         lt_floats(line_p(QP_MAX_IND))));
  for (int logn = 4; logn <= QP_MAX_IND; ++logn) {
    int rc = 0;
    QP_LINE_SWITCH(logn, rc = set_smem_limits<P_>(big));
    if (rc) return rc;
  }
  return 0;
}

void launch_xfwd(const XJob& job, const GridDims& g, const LineTables& tx, const DevStatus* st,
                 cudaStream_t s) {
  dim3 grid((g.ny + 1 + 7) / 8, job.ncomp);
  QP_LINE_SWITCH(g.indx, (launch_pdl(k_xfwd<P_>, grid, 256, xpass_smem(g), s, job, g, tx, st)));
}

void launch_xinv(const XJob& job, const GridDims& g, const LineTables& tx, const DevStatus* st,
                 cudaStream_t s) {
  dim3 grid((g.ny + 1 + 7) / 8, job.ncomp);
  QP_LINE_SWITCH(g.indx, (launch_pdl(k_xinv<P_>, grid, 256, xpass_smem(g), s, job, g, tx, st)));
}

void launch_ycol(const YJob& job, const GridDims& g, const LineTables& ty, const DevStatus* st,
                 cudaStream_t s) {
  dim3 grid((g.nx + 1 + 7) / 8);
  QP_LINE_SWITCH(g.indy, (launch_pdl(k_ycol<P_>, grid, 256, ypass_smem(g), s, job, g, ty, st)));
}

}  // namespace qp
