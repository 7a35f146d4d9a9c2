// qp_misc.cu -- Fourier-space solve kernels, field algebra, guard operations
// and the small per-slice kernels of the fused 3D step.
#include "qp_misc.cuh"

namespace qp {

namespace {

__device__ __forceinline__ bool kidx(const GridDims& g, int i, int* kx, int* ky) {
  const int n1 = g.ny + 1;
  if (i >= (g.nx + 1) * n1) return false;
  *kx = i / n1;
  *ky = i - *kx * n1;
  return true;
}

__global__ void k_kpoint(int op, GridDims g, KCoef K, KPtrs in, KPtrs out, float aa, float dex,
                         const DevStatus* st) {
  grid_dep_sync();
  if (st && st->error) return;
  int kx, ky;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (!kidx(g, i, &kx, &ky)) return;
  const long long o = (long long)kx * g.kp + ky;
  switch (op) {
    case KOP_POT:
      out.p[0][o] = k_pot(K, kx, ky, in.p[0][o]);
      break;
    case KOP_SMOOTH:
      out.p[0][o] = k_smooth(K, kx, ky, in.p[0][o]);
      break;
    case KOP_ELF: {
      float fx, fy;
      k_elf(K, kx, ky, in.p[0][o], &fx, &fy);
      out.p[0][o] = fx;
      out.p[1][o] = fy;
      break;
    }
    case KOP_BF: {
      float bx, by, bz;
      k_bf(K, kx, ky, in.p[0][o], in.p[1][o], in.p[2][o], &bx, &by, &bz);
      out.p[0][o] = bx;
      out.p[1][o] = by;
      out.p[2][o] = bz;
      break;
    }
    case KOP_BFQP: {
      // in: cu(3), dcu(2) (in/out), amu(3); out: bxy(2) (in/out)
      float dcx = in.p[3][o], dcy = in.p[4][o];
      float bx = out.p[0][o], by = out.p[1][o];
      k_bfqp(K, kx, ky, aa, 1.f / dex, in.p[2][o], &dcx, &dcy, in.p[5][o], in.p[6][o],
             in.p[7][o], &bx, &by);
      in.p[3][o] = dcx;
      in.p[4][o] = dcy;
      out.p[0][o] = bx;
      out.p[1][o] = by;
      break;
    }
    case KOP_DIV:
      out.p[0][o] = k_div(K, kx, ky, in.p[0][o], in.p[1][o]);
      break;
    case KOP_GRAD: {
      float fx, fy;
      k_grad(K, kx, ky, in.p[0][o], &fx, &fy);
      out.p[0][o] = fx;
      out.p[1][o] = fy;
      break;
    }
    case KOP_VPOT: {
      float ax, ay, az;
      k_vpot(K, kx, ky, in.p[0][o], in.p[1][o], in.p[2][o], &ax, &ay, &az);
      out.p[0][o] = ax;
      out.p[1][o] = ay;
      out.p[2][o] = az;
      break;
    }
  }
}

__global__ void k_lin(long long n, float* d, const float* a, const float* b, float v, int op,
                      const DevStatus* st) {
  grid_dep_sync();
  if (st && st->error) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    switch (op) {
      case LIN_FILL:
        d[i] = v;
        break;
      case LIN_SCALE:
        d[i] = a[i] * v;
        break;
      case LIN_ADD:
        d[i] = a[i] + b[i];
        break;
      case LIN_SUB:
        d[i] = a[i] - b[i];
        break;
      case LIN_COPY:
        d[i] = a[i];
        break;
    }
  }
}

// copyguard: row ny = row 0, every column (ufield2d_lib.f03:37-42)
__global__ void k_guard_copy(float* p, GridDims g, const DevStatus* st) {
  grid_dep_sync();
  if (st && st->error) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j <= g.nx + 1) p[(long long)g.ny * g.rp + j] = p[j];
}

// acopyguard: row 0 += row ny, row ny = 0 for columns 0..nx (ufield2d_lib.f03:90-97)
__global__ void k_guard_add(float* p, GridDims g, const DevStatus* st) {
  grid_dep_sync();
  if (st && st->error) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j <= g.nx) {
    float* top = p + (long long)g.ny * g.rp + j;
    p[j] = p[j] + *top;
    *top = 0.f;
  }
}

// bxyz assembly in Fourier space (simulation_class.f03:677-680 and 717-720):
//   bx = -dex*epw(2) - epwb(2); by = dex*epw(1) + epwb(1); bz = dex*bz
__global__ void k_assemble(GridDims g, float* bx, float* by, float* bz, const float* ex,
                           const float* ey, const float* ebx, const float* eby, float dex,
                           const DevStatus* st) {
  grid_dep_sync();
  if (st->error) return;
  int kx, ky;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (!kidx(g, i, &kx, &ky)) return;
  const long long o = (long long)kx * g.kp + ky;
  const float b1 = ey[o] * (-dex);
  const float b2 = ex[o] * dex;
  bz[o] = bz[o] * dex;
  bx[o] = b1 - eby[o];
  by[o] = b2 + ebx[o];
}

// end-of-slice extrapolation of the current in Fourier space
// (simulation_class.f03:725-726): dcu = dcu*dxi; cu(1:2) = cu(1:2) - dcu(1:2)
__global__ void k_extrap(GridDims g, float* cx, float* cy, float* dx, float* dy, float dxi,
                         const DevStatus* st) {
  grid_dep_sync();
  if (st->error) return;
  int kx, ky;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (!kidx(g, i, &kx, &ky)) return;
  const long long o = (long long)kx * g.kp + ky;
  const float a = dx[o] * dxi, b = dy[o] * dxi;
  dx[o] = a;
  dy[o] = b;
  cx[o] = cx[o] - a;
  cy[o] = cy[o] - b;
}

// Fourier-space scale of one plane, skipped after an error
__global__ void k_kscale(GridDims g, float* p, float v, const DevStatus* st) {
  grid_dep_sync();
  if (st->error) return;
  int kx, ky;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (!kidx(g, i, &kx, &ky)) return;
  const long long o = (long long)kx * g.kp + ky;
  p[o] = p[o] * v;
}

// End of a slice (simulation_class.f03:722-735): the final force
// fxy = -fxy + (by, -bx), then fxy *= dex -> bexyz(1:2), psit -> bexyz(3),
// bxyz(1:2) *= dex -> bbxyz, stored at 3D plane `cursor` (0-based; the
// reference's 1-based slice j+1 for slice j); fxy and bxyz are
// updated in place as in the reference.
__global__ void k_store3d(GridDims g, float* fx, float* fy, float* bx, float* by, const float* bz,
                          const float* psit, Planes3 be, Planes3 bb, float dex, int store,
                          int nplanes, float* zero_q, DevStatus* st) {
  grid_dep_sync();
  if (st->error) return;
  const int cur = st->cursor;
  if (store && (cur < 0 || cur >= nplanes)) {  // never store outside the 3D arrays
    if (threadIdx.x == 0) atomicCAS(&st->error, 0, -7);
    return;
  }
  // four nodes per thread: planes and rows are 16-byte aligned (rp = nx + 4)
  const long long n4 = g.rplane >> 2;
  const long long pl4 = (long long)cur * n4;
  float4* fx4 = reinterpret_cast<float4*>(fx);
  float4* fy4 = reinterpret_cast<float4*>(fy);
  float4* bx4 = reinterpret_cast<float4*>(bx);
  float4* by4 = reinterpret_cast<float4*>(by);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4;
       i += (long long)gridDim.x * blockDim.x) {
    // every load of the iteration first, so the thread waits for L2 once
    const float4 vfx = fx4[i], vfy = fy4[i], vbx = bx4[i], vby = by4[i];
    float4 vpt = make_float4(0.f, 0.f, 0.f, 0.f), vbz = vpt;
    if (store) {
      vpt = reinterpret_cast<const float4*>(psit)[i];
      vbz = reinterpret_cast<const float4*>(bz)[i];
    }
    float4 f1, f2, b1, b2;
    // f1 = (-fx + by) * dex, f2 = (-fy - bx) * dex; b1 = bx * dex, b2 = by * dex
    f1.x = (-1.f * vfx.x + vby.x) * dex;
    f1.y = (-1.f * vfx.y + vby.y) * dex;
    f1.z = (-1.f * vfx.z + vby.z) * dex;
    f1.w = (-1.f * vfx.w + vby.w) * dex;
    f2.x = (-1.f * vfy.x - vbx.x) * dex;
    f2.y = (-1.f * vfy.y - vbx.y) * dex;
    f2.z = (-1.f * vfy.z - vbx.z) * dex;
    f2.w = (-1.f * vfy.w - vbx.w) * dex;
    b1 = make_float4(vbx.x * dex, vbx.y * dex, vbx.z * dex, vbx.w * dex);
    b2 = make_float4(vby.x * dex, vby.y * dex, vby.z * dex, vby.w * dex);
    fx4[i] = f1;
    fy4[i] = f2;
    bx4[i] = b1;
    by4[i] = b2;
    if (store) {
      reinterpret_cast<float4*>(be.p[0])[pl4 + i] = f1;
      reinterpret_cast<float4*>(be.p[1])[pl4 + i] = f2;
      reinterpret_cast<float4*>(be.p[2])[pl4 + i] = vpt;
      reinterpret_cast<float4*>(bb.p[0])[pl4 + i] = b1;
      reinterpret_cast<float4*>(bb.p[1])[pl4 + i] = b2;
      reinterpret_cast<float4*>(bb.p[2])[pl4 + i] = vbz;
    }
    if (zero_q) reinterpret_cast<float4*>(zero_q)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  // the last CTA to finish advances the slice cursor
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const int done = atomicAdd(&st->store_ctas, 1);
    if (done == (int)gridDim.x - 1) {
      st->store_ctas = 0;
      st->cursor = st->cursor + 1;
      __threadfence();
    }
  }
}

__global__ void k_cursor(DevStatus* st, int v) {
  grid_dep_sync();
  if (st->error) return;
  st->cursor = v < 0 ? st->cursor + 1 : v;
}

}  // namespace

int launch_kpoint(int op, const GridDims& g, const KCoef& K, float* const* in, float* const* out,
                  float aa, float dex, const DevStatus* st, cudaStream_t s) {
  KPtrs a{}, b{};
  for (int i = 0; i < 8; ++i) {
    a.p[i] = in ? in[i] : nullptr;
    b.p[i] = out ? out[i] : nullptr;
  }
  const int n = (g.nx + 1) * (g.ny + 1);
  launch_pdl(k_kpoint, (n + 255) / 256, 256, 0, s, op, g, K, a, b, aa, dex, st);
  return 0;
}

void launch_lin(long long n, float* d, const float* a, const float* b, float v, int op,
                const DevStatus* st, cudaStream_t s) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  launch_pdl(k_lin, (int)blocks, 256, 0, s, n, d, a, b, v, op, st);
}

void launch_guard_copy(float* p, const GridDims& g, const DevStatus* st, cudaStream_t s) {
  launch_pdl(k_guard_copy, (g.nx + 2 + 255) / 256, 256, 0, s, p, g, st);
}

void launch_guard_add(float* p, const GridDims& g, const DevStatus* st, cudaStream_t s) {
  launch_pdl(k_guard_add, (g.nx + 1 + 255) / 256, 256, 0, s, p, g, st);
}

void launch_assemble(const GridDims& g, float* const* bxyz, float* const* epw,
                     float* const* epwb, float dex, const DevStatus* st, cudaStream_t s) {
  const int n = (g.nx + 1) * (g.ny + 1);
  launch_pdl(k_assemble, (n + 255) / 256, 256, 0, s, g, bxyz[0], bxyz[1], bxyz[2], epw[0], epw[1],
                                             epwb[0], epwb[1], dex, st);
}

void launch_extrap(const GridDims& g, float* const* cu, float* const* dcu, float dxi,
                   const DevStatus* st, cudaStream_t s) {
  const int n = (g.nx + 1) * (g.ny + 1);
  launch_pdl(k_extrap, (n + 255) / 256, 256, 0, s, g, cu[0], cu[1], dcu[0], dcu[1], dxi, st);
}

void launch_kscale(const GridDims& g, float* p, float v, const DevStatus* st, cudaStream_t s) {
  const int n = (g.nx + 1) * (g.ny + 1);
  launch_pdl(k_kscale, (n + 255) / 256, 256, 0, s, g, p, v, st);
}

void launch_cursor(DevStatus* st, int v, cudaStream_t s) {
  launch_pdl(k_cursor, 1, 1, 0, s, st, v);
}

void launch_store3d(const GridDims& g, float* const* fxy, float* const* bxyz, const float* psit,
                    const Planes3& be, const Planes3& bb, float dex, int store, int nplanes,
                    float* zero_q, DevStatus* st, cudaStream_t s) {
  long long blocks = ((g.rplane >> 2) + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  launch_pdl(k_store3d, (int)blocks, 256, 0, s, g, fxy[0], fxy[1], bxyz[0], bxyz[1], bxyz[2],
             psit, be, bb, dex, store, nplanes, zero_q, st);
}

}  // namespace qp
