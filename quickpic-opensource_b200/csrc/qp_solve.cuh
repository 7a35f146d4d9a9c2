// qp_solve.cuh -- k-space pointwise operators, one (kx, ky) mode at a time.
//
// Each function reproduces the per-mode result of one QuickPIC solver,
// including which modes it zeroes (kx = 0, kx = nx, ky = 0, ky = ny), so that
// the standalone kernels (class-level API) and the fused column kernels share
// one definition:
//   pot    MPPOTPD2       fpois2d_lib77.f:1701-1779
//   smooth MPPSMOOTHD2    fpois2d_lib77.f:1781-1843
//   elf    MPPOISD22      fpois2d_lib77.f:1532-1575
//   bf     MPPBBPOISD23   fpois2d_lib77.f:1845-1956  (ci = 1)
//   bfqp   PBPOISD22N_QP  fpois2d_lib77.f:1322-1421  (isign = 1, ci = 1)
//   div    MPPDIVFD2      fft2d_lib77.f:9170-9229
//   grad   MPPGRADFD2     fft2d_lib77.f:9231-9295
// ffre/ffim are the real and imaginary parts of the form-factor table ffd
// (affp*s/k^2, s), stored [kx][ky] with pitch ny, kx < nx, ky < ny.
#pragma once

#include "qp_common.cuh"

namespace qp {

struct KCoef {
  int nx, ny;
  float dnx, dny;  // 6.28318530717959 / (2 n), rounded to FP32 as the reference does
  const float* ffre;
  const float* ffim;
  __device__ __forceinline__ float re(int kx, int ky) const { return ffre[kx * ny + ky]; }
  __device__ __forceinline__ float im(int kx, int ky) const { return ffim[kx * ny + ky]; }
  __device__ __forceinline__ bool interior(int kx, int ky) const {
    return kx > 0 && kx < nx && ky > 0 && ky < ny;
  }
};

__device__ __forceinline__ float k_pot(const KCoef& K, int kx, int ky, float q) {
  return K.interior(kx, ky) ? K.re(kx, ky) * q : 0.f;
}

__device__ __forceinline__ float k_smooth(const KCoef& K, int kx, int ky, float q) {
  return K.interior(kx, ky) ? K.im(kx, ky) * q : 0.f;
}

__device__ __forceinline__ void k_elf(const KCoef& K, int kx, int ky, float q, float* fx,
                                      float* fy) {
  if (K.interior(kx, ky)) {
    const float at1 = K.re(kx, ky) * K.im(kx, ky);
    const float at3 = -at1 * q;
    *fx = (K.dnx * (float)kx) * at3;
    *fy = (K.dny * (float)ky) * at3;
  } else {
    *fx = 0.f;
    *fy = 0.f;
  }
}

__device__ __forceinline__ void k_bf(const KCoef& K, int kx, int ky, float cux, float cuy,
                                     float cuz, float* bx, float* by, float* bz) {
  *bx = 0.f;
  *by = 0.f;
  *bz = 0.f;
  if (kx >= K.nx || ky >= K.ny) return;
  const float dkx = K.dnx * (float)kx;
  const float dky = K.dny * (float)ky;
  if (kx > 0) {
    const float at1 = K.re(kx, ky) * K.im(kx, ky);
    if (ky > 0) {
      const float at2 = dky * at1, at3 = dkx * at1;
      *bx = at2 * cuz;
      *by = -at3 * cuz;
      *bz = at3 * cuy - at2 * cux;
    } else {
      *bz = (dkx * at1) * cuy;
    }
  } else if (ky > 0) {
    const float at1 = K.re(0, ky) * K.im(0, ky);
    *bz = -(dky * at1) * cux;
  }
}

// The transverse-B corrector.  dcu is updated in place (the reference writes
// the modified dcu back, and the slice loop extrapolates the current with it).
__device__ __forceinline__ void k_bfqp(const KCoef& K, int kx, int ky, float aa, float idex,
                                       float cuz, float* dcx, float* dcy, float amxx,
                                       float amyy, float amxy, float* bx, float* by) {
  const float bxo = *bx, byo = *by;
  *bx = 0.f;
  *by = 0.f;
  if (kx >= K.nx || ky >= K.ny) return;
  const float dkx = K.dnx * (float)kx;
  const float dky = K.dny * (float)ky;
  if (kx > 0) {
    if (ky > 0) {
      const float d1 = -*dcx + dkx * amxx - dky * amxy;
      const float aat1 = d1 - dkx * cuz * idex;
      const float d2 = -*dcy - dkx * amxy + dky * amyy;
      const float aat2 = d2 - dky * cuz * idex;
      float at2 = K.re(kx, ky);
      at2 = at2 / (1.f + aa * at2);
      const float at1 = at2 * K.im(kx, ky);
      *bx = at1 * aat1 + aa * at2 * bxo;
      *by = at1 * aat2 + aa * at2 * byo;
      *dcx = d1;
      *dcy = d2;
    } else {
      const float d1 = -*dcx + dkx * amxx;
      const float d2 = -*dcy - dkx * amxy;
      float at2 = K.re(kx, 0);
      at2 = at2 / (1.f + aa * at2);
      const float at1 = at2 * K.im(kx, 0);
      *by = at1 * d2 + aa * at2 * byo;
      *dcx = d1;
      *dcy = d2;
    }
  } else if (ky > 0) {
    const float d1 = -*dcx - dky * amxy;
    const float d2 = -*dcy + dky * amyy;
    float at2 = K.re(0, ky);
    at2 = at2 / (1.f + aa * at2);
    const float at1 = at2 * K.im(0, ky);
    *bx = at1 * d1 + aa * at2 * bxo;
    *dcx = d1;
    *dcy = d2;
  }
}

__device__ __forceinline__ float k_div(const KCoef& K, int kx, int ky, float fx, float fy) {
  if (!K.interior(kx, ky)) return 0.f;
  return -((K.dnx * (float)kx) * fx + (K.dny * (float)ky) * fy);
}

__device__ __forceinline__ void k_grad(const KCoef& K, int kx, int ky, float p, float* fx,
                                       float* fy) {
  if (K.interior(kx, ky)) {
    *fx = (K.dnx * (float)kx) * p;
    *fy = (K.dny * (float)ky) * p;
  } else {
    *fx = 0.f;
    *fy = 0.f;
  }
}

// standalone launches used by the class-level API
int launch_kpoint(int op, const GridDims& g, const KCoef& K, float* const* in, float* const* out,
                  float aa, float dex, const DevStatus* st, cudaStream_t s);
enum { KOP_POT = 0, KOP_SMOOTH, KOP_ELF, KOP_BF, KOP_BFQP, KOP_DIV, KOP_GRAD };

}  // namespace qp
