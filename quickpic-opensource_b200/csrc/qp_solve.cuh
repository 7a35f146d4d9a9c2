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
// All arithmetic uses round-to-nearest intrinsics in the reference's
// left-to-right order, so no multiply-add is contracted and each mode is
// bit-identical to the reference's FP32 build whatever the compile flags.
#pragma once

#include "qp_common.cuh"

namespace qp {

#define QM(a, b) __fmul_rn((a), (b))
#define QA(a, b) __fadd_rn((a), (b))
#define QS(a, b) __fsub_rn((a), (b))

struct KCoef {
  int nx, ny;
  float dnx, dny;  // 6.28318530717959 / (2 n), rounded to FP32 as the reference does
  const float* ffre;
  const float* ffim;
  // the form-factor tables are constant for the context's lifetime: read-only
  // loads, which the compiler may issue ahead of the kernels' stores
  __device__ __forceinline__ float re(int kx, int ky) const { return __ldg(ffre + kx * ny + ky); }
  __device__ __forceinline__ float im(int kx, int ky) const { return __ldg(ffim + kx * ny + ky); }
  __device__ __forceinline__ bool interior(int kx, int ky) const {
    return kx > 0 && kx < nx && ky > 0 && ky < ny;
  }
};

__device__ __forceinline__ float k_pot(const KCoef& K, int kx, int ky, float q) {
  return K.interior(kx, ky) ? QM(K.re(kx, ky), q) : 0.f;
}

__device__ __forceinline__ float k_smooth(const KCoef& K, int kx, int ky, float q) {
  return K.interior(kx, ky) ? QM(K.im(kx, ky), q) : 0.f;
}

__device__ __forceinline__ void k_elf(const KCoef& K, int kx, int ky, float q, float* fx,
                                      float* fy) {
  if (K.interior(kx, ky)) {
    const float at1 = QM(K.re(kx, ky), K.im(kx, ky));
    const float at3 = QM(-at1, q);
    *fx = QM(QM(K.dnx, (float)kx), at3);
    *fy = QM(QM(K.dny, (float)ky), at3);
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
  const float dkx = QM(K.dnx, (float)kx);
  const float dky = QM(K.dny, (float)ky);
  if (kx > 0) {
    const float at1 = QM(K.re(kx, ky), K.im(kx, ky));
    if (ky > 0) {
      const float at2 = QM(dky, at1), at3 = QM(dkx, at1);
      *bx = QM(at2, cuz);
      *by = QM(-at3, cuz);
      *bz = QS(QM(at3, cuy), QM(at2, cux));
    } else {
      *bz = QM(QM(dkx, at1), cuy);
    }
  } else if (ky > 0) {
    const float at1 = QM(K.re(0, ky), K.im(0, ky));
    *bz = QM(-QM(dky, at1), cux);
  }
}

// The vector potential (field2d%vpot: PBPOISD23 isign = 1,
// fpois2d_lib77.f:1085-1133, ci = 1): a = g s cu, with the reference's mode
// rules (ky = 0: y only; kx = 0: x only; ky = ny, kx = nx and (0,0): zero).
__device__ __forceinline__ void k_vpot(const KCoef& K, int kx, int ky, float cux, float cuy,
                                       float cuz, float* ax, float* ay, float* az) {
  *ax = 0.f;
  *ay = 0.f;
  *az = 0.f;
  if (kx >= K.nx || ky >= K.ny) return;
  if (kx > 0) {
    const float at1 = QM(K.re(kx, ky), K.im(kx, ky));
    if (ky > 0) {
      *ax = QM(at1, cux);
      *ay = QM(at1, cuy);
      *az = QM(at1, cuz);
    } else {
      *ay = QM(at1, cuy);
    }
  } else if (ky > 0) {
    *ax = QM(QM(K.re(0, ky), K.im(0, ky)), cux);
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
  const float dkx = QM(K.dnx, (float)kx);
  const float dky = QM(K.dny, (float)ky);
  if (kx > 0) {
    if (ky > 0) {
      const float d1 = QS(QA(-*dcx, QM(dkx, amxx)), QM(dky, amxy));
      const float aat1 = QS(d1, QM(QM(dkx, cuz), idex));
      const float d2 = QA(QS(-*dcy, QM(dkx, amxy)), QM(dky, amyy));
      const float aat2 = QS(d2, QM(QM(dky, cuz), idex));
      float at2 = K.re(kx, ky);
      at2 = __fdiv_rn(at2, QA(1.f, QM(aa, at2)));
      const float at1 = QM(at2, K.im(kx, ky));
      *bx = QA(QM(at1, aat1), QM(QM(aa, at2), bxo));
      *by = QA(QM(at1, aat2), QM(QM(aa, at2), byo));
      *dcx = d1;
      *dcy = d2;
    } else {
      const float d1 = QA(-*dcx, QM(dkx, amxx));
      const float d2 = QS(-*dcy, QM(dkx, amxy));
      float at2 = K.re(kx, 0);
      at2 = __fdiv_rn(at2, QA(1.f, QM(aa, at2)));
      const float at1 = QM(at2, K.im(kx, 0));
      *by = QA(QM(at1, d2), QM(QM(aa, at2), byo));
      *dcx = d1;
      *dcy = d2;
    }
  } else if (ky > 0) {
    const float d1 = QS(-*dcx, QM(dky, amxy));
    const float d2 = QA(-*dcy, QM(dky, amyy));
    float at2 = K.re(0, ky);
    at2 = __fdiv_rn(at2, QA(1.f, QM(aa, at2)));
    const float at1 = QM(at2, K.im(0, ky));
    *bx = QA(QM(at1, d1), QM(QM(aa, at2), bxo));
    *dcx = d1;
    *dcy = d2;
  }
}

__device__ __forceinline__ float k_div(const KCoef& K, int kx, int ky, float fx, float fy) {
  if (!K.interior(kx, ky)) return 0.f;
  return -QA(QM(QM(K.dnx, (float)kx), fx), QM(QM(K.dny, (float)ky), fy));
}

__device__ __forceinline__ void k_grad(const KCoef& K, int kx, int ky, float p, float* fx,
                                       float* fy) {
  if (K.interior(kx, ky)) {
    *fx = QM(QM(K.dnx, (float)kx), p);
    *fy = QM(QM(K.dny, (float)ky), p);
  } else {
    *fx = 0.f;
    *fy = 0.f;
  }
}

// bxyz assembly of one mode (simulation_class.f03:677-680 and 717-720):
//   bx = epw(2)*(-dex) - epwb(2); by = epw(1)*dex + epwb(1); bz = bz*dex
__device__ __forceinline__ void k_assemble_mode(float ex, float ey, float ebx, float eby,
                                                float dex, float* bx, float* by, float* bz) {
  *bx = QS(QM(ey, -dex), eby);
  *by = QA(QM(ex, dex), ebx);
  *bz = QM(*bz, dex);
}

// standalone launches used by the class-level API
int launch_kpoint(int op, const GridDims& g, const KCoef& K, float* const* in, float* const* out,
                  float aa, float dex, const DevStatus* st, cudaStream_t s);
enum { KOP_POT = 0, KOP_SMOOTH, KOP_ELF, KOP_BF, KOP_BFQP, KOP_DIV, KOP_GRAD, KOP_VPOT };

}  // namespace qp
