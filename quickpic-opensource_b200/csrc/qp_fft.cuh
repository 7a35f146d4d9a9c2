// qp_fft.cuh -- launch interface of the 2D sine/cosine transform passes.
#pragma once

#include "qp_common.cuh"

namespace qp {

struct LineTablesHost {
  char* base = nullptr;
  LineTables t{};
  int logn = 0;
};

int line_tables_build(LineTablesHost* t, int logn);
void line_tables_free(LineTablesHost* t);

constexpr int QP_MAX_JOB = 12;

// One component of an x pass.  xfwd: src/src2 are real planes, dst a k plane;
// xinv: src is a k plane, dst a real plane.  cursor_stride != 0 offsets the
// real-space side by cursor * cursor_stride floats (slice of a 3D array chosen
// by the device slice cursor).
struct XComp {
  const float* src;
  const float* src2;
  float* dst;
  float scale;
  int parity;  // 0 sine, 1 cosine
  long long cursor_stride;
  int cursor_planes;  // planes of that 3D array: a cursor outside them raises an error
};
struct XJob {
  XComp c[QP_MAX_JOB];
  int ncomp;
  // xinv only: real-space planes whose rows this launch clears (plane i is
  // cleared by the CTAs of component i % ncomp)
  float* zero[8];
  int nzero;
  int pass;  // predictor-corrector pass of the launch (pass_skipped), 0 = none
};

struct YComp {
  float* plane;
  float scale;
  int parity;
};
struct YJob {
  YComp c[QP_MAX_JOB];
  int ncomp;
};

int fft_kernels_init();
size_t xpass_smem(const GridDims& g);
size_t ypass_smem(const GridDims& g);
void launch_xfwd(const XJob& job, const GridDims& g, const LineTables& tx, const DevStatus* st,
                 cudaStream_t s);
void launch_xinv(const XJob& job, const GridDims& g, const LineTables& tx, const DevStatus* st,
                 cudaStream_t s);
void launch_ycol(const YJob& job, const GridDims& g, const LineTables& ty, const DevStatus* st,
                 cudaStream_t s);

}  // namespace qp
