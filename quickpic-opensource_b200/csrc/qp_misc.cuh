// qp_misc.cuh -- launch interface of the solve, algebra, guard and glue kernels.
#pragma once

#include "qp_common.cuh"
#include "qp_solve.cuh"

namespace qp {

struct KPtrs {
  float* p[8];
};
struct Planes3 {
  float* p[3];
};

enum { LIN_FILL = 0, LIN_SCALE, LIN_ADD, LIN_SUB, LIN_COPY };

void launch_lin(long long n, float* d, const float* a, const float* b, float v, int op,
                const DevStatus* st, cudaStream_t s);
void launch_guard_copy(float* p, const GridDims& g, const DevStatus* st, cudaStream_t s);
void launch_guard_add(float* p, const GridDims& g, const DevStatus* st, cudaStream_t s);
void launch_assemble(const GridDims& g, float* const* bxyz, float* const* epw,
                     float* const* epwb, float dex, const DevStatus* st, cudaStream_t s);
void launch_extrap(const GridDims& g, float* const* cu, float* const* dcu, float dxi,
                   const DevStatus* st, cudaStream_t s);
void launch_kscale(const GridDims& g, float* p, float v, const DevStatus* st, cudaStream_t s);
void launch_cursor(DevStatus* st, int v, cudaStream_t s);
// also clears zero_q (if not null) and advances the slice cursor
void launch_store3d(const GridDims& g, float* const* fxy, float* const* bxyz, const float* psit,
                    const Planes3& be, const Planes3& bb, float dex, int store, int nplanes,
                    float* zero_q, DevStatus* st, cudaStream_t s);

}  // namespace qp
