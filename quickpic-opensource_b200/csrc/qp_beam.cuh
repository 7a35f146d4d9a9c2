// qp_beam.cuh -- drive-beam particles on the device.
#pragma once

#include "qp_common.cuh"

namespace qp {

constexpr int BCOMP = 7;  // x, y, z, px, py, pz, q   (part(1..7), part3d_class.f03)

struct BeamBuf {
  float* c[BCOMP];
  long long np;
};

void launch_beam_aos_to_soa(const float* aos, const BeamBuf& b, cudaStream_t s);
void launch_lineout(const float* p, long long plane, long long off, int n, float* out,
                    cudaStream_t s);
void launch_beam_deposit(const BeamBuf& b, const GridDims& g, int nz, float* q3, DevStatus* st,
                         cudaStream_t s);

}  // namespace qp
