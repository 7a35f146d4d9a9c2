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

// The 3D fields a beam push gathers from: planes of the real-space layout,
// plane l = xi node l; e = bexyz (3 components), b = bbxyz (first 2 used).
struct Fields3 {
  const float* e[3];
  const float* b[2];
};

// PGBPUSH32L_QP: push every particle in place; keep[j] = 0 marks a particle
// that left [1, n-1) in x, y or z (conducting boundaries), counted in
// st->beam_drops.  qtmh = qbm*dt, dtcx = dt/dex, dtcz = dt/dxi.
void launch_beam_push(const BeamBuf& b, const GridDims& g, int nz, const Fields3& f, float qtmh,
                      float dtcx, float dtcz, float cofd1, int* keep, DevStatus* st,
                      cudaStream_t s);
// Stable compaction of the kept particles, in chunks of BEAM_CHUNK: per-chunk
// counts, then (after the host's exclusive scan of the counts) the scatter.
constexpr int BEAM_CHUNK = 4096;
void launch_beam_keep_count(const int* keep, long long np, int* counts, cudaStream_t s);
void launch_beam_scatter(const BeamBuf& src, const int* keep, const int* offsets,
                         const BeamBuf& dst, cudaStream_t s);

}  // namespace qp
