// qp_part.cuh -- tile-binned plasma particles and their kernels.
#pragma once

#include "qp_common.cuh"

namespace qp {

constexpr int TILE = 16;  // cells per tile side (part2d_class.f03:99, mx = my = 16)
constexpr int TN = TILE + 1;  // nodes per tile side
constexpr int NCOMP = 8;  // x, y, px, py, pz, p6, p7, q  (ppart(1..8))

// Structure-of-arrays particle buffer.
struct PartBuf {
  float* c[NCOMP];
  int* count;  // per tile
  int cap;     // slots per tile
};

// Movers in flight to their destination tile (filled by the push, drained by
// the insert kernel).
struct Inbox {
  float* c[NCOMP];
  unsigned long long* key;  // cell << 48 | source tile << 24 | source slot: deterministic order
  int* count;     // per destination tile
  int cap;        // slots per tile
};

struct TileGeom {
  int nx, ny, mx1, myp1, ntiles;
  int rp;
};

// field planes a particle kernel gathers from (real space)
struct GatherPlanes {
  const float* fx;   // fxy(1)
  const float* fy;   // fxy(2)
  const float* bx;   // bxyz(1)
  const float* by;   // bxyz(2)
  const float* bz;   // bxyz(3)
  const float* psit; // psit
  int combine;       // 1: the push uses -fxy + (by, -bx), the final slice force
  const float* psi;  // amjdp only, optional: form p6, p7 from psi first (extpsi)
  int pass;          // amjdp only: predictor-corrector pass (pass_skipped), 0 = none
  float* zero_q;     // push only, optional: clear the charge-plane nodes this tile
                     // owns (k_insert then deposits the next slice's charge)
};

int part_kernels_init();
// places the static scratch of qp_pmove_static on the current device (qp_noalloc.cu)
int pmove_static_reserve();
void launch_deposit_rho(const PartBuf& P, const TileGeom& tg, float* q, const DevStatus* st,
                        cudaStream_t s);
void launch_extpsi(const PartBuf& P, const TileGeom& tg, const float* psi, float qbm, float dex,
                   const DevStatus* st, cudaStream_t s);
void launch_amjdp(const PartBuf& P, const TileGeom& tg, const GatherPlanes& f, float* const* acc,
                  float qbm, float dt, float dex, float scale, const DevStatus* st,
                  cudaStream_t s);
// mode 0: push in place (partpush); 1: push A -> B with re-binning (push + pmove);
// 2: re-bin only (pmove) A -> B
void launch_push(int mode, const PartBuf& A, const PartBuf& B, const Inbox& ib,
                 const TileGeom& tg, const GatherPlanes& f, float qbm, float dt, float dex,
                 DevStatus* st, cudaStream_t s);
// deposit_q (optional): after the re-bin, deposit the charge of every
// particle of the tile into deposit_q (zero on entry), as k_deposit_rho does
void launch_insert(const PartBuf& B, const Inbox& ib, const TileGeom& tg, DevStatus* st,
                   cudaStream_t s, float* deposit_q = nullptr);

}  // namespace qp
