// qp_noalloc.cu -- particle re-binning (pmove) that allocates no device memory.
//
// Who needs this: a host code that hands all of a GPU's memory to its own
// allocator at start-up (a Fortran PIC driver that sizes its field and
// particle arrays once and then runs a time loop, or a job that shares the GPU
// under a fixed memory budget) cannot call cudaMalloc in the middle of a step:
// the memory may simply not be there, and cudaMalloc/cudaFree also stall the
// device while other streams are working.  Such a caller owns the particle
// buffers it passes in and out, but has nowhere to put the re-binning's own
// scratch (the mover inbox, its sort keys and the error status).
//
// qp_pmove_static runs the same two kernels as qp_species_pmove (the re-bin
// pass of k_push and the sorted insert, qp_part.cu), with that scratch carved
// out of one fixed array that lives in this file.  Every GPU on which this
// module is loaded holds the array until the process exits.
#include <mutex>
#include <string>

#include "qp_common.cuh"
#include "qp_part.cuh"
#include "../../include/qpgpu.h"

using namespace qp;

namespace {

// The scratch: the device status, then the per-tile inbox counts, the sort
// keys and the eight component planes of the inbox.  In host code this name is
// only a handle for the runtime; the device address comes from
// cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_pmove_scratch[QP_PMOVE_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
constexpr int kMaxInboxCap = 16384;  // the insert kernel sorts at most this many keys per tile
constexpr size_t kBytesPerMover = NCOMP * sizeof(float) + sizeof(unsigned long long);

std::mutex g_setup_mutex;
bool g_attr_done[kMaxDevices] = {};

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

int reject(int line, const std::string& msg) {
  qp_set_error("qp_noalloc.cu", line, msg.c_str());
  return -1;
}

// The scratch's device address on the current device.  The runtime loads this
// file's module (and places the array) at the first use of one of its symbols,
// so the lookup is what reserves the array on a device; it is repeated on
// every call, which keeps the address right after a context is torn down and
// re-created (cudaDeviceReset).
int scratch_address(unsigned char** out) {
  void* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_pmove_scratch);
  if (e != cudaSuccess)
    return reject(__LINE__, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  *out = static_cast<unsigned char*>(ptr);
  return 0;
}

// Once per device, with that device current: the insert kernel's
// shared-memory limit (a function attribute; it allocates nothing).
int setup_device(int dev) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_attr_done[dev]) {
    if (part_kernels_init() != 0) return reject(__LINE__, "insert kernel attribute set-up failed");
    g_attr_done[dev] = true;
  }
  return 0;
}

// A caller-supplied count outside [0, cap] would make the re-bin kernel read
// beyond its tile: flag it so that the following kernels return at once.
__global__ void k_check_counts(const int* count, int ntiles, int cap, DevStatus* st) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    const int c = count[t];
    if (c < 0 || c > cap) {
      atomicCAS(&st->error, 0, -5);
      atomicMax(&st->need_cap, c);
    }
  }
}

}  // namespace

namespace qp {
// Places the static scratch on the current device now, so that a caller who
// creates a context before handing the rest of the GPU's memory to its own
// allocator has the array reserved before that allocator takes its pool.
int pmove_static_reserve() {
  unsigned char* base = nullptr;
  return scratch_address(&base);
}
}  // namespace qp

extern "C" int qp_pmove_static(int indx, int indy, const float* const* part_in,
                               const int* count_in, int cap_in, float* const* part_out,
                               int* count_out, int cap_out, void* stream) {
  if (indx < 4 || indy < 4 || indx > QP_MAX_IND || indy > QP_MAX_IND)
    return reject(__LINE__, "pmove_static: indx and indy must lie in 4.." +
                                std::to_string(QP_MAX_IND));
  if (!part_in || !part_out || !count_in || !count_out)
    return reject(__LINE__, "pmove_static: null argument");
  if (cap_in < 1 || cap_out < 1) return reject(__LINE__, "pmove_static: capacities must be >= 1");
  for (int c = 0; c < NCOMP; ++c) {
    if (!part_in[c] || !part_out[c]) return reject(__LINE__, "pmove_static: null plane");
    if (part_in[c] == part_out[c]) return reject(__LINE__, "pmove_static: input and output alias");
  }
  if (count_in == count_out) return reject(__LINE__, "pmove_static: input and output alias");

  TileGeom tg{};
  tg.nx = 1 << indx;
  tg.ny = 1 << indy;
  tg.mx1 = (tg.nx - 1) / TILE + 1;
  tg.myp1 = (tg.ny - 1) / TILE + 1;
  tg.ntiles = tg.mx1 * tg.myp1;
  tg.rp = tg.nx + 4;

  // carve the scratch; the inbox gets what is left after the status and counts
  const size_t off_count = align256(sizeof(DevStatus));
  const size_t off_key = off_count + align256(sizeof(int) * (size_t)tg.ntiles);
  const size_t room = QP_PMOVE_STATIC_SCRATCH_BYTES > off_key + 256 * (NCOMP + 1)
                          ? QP_PMOVE_STATIC_SCRATCH_BYTES - off_key - 256 * (NCOMP + 1)
                          : 0;
  long long capin = (long long)(room / (kBytesPerMover * (size_t)tg.ntiles));
  if (capin > kMaxInboxCap) capin = kMaxInboxCap;
  capin &= ~3LL;
  if (capin < QP_PMOVE_STATIC_MIN_INBOX)
    return reject(__LINE__, "pmove_static: a " + std::to_string(tg.nx) + " x " +
                                std::to_string(tg.ny) + " grid has " +
                                std::to_string(tg.ntiles) + " tiles, more than the " +
                                std::to_string(QP_PMOVE_STATIC_SCRATCH_BYTES >> 20) +
                                " MiB static scratch can serve");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return reject(__LINE__, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return reject(__LINE__, "pmove_static: device index too large");
  unsigned char* base = nullptr;
  if (setup_device(dev) || scratch_address(&base)) return -1;

  DevStatus* st = reinterpret_cast<DevStatus*>(base);
  Inbox ib{};
  ib.cap = (int)capin;
  ib.count = reinterpret_cast<int*>(base + off_count);
  ib.key = reinterpret_cast<unsigned long long*>(base + off_key);
  size_t off = off_key + align256(sizeof(unsigned long long) * (size_t)tg.ntiles * ib.cap);
  for (int c = 0; c < NCOMP; ++c) {
    ib.c[c] = reinterpret_cast<float*>(base + off);
    off += align256(sizeof(float) * (size_t)tg.ntiles * ib.cap);
  }
  if (off > QP_PMOVE_STATIC_SCRATCH_BYTES) return reject(__LINE__, "pmove_static: scratch layout");

  PartBuf A{}, B{};
  for (int c = 0; c < NCOMP; ++c) {
    A.c[c] = const_cast<float*>(part_in[c]);
    B.c[c] = part_out[c];
  }
  A.count = const_cast<int*>(count_in);
  A.cap = cap_in;
  B.count = count_out;
  B.cap = cap_out;

  // the array keeps the previous call's contents: the status and the inbox
  // counts must start at zero
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if ((e = cudaMemsetAsync(st, 0, sizeof(DevStatus), s)) != cudaSuccess ||
      (e = cudaMemsetAsync(ib.count, 0, sizeof(int) * (size_t)tg.ntiles, s)) != cudaSuccess)
    return reject(__LINE__, cudaGetErrorString(e));
  k_check_counts<<<(tg.ntiles + 255) / 256, 256, 0, s>>>(count_in, tg.ntiles, cap_in, st);
  GatherPlanes f{};
  launch_push(2, A, B, ib, tg, f, 0.f, 1.f, 1.f, st, s);
  launch_insert(B, ib, tg, st, s);
  if ((e = cudaGetLastError()) != cudaSuccess) return reject(__LINE__, cudaGetErrorString(e));
  DevStatus h{};
  if ((e = cudaMemcpyAsync(&h, st, sizeof(DevStatus), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return reject(__LINE__, cudaGetErrorString(e));
  if (h.error == 0) return 0;
  if (h.error == -5)
    return reject(__LINE__, "pmove_static: a tile count lies outside 0.." +
                                std::to_string(cap_in) + " (found " +
                                std::to_string(h.need_cap) + ")");
  if (h.error == -4 || h.error == -3)
    return reject(__LINE__, "pmove_static: a particle position lies outside the grid (code " +
                                std::to_string(h.error) + ")");
  if (h.error == -6)
    return reject(__LINE__, "pmove_static: internal error, a tile's stayer count left its "
                            "slots (code -6)");
  if (h.error < 0)
    return reject(__LINE__, "pmove_static: internal error in the re-bin kernels (code " +
                                std::to_string(h.error) + ")");
  if (h.need_inbox > ib.cap)
    return reject(__LINE__, "pmove_static: " + std::to_string(h.need_inbox) +
                                " particles moved into one tile; the static scratch holds " +
                                std::to_string(ib.cap) + " per tile on this grid");
  return reject(__LINE__, "pmove_static: cap_out " + std::to_string(cap_out) +
                              " too small, a tile needs " + std::to_string(h.need_cap));
}
