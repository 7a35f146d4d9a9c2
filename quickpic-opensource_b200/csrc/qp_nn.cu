// qp_nn.cu -- the learned start of the B predictor-corrector: a 5-layer 3x3
// convolutional network (32 channels, BF16 weights and activations, FP32
// accumulation) on Fourier-space images, with its forward, data-gradient and
// weight-gradient kernels written on the Blackwell tensor cores (tcgen05.mma
// with the accumulator in tensor memory, operand tiles brought in by TMA), its
// training loop (Adam) and its use in the fused step.  It has no counterpart in
// the reference: it replaces the start of the pass loop (simulation_class.f03:676),
// where the reference starts slice j from the B_perp iterate of slice j-1.
//
// Why Fourier space: the quasi-static field equations are diagonal in the
// sine/cosine basis (each mode of B_perp answers the same mode of the current,
// through the form factor of fpois2d), so a network with an 11 x 11-mode
// receptive field sees the whole of the relation it has to learn, where in real
// space the same relation is a global Poisson solve.  The mode coordinates are
// input channels, so the network can learn the k-dependence.
//
// Convolution as an implicit GEMM (one CTA = 128 output pixels of one image row):
//   D[128 px][Cout] = sum over 9 taps and Cin:  X[px + shift(tap)][cin] W[tap][cin][cout]
// The input halo (3 rows x 130 pixels x Cin) is one TMA box of the
// channel-group-planar image [G][NB][H][W][8]; out-of-image rows and columns
// are filled with zeros by the TMA unit (the convolution's zero padding).  In
// shared memory the halo is [G][3][130][8] bf16, so 8 consecutive pixels of one
// channel group are 128 contiguous bytes: one core matrix of a K-major operand
// without swizzle.  The A operand of tap (dy, dx) is that tile addressed from
// start + (dy*130 + dx)*16 bytes, with the stride between channel groups as the
// K-direction core-matrix offset (LBO) and 128 bytes between 8-pixel groups
// (SBO).  B (the weights, Cout x 9*Cin) is staged once per CTA in the canonical
// K-major layout.  One thread issues the 9*Cin/16 MMAs (M=128, N=Cout, K=16)
// into a 32-column TMEM accumulator, commits them to an mbarrier, and the four
// warps read their 32 TMEM lanes back (tcgen05.ld 32x32b) for the epilogue.
// The halo of the CTA's next tile is loaded while the current one is computed.
//
// Weight gradient: dW[tap][cin][cout] = sum_px X[px + shift(tap)][cin] dY[px][cout],
// per tap a GEMM with M = cout, N = cin, K = pixels.  The reduction runs over
// pixels, so the threads first rewrite the TMA-loaded tiles as K-major
// operands (8 consecutive pixels of one channel in 16 bytes): dY as
// A[cout][pixels] and, for each of the 9 taps, the shifted window of X as
// B[cin][pixels].  M is padded to 128 (rows >= cout are zeros and are
// discarded); the 9 taps accumulate in 9 * cin TMEM columns over every tile of
// the CTA, and are added to the FP32 gradient once at the end.
//
// Every wait on an mbarrier is bounded (about 1 s of %globaltimer); on expiry
// the kernel records an error, waits (bounded) for its own copies and MMAs in
// flight, frees its tensor memory and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "qp_nn.cuh"
#include "../../include/qpgpu.h"

namespace qp {

int nn_total_params() {
  int n = 0;
  for (int l = 0; l < NN_LAYERS; ++l) n += nn_layer_params(l);
  return n;
}

namespace {

constexpr int TM = 128;             // output pixels per tile
constexpr int HW_ = TM + 2;         // halo width
constexpr int HALO_G = 3 * HW_ * 16;  // bytes of one channel group of the halo
constexpr uint64_t WAIT_NS = 1000000000ull;

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t su32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false after about WAIT_NS without the phase completing
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
  uint64_t t0 = 0;
  for (uint32_t i = 0;; ++i) {
    if (mbar_try(b, parity)) return true;
    if ((i & 255u) == 255u) {
      const uint64_t t = gtimer();
      if (t0 == 0) t0 = t;
      else if (t - t0 > WAIT_NS) return false;
    }
  }
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// TMA: a 5D box (8 channels, w pixels, h rows, 1 image, g groups) of the
// channel-group-planar image into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load5(void* dst, const CUtensorMap* map, uint64_t* bar, int x,
                                          int y, int b) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(su32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(x), "r"(y), "r"(b), "r"(0),
      "r"(su32(bar))
      : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   su32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// shared-memory matrix descriptor, no swizzle (layout type 0), sm100 version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor of kind::f16: BF16 x BF16 -> F32, M x N, majors
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          su32(bar))
      : "memory");
}
#define QP_TLD16(r, addr)                                                                     \
  asm volatile(                                                                               \
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13," \
      "%14,%15}, [%16];"                                                                      \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),  \
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),           \
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])                                                 \
      : "r"(addr))
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ void unpack8(uint4 u, float* f) {
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float2 v = __bfloat1622float2(h[i]);
    f[2 * i] = v.x;
    f[2 * i + 1] = v.y;
  }
}

// The start the network corrects: the quadratic extrapolation of the three
// previous slices' B_perp, per mode (the engine's predict = 2 start).
__device__ __forceinline__ float nn_base(float e1, float e0, float em) {
  return 3.f * (e1 - e0) + em;
}

// The network's correction of a mode, bounded: at most the size of the
// extrapolation step itself plus 5 % of the mode, and 0 if it is not finite.
// Out of its training distribution the network can then move the start only
// within the neighbourhood the extrapolation already spans; the passes that
// follow run to the tolerance from wherever the start is.
__device__ __forceinline__ float nn_bounded(float d, float step, float e1) {
  const float lim = fabsf(step) + 0.05f * fabsf(e1);
  if (!(fabsf(d) <= 3.0e38f)) return 0.f;
  return fminf(fmaxf(d, -lim), lim);
}

// ---------------------------------------------------------------- the kernels
enum { EPI_RELU = 0, EPI_MASK = 1, EPI_F32 = 2, EPI_EPW = 3 };

struct ConvArgs {
  const __nv_bfloat16* w;     // B operand in the canonical K-major layout (Cout x 9 Cin)
  const float* bias;          // Cout, or null
  __nv_bfloat16* out;         // EPI_RELU / EPI_MASK: [Cout/8][NB][H][W][8]
  const __nv_bfloat16* mask;  // EPI_MASK: the layer input [Cout/8][NB][H][W][8]
  float* out32;               // EPI_F32: [NB][2][H][W]
  NNSlicePlanes pl;           // EPI_EPW: the k-space planes
  const float* scale;         // EPI_EPW: scale[0] = the epw scale of this slice
  int kp;                     // EPI_EPW: k-space pitch
  int nx, ny;                 // EPI_EPW: grid
  int H, W, NB;               // output images (NB images of H x W)
  int b0;                     // first image of the launch in the input map
  int* err;                   // device error flag (nonzero on a wait that expired)
};

__device__ __forceinline__ void flag_error(int* err, int code) {
  if (err) atomicCAS(err, 0, code);
}

// One 3x3 convolution layer (stride 1, zero padding).  CIN, COUT in {16, 32}.
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(128) k_conv3x3(const __grid_constant__ CUtensorMap tin,
                                                 ConvArgs a) {
  constexpr int GIN = CIN / 8;
  constexpr int KSTEPS = 9 * CIN / 16;
  constexpr int WBYTES = COUT * 9 * CIN * 2;
  constexpr int HALO_BYTES = GIN * HALO_G;
  constexpr int HB = (HALO_BYTES + 127) & ~127;
  constexpr uint32_t LBO_B = (COUT / 8) * 128;
  constexpr uint32_t IDESC = idesc_bf16(128, COUT, 0, 0);
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* wsm = sm;
  unsigned char* halo[2] = {sm + WBYTES, sm + WBYTES + HB};
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + WBYTES + 2 * HB);  // [0,1] tma, [2] mma
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 3);
  int* s_err = reinterpret_cast<int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int segs = a.W / TM;
  const int ntiles = a.NB * a.H * segs;

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    *s_err = 0;
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(tslot, 32);
  // weights: global image of the shared layout, 16 bytes per thread and step
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.w);
    uint4* dst = reinterpret_cast<uint4*>(wsm);
    for (int i = tid; i < WBYTES / 16; i += 128) dst[i] = src[i];
  }
  fence_async_smem();
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tbase = *tslot;

  auto tile_coord = [&](int t, int& b, int& y, int& x0) {
    const int per = a.H * segs;
    b = t / per;
    const int r = t - b * per;
    y = r / segs;
    x0 = (r - y * segs) * TM;
  };
  auto issue = [&](int t, int buf) {
    int b, y, x0;
    tile_coord(t, b, y, x0);
    mbar_expect_tx(&bar[buf], (uint32_t)HALO_BYTES);
    tma_load5(halo[buf], &tin, &bar[buf], x0 - 1, y - 1, a.b0 + b);
  };

  int k = 0;
  // thread 0's record of what it has in flight, for the error path
  int pf_buf = -1, pf_k = 0;    // a prefetch not yet waited for: buffer and tile number
  bool mma_out = false;         // MMAs committed and not yet seen complete
  if (tid == 0 && (int)blockIdx.x < ntiles) {
    issue(blockIdx.x, 0);
    pf_buf = 0;
    pf_k = 0;
  }
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
    const int buf = k & 1;
    if (tid == 0) {
      const int tn = t + gridDim.x;
      if (mbar_wait(&bar[buf], (uint32_t)((k >> 1) & 1))) {
        pf_buf = -1;
        if (tn < ntiles) {  // the other buffer was freed by the previous tile's MMAs
          issue(tn, buf ^ 1);
          pf_buf = buf ^ 1;
          pf_k = k + 1;
        }
        tc_after();
        const uint32_t hbase = su32(halo[buf]);
        const uint32_t wbase = su32(wsm);
#pragma unroll 1
        for (int s = 0; s < KSTEPS; ++s) {
          const int tap = s / (CIN / 16), h = s - tap * (CIN / 16);
          const int dy = tap / 3, dx = tap - dy * 3;
          const uint32_t aa = hbase + (uint32_t)(2 * h * HALO_G + (dy * HW_ + dx) * 16);
          const uint64_t ad = sdesc(aa, HALO_G, 128);
          const uint64_t bd = sdesc(wbase + (uint32_t)(2 * s) * LBO_B, LBO_B, 128);
          mma_bf16(tbase, ad, bd, IDESC, s > 0 ? 1u : 0u);
        }
        mma_commit(&bar[2]);
        mma_out = true;
      } else {
        *s_err = 1;  // the halo never arrived: no MMA issued for this tile
      }
    }
    __syncthreads();
    if (*s_err) break;
    // every thread waits for the accumulator (bounded)
    if (!mbar_wait(&bar[2], (uint32_t)(k & 1))) atomicExch(s_err, 1);
    __syncthreads();
    if (*s_err) break;
    if (tid == 0) mma_out = false;
    tc_after();
    int b, y, x0;
    tile_coord(t, b, y, x0);
    const int x = x0 + warp * 32 + lane;
    float acc[32];
    {
      uint32_t r[16];
      const uint32_t ta = tbase + ((uint32_t)(warp * 32) << 16);
      QP_TLD16(r, ta);
#pragma unroll
      for (int i = 0; i < 16; ++i) acc[i] = __uint_as_float(r[i]);
      if (COUT == 32) {
        QP_TLD16(r, ta + 16);
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[16 + i] = __uint_as_float(r[i]);
      }
      tmem_wait_ld();
    }
    if (EPI == EPI_RELU || EPI == EPI_MASK) {
#pragma unroll
      for (int g = 0; g < COUT / 8; ++g) {
        const size_t o = ((((size_t)g * a.NB + b) * a.H + y) * a.W + x) * 8;
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = acc[8 * g + i] + (a.bias ? a.bias[8 * g + i] : 0.f);
        if (EPI == EPI_RELU) {
#pragma unroll
          for (int i = 0; i < 8; ++i) v[i] = fmaxf(v[i], 0.f);
        } else {
          float m[8];
          unpack8(*reinterpret_cast<const uint4*>(a.mask + o), m);
#pragma unroll
          for (int i = 0; i < 8; ++i) v[i] = m[i] > 0.f ? v[i] : 0.f;
        }
        uint4 u;
        u.x = pack_bf16(v[0], v[1]);
        u.y = pack_bf16(v[2], v[3]);
        u.z = pack_bf16(v[4], v[5]);
        u.w = pack_bf16(v[6], v[7]);
        *reinterpret_cast<uint4*>(a.out + o) = u;
      }
    } else if (EPI == EPI_F32) {
#pragma unroll
      for (int c = 0; c < NN_OUT; ++c)
        a.out32[(((size_t)b * NN_OUT + c) * a.H + y) * a.W + x] =
            acc[c] + (a.bias ? a.bias[c] : 0.f);
    } else {  // EPI_EPW: pixel (y, x) = mode (kx, ky); start of the slice's passes
      const int kx = y, ky = x;
      const size_t o = (size_t)kx * a.kp + ky;
      const float sB = a.scale[0];
      const float e1x = a.pl.epw_x[o], e1y = a.pl.epw_y[o];
      const float e0x = a.pl.prev_x[o], e0y = a.pl.prev_y[o];
      const float emx = a.pl.prev2_x[o], emy = a.pl.prev2_y[o];
      a.pl.prev2_x[o] = e0x;
      a.pl.prev2_y[o] = e0y;
      a.pl.prev_x[o] = e1x;
      a.pl.prev_y[o] = e1y;
      float px = nn_base(e1x, e0x, emx), py = nn_base(e1y, e0y, emy);
      if (kx >= 1 && ky >= 1) {  // the modes kx = 0, ky = 0 take the extrapolation alone
        px += nn_bounded(sB * (acc[0] + a.bias[0]), px - e1x, e1x);
        py += nn_bounded(sB * (acc[1] + a.bias[1]), py - e1y, e1y);
      }
      a.pl.epw_x[o] = px;
      a.pl.epw_y[o] = py;
    }
    tc_before();
    __syncthreads();
  }
  if (tid == 0 && *s_err) {
    // let this CTA's own copies and MMAs in flight land before its shared and
    // tensor memory are released (each wait bounded again)
    if (pf_buf >= 0) mbar_wait(&bar[pf_buf], (uint32_t)((pf_k >> 1) & 1));
    if (mma_out) mbar_wait(&bar[2], (uint32_t)(k & 1));
    flag_error(a.err, 1);
  }
  // EPI_EPW: the modes outside the conv image (the network's low-mode window)
  // take the quadratic extrapolation alone, spread over every CTA
  if (EPI == EPI_EPW && !*s_err) {
    const long long nm = (long long)(a.nx + 1) * (a.ny + 1);
    for (long long i = (long long)blockIdx.x * 128 + tid; i < nm; i += (long long)gridDim.x * 128) {
      const int kx = (int)(i / (a.ny + 1)), ky = (int)(i - (long long)kx * (a.ny + 1));
      if (kx < a.H && ky < a.W) continue;
      const size_t o = (size_t)kx * a.kp + ky;
      const float e1x = a.pl.epw_x[o], e1y = a.pl.epw_y[o];
      const float e0x = a.pl.prev_x[o], e0y = a.pl.prev_y[o];
      const float emx = a.pl.prev2_x[o], emy = a.pl.prev2_y[o];
      a.pl.prev2_x[o] = e0x;
      a.pl.prev2_y[o] = e0y;
      a.pl.prev_x[o] = e1x;
      a.pl.prev_y[o] = e1y;
      a.pl.epw_x[o] = nn_base(e1x, e0x, emx);
      a.pl.epw_y[o] = nn_base(e1y, e0y, emy);
    }
  }
  __syncthreads();
  if (warp == 0) tmem_dealloc(tbase, 32);
}


// ---------------------------------------------------------- weight gradient
struct WgradArgs {
  float* dw;        // [9][CIN][COUT] fp32, accumulated
  float* db;        // [COUT] fp32, accumulated
  const __nv_bfloat16* dy;  // the tile's dY (for the bias sums through shared memory)
  int couts;        // output channels that exist (the rest are padding)
  int H, W, NB;     // dY images
  int xb0;          // first image of the launch in the X map
  int* err;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_wgrad(const __grid_constant__ CUtensorMap tx,
                                               const __grid_constant__ CUtensorMap tdy,
                                               WgradArgs a) {
  constexpr int GIN = CIN / 8, GOUT = COUT / 8;
  constexpr int HALO_BYTES = GIN * HALO_G;
  constexpr int DY_BYTES = GOUT * TM * 16;
  constexpr int DY_OFF = (HALO_BYTES + 127) & ~127;               // TMA destinations 128-aligned
  constexpr int STG = ((DY_OFF + DY_BYTES) + 127) & ~127;        // one staging buffer
  constexpr int AT_BYTES = (TM / 8) * 128 * 16;                 // [16 pixel groups][128 rows][8]
  constexpr int XT_ONE = (TM / 8) * CIN * 16;                   // [16 pixel groups][CIN][8]
  constexpr uint32_t TCOLS = CIN == 32 ? 512 : 256;
  constexpr uint32_t IDESC = idesc_bf16(128, CIN, 0, 0);
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* stg[2] = {sm, sm + STG};
  unsigned char* at = sm + 2 * STG;
  unsigned char* xt = at + AT_BYTES;  // 9 copies, (dx, dy) major
  uint64_t* bar = reinterpret_cast<uint64_t*>(xt + 9 * XT_ONE);  // [0,1] tma, [2] mma
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 3);
  int* s_err = reinterpret_cast<int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int segs = a.W / TM;
  const int ntiles = a.NB * a.H * segs;

  if (tid == 0) {
    for (int i = 0; i < 3; ++i) mbar_init(&bar[i], 1);
    *s_err = 0;
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(tslot, TCOLS);
  {  // the rows of the A operand past the real output channels stay zero
    uint4* z = reinterpret_cast<uint4*>(at);
    for (int i = tid; i < AT_BYTES / 16; i += 128) z[i] = make_uint4(0, 0, 0, 0);
  }
  fence_async_smem();
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tbase = *tslot;

  auto tile_coord = [&](int t, int& b, int& y, int& x0) {
    const int per = a.H * segs;
    b = t / per;
    const int r = t - b * per;
    y = r / segs;
    x0 = (r - y * segs) * TM;
  };
  auto issue = [&](int t, int buf) {
    int b, y, x0;
    tile_coord(t, b, y, x0);
    mbar_expect_tx(&bar[buf], (uint32_t)(HALO_BYTES + DY_BYTES));
    tma_load5(stg[buf], &tx, &bar[buf], x0 - 1, y - 1, a.xb0 + b);
    tma_load5(stg[buf] + DY_OFF, &tdy, &bar[buf], x0, y, b);
  };

  float bsum = 0.f;  // thread c < COUT: sum of dY channel c
  int k = 0;
  int pf_buf = -1, pf_k = 0;
  int mma_last = -1;
  bool mma_seen = true;
  if (tid == 0 && (int)blockIdx.x < ntiles) {
    issue(blockIdx.x, 0);
    pf_buf = 0;
    pf_k = 0;
  }
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
    const int buf = k & 1;
    if (tid == 0) {
      // this tile's operands, and the transposed buffers free of the last tile's MMAs
      if (!mbar_wait(&bar[buf], (uint32_t)((k >> 1) & 1))) {
        *s_err = 1;
      } else {
        pf_buf = -1;
        if (mma_last >= 0 && !mma_seen) {
          if (mbar_wait(&bar[2], (uint32_t)(mma_last & 1))) mma_seen = true;
          else *s_err = 1;
        }
      }
    }
    __syncthreads();
    if (*s_err) break;
    if (tid == 0 && t + (int)gridDim.x < ntiles) {
      issue(t + gridDim.x, buf ^ 1);
      pf_buf = buf ^ 1;
      pf_k = k + 1;
    }
    // K-major operands from the channel-group tiles: A[cout][8 pixels] and,
    // for each tap, B[cin][8 pixels] of the shifted window
    const __nv_bfloat16* hx = reinterpret_cast<const __nv_bfloat16*>(stg[buf]);
    const __nv_bfloat16* hy = reinterpret_cast<const __nv_bfloat16*>(stg[buf] + DY_OFF);
    for (int it = tid; it < COUT * (TM / 8); it += 128) {
      const int m = it % COUT, kg = it / COUT;
      uint32_t w[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int p0 = kg * 8 + 2 * j;
        const __nv_bfloat16 v0 = hy[((m >> 3) * TM + p0) * 8 + (m & 7)];
        const __nv_bfloat16 v1 = hy[((m >> 3) * TM + p0 + 1) * 8 + (m & 7)];
        w[j] = (uint32_t)__bfloat16_as_ushort(v0) | ((uint32_t)__bfloat16_as_ushort(v1) << 16);
      }
      *reinterpret_cast<uint4*>(at + ((size_t)kg * 128 + m) * 16) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    for (int it = tid; it < 9 * (TM / 8) * CIN; it += 128) {
      const int n = it % CIN, r = it / CIN, kg = r % (TM / 8), tap = r / (TM / 8);
      const int dy = tap / 3, dx = tap - dy * 3;
      uint32_t w[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int p0 = dy * HW_ + kg * 8 + 2 * j + dx;
        const __nv_bfloat16 v0 = hx[((n >> 3) * 3 * HW_ + p0) * 8 + (n & 7)];
        const __nv_bfloat16 v1 = hx[((n >> 3) * 3 * HW_ + p0 + 1) * 8 + (n & 7)];
        w[j] = (uint32_t)__bfloat16_as_ushort(v0) | ((uint32_t)__bfloat16_as_ushort(v1) << 16);
      }
      *reinterpret_cast<uint4*>(xt + (size_t)tap * XT_ONE + ((size_t)kg * CIN + n) * 16) =
          make_uint4(w[0], w[1], w[2], w[3]);
    }
    if (tid < COUT) {
      for (int p = 0; p < TM; ++p) bsum += __bfloat162float(hy[((tid >> 3) * TM + p) * 8 + (tid & 7)]);
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_after();
      const uint32_t ab = su32(at), xb = su32(xt);
#pragma unroll 1
      for (int q = 0; q < TM / 16; ++q)
#pragma unroll 1
        for (int tap = 0; tap < 9; ++tap) {
          const uint64_t ad = sdesc(ab + (uint32_t)(2 * q * 128 * 16), 128 * 16, 128);
          const uint64_t bd =
              sdesc(xb + (uint32_t)(tap * XT_ONE + 2 * q * CIN * 16), CIN * 16, 128);
          mma_bf16(tbase + (uint32_t)(tap * CIN), ad, bd, IDESC, (k > 0 || q > 0) ? 1u : 0u);
        }
      mma_commit(&bar[2]);
      mma_last = k;
      mma_seen = false;
    }
  }
  if (tid == 0) {
    if (!*s_err && mma_last >= 0 && !mma_seen) {
      if (mbar_wait(&bar[2], (uint32_t)(mma_last & 1))) mma_seen = true;
      else *s_err = 2;
    }
    if (*s_err) {
      if (pf_buf >= 0) mbar_wait(&bar[pf_buf], (uint32_t)((pf_k >> 1) & 1));
      if (mma_last >= 0 && !mma_seen) mbar_wait(&bar[2], (uint32_t)(mma_last & 1));
      flag_error(a.err, 2);
    }
  }
  __syncthreads();
  // every CTA of the grid has at least one tile; the condition must be the
  // same in all 32 lanes of warp 0, whose tcgen05.ld is warp-synchronous
  // (mma_last is known to thread 0 only)
  if (!*s_err && (int)blockIdx.x < ntiles) {
    tc_after();
    if (warp == 0) {  // TMEM lanes 0..31 hold the rows cout = 0..31
      for (int tap = 0; tap < 9; ++tap)
        for (int c0 = 0; c0 < CIN; c0 += 16) {
          uint32_t r[16];
          QP_TLD16(r, tbase + (uint32_t)(tap * CIN + c0));
          tmem_wait_ld();
          if (lane < a.couts)
            for (int i = 0; i < 16; ++i)
              atomicAdd(&a.dw[((size_t)tap * CIN + c0 + i) * COUT + lane], __uint_as_float(r[i]));
        }
    }
    if (tid < a.couts) atomicAdd(&a.db[tid], bsum);
  }
  tc_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tbase, TCOLS);
}

// ------------------------------------------------------- features and records
__global__ void k_nn_norms(NNSlicePlanes p, int nx, int ny, int kp, float* part) {
  __shared__ float red[3][8];
  float sb = 0.f, sj = 0.f, sz = 0.f;
  const long long n = (long long)(nx + 1) * (ny + 1);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(i / (ny + 1)), ky = (int)(i - (long long)kx * (ny + 1));
    const size_t o = (size_t)kx * kp + ky;
    const float ex = p.epw_x[o], ey = p.epw_y[o];
    const float cx = p.cu_x[o], cy = p.cu_y[o], cz = p.cu_z[o];
    sb += ex * ex + ey * ey;
    sj += cx * cx + cy * cy;
    sz += cz * cz;
  }
  for (int off = 16; off; off >>= 1) {
    sb += __shfl_xor_sync(0xffffffffu, sb, off);
    sj += __shfl_xor_sync(0xffffffffu, sj, off);
    sz += __shfl_xor_sync(0xffffffffu, sz, off);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = sb;
    red[1][w] = sj;
    red[2][w] = sz;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    float v = 0.f;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v += red[threadIdx.x][i];
    part[3 * blockIdx.x + threadIdx.x] = v;
  }
}

// scales of the slice from the norm partials: epw, current (x, y), current z
__device__ void nn_scales(const float* part, int nx, int ny, float* sc) {
  if (threadIdx.x < 3) {
    float v = 0.f;
    for (int i = 0; i < NN_NORM_BLOCKS; ++i) v += part[3 * i + threadIdx.x];
    const float cnt = (float)(nx + 1) * (float)(ny + 1) * (threadIdx.x < 2 ? 2.f : 1.f);
    const float r = sqrtf(v / cnt);
    sc[threadIdx.x] = r > 1e-30f ? r : 0.f;
  }
  __syncthreads();
}

__device__ __forceinline__ float safe_div(float v, float s) { return s > 0.f ? v / s : 0.f; }

// the 16 input channels of mode (kx, ky): e1, e1 - e0, e0 - em1 (em1 = e(-1)),
// cu, coordinates, zeros
__device__ __forceinline__ void nn_feature(const NNSlicePlanes& p, size_t o, int kx, int ky,
                                           int nx, int ny, const float* sc, float e1x, float e1y,
                                           float e0x, float e0y, float emx, float emy, uint4* g0,
                                           uint4* g1) {
  float f[16];
  f[0] = safe_div(e1x, sc[0]);
  f[1] = safe_div(e1y, sc[0]);
  f[2] = safe_div(e1x - e0x, sc[0]);
  f[3] = safe_div(e1y - e0y, sc[0]);
  f[4] = safe_div(e0x - emx, sc[0]);
  f[5] = safe_div(e0y - emy, sc[0]);
  f[6] = safe_div(p.cu_x[o], sc[1]);
  f[7] = safe_div(p.cu_y[o], sc[1]);
  f[8] = safe_div(p.cu_z[o], sc[2]);
  f[9] = (float)kx / (float)nx;
  f[10] = (float)ky / (float)ny;
  f[11] = p.dxi * 25.6f;
  for (int i = NN_FEATURES; i < 16; ++i) f[i] = 0.f;
  g0->x = pack_bf16(f[0], f[1]);
  g0->y = pack_bf16(f[2], f[3]);
  g0->z = pack_bf16(f[4], f[5]);
  g0->w = pack_bf16(f[6], f[7]);
  g1->x = pack_bf16(f[8], f[9]);
  g1->y = pack_bf16(f[10], f[11]);
  g1->z = pack_bf16(f[12], f[13]);
  g1->w = pack_bf16(f[14], f[15]);
}

// inference: the input image [2][1][hc][wc][8] of the slice's low-mode
// window kx < hc, ky < wc; scale_out = the epw scale
__global__ void k_nn_features(NNSlicePlanes p, int nx, int ny, int kp, int hc, int wc,
                              const float* part, __nv_bfloat16* img, float* scale_out) {
  __shared__ float sc[3];
  nn_scales(part, nx, ny, sc);
  if (blockIdx.x == 0 && threadIdx.x == 0) scale_out[0] = sc[0];
  const long long n = (long long)hc * wc;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(i / wc), ky = (int)(i - (long long)kx * wc);
    const size_t o = (size_t)kx * kp + ky;
    uint4 g0, g1;
    nn_feature(p, o, kx, ky, nx, ny, sc, p.epw_x[o], p.epw_y[o], p.prev_x[o], p.prev_y[o],
               p.prev2_x[o], p.prev2_y[o], &g0, &g1);
    reinterpret_cast<uint4*>(img)[i] = g0;
    reinterpret_cast<uint4*>(img)[n + i] = g1;
  }
}

struct NNData {
  int cap;
  __nv_bfloat16* img;  // [2][cap][NN_CROP][NN_CROP][8]
  float* target;       // [cap][2][NN_CROP][NN_CROP]
  float* scale;        // [cap]
};

// recording, slice start: the crop's features into slot `slot`, the target
// slot = -(quadratic start) / scale, the scale; then the history moves one slice on
// for every mode (epw_prev2 <- epw_prev, epw_prev <- epw)
__global__ void k_nn_record_start(NNSlicePlanes p, int nx, int ny, int kp, const float* part,
                                  NNData d, int slot) {
  __shared__ float sc[3];
  nn_scales(part, nx, ny, sc);
  if (blockIdx.x == 0 && threadIdx.x == 0) d.scale[slot] = sc[0];
  const long long n = (long long)(nx + 1) * (ny + 1);
  const size_t C2 = (size_t)NN_CROP * NN_CROP;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(i / (ny + 1)), ky = (int)(i - (long long)kx * (ny + 1));
    const size_t o = (size_t)kx * kp + ky;
    const float e1x = p.epw_x[o], e1y = p.epw_y[o], e0x = p.prev_x[o], e0y = p.prev_y[o];
    const float emx = p.prev2_x[o], emy = p.prev2_y[o];
    if (kx < NN_CROP && ky < NN_CROP) {
      uint4 g0, g1;
      nn_feature(p, o, kx, ky, nx, ny, sc, e1x, e1y, e0x, e0y, emx, emy, &g0, &g1);
      const size_t px = (size_t)kx * NN_CROP + ky;
      uint4* im = reinterpret_cast<uint4*>(d.img);
      im[(size_t)slot * C2 + px] = g0;
      im[((size_t)d.cap + slot) * C2 + px] = g1;
      float* t = d.target + (size_t)slot * 2 * C2;
      t[px] = -safe_div(nn_base(e1x, e0x, emx), sc[0]);
      t[C2 + px] = -safe_div(nn_base(e1y, e0y, emy), sc[0]);
    }
    p.prev2_x[o] = e0x;
    p.prev2_y[o] = e0y;
    p.prev_x[o] = e1x;
    p.prev_y[o] = e1y;
  }
}

// recording, slice end: target slot += converged epw / scale
__global__ void k_nn_record_end(NNSlicePlanes p, int kp, NNData d, int slot) {
  const float sB = d.scale[slot];
  const size_t C2 = (size_t)NN_CROP * NN_CROP;
  float* t = d.target + (size_t)slot * 2 * C2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (int)C2; i += gridDim.x * blockDim.x) {
    const int kx = i / NN_CROP, ky = i - kx * NN_CROP;
    const size_t o = (size_t)kx * kp + ky;
    t[i] += safe_div(p.epw_x[o], sB);
    t[C2 + i] += safe_div(p.epw_y[o], sB);
  }
}

// recording, after the slice: a pair whose target is larger than the field
// itself (RMS over the crop above the epw scale: slices where B appears or
// changes shape abruptly, mostly at the head of the beam) is not a
// correction the network can learn from; its scale is set to 0, which takes
// it out of the loss
__global__ void k_nn_record_validate(NNData d, int slot) {
  __shared__ float red[32];
  const size_t C2 = (size_t)NN_CROP * NN_CROP;
  const float* t = d.target + (size_t)slot * 2 * C2;
  float v = 0.f;
  for (size_t i = threadIdx.x; i < 2 * C2; i += blockDim.x) v += t[i] * t[i];
  for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
    if (!(s / (float)(2 * C2) <= 1.f)) d.scale[slot] = 0.f;
  }
}

// ------------------------------------------------------------------ training
// MSE of the 2 outputs against the target (samples with scale 0 carry no
// weight); dY = 2 (y - t) / n as the last layer's output gradient
__global__ void k_nn_loss(const float* y, NNData d, int b0, int B, int H, int W, float inv_n,
                          __nv_bfloat16* dy, float* loss) {
  __shared__ float red[8];
  const long long n = (long long)B * H * W;
  const size_t C2 = (size_t)H * W;
  float l = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / C2);
    const size_t px = (size_t)(i - (long long)b * C2);
    const bool ok = d.scale[b0 + b] > 0.f;
    float g[2];
    for (int c = 0; c < 2; ++c) {
      const float e = ok ? y[((size_t)b * 2 + c) * C2 + px] -
                               d.target[((size_t)(b0 + b) * 2 + c) * C2 + px]
                         : 0.f;
      l += e * e;
      g[c] = 2.f * e * inv_n;
    }
    uint4 u0 = make_uint4(pack_bf16(g[0], g[1]), 0u, 0u, 0u);
    reinterpret_cast<uint4*>(dy)[i] = u0;
    reinterpret_cast<uint4*>(dy)[n + i] = make_uint4(0u, 0u, 0u, 0u);
  }
  for (int off = 16; off; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    float v = 0.f;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v += red[i];
    atomicAdd(loss, v * inv_n);
  }
}

// a minibatch: pairs idx[0..B) of the set copied into the batch buffers
__global__ void k_nn_gather(NNData src, const int* idx, NNData dst) {
  const size_t C2 = (size_t)NN_CROP * NN_CROP;
  const int b = blockIdx.y, slot = idx[b];
  const uint4* si = reinterpret_cast<const uint4*>(src.img);
  uint4* di = reinterpret_cast<uint4*>(dst.img);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < C2;
       i += (size_t)gridDim.x * blockDim.x) {
    di[(size_t)b * C2 + i] = si[(size_t)slot * C2 + i];
    di[((size_t)dst.cap + b) * C2 + i] = si[((size_t)src.cap + slot) * C2 + i];
    dst.target[((size_t)b * 2) * C2 + i] = src.target[((size_t)slot * 2) * C2 + i];
    dst.target[((size_t)b * 2 + 1) * C2 + i] = src.target[((size_t)slot * 2 + 1) * C2 + i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) dst.scale[b] = src.scale[slot];
}

__global__ void k_nn_adam(float* w, const float* g, float* m, float* v, int n, float lr,
                          float b1, float b2, float c1, float c2, float eps) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// the bf16 B operands of layer l from the fp32 master: forward (Cout x 9 Cin)
// and data gradient (Cin x 9 Cout, taps flipped), canonical K-major layouts
__global__ void k_nn_pack(const float* wl, int cin, int cout, __nv_bfloat16* wf,
                          __nv_bfloat16* wd) {
  const int n = 9 * cin * cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int t = i / (cin * cout), r = i - t * cin * cout, ci = r / cout, co = r - ci * cout;
    const __nv_bfloat16 v = __float2bfloat16_rn(wl[i]);
    {  // forward: n = co, k = t*cin + ci
      const int k = t * cin + ci;
      wf[((k >> 3) * (cout >> 3) + (co >> 3)) * 64 + (co & 7) * 8 + (k & 7)] = v;
    }
    {  // data gradient: n = ci, k = (8 - t)*cout + co
      const int k = (8 - t) * cout + co;
      wd[((k >> 3) * (cin >> 3) + (ci >> 3)) * 64 + (ci & 7) * 8 + (k & 7)] = v;
    }
  }
}


// ---------------------------------------------------------------- host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tensor map of a channel-group-planar image [G][NB][H][W][8] bf16 with a box
// of (8, box_w, box_h, 1, box_g); zero fill outside the image.
int make_map(CUtensorMap* m, const void* base, int G, int NB, int H, int W, int box_w, int box_h,
             int box_g) {
  auto fn = encode_fn();
  if (!fn) return -1;
  cuuint64_t dims[5] = {8, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)NB, (cuuint64_t)G};
  cuuint64_t strides[4] = {16, 16ull * W, 16ull * W * H, 16ull * W * H * NB};
  cuuint32_t box[5] = {8, (cuuint32_t)box_w, (cuuint32_t)box_h, 1, (cuuint32_t)box_g};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(base), dims,
                        strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -1;
}
int halo_map(CUtensorMap* m, const void* base, int G, int NB, int H, int W) {
  return make_map(m, base, G, NB, H, W, HW_, 3, G);
}
int tile_map(CUtensorMap* m, const void* base, int G, int NB, int H, int W) {
  return make_map(m, base, G, NB, H, W, TM, 1, G);
}

constexpr size_t conv_smem(int cin, int cout) {
  return (size_t)cout * 9 * cin * 2 + 2 * (size_t)(((cin / 8) * HALO_G + 127) & ~127) + 64;
}
constexpr size_t wgrad_smem(int cin, int cout) {
  return 2 * (size_t)(((((cin / 8) * HALO_G + 127) & ~127) + (cout / 8) * TM * 16 + 127) & ~127) +
         (size_t)(TM / 8) * 128 * 16 + 9 * (size_t)(TM / 8) * cin * 16 + 64;
}

int g_num_sms = 0;
int num_sms() {
  if (!g_num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

template <int CIN, int COUT, int EPI>
cudaError_t conv_launch(const CUtensorMap& tin, const ConvArgs& a, cudaStream_t s) {
  const size_t smem = conv_smem(CIN, COUT);
  cudaError_t e = cudaFuncSetAttribute(k_conv3x3<CIN, COUT, EPI>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int ntiles = a.NB * a.H * (a.W / TM);
  const int grid = std::min(ntiles, num_sms() * 4);
  k_conv3x3<CIN, COUT, EPI><<<grid, 128, smem, s>>>(tin, a);
  return cudaGetLastError();
}

template <int CIN, int COUT>
cudaError_t wgrad_launch(const CUtensorMap& tx, const CUtensorMap& tdy, const WgradArgs& a,
                         cudaStream_t s) {
  const size_t smem = wgrad_smem(CIN, COUT);
  cudaError_t e = cudaFuncSetAttribute(k_wgrad<CIN, COUT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int ntiles = a.NB * a.H * (a.W / TM);
  const int grid = std::min(ntiles, num_sms());
  k_wgrad<CIN, COUT><<<grid, 128, smem, s>>>(tx, tdy, a);
  return cudaGetLastError();
}

}  // namespace
}  // namespace qp

using namespace qp;

// The network: fp32 master parameters (layer l: W[9][cin][cout], bias[cout]),
// their bf16 forward and data-gradient operands, Adam moments, and the
// device error flag of the tensor-core kernels.
struct qp_nn {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* master = nullptr;
  float* grad = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  __nv_bfloat16* wf[NN_LAYERS] = {};
  __nv_bfloat16* wd[NN_LAYERS] = {};
  int off[NN_LAYERS] = {};
  int nparams = 0;
  long long adam_t = 0;
  int* err = nullptr;
  float* loss = nullptr;
};

// Training pairs recorded by a simulation: 128 x 128 crops (the low modes) of
// the 16-channel input image, the target correction and the epw scale, in
// recording order.
struct qp_nn_data {
  int device = 0;
  NNData d{};
  int count = 0;  // pairs recorded
};

namespace qp {
struct NNRuntime {
  int nx = 0, ny = 0, kp = 0;
  int hc = 0, wc = 0;             // the low-mode window the network corrects
  __nv_bfloat16* img = nullptr;   // [2][1][hc][wc][8]
  __nv_bfloat16* act[2] = {};     // [4][1][hc][wc][8]
  float* part = nullptr;          // norm partials
  float* scale = nullptr;         // the slice's epw scale
  CUtensorMap m_img, m_act[2];
};
}  // namespace qp

namespace {

int nn_fail(int line, const std::string& msg) {
  qp_set_error("qp_nn.cu", line, msg.c_str());
  return -1;
}
// QP_NN_TRACE=1: print each tensor-core launch and wait for it (diagnosis)
bool nn_trace() {
  static int t = -1;
  if (t < 0) {
    const char* e = std::getenv("QP_NN_TRACE");
    t = (e && e[0] == '1') ? 1 : 0;
  }
  return t == 1;
}
int nn_trace_point(const char* what, int layer, cudaStream_t s) {
  if (!nn_trace()) return 0;
  std::fprintf(stderr, "[qp_nn] %s layer %d ...", what, layer);
  std::fflush(stderr);
  const cudaError_t e = cudaStreamSynchronize(s);
  std::fprintf(stderr, " %s\n", cudaGetErrorString(e));
  std::fflush(stderr);
  return e == cudaSuccess ? 0 : -1;
}
#define NK(call)                                                              \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) return nn_fail(__LINE__, cudaGetErrorString(e_)); \
  } while (0)

int nn_pack(qp_nn* nn, cudaStream_t s) {
  for (int l = 0; l < NN_LAYERS; ++l) {
    k_nn_pack<<<64, 256, 0, s>>>(nn->master + nn->off[l], nn_cin(l), nn_cout(l), nn->wf[l],
                                  nn->wd[l]);
  }
  NK(cudaGetLastError());
  return 0;
}

const float* nn_bias(const qp_nn* nn, int l) {
  return nn->master + nn->off[l] + 9 * nn_cin(l) * nn_cout(l);
}

// forward of layers 1..5 over NB images of H x W.  in_map: halo map of the
// 16-channel input (its images b0 ..); act: 4 buffers [4][NB][H][W][8]
// (layer l's output in act[l], l = 0..3) with their halo maps; the last layer
// writes `out32` [NB][2][H][W] (training) or the slice start (epw planes).
int nn_forward(qp_nn* nn, const CUtensorMap& in_map, int b0, __nv_bfloat16* const* act,
               const CUtensorMap* act_map, int NB, int H, int W, float* out32,
               const NNSlicePlanes* pl, const float* scale, int kp, int nx, int ny,
               cudaStream_t s) {
  ConvArgs a{};
  a.H = H;
  a.W = W;
  a.NB = NB;
  a.err = nn->err;
  for (int l = 0; l < NN_LAYERS; ++l) {
    a.w = nn->wf[l];
    a.bias = nn_bias(nn, l);
    a.b0 = l == 0 ? b0 : 0;
    const CUtensorMap& tin = l == 0 ? in_map : act_map[l - 1];
    cudaError_t e;
    if (l < NN_LAYERS - 1) {
      a.out = act[l];
      e = l == 0 ? conv_launch<NN_CIN0, NN_CH, EPI_RELU>(tin, a, s)
                 : conv_launch<NN_CH, NN_CH, EPI_RELU>(tin, a, s);
    } else if (out32) {
      a.out32 = out32;
      e = conv_launch<NN_CH, NN_NLAST, EPI_F32>(tin, a, s);
    } else {
      a.pl = *pl;
      a.scale = scale;
      a.kp = kp;
      a.nx = nx;
      a.ny = ny;
      e = conv_launch<NN_CH, NN_NLAST, EPI_EPW>(tin, a, s);
    }
    if (e != cudaSuccess) return nn_fail(__LINE__, cudaGetErrorString(e));
    if (nn_trace_point("forward", l, s)) return nn_fail(__LINE__, "forward launch failed");
  }
  return 0;
}

// backward from dy5 = d loss / d output ([2][NB][H][W][8]): parameter
// gradients added into nn->grad.  in_map/b0: the 16-channel input; act and
// dx: 4 buffers each [4][NB][H][W][8] with halo and tile maps.
int nn_backward(qp_nn* nn, const CUtensorMap& in_map, int b0, __nv_bfloat16* const* act,
                const CUtensorMap* act_halo, __nv_bfloat16* dy5, const CUtensorMap& dy5_tile,
                const CUtensorMap& dy5_halo, __nv_bfloat16* const* dx, const CUtensorMap* dx_tile,
                const CUtensorMap* dx_halo, int NB, int H, int W, cudaStream_t s) {
  WgradArgs w{};
  w.H = H;
  w.W = W;
  w.NB = NB;
  w.err = nn->err;
  ConvArgs c{};
  c.H = H;
  c.W = W;
  c.NB = NB;
  c.err = nn->err;
  cudaError_t e;
  for (int l = NN_LAYERS - 1; l >= 0; --l) {
    const int cin = nn_cin(l), cout = nn_cout(l);
    float* gl = nn->grad + nn->off[l];
    w.dw = gl;
    w.db = gl + 9 * cin * cout;
    w.couts = l == NN_LAYERS - 1 ? NN_OUT : cout;
    w.xb0 = l == 0 ? b0 : 0;
    const CUtensorMap& xm = l == 0 ? in_map : act_halo[l - 1];
    const CUtensorMap& dym = l == NN_LAYERS - 1 ? dy5_tile : dx_tile[l];
    if (l == 0)
      e = wgrad_launch<NN_CIN0, NN_CH>(xm, dym, w, s);
    else if (l == NN_LAYERS - 1)
      e = wgrad_launch<NN_CH, NN_NLAST>(xm, dym, w, s);
    else
      e = wgrad_launch<NN_CH, NN_CH>(xm, dym, w, s);
    if (e != cudaSuccess) return nn_fail(__LINE__, cudaGetErrorString(e));
    if (nn_trace_point("wgrad", l, s)) return nn_fail(__LINE__, "wgrad launch failed");
    if (l == 0) break;
    // data gradient into layer l's input, masked by the ReLU of layer l-1
    c.w = nn->wd[l];
    c.bias = nullptr;
    c.b0 = 0;
    c.out = dx[l - 1];
    c.mask = act[l - 1];
    if (l == NN_LAYERS - 1)
      e = conv_launch<NN_NLAST, NN_CH, EPI_MASK>(dy5_halo, c, s);
    else
      e = conv_launch<NN_CH, NN_CH, EPI_MASK>(dx_halo[l], c, s);
    if (e != cudaSuccess) return nn_fail(__LINE__, cudaGetErrorString(e));
    if (nn_trace_point("dgrad", l, s)) return nn_fail(__LINE__, "dgrad launch failed");
  }
  return 0;
}

int nn_check_err(qp_nn* nn, cudaStream_t s) {
  int h = 0;
  NK(cudaMemcpyAsync(&h, nn->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  NK(cudaStreamSynchronize(s));
  if (h) return nn_fail(__LINE__, "tensor-core kernel: a bounded wait expired (code " +
                                      std::to_string(h) + ")");
  return 0;
}

// Work buffers of one forward/backward over NB images of H x W.
struct Work {
  int NB = 0, H = 0, W = 0;
  __nv_bfloat16* act[4] = {};
  __nv_bfloat16* dx[4] = {};
  __nv_bfloat16* dy5 = nullptr;
  float* out32 = nullptr;
  CUtensorMap act_halo[4], dx_halo[4], dx_tile[4], dy5_tile, dy5_halo;
  int alloc(int nb, int h, int w) {
    NB = nb;
    H = h;
    W = w;
    const size_t px = (size_t)nb * h * w;
    for (int i = 0; i < 4; ++i) {
      if (cudaMalloc(&act[i], px * NN_CH * 2) != cudaSuccess ||
          cudaMalloc(&dx[i], px * NN_CH * 2) != cudaSuccess)
        return -1;
      if (halo_map(&act_halo[i], act[i], NN_CH / 8, nb, h, w) ||
          halo_map(&dx_halo[i], dx[i], NN_CH / 8, nb, h, w) ||
          tile_map(&dx_tile[i], dx[i], NN_CH / 8, nb, h, w))
        return -2;
    }
    if (cudaMalloc(&dy5, px * NN_NLAST * 2) != cudaSuccess ||
        cudaMalloc(&out32, px * NN_OUT * sizeof(float)) != cudaSuccess)
      return -1;
    if (tile_map(&dy5_tile, dy5, NN_NLAST / 8, nb, h, w) ||
        halo_map(&dy5_halo, dy5, NN_NLAST / 8, nb, h, w))
      return -2;
    return 0;
  }
  void free_all() {
    for (int i = 0; i < 4; ++i) {
      cudaFree(act[i]);
      cudaFree(dx[i]);
    }
    cudaFree(dy5);
    cudaFree(out32);
  }
};

}  // namespace

// ------------------------------------------------------------------- C ABI
extern "C" int qp_nn_create(int device, unsigned long long seed, qp_nn** out) {
  if (!out) return nn_fail(__LINE__, "null argument");
  if (cudaSetDevice(device) != cudaSuccess) return nn_fail(__LINE__, "cudaSetDevice failed");
  if (!encode_fn()) return nn_fail(__LINE__, "cuTensorMapEncodeTiled is not available");
  qp_nn* nn = new qp_nn();
  nn->device = device;
  int o = 0;
  for (int l = 0; l < NN_LAYERS; ++l) {
    nn->off[l] = o;
    o += nn_layer_params(l);
  }
  nn->nparams = o;
  const size_t pb = sizeof(float) * (size_t)o;
  bool ok = cudaStreamCreateWithFlags(&nn->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&nn->master, pb) == cudaSuccess &&
            cudaMalloc(&nn->grad, pb) == cudaSuccess && cudaMalloc(&nn->m, pb) == cudaSuccess &&
            cudaMalloc(&nn->v, pb) == cudaSuccess &&
            cudaMalloc(&nn->err, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&nn->loss, sizeof(float)) == cudaSuccess;
  for (int l = 0; l < NN_LAYERS && ok; ++l) {
    const size_t wb = sizeof(__nv_bfloat16) * 9 * nn_cin(l) * nn_cout(l);
    ok = cudaMalloc(&nn->wf[l], wb) == cudaSuccess && cudaMalloc(&nn->wd[l], wb) == cudaSuccess;
  }
  if (!ok) {
    qp_nn_destroy(nn);
    return nn_fail(__LINE__, "out of device memory (network)");
  }
  // He initialisation for the ReLU layers; the last layer starts at zero, so an
  // untrained network is the quadratic extrapolation
  std::vector<float> h(o, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < NN_LAYERS - 1; ++l) {
    const int cin = l == 0 ? NN_FEATURES : nn_cin(l), cout = nn_cout(l);
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (9.f * cin)));
    for (int t = 0; t < 9; ++t)
      for (int ci = 0; ci < cin; ++ci)
        for (int co = 0; co < cout; ++co)
          h[nn->off[l] + (t * nn_cin(l) + ci) * cout + co] = nd(rng);
  }
  cudaMemcpy(nn->master, h.data(), pb, cudaMemcpyHostToDevice);
  cudaMemset(nn->m, 0, pb);
  cudaMemset(nn->v, 0, pb);
  cudaMemset(nn->err, 0, sizeof(int));
  if (nn_pack(nn, nn->stream) || cudaStreamSynchronize(nn->stream) != cudaSuccess) {
    qp_nn_destroy(nn);
    return nn_fail(__LINE__, "network set-up failed");
  }
  *out = nn;
  return 0;
}

extern "C" int qp_nn_destroy(qp_nn* nn) {
  if (!nn) return 0;
  cudaSetDevice(nn->device);
  if (nn->stream) cudaStreamSynchronize(nn->stream);
  for (void* p : {(void*)nn->master, (void*)nn->grad, (void*)nn->m, (void*)nn->v,
                  (void*)nn->err, (void*)nn->loss})
    if (p) cudaFree(p);
  for (int l = 0; l < NN_LAYERS; ++l) {
    if (nn->wf[l]) cudaFree(nn->wf[l]);
    if (nn->wd[l]) cudaFree(nn->wd[l]);
  }
  if (nn->stream) cudaStreamDestroy(nn->stream);
  delete nn;
  return 0;
}

extern "C" int qp_nn_num_params(const qp_nn* nn) { return nn ? nn->nparams : -1; }

extern "C" int qp_nn_get_params(qp_nn* nn, float* out) {
  if (!nn || !out) return nn_fail(__LINE__, "null argument");
  NK(cudaMemcpy(out, nn->master, sizeof(float) * nn->nparams, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int qp_nn_set_params(qp_nn* nn, const float* in) {
  if (!nn || !in) return nn_fail(__LINE__, "null argument");
  NK(cudaMemcpy(nn->master, in, sizeof(float) * nn->nparams, cudaMemcpyHostToDevice));
  if (nn_pack(nn, nn->stream)) return -1;
  NK(cudaStreamSynchronize(nn->stream));
  return 0;
}

namespace {
// host images [NB][16][H][W] fp32 -> device [2][NB][H][W][8] bf16 (through a
// host-side conversion; a test and set-up path, not the step's)
int upload_images(const float* in, int NB, int H, int W, __nv_bfloat16** dev) {
  const size_t px = (size_t)NB * H * W;
  std::vector<__nv_bfloat16> h(px * NN_CIN0);
  for (int b = 0; b < NB; ++b)
    for (int c = 0; c < NN_CIN0; ++c)
      for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
          const size_t src = (((size_t)b * NN_CIN0 + c) * H + y) * W + x;
          const size_t dst = ((((size_t)(c >> 3) * NB + b) * H + y) * W + x) * 8 + (c & 7);
          h[dst] = __float2bfloat16_rn(in[src]);
        }
  if (cudaMalloc(dev, h.size() * 2) != cudaSuccess) return -1;
  return cudaMemcpy(*dev, h.data(), h.size() * 2, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -1;
}

int check_shape(int NB, int H, int W) {
  if (NB < 1 || H < 1 || W < TM || W % TM != 0 || (long long)NB * H * W > (1LL << 28))
    return nn_fail(__LINE__, "network images: W must be a positive multiple of 128");
  return 0;
}
}  // namespace

extern "C" int qp_nn_forward(qp_nn* nn, const float* in, int NB, int H, int W, float* out) {
  if (!nn || !in || !out) return nn_fail(__LINE__, "null argument");
  if (check_shape(NB, H, W)) return -1;
  cudaSetDevice(nn->device);
  __nv_bfloat16* img = nullptr;
  Work wk;
  int rc = upload_images(in, NB, H, W, &img) || wk.alloc(NB, H, W) ? -1 : 0;
  CUtensorMap m_in;
  if (!rc && halo_map(&m_in, img, NN_CIN0 / 8, NB, H, W)) rc = -1;
  if (!rc) rc = nn_forward(nn, m_in, 0, wk.act, wk.act_halo, NB, H, W, wk.out32, nullptr, nullptr,
                           0, 0, 0, nn->stream);
  if (!rc) rc = nn_check_err(nn, nn->stream);
  if (!rc && cudaMemcpy(out, wk.out32, sizeof(float) * NN_OUT * (size_t)NB * H * W,
                        cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = nn_fail(__LINE__, "download failed");
  cudaFree(img);
  wk.free_all();
  return rc;
}

// Loss (mean squared error of the 2 outputs over every pixel) and its gradient
// with respect to every parameter, for images in[NB][16][H][W] and targets
// target[NB][2][H][W]; grad[] in the parameter layout.
extern "C" int qp_nn_loss_grad(qp_nn* nn, const float* in, const float* target, int NB, int H,
                               int W, double* loss, float* grad) {
  if (!nn || !in || !target || !grad) return nn_fail(__LINE__, "null argument");
  if (check_shape(NB, H, W)) return -1;
  cudaSetDevice(nn->device);
  cudaStream_t s = nn->stream;
  __nv_bfloat16* img = nullptr;
  Work wk;
  NNData d{};
  int rc = upload_images(in, NB, H, W, &img) || wk.alloc(NB, H, W) ? -1 : 0;
  const size_t px = (size_t)NB * H * W;
  std::vector<float> ones(NB, 1.f);
  if (!rc && (cudaMalloc(&d.target, sizeof(float) * 2 * px) != cudaSuccess ||
              cudaMalloc(&d.scale, sizeof(float) * NB) != cudaSuccess))
    rc = -1;
  if (!rc) {
    d.cap = NB;
    cudaMemcpy(d.target, target, sizeof(float) * 2 * px, cudaMemcpyHostToDevice);
    cudaMemcpy(d.scale, ones.data(), sizeof(float) * NB, cudaMemcpyHostToDevice);
  }
  CUtensorMap m_in;
  if (!rc && halo_map(&m_in, img, NN_CIN0 / 8, NB, H, W)) rc = -1;
  if (!rc) rc = nn_forward(nn, m_in, 0, wk.act, wk.act_halo, NB, H, W, wk.out32, nullptr, nullptr,
                           0, 0, 0, s);
  if (!rc) {
    cudaMemsetAsync(nn->loss, 0, sizeof(float), s);
    cudaMemsetAsync(nn->grad, 0, sizeof(float) * nn->nparams, s);
    k_nn_loss<<<256, 256, 0, s>>>(wk.out32, d, 0, NB, H, W, 1.f / (2.f * (float)px), wk.dy5,
                                  nn->loss);
    rc = nn_backward(nn, m_in, 0, wk.act, wk.act_halo, wk.dy5, wk.dy5_tile, wk.dy5_halo, wk.dx,
                     wk.dx_tile, wk.dx_halo, NB, H, W, s);
  }
  if (!rc) rc = nn_check_err(nn, s);
  float l = 0.f;
  if (!rc && (cudaMemcpy(&l, nn->loss, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
              cudaMemcpy(grad, nn->grad, sizeof(float) * nn->nparams, cudaMemcpyDeviceToHost) !=
                  cudaSuccess))
    rc = nn_fail(__LINE__, "download failed");
  if (loss) *loss = l;
  cudaFree(img);
  cudaFree(d.target);
  cudaFree(d.scale);
  wk.free_all();
  return rc;
}

// ------------------------------------------------------------- training set
extern "C" int qp_nn_data_create(int device, int capacity, qp_nn_data** out) {
  if (!out || capacity < 1) return nn_fail(__LINE__, "bad training-set arguments");
  if (cudaSetDevice(device) != cudaSuccess) return nn_fail(__LINE__, "cudaSetDevice failed");
  qp_nn_data* t = new qp_nn_data();
  t->device = device;
  t->d.cap = capacity;
  const size_t C2 = (size_t)NN_CROP * NN_CROP;
  if (cudaMalloc(&t->d.img, (size_t)capacity * C2 * NN_CIN0 * 2) != cudaSuccess ||
      cudaMalloc(&t->d.target, (size_t)capacity * C2 * 2 * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&t->d.scale, (size_t)capacity * sizeof(float)) != cudaSuccess) {
    qp_nn_data_destroy(t);
    return nn_fail(__LINE__, "out of device memory (training set)");
  }
  cudaMemset(t->d.scale, 0, (size_t)capacity * sizeof(float));
  *out = t;
  return 0;
}

extern "C" int qp_nn_data_destroy(qp_nn_data* t) {
  if (!t) return 0;
  cudaSetDevice(t->device);
  cudaDeviceSynchronize();
  if (t->d.img) cudaFree(t->d.img);
  if (t->d.target) cudaFree(t->d.target);
  if (t->d.scale) cudaFree(t->d.scale);
  delete t;
  return 0;
}

extern "C" int qp_nn_data_count(const qp_nn_data* t) { return t ? t->count : -1; }

// pair i (in recording order): features [16][128][128], target [2][128][128], scale
extern "C" int qp_nn_data_get(qp_nn_data* t, int i, float* img, float* target, float* scale) {
  if (!t || i < 0 || i >= t->count) return nn_fail(__LINE__, "training pair index out of range");
  const int slot = i;
  const size_t C2 = (size_t)NN_CROP * NN_CROP;
  std::vector<__nv_bfloat16> h(C2 * 8);
  for (int g = 0; g < 2 && img; ++g) {
    NK(cudaMemcpy(h.data(), t->d.img + ((size_t)g * t->d.cap + slot) * C2 * 8, h.size() * 2,
                  cudaMemcpyDeviceToHost));
    for (size_t p = 0; p < C2; ++p)
      for (int c = 0; c < 8; ++c) img[(size_t)(8 * g + c) * C2 + p] = __bfloat162float(h[p * 8 + c]);
  }
  if (target)
    NK(cudaMemcpy(target, t->d.target + (size_t)slot * 2 * C2, sizeof(float) * 2 * C2,
                  cudaMemcpyDeviceToHost));
  if (scale) NK(cudaMemcpy(scale, t->d.scale + slot, sizeof(float), cudaMemcpyDeviceToHost));
  return 0;
}

// Adam on minibatches of `batch` pairs drawn at random (seeded) from the
// recorded set; each minibatch is gathered into contiguous batch buffers.
extern "C" int qp_nn_train(qp_nn* nn, qp_nn_data* t, const qp_nn_train_desc* d,
                           qp_nn_train_stats* st) {
  if (!nn || !t || !d) return nn_fail(__LINE__, "null argument");
  if (t->count < d->batch || d->batch < 1 || d->steps < 1 || !(d->lr > 0.f))
    return nn_fail(__LINE__, "training: bad settings, or fewer pairs than one minibatch");
  cudaSetDevice(nn->device);
  cudaStream_t s = nn->stream;
  const int B = d->batch, H = NN_CROP, W = NN_CROP;
  const size_t C2 = (size_t)H * W;
  Work wk;
  NNData bt{};
  bt.cap = B;
  int* idx = nullptr;
  std::vector<int> hidx((size_t)d->steps * B);
  std::mt19937_64 rng(d->seed);
  std::uniform_int_distribution<int> pick(0, t->count - 1);
  for (auto& v : hidx) v = pick(rng);
  CUtensorMap m_in;
  int rc = 0;
  if (wk.alloc(B, H, W) || cudaMalloc(&bt.img, (size_t)B * C2 * NN_CIN0 * 2) != cudaSuccess ||
      cudaMalloc(&bt.target, (size_t)B * C2 * 2 * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&bt.scale, (size_t)B * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&idx, sizeof(int) * hidx.size()) != cudaSuccess ||
      halo_map(&m_in, bt.img, NN_CIN0 / 8, B, H, W))
    rc = nn_fail(__LINE__, "out of device memory (training buffers)");
  if (!rc && cudaMemcpy(idx, hidx.data(), sizeof(int) * hidx.size(), cudaMemcpyHostToDevice) !=
                 cudaSuccess)
    rc = nn_fail(__LINE__, "upload failed");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  const float inv_n = 1.f / (2.f * (float)B * H * W);
  const float b1 = 0.9f, b2 = 0.999f;
  // every step's minibatch loss, kept on the device and read once at the end
  float* hist = nullptr;
  if (!rc && (cudaMalloc(&hist, sizeof(float) * d->steps) != cudaSuccess ||
              cudaMemsetAsync(hist, 0, sizeof(float) * d->steps, s) != cudaSuccess))
    rc = nn_fail(__LINE__, "out of device memory (training buffers)");
  for (int it = 0; it < d->steps && !rc; ++it) {
    k_nn_gather<<<dim3(32, B), 256, 0, s>>>(t->d, idx + (size_t)it * B, bt);
    // the learning rate steps down to 0.3 and 0.1 of its start at 1/2 and 3/4 of the run
    const float lr = d->lr * (it < d->steps / 2 ? 1.f : (it < 3 * d->steps / 4 ? 0.3f : 0.1f));
    rc = nn_forward(nn, m_in, 0, wk.act, wk.act_halo, B, H, W, wk.out32, nullptr, nullptr, 0, 0,
                    0, s);
    if (rc) break;
    cudaMemsetAsync(nn->grad, 0, sizeof(float) * nn->nparams, s);
    k_nn_loss<<<256, 256, 0, s>>>(wk.out32, bt, 0, B, H, W, inv_n, wk.dy5, hist + it);
    rc = nn_backward(nn, m_in, 0, wk.act, wk.act_halo, wk.dy5, wk.dy5_tile, wk.dy5_halo, wk.dx,
                     wk.dx_tile, wk.dx_halo, B, H, W, s);
    if (rc) break;
    ++nn->adam_t;
    const float c1 = 1.f - std::pow(b1, (float)nn->adam_t);
    const float c2 = 1.f - std::pow(b2, (float)nn->adam_t);
    k_nn_adam<<<64, 256, 0, s>>>(nn->master, nn->grad, nn->m, nn->v, nn->nparams, lr, b1, b2, c1,
                                 c2, 1e-8f);
    rc = nn_pack(nn, s);
  }
  std::vector<float> losses(d->steps, 0.f);
  if (!rc && cudaMemcpyAsync(losses.data(), hist, sizeof(float) * d->steps,
                             cudaMemcpyDeviceToHost, s) != cudaSuccess)
    rc = nn_fail(__LINE__, "training loss download failed");
  cudaEventRecord(e1, s);
  if (!rc) rc = nn_check_err(nn, s);
  float ms = 0.f;
  if (!rc) {
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
  }
  cudaStreamSynchronize(s);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  wk.free_all();
  cudaFree(bt.img);
  cudaFree(bt.target);
  cudaFree(bt.scale);
  cudaFree(idx);
  cudaFree(hist);
  if (!rc && st) {
    // the mean minibatch loss over the first and over the last tenth of the run
    const int w = std::max(1, d->steps / 10);
    double a = 0.0, b = 0.0;
    for (int i = 0; i < w; ++i) {
      a += losses[i];
      b += losses[d->steps - 1 - i];
    }
    st->first_loss = a / w;
    st->last_loss = b / w;
    st->gpu_ms = ms;
    st->steps = d->steps;
  }
  return rc;
}

// ---------------------------------------------------------------- the step
namespace qp {

int nn_runtime_create(const GridDims& g, NNRuntime** out) {
  if (g.ny % TM != 0 || g.nx < 2)
    return nn_fail(__LINE__, "learned predictor: ny must be a multiple of 128");
  static_assert(NN_CROP == TM, "the network's window is one tile wide");
  if (!encode_fn()) return nn_fail(__LINE__, "cuTensorMapEncodeTiled is not available");
  NNRuntime* r = new NNRuntime();
  r->nx = g.nx;
  r->ny = g.ny;
  r->kp = g.kp;
  // the network corrects the modes it was trained on, kx, ky < 128 (the
  // training crop); the others take the quadratic extrapolation
  r->hc = std::min(g.nx, NN_CROP);
  r->wc = NN_CROP;
  const size_t px = (size_t)r->hc * r->wc;
  bool ok = cudaMalloc(&r->img, px * NN_CIN0 * 2) == cudaSuccess &&
            cudaMalloc(&r->act[0], px * NN_CH * 2) == cudaSuccess &&
            cudaMalloc(&r->act[1], px * NN_CH * 2) == cudaSuccess &&
            cudaMalloc(&r->part, sizeof(float) * 3 * NN_NORM_BLOCKS) == cudaSuccess &&
            cudaMalloc(&r->scale, sizeof(float)) == cudaSuccess;
  ok = ok && !halo_map(&r->m_img, r->img, NN_CIN0 / 8, 1, r->hc, r->wc) &&
       !halo_map(&r->m_act[0], r->act[0], NN_CH / 8, 1, r->hc, r->wc) &&
       !halo_map(&r->m_act[1], r->act[1], NN_CH / 8, 1, r->hc, r->wc);
  if (!ok) {
    nn_runtime_destroy(r);
    return nn_fail(__LINE__, "learned predictor set-up failed");
  }
  *out = r;
  return 0;
}

void nn_runtime_destroy(NNRuntime* r) {
  if (!r) return;
  for (void* p : {(void*)r->img, (void*)r->act[0], (void*)r->act[1], (void*)r->part,
                  (void*)r->scale})
    if (p) cudaFree(p);
  delete r;
}

int nn_predict(NNRuntime* r, const void* net, const NNSlicePlanes& p, const GridDims& g,
               DevStatus* st, cudaStream_t s) {
  qp_nn* nn = const_cast<qp_nn*>(static_cast<const qp_nn*>(net));
  k_nn_norms<<<NN_NORM_BLOCKS, 256, 0, s>>>(p, g.nx, g.ny, g.kp, r->part);
  k_nn_features<<<NN_NORM_BLOCKS, 256, 0, s>>>(p, g.nx, g.ny, g.kp, r->hc, r->wc, r->part,
                                                r->img, r->scale);
  // layers 1-4 ping-pong between the two activation buffers; every layer's
  // input is the previous output, so the four maps cycle through them
  __nv_bfloat16* act[4] = {r->act[0], r->act[1], r->act[0], r->act[1]};
  const CUtensorMap amap[4] = {r->m_act[0], r->m_act[1], r->m_act[0], r->m_act[1]};
  if (nn_forward(nn, r->m_img, 0, act, amap, 1, r->hc, r->wc, nullptr, &p, r->scale, g.kp, g.nx,
                 g.ny, s))
    return -1;
  (void)st;
  return 7;
}

int nn_record_start(NNRuntime* r, void* data, const NNSlicePlanes& p, const GridDims& g,
                    DevStatus* st, cudaStream_t s) {
  qp_nn_data* t = static_cast<qp_nn_data*>(data);
  (void)st;
  if (t->count >= t->d.cap) return 0;
  const int slot = t->count;
  k_nn_norms<<<NN_NORM_BLOCKS, 256, 0, s>>>(p, g.nx, g.ny, g.kp, r->part);
  k_nn_record_start<<<NN_NORM_BLOCKS * 4, 256, 0, s>>>(p, g.nx, g.ny, g.kp, r->part, t->d, slot);
  return 2;
}

int nn_record_end(NNRuntime* r, void* data, const NNSlicePlanes& p, const GridDims& g,
                  DevStatus* st, cudaStream_t s) {
  qp_nn_data* t = static_cast<qp_nn_data*>(data);
  (void)r;
  (void)st;
  if (t->count >= t->d.cap) return 0;
  const int slot = t->count;
  k_nn_record_end<<<64, 256, 0, s>>>(p, g.kp, t->d, slot);
  k_nn_record_validate<<<1, 1024, 0, s>>>(t->d, slot);
  t->count++;
  return 2;
}

}  // namespace qp
