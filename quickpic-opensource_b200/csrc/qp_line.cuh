// qp_line.cuh -- warp-level real sine (DST-I) and cosine (DCT-I) transforms.
//
// QuickPIC transforms each row and column of a field with the real sine and
// cosine transforms of Numerical Recipes (fft2d_lib77.f:4791-5493).  Their
// mathematical content is, for a line x[0..n] (n = 2^k):
//   sine   S[m] = 2 * sum_{j=1}^{n-1} x[j] sin(pi j m / n),          m = 0..n
//   cosine C[m] = x[0] + (-1)^m x[n] + 2 * sum_{j=1}^{n-1} x[j] cos(pi j m / n)
// (the reference's isign = +1 pass; its isign = -1 pass is the same transform
// scaled by 0.5/(nx*ny) along x and by 0.5 along y).  Here one warp computes
// one line in shared memory with the standard reduction of DST-I/DCT-I to a
// real FFT of length n (pre-twiddle, a complex FFT of n/2 points, real-FFT
// unscramble, and a prefix sum over the odd outputs); the complex FFT is a
// Stockham radix-4 (+ one radix-2) autosort, so no bit reversal is needed.
#pragma once

#include "qp_common.cuh"

namespace qp {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// exclusive warp scan
__device__ __forceinline__ float warp_excl_scan(float v, int lane) {
  float s = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    float t = __shfl_up_sync(0xffffffffu, s, o);
    if (lane >= o) s += t;
  }
  return s - v;
}

// Complex FFT (forward, exp(-i)) of N = 2^logN points held in shared memory
// at a; b is scratch of the same size.  Returns the buffer holding the result.
__device__ __forceinline__ float2* warp_cfft(float2* a, float2* b, int logN, const float2* tw,
                                             int lane) {
  const int N = 1 << logN;
  float2* src = a;
  float2* dst = b;
  int Ns = 1;
  const int n4 = N >> 2;
  for (int s = 0; s < (logN >> 1); ++s) {
    const int tstep = N / (4 * Ns);
    for (int j = lane; j < n4; j += 32) {
      const int k = j & (Ns - 1);
      float2 a0 = src[j], a1 = src[j + n4], a2 = src[j + 2 * n4], a3 = src[j + 3 * n4];
      if (Ns > 1) {
        const int st = k * tstep;
        a1 = cmul(a1, tw[st]);
        a2 = cmul(a2, tw[2 * st]);
        a3 = cmul(a3, tw[3 * st]);
      }
      float2 b0 = make_float2(a0.x + a2.x, a0.y + a2.y);
      float2 b1 = make_float2(a0.x - a2.x, a0.y - a2.y);
      float2 b2 = make_float2(a1.x + a3.x, a1.y + a3.y);
      float2 b3 = make_float2(a1.y - a3.y, a3.x - a1.x);  // -i * (a1 - a3)
      const int d = (j / Ns) * Ns * 4 + k;
      dst[d] = make_float2(b0.x + b2.x, b0.y + b2.y);
      dst[d + Ns] = make_float2(b1.x + b3.x, b1.y + b3.y);
      dst[d + 2 * Ns] = make_float2(b0.x - b2.x, b0.y - b2.y);
      dst[d + 3 * Ns] = make_float2(b1.x - b3.x, b1.y - b3.y);
    }
    __syncwarp();
    float2* t = src;
    src = dst;
    dst = t;
    Ns <<= 2;
  }
  if (logN & 1) {
    const int n2 = N >> 1;
    const int tstep = N / (2 * Ns);
    for (int j = lane; j < n2; j += 32) {
      const int k = j & (Ns - 1);
      float2 a0 = src[j], a1 = src[j + n2];
      if (Ns > 1) a1 = cmul(a1, tw[k * tstep]);
      const int d = (j / Ns) * Ns * 2 + k;
      dst[d] = make_float2(a0.x + a1.x, a0.y + a1.y);
      dst[d + Ns] = make_float2(a0.x - a1.x, a0.y - a1.y);
    }
    __syncwarp();
    float2* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

// Unnormalised DST-I (parity 0) or DCT-I (parity 1) of L[0..n], in place.
// L and S are per-warp shared buffers of at least n + 4 floats, 8-byte aligned.
static __device__ __noinline__ void warp_line_transform(float* L, float* S, int logn, int parity,
                                                 const LineTables& t, int lane) {
  const int n = 1 << logn;
  const int h = n >> 1;
  float sigma = 0.f;
  if (parity) {
    float acc = 0.f;
    for (int j = 1 + lane; j < n; j += 32) acc += L[j] * t.cs[j];
    acc = warp_sum(acc);
    sigma = 0.5f * (L[0] - L[n]) + acc;
  }
  __syncwarp();
  // pre-twiddle into the real sequence y[0..n-1]
  for (int j = 1 + lane; j < h; j += 32) {
    const float a = L[j], b = L[n - j], s = t.sn[j];
    const float p = a + b, m = a - b;
    if (parity == 0) {
      const float u = s * p, v = 0.5f * m;
      L[j] = u + v;
      L[n - j] = u - v;
    } else {
      const float u = 0.5f * p, v = s * m;
      L[j] = u - v;
      L[n - j] = u + v;
    }
  }
  if (lane == 0) {
    if (parity == 0) {
      L[0] = 0.f;
      L[h] = 2.f * L[h];
    } else {
      L[0] = 0.5f * (L[0] + L[n]);
    }
  }
  __syncwarp();
  // complex FFT of z[m] = y[2m] + i y[2m+1], m = 0..h-1
  float2* Z = warp_cfft(reinterpret_cast<float2*>(L), reinterpret_cast<float2*>(S), logn - 1,
                        t.tw, lane);
  float2* Y = (Z == reinterpret_cast<float2*>(L)) ? reinterpret_cast<float2*>(S)
                                                 : reinterpret_cast<float2*>(L);
  // real-FFT unscramble: Y[k] = sum_j y[j] exp(-2 pi i j k / n), k = 0..h
  for (int k = lane; k <= h; k += 32) {
    float2 y;
    if (k == 0 || k == h) {
      const float2 z0 = Z[0];
      y = make_float2(k == 0 ? z0.x + z0.y : z0.x - z0.y, 0.f);
    } else {
      const float2 A = Z[k];
      const float2 Bc = Z[h - k];
      const float2 B = make_float2(Bc.x, -Bc.y);
      const float2 E = make_float2(0.5f * (A.x + B.x), 0.5f * (A.y + B.y));
      const float2 D = make_float2(A.x - B.x, A.y - B.y);
      const float2 w = cmul(t.uw[k], D);
      y = make_float2(E.x + 0.5f * w.y, E.y - 0.5f * w.x);
    }
    Y[k] = y;
  }
  __syncwarp();
  // outputs: sine   S[2k] = -2 Im Y[k], S[2k+1] = Re Y[0] + 2 sum_{m=1..k} Re Y[m]
  //          cosine C[2k] =  2 Re Y[k], C[2k+1] = 2 sigma - 2 sum_{m=1..k} Im Y[m]
  const int c = (h >= 32) ? (h >> 5) : 1;
  const int active = h / c;
  float part = 0.f;
  const int k0 = lane * c;
  if (lane < active) {
    for (int i = 0; i < c; ++i) {
      const int k = k0 + i;
      const float2 y = Y[k];
      part += (parity == 0) ? (k == 0 ? y.x : 2.f * y.x) : (k == 0 ? 0.f : -2.f * y.y);
    }
  }
  float run = warp_excl_scan(part, lane);
  if (parity) run += 2.f * sigma;
  float2 yh = Y[h];
  __syncwarp();
  if (lane < active) {
    for (int i = 0; i < c; ++i) {
      const int k = k0 + i;
      const float2 y = Y[k];
      if (parity == 0) {
        run += (k == 0 ? y.x : 2.f * y.x);
        L[2 * k] = (k == 0) ? 0.f : -2.f * y.y;
      } else {
        run += (k == 0 ? 0.f : -2.f * y.y);
        L[2 * k] = 2.f * y.x;
      }
      L[2 * k + 1] = run;
    }
  }
  if (lane == 0) L[n] = parity ? 2.f * yh.x : 0.f;
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Register-resident form of the same transform for n = 64 P (P = 1..32).
//
// The n/2-point complex FFT is split as n/2 = P * 32: lane l holds the points
// m = l + 32 a (a = 0..P-1) in registers.  A P-point DFT over a runs in the
// lane's registers.  After a twiddle by exp(-2 pi i l k2 / (n/2)), a 32-point
// DFT over l runs across the lanes (radix-2 decimation in frequency with
// shuffles), which leaves Z[k2 + P * brev5(l)] in register k2 of lane l.  The
// pre-twiddle partners x[n - j], the unscramble partners Z[n/2 - k] and the
// prefix sum of the odd outputs are all lane shuffles, so the only memory
// traffic is the load of the line and one store of the result.

__device__ __forceinline__ int brev5(int v) { return (int)(__brev((unsigned)v) >> 27); }

template <int P>
__host__ __device__ constexpr int brev_p(int v) {
  int r = 0;
  for (int b = 1, rb = P >> 1; b < P; b <<= 1, rb >>= 1)
    if (v & b) r |= rb;
  return r;
}

__device__ __forceinline__ float2 shfl_xor2(float2 v, int m) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

__device__ __forceinline__ float2 shfl2(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// Unnormalised DST-I (parity 0) / DCT-I (parity 1) of the line
//   x[j] = in_scale * (in[j] + in2[j]),  j = 0..n   (in2 may be null)
// written to out[0..n] (shared memory, 16-byte aligned; may alias `in`).
// `in` and `in2` may point to global or shared memory, 8-byte aligned.
// The line of a register transform held by one lane: x[2m], x[2m+1] for
// m = lane + 32 a (a = 0..P-1) and, on lane 0, x[n].
template <int P>
struct LineRegs {
  float2 xp[P];
  float xn;
};

// 1. the line x = in_scale * (in + in2) into the lanes' registers.  A kernel
//    may issue this before it reads the device status, so that both loads
//    wait for L2 together.
template <int P>
__device__ __forceinline__ void reg_line_load(const float* in, const float* in2, float in_scale,
                                              LineRegs<P>& r, int lane) {
  constexpr int N = 64 * P;
#pragma unroll
  for (int a = 0; a < P; ++a) {
    const int m = lane + 32 * a;
    float2 v = *reinterpret_cast<const float2*>(in + 2 * m);
    if (in2) {
      const float2 w = *reinterpret_cast<const float2*>(in2 + 2 * m);
      v.x += w.x;
      v.y += w.y;
    }
    r.xp[a] = make_float2(v.x * in_scale, v.y * in_scale);
  }
  r.xn = 0.f;
  if (lane == 0) {
    float xn = in[N];
    if (in2) xn += in2[N];
    r.xn = xn * in_scale;
  }
}

// In-place 8-point DFT, natural order in and out (radix 2 x 4: the even
// outputs are the 4-point DFT of x[m] + x[m+4], the odd ones that of
// (x[m] - x[m+4]) exp(-2 pi i m / 8)).
__device__ __forceinline__ void dft8(float2 (&x)[8]) {
  const float r = 0.70710678118654752f;  // cos(pi / 4)
  const float2 a0 = make_float2(x[0].x + x[4].x, x[0].y + x[4].y);
  const float2 a1 = make_float2(x[0].x - x[4].x, x[0].y - x[4].y);
  const float2 b0 = make_float2(x[2].x + x[6].x, x[2].y + x[6].y);
  const float2 b1 = make_float2(x[2].x - x[6].x, x[2].y - x[6].y);
  const float2 c0 = make_float2(x[1].x + x[5].x, x[1].y + x[5].y);
  const float2 c1 = make_float2(x[1].x - x[5].x, x[1].y - x[5].y);
  const float2 d0 = make_float2(x[3].x + x[7].x, x[3].y + x[7].y);
  const float2 d1 = make_float2(x[3].x - x[7].x, x[3].y - x[7].y);
  // even outputs
  const float2 e0 = make_float2(a0.x + b0.x, a0.y + b0.y);
  const float2 e1 = make_float2(a0.x - b0.x, a0.y - b0.y);
  const float2 g0 = make_float2(c0.x + d0.x, c0.y + d0.y);
  const float2 g1 = make_float2(c0.x - d0.x, c0.y - d0.y);
  // odd outputs: b1 (-i), c1 exp(-i pi/4), d1 exp(-3 i pi/4)
  const float2 bb = make_float2(b1.y, -b1.x);
  const float2 cc = make_float2(r * (c1.x + c1.y), r * (c1.y - c1.x));
  const float2 dd = make_float2(r * (d1.y - d1.x), -r * (d1.x + d1.y));
  const float2 h0 = make_float2(a1.x + bb.x, a1.y + bb.y);
  const float2 h1 = make_float2(a1.x - bb.x, a1.y - bb.y);
  const float2 k0 = make_float2(cc.x + dd.x, cc.y + dd.y);
  const float2 k1 = make_float2(cc.x - dd.x, cc.y - dd.y);
  x[0] = make_float2(e0.x + g0.x, e0.y + g0.y);
  x[4] = make_float2(e0.x - g0.x, e0.y - g0.y);
  x[2] = make_float2(e1.x + g1.y, e1.y - g1.x);  // e1 - i g1
  x[6] = make_float2(e1.x - g1.y, e1.y + g1.x);  // e1 + i g1
  x[1] = make_float2(h0.x + k0.x, h0.y + k0.y);
  x[5] = make_float2(h0.x - k0.x, h0.y - k0.y);
  x[3] = make_float2(h1.x + k1.y, h1.y - k1.x);  // h1 - i k1
  x[7] = make_float2(h1.x - k1.y, h1.y + k1.x);  // h1 + i k1
}

// Steps 5-8 of the register transform for P = 8 (256-point complex FFT,
// 8 values per lane), through shared memory instead of 5 shuffle stages.
// In: w[k2] = f_k2(lane), the input of the 32-point DFT over the lanes.
// 5. The 32-point DFT as 8 x 4 (lane l = q + 4 b): the values move through
//    `out` so that lane t = 4 r + q holds f_r(q + 4 b), b = 0..7 (rows XOR-
//    swizzled by 4 (r & 3): the stores and the strided loads hit distinct
//    banks); an 8-point DFT over b, the twiddle exp(-2 pi i q c / 32), and a
//    4-point DFT over q across the four lanes of r (two shuffle stages) leave
//    Z[r + 8 (c + 8 brev2(q))] in register c.
// 6. Z goes back through `out` (swizzled by block) so that lane l holds its
//    block Z[8 l + k2] and the partners Z[256 - 8 l - k2] of the unscramble.
// 7-8. Unscramble, prefix sum and the output as in the shuffle form, with
//    the blocks in lane order.
template <int P>
__device__ __forceinline__ void reg_line_tail_xs(float2 (&w)[P], float* out, int parity,
                                                 float sigma, const float* T, const float2* uwl,
                                                 int lane) {
  static_assert(P == 8, "the exchange form is written for 512-point lines");
  constexpr int N = 64 * P;
  const unsigned FULL = 0xffffffffu;
  float2* X = reinterpret_cast<float2*>(out);  // 32 P float2 = N floats
#pragma unroll
  for (int k2 = 0; k2 < P; ++k2) X[32 * k2 + (lane ^ (4 * (k2 & 3)))] = w[k2];
  __syncwarp();
  const int r = lane >> 2, q = lane & 3;
  float2 f[8];
#pragma unroll
  for (int b = 0; b < 8; ++b) f[b] = X[32 * r + ((q + 4 * b) ^ (4 * (r & 3)))];
  dft8(f);
  const float2* w32 = reinterpret_cast<const float2*>(T + lt_w32(P)) + 8 * q;
#pragma unroll
  for (int c = 1; c < 8; ++c) f[c] = cmul(f[c], w32[c]);
  {
    // radix-2 DIF over q: lanes with bit 2 of q keep (p - v), times -i on q = 3
    const float sg = (q & 2) ? -1.f : 1.f;
    const bool rot = q == 3;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const float2 p = shfl_xor2(f[c], 2);
      const float2 d = make_float2(fmaf(sg, f[c].x, p.x), fmaf(sg, f[c].y, p.y));
      f[c] = rot ? make_float2(d.y, -d.x) : d;
    }
    const float sg1 = (q & 1) ? -1.f : 1.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const float2 p = shfl_xor2(f[c], 1);
      f[c] = make_float2(fmaf(sg1, f[c].x, p.x), fmaf(sg1, f[c].y, p.y));
    }
  }
  __syncwarp();  // every lane has read its exchange values before Z overwrites them
  const int qb = ((q & 1) << 1) | (q >> 1);  // brev2(q)
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int kap = c + 8 * qb;  // the block of this value
    X[8 * kap + (r ^ ((kap >> 1) & 7))] = f[c];
  }
  __syncwarp();
  float2 A[8], B[8];
  {
    const int sw = (lane >> 1) & 7;
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) A[k2] = X[8 * lane + (k2 ^ sw)];
    const int lp = 31 - lane, swp = (lp >> 1) & 7;
#pragma unroll
    for (int k2 = 1; k2 < 8; ++k2) B[k2] = X[8 * lp + ((8 - k2) ^ swp)];
    const int l0 = (32 - lane) & 31;
    B[0] = X[8 * l0 + ((l0 >> 1) & 7)];
  }
  float ev[P], od[P];
  float yh = 0.f;
  float run = 0.f;
#pragma unroll
  for (int k2 = 0; k2 < P; ++k2) {
    const int k = k2 + P * lane;
    const float2 a = A[k2];
    const float2 b = make_float2(B[k2].x, -B[k2].y);
    float2 Y;
    if (k == 0) {
      Y = make_float2(a.x + a.y, 0.f);
      yh = a.x - a.y;
    } else {
      const float2 E = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
      const float2 D = make_float2(a.x - b.x, a.y - b.y);
      const float2 u = cmul(uwl[32 * k2 + lane], D);
      Y = make_float2(E.x + 0.5f * u.y, E.y - 0.5f * u.x);
    }
    float term;
    if (parity == 0) {
      ev[k2] = (k == 0) ? 0.f : -2.f * Y.y;
      term = (k == 0) ? Y.x : 2.f * Y.x;
    } else {
      ev[k2] = 2.f * Y.x;
      term = (k == 0) ? 0.f : -2.f * Y.y;
    }
    run += term;
    od[k2] = run;
  }
  // exclusive scan of the block sums, blocks in lane order
  float inc = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const float u = __shfl_up_sync(FULL, inc, o);
    if (lane >= o) inc += u;
  }
  float base = inc - run;
  if (parity) base += 2.f * sigma;
  __syncwarp();  // every lane has read Z before the line overwrites it
  float* o = out + 2 * P * lane;
#pragma unroll
  for (int k2 = 0; k2 < P; k2 += 2)
    *reinterpret_cast<float4*>(o + 2 * k2) =
        make_float4(ev[k2], base + od[k2], ev[k2 + 1], base + od[k2 + 1]);
  if (lane == 0) out[N] = parity ? 2.f * yh : 0.f;
  __syncwarp();
}

// 2-8. the transform of a loaded line, written to out[0..n] (shared memory,
//      16-byte aligned; may alias the line's source)
template <int P>
__device__ __forceinline__ void reg_line_core(const LineRegs<P>& r, float* out, int parity,
                                              const float* T, int lane) {
  // T: the lane table of this line length staged in shared memory (lt_* layout)
  const float2* tw3 = reinterpret_cast<const float2*>(T + lt_tw3(P));
  const float2* tw4 = reinterpret_cast<const float2*>(T + lt_tw4(P));
  const float2* tw5 = reinterpret_cast<const float2*>(T + lt_tw5(P));
  const float2* uwl = reinterpret_cast<const float2*>(T + lt_uw(P));
  constexpr int N = 64 * P;
  const unsigned FULL = 0xffffffffu;
  const float2* xp = r.xp;
  const float xn = r.xn;
  __syncwarp();
  float sigma = 0.f;
  if (parity) {
    // sigma = 0.5 (x[0] - x[n]) + sum_{j=1}^{n-1} x[j] cos(pi j / n)
    float acc = 0.f;
#pragma unroll
    for (int a = 0; a < P; ++a) {
      const int j = 2 * (lane + 32 * a);
      if (j) acc += xp[a].x * T[lt_cs0(P) + 32 * a + lane];
      acc += xp[a].y * T[lt_cs1(P) + 32 * a + lane];
    }
    acc = warp_sum(acc);
    sigma = __shfl_sync(FULL, 0.5f * (xp[0].x - xn), 0) + acc;
  }
  // 2. pre-twiddle: z[a] = y[2m] + i y[2m+1]
  float2 z[P];
#pragma unroll
  for (int a = 0; a < P; ++a) {
    const int m = lane + 32 * a;
    float r0 = __shfl_sync(FULL, xp[P - 1 - a].x, (32 - lane) & 31);  // x[n - 2m]
    if (lane == 0) r0 = (a == 0) ? xn : xp[(P - a) % P].x;
    const float r1 = __shfl_xor_sync(FULL, xp[P - 1 - a].y, 31);  // x[n - 2m - 1]
    const float s0 = T[lt_sn0(P) + 32 * a + lane], s1 = T[lt_sn1(P) + 32 * a + lane];
    const float x0 = xp[a].x, x1 = xp[a].y;
    float y0, y1;
    if (parity == 0) {
      y0 = (m == 0) ? 0.f : s0 * (x0 + r0) + 0.5f * (x0 - r0);
      y1 = s1 * (x1 + r1) + 0.5f * (x1 - r1);
    } else {
      y0 = 0.5f * (x0 + r0) - s0 * (x0 - r0);
      y1 = 0.5f * (x1 + r1) - s1 * (x1 - r1);
    }
    z[a] = make_float2(y0, y1);
  }
  // 3. P-point DFT over a in registers (radix-2 DIF, output in bit-reversed order);
  //    exp(-2 pi i k / 32) = tw[k P]
#pragma unroll
  for (int s = P / 2; s >= 1; s >>= 1) {
#pragma unroll
    for (int i = 0; i < P; ++i) {
      if (!(i & s)) {
        const float2 A = z[i], B = z[i + s];
        z[i] = make_float2(A.x + B.x, A.y + B.y);
        float2 D = make_float2(A.x - B.x, A.y - B.y);
        const int k = (i & (s - 1)) * (16 / s);
        if (k == 8)
          D = make_float2(D.y, -D.x);  // exp(-2 pi i 8 / 32) = -i
        else if (k)
          D = cmul(D, tw3[k]);
        z[i + s] = D;
      }
    }
  }
  float2 w[P];
#pragma unroll
  for (int k2 = 0; k2 < P; ++k2) w[k2] = z[brev_p<P>(k2)];
  // 4. twiddle exp(-2 pi i lane k2 / (n/2))
#pragma unroll
  for (int k2 = 1; k2 < P; ++k2) w[k2] = cmul(w[k2], tw4[32 * k2 + lane]);
  if constexpr (line_xs(P)) {
    reg_line_tail_xs<P>(w, out, parity, sigma, T, uwl, lane);
    return;
  } else {
    // 5. 32-point DFT across the lanes (radix-2 DIF with shuffles): the lower
    //    lane of a pair keeps v + p, the upper one (p - v) * twiddle; written as
    //    fma(sign, v, p) times a twiddle that is 1 on the lower lanes (and on
    //    every lane in the last stage)
  #pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
      const bool hi = (lane & s) != 0;
      const float sg = hi ? -1.f : 1.f;
      // the table holds (1, 0) for the lower lanes of each stage
      const int si = (s == 16) ? 0 : (s == 8) ? 1 : (s == 4) ? 2 : 3;
      const float2 tws = (s > 1) ? tw5[32 * si + lane] : make_float2(1.f, 0.f);
  #pragma unroll
      for (int k2 = 0; k2 < P; ++k2) {
        const float2 v = w[k2];
        const float2 p = shfl_xor2(v, s);
        const float2 d = make_float2(fmaf(sg, v.x, p.x), fmaf(sg, v.y, p.y));
        w[k2] = (s > 1) ? cmul(d, tws) : d;
      }
    }
    // 6. real-FFT unscramble: Y[k] = sum_j y[j] exp(-2 pi i j k / n), k = k2 + P k1
    const int k1 = brev5(lane);
    const int src0 = brev5((32 - k1) & 31);
    float ev[P], od[P];
    float yh = 0.f;
    float run = 0.f;
  #pragma unroll
    for (int k2 = 0; k2 < P; ++k2) {
      float2 B = (k2 == 0) ? shfl2(w[0], src0) : shfl_xor2(w[(P - k2) % P], 31);
      B.y = -B.y;
      const int k = k2 + P * k1;
      const float2 A = w[k2];
      float2 Y;
      if (k == 0) {
        Y = make_float2(A.x + A.y, 0.f);
        yh = A.x - A.y;
      } else {
        const float2 E = make_float2(0.5f * (A.x + B.x), 0.5f * (A.y + B.y));
        const float2 D = make_float2(A.x - B.x, A.y - B.y);
        const float2 q = cmul(uwl[32 * k2 + lane], D);
        Y = make_float2(E.x + 0.5f * q.y, E.y - 0.5f * q.x);
      }
      // sine:   out[2k] = -2 Im Y[k], out[2k+1] = Re Y[0] + 2 sum_{m=1..k} Re Y[m]
      // cosine: out[2k] =  2 Re Y[k], out[2k+1] = 2 sigma - 2 sum_{m=1..k} Im Y[m]
      float term;
      if (parity == 0) {
        ev[k2] = (k == 0) ? 0.f : -2.f * Y.y;
        term = (k == 0) ? Y.x : 2.f * Y.x;
      } else {
        ev[k2] = 2.f * Y.x;
        term = (k == 0) ? 0.f : -2.f * Y.y;
      }
      run += term;
      od[k2] = run;
    }
    // 7. exclusive scan of the block sums in block order k1
    const float blk = __shfl_sync(FULL, run, k1);  // lane l: sum of block l
    float inc = blk;
  #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const float u = __shfl_up_sync(FULL, inc, o);
      if (lane >= o) inc += u;
    }
    float base = __shfl_sync(FULL, inc - blk, k1);
    if (parity) base += 2.f * sigma;
    __syncwarp();
    // 8. out[2k], out[2k+1] for the lane's block k = P k1 .. P k1 + P - 1
    float* o = out + 2 * P * k1;
    if (P == 1) {
      *reinterpret_cast<float2*>(o) = make_float2(ev[0], base + od[0]);
    } else {
  #pragma unroll
      for (int k2 = 0; k2 < P; k2 += 2)
        *reinterpret_cast<float4*>(o + 2 * k2) =
            make_float4(ev[k2], base + od[k2], ev[(k2 + 1) % P], base + od[(k2 + 1) % P]);
    }
    if (lane == 0) out[N] = parity ? 2.f * yh : 0.f;
    __syncwarp();
  }
}

template <int P>
__device__ __forceinline__ void reg_line(const float* in, const float* in2, float in_scale,
                                         float* out, int parity, const float* T, int lane) {
  LineRegs<P> r;
  reg_line_load<P>(in, in2, in_scale, r, lane);
  reg_line_core<P>(r, out, parity, T, lane);
}

// Per-warp line transform of x = in_scale * (in + in2) into the shared line
// `sline` (16-byte aligned, n + 4 floats).  P = n / 64 selects the register
// form; P = 0 (lines shorter than 64 points) goes through `sline` and the
// shared scratch `sscr` (n + 4 floats) with the shared-memory form.  Kernels
// are instantiated per P (QP_LINE_SWITCH) so that each holds only the
// registers its line length needs.
template <int P>
__device__ __forceinline__ void line_transform(const float* in, const float* in2, float in_scale,
                                               float* sline, float* sscr, int logn, int parity,
                                               const LineTables& t, const float* T, int lane) {
  if constexpr (P > 0) {
    reg_line<P>(in, in2, in_scale, sline, parity, T, lane);
  } else {
    const int n = 1 << logn;
    float v[2];
    // the line may alias sline: read everything before writing
    int c = 0;
    for (int j = lane; j <= n; j += 32) {
      float x = in[j];
      if (in2) x += in2[j];
      v[c++] = x * in_scale;
    }
    __syncwarp();
    c = 0;
    for (int j = lane; j <= n; j += 32) sline[j] = v[c++];
    __syncwarp();
    warp_line_transform(sline, sscr, logn, parity, t, lane);
  }
}

constexpr int line_p(int logn) { return logn < 6 ? 0 : 1 << (logn - 6); }

// Runs STMT with the compile-time constant P_ = line_p(logn).
#define QP_LINE_SWITCH(logn, STMT)                \
  switch (logn) {                                 \
    case 6: { constexpr int P_ = 1; STMT; } break;   \
    case 7: { constexpr int P_ = 2; STMT; } break;   \
    case 8: { constexpr int P_ = 4; STMT; } break;   \
    case 9: { constexpr int P_ = 8; STMT; } break;   \
    case 10: { constexpr int P_ = 16; STMT; } break; \
    case 11: { constexpr int P_ = 32; STMT; } break; \
    default: { constexpr int P_ = 0; STMT; } break;  \
  }

// Copy the lane table of a line length into shared memory (all threads of the
// block; the caller synchronises before the first transform).
__device__ __forceinline__ void stage_lane_table(float* T, const LineTables& t) {
  const float4* src = reinterpret_cast<const float4*>(t.lane);
  float4* dst = reinterpret_cast<float4*>(T);
  for (int i = threadIdx.x; i < (t.lane_floats >> 2); i += blockDim.x) dst[i] = __ldg(src + i);
}

// Coalesced copy of a shared line (n + 1 floats) to global memory, times sc.
__device__ __forceinline__ void line_store(float* dst, const float* sline, int n, float sc,
                                           int lane) {
  const float4* s4 = reinterpret_cast<const float4*>(sline);
  float4* d4 = reinterpret_cast<float4*>(dst);
  for (int i = lane; i < (n >> 2); i += 32) {
    const float4 v = s4[i];
    d4[i] = make_float4(v.x * sc, v.y * sc, v.z * sc, v.w * sc);
  }
  if (lane == 0) dst[n] = sline[n] * sc;
}

}  // namespace qp
