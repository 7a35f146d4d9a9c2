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

}  // namespace qp
