// qp_oracle.cpp -- CPU restatement of the QuickPIC per-slice hot path.
//
// TEST INFRASTRUCTURE ONLY (the checker; see qp_oracle.h).  PARITY UNPINNED:
// the reference has no golden vectors and cannot be compiled here, so this
// restatement is pinned by known-answer tests instead (tests/golden/).
//
// Every routine below restates one Fortran routine of QuickPIC-OpenSource and
// cites it as file:line.  Index arithmetic keeps the Fortran 1-based form
// through small accessor macros so each line can be compared with the source.
// `T` is the reference's `real` (float for PRECISION=SGL, double for DBL);
// variables the reference declares `double precision` stay double.

#include "qp_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

namespace {

constexpr int MX = 16, MY = 16;  // tile size, part2d_class.f03:99

template <class T>
struct Tables {
  // WPFST2RINIT, fft2d_lib77.f:3-50
  std::vector<int> mixup;
  std::vector<std::complex<T>> sctd;
  int indx, indy, nx, ny, nxy, nxhy;
  Tables(int indx_, int indy_) : indx(indx_), indy(indy_) {
    int indx1 = indx - 1;
    int indx1y = std::max(indx1, indy);
    nx = 1 << indx;
    ny = 1 << indy;
    nxy = std::max(nx, ny);
    nxhy = 1 << indx1y;
    mixup.resize(nxhy);
    for (int j = 1; j <= nxhy; ++j) {
      int lb = j - 1, ll = 0;
      for (int k = 1; k <= indx1y; ++k) {
        int jb = lb / 2;
        int it = lb - 2 * jb;
        lb = jb;
        ll = 2 * ll + it;
      }
      mixup[j - 1] = ll + 1;
    }
    sctd.resize(nxy);
    T dnxy = T(0.5) * T(6.28318530717959) / T(nxy);
    for (int j = 1; j <= nxy; ++j) {
      T arg = dnxy * T(j - 1);
      sctd[j - 1] = std::complex<T>(std::cos(arg), -std::sin(arg));
    }
  }
};

// One line of the Numerical-Recipes real sine (parity 0) or cosine (parity 1)
// transform, as the reference applies it per row or column.
//   x pass: PPFST2RMXX fft2d_lib77.f:4791-4964, PPFCT2RMXX 4966-5141
//   y pass: PPFST2RMXY fft2d_lib77.f:5143-5316, PPFCT2RMXY 5318-5493
// The x and y passes are the same algorithm on a line of n = 2**ind points;
// they differ only in the unscramble normalisation: x uses ani = 0.5/(nx*ny)
// for isign < 0, y uses 0.5; both use 1 for isign > 0.  The multi-component
// variants (PPFCST2RM2X ... PPFSSCT2RM23Y, fft2d_lib77.f:5659-9168) are the
// same per-component operations fused in one loop.
template <class T>
void nr_line(T* p, int s, int parity, int xpass, int isign, const Tables<T>& tb) {
#define F(j) p[((j)-1) * (ptrdiff_t)s]
  const int ind = xpass ? tb.indx : tb.indy;
  const int n = 1 << ind, nh = n / 2, nhh = n / 4, n3 = n + 3;
  const int nxy = tb.nxy, nxhy = tb.nxhy;
  const int nrb = nxhy / nh, nr = nxy / nh;
  T a, b;
  if (isign < 0) {
    if (xpass) {
      T ani = T(0.5) / (T(tb.nx) * T(tb.ny));
      a = ani;
      b = T(2.0) * ani;
    } else {
      a = T(0.5);
      b = T(1.0);
    }
  } else {
    a = T(1.0);
    b = T(2.0);
  }
  // create auxiliary array
  int kmr = nxy / n;
  double sum1 = 0.0;
  if (parity == 0) {
    for (int j = 2; j <= nh; ++j) {
      int j1 = 1 + kmr * (j - 1);
      T at2 = F(n + 2 - j);
      T at1 = F(j) + at2;
      at2 = F(j) - at2;
      at1 = -tb.sctd[j1 - 1].imag() * at1;
      at2 = T(0.5) * at2;
      F(j) = at1 + at2;
      F(n + 2 - j) = at1 - at2;
    }
    F(1) = T(0.0);
    F(nh + 1) = T(2.0) * F(nh + 1);
  } else {
    sum1 = (double)(T(0.5) * (F(1) - F(n + 1)));
    for (int j = 2; j <= nh; ++j) {
      int j1 = 1 + kmr * (j - 1);
      T at2 = F(n + 2 - j);
      T at1 = F(j) + at2;
      at2 = F(j) - at2;
      sum1 = sum1 + (double)(tb.sctd[j1 - 1].real() * at2);
      at2 = -tb.sctd[j1 - 1].imag() * at2;
      at1 = T(0.5) * at1;
      F(j) = at1 - at2;
      F(n + 2 - j) = at1 + at2;
    }
    F(1) = T(0.5) * (F(1) + F(n + 1));
    F(n + 1) = (T)sum1;
  }
  // bit-reverse array elements
  for (int j = 1; j <= nh; ++j) {
    int j1 = (tb.mixup[j - 1] - 1) / nrb + 1;
    if (j < j1) {
      T t2 = F(2 * j1 - 1), t3 = F(2 * j1);
      F(2 * j1 - 1) = F(2 * j - 1);
      F(2 * j1) = F(2 * j);
      F(2 * j - 1) = t2;
      F(2 * j) = t3;
    }
  }
  // then transform
  for (int m = 1; m <= ind - 1; ++m) {
    int ns = 1 << (m - 1), ns2 = ns + ns, km = nhh / ns;
    int kmr2 = 2 * km * nr;
    for (int k = 1; k <= km; ++k) {
      int k1 = ns2 * (k - 1), k2 = k1 + ns;
      for (int j = 1; j <= ns; ++j) {
        int j1 = j + k1, j2 = j + k2;
        std::complex<T> t1 = tb.sctd[1 + kmr2 * (j - 1) - 1];
        T t2 = t1.real() * F(2 * j2 - 1) - t1.imag() * F(2 * j2);
        T t3 = t1.imag() * F(2 * j2 - 1) + t1.real() * F(2 * j2);
        F(2 * j2 - 1) = F(2 * j1 - 1) - t2;
        F(2 * j2) = F(2 * j1) - t3;
        F(2 * j1 - 1) = F(2 * j1 - 1) + t2;
        F(2 * j1) = F(2 * j1) + t3;
      }
    }
  }
  // unscramble coefficients and normalize
  kmr = nxy / nh;
  for (int j = 2; j <= nhh; ++j) {
    std::complex<T> sc = tb.sctd[1 + kmr * (j - 1) - 1];
    T t1r = sc.imag(), t1i = -sc.real();
    T t4 = F(n3 - 2 * j);
    T t5 = -F(n3 - 2 * j + 1);
    T t2 = F(2 * j - 1) + t4;
    T t3 = F(2 * j) + t5;
    T t6 = F(2 * j - 1) - t4;
    t5 = F(2 * j) - t5;
    t4 = t6 * t1r - t5 * t1i;
    t5 = t6 * t1i + t5 * t1r;
    F(2 * j - 1) = a * (t2 + t4);
    F(2 * j) = a * (t3 + t5);
    F(n3 - 2 * j) = a * (t2 - t4);
    F(n3 - 2 * j + 1) = a * (t5 - t3);
  }
  F(nh + 1) = b * F(nh + 1);
  F(nh + 2) = -(b * F(nh + 2));
  {
    T t2 = b * (F(1) + F(2));
    F(2) = b * (F(1) - F(2));
    F(1) = t2;
  }
  F(n + 1) = b * F(n + 1);
  // perform recursion
  if (parity == 0) {
    sum1 = (double)(T(0.5) * F(1));
    F(1) = T(0.0);
    F(2) = (T)sum1;
    for (int j = 2; j <= nh; ++j) {
      sum1 = sum1 + (double)F(2 * j - 1);
      F(2 * j - 1) = -F(2 * j);
      F(2 * j) = (T)sum1;
    }
    F(n + 1) = T(0.0);
  } else {
    sum1 = (double)F(n + 1);
    F(n + 1) = F(2);
    F(2) = (T)sum1;
    for (int j = 2; j <= nh; ++j) {
      sum1 = sum1 - (double)F(2 * j);
      F(2 * j) = (T)sum1;
    }
  }
#undef F
}

// Parities (x, y) of every component for the field2d transform kinds,
// field2d_class.f03:157-227 -> fft2d_class.f03:121-413 -> the wrappers
// WPPFSST2RM 4479, WPPFCCT2RM 4713, WPPFCST2RM2 5495, WPPFSCT2RM2 5577,
// WPPFCST2RM3 6495, WPPFSCT2RM3 6577, WPPFSST2RM23 8640 (fft2d_lib77.f).
// 0 = sine, 1 = cosine.
bool kind_parity(int dim, int kind, int c, int* px, int* py) {
  static const int p1[3][2] = {{0, 0}, {1, 1}, {0, 0}};
  static const int p2[2][2][2] = {{{1, 0}, {0, 1}}, {{0, 1}, {1, 0}}};
  static const int p3[3][3][2] = {{{1, 0}, {0, 1}, {0, 0}},
                                  {{0, 1}, {1, 0}, {1, 1}},
                                  {{0, 0}, {0, 0}, {1, 1}}};
  if (dim == 1 && (kind == 1 || kind == 2)) {
    *px = p1[kind - 1][0];
    *py = p1[kind - 1][1];
    return true;
  }
  if (dim == 2 && (kind == 1 || kind == 2)) {
    *px = p2[kind - 1][c][0];
    *py = p2[kind - 1][c][1];
    return true;
  }
  if (dim == 3 && kind >= 1 && kind <= 3) {
    *px = p3[kind - 1][c][0];
    *py = p3[kind - 1][c][1];
    return true;
  }
  return false;
}

// Index helpers for the reference layouts.
struct Grid {
  int indx, indy, nx, ny, nxv, nypmx, nyv, kxp2d;
  Grid(int ix, int iy) : indx(ix), indy(iy) {
    nx = 1 << ix;
    ny = 1 << iy;
    nxv = nx + 2;
    nypmx = 2 * ny + 1;
    nyv = ny + 1;
    kxp2d = nx + 1;
  }
  size_t rs_size(int dim) const { return (size_t)dim * nxv * nypmx; }
  size_t ks_size(int dim) const { return (size_t)dim * nyv * kxp2d; }
  // rf(c, j, k), 1-based j (x) and k (y)
  size_t r(int dim, int c, int j, int k) const {
    return (size_t)(c - 1) + (size_t)dim * ((size_t)(j - 1) + (size_t)nxv * (size_t)(k - 1));
  }
  // g(c, k, j), 1-based k (ky) and j (kx)
  size_t g(int dim, int c, int k, int j) const {
    return (size_t)(c - 1) + (size_t)dim * ((size_t)(k - 1) + (size_t)nyv * (size_t)(j - 1));
  }
};

// PPNCGUARD2L single-rank branch, ufield2d_lib.f03:37-42: row ny+1 = row 1
template <class T>
void cguard(T* rs, int dim, const Grid& G) {
  size_t nxvt = (size_t)dim * G.nxv;
  for (size_t j = 0; j < nxvt; ++j) rs[j + nxvt * (size_t)G.ny] = rs[j];
}

// PPNACGUARD2L single-rank branch, ufield2d_lib.f03:90-97
template <class T>
void acguard(T* rs, int dim, const Grid& G) {
  for (int j = 1; j <= G.nx + 1; ++j)
    for (int c = 1; c <= dim; ++c) {
      rs[G.r(dim, c, j, 1)] = rs[G.r(dim, c, j, 1)] + rs[G.r(dim, c, j, G.ny + 1)];
      rs[G.r(dim, c, j, G.ny + 1)] = T(0);
    }
}

// fftrk: x pass over rows 1..ny+1, transpose (PPRTPOSE nvp=1,
// fft2d_lib.f03:675-683), y pass over columns 1..nx+1; result stays in g
// (ntpose = 1, fft2d_class.f03:139).
template <class T>
int fftrk(T* rs, T* ks, int dim, int kind, const Grid& G) {
  Tables<T> tb(G.indx, G.indy);
  int px[3], py[3];
  for (int c = 0; c < dim; ++c)
    if (!kind_parity(dim, kind, c, &px[c], &py[c])) return -1;
  for (int c = 1; c <= dim; ++c) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= G.ny + 1; ++i)
      nr_line(&rs[G.r(dim, c, 1, i)], dim, px[c - 1], 1, -1, tb);
  }
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= G.nx + 1; ++j)
    for (int k = 1; k <= G.ny + 1; ++k)
      for (int c = 1; c <= dim; ++c) ks[G.g(dim, c, k, j)] = rs[G.r(dim, c, j, k)];
  for (int c = 1; c <= dim; ++c) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= G.nx + 1; ++i)
      nr_line(&ks[G.g(dim, c, 1, i)], dim, py[c - 1], 0, -1, tb);
  }
  return 0;
}

// fftkr: y pass on g, transpose back, x pass; then the guard copy that
// fftkr_field2d performs (field2d_class.f03:222 -> ufield2d copyguard).
template <class T>
int fftkr(T* rs, T* ks, int dim, int kind, const Grid& G) {
  Tables<T> tb(G.indx, G.indy);
  int px[3], py[3];
  for (int c = 0; c < dim; ++c)
    if (!kind_parity(dim, kind, c, &px[c], &py[c])) return -1;
  for (int c = 1; c <= dim; ++c) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= G.nx + 1; ++i)
      nr_line(&ks[G.g(dim, c, 1, i)], dim, py[c - 1], 0, 1, tb);
  }
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= G.ny + 1; ++k)
    for (int j = 1; j <= G.nx + 1; ++j)
      for (int c = 1; c <= dim; ++c) rs[G.r(dim, c, j, k)] = ks[G.g(dim, c, k, j)];
  for (int c = 1; c <= dim; ++c) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= G.ny + 1; ++i)
      nr_line(&rs[G.r(dim, c, 1, i)], dim, px[c - 1], 1, 1, tb);
  }
  cguard(rs, dim, G);
  return 0;
}

// ---------------------------------------------------------------- solves
// Form-factor table, MPPOISD22 isign = 0, fpois2d_lib77.f:1509-1531, as
// prepared by ippoisd2init (fpois2d_class.f03:127-148).  Stored as
// (re, im) pairs of ffd(k, j), k = 1..ny, j = 1..nx.
template <class T>
void ffc_init(T* ffc, const Grid& G, T ax, T ay, T affp) {
  T dnx = T(6.28318530717959) / T(G.nx + G.nx);
  T dny = T(6.28318530717959) / T(G.ny + G.ny);
  int joff = -1;
  for (int j = 1; j <= G.nx; ++j) {
    T dkx = dnx * T(j + joff);
    T at1 = dkx * dkx;
    T at2 = (dkx * ax) * (dkx * ax);
    for (int k = 1; k <= G.ny; ++k) {
      T dky = dny * T(k - 1);
      T at3 = dky * dky + at1;
      T at4 = std::exp(-T(0.5) * ((dky * ay) * (dky * ay) + at2));
      size_t o = 2 * ((size_t)(k - 1) + (size_t)G.ny * (size_t)(j - 1));
      if (at3 == T(0)) {
        ffc[o] = affp;
        ffc[o + 1] = T(1.0);
      } else {
        ffc[o] = affp * at4 / at3;
        ffc[o + 1] = at4;
      }
    }
  }
}
#define FRE(k, j) ffc[2 * ((size_t)((k)-1) + (size_t)G.ny * (size_t)((j)-1))]
#define FIM(k, j) ffc[2 * ((size_t)((k)-1) + (size_t)G.ny * (size_t)((j)-1)) + 1]

// MPPOTPD2, fpois2d_lib77.f:1701-1779 (potential; field energy discarded)
template <class T>
void pot(const T* q, T* p, const T* ffc, const Grid& G) {
  int ny = G.ny, nx = G.nx;
  for (int j = 1; j <= nx; ++j) {
    if (j - 1 > 0) {
      for (int k = 2; k <= ny; ++k) {
        T at2 = FRE(k, j);
        T at3 = at2 * q[G.g(1, 1, k, j)];
        p[G.g(1, 1, k, j)] = at3;
      }
    }
    p[G.g(1, 1, 1, j)] = T(0);
    p[G.g(1, 1, ny + 1, j)] = T(0);
  }
  for (int k = 2; k <= ny; ++k) p[G.g(1, 1, k, 1)] = T(0);
  for (int k = 1; k <= ny + 1; ++k) p[G.g(1, 1, k, nx + 1)] = T(0);
}

// MPPSMOOTHD2, fpois2d_lib77.f:1781-1843
template <class T>
void smooth(const T* q, T* qs, const T* ffc, const Grid& G) {
  int ny = G.ny, nx = G.nx;
  for (int j = 1; j <= nx; ++j) {
    if (j - 1 > 0) {
      for (int k = 2; k <= ny; ++k) {
        T at1 = FIM(k, j);
        qs[G.g(1, 1, k, j)] = at1 * q[G.g(1, 1, k, j)];
      }
    }
    qs[G.g(1, 1, 1, j)] = T(0);
    qs[G.g(1, 1, ny + 1, j)] = T(0);
  }
  for (int k = 2; k <= ny; ++k) qs[G.g(1, 1, k, 1)] = T(0);
  for (int k = 1; k <= ny + 1; ++k) qs[G.g(1, 1, k, nx + 1)] = T(0);
}

// MPPOISD22 isign /= 0, fpois2d_lib77.f:1532-1575 (beam E-field, elf)
template <class T>
void elf(const T* q, T* fxy, const T* ffc, const Grid& G) {
  int ny = G.ny, nx = G.nx;
  T dnx = T(6.28318530717959) / T(nx + nx);
  T dny = T(6.28318530717959) / T(ny + ny);
  for (int j = 1; j <= nx; ++j) {
    T dkx = dnx * T(j - 1);
    if (j - 1 > 0) {
      for (int k = 2; k <= ny; ++k) {
        T at1 = FRE(k, j) * FIM(k, j);
        T at3 = -at1 * q[G.g(1, 1, k, j)];
        T at2 = dkx * at3;
        at3 = dny * T(k - 1) * at3;
        fxy[G.g(2, 1, k, j)] = at2;
        fxy[G.g(2, 2, k, j)] = at3;
      }
    }
    fxy[G.g(2, 1, 1, j)] = T(0);
    fxy[G.g(2, 2, 1, j)] = T(0);
    fxy[G.g(2, 1, ny + 1, j)] = T(0);
    fxy[G.g(2, 2, ny + 1, j)] = T(0);
  }
  for (int k = 2; k <= ny; ++k) {
    fxy[G.g(2, 1, k, 1)] = T(0);
    fxy[G.g(2, 2, k, 1)] = T(0);
  }
  for (int k = 1; k <= ny + 1; ++k) {
    fxy[G.g(2, 1, k, nx + 1)] = T(0);
    fxy[G.g(2, 2, k, nx + 1)] = T(0);
  }
}

// MPPBBPOISD23, fpois2d_lib77.f:1845-1956 (B from J, ci = 1)
template <class T>
void bf(const T* cu, T* bxy, const T* ffc, const Grid& G) {
  int ny = G.ny, nx = G.nx;
  T dnx = T(6.28318530717959) / T(nx + nx);
  T dny = T(6.28318530717959) / T(ny + ny);
  T ci = T(1.0), ci2 = ci * ci;
  for (int j = 1; j <= nx; ++j) {
    T dkx = dnx * T(j - 1);
    if (j - 1 > 0) {
      for (int k = 2; k <= ny; ++k) {
        T dky = dny * T(k - 1);
        T at1 = ci2 * FRE(k, j) * FIM(k, j);
        T at2 = dky * at1;
        T at3 = dkx * at1;
        bxy[G.g(3, 1, k, j)] = at2 * cu[G.g(3, 3, k, j)];
        bxy[G.g(3, 2, k, j)] = -at3 * cu[G.g(3, 3, k, j)];
        bxy[G.g(3, 3, k, j)] = at3 * cu[G.g(3, 2, k, j)] - at2 * cu[G.g(3, 1, k, j)];
      }
      T at1 = ci2 * FRE(1, j) * FIM(1, j);
      T at2 = dkx * at1;
      bxy[G.g(3, 1, 1, j)] = T(0);
      bxy[G.g(3, 2, 1, j)] = T(0);
      bxy[G.g(3, 3, 1, j)] = at2 * cu[G.g(3, 2, 1, j)];
    }
    bxy[G.g(3, 1, ny + 1, j)] = T(0);
    bxy[G.g(3, 2, ny + 1, j)] = T(0);
    bxy[G.g(3, 3, ny + 1, j)] = T(0);
  }
  for (int k = 2; k <= ny; ++k) {
    T dky = dny * T(k - 1);
    T at1 = ci2 * FRE(k, 1) * FIM(k, 1);
    T at2 = dky * at1;
    bxy[G.g(3, 1, k, 1)] = T(0);
    bxy[G.g(3, 2, k, 1)] = T(0);
    bxy[G.g(3, 3, k, 1)] = -at2 * cu[G.g(3, 1, k, 1)];
  }
  bxy[G.g(3, 1, 1, 1)] = T(0);
  bxy[G.g(3, 2, 1, 1)] = T(0);
  bxy[G.g(3, 3, 1, 1)] = T(0);
  for (int k = 1; k <= ny + 1; ++k)
    for (int c = 1; c <= 3; ++c) bxy[G.g(3, c, k, nx + 1)] = T(0);
}

// PBPOISD23 isign = 1, fpois2d_lib77.f:1085-1133, as called by ivppoisd2
// (fpois2d_class.f03:242-271) with ci = 1: the vector potential
// a(kx,ky) = ci^2 g(kx,ky) s(kx,ky) cu(kx,ky), with the reference's mode rules
// (ky = 0: y only; kx = 0: x only; ky = ny, kx = nx and (0,0): zero).
template <class T>
void vpot(const T* cu, T* a, const T* ffc, const Grid& G) {
  int ny = G.ny, nx = G.nx;
  T ci = T(1.0), ci2 = ci * ci;
  for (int j = 1; j <= nx; ++j) {
    if (j - 1 > 0) {
      for (int k = 2; k <= ny; ++k) {
        T at2 = ci2 * FRE(k, j);
        T at1 = at2 * FIM(k, j);
        a[G.g(3, 1, k, j)] = at1 * cu[G.g(3, 1, k, j)];
        a[G.g(3, 2, k, j)] = at1 * cu[G.g(3, 2, k, j)];
        a[G.g(3, 3, k, j)] = at1 * cu[G.g(3, 3, k, j)];
      }
      T at2 = ci2 * FRE(1, j);
      T at1 = at2 * FIM(1, j);
      a[G.g(3, 1, 1, j)] = T(0);
      a[G.g(3, 2, 1, j)] = at1 * cu[G.g(3, 2, 1, j)];
      a[G.g(3, 3, 1, j)] = T(0);
    }
    a[G.g(3, 1, ny + 1, j)] = T(0);
    a[G.g(3, 2, ny + 1, j)] = T(0);
    a[G.g(3, 3, ny + 1, j)] = T(0);
  }
  for (int k = 2; k <= ny; ++k) {
    T at2 = ci2 * FRE(k, 1);
    T at1 = at2 * FIM(k, 1);
    a[G.g(3, 1, k, 1)] = at1 * cu[G.g(3, 1, k, 1)];
    a[G.g(3, 2, k, 1)] = T(0);
    a[G.g(3, 3, k, 1)] = T(0);
  }
  a[G.g(3, 1, 1, 1)] = T(0);
  a[G.g(3, 2, 1, 1)] = T(0);
  a[G.g(3, 3, 1, 1)] = T(0);
  for (int k = 1; k <= ny + 1; ++k)
    for (int c = 1; c <= 3; ++c) a[G.g(3, c, k, nx + 1)] = T(0);
}

// PBPOISD22N_QP isign = 1, fpois2d_lib77.f:1322-1421, as called by
// jpbpoisd23n_qp (fpois2d_class.f03:444-495) with kxp2 = nx, ci = 1:
// the transverse-B corrector.  dcu is modified in place.
template <class T>
void bfqp(const T* cu, T* dcu, const T* amu, T* bxy, const T* ffc, T aa, T dex,
          const Grid& G) {
  int ny = G.ny, nx = G.nx;
  T idex = T(1.0) / dex;
  T dnx = T(6.28318530717959) / T(nx + nx);
  T dny = T(6.28318530717959) / T(ny + ny);
  T ci = T(1.0), ci2 = ci * ci;
#define CU(c, k, j) cu[G.g(3, c, k, j)]
#define DCU(c, k, j) dcu[G.g(2, c, k, j)]
#define AMU(c, k, j) amu[G.g(3, c, k, j)]
#define BXY(c, k, j) bxy[G.g(2, c, k, j)]
  for (int j = 1; j <= nx; ++j) {
    T dkx = dnx * T(j - 1);
    if (j - 1 > 0) {
      for (int k = 2; k <= ny; ++k) {
        T dky = dny * T(k - 1);
        DCU(1, k, j) = -DCU(1, k, j) + dkx * AMU(1, k, j) - dky * AMU(3, k, j);
        T aat1 = DCU(1, k, j) - dkx * CU(3, k, j) * idex;
        DCU(2, k, j) = -DCU(2, k, j) - dkx * AMU(3, k, j) + dky * AMU(2, k, j);
        T aat2 = DCU(2, k, j) - dky * CU(3, k, j) * idex;
        T at2 = FRE(k, j);
        at2 = ci2 * at2 / (T(1) + aa * at2);
        T at1 = at2 * FIM(k, j);
        BXY(1, k, j) = at1 * aat1 + aa * at2 * BXY(1, k, j);
        BXY(2, k, j) = at1 * aat2 + aa * at2 * BXY(2, k, j);
      }
      DCU(1, 1, j) = -DCU(1, 1, j) + dkx * AMU(1, 1, j);
      DCU(2, 1, j) = -DCU(2, 1, j) - dkx * AMU(3, 1, j);
      T at2 = FRE(1, j);
      at2 = ci2 * at2 / (T(1) + aa * at2);
      T at1 = at2 * FIM(1, j);
      BXY(1, 1, j) = T(0);
      BXY(2, 1, j) = at1 * DCU(2, 1, j) + aa * at2 * BXY(2, 1, j);
    }
    BXY(1, ny + 1, j) = T(0);
    BXY(2, ny + 1, j) = T(0);
  }
  for (int k = 2; k <= ny; ++k) {
    T dky = dny * T(k - 1);
    DCU(1, k, 1) = -DCU(1, k, 1) - dky * AMU(3, k, 1);
    DCU(2, k, 1) = -DCU(2, k, 1) + dky * AMU(2, k, 1);
    T at2 = FRE(k, 1);
    at2 = ci2 * at2 / (T(1) + aa * at2);
    T at1 = at2 * FIM(k, 1);
    BXY(1, k, 1) = at1 * DCU(1, k, 1) + aa * at2 * BXY(1, k, 1);
    BXY(2, k, 1) = T(0);
  }
  BXY(1, 1, 1) = T(0);
  BXY(2, 1, 1) = T(0);
  for (int k = 1; k <= ny + 1; ++k) {
    BXY(1, k, nx + 1) = T(0);
    BXY(2, k, nx + 1) = T(0);
  }
#undef CU
#undef DCU
#undef AMU
#undef BXY
}

// MPPDIVFD2, fft2d_lib77.f:9170-9229 (uses components 1 and 2 of f)
template <class T>
void divf(const T* f, T* df, int ndim, const Grid& G) {
  int ny = G.ny, nx = G.nx;
  T dnx = T(6.28318530717959) / T(nx + nx);
  T dny = T(6.28318530717959) / T(ny + ny);
  for (int j = 1; j <= nx; ++j) {
    T dkx = dnx * T(j - 1);
    if (j - 1 > 0) {
      for (int k = 2; k <= ny; ++k) {
        T dky = dny * T(k - 1);
        df[G.g(1, 1, k, j)] = -(dkx * f[G.g(ndim, 1, k, j)] + dky * f[G.g(ndim, 2, k, j)]);
      }
    }
    df[G.g(1, 1, 1, j)] = T(0);
    df[G.g(1, 1, ny + 1, j)] = T(0);
  }
  for (int k = 2; k <= ny; ++k) df[G.g(1, 1, k, 1)] = T(0);
  for (int k = 1; k <= ny + 1; ++k) df[G.g(1, 1, k, nx + 1)] = T(0);
}

// MPPGRADFD2, fft2d_lib77.f:9231-9295 (potential df -> 2-component f)
template <class T>
void gradf(const T* df, T* f, const Grid& G) {
  int ny = G.ny, nx = G.nx;
  T dnx = T(6.28318530717959) / T(nx + nx);
  T dny = T(6.28318530717959) / T(ny + ny);
  for (int j = 1; j <= nx; ++j) {
    T dkx = dnx * T(j - 1);
    if (j - 1 > 0) {
      for (int k = 2; k <= ny; ++k) {
        T dky = dny * T(k - 1);
        f[G.g(2, 1, k, j)] = dkx * df[G.g(1, 1, k, j)];
        f[G.g(2, 2, k, j)] = dky * df[G.g(1, 1, k, j)];
      }
    }
    f[G.g(2, 1, 1, j)] = T(0);
    f[G.g(2, 2, 1, j)] = T(0);
    f[G.g(2, 1, ny + 1, j)] = T(0);
    f[G.g(2, 2, ny + 1, j)] = T(0);
  }
  for (int k = 2; k <= ny; ++k) {
    f[G.g(2, 1, k, 1)] = T(0);
    f[G.g(2, 2, k, 1)] = T(0);
  }
  for (int k = 1; k <= ny + 1; ++k) {
    f[G.g(2, 1, k, nx + 1)] = T(0);
    f[G.g(2, 2, k, nx + 1)] = T(0);
  }
}
#undef FRE
#undef FIM

// ------------------------------------------------------------- particles
struct Tiles {
  int nx, ny, mx1, myp1, mxyp1, nxv, nypmx;
  Tiles(const Grid& G) {
    nx = G.nx;
    ny = G.ny;
    mx1 = (nx - 1) / MX + 1;
    myp1 = (ny - 1) / MY + 1;
    mxyp1 = mx1 * myp1;
    nxv = G.nxv;
    nypmx = G.nypmx;
  }
};
#define PP(i, n, k) ppart[(size_t)((i)-1) + 8 * ((size_t)((n)-1) + (size_t)nppmx * (size_t)((k)-1))]

// PPGPPOST2L, part2d_lib77.f:194-309.  Tile accumulators are formed in
// parallel; the global flush runs in tile order so the oracle is
// deterministic for any thread count.
template <class T>
void ppgppost2l(const T* ppart, T* q, const int* kpic, int nppmx, const Grid& G) {
  Tiles tl(G);
  const int S = (MX + 1) * (MY + 1);
  std::vector<T> sqall((size_t)tl.mxyp1 * S);
  int noff = 0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int k = 1; k <= tl.mxyp1; ++k) {
    int noffp = (k - 1) / tl.mx1;
    int moffp = MY * noffp;
    noffp = MX * (k - tl.mx1 * noffp - 1);
    int nppp = kpic[k - 1];
    int mnoff = moffp + noff - 1;
    T* sq = &sqall[(size_t)(k - 1) * S];
#define SQ(i, j) sq[((i)-1) + (MX + 1) * ((j)-1)]
    for (int j = 0; j < S; ++j) sq[j] = T(0);
    for (int j = 1; j <= nppp; ++j) {
      T x = PP(1, j, k), y = PP(2, j, k), qm = PP(8, j, k);
      int nn = (int)x, mm = (int)y;
      T dxp = qm * (x - T(nn));
      T dyp = y - T(mm);
      nn = nn - noffp + 1;
      mm = mm - mnoff;
      T amx = qm - dxp;
      T amy = T(1.0) - dyp;
      x = SQ(nn, mm) + amx * amy;
      y = SQ(nn + 1, mm) + dxp * amy;
      SQ(nn, mm) = x;
      SQ(nn + 1, mm) = y;
      x = SQ(nn, mm + 1) + amx * dyp;
      y = SQ(nn + 1, mm + 1) + dxp * dyp;
      SQ(nn, mm + 1) = x;
      SQ(nn + 1, mm + 1) = y;
    }
  }
  for (int k = 1; k <= tl.mxyp1; ++k) {
    int noffp = (k - 1) / tl.mx1;
    int moffp = MY * noffp;
    noffp = MX * (k - tl.mx1 * noffp - 1);
    T* sq = &sqall[(size_t)(k - 1) * S];
    size_t nxv = tl.nxv;
#define Q(i, j) q[(size_t)((i)-1) + nxv * (size_t)((j)-1)]
    int nn = std::min(MX, tl.nxv - noffp);
    int mm = std::min(MY, tl.nypmx - moffp);
    for (int j = 2; j <= mm; ++j)
      for (int i = 2; i <= nn; ++i) Q(i + noffp, j + moffp) += SQ(i, j);
    mm = std::min(MY + 1, tl.nypmx - moffp);
    for (int i = 2; i <= nn; ++i) {
      Q(i + noffp, 1 + moffp) += SQ(i, 1);
      if (mm > MY) Q(i + noffp, mm + moffp) += SQ(i, mm);
    }
    nn = std::min(MX + 1, tl.nxv - noffp);
    for (int j = 1; j <= mm; ++j) {
      Q(1 + noffp, j + moffp) += SQ(1, j);
      if (nn > MX) Q(nn + noffp, j + moffp) += SQ(nn, j);
    }
#undef Q
#undef SQ
  }
}

// WPGPSIPOST2L_QP, part2d_lib77.f:2207-2284
template <class T>
void wpgpsipost2l_qp(T* ppart, const T* psi, const int* kpic, T qbm, int nppmx,
                     const Grid& G, T dex) {
  Tiles tl(G);
  T dx2 = dex * dex;
  int noff = 0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int k = 1; k <= tl.mxyp1; ++k) {
    int noffp = (k - 1) / tl.mx1;
    int moffp = MY * noffp;
    noffp = MX * (k - tl.mx1 * noffp - 1);
    int nppp = kpic[k - 1];
    int mnoff = moffp + noff - 1;
    T spsi[(MX + 1) * (MY + 1)];
#define SPSI(i, j) spsi[((i)-1) + (MX + 1) * ((j)-1)]
    int nn = std::min(MX, tl.nx - noffp) + 1;
    int mm = std::min(MY, tl.ny - moffp) + 1;
    for (int j = 1; j <= mm; ++j)
      for (int i = 1; i <= nn; ++i)
        SPSI(i, j) = psi[(size_t)(i + noffp - 1) + (size_t)tl.nxv * (size_t)(j + moffp - 1)];
    for (int j = 1; j <= nppp; ++j) {
      T x = PP(1, j, k), y = PP(2, j, k), vx = PP(3, j, k), vy = PP(4, j, k);
      nn = (int)x;
      mm = (int)y;
      T dxp = x - T(nn), dyp = y - T(mm);
      nn = nn - noffp + 1;
      mm = mm - mnoff;
      T amx = T(1.0) - dxp, amy = T(1.0) - dyp;
      T dx = amx * SPSI(nn, mm);
      dx = amy * (dxp * SPSI(nn + 1, mm) + dx);
      T acx = amx * SPSI(nn, mm + 1);
      dx = dx + dyp * (dxp * SPSI(nn + 1, mm + 1) + acx);
      dx = -dx * dx2 * qbm;
      PP(7, j, k) = T(1.0) + dx;
      PP(6, j, k) = dx + (dx2 * (vx * vx + vy * vy) - dx * dx - T(2.) * dx) /
                             (T(2.) * (T(1.) + dx)) + T(1.0);
    }
#undef SPSI
  }
}

// PPGRDCJPPOST2L_QP, part2d_lib77.f:311-768
template <class T>
void ppgrdcjppost2l_qp(T* ppart, const T* fxy, const T* bxy, const T* psit, T* cu,
                       T* dcu, T* amu, const int* kpic, T qbm, T dt, T ci, int nppmx,
                       const Grid& G, T dex) {
  Tiles tl(G);
  const int S = (MX + 1) * (MY + 1);
  std::vector<T> acc((size_t)tl.mxyp1 * S * 8);
  int noff = 0;
  T qtmh = T(0.5) * qbm * dt;
  T dti = T(1.0) / dt;
  T idex = T(1.0) / dex;
  (void)ci;
  const size_t nxv = tl.nxv;
#pragma omp parallel for schedule(dynamic, 4)
  for (int k = 1; k <= tl.mxyp1; ++k) {
    int noffp = (k - 1) / tl.mx1;
    int moffp = MY * noffp;
    noffp = MX * (k - tl.mx1 * noffp - 1);
    int nppp = kpic[k - 1];
    int mnoff = moffp + noff - 1;
    T sfxy[2 * S], sbxy[3 * S], spsit[S];
#define IJ(i, j) (((i)-1) + (MX + 1) * ((j)-1))
    int nn = std::min(MX, tl.nx - noffp) + 1;
    int mm = std::min(MY, tl.ny - moffp) + 1;
    for (int j = 1; j <= mm; ++j)
      for (int i = 1; i <= nn; ++i) {
        size_t gi = (size_t)(i + noffp - 1) + nxv * (size_t)(j + moffp - 1);
        sfxy[2 * IJ(i, j)] = fxy[2 * gi];
        sfxy[2 * IJ(i, j) + 1] = fxy[2 * gi + 1];
        sbxy[3 * IJ(i, j)] = bxy[3 * gi];
        sbxy[3 * IJ(i, j) + 1] = bxy[3 * gi + 1];
        sbxy[3 * IJ(i, j) + 2] = bxy[3 * gi + 2];
        spsit[IJ(i, j)] = psit[gi];
      }
    T* a = &acc[(size_t)(k - 1) * S * 8];
    // component order in a: scu(1..3) dcu(1..2) amu(1..3)
    for (int j = 0; j < S * 8; ++j) a[j] = T(0);
#define SCU(c, ij) a[(ij) * 8 + (c)-1]
#define SDCU(c, ij) a[(ij) * 8 + 3 + (c)-1]
#define SAMU(c, ij) a[(ij) * 8 + 5 + (c)-1]
    for (int j = 1; j <= nppp; ++j) {
      T x = PP(1, j, k), y = PP(2, j, k), p6 = PP(6, j, k), p7 = PP(7, j, k),
        qm = PP(8, j, k);
      nn = (int)x;
      mm = (int)y;
      T dxp = x - T(nn), dyp = y - T(mm);
      nn = nn - noffp + 1;
      mm = mm - mnoff;
      T amx = T(1.0) - dxp, amy = T(1.0) - dyp;
      T inv_part_7 = T(1.0) / p7;
      T qtmh1 = qtmh * inv_part_7;
      T qtmh2 = qtmh1 * p6;
      int i00 = IJ(nn, mm), i10 = IJ(nn + 1, mm), i01 = IJ(nn, mm + 1),
          i11 = IJ(nn + 1, mm + 1);
      // find electric field
      T dx = amx * sfxy[2 * i00];
      T dy = amx * sfxy[2 * i00 + 1];
      T dz = amx * spsit[i00];
      dx = amy * (dxp * sfxy[2 * i10] + dx);
      dy = amy * (dxp * sfxy[2 * i10 + 1] + dy);
      dz = amy * (dxp * spsit[i10] + dz);
      T acx = amx * sfxy[2 * i01];
      T acy = amx * sfxy[2 * i01 + 1];
      T acz = amx * spsit[i01];
      dx = dx + dyp * (dxp * sfxy[2 * i11] + acx);
      dy = dy + dyp * (dxp * sfxy[2 * i11 + 1] + acy);
      dz = dz + dyp * (dxp * spsit[i11] + acz);
      // find magnetic field
      T ox = amx * sbxy[3 * i00];
      T oy = amx * sbxy[3 * i00 + 1];
      T oz = amx * sbxy[3 * i00 + 2];
      ox = amy * (dxp * sbxy[3 * i10] + ox);
      oy = amy * (dxp * sbxy[3 * i10 + 1] + oy);
      oz = amy * (dxp * sbxy[3 * i10 + 2] + oz);
      acx = amx * sbxy[3 * i01];
      acy = amx * sbxy[3 * i01 + 1];
      acz = amx * sbxy[3 * i01 + 2];
      ox = ox + dyp * (dxp * sbxy[3 * i11] + acx);
      oy = oy + dyp * (dxp * sbxy[3 * i11 + 1] + acy);
      oz = oz + dyp * (dxp * sbxy[3 * i11 + 2] + acz);
      // calculate half impulse
      T ddx = T(-1.0) * qtmh2 * dx + qtmh * oy;
      T ddy = T(-1.0) * qtmh2 * dy - qtmh * ox;
      // half acceleration
      T vx = PP(3, j, k), vy = PP(4, j, k);
      acx = vx + ddx;
      acy = vy + ddy;
      T omzt = qtmh1 * oz;
      T omt = omzt * omzt;
      T anorm = T(2.0) / (T(1.0) + omt);
      T rot1 = T(0.5) * (T(1.0) - omt);
      T rot2 = omzt;
      T v1 = (rot1 * acx + rot2 * acy) * anorm + ddx;
      T v2 = (rot1 * acy - rot2 * acx) * anorm + ddy;
      T qm1 = qm * inv_part_7;
      amx = qm1 * amx;
      dxp = qm1 * dxp;
      ox = T(0.5) * (v1 + vx);
      oy = T(0.5) * (v2 + vy);
      oz = T(0.5) * (T(1.0) + dex * dex * (ox * ox + oy * oy)) * inv_part_7 - T(0.5) * p7;
      PP(6, j, k) = p7 + oz;
      oz = oz * idex;
      vx = (v1 - vx) * dti;
      vy = (v2 - vy) * dti;
      dz = qbm * (dz + (dx * ox + dy * oy) * dex * dex * inv_part_7);
      dx = amx * amy;
      dy = dxp * amy;
      v1 = ox * ox * inv_part_7;
      v2 = oy * oy * inv_part_7;
      T v3 = ox * oy * inv_part_7;
      vx = vx + ox * dz * inv_part_7;
      vy = vy + oy * dz * inv_part_7;
      auto dep = [&](int ij, T w) {
        SAMU(1, ij) = SAMU(1, ij) + v1 * w;
        SAMU(2, ij) = SAMU(2, ij) + v2 * w;
        SAMU(3, ij) = SAMU(3, ij) + v3 * w;
        SDCU(1, ij) = SDCU(1, ij) + vx * w;
        SDCU(2, ij) = SDCU(2, ij) + vy * w;
        SCU(1, ij) = SCU(1, ij) + ox * w;
        SCU(2, ij) = SCU(2, ij) + oy * w;
        SCU(3, ij) = SCU(3, ij) + oz * w;
      };
      dep(i00, dx);
      dx = amx * dyp;
      dep(i10, dy);
      dy = dxp * dyp;
      dep(i01, dx);
      dep(i11, dy);
    }
  }
  // flush in tile order: interior, then the edges the reference updates
  // with OMP ATOMIC (part2d_lib77.f:664-766)
  for (int k = 1; k <= tl.mxyp1; ++k) {
    int noffp = (k - 1) / tl.mx1;
    int moffp = MY * noffp;
    noffp = MX * (k - tl.mx1 * noffp - 1);
    T* a = &acc[(size_t)(k - 1) * S * 8];
    auto add = [&](int i, int j) {
      size_t gi = (size_t)(i + noffp - 1) + nxv * (size_t)(j + moffp - 1);
      int ij = IJ(i, j);
      amu[3 * gi] += SAMU(1, ij);
      amu[3 * gi + 1] += SAMU(2, ij);
      amu[3 * gi + 2] += SAMU(3, ij);
      dcu[2 * gi] += SDCU(1, ij);
      dcu[2 * gi + 1] += SDCU(2, ij);
      cu[3 * gi] += SCU(1, ij);
      cu[3 * gi + 1] += SCU(2, ij);
      cu[3 * gi + 2] += SCU(3, ij);
    };
    int nn = std::min(MX, tl.nxv - noffp);
    int mm = std::min(MY, tl.nypmx - moffp);
    for (int j = 2; j <= mm; ++j)
      for (int i = 2; i <= nn; ++i) add(i, j);
    mm = std::min(MY + 1, tl.nypmx - moffp);
    for (int i = 2; i <= nn; ++i) {
      add(i, 1);
      if (mm > MY) add(i, mm);
    }
    nn = std::min(MX + 1, tl.nxv - noffp);
    for (int j = 1; j <= mm; ++j) {
      add(1, j);
      if (nn > MX) add(nn, j);
    }
  }
#undef SCU
#undef SDCU
#undef SAMU
#undef IJ
}

// PPGRBPPUSHF23L_QP, part2d_lib77.f:1066-1408.  Returns irc (0, or the
// largest ihole count when ntmax overflowed).
template <class T>
int ppgrbppushf23l_qp(T* ppart, const T* fxy, const T* bxy, const T* psit, const int* kpic,
                      int* ncl, int* ihole, T qbm, T dt, T ci, int nppmx, int ntmax,
                      const Grid& G, T dex) {
  Tiles tl(G);
  const int S = (MX + 1) * (MY + 1);
  int noff = 0;
  int nyp = tl.ny;
  T idex = T(1.0) / dex;
  T qtmh = T(0.5) * qbm * dt;
  (void)ci;
  T anx = T(tl.nx), any = T(tl.ny);
  const size_t nxv = tl.nxv;
  int irc = 0;
#define IH(i, n, k) ihole[(size_t)((i)-1) + 2 * ((size_t)((n)-1) + (size_t)(ntmax + 1) * (size_t)((k)-1))]
#pragma omp parallel for schedule(dynamic, 4) reduction(max : irc)
  for (int k = 1; k <= tl.mxyp1; ++k) {
    int noffp = (k - 1) / tl.mx1;
    int moffp = MY * noffp;
    noffp = MX * (k - tl.mx1 * noffp - 1);
    int nppp = kpic[k - 1];
    int nn = std::min(MX, tl.nx - noffp);
    int mm = std::min(MY, nyp - moffp);
    T edgelx = T(noffp), edgerx = T(noffp + nn);
    T edgely = T(noff + moffp), edgery = T(noff + moffp + mm);
    int ih = 0, nh = 0;
    int mnoff = moffp + noff - 1;
    T sfxy[2 * S], sbxy[3 * S], spsit[S];
#define IJ(i, j) (((i)-1) + (MX + 1) * ((j)-1))
    for (int j = 1; j <= mm + 1; ++j)
      for (int i = 1; i <= nn + 1; ++i) {
        size_t gi = (size_t)(i + noffp - 1) + nxv * (size_t)(j + moffp - 1);
        sfxy[2 * IJ(i, j)] = fxy[2 * gi];
        sfxy[2 * IJ(i, j) + 1] = fxy[2 * gi + 1];
        sbxy[3 * IJ(i, j)] = bxy[3 * gi];
        sbxy[3 * IJ(i, j) + 1] = bxy[3 * gi + 1];
        sbxy[3 * IJ(i, j) + 2] = bxy[3 * gi + 2];
        spsit[IJ(i, j)] = psit[gi];
      }
    for (int j = 1; j <= 8; ++j) ncl[(j - 1) + 8 * (k - 1)] = 0;
    for (int j = 1; j <= nppp; ++j) {
      T x = PP(1, j, k), y = PP(2, j, k);
      nn = (int)x;
      mm = (int)y;
      T p6 = PP(6, j, k), p7 = PP(7, j, k);
      T qtmh1 = qtmh / p7;
      T qtmh2 = qtmh1 * p6;
      T dxp = x - T(nn), dyp = y - T(mm);
      nn = nn - noffp + 1;
      mm = mm - mnoff;
      T amx = T(1.0) - dxp, amy = T(1.0) - dyp;
      int i00 = IJ(nn, mm), i10 = IJ(nn + 1, mm), i01 = IJ(nn, mm + 1),
          i11 = IJ(nn + 1, mm + 1);
      T dx = amx * sfxy[2 * i00];
      T dy = amx * sfxy[2 * i00 + 1];
      T dz = amx * spsit[i00];
      dx = amy * (dxp * sfxy[2 * i10] + dx);
      dy = amy * (dxp * sfxy[2 * i10 + 1] + dy);
      dz = amy * (dxp * spsit[i10] + dz);
      T acx = amx * sfxy[2 * i01];
      T acy = amx * sfxy[2 * i01 + 1];
      T acz = amx * spsit[i01];
      dx = dx + dyp * (dxp * sfxy[2 * i11] + acx);
      dy = dy + dyp * (dxp * sfxy[2 * i11 + 1] + acy);
      dz = dz + dyp * (dxp * spsit[i11] + acz);
      dz = dz * idex;
      T ox = amx * sbxy[3 * i00];
      T oy = amx * sbxy[3 * i00 + 1];
      T oz = amx * sbxy[3 * i00 + 2];
      ox = amy * (dxp * sbxy[3 * i10] + ox);
      oy = amy * (dxp * sbxy[3 * i10 + 1] + oy);
      oz = amy * (dxp * sbxy[3 * i10 + 2] + oz);
      acx = amx * sbxy[3 * i01];
      acy = amx * sbxy[3 * i01 + 1];
      acz = amx * sbxy[3 * i01 + 2];
      ox = ox + dyp * (dxp * sbxy[3 * i11] + acx);
      oy = oy + dyp * (dxp * sbxy[3 * i11 + 1] + acy);
      oz = oz + dyp * (dxp * sbxy[3 * i11 + 2] + acz);
      ox = ox * dex;
      oy = oy * dex;
      dx = qtmh2 * dx;
      dy = qtmh2 * dy;
      dz = qtmh2 * dz;
      acx = PP(3, j, k) + dx;
      acy = PP(4, j, k) + dy;
      acz = PP(5, j, k) + dz;
      T omxt = qtmh1 * ox, omyt = qtmh1 * oy, omzt = qtmh1 * oz;
      T omt = omxt * omxt + omyt * omyt + omzt * omzt;
      T anorm = T(2.0) / (T(1.0) + omt);
      omt = T(0.5) * (T(1.0) - omt);
      T rot4 = omxt * omyt, rot7 = omxt * omzt, rot8 = omyt * omzt;
      T rot1 = omt + omxt * omxt, rot5 = omt + omyt * omyt, rot9 = omt + omzt * omzt;
      T rot2 = omzt + rot4;
      rot4 = -omzt + rot4;
      T rot3 = -omyt + rot7;
      rot7 = omyt + rot7;
      T rot6 = omxt + rot8;
      rot8 = -omxt + rot8;
      dx = (rot1 * acx + rot2 * acy + rot3 * acz) * anorm + dx;
      dy = (rot4 * acx + rot5 * acy + rot6 * acz) * anorm + dy;
      dz = (rot7 * acx + rot8 * acy + rot9 * acz) * anorm + dz;
      PP(3, j, k) = dx;
      PP(4, j, k) = dy;
      PP(5, j, k) = dz;
      T dtc1 = dt / (std::sqrt(T(1) + (dx * dx + dy * dy + dz * dz) * dex * dex) - dz * dex);
      dx = x + dx * dtc1;
      dy = y + dy * dtc1;
      PP(1, j, k) = dx;
      PP(2, j, k) = dy;
      mm = 0;
      if (dx >= edgerx) {
        mm = 2;
      } else if (dx < edgelx) {
        mm = 1;
        if (dx < T(0.0)) {
          dx = dx + anx;
          if (dx >= anx) {
            PP(1, j, k) = T(0.0);
            mm = 0;
          }
        }
      }
      if (dy >= edgery) {
        mm = mm + 6;
      } else if (dy < edgely) {
        mm = mm + 3;
        if (dy < T(0.0)) {
          dy = dy + any;
          if (dy >= any) {
            PP(2, j, k) = T(0.0);
            mm = mm - 3;
          }
        }
      }
      if (mm > 0) {
        ncl[(mm - 1) + 8 * (k - 1)] += 1;
        ih = ih + 1;
        if (ih <= ntmax) {
          IH(1, ih + 1, k) = j;
          IH(2, ih + 1, k) = mm;
        } else {
          nh = 1;
        }
      }
    }
    if (nh > 0) irc = std::max(irc, 1);
    IH(1, 1, k) = ih;
#undef IJ
  }
  if (irc > 0) {
    int ih = 0;
    for (int k = 1; k <= tl.mxyp1; ++k) ih = std::max(ih, IH(1, 1, k));
    irc = ih;
  }
  return irc;
}

// pmove for one rank (part2d_class.f03:360-594 with list = .true.):
// PPPORDERF2LA part2d_lib77.f:1659-1811, PPPMOVE2 nvp==1 part2d_lib.f03:291-313,
// PPPORDER2LB part2d_lib77.f:1813-2028.  Buffers are sized so that only the
// ppart overflow (irc2(1) = 4) can occur; then the required nppmx is returned
// and ppart, kpic are restored from a snapshot, which matches the reference's
// recovery (PPPRSTOR2L, copy out, grow, copy in, redo PPPORDER2LB).
template <class T>
int pmove(T* ppart, int* kpic, int* ncl, int* ihole, int nppmx, int ntmax, const Grid& G) {
  Tiles tl(G);
  const int idimp = 8, mx1 = tl.mx1, myp1 = tl.myp1, mxyp1 = tl.mxyp1;
  int npbmx = nppmx;
  int total = 0;
  for (int k = 0; k < mxyp1; ++k) total += kpic[k];
  int nbmax = std::max(1, total);
  std::vector<T> ppbuff((size_t)idimp * npbmx * mxyp1);
  std::vector<T> sbufl((size_t)idimp * nbmax), sbufr((size_t)idimp * nbmax);
  std::vector<T> rbufl((size_t)idimp * nbmax), rbufr((size_t)idimp * nbmax);
  std::vector<int> ncll(3 * mx1), nclr(3 * mx1), mcll(3 * mx1), mclr(3 * mx1);
  std::vector<T> save_pp(ppart, ppart + (size_t)idimp * nppmx * mxyp1);
  std::vector<int> save_kpic(kpic, kpic + mxyp1);
  std::vector<int> save_ncl(ncl, ncl + 8 * (size_t)mxyp1);
#define PB(i, n, k) ppbuff[(size_t)((i)-1) + idimp * ((size_t)((n)-1) + (size_t)npbmx * (size_t)((k)-1))]
#define NCL(i, k) ncl[((i)-1) + 8 * ((k)-1)]
#define NCLL(i, k) ncll[((i)-1) + 3 * ((k)-1)]
#define NCLR(i, k) nclr[((i)-1) + 3 * ((k)-1)]
#define MCLL(i, k) mcll[((i)-1) + 3 * ((k)-1)]
#define MCLR(i, k) mclr[((i)-1) + 3 * ((k)-1)]
#define SBL(i, n) sbufl[(size_t)((i)-1) + idimp * (size_t)((n)-1)]
#define SBR(i, n) sbufr[(size_t)((i)-1) + idimp * (size_t)((n)-1)]
#define RBL(i, n) rbufl[(size_t)((i)-1) + idimp * (size_t)((n)-1)]
#define RBR(i, n) rbufr[(size_t)((i)-1) + idimp * (size_t)((n)-1)]
  int irc2_1 = 0;
  // ---- PPPORDERF2LA
  for (int k = 1; k <= mxyp1; ++k) {
    int isum = 0;
    for (int j = 1; j <= 8; ++j) {
      int ist = NCL(j, k);
      NCL(j, k) = isum;
      isum += ist;
    }
    int nh = IH(1, 1, k);
    int ip = 0;
    for (int j = 1; j <= nh; ++j) {
      int j1 = IH(1, j + 1, k);
      int ist = IH(2, j + 1, k);
      int ii = NCL(ist, k) + 1;
      if (ii <= npbmx) {
        for (int i = 1; i <= idimp; ++i) PB(i, ii, k) = PP(i, j1, k);
      } else {
        ip = 1;
      }
      NCL(ist, k) = ii;
    }
    if (ip > 0) irc2_1 = 2;
  }
  if (irc2_1 > 0) return -2;  // cannot happen: npbmx = nppmx
  int kk = mx1 * (myp1 - 1);
  for (int k = 1; k <= mx1; ++k) {
    NCLL(1, k) = NCL(5, k) - NCL(2, k);
    NCLR(1, k) = NCL(8, k + kk) - NCL(5, k + kk);
  }
  kk = 1;
  while (kk < mx1) {
    for (int k = 1; k <= mx1; ++k) {
      int ii = (k - 1) / kk;
      int nn = kk * ii;
      int mm = 2 * nn + kk - 1;
      nn = nn + k + kk;
      if (nn <= mx1) {
        NCLL(1, nn) = NCLL(1, nn) + NCLL(1, mm + 1);
        NCLR(1, nn) = NCLR(1, nn) + NCLR(1, mm + 1);
      }
    }
    kk = kk + kk;
  }
  kk = mx1 * (myp1 - 1);
  for (int k = 1; k <= mx1; ++k) {
    int ii = NCL(5, k) - NCL(2, k);
    int nn = NCLL(1, k) - ii;
    for (int j = 1; j <= std::min(ii, nbmax - nn); ++j)
      for (int i = 1; i <= idimp; ++i) SBL(i, j + nn) = PB(i, j + NCL(2, k), k);
    for (int i = 1; i <= 3; ++i) NCLL(i, k) = NCL(i + 2, k) - NCL(2, k) + nn;
    ii = NCL(8, k + kk) - NCL(5, k + kk);
    int mm = NCLR(1, k) - ii;
    for (int j = 1; j <= std::min(ii, nbmax - mm); ++j)
      for (int i = 1; i <= idimp; ++i) SBR(i, j + mm) = PB(i, j + NCL(5, k + kk), k + kk);
    for (int i = 1; i <= 3; ++i) NCLR(i, k) = NCL(i + 5, k + kk) - NCL(5, k + kk) + mm;
  }
  // ---- PPPMOVE2, nvp == 1
  for (int j = 1; j <= mx1; ++j)
    for (int i = 1; i <= 3; ++i) MCLL(i, j) = NCLR(i, j);
  for (int j = 1; j <= mx1; ++j)
    for (int i = 1; i <= 3; ++i) MCLR(i, j) = NCLL(i, j);
  for (int j = 1; j <= NCLR(3, mx1); ++j)
    for (int i = 1; i <= idimp; ++i) RBL(i, j) = SBR(i, j);
  for (int j = 1; j <= NCLL(3, mx1); ++j)
    for (int i = 1; i <= idimp; ++i) RBR(i, j) = SBL(i, j);
  // ---- PPPORDER2LB
  T anx = T(tl.nx), any = T(tl.ny);
  int need = 0;
  for (int k = 1; k <= mxyp1; ++k) {
    int nppp = kpic[k - 1];
    int ky = (k - 1) / mx1 + 1;
    int kk2 = (ky - 1) * mx1;
    int kl = (ky - 2) * mx1;
    int kr = ky * mx1;
    int kx = k - (ky - 1) * mx1;
    int kxl = kx - 1;
    if (kxl < 1) kxl = kxl + mx1;
    int kxr = kx + 1;
    if (kxr > mx1) kxr = kxr - mx1;
    int ks[8] = {kxr + kk2, kxl + kk2, kx + kr, kxr + kr, kxl + kr, kx + kl, kxr + kl, kxl + kl};
    int nh = IH(1, 1, k);
    int noff = 0, moff = 0;
    if (ky == 1) {
      if (kx > 1) noff = MCLL(3, kx - 1);
    }
    if (ky == myp1) {
      if (kx > 1) moff = MCLR(3, kx - 1);
    }
    int ncoff = 0, ih = 0, ist = 0, j1 = 0;
    for (int ii = 1; ii <= 8; ++ii) {
      int ip;
      if (ks[ii - 1] <= 0) {
        if (ii > 6) noff = MCLL(ii - 6, ks[ii - 1] + mx1);
        ip = MCLL(ii - 5, ks[ii - 1] + mx1) - noff;
      } else if (ks[ii - 1] > mxyp1) {
        if (ii > 3) moff = MCLR(ii - 3, ks[ii - 1] - mxyp1);
        ip = MCLR(ii - 2, ks[ii - 1] - mxyp1) - moff;
      } else {
        if (ii > 1) ncoff = NCL(ii - 1, ks[ii - 1]);
        ip = NCL(ii, ks[ii - 1]) - ncoff;
      }
      for (int j = 1; j <= ip; ++j) {
        ih = ih + 1;
        if (ih <= nh) {
          j1 = IH(1, ih + 1, k);
        } else {
          j1 = nppp + 1;
          nppp = j1;
        }
        if (j1 <= nppmx) {
          const T* src;
          if (ks[ii - 1] <= 0)
            src = &RBL(1, j + noff);
          else if (ks[ii - 1] > mxyp1)
            src = &RBR(1, j + moff);
          else
            src = &PB(1, j + ncoff, ks[ii - 1]);
          T dx = src[0];
          if (dx < T(0.0)) dx = dx + anx;
          if (dx >= anx) dx = dx - anx;
          PP(1, j1, k) = dx;
          T dy = src[1];
          if (dy < T(0.0)) dy = dy + any;
          if (dy >= any) dy = dy - any;
          PP(2, j1, k) = dy;
          for (int i = 3; i <= idimp; ++i) PP(i, j1, k) = src[i - 1];
        } else {
          ist = 1;
        }
      }
    }
    if (ih < nh) {
      IH(2, 1, k) = -(ih + 1);
    } else {
      IH(2, 1, k) = nppp;
    }
    if (ist > 0) {
      irc2_1 = 4;
    }
    need = std::max(need, IH(2, 1, k));
  }
  if (irc2_1 == 4) {
    std::memcpy(ppart, save_pp.data(), save_pp.size() * sizeof(T));
    std::memcpy(kpic, save_kpic.data(), save_kpic.size() * sizeof(int));
    std::memcpy(ncl, save_ncl.data(), save_ncl.size() * sizeof(int));
    return std::max(need, 1);
  }
  for (int k = 1; k <= mxyp1; ++k) {
    int ih = IH(2, 1, k);
    if (ih < 0) {
      int nppp = kpic[k - 1];
      int nh = IH(1, 1, k);
      int ip = nh + ih + 1;
      for (int j = 1; j <= ip; ++j) {
        int j1 = nppp - j + 1;
        int j2 = IH(1, nh - j + 2, k);
        if (j1 > j2) {
          for (int i = 1; i <= idimp; ++i) PP(i, j2, k) = PP(i, j1, k);
        }
      }
      kpic[k - 1] = nppp - ip;
    } else {
      kpic[k - 1] = IH(2, 1, k);
    }
  }
#undef PB
#undef NCL
#undef NCLL
#undef NCLR
#undef MCLL
#undef MCLR
#undef SBL
#undef SBR
#undef RBL
#undef RBR
  return 0;
}
#undef IH

// PPDBLKP2L, part2d_lib77.f:15-77 (idimp = 8, noff = 0)
template <class T>
int ppdblkp2l(const T* part, int* kpic, int npp, int* nppmx, const Grid& G) {
  Tiles tl(G);
  int ierr = 0;
  for (int k = 0; k < tl.mxyp1; ++k) kpic[k] = 0;
  for (int j = 1; j <= npp; ++j) {
    int n = (int)part[8 * (size_t)(j - 1)];
    n = n / MX + 1;
    int m = (int)part[8 * (size_t)(j - 1) + 1];
    m = m / MY;
    m = n + tl.mx1 * m;
    if (m <= tl.mxyp1)
      kpic[m - 1] += 1;
    else
      ierr = std::max(ierr, m - tl.mxyp1);
  }
  int isum = 0, npx = 0;
  for (int k = 0; k < tl.mxyp1; ++k) {
    npx = std::max(npx, kpic[k]);
    isum += kpic[k];
  }
  *nppmx = npx;
  if (ierr > 0) return ierr;
  if (isum != npp) return -1;
  return 0;
}

// PPPMOVIN2L, part2d_lib77.f:79-131
template <class T>
int pppmovin2l(const T* part, T* ppart, int* kpic, int npp, int nppmx, const Grid& G) {
  Tiles tl(G);
  int ierr = 0;
  for (int k = 0; k < tl.mxyp1; ++k) kpic[k] = 0;
  for (int j = 1; j <= npp; ++j) {
    int n = (int)part[8 * (size_t)(j - 1)];
    n = n / MX + 1;
    int m = (int)part[8 * (size_t)(j - 1) + 1];
    m = m / MY;
    m = n + tl.mx1 * m;
    int ip = kpic[m - 1] + 1;
    if (ip <= nppmx) {
      for (int i = 1; i <= 8; ++i) PP(i, ip, m) = part[(size_t)(i - 1) + 8 * (size_t)(j - 1)];
    } else {
      ierr = std::max(ierr, ip - nppmx);
    }
    kpic[m - 1] = ip;
  }
  return ierr;
}

// PPPCHECK2L, part2d_lib77.f:133-192: returns 0 or the 1-based bad tile
template <class T>
int pppcheck2l(const T* ppart, const int* kpic, int nppmx, const Grid& G) {
  Tiles tl(G);
  int irc = 0;
  for (int k = 1; k <= tl.mxyp1; ++k) {
    int noffp = (k - 1) / tl.mx1;
    int moffp = MY * noffp;
    noffp = MX * (k - tl.mx1 * noffp - 1);
    int nn = std::min(MX, tl.nx - noffp);
    int mm = std::min(MY, tl.ny - moffp);
    T edgelx = T(noffp), edgerx = T(noffp + nn);
    T edgely = T(moffp), edgery = T(moffp + mm);
    for (int j = 1; j <= kpic[k - 1]; ++j) {
      T dx = PP(1, j, k), dy = PP(2, j, k);
      int ist = 0;
      if (dx < edgelx) ist = 1;
      if (dx >= edgerx) ist = 2;
      if (dy < edgely) ist += 3;
      if (dy >= edgery) ist += 6;
      if (ist > 0) irc = k;
    }
  }
  return irc;
}
#undef PP

// dist2d_000 single-rank branch, fdist2d_class.f03:212-316 (uniform profile,
// noff = 0 < ny so cells i = 2..nx-1, j = 2..ny)
template <class T>
int dist2d_000(T* part, int npmax, int* npp, int xppc, int yppc, T qsign_q, T den,
               const Grid& G) {
  T den_temp = T(1.0);
  T qm = den_temp * den * qsign_q / std::abs(qsign_q) / T(xppc) / T(yppc);
  int nps = 1;
  int noff = 0;
  for (int i = 2; i <= G.nx - 1; ++i)
    for (int j = 2; j <= G.ny; ++j)
      for (int ix = 0; ix <= xppc - 1; ++ix)
        for (int iy = 0; iy <= yppc - 1; ++iy) {
          if (nps > npmax) return -1;
          T* pt = &part[8 * (size_t)(nps - 1)];
          pt[0] = (T(ix) + T(0.5)) / T(xppc) + T(i) - T(1);
          pt[1] = (T(iy) + T(0.5)) / T(yppc) + T(j) - T(1) + T(noff);
          pt[2] = T(0.0);
          pt[3] = T(0.0);
          pt[4] = T(0.0);
          pt[5] = T(1.0);
          pt[6] = T(1.0);
          pt[7] = qm;
          nps = nps + 1;
        }
  *npp = nps - 1;
  return 0;
}

// The other plasma loaders of fdist2d_class.f03 for one rank (noff = 0 < ny):
// init_fdist2d_010/011/012 (318-387, 525-590, 713-776) convert the lengths to
// cells, dist2d_010 (389-523) keeps the particles on or between two ellipses,
// dist2d_011 (592-711) weights the charge by a Gaussian ring and dist2d_012
// (778-950) by a piecewise-linear f(r); all take the longitudinal factor
// den_temp (421-438) of a 'piecewise' profile.  pr = profile, xppc, yppc, q,
// den, box x min/max, box y min/max, indx, indy, center x/y, inner radius x/y,
// outer radius x/y, radius, width, s, nr, ns, then r(nr), fr(nr), s(ns), fs(ns).
template <class T>
int dist2d_prof(T* part, int npmax, int* npp, const T* pr) {
  const int npf = (int)pr[0], xppc = (int)pr[1], yppc = (int)pr[2];
  const T q = pr[3], den = pr[4];
  const int indx = (int)pr[9], indy = (int)pr[10];
  const Grid G(indx, indy);
  const T dx = (pr[6] - pr[5]) / T(1 << indx), dy = (pr[8] - pr[7]) / T(1 << indy);
  const T cx = (pr[11] - pr[5]) / dx, cy = (pr[12] - pr[7]) / dy;
  const T irx = pr[13] / dx, iry = pr[14] / dy, orx = pr[15] / dx, ory = pr[16] / dy;
  const T r0 = pr[17] / dx, sigr = pr[18] / dx;
  const T s = pr[19];
  const int nr = (int)pr[20], ns = (int)pr[21];
  std::vector<T> r(nr), fr(nr), ls(ns), lfs(ns);
  for (int k = 0; k < nr; ++k) {
    r[k] = pr[22 + k] / dx;
    fr[k] = pr[22 + nr + k];
  }
  for (int k = 0; k < ns; ++k) {
    ls[k] = pr[22 + 2 * nr + k];
    lfs[k] = pr[22 + 2 * nr + ns + k];
  }
  T den_temp = T(1.0);
  if (ns > 0) {
    if (s < ls[0] || s > ls[ns - 1]) return -2;
    for (int i = 2; i <= ns; ++i) {
      if (ls[i - 1] < ls[i - 2]) return -3;
      if (s <= ls[i - 1]) {
        den_temp = lfs[i - 2] + (lfs[i - 1] - lfs[i - 2]) / (ls[i - 1] - ls[i - 2]) *
                                    (s - ls[i - 2]);
        break;
      }
    }
  }
  const T qm = den_temp * den * q / std::abs(q) / T(xppc) / T(yppc);
  const T iirx2 = T(1.0) / (irx * irx), iiry2 = T(1.0) / (iry * iry);
  const T iorx2 = T(1.0) / (orx * orx), iory2 = T(1.0) / (ory * ory);
  const T isigr2 = T(0.5) / (sigr * sigr);
  int nps = 1;
  for (int i = 2; i <= G.nx - 1; ++i)
    for (int j = 2; j <= G.ny; ++j)
      for (int ix = 0; ix <= xppc - 1; ++ix)
        for (int iy = 0; iy <= yppc - 1; ++iy) {
          const T x = (T(ix) + T(0.5)) / T(xppc) + T(i) - T(1);
          const T y = (T(iy) + T(0.5)) / T(yppc) + T(j) - T(1) + T(0);
          T qp = qm;
          if (npf == 10) {
            if (((x - cx) * (x - cx) * iirx2 + (y - cy) * (y - cy) * iiry2 < T(1)) ||
                ((x - cx) * (x - cx) * iorx2 + (y - cy) * (y - cy) * iory2 > T(1)))
              continue;
          } else if (npf == 11) {
            const T rr = std::sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy));
            qp = qm * std::exp(-(rr - r0) * (rr - r0) * isigr2);
          } else if (npf == 12) {
            const T rr = std::sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy));
            if (rr < r[0] || rr > r[nr - 1]) continue;
            for (int ii = 2; ii <= nr; ++ii) {
              if (r[ii - 1] <= r[ii - 2]) return -4;
              if (rr <= r[ii - 1]) {
                den_temp = fr[ii - 2] + (fr[ii - 1] - fr[ii - 2]) / (r[ii - 1] - r[ii - 2]) *
                                            (rr - r[ii - 2]);
                break;
              }
            }
            qp = qm * den_temp;
          } else if (npf != 0) {
            return -5;
          }
          if (nps > npmax) return -1;
          T* pt = &part[8 * (size_t)(nps - 1)];
          pt[0] = x;
          pt[1] = y;
          pt[2] = T(0.0);
          pt[3] = T(0.0);
          pt[4] = T(0.0);
          pt[5] = T(1.0);
          pt[6] = T(1.0);
          pt[7] = qp;
          nps = nps + 1;
        }
  *npp = nps - 1;
  return 0;
}

}  // namespace

// ---------------------------------------------------------------- ranorm
// ranorm, part3d_lib77.f:1324-1383 (Box-Muller on two 48-bit LCGs with the
// fixed seeds of the DATA statement).  The state is global like the
// Fortran SAVE variables.
namespace {
struct RanormState {
  int r1 = 885098780, r2 = 1824280461, r4 = 1396483093, r5 = 55318673;
  int iflg = 0;
  double r0 = 0.0;
};
RanormState g_ran;
}  // namespace

extern "C" void oq_ranorm_reset(void) { g_ran = RanormState(); }

extern "C" double oq_ranorm(void) {
  RanormState& s = g_ran;
  const double h1l = 65531.0, h1u = 32767.0, h2l = 65525.0;
  if (s.iflg != 0) {
    double v = s.r0;
    s.r0 = 0.0;
    s.iflg = 0;
    return v;
  }
  int isc = 65536;
  double asc = (double)isc;
  double bsc = asc * asc;
  int i1 = s.r1 - (s.r1 / isc) * isc;
  double r3 = h1l * (double)s.r1 + asc * h1u * (double)i1;
  i1 = (int)(r3 / bsc);
  r3 = r3 - (double)i1 * bsc;
  bsc = 0.5 * bsc;
  i1 = s.r2 / isc;
  isc = s.r2 - i1 * isc;
  s.r0 = h1l * (double)s.r2 + asc * h1u * (double)isc;
  asc = 1.0 / bsc;
  isc = (int)(s.r0 * asc);
  s.r2 = (int)(s.r0 - (double)isc * bsc);
  r3 = r3 + ((double)isc + 2.0 * h1u * (double)i1);
  isc = (int)(r3 * asc);
  s.r1 = (int)(r3 - (double)isc * bsc);
  double temp = std::sqrt(-2.0 * std::log(((double)s.r1 + (double)s.r2 * asc) * asc));
  isc = 65536;
  asc = (double)isc;
  bsc = asc * asc;
  i1 = s.r4 - (s.r4 / isc) * isc;
  r3 = h2l * (double)s.r4 + asc * h1u * (double)i1;
  i1 = (int)(r3 / bsc);
  r3 = r3 - (double)i1 * bsc;
  bsc = 0.5 * bsc;
  i1 = s.r5 / isc;
  isc = s.r5 - i1 * isc;
  s.r0 = h2l * (double)s.r5 + asc * h1u * (double)isc;
  asc = 1.0 / bsc;
  isc = (int)(s.r0 * asc);
  s.r5 = (int)(s.r0 - (double)isc * bsc);
  r3 = r3 + ((double)isc + 2.0 * h1u * (double)i1);
  isc = (int)(r3 * asc);
  s.r4 = (int)(r3 - (double)isc * bsc);
  s.r0 = 6.28318530717959 * (((double)s.r4 + (double)s.r5 * asc) * asc);
  double v = temp * std::sin(s.r0);
  s.r0 = temp * std::cos(s.r0);
  s.iflg = 1;
  return v;
}

namespace {

// init_fdist3d_000 charge normalisation, fdist3d_class.f03:311-316
template <class T>
T beam_qm(T q, T np, const T* sig, const T* lo, const T* hi, int indx, int indy, int indz,
          int npx, int npy, int npz) {
  T dx = (hi[0] - lo[0]) / T(1 << indx);
  T dy = (hi[1] - lo[1]) / T(1 << indy);
  T dz = (hi[2] - lo[2]) / T(1 << indz);
  T qm = q / std::abs(q) * std::abs(np) * std::pow(T(2) * T(3.1415926535897932), T(1.5)) *
         sig[0] * sig[1] * sig[2];
  qm = qm / dx / dy / dz;
  qm = qm / T(npx);
  qm = qm / T(npy);
  qm = qm / T(npz);
  return qm;
}

// PRVDIST32_RANDOM, part3d_lib77.f:411-552 (one partition, edges = the box)
template <class T>
int prvdist32_random(T* part, int npmax, int* npp, T qm, T vtx, T vty, T vtz, T vdx, T vdy,
                     T vdz, int npx, int npy, int npz, int nx, int ny, int nz, T sigx,
                     T sigy, T sigz, T x0, T y0, T z0, const T* cx, const T* cy,
                     bool lquiet) {
  int ierr = 0;
  int npt = 1;
  T edges[4] = {T(0), T(ny), T(0), T(nz)};
  T x2 = T(2.0) * x0, y2 = T(2.0) * y0;
  T borderlx = std::max(x0 - T(5.0) * sigx, T(1.0));
  T borderly = std::max(y0 - T(5.0) * sigy, T(1.0));
  T borderlz = std::max(z0 - T(5.0) * sigz, T(1.0));
  T borderx = std::min(x0 + T(5.0) * sigx, T(nx - 1));
  T bordery = std::min(y0 + T(5.0) * sigy, T(ny - 1));
  T borderz = std::min(z0 + T(5.0) * sigz, T(nz - 1));
  int n = 0;
  auto put = [&](T px, T py, T pz, T vx, T vy, T vz) {
    if (npt < npmax) {
      npt = n + 1;
      T* p = &part[7 * (size_t)(npt - 1)];
      p[0] = px;
      p[1] = py;
      p[2] = pz;
      p[3] = vx;
      p[4] = vy;
      p[5] = vz;
      p[6] = qm;
      n = npt;
    } else {
      ierr += 1;
    }
  };
  int j = 0, l = npz;
  while (j < npx) {
    int k = 0;
    while (k < npy) {
      l = l - npz;
      while (l < npz) {
        T tempz, tempx, tempy;
        do {
          tempz = (T)((double)z0 + (double)sigz * oq_ranorm());
        } while (tempz >= borderz || tempz <= borderlz);
        do {
          tempx = (T)((double)x0 + (double)sigx * oq_ranorm());
        } while (tempx >= borderx || tempx <= borderlx);
        do {
          tempy = (T)((double)y0 + (double)sigy * oq_ranorm());
        } while (tempy >= bordery || tempy <= borderly);
        T tvtx = (T)((double)vtx * oq_ranorm() + (double)vdx);
        T tvty = (T)((double)vty * oq_ranorm() + (double)vdy);
        T tvtz = (T)((double)vtz * oq_ranorm() + (double)vdz);
        tvtz = std::sqrt(tvtz * tvtz - T(1) - tvtx * tvtx - tvty * tvty);
        if (tempy >= edges[0] && tempy < edges[1] && tempz >= edges[2] && tempz < edges[3]) {
          T dzz = tempz - z0;
          T tempxx = -(cx[0] * (dzz * dzz)) - cx[1] * dzz - cx[2];
          T tempyy = -(cy[0] * (dzz * dzz)) - cy[1] * dzz - cy[2];
          put(tempx + tempxx, tempy + tempyy, tempz, tvtx, tvty, tvtz);
          if (lquiet) put(x2 - tempx + tempxx, y2 - tempy + tempyy, tempz, -tvtx, -tvty, tvtz);
        }
        l = l + 1;
        if (lquiet) l = l + 1;
      }
      k = k + 1;
    }
    j = j + 1;
  }
  *npp = n;
  return ierr;
}

// Stand-in for the Fortran intrinsic RANDOM_NUMBER that PRVDIST32_RAN_PFL
// calls (a compiler runtime's generator, which the reference does not pin):
// SplitMix64 (Steele, Lea, Flood 2014) from a 64-bit seed, each number the
// top 24 bits of an output times 2^-24.  The engine's loader defines the same.
struct OUniform {
  uint64_t s;
  float next() {
    s += 0x9e3779b97f4a7c15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z = z ^ (z >> 31);
    return (float)(z >> 40) * (1.0f / 16777216.0f);
  }
};

// init_fdist3d_001 fdist3d_class.f03:508-518 (sumz, the trapezoid integral
// of fz over z, and the conversion z = (z - min) / dz) and the table of
// dist3d_001 600-611: zf(i), i = 1..nz, linear between the points.
template <class T>
int dist3d_001_zf(const T* z, const T* fz, int nzf, T zmin, T dz, int nz, T* zf, T* sumz) {
  T sum = T(0.0);
  for (int ii = 2; ii <= nzf; ++ii) {
    if (z[ii - 1] <= z[ii - 2]) return -1;  // "Piecewise_z is not monotonically increasing"
    sum = sum + (fz[ii - 1] + fz[ii - 2]) * (z[ii - 1] - z[ii - 2]) * T(0.5);
  }
  *sumz = sum;
  std::vector<T> zz(nzf);
  for (int ii = 1; ii <= nzf; ++ii) zz[ii - 1] = (z[ii - 1] - zmin) / dz;
  for (int i = 1; i <= nz; ++i) {
    zf[i - 1] = T(0.0);
    for (int j = 2; j <= nzf; ++j) {
      if (((T)i >= zz[j - 2]) && ((T)i < zz[j - 1])) {
        zf[i - 1] = fz[j - 1] + (fz[j - 2] - fz[j - 1]) / (zz[j - 2] - zz[j - 1]) * ((T)i - zz[j - 1]);
        break;
      }
    }
  }
  return 0;
}

// init_fdist3d_001 521-526 (e = 1, sz = sumz) and init_fdist3d_002 732-737
// (e = 1.5, sz = sigz): the charge of one macro-particle.
template <class T>
T beam_qm2(T qm, T np, T e, T sx, T sy, T sz, T dx, T dy, T dz, int npx, int npy, int npz) {
  const T twopi = T(2) * (T)3.1415926535897932f;
  qm = qm / std::abs(qm) * std::abs(np) * (e == T(1) ? twopi : (T)std::pow(twopi, e)) * sx * sy *
       sz;
  qm = qm / dx / dy / dz;
  qm = qm / (T)npx;
  qm = qm / (T)npy;
  qm = qm / (T)npz;
  return qm;
}

// PRVDIST32_RAN_PFL, part3d_lib77.f:193-410, one partition (edges 0, ny,
// 0, nz).  dp(nz) is the longitudinal profile and is rescaled in place as in
// the reference.  The reference stores while npt <= npmax, which lets npp
// reach npmax + 1, one past its array; here a particle is stored only while
// npp < npmax and each refused one counts in ierr.  An all-zero profile
// returns no particles (the reference would draw forever).
template <class T>
int prvdist32_ran_pfl(T* part, int npmax, int* npp, T qm, T x0, T y0, T z0, T sigx, T sigy,
                      T vtx, T vty, T vtz, T vdx, T vdy, T vdz, const T* cx, const T* cy, int npx,
                      int npy, int npz, int nx, int ny, int nz, T* dp, bool lquiet,
                      uint64_t seed) {
  int ierr = 0;
  (void)vdx;
  (void)vdy;
  const T edges[4] = {T(0), T(ny), T(0), T(nz)};
  int npt = 1;
  const T x2 = T(2.0) * x0, y2 = T(2.0) * y0;
  const T borderlx = std::max(x0 - T(5.0) * sigx, T(1.0));
  const T borderly = std::max(y0 - T(5.0) * sigy, T(1.0));
  const T borderx = std::min(x0 + T(5.0) * sigx, T(nx - 1));
  const T bordery = std::min(y0 + T(5.0) * sigy, T(ny - 1));
  const int nz1 = nz - 1;
  T amax = T(0);
  for (int i = 1; i <= nz; ++i) {
    dp[i - 1] = std::abs(dp[i - 1]);
    amax = std::max(amax, dp[i - 1]);
  }
  *npp = 0;
  if (!(amax > T(0)) || nz1 < 1) return 0;
  amax = amax * (T)1.2f;
  for (int i = 1; i <= nz; ++i) dp[i - 1] = dp[i - 1] / amax;
  OUniform uni{seed};
  T tmpu[1024], tmpz[1024];
  int cnt = 0;
  int j = 0, l = npz;
  while (j < npx) {
    int k = 0;
    while (k < npy) {
      l = l - npz;
      while (l < npz) {
        if (cnt <= 0) {  // call RANDOM_NUMBER(tmpu); call RANDOM_NUMBER(tmpz)
          for (int i = 0; i < 1024; ++i) tmpu[i] = (T)uni.next();
          for (int i = 0; i < 1024; ++i) tmpz[i] = (T)uni.next();
          cnt = 1024;
        }
        const T u = tmpu[cnt - 1];
        const T tempz = tmpz[cnt - 1] * (T)nz1;
        cnt = cnt - 1;
        int zi = (int)tempz;
        if (zi > nz1 - 1) zi = nz1 - 1;
        const T zf = tempz - (T)zi;
        const T zs = T(1.) - zf;
        zi = zi + 1;
        const T dpi = dp[zi - 1] * zs + dp[zi] * zf;
        if (u <= dpi) {
          T tempx, tempy;
          do {
            tempx = (T)((double)x0 + (double)sigx * oq_ranorm());
          } while (tempx >= borderx || tempx <= borderlx);
          do {
            tempy = (T)((double)y0 + (double)sigy * oq_ranorm());
          } while (tempy >= bordery || tempy <= borderly);
          if ((tempy < edges[1]) && (tempy > edges[0]) && (tempz < edges[3]) &&
              (tempz > edges[2])) {
            const T tvtx = (T)((double)vtx * oq_ranorm());
            const T tvty = (T)((double)vty * oq_ranorm());
            T tvtz = (T)((double)vtz * oq_ranorm() + (double)vdz);
            tvtz = std::sqrt(tvtz * tvtz - T(1) - tvtx * tvtx - tvty * tvty);
            T tempxx = T(0), tempyy = T(0);
            if (npt <= npmax && *npp < npmax) {
              npt = *npp + 1;
              T* p = &part[7 * (size_t)(npt - 1)];
              p[2] = tempz;
              const T d = p[2] - z0;
              tempxx = -(cx[0] * (d * d)) - cx[1] * d - cx[2];
              p[0] = tempx + tempxx;
              tempyy = -(cy[0] * (d * d)) - cy[1] * d - cy[2];
              p[1] = tempy + tempyy;
              p[3] = tvtx;
              p[4] = tvty;
              p[5] = tvtz;
              p[6] = qm;
              *npp = npt;
            } else {
              ierr = ierr + 1;
            }
            if (lquiet) {
              if (npt <= npmax && *npp < npmax) {
                npt = *npp + 1;
                T* p = &part[7 * (size_t)(npt - 1)];
                p[2] = tempz;
                p[0] = x2 - tempx + tempxx;
                p[1] = y2 - tempy + tempyy;
                p[3] = -tvtx;
                p[4] = -tvty;
                p[5] = tvtz;
                p[6] = qm;
                *npp = npt;
              } else {
                ierr = ierr + 1;
              }
            }
          }
          l = l + 1;
          if (lquiet) l = l + 1;
        }
      }
      k = k + 1;
    }
    j = j + 1;
  }
  return ierr;
}

// PRVDIST32_TWISS, part3d_lib77.f:1-191, one partition.  tempx, tempy, tempz
// and at1 are double precision in the reference, tx, ty and the velocities
// real; the drift sums at its end are computed but never applied, and are
// left out.  Storage as in prvdist32_ran_pfl (npt <= npmax, at most npmax).
template <class T>
int prvdist32_twiss(T* part, int npmax, int* npp, T qm, T alpha_x, T alpha_y, T beta_x,
                    T beta_y, T emt_x, T emt_y, T sigz, T vdz, T vtz, int npx, int npy, int npz,
                    int nx, int ny, int nz, T x0, T y0, T z0, T gamma, bool lquiet) {
  int ierr = 0;
  int npt = 1;
  *npp = 0;
  const T edges[4] = {T(0), T(ny), T(0), T(nz)};
  const T x2 = T(2.0) * x0, y2 = T(2.0) * y0;
  const T sigx = std::sqrt(beta_x * emt_x / gamma);
  const T sigy = std::sqrt(beta_y * emt_y / gamma);
  const T vtx = emt_x / sigx, vty = emt_y / sigy;
  const T borderlx = std::max(x0 - T(3.0) * sigx, T(1.0));
  const T borderly = std::max(y0 - T(3.0) * sigy, T(1.0));
  const T borderlz = std::max(z0 - T(3.0) * sigz, T(1.0));
  const T borderx = std::min(x0 + T(3.0) * sigx, T(nx - 1));
  const T bordery = std::min(y0 + T(3.0) * sigy, T(ny - 1));
  const T borderz = std::min(z0 + T(3.0) * sigz, T(nz - 1));
  int j = 0, l = npz;
  while (j < npx) {
    int k = 0;
    while (k < npy) {
      l = l - npz;
      while (l < npz) {
        double tempz, tempx, tempy;
        T tx, ty;
      L10:
        tempz = (double)z0 + (double)sigz * oq_ranorm();
        if (tempz >= (double)borderz || tempz <= (double)borderlz) goto L10;
      L20:
        tx = (T)oq_ranorm();
        tempx = (double)(x0 + sigx * tx);
        if (tempx >= (double)borderx || tempx <= (double)borderlx) goto L20;
      L30:
        ty = (T)oq_ranorm();
        tempy = (double)(y0 + sigy * ty);
        if (tempy >= (double)bordery || tempy <= (double)borderly) goto L30;
        if ((tx * tx + ty * ty) > T(9.0)) goto L20;
        T tvtx = (T)((double)vtx * oq_ranorm());
        T tvty = (T)((double)vty * oq_ranorm());
        const T tvtz = (T)((double)vtz * oq_ranorm() + (double)vdz);
        tvtx = (T)((double)tvtx - (double)(gamma * alpha_x / beta_x) * (tempx - (double)x0));
        tvty = (T)((double)tvty - (double)(gamma * alpha_y / beta_y) * (tempy - (double)y0));
        if ((tempy >= (double)edges[0]) && (tempy < (double)edges[1]) &&
            (tempz >= (double)edges[2]) && (tempz < (double)edges[3])) {
          if (npt <= npmax && *npp < npmax) {
            npt = *npp + 1;
            T* p = &part[7 * (size_t)(npt - 1)];
            p[2] = (T)tempz;
            p[0] = (T)tempx;
            p[1] = (T)tempy;
            p[3] = tvtx;
            p[4] = tvty;
            p[5] = tvtz;
            p[6] = qm;
            *npp = npt;
          } else {
            ierr = ierr + 1;
          }
          if (lquiet) {
            if (npt <= npmax && *npp < npmax) {
              npt = *npp + 1;
              T* p = &part[7 * (size_t)(npt - 1)];
              p[2] = (T)tempz;
              p[0] = (T)((double)x2 - tempx);
              p[1] = (T)((double)y2 - tempy);
              p[3] = -tvtx;
              p[4] = -tvty;
              p[5] = tvtz;
              p[6] = qm;
              *npp = npt;
            } else {
              ierr = ierr + 1;
            }
          }
        }
        l = l + 1;
        if (lquiet) l = l + 1;
      }
      k = k + 1;
    }
    j = j + 1;
  }
  return ierr;
}

// dist3d_003, fdist3d_class.f03:899-974: npt lines "z x y vz vx vy q" read
// from a text file (blank-separated numbers), converted to cells and kept
// when inside the box.  Returns -1 on a failed read, -2 past npmax.
template <class T>
int dist3d_003(const char* file, int npt, T* part, int npmax, int* npp, T x0, T y0, T dx, T dy,
               T dz, T cwp, int nx, int ny, int nz) {
  std::FILE* f = std::fopen(file, "r");
  if (!f) return -1;
  int nps = 1;
  for (int i = 1; i <= npt; ++i) {
    // a REAL read: each decimal rounded once to T
    T v[7];
    const char* fmt = sizeof(T) == sizeof(float) ? "%f %f %f %f %f %f %f"
                                                 : "%lf %lf %lf %lf %lf %lf %lf";
    if (std::fscanf(f, fmt, &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6]) != 7) {
      std::fclose(f);
      return -1;
    }
    T tempz = v[0], tempx = v[1], tempy = v[2];
    const T tempvz = v[3], tempvx = v[4], tempvy = v[5], tempq = v[6];
    tempx = tempx / cwp / dx + x0;
    tempy = tempy / cwp / dy + y0;
    tempz = -(tempz / cwp / dz);
    if ((tempx >= T(1)) && tempx <= T(nx - 1) && (tempy >= T(0)) && (tempy < T(ny)) &&
        (tempz >= T(0)) && (tempz < T(nz))) {
      if (nps > npmax) {
        std::fclose(f);
        return -2;
      }
      T* p = &part[7 * (size_t)(nps - 1)];
      p[0] = tempx;
      p[3] = tempvx;
      p[1] = tempy;
      p[4] = tempvy;
      p[2] = tempz;
      p[5] = tempvz;
      p[6] = tempq;
      nps = nps + 1;
    }
  }
  *npp = nps - 1;
  std::fclose(f);
  return 0;
}

// dist3d_100, fdist3d_class.f03:1081-1166, one partition (noff = 0, nd2p =
// ny, nd3p = nz).  Returns -2 past npmax.
template <class T>
int dist3d_100(T* part, int npmax, int* npp, const int* ppc, T qm, T np, T gamma, const T* bc,
               const T* lb_in, const T* ub_in, T r1, T r2, int nx, int ny, int nz) {
  T lb[3], ub[3];
  *npp = 0;
  lb[0] = std::max(lb_in[0], T(0.0));
  ub[0] = std::min(ub_in[0], (T)nx);
  if (lb_in[1] > (T)ny || ub_in[1] < T(0)) return 0;
  lb[1] = std::max(lb_in[1], T(0));
  ub[1] = std::min(ub_in[1], (T)ny);
  if (lb_in[2] > (T)nz || ub_in[2] < T(0)) return 0;
  lb[2] = std::max(lb_in[2], T(0));
  ub[2] = std::min(ub_in[2], (T)nz);
  int nps = 1;
  for (int i = (int)lb[0]; i <= (int)ub[0] - 1; ++i)
    for (int j = (int)lb[1]; j <= (int)ub[1] - 1; ++j)
      for (int k = (int)lb[2]; k <= (int)ub[2] - 1; ++k)
        for (int ix = 0; ix <= ppc[0] - 1; ++ix)
          for (int iy = 0; iy <= ppc[1] - 1; ++iy)
            for (int iz = 0; iz <= ppc[2] - 1; ++iz) {
              if (nps > npmax) return -2;
              const T tx = ((T)ix + T(0.5)) / (T)ppc[0] + (T)i - T(1);
              const T ty = ((T)iy + T(0.5)) / (T)ppc[1] + (T)j - T(1);
              const T tz = ((T)iz + T(0.5)) / (T)ppc[2] + (T)k - T(1);
              T* p = &part[7 * (size_t)(nps - 1)];
              p[0] = tx;
              p[1] = ty;
              p[2] = tz;
              p[3] = T(0.0);
              p[4] = T(0.0);
              p[5] = gamma;
              const T a1 = std::abs(tz - bc[2]);
              const T a2 = std::sqrt((tx - bc[0]) * (tx - bc[0]) + (ty - bc[1]) * (ty - bc[1]));
              const T a3 = std::abs(a2 - r1);
              const T a4 = a1 * a1 + a3 * a3;
              p[6] = qm * np * std::exp(-(a4 / (r2 * r2) * T(0.5)));
              nps = nps + 1;
            }
  *npp = nps - 1;
  return 0;
}

// The static branch of dist3d_000 (fdist3d_class.f03:392-408) and dist3d_001
// (613-630), one partition: q3(i, j, k) for i = 1..nx, j = 1..ny, k = 1..nz
// of a (nx+2, ny+1, nz+1) array; zf = null takes the Gaussian in z of 000.
template <class T>
void beam_static(T np, T x0, T y0, T z0, T sigx, T sigy, T sigz, const T* cx, const T* cy,
                 const T* zf, int nx, int ny, int nz, T* q3) {
  const size_t nxv = (size_t)nx + 2, nyv = (size_t)ny + 1;
  for (int k = 1; k <= nz; ++k) {
    const T zval = (T)(k - 1) - z0;
    const T cx0 = -(cx[0] * (zval * zval)) - cx[1] * zval - cx[2];
    const T cy0 = -(cy[0] * (zval * zval)) - cy[1] * zval - cy[2];
    const T t1 = zf ? np * zf[k - 1] : np * std::exp(-(zval * zval / T(2.0) / (sigz * sigz)));
    for (int i = 1; i <= nx; ++i) {
      const T xval = (T)(i - 1);
      const T dx = xval - x0 + cx0;
      const T t2 = t1 * std::exp(-(dx * dx / T(2.0) / (sigx * sigx)));
      for (int j = 1; j <= ny; ++j) {
        const T yval = (T)(j - 1);
        const T dy = yval - y0 + cy0;
        q3[(size_t)(i - 1) + nxv * ((size_t)(j - 1) + nyv * (size_t)(k - 1))] =
            t2 * std::exp(-(dy * dy / T(2.0) / (sigy * sigy)));
      }
    }
  }
}

// PGBPUSH32L_QP, part3d_lib77.f:630-786 (one partition, noff = 0): the
// quasi-static beam push with the 3D fields of the step.  fxyz and bxyz are
// (3, nxv, nypmx, nzpmx); only the first two components of bxyz are used.
// With ipbc = 1 (conducting, the only solver, spect2d_class.f03:19) a particle
// that leaves [1, n-1) in x, y or z is dropped: the last particle takes its
// slot and is pushed in its place, as the reference does.  Returns the new
// particle count.
template <class T>
int pgbpush32l_qp(T* part, int npp, const T* fxyz, const T* bxyz, T qbm, T dt, T dtc, int nx,
                  int ny, int nz, int nxv, int nypmx, int ipbc, T deltax, T deltaz, T cofd) {
  const T qtmh = qbm * dt;
  const T dtcx = dtc / deltax;
  const T dtcz = dtc / deltaz;
  const T cofd1 = cofd / dt;
  T edgelx = T(0), edgely = T(0), edgelz = T(0), edgerx = T(0), edgery = T(0), edgerz = T(0);
  if (ipbc == 1) {
    edgelx = edgely = edgelz = T(1.);
    edgerx = T(nx - 1);
    edgery = T(ny - 1);
    edgerz = T(nz - 1);
  }
  const int mnoff = -1, lnoff = -1;
#define F3(a, c, b, l)                                                                   \
  a[(size_t)((c)-1) +                                                                  \
    3 * ((size_t)((b)-1) + (size_t)nxv * ((size_t)((l)-1) + (size_t)nypmx * (size_t)(lz - 1)))]
  int inpp = npp;
  int j = 1;
  while (j <= inpp) {
    T* p = &part[7 * (size_t)(j - 1)];
    int nn = (int)p[0], mm = (int)p[1], lz = (int)p[2];
    T dxp = p[0] - T(nn);
    T dyp = p[1] - T(mm);
    T dzp = p[2] - T(lz);
    nn = nn + 1;
    T amx = T(1.) - dxp;
    T amy = T(1.) - dyp;
    const int np = nn + 1;
    mm = mm - mnoff;
    T dx1 = dxp * dyp;
    dyp = amx * dyp;
    const int mp = mm + 1;
    amx = amx * amy;
    T amz = T(1.) - dzp;
    lz = lz - lnoff;
    amy = dxp * amy;
    // trilinear gather of component c of field a at (nn..np, mm..mp, lz..lz+1)
    auto tri = [&](const T* a, int c) {
      T lo = amx * F3(a, c, nn, mm) + amy * F3(a, c, np, mm) + dyp * F3(a, c, nn, mp) +
             dx1 * F3(a, c, np, mp);
      ++lz;
      T hi = amx * F3(a, c, nn, mm) + amy * F3(a, c, np, mm) + dyp * F3(a, c, nn, mp) +
             dx1 * F3(a, c, np, mp);
      --lz;
      return amz * lo + dzp * hi;
    };
    T dx = tri(fxyz, 1), dy = tri(fxyz, 2), dz = tri(fxyz, 3);
    const T ox = tri(bxyz, 1), oy = tri(bxyz, 2);
    dx = dx - oy;
    dy = dy + ox;
    const T delx = qtmh * dx, dely = qtmh * dy, delz = qtmh * dz;
    dx = p[3] + delx;
    dy = p[4] + dely;
    dz = p[5] + delz;
    p[3] = dx;
    p[4] = dy;
    const T p2t = dx * dx + dy * dy;
    const T p2l = dz * dz;
    const T p2 = p2t + p2l;
    const T ngamma = std::sqrt(T(1.) + p2);
    const T dtgx = dtcx / ngamma;
    const T dtgy = dtcx / ngamma;
    const T one_minus_vz = (T(1.) + p2t) / (dz * (dz + ngamma));
    dz = dz - cofd1 * ngamma * ((delx * delx + dely * dely) * dz - delz * (delx * dx + dely * dy));
    p[5] = dz;
    dx = p[0] + dx * dtgx;
    dy = p[1] + dy * dtgy;
    dz = p[2] + one_minus_vz * dtcz;
    if (ipbc == 1 && (dx < edgelx || dx >= edgerx || dy < edgely || dy >= edgery ||
                      dz < edgelz || dz >= edgerz)) {
      if (j == inpp) {
        --inpp;
        break;
      }
      std::copy(&part[7 * (size_t)(inpp - 1)], &part[7 * (size_t)inpp], p);
      --inpp;
      continue;  // push the particle moved into slot j
    }
    p[0] = dx;
    p[1] = dy;
    p[2] = dz;
    ++j;
  }
#undef F3
  return inpp;
}

// PGPOST32L, part3d_lib77.f:554-628 (one partition, noff = 0)
template <class T>
void pgpost32l(const T* part, int npp, T* q, int nxv, int nypmx) {
  int mnoff = -1, lnoff = -1;
  for (int j = 1; j <= npp; ++j) {
    const T* p = &part[7 * (size_t)(j - 1)];
    int nn = (int)p[0], mm = (int)p[1], ll = (int)p[2];
    T qm = p[6];
    T dxp = qm * (p[0] - T(nn));
    T dyp = p[1] - T(mm);
    T dzp = p[2] - T(ll);
    nn = nn + 1;
    T amx = qm - dxp;
    T amy = T(1.) - dyp;
    int np = nn + 1;
    mm = mm - mnoff;
    T dx1 = dxp * dyp;
    dyp = amx * dyp;
    int mp = mm + 1;
    amx = amx * amy;
    T amz = T(1.) - dzp;
    ll = ll - lnoff;
    amy = dxp * amy;
    int lp = ll + 1;
#define Q3(a, b, c) q[(size_t)((a)-1) + (size_t)nxv * ((size_t)((b)-1) + (size_t)nypmx * (size_t)((c)-1))]
    Q3(nn, mm, ll) += amx * amz;
    Q3(np, mm, ll) += amy * amz;
    Q3(nn, mp, ll) += dyp * amz;
    Q3(np, mp, ll) += dx1 * amz;
    Q3(nn, mm, lp) += amx * dzp;
    Q3(np, mm, lp) += amy * dzp;
    Q3(nn, mp, lp) += dyp * dzp;
    Q3(np, mp, lp) += dx1 * dzp;
#undef Q3
  }
}

}  // namespace

#include "qp_oracle_sim.inc"

// ------------------------------------------------------------ C exports
#define OQ_DEF(T, S)                                                                      \
  extern "C" int oq_fftrk_##S(T* rs, T* ks, int dim, int kind, int indx, int indy) {    \
    return fftrk<T>(rs, ks, dim, kind, Grid(indx, indy));                               \
  }                                                                                     \
  extern "C" int oq_fftkr_##S(T* rs, T* ks, int dim, int kind, int indx, int indy) {    \
    return fftkr<T>(rs, ks, dim, kind, Grid(indx, indy));                               \
  }                                                                                     \
  extern "C" int oq_line_##S(T* line, int stride, int parity, int xpass, int isign,     \
                             int indx, int indy) {                                      \
    Tables<T> tb(indx, indy);                                                           \
    nr_line<T>(line, stride, parity, xpass, isign, tb);                                 \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_ffc_##S(T* ffc, int indx, int indy, T ax, T ay, T affp) {           \
    ffc_init<T>(ffc, Grid(indx, indy), ax, ay, affp);                                   \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_pot_##S(const T* q, T* p, const T* ffc, int indx, int indy) {       \
    pot<T>(q, p, ffc, Grid(indx, indy));                                                \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_smooth_##S(const T* q, T* qs, const T* ffc, int indx, int indy) {   \
    smooth<T>(q, qs, ffc, Grid(indx, indy));                                            \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_elf_##S(const T* q, T* fxy, const T* ffc, int indx, int indy) {     \
    elf<T>(q, fxy, ffc, Grid(indx, indy));                                              \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_bf_##S(const T* cu, T* bxy, const T* ffc, int indx, int indy) {     \
    bf<T>(cu, bxy, ffc, Grid(indx, indy));                                              \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_vpot_##S(const T* cu, T* a, const T* ffc, int indx, int indy) {    \
    vpot<T>(cu, a, ffc, Grid(indx, indy));                                              \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_bfqp_##S(const T* cu, T* dcu, const T* amu, T* bxy, const T* ffc,   \
                             T aa, T dex, int indx, int indy) {                         \
    bfqp<T>(cu, dcu, amu, bxy, ffc, aa, dex, Grid(indx, indy));                         \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_div_##S(const T* f, T* df, int ndim, int indx, int indy) {          \
    divf<T>(f, df, ndim, Grid(indx, indy));                                             \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_grad_##S(const T* df, T* f, int indx, int indy) {                   \
    gradf<T>(df, f, Grid(indx, indy));                                                  \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_cguard_##S(T* rs, int dim, int indx, int indy) {                    \
    cguard<T>(rs, dim, Grid(indx, indy));                                               \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_acguard_##S(T* rs, int dim, int indx, int indy) {                   \
    acguard<T>(rs, dim, Grid(indx, indy));                                              \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_ppgppost2l_##S(const T* ppart, T* q, const int* kpic, int nppmx,    \
                                   int indx, int indy) {                                \
    ppgppost2l<T>(ppart, q, kpic, nppmx, Grid(indx, indy));                             \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_wpgpsipost2l_qp_##S(T* ppart, const T* psi, const int* kpic, T qbm, \
                                        int nppmx, int indx, int indy, T dex) {         \
    wpgpsipost2l_qp<T>(ppart, psi, kpic, qbm, nppmx, Grid(indx, indy), dex);            \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_ppgrdcjppost2l_qp_##S(T* ppart, const T* fxy, const T* bxy,         \
                                          const T* psit, T* cu, T* dcu, T* amu,         \
                                          const int* kpic, T qbm, T dt, T ci,           \
                                          int nppmx, int indx, int indy, T dex) {       \
    ppgrdcjppost2l_qp<T>(ppart, fxy, bxy, psit, cu, dcu, amu, kpic, qbm, dt, ci, nppmx, \
                         Grid(indx, indy), dex);                                        \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_ppgrbppushf23l_qp_##S(T* ppart, const T* fxy, const T* bxy,         \
                                          const T* psit, const int* kpic, int* ncl,     \
                                          int* ihole, T qbm, T dt, T ci, int nppmx,     \
                                          int ntmax, int indx, int indy, T dex) {       \
    return ppgrbppushf23l_qp<T>(ppart, fxy, bxy, psit, kpic, ncl, ihole, qbm, dt, ci,   \
                                nppmx, ntmax, Grid(indx, indy), dex);                   \
  }                                                                                     \
  extern "C" int oq_pmove_##S(T* ppart, int* kpic, int* ncl, int* ihole, int nppmx,     \
                              int ntmax, int indx, int indy) {                          \
    return pmove<T>(ppart, kpic, ncl, ihole, nppmx, ntmax, Grid(indx, indy));           \
  }                                                                                     \
  extern "C" int oq_ppdblkp2l_##S(const T* part, int* kpic, int npp, int* nppmx_out,    \
                                  int indx, int indy) {                                 \
    return ppdblkp2l<T>(part, kpic, npp, nppmx_out, Grid(indx, indy));                  \
  }                                                                                     \
  extern "C" int oq_pppmovin2l_##S(const T* part, T* ppart, int* kpic, int npp,         \
                                   int nppmx, int indx, int indy) {                     \
    return pppmovin2l<T>(part, ppart, kpic, npp, nppmx, Grid(indx, indy));              \
  }                                                                                     \
  extern "C" int oq_pppcheck2l_##S(const T* ppart, const int* kpic, int nppmx,          \
                                   int indx, int indy) {                                \
    return pppcheck2l<T>(ppart, kpic, nppmx, Grid(indx, indy));                         \
  }                                                                                     \
  extern "C" int oq_dist2d_000_##S(T* part, int npmax, int* npp, int xppc, int yppc,    \
                                   T qm, T den, int indx, int indy) {                   \
    return dist2d_000<T>(part, npmax, npp, xppc, yppc, qm, den, Grid(indx, indy));      \
  }                                                                                     \
  extern "C" int oq_dist2d_prof_##S(T* part, int npmax, int* npp, const T* pr) {       \
    return dist2d_prof<T>(part, npmax, npp, pr);                                        \
  }                                                                                     \
  extern "C" int oq_beam_qm_##S(T q, T np, const T* sig, const T* lo, const T* hi,      \
                                int indx, int indy, int indz, int npx, int npy,         \
                                int npz, T* qm_out) {                                   \
    *qm_out = beam_qm<T>(q, np, sig, lo, hi, indx, indy, indz, npx, npy, npz);          \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_prvdist32_random_##S(                                               \
      T* part, int npmax, int* npp, T qm, T vtx, T vty, T vtz, T vdz, int npx, int npy, \
      int npz, int indx, int indy, int indz, T sigx, T sigy, T sigz, T x0, T y0, T z0,  \
      const T* cx, const T* cy, int quiet) {                                            \
    return prvdist32_random<T>(part, npmax, npp, qm, vtx, vty, vtz, T(0), T(0), vdz,    \
                               npx, npy, npz, 1 << indx, 1 << indy, 1 << indz, sigx,    \
                               sigy, sigz, x0, y0, z0, cx, cy, quiet != 0);             \
  }                                                                                     \
  extern "C" int oq_dist3d_001_zf_##S(const T* z, const T* fz, int nzf, T zmin, T dz,   \
                                     int nz, T* zf, T* sumz) {                          \
    return dist3d_001_zf<T>(z, fz, nzf, zmin, dz, nz, zf, sumz);                        \
  }                                                                                     \
  extern "C" int oq_beam_qm2_##S(T q, T np, T e, T sx, T sy, T sz, T dx, T dy, T dz,    \
                                 int npx, int npy, int npz, T* qm_out) {                \
    *qm_out = beam_qm2<T>(q, np, e, sx, sy, sz, dx, dy, dz, npx, npy, npz);             \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_prvdist32_ran_pfl_##S(                                              \
      T* part, int npmax, int* npp, T qm, T x0, T y0, T z0, T sigx, T sigy, T vtx, T vty, \
      T vtz, T vdz, const T* cx, const T* cy, int npx, int npy, int npz, int nx, int ny, \
      int nz, T* dp, int quiet, unsigned long long seed) {                              \
    return prvdist32_ran_pfl<T>(part, npmax, npp, qm, x0, y0, z0, sigx, sigy, vtx, vty, \
                                vtz, T(0), T(0), vdz, cx, cy, npx, npy, npz, nx, ny, nz, \
                                dp, quiet != 0, seed);                                  \
  }                                                                                     \
  extern "C" int oq_prvdist32_twiss_##S(                                                \
      T* part, int npmax, int* npp, T qm, const T* alpha, const T* beta, const T* emt,  \
      T sigz, T vdz, T vtz, int npx, int npy, int npz, int nx, int ny, int nz, T x0,    \
      T y0, T z0, int quiet) {                                                          \
    return prvdist32_twiss<T>(part, npmax, npp, qm, alpha[0], alpha[1], beta[0],        \
                              beta[1], emt[0], emt[1], sigz, vdz, vtz, npx, npy, npz,   \
                              nx, ny, nz, x0, y0, z0, vdz, quiet != 0);                 \
  }                                                                                     \
  extern "C" int oq_dist3d_003_##S(const char* file, int npt, T* part, int npmax,       \
                                   int* npp, T x0, T y0, T dx, T dy, T dz, T cwp,       \
                                   int nx, int ny, int nz) {                            \
    return dist3d_003<T>(file, npt, part, npmax, npp, x0, y0, dx, dy, dz, cwp, nx, ny,  \
                         nz);                                                           \
  }                                                                                     \
  extern "C" int oq_dist3d_100_##S(T* part, int npmax, int* npp, const int* ppc, T qm,  \
                                   T np, T gamma, const T* bc, const T* lb,             \
                                   const T* ub, T r1, T r2, int nx, int ny, int nz) {   \
    return dist3d_100<T>(part, npmax, npp, ppc, qm, np, gamma, bc, lb, ub, r1, r2, nx,  \
                         ny, nz);                                                       \
  }                                                                                     \
  extern "C" int oq_beam_static_##S(T np, T x0, T y0, T z0, T sigx, T sigy, T sigz,    \
                                    const T* cx, const T* cy, const T* zf, int nx,      \
                                    int ny, int nz, T* q3) {                            \
    beam_static<T>(np, x0, y0, z0, sigx, sigy, sigz, cx, cy, zf, nx, ny, nz, q3);       \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_pgbpush32l_qp_##S(T* part, int npp, const T* fxyz, const T* bxyz,  \
                                      T qbm, T dt, T dex, T dxi, int indx, int indy,    \
                                      int indz) {                                       \
    return pgbpush32l_qp<T>(part, npp, fxyz, bxyz, qbm, dt, dt, 1 << indx, 1 << indy,   \
                            1 << indz, (1 << indx) + 2, (1 << indy) + 1, 1, dex, dxi,   \
                            T(0));                                                      \
  }                                                                                     \
  extern "C" int oq_pgpost32l_##S(const T* part, int npp, T* q3, int indx, int indy,    \
                                  int indz) {                                           \
    (void)indz;                                                                         \
    pgpost32l<T>(part, npp, q3, (1 << indx) + 2, (1 << indy) + 1);                      \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" void* oq_sim_create_##S(const T* params, int nparams) {                    \
    return sim_create<T>(params, nparams);                                              \
  }                                                                                     \
  extern "C" int oq_sim_destroy_##S(void* h) {                                          \
    delete static_cast<OSim<T>*>(h);                                                    \
    return 0;                                                                           \
  }                                                                                     \
  extern "C" int oq_sim_begin3d_##S(void* h) { return static_cast<OSim<T>*>(h)->begin3d(); } \
  extern "C" int oq_sim_slice_##S(void* h, int j) { return static_cast<OSim<T>*>(h)->slice(j); } \
  extern "C" int oq_sim_step3d_##S(void* h) { return static_cast<OSim<T>*>(h)->step3d(); } \
  extern "C" int oq_sim_get_##S(void* h, int what, T* out, long long n) {               \
    return static_cast<OSim<T>*>(h)->get(what, out, n);                                 \
  }                                                                                     \
  extern "C" long long oq_sim_size_##S(void* h, int what) {                             \
    return static_cast<OSim<T>*>(h)->size(what);                                        \
  }                                                                                     \
  extern "C" int oq_sim_set_##S(void* h, int what, const T* in, long long n) {          \
    return static_cast<OSim<T>*>(h)->set(what, in, n);                                  \
  }

OQ_DEF(float, f)
OQ_DEF(double, d)
