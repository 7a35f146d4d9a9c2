// qp_loader.cpp -- host-side initial conditions and tables of the engine.
//
// These run once per species, beam or context, not per slice:
//  * uniform plasma of profile 0 (dist2d_000, fdist2d_class.f03:212-316, one
//    rank: cells i = 2..nx-1, j = 2..ny, particle order i, j, ix, iy);
//  * the tri-Gaussian beam of profile 0 drawn by PRVDIST32_RANDOM
//    (part3d_lib77.f:411-552) from the Box-Muller generator ranorm
//    (part3d_lib77.f:1324-1383, two 48-bit LCGs in double precision with the
//    fixed seeds of its DATA statement), with the charge normalisation of
//    init_fdist3d_000 (fdist3d_class.f03:311-316);
//  * the beams of profiles 1 (PRVDIST32_RAN_PFL), 2 (PRVDIST32_TWISS), 3 (a
//    particle file), 100 (a ring) and the analytic density of static beams
//    (fdist3d_class.f03:423-1166, part3d_lib77.f:1-410);
//  * the Poisson form-factor table of MPPOISD22 isign = 0
//    (fpois2d_lib77.f:1509-1531) with ax = ay = 0.912871, affp = 1
//    (field2d_class.f03:129).
// Arithmetic is kept in the reference's precision and order (FP32 `real`,
// double where the reference declares double precision), so the device
// starts from the same bits as the reference's SGL build.
#include "qp_loader.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>

namespace qp {

double Ranorm::next() {
  const double h1l = 65531.0, h1u = 32767.0, h2l = 65525.0;
  if (iflg != 0) {
    const double v = r0;
    r0 = 0.0;
    iflg = 0;
    return v;
  }
  int isc = 65536;
  double asc = (double)isc;
  double bsc = asc * asc;
  int i1 = r1 - (r1 / isc) * isc;
  double r3 = h1l * (double)r1 + asc * h1u * (double)i1;
  i1 = (int)(r3 / bsc);
  r3 = r3 - (double)i1 * bsc;
  bsc = 0.5 * bsc;
  i1 = r2 / isc;
  isc = r2 - i1 * isc;
  r0 = h1l * (double)r2 + asc * h1u * (double)isc;
  asc = 1.0 / bsc;
  isc = (int)(r0 * asc);
  r2 = (int)(r0 - (double)isc * bsc);
  r3 = r3 + ((double)isc + 2.0 * h1u * (double)i1);
  isc = (int)(r3 * asc);
  r1 = (int)(r3 - (double)isc * bsc);
  const double temp = std::sqrt(-2.0 * std::log(((double)r1 + (double)r2 * asc) * asc));
  isc = 65536;
  asc = (double)isc;
  bsc = asc * asc;
  i1 = r4 - (r4 / isc) * isc;
  r3 = h2l * (double)r4 + asc * h1u * (double)i1;
  i1 = (int)(r3 / bsc);
  r3 = r3 - (double)i1 * bsc;
  bsc = 0.5 * bsc;
  i1 = r5 / isc;
  isc = r5 - i1 * isc;
  r0 = h2l * (double)r5 + asc * h1u * (double)isc;
  asc = 1.0 / bsc;
  isc = (int)(r0 * asc);
  r5 = (int)(r0 - (double)isc * bsc);
  r3 = r3 + ((double)isc + 2.0 * h1u * (double)i1);
  isc = (int)(r3 * asc);
  r4 = (int)(r3 - (double)isc * bsc);
  r0 = 6.28318530717959 * (((double)r4 + (double)r5 * asc) * asc);
  const double v = temp * std::sin(r0);
  r0 = temp * std::cos(r0);
  iflg = 1;
  return v;
}

long long plasma_uniform(int nx, int ny, int xppc, int yppc, float q, float den,
                         std::vector<float> (&c)[8]) {
  const float qm = 1.0f * den * q / std::fabs(q) / (float)xppc / (float)yppc;
  const long long n = (long long)(nx - 2) * (ny - 1) * xppc * yppc;
  for (auto& v : c) {
    v.clear();
    v.reserve(n);
  }
  for (int i = 2; i <= nx - 1; ++i)
    for (int j = 2; j <= ny; ++j)
      for (int ix = 0; ix < xppc; ++ix)
        for (int iy = 0; iy < yppc; ++iy) {
          c[0].push_back(((float)ix + 0.5f) / (float)xppc + (float)i - 1.0f);
          c[1].push_back(((float)iy + 0.5f) / (float)yppc + (float)j - 1.0f + 0.0f);
          c[2].push_back(0.f);
          c[3].push_back(0.f);
          c[4].push_back(0.f);
          c[5].push_back(1.f);
          c[6].push_back(1.f);
          c[7].push_back(qm);
        }
  return n;
}

// The longitudinal factor den_temp of dist2d_0xx (fdist2d_class.f03:421-438):
// 1 without a profile, else linear between the points (s[i], fs[i]).
static bool longitudinal(const PlasmaProfile& p, float s, float* den, std::string* err) {
  *den = 1.0f;
  const int n = (int)p.fs.size();
  if (n == 0) return true;
  if ((int)p.s.size() != n) {
    *err = "piecewise_density and piecewise_s have different sizes";
    return false;
  }
  if (s < p.s[0] || s > p.s[n - 1]) {
    *err = "The s is out of the bound!";
    return false;
  }
  for (int i = 1; i < n; ++i) {
    if (p.s[i] < p.s[i - 1]) {
      *err = "s is not monotonically increasing!";
      return false;
    }
    if (s <= p.s[i]) {
      *den = p.fs[i - 1] + (p.fs[i] - p.fs[i - 1]) / (p.s[i] - p.s[i - 1]) * (s - p.s[i - 1]);
      break;
    }
  }
  return true;
}

bool plasma_qm(const PlasmaProfile& p, float s, float* qm, std::string* err) {
  float den_temp;
  if (!longitudinal(p, s, &den_temp, err)) return false;
  *qm = den_temp * p.den * p.q / std::fabs(p.q) / (float)p.xppc / (float)p.yppc;
  return true;
}

long long plasma_load(const PlasmaProfile& p, int nx, int ny, float s, bool factor_only,
                      std::vector<float> (&c)[8], std::string* err) {
  float den_temp, qm_s;
  if (!longitudinal(p, s, &den_temp, err) || !plasma_qm(p, s, &qm_s, err)) return -1;
  const float qm = factor_only ? 1.0f : qm_s;
  const int nr = (int)p.r.size();
  if (p.profile == 12) {
    if (nr < 2 || (int)p.fr.size() != nr) {
      *err = "The piecewise_radial_density and r array have different sizes!";
      return -1;
    }
    for (int k = 1; k < nr; ++k)
      if (p.r[k] <= p.r[k - 1]) {
        *err = "r is not monotonically increasing!";
        return -1;
      }
  } else if (p.profile != 0 && p.profile != 10 && p.profile != 11) {
    *err = "Invalid species profile number: " + std::to_string(p.profile);
    return -1;
  }
  // fdist2d_010: reciprocal squared radii; fdist2d_011: 0.5 / sigr^2
  const float iirx2 = 1.0f / (p.irx * p.irx), iiry2 = 1.0f / (p.iry * p.iry);
  const float iorx2 = 1.0f / (p.orx * p.orx), iory2 = 1.0f / (p.ory * p.ory);
  const float isigr2 = 0.5f / (p.sigr * p.sigr);
  for (auto& v : c) v.clear();
  for (int i = 2; i <= nx - 1; ++i)
    for (int j = 2; j <= ny; ++j)
      for (int ix = 0; ix < p.xppc; ++ix)
        for (int iy = 0; iy < p.yppc; ++iy) {
          const float x = ((float)ix + 0.5f) / (float)p.xppc + (float)i - 1.0f;
          const float y = ((float)iy + 0.5f) / (float)p.yppc + (float)j - 1.0f + 0.0f;
          float q = qm;
          if (p.profile == 10) {
            const float dx2 = (x - p.cx) * (x - p.cx), dy2 = (y - p.cy) * (y - p.cy);
            if (dx2 * iirx2 + dy2 * iiry2 < 1.0f || dx2 * iorx2 + dy2 * iory2 > 1.0f) continue;
          } else if (p.profile == 11) {
            const float rr = std::sqrt((x - p.cx) * (x - p.cx) + (y - p.cy) * (y - p.cy));
            q = qm * std::exp(-((rr - p.r0) * (rr - p.r0)) * isigr2);
          } else if (p.profile == 12) {
            const float rr = std::sqrt((x - p.cx) * (x - p.cx) + (y - p.cy) * (y - p.cy));
            if (rr < p.r[0] || rr > p.r[nr - 1]) continue;
            float f = den_temp;
            for (int k = 1; k < nr; ++k)
              if (rr <= p.r[k]) {
                f = p.fr[k - 1] + (p.fr[k] - p.fr[k - 1]) / (p.r[k] - p.r[k - 1]) * (rr - p.r[k - 1]);
                break;
              }
            q = qm * f;
          }
          c[0].push_back(x);
          c[1].push_back(y);
          c[2].push_back(0.f);
          c[3].push_back(0.f);
          c[4].push_back(0.f);
          c[5].push_back(1.f);
          c[6].push_back(1.f);
          c[7].push_back(q);
        }
  return (long long)c[0].size();
}

float beam_charge(float q, float peak, const float sig[3], const float lo[3], const float hi[3],
                  int indx, int indy, int indz, int npx, int npy, int npz) {
  const float dx = (hi[0] - lo[0]) / (float)(1 << indx);
  const float dy = (hi[1] - lo[1]) / (float)(1 << indy);
  const float dz = (hi[2] - lo[2]) / (float)(1 << indz);
  float qm = q / std::fabs(q) * std::fabs(peak) *
             std::pow(2.0f * 3.1415926535897932f, 1.5f) * sig[0] * sig[1] * sig[2];
  qm = qm / dx / dy / dz;
  qm = qm / (float)npx;
  qm = qm / (float)npy;
  qm = qm / (float)npz;
  return qm;
}

long long beam_random(Ranorm& rng, const BeamLoad& b, std::vector<float> (&c)[7], int* ierr) {
  for (auto& v : c) v.clear();
  *ierr = 0;
  const float x0 = b.x0, y0 = b.y0, z0 = b.z0;
  const float sigx = b.sigx, sigy = b.sigy, sigz = b.sigz;
  const float x2 = 2.0f * x0, y2 = 2.0f * y0;
  const float borderlx = std::max(x0 - 5.0f * sigx, 1.0f);
  const float borderly = std::max(y0 - 5.0f * sigy, 1.0f);
  const float borderlz = std::max(z0 - 5.0f * sigz, 1.0f);
  const float borderx = std::min(x0 + 5.0f * sigx, (float)(b.nx - 1));
  const float bordery = std::min(y0 + 5.0f * sigy, (float)(b.ny - 1));
  const float borderz = std::min(z0 + 5.0f * sigz, (float)(b.nz - 1));
  long long n = 0, npt = 1;
  auto put = [&](float px, float py, float pz, float vx, float vy, float vz) {
    if (npt < b.npmax) {
      npt = n + 1;
      c[0].push_back(px);
      c[1].push_back(py);
      c[2].push_back(pz);
      c[3].push_back(vx);
      c[4].push_back(vy);
      c[5].push_back(vz);
      c[6].push_back(b.qm);
      n = npt;
    } else {
      *ierr += 1;
    }
  };
  int j = 0, l = b.npz;
  while (j < b.npx) {
    int k = 0;
    while (k < b.npy) {
      l = l - b.npz;
      while (l < b.npz) {
        float tz, tx, ty;
        do {
          tz = (float)((double)z0 + (double)sigz * rng.next());
        } while (tz >= borderz || tz <= borderlz);
        do {
          tx = (float)((double)x0 + (double)sigx * rng.next());
        } while (tx >= borderx || tx <= borderlx);
        do {
          ty = (float)((double)y0 + (double)sigy * rng.next());
        } while (ty >= bordery || ty <= borderly);
        const float vx = (float)((double)b.vtx * rng.next() + 0.0);
        const float vy = (float)((double)b.vty * rng.next() + 0.0);
        float vz = (float)((double)b.vtz * rng.next() + (double)b.vdz);
        vz = std::sqrt(vz * vz - 1.0f - vx * vx - vy * vy);
        if (ty >= 0.0f && ty < (float)b.ny && tz >= 0.0f && tz < (float)b.nz) {
          // centroid offsets -(c0 (z-z0)^2 + c1 (z-z0) + c2), in cells
          const float dzz = tz - z0;
          const float txx = -(b.cx[0] * (dzz * dzz)) - b.cx[1] * dzz - b.cx[2];
          const float tyy = -(b.cy[0] * (dzz * dzz)) - b.cy[1] * dzz - b.cy[2];
          put(tx + txx, ty + tyy, tz, vx, vy, vz);
          if (b.quiet) put(x2 - tx + txx, y2 - ty + tyy, tz, -vx, -vy, vz);
        }
        l = l + 1;
        if (b.quiet) l = l + 1;
      }
      k = k + 1;
    }
    j = j + 1;
  }
  return n;
}

float Uniform::next() {
  s += 0x9e3779b97f4a7c15ull;
  unsigned long long z = s;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z = z ^ (z >> 31);
  return (float)(z >> 40) * (1.0f / 16777216.0f);
}

bool beam_zprofile(const std::vector<float>& z, const std::vector<float>& fz, float zl, float dz,
                   int nz, std::vector<float>* zf, float* sumz) {
  const size_t nzf = z.size();
  if (nzf < 2 || fz.size() != nzf) return false;
  float sum = 0.0f;
  for (size_t ii = 1; ii < nzf; ++ii) {
    if (z[ii] <= z[ii - 1]) return false;
    sum = sum + (fz[ii] + fz[ii - 1]) * (z[ii] - z[ii - 1]) * 0.5f;
  }
  *sumz = sum;
  std::vector<float> zc(nzf);
  for (size_t ii = 0; ii < nzf; ++ii) zc[ii] = (z[ii] - zl) / dz;
  zf->assign(nz, 0.0f);
  for (int i = 1; i <= nz; ++i) {
    const float ri = (float)i;
    for (size_t j = 1; j < nzf; ++j) {
      if (ri >= zc[j - 1] && ri < zc[j]) {
        (*zf)[i - 1] = fz[j] + (fz[j - 1] - fz[j]) / (zc[j - 1] - zc[j]) * (ri - zc[j]);
        break;
      }
    }
  }
  return true;
}

float beam_charge_q(float q, float peak, float e, float sx, float sy, float sz, float dx, float dy,
                    float dz, int npx, int npy, int npz) {
  const float twopi = 2.0f * 3.1415926535897932f;
  float qm = q / std::fabs(q) * std::fabs(peak) * (e == 1.0f ? twopi : std::pow(twopi, e)) * sx *
             sy * sz;
  qm = qm / dx / dy / dz;
  qm = qm / (float)npx;
  qm = qm / (float)npy;
  qm = qm / (float)npz;
  return qm;
}

// The reference's "npt <= npmax" test lets a partition take npmax + 1
// particles, one past its array; here a particle is stored only while fewer
// than npmax are, and each one refused counts in *ierr.
long long beam_ran_pfl(Ranorm& rng, Uniform& uni, const BeamLoad& b, std::vector<float> (&c)[7],
                       int* ierr) {
  for (auto& v : c) v.clear();
  *ierr = 0;
  const float x0 = b.x0, y0 = b.y0, z0 = b.z0;
  const float sigx = b.sigx, sigy = b.sigy;
  const float x2 = 2.0f * x0, y2 = 2.0f * y0;
  const float borderlx = std::max(x0 - 5.0f * sigx, 1.0f);
  const float borderly = std::max(y0 - 5.0f * sigy, 1.0f);
  const float borderx = std::min(x0 + 5.0f * sigx, (float)(b.nx - 1));
  const float bordery = std::min(y0 + 5.0f * sigy, (float)(b.ny - 1));
  const int nz1 = b.nz - 1;
  std::vector<float> dp(b.zf);
  float amax = 0.0f;
  for (float& v : dp) {
    v = std::fabs(v);
    amax = std::max(amax, v);
  }
  // an all-zero profile accepts nothing (the reference would draw forever)
  if (!(amax > 0.0f) || (int)dp.size() < b.nz || nz1 < 1) return 0;
  amax = amax * 1.2f;
  for (float& v : dp) v = v / amax;
  long long n = 0, npt = 1;
  auto put = [&](float px, float py, float pz, float vx, float vy, float vz) {
    if (npt <= b.npmax && n < b.npmax) {
      npt = n + 1;
      c[0].push_back(px);
      c[1].push_back(py);
      c[2].push_back(pz);
      c[3].push_back(vx);
      c[4].push_back(vy);
      c[5].push_back(vz);
      c[6].push_back(b.qm);
      n = npt;
    } else {
      *ierr += 1;
    }
  };
  float tmpu[1024], tmpz[1024];
  int cnt = 0;
  int j = 0, l = b.npz;
  while (j < b.npx) {
    int k = 0;
    while (k < b.npy) {
      l = l - b.npz;
      while (l < b.npz) {
        if (cnt <= 0) {
          for (float& v : tmpu) v = uni.next();
          for (float& v : tmpz) v = uni.next();
          cnt = 1024;
        }
        const float u = tmpu[cnt - 1];
        const float tempz = tmpz[cnt - 1] * (float)nz1;
        cnt = cnt - 1;
        int zi = (int)tempz;
        if (zi > nz1 - 1) zi = nz1 - 1;  // tempz < nz - 1 always: never read past dp
        const float zf = tempz - (float)zi;
        const float zs = 1.0f - zf;
        zi = zi + 1;
        const float dpi = dp[zi - 1] * zs + dp[zi] * zf;
        if (u <= dpi) {
          float tx, ty;
          do {
            tx = (float)((double)x0 + (double)sigx * rng.next());
          } while (tx >= borderx || tx <= borderlx);
          do {
            ty = (float)((double)y0 + (double)sigy * rng.next());
          } while (ty >= bordery || ty <= borderly);
          if (ty < (float)b.ny && ty > 0.0f && tempz < (float)b.nz && tempz > 0.0f) {
            const float vx = (float)((double)b.vtx * rng.next());
            const float vy = (float)((double)b.vty * rng.next());
            float vz = (float)((double)b.vtz * rng.next() + (double)b.vdz);
            vz = std::sqrt(vz * vz - 1.0f - vx * vx - vy * vy);
            const float dzz = tempz - z0;
            const float txx = -(b.cx[0] * (dzz * dzz)) - b.cx[1] * dzz - b.cx[2];
            const float tyy = -(b.cy[0] * (dzz * dzz)) - b.cy[1] * dzz - b.cy[2];
            put(tx + txx, ty + tyy, tempz, vx, vy, vz);
            if (b.quiet) put(x2 - tx + txx, y2 - ty + tyy, tempz, -vx, -vy, vz);
          }
          l = l + 1;
          if (b.quiet) l = l + 1;
        }
      }
      k = k + 1;
    }
    j = j + 1;
  }
  return n;
}

long long beam_twiss(Ranorm& rng, const BeamLoad& b, std::vector<float> (&c)[7], int* ierr) {
  for (auto& v : c) v.clear();
  *ierr = 0;
  const float x0 = b.x0, y0 = b.y0, z0 = b.z0, sigz = b.sigz, gamma = b.vdz;
  const float x2 = 2.0f * x0, y2 = 2.0f * y0;
  const float sigx = std::sqrt(b.betax * b.emitx / gamma);
  const float sigy = std::sqrt(b.betay * b.emity / gamma);
  const float vtx = b.emitx / sigx, vty = b.emity / sigy;
  const float borderlx = std::max(x0 - 3.0f * sigx, 1.0f);
  const float borderly = std::max(y0 - 3.0f * sigy, 1.0f);
  const float borderlz = std::max(z0 - 3.0f * sigz, 1.0f);
  const float borderx = std::min(x0 + 3.0f * sigx, (float)(b.nx - 1));
  const float bordery = std::min(y0 + 3.0f * sigy, (float)(b.ny - 1));
  const float borderz = std::min(z0 + 3.0f * sigz, (float)(b.nz - 1));
  const float gax = gamma * b.alphax / b.betax, gay = gamma * b.alphay / b.betay;
  long long n = 0, npt = 1;
  auto put = [&](float px, float py, float pz, float vx, float vy, float vz) {
    if (npt <= b.npmax && n < b.npmax) {
      npt = n + 1;
      c[0].push_back(px);
      c[1].push_back(py);
      c[2].push_back(pz);
      c[3].push_back(vx);
      c[4].push_back(vy);
      c[5].push_back(vz);
      c[6].push_back(b.qm);
      n = npt;
    } else {
      *ierr += 1;
    }
  };
  int j = 0, l = b.npz;
  while (j < b.npx) {
    int k = 0;
    while (k < b.npy) {
      l = l - b.npz;
      while (l < b.npz) {
        double tempz, tempx, tempy;
        do {
          tempz = (double)z0 + (double)sigz * rng.next();
        } while (tempz >= (double)borderz || tempz <= (double)borderlz);
        float tx, ty;
        for (;;) {
          do {
            tx = (float)rng.next();
            tempx = (double)(x0 + sigx * tx);
          } while (tempx >= (double)borderx || tempx <= (double)borderlx);
          do {
            ty = (float)rng.next();
            tempy = (double)(y0 + sigy * ty);
          } while (tempy >= (double)bordery || tempy <= (double)borderly);
          if (!(tx * tx + ty * ty > 9.0f)) break;
        }
        float tvtx = (float)((double)vtx * rng.next());
        float tvty = (float)((double)vty * rng.next());
        const float tvtz = (float)((double)b.vtz * rng.next() + (double)b.vdz);
        tvtx = (float)((double)tvtx - (double)gax * (tempx - (double)x0));
        tvty = (float)((double)tvty - (double)gay * (tempy - (double)y0));
        if (tempy >= 0.0 && tempy < (double)b.ny && tempz >= 0.0 && tempz < (double)b.nz) {
          put((float)tempx, (float)tempy, (float)tempz, tvtx, tvty, tvtz);
          if (b.quiet)
            put((float)((double)x2 - tempx), (float)((double)y2 - tempy), (float)tempz, -tvtx,
                -tvty, tvtz);
        }
        l = l + 1;
        if (b.quiet) l = l + 1;
      }
      k = k + 1;
    }
    j = j + 1;
  }
  return n;
}

// One list-directed read of 7 reals: a new line, continued on the next lines
// while fewer than 7 values were found; values are separated by blanks or
// commas, a Fortran exponent letter d/D reads as e.
static bool read7(std::FILE* f, float v[7]) {
  int got = 0;
  char line[4096];
  while (got < 7) {
    if (!std::fgets(line, sizeof line, f)) return false;
    for (char* p = line; *p; ++p)
      if (*p == ',') *p = ' ';
      else if (*p == 'd' || *p == 'D') *p = 'e';
    char* p = line;
    while (got < 7) {
      char* e = nullptr;
      const float x = std::strtof(p, &e);
      if (e == p) {
        while (*e == ' ' || *e == '\t' || *e == '\r' || *e == '\n') ++e;
        if (*e != 0) return false;  // not a number
        break;
      }
      v[got++] = x;
      p = e;
    }
  }
  return true;
}

long long beam_file(const std::string& file, long long npt, float x0, float y0, float cwp,
                    float dx, float dy, float dz, int nx, int ny, int nz,
                    std::vector<float> (&c)[7], std::string* err) {
  for (auto& v : c) v.clear();
  std::FILE* f = std::fopen(file.c_str(), "r");
  if (!f) {
    *err = "cannot open the beam file " + file;
    return -1;
  }
  long long n = 0;
  for (long long i = 0; i < npt; ++i) {
    float v[7];
    if (!read7(f, v)) {
      std::fclose(f);
      *err = "read beam file error at particle " + std::to_string(i + 1);
      return -1;
    }
    const float tx = v[1] / cwp / dx + x0;
    const float ty = v[2] / cwp / dy + y0;
    const float tz = -(v[0] / cwp / dz);
    if (tx >= 1.0f && tx <= (float)(nx - 1) && ty >= 0.0f && ty < (float)ny && tz >= 0.0f &&
        tz < (float)nz) {
      c[0].push_back(tx);
      c[3].push_back(v[4]);
      c[1].push_back(ty);
      c[4].push_back(v[5]);
      c[2].push_back(tz);
      c[5].push_back(v[3]);
      c[6].push_back(v[6]);
      ++n;
    }
  }
  std::fclose(f);
  return n;
}

long long beam_ring(const int ppc[3], float qm, float np, float gamma, const float bc[3],
                    const float lb_in[3], const float ub_in[3], float r1, float r2, int nx, int ny,
                    int nz, std::vector<float> (&c)[7]) {
  for (auto& v : c) v.clear();
  float lb[3], ub[3];
  lb[0] = std::max(lb_in[0], 0.0f);
  ub[0] = std::min(ub_in[0], (float)nx);
  const int nd[3] = {nx, ny, nz};
  for (int a = 1; a < 3; ++a) {
    if (lb_in[a] > (float)nd[a] || ub_in[a] < 0.0f) return 0;
    lb[a] = std::max(lb_in[a], 0.0f);
    ub[a] = std::min(ub_in[a], (float)nd[a]);
  }
  const float r22 = r2 * r2;
  long long n = 0;
  for (int i = (int)lb[0]; i <= (int)ub[0] - 1; ++i)
    for (int j = (int)lb[1]; j <= (int)ub[1] - 1; ++j)
      for (int k = (int)lb[2]; k <= (int)ub[2] - 1; ++k)
        for (int ix = 0; ix < ppc[0]; ++ix)
          for (int iy = 0; iy < ppc[1]; ++iy)
            for (int iz = 0; iz < ppc[2]; ++iz) {
              const float tx = ((float)ix + 0.5f) / (float)ppc[0] + (float)i - 1.0f;
              const float ty = ((float)iy + 0.5f) / (float)ppc[1] + (float)j - 1.0f;
              const float tz = ((float)iz + 0.5f) / (float)ppc[2] + (float)k - 1.0f;
              const float a1 = std::fabs(tz - bc[2]);
              const float a2 = std::sqrt((tx - bc[0]) * (tx - bc[0]) + (ty - bc[1]) * (ty - bc[1]));
              const float a3 = std::fabs(a2 - r1);
              const float a4 = a1 * a1 + a3 * a3;
              c[0].push_back(tx);
              c[1].push_back(ty);
              c[2].push_back(tz);
              c[3].push_back(0.0f);
              c[4].push_back(0.0f);
              c[5].push_back(gamma);
              c[6].push_back(qm * np * std::exp(-(a4 / r22 * 0.5f)));
              ++n;
            }
  return n;
}

void beam_static_plane(float amp, float x0, float y0, float z0, float sigx, float sigy,
                       float sigz, const float cx[3], const float cy[3],
                       const std::vector<float>& zf, int nx, int ny, int k, long long ld,
                       float* plane) {
  const float zval = (float)k - z0;
  const float cx0 = -(cx[0] * (zval * zval)) - cx[1] * zval - cx[2];
  const float cy0 = -(cy[0] * (zval * zval)) - cy[1] * zval - cy[2];
  const float t1 =
      zf.empty() ? amp * std::exp(-(zval * zval / 2.0f / (sigz * sigz))) : amp * zf[k];
  std::vector<float> ey(ny);
  for (int j = 0; j < ny; ++j) {
    const float d = (float)j - y0 + cy0;
    ey[j] = std::exp(-(d * d / 2.0f / (sigy * sigy)));
  }
  for (int i = 0; i < nx; ++i) {
    const float d = (float)i - x0 + cx0;
    const float t2 = t1 * std::exp(-(d * d / 2.0f / (sigx * sigx)));
    for (int j = 0; j < ny; ++j) plane[(size_t)j * ld + i] = t2 * ey[j];
  }
}

void form_factor(int nx, int ny, float ax, float ay, float affp, std::vector<float>& re,
                 std::vector<float>& im) {
  re.assign((size_t)nx * ny, 0.f);
  im.assign((size_t)nx * ny, 0.f);
  const float dnx = 6.28318530717959f / (float)(nx + nx);
  const float dny = 6.28318530717959f / (float)(ny + ny);
  for (int kx = 0; kx < nx; ++kx) {
    const float dkx = dnx * (float)kx;
    const float at1 = dkx * dkx;
    const float at2 = (dkx * ax) * (dkx * ax);
    for (int ky = 0; ky < ny; ++ky) {
      const float dky = dny * (float)ky;
      const float at3 = dky * dky + at1;
      const float at4 = std::exp(-0.5f * ((dky * ay) * (dky * ay) + at2));
      const size_t o = (size_t)kx * ny + ky;
      if (at3 == 0.0f) {
        re[o] = affp;
        im[o] = 1.0f;
      } else {
        re[o] = affp * at4 / at3;
        im[o] = at4;
      }
    }
  }
}

}  // namespace qp
