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
//  * the Poisson form-factor table of MPPOISD22 isign = 0
//    (fpois2d_lib77.f:1509-1531) with ax = ay = 0.912871, affp = 1
//    (field2d_class.f03:129).
// Arithmetic is kept in the reference's precision and order (FP32 `real`,
// double where the reference declares double precision), so the device
// starts from the same bits as the reference's SGL build.
#include "qp_loader.h"

#include <algorithm>
#include <cmath>

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

long long plasma_load(const PlasmaProfile& p, int nx, int ny, float s,
                      std::vector<float> (&c)[8], std::string* err) {
  float den_temp;
  if (!longitudinal(p, s, &den_temp, err)) return -1;
  const float qm = den_temp * p.den * p.q / std::fabs(p.q) / (float)p.xppc / (float)p.yppc;
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
          // centroid offsets are zero for the profile-0 beams this engine loads
          const float txx = 0.0f, tyy = 0.0f;
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
