// qp_loader.h -- host-side initial conditions and tables (see qp_loader.cpp).
#pragma once

#include <string>
#include <vector>

namespace qp {

// ranorm's generator state; one per context (the reference's SAVE state).
struct Ranorm {
  int r1 = 885098780, r2 = 1824280461, r4 = 1396483093, r5 = 55318673;
  int iflg = 0;
  double r0 = 0.0;
  double next();
};

// Uniform plasma of profile 0; returns the number of particles; c[0..7] get
// x, y, px, py, pz, p6, p7, q in the loader's order.
long long plasma_uniform(int nx, int ny, int xppc, int yppc, float q, float den,
                         std::vector<float> (&c)[8]);

// A plasma profile with its lengths already in cells (the init_fdist2d_0xx
// conversions): profile 0, 10, 11 or 12 (see qp_species_desc).
struct PlasmaProfile {
  int profile = 0;
  int xppc = 1, yppc = 1;
  float q = -1.f, den = 1.f;
  float cx = 0.f, cy = 0.f;
  float irx = 0.f, iry = 0.f, orx = 0.f, ory = 0.f;  // 10
  float r0 = 0.f, sigr = 0.f;                       // 11
  std::vector<float> r, fr;                         // 12
  std::vector<float> s, fs;                         // longitudinal piecewise
};

// Loads profile p at propagation distance s (dist2d_0xx for one rank:
// cells i = 2..nx-1, j = 2..ny, order i, j, ix, iy).  Returns the number of
// particles, or -1 with a message in *err.
long long plasma_load(const PlasmaProfile& p, int nx, int ny, float s,
                      std::vector<float> (&c)[8], std::string* err);

struct BeamLoad {
  int npx, npy, npz, nx, ny, nz;
  float qm, vtx, vty, vtz, vdz;
  float sigx, sigy, sigz;  // in cells
  float x0, y0, z0;        // centre in cells
  bool quiet;
  long long npmax;
};

float beam_charge(float q, float peak, const float sig[3], const float lo[3], const float hi[3],
                  int indx, int indy, int indz, int npx, int npy, int npz);
long long beam_random(Ranorm& rng, const BeamLoad& b, std::vector<float> (&c)[7], int* ierr);

void form_factor(int nx, int ny, float ax, float ay, float affp, std::vector<float>& re,
                 std::vector<float>& im);

}  // namespace qp
