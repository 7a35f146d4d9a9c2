// qp_loader.h -- host-side initial conditions and tables (see qp_loader.cpp).
#pragma once

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
