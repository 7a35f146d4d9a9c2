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

// The charge per particle of profile p before its transverse factor, at
// propagation distance s: den_temp(s) * den * sign(q) / (xppc * yppc)
// (dist2d_0xx, fdist2d_class.f03:246-248 with 421-438).  false with *err on a
// bad longitudinal profile.
bool plasma_qm(const PlasmaProfile& p, float s, float* qm, std::string* err);

// Loads profile p at propagation distance s (dist2d_0xx for one rank:
// cells i = 2..nx-1, j = 2..ny, order i, j, ix, iy).  Returns the number of
// particles, or -1 with a message in *err.  With factor_only, c[7] holds the
// transverse factor of each particle's charge (1, or the profile's weight)
// and the charge is qm(s) * c[7], the same single product the loader forms.
long long plasma_load(const PlasmaProfile& p, int nx, int ny, float s, bool factor_only,
                      std::vector<float> (&c)[8], std::string* err);

// One beam's loader parameters with lengths in cells (the init_fdist3d_0xx
// conversions).  Profile 0 uses sig*, cx, cy; profile 1 sigx, sigy, cx, cy
// and zf; profile 2 the Twiss fields, sigz and vtz.
struct BeamLoad {
  int npx, npy, npz, nx, ny, nz;
  float qm, vtx, vty, vtz, vdz;
  float sigx, sigy, sigz;  // in cells
  float x0, y0, z0;        // centre in cells
  bool quiet;
  long long npmax;
  float cx[3] = {0.f, 0.f, 0.f}, cy[3] = {0.f, 0.f, 0.f};  // centroid polynomials
  std::vector<float> zf;                                   // profile 1: density of slice i = 1..nz
  float alphax = 0.f, alphay = 0.f, betax = 0.f, betay = 0.f, emitx = 0.f, emity = 0.f;
};

// Uniform numbers in [0, 1) for the longitudinal acceptance draws of
// PRVDIST32_RAN_PFL, where the reference calls the Fortran intrinsic
// RANDOM_NUMBER (a compiler runtime's generator, not part of the reference):
// SplitMix64 (Steele, Lea, Flood 2014) from a 64-bit seed, each number the
// top 24 bits of an output times 2^-24.
struct Uniform {
  unsigned long long s;
  explicit Uniform(unsigned long long seed) : s(seed) {}
  float next();
};

float beam_charge(float q, float peak, const float sig[3], const float lo[3], const float hi[3],
                  int indx, int indy, int indz, int npx, int npy, int npz);
// PRVDIST32_RANDOM (profile 0): tri-Gaussian, 5-sigma cut, centroid offsets.
long long beam_random(Ranorm& rng, const BeamLoad& b, std::vector<float> (&c)[7], int* ierr);

// Profile 1 (fdist3d_001): the piecewise longitudinal profile fz at z (box
// units) as the density of slices i = 1..nz (dist3d_001, fdist3d_class.f03:
// 600-611), with zl the box's lower z and dz the cell size; *sumz gets the
// trapezoid integral of fz over z (init_fdist3d_001, 508-518).  Returns false
// when z does not increase.
bool beam_zprofile(const std::vector<float>& z, const std::vector<float>& fz, float zl, float dz,
                   int nz, std::vector<float>* zf, float* sumz);
// Charge per particle of profiles 1 and 2: q/|q| |peak| (2 pi)^e sx sy sz /
// (dx dy dz npx npy npz), e = 1 with sz = sumz (001) or 1.5 with sz = sigmaz (002).
float beam_charge_q(float q, float peak, float e, float sx, float sy, float sz, float dx, float dy,
                    float dz, int npx, int npy, int npz);
// PRVDIST32_RAN_PFL (part3d_lib77.f:193-410): Gaussian in x and y, the
// longitudinal profile b.zf by acceptance-rejection with uniform draws.
long long beam_ran_pfl(Ranorm& rng, Uniform& uni, const BeamLoad& b, std::vector<float> (&c)[7],
                       int* ierr);
// PRVDIST32_TWISS (part3d_lib77.f:1-191): Twiss-parameter beam, 3-sigma cut,
// circular cut at 3 in the normalised transverse draws.
long long beam_twiss(Ranorm& rng, const BeamLoad& b, std::vector<float> (&c)[7], int* ierr);
// dist3d_003 (fdist3d_class.f03:899-974): up to npt particles read from a
// text file of lines "z x y pz px py q" in physical units, kept when inside
// the box.  Returns -1 with a message in *err when the file cannot be read.
long long beam_file(const std::string& file, long long npt, float x0, float y0, float cwp,
                    float dx, float dy, float dz, int nx, int ny, int nz,
                    std::vector<float> (&c)[7], std::string* err);
// dist3d_100 (fdist3d_class.f03:1081-1166): a ring of radius r1 and width
// r2 (cells), ppc particles per cell in the box [lb, ub] (cells), weights
// qm np exp(-((z - bcz)^2 + (|r - bc| - r1)^2) / (2 r2^2)).
long long beam_ring(const int ppc[3], float qm, float np, float gamma, const float bc[3],
                    const float lb[3], const float ub[3], float r1, float r2, int nx, int ny,
                    int nz, std::vector<float> (&c)[7]);
// The analytic density of a static beam (profiles 0 and 1 with static =
// true, dist3d_000/001 fdist3d_class.f03:392-408, 613-630) on slice k
// (0-based) as an (nx) x (ny) plane, row y at y * ld: Gaussian in z with
// sigz (zf empty) or the profile zf.
void beam_static_plane(float amp, float x0, float y0, float z0, float sigx, float sigy,
                       float sigz, const float cx[3], const float cy[3],
                       const std::vector<float>& zf, int nx, int ny, int k, long long ld,
                       float* plane);

void form_factor(int nx, int ny, float ax, float ay, float affp, std::vector<float>& re,
                 std::vector<float>& im);

}  // namespace qp
