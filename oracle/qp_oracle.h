/*
 * qp_oracle.h -- CPU oracle for the QuickPIC per-slice quasi-static path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the B200 engine
 * (libqpgpu); only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  The product never links it.
 *
 * It restates, routine by routine, the Fortran 77 kernels and the Fortran 2003
 * slice loop of QuickPIC-OpenSource (file:line citations beside each function
 * in qp_oracle.cpp), templated on the reference's `real` type:
 *   suffix _f  = float   (the reference's PRECISION=SGL build)
 *   suffix _d  = double  (the reference's default PRECISION=DBL build)
 *
 * PARITY UNPINNED: the reference ships no tests, golden vectors or fixtures,
 * and it cannot be compiled in this environment (no Fortran compiler, no MPI,
 * no HDF5).  The restatement is checked instead against independent
 * known-answer tests (closed-form sine/cosine transforms from scipy, eigenmode
 * Poisson solves, charge conservation, rotation invariants, the ranorm LCG
 * evaluated by hand) kept under tests/golden/.
 *
 * Array layouts are exactly the reference's column-major layouts:
 *   real-space field  rf(dim, nx+2, 2*ny+1)      (ufield2d_class.f03:129)
 *   k-space field     g (dim, ny+1, nx+1)         (ufield2d_class.f03:198)
 *   tiled particles   ppart(8, nppmx, mxyp1), kpic(mxyp1)  (part2d_class.f03:170)
 *   beam particles    part(7, npmax)              (part3d_class.f03)
 *   3D field          q(nx+2, ny+1, nz+1)         (ufield3d_class.f03:116)
 * All integers are 32-bit; every function returns 0 on success.
 */
#ifndef QP_ORACLE_H
#define QP_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define OQ_DECL(T, S)                                                                   \
  /* 2D transforms of one field2d (fftrk / fftkr incl. guard copy), kinds as         \
     field2d_class.f03:157-227 */                                                     \
  int oq_fftrk_##S(T* rs, T* ks, int dim, int kind, int indx, int indy);             \
  int oq_fftkr_##S(T* rs, T* ks, int dim, int kind, int indx, int indy);             \
  /* one 1D pass on a strided line: sine (parity 0) or cosine (1); xpass 1 = x      \
     normalisation, 0 = y normalisation; isign as the reference */                   \
  int oq_line_##S(T* line, int stride, int parity, int xpass, int isign, int indx,   \
                  int indy);                                                         \
  /* k-space solves (fpois2d_lib77.f, fft2d_lib77.f) */                             \
  int oq_ffc_##S(T* ffc_re_im, int indx, int indy, T ax, T ay, T affp);             \
  int oq_pot_##S(const T* q, T* pot, const T* ffc, int indx, int indy);             \
  int oq_smooth_##S(const T* q, T* qs, const T* ffc, int indx, int indy);           \
  int oq_elf_##S(const T* q, T* fxy, const T* ffc, int indx, int indy);             \
  int oq_bf_##S(const T* cu, T* bxy, const T* ffc, int indx, int indy);             \
  int oq_vpot_##S(const T* cu, T* a, const T* ffc, int indx, int indy);            \
  int oq_bfqp_##S(const T* cu, T* dcu, const T* amu, T* bxy, const T* ffc, T aa,    \
                  T dex, int indx, int indy);                                        \
  int oq_div_##S(const T* f, T* df, int ndim, int indx, int indy);                  \
  int oq_grad_##S(const T* df, T* f, int indx, int indy);                           \
  /* guard-cell operations, single-rank branches (ufield2d_lib.f03) */               \
  int oq_cguard_##S(T* rs, int dim, int indx, int indy);                            \
  int oq_acguard_##S(T* rs, int dim, int indx, int indy);                           \
  /* plasma particle kernels (part2d_lib77.f); tiles are 16x16 */                   \
  int oq_ppgppost2l_##S(const T* ppart, T* q, const int* kpic, int nppmx, int indx, \
                        int indy);                                                   \
  int oq_wpgpsipost2l_qp_##S(T* ppart, const T* psi, const int* kpic, T qbm,        \
                             int nppmx, int indx, int indy, T dex);                  \
  int oq_ppgrdcjppost2l_qp_##S(T* ppart, const T* fxy, const T* bxy, const T* psit, \
                               T* cu, T* dcu, T* amu, const int* kpic, T qbm, T dt, \
                               T ci, int nppmx, int indx, int indy, T dex);          \
  int oq_ppgrbppushf23l_qp_##S(T* ppart, const T* fxy, const T* bxy, const T* psit, \
                               const int* kpic, int* ncl, int* ihole, T qbm, T dt,  \
                               T ci, int nppmx, int ntmax, int indx, int indy,      \
                               T dex);                                               \
  /* pmove: PPPORDERF2LA + PPPMOVE2(nvp=1) + PPPORDER2LB; returns 0, or the        \
     required nppmx (>0) when ppart would overflow (ppart then unchanged) */         \
  int oq_pmove_##S(T* ppart, int* kpic, int* ncl, int* ihole, int nppmx, int ntmax, \
                   int indx, int indy);                                              \
  int oq_ppdblkp2l_##S(const T* part, int* kpic, int npp, int* nppmx_out, int indx,  \
                       int indy);                                                    \
  int oq_pppmovin2l_##S(const T* part, T* ppart, int* kpic, int npp, int nppmx,     \
                        int indx, int indy);                                         \
  int oq_pppcheck2l_##S(const T* ppart, const int* kpic, int nppmx, int indx,       \
                        int indy);                                                   \
  /* loaders */                                                                      \
  int oq_dist2d_prof_##S(T* part, int npmax, int* npp, const T* pr);               \
  int oq_dist2d_000_##S(T* part, int npmax, int* npp, int xppc, int yppc, T qm,     \
                        T den, int indx, int indy);                                  \
  int oq_beam_qm_##S(T q, T np, const T* sig, const T* box_lo, const T* box_hi,     \
                     int indx, int indy, int indz, int npx, int npy, int npz,       \
                     T* qm_out);                                                     \
  int oq_prvdist32_random_##S(T* part, int npmax, int* npp, T qm, T vtx, T vty,     \
                              T vtz, T vdz, int npx, int npy, int npz, int indx,    \
                              int indy, int indz, T sigx, T sigy, T sigz, T x0,     \
                              T y0, T z0, const T* cx, const T* cy, int quiet);     \
  /* beam profiles 1, 2, 3, 100 and static densities (fdist3d_class.f03) */        \
  int oq_dist3d_001_zf_##S(const T* z, const T* fz, int nzf, T zmin, T dz, int nz,   \
                           T* zf, T* sumz);                                          \
  int oq_beam_qm2_##S(T q, T np, T e, T sx, T sy, T sz, T dx, T dy, T dz, int npx,  \
                      int npy, int npz, T* qm_out);                                  \
  int oq_prvdist32_ran_pfl_##S(T* part, int npmax, int* npp, T qm, T x0, T y0, T z0,\
                               T sigx, T sigy, T vtx, T vty, T vtz, T vdz,          \
                               const T* cx, const T* cy, int npx, int npy, int npz, \
                               int nx, int ny, int nz, T* dp, int quiet,            \
                               unsigned long long seed);                             \
  int oq_prvdist32_twiss_##S(T* part, int npmax, int* npp, T qm, const T* alpha,    \
                             const T* beta, const T* emt, T sigz, T vdz, T vtz,     \
                             int npx, int npy, int npz, int nx, int ny, int nz,     \
                             T x0, T y0, T z0, int quiet);                           \
  int oq_dist3d_003_##S(const char* file, int npt, T* part, int npmax, int* npp,    \
                        T x0, T y0, T dx, T dy, T dz, T cwp, int nx, int ny, int nz);\
  int oq_dist3d_100_##S(T* part, int npmax, int* npp, const int* ppc, T qm, T np,   \
                        T gamma, const T* bc, const T* lb, const T* ub, T r1, T r2, \
                        int nx, int ny, int nz);                                     \
  int oq_beam_static_##S(T np, T x0, T y0, T z0, T sigx, T sigy, T sigz,            \
                         const T* cx, const T* cy, const T* zf, int nx, int ny,     \
                         int nz, T* q3);                                             \
  int oq_pgpost32l_##S(const T* part, int npp, T* q3, int indx, int indy, int indz);\
  /* beam push PGBPUSH32L_QP with the 3D fields (3, nx+2, ny+1, nz+1); conducting  \
     boundaries drop particles; returns the new count */                             \
  int oq_pgbpush32l_qp_##S(T* part, int npp, const T* fxyz, const T* bxyz, T qbm,   \
                           T dt, T dex, T dxi, int indx, int indy, int indz);        \
  /* full simulation driver (simulation_class.f03:593-769) */                        \
  void* oq_sim_create_##S(const T* params, int nparams);                            \
  int oq_sim_destroy_##S(void* h);                                                   \
  int oq_sim_step3d_##S(void* h);                                                    \
  int oq_sim_slice_##S(void* h, int j);                                              \
  int oq_sim_begin3d_##S(void* h);                                                   \
  int oq_sim_get_##S(void* h, int what, T* out, long long n);                        \
  long long oq_sim_size_##S(void* h, int what);

OQ_DECL(float, f)
OQ_DECL(double, d)
#undef OQ_DECL

/* ranorm (part3d_lib77.f:1324-1383): reset to the fixed seeds, or draw */
void oq_ranorm_reset(void);
double oq_ranorm(void);

#ifdef __cplusplus
}
#endif
#endif
