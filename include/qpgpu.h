/*
 * qpgpu.h -- C ABI of the B200 engine for QuickPIC's per-slice quasi-static path.
 *
 * The engine replaces, behind QuickPIC's own Fortran class API, the plasma
 * push and deposits (species2d / part2d), the 2D sine/cosine Poisson and B
 * solves (field2d / fpois2d / fft2d) and the beam 3D deposit (beam3d / part3d)
 * on one GPU.  A Fortran caller binds these entry points with iso_c_binding
 * (bind(C) interfaces, one per function); every argument is a plain
 * pointer, integer or float, and no call retains a host pointer after it
 * returns.  Each function below names the reference routine it replaces
 * (paths relative to QuickPIC-OpenSource/source).
 *
 * Conventions
 *  - Every call returns int: 0 = success; > 0 = recoverable capacity
 *    overflow (the required capacity is in qp_ctx_last_need(), the caller
 *    grows and retries, as part2d%pmove does, part2d_class.f03:429-579);
 *    < 0 = fatal error (message in qp_ctx_last_error()), which the Fortran
 *    shim maps to err%equit (perrors_class.f03:96-118).
 *  - Host arrays use the reference's column-major layouts:
 *      real-space field  rf(dim, nx+2, 2*ny+1)    (ufield2d_class.f03:129)
 *      k-space field     rf(dim, ny+1, nx+1)      (ufield2d_class.f03:198)
 *      tiled particles   ppart(8, nppmx, ntiles), kpic(ntiles)
 *                        (part2d_class.f03:170; tiles of 16 x 16 cells)
 *      beam particles    part(7, np)              (part3d_class.f03)
 *      3D field          rf(dim, nx+2, ny+1, nz+1) (ufield3d_class.f03:116)
 *  - A field keeps the reference's state flag (0 = real space, 1 = Fourier
 *    space, field2d_class.f03:24-26); operations check it like the reference
 *    and fail with "data is in ks" / "data is in rs" otherwise.
 *  - Calls on one context are stream-ordered on the context's CUDA stream.
 *    One host thread per context.
 */
#ifndef QPGPU_H
#define QPGPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qp_ctx qp_ctx;
typedef struct qp_field2d qp_field2d;
typedef struct qp_species qp_species;
typedef struct qp_beam qp_beam;
typedef struct qp_sim qp_sim;

/* ------------------------------------------------------------- context */

/* Grid description: the simulation.{indx,indy,indz,box} keys of the input
 * deck (simulation_class.f03:171-184).  4 <= indx, indy <= 11. */
typedef struct {
  int indx, indy, indz;
  double box[3][2]; /* box.x(1:2), box.y(1:2), box.z(1:2) in c/wp */
} qp_grid_desc;

/* Creates a context on CUDA device `device` (replaces the per-rank set-up of
 * simulation%new for one rank and one stage, simulation_class.f03:151-224). */
int qp_ctx_create(const qp_grid_desc* grid, int device, qp_ctx** out);
int qp_ctx_destroy(qp_ctx* ctx);
/* Blocks until all work queued on the context has finished. */
int qp_ctx_sync(qp_ctx* ctx);
/* Required capacity after a call returned > 0. */
long long qp_ctx_last_need(const qp_ctx* ctx);
/* Message of the last failed call (static storage of the context). */
const char* qp_ctx_last_error(const qp_ctx* ctx);
/* dex = dx (transverse cell size) and dxi = dz (slice width) in c/wp. */
int qp_ctx_spacing(const qp_ctx* ctx, float* dex, float* dxi);
/* Device-time stopwatch on the context's stream (no reference counterpart;
 * the reference logs wall-clock stamps, perrors_class.f03:120-134):
 * start records an event, stop records a second one, waits for it and
 * returns the elapsed milliseconds. */
int qp_ctx_timer_start(qp_ctx* ctx);
int qp_ctx_timer_stop(qp_ctx* ctx, double* ms);

/* -------------------------------------------------------------- field2d */

/* field2d%new (field2d_class.f03:82-138) with fftflag = .true.: dim = 1..3
 * components, state = 0 (real space) or 1 (Fourier space). */
int qp_field2d_create(qp_ctx* ctx, int dim, int state, qp_field2d** out);
int qp_field2d_destroy(qp_field2d* f);
int qp_field2d_state(const qp_field2d* f);
int qp_field2d_dim(const qp_field2d* f);
/* Copy real-space data rf(dim, nx+2, 2*ny+1) in / out; upload sets state 0. */
int qp_field2d_upload_rs(qp_field2d* f, const float* rf);
int qp_field2d_download_rs(qp_field2d* f, float* rf);
/* Copy Fourier-space data rf(dim, ny+1, nx+1) in / out; upload sets state 1. */
int qp_field2d_upload_ks(qp_field2d* f, const float* kf);
int qp_field2d_download_ks(qp_field2d* f, float* kf);

/* field2d%fftrk / %fftkr (field2d_class.f03:157-227): kind 1, 2, 3 select the
 * sine/cosine parities of fft2d%fsst / %fcct / %fs3t (fft2d_class.f03:121-413).
 * fftkr ends with the guard copy (ufield2d copyguard). */
int qp_field2d_fftrk(qp_field2d* f, int kind);
int qp_field2d_fftkr(qp_field2d* f, int kind);

/* Fourier-space solves; `src` must be in state 1, `dst` is left in state 1. */
int qp_field2d_pot(qp_field2d* src, qp_field2d* dst);    /* MPPOTPD2 via field2d%pot 295-316 */
int qp_field2d_smooth(qp_field2d* src, qp_field2d* dst); /* MPPSMOOTHD2 via field2d%smooth 341-362 */
int qp_field2d_elf(qp_field2d* src, qp_field2d* dst);    /* MPPOISD22 via field2d%elf 364-385 */
int qp_field2d_bf(qp_field2d* src, qp_field2d* dst);     /* MPPBBPOISD23 via field2d%bf 387-408 */
int qp_field2d_vpot(qp_field2d* src, qp_field2d* dst);   /* PBPOISD23 isign=1 via field2d%vpot 318-339 */
int qp_field2d_div(qp_field2d* src, qp_field2d* dst);    /* MPPDIVFD2 via field2d%div 229-249 */
int qp_field2d_grad(qp_field2d* src, qp_field2d* dst);   /* MPPGRADFD2 via field2d%grad 251-271 */
/* field2d%bfqp (field2d_class.f03:410-432 -> PBPOISD22N_QP): the transverse-B
 * corrector; dcu is modified in place, bxy (2 components) is read and written. */
int qp_field2d_bfqp(qp_field2d* cu, qp_field2d* dcu, qp_field2d* amu, qp_field2d* bxy, float c,
                    float dex);

/* Field algebra of field2d/ufield2d (ufield2d_class.f03:558-811), applied to
 * the real- or Fourier-space data according to the operands' state.
 * Component lists are 1-based like the Fortran (/1,2/) arrays. */
int qp_field2d_as(qp_field2d* f, float value);                    /* asc: rs = value, state 0 */
int qp_field2d_copy(qp_field2d* dst, qp_field2d* src);            /* asa */
int qp_field2d_add(qp_field2d* dst, qp_field2d* a1, qp_field2d* a2);       /* sum1 */
int qp_field2d_sub(qp_field2d* dst, qp_field2d* a1, qp_field2d* a2);       /* minus1 */
int qp_field2d_mult(qp_field2d* dst, qp_field2d* a1, float value);         /* multiply1 */
int qp_field2d_add_comp(qp_field2d* dst, qp_field2d* a1, qp_field2d* a2, const int* dim,
                        const int* dim1, const int* dim2, int n);          /* sum2 */
int qp_field2d_sub_comp(qp_field2d* dst, qp_field2d* a1, qp_field2d* a2, const int* dim,
                        const int* dim1, const int* dim2, int n);          /* minus2 */
int qp_field2d_mult_comp(qp_field2d* dst, qp_field2d* a1, const int* dim, const int* dim1,
                         const float* value, int n);                       /* multiply2 */
int qp_field2d_cg(qp_field2d* f); /* copyguard: row ny = row 0 (ufield2d_lib.f03:37-42) */
int qp_field2d_ag(qp_field2d* f); /* acopyguard: row 0 += row ny (ufield2d_lib.f03:90-97) */

/* ------------------------------------------------------------ species2d */

/* Plasma species (species(i) of the input, fdist2d_class.f03) with the keys
 * {profile, ppc, q, m, density}; xtras is part2d's buffer headroom (0.2 in
 * the reference, part2d_class.f03:62).  profile selects the loader:
 *   0  uniform                        (fdist2d_000, 212-316)
 *   10 elliptic hollow channel        (fdist2d_010, 318-523): the particles
 *      on or between the inner and the outer ellipse about center
 *   11 Gaussian ring                  (fdist2d_011, 525-711): charge weight
 *      exp(-(r - radius)^2 / (2 width^2))
 *   12 tabulated radial density f(r)  (fdist2d_012, 713-950), linear between
 *      the nr points (r[i], fr[i]), no particles outside [r[0], r[nr-1]]
 * Lengths (center, radii, width, r) are in the units of the box.  With ns > 0
 * the density is also scaled by the piecewise-linear longitudinal profile
 * (s[i], fs[i]) at the s given to qp_species_create / qp_species_renew
 * (longitudinal_profile = 'piecewise'); the arrays are read during those calls
 * only.  Unused fields may be zero. */
typedef struct {
  int profile;
  int ppc[2];
  float q, m, density;
  float xtras;
  float center[2];                        /* 10, 11, 12 */
  float inner_radius[2], outer_radius[2]; /* 10: x and y radii */
  float radius, width;                    /* 11 */
  int nr;                                 /* 12 */
  const float* r;
  const float* fr;
  int ns;                                 /* longitudinal piecewise density */
  const float* s;
  const float* fs;
} qp_species_desc;

/* species2d%new (species2d_class.f03:74-118): loads and bins the particles
 * (PPDBLKP2L, PPPMOVIN2L, PPPCHECK2L) and forms the ion background qn. */
int qp_species_create(qp_ctx* ctx, const qp_species_desc* d, float s, qp_species** out);
int qp_species_destroy(qp_species* sp);
/* species2d%renew (species2d_class.f03:138-164): fresh plasma for the next 3D step. */
int qp_species_renew(qp_species* sp, float s);
/* species2d%qdp (166-185): q_species = deposit (PPGPPOST2L) + guard add;
 * qe = q_species + qe; qe = qn + qe.  qe must be in state 0. */
int qp_species_qdp(qp_species* sp, qp_field2d* qe);
/* species2d%extpsi (256-272 -> WPGPSIPOST2L_QP). */
int qp_species_extpsi(qp_species* sp, qp_field2d* psi, float dex);
/* species2d%amjdp (187-218 -> PPGRDCJPPOST2L_QP): adds the species' current,
 * acceleration and momentum-flux densities to cu, dcu, amu (state 0). */
int qp_species_amjdp(qp_species* sp, qp_field2d* fxy, qp_field2d* bxyz, qp_field2d* psit,
                     qp_field2d* cu, qp_field2d* amu, qp_field2d* dcu, float dex);
/* species2d%push (220-237) = part2d%partpush (PPGRBPPUSHF23L_QP) + pmove. */
int qp_species_push(qp_species* sp, qp_field2d* fxy, qp_field2d* bxyz, qp_field2d* psit,
                    float dex);
/* The two halves of push: part2d%partpush (part2d_class.f03:315-358, in place,
 * no re-binning) and part2d%pmove (360-594, re-binning into tiles). */
int qp_species_partpush(qp_species* sp, qp_field2d* fxy, qp_field2d* bxyz, qp_field2d* psit,
                        float dex);
int qp_species_pmove(qp_species* sp);
/* The re-bin of qp_species_pmove for callers that cannot allocate device
 * memory while they run (a host code whose allocator owns the GPU's memory,
 * or a job held to a fixed memory budget).  This entry point has no
 * counterpart in the reference.  The caller owns both particle buffers, as
 * device pointers: part_in[8] / part_out[8] hold the eight component planes
 * of ntiles * cap floats (tile t in [t*cap, t*cap + count[t])), count_in /
 * count_out one int per tile; ntiles = (2^indx / 16) * (2^indy / 16).  The
 * output equals qp_species_pmove's on the same input.  The mover inbox and
 * the status live in one fixed device array of
 * QP_PMOVE_STATIC_SCRATCH_BYTES, which a GPU holds from the moment the
 * library first touches the array there until the process exits.  The CUDA
 * runtime loads the array's module lazily (the default since CUDA 12.2), so
 * that moment is qp_ctx_create on the device, or else the first
 * qp_pmove_static call on it: a caller that hands the GPU's memory to its own
 * allocator makes one of those calls first (or runs with
 * CUDA_MODULE_LOADING=EAGER, which places the array when the library loads).
 * After that no call allocates or frees device memory.  The
 * inbox takes min(16384, about 16 MiB / (40 B * ntiles)) movers per tile
 * (408 on a 512 x 512 grid, 100 on 1024 x 1024); grids that leave fewer than
 * QP_PMOVE_STATIC_MIN_INBOX are rejected, and so is a step that moves more
 * particles into one tile, or fills an output tile beyond cap_out: those
 * return -1 with the sizes in qp_ctx_last_error(NULL) and leave the input
 * untouched (there is no grow-and-retry).  Every call looks up the array's
 * device address on the current device (so it stays valid across a
 * cudaDeviceReset) and shares the one array: calls that overlap on the GPU
 * (other streams, other host threads) race.  The call runs on `stream`
 * (a cudaStream_t; NULL = the legacy default stream) and returns after it
 * has synchronised that stream, so it cannot be captured into a CUDA graph. */
#define QP_PMOVE_STATIC_SCRATCH_BYTES (16u << 20)
#define QP_PMOVE_STATIC_MIN_INBOX 64
int qp_pmove_static(int indx, int indy, const float* const* part_in, const int* count_in,
                    int cap_in, float* const* part_out, int* count_out, int cap_out,
                    void* stream);
/* species2d%cbq (399-418): q_species(1) += cu_species(3); smooth; store as
 * slice `pos` (1-based) of the species' 3D charge q3. */
int qp_species_cbq(qp_species* sp, int pos);
/* Particle data in the reference's tiled layout: ppart(8, nppmx_ld, ntiles),
 * kpic(ntiles).  nppmx_ld must be >= qp_species_nppmx(). */
int qp_species_ntiles(const qp_species* sp);
int qp_species_nppmx(const qp_species* sp);
long long qp_species_np(qp_species* sp);
int qp_species_download(qp_species* sp, float* ppart, int* kpic, int nppmx_ld);
int qp_species_upload(qp_species* sp, const float* ppart, const int* kpic, int nppmx_ld);
/* The ion background qn (real space, (1, nx+2, 2*ny+1)) and the species'
 * own charge density q after the last qdp/cbq. */
int qp_species_download_qn(qp_species* sp, float* rf);
int qp_species_download_q(qp_species* sp, float* rf);
/* Slice `pos` (1-based) of the species' 3D smoothed charge q3 as (nx+2, ny+1). */
int qp_species_download_q3(qp_species* sp, int pos, float* rf);

/* --------------------------------------------------------------- beam3d */

/* A beam3d and its fdist3d profile (fdist3d_class.f03), with the keys of
 * beam(i) in the input file.  Lengths are in the box's units, like the input.
 * Beams created on one context draw from one ranorm sequence, in creation
 * order, like the reference.
 *  profile 0 (fdist3d_000, 222-421): tri-Gaussian by PRVDIST32_RANDOM
 *    (part3d_lib77.f:411-552) with ranorm's fixed seeds (1324-1383): np,
 *    q, m, gamma, peak_density, quiet_start, center, sigma, sigma_v, npmax,
 *    centroid_x, centroid_y, static_density;
 *  profile 1 (fdist3d_001, 423-650): Gaussian in x, y and the piecewise
 *    profile fz(z) in z by PRVDIST32_RAN_PFL (part3d_lib77.f:193-410): as
 *    profile 0 without sigma[2], plus piecewise_z/fz (npiece points, z
 *    increasing).  Its longitudinal acceptance draws use RANDOM_NUMBER in the
 *    reference, a compiler runtime's generator; here SplitMix64 from `seed`;
 *  profile 2 (fdist3d_002, 652-821): Twiss beam by PRVDIST32_TWISS
 *    (part3d_lib77.f:1-191): np, q, m, gamma, peak_density, quiet_start,
 *    center, alpha, beta, emittance, sigma[2] = sigmaz, sigma_v[2] =
 *    sigma_vz, npmax;
 *  profile 3 (fdist3d_003, 823-974): np[0] particles read from the text
 *    file file_name, one "z x y pz px py q" per line, positions in
 *    micrometres (divided by c/omega_p = 5.32150254e9 / sqrt(n0) um, n0 the
 *    plasma density in cm^-3; z measured backwards from the box front; x, y
 *    from center), momenta and charge as they are; particles outside the box
 *    are left out;
 *  profile 100 (fdist3d_100, 976-1166): ring of radius r1 and width r2 about
 *    center, ppc particles per cell in the box range_x/y/z, weights q/|q|
 *    peak_density exp(-(dz^2 + (r - r1)^2) / (2 r2^2)) / (ppc product), pz =
 *    gamma.
 * static_density = 1 (beam(i).static, profiles 0 and 1) puts the profile's
 * analytic density on the 3D grid and loads no particles: no deposit, no
 * push.  frozen = 1 is beam(i).evolution = false: the push leaves the beam
 * where it is (push_beam3d, beam3d_class.f03:169-172). */
typedef struct {
  int profile;
  int np[3];
  float q, m, gamma, peak_density;
  int quiet_start;
  float center[3], sigma[3], sigma_v[3];
  long long npmax;
  float centroid_x[3], centroid_y[3];
  int static_density, frozen, npiece;
  int ppc[3];
  const float* piecewise_z;
  const float* piecewise_fz;
  const char* file_name;
  unsigned long long seed;
  float alpha[2], beta[2], emittance[2];
  float n0;
  float range_x[2], range_y[2], range_z[2];
  float r1, r2;
  float reserved[1];
} qp_beam_desc;

int qp_beam_create(qp_ctx* ctx, const qp_beam_desc* d, qp_beam** out);
int qp_beam_destroy(qp_beam* b);
long long qp_beam_np(const qp_beam* b);
/* beam3d%qdp (beam3d_class.f03:111-134 -> PGPOST32L): 3D charge deposit. */
int qp_beam_qdp(qp_beam* b);
/* beam3d%qdp(q, slice) (qdpcopy_beam3d 136-153): q(rs) += slice `slice`
 * (1-based) of the beam's 3D charge; q must be in state 0. */
int qp_beam_qdpcopy(qp_beam* b, qp_field2d* q, int slice);
int qp_beam_download(qp_beam* b, float* part /* (7, np) */);
/* Replace the beam's particles with part(7, np) from host memory (np at most
 * the particle count the beam was created with); the restart read of beam
 * particles, part3d%rrst (part3d_class.f03:315-331), without the HDF5 file. */
int qp_beam_upload(qp_beam* b, const float* part, long long np);
int qp_beam_download_q3d(qp_beam* b, float* rf /* (nx+2, ny+1, nz+1) */);
/* Beam restart (beam3d%wrst / %rrst, beam3d_class.f03:220-290 -> hdf5io
 * wpart / rpart, hdf5io_class.f03:1301-1422) in the reference's path layout
 * dir/RST/Beam-NNNN/RST-beamNNNN-RRRRRRRRRR_SSSSSSSS (beam from 1, rank,
 * dump step; simulation_class.f03:1261-1277) with the reference's content,
 * the particle count tp and part(7, tp).  The HDF5 container is not built
 * (no HDF5 library in this build): the file ends in .qprst and holds
 * "QPRST001", tp (int64) and part(7, tp) (float32, column-major).  read
 * replaces the beam's particles (tp must fit its capacity). */
int qp_beam_write_restart(qp_beam* b, const char* dir, int beam, int rank, int step);
int qp_beam_read_restart(qp_beam* b, const char* dir, int beam, int rank, int step);

/* ----------------------------------------------------- fused 3D step */

/* The whole 3D step of go_simulation (simulation_class.f03:611-764) for the
 * species and beams given, with all state on the GPU: beam deposit, the
 * per-slice loop (643-736) as one fixed sequence of kernel launches per
 * slice, and the species renew.
 * iter = fixed number of B predictor-corrector passes (simulation.iter);
 * tol = 0 runs exactly iter passes per slice, as the reference does; tol > 0
 * stops a slice's passes after the first one whose relative change of the
 * transverse B, |epw - epw_prev| / |epw| over all Fourier modes, is at most
 * tol, and runs at most iter passes (one plasma species only; the passes
 * actually run are returned in qp_step_stats.iterations);
 * store3d = 1 keeps the 3D fields bexyz, bbxyz and the species q3;
 * predict = 1 starts each slice's B passes from the linear extrapolation
 * 2 epw(j-1) - epw(j-2) of the transverse B of the two previous slices,
 * predict = 2 from the quadratic 3 epw(j-1) - 3 epw(j-2) + epw(j-3),
 * predict = 3 from the learned network (qp_sim_set_predictor), instead
 * of epw(j-1) (the reference's start); with tol > 0 the passes still run to
 * the same tolerance;
 * vpot = 1 (with store3d = 1, one species) also keeps the vector potential
 * vpot3d of every slice (simulation_class.f03:711-716: field2d%vpot of the
 * last pass's current, fftkr, times -dex), downloaded as "vpot";
 * use_graphs = 1 captures a slice's launches as a CUDA graph, once per
 * particle-buffer parity and number of passes enqueued, and replays it for
 * every slice with the same two (a replay first checks every pointer and
 * value the graph holds against the current ones and captures again when a
 * buffer was grown or replaced); the results are the same as with direct
 * launches; ignored while recording and in checked mode (QP_SYNC_CHECK=1);
 * dt = the 3D time step (simulation.dt): dt > 0 (with store3d = 1) ends the
 * step with beam3d%push of every beam with the stored bexyz, bbxyz
 * (simulation_class.f03:753-757), dt = 0 leaves the beams where they are. */
typedef struct {
  int iter;
  int store3d;
  int use_graphs;
  float dt;
  float tol;
  int vpot;
  int predict;
  int reserved[1];
} qp_sim_desc;

typedef struct {
  int slices;          /* slices advanced */
  int iterations;      /* predictor-corrector passes run */
  int regrowths;       /* particle-buffer growths (overflow recoveries) */
  int kernels;         /* kernel launches of the step */
  double gpu_ms;       /* device time of the step */
  int unconverged;     /* with tol > 0: slices whose iter-th pass still missed tol */
} qp_step_stats;

int qp_sim_create(qp_ctx* ctx, const qp_sim_desc* d, qp_species* const* species, int nspecies,
                  qp_beam* const* beams, int nbeams, qp_sim** out);
int qp_sim_destroy(qp_sim* sim);
/* beam3d%push (beam3d_class.f03:155-180 -> part3d%partpush, PGBPUSH32L_QP,
 * part3d_lib77.f:630-786) of beam b with the 3D fields bexyz, bbxyz of the
 * last step of `sim` (store3d = 1) and time step dt.  Conducting boundaries:
 * a particle that leaves [1, n-1) cells in x, y or z is dropped; the
 * remaining ones keep their order.  With one pipeline stage part3d%pmove
 * (PMOVE32) has nothing to move, so this is the whole beam3d%push. */
int qp_beam_push(qp_beam* b, qp_sim* sim, float dt);
/* One 3D step; `stats` may be NULL.  The species are renewed at the end.
 * Equal to qp_sim_begin3d, qp_sim_slices(nz), qp_sim_end3d. */
int qp_sim_step3d(qp_sim* sim, qp_step_stats* stats);
/* The 3D step in the three parts of go_simulation, so that a caller can stop
 * between slices (to read or restore the state a slice hands to the next):
 * qp_sim_begin3d = the start of the step (simulation_class.f03:611-641: beam
 * deposits, the fields handed to slice 1, the slice cursor at 1);
 * qp_sim_slices = the next n slices of the loop 643-736 (grow-and-retry
 * included; between calls the species' live particles are in the buffer
 * that qp_species_download/upload read and write);
 * qp_sim_end3d = the end of the step (741-764: beam push when dt > 0,
 * species renew), once all nz slices have run; `stats` as qp_sim_step3d
 * (gpu_ms spans begin3d to end3d, caller pauses included).
 * qp_sim_next_slice = the slice the next qp_sim_slices call starts with
 * (1-based), 0 when no step is in progress. */
int qp_sim_begin3d(qp_sim* sim);
int qp_sim_slices(qp_sim* sim, int n);
int qp_sim_end3d(qp_sim* sim, qp_step_stats* stats);
int qp_sim_next_slice(const qp_sim* sim);
/* use_graphs: slice graphs captured so far (each capture follows a new pass
 * count, parity or a replaced buffer; replays are not counted); -1 for NULL */
int qp_sim_graph_captures(const qp_sim* sim);
/* The Fourier-space fields a slice hands to the next, reference k-space
 * layout (dim, ny+1, nx+1): "epw" (transverse-B iterate, dim 2), "cu_k"
 * (current after the xi extrapolation, dim 3), and with predict > 0
 * "epw_prev" / "epw_prev2" (B_perp of earlier slices, dim 2).  With the
 * species particles they are the whole state between two slices; download
 * them with qp_sim_download_field. */
int qp_sim_upload_field(qp_sim* sim, const char* name, const float* in);
/* One plane (0-based index 0..nz) of a 3D array, reference layout: "bexyz",
 * "bbxyz", "vpot" (3, nx+2, ny+1) and "q3" (nx+2, ny+1) as stored by the
 * slice of that index (store3d = 1); "qb" (nx+2, ny+1) the beam charge
 * plane the slice of that index reads (ufield3d%copyadd in qdpcopy,
 * simulation_class.f03:645-650). */
int qp_sim_download_plane(qp_sim* sim, const char* name, int plane, float* out);
/* Fields of the last slice (real space or Fourier space, reference layout):
 * name = "psi", "fxy", "bxyz", "psit", "cu", "dcu", "amu" (rs) or
 * "epw", "cu_k", "epwb", "epw_prev", "epw_prev2" (ks). */
int qp_sim_download_field(qp_sim* sim, const char* name, float* out);
/* 3D fields (3, nx+2, ny+1, nz+1): "bexyz" or "bbxyz"; species 3D charge
 * (nx+2, ny+1, nz+1): "q3". */
int qp_sim_download_3d(qp_sim* sim, const char* name, float* out);
/* Component comp (1..3) of the 3D field bexyz on the axis node (nx/2, ny/2)
 * of every slice: out(nz+1), the on-axis wake lineout.  A 1D cut of the 3D
 * field that the reference's field slice diagnostics write to HDF5 files
 * (init_diag, simulation_class.f03:771-1100), read here without a file. */
int qp_sim_download_lineout(qp_sim* sim, int comp, float* out);
/* Per-kernel device times of one whole 3D step (the timing side of the
 * reference's per-step ELOG stamps, simulation_class.f03:614-645), with
 * `nslices` slices sampled at an even stride across the box (slice
 * 1 + floor((2i+1) nz / (2 nslices)), i = 0..nslices-1) and an event pair
 * around every launch of a sampled slice.  The step runs under the
 * simulation's own settings, tolerance included, and advances it by one 3D
 * step.  Kernel names are written newline-separated into `names`; ms[i],
 * count[i] and bytes[i] are the total milliseconds, launches and
 * algorithmic bytes (minimal FP32 traffic of the work done) of name i.
 * Under a tolerance, launches of passes after the one at which their slice
 * stopped return at once and are reported as "<kernel>:skipped" with no
 * bytes.  Returns the number of names (<= max), or < 0 on error. */
int qp_sim_profile(qp_sim* sim, int nslices, char* names, int names_len, double* ms, int* count,
                   double* bytes, int max);

/* -------------------------------------------- learned start of the B passes */

/* A convolutional network (5 layers of 3x3 convolutions, 32 channels, BF16
 * weights and activations, FP32 accumulation, on the BF16 tensor cores) that
 * predicts the start of each slice's B predictor-corrector passes: a
 * correction, per Fourier mode, of the quadratic extrapolation
 * 3 epw(j-1) - 3 epw(j-2) + epw(j-3), from epw(j-1) and the differences of
 * the three previous slices' B_perp, the current handed to the slice (cu_k)
 * and the mode coordinates, for the modes kx, ky < 128 (the window it is
 * trained on; the other modes start from the extrapolation alone).  It has no counterpart in the
 * reference, whose passes start from epw(j-1) (simulation_class.f03:676); it
 * replaces that start when qp_sim_desc.predict = 3, and the passes still run
 * to the tolerance.  Layer l: weights W[9][cin][cout] (tap = 3 dy + dx, dy and
 * dx the row and column offsets + 1) then bias[cout]; cin = 16 for layer 1
 * (9 input features, the rest zero), 32 otherwise; cout = 32, and 16 for
 * layer 5 (2 outputs used).  An untrained network (seeded He initialisation,
 * last layer zero) is the quadratic extrapolation. */
typedef struct qp_nn qp_nn;
typedef struct qp_nn_data qp_nn_data;
int qp_nn_create(int device, unsigned long long seed, qp_nn** out);
int qp_nn_destroy(qp_nn* nn);
int qp_nn_num_params(const qp_nn* nn);
int qp_nn_get_params(qp_nn* nn, float* out);
int qp_nn_set_params(qp_nn* nn, const float* in);
/* Forward of nb images in[nb][16][h][w] (w a multiple of 128) to
 * out[nb][2][h][w] (zero padding at the image edges). */
int qp_nn_forward(qp_nn* nn, const float* in, int nb, int h, int w, float* out);
/* Mean squared error of the 2 outputs against target[nb][2][h][w] and its
 * gradient with respect to every parameter (the parameter layout above). */
int qp_nn_loss_grad(qp_nn* nn, const float* in, const float* target, int nb, int h, int w,
                    double* loss, float* grad);
/* Training pairs recorded from simulations (qp_sim_record): for each slice,
 * the 128 x 128 low-mode crop of the network's 16 input channels, the target
 * (the converged epw minus the quadratic extrapolation, over the epw scale)
 * and the scale (the RMS of epw(j-1); 0 marks a pair left out of training:
 * no field to scale, or a target larger than the field itself). */
int qp_nn_data_create(int device, int capacity, qp_nn_data** out);
int qp_nn_data_destroy(qp_nn_data* t);
int qp_nn_data_count(const qp_nn_data* t);
int qp_nn_data_get(qp_nn_data* t, int i, float* img /* [16][128][128] */,
                   float* target /* [2][128][128] */, float* scale);
typedef struct {
  int steps;               /* Adam steps */
  int batch;               /* pairs per minibatch */
  float lr;                /* learning rate (x0.3 after half the steps, x0.1 after 3/4) */
  int reserved;
  unsigned long long seed; /* minibatch draws */
} qp_nn_train_desc;
typedef struct {
  double first_loss, last_loss; /* mean minibatch loss of the first and the last tenth */
  double gpu_ms;                /* device time of the training */
  int steps;
  int reserved;
} qp_nn_train_stats;
/* Trains the network on the GPU with its own forward, data-gradient and
 * weight-gradient kernels. */
int qp_nn_train(qp_nn* nn, qp_nn_data* t, const qp_nn_train_desc* d, qp_nn_train_stats* st);
/* Every following slice of `sim` records one training pair into t until it
 * is full (NULL stops).  Needs nx, ny >= 128 and ny a multiple of 128. */
int qp_sim_record(qp_sim* sim, qp_nn_data* t);
/* The network that starts the passes of a simulation created with
 * predict = 3 (ny a multiple of 128).  The simulation keeps a pointer. */
int qp_sim_set_predictor(qp_sim* sim, qp_nn* nn);

/* ------------------------------------------------------ batched scan */

/* A parameter scan over independent instances (a density, current or beam
 * size scan): n simulations, each on its own context, advanced by `steps` 3D
 * steps each.  `workers` host threads take instances from a queue, largest
 * first, and step them on their own streams, so the instances' kernels
 * overlap on the GPU; workers <= 0 (or > n) runs one per instance, 1 steps
 * the instances one after another.  The scan is timed on the device, from a
 * start event every instance stream waits on to the last instance's end. */
typedef struct {
  int steps;
  int workers;
} qp_scan_desc;

typedef struct {
  double gpu_ms;              /* device time of the whole scan */
  long long particle_slices;  /* sum over instances and steps of Np * nz */
  int workers;                /* worker threads used */
  int failed;                 /* instances whose step returned an error */
} qp_scan_stats;

int qp_scan_run(qp_sim* const* sims, int n, const qp_scan_desc* d, qp_scan_stats* out);
/* Autotuner of the scan's concurrency: times probe_steps steps of every
 * instance with 1, 2, 4, ... and n workers and returns the count with the
 * highest particle-slices per second (and that rate).  The probes advance
 * the instances by probe_steps times the number of candidates. */
int qp_scan_tune(qp_sim* const* sims, int n, int probe_steps, int* best_workers,
                 double* best_rate);

#ifdef __cplusplus
}
#endif
#endif
