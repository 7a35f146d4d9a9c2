// qp_api.cu -- implementation of the C ABI declared in include/qpgpu.h.
//
// Handles own their device memory.  Field handles carry the reference's
// real/Fourier state flag and check it the way field2d does.  The species
// handle owns two tile-binned particle buffers (the push reads one and writes
// the other) and the mover inbox; overflow of either is detected on the
// device, and the call grows the buffers by (1 + xtras) and retries, as
// part2d%pmove does (part2d_class.f03:429-579).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/qpgpu.h"
#include "qp_beam.cuh"
#include "qp_fft.cuh"
#include "qp_loader.h"
#include "qp_misc.cuh"
#include "qp_nn.cuh"
#include "qp_part.cuh"
#include "qp_slice.cuh"

using namespace qp;

static thread_local std::string g_last_error;

void qp_set_error(const char* file, int line, const char* msg) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s:%d: %s", file, line, msg);
  g_last_error = buf;
}

#define CK(call)                                                                 \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) return fail(ctx, __LINE__, cudaGetErrorString(e_));   \
  } while (0)

struct qp_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  GridDims g{};
  int indz = 0, nz = 0;
  double box[3][2];
  float dex = 0, dy = 0, dxi = 0;
  LineTablesHost tx, ty;
  float* ffre = nullptr;
  float* ffim = nullptr;
  KCoef kc{};
  TileGeom tg{};
  DevStatus* st = nullptr;  // device
  std::string err;
  long long need = 0;
  Ranorm rng;
  float* staging = nullptr;  // device scratch for layout conversion
  size_t staging_bytes = 0;
  cudaEvent_t t0 = nullptr, t1 = nullptr;  // qp_ctx_timer_start / _stop
};

static int fail(qp_ctx* ctx, int line, const std::string& msg) {
  char buf[64];
  snprintf(buf, sizeof(buf), "qp_api.cu:%d: ", line);
  if (ctx) ctx->err = std::string(buf) + msg;
  g_last_error = std::string(buf) + msg;
  return -1;
}

struct qp_field2d {
  qp_ctx* ctx;
  int dim;
  int state;
  float* rs[3];
  float* ks[3];
};

struct qp_species {
  qp_ctx* ctx;
  qp_species_desc d;
  float qbm, dt;
  PartBuf A{}, B{}, P0{};  // live, spare, pristine (renew)
  Inbox ib{};
  int nppmx0 = 0;          // reference-equivalent capacity
  long long np = 0;
  qp_field2d* q = nullptr;     // species charge (rs + ks, used by cbq)
  qp_field2d* qn = nullptr;    // ion background
  qp_field2d* cusp = nullptr;  // per-species accumulators of the class API
  qp_field2d* dcusp = nullptr;
  qp_field2d* amusp = nullptr;
  float* q3 = nullptr;         // (nz+1) real planes
  float* q3_first = nullptr;   // slice-1 plane after renew (pristine)
  int regrowths = 0;
  PlasmaProfile prof;          // the loader's profile, lengths in cells
};

struct qp_beam {
  qp_ctx* ctx;
  BeamBuf b{};
  float* q3d = nullptr;  // (nz+1) real planes
  float qbm = 0.f;       // charge-to-mass ratio q/m of the push
  long long cap = 0;     // particle slots of each plane (the count at creation)
  int* keep = nullptr;   // per-particle flags of the push (allocated by the first push)
  bool is_static = false;  // analytic density on the grid, no particles
  bool frozen = false;     // evolution = false: the push leaves it alone
};

// ------------------------------------------------------------ helpers
static int sync_status(qp_ctx* ctx, DevStatus* out) {
  CK(cudaMemcpyAsync(out, ctx->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

static int clear_status(qp_ctx* ctx, int keep_cursor) {
  DevStatus s{};
  if (keep_cursor) {  // a recovery within a step: keep its cursor and pass count
    DevStatus cur;
    if (sync_status(ctx, &cur)) return -1;
    s.cursor = cur.cursor;
    s.passes = cur.passes;
    s.unconverged = cur.unconverged;
  }
  CK(cudaMemcpyAsync(ctx->st, &s, sizeof(DevStatus), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

static int ensure_staging(qp_ctx* ctx, size_t bytes) {
  if (ctx->staging_bytes >= bytes) return 0;
  if (ctx->staging) cudaFree(ctx->staging);
  ctx->staging = nullptr;
  ctx->staging_bytes = 0;
  CK(cudaMalloc(&ctx->staging, bytes));
  ctx->staging_bytes = bytes;
  return 0;
}

// Zero freshly allocated device memory before anything else can touch it.
// The contexts' streams are non-blocking, so a memset left pending on the
// legacy default stream could land after later work on a context stream.
static int zero_now(void* p, size_t bytes) {
  if (cudaMemset(p, 0, bytes) != cudaSuccess) return -1;
  return cudaStreamSynchronize(cudaStreamLegacy) == cudaSuccess ? 0 : -1;
}

static float* dalloc(size_t n, bool zero = true) {
  float* p = nullptr;
  if (cudaMalloc(&p, sizeof(float) * std::max<size_t>(n, 1)) != cudaSuccess) return nullptr;
  if (zero && zero_now(p, sizeof(float) * std::max<size_t>(n, 1))) {
    cudaFree(p);
    return nullptr;
  }
  return p;
}

// --------------------------------------------------------------- context
extern "C" int qp_ctx_create(const qp_grid_desc* grid, int device, qp_ctx** out) {
  qp_ctx* ctx = nullptr;
  if (!grid || !out) return fail(nullptr, __LINE__, "null argument");
  if (grid->indx < 4 || grid->indy < 4 || grid->indx > QP_MAX_IND || grid->indy > QP_MAX_IND ||
      grid->indz < 1 || grid->indz > 14)
    return fail(nullptr, __LINE__, "grid exponents out of range (4 <= indx, indy <= 11)");
  ctx = new qp_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete ctx;
    return fail(nullptr, __LINE__, "cudaSetDevice failed");
  }
  ctx->g = make_dims(grid->indx, grid->indy);
  ctx->indz = grid->indz;
  ctx->nz = 1 << grid->indz;
  std::memcpy(ctx->box, grid->box, sizeof(ctx->box));
  ctx->dex = (float)((float)(grid->box[0][1]) - (float)(grid->box[0][0])) / (float)ctx->g.nx;
  ctx->dy = (float)((float)(grid->box[1][1]) - (float)(grid->box[1][0])) / (float)ctx->g.ny;
  ctx->dxi = (float)((float)(grid->box[2][1]) - (float)(grid->box[2][0])) / (float)ctx->nz;
  CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  if (fft_kernels_init() || part_kernels_init() || slice_kernels_init())
    return fail(ctx, __LINE__, "kernel init failed");
  // the fixed scratch array of qp_pmove_static is placed on the device with
  // the context, before a caller's own allocator can take the rest
  if (pmove_static_reserve()) return fail(ctx, __LINE__, "static scratch set-up failed");
  if (line_tables_build(&ctx->tx, grid->indx)) return fail(ctx, __LINE__, "table alloc failed");
  if (grid->indy == grid->indx)
    ctx->ty = ctx->tx;
  else if (line_tables_build(&ctx->ty, grid->indy))
    return fail(ctx, __LINE__, "table alloc failed");
  std::vector<float> re, im;
  form_factor(ctx->g.nx, ctx->g.ny, 0.912871f, 0.912871f, 1.0f, re, im);
  ctx->ffre = dalloc(re.size(), false);
  ctx->ffim = dalloc(im.size(), false);
  if (!ctx->ffre || !ctx->ffim) return fail(ctx, __LINE__, "out of device memory");
  CK(cudaMemcpy(ctx->ffre, re.data(), sizeof(float) * re.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->ffim, im.data(), sizeof(float) * im.size(), cudaMemcpyHostToDevice));
  ctx->kc.nx = ctx->g.nx;
  ctx->kc.ny = ctx->g.ny;
  ctx->kc.dnx = 6.28318530717959f / (float)(ctx->g.nx + ctx->g.nx);
  ctx->kc.dny = 6.28318530717959f / (float)(ctx->g.ny + ctx->g.ny);
  ctx->kc.ffre = ctx->ffre;
  ctx->kc.ffim = ctx->ffim;
  ctx->tg.nx = ctx->g.nx;
  ctx->tg.ny = ctx->g.ny;
  ctx->tg.mx1 = (ctx->g.nx - 1) / TILE + 1;
  ctx->tg.myp1 = (ctx->g.ny - 1) / TILE + 1;
  ctx->tg.ntiles = ctx->tg.mx1 * ctx->tg.myp1;
  ctx->tg.rp = ctx->g.rp;
  CK(cudaMalloc(&ctx->st, sizeof(DevStatus)));
  if (zero_now(ctx->st, sizeof(DevStatus))) return fail(ctx, __LINE__, "status set-up failed");
  CK(cudaDeviceSynchronize());
  *out = ctx;
  return 0;
}

extern "C" int qp_ctx_destroy(qp_ctx* ctx) {
  if (!ctx) return 0;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->ty.base != ctx->tx.base) line_tables_free(&ctx->ty);
  line_tables_free(&ctx->tx);
  cudaFree(ctx->ffre);
  cudaFree(ctx->ffim);
  cudaFree(ctx->st);
  if (ctx->staging) cudaFree(ctx->staging);
  if (ctx->t0) cudaEventDestroy(ctx->t0);
  if (ctx->t1) cudaEventDestroy(ctx->t1);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return 0;
}

extern "C" int qp_ctx_sync(qp_ctx* ctx) {
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

extern "C" long long qp_ctx_last_need(const qp_ctx* ctx) { return ctx ? ctx->need : 0; }

extern "C" const char* qp_ctx_last_error(const qp_ctx* ctx) {
  if (ctx && !ctx->err.empty()) return ctx->err.c_str();
  return g_last_error.c_str();
}

extern "C" int qp_ctx_spacing(const qp_ctx* ctx, float* dex, float* dxi) {
  if (dex) *dex = ctx->dex;
  if (dxi) *dxi = ctx->dxi;
  return 0;
}

// --------------------------------------------------------------- field2d
static qp_field2d* field_new(qp_ctx* ctx, int dim, int state) {
  qp_field2d* f = new qp_field2d();
  f->ctx = ctx;
  f->dim = dim;
  f->state = state;
  for (int c = 0; c < 3; ++c) {
    f->rs[c] = nullptr;
    f->ks[c] = nullptr;
  }
  for (int c = 0; c < dim; ++c) {
    f->rs[c] = dalloc(ctx->g.rplane);
    f->ks[c] = dalloc(ctx->g.kplane);
    if (!f->rs[c] || !f->ks[c]) return nullptr;
  }
  return f;
}

static void field_free(qp_field2d* f) {
  if (!f) return;
  for (int c = 0; c < 3; ++c) {
    if (f->rs[c]) cudaFree(f->rs[c]);
    if (f->ks[c]) cudaFree(f->ks[c]);
  }
  delete f;
}

extern "C" int qp_field2d_create(qp_ctx* ctx, int dim, int state, qp_field2d** out) {
  if (!ctx || dim < 1 || dim > 3 || (state != 0 && state != 1))
    return fail(ctx, __LINE__, "invalid field dimension or state");
  qp_field2d* f = field_new(ctx, dim, state);
  if (!f) return fail(ctx, __LINE__, "out of device memory");
  *out = f;
  return 0;
}

extern "C" int qp_field2d_destroy(qp_field2d* f) {
  if (f) {
    cudaStreamSynchronize(f->ctx->stream);
    field_free(f);
  }
  return 0;
}

extern "C" int qp_field2d_state(const qp_field2d* f) { return f->state; }
extern "C" int qp_field2d_dim(const qp_field2d* f) { return f->dim; }

extern "C" int qp_field2d_upload_rs(qp_field2d* f, const float* rf) {
  qp_ctx* ctx = f->ctx;
  const GridDims& g = ctx->g;
  const int nxv = g.nx + 2;
  std::vector<float> h((size_t)f->dim * g.rplane, 0.f);
  for (int c = 0; c < f->dim; ++c)
    for (int y = 0; y <= g.ny; ++y)
      for (int x = 0; x < nxv; ++x)
        h[(size_t)c * g.rplane + (size_t)y * g.rp + x] =
            rf[(size_t)c + (size_t)f->dim * ((size_t)x + (size_t)nxv * y)];
  for (int c = 0; c < f->dim; ++c)
    CK(cudaMemcpyAsync(f->rs[c], &h[(size_t)c * g.rplane], sizeof(float) * g.rplane,
                       cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  f->state = 0;
  return 0;
}

extern "C" int qp_field2d_download_rs(qp_field2d* f, float* rf) {
  qp_ctx* ctx = f->ctx;
  const GridDims& g = ctx->g;
  const int nxv = g.nx + 2, nypmx = 2 * g.ny + 1;
  std::vector<float> h((size_t)f->dim * g.rplane);
  for (int c = 0; c < f->dim; ++c)
    CK(cudaMemcpyAsync(&h[(size_t)c * g.rplane], f->rs[c], sizeof(float) * g.rplane,
                       cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  std::memset(rf, 0, sizeof(float) * (size_t)f->dim * nxv * nypmx);
  for (int c = 0; c < f->dim; ++c)
    for (int y = 0; y <= g.ny; ++y)
      for (int x = 0; x < nxv; ++x)
        rf[(size_t)c + (size_t)f->dim * ((size_t)x + (size_t)nxv * y)] =
            h[(size_t)c * g.rplane + (size_t)y * g.rp + x];
  return 0;
}

extern "C" int qp_field2d_upload_ks(qp_field2d* f, const float* kf) {
  qp_ctx* ctx = f->ctx;
  const GridDims& g = ctx->g;
  std::vector<float> h((size_t)f->dim * g.kplane, 0.f);
  for (int c = 0; c < f->dim; ++c)
    for (int kx = 0; kx <= g.nx; ++kx)
      for (int ky = 0; ky <= g.ny; ++ky)
        h[(size_t)c * g.kplane + (size_t)kx * g.kp + ky] =
            kf[(size_t)c + (size_t)f->dim * ((size_t)ky + (size_t)(g.ny + 1) * kx)];
  for (int c = 0; c < f->dim; ++c)
    CK(cudaMemcpyAsync(f->ks[c], &h[(size_t)c * g.kplane], sizeof(float) * g.kplane,
                       cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  f->state = 1;
  return 0;
}

extern "C" int qp_field2d_download_ks(qp_field2d* f, float* kf) {
  qp_ctx* ctx = f->ctx;
  const GridDims& g = ctx->g;
  std::vector<float> h((size_t)f->dim * g.kplane);
  for (int c = 0; c < f->dim; ++c)
    CK(cudaMemcpyAsync(&h[(size_t)c * g.kplane], f->ks[c], sizeof(float) * g.kplane,
                       cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int c = 0; c < f->dim; ++c)
    for (int kx = 0; kx <= g.nx; ++kx)
      for (int ky = 0; ky <= g.ny; ++ky)
        kf[(size_t)c + (size_t)f->dim * ((size_t)ky + (size_t)(g.ny + 1) * kx)] =
            h[(size_t)c * g.kplane + (size_t)kx * g.kp + ky];
  return 0;
}

// sine (0) / cosine (1) parity of component c along x (axis 0) or y (axis 1)
// for the transform kinds of field2d%fftrk/fftkr (see kind_parity in the
// fft2d_class.f03:121-413 dispatch): kind 1 = fsst, 2 = fcct, 3 = fs3t.
static bool parity_of(int dim, int kind, int c, int* px, int* py) {
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

static int fft_rk(qp_ctx* ctx, float* const* rs, float* const* ks, const float* const* add,
                  int dim, const int* px, const int* py) {
  const GridDims& g = ctx->g;
  XJob xj{};
  YJob yj{};
  xj.ncomp = yj.ncomp = dim;
  const float norm = 0.25f / ((float)g.nx * (float)g.ny);
  for (int c = 0; c < dim; ++c) {
    xj.c[c] = XComp{rs[c], add ? add[c] : nullptr, ks[c], 1.0f, px[c], 0};
    yj.c[c] = YComp{ks[c], norm, py[c]};
  }
  launch_xfwd(xj, g, ctx->tx.t, ctx->st, ctx->stream);
  launch_ycol(yj, g, ctx->ty.t, ctx->st, ctx->stream);
  return 0;
}

static int fft_kr(qp_ctx* ctx, float* const* rs, float* const* ks, int dim, const int* px,
                  const int* py) {
  const GridDims& g = ctx->g;
  XJob xj{};
  YJob yj{};
  xj.ncomp = yj.ncomp = dim;
  for (int c = 0; c < dim; ++c) {
    yj.c[c] = YComp{ks[c], 1.0f, py[c]};
    xj.c[c] = XComp{ks[c], nullptr, rs[c], 1.0f, px[c], 0};
  }
  launch_ycol(yj, g, ctx->ty.t, ctx->st, ctx->stream);
  launch_xinv(xj, g, ctx->tx.t, ctx->st, ctx->stream);
  return 0;
}

extern "C" int qp_field2d_fftrk(qp_field2d* f, int kind) {
  qp_ctx* ctx = f->ctx;
  if (f->state != 0) return fail(ctx, __LINE__, "fftrk_field2d: data is in ks");
  int px[3], py[3];
  for (int c = 0; c < f->dim; ++c)
    if (!parity_of(f->dim, kind, c, &px[c], &py[c]))
      return fail(ctx, __LINE__, "fftrk_field2d: wrong fft kind");
  fft_rk(ctx, f->rs, f->ks, nullptr, f->dim, px, py);
  CK(cudaGetLastError());
  f->state = 1;
  return 0;
}

extern "C" int qp_field2d_fftkr(qp_field2d* f, int kind) {
  qp_ctx* ctx = f->ctx;
  if (f->state != 1) return fail(ctx, __LINE__, "fftkr_field2d: data is in rs");
  int px[3], py[3];
  for (int c = 0; c < f->dim; ++c)
    if (!parity_of(f->dim, kind, c, &px[c], &py[c]))
      return fail(ctx, __LINE__, "fftkr_field2d: wrong fft kind");
  fft_kr(ctx, f->rs, f->ks, f->dim, px, py);
  CK(cudaGetLastError());
  f->state = 0;
  return 0;
}

static int kop(qp_ctx* ctx, int op, qp_field2d* src, qp_field2d* dst, int need_src,
               int need_dst) {
  if (src->state != 1) return fail(ctx, __LINE__, "data is in rs");
  if (src->dim < need_src || dst->dim < need_dst)
    return fail(ctx, __LINE__, "invalid vector size");
  float* in[8] = {src->ks[0], src->ks[1], src->ks[2]};
  float* out[8] = {dst->ks[0], dst->ks[1], dst->ks[2]};
  launch_kpoint(op, ctx->g, ctx->kc, in, out, 0.f, 1.f, ctx->st, ctx->stream);
  CK(cudaGetLastError());
  dst->state = 1;
  return 0;
}

extern "C" int qp_field2d_pot(qp_field2d* s, qp_field2d* d) { return kop(s->ctx, KOP_POT, s, d, 1, 1); }
extern "C" int qp_field2d_smooth(qp_field2d* s, qp_field2d* d) { return kop(s->ctx, KOP_SMOOTH, s, d, 1, 1); }
extern "C" int qp_field2d_elf(qp_field2d* s, qp_field2d* d) { return kop(s->ctx, KOP_ELF, s, d, 1, 2); }
extern "C" int qp_field2d_bf(qp_field2d* s, qp_field2d* d) {
  if (s->dim != 3) return fail(s->ctx, __LINE__, "jpbpoisd23: invalid cu vector size");
  return kop(s->ctx, KOP_BF, s, d, 3, 3);
}
extern "C" int qp_field2d_vpot(qp_field2d* s, qp_field2d* d) {
  if (s->dim != 3 || d->dim != 3) return fail(s->ctx, __LINE__, "ivpotd2: invalid vector size");
  return kop(s->ctx, KOP_VPOT, s, d, 3, 3);
}
extern "C" int qp_field2d_div(qp_field2d* s, qp_field2d* d) { return kop(s->ctx, KOP_DIV, s, d, 2, 1); }
extern "C" int qp_field2d_grad(qp_field2d* s, qp_field2d* d) { return kop(s->ctx, KOP_GRAD, s, d, 1, 2); }

extern "C" int qp_field2d_bfqp(qp_field2d* cu, qp_field2d* dcu, qp_field2d* amu, qp_field2d* bxy,
                               float c, float dex) {
  qp_ctx* ctx = cu->ctx;
  if (cu->state != 1 || dcu->state != 1 || amu->state != 1)
    return fail(ctx, __LINE__, "bfield_qp_field2d: data is in rs");
  if (cu->dim != 3 || dcu->dim != 2 || amu->dim != 3 || bxy->dim != 2)
    return fail(ctx, __LINE__, "bfield_qp_field2d: invalid vector size");
  float* in[8] = {cu->ks[0], cu->ks[1], cu->ks[2], dcu->ks[0], dcu->ks[1],
                  amu->ks[0], amu->ks[1], amu->ks[2]};
  float* out[8] = {bxy->ks[0], bxy->ks[1]};
  launch_kpoint(KOP_BFQP, ctx->g, ctx->kc, in, out, c, dex, ctx->st, ctx->stream);
  CK(cudaGetLastError());
  bxy->state = 1;
  return 0;
}

static float* const* planes(qp_field2d* f, int state) { return state == 0 ? f->rs : f->ks; }
static long long plane_n(qp_ctx* ctx, int state) {
  return state == 0 ? ctx->g.rplane : ctx->g.kplane;
}

extern "C" int qp_field2d_as(qp_field2d* f, float value) {
  qp_ctx* ctx = f->ctx;
  for (int c = 0; c < f->dim; ++c)
    launch_lin(ctx->g.rplane, f->rs[c], nullptr, nullptr, value, LIN_FILL, ctx->st, ctx->stream);
  f->state = 0;
  CK(cudaGetLastError());
  return 0;
}

extern "C" int qp_field2d_copy(qp_field2d* d, qp_field2d* s) {
  qp_ctx* ctx = d->ctx;
  const int st = s->state;
  for (int c = 0; c < std::min(d->dim, s->dim); ++c)
    launch_lin(plane_n(ctx, st), planes(d, st)[c], planes(s, st)[c], nullptr, 0.f, LIN_COPY,
               ctx->st, ctx->stream);
  d->state = st;
  CK(cudaGetLastError());
  return 0;
}

static int binop(qp_field2d* d, qp_field2d* a, qp_field2d* b, int op) {
  qp_ctx* ctx = d->ctx;
  if (a->state != b->state) return fail(ctx, __LINE__, "states are different");
  const int st = a->state;
  for (int c = 0; c < d->dim; ++c)
    launch_lin(plane_n(ctx, st), planes(d, st)[c], planes(a, st)[c], planes(b, st)[c], 0.f, op,
               ctx->st, ctx->stream);
  d->state = st;
  CK(cudaGetLastError());
  return 0;
}

extern "C" int qp_field2d_add(qp_field2d* d, qp_field2d* a, qp_field2d* b) { return binop(d, a, b, LIN_ADD); }
extern "C" int qp_field2d_sub(qp_field2d* d, qp_field2d* a, qp_field2d* b) { return binop(d, a, b, LIN_SUB); }

extern "C" int qp_field2d_mult(qp_field2d* d, qp_field2d* a, float value) {
  qp_ctx* ctx = d->ctx;
  const int st = a->state;
  for (int c = 0; c < d->dim; ++c)
    launch_lin(plane_n(ctx, st), planes(d, st)[c], planes(a, st)[c], nullptr, value, LIN_SCALE,
               ctx->st, ctx->stream);
  d->state = st;
  CK(cudaGetLastError());
  return 0;
}

static int binop_comp(qp_field2d* d, qp_field2d* a, qp_field2d* b, const int* dim,
                      const int* dim1, const int* dim2, int n, int op) {
  qp_ctx* ctx = d->ctx;
  if (a->state != b->state) return fail(ctx, __LINE__, "states are different");
  const int st = a->state;
  for (int i = 0; i < n; ++i) {
    if (dim[i] < 1 || dim[i] > d->dim || dim1[i] < 1 || dim1[i] > a->dim || dim2[i] < 1 ||
        dim2[i] > b->dim)
      return fail(ctx, __LINE__, "component index out of range");
    launch_lin(plane_n(ctx, st), planes(d, st)[dim[i] - 1], planes(a, st)[dim1[i] - 1],
               planes(b, st)[dim2[i] - 1], 0.f, op, ctx->st, ctx->stream);
  }
  d->state = st;
  CK(cudaGetLastError());
  return 0;
}

extern "C" int qp_field2d_add_comp(qp_field2d* d, qp_field2d* a, qp_field2d* b, const int* dim,
                                   const int* dim1, const int* dim2, int n) {
  return binop_comp(d, a, b, dim, dim1, dim2, n, LIN_ADD);
}
extern "C" int qp_field2d_sub_comp(qp_field2d* d, qp_field2d* a, qp_field2d* b, const int* dim,
                                   const int* dim1, const int* dim2, int n) {
  return binop_comp(d, a, b, dim, dim1, dim2, n, LIN_SUB);
}

extern "C" int qp_field2d_mult_comp(qp_field2d* d, qp_field2d* a, const int* dim, const int* dim1,
                                    const float* value, int n) {
  qp_ctx* ctx = d->ctx;
  const int st = a->state;
  // multiply2 reads a1 and writes this element by element; when this == a1 and
  // the component lists overlap, compute into scratch first so that every
  // product uses the input value (the reference's loop order gives the same
  // result for the lists QuickPIC uses).
  for (int i = 0; i < n; ++i) {
    if (dim[i] < 1 || dim[i] > d->dim || dim1[i] < 1 || dim1[i] > a->dim)
      return fail(ctx, __LINE__, "component index out of range");
    launch_lin(plane_n(ctx, st), planes(d, st)[dim[i] - 1], planes(a, st)[dim1[i] - 1], nullptr,
               value[i], LIN_SCALE, ctx->st, ctx->stream);
  }
  d->state = st;
  CK(cudaGetLastError());
  return 0;
}

extern "C" int qp_field2d_cg(qp_field2d* f) {
  qp_ctx* ctx = f->ctx;
  if (f->state != 0) return fail(ctx, __LINE__, "copyguard_field2d: data is in ks");
  for (int c = 0; c < f->dim; ++c) launch_guard_copy(f->rs[c], ctx->g, ctx->st, ctx->stream);
  CK(cudaGetLastError());
  return 0;
}

extern "C" int qp_field2d_ag(qp_field2d* f) {
  qp_ctx* ctx = f->ctx;
  if (f->state != 0) return fail(ctx, __LINE__, "acopyguard_field2d: data is in ks");
  for (int c = 0; c < f->dim; ++c) launch_guard_add(f->rs[c], ctx->g, ctx->st, ctx->stream);
  CK(cudaGetLastError());
  return 0;
}

// --------------------------------------------------------------- species
// Tile capacities are rounded up to a multiple of 4 so every tile segment
// starts on a 16-byte boundary (the particle kernels use float4 accesses).
static int part_alloc(PartBuf* P, int ntiles, int cap) {
  cap = (cap + 3) & ~3;
  P->cap = cap;
  for (int c = 0; c < NCOMP; ++c) {
    P->c[c] = dalloc((size_t)ntiles * cap);
    if (!P->c[c]) return -1;
  }
  if (cudaMalloc(&P->count, sizeof(int) * ntiles) != cudaSuccess) return -1;
  return zero_now(P->count, sizeof(int) * ntiles);
}

static void part_free(PartBuf* P) {
  for (int c = 0; c < NCOMP; ++c)
    if (P->c[c]) cudaFree(P->c[c]);
  if (P->count) cudaFree(P->count);
  *P = PartBuf{};
}

static int inbox_alloc(Inbox* ib, int ntiles, int cap) {
  ib->cap = cap;
  for (int c = 0; c < NCOMP; ++c) {
    ib->c[c] = dalloc((size_t)ntiles * cap, false);
    if (!ib->c[c]) return -1;
  }
  if (cudaMalloc(&ib->key, sizeof(unsigned long long) * (size_t)ntiles * cap) != cudaSuccess)
    return -1;
  if (cudaMalloc(&ib->count, sizeof(int) * ntiles) != cudaSuccess) return -1;
  return zero_now(ib->count, sizeof(int) * ntiles);
}

static void inbox_free(Inbox* ib) {
  for (int c = 0; c < NCOMP; ++c)
    if (ib->c[c]) cudaFree(ib->c[c]);
  if (ib->key) cudaFree(ib->key);
  if (ib->count) cudaFree(ib->count);
  *ib = Inbox{};
}

// copy the tiles of `src` into `dst` (which may have a larger capacity)
static int part_copy(qp_ctx* ctx, PartBuf& dst, const PartBuf& src) {
  const int nt = ctx->tg.ntiles;
  for (int c = 0; c < NCOMP; ++c)
    CK(cudaMemcpy2DAsync(dst.c[c], sizeof(float) * dst.cap, src.c[c], sizeof(float) * src.cap,
                         sizeof(float) * std::min(src.cap, dst.cap), nt, cudaMemcpyDeviceToDevice,
                         ctx->stream));
  CK(cudaMemcpyAsync(dst.count, src.count, sizeof(int) * nt, cudaMemcpyDeviceToDevice,
                     ctx->stream));
  return 0;
}

// species q / qn / q3 bookkeeping after (re)loading: qn = -(deposit + guard
// add); q = qn; smoothed q -> q3 slice 1 (species2d_class.f03:104-115).
static int species_background(qp_species* sp) {
  qp_ctx* ctx = sp->ctx;
  const GridDims& g = ctx->g;
  launch_lin(g.rplane, sp->qn->rs[0], nullptr, nullptr, 0.f, LIN_FILL, ctx->st, ctx->stream);
  launch_deposit_rho(sp->A, ctx->tg, sp->qn->rs[0], ctx->st, ctx->stream);
  launch_lin(g.rplane, sp->q->rs[0], sp->qn->rs[0], nullptr, 0.f, LIN_COPY, ctx->st, ctx->stream);
  sp->q->state = 0;
  int px = 0, py = 0;
  fft_rk(ctx, sp->q->rs, sp->q->ks, nullptr, 1, &px, &py);
  float* in[8] = {sp->q->ks[0]};
  float* out[8] = {sp->q->ks[0]};
  launch_kpoint(KOP_SMOOTH, g, ctx->kc, in, out, 0.f, 1.f, ctx->st, ctx->stream);
  fft_kr(ctx, sp->q->rs, sp->q->ks, 1, &px, &py);
  if (sp->q3)
    CK(cudaMemcpyAsync(sp->q3, sp->q->rs[0], sizeof(float) * g.rplane, cudaMemcpyDeviceToDevice,
                       ctx->stream));
  launch_lin(g.rplane, sp->qn->rs[0], sp->qn->rs[0], nullptr, -1.0f, LIN_SCALE, ctx->st,
             ctx->stream);
  CK(cudaGetLastError());
  return 0;
}

// The profile of a species descriptor with its lengths in cells, converted
// in FP32 as init_fdist2d_0xx does (fdist2d_class.f03:164-210, 318-387,
// 525-590, 713-776): c = (center - box min) / (box length / 2^ind).
static int species_profile(qp_ctx* ctx, const qp_species_desc* d, PlasmaProfile* p) {
  p->profile = d->profile;
  p->xppc = d->ppc[0];
  p->yppc = d->ppc[1];
  p->q = d->q;
  p->den = d->density;
  const float xmin = (float)ctx->box[0][0], xmax = (float)ctx->box[0][1];
  const float ymin = (float)ctx->box[1][0], ymax = (float)ctx->box[1][1];
  const float dx = (xmax - xmin) / (float)(1 << ctx->g.indx);
  const float dy = (ymax - ymin) / (float)(1 << ctx->g.indy);
  p->cx = (d->center[0] - xmin) / dx;
  p->cy = (d->center[1] - ymin) / dy;
  p->irx = d->inner_radius[0] / dx;
  p->iry = d->inner_radius[1] / dy;
  p->orx = d->outer_radius[0] / dx;
  p->ory = d->outer_radius[1] / dy;
  p->r0 = d->radius / dx;
  p->sigr = d->width / dx;
  if (d->profile == 12) {
    if (d->nr < 2 || !d->r || !d->fr) return fail(ctx, __LINE__, "profile 12 needs nr >= 2 points");
    p->r.resize(d->nr);
    p->fr.assign(d->fr, d->fr + d->nr);
    for (int k = 0; k < d->nr; ++k) p->r[k] = d->r[k] / dx;
  }
  if (d->ns > 0) {
    if (!d->s || !d->fs) return fail(ctx, __LINE__, "longitudinal profile: null arrays");
    p->s.assign(d->s, d->s + d->ns);
    p->fs.assign(d->fs, d->fs + d->ns);
  }
  if (d->profile == 10 && !(p->irx > 0.f && p->iry > 0.f && p->orx > 0.f && p->ory > 0.f))
    return fail(ctx, __LINE__, "profile 10 needs positive inner and outer radii");
  if (d->profile == 11 && !(p->sigr > 0.f)) return fail(ctx, __LINE__, "profile 11 needs width > 0");
  return 0;
}

// Loads the species' profile at s (PPDBLKP2L: particles per tile and nppmx;
// PPPMOVIN2L: a stable copy into the tiles) into the pristine buffer P0 and
// the live buffer A, growing the buffers when the load needs more room.
// species2d%renew at s (species2d_class.f03:138-164 -> part2d%renew,
// part2d_class.f03:226-254): the particles of the profile, which depend on s
// only through the longitudinal density factor, come from the pristine copy
// on the device, with charge qm(s) * (transverse factor): no host reload.
static int species_renew_device(qp_species* sp, float s) {
  qp_ctx* ctx = sp->ctx;
  const TileGeom& tg = ctx->tg;
  float qm = 0.f;
  std::string err;
  if (!plasma_qm(sp->prof, s, &qm, &err)) return fail(ctx, __LINE__, "plasma loader: " + err);
  if (sp->A.cap < sp->P0.cap) return fail(ctx, __LINE__, "renew: capacity shrank");
  const long long n = (long long)tg.ntiles * sp->A.cap;
  for (int k = 0; k < NCOMP; ++k)
    launch_lin(n, sp->A.c[k], nullptr, nullptr, 0.f, LIN_FILL, ctx->st, ctx->stream);
  if (part_copy(ctx, sp->A, sp->P0)) return -1;
  launch_lin(n, sp->A.c[7], sp->A.c[7], nullptr, qm, LIN_SCALE, ctx->st, ctx->stream);
  CK(cudaGetLastError());
  return 0;
}

static int species_load(qp_species* sp, float s) {
  qp_ctx* ctx = sp->ctx;
  const GridDims& g = ctx->g;
  const TileGeom& tg = ctx->tg;
  std::vector<float> c[8];
  std::string err;
  // the pristine copy holds each particle's transverse charge factor; renew
  // multiplies it by the longitudinal qm(s) on the device
  const long long np = plasma_load(sp->prof, g.nx, g.ny, s, true, c, &err);
  if (np < 0) return fail(ctx, __LINE__, "plasma loader: " + err);
  sp->np = np;
  std::vector<int> cnt(tg.ntiles, 0), tile(np);
  for (long long n = 0; n < np; ++n) {
    const int tx = (int)c[0][n] / TILE, ty = (int)c[1][n] / TILE;
    tile[n] = tx + tg.mx1 * ty;
    cnt[tile[n]]++;
  }
  int nppmx = 0;
  for (int v : cnt) nppmx = std::max(nppmx, v);
  const float xtras = sp->d.xtras > 0 ? sp->d.xtras : 0.2f;
  const int nppmx0 = (int)((1.0f + xtras) * (float)nppmx);
  if (sp->P0.cap == 0 || nppmx0 > sp->P0.cap) {
    CK(cudaStreamSynchronize(ctx->stream));
    const int want = std::max({nppmx0, sp->A.cap, 1});
    part_free(&sp->P0);
    if (part_alloc(&sp->P0, tg.ntiles, std::max(nppmx0, 1)))
      return fail(ctx, __LINE__, "out of device memory (particles)");
    if (sp->A.cap < sp->P0.cap) {
      part_free(&sp->A);
      part_free(&sp->B);
      if (part_alloc(&sp->A, tg.ntiles, want) || part_alloc(&sp->B, tg.ntiles, want))
        return fail(ctx, __LINE__, "out of device memory (particles)");
    }
  }
  sp->nppmx0 = std::max(sp->nppmx0, nppmx0);
  if (!sp->ib.count) {
    const int capin = std::max(64, (int)(xtras * (float)nppmx));
    if (inbox_alloc(&sp->ib, tg.ntiles, capin)) return fail(ctx, __LINE__, "out of device memory");
  }
  const int cap = sp->P0.cap;  // rounded up to a multiple of 4 by part_alloc
  std::vector<float> h((size_t)tg.ntiles * cap, 0.f);
  std::vector<int> pos(tg.ntiles, 0);
  std::vector<long long> slot(np);
  for (long long n = 0; n < np; ++n) slot[n] = (long long)tile[n] * cap + pos[tile[n]]++;
  CK(cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < NCOMP; ++k) {
    std::fill(h.begin(), h.end(), 0.f);
    for (long long n = 0; n < np; ++n) h[slot[n]] = c[k][n];
    CK(cudaMemcpy(sp->P0.c[k], h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(sp->P0.count, cnt.data(), sizeof(int) * tg.ntiles, cudaMemcpyHostToDevice));
  return species_renew_device(sp, s);
}

extern "C" int qp_species_create(qp_ctx* ctx, const qp_species_desc* d, float s,
                                 qp_species** out) {
  if (!ctx || !d || !out) return fail(ctx, __LINE__, "null argument");
  if (d->ppc[0] < 1 || d->ppc[1] < 1) return fail(ctx, __LINE__, "invalid ppc");
  qp_species* sp = new qp_species();
  sp->ctx = ctx;
  sp->d = *d;
  sp->d.r = sp->d.fr = sp->d.s = sp->d.fs = nullptr;  // the arrays are copied into prof
  sp->qbm = d->q / d->m;
  sp->dt = ctx->dxi;
  const GridDims& g = ctx->g;
  if (species_profile(ctx, d, &sp->prof) || species_load(sp, s)) {
    qp_species_destroy(sp);
    return -1;
  }
  sp->q = field_new(ctx, 1, 0);
  sp->qn = field_new(ctx, 1, 0);
  sp->cusp = field_new(ctx, 3, 0);
  sp->dcusp = field_new(ctx, 2, 0);
  sp->amusp = field_new(ctx, 3, 0);
  if (!sp->q || !sp->qn || !sp->cusp || !sp->dcusp || !sp->amusp)
    return fail(ctx, __LINE__, "out of device memory");
  sp->q3 = dalloc((size_t)(ctx->nz + 1) * g.rplane);
  sp->q3_first = dalloc(g.rplane);
  if (!sp->q3 || !sp->q3_first) return fail(ctx, __LINE__, "out of device memory");
  if (species_background(sp)) return -1;
  CK(cudaMemcpyAsync(sp->q3_first, sp->q3, sizeof(float) * g.rplane, cudaMemcpyDeviceToDevice,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  DevStatus st;
  if (sync_status(ctx, &st)) return -1;
  if (st.error) return fail(ctx, __LINE__, "species load: particle outside its tile");
  *out = sp;
  return 0;
}

extern "C" int qp_species_destroy(qp_species* sp) {
  if (!sp) return 0;
  cudaStreamSynchronize(sp->ctx->stream);
  part_free(&sp->A);
  part_free(&sp->B);
  part_free(&sp->P0);
  inbox_free(&sp->ib);
  field_free(sp->q);
  field_free(sp->qn);
  field_free(sp->cusp);
  field_free(sp->dcusp);
  field_free(sp->amusp);
  cudaFree(sp->q3);
  cudaFree(sp->q3_first);
  delete sp;
  return 0;
}

// A transverse profile is deterministic, so renew restores the pristine copy of
// the loaded, binned plasma and its background (same bits as a fresh load).
// With a longitudinal profile the density depends on s: the plasma is loaded
// afresh at s (species2d%renew, species2d_class.f03:138-164).
extern "C" int qp_species_renew(qp_species* sp, float s) {
  qp_ctx* ctx = sp->ctx;
  if (species_renew_device(sp, s) || species_background(sp)) return -1;
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

extern "C" int qp_species_qdp(qp_species* sp, qp_field2d* qe) {
  qp_ctx* ctx = sp->ctx;
  if (qe->state != 0) return fail(ctx, __LINE__, "sum: states are different");
  const GridDims& g = ctx->g;
  float* q = sp->q->rs[0];
  launch_lin(g.rplane, q, nullptr, nullptr, 0.f, LIN_FILL, ctx->st, ctx->stream);
  launch_deposit_rho(sp->A, ctx->tg, q, ctx->st, ctx->stream);
  sp->q->state = 0;
  launch_lin(g.rplane, qe->rs[0], q, qe->rs[0], 0.f, LIN_ADD, ctx->st, ctx->stream);
  launch_lin(g.rplane, qe->rs[0], sp->qn->rs[0], qe->rs[0], 0.f, LIN_ADD, ctx->st, ctx->stream);
  CK(cudaGetLastError());
  return 0;
}

static int check_particles(qp_ctx* ctx, const char* where) {
  DevStatus st;
  if (sync_status(ctx, &st)) return -1;
  if (st.error < 0) {
    clear_status(ctx, 1);
    return fail(ctx, __LINE__, std::string(where) + ": particle outside its tile (code " +
                                   std::to_string(st.error) + ")");
  }
  return 0;
}

extern "C" int qp_species_extpsi(qp_species* sp, qp_field2d* psi, float dex) {
  qp_ctx* ctx = sp->ctx;
  if (psi->state != 0) return fail(ctx, __LINE__, "extpsi: data is in ks");
  launch_extpsi(sp->A, ctx->tg, psi->rs[0], sp->qbm, dex, ctx->st, ctx->stream);
  CK(cudaGetLastError());
  return check_particles(ctx, "extpsi");
}

static GatherPlanes gplanes(qp_field2d* fxy, qp_field2d* bxyz, qp_field2d* psit, int combine) {
  GatherPlanes f{};
  f.fx = fxy->rs[0];
  f.fy = fxy->rs[1];
  f.bx = bxyz->rs[0];
  f.by = bxyz->rs[1];
  f.bz = bxyz->rs[2];
  f.psit = psit->rs[0];
  f.combine = combine;
  return f;
}

extern "C" int qp_species_amjdp(qp_species* sp, qp_field2d* fxy, qp_field2d* bxyz,
                                qp_field2d* psit, qp_field2d* cu, qp_field2d* amu,
                                qp_field2d* dcu, float dex) {
  qp_ctx* ctx = sp->ctx;
  const GridDims& g = ctx->g;
  if (fxy->dim != 2 || bxyz->dim != 3 || cu->dim != 3 || dcu->dim != 2 || amu->dim != 3)
    return fail(ctx, __LINE__, "amjdp: invalid vector size");
  float* acc[8] = {sp->cusp->rs[0], sp->cusp->rs[1], sp->cusp->rs[2], sp->dcusp->rs[0],
                   sp->dcusp->rs[1], sp->amusp->rs[0], sp->amusp->rs[1], sp->amusp->rs[2]};
  for (int i = 0; i < 8; ++i)
    launch_lin(g.rplane, acc[i], nullptr, nullptr, 0.f, LIN_FILL, ctx->st, ctx->stream);
  launch_amjdp(sp->A, ctx->tg, gplanes(fxy, bxyz, psit, 0), acc, sp->qbm, sp->dt, dex, 1.0f,
               ctx->st, ctx->stream);
  for (int c = 0; c < 3; ++c)
    launch_lin(g.rplane, cu->rs[c], sp->cusp->rs[c], cu->rs[c], 0.f, LIN_ADD, ctx->st, ctx->stream);
  for (int c = 0; c < 2; ++c)
    launch_lin(g.rplane, dcu->rs[c], sp->dcusp->rs[c], dcu->rs[c], 0.f, LIN_ADD, ctx->st,
               ctx->stream);
  for (int c = 0; c < 3; ++c)
    launch_lin(g.rplane, amu->rs[c], sp->amusp->rs[c], amu->rs[c], 0.f, LIN_ADD, ctx->st,
               ctx->stream);
  for (int c = 0; c < 3; ++c)
    launch_lin(g.rplane, sp->cusp->rs[c], sp->cusp->rs[c], nullptr, dex, LIN_SCALE, ctx->st,
               ctx->stream);
  cu->state = dcu->state = amu->state = 0;
  CK(cudaGetLastError());
  return check_particles(ctx, "amjdp");
}

// push (mode 1) or re-bin (mode 2) from A into B, with overflow recovery;
// on success B becomes the live buffer.
static int push_rebin(qp_species* sp, int mode, const GatherPlanes& f, float dex) {
  qp_ctx* ctx = sp->ctx;
  const int nt = ctx->tg.ntiles;
  for (int attempt = 0; attempt < 12; ++attempt) {
    if (sp->B.cap < sp->A.cap) {
      part_free(&sp->B);
      if (part_alloc(&sp->B, nt, sp->A.cap)) return fail(ctx, __LINE__, "out of device memory");
    }
    launch_push(mode, sp->A, sp->B, sp->ib, ctx->tg, f, sp->qbm, sp->dt, dex, ctx->st,
                ctx->stream);
    launch_insert(sp->B, sp->ib, ctx->tg, ctx->st, ctx->stream);
    CK(cudaGetLastError());
    DevStatus st;
    if (sync_status(ctx, &st)) return -1;
    if (st.error == 0) {
      std::swap(sp->A, sp->B);
      return 0;
    }
    if (st.error < 0) {
      clear_status(ctx, 1);
      return fail(ctx, __LINE__, "push: particle outside its tile (code " +
                                     std::to_string(st.error) + ")");
    }
    // capacity overflow: grow by (1 + xtras) and retry from the intact input
    const float xtras = sp->d.xtras > 0 ? sp->d.xtras : 0.2f;
    sp->regrowths++;
    if (st.need_cap > sp->B.cap) {
      const int ncap = (int)((1.0f + xtras) * (float)st.need_cap);
      ctx->need = ncap;
      part_free(&sp->B);
      if (part_alloc(&sp->B, nt, ncap)) return fail(ctx, __LINE__, "out of device memory");
    }
    if (st.need_inbox > sp->ib.cap) {
      const int ncap = (int)((1.0f + xtras) * (float)st.need_inbox);
      inbox_free(&sp->ib);
      if (inbox_alloc(&sp->ib, nt, ncap)) return fail(ctx, __LINE__, "out of device memory");
    }
    CK(cudaMemsetAsync(sp->ib.count, 0, sizeof(int) * nt, ctx->stream));
    if (clear_status(ctx, 1)) return -1;
  }
  return fail(ctx, __LINE__, "push: buffer growth did not converge");
}

extern "C" int qp_species_push(qp_species* sp, qp_field2d* fxy, qp_field2d* bxyz,
                               qp_field2d* psit, float dex) {
  return push_rebin(sp, 1, gplanes(fxy, bxyz, psit, 0), dex);
}

extern "C" int qp_species_partpush(qp_species* sp, qp_field2d* fxy, qp_field2d* bxyz,
                                   qp_field2d* psit, float dex) {
  qp_ctx* ctx = sp->ctx;
  launch_push(0, sp->A, sp->A, sp->ib, ctx->tg, gplanes(fxy, bxyz, psit, 0), sp->qbm, sp->dt, dex,
              ctx->st, ctx->stream);
  CK(cudaGetLastError());
  return check_particles(ctx, "partpush");
}

extern "C" int qp_species_pmove(qp_species* sp) {
  GatherPlanes f{};
  return push_rebin(sp, 2, f, 1.0f);
}

extern "C" int qp_species_cbq(qp_species* sp, int pos) {
  qp_ctx* ctx = sp->ctx;
  const GridDims& g = ctx->g;
  if (pos < 1 || pos > ctx->nz + 1) return fail(ctx, __LINE__, "cbq: slice out of range");
  int px = 0, py = 0;
  const float* add[1] = {sp->cusp->rs[2]};
  fft_rk(ctx, sp->q->rs, sp->q->ks, add, 1, &px, &py);
  float* in[8] = {sp->q->ks[0]};
  launch_kpoint(KOP_SMOOTH, g, ctx->kc, in, in, 0.f, 1.f, ctx->st, ctx->stream);
  fft_kr(ctx, sp->q->rs, sp->q->ks, 1, &px, &py);
  CK(cudaMemcpyAsync(sp->q3 + (size_t)(pos - 1) * g.rplane, sp->q->rs[0],
                     sizeof(float) * g.rplane, cudaMemcpyDeviceToDevice, ctx->stream));
  sp->q->state = 0;
  CK(cudaGetLastError());
  return 0;
}

extern "C" int qp_species_ntiles(const qp_species* sp) { return sp->ctx->tg.ntiles; }
extern "C" int qp_species_nppmx(const qp_species* sp) { return sp->A.cap; }

extern "C" long long qp_species_np(qp_species* sp) {
  qp_ctx* ctx = sp->ctx;
  std::vector<int> cnt(ctx->tg.ntiles);
  if (cudaMemcpyAsync(cnt.data(), sp->A.count, sizeof(int) * cnt.size(), cudaMemcpyDeviceToHost,
                      ctx->stream) != cudaSuccess)
    return -1;
  cudaStreamSynchronize(ctx->stream);
  long long n = 0;
  for (int v : cnt) n += v;
  return n;
}

extern "C" int qp_species_download(qp_species* sp, float* ppart, int* kpic, int nppmx_ld) {
  qp_ctx* ctx = sp->ctx;
  const int nt = ctx->tg.ntiles, cap = sp->A.cap;
  std::vector<int> cnt(nt);
  CK(cudaMemcpyAsync(cnt.data(), sp->A.count, sizeof(int) * nt, cudaMemcpyDeviceToHost,
                     ctx->stream));
  std::vector<float> h((size_t)nt * cap);
  CK(cudaStreamSynchronize(ctx->stream));
  int mx = 0;
  for (int v : cnt) mx = std::max(mx, v);
  if (nppmx_ld < mx) return fail(ctx, __LINE__, "download: nppmx_ld too small");
  std::memset(ppart, 0, sizeof(float) * 8 * (size_t)nppmx_ld * nt);
  for (int c = 0; c < NCOMP; ++c) {
    CK(cudaMemcpy(h.data(), sp->A.c[c], sizeof(float) * h.size(), cudaMemcpyDeviceToHost));
    for (int t = 0; t < nt; ++t)
      for (int n = 0; n < cnt[t]; ++n)
        ppart[(size_t)c + 8 * ((size_t)n + (size_t)nppmx_ld * t)] = h[(size_t)t * cap + n];
  }
  std::memcpy(kpic, cnt.data(), sizeof(int) * nt);
  return 0;
}

extern "C" int qp_species_upload(qp_species* sp, const float* ppart, const int* kpic,
                                 int nppmx_ld) {
  qp_ctx* ctx = sp->ctx;
  const int nt = ctx->tg.ntiles;
  int mx = 0;
  for (int t = 0; t < nt; ++t) mx = std::max(mx, kpic[t]);
  if (mx > sp->A.cap) {
    part_free(&sp->A);
    if (part_alloc(&sp->A, nt, mx)) return fail(ctx, __LINE__, "out of device memory");
  }
  const int cap = sp->A.cap;
  std::vector<float> h((size_t)nt * cap);
  for (int c = 0; c < NCOMP; ++c) {
    std::fill(h.begin(), h.end(), 0.f);
    for (int t = 0; t < nt; ++t)
      for (int n = 0; n < kpic[t]; ++n)
        h[(size_t)t * cap + n] = ppart[(size_t)c + 8 * ((size_t)n + (size_t)nppmx_ld * t)];
    CK(cudaMemcpy(sp->A.c[c], h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(sp->A.count, kpic, sizeof(int) * nt, cudaMemcpyHostToDevice));
  return 0;
}

extern "C" int qp_species_download_qn(qp_species* sp, float* rf) {
  sp->qn->state = 0;
  return qp_field2d_download_rs(sp->qn, rf);
}

extern "C" int qp_species_download_q(qp_species* sp, float* rf) {
  return qp_field2d_download_rs(sp->q, rf);
}

extern "C" int qp_species_download_q3(qp_species* sp, int pos, float* rf) {
  qp_ctx* ctx = sp->ctx;
  const GridDims& g = ctx->g;
  if (pos < 1 || pos > ctx->nz + 1) return fail(ctx, __LINE__, "q3: slice out of range");
  std::vector<float> h(g.rplane);
  CK(cudaMemcpyAsync(h.data(), sp->q3 + (size_t)(pos - 1) * g.rplane, sizeof(float) * g.rplane,
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const int nxv = g.nx + 2;
  for (int y = 0; y <= g.ny; ++y)
    for (int x = 0; x < nxv; ++x) rf[(size_t)x + (size_t)nxv * y] = h[(size_t)y * g.rp + x];
  return 0;
}

// ------------------------------------------------------------------ beam
// init_fdist3d_0xx conversions of a beam's keys to cells and its charge per
// particle, then the profile's loader (fdist3d_class.f03:222-1166).
extern "C" int qp_beam_create(qp_ctx* ctx, const qp_beam_desc* d, qp_beam** out) {
  if (!ctx || !d || !out) return fail(ctx, __LINE__, "null argument");
  const int pf = d->profile;
  if (pf != 0 && pf != 1 && pf != 2 && pf != 3 && pf != 100)
    return fail(ctx, __LINE__, "beam profile must be 0, 1, 2, 3 or 100");
  if (d->static_density && pf != 0 && pf != 1)
    return fail(ctx, __LINE__, "only beam profiles 0 and 1 can be static");
  if (pf <= 2 && (d->np[0] < 1 || d->np[1] < 1 || d->np[2] < 1))
    return fail(ctx, __LINE__, "beam np must be at least 1 in each direction");
  if (!(d->q != 0.f)) return fail(ctx, __LINE__, "beam q must not be 0");
  const GridDims& g = ctx->g;
  float lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = (float)ctx->box[a][0];
    hi[a] = (float)ctx->box[a][1];
  }
  const float dx = (hi[0] - lo[0]) / (float)g.nx;
  const float dy = (hi[1] - lo[1]) / (float)g.ny;
  const float dz = (hi[2] - lo[2]) / (float)ctx->nz;
  BeamLoad L;
  L.npx = d->np[0];
  L.npy = d->np[1];
  L.npz = d->np[2];
  L.nx = g.nx;
  L.ny = g.ny;
  L.nz = ctx->nz;
  L.vtx = d->sigma_v[0];
  L.vty = d->sigma_v[1];
  L.vtz = d->sigma_v[2];
  L.vdz = d->gamma;
  L.sigx = d->sigma[0] / dx;
  L.sigy = d->sigma[1] / dy;
  L.sigz = d->sigma[2] / dz;
  L.x0 = (d->center[0] - lo[0]) / dx;
  L.y0 = (d->center[1] - lo[1]) / dy;
  L.z0 = (d->center[2] - lo[2]) / dz;
  L.quiet = d->quiet_start != 0;
  // centroid polynomials in cells: c1 dz dz / dx, c2 dz / dx, c3 / dx
  L.cx[0] = d->centroid_x[0] * dz * dz / dx;
  L.cx[1] = d->centroid_x[1] * dz / dx;
  L.cx[2] = d->centroid_x[2] / dx;
  L.cy[0] = d->centroid_y[0] * dz * dz / dy;
  L.cy[1] = d->centroid_y[1] * dz / dy;
  L.cy[2] = d->centroid_y[2] / dy;
  const long long nfull = (long long)L.npx * L.npy * L.npz;
  L.npmax = d->npmax > 0 ? d->npmax : nfull + 8;
  std::vector<float> c[7];
  long long n = 0;
  int ierr = 0;
  bool outside = false;  // a profile-1 beam whose z range misses the box
  if (pf == 0) {
    L.qm = beam_charge(d->q, d->peak_density, d->sigma, lo, hi, g.indx, g.indy, ctx->indz, L.npx,
                       L.npy, L.npz);
    if (!d->static_density) n = beam_random(ctx->rng, L, c, &ierr);
  } else if (pf == 1) {
    if (d->npiece < 2 || !d->piecewise_z || !d->piecewise_fz)
      return fail(ctx, __LINE__, "beam profile 1 needs at least 2 piecewise points");
    const std::vector<float> z(d->piecewise_z, d->piecewise_z + d->npiece);
    const std::vector<float> fz(d->piecewise_fz, d->piecewise_fz + d->npiece);
    float sumz = 0.f;
    if (!beam_zprofile(z, fz, lo[2], dz, ctx->nz, &L.zf, &sumz))
      return fail(ctx, __LINE__, "Piecewise_z is not monotonically increasing");
    L.qm = beam_charge_q(d->q, d->peak_density, 1.f, d->sigma[0], d->sigma[1], sumz, dx, dy, dz,
                         L.npx, L.npy, L.npz);
    outside = (z.front() - lo[2]) / dz >= (float)ctx->nz || (z.back() - lo[2]) / dz <= 0.f;
    if (!d->static_density && !outside) {
      Uniform uni(d->seed ? d->seed : 0x5eedull);
      n = beam_ran_pfl(ctx->rng, uni, L, c, &ierr);
    }
  } else if (pf == 2) {
    const float sx = std::sqrt(d->beta[0] * d->emittance[0] / d->gamma);
    const float sy = std::sqrt(d->beta[1] * d->emittance[1] / d->gamma);
    L.qm = beam_charge_q(d->q, d->peak_density, 1.5f, sx, sy, d->sigma[2], dx, dy, dz, L.npx,
                         L.npy, L.npz);
    L.alphax = d->alpha[0];
    L.alphay = d->alpha[1];
    L.betax = d->beta[0] / dx;
    L.betay = d->beta[1] / dy;
    L.emitx = d->emittance[0] / dx;
    L.emity = d->emittance[1] / dy;
    if (!(L.betax > 0.f && L.betay > 0.f && L.emitx > 0.f && L.emity > 0.f && d->gamma > 0.f))
      return fail(ctx, __LINE__, "beam profile 2 needs beta, emittance and gamma > 0");
    n = beam_twiss(ctx->rng, L, c, &ierr);
  } else if (pf == 3) {
    if (!d->file_name || d->np[0] < 0 || !(d->n0 > 0.f))
      return fail(ctx, __LINE__, "beam profile 3 needs file_name, np[0] >= 0 and n0 > 0");
    const float cwp = 5.32150254f * 1e9f / std::sqrt(d->n0);
    std::string err;
    n = beam_file(d->file_name, d->np[0], L.x0, L.y0, cwp, dx, dy, dz, g.nx, g.ny, ctx->nz, c,
                  &err);
    if (n < 0) return fail(ctx, __LINE__, err);
    if (d->npmax > 0 && n > d->npmax) ierr = (int)(n - d->npmax);
  } else {
    if (d->ppc[0] < 1 || d->ppc[1] < 1 || d->ppc[2] < 1 || !(d->r2 != 0.f))
      return fail(ctx, __LINE__, "beam profile 100 needs ppc >= 1 and r2 != 0");
    const float qm = d->q / std::fabs(d->q) / (float)d->ppc[0] / (float)d->ppc[1] /
                     (float)d->ppc[2];
    const float bc[3] = {L.x0, L.y0, L.z0};
    const float* rg[3] = {d->range_x, d->range_y, d->range_z};
    const float del[3] = {dx, dy, dz};
    float lb[3], ub[3];
    for (int a = 0; a < 3; ++a) {
      lb[a] = (rg[a][0] - lo[a]) / del[a];
      ub[a] = (rg[a][1] - lo[a]) / del[a];
    }
    n = beam_ring(d->ppc, qm, d->peak_density, d->gamma, bc, lb, ub, d->r1 / dx, d->r2 / dx, g.nx,
                  g.ny, ctx->nz, c);
    if (d->npmax > 0 && n > d->npmax) ierr = (int)(n - d->npmax);
  }
  if (ierr) return fail(ctx, __LINE__, "beam loader: npmax too small");
  qp_beam* b = new qp_beam();
  b->ctx = ctx;
  b->b.np = n;
  b->cap = n;
  b->qbm = d->q / d->m;
  b->is_static = d->static_density != 0;
  b->frozen = d->frozen != 0 || b->is_static;
  for (int k = 0; k < BCOMP; ++k) {
    b->b.c[k] = dalloc(n, false);
    if (!b->b.c[k]) return fail(ctx, __LINE__, "out of device memory");
    if (n > 0)
      CK(cudaMemcpy(b->b.c[k], c[k].data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  }
  b->q3d = dalloc((size_t)(ctx->nz + 1) * g.rplane);
  if (!b->q3d) return fail(ctx, __LINE__, "out of device memory");
  if (b->is_static && !outside) {
    // dist3d_000/001 with static = true: the density np q/|q| times the
    // profile on nodes x < nx, y < ny of slices 1..nz
    const float amp = d->peak_density * L.qm / std::fabs(L.qm);
    const float sigz = d->sigma[2] / dz;
    std::vector<float> plane(g.rplane, 0.f);
    for (int k = 0; k < ctx->nz; ++k) {
      beam_static_plane(amp, L.x0, L.y0, L.z0, L.sigx, L.sigy, sigz, L.cx, L.cy,
                        pf == 1 ? L.zf : std::vector<float>(), g.nx, g.ny, k, g.rp, plane.data());
      CK(cudaMemcpy(b->q3d + (size_t)k * g.rplane, plane.data(), sizeof(float) * g.rplane,
                    cudaMemcpyHostToDevice));
    }
  }
  *out = b;
  return 0;
}

extern "C" int qp_beam_destroy(qp_beam* b) {
  if (!b) return 0;
  cudaStreamSynchronize(b->ctx->stream);
  for (int k = 0; k < BCOMP; ++k) cudaFree(b->b.c[k]);
  cudaFree(b->q3d);
  if (b->keep) cudaFree(b->keep);
  delete b;
  return 0;
}

extern "C" long long qp_beam_np(const qp_beam* b) { return b->b.np; }

extern "C" int qp_beam_qdp(qp_beam* b) {
  qp_ctx* ctx = b->ctx;
  const GridDims& g = ctx->g;
  if (b->is_static) return 0;  // qdeposit_beam3d skips static beams
  CK(cudaMemsetAsync(b->q3d, 0, sizeof(float) * (size_t)(ctx->nz + 1) * g.rplane, ctx->stream));
  launch_beam_deposit(b->b, g, ctx->nz, b->q3d, ctx->st, ctx->stream);
  CK(cudaGetLastError());
  DevStatus st;
  if (sync_status(ctx, &st)) return -1;
  if (st.error) {
    clear_status(ctx, 1);
    return fail(ctx, __LINE__, "beam deposit: particle outside the grid");
  }
  return 0;
}

extern "C" int qp_beam_qdpcopy(qp_beam* b, qp_field2d* q, int slice) {
  qp_ctx* ctx = b->ctx;
  if (slice < 1 || slice > ctx->nz + 1) return fail(ctx, __LINE__, "qdpcopy: slice out of range");
  if (q->state != 0) return fail(ctx, __LINE__, "copyadd: data is in ks");
  const GridDims& g = ctx->g;
  launch_lin(g.rplane, q->rs[0], q->rs[0], b->q3d + (size_t)(slice - 1) * g.rplane, 0.f, LIN_ADD,
             ctx->st, ctx->stream);
  CK(cudaGetLastError());
  return 0;
}

extern "C" int qp_beam_upload(qp_beam* b, const float* part, long long np) {
  qp_ctx* ctx = b->ctx;
  if (np < 0 || np > b->cap)
    return fail(ctx, __LINE__, "beam upload: more particles than the beam holds (" +
                                   std::to_string(b->cap) + ")");
  b->b.np = np;
  if (ensure_staging(ctx, sizeof(float) * 7 * (size_t)np)) return -1;
  CK(cudaMemcpyAsync(ctx->staging, part, sizeof(float) * 7 * (size_t)np, cudaMemcpyHostToDevice,
                     ctx->stream));
  launch_beam_aos_to_soa(ctx->staging, b->b, ctx->stream);
  CK(cudaGetLastError());
  return 0;
}

extern "C" int qp_beam_download(qp_beam* b, float* part) {
  qp_ctx* ctx = b->ctx;
  std::vector<float> h(b->b.np);
  for (int k = 0; k < BCOMP; ++k) {
    CK(cudaMemcpy(h.data(), b->b.c[k], sizeof(float) * h.size(), cudaMemcpyDeviceToHost));
    for (long long n = 0; n < b->b.np; ++n) part[(size_t)k + 7 * (size_t)n] = h[n];
  }
  return 0;
}

extern "C" int qp_beam_download_q3d(qp_beam* b, float* rf) {
  qp_ctx* ctx = b->ctx;
  const GridDims& g = ctx->g;
  const size_t np3 = (size_t)(ctx->nz + 1) * g.rplane;
  std::vector<float> h(np3);
  CK(cudaMemcpy(h.data(), b->q3d, sizeof(float) * np3, cudaMemcpyDeviceToHost));
  const int nxv = g.nx + 2;
  for (int l = 0; l <= ctx->nz; ++l)
    for (int y = 0; y <= g.ny; ++y)
      for (int x = 0; x < nxv; ++x)
        rf[(size_t)x + (size_t)nxv * ((size_t)y + (size_t)(g.ny + 1) * l)] =
            h[(size_t)l * g.rplane + (size_t)y * g.rp + x];
  return 0;
}

// ---------------------------------------------------------------- beam restart
// The reference writes a beam's restart (beam3d%wrst -> part3d%wrst ->
// hdf5io wpart, hdf5io_class.f03:1301-1360) as
//   ./RST/Beam-NNNN/RST-beamNNNN-RRRRRRRRRR_SSSSSSSS.h5
// (beam NNNN from 1, rank R, dump S; simulation_class.f03:1261-1277) holding
// the root attribute tp = particle count and one dataset named
// RST-beamNNNN-RRRRRRRRRR with part(7, tp).  This build has no HDF5 library,
// so the same path carries the suffix .qprst instead of .h5 and the same
// content in a flat container: the 8 bytes "QPRST001", tp as a little-endian
// int64, then part(7, tp) as float32, column-major.
static std::string restart_path(const char* dir, int beam, int rank, int step) {
  char tail[96];
  std::snprintf(tail, sizeof(tail), "RST/Beam-%04d/RST-beam%04d-%010d_%08d.qprst", beam, beam,
                rank, step);
  std::string d = dir && dir[0] ? std::string(dir) : std::string(".");
  if (d.back() != '/') d += '/';
  return d + tail;
}

extern "C" int qp_beam_write_restart(qp_beam* b, const char* dir, int beam, int rank, int step) {
  if (!b) return fail(nullptr, __LINE__, "null beam");
  qp_ctx* ctx = b->ctx;
  if (beam < 1 || beam > 9999 || rank < 0 || step < 0 || step > 99999999)
    return fail(ctx, __LINE__, "restart: beam 1..9999, rank >= 0, step 0..99999999");
  const std::string path = restart_path(dir, beam, rank, step);
  const std::string folder = path.substr(0, path.rfind('/'));
  const std::string mk = "mkdir -p '" + folder + "'";
  if (folder.find('\'') != std::string::npos || std::system(mk.c_str()) != 0)
    return fail(ctx, __LINE__, "restart: cannot create " + folder);
  const long long np = b->b.np;
  std::vector<float> part((size_t)7 * np);
  if (np > 0 && qp_beam_download(b, part.data())) return -1;
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return fail(ctx, __LINE__, "restart: cannot write " + path);
  const long long tp = np;
  bool ok = std::fwrite("QPRST001", 1, 8, f) == 8 && std::fwrite(&tp, 8, 1, f) == 1 &&
            (np == 0 || std::fwrite(part.data(), sizeof(float), part.size(), f) == part.size());
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return fail(ctx, __LINE__, "restart: short write to " + path);
  return 0;
}

extern "C" int qp_beam_read_restart(qp_beam* b, const char* dir, int beam, int rank, int step) {
  if (!b) return fail(nullptr, __LINE__, "null beam");
  qp_ctx* ctx = b->ctx;
  const std::string path = restart_path(dir, beam, rank, step);
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return fail(ctx, __LINE__, "restart: cannot open " + path);
  char magic[8];
  long long tp = -1;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "QPRST001", 8) == 0 &&
            std::fread(&tp, 8, 1, f) == 1 && tp >= 0 && tp <= b->cap;
  std::vector<float> part;
  if (ok) {
    part.resize((size_t)7 * tp);
    ok = tp == 0 || std::fread(part.data(), sizeof(float), part.size(), f) == part.size();
  }
  std::fclose(f);
  if (!ok) return fail(ctx, __LINE__, "restart: " + path + " is not a beam restart of this beam");
  if (qp_beam_upload(b, part.data(), tp)) return -1;
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

#include "qp_sim.inc"
#include "qp_scan.inc"
