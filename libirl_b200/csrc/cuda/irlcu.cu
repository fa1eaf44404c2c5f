// irlcu.cu -- device context and the extern "C" entry points of include/irlcu.h.
//
// The host C driver (IrlOsem / IrlGenprj) owns the control flow; this file
// owns device memory and sequences the kernels of one batched stage.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <array>
#include <vector>

#include "irlcu_internal.cuh"
#include "../host/irl_geom.h"

namespace irlcu {

Ctx *g_ctx = nullptr;
long long g_launch_count = 0;
static char g_err[1024] = "";
// stream of the context being built or torn down before it is current
static cudaStream_t g_init_stream = nullptr;

// ------------------------------------------------------- stage profiling
struct ProfRec {
  int stage;
  cudaEvent_t a, b;
  double flops, bytes;
  int launches;
};
static bool g_prof_on = false;
static std::vector<ProfRec> g_prof;
static std::vector<cudaEvent_t> g_prof_pool;
static size_t g_prof_used = 0;
static irlcu_profile g_prof_acc;

static cudaEvent_t prof_event() {
  if (g_prof_used == g_prof_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    g_prof_pool.push_back(e);
  }
  return g_prof_pool[g_prof_used++];
}

// RAII bracket of one stage on stream st
struct Stage {
  int stage;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
  long long l0;
  double flops = 0, bytes = 0;
  Stage(int s, cudaStream_t st_) : stage(s), st(st_), l0(g_launch_count) {
    if (g_prof_on && (a = prof_event())) cudaEventRecord(a, st);
  }
  ~Stage() {
    if (!a) return;
    cudaEvent_t b = prof_event();
    if (!b) return;
    cudaEventRecord(b, st);
    g_prof.push_back(ProfRec{stage, a, b, flops, bytes, (int)(g_launch_count - l0)});
  }
};

// algorithmic FLOPs of the DRF convolutions of a batch (2 per tap per
// output pixel, taps = the PSF's own extent, planes with distance > 0)
// 5 L log2 L per complex line transform of length L
static double fft5(double L) { return 5.0 * L * std::log2(L); }

// algorithmic FLOPs of the DRF stage: 2 per PSF tap per output pixel for the
// direct convolution; for the Fourier-domain engine the line transforms
// (two real rows per complex line) and the spectral products
static double drf_flops(const Ctx &c, const DrfDev *d, const int *views, int nv, bool forward) {
  if (!d || !d->psf) return 0.0;
  if (d->fft.on) {
    const DrfFft &F = d->fft;
    const double rows = 0.5 * F.G * fft5(F.Mx), cols = F.Mxh * fft5(F.Mz), mul = 8.0 * F.Mz * F.Mxh;
    const double inv_rows = 0.5 * c.nz * fft5(F.Mx);
    if (forward) return (double)nv * (c.n * (rows + cols + mul) + cols + inv_rows);
    return (double)nv * c.n * (rows + 2.0 * cols + mul + inv_rows);
  }
  double f = 0.0;
  for (int i = 0; i < nv; ++i)
    for (int y = 0; y < c.n; ++y) {
      const int id = d->h_rows[(size_t)views[i] * c.n + y];
      if (id >= 0) f += 2.0 * (double)c.pln * d->h_taps[id];
    }
  return f;
}

int set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int halo_instance(int h);
size_t forward_partial_elems(int n, int nz, int max_batch);
void free_rotate_scratch(Ctx &c);
void esse_free(Ctx &c);

cudaError_t dev_alloc(void **p, size_t bytes, cudaStream_t st) {
  static bool ready[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && !ready[dev]) {
    cudaMemPool_t pool;
    if ((e = cudaDeviceGetDefaultMemPool(&pool, dev)) != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
    // a block freed on another context's stream is not handed out with an
    // inserted wait on that stream: with several reconstructions in flight
    // (IrlOsemBatch) such a wait, followed by this function's stream
    // synchronisation, would hold the host until the other problem's queued
    // work reached the free
    int no = 0;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no)) != cudaSuccess) return e;
    ready[dev] = true;
  }
  if ((e = cudaMallocAsync(p, bytes, st)) != cudaSuccess) return e;
  return cudaStreamSynchronize(st);
}

void dev_free(void *p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}

// allocations, uploads and memsets of the current context go on its stream:
// the context's kernels run on a non-blocking stream, which is not ordered
// after legacy-stream copies or memsets (a pageable cudaMemcpy may return
// before its DMA lands, a cudaMemset before it runs)
static cudaStream_t alloc_stream() { return g_ctx ? g_ctx->st : g_init_stream; }

template <class T>
static int dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) return IRLCU_OK;
  cudaError_t e = dev_alloc_t(p, count, alloc_stream());
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(IRLCU_ENOMEM, "device allocation of %zu bytes failed: %s", count * sizeof(T),
                     cudaGetErrorString(e));
  }
  return IRLCU_OK;
}

template <class T>
static void dfree(T *&p) {
  dev_free(p, alloc_stream());
  p = nullptr;
}

static void graphs_clear(Ctx &c) {
  for (GraphRec &g : c.graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  c.graphs.clear();
  c.graph_seen.clear();
}

static void free_ctx(Ctx *c) {
  if (!c) return;
  Ctx *const cur = g_ctx;
  g_ctx = c;  // dfree orders the frees on this context's stream
  cudaStreamSynchronize(c->st);
  graphs_clear(*c);
  dfree(c->sur_scale);
  dfree(c->sur_work);
  dfree(c->sur_static);
  dfree(c->dviews_all);
  dfree(c->dvp_all);
  dfree(c->rot.hdr);
  dfree(c->rot.row_sh);
  dfree(c->rot.row_f1);
  dfree(c->rot.row_f2);
  dfree(c->rot.col_sh);
  dfree(c->rot.col_f1);
  dfree(c->rot.col_f2);
  dfree(c->rot.sn);
  dfree(c->rot.cs);
  dfree(c->sup_start);
  dfree(c->sup_end);
  dfree(c->est);
  dfree(c->atn);
  dfree(c->prj);
  dfree(c->scatest);
  dfree(c->prjscat);
  dfree(c->upd);
  dfree(c->norm);
  dfree(c->colmask);
  dfree(c->tE);
  dfree(c->tS);
  dfree(c->tMu);
  dfree(c->wrot);
  dfree(c->wbck);
  dfree(c->wprj);
  dfree(c->wprj2);
  dfree(c->wpart);
  dfree(c->wavg);
  dfree(c->dviews);
  dfree(c->dvp);
  for (int w = 0; w < 2; ++w) {
    dfree(c->drf[w].psf);
    dfree(c->drf[w].pad_rows);
    dfree(c->drf[w].row_idist);
    drf_fft_free(*c, c->drf[w]);
  }
  drf_fft_work_free(*c);
  esse_free(*c);
  free_rotate_scratch(*c);
  for (int k = 0; k < 2; ++k) {
    if (c->snap_copied[k]) cudaEventSynchronize(c->snap_copied[k]);
    dfree(c->snap[k]);  // snap_host[k] belongs to the process-wide pinned pair
    if (c->snap_made[k]) cudaEventDestroy(c->snap_made[k]);
    if (c->snap_copied[k]) cudaEventDestroy(c->snap_copied[k]);
  }
  if (c->snap_st) cudaStreamDestroy(c->snap_st);
  if (c->up_st) cudaStreamDestroy(c->up_st);
  for (auto &v : c->trial_ev)
    for (auto &e : v) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
  for (auto &e : c->ev) cudaEventDestroy(e);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  g_ctx = cur == c ? nullptr : cur;
}

#define TRY(x)                 \
  do {                         \
    int rc_ = (x);             \
    if (rc_) return rc_;       \
  } while (0)

static int need_ctx() {
  if (!g_ctx) return set_error(IRLCU_ESTATE, "irlcu_init has not been called");
  return IRLCU_OK;
}

// internal [y][z][x] -> external [z][y][x] (irl.h layout); x stays contiguous
__global__ void k_to_external(const float *__restrict__ in, float *__restrict__ out, int n, int nz) {
  const size_t vox = (size_t)n * nz * n;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < vox; e += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(e % n);
    const size_t r = e / n;
    const int z = (int)(r % nz), y = (int)(r / nz);
    out[((size_t)z * n + y) * n + x] = in[e];
  }
}

// the inverse of k_to_external, with irlosem.c's scaling and clamp of the
// attenuation map folded in (one float multiply, then x < 0 -> +0)
__global__ void k_from_external(const float *__restrict__ in, float *__restrict__ out, int n, int nz, float scale,
                                int clamp) {
  const size_t vox = (size_t)n * nz * n;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < vox; e += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(e % n);
    const size_t r = e / n;
    const int z = (int)(r % nz), y = (int)(r / nz);
    float v = in[((size_t)z * n + y) * n + x];
    if (scale > 0.0f && scale != 1.0f) v = __fmul_rn(v, scale);
    if (clamp && v < 0.0f) v = 0.0f;
    out[e] = v;
  }
}

}  // namespace irlcu

using namespace irlcu;

extern "C" {

const char *irlcu_error_string(void) { return g_err; }

int irlcu_init(const irlcu_geom *g) {
  if (g_ctx) irlcu_shutdown();
  if (!g || g->n <= 0 || g->nz <= 0 || g->nviews <= 0)
    return set_error(IRLCU_EARG, "bad geometry");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(IRLCU_ECUDA, "no CUDA device is available; libirl_b200 has no CPU path");
  Ctx *c = new Ctx();
  c->g = *g;
  if (c->g.max_batch <= 0) c->g.max_batch = 16;
  if (c->g.max_batch > g->nviews) c->g.max_batch = g->nviews;
  c->n = g->n;
  c->nz = g->nz;
  c->nv = g->nviews;
  c->pln = (size_t)c->nz * c->n;
  c->vox = c->pln * c->n;
  g_ctx = c;
  CU_TRY(cudaGetDevice(&c->dev));
  CU_TRY(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  CU_TRY(cudaStreamCreateWithFlags(&c->up_st, cudaStreamNonBlocking));
  for (auto &e : c->ev) CU_TRY(cudaEventCreate(&e));
  const int n = c->n, R = 2 * c->nv;
  TRY(dalloc(&c->rot.hdr, (size_t)4 * R));
  TRY(dalloc(&c->rot.row_sh, (size_t)n * R));
  TRY(dalloc(&c->rot.row_f1, (size_t)n * R));
  TRY(dalloc(&c->rot.row_f2, (size_t)n * R));
  TRY(dalloc(&c->rot.col_sh, (size_t)2 * n * R));
  TRY(dalloc(&c->rot.col_f1, (size_t)2 * n * R));
  TRY(dalloc(&c->rot.col_f2, (size_t)2 * n * R));
  TRY(dalloc(&c->rot.sn, (size_t)R));
  TRY(dalloc(&c->rot.cs, (size_t)R));
  TRY(dalloc(&c->sup_start, (size_t)n));
  TRY(dalloc(&c->sup_end, (size_t)n));
  {
    std::vector<int> st(n), en(n);
    irl_shear_support(n, st.data(), en.data());
    CU_TRY(cudaMemcpyAsync(c->sup_start, st.data(), n * sizeof(int), cudaMemcpyHostToDevice, alloc_stream()));
    CU_TRY(cudaMemcpyAsync(c->sup_end, en.data(), n * sizeof(int), cudaMemcpyHostToDevice, alloc_stream()));
  }
  const int B = c->g.max_batch;
  TRY(dalloc(&c->est, c->vox));
  TRY(dalloc(&c->upd, c->vox));
  TRY(dalloc(&c->prj, c->pln * c->nv));
  TRY(dalloc(&c->colmask, (size_t)c->nv * n));
  TRY(dalloc(&c->wrot, c->vox * B));
  TRY(dalloc(&c->wbck, c->vox * B));
  TRY(dalloc(&c->wprj, c->pln * B));
  TRY(dalloc(&c->wprj2, c->pln * B * 2));
  c->wpart_elems = forward_partial_elems(n, c->nz, B);
  TRY(dalloc(&c->wpart, c->wpart_elems));
  TRY(dalloc(&c->dviews, (size_t)c->nv));
  TRY(dalloc(&c->dvp, (size_t)c->nv));
  CU_TRY(cudaMemsetAsync(c->prj, 0, c->pln * c->nv * sizeof(float), alloc_stream()));
  CU_TRY(cudaMemsetAsync(c->upd, 0, c->vox * sizeof(float), alloc_stream()));
  std::vector<unsigned char> ones((size_t)c->nv * n, 3);
  CU_TRY(cudaMemcpyAsync(c->colmask, ones.data(), ones.size(), cudaMemcpyHostToDevice, alloc_stream()));
  // the buffers are zeroed before irlcu_upload_now may write them from the
  // copy stream
  CU_TRY(cudaStreamSynchronize(c->st));
  return IRLCU_OK;
}

void irlcu_shutdown(void) {
  free_ctx(g_ctx);
  g_ctx = nullptr;
}

int irlcu_set_angles(const float *angles) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  const int n = c.n, R = 2 * c.nv;
  std::vector<int> hdr(4 * R), rsh((size_t)n * R), csh((size_t)2 * n * R);
  std::vector<float> rf1((size_t)n * R), rf2((size_t)n * R), cf1((size_t)2 * n * R), cf2((size_t)2 * n * R);
  std::vector<float> sn(R), cs(R);
  for (int r = 0; r < R; ++r) {
    const float a = angles[r % c.nv];
    // libirl passes 0.5*M_PI+fAngle and -0.5*M_PI-fAngle (double) to a
    // float parameter (prjbck.c:131, 409; rot3dpar: prjbck.c:135, 413)
    const float ang = r < c.nv ? (float)(0.5 * M_PI + a) : (float)(-0.5 * M_PI - a);
    irl_shear_tab t;
    t.row_sh = &rsh[(size_t)r * n];
    t.row_f1 = &rf1[(size_t)r * n];
    t.row_f2 = &rf2[(size_t)r * n];
    t.col_sh = &csh[(size_t)r * 2 * n];
    t.col_f1 = &cf1[(size_t)r * 2 * n];
    t.col_f2 = &cf2[(size_t)r * 2 * n];
    irl_shear_table(ang, n, &t);
    if (t.mdim > 2 * n) return set_error(IRLCU_EARG, "shear margin too large");
    if (t.mdim > c.max_mdim) c.max_mdim = t.mdim;
    hdr[4 * r] = t.b90;
    hdr[4 * r + 1] = t.b180;
    hdr[4 * r + 2] = t.iadd;
    hdr[4 * r + 3] = t.mdim;
    const float ang3 = r < c.nv ? (float)(0.5 * M_PI + a) : (float)(-a - 0.5 * M_PI);
    irl_rot3dpar_sincos(ang3, &sn[r], &cs[r]);
  }
  CU_TRY(cudaMemcpyAsync(c.rot.hdr, hdr.data(), hdr.size() * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.row_sh, rsh.data(), rsh.size() * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.row_f1, rf1.data(), rf1.size() * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.row_f2, rf2.data(), rf2.size() * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.col_sh, csh.data(), csh.size() * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.col_f1, cf1.data(), cf1.size() * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.col_f2, cf2.data(), cf2.size() * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.sn, sn.data(), sn.size() * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.cs, cs.data(), cs.size() * 4, cudaMemcpyHostToDevice, alloc_stream()));
  return IRLCU_OK;
}

// ------------------------------------------------------ shape autotuner
// The three-shear rotation has two kernel shapes: one slice per CTA (two
// CTAs per SM) and two slices per CTA (one 1024-thread CTA per SM, shared
// index work).  Which is faster depends on where a launch finds its
// source and on what runs around it, which a stand-alone timing at set-up
// did not reproduce.  So the shapes are tried on the real work: the first
// two whole iterations of a context (irlcu_osem_iteration) run eagerly, the
// first with the one-slice and the second with the two-slice kernel, every
// rotation launch timed with events, per source kind (one volume shared by
// all views: the estimate; a volume per view: the backprojections).  From
// the third iteration on, each kind keeps the shape with the smaller total,
// before any iteration is captured into a graph.  Both shapes give the
// same bits, so the trial iterations are ordinary iterations.
// IRLCU_SHEAR_PAIR = 0 / 1 skips the trial and forces a shape.
static float g_shear_ms[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
static int g_shear_form[2] = {-1, -1};
static bool g_shape_trials = true;  // off inside IrlOsemBatch (no host waits)
struct ShearKey {
  int n, nz, batch;
  bool operator==(const ShearKey &o) const { return n == o.n && nz == o.nz && batch == o.batch; }
};
static std::vector<std::pair<ShearKey, std::array<int, 2>>> g_shear_cache;  // per geometry, for the process

// sums the finished trial iteration's launch times into trial_ms[.][form]
static int shear_trial_collect(Ctx &c, int form) {
  for (int kind = 0; kind < 2; ++kind) {
    float tot = 0.f;
    for (auto &e : c.trial_ev[kind]) {
      float ms = 0.f;
      if (cudaEventSynchronize(e.second) == cudaSuccess && cudaEventElapsedTime(&ms, e.first, e.second) == cudaSuccess)
        tot += ms;
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
    c.trial_ev[kind].clear();
    c.trial_ms[kind][form] = tot;
  }
  return IRLCU_OK;
}

// advances the trial before iteration launches; returns true while the
// coming iteration is a trial iteration (to be run eagerly)
static bool shear_trial_step(Ctx &c) {
  if (!c.g.fast_rotate || c.shear_trial >= 3 || getenv("IRLCU_SHEAR_PAIR")) return false;
  const ShearKey key{c.n, c.nz, std::min(c.g.max_batch, c.nv)};
  if (c.shear_trial == 0) {
    for (const auto &e : g_shear_cache)
      if (e.first == key) {
        c.shear_form[0] = e.second[0];
        c.shear_form[1] = e.second[1];
        c.shear_trial = 3;
        return false;
      }
    if (!g_shape_trials) return false;
    c.trial_form = 0;
    c.shear_trial = 1;
    return true;
  }
  shear_trial_collect(c, c.trial_form);
  if (c.shear_trial == 1) {
    c.trial_form = 1;
    c.shear_trial = 2;
    return true;
  }
  c.trial_form = -1;
  c.shear_trial = 3;
  for (int kind = 0; kind < 2; ++kind) {
    const float one = c.trial_ms[kind][0], two = c.trial_ms[kind][1];
    c.shear_form[kind] = (two > 0.f && two < one) ? 1 : 0;
    g_shear_ms[kind][0] = one;
    g_shear_ms[kind][1] = two;
    g_shear_form[kind] = c.shear_form[kind];
  }
  g_shear_cache.push_back({key, {c.shear_form[0], c.shear_form[1]}});
  return false;
}

int irlcu_mem_info(size_t *free_bytes, size_t *total_bytes) {
  size_t fr = 0, tot = 0;
  CU_TRY(cudaMemGetInfo(&fr, &tot));
  // blocks the stream-ordered pool keeps for reuse count as free
  int dev = 0;
  cudaMemPool_t pool;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
      fr += (size_t)(reserved - used);
  }
  if (free_bytes) *free_bytes = fr;
  if (total_bytes) *total_bytes = tot;
  return IRLCU_OK;
}

static bool g_graphs_on = true;  // off inside IrlOsemBatch (eager iterations)

int irlcu_iteration_graphs(int on) {
  const int prev = g_graphs_on ? 1 : 0;
  g_graphs_on = on != 0;
  return prev;
}

int irlcu_shape_trials(int on) {
  const int prev = g_shape_trials ? 1 : 0;
  g_shape_trials = on != 0;
  return prev;
}

int irlcu_shear_tuning(float ms[4], int form[2]) {
  for (int k = 0; k < 2; ++k) {
    ms[2 * k] = g_shear_ms[k][0];
    ms[2 * k + 1] = g_shear_ms[k][1];
    form[k] = g_shear_form[k];
  }
  return IRLCU_OK;
}

// ------------------------------------------------------------ autotuner
// DRF engine per table: the direct kernels and the Fourier-domain engine
// compute the same convolution; which is faster depends on the PSF size,
// the plane size and the batch.  One projection plus backprojection of a
// subset batch (views 0 .. B-1 of this geometry) is timed with each, after
// one untimed run, and the faster is kept.  Decisions are cached per
// (n, nz, half-width, distances, pad, batch, views) for the process.
enum { ENGINE_TUNE = 0, ENGINE_DIRECT = 1, ENGINE_FFT = 2 };

struct TuneKey {
  int n, nz, halo, ndist, pad, batch, nv;
  bool operator==(const TuneKey &o) const {
    return n == o.n && nz == o.nz && halo == o.halo && ndist == o.ndist && pad == o.pad && batch == o.batch &&
           nv == o.nv;
  }
};
static std::vector<std::pair<TuneKey, bool>> g_tune_cache;
static float g_tune_ms[2] = {0.f, 0.f};  // last timing: direct, Fourier domain

static int upload_views(const int *views, int nv, const irlcu_view_parm *vp);

static int time_drf(Ctx &c, const DrfDev &D, int B, float *ms) {
  for (int rep = 0; rep < 2; ++rep) {
    if (rep == 1) CU_TRY(cudaEventRecord(c.ev[4], c.st));
    TRY(launch_project(c, c.wrot, c.dviews, B, nullptr, &D, 1.0f, c.wprj));
    TRY(launch_backproject(c, c.wprj, c.dviews, B, nullptr, &D, 1.0f, c.wbck));
  }
  CU_TRY(cudaEventRecord(c.ev[5], c.st));
  CU_TRY(cudaEventSynchronize(c.ev[5]));
  CU_TRY(cudaEventElapsedTime(ms, c.ev[4], c.ev[5]));
  return IRLCU_OK;
}

static int drf_autotune(Ctx &c, DrfDev &D, int max_pad, bool *fft) {
  const int B = std::min(c.g.max_batch, c.nv);
  const TuneKey key{c.n, c.nz, D.halo, D.ndist, max_pad, B, c.nv};
  for (const auto &e : g_tune_cache)
    if (e.first == key) {
      *fft = e.second;
      return IRLCU_OK;
    }
  std::vector<int> views(B);
  for (int i = 0; i < B; ++i) views[i] = i;
  TRY(upload_views(views.data(), B, nullptr));
  CU_TRY(cudaMemsetAsync(c.wrot, 0, sizeof(float) * c.vox * B, c.st));
  D.fft.on = false;
  TRY(time_drf(c, D, B, &g_tune_ms[0]));
  D.fft.on = true;
  TRY(time_drf(c, D, B, &g_tune_ms[1]));
  *fft = g_tune_ms[1] < g_tune_ms[0];
  D.fft.on = *fft;
  g_tune_cache.push_back({key, *fft});
  return IRLCU_OK;
}

int irlcu_set_drf(int which, const irlcu_drf *d) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  if (which < 0 || which > 1) return set_error(IRLCU_EARG, "bad DRF slot %d", which);
  DrfDev &D = c.drf[which];
  dfree(D.psf);
  dfree(D.pad_rows);
  dfree(D.row_idist);
  drf_fft_free(c, D);
  D = DrfDev{};
  if (!d) return IRLCU_OK;
  // engine: the direct kernels take half-widths up to 32, the Fourier-domain
  // engine any that fits its grid.  IRLCU_DRF_ENGINE = direct | fft | auto;
  // auto (the default) times both on this table and keeps the faster
  const int Hd = halo_instance(d->halo);
  const char *eng = getenv("IRLCU_DRF_ENGINE");
  int mode = ENGINE_TUNE;
  if (eng && !strcmp(eng, "direct")) mode = ENGINE_DIRECT;
  if (eng && !strcmp(eng, "fft")) mode = ENGINE_FFT;
  if (Hd < 0) {
    if (mode == ENGINE_DIRECT)
      return set_error(IRLCU_EARG, "DRF half-width %d exceeds the direct-convolution limit (32)", d->halo);
    mode = ENGINE_FFT;
  }
  const int H = Hd >= 0 ? Hd : d->halo;
  const int PW = 2 * H + 1, PLD = (PW + 3) & ~3, w = 2 * d->halo + 1;
  std::vector<float> pad((size_t)d->ndist * PW * PLD, 0.f);
  for (int i = 0; i < d->ndist; ++i)
    for (int yy = 0; yy < w; ++yy)
      for (int xx = 0; xx < w; ++xx)
        pad[(size_t)i * PW * PLD + (size_t)(yy + H - d->halo) * PLD + (xx + H - d->halo)] =
            d->psf[(size_t)i * w * w + (size_t)yy * w + xx];
  TRY(dalloc(&D.psf, pad.size()));
  CU_TRY(cudaMemcpyAsync(D.psf, pad.data(), pad.size() * 4, cudaMemcpyHostToDevice, alloc_stream()));
  TRY(dalloc(&D.pad_rows, (size_t)d->ndist));
  CU_TRY(cudaMemcpyAsync(D.pad_rows, d->pad_rows, d->ndist * 4, cudaMemcpyHostToDevice, alloc_stream()));
  TRY(dalloc(&D.row_idist, (size_t)c.nv * c.n));
  CU_TRY(cudaMemcpyAsync(D.row_idist, d->row_idist, (size_t)c.nv * c.n * 4, cudaMemcpyHostToDevice, alloc_stream()));
  D.ndist = d->ndist;
  D.halo = H;
  D.pstride = PLD;
  D.avg_rows = d->avg_rows;
  D.h_rows.assign(d->row_idist, d->row_idist + (size_t)c.nv * c.n);
  D.h_taps.resize(d->ndist);
  for (int i = 0; i < d->ndist; ++i) D.h_taps[i] = d->taps ? d->taps[i] : w * w;
  if (mode != ENGINE_DIRECT) {
    int max_pad = 0;
    if (d->avg_rows > 0)
      for (int i = 0; i < d->ndist; ++i) max_pad = std::max(max_pad, d->pad_rows[i]);
    TRY(drf_fft_setup(c, D, max_pad));
    if (mode == ENGINE_TUNE) {
      bool fft = true;
      TRY(drf_autotune(c, D, max_pad, &fft));
      if (!fft) drf_fft_free(c, D);
    }
  }
  return IRLCU_OK;
}

int irlcu_set_column_mask(const unsigned char *mask) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  CU_TRY(cudaMemcpyAsync(c.colmask, mask, (size_t)c.nv * c.n, cudaMemcpyHostToDevice, alloc_stream()));
  return IRLCU_OK;
}

static int buf_ptr(int buf, int index, float **p, size_t *count, bool alloc) {
  Ctx &c = *g_ctx;
  switch (buf) {
    case IRLCU_BUF_EST: *p = c.est; *count = c.vox; return IRLCU_OK;
    case IRLCU_BUF_UPDATE: *p = c.upd; *count = c.vox; return IRLCU_OK;
    case IRLCU_BUF_PRJ: *p = c.prj; *count = c.pln * c.nv; return IRLCU_OK;
    case IRLCU_BUF_ATN:
      if (!c.atn && alloc) TRY(dalloc(&c.atn, c.vox));
      *p = c.atn; *count = c.vox; return IRLCU_OK;
    case IRLCU_BUF_SCATEST:
      if (!c.scatest && alloc) TRY(dalloc(&c.scatest, c.pln * c.nv));
      *p = c.scatest; *count = c.pln * c.nv; return IRLCU_OK;
    case IRLCU_BUF_PRJSCAT:
      if (!c.prjscat && alloc) {
        TRY(dalloc(&c.prjscat, c.pln * c.nv));
        CU_TRY(cudaMemsetAsync(c.prjscat, 0, c.pln * c.nv * 4, alloc_stream()));
      }
      *p = c.prjscat; *count = c.pln * c.nv; return IRLCU_OK;
    case IRLCU_BUF_NORM:
      if (index < 0 || index >= c.nsub) return set_error(IRLCU_EARG, "norm index %d out of range", index);
      *p = c.norm + (size_t)index * c.vox; *count = c.vox; return IRLCU_OK;
  }
  return set_error(IRLCU_EARG, "unknown buffer %d", buf);
}

int irlcu_upload(int buf, int index, const float *host, size_t count) {
  TRY(need_ctx());
  float *p;
  size_t cap;
  TRY(buf_ptr(buf, index, &p, &cap, true));
  if (count > cap) return set_error(IRLCU_EARG, "upload of %zu floats exceeds buffer %d (%zu)", count, buf, cap);
  CU_TRY(cudaMemcpyAsync(p, host, count * 4, cudaMemcpyHostToDevice, g_ctx->st));
  CU_TRY(cudaStreamSynchronize(g_ctx->st));
  return IRLCU_OK;
}

int irlcu_upload_now(int buf, int index, const float *host, size_t count) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  CU_TRY(cudaSetDevice(c.dev));  // the calling thread may be a helper thread
  float *p;
  size_t cap;
  TRY(buf_ptr(buf, index, &p, &cap, false));
  if (!p) return set_error(IRLCU_ESTATE, "buffer %d not allocated", buf);
  if (count > cap) return set_error(IRLCU_EARG, "upload of %zu floats exceeds buffer %d (%zu)", count, buf, cap);
  CU_TRY(cudaMemcpyAsync(p, host, count * 4, cudaMemcpyHostToDevice, c.up_st));
  CU_TRY(cudaStreamSynchronize(c.up_st));
  return IRLCU_OK;
}

int irlcu_download(int buf, int index, float *host, size_t count) {
  TRY(need_ctx());
  float *p;
  size_t cap;
  TRY(buf_ptr(buf, index, &p, &cap, false));
  if (!p) return set_error(IRLCU_ESTATE, "buffer %d not allocated", buf);
  if (count > cap) return set_error(IRLCU_EARG, "download of %zu floats exceeds buffer %d", count, buf);
  CU_TRY(cudaMemcpyAsync(host, p, count * 4, cudaMemcpyDeviceToHost, g_ctx->st));
  CU_TRY(cudaStreamSynchronize(g_ctx->st));
  if (g_ctx->sur) TRY(sur_tc_status(g_ctx->st));
  return IRLCU_OK;
}

int irlcu_zero(int buf, int index) {
  TRY(need_ctx());
  float *p;
  size_t cap;
  TRY(buf_ptr(buf, index, &p, &cap, true));
  CU_TRY(cudaMemsetAsync(p, 0, cap * 4, g_ctx->st));
  return IRLCU_OK;
}

int irlcu_download_external(int buf, float *host) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  float *p;
  size_t cap;
  TRY(buf_ptr(buf, 0, &p, &cap, false));
  if (!p || cap != c.vox) return set_error(IRLCU_EARG, "buffer %d is not a volume", buf);
  k_to_external<<<592, 256, 0, c.st>>>(p, c.wbck, c.n, c.nz);
  CU_LAUNCHED();
  CU_TRY(cudaMemcpyAsync(host, c.wbck, c.vox * 4, cudaMemcpyDeviceToHost, c.st));
  CU_TRY(cudaStreamSynchronize(c.st));
  if (c.sur) TRY(sur_tc_status(c.st));
  return IRLCU_OK;
}

int irlcu_upload_external(int buf, const float *host, float scale, int clamp) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  float *p;
  size_t cap;
  TRY(buf_ptr(buf, 0, &p, &cap, true));
  if (!p || cap != c.vox) return set_error(IRLCU_EARG, "buffer %d is not a volume", buf);
  // into wbck (vox * max_batch floats); the host array is free once the
  // copy has landed, before the transposition is queued
  CU_TRY(cudaMemcpyAsync(c.wbck, host, c.vox * 4, cudaMemcpyHostToDevice, c.st));
  CU_TRY(cudaStreamSynchronize(c.st));
  k_from_external<<<592, 256, 0, c.st>>>(c.wbck, p, c.n, c.nz, scale, clamp);
  CU_LAUNCHED();
  return IRLCU_OK;
}

// The iteration callback's copy of the estimate without stalling the
// device: the external-layout snapshot is taken on the context stream right
// after the iteration's kernels, then copied to pinned host memory on a
// stream of its own, so that the next iteration's kernels (queued by the
// host meanwhile) run during the copy and the callback.
// The pinned host pair is kept for the process and reused by every later
// context (pinning 2 x 8 MB takes milliseconds, more than a short
// reconstruction's callbacks save).  Only the session with a callback uses
// it, one at a time, and a context waits for its copies before it ends.
static float *g_pin[2] = {nullptr, nullptr};
static size_t g_pin_cap = 0;

int irlcu_snapshot_begin(int slot) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  if (slot < 0 || slot > 1) return set_error(IRLCU_EARG, "snapshot slot %d", slot);
  if (!c.est) return set_error(IRLCU_ESTATE, "no estimate to snapshot");
  if (!c.snap_st) CU_TRY(cudaStreamCreateWithFlags(&c.snap_st, cudaStreamNonBlocking));
  if (g_pin_cap < c.vox) {
    for (int k = 0; k < 2; ++k) {
      if (g_pin[k]) CU_TRY(cudaFreeHost(g_pin[k]));
      g_pin[k] = nullptr;
    }
    g_pin_cap = 0;
    for (int k = 0; k < 2; ++k) CU_TRY(cudaMallocHost(&g_pin[k], c.vox * sizeof(float)));
    g_pin_cap = c.vox;
  }
  if (!c.snap[slot]) {
    TRY(dalloc(&c.snap[slot], c.vox));
    CU_TRY(cudaEventCreateWithFlags(&c.snap_made[slot], cudaEventDisableTiming));
    CU_TRY(cudaEventCreateWithFlags(&c.snap_copied[slot], cudaEventDisableTiming));
  }
  c.snap_host[slot] = g_pin[slot];
  k_to_external<<<592, 256, 0, c.st>>>(c.est, c.snap[slot], c.n, c.nz);
  CU_LAUNCHED();
  CU_TRY(cudaEventRecord(c.snap_made[slot], c.st));
  CU_TRY(cudaStreamWaitEvent(c.snap_st, c.snap_made[slot], 0));
  CU_TRY(cudaMemcpyAsync(c.snap_host[slot], c.snap[slot], c.vox * sizeof(float), cudaMemcpyDeviceToHost, c.snap_st));
  CU_TRY(cudaEventRecord(c.snap_copied[slot], c.snap_st));
  return IRLCU_OK;
}

int irlcu_snapshot_end(int slot, float **host) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  if (slot < 0 || slot > 1 || !c.snap_copied[slot]) return set_error(IRLCU_ESTATE, "no snapshot in slot %d", slot);
  CU_TRY(cudaEventSynchronize(c.snap_copied[slot]));
  *host = c.snap_host[slot];
  return IRLCU_OK;
}

int irlcu_alloc_norm(int nsubsets) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  dfree(c.norm);
  c.nsub = 0;
  TRY(dalloc(&c.norm, c.vox * nsubsets));
  c.nsub = nsubsets;
  return IRLCU_OK;
}

static int upload_views(const int *views, int nv, const irlcu_view_parm *vp) {
  Ctx &c = *g_ctx;
  if (nv <= 0 || nv > c.g.max_batch) return set_error(IRLCU_EARG, "batch of %d views (max %d)", nv, c.g.max_batch);
  for (int i = 0; i < nv; ++i)
    if (views[i] < 0 || views[i] >= c.nv) return set_error(IRLCU_EARG, "view index %d out of range", views[i]);
  CU_TRY(cudaMemcpyAsync(c.dviews, views, nv * sizeof(int), cudaMemcpyHostToDevice, c.st));
  if (vp) CU_TRY(cudaMemcpyAsync(c.dvp, vp, nv * sizeof(irlcu_view_parm), cudaMemcpyHostToDevice, c.st));
  return IRLCU_OK;
}

// the surrogate's iteration-invariant input channels of every view, from
// the current per-view mu and S tables (not inside a graph capture)
static int sur_static_ensure(Ctx &c) {
  if (c.sur_static_ok || !c.tMu || !c.tS || c.n % (4 * SUR_P) || c.n != c.nz) return IRLCU_OK;
  const size_t P = (size_t)SUR_P * SUR_P * SUR_P;
  if (!c.sur_static) TRY(dalloc(&c.sur_static, (size_t)c.nv * P));  // one BF16 pair per float
  TRY(launch_sur_static(c.st, c.tMu, c.tS, c.nv, c.n, c.vox, c.sur_static));
  c.sur_static_ok = true;
  return IRLCU_OK;
}

int irlcu_prepare_attenuation(int need_srf) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  if (!c.atn) return set_error(IRLCU_ESTATE, "attenuation map not uploaded");
  c.sur_static_ok = false;
  if (!c.tE) TRY(dalloc(&c.tE, c.vox * c.nv));
  if (need_srf) {
    if (!c.tS) TRY(dalloc(&c.tS, c.vox * c.nv));
    if (!c.tMu) TRY(dalloc(&c.tMu, c.vox * c.nv));
  }
  const int B = c.g.max_batch;
  std::vector<int> views(B);
  for (int v0 = 0; v0 < c.nv; v0 += B) {
    const int nb = std::min(B, c.nv - v0);
    for (int i = 0; i < nb; ++i) views[i] = v0 + i;
    TRY(upload_views(views.data(), nb, nullptr));
    float *rmu = need_srf ? c.tMu + (size_t)v0 * c.vox : c.wrot;
    TRY(launch_rotate(c, c.atn, 0, rmu, c.vox, c.dviews, nb, 0));
    TRY(launch_atn_tables(c, rmu, c.tE + (size_t)v0 * c.vox, need_srf ? c.tS + (size_t)v0 * c.vox : nullptr, nb));
  }
  if (need_srf && c.sur) TRY(sur_static_ensure(c));
  return IRLCU_OK;
}

// rotated source of the batch in wrot (act) and, with SRF, act+scatter in src
// any view of the batch kept on ESSE
static bool sur_flagged(const Ctx &c, const int *hviews, int nv) {
  if (c.sur_flags.empty()) return false;
  for (int i = 0; i < nv; ++i)
    if (c.sur_flags[hviews[i]]) return true;
  return false;
}

static int forward_batch(int nv, const int *hviews, int model, float primary, float *out, float *out_nosrf) {
  Ctx &c = *g_ctx;
  RotCollapse col;
  {
    Stage s(IRLCU_ST_ROTATE, c.st);
    s.bytes = 8.0 * (double)c.vox * nv;  // read the estimate, write each rotated copy
    // ESSE's collapse of the rotated volumes rides on the rotation when this
    // batch takes the ESSE path
    const bool esse_path = (model & MODEL_SRF_BIT) && c.esse.on && !(c.sur && !sur_flagged(c, hviews, nv));
    if (!esse_path || !esse_collapse_target(c, nv, &col)) col.out = nullptr;
    TRY(launch_rotate(c, c.est, 0, c.wrot, c.vox, c.dviews, nv, 0, col.out ? &col : nullptr));
  }
  const float *E = (model & MODEL_ATN_BIT) ? c.tE : nullptr;
  const DrfDev *drf = (model & MODEL_DRF_BIT) ? &c.drf[0] : nullptr;
  const float *src = c.wrot;
  float scale = primary;
  if ((model & MODEL_SRF_BIT) && c.sur && c.esse.on && !sur_flagged(c, hviews, nv)) {
    // learned scatter: primary projection + the network's scatter projection
    {
      Stage s(IRLCU_ST_PROJECT, c.st);
      s.flops = drf_flops(c, drf, hviews, nv, true);
      s.bytes = (E ? 8.0 : 4.0) * (double)c.vox * nv;
      TRY(launch_project(c, c.wrot, c.dviews, nv, E, drf, primary, out));
    }
    if (out_nosrf)
      CU_TRY(cudaMemcpyAsync(out_nosrf, out, sizeof(float) * c.pln * nv, cudaMemcpyDeviceToDevice, c.st));
    Stage s(IRLCU_ST_ESSE, c.st);
    if (c.sur_static_ok)
      TRY(launch_sur_inputs_static(c.st, c.wrot, c.vox, c.sur_static, c.dviews, nv, c.n, c.sur_scale,
                                   sur_input(c.sur), c.sur_work));
    else
      TRY(launch_sur_inputs(c.st, c.wrot, c.vox, c.tMu, c.tS, c.dviews, nv, c.n, c.vox, c.sur_scale,
                            sur_input(c.sur), c.sur_work));
    const float *y = nullptr;
    TRY(sur_infer(c.sur, c.st, nv, &y));
    return launch_scale_views_up(c.st, y, c.sur_scale, out, c.n, nv, 1);
  }
  if (model & MODEL_SRF_BIT) {
    if (!c.esse.on && !c.esse.zero) return set_error(IRLCU_ESTATE, "scatter model requested but not set up");
    if (!c.tS) return set_error(IRLCU_ESTATE, "scatter model needs the attenuation tables");
    Stage s(IRLCU_ST_ESSE, c.st);
    TRY(launch_esse(c, c.wrot, c.dviews, nv, primary, c.wbck, col.done));
    src = c.wbck;
    scale = 1.0f;
  }
  for (int pass = 0; pass < (out_nosrf ? 2 : 1); ++pass) {
    Stage s(IRLCU_ST_PROJECT, c.st);
    s.flops = drf_flops(c, drf, hviews, nv, true);
    // algorithmic bytes: source and attenuation factor of every plane
    s.bytes = (E ? 8.0 : 4.0) * (double)c.vox * nv;
    if (pass == 0)
      TRY(launch_project(c, src, c.dviews, nv, E, drf, scale, out));
    else
      TRY(launch_project(c, c.wrot, c.dviews, nv, E, drf, primary, out_nosrf));
  }
  return IRLCU_OK;
}

int irlcu_project(int nv, const int *views, int model, float primary_fac, float *dst, int dst_on_device) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  for (int v0 = 0; v0 < nv; v0 += c.g.max_batch) {
    const int nb = std::min(c.g.max_batch, nv - v0);
    TRY(upload_views(views + v0, nb, nullptr));
    TRY(forward_batch(nb, views + v0, model, primary_fac, c.wprj, nullptr));
    CU_TRY(cudaMemcpyAsync(dst + (size_t)v0 * c.pln, c.wprj, (size_t)nb * c.pln * 4,
                           dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c.st));
  }
  CU_TRY(cudaStreamSynchronize(c.st));
  return IRLCU_OK;
}

// the device work of one subset batch whose views and parameters are at
// c.dviews / c.dvp; hviews: the same view indices on the host (accounting)
static int osem_subset_body(int nv, const int *hviews, bool need_nosrf, int model, int bck_model, int subset,
                            int use_scatest, int apply_update, int accumulate_from_update) {
  Ctx &c = *g_ctx;
  float *calc = c.wprj;
  float *calc_nosrf = c.wprj2;
  float *ratio = c.wprj2 + c.pln * c.g.max_batch;
  if (!c.capturing) CU_TRY(cudaEventRecord(c.ev[0], c.st));
  TRY(forward_batch(nv, hviews, model, 1.0f, calc, need_nosrf ? calc_nosrf : nullptr));
  if (!c.capturing) CU_TRY(cudaEventRecord(c.ev[1], c.st));
  {
    Stage s(IRLCU_ST_REDUCE, c.st);
    s.bytes = 16.0 * (double)c.pln * nv;
    TRY(launch_ratio(c, calc, calc_nosrf, c.dviews, c.dvp, nv, use_scatest, ratio));
  }
  const float *E = (bck_model & MODEL_ATN_BIT) ? c.tE : nullptr;
  const DrfDev *drf = nullptr;
  if (bck_model & MODEL_DRF_BIT) drf = c.drf[1].psf ? &c.drf[1] : &c.drf[0];
  {
    Stage s(IRLCU_ST_BACKPROJECT, c.st);
    s.flops = drf_flops(c, drf, hviews, nv, false);
    s.bytes = (E ? 8.0 : 4.0) * (double)c.vox * nv;  // attenuation factor read, plane written
    TRY(launch_backproject(c, ratio, c.dviews, nv, E, drf, 1.0f, c.wbck));
  }
  if (!c.capturing) CU_TRY(cudaEventRecord(c.ev[2], c.st));
  {
    Stage s(IRLCU_ST_ACCUM, c.st);
    // unrotation (read + write per view), accumulation read per view, and
    // the update / estimate read-modify-write
    s.bytes = 12.0 * (double)c.vox * nv + 16.0 * (double)c.vox;
    TRY(launch_unrotate_accumulate(c, c.wbck, c.dviews, nv, c.upd, accumulate_from_update,
                                   apply_update ? ACC_EM : 0, c.est,
                                   apply_update ? c.norm + (size_t)subset * c.vox : nullptr));
  }
  if (!c.capturing) CU_TRY(cudaEventRecord(c.ev[3], c.st));
  return IRLCU_OK;
}

static int need_prjscat_buffer(Ctx &c) {
  if (c.prjscat) return IRLCU_OK;
  float *p;
  size_t cap;
  return buf_ptr(IRLCU_BUF_PRJSCAT, 0, &p, &cap, true);
}

int irlcu_osem_subset(int nv, const int *views, const irlcu_view_parm *vp, int model, int bck_model, int subset,
                      int use_scatest, int apply_update, int accumulate_from_update) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  if (apply_update && (subset < 0 || subset >= c.nsub)) return set_error(IRLCU_EARG, "bad subset %d", subset);
  if (use_scatest && !c.scatest) return set_error(IRLCU_ESTATE, "scatter estimate not uploaded");
  bool need_nosrf = false, need_prjscat = false;
  for (int i = 0; i < nv; ++i) {
    need_nosrf |= vp[i].scat_mode == 2;
    need_prjscat |= vp[i].scat_mode != 0;
  }
  if (need_prjscat) TRY(need_prjscat_buffer(c));
  TRY(upload_views(views, nv, vp));
  return osem_subset_body(nv, views, need_nosrf, model, bck_model, subset, use_scatest, apply_update,
                          accumulate_from_update);
}

int irlcu_set_subsets(int nsub, int per, const int *views, const irlcu_view_parm *vp) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  if (nsub <= 0 || per <= 0 || nsub > c.nsub) return set_error(IRLCU_EARG, "bad subsets %d x %d", nsub, per);
  const size_t tot = (size_t)nsub * per;
  for (size_t i = 0; i < tot; ++i)
    if (views[i] < 0 || views[i] >= c.nv) return set_error(IRLCU_EARG, "view index %d out of range", views[i]);
  graphs_clear(c);
  dfree(c.dviews_all);
  dfree(c.dvp_all);
  TRY(dalloc(&c.dviews_all, tot));
  TRY(dalloc(&c.dvp_all, tot));
  c.h_views_all.assign(views, views + tot);
  c.h_vp_all.assign(vp, vp + tot);
  for (auto &q : c.h_vp_all) q.scat_mode = 0;
  c.vp_scat_mode = 0;
  CU_TRY(cudaMemcpyAsync(c.dviews_all, views, tot * sizeof(int), cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.dvp_all, c.h_vp_all.data(), tot * sizeof(irlcu_view_parm), cudaMemcpyHostToDevice, alloc_stream()));
  c.nsub_all = nsub;
  c.per_all = per;
  return IRLCU_OK;
}

// every subset of one iteration, in batches of max_batch views
static int run_subsets(Ctx &c, int model, int bck_model, int use_scatest, int scat_mode) {
  int *dv0 = c.dviews;
  irlcu_view_parm *dp0 = c.dvp;
  int rc = IRLCU_OK;
  const int per = c.per_all, B = c.g.max_batch;
  for (int s = 0; s < c.nsub_all && !rc; ++s)
    for (int m0 = 0; m0 < per && !rc; m0 += B) {
      const int nb = std::min(B, per - m0);
      const size_t off = (size_t)s * per + m0;
      c.dviews = c.dviews_all + off;
      c.dvp = c.dvp_all + off;
      rc = osem_subset_body(nb, c.h_views_all.data() + off, scat_mode == 2, model, bck_model, s, use_scatest,
                            m0 + nb >= per, m0 > 0);
    }
  c.dviews = dv0;
  c.dvp = dp0;
  return rc;
}

int irlcu_osem_iteration(int model, int bck_model, int use_scatest, int scat_mode) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  if (!c.dviews_all) return set_error(IRLCU_ESTATE, "irlcu_set_subsets has not been called");
  if (use_scatest && !c.scatest) return set_error(IRLCU_ESTATE, "scatter estimate not uploaded");
  if (scat_mode < 0 || scat_mode > 2) return set_error(IRLCU_EARG, "bad scatter mode %d", scat_mode);
  if (scat_mode != 0) TRY(need_prjscat_buffer(c));
  if (scat_mode != c.vp_scat_mode) {  // ordered on the stream before this iteration's kernels
    for (auto &q : c.h_vp_all) q.scat_mode = scat_mode;
    CU_TRY(cudaMemcpyAsync(c.dvp_all, c.h_vp_all.data(), c.h_vp_all.size() * sizeof(irlcu_view_parm),
                           cudaMemcpyHostToDevice, c.st));
    c.vp_scat_mode = scat_mode;
  }
  // stage profiling needs the eager launches (events around every stage)
  if (g_prof_on) return run_subsets(c, model, bck_model, use_scatest, scat_mode);
  const int key = (model & 15) | (bck_model & 15) << 4 | (use_scatest ? 1 : 0) << 8 | scat_mode << 9;
  if (shear_trial_step(c)) {  // a shape-autotuner trial iteration: eager, its rotations timed
    bool seen = false;
    for (int k : c.graph_seen) seen |= k == key;
    if (!seen) c.graph_seen.push_back(key);
    return run_subsets(c, model, bck_model, use_scatest, scat_mode);
  }
  for (const GraphRec &g : c.graphs)
    if (g.key == key) {
      CU_TRY(cudaGraphLaunch(g.exec, c.st));
      g_launch_count += g.kernels;
      return IRLCU_OK;
    }
  const char *env = getenv("IRLCU_GRAPHS");
  const bool graphs = g_graphs_on && !(env && !strcmp(env, "0"));
  bool seen = false;
  for (int k : c.graph_seen) seen |= k == key;
  if (!graphs || !seen) {
    if (!seen) c.graph_seen.push_back(key);
    return run_subsets(c, model, bck_model, use_scatest, scat_mode);
  }
  // capture the iteration once, then replay it
  CU_TRY(cudaStreamBeginCapture(c.st, cudaStreamCaptureModeThreadLocal));
  const long long l0 = g_launch_count;
  c.capturing = true;
  const int rc = run_subsets(c, model, bck_model, use_scatest, scat_mode);
  c.capturing = false;
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(c.st, &graph);
  const long long kernels = g_launch_count - l0;
  g_launch_count = l0;
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ce != cudaSuccess) return set_error(IRLCU_ECUDA, "iteration capture: %s", cudaGetErrorString(ce));
  GraphRec g{key, nullptr, kernels};
  const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return set_error(IRLCU_ECUDA, "iteration graph: %s", cudaGetErrorString(ie));
  c.graphs.push_back(g);
  CU_TRY(cudaGraphLaunch(g.exec, c.st));
  g_launch_count += g.kernels;
  return IRLCU_OK;
}

// ------------------------------------------------ learned scatter surrogate

// pooling work buffer of max_batch views
static int sur_work_ensure(Ctx &c) {
  if (c.sur_work) return IRLCU_OK;
  const size_t P = (size_t)SUR_P * SUR_P * SUR_P;
  return dalloc(&c.sur_work, (size_t)c.g.max_batch * (P + SUR_POOL_PARTS));
}

static int sur_geometry(const Ctx &c, irlcu_sur *net, int model) {
  if (!net) return set_error(IRLCU_EARG, "surrogate: null network");
  if ((c.n != 128 && c.n != 256) || c.nz != c.n)
    return set_error(IRLCU_EARG, "surrogate: the network takes 128^3 or 256^3 volumes (here %d x %d)", c.n, c.nz);
  if (!(model & MODEL_SRF_BIT) || !c.esse.on || !c.tS || !c.tMu)
    return set_error(IRLCU_ESTATE, "surrogate: the scatter model (ESSE) must be set up");
  return IRLCU_OK;
}

// ESSE scatter projections of a batch (views at c.dviews) into t; the
// rotated activity stays in c.wrot
static int esse_scatter(Ctx &c, int nv, const int *hviews, int model, float *t) {
  irlcu_sur *keep = c.sur;
  c.sur = nullptr;  // the targets come from ESSE
  const int rc = forward_batch(nv, hviews, model, 1.0f, c.wprj, c.wprj2);
  c.sur = keep;
  TRY(rc);
  return launch_sub(c.st, c.wprj, c.wprj2, t, c.pln * nv);
}

int irlcu_sur_pairs(int nv, const int *views, int model, void *x_out, float *t_out, float *scale_out) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  if (nv < 1 || nv > c.g.max_batch)
    return set_error(IRLCU_EARG, "surrogate pairs: batch %d outside 1..%d", nv, c.g.max_batch);
  if ((c.n != 128 && c.n != 256) || c.nz != c.n)
    return set_error(IRLCU_EARG, "surrogate pairs: 128^3 or 256^3 volumes only");
  if (!(model & MODEL_SRF_BIT) || !c.esse.on || !c.tS || !c.tMu)
    return set_error(IRLCU_ESTATE, "surrogate pairs: ESSE is not set up");
  TRY(upload_views(views, nv, nullptr));
  TRY(esse_scatter(c, nv, views, model, c.wprj));
  TRY(sur_work_ensure(c));
  TRY(launch_sur_inputs(c.st, c.wrot, c.vox, c.tMu, c.tS, c.dviews, nv, c.n, c.vox, scale_out, x_out, c.sur_work));
  TRY(launch_div_views_down(c.st, c.wprj, scale_out, t_out, c.n, nv));
  CU_TRY(cudaStreamSynchronize(c.st));
  return IRLCU_OK;
}

int irlcu_sur_check(irlcu_sur *net, int nv, const int *views, int model, float *nrmse) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  TRY(sur_geometry(c, net, model));
  const int B = std::min(sur_max_batch(net), c.g.max_batch);
  TRY(sur_work_ensure(c));
  float *scale = nullptr;
  TRY(dalloc(&scale, (size_t)B));
  std::vector<float> y(c.pln * B), t(c.pln * B);
  int rc = IRLCU_OK;
  for (int v0 = 0; v0 < nv && !rc; v0 += B) {
    const int nb = std::min(B, nv - v0);
    if ((rc = upload_views(views + v0, nb, nullptr))) break;
    if ((rc = esse_scatter(c, nb, views + v0, model, c.wprj))) break;
    if ((rc = launch_sur_inputs(c.st, c.wrot, c.vox, c.tMu, c.tS, c.dviews, nb, c.n, c.vox, scale, sur_input(net),
                                c.sur_work)))
      break;
    const float *yd = nullptr;
    if ((rc = sur_infer(net, c.st, nb, &yd))) break;
    if ((rc = launch_scale_views_up(c.st, yd, scale, c.wprj2, c.n, nb, 0))) break;
    if (cudaMemcpyAsync(y.data(), c.wprj2, sizeof(float) * c.pln * nb, cudaMemcpyDeviceToHost, c.st) ||
        cudaMemcpyAsync(t.data(), c.wprj, sizeof(float) * c.pln * nb, cudaMemcpyDeviceToHost, c.st) ||
        cudaStreamSynchronize(c.st)) {
      rc = set_error(IRLCU_ECUDA, "surrogate check: copy failed");
      break;
    }
    if ((rc = sur_tc_status(c.st))) break;
    for (int b = 0; b < nb; ++b) {
      double e2 = 0.0, t2 = 0.0;
      for (size_t i = 0; i < c.pln; ++i) {
        const double d = (double)y[b * c.pln + i] - t[b * c.pln + i];
        e2 += d * d;
        t2 += (double)t[b * c.pln + i] * t[b * c.pln + i];
      }
      nrmse[v0 + b] = (float)(t2 > 0 ? std::sqrt(e2 / t2) : (e2 > 0 ? 1.0 : 0.0));
    }
  }
  dfree(scale);
  return rc;
}

int irlcu_set_surrogate(irlcu_sur *net, const unsigned char *flags) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  graphs_clear(c);  // captured iterations may hold the other projector
  if (!net) {
    c.sur = nullptr;
    c.sur_flags.clear();
    return IRLCU_OK;
  }
  TRY(sur_geometry(c, net, MODEL_SRF_BIT));
  if (sur_max_batch(net) < c.g.max_batch)
    return set_error(IRLCU_EARG, "surrogate: network batch %d below the context's %d", sur_max_batch(net),
                     c.g.max_batch);
  if (!c.sur_scale) TRY(dalloc(&c.sur_scale, (size_t)c.g.max_batch));
  TRY(sur_work_ensure(c));
  c.sur = net;
  TRY(sur_static_ensure(c));
  if (flags)
    c.sur_flags.assign(flags, flags + c.nv);
  else
    c.sur_flags.clear();
  return IRLCU_OK;
}

void *irlcu_ctx_detach(void) {
  Ctx *c = g_ctx;
  g_ctx = nullptr;
  return c;
}

int irlcu_ctx_attach(void *ctx) {
  if (g_ctx && g_ctx != ctx) return set_error(IRLCU_ESTATE, "another context is current; detach it first");
  g_ctx = static_cast<Ctx *>(ctx);
  return IRLCU_OK;
}

int irlcu_norm_subset(int nv, const int *views, const float *view_time, int bck_model, int subset) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  if (subset < 0 || subset >= c.nsub) return set_error(IRLCU_EARG, "bad subset %d", subset);
  float *norm = c.norm + (size_t)subset * c.vox;
  CU_TRY(cudaMemsetAsync(norm, 0, c.vox * 4, c.st));
  const int B = c.g.max_batch;
  for (int v0 = 0; v0 < nv; v0 += B) {
    const int nb = std::min(B, nv - v0);
    std::vector<irlcu_view_parm> vp(nb);
    for (int i = 0; i < nb; ++i) vp[i].view_time = view_time[v0 + i];
    TRY(upload_views(views + v0, nb, vp.data()));
    // the per-view times travel in dvp; the mask kernel reads view_time
    float *planes = c.wprj2;
    float *vt = c.wprj;  // nb floats of scratch
    std::vector<float> vth(view_time + v0, view_time + v0 + nb);
    CU_TRY(cudaMemcpyAsync(vt, vth.data(), nb * 4, cudaMemcpyHostToDevice, c.st));
    TRY(launch_norm_planes(c, c.dviews, vt, nb, nullptr, planes));
    const float *E = (bck_model & MODEL_ATN_BIT) ? c.tE : nullptr;
    const DrfDev *drf = nullptr;
    if (bck_model & MODEL_DRF_BIT) drf = c.drf[1].psf ? &c.drf[1] : &c.drf[0];
    TRY(launch_backproject(c, planes, c.dviews, nb, E, drf, 1.0f, c.wbck));
    const bool last = v0 + nb >= nv;
    TRY(launch_unrotate_accumulate(c, c.wbck, c.dviews, nb, norm, 1, last ? ACC_INVERT : 0, nullptr, nullptr));
  }
  return IRLCU_OK;
}

int irlcu_rotate_volume(float angle, const float *src, float *dst, int pb_flag, int on_device) {
  (void)pb_flag;
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  // a one-off rotation through a temporary table slot: use view 0's slots
  // by rebuilding them for this angle
  const int n = c.n;
  std::vector<int> hdr(4), rsh(n), csh(2 * n);
  std::vector<float> rf1(n), rf2(n), cf1(2 * n), cf2(2 * n);
  irl_shear_tab t{0, 0, 0, 0, rsh.data(), rf1.data(), rf2.data(), csh.data(), cf1.data(), cf2.data()};
  irl_shear_table(angle, n, &t);
  if (t.mdim > c.max_mdim) c.max_mdim = t.mdim;
  hdr = {t.b90, t.b180, t.iadd, t.mdim};
  float sn, cs;
  irl_rot3dpar_sincos(angle, &sn, &cs);
  // the last unrotation slot (index 2*nv-1) is borrowed and restored by the
  // caller through irlcu_set_angles when needed
  const int r = 2 * c.nv - 1;
  CU_TRY(cudaMemcpyAsync(c.rot.hdr + 4 * r, hdr.data(), 16, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.row_sh + (size_t)r * n, rsh.data(), n * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.row_f1 + (size_t)r * n, rf1.data(), n * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.row_f2 + (size_t)r * n, rf2.data(), n * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.col_sh + (size_t)r * 2 * n, csh.data(), 2 * n * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.col_f1 + (size_t)r * 2 * n, cf1.data(), 2 * n * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.col_f2 + (size_t)r * 2 * n, cf2.data(), 2 * n * 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.sn + r, &sn, 4, cudaMemcpyHostToDevice, alloc_stream()));
  CU_TRY(cudaMemcpyAsync(c.rot.cs + r, &cs, 4, cudaMemcpyHostToDevice, alloc_stream()));
  int zero = 0;
  TRY(upload_views(&zero, 1, nullptr));
  const float *s = src;
  float *d = dst;
  if (!on_device) {
    CU_TRY(cudaMemcpyAsync(c.wbck, src, c.vox * 4, cudaMemcpyHostToDevice, c.st));
    s = c.wbck;
    d = c.wrot;
  }
  // rot_base chosen so rot_base + views[0] == r
  TRY(launch_rotate(c, s, 0, d, c.vox, c.dviews, 1, r));
  if (!on_device) CU_TRY(cudaMemcpyAsync(dst, c.wrot, c.vox * 4, cudaMemcpyDeviceToHost, c.st));
  CU_TRY(cudaStreamSynchronize(c.st));
  return IRLCU_OK;
}

// Allocates nothing: tables and intermediate live in a static device array
// (k_rotate.cu), for callers that must not allocate device memory (see the
// declaration in irlcu.h).
int irlcu_rotate_volume_noalloc(float angle, const float *src, float *dst, int n, int nz) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  int cur = -1;
  CU_TRY(cudaGetDevice(&cur));
  if (cur != c.dev)
    return set_error(IRLCU_EARG,
                     "irlcu_rotate_volume_noalloc: device %d is current, but the library was initialised on device "
                     "%d; make device %d current first",
                     cur, c.dev, c.dev);
  TRY(launch_rotate_noalloc(c.st, c.dev, angle, src, dst, n, nz));
  CU_TRY(cudaStreamSynchronize(c.st));
  return IRLCU_OK;
}

int irlcu_grids(int out[5]) {
  TRY(need_ctx());
  const Ctx &c = *g_ctx;
  const DrfFft &F = c.drf[0].fft;
  out[0] = F.on ? F.Mz : 0;
  out[1] = F.on ? F.Mx : 0;
  out[2] = c.esse.on ? c.esse.kx : 0;
  out[3] = c.esse.on ? c.esse.ky : 0;
  out[4] = c.esse.on ? c.esse.kz : 0;
  return IRLCU_OK;
}

int irlcu_drf_tuning(float ms[2]) {
  ms[0] = g_tune_ms[0];
  ms[1] = g_tune_ms[1];
  return IRLCU_OK;
}

void *irlcu_stream(void) { return g_ctx ? (void *)g_ctx->st : nullptr; }

long long irlcu_launch_count(void) { return g_launch_count; }

int irlcu_profile_enable(int on) {
  if (g_ctx) cudaStreamSynchronize(g_ctx->st);
  g_prof.clear();
  g_prof_used = 0;
  std::memset(&g_prof_acc, 0, sizeof(g_prof_acc));
  g_prof_on = on != 0;
  return IRLCU_OK;
}

int irlcu_profile_read(irlcu_profile *out) {
  for (const ProfRec &r : g_prof) {
    float ms = 0.f;
    CU_TRY(cudaEventSynchronize(r.b));
    CU_TRY(cudaEventElapsedTime(&ms, r.a, r.b));
    g_prof_acc.ms[r.stage] += ms;
    g_prof_acc.flops[r.stage] += r.flops;
    g_prof_acc.bytes[r.stage] += r.bytes;
    g_prof_acc.launches[r.stage] += r.launches;
  }
  g_prof.clear();
  g_prof_used = 0;
  if (out) *out = g_prof_acc;
  return IRLCU_OK;
}

int irlcu_stage_times(float *ms, int nmax) {
  TRY(need_ctx());
  Ctx &c = *g_ctx;
  CU_TRY(cudaEventSynchronize(c.ev[3]));
  for (int i = 0; i < 3 && i < nmax; ++i) CU_TRY(cudaEventElapsedTime(&ms[i], c.ev[i], c.ev[i + 1]));
  return IRLCU_OK;
}

}  // extern "C"
