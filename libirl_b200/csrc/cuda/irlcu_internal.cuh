// irlcu_internal.cuh -- device context and kernel launchers shared by the
// CUDA translation units of libirl_b200.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <vector>

#include "irlcu.h"

namespace irlcu {

constexpr int MODEL_ATN_BIT = 1, MODEL_DRF_BIT = 2, MODEL_SRF_BIT = 4;

// Rotation tables of a batch of rotations, in device memory.  For rotation
// r: hdr[4r..4r+3] = {b90, b180, iadd, mdim}; row tables have n entries,
// column tables 2n; sin/cos for the bilinear rotator.
struct RotTabs {
  int *hdr;
  int *row_sh;
  float *row_f1, *row_f2;
  int *col_sh;
  float *col_f1, *col_f2;
  float *sn, *cs;
};

// Fourier-domain form of a DRF table (k_drf_fft.cu): planes on an Mz x Mx
// grid, plane row z at grid row z + P; spectra of the quadrant-swapped PSFs
// plus an identity spectrum for rows without DRF, scaled by 1/(Mz Mx).
struct DrfFft {
  bool on = false;
  int Mz = 0, Mx = 0, Mxh = 0;  // grid; Mxh = Mx/2 + 1 half-spectrum bins
  int P = 0, G = 0;             // row offset; rows that can be nonzero
  float2 *H = nullptr;          // [ndist + 1][Mz][Mxh]
  float2 *twx = nullptr, *twz = nullptr;
  bool fused = false;           // square grid (Mz == Mx), one CTA per plane
};

struct DrfDev {
  int ndist = 0, halo = -1, avg_rows = 0;
  float *psf = nullptr;       // ndist * (2h+1) * pstride
  int pstride = 0;            // row stride of a PSF (multiple of 4 floats)
  int *pad_rows = nullptr;    // per distance
  int *row_idist = nullptr;   // nviews * n
  std::vector<int> h_rows;    // host copy of row_idist (work accounting)
  std::vector<int> h_taps;    // per distance: taps of the unpadded PSF
  DrfFft fft;                 // on: the convolution runs in the Fourier domain
};

struct EsseDev {
  bool on = false;
  bool zero = false;          // kernel scatter factor 0: zero effective source
  int kx = 0, ky = 0, kz = 0, collapse = 1, nterms = 1;
  float mu0 = 0, mu_avg = 0, pix = 0, cntr = 0;
  int kxh = 0;                // kx/2 + 1 complex bins along x
  float2 *kft[3] = {nullptr, nullptr, nullptr};  // kernel spectra [ky][kz][kxh]
  float2 *kftT[3] = {nullptr, nullptr, nullptr}; // kx-major copies [kxh][ky][kz]
  bool fused = false;         // y-z transforms in one shared-memory kernel
  bool yz_reg = false;        // ... with register transforms (kftT in position order)
};

// ESSE work buffers of one context (k_esse.cu)
struct EsseWork {
  float2 *twx = nullptr, *twy = nullptr, *twz = nullptr;
  float2 *A = nullptr, *Bf = nullptr, *C2[2] = {nullptr, nullptr}, *D[2] = {nullptr, nullptr};
  float *g[2] = {nullptr, nullptr};
  float *T[2] = {nullptr, nullptr};   // smoothed terms (coarse in x after the z pass)
  float *Tc[2] = {nullptr, nullptr};  // terms after the y pass, coarse in z and x
  int batch = 0;
  int nxv = 0, nyv = 0, nzv = 0;
};

// Fourier-domain DRF work buffers of one context, sized for the largest
// table (k_drf_fft.cu)
struct DfftWork {
  float2 *S = nullptr;     // row spectra of a batch of planes
  size_t s_elems = 0;
  float2 *part = nullptr;  // forward partial sums
  size_t part_elems = 0;
  float2 *Y = nullptr;     // forward column results
  size_t y_elems = 0;
};

struct GraphRec {
  int key;                  // model bits, scatter estimate, scatter mode
  cudaGraphExec_t exec;
  long long kernels;        // kernel launches in the graph
};

struct Ctx {
  irlcu_geom g{};
  int n = 0, nz = 0, nv = 0;
  size_t vox = 0, pln = 0;
  int dev = -1;               // the device current at irlcu_init; c.st belongs to it
  // three-shear kernel per source kind (0: one source shared by all views,
  // 1: a source per view): 0 one slice per CTA, 1 two slices per CTA,
  // -1 not tuned (launch_rotate's default); set by the shape autotuner
  mutable int shear_form[2] = {-1, -1};
  // shape autotuner trial (irlcu_osem_iteration): state 0 pending, 1 and 2
  // the trial iterations with form 0 and 1 in flight, 3 decided; while a
  // trial iteration runs, launch_rotate times every launch (events per kind)
  int shear_trial = 0;
  mutable int trial_form = -1;
  mutable std::vector<std::pair<cudaEvent_t, cudaEvent_t>> trial_ev[2];
  float trial_ms[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // [kind][form], ms per iteration
  cudaStream_t st = nullptr;
  cudaStream_t up_st = nullptr;  // irlcu_upload_now: copies beside the queued kernels
  cudaEvent_t ev[16];
  int nsub = 0;

  // rotation tables: [0, nv) rotate by 0.5*pi + angle, [nv, 2nv) unrotate
  RotTabs rot{};
  int max_mdim = 0;           // widest three-shear intermediate image in use
  int *sup_start = nullptr, *sup_end = nullptr;

  // persistent volumes / planes
  float *est = nullptr, *atn = nullptr, *prj = nullptr, *scatest = nullptr;
  float *prjscat = nullptr, *upd = nullptr, *norm = nullptr;
  unsigned char *colmask = nullptr;  // nv * n measured columns

  // per-view iteration-invariant tables [view][y][z][x]
  float *tE = nullptr;    // exp(-cumulative attenuation) at pixel centres
  float *tS = nullptr;    // cumulative attenuation (ESSE depth), SRF only
  float *tMu = nullptr;   // rotated attenuation map (ESSE density), SRF only

  // batch work space (max_batch views)
  float *wrot = nullptr;    // rotated activity / source, B volumes
  float *wbck = nullptr;    // backprojected rotated volumes, B volumes
  float *wprj = nullptr;    // B projection planes
  float *wprj2 = nullptr;   // B projection planes (second projection)
  float *wpart = nullptr;   // forward partial sums
  size_t wpart_elems = 0;
  float *wavg = nullptr;    // axial-pad average rows, B * n * 2 * n
  int *dviews = nullptr;    // B view indices
  irlcu_view_parm *dvp = nullptr;

  DrfDev drf[2];
  EsseDev esse;
  float *wfft = nullptr;    // ESSE work: B * spectra
  size_t wfft_elems = 0;
  float *weff = nullptr;    // ESSE expanded terms, B volumes x2
  EsseWork ew;
  DfftWork dw;

  // every subset's views and per-view parameters (irlcu_set_subsets) and
  // the CUDA graphs of whole iterations (irlcu_osem_iteration)
  int *dviews_all = nullptr;
  irlcu_view_parm *dvp_all = nullptr;
  std::vector<int> h_views_all;
  std::vector<irlcu_view_parm> h_vp_all;
  int nsub_all = 0, per_all = 0, vp_scat_mode = 0;
  std::vector<GraphRec> graphs;
  std::vector<int> graph_seen;   // keys run eagerly once
  bool capturing = false;

  // learned scatter surrogate in place of ESSE (irlcu_set_surrogate)
  irlcu_sur *sur = nullptr;
  std::vector<unsigned char> sur_flags;   // per view: 1 = ESSE for that view
  float *sur_scale = nullptr;             // max_batch activity means
  float *sur_work = nullptr;              // pooling work of max_batch views
  float *sur_static = nullptr;            // pooled mu and exp(-S) channels of every view (BF16 pairs)
  bool sur_static_ok = false;             // ... computed from the current attenuation tables
  // estimate snapshots for the iteration callback (irlcu_snapshot_*): a
  // device copy in external layout and a pinned host copy per slot, copied
  // on their own stream while the next iteration runs
  float *snap[2] = {nullptr, nullptr};
  float *snap_host[2] = {nullptr, nullptr};
  cudaStream_t snap_st = nullptr;
  cudaEvent_t snap_made[2] = {nullptr, nullptr}, snap_copied[2] = {nullptr, nullptr};
  // three-shear intermediate for slices beyond shared memory, grown on use
  mutable float *xscratch = nullptr;
  mutable size_t xscratch_elems = 0;
};

extern Ctx *g_ctx;

// Device memory of a context: stream-ordered allocations from the device's
// default pool, whose release threshold is raised so that freed memory stays
// cached for the next context (set-up reuses it without reaching the driver
// and teardown never synchronises the device).  dev_alloc waits for its
// stream, so the memory can be used at once by any stream or copy.
cudaError_t dev_alloc(void **p, size_t bytes, cudaStream_t st);
void dev_free(void *p, cudaStream_t st);
template <class T>
inline cudaError_t dev_alloc_t(T **p, size_t count, cudaStream_t st) {
  return dev_alloc(reinterpret_cast<void **>(p), count * sizeof(T), st);
}

// error helpers
int set_error(int code, const char *fmt, ...);
#define CU_TRY(x)                                                         \
  do {                                                                    \
    cudaError_t e_ = (x);                                                 \
    if (e_ != cudaSuccess)                                                \
      return ::irlcu::set_error(IRLCU_ECUDA, "%s:%d %s: %s", __FILE__,    \
                                __LINE__, #x, cudaGetErrorString(e_));    \
  } while (0)

// every kernel launch is followed by CU_LAUNCHED(): it counts the launch
// (irlcu_launch_count) and checks the launch status
extern long long g_launch_count;
#define CU_LAUNCHED()                      \
  do {                                     \
    ++::irlcu::g_launch_count;             \
    CU_TRY(cudaGetLastError());            \
  } while (0)

// ---- launchers (each defined in its kernel file) ----

// ESSE's CollapseByFac by 2 of the rotated volumes, taken by the two-slice
// shear while it writes them (out[v][y'][z'][x'], nyv x nzv x nxv per
// view); `done` reports whether it did
struct RotCollapse {
  float *out = nullptr;
  int nyv = 0, nzv = 0, nxv = 0;
  bool done = false;
};

// rotation of nv volumes: dst[v] = rotate(src[v or shared], tab rot_base+views[v])
int launch_rotate(const Ctx &c, const float *src, size_t src_stride, float *dst,
                  size_t dst_stride, const int *dviews, int nv, int rot_base, RotCollapse *col = nullptr);

// three-shear rotation of one device volume with every buffer in a static
// device array (irlcu_rotate_volume_noalloc); enqueued on `st`
int launch_rotate_noalloc(cudaStream_t st, int dev, float angle, const float *src, float *dst, int n, int nz);

// cumulative attenuation tables of nv views from rotated maps in tMu-like
// buffer `rmu` (stride vox): writes E (and S if not null)
int launch_atn_tables(const Ctx &c, const float *rmu, float *E, float *S, int nv);

// forward DRF projection: out[v] = sum_y conv(src[v][y] * E[view][y]) * scale
int launch_project(const Ctx &c, const float *src, const int *dviews, int nv,
                   const float *E, const DrfDev *drf, float scale, float *out);

// backprojection planes: bck[v][y] = conv(plane[v] * E[view][y]) * scale
int launch_backproject(const Ctx &c, const float *planes, const int *dviews, int nv,
                       const float *E, const DrfDev *drf, float scale, float *bck);

// Fourier-domain DRF engine (k_drf_fft.cu); max_pad: the largest axial pad
int drf_fft_setup(Ctx &c, DrfDev &D, int max_pad);
void drf_fft_free(Ctx &c, DrfDev &D);
void drf_fft_work_free(Ctx &c);
int launch_project_fft(const Ctx &c, const float *src, const int *dviews, int nv, const float *E, const DrfDev &D,
                       float scale, float *out);
int launch_backproject_fft(const Ctx &c, const float *planes, const int *dviews, int nv, const float *E,
                           const DrfDev &D, float scale, float *bck);

// unrotate nv backprojected volumes and accumulate into acc with the
// per-view clamp; then optionally est *= acc * norm or acc = invert(acc)
#define ACC_EM 1
#define ACC_INVERT 2
int launch_unrotate_accumulate(const Ctx &c, const float *bck, const int *dviews, int nv,
                               float *acc, int start_from_acc, int mode, float *est,
                               const float *norm);

// OSEM ratio epilogue for nv views
int launch_ratio(const Ctx &c, const float *calc, const float *calc_nosrf,
                 const int *dviews, const irlcu_view_parm *dvp, int nv,
                 int use_scatest, float *ratio);

// norm mask planes
int launch_norm_planes(const Ctx &c, const int *dviews, const float *vt_dev, int nv,
                       const unsigned char *normcols, float *planes);

// learned scatter surrogate (k_surrogate.cu)
int sur_max_batch(const irlcu_sur *s);
int sur_tc_status(cudaStream_t st);
void *sur_input(irlcu_sur *s);
int sur_infer(irlcu_sur *s, cudaStream_t st, int B, const float **y);
// The network's input grid: SUR_P^3 means of (n / SUR_P)^3 voxels (n a
// multiple of 4 SUR_P: 128 or 256).  work: nv * (SUR_P^3 + SUR_POOL_PARTS) floats
constexpr int SUR_P = 32;
constexpr int SUR_POOL_PARTS = 128;
int launch_sur_static(cudaStream_t st, const float *mu, const float *S, int nviews, int n, size_t vox, void *stat);
int launch_sur_inputs_static(cudaStream_t st, const float *act, size_t act_stride, const void *stat,
                             const int *dviews, int nv, int n, float *scale, void *out, float *work);
int launch_sur_inputs(cudaStream_t st, const float *act, size_t act_stride, const float *mu, const float *S,
                      const int *dviews, int nv, int n, size_t vox, float *scale, void *out, float *work);
int launch_sub(cudaStream_t st, const float *a, const float *b, float *out, size_t n);
int launch_scale_views(cudaStream_t st, const float *x, const float *s, float *y, int P, int nb, int accumulate);
int launch_div_views(cudaStream_t st, const float *a, const float *s, float *out, int P, int nb);
// the network's 128 x 128 output onto n x n projections (bilinear) and n x n
// targets onto 128 x 128 (f x f means); n = 128 is the plain scale / divide
int launch_scale_views_up(cudaStream_t st, const float *x, const float *s, float *y, int n, int nb, int accumulate);
int launch_div_views_down(cudaStream_t st, const float *a, const float *s, float *out, int n, int nb);

// ESSE effective source: src[v] = rot[v]*primary + effsrc(rot[v], view)
int esse_setup(Ctx &c, const irlcu_esse *e);
int launch_esse(Ctx &c, const float *rot, const int *dviews, int nv, float primary,
                float *src, bool collapsed = false);
// where the rotation may leave ESSE's collapsed input for a batch of nv
// views (RotCollapse), or false when this ESSE set-up reads it otherwise
bool esse_collapse_target(const Ctx &c, int nv, RotCollapse *col);

}  // namespace irlcu
