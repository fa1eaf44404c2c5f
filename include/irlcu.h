/*
 * irlcu.h -- device-side C ABI of libirl_b200.
 *
 * This is the thin layer between the host C driver (IrlOsem, IrlGenprj,
 * set-up) and the sm_100a CUDA kernels.  Every entry point takes plain
 * pointers and sizes and returns an int status (0 = OK, otherwise an
 * IRLCU_E* code; irlcu_error_string() gives the message).
 *
 * It replaces libirl's internal projector seam (irlprivate.h:461-517:
 * InitPrj, Project, BackProject, FreePrj) and the OSEM inner loop of
 * osemrecon.c:687-863.  Instead of one view per call it works on all the
 * views of a subset at once: rotation, ESSE scatter source, attenuated DRF
 * projection, ratio, DRF backprojection, unrotation, per-view clamped
 * accumulation and the EM update run as a few batched kernels.
 *
 * Layouts on the device (x fastest throughout):
 *   volume      [y][z][x]  N*Nz*N      (libirl's internal layout)
 *   projection  [z][x]     Nz*N per view
 *   per-view tables [view][y][z][x]    rotated frame of each view
 *
 * One context per process, like libirl (non-reentrant; one device).
 */
#ifndef IRLCU_H
#define IRLCU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IRLCU_OK 0
#define IRLCU_ECUDA 101     /* a CUDA call failed */
#define IRLCU_EARG 102      /* bad argument or size */
#define IRLCU_ESTATE 103    /* call out of order (e.g. no context) */
#define IRLCU_ENOMEM 104    /* device allocation failed */

/* problem geometry; NumRotPixs == NumPixels as in libirl (IrlSetup.c:60) */
typedef struct {
	int n;            /* NumPixels */
	int nz;           /* NumSlices */
	int nviews;       /* NumAngles */
	int fast_rotate;  /* 1: three-shear rotation, 0: bilinear (rot3dpar) */
	int max_batch;    /* views processed per batched launch (>= views per subset) */
} irlcu_geom;

/* DRF table as the kernels use it: every PSF zero-padded and centred in a
   (2*halo+1)^2 grid; row_idist[view*n + row] = table index for that rotated
   row or -1 where libirl skips the convolution (distance <= 0). */
typedef struct {
	int ndist;
	int halo;                 /* max(MaxOffsX, MaxOffsY) - 1 over the table */
	const float *psf;         /* ndist * (2*halo+1)^2, host memory */
	const int *pad_rows;      /* per distance: min(iAxialPadLength, MaxOffsY-1) */
	const int *row_idist;     /* nviews * n, host memory */
	int avg_rows;             /* iAxialAvgLength, clamped to [0, nz] */
	const int *taps;          /* per distance: (2*MaxOffsX-1)*(2*MaxOffsY-1),
	                             the PSF's own extent (work accounting) */
} irlcu_drf;

/* ESSE scatter model (krnlprj3d.c:349-365, 676-954).  The kernel comes in
   its KRNL-file form (one quadrant, [ndepths][noffs][noffs]); the device
   expands it to the grids K and K (mu - mu_avg) of pfReorder3dKrnl
   (krnlprj3d.c:43-128, irlcu_esse_expand) and transforms them. */
typedef struct {
	int kx, ky, kz;           /* FFT grid: offsets (x), depths (y), slices (z) */
	int collapse;             /* SrfCollapseFac */
	int nterms;               /* Taylor terms, 1 or 2 */
	float mu0, mu_avg, pix, cntr_pix_fac;
	int noffs, ndepths;       /* NumXYoffs, NumDists */
	const float *krnl;        /* pfKrnl, [ndepths][noffs][noffs], host */
	const float *mu;          /* pfKrnlMu, same layout, host */
	float kmu_outside;        /* K (mu - mu_avg) where K is 0 */
} irlcu_esse;

/* per-view scalars of the OSEM update (osemrecon.c:727-827) */
typedef struct {
	float view_time;          /* ViewTime */
	float sensitivity;        /* Sensitivity */
	int scat_mode;            /* 0 none, 1 add stored estimate, 2 store
	                             (with-SRF minus no-SRF) estimate */
} irlcu_view_parm;

int irlcu_init(const irlcu_geom *g);
void irlcu_shutdown(void);
const char *irlcu_error_string(void);

/* rotation angles of every view (radians, as in PrjView_t.Angle) */
int irlcu_set_angles(const float *angles);
/* DRF tables: which = 0 projector, 1 backprojector */
int irlcu_set_drf(int which, const irlcu_drf *d);
int irlcu_set_esse(const irlcu_esse *e);
/* The ESSE grid of one term (0: K, 1: K (mu - mu_avg)), [ky][kz][kx], as
   irlcu_set_esse builds it on the device, copied to host memory out. */
int irlcu_esse_expand(const irlcu_esse *e, int term, float *out);
/* measured-bin mask of each view: nviews*n column flags (1 measured) */
int irlcu_set_column_mask(const unsigned char *mask);

/* volume / projection buffers */
#define IRLCU_BUF_EST 0      /* estimate, volume */
#define IRLCU_BUF_ATN 1      /* attenuation map (per pixel), volume */
#define IRLCU_BUF_PRJ 2      /* measured projections, nviews planes */
#define IRLCU_BUF_SCATEST 3  /* additive scatter estimate, nviews planes */
#define IRLCU_BUF_PRJSCAT 4  /* stored scatter projections, nviews planes */
#define IRLCU_BUF_UPDATE 5   /* subset update image, volume */
#define IRLCU_BUF_NORM 6     /* inverted norm image of subset `index`, volume */
int irlcu_upload(int buf, int index, const float *host, size_t count);
/* irlcu_upload on the context's copy stream: it does not wait for the
   kernels queued on the library stream, and returns once the copy has
   landed, so that later work sees it.  The buffer must exist and no queued
   kernel may use it.  Callable from a helper thread of the calling one
   (never at the same time as an irlcu call that changes the context). */
int irlcu_upload_now(int buf, int index, const float *host, size_t count);
int irlcu_download(int buf, int index, float *host, size_t count);
int irlcu_zero(int buf, int index);
/* a volume buffer copied to the host in libirl's external layout
   [z][y][x] (the transposition runs on the device) */
int irlcu_download_external(int buf, float *host);
/* a volume given in libirl's external layout [z][y][x] into a volume
   buffer (internal layout [y][z][x]; the transposition runs on the device),
   each value multiplied by scale when scale > 0 and scale != 1 (one float
   multiply, as irlosem.c:212-215 scales the attenuation map) and set to 0
   when below 0 with clamp (vZeroNeg).  The host array may be changed once
   the call returns; the device work is queued on the library stream. */
int irlcu_upload_external(int buf, const float *host, float scale, int clamp);
int irlcu_alloc_norm(int nsubsets);

/* Builds the per-view rotated attenuation tables from IRLCU_BUF_ATN
   (rotated map, cumulative half-pixel sums and exp(-sum)).  Asynchronous:
   returns once the work is queued on the library stream. */
int irlcu_prepare_attenuation(int need_srf);

/* Raw projections of the estimate for views[0..nv) into host or device
   memory dst (nv*nz*n floats), libirl Project() with fAtnFac = 1. */
int irlcu_project(int nv, const int *views, int model, float primary_fac,
	float *dst, int dst_on_device);

/* One OSEM subset (osemrecon.c:694-852): projections, ratio against
   IRLCU_BUF_PRJ, backprojection, clamped accumulation into UPDATE and
   EM update of EST with NORM[subset].  model = projector model bits for
   this iteration; bck_model = backprojector bits. */
int irlcu_osem_subset(int nv, const int *views, const irlcu_view_parm *vp,
	int model, int bck_model, int subset, int use_scatest, int apply_update,
	int accumulate_from_update);

/* Views of every subset for irlcu_osem_iteration: views[s*per + m] and the
   per-view ViewTime / Sensitivity in vp (its scat_mode is ignored); kept on
   the device. */
int irlcu_set_subsets(int nsub, int per, const int *views, const irlcu_view_parm *vp);

/* One OSEM iteration over every subset set by irlcu_set_subsets: the
   subset loop of osemrecon.c:687-863 without hooks, each subset as
   irlcu_osem_subset in batches of max_batch views, scat_mode for every
   view.  The first call with a given (model, bck_model, use_scatest,
   scat_mode) runs eagerly; later ones replay a CUDA graph captured from the
   second (set IRLCU_GRAPHS=0 to always run eagerly).  Asynchronous: returns
   once the work is enqueued on the library stream. */
int irlcu_osem_iteration(int model, int bck_model, int use_scatest, int scat_mode);

/* Several device contexts per process (one per reconstruction of a batch):
   irlcu_ctx_detach returns the current context and leaves none current, so
   that the next irlcu_init creates a new one; irlcu_ctx_attach makes a
   detached context current again (none may be current). */
void *irlcu_ctx_detach(void);
int irlcu_ctx_attach(void *ctx);

/* Normalisation image of one subset (osemrecon.c:282-320): backprojects
   the measured-bin mask times ViewTime of each view, clamps after each,
   inverts with a 1e-6 floor and stores it as NORM[subset].  Asynchronous:
   returns once the work is queued on the library stream. */
int irlcu_norm_subset(int nv, const int *views, const float *view_time,
	int bck_model, int subset);

/* Rotation of IRLCU_BUF_EST-layout volumes (libirl vShearsRotate /
   rot3dpar): src and dst are device or host pointers of n*nz*n floats. */
int irlcu_rotate_volume(float angle, const float *src, float *dst, int pb_flag, int on_device);

/* Three-shear rotation (vShearsRotate) of one device-resident volume that
   allocates nothing.  It has no counterpart in libirl, which mallocs its
   mDim^2 scratch on every call (fastrotate.c:391-394).

   It is for callers that must not allocate device memory: a per-angle hook
   or a process beside a running reconstruction whose resident tables
   already fill the device, and latency-bound callers that cannot absorb the
   device-wide synchronisation of cudaMalloc/cudaFree.  irlcu_rotate_volume
   lazily cudaMallocs an n*nz*mdim intermediate when a slice does not fit in
   shared memory.

   Instead this function keeps its rotation tables and that intermediate in
   one file-scope device array of IRLCU_NOALLOC_SCRATCH_BYTES, part of the
   library's module image.  Limits: 1 <= n <= IRLCU_NOALLOC_MAX_N and
   nz*n*mdim floats <= IRLCU_NOALLOC_X_FLOATS, where mdim < 2n is the
   intermediate side for this angle (n = nz = 128: at most 4.2 M floats).
   Larger sizes return IRLCU_EARG before any device access.

   src and dst are device pointers of n*nz*n floats ([y][z][x]), distinct,
   on the device that was current at irlcu_init; that device must be the
   current one (otherwise IRLCU_EARG).  The results are bit-identical to
   irlcu_rotate_volume with a fast-rotation context.

   The call is synchronous: it copies its tables from a static host buffer
   to the array on the library stream, launches the two shear kernels and
   synchronises the stream before returning.  So it must not be made while
   the library stream is being captured into a CUDA graph.  The first call
   on a device looks up the array's address with cudaGetSymbolAddress (which
   may load the module).  There is one scratch array per device and one host
   staging buffer, so overlapping calls (from several host threads) race. */
#define IRLCU_NOALLOC_SCRATCH_BYTES (32u << 20)
#define IRLCU_NOALLOC_TAB_BYTES (64u << 10)
#define IRLCU_NOALLOC_X_FLOATS ((IRLCU_NOALLOC_SCRATCH_BYTES - IRLCU_NOALLOC_TAB_BYTES) / 4u)
#define IRLCU_NOALLOC_MAX_N 1024
int irlcu_rotate_volume_noalloc(float angle, const float *src, float *dst, int n, int nz);

/* The shape autotuner's last decision for the three-shear rotation, made
   from a context's first two whole iterations (irlcu_osem_iteration runs
   the first with the one-slice and the second with the two-slice kernel,
   timing every rotation launch) and cached per (n, nz, batch) for the
   process: ms[0..1] one- and two-slice time per iteration of the rotations
   from the shared estimate, ms[2..3] the same for the unrotations of the
   per-view backprojections; form[k] = 1 where the two-slice kernel was
   kept. */
int irlcu_shear_tuning(float ms[4], int form[2]);
/* Switches the trial iterations on or off (default on; IrlOsemBatch turns
   them off so that the host never waits for the device between problems);
   returns the previous setting. */
int irlcu_shape_trials(int on);
/* Switches the capture and replay of whole iterations as CUDA graphs on or
   off (default on; returns the previous setting).  Off, every iteration
   launches its kernels one by one.  IrlOsemBatch turns it off for its
   problems: with several reconstructions in flight on their own streams,
   capturing and instantiating each problem's iteration graph on the host
   while the device runs the others measured slower (32-problem batch:
   1.12 s with graphs, 0.70 s eager, 0.94 s for the problems one after
   another). */
int irlcu_iteration_graphs(int on);

/* Device memory that new contexts can use: cudaMemGetInfo's free bytes
   plus what the stream-ordered pool holds unused; and the total. */
int irlcu_mem_info(size_t *free_bytes, size_t *total_bytes);

/* Iteration-callback snapshots of the estimate, overlapped with the next
   iteration: irlcu_snapshot_begin(slot) queues, after the work queued so
   far, a copy of the estimate in external layout into the slot's pinned
   host buffer (slot 0 or 1); irlcu_snapshot_end(slot, &p) waits for that
   copy and sets p to the buffer, valid until the slot's next begin or the
   context's end. */
int irlcu_snapshot_begin(int slot);
int irlcu_snapshot_end(int slot, float **host);

/* Body-contour orbit edges for ComputeOrbit (computeorbit.c:81-147): img
   is the thresholded n x n body image (host); for each view, rotated by
   (sn[v], cs[v]) onto an m x m grid with the bilinear rotator of
   rot3dpar.c:19-198, consumed[v] is one more than the first row (from
   row 0, the detector side) that holds a positive sample, or m/2 when the
   first m/2 rows hold none, which is the row count libirl's search loop
   leaves behind.  Synchronous; needs no context (allocates its own small
   device buffers). */
int irlcu_orbit_edges(const float *img, int n, int m, const float *sn, const float *cs, int nviews,
	int *consumed);

/* synchronous wall-clock of the last batched call's stages, for tracing */
int irlcu_stage_times(float *ms, int nmax);

/* The CUDA stream every kernel of the library is launched on (a
   cudaStream_t), so callers can time or order work against it. */
void *irlcu_stream(void);

/* ---- learned scatter surrogate (no libirl counterpart) ----
   A 3D-conv encoder / 2D decoder (1,653,153 parameters, BF16 weights and
   activations, FP32 accumulation) that maps a view's rotated activity,
   attenuation and depth, 4x4x4-pooled to 32^3 x 3 channels, to the view's
   ESSE scatter projection, 128 x 128 (N = Nz = 128 only).  Input and target
   are divided by the view's mean rotated activity.  Training and inference
   run on hand-written kernels; the GPU ESSE path generates the targets and
   stays the fallback. */
typedef struct irlcu_sur irlcu_sur;
/* network for batches of up to max_batch views, weights He-initialised from seed */
int irlcu_sur_create(int max_batch, unsigned long long seed, irlcu_sur **net);
void irlcu_sur_destroy(irlcu_sur *net);
size_t irlcu_sur_nparams(const irlcu_sur *net);
/* FP32 parameter vector (per layer: weights [co][k] then bias [co]) */
int irlcu_sur_get_weights(irlcu_sur *net, float *host, size_t n);
int irlcu_sur_set_weights(irlcu_sur *net, const float *host, size_t n);
/* x: device BF16 [B][32][32][32][3] (channels last); y, t: device FP32 [B][128*128] */
int irlcu_sur_forward(irlcu_sur *net, int B, const void *x, float *y);
/* Test hook for the bounded waits of the tensor-core convolutions: how many
   times a stage-refill wait polls its mbarrier before it gives up (default
   and maximum 4,194,304); returns the previous value.  With 0 every such
   wait runs out at once: the kernel sets its error flag, issues no further
   copies or MMAs, waits for its copies in flight and (at the full limit)
   for its last MMAs, frees its TMEM and returns, and the entry point
   returns IRLCU_ECUDA ("... wait timed out").  The output of that call is
   undefined; the context stays usable. */
unsigned irlcu_sur_test_refill_wait(unsigned polls);
/* mean squared error against t and its gradient (grad_host: nparams floats, or NULL) */
int irlcu_sur_gradient(irlcu_sur *net, int B, const void *x, const float *t, float *loss, float *grad_host);
/* one Adam step (beta 0.9 / 0.999) at learning rate lr; *loss before the step */
int irlcu_sur_train_step(irlcu_sur *net, int B, const void *x, const float *t, float lr, float *loss);

/* Training pairs of views[0..nv) from the current context's estimate (the
   phantom): x_out the network inputs (device BF16 [nv][32][32][32][3]),
   t_out the ESSE scatter projections divided by the view's activity mean
   (device FP32 [nv][Nz*N]), scale_out those means (device FP32 [nv]).
   model: projector bits with the scatter model (attenuation 1, DRF 2,
   scatter 4). */
int irlcu_sur_pairs(int nv, const int *views, int model, void *x_out, float *t_out, float *scale_out);

/* Use net in place of the ESSE projector for every view whose flag is 0
   (flags: nviews bytes, 1 = keep ESSE for that view, NULL = none);
   net == NULL switches back to ESSE.  The network must outlive its use. */
int irlcu_set_surrogate(irlcu_sur *net, const unsigned char *flags);

/* Per-view NRMSE (||surrogate - ESSE|| / ||ESSE|| of the scatter
   projection) of views[0..nv) on the current estimate, into nrmse[nv]. */
int irlcu_sur_check(irlcu_sur *net, int nv, const int *views, int model, float *nrmse);

/* Transform grids in use (0 where not set up): out[0..1] = Mz, Mx of the
   projector's Fourier-domain DRF engine (0, 0: direct convolution),
   out[2..4] = Kx, Ky, Kz of the ESSE grid. */
int irlcu_grids(int out[5]);

/* The DRF engine autotuner's last measurement (ms for one projection plus
   backprojection of a subset batch): ms[0] direct kernels, ms[1] the
   Fourier-domain engine; zeros before the first tuning. */
int irlcu_drf_tuning(float ms[2]);

/* Kernel launches issued by the library since the context was created. */
long long irlcu_launch_count(void);

/* Stage profiling.  While enabled, every stage of irlcu_osem_subset is
   bracketed by CUDA events on the library stream; irlcu_profile_read()
   waits for them and returns per-stage totals since the last enable:
   device milliseconds, launches, and the algorithmic work of the stage
   (FLOPs for the DRF convolutions, bytes for the memory-bound stages). */
#define IRLCU_NSTAGE 8
#define IRLCU_ST_ROTATE 0      /* rotation of the estimate */
#define IRLCU_ST_ESSE 1        /* effective scatter source */
#define IRLCU_ST_PROJECT 2     /* attenuated DRF projection (conv kernel) */
#define IRLCU_ST_REDUCE 3      /* partial-sum reduction + ratio epilogue */
#define IRLCU_ST_BACKPROJECT 4 /* attenuated DRF backprojection (conv kernel) */
#define IRLCU_ST_ACCUM 5       /* unrotation + clamped accumulation + EM update */
typedef struct {
	double ms[IRLCU_NSTAGE];
	double flops[IRLCU_NSTAGE];
	double bytes[IRLCU_NSTAGE];
	long long launches[IRLCU_NSTAGE];
} irlcu_profile;
int irlcu_profile_enable(int on);
int irlcu_profile_read(irlcu_profile *out);

#ifdef __cplusplus
}
#endif

#endif /* IRLCU_H */
