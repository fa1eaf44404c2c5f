// k_drf.cu -- attenuated, depth-dependent DRF projector and backprojector.
//
// libirl Project / BackProject (prjbck.c:68-427) process one rotated row
// ("plane", a z-by-x image at depth y) at a time: attenuate it with the
// cumulative attenuation up to the row centre, convolve it with the PSF of
// the row's collimator distance (conv2d_ypad.c:39-108, direct "same"
// convolution, x zero padded, y optionally padded with averaged end rows),
// and either sum the planes into a projection (Project) or store each plane
// into the rotated volume (BackProject).
//
// Here a CTA owns a 64 x 64 output tile of a plane.  The attenuated input
// tile plus a halo of H pixels is staged in shared memory together with the
// PSF (zero-padded to (2H+1)^2).  Each thread keeps a 4 x BX block of
// outputs in registers and streams input rows through a register window,
// so every shared-memory load feeds 4*BX FMAs per PSF column.
//
// Forward: the (view, tile, plane) tasks are split evenly over a grid sized
// to the machine; a CTA accumulates consecutive planes of a tile in
// registers and writes at most two partial tiles, which a second kernel
// sums in a fixed order (deterministic) and scales.
// Backward: one CTA per (view, plane, tile) writes its plane tile.
//
// The arithmetic is FP32 with FMA; summation order differs from libirl's
// (which adds taps row-major and planes in order), so results agree to
// float rounding, not bit for bit.
#include <cstdio>

#include "irlcu_internal.cuh"

namespace irlcu {

constexpr int TZ = 64, TX = 64, BZ = 4;

template <int H>
struct Cfg {
  static constexpr int BX = (H <= 16) ? 8 : 4;
  static constexpr int NTX = TX / BX, NTZ = TZ / BZ;
  static constexpr int NT = NTX * NTZ;
  static constexpr int TW = TX + 2 * H;
  static constexpr int LD = (TW + 3) & ~3;
  static constexpr int TH = TZ + 2 * H;
  static constexpr int PW = 2 * H + 1;
  static constexpr int PLD = (PW + 3) & ~3;
  static constexpr int WIN = BX + 2 * H;
  static constexpr int SMEM = (TH * LD + PW * PLD) * 4;
};

struct PlaneSrc {
  const float *a;   // plane base [z][x] (row stride n)
  const float *e;   // attenuation factor plane or null (=1)
};

// value of the attenuated, axially padded plane at (pz, px)
__device__ __forceinline__ float plane_val(const PlaneSrc &p, int pz, int px, int n, int nz, int pady,
                                           int avgy) {
  if (px < 0 || px >= n) return 0.f;
  if (pz >= 0 && pz < nz) {
    const float a = __ldg(p.a + (size_t)pz * n + px);
    return p.e ? a * __ldg(p.e + (size_t)pz * n + px) : a;
  }
  if (pady <= 0 || avgy <= 0) return 0.f;
  if (pz < -pady || pz >= nz + pady) return 0.f;
  // pfAvgRows (pad2d.c:92-122): row sum in order, divided when > 1 row
  const int r0 = pz < 0 ? 0 : nz - avgy;
  float s = 0.f;
  for (int r = 0; r < avgy; ++r) {
    const float a = __ldg(p.a + (size_t)(r0 + r) * n + px);
    s = __fadd_rn(s, p.e ? a * __ldg(p.e + (size_t)(r0 + r) * n + px) : a);
  }
  return avgy > 1 ? __fdiv_rn(s, (float)avgy) : s;
}

template <int H>
__device__ __forceinline__ void stage_tile(float *tile, const PlaneSrc &p, int zt0, int xt0, int n, int nz,
                                           int pady, int avgy) {
  using C = Cfg<H>;
  for (int e = threadIdx.x; e < C::TH * C::TW; e += C::NT) {
    const int R = e / C::TW, Cc = e - R * C::TW;
    tile[R * C::LD + Cc] = plane_val(p, zt0 - H + R, xt0 - H + Cc, n, nz, pady, avgy);
  }
}

template <int H>
__device__ __forceinline__ void stage_psf(float *ps, const float *__restrict__ psf_tab, int idist) {
  using C = Cfg<H>;
  const float *src = psf_tab + (size_t)idist * C::PW * C::PLD;
  for (int e = threadIdx.x; e < C::PW * C::PLD; e += C::NT) ps[e] = __ldg(src + e);
}

// acc[zz][j] += sum over taps; the tile and PSF are in shared memory
template <int H>
__device__ __forceinline__ void conv_tile(const float *tile, const float *ps, int z0, int x0,
                                          float (&acc)[BZ][Cfg<H>::BX]) {
  using C = Cfg<H>;
  constexpr int BX = C::BX;
#pragma unroll 1
  for (int r = 0; r < BZ + 2 * H; ++r) {
    float in[C::WIN];
    const float *row = tile + (z0 + r) * C::LD + x0;
#pragma unroll
    for (int m = 0; m < C::WIN; m += 4) {
      const float4 q = *reinterpret_cast<const float4 *>(row + m);
      in[m] = q.x;
      in[m + 1] = q.y;
      in[m + 2] = q.z;
      in[m + 3] = q.w;
    }
#pragma unroll
    for (int zz = 0; zz < BZ; ++zz) {
      const int py = zz + 2 * H - r;
      if (py >= 0 && py <= 2 * H) {
        const float *prow = ps + py * C::PLD;
#pragma unroll
        for (int q4 = 0; q4 < C::PLD / 4; ++q4) {
          const float4 w4 = *reinterpret_cast<const float4 *>(prow + 4 * q4);
          const float w[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int px = 4 * q4 + u;
            if (px < C::PW) {
#pragma unroll
              for (int j = 0; j < BX; ++j) acc[zz][j] = fmaf(w[u], in[j + 2 * H - px], acc[zz][j]);
            }
          }
        }
      }
    }
  }
}

template <int H>
__device__ __forceinline__ void add_center(const float *tile, int z0, int x0, float (&acc)[BZ][Cfg<H>::BX]) {
  using C = Cfg<H>;
#pragma unroll
  for (int zz = 0; zz < BZ; ++zz)
#pragma unroll
    for (int j = 0; j < C::BX; ++j) acc[zz][j] += tile[(z0 + zz + H) * C::LD + x0 + j + H];
}

struct FwdArgs {
  const float *src;        // nv volumes [y][z][x]
  const float *E;          // per-view tables or null
  const int *views;        // batch -> view
  const float *psf;        // padded PSF table or null
  const int *row_idist;    // [view][y] or null
  const int *pad_rows;     // per distance or null
  int avgy;
  int n, nz, nv, ntx, ntiles;
  long long T;             // total tasks
  float *part;             // partial tiles [G][2][TZ*TX]
};

template <int H>
__global__ void __launch_bounds__(Cfg<H>::NT) k_drf_forward(FwdArgs a) {
  using C = Cfg<H>;
  extern __shared__ __align__(16) float sm[];
  float *tile = sm;
  float *ps = sm + C::TH * C::LD;
  const int tid = threadIdx.x;
  const int tx = tid % C::NTX, tz = tid / C::NTX;
  const int z0 = tz * BZ, x0 = tx * C::BX;
  const long long G = gridDim.x, c = blockIdx.x;
  const long long t0 = c * a.T / G, t1 = (c + 1) * a.T / G;
  const size_t vox = (size_t)a.n * a.nz * a.n, pln = (size_t)a.nz * a.n;
  float acc[BZ][C::BX];
#pragma unroll
  for (int zz = 0; zz < BZ; ++zz)
#pragma unroll
    for (int j = 0; j < C::BX; ++j) acc[zz][j] = 0.f;
  int slot = 0;
  long long seg_prev = t0 / a.n;
  for (long long t = t0; t < t1; ++t) {
    const long long seg = t / a.n;
    if (seg != seg_prev) {  // flush the finished segment
      float *p = a.part + ((size_t)c * 2 + slot) * (TZ * TX);
#pragma unroll
      for (int zz = 0; zz < BZ; ++zz)
#pragma unroll
        for (int j = 0; j < C::BX; ++j) {
          p[(z0 + zz) * TX + x0 + j] = acc[zz][j];
          acc[zz][j] = 0.f;
        }
      slot = 1;
      seg_prev = seg;
    }
    const int y = (int)(t - seg * a.n);
    const int tile_i = (int)(seg % a.ntiles);
    const int bv = (int)(seg / a.ntiles);
    const int view = a.views[bv];
    const int zt0 = (tile_i / a.ntx) * TZ, xt0 = (tile_i % a.ntx) * TX;
    const int idist = a.row_idist ? a.row_idist[(size_t)view * a.n + y] : -1;
    const int pady = (idist >= 0 && a.pad_rows) ? a.pad_rows[idist] : 0;
    PlaneSrc p{a.src + (size_t)bv * vox + (size_t)y * pln, a.E ? a.E + (size_t)view * vox + (size_t)y * pln : nullptr};
    __syncthreads();
    stage_tile<H>(tile, p, zt0, xt0, a.n, a.nz, pady, a.avgy);
    if (idist >= 0) stage_psf<H>(ps, a.psf, idist);
    __syncthreads();
    if (idist >= 0)
      conv_tile<H>(tile, ps, z0, x0, acc);
    else
      add_center<H>(tile, z0, x0, acc);
  }
  float *p = a.part + ((size_t)c * 2 + slot) * (TZ * TX);
#pragma unroll
  for (int zz = 0; zz < BZ; ++zz)
#pragma unroll
    for (int j = 0; j < C::BX; ++j) p[(z0 + zz) * TX + x0 + j] = acc[zz][j];
}

// sum of the partial tiles of every (view, tile) segment, in CTA order
__global__ void k_forward_reduce(const float *__restrict__ part, long long T, long long G, int n, int nz,
                                 int ntx, int ntiles, int nv, float scale, float *__restrict__ out) {
  const size_t pln = (size_t)nz * n;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)nv * pln) return;
  const int bv = (int)(e / pln);
  const int rem = (int)(e - (size_t)bv * pln);
  const int Z = rem / n, X = rem - Z * n;
  const int tile_i = (Z / TZ) * ntx + X / TX;
  const long long seg = (long long)bv * ntiles + tile_i;
  const long long tf = seg * n, tl = seg * n + n - 1;
  const long long cf = ((tf + 1) * G + T - 1) / T - 1;
  const long long cl = ((tl + 1) * G + T - 1) / T - 1;
  const int off = (Z % TZ) * TX + (X % TX);
  float s = 0.f;
  for (long long c = cf; c <= cl; ++c) {
    const long long first_seg = (c * T / G) / n;
    const int slot = first_seg == seg ? 0 : 1;
    s += part[((size_t)c * 2 + slot) * (TZ * TX) + off];
  }
  out[e] = s * scale;
}

struct BckArgs {
  const float *planes;     // nv planes [z][x]
  const float *E;
  const int *views;
  const float *psf;
  const int *row_idist;
  const int *pad_rows;
  int avgy;
  int n, nz, ntx, ntiles;
  float scale;
  float *out;              // nv volumes [y][z][x]
};

template <int H>
__global__ void __launch_bounds__(Cfg<H>::NT) k_drf_backward(BckArgs a) {
  using C = Cfg<H>;
  extern __shared__ __align__(16) float sm[];
  float *tile = sm;
  float *ps = sm + C::TH * C::LD;
  const int tid = threadIdx.x;
  const int tx = tid % C::NTX, tz = tid / C::NTX;
  const int z0 = tz * BZ, x0 = tx * C::BX;
  // blockIdx.x = tile, blockIdx.y = plane y, blockIdx.z = batch view
  const int tile_i = blockIdx.x, y = blockIdx.y, bv = blockIdx.z;
  const int view = a.views[bv];
  const size_t vox = (size_t)a.n * a.nz * a.n, pln = (size_t)a.nz * a.n;
  const int zt0 = (tile_i / a.ntx) * TZ, xt0 = (tile_i % a.ntx) * TX;
  const int idist = a.row_idist ? a.row_idist[(size_t)view * a.n + y] : -1;
  const int pady = (idist >= 0 && a.pad_rows) ? a.pad_rows[idist] : 0;
  PlaneSrc p{a.planes + (size_t)bv * pln, a.E ? a.E + (size_t)view * vox + (size_t)y * pln : nullptr};
  stage_tile<H>(tile, p, zt0, xt0, a.n, a.nz, pady, a.avgy);
  if (idist >= 0) stage_psf<H>(ps, a.psf, idist);
  __syncthreads();
  float acc[BZ][C::BX];
#pragma unroll
  for (int zz = 0; zz < BZ; ++zz)
#pragma unroll
    for (int j = 0; j < C::BX; ++j) acc[zz][j] = 0.f;
  if (idist >= 0)
    conv_tile<H>(tile, ps, z0, x0, acc);
  else
    add_center<H>(tile, z0, x0, acc);
  float *o = a.out + (size_t)bv * vox + (size_t)y * pln;
#pragma unroll
  for (int zz = 0; zz < BZ; ++zz) {
    const int Z = zt0 + z0 + zz;
    if (Z >= a.nz) continue;
#pragma unroll
    for (int j = 0; j < C::BX; ++j) {
      const int X = xt0 + x0 + j;
      if (X < a.n) o[(size_t)Z * a.n + X] = acc[zz][j] * a.scale;
    }
  }
}

// -------------------------------------------------------------- launchers

static const int kHalos[] = {0, 4, 8, 12, 16, 24, 32};

int halo_instance(int h) {
  for (int k : kHalos)
    if (h <= k) return k;
  return -1;
}

static long long g_fwd_grid = 0;

#define TRY_FFT(x)           \
  do {                       \
    int rc_ = (x);           \
    if (rc_) return rc_;     \
  } while (0)

template <int H>
static int fwd_launch(const Ctx &c, FwdArgs a) {
  using C = Cfg<H>;
  static bool configured = false;
  if (!configured) {
    CU_TRY(cudaFuncSetAttribute(k_drf_forward<H>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
    configured = true;
  }
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  CU_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_drf_forward<H>, C::NT, C::SMEM));
  if (per_sm < 1) per_sm = 1;
  long long G = (long long)nsm * per_sm;
  const long long nseg = a.T / a.n;
  if (G < nseg) G = nseg;             // every CTA spans at most two segments
  if (G > a.T) G = a.T;
  const size_t need = (size_t)G * 2 * TZ * TX;
  if (need > c.wpart_elems) return set_error(IRLCU_EARG, "forward partial buffer too small (%zu < %zu)", c.wpart_elems, need);
  a.part = c.wpart;
  g_fwd_grid = G;
  k_drf_forward<H><<<(unsigned)G, C::NT, C::SMEM, c.st>>>(a);
  CU_LAUNCHED();
  return IRLCU_OK;
}

template <int H>
static int bck_launch(const Ctx &c, BckArgs a, int nv) {
  using C = Cfg<H>;
  static bool configured = false;
  if (!configured) {
    CU_TRY(cudaFuncSetAttribute(k_drf_backward<H>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
    configured = true;
  }
  dim3 grid(a.ntiles, a.n, nv);
  k_drf_backward<H><<<grid, C::NT, C::SMEM, c.st>>>(a);
  CU_LAUNCHED();
  return IRLCU_OK;
}

#define DISPATCH_H(h, F, ...)                  \
  switch (h) {                                 \
    case 0: return F<0>(__VA_ARGS__);          \
    case 4: return F<4>(__VA_ARGS__);          \
    case 8: return F<8>(__VA_ARGS__);          \
    case 12: return F<12>(__VA_ARGS__);        \
    case 16: return F<16>(__VA_ARGS__);        \
    case 24: return F<24>(__VA_ARGS__);        \
    case 32: return F<32>(__VA_ARGS__);        \
    default: return set_error(IRLCU_EARG, "unsupported DRF halo %d", h); \
  }

static int forward_dispatch(int h, const Ctx &c, FwdArgs a) { DISPATCH_H(h, fwd_launch, c, a) }
static int backward_dispatch(int h, const Ctx &c, BckArgs a, int nv) { DISPATCH_H(h, bck_launch, c, a, nv) }

int launch_project(const Ctx &c, const float *src, const int *dviews, int nv, const float *E, const DrfDev *drf,
                   float scale, float *out) {
  if (nv <= 0) return IRLCU_OK;
  if (drf && drf->psf && drf->fft.on) {
    TRY_FFT(launch_project_fft(c, src, dviews, nv, E, *drf, scale, out));
    return IRLCU_OK;
  }
  FwdArgs a{};
  a.src = src;
  a.E = E;
  a.views = dviews;
  const bool use = drf && drf->psf;
  a.psf = use ? drf->psf : nullptr;
  a.row_idist = use ? drf->row_idist : nullptr;
  a.pad_rows = use ? drf->pad_rows : nullptr;
  a.avgy = use ? drf->avg_rows : 0;
  a.n = c.n;
  a.nz = c.nz;
  a.nv = nv;
  a.ntx = (c.n + TX - 1) / TX;
  a.ntiles = a.ntx * ((c.nz + TZ - 1) / TZ);
  a.T = (long long)nv * a.ntiles * c.n;
  const int h = use ? drf->halo : 0;
  int rc = forward_dispatch(h, c, a);
  if (rc) return rc;
  const size_t tot = (size_t)nv * c.pln;
  k_forward_reduce<<<(unsigned)((tot + 255) / 256), 256, 0, c.st>>>(c.wpart, a.T, g_fwd_grid, c.n, c.nz, a.ntx,
                                                                      a.ntiles, nv, scale, out);
  CU_LAUNCHED();
  return IRLCU_OK;
}

int launch_backproject(const Ctx &c, const float *planes, const int *dviews, int nv, const float *E,
                       const DrfDev *drf, float scale, float *bck) {
  if (nv <= 0) return IRLCU_OK;
  if (drf && drf->psf && drf->fft.on) return launch_backproject_fft(c, planes, dviews, nv, E, *drf, scale, bck);
  BckArgs a{};
  a.planes = planes;
  a.E = E;
  a.views = dviews;
  const bool use = drf && drf->psf;
  a.psf = use ? drf->psf : nullptr;
  a.row_idist = use ? drf->row_idist : nullptr;
  a.pad_rows = use ? drf->pad_rows : nullptr;
  a.avgy = use ? drf->avg_rows : 0;
  a.n = c.n;
  a.nz = c.nz;
  a.ntx = (c.n + TX - 1) / TX;
  a.ntiles = a.ntx * ((c.nz + TZ - 1) / TZ);
  a.scale = scale;
  a.out = bck;
  const int h = use ? drf->halo : 0;
  return backward_dispatch(h, c, a, nv);
}

size_t forward_partial_elems(int n, int nz, int max_batch) {
  // upper bound of the forward grid: one CTA per task at most, and at least
  // one per segment; callers size the buffer for the larger of the machine
  // grid (<= 148 SMs x 16 CTAs) and the segment count
  const long long ntiles = (long long)((n + TX - 1) / TX) * ((nz + TZ - 1) / TZ);
  long long G = 148LL * 16;
  if (G < (long long)max_batch * ntiles) G = (long long)max_batch * ntiles;
  return (size_t)G * 2 * TZ * TX;
}

// ------------------------------------------------- attenuation tables
// S += mu/2; value at the row centre; S += mu/2 (prjbck.c:212-214, 248-250);
// E = exp(-S) evaluated in double as libirl does (prjbck.c:221-222).
__global__ void k_atn_tables(const float *__restrict__ rmu, float *__restrict__ E, float *__restrict__ S, int n,
                             int nz, int nv) {
  const size_t pln = (size_t)nz * n, vox = pln * n;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)nv * pln) return;
  const size_t v = e / pln, i = e - v * pln;
  const float *m = rmu + v * vox + i;
  float s = 0.f;
  for (int y = 0; y < n; ++y) {
    const float h = 0.5f * __ldg(m + (size_t)y * pln);
    s = __fadd_rn(s, h);
    if (S) S[v * vox + (size_t)y * pln + i] = s;
    if (E) E[v * vox + (size_t)y * pln + i] = (float)exp(-(double)s);
    s = __fadd_rn(s, h);
  }
}

int launch_atn_tables(const Ctx &c, const float *rmu, float *E, float *S, int nv) {
  const size_t tot = (size_t)nv * c.pln;
  k_atn_tables<<<(unsigned)((tot + 255) / 256), 256, 0, c.st>>>(rmu, E, S, c.n, c.nz, nv);
  CU_LAUNCHED();
  return IRLCU_OK;
}

}  // namespace irlcu
