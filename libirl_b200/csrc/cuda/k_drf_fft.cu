// k_drf_fft.cu -- the depth-dependent DRF convolution of the projector and
// backprojector evaluated in the Fourier domain.
//
// Both of libirl's convolution paths compute, per rotated row y (a z-by-x
// plane), a linear "same" convolution of the attenuated plane with the PSF
// of the row's distance:
//   * conv2d_ypad (conv2d_ypad.c:39-108): x zero padded, z padded by up to
//     pady rows holding the mean of the avgy end rows (pad2d.c:21-141);
//   * conv2dPsfFFT (conv2dPsfFFT.c:53-117): the plane zero padded into the
//     upper-left corner of a 2N x 2Nz grid, the PSF quadrant-swapped
//     (padswap.c:21-119), a circular convolution and the upper-left crop --
//     for a PSF half-width h <= N the same linear convolution with no axial
//     padding (the FFT-flagged tables are uploaded with pady = 0).
// Here every plane is placed in an Mz x Mx grid (products of 2, 3, 5, 7)
// with its row z at grid row z + P, P the largest axial pad of the table,
// Mx >= n + h and Mz >= nz + P + h, so the circular convolution on the grid
// equals the linear one on every output pixel.  The PSF spectra H[d] (plus
// an identity spectrum for rows without DRF, prjbck.c:233) are computed
// once per table and carry the 1/(Mz Mx) normalisation.
//
// Forward (Project, prjbck.c:217-240), per batch of views:
//   rows:    R2C along x of every grid row of every plane (two real rows per
//            complex line) -> S[b][y][g][kx], g < G = nz + 2P;
//   columns: per (view, kx chunk, plane group) FFT along g, multiply by
//            H[d(y)], accumulate over the group's planes -> partial sums;
//   finish:  per (view, kx chunk) the partial sums in group order, inverse
//            FFT along g, rows P..P+nz-1 -> Y[b][z][kx];
//   rows:    C2R along x, crop x < n, times the projector scale.
// Backward (BackProject, prjbck.c:340-408), per batch of views:
//   rows:    R2C of ratio * E(y) for every plane y -> S;
//   columns: per (view, plane, kx chunk) FFT, multiply by H[d(y)], inverse
//            FFT, rows P..P+nz-1 written back in place;
//   rows:    C2R, crop, scale -> the backprojected volume [b][y][z][x].
// Work per plane is O(Mz Mx log(Mz Mx)) instead of O(nz n (2h+1)^2); results
// agree with the direct convolution to FP32 FFT rounding.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>

#include "drf_plane.cuh"
#include "fft_core.cuh"
#include "irlcu_internal.cuh"

namespace irlcu {

constexpr int FT_NT = 256;

#define TRY_RC(x)            \
  do {                       \
    int rc_ = (x);           \
    if (rc_) return rc_;     \
  } while (0)

// row pairs per CTA of the x passes, columns per CTA of the z passes
template <int L>
__host__ __device__ constexpr int rows_pairs() { return L <= 256 ? 8 : (L <= 512 ? 4 : 2); }
template <int L>
__host__ __device__ constexpr int col_chunk() { return L <= 256 ? 16 : (L <= 512 ? 8 : 4); }
template <int L>
__host__ __device__ constexpr size_t col_smem() { return sizeof(float2) * ((size_t)2 * col_chunk<L>() * (L + 1) + L); }

// ------------------------------------------------------------ x passes

struct RowSrc {
  // MODE_PLANE: grid row g of plane (b, y) holds row z = g - P of
  //   a[b*a_bs + y*a_ys] * E[view][y] (x < n), or the averaged pad rows
  // MODE_PSF:   grid row g of "plane" d holds the quadrant-swapped PSF d
  //   (d == ndist: the identity)
  int mode;
  const float *a;
  size_t a_bs, a_ys;
  const float *E;
  const int *views;
  const int *row_idist;
  const int *pad_rows;
  int avgy;
  const float *psf;   // padded tables: ndist * (2h+1) * pstride
  int h, pstride, ndist;
  int n, nz, P, G;    // G: grid rows that can be nonzero
  int Mz;
  float2 *out;        // [b][plane][G][Mxh]
  int Mxh, nplanes;
};
constexpr int MODE_PLANE = 0, MODE_PSF = 1;

// index of grid offset g in a centred (2h+1) table, or -1
__device__ __forceinline__ int centred(int g, int M, int h) {
  if (g <= h) return h + g;
  if (g >= M - h) return h + g - M;
  return -1;
}

template <int L>
__global__ void __launch_bounds__(FT_NT) k_dfft_rows_fwd(RowSrc a, const float2 *__restrict__ twg) {
  constexpr int PR = rows_pairs<L>(), LS = L + 1;
  __shared__ float2 tw[L];
  __shared__ float2 sa[PR * LS], sb[PR * LS];
  for (int i = threadIdx.x; i < L; i += FT_NT) tw[i] = twg[i];
  const int b = blockIdx.z, y = blockIdx.y, g0 = blockIdx.x * 2 * PR;
  const int G = a.G, n = a.n;
  const float *ap = nullptr, *ep = nullptr;
  int pady = 0;
  const float *psf = nullptr;
  if (a.mode == MODE_PLANE) {
    const int view = a.views[b];
    const size_t pln = (size_t)a.nz * n;
    ap = a.a + (size_t)b * a.a_bs + (size_t)y * a.a_ys;
    ep = a.E ? a.E + ((size_t)view * n + y) * pln : nullptr;
    const int idist = a.row_idist ? a.row_idist[(size_t)view * n + y] : -1;
    pady = (idist >= 0 && a.pad_rows) ? a.pad_rows[idist] : 0;
  } else if (y < a.ndist) {
    psf = a.psf + (size_t)y * (2 * a.h + 1) * a.pstride;
  }
#pragma unroll 4
  for (int e = threadIdx.x; e < PR * L; e += FT_NT) {
    const int w = e / L, x = e - w * L;
    float v[2] = {0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int g = g0 + 2 * w + q;
      if (g >= G) continue;
      if (a.mode == MODE_PLANE) {
        if (x < n) v[q] = plane_pad_val(ap, ep, g - a.P, x, n, a.nz, pady, a.avgy);
      } else if (psf) {
        const int py = centred(g, a.Mz, a.h), px = centred(x, L, a.h);
        if (py >= 0 && px >= 0) v[q] = __ldg(psf + (size_t)py * a.pstride + px);
      } else {
        v[q] = (g == 0 && x == 0) ? 1.f : 0.f;
      }
    }
    sa[w * LS + x] = make_float2(v[0], v[1]);
  }
  __syncthreads();
  const float2 *res = fft_lines<L>(sa, sb, PR, LS, tw, 1.f);
  // two real rows from one complex line: A = (Z[k] + conj Z[L-k]) / 2,
  // B = (Z[k] - conj Z[L-k]) / 2i
  const int Mxh = a.Mxh;
#pragma unroll 4
  for (int e = threadIdx.x; e < PR * Mxh; e += FT_NT) {
    const int w = e / Mxh, k = e - w * Mxh;
    const int g = g0 + 2 * w;
    if (g >= G) continue;
    const float2 zk = res[w * LS + k];
    const float2 zm = res[w * LS + (k == 0 ? 0 : L - k)];
    float2 *o = a.out + (((size_t)b * a.nplanes + y) * G + g) * Mxh + k;
    o[0] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    if (g + 1 < G) o[Mxh] = make_float2(0.5f * (zk.y + zm.y), 0.5f * (zm.x - zk.x));
  }
}

// C2R along x of row pairs: row (b, p, z) of the input at
//   in[((b*np + p)*rs + r0 + z)*Mxh]; output x < n at out[((b*np + p)*nz + z)*n]
struct RowInv {
  const float2 *in;
  int np, rs, r0, Mxh;
  float *out;
  int n, nz;
  float scale;
};

template <int L>
__global__ void __launch_bounds__(FT_NT) k_dfft_rows_inv(RowInv a, const float2 *__restrict__ twg) {
  constexpr int PR = rows_pairs<L>(), LS = L + 1;
  __shared__ float2 tw[L];
  __shared__ float2 sa[PR * LS], sb[PR * LS];
  for (int i = threadIdx.x; i < L; i += FT_NT) tw[i] = twg[i];
  const int b = blockIdx.z, p = blockIdx.y, z0 = blockIdx.x * 2 * PR;
  const int Mxh = a.Mxh, nz = a.nz;
  const size_t rbase = ((size_t)b * a.np + p) * a.rs + a.r0;
  // Z = A + iB from the half spectra of rows z (A) and z+1 (B)
#pragma unroll 4
  for (int e = threadIdx.x; e < PR * Mxh; e += FT_NT) {
    const int w = e / Mxh, k = e - w * Mxh;
    const int z = z0 + 2 * w;
    float2 A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
    if (z < nz) A = a.in[(rbase + z) * Mxh + k];
    if (z + 1 < nz) B = a.in[(rbase + z + 1) * Mxh + k];
    sa[w * LS + k] = make_float2(A.x - B.y, A.y + B.x);
    if (k > 0 && L - k >= Mxh) sa[w * LS + L - k] = make_float2(A.x + B.y, B.x - A.y);
  }
  __syncthreads();
  const float2 *res = fft_lines<L>(sa, sb, PR, LS, tw, -1.f);
  const int n = a.n;
  for (int e = threadIdx.x; e < PR * 2 * n; e += FT_NT) {
    const int w = e / (2 * n), r = e - w * 2 * n, q = r / n, x = r - q * n;
    const int z = z0 + 2 * w + q;
    if (z >= nz) continue;
    const float2 v = res[w * LS + x];
    a.out[(((size_t)b * a.np + p) * nz + z) * n + x] = (q ? v.y : v.x) * a.scale;
  }
}

// ------------------------------------------------------------ z passes

// column chunk [c][g] of lines c < CK (kx = k0 + c), g < L, from rows
// [g][kx] of `src` (row stride Mxh); rows g >= valid are zero
template <int L>
__device__ __forceinline__ void load_cols(float2 *s, const float2 *src, int k0, int Mxh, int valid) {
  constexpr int CK = col_chunk<L>(), LS = L + 1;
#pragma unroll 4
  for (int e = threadIdx.x; e < CK * L; e += FT_NT) {
    const int c = e % CK, g = e / CK, k = k0 + c;
    s[c * LS + g] = (g < valid && k < Mxh) ? src[(size_t)g * Mxh + k] : make_float2(0.f, 0.f);
  }
}

struct ColArgsD {
  const float2 *in;    // rows [b][plane][G][Mxh]
  float2 *out;
  const float2 *H;     // [ndist+1][Mz][Mxh]
  const int *views;
  const int *row_idist;
  int ndist, nplanes, G, P, nz, Mxh;
  float hscale;        // COL_H: normalisation of the spectra
  float2 *part;        // COL_FWD partial sums [pg][b][Mz][Mxh]
  int npg, nb;
};
constexpr int COL_H = 0, COL_BCK = 1;

__device__ __forceinline__ int spectrum_of(const ColArgsD &a, int b, int y) {
  const int view = a.views[b];
  const int d = a.row_idist ? a.row_idist[(size_t)view * a.nplanes + y] : -1;
  return d >= 0 ? d : a.ndist;
}

// COL_H: H[d] = FFT_g(rows) * hscale (all rows).  COL_BCK: per plane FFT,
// multiply by H[d(y)], inverse FFT, rows P..P+nz-1 back in place.
template <int L>
__global__ void __launch_bounds__(FT_NT) k_dfft_cols(ColArgsD a, int mode, const float2 *__restrict__ twg) {
  constexpr int CK = col_chunk<L>(), LS = L + 1;
  extern __shared__ __align__(16) float2 cs[];
  float2 *tw = cs, *s0 = cs + L, *s1 = s0 + CK * LS;
  for (int i = threadIdx.x; i < L; i += FT_NT) tw[i] = twg[i];
  const int k0 = blockIdx.x * CK, y = blockIdx.y, b = blockIdx.z;
  const int Mxh = a.Mxh;
  const size_t plane = ((size_t)b * a.nplanes + y) * a.G;
  load_cols<L>(s0, a.in + plane * Mxh, k0, Mxh, a.G);
  __syncthreads();
  float2 *res = fft_lines<L>(s0, s1, CK, LS, tw, 1.f);
  if (mode == COL_H) {
  #pragma unroll 4
  for (int e = threadIdx.x; e < CK * L; e += FT_NT) {
      const int c = e % CK, g = e / CK, k = k0 + c;
      if (k < Mxh) a.out[(plane + g) * Mxh + k] = cscale(res[c * LS + g], a.hscale);
    }
    return;
  }
  const float2 *Hd = a.H + (size_t)spectrum_of(a, b, y) * L * Mxh;
#pragma unroll 4
  for (int e = threadIdx.x; e < CK * L; e += FT_NT) {
    const int c = e % CK, g = e / CK, k = k0 + c;
    if (k < Mxh) res[c * LS + g] = cmul(res[c * LS + g], __ldg(Hd + (size_t)g * Mxh + k));
  }
  __syncthreads();
  float2 *other = res == s0 ? s1 : s0;
  res = fft_lines<L>(res, other, CK, LS, tw, -1.f);
  for (int e = threadIdx.x; e < CK * a.nz; e += FT_NT) {
    const int c = e % CK, z = e / CK, k = k0 + c;
    if (k < Mxh) a.out[(plane + a.P + z) * Mxh + k] = res[c * LS + a.P + z];
  }
}

// forward: per (kx chunk, view, plane group) sum over the group's planes of
// FFT_g(plane) * H[d(y)] -> part[pg][b][g][kx]
template <int L>
__global__ void __launch_bounds__(FT_NT) k_dfft_cols_fwd(ColArgsD a, const float2 *__restrict__ twg) {
  constexpr int CK = col_chunk<L>(), LS = L + 1;
  constexpr int NE = (CK * L + FT_NT - 1) / FT_NT;
  extern __shared__ __align__(16) float2 cs[];
  float2 *tw = cs, *s0 = cs + L, *s1 = s0 + CK * LS;
  for (int i = threadIdx.x; i < L; i += FT_NT) tw[i] = twg[i];
  const int k0 = blockIdx.x * CK, b = blockIdx.y, pg = blockIdx.z;
  const int Mxh = a.Mxh;
  const int per = (a.nplanes + a.npg - 1) / a.npg;
  const int y0 = pg * per, y1 = min(a.nplanes, y0 + per);
  float2 acc[NE];
#pragma unroll
  for (int i = 0; i < NE; ++i) acc[i] = make_float2(0.f, 0.f);
  for (int y = y0; y < y1; ++y) {
    const size_t plane = ((size_t)b * a.nplanes + y) * a.G;
    __syncthreads();
    load_cols<L>(s0, a.in + plane * Mxh, k0, Mxh, a.G);
    __syncthreads();
    const float2 *res = fft_lines<L>(s0, s1, CK, LS, tw, 1.f);
    const float2 *Hd = a.H + (size_t)spectrum_of(a, b, y) * L * Mxh;
#pragma unroll
    for (int i = 0; i < NE; ++i) {
      const int e = threadIdx.x + i * FT_NT;
      const int c = e % CK, g = e / CK, k = k0 + c;
      if (e < CK * L && k < Mxh) {
        const float2 v = cmul(res[c * LS + g], __ldg(Hd + (size_t)g * Mxh + k));
        acc[i] = cadd(acc[i], v);
      }
    }
  }
  float2 *P = a.part + ((size_t)pg * a.nb + b) * L * Mxh;
#pragma unroll
  for (int i = 0; i < NE; ++i) {
    const int e = threadIdx.x + i * FT_NT;
    const int c = e % CK, g = e / CK, k = k0 + c;
    if (e < CK * L && k < Mxh) P[(size_t)g * Mxh + k] = acc[i];
  }
}

// forward: partial sums in group order, inverse FFT along g, rows
// P..P+nz-1 -> out[b][z][kx]
template <int L>
__global__ void __launch_bounds__(FT_NT) k_dfft_fwd_finish(ColArgsD a, const float2 *__restrict__ twg) {
  constexpr int CK = col_chunk<L>(), LS = L + 1;
  extern __shared__ __align__(16) float2 cs[];
  float2 *tw = cs, *s0 = cs + L, *s1 = s0 + CK * LS;
  for (int i = threadIdx.x; i < L; i += FT_NT) tw[i] = twg[i];
  const int k0 = blockIdx.x * CK, b = blockIdx.y;
  const int Mxh = a.Mxh;
#pragma unroll 4
  for (int e = threadIdx.x; e < CK * L; e += FT_NT) {
    const int c = e % CK, g = e / CK, k = k0 + c;
    float2 v = make_float2(0.f, 0.f);
    if (k < Mxh)
      for (int pg = 0; pg < a.npg; ++pg) v = cadd(v, a.part[(((size_t)pg * a.nb + b) * L + g) * Mxh + k]);
    s0[c * LS + g] = v;
  }
  __syncthreads();
  const float2 *res = fft_lines<L>(s0, s1, CK, LS, tw, -1.f);
  for (int e = threadIdx.x; e < CK * a.nz; e += FT_NT) {
    const int c = e % CK, z = e / CK, k = k0 + c;
    if (k < Mxh) a.out[((size_t)b * a.nz + z) * Mxh + k] = res[c * LS + a.P + z];
  }
}

// ------------------------------------------------- one CTA per plane
// Square grids L x L (L = Mz = Mx) whose half spectrum fits shared memory:
// the row transforms, column transforms, PSF product and inverses of a
// plane run in one CTA (drf_plane.cuh), so the row spectra never travel
// through global memory.
//   backward: one CTA per (plane y, view b) -> bck[b][y][z][x];
//   forward:  one CTA per (plane group pg, view b) accumulates
//             sum_y H[d(y)] * FFT2(plane y) in registers -> part[pg][b];
//             the finish CTA of view b adds the groups in order, inverts
//             and writes out[b][z][x].

struct PlaneArgs {
  const float *a;       // plane (b, y) at a + b*a_bs + y*a_ys, [z][x]
  size_t a_bs, a_ys;
  const float *E;       // attenuation factors [view][y][z][x] or null
  const int *views, *row_idist, *pad_rows;
  int avgy, ndist;
  const float2 *H;      // [ndist + 1][L][L/2 + 1]
  int n, nz, P, G, nplanes;
  float scale;
  float *out;           // backward [b][y][z][x]; forward [b][z][x]
  float2 *part;         // forward partial sums [pg][b][L][L/2 + 1]
  int npg, nb;
};

// source of plane (b, y) and its PSF spectrum (the identity for rows
// without DRF, prjbck.c:233)
template <int L>
__device__ __forceinline__ const float2 *dp_plane_src(const PlaneArgs &a, int b, int y, PlaneSrc &p) {
  const int view = a.views[b];
  const size_t pln = (size_t)a.nz * a.n;
  p.a = a.a + (size_t)b * a.a_bs + (size_t)y * a.a_ys;
  p.e = a.E ? a.E + ((size_t)view * a.nplanes + y) * pln : nullptr;
  const int d = a.row_idist ? a.row_idist[(size_t)view * a.nplanes + y] : -1;
  p.pady = (d >= 0 && a.pad_rows) ? a.pad_rows[d] : 0;
  p.n = a.n;
  p.nz = a.nz;
  p.P = a.P;
  p.avgy = a.avgy;
  return a.H + (size_t)(d >= 0 ? d : a.ndist) * L * DPlane<L>::H;
}

// grid rows 0 .. G-1 of the plane -> half spectra S[g][kx].  Ends with a barrier.
template <int L>
__device__ __forceinline__ void dp_rows_forward(int tid, const PlaneSrc &p, int G, float2 *S, float2 *X,
                                                const float2 *twr) {
  using D = DPlane<L>;
  const int nl = (G + 1) / 2;
  const int src = dp_partner<L>(tid) & 31;
  for (int w0 = 0; w0 < nl; w0 += D::LINES) {
    dp_rows_fwd_a<L>(tid, w0, p, G, X, twr);
    __syncthreads();
    float2 u[D::N2], q[D::N2];
    dp_rows_b<L, false>(tid, X, u);
#pragma unroll
    for (int t = 0; t < D::N2; ++t) {
      q[t].x = __shfl_sync(0xffffffffu, u[t].x, src);
      q[t].y = __shfl_sync(0xffffffffu, u[t].y, src);
    }
    dp_rows_fwd_store<L>(tid, w0, G, u, q, S);
    __syncthreads();
  }
}

// spectrum rows r0 .. r0+nz-1 -> output rows [z][x], x < n, times scale
template <int L, bool PERM>
__device__ __forceinline__ void dp_rows_inverse(int tid, const float2 *S, float2 *X, const float2 *twr, int r0,
                                                int nz, int n, float *out, float scale) {
  using D = DPlane<L>;
  const int nl = (nz + 1) / 2;
  for (int w0 = 0; w0 < nl; w0 += D::LINES) {
    dp_rows_inv_a<L, PERM>(tid, w0, S, X, twr, r0, nz);
    __syncthreads();
    float2 u[D::N2];
    dp_rows_b<L, true>(tid, X, u);
    dp_rows_inv_store<L>(tid, w0, u, out, n, nz, scale);
    __syncthreads();
  }
}

// persistent: CTA i takes planes i, i + gridDim.x, ... (plane p = view
// p / nplanes, row p mod nplanes) and prefetches its next plane into L2
template <int L>
__global__ void __launch_bounds__(DP_NT, 1) k_dplane_bck(PlaneArgs a, const float2 *__restrict__ twg) {
  using D = DPlane<L>;
  extern __shared__ __align__(16) float2 dsm[];
  float2 *S = dsm, *X = S + D::S_ELEMS, *tw = X + D::X_ELEMS, *twr = tw + L;
  const int tid = threadIdx.x, total = a.nb * a.nplanes;
  dp_twiddles<L>(tid, tw, twr, twg);
  for (int pl = blockIdx.x; pl < total; pl += gridDim.x) {
    const int b = pl / a.nplanes, y = pl - b * a.nplanes;
    PlaneSrc p;
    const float2 *Hd = dp_plane_src<L>(a, b, y, p);
    if (pl + (int)gridDim.x < total) {
      const int nx = pl + gridDim.x, bn = nx / a.nplanes;
      PlaneSrc pn;
      dp_plane_src<L>(a, bn, nx - bn * a.nplanes, pn);
      dp_prefetch_plane(tid, pn);
    }
    __syncthreads();
    dp_rows_forward<L>(tid, p, a.G, S, X, twr);
    dp_cols_a<L>(tid, S, tw, a.G);
    __syncthreads();
    dp_cols_b_bck<L>(tid, S, tw, Hd);
    __syncthreads();
    dp_cols_c<L>(tid, S, a.P, a.P + a.nz);
    __syncthreads();
    dp_rows_inverse<L, false>(tid, S, X, twr, a.P, a.nz, a.n, a.out + ((size_t)b * a.nplanes + y) * a.nz * a.n,
                              a.scale);
  }
}

template <int L>
__global__ void __launch_bounds__(DP_NT, 1) k_dplane_fwd(PlaneArgs a, const float2 *__restrict__ twg) {
  using D = DPlane<L>;
  extern __shared__ __align__(16) float2 dsm[];
  float2 *S = dsm, *X = S + D::S_ELEMS, *tw = X + D::X_ELEMS, *twr = tw + L;
  const int tid = threadIdx.x, pg = blockIdx.x, b = blockIdx.y;
  const int y0 = pg * a.nplanes / a.npg, y1 = (pg + 1) * a.nplanes / a.npg;
  dp_twiddles<L>(tid, tw, twr, twg);
  float2 acc[D::NRB][D::N2];
#pragma unroll
  for (int r = 0; r < D::NRB; ++r)
#pragma unroll
    for (int k = 0; k < D::N2; ++k) acc[r][k] = make_float2(0.f, 0.f);
  __syncthreads();
  for (int y = y0; y < y1; ++y) {
    PlaneSrc p;
    const float2 *Hd = dp_plane_src<L>(a, b, y, p);
    if (y + 1 < y1) {
      PlaneSrc pn;
      dp_plane_src<L>(a, b, y + 1, pn);
      dp_prefetch_plane(tid, pn);
    }
    dp_rows_forward<L>(tid, p, a.G, S, X, twr);
    dp_cols_a<L>(tid, S, tw, a.G);
    __syncthreads();
    dp_cols_b_acc<L>(tid, S, Hd, acc);
    __syncthreads();
  }
  dp_store_acc<L>(tid, a.part + ((size_t)pg * a.nb + b) * L * D::H, acc);
}

template <int L>
__global__ void __launch_bounds__(DP_NT, 1) k_dplane_fwd_finish(PlaneArgs a, const float2 *__restrict__ twg) {
  using D = DPlane<L>;
  extern __shared__ __align__(16) float2 dsm[];
  float2 *S = dsm, *X = S + D::S_ELEMS, *tw = X + D::X_ELEMS, *twr = tw + L;
  const int tid = threadIdx.x, b = blockIdx.x;
  dp_twiddles<L>(tid, tw, twr, twg);
  __syncthreads();
  dp_fin_b<L>(tid, S, tw, a.part + (size_t)b * L * D::H, (size_t)a.nb * L * D::H, a.npg);
  __syncthreads();
  dp_fin_c<L>(tid, S);
  __syncthreads();
  dp_rows_inverse<L, true>(tid, S, X, twr, a.P, a.nz, a.n, a.out + (size_t)b * a.nz * a.n, a.scale);
}

// -------------------------------------------------------------- host side

// grid lengths with instantiated kernels
static const int kLens[] = {16, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256, 320, 384, 512, 640, 768, 1024};

static int grid_len(int need) {
  for (int L : kLens)
    if (L >= need) return L;
  return -1;
}

#define DFFT_DISPATCH(L, ...)                                                       \
  switch (L) {                                                                     \
    case 16: { constexpr int LL = 16; __VA_ARGS__; } break;                       \
    case 24: { constexpr int LL = 24; __VA_ARGS__; } break;                       \
    case 32: { constexpr int LL = 32; __VA_ARGS__; } break;                       \
    case 40: { constexpr int LL = 40; __VA_ARGS__; } break;                       \
    case 48: { constexpr int LL = 48; __VA_ARGS__; } break;                       \
    case 64: { constexpr int LL = 64; __VA_ARGS__; } break;                       \
    case 80: { constexpr int LL = 80; __VA_ARGS__; } break;                       \
    case 96: { constexpr int LL = 96; __VA_ARGS__; } break;                       \
    case 128: { constexpr int LL = 128; __VA_ARGS__; } break;                     \
    case 160: { constexpr int LL = 160; __VA_ARGS__; } break;                     \
    case 192: { constexpr int LL = 192; __VA_ARGS__; } break;                     \
    case 256: { constexpr int LL = 256; __VA_ARGS__; } break;                     \
    case 320: { constexpr int LL = 320; __VA_ARGS__; } break;                     \
    case 384: { constexpr int LL = 384; __VA_ARGS__; } break;                     \
    case 512: { constexpr int LL = 512; __VA_ARGS__; } break;                     \
    case 640: { constexpr int LL = 640; __VA_ARGS__; } break;                     \
    case 768: { constexpr int LL = 768; __VA_ARGS__; } break;                     \
    case 1024: { constexpr int LL = 1024; __VA_ARGS__; } break;                   \
    default: return set_error(IRLCU_EARG, "DRF FFT length %d not supported", L);   \
  }

// square grid lengths of the one-CTA-per-plane kernels
static const int kPlaneLens[] = {32, 40, 48, 64, 80, 96, 128, 160, 192};

#define DPLANE_DISPATCH(L, ...)                                                    \
  switch (L) {                                                                    \
    case 32: { constexpr int LL = 32; __VA_ARGS__; } break;                      \
    case 40: { constexpr int LL = 40; __VA_ARGS__; } break;                      \
    case 48: { constexpr int LL = 48; __VA_ARGS__; } break;                      \
    case 64: { constexpr int LL = 64; __VA_ARGS__; } break;                      \
    case 80: { constexpr int LL = 80; __VA_ARGS__; } break;                      \
    case 96: { constexpr int LL = 96; __VA_ARGS__; } break;                      \
    case 128: { constexpr int LL = 128; __VA_ARGS__; } break;                    \
    case 160: { constexpr int LL = 160; __VA_ARGS__; } break;                    \
    case 192: { constexpr int LL = 192; __VA_ARGS__; } break;                    \
    default: return set_error(IRLCU_EARG, "DRF plane length %d not supported", L); \
  }

static size_t dplane_smem(int L) {
  size_t sm = 0;
  switch (L) {
#define DPLANE_SMEM_CASE(X) case X: sm = DPlane<X>::SMEM; break;
    DPLANE_SMEM_CASE(32) DPLANE_SMEM_CASE(40) DPLANE_SMEM_CASE(48) DPLANE_SMEM_CASE(64) DPLANE_SMEM_CASE(80)
    DPLANE_SMEM_CASE(96) DPLANE_SMEM_CASE(128) DPLANE_SMEM_CASE(160) DPLANE_SMEM_CASE(192)
#undef DPLANE_SMEM_CASE
    default: break;
  }
  return sm;
}

// the one-CTA-per-plane form for an L x L grid: instantiated length, shared
// memory within the device limit, not switched off (IRLCU_DRF_PLANE=0)
static bool dplane_usable(int L) {
  const char *env = getenv("IRLCU_DRF_PLANE");
  if (env && env[0] == '0') return false;
  bool len = false;
  for (int l : kPlaneLens) len = len || l == L;
  if (!len) return false;
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return dplane_smem(L) <= (size_t)maxsm;
}

template <int L>
static int dplane_attrs() {
  static bool done = false;
  if (done) return IRLCU_OK;
  const int sm = (int)DPlane<L>::SMEM;
  CU_TRY(cudaFuncSetAttribute(k_dplane_bck<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CU_TRY(cudaFuncSetAttribute(k_dplane_fwd<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CU_TRY(cudaFuncSetAttribute(k_dplane_fwd_finish<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  done = true;
  return IRLCU_OK;
}

static int sm_count() {
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 1;
  }
  return nsm;
}

// plane groups of the forward pass: one CTA per SM over the batch
static int dplane_groups(int nv, int nplanes) {
  const int g = sm_count() / std::max(nv, 1);
  return std::max(1, std::min(g, std::min(16, nplanes)));
}

// CTAs of the persistent backward pass: one per SM
static int dplane_ctas(int planes) { return std::max(1, std::min(planes, sm_count())); }

template <int L>
static int set_col_attrs() {
  static bool done = false;
  if (done) return IRLCU_OK;
  const int sm = (int)col_smem<L>();
  CU_TRY(cudaFuncSetAttribute(k_dfft_cols<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CU_TRY(cudaFuncSetAttribute(k_dfft_cols_fwd<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CU_TRY(cudaFuncSetAttribute(k_dfft_fwd_finish<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  done = true;
  return IRLCU_OK;
}



static int grow(cudaStream_t st, float2 **p, size_t *have, size_t need) {
  if (need <= *have) return IRLCU_OK;
  dev_free(*p, st);
  *p = nullptr;
  *have = 0;
  CU_TRY(dev_alloc_t(p, need, st));
  *have = need;
  return IRLCU_OK;
}

void drf_fft_free(Ctx &c, DrfDev &D) {
  dev_free(D.fft.H, c.st);
  dev_free(D.fft.twx, c.st);
  dev_free(D.fft.twz, c.st);
  D.fft = DrfFft{};
}

void drf_fft_work_free(Ctx &c) {
  dev_free(c.dw.S, c.st);
  dev_free(c.dw.part, c.st);
  dev_free(c.dw.Y, c.st);
  c.dw = DfftWork{};
}

// plane groups of the forward column pass
static int fwd_groups(int nplanes) { return nplanes < 16 ? nplanes : 16; }

int drf_fft_setup(Ctx &c, DrfDev &D, int max_pad) {
  drf_fft_free(c, D);
  const int n = c.n, nz = c.nz, h = D.halo;
  int Mx = grid_len(n + h), Mz = grid_len(nz + max_pad + h);
  if (Mx < 0 || Mz < 0 || Mx < 2 * h + 1 || Mz < 2 * h + 1)
    return set_error(IRLCU_EARG, "DRF FFT grid for n=%d nz=%d h=%d pad=%d exceeds %d", n, nz, h, max_pad, 1024);
  DrfFft &F = D.fft;
  // one CTA per plane on a square grid when it fits shared memory (a larger
  // grid than needed along one axis leaves the linear convolution unchanged)
  F.fused = dplane_usable(std::max(Mx, Mz));
  if (F.fused) Mx = Mz = std::max(Mx, Mz);
  F.Mx = Mx;
  F.Mz = Mz;
  F.Mxh = Mx / 2 + 1;
  F.P = max_pad;
  F.G = nz + 2 * max_pad;
  if (F.G > Mz) F.G = Mz;
  TRY_RC(upload_twiddle_table(c.st, &F.twx, Mx));
  TRY_RC(upload_twiddle_table(c.st, &F.twz, Mz));
  const int nspec = D.ndist + 1;
  CU_TRY(dev_alloc_t(&F.H, (size_t)nspec * Mz * F.Mxh, c.st));
  // work: row spectra for max_batch views (also holds the PSF rows here)
  const int B = c.g.max_batch;
  // (the plane form needs only the partial sums; S holds the PSF rows here)
  const size_t s_need = (size_t)nspec * Mz * F.Mxh;
  TRY_RC(grow(c.st, &c.dw.S, &c.dw.s_elems, F.fused ? s_need : std::max((size_t)B * n * F.G * F.Mxh, s_need)));
  TRY_RC(grow(c.st, &c.dw.part, &c.dw.part_elems, (size_t)fwd_groups(n) * B * Mz * F.Mxh));
  if (!F.fused) TRY_RC(grow(c.st, &c.dw.Y, &c.dw.y_elems, (size_t)B * nz * F.Mxh));
  // spectra of the quadrant-swapped PSFs (and the identity), 1/(Mz Mx)
  RowSrc r{};
  r.mode = MODE_PSF;
  r.psf = D.psf;
  r.h = h;
  r.pstride = D.pstride;
  r.ndist = D.ndist;
  r.n = n;
  r.nz = nz;
  r.G = Mz;
  r.Mz = Mz;
  r.out = c.dw.S;
  r.Mxh = F.Mxh;
  r.nplanes = nspec;
  DFFT_DISPATCH(Mx, {
    dim3 grid((Mz + 2 * rows_pairs<LL>() - 1) / (2 * rows_pairs<LL>()), nspec, 1);
    k_dfft_rows_fwd<LL><<<grid, FT_NT, 0, c.st>>>(r, F.twx);
    CU_LAUNCHED();
  });
  ColArgsD ca{};
  ca.in = c.dw.S;
  ca.out = F.H;
  ca.nplanes = nspec;
  ca.G = Mz;
  ca.Mxh = F.Mxh;
  ca.hscale = (float)(1.0 / ((double)Mz * Mx));
  DFFT_DISPATCH(Mz, {
    TRY_RC(set_col_attrs<LL>());
    dim3 grid((F.Mxh + col_chunk<LL>() - 1) / col_chunk<LL>(), nspec, 1);
    k_dfft_cols<LL><<<grid, FT_NT, col_smem<LL>(), c.st>>>(ca, COL_H, F.twz);
    CU_LAUNCHED();
  });
  CU_TRY(cudaStreamSynchronize(c.st));
  F.on = true;
  return IRLCU_OK;
}

static RowSrc plane_rows(const Ctx &c, const DrfDev &D, const float *a, size_t a_bs, size_t a_ys, const float *E,
                         const int *dviews) {
  RowSrc r{};
  r.mode = MODE_PLANE;
  r.a = a;
  r.a_bs = a_bs;
  r.a_ys = a_ys;
  r.E = E;
  r.views = dviews;
  r.row_idist = D.row_idist;
  r.pad_rows = D.pad_rows;
  r.avgy = D.avg_rows;
  r.n = c.n;
  r.nz = c.nz;
  r.P = D.fft.P;
  r.G = D.fft.G;
  r.Mz = D.fft.Mz;
  r.out = c.dw.S;
  r.Mxh = D.fft.Mxh;
  r.nplanes = c.n;
  return r;
}

static ColArgsD col_args(const Ctx &c, const DrfDev &D, const int *dviews, int nv) {
  ColArgsD a{};
  a.in = c.dw.S;
  a.H = D.fft.H;
  a.views = dviews;
  a.row_idist = D.row_idist;
  a.ndist = D.ndist;
  a.nplanes = c.n;
  a.G = D.fft.G;
  a.P = D.fft.P;
  a.nz = c.nz;
  a.Mxh = D.fft.Mxh;
  a.part = c.dw.part;
  a.npg = fwd_groups(c.n);
  a.nb = nv;
  return a;
}

static PlaneArgs plane_args(const Ctx &c, const DrfDev &D, const float *a, size_t a_bs, size_t a_ys, const float *E,
                            const int *dviews, float scale, float *out) {
  PlaneArgs p{};
  p.a = a;
  p.a_bs = a_bs;
  p.a_ys = a_ys;
  p.E = E;
  p.views = dviews;
  p.row_idist = D.row_idist;
  p.pad_rows = D.pad_rows;
  p.avgy = D.avg_rows;
  p.ndist = D.ndist;
  p.H = D.fft.H;
  p.n = c.n;
  p.nz = c.nz;
  p.P = D.fft.P;
  p.G = D.fft.G;
  p.nplanes = c.n;
  p.scale = scale;
  p.out = out;
  return p;
}

static int launch_project_plane(const Ctx &c, const float *src, const int *dviews, int nv, const float *E,
                                const DrfDev &D, float scale, float *out) {
  const DrfFft &F = D.fft;
  PlaneArgs a = plane_args(c, D, src, c.vox, c.pln, E, dviews, scale, out);
  a.part = c.dw.part;
  a.nb = nv;
  a.npg = dplane_groups(nv, c.n);
  if ((size_t)a.npg * nv * F.Mz * F.Mxh > c.dw.part_elems)
    return set_error(IRLCU_EARG, "DRF FFT batch of %d views exceeds the work buffers", nv);
  DPLANE_DISPATCH(F.Mx, {
    TRY_RC(dplane_attrs<LL>());
    k_dplane_fwd<LL><<<dim3(a.npg, nv), DP_NT, DPlane<LL>::SMEM, c.st>>>(a, F.twx);
    CU_LAUNCHED();
    k_dplane_fwd_finish<LL><<<nv, DP_NT, DPlane<LL>::SMEM, c.st>>>(a, F.twx);
    CU_LAUNCHED();
  });
  return IRLCU_OK;
}

int launch_project_fft(const Ctx &c, const float *src, const int *dviews, int nv, const float *E, const DrfDev &D,
                       float scale, float *out) {
  const DrfFft &F = D.fft;
  if (F.fused) return launch_project_plane(c, src, dviews, nv, E, D, scale, out);
  if ((size_t)nv * c.n * F.G * F.Mxh > c.dw.s_elems || (size_t)nv * c.nz * F.Mxh > c.dw.y_elems ||
      (size_t)fwd_groups(c.n) * nv * F.Mz * F.Mxh > c.dw.part_elems)
    return set_error(IRLCU_EARG, "DRF FFT batch of %d views exceeds the work buffers", nv);
  const RowSrc r = plane_rows(c, D, src, c.vox, c.pln, E, dviews);
  DFFT_DISPATCH(F.Mx, {
    dim3 grid((F.G + 2 * rows_pairs<LL>() - 1) / (2 * rows_pairs<LL>()), c.n, nv);
    k_dfft_rows_fwd<LL><<<grid, FT_NT, 0, c.st>>>(r, F.twx);
    CU_LAUNCHED();
  });
  ColArgsD a = col_args(c, D, dviews, nv);
  a.out = c.dw.Y;
  DFFT_DISPATCH(F.Mz, {
    TRY_RC(set_col_attrs<LL>());
    const int nch = (F.Mxh + col_chunk<LL>() - 1) / col_chunk<LL>();
    k_dfft_cols_fwd<LL><<<dim3(nch, nv, a.npg), FT_NT, col_smem<LL>(), c.st>>>(a, F.twz);
    CU_LAUNCHED();
    k_dfft_fwd_finish<LL><<<dim3(nch, nv, 1), FT_NT, col_smem<LL>(), c.st>>>(a, F.twz);
    CU_LAUNCHED();
  });
  RowInv ri{};
  ri.in = c.dw.Y;
  ri.np = 1;
  ri.rs = c.nz;
  ri.r0 = 0;
  ri.Mxh = F.Mxh;
  ri.out = out;
  ri.n = c.n;
  ri.nz = c.nz;
  ri.scale = scale;
  DFFT_DISPATCH(F.Mx, {
    dim3 grid((c.nz + 2 * rows_pairs<LL>() - 1) / (2 * rows_pairs<LL>()), 1, nv);
    k_dfft_rows_inv<LL><<<grid, FT_NT, 0, c.st>>>(ri, F.twx);
    CU_LAUNCHED();
  });
  return IRLCU_OK;
}

int launch_backproject_fft(const Ctx &c, const float *planes, const int *dviews, int nv, const float *E,
                           const DrfDev &D, float scale, float *bck) {
  const DrfFft &F = D.fft;
  if (F.fused) {
    PlaneArgs a = plane_args(c, D, planes, c.pln, 0, E, dviews, scale, bck);
    a.nb = nv;
    DPLANE_DISPATCH(F.Mx, {
      TRY_RC(dplane_attrs<LL>());
      k_dplane_bck<LL><<<dplane_ctas(nv * c.n), DP_NT, DPlane<LL>::SMEM, c.st>>>(a, F.twx);
      CU_LAUNCHED();
    });
    return IRLCU_OK;
  }
  if ((size_t)nv * c.n * F.G * F.Mxh > c.dw.s_elems)
    return set_error(IRLCU_EARG, "DRF FFT batch of %d views exceeds the work buffers", nv);
  const RowSrc r = plane_rows(c, D, planes, c.pln, 0, E, dviews);
  DFFT_DISPATCH(F.Mx, {
    dim3 grid((F.G + 2 * rows_pairs<LL>() - 1) / (2 * rows_pairs<LL>()), c.n, nv);
    k_dfft_rows_fwd<LL><<<grid, FT_NT, 0, c.st>>>(r, F.twx);
    CU_LAUNCHED();
  });
  ColArgsD a = col_args(c, D, dviews, nv);
  a.out = c.dw.S;
  DFFT_DISPATCH(F.Mz, {
    TRY_RC(set_col_attrs<LL>());
    const int nch = (F.Mxh + col_chunk<LL>() - 1) / col_chunk<LL>();
    k_dfft_cols<LL><<<dim3(nch, c.n, nv), FT_NT, col_smem<LL>(), c.st>>>(a, COL_BCK, F.twz);
    CU_LAUNCHED();
  });
  RowInv ri{};
  ri.in = c.dw.S;
  ri.np = c.n;
  ri.rs = F.G;
  ri.r0 = F.P;
  ri.Mxh = F.Mxh;
  ri.out = bck;
  ri.n = c.n;
  ri.nz = c.nz;
  ri.scale = scale;
  DFFT_DISPATCH(F.Mx, {
    dim3 grid((c.nz + 2 * rows_pairs<LL>() - 1) / (2 * rows_pairs<LL>()), c.n, nv);
    k_dfft_rows_inv<LL><<<grid, FT_NT, 0, c.st>>>(ri, F.twx);
    CU_LAUNCHED();
  });
  return IRLCU_OK;
}

}  // namespace irlcu
