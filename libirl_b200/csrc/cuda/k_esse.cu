// k_esse.cu -- ESSE effective scatter source on the GPU (libirl
// krnlprj3d.c:676-954, CalcEffScatterSource) and the FFT it needs.
//
// Per view of a batch (all in the view's rotated frame, layout [y][z][x]):
//   1. collapse the rotated activity by c (sum pooling, CollapseByFac) and
//      zero-pad it into the Ky x Kz x Kx FFT grid: a streaming pass
//      (k_esse_collapse) ahead of the register x transform, or fused into
//      the first FFT pass of the pass form; only the rows that hold data
//      are transformed;
//   2. forward 3D DFT (x, z, y passes; z and y skip the known-zero lines);
//   3. for the zeroth and first Taylor terms: multiply by the kernel spectra
//      K^ and (K (mu - mu_avg))^, inverse 3D DFT (y, z, x passes, each
//      keeping only the cropped output region), i.e. the circular
//      convolution of krnlprj3d.c:783-790, 815-817;
//   4. expand by c with libirl's recursive (in place) (c+1)-point smoothing
//      along y, then z, then x (ExpandByFac, krnlprj3d.c:595-673); lines
//      that receive the same inputs are smoothed once (coarse z and x after
//      the y pass, coarse x after the z pass);
//   5. combine with the depth and density terms: eff = T0 - d*T1,
//      eff *= exp(d*(mu0-mu_avg)), eff += act*CntrPixFac, eff *= mu/(mu0*pix),
//      clamp at 0 (krnlprj3d.c:833-946), and form the projector source
//      act*fPrimaryFac + eff (prjbck.c:170-173).
// Steps 4-5 round exactly like libirl's float code.  The DFTs are FP32
// (libirl uses an external FFT library), so the source agrees with libirl to
// FFT rounding rather than bit for bit.
//
// FFT: batched line transforms of fft_core.cuh; the ESSE grids are powers
// of two from 8 to 1024.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "esse_rows.cuh"
#include "esse_walk.cuh"
#include "esse_yz.cuh"
#include "fft_core.cuh"
#include "irlcu_internal.cuh"

namespace irlcu {

#define TRY_ESSE(x)      \
  do {                 \
    int rc_ = (x);     \
    if (rc_) return rc_; \
  } while (0)

// ----------------------------------------------------------- pass kernels

// Row pass (x axis).  Forward: input real rows from a loader, output bins
// [0, L/2] of every row.  Inverse: input bins [0, L/2] (Hermitian
// extension), output real part * scale for x < nx_out.
struct RowFwdArgs {
  // collapsed rotated activity source (ESSE) or a plain real grid (kernel)
  const float *rot;     // B volumes [n][nz][n] (rotated activity) or null
  const float *grid;    // real grid [Ky][Kz][Kx] (kernel set-up) or null
  int n, nz, c;         // full volume size and collapse factor
  int nyv, nzv, nxv;    // valid (collapsed) extents: rows y'<nyv, z'<nzv, x'<nxv
  size_t vox;
  float2 *out;          // [B][nyv][zext][kxh] with zext >= nzv, or kx-major
  int zext, kxh;
  int kmajor;           // 1: out is [B][kxh][nyv][nzv] (planes of fixed kx)
  const float *pre;     // register form: B collapsed volumes [nyv][nzv][nxv], or null
};

// rows per CTA of the x passes (host: row_wr)
template <int L>
__host__ __device__ constexpr int row_lines() { return (L <= 128) ? 16 : (L <= 256 ? 4 : 2); }

template <int L>
__global__ void k_fft_row_fwd(RowFwdArgs a, const float2 *__restrict__ twg) {
  constexpr int WR = row_lines<L>();
  constexpr int LS = L + 1;  // padded line stride: row-major walks are conflict-free
  __shared__ float2 tw[L];
  __shared__ float2 sa[WR * LS], sb[WR * LS];
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = twg[i];
  const int b = blockIdx.y;
  const int row0 = blockIdx.x * WR;  // row = y' * nzv + z'
  const int nrows = a.nyv * a.nzv;
  for (int e = threadIdx.x; e < WR * L; e += blockDim.x) {
    const int w = e / L, x = e - w * L, row = row0 + w;
    float v = 0.f;
    if (row < nrows && x < a.nxv) {
      const int yy = row / a.nzv, zz = row - yy * a.nzv;
      if (a.rot && a.c == 2 && (a.n & 1) == 0) {
        // CollapseByFac (krnlprj3d.c:549-593) for c = 2: the two x offsets
        // of a (y, z) offset pair are one aligned float2
        const float *r = a.rot + (size_t)b * a.vox;
        float t = 0.f;
#pragma unroll
        for (int k = 0; k < 2; ++k)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const float2 q = __ldg(reinterpret_cast<const float2 *>(
                r + ((size_t)(yy * 2 + k) * a.nz + (zz * 2 + j)) * a.n + x * 2));
            t = __fadd_rn(__fadd_rn(t, q.x), q.y);
          }
        v = t;
      } else if (a.rot) {
        // CollapseByFac (krnlprj3d.c:549-593): sum over y, then z, then x offsets
        const float *r = a.rot + (size_t)b * a.vox;
        float t = 0.f;
        for (int k = 0; k < a.c; ++k)
          for (int j = 0; j < a.c; ++j)
            for (int i = 0; i < a.c; ++i)
              t = __fadd_rn(t, __ldg(r + ((size_t)(yy * a.c + k) * a.nz + (zz * a.c + j)) * a.n + x * a.c + i));
        v = t;
      } else {
        v = __ldg(a.grid + ((size_t)yy * a.zext + zz) * L + x);
      }
    }
    sa[w * LS + x] = make_float2(v, 0.f);
  }
  __syncthreads();
  float2 *res = fft_lines<L>(sa, sb, WR, LS, tw, 1.f);
  const int kxh = a.kxh;
  if (a.kmajor) {
    // kx-major: consecutive threads take consecutive rows (contiguous in out)
    for (int e = threadIdx.x; e < WR * kxh; e += blockDim.x) {
      const int k = e / WR, w = e - k * WR, row = row0 + w;
      if (row >= nrows) continue;
      a.out[((size_t)b * kxh + k) * nrows + row] = res[w * LS + k];
    }
  } else {
    for (int e = threadIdx.x; e < WR * kxh; e += blockDim.x) {
      const int w = e / kxh, k = e - w * kxh, row = row0 + w;
      if (row >= nrows) continue;
      const int yy = row / a.nzv, zz = row - yy * a.nzv;
      a.out[(((size_t)b * a.nyv + yy) * a.zext + zz) * kxh + k] = res[w * LS + k];
    }
  }
}

struct RowInvArgs {
  const float2 *in[2];  // [B][nyv][nzv][kxh] per term, or kx-major [B][kxh][nyv][nzv]
  float *out[2];        // [B][nyv][nzv][nxv] per term (cropped real grid)
  int nt, nyv, nzv, nxv, kxh;
  float scale;
  int kmajor;
};

template <int L>
__global__ void k_fft_row_inv(RowInvArgs a, const float2 *__restrict__ twg) {
  constexpr int WR = row_lines<L>();
  constexpr int LS = L + 1;  // padded line stride: row-major walks are conflict-free
  __shared__ float2 tw[L];
  __shared__ float2 sa[WR * LS], sb[WR * LS];
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = twg[i];
  const int b = blockIdx.y;
  const int row0 = blockIdx.x * WR;
  const int nrows = a.nyv * a.nzv;
  for (int t = 0; t < a.nt; ++t) {
    __syncthreads();
    if (a.kmajor) {
      // kx-major input: consecutive threads read consecutive rows; the
      // conjugate-symmetric half is filled from shared memory below
      for (int e = threadIdx.x; e < WR * a.kxh; e += blockDim.x) {
        const int k = e / WR, w = e - k * WR, row = row0 + w;
        sa[w * LS + k] = row < nrows ? a.in[t][((size_t)b * a.kxh + k) * nrows + row] : make_float2(0.f, 0.f);
      }
      __syncthreads();
      for (int e = threadIdx.x; e < WR * (L - a.kxh); e += blockDim.x) {
        const int w = e / (L - a.kxh), k = a.kxh + (e - w * (L - a.kxh));
        const float2 c = sa[w * LS + (L - k)];
        sa[w * LS + k] = make_float2(c.x, -c.y);
      }
    } else {
      for (int e = threadIdx.x; e < WR * L; e += blockDim.x) {
        const int w = e / L, k = e - w * L, row = row0 + w;
        float2 v = make_float2(0.f, 0.f);
        if (row < nrows) {
          const int kk = k < a.kxh ? k : L - k;
          const float2 c = a.in[t][((size_t)b * nrows + row) * a.kxh + kk];
          v = k < a.kxh ? c : make_float2(c.x, -c.y);
        }
        sa[w * LS + k] = v;
      }
    }
    __syncthreads();
    float2 *res = fft_lines<L>(sa, sb, WR, LS, tw, -1.f);
    for (int e = threadIdx.x; e < WR * a.nxv; e += blockDim.x) {
      const int w = e / a.nxv, x = e - w * a.nxv, row = row0 + w;
      if (row >= nrows) continue;
      a.out[t][((size_t)b * nrows + row) * a.nxv + x] = res[w * LS + x].x * a.scale;
    }
  }
}

// x transforms with register transforms (esse_rows.cuh), kx-major layout:
// one CTA per ER_LW row pairs of a view (and term)
// CollapseByFac of nb rotated volumes into [b][y'][z'][x'], a thread per
// collapsed value (consecutive x' in consecutive threads), summed as in
// er_collapse
__global__ void __launch_bounds__(256) k_esse_collapse(const float *__restrict__ rot, size_t vox, int n, int nz, int c,
                                                       int nyv, int nzv, int nxv, int nb, float *__restrict__ out) {
  const size_t per = (size_t)nyv * nzv * nxv;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)nb * per) return;
  const int b = (int)(e / per);
  const size_t i = e - (size_t)b * per;
  const int x = (int)(i % nxv);
  const size_t r = i / nxv;
  const int y = (int)(r / nzv), z = (int)(r - (size_t)y * nzv);
  out[e] = er_collapse(rot + (size_t)b * vox, n, nz, c, y, z, x);
}

template <int L, bool PRE>
__global__ void __launch_bounds__(ER_NT, 2) k_esse_row_fwd_reg(RowFwdArgs a, const float2 *__restrict__ twg) {
  using D = ERow<L>;
  extern __shared__ __align__(16) float2 ers[];
  float2 *X = ers, *tw = X + D::X_ELEMS;
  const int tid = threadIdx.x, b = blockIdx.y, w0 = blockIdx.x * ER_LW;
  const int nrows = a.nyv * a.nzv;
  for (int i = tid; i < L; i += ER_NT) tw[i] = twg[i];
  __syncthreads();
  er_fwd_a<L, PRE>(tid, w0, X, tw, a.rot + (size_t)b * a.vox, a.n, a.nz, a.c, a.nzv, a.nxv, nrows,
                   PRE ? a.pre + (size_t)b * nrows * a.nxv : nullptr);
  __syncthreads();
  constexpr int NB = (ER_LW * D::N1 + ER_NT - 1) / ER_NT;
  float2 u[NB][D::N2];
#pragma unroll
  for (int r = 0; r < NB; ++r) {
    const int it = tid + r * ER_NT;
    if (it < ER_LW * D::N1) er_b<L, false>(it, X, u[r]);
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < NB; ++r) {
    const int it = tid + r * ER_NT;
    if (it < ER_LW * D::N1) er_fwd_b_store<L>(it, u[r], X);
  }
  __syncthreads();
  er_fwd_unpack<L>(tid, w0, X, a.out + (size_t)b * a.kxh * nrows, nrows);
}

// grid (row-pair blocks, view, term)
template <int L>
__global__ void __launch_bounds__(ER_NT, 3) k_esse_row_inv_reg(RowInvArgs a, const float2 *__restrict__ twg) {
  using D = ERow<L>;
  extern __shared__ __align__(16) float2 ers[];
  float2 *X = ers, *tw = X + D::X_ELEMS;
  const int tid = threadIdx.x, b = blockIdx.y, t = blockIdx.z, w0 = blockIdx.x * ER_LW;
  const int nrows = a.nyv * a.nzv;
  for (int i = tid; i < L; i += ER_NT) tw[i] = twg[i];
  __syncthreads();
  er_inv_a<L>(tid, w0, X, tw, (t ? a.in[1] : a.in[0]) + (size_t)b * a.kxh * nrows, nrows);
  __syncthreads();
  float *out = (t ? a.out[1] : a.out[0]) + (size_t)b * nrows * a.nxv;
  for (int it = tid; it < ER_LW * D::N1; it += ER_NT) {
    float2 u[D::N2];
    er_b<L, true>(it, X, u);
    er_inv_b_store<L>(it, w0, u, out, nrows, a.nxv, a.scale);
  }
}

static bool er_len_ok(int L) { return L == 32 || L == 64 || L == 128 || L == 256; }

static int er_attrs(int L) {
  static bool done = false;
  if (done) return IRLCU_OK;
  CU_TRY(cudaFuncSetAttribute(k_esse_row_fwd_reg<256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ERow<256>::SMEM));
  CU_TRY(cudaFuncSetAttribute(k_esse_row_fwd_reg<256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ERow<256>::SMEM));
  CU_TRY(cudaFuncSetAttribute(k_esse_row_inv_reg<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ERow<256>::SMEM));
  (void)L;
  done = true;
  return IRLCU_OK;
}

#define ER_DISPATCH(L, ...)                                  \
  switch (L) {                                               \
    case 32: { constexpr int LL = 32; __VA_ARGS__; } break;  \
    case 64: { constexpr int LL = 64; __VA_ARGS__; } break;  \
    case 128: { constexpr int LL = 128; __VA_ARGS__; } break; \
    default: { constexpr int LL = 256; __VA_ARGS__; } break; \
  }

// Column pass (z or y axis): lines are (outer, kx); 16 consecutive kx per
// CTA for coalescing.  Input point p of line (b, o, kx) at
//   in + b*in_bs + o*in_os + p*in_ps + kx      (zero for p >= in_valid)
// output point p (< out_valid) at the same form with out_*; optionally the
// input is multiplied by nt kernel spectra (each with its own strides,
// batch-invariant) producing nt outputs.
struct ColArgs {
  const float2 *in;
  size_t in_bs, in_os, in_ps;
  int in_valid;
  const float2 *mul[2];
  size_t mul_os, mul_ps;
  float2 *out[2];
  size_t out_bs, out_os, out_ps;
  int out_valid;
  int nt, kxh, nouter;
  float s;
};

constexpr int CW = 16;

template <int L>
__global__ void k_fft_col(ColArgs a, const float2 *__restrict__ twg) {
  extern __shared__ __align__(16) float2 smc[];
  constexpr int LS = L + 1;              // odd line stride: the kx-fastest loads and stores are conflict-free
  float2 *tw = smc;
  float2 *sa = smc + L;                  // [CW][LS]
  float2 *sb = sa + CW * LS;
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = twg[i];
  const int kx0 = blockIdx.x * CW, o = blockIdx.y, b = blockIdx.z;
  const int wv = min(CW, a.kxh - kx0);
  for (int t = 0; t < a.nt; ++t) {
    __syncthreads();
    for (int e = threadIdx.x; e < L * CW; e += blockDim.x) {
      const int p = e / CW, w = e - p * CW;  // w fastest: coalesced along kx
      float2 v = make_float2(0.f, 0.f);
      if (w < wv && p < a.in_valid) {
        v = a.in[(size_t)b * a.in_bs + (size_t)o * a.in_os + (size_t)p * a.in_ps + kx0 + w];
        if (a.mul[t]) v = cmul(v, __ldg(&a.mul[t][(size_t)o * a.mul_os + (size_t)p * a.mul_ps + kx0 + w]));
      }
      sa[w * LS + p] = v;
    }
    __syncthreads();
    float2 *res = fft_lines<L>(sa, sb, CW, LS, tw, a.s);
    for (int e = threadIdx.x; e < a.out_valid * CW; e += blockDim.x) {
      const int p = e / CW, w = e - p * CW;
      if (w < wv)
        a.out[t][(size_t)b * a.out_bs + (size_t)o * a.out_os + (size_t)p * a.out_ps + kx0 + w] = res[w * LS + p];
    }
  }
}

// ------------------------------------------------ fused y-z plane kernel
// One CTA per (view, kx) holds the whole (y, z) plane of that x-frequency
// in shared memory: forward z and y transforms, then for each Taylor term
// the spectral product, the inverse y transform (in chunks of lines, keeping
// only y < nyv) and the inverse z transform (keeping z < nzv).  Planes are
// exchanged with the x passes in kx-major layout [view][kx][y][z].

constexpr int YZ_NT = 512;   // threads per CTA
constexpr int YZ_CH = 16;    // z lines per inverse-y chunk

// in-place Stockham pass over W lines of L points, point i of line w at
// base[w*ls + i*es]; every thread stages its butterflies in registers, so
// reads complete (barrier) before any write.  WFAST: consecutive threads
// take consecutive lines (use when ls == 1) instead of consecutive points.
template <int L, int R, int MAXW, bool WFAST, int Ns>
__device__ __forceinline__ void ip_pass(float2 *base, int W, int ls, int es, const float2 *tw, float s) {
  constexpr int JPL = L / R;
  constexpr int MAXJ = (MAXW * JPL + YZ_NT - 1) / YZ_NT;
  const int jobs = W * JPL;
  float2 v[MAXJ][R];
  int dst[MAXJ];
  constexpr int step = L / (Ns * R);
#pragma unroll
  for (int jj = 0; jj < MAXJ; ++jj) {
    const int q = threadIdx.x + jj * YZ_NT;
    dst[jj] = -1;
    if (q < jobs) {
      int w, j;
      if (WFAST) {
        w = q % W;
        j = q / W;
      } else {
        w = q / JPL;
        j = q - w * JPL;
      }
      const int k = j % Ns;
      const float2 *src = base + w * ls;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        float2 x = src[(j + r * JPL) * es];
        if (r > 0 && k > 0) {
          float2 t = tw[(r * k * step) & (L - 1)];
          t.y *= s;
          x = cmul(x, t);
        }
        v[jj][r] = x;
      }
      dst[jj] = w * ls + ((j / Ns) * Ns * R + k) * es;
    }
  }
  __syncthreads();
#pragma unroll
  for (int jj = 0; jj < MAXJ; ++jj) {
    if (dst[jj] >= 0) {
      dft_r<R>(v[jj], s);
#pragma unroll
      for (int r = 0; r < R; ++r) base[dst[jj] + r * Ns * es] = v[jj][r];
    }
  }
  __syncthreads();
}

// radix 8 while possible, 4 x 4 instead of 8 x 2 (fewer staged jobs);
// the pass sequence is unrolled at compile time
__host__ __device__ constexpr int ip_radix(int rem) { return (rem >= 8 && rem != 16) ? 8 : (rem == 4 || rem == 16) ? 4 : 2; }

template <int L, int MAXW, bool WFAST, int Ns>
struct IpPlan {
  static __device__ __forceinline__ void run(float2 *base, int W, int ls, int es, const float2 *tw, float s) {
    if constexpr (Ns < L) {
      constexpr int R = ip_radix(L / Ns);
      ip_pass<L, R, MAXW, WFAST, Ns>(base, W, ls, es, tw, s);
      IpPlan<L, MAXW, WFAST, Ns * R>::run(base, W, ls, es, tw, s);
    }
  }
};

// transforms W lines in chunks of at most MAXW lines (bounds the registers
// that stage one pass of a chunk)
template <int L, int MAXW, bool WFAST>
__device__ void fft_ip(float2 *base_all, int W, int ls, int es, const float2 *tw, float s) {
  for (int w0 = 0; w0 < W; w0 += MAXW) {
    float2 *base = base_all + (size_t)w0 * ls;
    const int Wc = min(MAXW, W - w0);
    IpPlan<L, MAXW, WFAST, 1>::run(base, Wc, ls, es, tw, s);
  }
}

struct YzArgs {
  const float2 *A;      // [B][kxh][nyv][nzv] after the forward x pass
  const float2 *K[2];   // kernel spectra, kx-major [kxh][L(y)][L(z)]
  float2 *D[2];         // [B][kxh][nyv][nzv] per term
  int kxh, nyv, nzv, nt;
};

template <int L>
__global__ void __launch_bounds__(YZ_NT, 1) k_esse_yz(YzArgs a, const float2 *__restrict__ twg) {
  extern __shared__ __align__(16) float2 yzs[];
  float2 *tw = yzs;                       // L
  float2 *F = tw + L;                     // [L(y)][L(z)]
  float2 *G = F + L * L;                  // [nyv][L(z)]
  float2 *S = G + (size_t)a.nyv * L;      // [L(y)][YZ_CH]
  const int kx = blockIdx.x, b = blockIdx.y, tid = threadIdx.x;
  const int nyv = a.nyv, nzv = a.nzv;
  for (int i = tid; i < L; i += YZ_NT) tw[i] = twg[i];
  const float2 *A = a.A + ((size_t)b * a.kxh + kx) * nyv * nzv;
  for (int e = tid; e < L * L; e += YZ_NT) {
    const int y = e / L, z = e - y * L;
    F[e] = (y < nyv && z < nzv) ? A[y * nzv + z] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  constexpr int MW = L >= 128 ? 32 : L;        // lines per staged chunk
  fft_ip<L, MW, false>(F, nyv, L, 1, tw, 1.f);  // z lines of the nonzero rows
  fft_ip<L, MW, true>(F, L, 1, L, tw, 1.f);     // y lines of every z
  for (int t = 0; t < a.nt; ++t) {
    const float2 *K = a.K[t] + (size_t)kx * L * L;
    for (int z0 = 0; z0 < L; z0 += YZ_CH) {
      for (int e = tid; e < L * YZ_CH; e += YZ_NT) {
        const int y = e / YZ_CH, zz = e - y * YZ_CH;
        S[e] = cmul(F[y * L + z0 + zz], __ldg(K + (size_t)y * L + z0 + zz));
      }
      __syncthreads();
      fft_ip<L, YZ_CH, true>(S, YZ_CH, 1, YZ_CH, tw, -1.f);  // inverse y
      for (int e = tid; e < nyv * YZ_CH; e += YZ_NT) {
        const int y = e / YZ_CH, zz = e - y * YZ_CH;
        G[y * L + z0 + zz] = S[e];
      }
      __syncthreads();
    }
    fft_ip<L, MW, false>(G, nyv, L, 1, tw, -1.f);  // inverse z of the kept rows
    float2 *D = a.D[t] + ((size_t)b * a.kxh + kx) * nyv * nzv;
    for (int e = tid; e < nyv * nzv; e += YZ_NT) {
      const int y = e / nzv, z = e - y * nzv;
      D[e] = G[y * L + z];
    }
    __syncthreads();
  }
}

// y-z plane with register transforms (esse_yz.cuh): one CTA per (kx, view),
// every transform in place in the plane; both terms from one forward
// spectrum.  Needs nyv <= L / 2 (the terms' cropped rows share the plane).
template <int L>
__global__ void __launch_bounds__(EY_NT, 1) k_esse_yz_reg(YzArgs a, const float2 *__restrict__ twg) {
  using D = EYz<L>;
  extern __shared__ __align__(16) float2 eys[];
  float2 *F = eys, *C = F + D::F_ELEMS, *tw = C + 2 * D::C_ELEMS;
  const int kx = blockIdx.x, b = blockIdx.y, tid = threadIdx.x;
  const int nyv = a.nyv, nzv = a.nzv, nt = a.nt;
  for (int i = tid; i < L; i += EY_NT) tw[i] = twg[i];
  const size_t plane = ((size_t)b * a.kxh + kx) * nyv * nzv;
  ey_load<L>(tid, F, a.A + plane, nyv, nzv);
  __syncthreads();
  ey_z_fwd_a<L>(tid, F, tw, nyv, nzv);
  __syncthreads();
  ey_z_fwd_b<L>(tid, F, nyv);
  __syncthreads();
  ey_y_fwd_a<L>(tid, F, tw, nyv);
  __syncthreads();
  const float2 *K0 = a.K[0] + (size_t)kx * L * L;
  const float2 *K1 = nt > 1 ? a.K[1] + (size_t)kx * L * L : K0;
  for (int z0 = 0; z0 < L; z0 += EY_ZC) {
    ey_y_mid<L>(tid, F, C, tw, K0, K1, nt, z0);
    __syncthreads();
    ey_y_inv_c<L>(tid, F, C, nt, nyv, z0);
    __syncthreads();
  }
  ey_z_inv_b<L>(tid, F, tw, nt * nyv);
  __syncthreads();
  ey_z_inv_c<L>(tid, F, nt * nyv, nzv);
  __syncthreads();
  ey_store<L>(tid, F, a.D[0] + plane, nt > 1 ? a.D[1] + plane : nullptr, nt, nyv, nzv);
}

// [ky][kz][kxh] -> [kxh][ky][p], p the position of kz after the forward z
// transform of k_esse_yz_reg (kz = (p mod N2) N1 + p / N2)
__global__ void k_spec_kpos(const float2 *__restrict__ in, float2 *__restrict__ out, int L, int kxh, int N1, int N2) {
  const size_t tot = (size_t)L * L * kxh;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    const int p = (int)(e % L);
    const size_t r = e / L;
    const int ky = (int)(r % L), kx = (int)(r / L);
    const int kz = (p % N2) * N1 + p / N2;
    out[e] = in[((size_t)ky * L + kz) * kxh + kx];
  }
}

static size_t yz_smem(int L, int nyv) { return sizeof(float2) * ((size_t)L + (size_t)L * L + (size_t)nyv * L + (size_t)L * YZ_CH); }

// [ky][kz][kxh] -> [kxh][ky][kz]
__global__ void k_spec_kmajor(const float2 *__restrict__ in, float2 *__restrict__ out, int ky, int kz, int kxh) {
  const size_t tot = (size_t)ky * kz * kxh;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    const int kx = (int)(e % kxh);
    const size_t r = e / kxh;  // y * kz + z
    out[(size_t)kx * ky * kz + r] = in[e];
  }
}

// ------------------------------------------------- expansion / smoothing

// The expansion replicates each coarse value over a c x c x c block, so a
// fine (z, x) line's inputs along y depend only on (z / c, x / c): after the
// y smoothing every c x c group of lines holds the same values, and after
// the z smoothing every group of c lines along x does.  The terms are
// therefore kept at coarse z and x after the y pass, and at coarse x after
// the z pass; the x pass expands x as it stages its rows.

// expansion along y with the y smoothing: thread per (term, b, zc, xc)
// coarse line; g = cropped coarse result [B][nyv][nzv][nxv]; output
// t[b][y][zc][xc] (y fine)
template <int C>
__global__ void __launch_bounds__(256) k_expand_y(const float *__restrict__ g0, const float *__restrict__ g1,
                                                   float *__restrict__ t0, float *__restrict__ t1, int nt, int n,
                                                   int nyv, int nzv, int nxv, int nb) {
  const size_t gs = (size_t)nzv * nxv, per = (size_t)nb * gs;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)nt * per) return;
  const int t = (int)(e / per);
  const int b = (int)((e - t * per) / gs);
  const size_t i = e - t * per - (size_t)b * gs;  // zc * nxv + xc
  {
    const float *g = (t == 0 ? g0 : g1) + (size_t)b * nyv * gs + i;
    float *o = (t == 0 ? t0 : t1) + (size_t)b * n * gs + i;
    coarse_walk<C, true, true>(g, gs, nyv, o, gs);
  }
}

// z expansion with the z smoothing: thread per (term, b, y, xc); input
// tc[b][y][zc][xc], output u[b][y][z][xc] with every entry written (entries
// z < h and z >= nz - h keep their input value, as the in-place pass leaves
// them)
template <int C>
__global__ void __launch_bounds__(256) k_smooth_z(const float *__restrict__ tc0, const float *__restrict__ tc1,
                                                   float *__restrict__ u0, float *__restrict__ u1, int nt, int n,
                                                   int nz, int nzv, int nxv, int nb) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t lines = (size_t)nb * n * nxv;
  if (e >= (size_t)nt * lines) return;
  const int t = (int)(e / lines);
  const size_t by = (e - t * lines) / nxv;  // b * n + y
  const int xc = (int)(e - t * lines - by * nxv);
  {
    const float *in = (t == 0 ? tc0 : tc1) + by * nzv * nxv + xc;
    float *o = (t == 0 ? u0 : u1) + by * nz * nxv + xc;
    coarse_walk<C, false, true>(in, nxv, nzv, o, nxv);
  }
}

// recursive smoothing along x (rows staged in shared memory) fused with the
// depth/density combination and the projector source.
struct CombineArgs {
  const float *t0, *t1;   // terms after the z pass [B][n][nz][n / c] (coarse x)
  const float *rot;       // rotated activity [B][n][nz][n]
  const float *S, *mu;    // per-view tables [view][n][nz][n]
  const int *views;
  float *src;             // output [B][n][nz][n]
  int n, nz, c, nt;
  float cnv;              // (float)(1.0/mu0)
  float fmu;              // mu0 - mu_avg
  float cntr;             // CntrPixFac
  float cnv_pix;          // cnv / pixsize
  float primary;
};

// one voxel of the combination (krnlprj3d.c:833-946) and the projector
// source (prjbck.c:170-173), rounded like libirl's float code
__device__ __forceinline__ float combine_one(const CombineArgs &a, float T0, float T1, float S, float act, float mu) {
  const float d = __fmul_rn(S, a.cnv);
  float eff = T0;
  if (a.nt > 1) eff = __fsub_rn(eff, __fmul_rn(d, T1));
  eff = (float)((double)eff * exp((double)__fmul_rn(d, a.fmu)));
  if (a.cntr > 0.f) eff = __fadd_rn(eff, __fmul_rn(act, a.cntr));
  eff = __fmul_rn(eff, __fmul_rn(mu, a.cnv_pix));
  if (eff < 0.f) eff = 0.f;
  return __fadd_rn(__fmul_rn(act, a.primary), eff);
}

// CTA of 32 x CX_TY threads per (b, y, block of XZB z rows).  The terms'
// rows arrive coarse in x (n / C values, each standing for C fine ones) and
// are staged as they are; one thread per (term, row) walks the fine x
// positions, reading its inputs from the coarse row (never overwritten, so
// every read sees an input as libirl's in-place walk does) and writing the
// smoothed fine row.  Rows have odd strides, so the row walks are free of
// bank conflicts.  C = 1 (no smoothing): the combination reads the staged
// rows.
constexpr int XZB = 32;
constexpr int CX_TY = 8;

static size_t smooth_x_smem(int n, int c) { return sizeof(float) * 2 * XZB * ((size_t)(n + 1) + (n / c + 1)); }

template <int C>
__global__ void __launch_bounds__(32 * CX_TY) k_smooth_x_combine(CombineArgs a) {
  constexpr int H = C / 2;
  extern __shared__ float smx[];  // fine rows [2][XZB][n + 1], coarse rows [2][XZB][n / C + 1]
  const int n = a.n, nz = a.nz, ld = n + 1, tn = n / C, lq = tn + 1;
  float *F = smx, *Q = smx + (size_t)2 * XZB * ld;
  const int y = blockIdx.x, z0 = blockIdx.y * XZB, b = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int rows = min(XZB, nz - z0);
  const size_t pln = (size_t)nz * n, vox = pln * n;
  const size_t base = (size_t)b * vox + (size_t)y * pln + (size_t)z0 * n;
  const size_t tbase = ((size_t)b * n + y) * nz * tn + (size_t)z0 * tn;
  const bool tvec = (tn & 3) == 0;  // coarse rows of whole float4s (16-byte aligned)
  const int tn4 = tn >> 2;
  for (int t = 0; t < a.nt; ++t) {
    const float *src = (t == 0 ? a.t0 : a.t1) + tbase;
    float *dst = Q + (size_t)t * XZB * lq;
    if (tvec) {
      for (int e = tid; e < rows * tn4; e += 32 * CX_TY) {
        const int rr = e / tn4, q4 = (e - rr * tn4) * 4;
        const float4 v = __ldg(reinterpret_cast<const float4 *>(src + (size_t)rr * tn + q4));
        float *d = dst + rr * lq + q4;
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
        d[3] = v.w;
      }
    } else {
      for (int rr = ty; rr < rows; rr += CX_TY)
        for (int xx = tx; xx < tn; xx += 32) dst[rr * lq + xx] = src[(size_t)rr * tn + xx];
    }
  }
  __syncthreads();
  const float *R = Q;  // rows the combination reads, stride lr
  int lr = lq;
  if (H > 0) {
    if (tid < a.nt * XZB && (tid % XZB) < rows) {
      const float *qrow = Q + (size_t)tid * lq;  // (term, row) = (tid / XZB, tid % XZB)
      float *frow = F + (size_t)tid * ld;
      coarse_walk<C, false, false>(qrow, 1, tn, frow, 1);
    }
    __syncthreads();
    R = F;
    lr = ld;
  }
  const int view = a.views[b];
  const size_t tb = (size_t)view * vox + (size_t)y * pln + (size_t)z0 * n;
  if ((n & 3) == 0) {
    const int n4 = n >> 2;
    for (int e = tid; e < rows * n4; e += 32 * CX_TY) {
      const int rr = e / n4, x = (e - rr * n4) * 4;
      const size_t g = (size_t)rr * n + x;
      const float4 S4 = __ldg(reinterpret_cast<const float4 *>(a.S + tb + g));
      const float4 A4 = __ldg(reinterpret_cast<const float4 *>(a.rot + base + g));
      const float4 M4 = __ldg(reinterpret_cast<const float4 *>(a.mu + tb + g));
      const float Sv[4] = {S4.x, S4.y, S4.z, S4.w}, Av[4] = {A4.x, A4.y, A4.z, A4.w};
      const float Mv[4] = {M4.x, M4.y, M4.z, M4.w};
      float out[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float T0 = R[rr * lr + x + q];
        const float T1 = a.nt > 1 ? R[(XZB + rr) * lr + x + q] : 0.f;
        out[q] = combine_one(a, T0, T1, Sv[q], Av[q], Mv[q]);
      }
      *reinterpret_cast<float4 *>(a.src + base + g) = make_float4(out[0], out[1], out[2], out[3]);
    }
    return;
  }
  for (int rr = ty; rr < rows; rr += CX_TY) {
    for (int xx = tx; xx < n; xx += 32) {
      const size_t e = (size_t)rr * n + xx;
      const float T0 = R[rr * lr + xx];
      const float T1 = a.nt > 1 ? R[(XZB + rr) * lr + xx] : 0.f;
      a.src[base + e] = combine_one(a, T0, T1, __ldg(a.S + tb + e), __ldg(a.rot + base + e), __ldg(a.mu + tb + e));
    }
  }
}

__global__ void k_scale_copy(const float *__restrict__ in, float *__restrict__ out, float s, size_t n) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) out[e] = __fmul_rn(in[e], s);
}

// -------------------------------------------------------------- host side




int upload_twiddle_table(cudaStream_t st, float2 **d, int L) {
  std::vector<float2> h(L);
  for (int m = 0; m < L; ++m) {
    const double a = -2.0 * M_PI * (double)m / (double)L;
    h[m] = make_float2((float)cos(a), (float)sin(a));
  }
  CU_TRY(dev_alloc_t(d, (size_t)L, st));
  CU_TRY(cudaMemcpyAsync(*d, h.data(), sizeof(float2) * L, cudaMemcpyHostToDevice, st));
  return IRLCU_OK;
}

static int upload_twiddles(float2 **d, int L) { return upload_twiddle_table(g_ctx->st, d, L); }

// ESSE grid sides with instantiated kernels: products of 2, 3, 5, 7 that
// ceil(2 N / c) takes for the usual volume sizes and collapse factors
#define ESSE_LENS(X) X(8) X(16) X(24) X(32) X(40) X(48) X(64) X(80) X(96) X(112) X(128) X(160) X(192) X(224) X(256) X(320) X(384) X(512) X(1024)

#define LDISPATCH(L, KERNEL, GRID, BLOCK, SMEM, ST, ...)                        \
  switch (L) {                                                                  \
    LCASES(KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__)                           \
    default: return set_error(IRLCU_EARG, "FFT length %d not supported", L);   \
  }
#define LCASE_1(L, KERNEL, GRID, BLOCK, SMEM, ST, ...) \
  case L: KERNEL<L><<<GRID, BLOCK, SMEM, ST>>>(__VA_ARGS__); break;
#define LCASES(KERNEL, GRID, BLOCK, SMEM, ST, ...) \
  LCASE_1(8, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(16, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(24, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(32, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(40, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(48, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(64, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(80, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(96, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(112, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(128, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(160, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(192, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(224, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(256, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(320, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(384, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(512, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__) \
  LCASE_1(1024, KERNEL, GRID, BLOCK, SMEM, ST, __VA_ARGS__)

static bool esse_len_ok(int L) {
  switch (L) {
#define LOK(L) case L:
    ESSE_LENS(LOK)
#undef LOK
    return true;
    default: return false;
  }
}

static int row_wr(int L) { return (L <= 128) ? 16 : (L <= 256 ? 4 : 2); }  // row_lines<L>()

static int col_smem(int L) { return (int)(sizeof(float2) * (L + 2 * CW * (L + 1))); }
// threads of a column-pass CTA: 512 for long lines (more warps to hide the
// shared-memory passes), 256 below
static int col_nt(int L) { return L >= 256 ? 512 : 256; }

static int set_col_attr(int L) {
  const int sm = col_smem(L);
  switch (L) {
#define LATTR(L)                                                                                  \
  case L:                                                                                         \
    CU_TRY(cudaFuncSetAttribute(k_fft_col<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm)); \
    break;
    ESSE_LENS(LATTR)
#undef LATTR
    default: return set_error(IRLCU_EARG, "FFT length %d not supported", L);
  }
  return IRLCU_OK;
}

// forward 3D transform of nb volumes.  Row pass from `rot` (collapse) or
// `grid`; valid input extents (nyv, nzv, nxv) of a (Ky, Kz, Kx) grid.
// Result: full spectrum [nb][Ky][Kz][kxh] in `out`; `tmpA`/`tmpB` scratch.
static int fft3_forward(cudaStream_t st, const EsseDev &E, const float *rot, const float *grid, int n, int nz,
                        int c, int nyv, int nzv, int nxv, int nb, float2 *tmpA, float2 *tmpB, float2 *out) {
  const int kxh = E.kxh;
  // x rows -> tmpA [nb][nyv][nzv][kxh]
  RowFwdArgs ra{};
  ra.rot = rot;
  ra.grid = grid;
  ra.n = n;
  ra.nz = nz;
  ra.c = c;
  ra.nyv = nyv;
  ra.nzv = nzv;
  ra.nxv = nxv;
  ra.vox = (size_t)n * nz * n;
  ra.out = tmpA;
  ra.zext = nzv;
  ra.kxh = kxh;
  {
    dim3 grid_((nyv * nzv + row_wr(E.kx) - 1) / row_wr(E.kx), nb);
    LDISPATCH(E.kx, k_fft_row_fwd, grid_, 256, 0, st, ra, g_ctx->ew.twx);
    CU_LAUNCHED();
  }
  // z lines (outer = y' < nyv) -> tmpB [nb][nyv][Kz][kxh]
  ColArgs za{};
  za.in = tmpA;
  za.in_bs = (size_t)nyv * nzv * kxh;
  za.in_os = (size_t)nzv * kxh;
  za.in_ps = kxh;
  za.in_valid = nzv;
  za.out[0] = tmpB;
  za.out_bs = (size_t)nyv * E.kz * kxh;
  za.out_os = (size_t)E.kz * kxh;
  za.out_ps = kxh;
  za.out_valid = E.kz;
  za.nt = 1;
  za.kxh = kxh;
  za.s = 1.f;
  {
    dim3 grid_((kxh + CW - 1) / CW, nyv, nb);
    LDISPATCH(E.kz, k_fft_col, grid_, col_nt(E.kz), col_smem(E.kz), st, za, g_ctx->ew.twz);
    CU_LAUNCHED();
  }
  // y lines (outer = z < Kz) -> out [nb][Ky][Kz][kxh]
  ColArgs ya{};
  ya.in = tmpB;
  ya.in_bs = (size_t)nyv * E.kz * kxh;
  ya.in_os = kxh;
  ya.in_ps = (size_t)E.kz * kxh;
  ya.in_valid = nyv;
  ya.out[0] = out;
  ya.out_bs = (size_t)E.ky * E.kz * kxh;
  ya.out_os = kxh;
  ya.out_ps = (size_t)E.kz * kxh;
  ya.out_valid = E.ky;
  ya.nt = 1;
  ya.kxh = kxh;
  ya.s = 1.f;
  {
    dim3 grid_((kxh + CW - 1) / CW, E.kz, nb);
    LDISPATCH(E.ky, k_fft_col, grid_, col_nt(E.ky), col_smem(E.ky), st, ya, g_ctx->ew.twy);
    CU_LAUNCHED();
  }
  return IRLCU_OK;
}

void esse_free(Ctx &c) {
  for (int t = 0; t < 3; ++t) {
    dev_free(c.esse.kft[t], c.st), c.esse.kft[t] = nullptr;
    dev_free(c.esse.kftT[t], c.st), c.esse.kftT[t] = nullptr;
  }
  c.esse.on = false;
  c.esse.zero = false;
  c.esse.fused = false;
  c.esse.yz_reg = false;
  EsseWork &w = c.ew;
  dev_free(w.twx, c.st);
  dev_free(w.twy, c.st);
  dev_free(w.twz, c.st);
  dev_free(w.A, c.st);
  dev_free(w.Bf, c.st);
  for (int t = 0; t < 2; ++t) {
    dev_free(w.C2[t], c.st);
    dev_free(w.D[t], c.st);
    dev_free(w.g[t], c.st);
    dev_free(w.T[t], c.st);
    dev_free(w.Tc[t], c.st);
  }
  c.ew = EsseWork{};
}

// pfReorder3dKrnl (krnlprj3d.c:43-128) read backwards: each grid point
// [z][y][x] of the oxd x oyd x ozd grid finds the file value that lands on
// it, if any.  Offsets below the half-widths xmin = min(noffs, oxd/2) map
// to themselves, their mirrors oxd - ix (ix > 0) back; depth plane z holds
// file depth ozd/2 + ndepths/2 - 1 - u, u the plane before the half-axis
// rotation.  Term 0 writes K (0 elsewhere), term 1 K (mu - mu_avg) (one
// float subtraction and one product; `outside` elsewhere).
__global__ void k_esse_expand(const float *__restrict__ kf, const float *__restrict__ mf, int noffs, int ndepths,
                              int oxd, int oyd, int ozd, int term, float mu_avg, float outside,
                              float *__restrict__ grid) {
  const size_t total = (size_t)oxd * oyd * ozd;
  const int xmin = min(noffs, oxd / 2), ymin = min(noffs, oyd / 2);
  for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(g % oxd);
    const size_t r = g / oxd;
    const int y = (int)(r % oyd), z = (int)(r / oyd);
    const int ix = x < xmin ? x : (x >= oxd - xmin + 1 ? oxd - x : -1);
    const int iy = y < ymin ? y : (y >= oyd - ymin + 1 ? oyd - y : -1);
    const int u = z < ozd / 2 ? z + ozd / 2 : z - ozd / 2;
    const int iz = ozd / 2 + ndepths / 2 - 1 - u;
    float v;
    if (ix >= 0 && iy >= 0 && iz >= 0 && iz < ndepths) {
      const size_t f = (size_t)ix + (size_t)noffs * (iy + (size_t)noffs * iz);
      v = term == 0 ? kf[f] : __fmul_rn(__fsub_rn(mf[f], mu_avg), kf[f]);
    } else {
      v = term == 0 ? 0.0f : outside;
    }
    grid[g] = v;
  }
}

// the file-form kernel of e on the device (two arrays of noffs^2 * ndepths)
static int esse_file_upload(Ctx &c, const irlcu_esse *e, float **dk, float **dm) {
  *dk = *dm = nullptr;
  if (e->noffs <= 0 || e->ndepths <= 0 || !e->krnl || !e->mu)
    return set_error(IRLCU_EARG, "ESSE kernel of %d x %d x %d offsets", e->noffs, e->noffs, e->ndepths);
  const size_t fc = (size_t)e->noffs * e->noffs * e->ndepths;
  CU_TRY(dev_alloc(reinterpret_cast<void **>(dk), sizeof(float) * fc, c.st));
  CU_TRY(dev_alloc(reinterpret_cast<void **>(dm), sizeof(float) * fc, c.st));
  CU_TRY(cudaMemcpyAsync(*dk, e->krnl, sizeof(float) * fc, cudaMemcpyHostToDevice, c.st));
  CU_TRY(cudaMemcpyAsync(*dm, e->mu, sizeof(float) * fc, cudaMemcpyHostToDevice, c.st));
  return IRLCU_OK;
}

// the grid of one term: pfReorder3dKrnl's (oxd, oyd, ozd) = (kx, kz, ky)
static int esse_expand(Ctx &c, const irlcu_esse *e, const float *dk, const float *dm, int term, float *grid) {
  k_esse_expand<<<148 * 8, 256, 0, c.st>>>(dk, dm, e->noffs, e->ndepths, e->kx, e->kz, e->ky, term, e->mu_avg,
                                           e->kmu_outside, grid);
  CU_LAUNCHED();
  return IRLCU_OK;
}

int esse_setup(Ctx &c, const irlcu_esse *e) {
  esse_free(c);
  if (!e) {  // scatter factor 0: the effective source is zero
    c.esse.zero = true;
    return IRLCU_OK;
  }
  EsseDev &E = c.esse;
  if (!esse_len_ok(e->kx) || !esse_len_ok(e->ky) || !esse_len_ok(e->kz) || e->ky > 512 || e->kz > 512)
    return set_error(IRLCU_EARG,
                     "ESSE FFT grid %d x %d x %d: sides must be one of 8..1024 with factors 2, 3, 5, 7 "
                     "(instantiated lengths) and at most 512 along y, z",
                     e->kx, e->ky, e->kz);
  if (e->nterms < 1 || e->nterms > 2)
    return set_error(IRLCU_EARG, "ESSE with %d Taylor terms is not supported (1 or 2)", e->nterms);
  E.kx = e->kx;
  E.ky = e->ky;
  E.kz = e->kz;
  E.kxh = e->kx / 2 + 1;
  E.collapse = e->collapse;
  E.nterms = e->nterms;
  E.mu0 = e->mu0;
  E.mu_avg = e->mu_avg;
  E.pix = e->pix;
  E.cntr = e->cntr_pix_fac;
  EsseWork &w = c.ew;
  // CollapseByFac (krnlprj3d.c:559-562) requires the factor to divide the
  // image dimensions
  if (E.collapse < 1 || c.n % E.collapse != 0 || c.nz % E.collapse != 0)
    return set_error(IRLCU_EARG, "ESSE collapse factor %d does not evenly divide the image dimensions %d, %d",
                     E.collapse, c.n, c.nz);
  w.nxv = c.n / E.collapse;
  w.nyv = c.n / E.collapse;
  w.nzv = c.nz / E.collapse;
  if (w.nxv > E.kx || w.nyv > E.ky || w.nzv > E.kz)
    return set_error(IRLCU_EARG, "Collapsed activity image can not be larger than kernel image");
  {
    int rc;
    if ((rc = upload_twiddles(&w.twx, E.kx))) return rc;
    if ((rc = upload_twiddles(&w.twy, E.ky))) return rc;
    if ((rc = upload_twiddles(&w.twz, E.kz))) return rc;
    if ((rc = set_col_attr(E.ky))) return rc;
    if ((rc = set_col_attr(E.kz))) return rc;
  }
  const int B = c.g.max_batch;
  w.batch = B;
  const size_t spec = (size_t)E.ky * E.kz * E.kxh;
  CU_TRY(dev_alloc(reinterpret_cast<void **>(&w.A), sizeof(float2) * (size_t)B * w.nyv * E.kz * E.kxh, c.st));
  CU_TRY(dev_alloc(reinterpret_cast<void **>(&w.Bf), sizeof(float2) * (size_t)B * spec, c.st));
  for (int t = 0; t < 2; ++t) {
    CU_TRY(dev_alloc(reinterpret_cast<void **>(&w.C2[t]), sizeof(float2) * (size_t)B * w.nyv * E.kz * E.kxh, c.st));
    CU_TRY(dev_alloc(reinterpret_cast<void **>(&w.D[t]), sizeof(float2) * (size_t)B * w.nyv * w.nzv * E.kxh, c.st));
    CU_TRY(dev_alloc(reinterpret_cast<void **>(&w.g[t]), sizeof(float) * (size_t)B * w.nyv * w.nzv * w.nxv, c.st));
    CU_TRY(dev_alloc(reinterpret_cast<void **>(&w.T[t]), sizeof(float) * (size_t)B * c.n * c.nz * w.nxv, c.st));
    CU_TRY(dev_alloc(reinterpret_cast<void **>(&w.Tc[t]), sizeof(float) * (size_t)B * c.n * w.nzv * w.nxv, c.st));
  }
  // kernel spectra: the grids expanded from the file form on the device,
  // then their forward transforms
  {
    float *dk = nullptr, *dm = nullptr, *dgrid = nullptr;
    float2 *ta = nullptr, *tb = nullptr;
    int rc = esse_file_upload(c, e, &dk, &dm);
    if (!rc && dev_alloc(reinterpret_cast<void **>(&dgrid), sizeof(float) * (size_t)E.kx * E.ky * E.kz, c.st))
      rc = set_error(IRLCU_ENOMEM, "ESSE grid");
    if (!rc && (dev_alloc(reinterpret_cast<void **>(&ta), sizeof(float2) * spec, c.st) ||
                dev_alloc(reinterpret_cast<void **>(&tb), sizeof(float2) * spec, c.st)))
      rc = set_error(IRLCU_ENOMEM, "ESSE transform work");
    for (int t = 0; !rc && t < E.nterms; ++t) {
      if (dev_alloc(reinterpret_cast<void **>(&E.kft[t]), sizeof(float2) * spec, c.st)) {
        rc = set_error(IRLCU_ENOMEM, "ESSE kernel spectrum");
        break;
      }
      rc = esse_expand(c, e, dk, dm, t, dgrid);
      if (!rc) rc = fft3_forward(c.st, E, nullptr, dgrid, c.n, c.nz, 1, E.ky, E.kz, E.kx, 1, ta, tb, E.kft[t]);
    }
    if (!rc && cudaStreamSynchronize(c.st) != cudaSuccess) rc = set_error(IRLCU_ECUDA, "ESSE kernel spectra");
    dev_free(ta, c.st);
    dev_free(tb, c.st);
    dev_free(dgrid, c.st);
    dev_free(dk, c.st);
    dev_free(dm, c.st);
    if (rc) return rc;
  }
  // fused y-z kernel when the plane fits in shared memory: the register
  // form when the cropped rows of both terms fit the plane (nyv <= L/2),
  // else the pass form (IRLCU_ESSE_YZ=pass forces the latter)
  {
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int L = E.ky;
    const char *yzenv = getenv("IRLCU_ESSE_YZ");
    size_t rsm = 0;
    switch (L) {
      case 32: rsm = EYz<32>::SMEM; break;
      case 64: rsm = EYz<64>::SMEM; break;
      case 128: rsm = EYz<128>::SMEM; break;
      default: break;
    }
    if (E.ky == E.kz && rsm && 2 * w.nyv <= L && rsm <= (size_t)maxsm && !(yzenv && !strcmp(yzenv, "pass"))) {
      const int N1 = L % 16 == 0 ? 16 : 8;
      for (int t = 0; t < E.nterms; ++t) {
        CU_TRY(dev_alloc(reinterpret_cast<void **>(&E.kftT[t]), sizeof(float2) * spec, c.st));
        k_spec_kpos<<<592, 256, 0, c.st>>>(E.kft[t], E.kftT[t], L, E.kxh, N1, L / N1);
        CU_LAUNCHED();
      }
      switch (L) {
        case 32: CU_TRY(cudaFuncSetAttribute(k_esse_yz_reg<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsm)); break;
        case 64: CU_TRY(cudaFuncSetAttribute(k_esse_yz_reg<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsm)); break;
        default: CU_TRY(cudaFuncSetAttribute(k_esse_yz_reg<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsm)); break;
      }
      CU_TRY(cudaStreamSynchronize(c.st));
      E.fused = true;
      E.yz_reg = true;
    }
    const size_t sm = yz_smem(L, w.nyv);
    if (!E.fused && E.ky == E.kz && (L == 32 || L == 64 || L == 128) && sm <= (size_t)maxsm) {
      for (int t = 0; t < E.nterms; ++t) {
        CU_TRY(dev_alloc(reinterpret_cast<void **>(&E.kftT[t]), sizeof(float2) * spec, c.st));
        k_spec_kmajor<<<592, 256, 0, c.st>>>(E.kft[t], E.kftT[t], E.ky, E.kz, E.kxh);
        CU_LAUNCHED();
      }
      switch (L) {
        case 32: CU_TRY(cudaFuncSetAttribute(k_esse_yz<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); break;
        case 64: CU_TRY(cudaFuncSetAttribute(k_esse_yz<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); break;
        default: CU_TRY(cudaFuncSetAttribute(k_esse_yz<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); break;
      }
      CU_TRY(cudaStreamSynchronize(c.st));
      E.fused = true;
    }
  }
  E.on = true;
  return IRLCU_OK;
}

static int esse_expand_combine(Ctx &c, const float *rot, const int *dviews, int nv, float primary, float *src);

bool esse_collapse_target(const Ctx &c, int nv, RotCollapse *col) {
  const EsseDev &E = c.esse;
  const EsseWork &w = c.ew;
  if (!E.on || !E.fused || !E.yz_reg || !er_len_ok(E.kx) || E.collapse != 2 || nv > w.batch || !w.g[0] ||
      (c.n & 1) || (c.nz & 1))
    return false;
  col->out = w.g[0];
  col->nyv = w.nyv;
  col->nzv = w.nzv;
  col->nxv = w.nxv;
  col->done = false;
  return true;
}

int launch_esse(Ctx &c, const float *rot, const int *dviews, int nv, float primary, float *src, bool collapsed) {
  EsseDev &E = c.esse;
  EsseWork &w = c.ew;
  if (!E.on) {
    // libirl returns a zero effective source when the kernel's scatter
    // factor is 0 (krnlprj3d.c:714-722): src = act * primary
    const size_t tot = (size_t)nv * c.vox;
    k_scale_copy<<<(unsigned)((tot + 255) / 256), 256, 0, c.st>>>(rot, src, primary, tot);
    CU_LAUNCHED();
    return IRLCU_OK;
  }
  if (nv > w.batch) return set_error(IRLCU_EARG, "ESSE batch %d exceeds %d", nv, w.batch);
  const int kxh = E.kxh, nyv = w.nyv, nzv = w.nzv, nxv = w.nxv;
  if (E.fused) {
    // x rows (collapse fused) -> A kx-major; y-z planes -> D[t]; x rows -> g[t]
    RowFwdArgs ra{};
    ra.rot = rot;
    ra.n = c.n;
    ra.nz = c.nz;
    ra.c = E.collapse;
    ra.nyv = nyv;
    ra.nzv = nzv;
    ra.nxv = nxv;
    ra.vox = c.vox;
    ra.out = w.A;
    ra.zext = nzv;
    ra.kxh = kxh;
    ra.kmajor = 1;
    // x transforms: register form unless IRLCU_ESSE_YZ=pass selects the
    // pass forms of all three transforms
    const bool reg_rows = er_len_ok(E.kx) && E.yz_reg;
    const int lines = (nyv * nzv + 1) / 2;
    if (reg_rows) {
      TRY_ESSE(er_attrs(E.kx));
      if (E.collapse > 1 && collapsed) {
        ra.pre = w.g[0];  // the two-slice rotation left the collapse there
      } else if (E.collapse > 1) {
        // the collapse as its own streaming pass into g[0] (free until the
        // x inverse writes it); in a shape-autotuner trial it counts with
        // the rotation it follows, which the two-slice form folds it into
        const size_t tot = (size_t)nv * nyv * nzv * nxv;
        const bool timed = c.trial_form >= 0 && !c.capturing;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (timed) {
          CU_TRY(cudaEventCreate(&e0));
          CU_TRY(cudaEventCreate(&e1));
          c.trial_ev[0].push_back({e0, e1});
          CU_TRY(cudaEventRecord(e0, c.st));
        }
        k_esse_collapse<<<(unsigned)((tot + 255) / 256), 256, 0, c.st>>>(rot, c.vox, c.n, c.nz, E.collapse, nyv, nzv,
                                                                         nxv, nv, w.g[0]);
        CU_LAUNCHED();
        if (timed) CU_TRY(cudaEventRecord(e1, c.st));
        ra.pre = w.g[0];
      }
      dim3 grid_((lines + ER_LW - 1) / ER_LW, nv);
      if (ra.pre) {
        ER_DISPATCH(E.kx, k_esse_row_fwd_reg<LL, true><<<grid_, ER_NT, ERow<LL>::SMEM, c.st>>>(ra, w.twx));
      } else {
        ER_DISPATCH(E.kx, k_esse_row_fwd_reg<LL, false><<<grid_, ER_NT, ERow<LL>::SMEM, c.st>>>(ra, w.twx));
      }
      CU_LAUNCHED();
    } else {
      dim3 grid_((nyv * nzv + row_wr(E.kx) - 1) / row_wr(E.kx), nv);
      LDISPATCH(E.kx, k_fft_row_fwd, grid_, 256, 0, c.st, ra, w.twx);
      CU_LAUNCHED();
    }
    YzArgs ya{};
    ya.A = w.A;
    ya.K[0] = E.kftT[0];
    ya.K[1] = E.nterms > 1 ? E.kftT[1] : nullptr;
    ya.D[0] = w.D[0];
    ya.D[1] = w.D[1];
    ya.kxh = kxh;
    ya.nyv = nyv;
    ya.nzv = nzv;
    ya.nt = E.nterms;
    if (E.yz_reg) {
      dim3 grid_(kxh, nv);
      switch (E.ky) {
        case 32: k_esse_yz_reg<32><<<grid_, EY_NT, EYz<32>::SMEM, c.st>>>(ya, w.twy); break;
        case 64: k_esse_yz_reg<64><<<grid_, EY_NT, EYz<64>::SMEM, c.st>>>(ya, w.twy); break;
        default: k_esse_yz_reg<128><<<grid_, EY_NT, EYz<128>::SMEM, c.st>>>(ya, w.twy); break;
      }
      CU_LAUNCHED();
    } else {
      dim3 grid_(kxh, nv);
      const size_t sm = yz_smem(E.ky, nyv);
      switch (E.ky) {
        case 32: k_esse_yz<32><<<grid_, YZ_NT, sm, c.st>>>(ya, w.twy); break;
        case 64: k_esse_yz<64><<<grid_, YZ_NT, sm, c.st>>>(ya, w.twy); break;
        default: k_esse_yz<128><<<grid_, YZ_NT, sm, c.st>>>(ya, w.twy); break;
      }
      CU_LAUNCHED();
    }
    RowInvArgs ri{};
    ri.in[0] = w.D[0];
    ri.in[1] = w.D[1];
    ri.out[0] = w.g[0];
    ri.out[1] = w.g[1];
    ri.nt = E.nterms;
    ri.nyv = nyv;
    ri.nzv = nzv;
    ri.nxv = nxv;
    ri.kxh = kxh;
    ri.scale = (float)(1.0 / ((double)E.kx * E.ky * E.kz));
    ri.kmajor = 1;
    if (reg_rows) {
      dim3 grid_((lines + ER_LW - 1) / ER_LW, nv, E.nterms);
      ER_DISPATCH(E.kx, k_esse_row_inv_reg<LL><<<grid_, ER_NT, ERow<LL>::SMEM, c.st>>>(ri, w.twx));
      CU_LAUNCHED();
    } else {
      dim3 grid_((nyv * nzv + row_wr(E.kx) - 1) / row_wr(E.kx), nv);
      LDISPATCH(E.kx, k_fft_row_inv, grid_, 256, 0, c.st, ri, w.twx);
      CU_LAUNCHED();
    }
    return esse_expand_combine(c, rot, dviews, nv, primary, src);
  }
  // forward: rot -> Bf (full spectrum)
  int rc = fft3_forward(c.st, E, rot, nullptr, c.n, c.nz, E.collapse, nyv, nzv, nxv, nv, w.A, w.C2[0], w.Bf);
  if (rc) return rc;
  // inverse y with the spectral products -> C2[t] [nv][nyv][Kz][kxh]
  ColArgs ya{};
  ya.in = w.Bf;
  ya.in_bs = (size_t)E.ky * E.kz * kxh;
  ya.in_os = kxh;
  ya.in_ps = (size_t)E.kz * kxh;
  ya.in_valid = E.ky;
  ya.mul[0] = E.kft[0];
  ya.mul[1] = E.nterms > 1 ? E.kft[1] : nullptr;
  ya.mul_os = kxh;
  ya.mul_ps = (size_t)E.kz * kxh;
  ya.out[0] = w.C2[0];
  ya.out[1] = w.C2[1];
  ya.out_bs = (size_t)nyv * E.kz * kxh;
  ya.out_os = kxh;
  ya.out_ps = (size_t)E.kz * kxh;
  ya.out_valid = nyv;
  ya.nt = E.nterms;
  ya.kxh = kxh;
  ya.s = -1.f;
  {
    dim3 grid_((kxh + CW - 1) / CW, E.kz, nv);
    LDISPATCH(E.ky, k_fft_col, grid_, col_nt(E.ky), col_smem(E.ky), c.st, ya, w.twy);
    CU_LAUNCHED();
  }
  // inverse z -> D[t] [nv][nyv][nzv][kxh]
  for (int t = 0; t < E.nterms; ++t) {
    ColArgs za{};
    za.in = w.C2[t];
    za.in_bs = (size_t)nyv * E.kz * kxh;
    za.in_os = (size_t)E.kz * kxh;
    za.in_ps = kxh;
    za.in_valid = E.kz;
    za.out[0] = w.D[t];
    za.out_bs = (size_t)nyv * nzv * kxh;
    za.out_os = (size_t)nzv * kxh;
    za.out_ps = kxh;
    za.out_valid = nzv;
    za.nt = 1;
    za.kxh = kxh;
    za.s = -1.f;
    dim3 grid_((kxh + CW - 1) / CW, nyv, nv);
    LDISPATCH(E.kz, k_fft_col, grid_, col_nt(E.kz), col_smem(E.kz), c.st, za, w.twz);
    CU_LAUNCHED();
  }
  // inverse x (real part, cropped, 1/(Kx Ky Kz)) -> g[t] [nv][nyv][nzv][nxv]
  RowInvArgs ri{};
  ri.in[0] = w.D[0];
  ri.in[1] = w.D[1];
  ri.out[0] = w.g[0];
  ri.out[1] = w.g[1];
  ri.nt = E.nterms;
  ri.nyv = nyv;
  ri.nzv = nzv;
  ri.nxv = nxv;
  ri.kxh = kxh;
  ri.scale = (float)(1.0 / ((double)E.kx * E.ky * E.kz));
  {
    dim3 grid_((nyv * nzv + row_wr(E.kx) - 1) / row_wr(E.kx), nv);
    LDISPATCH(E.kx, k_fft_row_inv, grid_, 256, 0, c.st, ri, w.twx);
    CU_LAUNCHED();
  }
  return esse_expand_combine(c, rot, dviews, nv, primary, src);
}

// expansion + smoothing (y, z), then x smoothing fused with the combine
static int esse_expand_combine(Ctx &c, const float *rot, const int *dviews, int nv, float primary, float *src) {
  EsseDev &E = c.esse;
  EsseWork &w = c.ew;
  const int nyv = w.nyv, nzv = w.nzv, nxv = w.nxv;
  const int cf = E.collapse;
  // c = 1: the cropped grid is the full-resolution term and needs no
  // smoothing; otherwise y expansion and smoothing (coarse z and x), then z
  // expansion and smoothing (coarse x)
  if (cf > 1) {
    const unsigned gy = (unsigned)(((size_t)E.nterms * nv * nzv * nxv + 255) / 256);
    const unsigned gz = (unsigned)(((size_t)E.nterms * nv * c.n * nxv + 255) / 256);
#define EXPAND_Z(C)                                                                                            \
  case C:                                                                                                      \
    k_expand_y<C><<<gy, 256, 0, c.st>>>(w.g[0], w.g[1], w.Tc[0], w.Tc[1], E.nterms, c.n, nyv, nzv, nxv, nv);    \
    CU_LAUNCHED();                                                                                             \
    k_smooth_z<C><<<gz, 256, 0, c.st>>>(w.Tc[0], w.Tc[1], w.T[0], w.T[1], E.nterms, c.n, c.nz, nzv, nxv, nv);   \
    CU_LAUNCHED();                                                                                             \
    break;
    switch (cf) {
      EXPAND_Z(2)
      EXPAND_Z(3)
      EXPAND_Z(4)
      EXPAND_Z(5)
      EXPAND_Z(6)
      EXPAND_Z(7)
      default:
        return set_error(IRLCU_EARG, "ESSE collapse factor %d not supported (1..7)", cf);
    }
#undef EXPAND_Z
  }
  CombineArgs ca{};
  ca.t0 = cf > 1 ? w.T[0] : w.g[0];
  ca.t1 = cf > 1 ? w.T[1] : w.g[1];
  ca.rot = rot;
  ca.S = c.tS;
  ca.mu = c.tMu;
  ca.views = dviews;
  ca.src = src;
  ca.n = c.n;
  ca.nz = c.nz;
  ca.c = cf;
  ca.nt = E.nterms;
  ca.cnv = (float)(1.0 / (double)E.mu0);
  ca.fmu = E.mu0 - E.mu_avg;
  ca.cntr = E.cntr;
  ca.cnv_pix = ca.cnv / E.pix;
  ca.primary = primary;
  {
    dim3 grid_(c.n, (c.nz + XZB - 1) / XZB, nv);
    const size_t sm = smooth_x_smem(c.n, cf);
    static size_t configured[8] = {};
    if (cf < 1 || cf > 7) return set_error(IRLCU_EARG, "ESSE collapse factor %d not supported (1..7)", cf);
    if (sm > 48 * 1024 && sm > configured[cf]) {
      switch (cf) {
#define SXC_ATTR(C) \
  case C: CU_TRY(cudaFuncSetAttribute(k_smooth_x_combine<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); break;
        SXC_ATTR(1) SXC_ATTR(2) SXC_ATTR(3) SXC_ATTR(4) SXC_ATTR(5) SXC_ATTR(6) SXC_ATTR(7)
#undef SXC_ATTR
      }
      configured[cf] = sm;
    }
    const dim3 blk(32, CX_TY);
    switch (cf) {
#define SXC_LAUNCH(C) \
  case C: k_smooth_x_combine<C><<<grid_, blk, sm, c.st>>>(ca); break;
      SXC_LAUNCH(1) SXC_LAUNCH(2) SXC_LAUNCH(3) SXC_LAUNCH(4) SXC_LAUNCH(5) SXC_LAUNCH(6) SXC_LAUNCH(7)
#undef SXC_LAUNCH
    }
    CU_LAUNCHED();
  }
  return IRLCU_OK;
}

}  // namespace irlcu

extern "C" int irlcu_set_esse(const irlcu_esse *e) {
  if (!irlcu::g_ctx) return irlcu::set_error(IRLCU_ESTATE, "irlcu_init has not been called");
  return irlcu::esse_setup(*irlcu::g_ctx, e);
}

extern "C" int irlcu_esse_expand(const irlcu_esse *e, int term, float *out) {
  using namespace irlcu;
  if (!g_ctx) return set_error(IRLCU_ESTATE, "irlcu_init has not been called");
  if (!e || !out || term < 0 || term > 1 || e->kx <= 0 || e->ky <= 0 || e->kz <= 0)
    return set_error(IRLCU_EARG, "irlcu_esse_expand: bad arguments");
  Ctx &c = *g_ctx;
  const size_t total = (size_t)e->kx * e->ky * e->kz;
  float *dk = nullptr, *dm = nullptr, *dgrid = nullptr;
  int rc = esse_file_upload(c, e, &dk, &dm);
  if (!rc && dev_alloc(reinterpret_cast<void **>(&dgrid), sizeof(float) * total, c.st))
    rc = set_error(IRLCU_ENOMEM, "ESSE grid");
  if (!rc) rc = esse_expand(c, e, dk, dm, term, dgrid);
  if (!rc && cudaMemcpyAsync(out, dgrid, sizeof(float) * total, cudaMemcpyDeviceToHost, c.st) != cudaSuccess)
    rc = set_error(IRLCU_ECUDA, "ESSE grid download");
  if (!rc && cudaStreamSynchronize(c.st) != cudaSuccess) rc = set_error(IRLCU_ECUDA, "ESSE grid download");
  dev_free(dgrid, c.st);
  dev_free(dk, c.st);
  dev_free(dm, c.st);
  return rc;
}
