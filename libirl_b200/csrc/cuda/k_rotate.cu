// k_rotate.cu -- volume rotation kernels of libirl_b200.
//
//  * three-shear rotation (libirl fastrotate.c:330-563, vShearsRotate):
//    one CTA rotates one z-slice of one view.  The slice is staged in shared
//    memory, pass 1 (x shear) writes the intermediate image X to shared
//    memory, and passes 2 (y shear) and 3 (x shear) are fused: each output
//    pixel reads the four X values it depends on.  Shifts and weights come
//    from host tables (irl_geom.c) and every product/sum is rounded exactly
//    like libirl's float C code (no FMA contraction), so the result is
//    bit-identical to vShearsRotate.
//  * bilinear rotation (rot3dpar.c:19-198): one thread per output (x, y)
//    column, looping over slices.
//  * the per-view clamped accumulation of unrotated backprojections and the
//    EM update / norm inversion epilogue (prjbck.c:418-426,
//    osemrecon.c:317-320, 850-852).
//
// Volume layout [y][z][x]; a slice k is the set of rows y*nz*n + k*n.
#include <cooperative_groups.h>
#include <cstdio>
#include <cstdlib>

#include "irlcu_internal.cuh"
#include "../host/irl_geom.h"

namespace cg = cooperative_groups;

namespace irlcu {

__device__ __forceinline__ float lerp2(float f1, float a, float f2, float b) {
  // f1*a + f2*b with the two products and the sum each rounded once
  return __fadd_rn(__fmul_rn(f1, a), __fmul_rn(f2, b));
}

struct RotHdr {
  int b90, b180, iadd, mdim;
};

// ---------------------------------------------------------------- pass 1
// X[r][i] of one slice (r = source row j, i < mdim); `S(y, x)` reads the
// source slice.
template <class Src>
__device__ __forceinline__ float shear_pass1(const Src &S, int n, const RotHdr &h, int j, int i,
                                             int sh, float f1, float f2, int st, int en) {
  const int iStart = st - sh, iEnd = en - sh - 1;
  if (i < iStart + h.iadd || i >= iEnd + h.iadd) return 0.f;
  if (h.b180 == 0) {
    const int t = sh - h.iadd;
    if (h.b90 == 0) return lerp2(f1, S(j, i + t), f2, S(j, i + t + 1));
    const int jj = n - j - 1;
    return lerp2(f1, S(i + t, jj), f2, S(i + t + 1, jj));
  } else {
    const int t = sh - h.iadd + 1;
    if (h.b90 == 0) {
      const int jj = n - j - 1;
      return lerp2(f1, S(jj, n - i - t), f2, S(jj, n - i - t - 1));
    }
    return lerp2(f1, S(n - i - t, j), f2, S(n - i - t - 1, j));
  }
}

// ------------------------------------------------------------ pass 2 + 3
// output pixel (j, x) from the intermediate image X (rows r in [0, n)
// correspond to rows r + iadd of libirl's mdim x mdim pfShiftedX).
template <class Xs>
__device__ __forceinline__ float shear_pass23(const Xs &X, int n, const RotHdr &h, int j, int x,
                                              int sh, float f1, float f2, int st, int en,
                                              const int *__restrict__ csh,
                                              const float *__restrict__ cf1,
                                              const float *__restrict__ cf2) {
  if (x < st + 1 || x >= en - 1) return 0.f;
  const int jj = j + h.iadd;
  const int a = x + sh + h.iadd;
  float y2[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int c = a + q;
    float v = 0.f;
    if (c >= 0 && c < h.mdim) {
      const int jt = csh[c];
      const int jS = max(0, -jt), jE = min(h.mdim, h.mdim - jt - 1);
      if (jj >= jS && jj < jE) {
        const int r0 = jj + jt - h.iadd;  // X row of ShiftedX[jj + jt]
        const float x0 = (r0 >= 0 && r0 < n) ? X(r0, c) : 0.f;
        const float x1 = (r0 + 1 >= 0 && r0 + 1 < n) ? X(r0 + 1, c) : 0.f;
        v = lerp2(cf1[c], x0, cf2[c], x1);
      }
    }
    y2[q] = v;
  }
  return lerp2(f1, y2[0], f2, y2[1]);
}

struct SmemSlice {
  const float *p;
  int n;
  __device__ float operator()(int y, int x) const { return p[y * n + x]; }
};
struct SmemX {
  const float *p;
  int ld;
  __device__ float operator()(int r, int c) const { return p[r * ld + c]; }
};
struct GlobSlice {  // rows y*nz*n + k*n of a volume; outside the slice: 0
  const float *__restrict__ p;
  int n;
  size_t rs;
  __device__ float operator()(int y, int x) const {
    return (y < 0 || y >= n || x < 0 || x >= n) ? 0.f : __ldg(p + (size_t)y * rs + x);
  }
};
struct GlobX {
  const float *__restrict__ p;
  int ld;
  __device__ float operator()(int r, int c) const { return __ldg(p + (size_t)r * ld + c); }
};

__device__ __forceinline__ RotHdr load_hdr(const RotTabs &T, int r) {
  RotHdr h;
  h.b90 = T.hdr[4 * r];
  h.b180 = T.hdr[4 * r + 1];
  h.iadd = T.hdr[4 * r + 2];
  h.mdim = T.hdr[4 * r + 3];
  return h;
}

// Path A: whole slice and X in shared memory, one CTA of 32 x 16 threads
// per (slice, view).  The slice is stored with an odd row stride (n + 1) so
// that the column walks of the 90-degree-flipped cases are free of bank
// conflicts; the rotation's tables are copied to shared memory once.
// grid (nz, nv).
constexpr int SH_TX = 32, SH_TY = 16;

// STAGE = false: pass 1 reads the source slice from global memory (L1 /
// L2) instead of staging it, which halves the shared memory per CTA
template <bool STAGE>
__global__ void __launch_bounds__(SH_TX *SH_TY) k_shear_smem(const float *__restrict__ src, size_t src_stride,
                                                             float *__restrict__ dst, size_t dst_stride,
                                                             const int *__restrict__ views, int rot_base,
                                                             RotTabs T, const int *__restrict__ sup_st,
                                                             const int *__restrict__ sup_en, int n, int nz,
                                                             int xld) {
  extern __shared__ float sm[];
  const int ld = n + 1;
  float *s_slice = sm;                                   // n * ld (STAGE)
  float *s_x = STAGE ? s_slice + (size_t)n * ld : sm;    // n * xld
  int *t_rsh = reinterpret_cast<int *>(s_x + (size_t)n * xld);
  int *t_st = t_rsh + n, *t_en = t_st + n;
  float *t_rf1 = reinterpret_cast<float *>(t_en + n), *t_rf2 = t_rf1 + n;
  int *t_csh = reinterpret_cast<int *>(t_rf2 + n);
  float *t_cf1 = reinterpret_cast<float *>(t_csh + xld), *t_cf2 = t_cf1 + xld;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * SH_TX + tx, nt = SH_TX * SH_TY;
  const int k = blockIdx.x, v = blockIdx.y;
  const int r = rot_base + views[v];
  const RotHdr h = load_hdr(T, r);
  const float *s = src + (size_t)v * src_stride + (size_t)k * n;
  float *d = dst + (size_t)v * dst_stride + (size_t)k * n;
  const size_t rs = (size_t)nz * n;
  for (int i = tid; i < n; i += nt) {
    t_rsh[i] = T.row_sh[(size_t)r * n + i];
    t_rf1[i] = T.row_f1[(size_t)r * n + i];
    t_rf2[i] = T.row_f2[(size_t)r * n + i];
    t_st[i] = sup_st[i];
    t_en[i] = sup_en[i];
  }
  for (int i = tid; i < h.mdim; i += nt) {
    t_csh[i] = T.col_sh[(size_t)r * 2 * n + i];
    t_cf1[i] = T.col_f1[(size_t)r * 2 * n + i];
    t_cf2[i] = T.col_f2[(size_t)r * 2 * n + i];
  }
  if (!STAGE) {
  } else if ((n & 3) == 0) {
    const int n4 = n >> 2;
#pragma unroll 4
    for (int y = ty; y < n; y += SH_TY)
      for (int q = tx; q < n4; q += SH_TX) {
        const float4 val = __ldg(reinterpret_cast<const float4 *>(s + (size_t)y * rs) + q);
        float *o = s_slice + y * ld + 4 * q;
        o[0] = val.x;
        o[1] = val.y;
        o[2] = val.z;
        o[3] = val.w;
      }
  } else {
    for (int y = ty; y < n; y += SH_TY)
      for (int x = tx; x < n; x += SH_TX) s_slice[y * ld + x] = __ldg(s + (size_t)y * rs + x);
  }
  __syncthreads();
  // source slice element (row y, column x)
  // taps outside the slice read as 0 (weight 0: see shear_tap)
  auto SL = [&](int yy, int xx) -> float {
    if (yy < 0 || yy >= n || xx < 0 || xx >= n) return 0.f;
    if (STAGE) return s_slice[yy * ld + xx];
    return __ldg(s + (size_t)yy * rs + xx);
  };
  // pass 1 (x shear): X row j from source row j (or column, when flipped)
  for (int j = ty; j < n; j += SH_TY) {
    const int sh = t_rsh[j], st = t_st[j], en = t_en[j];
    const float f1 = t_rf1[j], f2 = t_rf2[j];
    const int lo = st - sh + h.iadd, hi = en - sh - 1 + h.iadd;
    float *xr = s_x + (size_t)j * xld;
    for (int i = tx; i < h.mdim; i += SH_TX) {
      float val = 0.f;
      if (i >= lo && i < hi) {
        if (h.b180 == 0) {
          const int t = i + sh - h.iadd;
          if (h.b90 == 0)
            val = lerp2(f1, SL(j, t), f2, SL(j, t + 1));
          else
            val = lerp2(f1, SL(t, n - j - 1), f2, SL(t + 1, n - j - 1));
        } else {
          const int t = n - i - (sh - h.iadd + 1);
          if (h.b90 == 0)
            val = lerp2(f1, SL(n - j - 1, t), f2, SL(n - j - 1, t - 1));
          else
            val = lerp2(f1, SL(t, j), f2, SL(t - 1, j));
        }
      }
      xr[i] = val;
    }
  }
  __syncthreads();
  // passes 2 + 3 (y shear, then x shear) per output pixel
  for (int j = ty; j < n; j += SH_TY) {
    const int sh = t_rsh[j], st = t_st[j], en = t_en[j];
    const float f1 = t_rf1[j], f2 = t_rf2[j];
    const int jj = j + h.iadd;
    float *orow = d + (size_t)j * rs;
    for (int x = tx; x < n; x += SH_TX) {
      float out = 0.f;
      if (x >= st + 1 && x < en - 1) {
        const int a = x + sh + h.iadd;
        float y2[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int c = a + q;
          float yv = 0.f;
          if (c >= 0 && c < h.mdim) {
            const int jt = t_csh[c];
            if (jj >= max(0, -jt) && jj < min(h.mdim, h.mdim - jt - 1)) {
              const int r0 = jj + jt - h.iadd;
              const float x0 = (r0 >= 0 && r0 < n) ? s_x[(size_t)r0 * xld + c] : 0.f;
              const float x1 = (r0 + 1 >= 0 && r0 + 1 < n) ? s_x[(size_t)(r0 + 1) * xld + c] : 0.f;
              yv = lerp2(t_cf1[c], x0, t_cf2[c], x1);
            }
          }
          y2[q] = yv;
        }
        out = lerp2(f1, y2[0], f2, y2[1]);
      }
      orow[x] = out;
    }
  }
}

// Column-walk form: one CTA of 32 x 16 threads per (slice, view), only X in
// shared memory (two CTAs per SM).
//   pass 1: X[j][i] from the source slice through L1; the thread index runs
//           along the source row that the rotation reads contiguously (i
//           for the unflipped cases, j for the 90-degree-flipped ones);
//   pass 2: the y shear in place: each column c of X is shifted by its own
//           csh[c] with weights cf1[c], cf2[c], a warp per column stepping
//           32 rows at a time away from the rows it still has to read
//           (ascending for csh >= 0, descending otherwise), so every
//           intermediate value is computed once and every warp has work;
//   pass 3: the second x shear, two reads of the y-sheared row per output.
// Every product and sum is rounded as in the fused form above, so the
// output is the same bit for bit.
// Pass 1 reads source taps p(i) and p(i+1) of one source line (taps
// outside [0, n) read as 0: for odd n the middle row's last second tap is
// one past the line, with weight f2 = 0 exactly), where
//   b180 = 0: p(i) = i + sh - iadd,            line = row j (col n-j-1 if b90)
//   b180 = 1: p(i) = n - i - (sh - iadd + 1),  line = row n-j-1 (col j if b90)
// so the second tap of i is the first tap of i + 1.
//   unflipped (rows): a warp per row j, lanes along i; the second tap comes
//     from the next lane;
//   flipped (columns): a lane per j (consecutive columns of the source),
//     walking a quarter of the i range with the tap carried along.
__device__ __forceinline__ int shear_tap(const RotHdr &h, int n, int sh, int i) {
  return h.b180 ? n - i - (sh - h.iadd + 1) : i + sh - h.iadd;
}

// per row j of pass 1: tap(i) = c0 + dir i; taps are read for i in
// [la, lb] (the valid interval [lo, min(hi, mdim)] clipped to taps inside
// [0, n)); values for i in [lo, vb)
struct ShearRow {
  int dir, c0, lo, vb, la, lb;
  float f1, f2;
};

__device__ __forceinline__ ShearRow shear_row(const RotHdr &h, int n, int j, const int *t_rsh, const float *t_rf1,
                                              const float *t_rf2, const int *t_st, const int *t_en) {
  ShearRow r;
  const int sh = t_rsh[j];
  r.lo = t_st[j] - sh + h.iadd;
  const int hi = t_en[j] - sh - 1 + h.iadd;
  r.vb = min(hi, h.mdim);
  r.dir = h.b180 ? -1 : 1;
  r.c0 = h.b180 ? n - sh + h.iadd - 1 : sh - h.iadd;
  r.la = max(r.lo, h.b180 ? r.c0 - n + 1 : -r.c0);
  r.lb = min(r.vb, h.b180 ? r.c0 : n - 1 - r.c0);
  r.f1 = t_rf1[j];
  r.f2 = t_rf2[j];
  return r;
}

__device__ __forceinline__ void shear_pass1_rows(const float *__restrict__ s, int rs, float *s_x, int xld, int n,
                                                 const RotHdr &h, const int *t_rsh, const float *t_rf1,
                                                 const float *t_rf2, const int *t_st, const int *t_en, int warp,
                                                 int lane) {
  for (int j = warp; j < n; j += SH_TY) {
    const ShearRow r = shear_row(h, n, j, t_rsh, t_rf1, t_rf2, t_st, t_en);
    const float *line = s + (h.b180 ? n - j - 1 : j) * rs + r.c0;  // tap(i) at line[dir i]
    float *xr = s_x + j * xld;
    float v = (lane >= r.la && lane <= r.lb) ? __ldg(line + r.dir * lane) : 0.f;
    for (int i0 = 0; i0 < h.mdim; i0 += SH_TX) {
      const int i = i0 + lane, inx = i + SH_TX;
      const float vn = (inx >= r.la && inx <= r.lb) ? __ldg(line + r.dir * inx) : 0.f;
      // second tap of i = tap(i + 1): the next lane's, lane 0's next chunk for lane 31
      const float sec = __shfl_sync(0xffffffffu, lane == 0 ? vn : v, (lane + 1) & (SH_TX - 1));
      if (i < h.mdim) xr[i] = (i >= r.lo && i < r.vb) ? lerp2(r.f1, v, r.f2, sec) : 0.f;
      v = vn;
    }
  }
}

__device__ __forceinline__ void shear_pass1_cols(const float *__restrict__ s, int rs, float *s_x, int xld, int n,
                                                 const RotHdr &h, const int *t_rsh, const float *t_rf1,
                                                 const float *t_rf2, const int *t_st, const int *t_en, int tid) {
  constexpr int NCH = 4;  // i chunks per j
  const int nt = SH_TX * SH_TY;
  const int per = (h.mdim + NCH - 1) / NCH;
  for (int e = tid; e < n * NCH; e += nt) {
    const int ch = e / n, j = e - ch * n;
    const ShearRow r = shear_row(h, n, j, t_rsh, t_rf1, t_rf2, t_st, t_en);
    const int step = r.dir * rs;
    const float *col = s + (h.b180 ? j : n - j - 1) + r.c0 * rs;  // tap(i) at col[i step]
    float *xc = s_x + j * xld;
    const int i0 = ch * per, i1 = min(h.mdim, i0 + per);
    float v = (i0 >= r.la && i0 <= r.lb) ? __ldg(col + i0 * step) : 0.f;
    const float *pn = col + (i0 + 1) * step;
    for (int i = i0; i < i1; ++i, pn += step) {
      const float vn = (i + 1 >= r.la && i + 1 <= r.lb) ? __ldg(pn) : 0.f;
      xc[i] = (i >= r.lo && i < r.vb) ? lerp2(r.f1, v, r.f2, vn) : 0.f;
      v = vn;
    }
  }
}

__global__ void __launch_bounds__(SH_TX *SH_TY, 2) k_shear_cw(const float *__restrict__ src, size_t src_stride,
                                                             float *__restrict__ dst, size_t dst_stride,
                                                             const int *__restrict__ views, int rot_base,
                                                             RotTabs T, const int *__restrict__ sup_st,
                                                             const int *__restrict__ sup_en, int n, int nz,
                                                             int xld) {
  extern __shared__ float sm[];
  float *s_x = sm;  // n * xld
  int *t_rsh = reinterpret_cast<int *>(s_x + (size_t)n * xld);
  int *t_st = t_rsh + n, *t_en = t_st + n;
  float *t_rf1 = reinterpret_cast<float *>(t_en + n), *t_rf2 = t_rf1 + n;
  int *t_csh = reinterpret_cast<int *>(t_rf2 + n);
  float *t_cf1 = reinterpret_cast<float *>(t_csh + xld), *t_cf2 = t_cf1 + xld;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * SH_TX + tx, nt = SH_TX * SH_TY;
  const int k = blockIdx.x, v = blockIdx.y;
  const int r = rot_base + views[v];
  const RotHdr h = load_hdr(T, r);
  const float *s = src + (size_t)v * src_stride + (size_t)k * n;
  float *d = dst + (size_t)v * dst_stride + (size_t)k * n;
  const int rs = nz * n;
  for (int i = tid; i < n; i += nt) {
    t_rsh[i] = T.row_sh[(size_t)r * n + i];
    t_rf1[i] = T.row_f1[(size_t)r * n + i];
    t_rf2[i] = T.row_f2[(size_t)r * n + i];
    t_st[i] = sup_st[i];
    t_en[i] = sup_en[i];
  }
  for (int i = tid; i < h.mdim; i += nt) {
    t_csh[i] = T.col_sh[(size_t)r * 2 * n + i];
    t_cf1[i] = T.col_f1[(size_t)r * 2 * n + i];
    t_cf2[i] = T.col_f2[(size_t)r * 2 * n + i];
  }
  __syncthreads();
  if (h.b90)
    shear_pass1_cols(s, rs, s_x, xld, n, h, t_rsh, t_rf1, t_rf2, t_st, t_en, tid);
  else
    shear_pass1_rows(s, rs, s_x, xld, n, h, t_rsh, t_rf1, t_rf2, t_st, t_en, ty, tx);
  __syncthreads();
  // pass 2: Y[j][c] = lerp(X[j+jt][c], X[j+jt+1][c]) for jj = j + iadd in
  // [max(0, -jt), min(mdim, mdim - jt - 1)), else 0; X rows outside [0, n)
  // are 0.  A warp per column c, in place, 32 rows per step: all lanes
  // load before any stores, and the rows read lie on the far side of the
  // rows already written (at or past the step's first row for jt >= 0,
  // walking down; at or before its last row for jt < 0, walking up), so
  // every load sees X.
  for (int c = ty; c < h.mdim; c += SH_TY) {
    const int jt = t_csh[c];
    const float w1 = t_cf1[c], w2 = t_cf2[c];
    const int jlo = max(0, -jt) - h.iadd, jhi = min(h.mdim, h.mdim - jt - 1) - h.iadd;
    float *col = s_x + c;
    if (jt >= 0) {
      for (int j0 = 0; j0 < n; j0 += SH_TX) {
        const int j = j0 + tx, r0 = j + jt;
        const float x0 = (j < n && r0 < n) ? col[r0 * xld] : 0.f;
        const float x1 = (j < n && r0 + 1 < n) ? col[(r0 + 1) * xld] : 0.f;
        __syncwarp();
        if (j < n) col[j * xld] = (j >= jlo && j < jhi) ? lerp2(w1, x0, w2, x1) : 0.f;
      }
    } else {
      for (int j0 = n - 1; j0 >= 0; j0 -= SH_TX) {
        const int j = j0 - tx, r0 = j + jt;
        const float x0 = (j >= 0 && r0 >= 0) ? col[r0 * xld] : 0.f;
        const float x1 = (j >= 0 && r0 + 1 >= 0) ? col[(r0 + 1) * xld] : 0.f;
        __syncwarp();
        if (j >= 0) col[j * xld] = (j >= jlo && j < jhi) ? lerp2(w1, x0, w2, x1) : 0.f;
      }
    }
    __syncwarp();
  }
  __syncthreads();
  // pass 3: output (j, x) = lerp(Y[j][a], Y[j][a+1]), a = x + sh + iadd, for
  // x in [st + 1, en - 1); a warp per row, the second tap from the next lane
  for (int j = ty; j < n; j += SH_TY) {
    const int off = t_rsh[j] + h.iadd, xa = t_st[j] + 1, xb = t_en[j] - 1;
    const float f1 = t_rf1[j], f2 = t_rf2[j];
    const float *yr = s_x + j * xld;
    float *orow = d + (size_t)j * rs;
    int a = tx + off;
    float y = (a >= 0 && a < h.mdim) ? yr[a] : 0.f;
    for (int x0 = 0; x0 < n; x0 += SH_TX) {
      const int x = x0 + tx;
      a += SH_TX;
      const float yn = (a >= 0 && a < h.mdim) ? yr[a] : 0.f;
      const float sec = __shfl_sync(0xffffffffu, tx == 0 ? yn : y, (tx + 1) & (SH_TX - 1));
      if (x < n) orow[x] = (x >= xa && x < xb) ? lerp2(f1, y, f2, sec) : 0.f;
      y = yn;
    }
  }
}

// Two-slice form of the column-walk shear: one CTA of 32 x SH2_TY threads
// rotates the adjacent slices k0 = 2 blockIdx.x and k0 + 1 of one view.
// Both slices use the same rotation, so every shift, weight, bound and
// address is computed once for the pair: the intermediate image holds
// float2 pairs (slice k0, slice k0 + 1), each shared-memory access moves
// both values, and only the loads, shuffles, products and global stores are
// per slice.  The passes and every rounding are those of k_shear_cw, so the
// output is the same bit for bit.  For an odd slice count the last CTA has
// one slice; its second lane reads nothing and stores nothing.
//
// With COL (even n, even slice count) the CTA also writes ESSE's
// CollapseByFac by 2 of the pair (out[v][y/2][k0/2][x/2], nyv x nzv x n/2
// per view): the 2 x 2 x 2 sums of its output values, added in the order of
// the separate collapse (row y, then y + 1; slice k0, then k0 + 1; x, then
// x + 1), so ESSE reads the same bits without a pass over the rotated
// volumes.  Pass 3 then runs a warp per row pair.
constexpr int SH2_TY = 32;

template <bool COL>
__global__ void __launch_bounds__(SH_TX *SH2_TY, 1) k_shear_cw2(const float *__restrict__ src, size_t src_stride,
                                                               float *__restrict__ dst, size_t dst_stride,
                                                               const int *__restrict__ views, int rot_base,
                                                               RotTabs T, const int *__restrict__ sup_st,
                                                               const int *__restrict__ sup_en, int n, int nz,
                                                               int xld, float *__restrict__ col_out, int nyv,
                                                               int nzv) {
  extern __shared__ float sm[];
  float2 *s_x = reinterpret_cast<float2 *>(sm);  // n * xld pairs
  int *t_rsh = reinterpret_cast<int *>(s_x + (size_t)n * xld);
  int *t_st = t_rsh + n, *t_en = t_st + n;
  float *t_rf1 = reinterpret_cast<float *>(t_en + n), *t_rf2 = t_rf1 + n;
  int *t_csh = reinterpret_cast<int *>(t_rf2 + n);
  float *t_cf1 = reinterpret_cast<float *>(t_csh + xld), *t_cf2 = t_cf1 + xld;

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * SH_TX + tx, nt = SH_TX * SH2_TY;
  const int k0 = 2 * blockIdx.x, v = blockIdx.y;
  const bool two = k0 + 1 < nz;
  const int r = rot_base + views[v];
  const RotHdr h = load_hdr(T, r);
  const float *s = src + (size_t)v * src_stride + (size_t)k0 * n;  // slice k0 + 1 at s + n
  float *d = dst + (size_t)v * dst_stride + (size_t)k0 * n;
  const int rs = nz * n;
  // the pair's source rows (row y of both slices: 2n contiguous floats)
  // into L2 while the tables load, so that pass 1's walks find them there
  {
    const int lines = (2 * n * 4 + 127) / 128, rb = two ? 2 * n * 4 : n * 4;
    for (int e = tid; e < n * lines; e += nt) {
      const int y = e / lines, o = (e - y * lines) * 128;
      if (o < rb) asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char *>(s + (size_t)y * rs) + o));
    }
  }
  for (int i = tid; i < n; i += nt) {
    t_rsh[i] = T.row_sh[(size_t)r * n + i];
    t_rf1[i] = T.row_f1[(size_t)r * n + i];
    t_rf2[i] = T.row_f2[(size_t)r * n + i];
    t_st[i] = sup_st[i];
    t_en[i] = sup_en[i];
  }
  for (int i = tid; i < h.mdim; i += nt) {
    t_csh[i] = T.col_sh[(size_t)r * 2 * n + i];
    t_cf1[i] = T.col_f1[(size_t)r * 2 * n + i];
    t_cf2[i] = T.col_f2[(size_t)r * 2 * n + i];
  }
  __syncthreads();
  const float2 zero2 = make_float2(0.f, 0.f);
  if (!h.b90) {
    // pass 1, rows: a warp per row, the second tap from the next lane
    for (int j = ty; j < n; j += SH2_TY) {
      const ShearRow rw = shear_row(h, n, j, t_rsh, t_rf1, t_rf2, t_st, t_en);
      const float *line = s + (h.b180 ? n - j - 1 : j) * rs + rw.c0;  // tap(i) at line[dir i]
      float2 *xr = s_x + j * xld;
      const bool in0 = tx >= rw.la && tx <= rw.lb;
      float a0 = in0 ? __ldg(line + rw.dir * tx) : 0.f;
      float a1 = (in0 && two) ? __ldg(line + rw.dir * tx + n) : 0.f;
      for (int i0 = 0; i0 < h.mdim; i0 += SH_TX) {
        const int i = i0 + tx, inx = i + SH_TX;
        const bool in = inx >= rw.la && inx <= rw.lb;
        const float *pp = line + rw.dir * inx;
        const float b0 = in ? __ldg(pp) : 0.f, b1 = (in && two) ? __ldg(pp + n) : 0.f;
        const float c0 = __shfl_sync(0xffffffffu, tx == 0 ? b0 : a0, (tx + 1) & (SH_TX - 1));
        const float c1 = __shfl_sync(0xffffffffu, tx == 0 ? b1 : a1, (tx + 1) & (SH_TX - 1));
        if (i < h.mdim)
          xr[i] = (i >= rw.lo && i < rw.vb) ? make_float2(lerp2(rw.f1, a0, rw.f2, c0), lerp2(rw.f1, a1, rw.f2, c1))
                                            : zero2;
        a0 = b0;
        a1 = b1;
      }
    }
  } else {
    // pass 1, columns (90-degree flips): a thread per (chunk, j) walks i
    constexpr int NCH = 4;
    const int per = (h.mdim + NCH - 1) / NCH;
    for (int e = tid; e < n * NCH; e += nt) {
      const int ch = e / n, j = e - ch * n;
      const ShearRow rw = shear_row(h, n, j, t_rsh, t_rf1, t_rf2, t_st, t_en);
      const int step = rw.dir * rs;
      const float *col = s + (h.b180 ? j : n - j - 1) + rw.c0 * rs;  // tap(i) at col[i step]
      float2 *xc = s_x + j * xld;
      const int i0 = ch * per, i1 = min(h.mdim, i0 + per);
      const bool in0 = i0 >= rw.la && i0 <= rw.lb;
      float a0 = in0 ? __ldg(col + i0 * step) : 0.f;
      float a1 = (in0 && two) ? __ldg(col + i0 * step + n) : 0.f;
      const float *pn = col + (i0 + 1) * step;
      for (int i = i0; i < i1; ++i, pn += step) {
        const bool in = i + 1 >= rw.la && i + 1 <= rw.lb;
        const float b0 = in ? __ldg(pn) : 0.f, b1 = (in && two) ? __ldg(pn + n) : 0.f;
        xc[i] = (i >= rw.lo && i < rw.vb) ? make_float2(lerp2(rw.f1, a0, rw.f2, b0), lerp2(rw.f1, a1, rw.f2, b1))
                                          : zero2;
        a0 = b0;
        a1 = b1;
      }
    }
  }
  __syncthreads();
  // pass 2: the y shear in place, a warp per column (see k_shear_cw)
  for (int c = ty; c < h.mdim; c += SH2_TY) {
    const int jt = t_csh[c];
    const float w1 = t_cf1[c], w2 = t_cf2[c];
    const int jlo = max(0, -jt) - h.iadd, jhi = min(h.mdim, h.mdim - jt - 1) - h.iadd;
    float2 *col = s_x + c;
    if (jt >= 0) {
      for (int j0 = 0; j0 < n; j0 += SH_TX) {
        const int j = j0 + tx, r0 = j + jt;
        const float2 x0 = (j < n && r0 < n) ? col[r0 * xld] : zero2;
        const float2 x1 = (j < n && r0 + 1 < n) ? col[(r0 + 1) * xld] : zero2;
        __syncwarp();
        if (j < n)
          col[j * xld] = (j >= jlo && j < jhi) ? make_float2(lerp2(w1, x0.x, w2, x1.x), lerp2(w1, x0.y, w2, x1.y))
                                               : zero2;
      }
    } else {
      for (int j0 = n - 1; j0 >= 0; j0 -= SH_TX) {
        const int j = j0 - tx, r0 = j + jt;
        const float2 x0 = (j >= 0 && r0 >= 0) ? col[r0 * xld] : zero2;
        const float2 x1 = (j >= 0 && r0 + 1 >= 0) ? col[(r0 + 1) * xld] : zero2;
        __syncwarp();
        if (j >= 0)
          col[j * xld] = (j >= jlo && j < jhi) ? make_float2(lerp2(w1, x0.x, w2, x1.x), lerp2(w1, x0.y, w2, x1.y))
                                               : zero2;
      }
    }
    __syncwarp();
  }
  __syncthreads();
  // pass 3: the second x shear, a warp per row, the second tap from the next lane
  if (!COL) {
    for (int j = ty; j < n; j += SH2_TY) {
      const int off = t_rsh[j] + h.iadd, xa = t_st[j] + 1, xb = t_en[j] - 1;
      const float f1 = t_rf1[j], f2 = t_rf2[j];
      const float2 *yr = s_x + j * xld;
      float *orow = d + (size_t)j * rs;
      int a = tx + off;
      float2 y = (a >= 0 && a < h.mdim) ? yr[a] : zero2;
      for (int x0 = 0; x0 < n; x0 += SH_TX) {
        const int x = x0 + tx;
        a += SH_TX;
        const float2 yn = (a >= 0 && a < h.mdim) ? yr[a] : zero2;
        const float s0 = __shfl_sync(0xffffffffu, tx == 0 ? yn.x : y.x, (tx + 1) & (SH_TX - 1));
        const float s1 = __shfl_sync(0xffffffffu, tx == 0 ? yn.y : y.y, (tx + 1) & (SH_TX - 1));
        if (x < n) {
          const bool in = x >= xa && x < xb;
          orow[x] = in ? lerp2(f1, y.x, f2, s0) : 0.f;
          if (two) orow[x + n] = in ? lerp2(f1, y.y, f2, s1) : 0.f;
        }
        y = yn;
      }
    }
  } else {
    // a warp per row pair (2p, 2p + 1), both rows a chunk at a time, so the
    // collapse of each 2 x 2 x 2 block is added in registers
    for (int p = ty; p < (n >> 1); p += SH2_TY) {
      const int ja = 2 * p, jb = ja + 1;
      const int offa = t_rsh[ja] + h.iadd, xaa = t_st[ja] + 1, xba = t_en[ja] - 1;
      const int offb = t_rsh[jb] + h.iadd, xab = t_st[jb] + 1, xbb = t_en[jb] - 1;
      const float f1a = t_rf1[ja], f2a = t_rf2[ja], f1b = t_rf1[jb], f2b = t_rf2[jb];
      const float2 *yra = s_x + ja * xld, *yrb = s_x + jb * xld;
      float *oa = d + (size_t)ja * rs, *ob = d + (size_t)jb * rs;
      float *co = col_out + (((size_t)v * nyv + p) * nzv + (k0 >> 1)) * (n >> 1);
      int aa = tx + offa, ab = tx + offb;
      float2 ya = (aa >= 0 && aa < h.mdim) ? yra[aa] : zero2;
      float2 yb = (ab >= 0 && ab < h.mdim) ? yrb[ab] : zero2;
      for (int x0 = 0; x0 < n; x0 += SH_TX) {
        const int x = x0 + tx;
        aa += SH_TX;
        ab += SH_TX;
        const float2 yna = (aa >= 0 && aa < h.mdim) ? yra[aa] : zero2;
        const float2 ynb = (ab >= 0 && ab < h.mdim) ? yrb[ab] : zero2;
        const int src_lane = (tx + 1) & (SH_TX - 1);
        const float sa0 = __shfl_sync(0xffffffffu, tx == 0 ? yna.x : ya.x, src_lane);
        const float sa1 = __shfl_sync(0xffffffffu, tx == 0 ? yna.y : ya.y, src_lane);
        const float sb0 = __shfl_sync(0xffffffffu, tx == 0 ? ynb.x : yb.x, src_lane);
        const float sb1 = __shfl_sync(0xffffffffu, tx == 0 ? ynb.y : yb.y, src_lane);
        float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f;
        if (x < n) {
          const bool ina = x >= xaa && x < xba, inb = x >= xab && x < xbb;
          a0 = ina ? lerp2(f1a, ya.x, f2a, sa0) : 0.f;
          a1 = ina ? lerp2(f1a, ya.y, f2a, sa1) : 0.f;
          b0 = inb ? lerp2(f1b, yb.x, f2b, sb0) : 0.f;
          b1 = inb ? lerp2(f1b, yb.y, f2b, sb1) : 0.f;
          oa[x] = a0;
          oa[x + n] = a1;
          ob[x] = b0;
          ob[x + n] = b1;
        }
        // the next x of each value, from the next lane
        const float na0 = __shfl_down_sync(0xffffffffu, a0, 1), na1 = __shfl_down_sync(0xffffffffu, a1, 1);
        const float nb0 = __shfl_down_sync(0xffffffffu, b0, 1), nb1 = __shfl_down_sync(0xffffffffu, b1, 1);
        if (!(tx & 1) && x < n) {
          float t = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(0.f, a0), na0), a1), na1);
          t = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(t, b0), nb0), b1), nb1);
          co[x >> 1] = t;
        }
        ya = yna;
        yb = ynb;
      }
    }
  }
}

// Column-split form, for slices whose intermediate image does not fit
// shared memory (n = 256: 256 x 277 floats): one CTA per (slice, view).
// Pass 2 treats every column of X on its own, so the CTA runs passes 1 and
// 2 for one block of columns at a time in shared memory and stores each
// finished block of Y to a global work area (row-major, ldy per row); pass
// 3 then reads Y's rows from there (just written, from L2).  Every value is
// computed and rounded as in k_shear_cw, so the output is the same bit for
// bit.  SPLIT_CB columns per block (the last may be shorter).
constexpr int SPLIT_CB = 144;

__global__ void __launch_bounds__(SH_TX *SH_TY, 1) k_shear_split(const float *__restrict__ src, size_t src_stride,
                                                                float *__restrict__ dst, size_t dst_stride,
                                                                float *__restrict__ ywork, int ldy,
                                                                const int *__restrict__ views, int rot_base,
                                                                RotTabs T, const int *__restrict__ sup_st,
                                                                const int *__restrict__ sup_en, int n, int nz) {
  constexpr int XS = SPLIT_CB | 1;  // odd stride: conflict-free column walks
  extern __shared__ float sm[];
  float *s_x = sm;  // n * XS
  int *t_rsh = reinterpret_cast<int *>(s_x + (size_t)n * XS);
  int *t_st = t_rsh + n, *t_en = t_st + n;
  float *t_rf1 = reinterpret_cast<float *>(t_en + n), *t_rf2 = t_rf1 + n;
  int *t_csh = reinterpret_cast<int *>(t_rf2 + n);
  float *t_cf1 = reinterpret_cast<float *>(t_csh + 2 * n), *t_cf2 = t_cf1 + 2 * n;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * SH_TX + tx, nt = SH_TX * SH_TY;
  const int k = blockIdx.x, v = blockIdx.y;
  const int r = rot_base + views[v];
  const RotHdr h = load_hdr(T, r);
  const float *s = src + (size_t)v * src_stride + (size_t)k * n;
  float *d = dst + (size_t)v * dst_stride + (size_t)k * n;
  float *yw = ywork + ((size_t)v * nz + k) * (size_t)n * ldy;
  const int rs = nz * n;
  for (int i = tid; i < n; i += nt) {
    t_rsh[i] = T.row_sh[(size_t)r * n + i];
    t_rf1[i] = T.row_f1[(size_t)r * n + i];
    t_rf2[i] = T.row_f2[(size_t)r * n + i];
    t_st[i] = sup_st[i];
    t_en[i] = sup_en[i];
  }
  for (int i = tid; i < h.mdim; i += nt) {
    t_csh[i] = T.col_sh[(size_t)r * 2 * n + i];
    t_cf1[i] = T.col_f1[(size_t)r * 2 * n + i];
    t_cf2[i] = T.col_f2[(size_t)r * 2 * n + i];
  }
  __syncthreads();
  for (int c0 = 0; c0 < h.mdim; c0 += SPLIT_CB) {
    const int c1 = min(h.mdim, c0 + SPLIT_CB);
    // pass 1 for columns [c0, c1): X[j][i] at s_x[j XS + i - c0]
    if (!h.b90) {
      for (int j = ty; j < n; j += SH_TY) {
        const ShearRow rw = shear_row(h, n, j, t_rsh, t_rf1, t_rf2, t_st, t_en);
        const float *line = s + (h.b180 ? n - j - 1 : j) * rs + rw.c0;
        float *xr = s_x + j * XS;  // column i at xr[i - c0]
        const int i00 = c0 + tx;
        float a = (i00 >= rw.la && i00 <= rw.lb) ? __ldg(line + rw.dir * i00) : 0.f;
        for (int i0 = c0; i0 < c1; i0 += SH_TX) {
          const int i = i0 + tx, inx = i + SH_TX;
          const float b = (inx >= rw.la && inx <= rw.lb) ? __ldg(line + rw.dir * inx) : 0.f;
          const float sec = __shfl_sync(0xffffffffu, tx == 0 ? b : a, (tx + 1) & (SH_TX - 1));
          if (i < c1) xr[i - c0] = (i >= rw.lo && i < rw.vb) ? lerp2(rw.f1, a, rw.f2, sec) : 0.f;
          a = b;
        }
      }
    } else {
      constexpr int NCH = 4;
      const int per = (c1 - c0 + NCH - 1) / NCH;
      for (int e = tid; e < n * NCH; e += nt) {
        const int ch = e / n, j = e - ch * n;
        const int i0 = c0 + ch * per, i1 = min(c1, i0 + per);
        if (i0 >= i1) continue;
        const ShearRow rw = shear_row(h, n, j, t_rsh, t_rf1, t_rf2, t_st, t_en);
        const int step = rw.dir * rs;
        const float *col = s + (h.b180 ? j : n - j - 1) + rw.c0 * rs;
        float *xc = s_x + j * XS;  // column i at xc[i - c0]
        float a = (i0 >= rw.la && i0 <= rw.lb) ? __ldg(col + i0 * step) : 0.f;
        const float *pn = col + (i0 + 1) * step;
        for (int i = i0; i < i1; ++i, pn += step) {
          const float b = (i + 1 >= rw.la && i + 1 <= rw.lb) ? __ldg(pn) : 0.f;
          xc[i - c0] = (i >= rw.lo && i < rw.vb) ? lerp2(rw.f1, a, rw.f2, b) : 0.f;
          a = b;
        }
      }
    }
    __syncthreads();
    // pass 2 in place for the block's columns (see k_shear_cw), then Y to ywork
    for (int c = c0 + ty; c < c1; c += SH_TY) {
      const int jt = t_csh[c];
      const float w1 = t_cf1[c], w2 = t_cf2[c];
      const int jlo = max(0, -jt) - h.iadd, jhi = min(h.mdim, h.mdim - jt - 1) - h.iadd;
      float *col = s_x + (c - c0);
      if (jt >= 0) {
        for (int j0 = 0; j0 < n; j0 += SH_TX) {
          const int j = j0 + tx, r0 = j + jt;
          const float x0 = (j < n && r0 < n) ? col[r0 * XS] : 0.f;
          const float x1 = (j < n && r0 + 1 < n) ? col[(r0 + 1) * XS] : 0.f;
          __syncwarp();
          if (j < n) col[j * XS] = (j >= jlo && j < jhi) ? lerp2(w1, x0, w2, x1) : 0.f;
        }
      } else {
        for (int j0 = n - 1; j0 >= 0; j0 -= SH_TX) {
          const int j = j0 - tx, r0 = j + jt;
          const float x0 = (j >= 0 && r0 >= 0) ? col[r0 * XS] : 0.f;
          const float x1 = (j >= 0 && r0 + 1 >= 0) ? col[(r0 + 1) * XS] : 0.f;
          __syncwarp();
          if (j >= 0) col[j * XS] = (j >= jlo && j < jhi) ? lerp2(w1, x0, w2, x1) : 0.f;
        }
      }
      __syncwarp();
    }
    __syncthreads();
    for (int j = ty; j < n; j += SH_TY)
      for (int c = c0 + tx; c < c1; c += SH_TX) yw[(size_t)j * ldy + c] = s_x[j * XS + (c - c0)];
    __syncthreads();
  }
  // pass 3 from the Y rows in ywork (written above by this CTA)
  for (int j = ty; j < n; j += SH_TY) {
    const int off = t_rsh[j] + h.iadd, xa = t_st[j] + 1, xb = t_en[j] - 1;
    const float f1 = t_rf1[j], f2 = t_rf2[j];
    const float *yr = yw + (size_t)j * ldy;
    float *orow = d + (size_t)j * rs;
    int a = tx + off;
    float y = (a >= 0 && a < h.mdim) ? yr[a] : 0.f;
    for (int x0 = 0; x0 < n; x0 += SH_TX) {
      const int x = x0 + tx;
      a += SH_TX;
      const float yn = (a >= 0 && a < h.mdim) ? yr[a] : 0.f;
      const float sec = __shfl_sync(0xffffffffu, tx == 0 ? yn : y, (tx + 1) & (SH_TX - 1));
      if (x < n) orow[x] = (x >= xa && x < xb) ? lerp2(f1, y, f2, sec) : 0.f;
      y = yn;
    }
  }
}

// Cluster form, for slices whose intermediate image does not fit one SM's
// shared memory (n = 256: 256 x 277 floats): a cluster of two CTAs per
// (slice, view), CTA q holding X's columns [q cb, q cb + cb).  Passes 1 and
// 2 treat every column on its own, so each CTA runs them for its half;
// after a cluster barrier pass 3 reads Y's rows from both halves (the
// partner's through distributed shared memory), each CTA writing half of
// the output rows, and a second barrier keeps both halves alive until both
// CTAs are done.  Every value is computed and rounded as in k_shear_cw, so
// the output is the same bit for bit.
constexpr int CL_TY = 32;  // warps per CTA of the cluster form

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(SH_TX *CL_TY, 1)
    k_shear_cl2(const float *__restrict__ src, size_t src_stride, float *__restrict__ dst, size_t dst_stride,
                const int *__restrict__ views, int rot_base, RotTabs T, const int *__restrict__ sup_st,
                const int *__restrict__ sup_en, int n, int nz, int cb, int xs) {
  cg::cluster_group cl = cg::this_cluster();
  const int q = (int)cl.block_rank();
  extern __shared__ float sm[];
  float *s_x = sm;  // n * xs: column c0 + i at s_x[j xs + i]
  int *t_rsh = reinterpret_cast<int *>(s_x + (size_t)n * xs);
  int *t_st = t_rsh + n, *t_en = t_st + n;
  float *t_rf1 = reinterpret_cast<float *>(t_en + n), *t_rf2 = t_rf1 + n;
  int *t_csh = reinterpret_cast<int *>(t_rf2 + n);
  float *t_cf1 = reinterpret_cast<float *>(t_csh + 2 * n), *t_cf2 = t_cf1 + 2 * n;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * SH_TX + tx, nt = SH_TX * CL_TY;
  const int k = blockIdx.x >> 1, v = blockIdx.y;
  const int r = rot_base + views[v];
  const RotHdr h = load_hdr(T, r);
  const float *s = src + (size_t)v * src_stride + (size_t)k * n;
  float *d = dst + (size_t)v * dst_stride + (size_t)k * n;
  const int rs = nz * n;
  for (int i = tid; i < n; i += nt) {
    t_rsh[i] = T.row_sh[(size_t)r * n + i];
    t_rf1[i] = T.row_f1[(size_t)r * n + i];
    t_rf2[i] = T.row_f2[(size_t)r * n + i];
    t_st[i] = sup_st[i];
    t_en[i] = sup_en[i];
  }
  for (int i = tid; i < h.mdim; i += nt) {
    t_csh[i] = T.col_sh[(size_t)r * 2 * n + i];
    t_cf1[i] = T.col_f1[(size_t)r * 2 * n + i];
    t_cf2[i] = T.col_f2[(size_t)r * 2 * n + i];
  }
  __syncthreads();
  const int c0 = q * cb, c1 = min(h.mdim, c0 + cb);  // empty when X is narrower than one half
  // pass 1 for columns [c0, c1)
  if (!h.b90) {
    for (int j = ty; j < n; j += CL_TY) {
      const ShearRow rw = shear_row(h, n, j, t_rsh, t_rf1, t_rf2, t_st, t_en);
      const float *line = s + (h.b180 ? n - j - 1 : j) * rs + rw.c0;
      float *xr = s_x + j * xs;
      const int i00 = c0 + tx;
      float a = (i00 >= rw.la && i00 <= rw.lb) ? __ldg(line + rw.dir * i00) : 0.f;
      for (int i0 = c0; i0 < c1; i0 += SH_TX) {
        const int i = i0 + tx, inx = i + SH_TX;
        const float b = (inx >= rw.la && inx <= rw.lb) ? __ldg(line + rw.dir * inx) : 0.f;
        const float sec = __shfl_sync(0xffffffffu, tx == 0 ? b : a, (tx + 1) & (SH_TX - 1));
        if (i < c1) xr[i - c0] = (i >= rw.lo && i < rw.vb) ? lerp2(rw.f1, a, rw.f2, sec) : 0.f;
        a = b;
      }
    }
  } else {
    constexpr int NCH = 4;
    const int per = (c1 - c0 + NCH - 1) / NCH;
    for (int e = tid; e < n * NCH; e += nt) {
      const int ch = e / n, j = e - ch * n;
      const int i0 = c0 + ch * per, i1 = min(c1, i0 + per);
      if (i0 >= i1) continue;
      const ShearRow rw = shear_row(h, n, j, t_rsh, t_rf1, t_rf2, t_st, t_en);
      const int step = rw.dir * rs;
      const float *col = s + (h.b180 ? j : n - j - 1) + rw.c0 * rs;
      float *xc = s_x + j * xs;
      float a = (i0 >= rw.la && i0 <= rw.lb) ? __ldg(col + i0 * step) : 0.f;
      const float *pn = col + (i0 + 1) * step;
      for (int i = i0; i < i1; ++i, pn += step) {
        const float b = (i + 1 >= rw.la && i + 1 <= rw.lb) ? __ldg(pn) : 0.f;
        xc[i - c0] = (i >= rw.lo && i < rw.vb) ? lerp2(rw.f1, a, rw.f2, b) : 0.f;
        a = b;
      }
    }
  }
  __syncthreads();
  // pass 2 in place for the half's columns (see k_shear_cw)
  for (int c = c0 + ty; c < c1; c += CL_TY) {
    const int jt = t_csh[c];
    const float w1 = t_cf1[c], w2 = t_cf2[c];
    const int jlo = max(0, -jt) - h.iadd, jhi = min(h.mdim, h.mdim - jt - 1) - h.iadd;
    float *col = s_x + (c - c0);
    if (jt >= 0) {
      for (int j0 = 0; j0 < n; j0 += SH_TX) {
        const int j = j0 + tx, r0 = j + jt;
        const float x0 = (j < n && r0 < n) ? col[r0 * xs] : 0.f;
        const float x1 = (j < n && r0 + 1 < n) ? col[(r0 + 1) * xs] : 0.f;
        __syncwarp();
        if (j < n) col[j * xs] = (j >= jlo && j < jhi) ? lerp2(w1, x0, w2, x1) : 0.f;
      }
    } else {
      for (int j0 = n - 1; j0 >= 0; j0 -= SH_TX) {
        const int j = j0 - tx, r0 = j + jt;
        const float x0 = (j >= 0 && r0 >= 0) ? col[r0 * xs] : 0.f;
        const float x1 = (j >= 0 && r0 + 1 >= 0) ? col[(r0 + 1) * xs] : 0.f;
        __syncwarp();
        if (j >= 0) col[j * xs] = (j >= jlo && j < jhi) ? lerp2(w1, x0, w2, x1) : 0.f;
      }
    }
    __syncwarp();
  }
  // both halves of Y complete
  cl.sync();
  const float *half0 = cl.map_shared_rank(s_x, 0), *half1 = cl.map_shared_rank(s_x, 1);
  // pass 3 for rows [q n / 2, (q + 1) n / 2): Y[j][a] from the half that holds column a
  const int jb = q * n / 2, je = (q + 1) * n / 2;
  for (int j = jb + ty; j < je; j += CL_TY) {
    const int off = t_rsh[j] + h.iadd, xa = t_st[j] + 1, xb = t_en[j] - 1;
    const float f1 = t_rf1[j], f2 = t_rf2[j];
    const float *y0 = half0 + (size_t)j * xs, *y1 = half1 + (size_t)j * xs;
    float *orow = d + (size_t)j * rs;
    int a = tx + off;
    float y = (a >= 0 && a < h.mdim) ? (a < cb ? y0[a] : y1[a - cb]) : 0.f;
    for (int x0 = 0; x0 < n; x0 += SH_TX) {
      const int x = x0 + tx;
      a += SH_TX;
      const float yn = (a >= 0 && a < h.mdim) ? (a < cb ? y0[a] : y1[a - cb]) : 0.f;
      const float sec = __shfl_sync(0xffffffffu, tx == 0 ? yn : y, (tx + 1) & (SH_TX - 1));
      if (x < n) orow[x] = (x >= xa && x < xb) ? lerp2(f1, y, f2, sec) : 0.f;
      y = yn;
    }
  }
  // the partner may still read this CTA's half
  cl.sync();
}

static size_t shear_cl2_smem_bytes(int n, int xs) {
  return sizeof(float) * ((size_t)n * xs + 5 * (size_t)n + 3 * 2 * (size_t)n);
}

static size_t shear_split_smem_bytes(int n) {
  return sizeof(float) * ((size_t)n * (SPLIT_CB | 1) + 5 * (size_t)n + 3 * 2 * (size_t)n);
}

static size_t shear2_smem_bytes(int n, int xld) {
  return sizeof(float2) * (size_t)n * xld + sizeof(float) * (5 * (size_t)n + 3 * (size_t)xld);
}

static size_t shear_smem_bytes(int n, int xld, bool stage) {
  return sizeof(float) * ((stage ? (size_t)n * (n + 1) : 0) + (size_t)n * xld + 5 * (size_t)n + 3 * (size_t)xld);
}

// Path B, for slices too large for shared memory: pass 1 into a global
// scratch X[v][k][n][xld], then passes 2+3.  grid (nz, nv).
__global__ void __launch_bounds__(512) k_shear_pass1_glob(const float *__restrict__ src, size_t src_stride,
                                                          float *__restrict__ xs, const int *__restrict__ views,
                                                          int rot_base, RotTabs T,
                                                          const int *__restrict__ sup_st,
                                                          const int *__restrict__ sup_en, int n, int nz, int xld) {
  const int k = blockIdx.x, v = blockIdx.y;
  const int r = rot_base + views[v];
  const RotHdr h = load_hdr(T, r);
  GlobSlice S{src + (size_t)v * src_stride + (size_t)k * n, n, (size_t)nz * n};
  float *xo = xs + ((size_t)v * nz + k) * (size_t)n * xld;
  const int *rsh = T.row_sh + (size_t)r * n;
  const float *rf1 = T.row_f1 + (size_t)r * n, *rf2 = T.row_f2 + (size_t)r * n;
  for (int e = threadIdx.x; e < n * h.mdim; e += blockDim.x) {
    const int j = e / h.mdim, i = e - j * h.mdim;
    xo[(size_t)j * xld + i] = shear_pass1(S, n, h, j, i, rsh[j], rf1[j], rf2[j], sup_st[j], sup_en[j]);
  }
}

__global__ void __launch_bounds__(512) k_shear_pass23_glob(const float *__restrict__ xs, float *__restrict__ dst,
                                                           size_t dst_stride, const int *__restrict__ views,
                                                           int rot_base, RotTabs T,
                                                           const int *__restrict__ sup_st,
                                                           const int *__restrict__ sup_en, int n, int nz, int xld) {
  const int k = blockIdx.x, v = blockIdx.y;
  const int r = rot_base + views[v];
  const RotHdr h = load_hdr(T, r);
  GlobX X{xs + ((size_t)v * nz + k) * (size_t)n * xld, xld};
  float *d = dst + (size_t)v * dst_stride;
  const size_t rs = (size_t)nz * n;
  const int *rsh = T.row_sh + (size_t)r * n;
  const float *rf1 = T.row_f1 + (size_t)r * n, *rf2 = T.row_f2 + (size_t)r * n;
  const int *csh = T.col_sh + (size_t)r * 2 * n;
  const float *cf1 = T.col_f1 + (size_t)r * 2 * n, *cf2 = T.col_f2 + (size_t)r * 2 * n;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int j = e / n, x = e - j * n;
    d[(size_t)j * rs + (size_t)k * n + x] =
        shear_pass23(X, n, h, j, x, rsh[j], rf1[j], rf2[j], sup_st[j], sup_en[j], csh, cf1, cf2);
  }
}

// Bilinear rotation (rot3dpar.c:19-198, non-FAST branch).  One thread per
// output (x, y); NumPixels == NumRotPixs.  grid (ceil(n*n/256), nv).
__global__ void k_rot3dpar(const float *__restrict__ src, size_t src_stride, float *__restrict__ dst,
                           size_t dst_stride, const int *__restrict__ views, int rot_base, RotTabs T,
                           int n, int nz) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * n) return;
  const int v = blockIdx.y;
  const int r = rot_base + views[v];
  const float Sin = T.sn[r], Cos = T.cs[r];
  const int NewY = e / n, NewX = e - NewY * n;
  const int Dim = n;
  const float Axis = 0.5f * (float)(Dim - 1);  // 0.5*(NewDim-1): exact in float
  const float Radius = 0.5f * (float)Dim;
  const float *s = src + (size_t)v * src_stride;
  float *d = dst + (size_t)v * dst_stride;
  const size_t rs = (size_t)nz * n;
  // row extent (rot3dpar.c:98-101) with the C expression types:
  // (Radius - NewY) is float, "- .5" and the rest double
  const double t = __dsub_rn((double)__fsub_rn(Radius, (float)NewY), 0.5);
  int NumPix = (int)__dadd_rn(sqrt(__dsub_rn((double)__fmul_rn(Radius, Radius), __dmul_rn(t, t))), 0.5);
  NumPix *= 2;
  const int Head = (int)(0.5 * (double)(Dim - NumPix));
  const int Tail = Head + NumPix - 1;
  if (NewX < Head || NewX > Tail) {
    for (int z = 0; z < nz; ++z) d[(size_t)NewY * rs + (size_t)z * n + NewX] = 0.f;
    return;
  }
  // For odd sizes libirl's middle row gets NumPix = Dim + 1, so its loop
  // also evaluates NewX = Dim; that store lands on x = 0 of the next slice
  // of the same row (written earlier in the loop), and for the last slice
  // on x = 0 of the next row (rewritten later).  The thread of x = 0
  // reproduces the result: slices z >= 1 take the NewX = Dim value of z-1.
  const bool spill = (NewX == 0 && Tail >= Dim);
  const float Y = (float)NewY - Axis;
  for (int pass = 0; pass < (spill ? 2 : 1); ++pass) {
    const int NX = pass == 0 ? NewX : Dim;
    const float X = (float)NX - Axis;
    const float FloatX = __fadd_rn(__fsub_rn(__fmul_rn(X, Cos), __fmul_rn(Y, Sin)), Axis);
    const float FloatY = __fadd_rn(__fadd_rn(__fmul_rn(X, Sin), __fmul_rn(Y, Cos)), Axis);
    const int OldX = (int)FloatX, OldY = (int)FloatY;
    bool z0o = false, z1o = false, z2o = false, z3o = false;
    if (OldX < 0 || OldX >= Dim) z0o = z1o = true;
    if (OldY < 0 || OldY >= Dim) z0o = z2o = true;
    if (OldX + 1 < 0 || OldX + 1 >= Dim) z2o = z3o = true;
    if (OldY + 1 < 0 || OldY + 1 >= Dim) z1o = z3o = true;
    const float fy = __fsub_rn(FloatY, (float)OldY), fx = __fsub_rn(FloatX, (float)OldX);
    for (int z = 0; z < (pass == 0 ? nz : nz - 1); ++z) {
      const float z0 = z0o ? 0.f : __ldg(s + (size_t)OldY * rs + (size_t)z * n + OldX);
      const float z1 = z1o ? 0.f : __ldg(s + (size_t)(OldY + 1) * rs + (size_t)z * n + OldX);
      const float z2 = z2o ? 0.f : __ldg(s + (size_t)OldY * rs + (size_t)z * n + OldX + 1);
      const float z3 = z3o ? 0.f : __ldg(s + (size_t)(OldY + 1) * rs + (size_t)z * n + OldX + 1);
      float z01 = __fadd_rn(z0, __fmul_rn(fy, __fsub_rn(z1, z0)));
      float z23 = __fadd_rn(z2, __fmul_rn(fy, __fsub_rn(z3, z2)));
      if (FloatY < 0) {
        z01 = z0;
        z23 = z2;
      }
      float z0123 = __fadd_rn(z01, __fmul_rn(fx, __fsub_rn(z23, z01)));
      if (FloatX < 0) z0123 = z01;
      if (pass == 0)
        d[(size_t)NewY * rs + (size_t)z * n + NewX] = z0123;
      else
        d[(size_t)NewY * rs + (size_t)(z + 1) * n] = z0123;
    }
  }
}


static int launch_rotate_impl(const Ctx &c, const float *src, size_t src_stride, float *dst, size_t dst_stride,
                              const int *dviews, int nv, int rot_base, RotCollapse *col);

// During a shape-autotuner trial iteration every three-shear launch is
// bracketed by events, per source kind (irlcu_osem_iteration sums them).
int launch_rotate(const Ctx &c, const float *src, size_t src_stride, float *dst, size_t dst_stride,
                  const int *dviews, int nv, int rot_base, RotCollapse *col) {
  const bool timed = c.trial_form >= 0 && c.g.fast_rotate && !c.capturing && nv > 0;
  if (!timed) return launch_rotate_impl(c, src, src_stride, dst, dst_stride, dviews, nv, rot_base, col);
  const int kind = src_stride == 0 ? 0 : 1;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CU_TRY(cudaEventCreate(&e0));
  CU_TRY(cudaEventCreate(&e1));
  c.trial_ev[kind].push_back({e0, e1});
  CU_TRY(cudaEventRecord(e0, c.st));
  const int rc = launch_rotate_impl(c, src, src_stride, dst, dst_stride, dviews, nv, rot_base, col);
  CU_TRY(cudaEventRecord(e1, c.st));
  return rc;
}

static int launch_rotate_impl(const Ctx &c, const float *src, size_t src_stride, float *dst, size_t dst_stride,
                              const int *dviews, int nv, int rot_base, RotCollapse *col) {
  if (col) col->done = false;
  if (nv <= 0) return IRLCU_OK;
  const int n = c.n, nz = c.nz;
  if (!c.g.fast_rotate) {
    dim3 grid((n * n + 255) / 256, nv);
    k_rot3dpar<<<grid, 256, 0, c.st>>>(src, src_stride, dst, dst_stride, dviews, rot_base, c.rot, n, nz);
    CU_LAUNCHED();
    return IRLCU_OK;
  }
  // widest intermediate image over the rotations in use (mdim < 2n)
  const int xld = c.max_mdim > 0 ? c.max_mdim : 2 * n;
  int dev = 0, maxsm = 0, smsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&smsm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  // stage the slice only while two CTAs still fit an SM; otherwise pass 1
  // reads the slice through L1 and the CTA keeps only X
  // (IRLCU_SHEAR_STAGE = 1 / 0 forces either form)
  const size_t sm_stage = shear_smem_bytes(n, xld, true), sm_glob = shear_smem_bytes(n, xld, false);
  const char *env = getenv("IRLCU_SHEAR_STAGE");
  // column-walk form unless IRLCU_SHEAR_STAGE selects the fused one; its
  // X rows get an odd stride (bank-conflict-free column walks)
  const int xo = xld | 1;
  const size_t smc = shear_smem_bytes(n, xo, false);
  // two slices per CTA where their pair image fits, as the shape autotuner
  // decided for this kind of source (one volume shared by all views, or one
  // per view; Ctx::shear_form), else by default.  IRLCU_SHEAR_PAIR = 0 / 1
  // forces either form.
  const char *pair_env = getenv("IRLCU_SHEAR_PAIR");
  const size_t smc2 = shear2_smem_bytes(n, xo);
  const int kind = src_stride == 0 ? 0 : 1, tuned = c.trial_form >= 0 ? c.trial_form : c.shear_form[kind];
  const bool pair = pair_env ? pair_env[0] == '1' : (tuned >= 0 ? tuned == 1 : true);
  if (!env && pair && smc2 <= (size_t)maxsm) {
    // with the collapse where its buffers fit too (even n and slice count,
    // the collapsed sizes those of the rotated volume)
    const size_t smcc = smc2;
    const bool fuse = col && col->out && !(n & 1) && !(nz & 1) && col->nyv == n / 2 && col->nzv == nz / 2 &&
                      col->nxv == n / 2;
    if (fuse) {
      static size_t s_cw2c = 0;
      if (smcc > s_cw2c) {
        CU_TRY(cudaFuncSetAttribute(k_shear_cw2<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smcc));
        s_cw2c = smcc;
      }
      k_shear_cw2<true><<<dim3(nz / 2, nv), dim3(SH_TX, SH2_TY), smcc, c.st>>>(
          src, src_stride, dst, dst_stride, dviews, rot_base, c.rot, c.sup_start, c.sup_end, n, nz, xo, col->out,
          col->nyv, col->nzv);
      CU_LAUNCHED();
      col->done = true;
      return IRLCU_OK;
    }
    static size_t s_cw2 = 0;
    if (smc2 > s_cw2) {
      CU_TRY(cudaFuncSetAttribute(k_shear_cw2<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc2));
      s_cw2 = smc2;
    }
    k_shear_cw2<false><<<dim3((nz + 1) / 2, nv), dim3(SH_TX, SH2_TY), smc2, c.st>>>(
        src, src_stride, dst, dst_stride, dviews, rot_base, c.rot, c.sup_start, c.sup_end, n, nz, xo, nullptr, 0, 0);
    CU_LAUNCHED();
    return IRLCU_OK;
  }
  if (!env && smc <= (size_t)maxsm) {
    static size_t s_cw = 0;
    if (smc > s_cw) {
      CU_TRY(cudaFuncSetAttribute(k_shear_cw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc));
      s_cw = smc;
    }
    k_shear_cw<<<dim3(nz, nv), dim3(SH_TX, SH_TY), smc, c.st>>>(src, src_stride, dst, dst_stride, dviews, rot_base,
                                                                c.rot, c.sup_start, c.sup_end, n, nz, xo);
    CU_LAUNCHED();
    return IRLCU_OK;
  }
  bool stage = 2 * sm_stage + 2048 <= (size_t)smsm;
  if (env && env[0] == '1') stage = true;
  if (env && env[0] == '0') stage = false;
  if (stage && sm_stage > (size_t)maxsm) stage = false;
  const size_t smem = stage ? sm_stage : sm_glob;
  dim3 grid(nz, nv);
  if (smem <= (size_t)maxsm) {
    static size_t s_conf[2] = {0, 0};
    if (smem > s_conf[stage]) {
      if (stage)
        CU_TRY(cudaFuncSetAttribute(k_shear_smem<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      else
        CU_TRY(cudaFuncSetAttribute(k_shear_smem<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      s_conf[stage] = smem;
    }
    if (stage)
      k_shear_smem<true><<<grid, dim3(SH_TX, SH_TY), smem, c.st>>>(src, src_stride, dst, dst_stride, dviews,
                                                                  rot_base, c.rot, c.sup_start, c.sup_end, n, nz, xld);
    else
      k_shear_smem<false><<<grid, dim3(SH_TX, SH_TY), smem, c.st>>>(src, src_stride, dst, dst_stride, dviews,
                                                                   rot_base, c.rot, c.sup_start, c.sup_end, n, nz, xld);
    CU_LAUNCHED();
    return IRLCU_OK;
  }
  // cluster form where half of X fits one SM (IRLCU_SHEAR_CLUSTER=0 skips
  // it for the column-split form below)
  {
    const char *cl_env = getenv("IRLCU_SHEAR_CLUSTER");
    const int cb = (xld + 1) / 2, xs = cb | 1;
    const size_t smcl = shear_cl2_smem_bytes(n, xs);
    if (!env && !(cl_env && cl_env[0] == '0') && smcl <= (size_t)maxsm) {
      static size_t s_cl = 0;
      if (smcl > s_cl) {
        CU_TRY(cudaFuncSetAttribute(k_shear_cl2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smcl));
        s_cl = smcl;
      }
      k_shear_cl2<<<dim3(2 * nz, nv), dim3(SH_TX, CL_TY), smcl, c.st>>>(
          src, src_stride, dst, dst_stride, dviews, rot_base, c.rot, c.sup_start, c.sup_end, n, nz, cb, xs);
      CU_LAUNCHED();
      return IRLCU_OK;
    }
  }
  // column-split form where its block of columns fits (IRLCU_SHEAR_SPLIT=0
  // keeps the two global-memory kernels below)
  const char *split_env = getenv("IRLCU_SHEAR_SPLIT");
  const size_t sms = shear_split_smem_bytes(n);
  if (!env && !(split_env && split_env[0] == '0') && sms <= (size_t)maxsm) {
    const size_t needy = (size_t)nv * nz * n * xld;
    if (needy > c.xscratch_elems) {
      dev_free(c.xscratch, c.st);
      c.xscratch = nullptr;
      c.xscratch_elems = 0;
      CU_TRY(dev_alloc_t(&c.xscratch, needy, c.st));
      c.xscratch_elems = needy;
    }
    static size_t s_split = 0;
    if (sms > s_split) {
      CU_TRY(cudaFuncSetAttribute(k_shear_split, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sms));
      s_split = sms;
    }
    k_shear_split<<<dim3(nz, nv), dim3(SH_TX, SH_TY), sms, c.st>>>(src, src_stride, dst, dst_stride, c.xscratch,
                                                                   xld, dviews, rot_base, c.rot, c.sup_start,
                                                                   c.sup_end, n, nz);
    CU_LAUNCHED();
    return IRLCU_OK;
  }
  const size_t need = (size_t)nv * nz * n * xld;
  if (need > c.xscratch_elems) {
    dev_free(c.xscratch, c.st);
    c.xscratch = nullptr;
    c.xscratch_elems = 0;
    CU_TRY(dev_alloc_t(&c.xscratch, need, c.st));
    c.xscratch_elems = need;
  }
  k_shear_pass1_glob<<<grid, 512, 0, c.st>>>(src, src_stride, c.xscratch, dviews, rot_base, c.rot,
                                             c.sup_start, c.sup_end, n, nz, xld);
  CU_LAUNCHED();
  k_shear_pass23_glob<<<grid, 512, 0, c.st>>>(c.xscratch, dst, dst_stride, dviews, rot_base, c.rot,
                                              c.sup_start, c.sup_end, n, nz, xld);
  CU_LAUNCHED();
  return IRLCU_OK;
}

void free_rotate_scratch(Ctx &c) {
  dev_free(c.xscratch, c.st);
  c.xscratch = nullptr;
  c.xscratch_elems = 0;
}

// ---------------------------------------------------------- accumulation
// acc = clamp(acc + vol[v]) for v in order (prjbck.c:418-426), then the
// epilogue: ACC_EM est *= acc * norm (osemrecon.c:850-852) or ACC_INVERT
// acc = acc < 1e-6 ? 0 : 1/acc (osemrecon.c:317-320).
__global__ void k_accumulate(const float *__restrict__ vols, size_t vstride, int nv, float *__restrict__ acc,
                             int start_from_acc, int mode, float *__restrict__ est,
                             const float *__restrict__ norm, size_t vox) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < vox; i += (size_t)gridDim.x * blockDim.x) {
    float a = start_from_acc ? acc[i] : 0.f;
    for (int v = 0; v < nv; ++v) {
      a = __fadd_rn(a, __ldg(vols + (size_t)v * vstride + i));
      if ((double)a < 1.0e-5) a = 0.f;
    }
    if (mode == ACC_INVERT) {
      a = (double)a < 1e-6 ? 0.f : (float)(1.0 / (double)a);
    } else if (mode == ACC_EM) {
      est[i] = __fmul_rn(est[i], __fmul_rn(a, __ldg(norm + i)));
    }
    acc[i] = a;
  }
}

int launch_unrotate_accumulate(const Ctx &c, const float *bck, const int *dviews, int nv, float *acc,
                               int start_from_acc, int mode, float *est, const float *norm) {
  // unrotate every backprojected volume in place into wrot, then accumulate
  int rc = launch_rotate(c, bck, c.vox, c.wrot, c.vox, dviews, nv, c.nv);
  if (rc) return rc;
  int blocks = (int)((c.vox + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_accumulate<<<blocks, 256, 0, c.st>>>(c.wrot, c.vox, nv, acc, start_from_acc, mode, est, norm, c.vox);
  CU_LAUNCHED();
  return IRLCU_OK;
}

}  // namespace irlcu

// ----------------------------------------------- allocation-free rotation
// The three-shear rotation of irlcu_rotate_volume_noalloc runs the two
// global-memory kernels above with every buffer inside this file-scope
// array: rotation tables in the first IRLCU_NOALLOC_TAB_BYTES, then the
// pass-1 intermediate X[k][j][i] (i < mdim) of every slice.  The array is
// part of the module image, so the entry point calls no allocator.  Pass 2/3
// read only X entries that pass 1 of the same call wrote (c < mdim, rows
// < n), so nothing in it has to start at zero.
namespace irlcu {

static __device__ __align__(256) unsigned char g_noalloc_scratch[IRLCU_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int NA_MAXDEV = 64;
void *g_noalloc_addr[NA_MAXDEV];  // per device, looked up on first use

// host staging of the table region, laid out like the device copy (each
// table starts at a multiple of 64 words = 256 bytes)
constexpr int NA_SEG = 64;
constexpr int na_round(int w) { return (w + NA_SEG - 1) / NA_SEG * NA_SEG; }
struct NaLayout {
  int hdr, row_sh, row_f1, row_f2, col_sh, col_f1, col_f2, sn, cs, st, en, views, words;
};
NaLayout na_layout(int n) {
  NaLayout L{};
  int w = 0;
  L.hdr = w;    w += na_round(4);
  L.row_sh = w; w += na_round(n);
  L.row_f1 = w; w += na_round(n);
  L.row_f2 = w; w += na_round(n);
  L.col_sh = w; w += na_round(2 * n);
  L.col_f1 = w; w += na_round(2 * n);
  L.col_f2 = w; w += na_round(2 * n);
  L.sn = w;     w += na_round(1);
  L.cs = w;     w += na_round(1);
  L.st = w;     w += na_round(n);
  L.en = w;     w += na_round(n);
  L.views = w;  w += na_round(1);
  L.words = w;
  return L;
}
static_assert((4 * (NA_SEG * 8 + 13 * IRLCU_NOALLOC_MAX_N)) <= (int)IRLCU_NOALLOC_TAB_BYTES,
              "rotation tables of the largest n must fit the table region");
uint32_t g_na_host[IRLCU_NOALLOC_TAB_BYTES / 4];

}  // namespace

int launch_rotate_noalloc(cudaStream_t st, int dev, float angle, const float *src, float *dst, int n, int nz) {
  if (n < 1 || nz < 1 || n > IRLCU_NOALLOC_MAX_N)
    return set_error(IRLCU_EARG, "irlcu_rotate_volume_noalloc: n = %d, nz = %d outside 1 <= n <= %d, nz >= 1", n,
                     nz, IRLCU_NOALLOC_MAX_N);
  if (src == nullptr || dst == nullptr || src == dst)
    return set_error(IRLCU_EARG, "irlcu_rotate_volume_noalloc: src and dst must be distinct device pointers");
  // host tables straight into the staging words (no heap)
  const NaLayout L = na_layout(n);
  int32_t *wi = reinterpret_cast<int32_t *>(g_na_host);
  float *wf = reinterpret_cast<float *>(g_na_host);
  irl_shear_tab t{0, 0, 0, 0, wi + L.row_sh, wf + L.row_f1, wf + L.row_f2, wi + L.col_sh, wf + L.col_f1, wf + L.col_f2};
  irl_shear_table(angle, n, &t);
  const size_t need = (size_t)nz * n * (size_t)t.mdim;
  if (need > (size_t)IRLCU_NOALLOC_X_FLOATS)
    return set_error(IRLCU_EARG,
                     "irlcu_rotate_volume_noalloc: intermediate of nz*n*mdim = %d*%d*%d = %zu floats exceeds the "
                     "static scratch of %u floats",
                     nz, n, t.mdim, need, (unsigned)IRLCU_NOALLOC_X_FLOATS);
  wi[L.hdr + 0] = t.b90;
  wi[L.hdr + 1] = t.b180;
  wi[L.hdr + 2] = t.iadd;
  wi[L.hdr + 3] = t.mdim;
  wf[L.sn] = 0.f;
  wf[L.cs] = 0.f;
  irl_shear_support(n, wi + L.st, wi + L.en);
  wi[L.views] = 0;

  // dev is the library's device and the current one (checked by the caller),
  // so the symbol lookup below resolves on the device that runs `st`
  if (dev < 0 || dev >= NA_MAXDEV)
    return set_error(IRLCU_EARG, "irlcu_rotate_volume_noalloc: device %d beyond %d", dev, NA_MAXDEV);
  if (g_noalloc_addr[dev] == nullptr) {
    void *p = nullptr;
    CU_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = p;
  }
  unsigned char *base = static_cast<unsigned char *>(g_noalloc_addr[dev]);
  CU_TRY(cudaMemcpyAsync(base, g_na_host, (size_t)L.words * 4, cudaMemcpyHostToDevice, st));
  int32_t *di = reinterpret_cast<int32_t *>(base);
  float *df = reinterpret_cast<float *>(base);
  RotTabs T{di + L.hdr, di + L.row_sh, df + L.row_f1, df + L.row_f2, di + L.col_sh,
            df + L.col_f1, df + L.col_f2, df + L.sn, df + L.cs};
  float *xs = reinterpret_cast<float *>(base + IRLCU_NOALLOC_TAB_BYTES);
  const dim3 grid(nz, 1);
  k_shear_pass1_glob<<<grid, 512, 0, st>>>(src, 0, xs, di + L.views, 0, T, di + L.st, di + L.en, n, nz, t.mdim);
  CU_LAUNCHED();
  k_shear_pass23_glob<<<grid, 512, 0, st>>>(xs, dst, 0, di + L.views, 0, T, di + L.st, di + L.en, n, nz, t.mdim);
  CU_LAUNCHED();
  return IRLCU_OK;
}

}  // namespace irlcu
