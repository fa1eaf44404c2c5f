// esse_rows.cuh -- phases of the x transforms of the ESSE convolution with
// the two-level register transforms of reg_fft.cuh (kernels in k_esse.cu).
//
// Rows (y', z') of the collapsed volume, r = y' nzv + z', are transformed
// in pairs: rows 2w and 2w + 1 are the real and imaginary parts of one
// complex line w.  A CTA of ER_NT threads takes ER_LW lines per round.
//   forward:  step A (N2 threads per line) computes the collapsed values
//             x' < nxv (CollapseByFac fused into the load), the N1-point
//             DFTs and the twiddle; step B (N1 threads per line) the N2-point
//             DFTs, leaving Z[k1 + N1 k2] of each line in shared memory; the
//             unpack phase splits Z into the two rows' half spectra and
//             writes them kx-major, out[k][r] (rows 2w, 2w+1 as one 16-byte
//             store, consecutive lines in consecutive threads);
//   inverse:  step A reads the two rows' half spectra kx-major (consecutive
//             lines in consecutive threads), forms Z = A + iB over the full
//             length and runs the N1-point DFTs; step B the N2-point DFTs,
//             real part -> row 2w, imaginary part -> row 2w + 1, x < nxv,
//             times the scale.
// Every phase is a function of the thread index so that a host emulation
// of the CTA runs the same code.
#pragma once

#include "reg_fft.cuh"

namespace irlcu {

constexpr int ER_NT = 256;  // threads per CTA
constexpr int ER_LW = 32;   // lines (row pairs) per CTA round

template <int L>
struct ERow {
  static constexpr int N1 = LineSplit<L>::N1, N2 = LineSplit<L>::N2;
  static constexpr int XI = (ER_LW * N2) | 1;  // exchange buffer stride per k1 (odd)
  static constexpr int ZS = L + 1;             // line stride of the unpack buffer (odd)
  static constexpr int X_ELEMS = N1 * XI > ER_LW * ZS ? N1 * XI : ER_LW * ZS;
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)X_ELEMS + L);
  static constexpr int H = L / 2 + 1;
};

#ifdef __CUDA_ARCH__
__device__ __forceinline__ float2 er_ld2(const float2 *p) { return __ldg(p); }
__device__ __forceinline__ float er_ld(const float *p) { return __ldg(p); }
#else
inline float2 er_ld2(const float2 *p) { return *p; }
inline float er_ld(const float *p) { return *p; }
#endif

// CollapseByFac (krnlprj3d.c:549-593): sum over y, then z, then x offsets,
// in that order, of the rotated activity rot [n][nz][n]
__device__ __forceinline__ float er_collapse(const float *rot, int n, int nz, int c, int yy, int zz, int x) {
  if (c == 2 && (n & 1) == 0) {
    float t = 0.f;
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const float2 q = er_ld2(reinterpret_cast<const float2 *>(rot + ((size_t)(yy * 2 + k) * nz + (zz * 2 + j)) * n + x * 2));
        t = __fadd_rn(__fadd_rn(t, q.x), q.y);
      }
    return t;
  }
  float t = 0.f;
  for (int k = 0; k < c; ++k)
    for (int j = 0; j < c; ++j)
      for (int i = 0; i < c; ++i)
        t = __fadd_rn(t, er_ld(rot + ((size_t)(yy * c + k) * nz + (zz * c + j)) * n + x * c + i));
  return t;
}

// exchange index of (line wl, n2): forward n2 fastest, inverse line fastest
// (the order of the step A items, so that step A stores are consecutive)
template <int L, bool INV>
__device__ __forceinline__ int er_xi(int wl, int n2) {
  return INV ? n2 * ER_LW + wl : wl * ERow<L>::N2 + n2;
}

// forward step A, round of lines w0 .. w0 + ER_LW - 1 (item: n2 fastest);
// the collapsed values come from pre (rows [nrows][nxv], already collapsed
// by k_esse_collapse) when PRE, else from rot
template <int L, bool PRE = false>
__device__ __forceinline__ void er_fwd_a(int tid, int w0, float2 *X, const float2 *tw, const float *rot, int n,
                                         int nz, int c, int nzv, int nxv, int nrows, const float *pre = nullptr) {
  using D = ERow<L>;
  for (int it = tid; it < ER_LW * D::N2; it += ER_NT) {
    const int wl = it / D::N2, n2 = it - wl * D::N2;
    const int r0 = 2 * (w0 + wl);
    const bool h0 = r0 < nrows, h1 = r0 + 1 < nrows;
    const int y0 = r0 / nzv, z0 = r0 - y0 * nzv, y1 = (r0 + 1) / nzv, z1 = (r0 + 1) - y1 * nzv;
    float2 v[D::N1];
#pragma unroll
    for (int n1 = 0; n1 < D::N1; ++n1) {
      const int x = n2 + D::N2 * n1;
      float re = 0.f, im = 0.f;
      if (x < nxv) {
        if constexpr (PRE) {
          if (h0) re = er_ld(pre + (size_t)r0 * nxv + x);
          if (h1) im = er_ld(pre + (size_t)(r0 + 1) * nxv + x);
        } else {
          if (h0) re = er_collapse(rot, n, nz, c, y0, z0, x);
          if (h1) im = er_collapse(rot, n, nz, c, y1, z1, x);
        }
      }
      v[n1] = make_float2(re, im);
    }
    RDft<D::N1, false>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < D::N1; ++k1) v[k1] = twiddle<false>(v[k1], tw[n2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < D::N1; ++k1) X[k1 * D::XI + er_xi<L, false>(wl, n2)] = v[k1];
  }
}

// step B, both directions (item: k1 fastest): u[k2] = Z[k1 + N1 k2]; reads
// at the odd stride XI between consecutive threads
template <int L, bool INV>
__device__ __forceinline__ void er_b(int it, const float2 *X, float2 *u) {
  using D = ERow<L>;
  const int wl = it / D::N1, k1 = it - wl * D::N1;
#pragma unroll
  for (int n2 = 0; n2 < D::N2; ++n2) u[n2] = X[k1 * D::XI + er_xi<L, INV>(wl, n2)];
  RDft<D::N2, INV>::run(u);
}

// forward step B store: Z of line wl -> Zs[wl][k] (natural order)
template <int L>
__device__ __forceinline__ void er_fwd_b_store(int it, const float2 *u, float2 *Zs) {
  using D = ERow<L>;
  const int wl = it / D::N1, k1 = it - wl * D::N1;
#pragma unroll
  for (int k2 = 0; k2 < D::N2; ++k2) Zs[wl * D::ZS + k1 + D::N1 * k2] = u[k2];
}

// forward unpack (item: line fastest): A = (Z[k] + conj Z[L-k]) / 2 -> row
// 2w, B = (Z[k] - conj Z[L-k]) / 2i -> row 2w + 1, out[k][r] for k <= L/2
template <int L>
__device__ __forceinline__ void er_fwd_unpack(int tid, int w0, const float2 *Zs, float2 *out, int nrows) {
  using D = ERow<L>;
  for (int it = tid; it < ER_LW * D::H; it += ER_NT) {
    const int k = it / ER_LW, wl = it - k * ER_LW;
    const int r0 = 2 * (w0 + wl);
    if (r0 >= nrows) continue;
    const float2 zk = Zs[wl * D::ZS + k], zm = Zs[wl * D::ZS + (k == 0 ? 0 : L - k)];
    float2 *o = out + (size_t)k * nrows + r0;
    o[0] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    if (r0 + 1 < nrows) o[1] = make_float2(0.5f * (zk.y + zm.y), 0.5f * (zm.x - zk.x));
  }
}

// inverse step A (item: line fastest): Z = A + iB from the half spectra
// in[k][r] of rows 2w, 2w + 1, then the N1-point inverse DFTs
template <int L>
__device__ __forceinline__ void er_inv_a(int tid, int w0, float2 *X, const float2 *tw, const float2 *in, int nrows) {
  using D = ERow<L>;
  for (int it = tid; it < ER_LW * D::N2; it += ER_NT) {
    const int n2 = it / ER_LW, wl = it - n2 * ER_LW;
    const int r0 = 2 * (w0 + wl);
    const bool h0 = r0 < nrows, h1 = r0 + 1 < nrows;
    float2 v[D::N1];
#pragma unroll
    for (int n1 = 0; n1 < D::N1; ++n1) {
      const int k = n2 + D::N2 * n1;
      const bool lo = k <= L / 2;
      const int kk = lo ? k : L - k;
      const float2 *p = in + (size_t)kk * nrows + r0;
      const float2 A = h0 ? er_ld2(p) : make_float2(0.f, 0.f);
      const float2 B = h1 ? er_ld2(p + 1) : make_float2(0.f, 0.f);
      v[n1] = lo ? make_float2(A.x - B.y, A.y + B.x) : make_float2(A.x + B.y, B.x - A.y);
    }
    RDft<D::N1, true>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < D::N1; ++k1) v[k1] = twiddle<true>(v[k1], tw[n2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < D::N1; ++k1) X[k1 * D::XI + er_xi<L, true>(wl, n2)] = v[k1];
  }
}

// inverse step B store: real part -> row 2w, imaginary -> row 2w + 1,
// out[r][x] for x < nxv, times scale
template <int L>
__device__ __forceinline__ void er_inv_b_store(int it, int w0, const float2 *u, float *out, int nrows, int nxv,
                                               float scale) {
  using D = ERow<L>;
  const int wl = it / D::N1, k1 = it - wl * D::N1;
  const int r0 = 2 * (w0 + wl);
  if (r0 >= nrows) return;
  const bool two = r0 + 1 < nrows;
#pragma unroll
  for (int k2 = 0; k2 < D::N2; ++k2) {
    const int x = k1 + D::N1 * k2;
    if (x < nxv) {
      out[(size_t)r0 * nxv + x] = u[k2].x * scale;
      if (two) out[(size_t)(r0 + 1) * nxv + x] = u[k2].y * scale;
    }
  }
}

}  // namespace irlcu
