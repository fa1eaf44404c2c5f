// drf_plane.cuh -- phases of the one-CTA-per-plane form of the Fourier-domain
// DRF convolution (kernels in k_drf_fft.cu).
//
// One CTA of DP_NT threads holds a whole plane's half spectrum
// S[row][kx] (L rows, H = L/2 + 1 bins, row stride H) in shared memory and
// runs, with the two-level register transforms of reg_fft.cuh (L = N1 N2):
//   rows:     pairs of grid rows (g, g+1) as the real and imaginary parts
//             of one complex line; step A (N2 threads per line, N1-point
//             DFTs, twiddle) -> exchange buffer X -> step B (N1 threads per
//             line, N2-point DFTs) -> the two rows' half spectra, Z[k] and
//             Z[L-k] meeting through a warp shuffle;
//   columns:  in place in S.  Step A leaves Y[n2][k1] at row n2 + N2 k1;
//             step B holds X[k1 + N1 k2] in registers (the spectrum, in
//             natural frequency order k1 + N1 k2), where the backward pass
//             multiplies by the PSF spectrum and runs the first half of the
//             inverse, and the forward pass accumulates the product over
//             the planes of a group; step C finishes the inverse column
//             transform with the output rows in natural order;
//   rows:     the inverse of the row step (C2R of row pairs), cropped to
//             x < n and scaled, written to global memory.
// Every phase is a function of the thread index so that a host emulation
// of the CTA runs the same code.
#pragma once

#include "reg_fft.cuh"

namespace irlcu {

constexpr int DP_NT = 512;

template <int L>
struct DPlane {
  static constexpr int N1 = LineSplit<L>::N1, N2 = LineSplit<L>::N2;
  static constexpr int H = L / 2 + 1;             // half-spectrum bins (row stride of S)
  static constexpr int LINES = DP_NT / N1;        // row pairs per round
  static constexpr int XI = (LINES * N2) | 1;     // odd stride of the exchange buffer
  static constexpr int S_ELEMS = L * H;
  static constexpr int X_ELEMS = N1 * XI;
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)S_ELEMS + X_ELEMS + 2 * L);
  static constexpr int NRB = (N1 * H + DP_NT - 1) / DP_NT;  // column step-B items per thread
  static_assert(LINES * N2 <= DP_NT, "row step A needs one item per thread");
};

#ifdef __CUDA_ARCH__
__device__ __forceinline__ float2 dp_ld(const float2 *p) { return __ldg(p); }
#else
inline float2 dp_ld(const float2 *p) { return *p; }
#endif

__device__ __forceinline__ float plane_in(const float *a, const float *e, int i) {
  const float v = __ldg(a + i);
  return e ? __fmul_rn(v, __ldg(e + i)) : v;
}

// value of the attenuated, axially padded plane at (z, x), x < n
__device__ __forceinline__ float plane_pad_val(const float *a, const float *e, int z, int x, int n, int nz,
                                               int pady, int avgy) {
  if (z >= 0 && z < nz) return plane_in(a, e, z * n + x);
  if (pady <= 0 || avgy <= 0 || z < -pady || z >= nz + pady) return 0.f;
  // pfAvgRows (pad2d.c:92-122): row sum in order, divided when > 1 row
  const int r0 = z < 0 ? 0 : nz - avgy;
  float s = 0.f;
  for (int r = 0; r < avgy; ++r) s = __fadd_rn(s, plane_in(a, e, (r0 + r) * n + x));
  return avgy > 1 ? __fdiv_rn(s, (float)avgy) : s;
}

// one plane's source: grid row g holds plane row z = g - P
struct PlaneSrc {
  const float *a, *e;  // plane [z][x]; attenuation factors of the plane or null
  int n, nz, P, pady, avgy;
};

__device__ __forceinline__ float psrc_val(const PlaneSrc &p, int g, int x) {
  return plane_pad_val(p.a, p.e, g - p.P, x, p.n, p.nz, p.pady, p.avgy);
}

// tw[m] = W_L^m; twr[k1 * N2 + n2] = W_L^(n2 k1) (row step A: consecutive
// threads read consecutive entries)
template <int L>
__device__ __forceinline__ void dp_twiddles(int tid, float2 *tw, float2 *twr, const float2 *twg) {
  using D = DPlane<L>;
  for (int i = tid; i < L; i += DP_NT) {
    tw[i] = twg[i];
    const int k1 = i / D::N2, n2 = i - k1 * D::N2;
    twr[i] = twg[n2 * k1];
  }
}

// ---------------------------------------------------------------- rows

// L2 prefetch of the plane's source rows (and attenuation factors), one
// 128-byte line per thread and step, ahead of the row transforms
__device__ __forceinline__ void dp_prefetch_plane(int tid, const PlaneSrc &p) {
#ifdef __CUDA_ARCH__
  const int bytes = p.nz * p.n * 4;
  const char *a = reinterpret_cast<const char *>(p.a), *e = reinterpret_cast<const char *>(p.e);
  for (int o = tid * 128; o < bytes; o += DP_NT * 128) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(a + o));
    if (e) asm volatile("prefetch.global.L2 [%0];" ::"l"(e + o));
  }
#endif
}

// forward step A of round w0: line w = w0 + tid / N2 holds grid rows 2w
// (real) and 2w + 1 (imaginary); x[n2 + N2 n1] -> Y[n2][k1] W^(n2 k1)
template <int L>
__device__ __forceinline__ void dp_rows_fwd_a(int tid, int w0, const PlaneSrc &p, int G, float2 *X,
                                              const float2 *twr) {
  using D = DPlane<L>;
  if (tid >= D::LINES * D::N2) return;
  const int wl = tid / D::N2, n2 = tid - wl * D::N2, g = 2 * (w0 + wl);
  const int n = p.n, z0 = g - p.P;
  float2 v[D::N1];
  if (g + 1 < G && z0 >= 0 && z0 + 1 < p.nz) {
    // both rows inside the plane: no padding logic per element
    const float *a0 = p.a + z0 * n + n2;
    if (p.e) {
      const float *e0 = p.e + z0 * n + n2;
#pragma unroll
      for (int n1 = 0; n1 < D::N1; ++n1) {
        const int o = D::N2 * n1;
        v[n1] = n2 + o < n ? make_float2(__fmul_rn(__ldg(a0 + o), __ldg(e0 + o)),
                                         __fmul_rn(__ldg(a0 + n + o), __ldg(e0 + n + o)))
                           : make_float2(0.f, 0.f);
      }
    } else {
#pragma unroll
      for (int n1 = 0; n1 < D::N1; ++n1) {
        const int o = D::N2 * n1;
        v[n1] = n2 + o < n ? make_float2(__ldg(a0 + o), __ldg(a0 + n + o)) : make_float2(0.f, 0.f);
      }
    }
  } else {
#pragma unroll
    for (int n1 = 0; n1 < D::N1; ++n1) {
      const int x = n2 + D::N2 * n1;
      float re = 0.f, im = 0.f;
      if (x < n && g < G) {
        re = psrc_val(p, g, x);
        if (g + 1 < G) im = psrc_val(p, g + 1, x);
      }
      v[n1] = make_float2(re, im);
    }
  }
  RDft<D::N1, false>::run(v);
#pragma unroll
  for (int k1 = 1; k1 < D::N1; ++k1) v[k1] = twiddle<false>(v[k1], twr[k1 * D::N2 + n2]);
#pragma unroll
  for (int k1 = 0; k1 < D::N1; ++k1) X[k1 * D::XI + tid] = v[k1];
}

// step B (both directions): u[k2] = Z[k1 + N1 k2] of line tid / N1
template <int L, bool INV>
__device__ __forceinline__ void dp_rows_b(int tid, const float2 *X, float2 *u) {
  using D = DPlane<L>;
  const int wl = tid / D::N1, k1 = tid - wl * D::N1;
#pragma unroll
  for (int n2 = 0; n2 < D::N2; ++n2) u[n2] = X[k1 * D::XI + wl * D::N2 + n2];
  RDft<D::N2, INV>::run(u);
}

// the thread of the same line holding Z[L - k] for this thread's Z[k]
template <int L>
__device__ __forceinline__ int dp_partner(int tid) {
  constexpr int N1 = DPlane<L>::N1;
  return (tid & ~(N1 - 1)) | ((N1 - (tid & (N1 - 1))) & (N1 - 1));
}

// forward step B store: q[t] = slot t of the partner thread.  For k1 > 0,
// Z[L - k] = partner slot N2 - 1 - k2; for k1 = 0, slot (N2 - k2) mod N2.
// A = (Z[k] + conj Z[L-k]) / 2, B = (Z[k] - conj Z[L-k]) / 2i -> rows g, g+1
template <int L>
__device__ __forceinline__ void dp_rows_fwd_store(int tid, int w0, int G, const float2 *u, const float2 *q,
                                                  float2 *S) {
  using D = DPlane<L>;
  const int wl = tid / D::N1, k1 = tid - wl * D::N1, g = 2 * (w0 + wl);
  if (g >= G) return;
  const bool two = g + 1 < G;
#pragma unroll
  for (int k2 = 0; k2 < D::N2; ++k2) {
    const int k = k1 + D::N1 * k2;
    if (k <= L / 2) {
      const float2 zk = u[k2], zm = k1 ? q[D::N2 - 1 - k2] : q[(D::N2 - k2) % D::N2];
      S[g * D::H + k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      if (two) S[(g + 1) * D::H + k] = make_float2(0.5f * (zk.y + zm.y), 0.5f * (zm.x - zk.x));
    }
  }
}

// grid position of spectrum row r: natural, or r / N2 + N1 (r mod N2) after
// the forward finish's column inverse
template <int L, bool PERM>
__device__ __forceinline__ int dp_row_pos(int r) {
  using D = DPlane<L>;
  if constexpr (PERM) {
    const int q = r / D::N2;
    return q + D::N1 * (r - q * D::N2);
  } else {
    return r;
  }
}

// inverse step A of round w0: line w holds rows z = 2w (real) and 2w + 1
// (imaginary) of the output, read from spectrum rows r0 + z
template <int L, bool PERM>
__device__ __forceinline__ void dp_rows_inv_a(int tid, int w0, const float2 *S, float2 *X, const float2 *twr,
                                              int r0, int nz) {
  using D = DPlane<L>;
  if (tid >= D::LINES * D::N2) return;
  const int wl = tid / D::N2, n2 = tid - wl * D::N2, z = 2 * (w0 + wl);
  const bool ha = z < nz, hb = z + 1 < nz;
  const int ra = ha ? dp_row_pos<L, PERM>(r0 + z) : 0, rb = hb ? dp_row_pos<L, PERM>(r0 + z + 1) : 0;
  float2 v[D::N1];
#pragma unroll
  for (int n1 = 0; n1 < D::N1; ++n1) {
    const int k = n2 + D::N2 * n1;
    const bool lo = k <= L / 2;
    const int kk = lo ? k : L - k;
    const float2 A = ha ? S[ra * D::H + kk] : make_float2(0.f, 0.f);
    const float2 B = hb ? S[rb * D::H + kk] : make_float2(0.f, 0.f);
    v[n1] = lo ? make_float2(A.x - B.y, A.y + B.x) : make_float2(A.x + B.y, B.x - A.y);
  }
  RDft<D::N1, true>::run(v);
#pragma unroll
  for (int k1 = 1; k1 < D::N1; ++k1) v[k1] = twiddle<true>(v[k1], twr[k1 * D::N2 + n2]);
#pragma unroll
  for (int k1 = 0; k1 < D::N1; ++k1) X[k1 * D::XI + tid] = v[k1];
}

// inverse step B store: x[k1 + N1 k2] of rows z (real part), z + 1
// (imaginary part), x < n, times scale
template <int L>
__device__ __forceinline__ void dp_rows_inv_store(int tid, int w0, const float2 *u, float *out, int n, int nz,
                                                  float scale) {
  using D = DPlane<L>;
  const int wl = tid / D::N1, k1 = tid - wl * D::N1, z = 2 * (w0 + wl);
  if (z >= nz) return;
  const bool two = z + 1 < nz;
#pragma unroll
  for (int k2 = 0; k2 < D::N2; ++k2) {
    const int x = k1 + D::N1 * k2;
    if (x < n) {
      out[(size_t)z * n + x] = u[k2].x * scale;
      if (two) out[(size_t)(z + 1) * n + x] = u[k2].y * scale;
    }
  }
}

// ------------------------------------------------------------- columns

// step A: column c, rows n2 + N2 n1 (rows >= G are zero) -> Y[n2][k1]
// W^(n2 k1) at row n2 + N2 k1
template <int L>
__device__ __forceinline__ void dp_cols_a(int tid, float2 *S, const float2 *tw, int G) {
  using D = DPlane<L>;
  for (int i = tid; i < D::N2 * D::H; i += DP_NT) {
    const int n2 = i / D::H, c = i - n2 * D::H;
    float2 v[D::N1];
#pragma unroll
    for (int n1 = 0; n1 < D::N1; ++n1) {
      const int r = n2 + D::N2 * n1;
      v[n1] = r < G ? S[r * D::H + c] : make_float2(0.f, 0.f);
    }
    RDft<D::N1, false>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < D::N1; ++k1) v[k1] = twiddle<false>(v[k1], tw[n2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < D::N1; ++k1) S[(n2 + D::N2 * k1) * D::H + c] = v[k1];
  }
}

// backward step B: spectrum X[k1 + N1 k2] times the PSF spectrum, then the
// N2-point inverse and the twiddle conj W^(k1 m2), back to row m2 + N2 k1
template <int L>
__device__ __forceinline__ void dp_cols_b_bck(int tid, float2 *S, const float2 *tw, const float2 *Hd) {
  using D = DPlane<L>;
  for (int j = tid; j < D::N1 * D::H; j += DP_NT) {
    const int k1 = j / D::H, c = j - k1 * D::H;
    float2 u[D::N2], h[D::N2];
#pragma unroll
    for (int k2 = 0; k2 < D::N2; ++k2) h[k2] = dp_ld(Hd + (k1 + D::N1 * k2) * D::H + c);
#pragma unroll
    for (int n2 = 0; n2 < D::N2; ++n2) u[n2] = S[(n2 + D::N2 * k1) * D::H + c];
    RDft<D::N2, false>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < D::N2; ++k2) u[k2] = cmul(u[k2], h[k2]);
    RDft<D::N2, true>::run(u);
#pragma unroll
    for (int m2 = 1; m2 < D::N2; ++m2) u[m2] = twiddle<true>(u[m2], tw[k1 * m2]);
#pragma unroll
    for (int m2 = 0; m2 < D::N2; ++m2) S[(m2 + D::N2 * k1) * D::H + c] = u[m2];
  }
}

// step C: N1-point inverses; output rows r = m2 + N2 m1 in [r0, r1) stored
template <int L>
__device__ __forceinline__ void dp_cols_c(int tid, float2 *S, int r0, int r1) {
  using D = DPlane<L>;
  for (int i = tid; i < D::N2 * D::H; i += DP_NT) {
    const int m2 = i / D::H, c = i - m2 * D::H;
    float2 v[D::N1];
#pragma unroll
    for (int k1 = 0; k1 < D::N1; ++k1) v[k1] = S[(m2 + D::N2 * k1) * D::H + c];
    RDft<D::N1, true>::run(v);
#pragma unroll
    for (int m1 = 0; m1 < D::N1; ++m1) {
      const int r = m2 + D::N2 * m1;
      if (r >= r0 && r < r1) S[r * D::H + c] = v[m1];
    }
  }
}

// forward step B: acc[rr][k2] += X[k1 + N1 k2] * H, item j = tid + rr DP_NT
template <int L>
__device__ __forceinline__ void dp_cols_b_acc(int tid, const float2 *S, const float2 *Hd,
                                              float2 (*acc)[DPlane<L>::N2]) {
  using D = DPlane<L>;
#pragma unroll
  for (int rr = 0; rr < D::NRB; ++rr) {
    const int j = tid + rr * DP_NT;
    if (j < D::N1 * D::H) {
      const int k1 = j / D::H, c = j - k1 * D::H;
      float2 u[D::N2];
#pragma unroll
      for (int n2 = 0; n2 < D::N2; ++n2) u[n2] = S[(n2 + D::N2 * k1) * D::H + c];
      RDft<D::N2, false>::run(u);
#pragma unroll
      for (int k2 = 0; k2 < D::N2; ++k2)
        acc[rr][k2] = cadd(acc[rr][k2], cmul(u[k2], dp_ld(Hd + (k1 + D::N1 * k2) * D::H + c)));
    }
  }
}

// forward partial sums of item j = tid + rr DP_NT -> part[k][c]
template <int L>
__device__ __forceinline__ void dp_store_acc(int tid, float2 *part, float2 (*acc)[DPlane<L>::N2]) {
  using D = DPlane<L>;
#pragma unroll
  for (int rr = 0; rr < D::NRB; ++rr) {
    const int j = tid + rr * DP_NT;
    if (j < D::N1 * D::H) {
      const int k1 = j / D::H, c = j - k1 * D::H;
#pragma unroll
      for (int k2 = 0; k2 < D::N2; ++k2) part[(size_t)(k1 + D::N1 * k2) * D::H + c] = acc[rr][k2];
    }
  }
}

// forward finish step B: the spectrum (natural order, partial sums of npg
// groups added in group order), N2-point inverse, conj W^(k1 m2), stored at
// row k1 + N1 m2
template <int L>
__device__ __forceinline__ void dp_fin_b(int tid, float2 *S, const float2 *tw, const float2 *part, size_t pg_stride,
                                         int npg) {
  using D = DPlane<L>;
  for (int j = tid; j < D::N1 * D::H; j += DP_NT) {
    const int k1 = j / D::H, c = j - k1 * D::H;
    float2 u[D::N2];
#pragma unroll
    for (int k2 = 0; k2 < D::N2; ++k2) u[k2] = make_float2(0.f, 0.f);
    for (int pg = 0; pg < npg; ++pg) {
      const float2 *pp = part + pg * pg_stride + c;
#pragma unroll
      for (int k2 = 0; k2 < D::N2; ++k2) u[k2] = cadd(u[k2], dp_ld(pp + (k1 + D::N1 * k2) * D::H));
    }
    RDft<D::N2, true>::run(u);
#pragma unroll
    for (int m2 = 1; m2 < D::N2; ++m2) u[m2] = twiddle<true>(u[m2], tw[k1 * m2]);
#pragma unroll
    for (int m2 = 0; m2 < D::N2; ++m2) S[(k1 + D::N1 * m2) * D::H + c] = u[m2];
  }
}

// forward finish step C: N1-point inverses; natural row m2 + N2 m1 ends at
// position m1 + N1 m2 (dp_row_pos<L, true>)
template <int L>
__device__ __forceinline__ void dp_fin_c(int tid, float2 *S) {
  using D = DPlane<L>;
  for (int i = tid; i < D::N2 * D::H; i += DP_NT) {
    const int m2 = i / D::H, c = i - m2 * D::H;
    float2 v[D::N1];
#pragma unroll
    for (int k1 = 0; k1 < D::N1; ++k1) v[k1] = S[(k1 + D::N1 * m2) * D::H + c];
    RDft<D::N1, true>::run(v);
#pragma unroll
    for (int m1 = 0; m1 < D::N1; ++m1) S[(m1 + D::N1 * m2) * D::H + c] = v[m1];
  }
}

}  // namespace irlcu
