// esse_yz.cuh -- phases of the y-z part of the ESSE convolution for one kx
// plane of one view, in one CTA (kernel in k_esse.cu).
//
// The plane F[y][z] (L x L complex, L = Ky = Kz = N1 N2) holds the x
// spectra A[y][z] of the collapsed volume (y < nyv, z < nzv, zero
// elsewhere).  With the two-level register transforms of reg_fft.cuh, all
// in place in F:
//   z forward (rows y < nyv): step A, then step B leaving the spectrum at
//       position p = k2 + N2 k1 for frequency kz = k1 + N1 k2;
//   y forward (all L positions): step A; step B runs per term, fused with
//       the product by the kernel spectrum (stored in the same position
//       order, K[kx][ky][p]) and the first half of the inverse y
//       transform, for a chunk of ZC positions at a time into the chunk
//       buffer C[t]; step C of the inverse keeps rows y < nyv and writes
//       them into the chunk's columns of F, which are no longer needed:
//       rows [t nyv, (t+1) nyv) of F hold term t afterwards;
//   z inverse (rows of both terms): steps B and C from the position order
//       back to natural z.
// Rows are swizzled (element (r, p) at r L + (p ^ (r mod 16))) so that walks
// along a row by consecutive rows and walks along a column by consecutive
// positions are both free of bank conflicts.  Every phase is a function of
// the thread index so that a host emulation of the CTA runs the same code.
#pragma once

#include "reg_fft.cuh"

namespace irlcu {

constexpr int EY_NT = 512;  // threads per CTA
constexpr int EY_ZC = 32;   // positions per chunk of the y inverse

template <int L>
struct EYz {
  static constexpr int N1 = LineSplit<L>::N1, N2 = LineSplit<L>::N2;
  static constexpr int F_ELEMS = L * L;
  static constexpr int C_ELEMS = L * EY_ZC;  // per term
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)F_ELEMS + 2 * C_ELEMS + L);
  static_assert(L % 16 == 0 && L % EY_ZC == 0, "ESSE plane length");
};

template <int L>
__device__ __forceinline__ int ey_at(int r, int p) {
  return r * L + (p ^ (r & 15));
}

#ifdef __CUDA_ARCH__
__device__ __forceinline__ float2 ey_ld(const float2 *p) { return __ldg(p); }
#else
inline float2 ey_ld(const float2 *p) { return *p; }
#endif

// P0: A[y][z] (y < nyv, z < nzv, row stride nzv) -> F
template <int L>
__device__ __forceinline__ void ey_load(int tid, float2 *F, const float2 *A, int nyv, int nzv) {
  for (int e = tid; e < nyv * nzv; e += EY_NT) {
    const int y = e / nzv, z = e - y * nzv;
    F[ey_at<L>(y, z)] = ey_ld(A + e);
  }
}

// P1: z forward step A, rows y < nyv (item: y fastest, then n2)
template <int L>
__device__ __forceinline__ void ey_z_fwd_a(int tid, float2 *F, const float2 *tw, int nyv, int nzv) {
  using D = EYz<L>;
  for (int i = tid; i < nyv * D::N2; i += EY_NT) {
    const int n2 = i / nyv, y = i - n2 * nyv;
    float2 v[D::N1];
#pragma unroll
    for (int n1 = 0; n1 < D::N1; ++n1) {
      const int z = n2 + D::N2 * n1;
      v[n1] = z < nzv ? F[ey_at<L>(y, z)] : make_float2(0.f, 0.f);
    }
    RDft<D::N1, false>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < D::N1; ++k1) v[k1] = twiddle<false>(v[k1], tw[n2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < D::N1; ++k1) F[ey_at<L>(y, n2 + D::N2 * k1)] = v[k1];
  }
}

// P2: z forward step B: kz = k1 + N1 k2 at position k2 + N2 k1
template <int L>
__device__ __forceinline__ void ey_z_fwd_b(int tid, float2 *F, int nyv) {
  using D = EYz<L>;
  for (int i = tid; i < nyv * D::N1; i += EY_NT) {
    const int k1 = i / nyv, y = i - k1 * nyv;
    float2 u[D::N2];
#pragma unroll
    for (int n2 = 0; n2 < D::N2; ++n2) u[n2] = F[ey_at<L>(y, n2 + D::N2 * k1)];
    RDft<D::N2, false>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < D::N2; ++k2) F[ey_at<L>(y, k2 + D::N2 * k1)] = u[k2];
  }
}

// P3: y forward step A over every position p (rows y >= nyv are zero)
template <int L>
__device__ __forceinline__ void ey_y_fwd_a(int tid, float2 *F, const float2 *tw, int nyv) {
  using D = EYz<L>;
  for (int i = tid; i < L * D::N2; i += EY_NT) {
    const int n2 = i / L, p = i - n2 * L;
    float2 v[D::N1];
#pragma unroll
    for (int n1 = 0; n1 < D::N1; ++n1) {
      const int y = n2 + D::N2 * n1;
      v[n1] = y < nyv ? F[ey_at<L>(y, p)] : make_float2(0.f, 0.f);
    }
    RDft<D::N1, false>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < D::N1; ++k1) v[k1] = twiddle<false>(v[k1], tw[n2 * k1]);
#pragma unroll
    for (int k1 = 0; k1 < D::N1; ++k1) F[ey_at<L>(n2 + D::N2 * k1, p)] = v[k1];
  }
}

// P4: for positions z0 .. z0+ZC-1: y forward step B (ky = k1 + N1 k2), the
// product by each term's spectrum K[t][ky][p] (this kx plane, row stride
// L), the N2-point inverse and conj W^(k1 m2) -> C[t][m2 + N2 k1][pl]
template <int L>
__device__ __forceinline__ void ey_y_mid(int tid, const float2 *F, float2 *C, const float2 *tw,
                                         const float2 *K0, const float2 *K1, int nt, int z0) {
  using D = EYz<L>;
  for (int i = tid; i < EY_ZC * D::N1; i += EY_NT) {
    const int k1 = i / EY_ZC, pl = i - k1 * EY_ZC, p = z0 + pl;
    float2 h0[D::N2], h1[D::N2], u[D::N2];
#pragma unroll
    for (int k2 = 0; k2 < D::N2; ++k2) {
      const int ky = k1 + D::N1 * k2;
      h0[k2] = ey_ld(K0 + ky * L + p);
      h1[k2] = nt > 1 ? ey_ld(K1 + ky * L + p) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int n2 = 0; n2 < D::N2; ++n2) u[n2] = F[ey_at<L>(n2 + D::N2 * k1, p)];
    RDft<D::N2, false>::run(u);
    for (int t = 0; t < nt; ++t) {
      float2 w[D::N2];
#pragma unroll
      for (int k2 = 0; k2 < D::N2; ++k2) w[k2] = cmul(u[k2], t ? h1[k2] : h0[k2]);
      RDft<D::N2, true>::run(w);
#pragma unroll
      for (int m2 = 1; m2 < D::N2; ++m2) w[m2] = twiddle<true>(w[m2], tw[k1 * m2]);
      float2 *Ct = C + t * D::C_ELEMS;
#pragma unroll
      for (int m2 = 0; m2 < D::N2; ++m2) Ct[(m2 + D::N2 * k1) * EY_ZC + pl] = w[m2];
    }
  }
}

// P5: y inverse step C: y = m2 + N2 m1 < nyv of term t -> F row t nyv + y
template <int L>
__device__ __forceinline__ void ey_y_inv_c(int tid, float2 *F, const float2 *C, int nt, int nyv, int z0) {
  using D = EYz<L>;
  for (int i = tid; i < nt * D::N2 * EY_ZC; i += EY_NT) {
    const int tm = i / EY_ZC, pl = i - tm * EY_ZC;
    const int t = tm / D::N2, m2 = tm - t * D::N2;
    const float2 *Ct = C + t * D::C_ELEMS;
    float2 v[D::N1];
#pragma unroll
    for (int k1 = 0; k1 < D::N1; ++k1) v[k1] = Ct[(m2 + D::N2 * k1) * EY_ZC + pl];
    RDft<D::N1, true>::run(v);
#pragma unroll
    for (int m1 = 0; m1 < D::N1; ++m1) {
      const int y = m2 + D::N2 * m1;
      if (y < nyv) F[ey_at<L>(t * nyv + y, z0 + pl)] = v[m1];
    }
  }
}

// P6: z inverse step B on rows r < nr: X[k1 + N1 k2] at k2 + N2 k1 ->
// conj W^(k1 m2) Z[k1][m2] at m2 + N2 k1
template <int L>
__device__ __forceinline__ void ey_z_inv_b(int tid, float2 *F, const float2 *tw, int nr) {
  using D = EYz<L>;
  for (int i = tid; i < nr * D::N1; i += EY_NT) {
    const int k1 = i / nr, r = i - k1 * nr;
    float2 u[D::N2];
#pragma unroll
    for (int k2 = 0; k2 < D::N2; ++k2) u[k2] = F[ey_at<L>(r, k2 + D::N2 * k1)];
    RDft<D::N2, true>::run(u);
#pragma unroll
    for (int m2 = 1; m2 < D::N2; ++m2) u[m2] = twiddle<true>(u[m2], tw[k1 * m2]);
#pragma unroll
    for (int m2 = 0; m2 < D::N2; ++m2) F[ey_at<L>(r, m2 + D::N2 * k1)] = u[m2];
  }
}

// P7: z inverse step C: natural z = m2 + N2 m1 (only z < nzv stored)
template <int L>
__device__ __forceinline__ void ey_z_inv_c(int tid, float2 *F, int nr, int nzv) {
  using D = EYz<L>;
  for (int i = tid; i < nr * D::N2; i += EY_NT) {
    const int m2 = i / nr, r = i - m2 * nr;
    float2 v[D::N1];
#pragma unroll
    for (int k1 = 0; k1 < D::N1; ++k1) v[k1] = F[ey_at<L>(r, m2 + D::N2 * k1)];
    RDft<D::N1, true>::run(v);
#pragma unroll
    for (int m1 = 0; m1 < D::N1; ++m1) {
      const int z = m2 + D::N2 * m1;
      if (z < nzv) F[ey_at<L>(r, z)] = v[m1];
    }
  }
}

// P8: F rows t nyv + y, z < nzv -> D[t][y][z] (row stride nzv)
template <int L>
__device__ __forceinline__ void ey_store(int tid, const float2 *F, float2 *D0, float2 *D1, int nt, int nyv,
                                         int nzv) {
  for (int e = tid; e < nt * nyv * nzv; e += EY_NT) {
    const int r = e / nzv, z = e - r * nzv;
    const int t = r >= nyv, y = r - t * nyv;
    (t ? D1 : D0)[y * nzv + z] = F[ey_at<L>(r, z)];
  }
}

}  // namespace irlcu
