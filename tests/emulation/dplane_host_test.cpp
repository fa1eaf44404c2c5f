// Host emulation of the one-CTA-per-plane DRF kernels: every phase of
// drf_plane.cuh runs for all threads of a CTA, in forward and in reverse
// thread order (a phase that depended on another thread of the same phase
// would differ), against a direct circular convolution in double.
// host emulation of the fused per-plane DRF kernels (phases of drf_plane.cuh)
#include <cstdio>
#include <cmath>
#include <vector>
#include <random>
#include <complex>
#include <algorithm>
struct D3 { int x, y, z; }; static D3 threadIdx, blockDim;
static inline void __syncthreads() {}
#include <cuda_runtime.h>
static inline float __ldg(const float *p) { return *p; }
static inline float __fmul_rn(float a, float b) { return a * b; }
static inline float __fadd_rn(float a, float b) { return a + b; }
static inline float __fdiv_rn(float a, float b) { return a / b; }
#include "drf_plane.cuh"
using namespace irlcu;
static double g_worst = 0;
static double track(double e) { if (!(e <= g_worst)) g_worst = e; return e; }
using cd = std::complex<double>;

template <int L> struct Case {
  using D = DPlane<L>;
  int n, nz, P, G, pady, avgy, hh, nplanes, ndist;
  std::vector<float> a, e;          // [y][z][x]
  std::vector<float> psf;           // [d][L][L] real grid (wrapped)
  std::vector<float2> Hs;           // [d][L][H]
  std::vector<float2> twg;
  std::vector<int> dist;            // per plane
};

template <int L> void make_case(Case<L> &C, int n, int nz, int P, int G, int pady, int avgy, int hh, int nplanes, int ndist, unsigned seed) {
  using D = DPlane<L>;
  std::mt19937 rng(seed); std::uniform_real_distribution<float> U(0, 1);
  C.n = n; C.nz = nz; C.P = P; C.G = G; C.pady = pady; C.avgy = avgy; C.hh = hh; C.nplanes = nplanes; C.ndist = ndist;
  C.a.resize((size_t)nplanes * nz * n); C.e.resize(C.a.size());
  for (auto &v : C.a) v = U(rng); for (auto &v : C.e) v = 0.5f + 0.5f * U(rng);
  C.psf.assign((size_t)ndist * L * L, 0.f);
  for (int d = 0; d < ndist; ++d) for (int dy = -hh; dy <= hh; ++dy) for (int dx = -hh; dx <= hh; ++dx)
    C.psf[(size_t)d * L * L + ((dy + L) % L) * L + ((dx + L) % L)] = U(rng);
  C.Hs.resize((size_t)ndist * L * D::H);
  for (int d = 0; d < ndist; ++d) {
    std::vector<cd> R((size_t)L * D::H);
    for (int g = 0; g < L; ++g) for (int k = 0; k < D::H; ++k) { cd s = 0; for (int x = 0; x < L; ++x) s += (double)C.psf[(size_t)d*L*L + g*L + x] * std::polar(1.0, -2*M_PI*(double)x*k/L); R[g*D::H+k] = s; }
    for (int kz = 0; kz < L; ++kz) for (int k = 0; k < D::H; ++k) { cd s = 0; for (int g = 0; g < L; ++g) s += R[g*D::H+k] * std::polar(1.0, -2*M_PI*(double)g*kz/L); s /= (double)L * L; C.Hs[(size_t)d*L*D::H + kz*D::H + k] = make_float2((float)s.real(), (float)s.imag()); }
  }
  C.twg.resize(L);
  for (int m = 0; m < L; ++m) C.twg[m] = make_float2((float)cos(-2*M_PI*m/L), (float)sin(-2*M_PI*m/L));
  C.dist.resize(nplanes); for (int y = 0; y < nplanes; ++y) C.dist[y] = y % ndist;
}

template <int L> PlaneSrc src_of(const Case<L> &C, int y) {
  PlaneSrc p; p.a = C.a.data() + (size_t)y * C.nz * C.n; p.e = C.e.data() + (size_t)y * C.nz * C.n;
  p.n = C.n; p.nz = C.nz; p.P = C.P; p.pady = C.pady; p.avgy = C.avgy; return p;
}

// direct circular convolution on the L x L grid, rows P .. P+nz-1
template <int L> void ref_plane(const Case<L> &C, int y, std::vector<double> &out) {
  PlaneSrc p = src_of(C, y);
  std::vector<double> grid((size_t)L * L, 0.0);
  for (int g = 0; g < C.G; ++g) for (int x = 0; x < C.n; ++x) grid[g * L + x] = psrc_val(p, g, x);
  const float *ps = C.psf.data() + (size_t)C.dist[y] * L * L;
  for (int z = 0; z < C.nz; ++z) for (int x = 0; x < C.n; ++x) {
    double s = 0; const int g = z + C.P;
    for (int dy = -C.hh; dy <= C.hh; ++dy) for (int dx = -C.hh; dx <= C.hh; ++dx)
      s += grid[((g - dy + L) % L) * L + ((x - dx + L) % L)] * ps[((dy + L) % L) * L + ((dx + L) % L)];
    out[(size_t)z * C.n + x] += s;
  }
}

template <class F> void for_threads(bool rev, F f) { if (rev) for (int t = DP_NT - 1; t >= 0; --t) f(t); else for (int t = 0; t < DP_NT; ++t) f(t); }

template <int L> void emu_rows_fwd(const Case<L> &C, const PlaneSrc &p, float2 *S, float2 *X, const float2 *twr, bool rev) {
  using D = DPlane<L>;
  const int nl = (C.G + 1) / 2;
  std::vector<float2> U((size_t)DP_NT * D::N2);
  for (int w0 = 0; w0 < nl; w0 += D::LINES) {
    for_threads(rev, [&](int t) { dp_rows_fwd_a<L>(t, w0, p, C.G, X, twr); });
    for_threads(rev, [&](int t) { dp_rows_b<L, false>(t, X, &U[(size_t)t * D::N2]); });
    for_threads(rev, [&](int t) { dp_rows_fwd_store<L>(t, w0, C.G, &U[(size_t)t * D::N2], &U[(size_t)dp_partner<L>(t) * D::N2], S); });
  }
}

template <int L, bool PERM> void emu_rows_inv(const Case<L> &C, const float2 *S, float2 *X, const float2 *twr, float *out, float scale, bool rev) {
  using D = DPlane<L>;
  const int nl = (C.nz + 1) / 2;
  std::vector<float2> U((size_t)DP_NT * D::N2);
  for (int w0 = 0; w0 < nl; w0 += D::LINES) {
    for_threads(rev, [&](int t) { dp_rows_inv_a<L, PERM>(t, w0, S, X, twr, C.P, C.nz); });
    for_threads(rev, [&](int t) { float2 *u = &U[(size_t)t * D::N2]; dp_rows_b<L, true>(t, X, u); dp_rows_inv_store<L>(t, w0, u, out, C.n, C.nz, scale); });
  }
}

template <int L> double run_bck(const Case<L> &C, bool rev) {
  using D = DPlane<L>;
  double e2 = 0, r2 = 0;
  for (int y = 0; y < C.nplanes; ++y) {
    std::vector<float2> S(D::S_ELEMS, make_float2(NAN, NAN)), X(D::X_ELEMS, make_float2(NAN, NAN)), tw(L), twr(L);
    for_threads(rev, [&](int t) { dp_twiddles<L>(t, tw.data(), twr.data(), C.twg.data()); });
    PlaneSrc p = src_of(C, y);
    const float2 *Hd = C.Hs.data() + (size_t)C.dist[y] * L * D::H;
    emu_rows_fwd<L>(C, p, S.data(), X.data(), twr.data(), rev);
    for_threads(rev, [&](int t) { dp_cols_a<L>(t, S.data(), tw.data(), C.G); });
    for_threads(rev, [&](int t) { dp_cols_b_bck<L>(t, S.data(), tw.data(), Hd); });
    for_threads(rev, [&](int t) { dp_cols_c<L>(t, S.data(), C.P, C.P + C.nz); });
    std::vector<float> out((size_t)C.nz * C.n, NAN);
    emu_rows_inv<L, false>(C, S.data(), X.data(), twr.data(), out.data(), 0.5f, rev);
    std::vector<double> ref((size_t)C.nz * C.n, 0.0);
    ref_plane<L>(C, y, ref);
    for (size_t i = 0; i < ref.size(); ++i) { const double r = 0.5 * ref[i]; e2 += (out[i] - r) * (out[i] - r); r2 += r * r; }
  }
  return std::sqrt(e2 / r2);
}

template <int L> double run_fwd(const Case<L> &C, int npg, bool rev) {
  using D = DPlane<L>;
  std::vector<float2> part((size_t)npg * L * D::H, make_float2(NAN, NAN));
  for (int pg = 0; pg < npg; ++pg) {
    std::vector<float2> S(D::S_ELEMS, make_float2(NAN, NAN)), X(D::X_ELEMS, make_float2(NAN, NAN)), tw(L), twr(L);
    for_threads(rev, [&](int t) { dp_twiddles<L>(t, tw.data(), twr.data(), C.twg.data()); });
    std::vector<float2> acc((size_t)DP_NT * D::NRB * D::N2, make_float2(0.f, 0.f));
    const int y0 = pg * C.nplanes / npg, y1 = (pg + 1) * C.nplanes / npg;
    for (int y = y0; y < y1; ++y) {
      PlaneSrc p = src_of(C, y);
      const float2 *Hd = C.Hs.data() + (size_t)C.dist[y] * L * D::H;
      emu_rows_fwd<L>(C, p, S.data(), X.data(), twr.data(), rev);
      for_threads(rev, [&](int t) { dp_cols_a<L>(t, S.data(), tw.data(), C.G); });
      for_threads(rev, [&](int t) { dp_cols_b_acc<L>(t, S.data(), Hd, reinterpret_cast<float2 (*)[D::N2]>(&acc[(size_t)t * D::NRB * D::N2])); });
    }
    for_threads(rev, [&](int t) { dp_store_acc<L>(t, part.data() + (size_t)pg * L * D::H, reinterpret_cast<float2 (*)[D::N2]>(&acc[(size_t)t * D::NRB * D::N2])); });
  }
  std::vector<float2> S(D::S_ELEMS, make_float2(NAN, NAN)), X(D::X_ELEMS, make_float2(NAN, NAN)), tw(L), twr(L);
  for_threads(rev, [&](int t) { dp_twiddles<L>(t, tw.data(), twr.data(), C.twg.data()); });
  for_threads(rev, [&](int t) { dp_fin_b<L>(t, S.data(), tw.data(), part.data(), (size_t)L * D::H, npg); });
  for_threads(rev, [&](int t) { dp_fin_c<L>(t, S.data()); });
  std::vector<float> out((size_t)C.nz * C.n, NAN);
  emu_rows_inv<L, true>(C, S.data(), X.data(), twr.data(), out.data(), 2.0f, rev);
  std::vector<double> ref((size_t)C.nz * C.n, 0.0);
  for (int y = 0; y < C.nplanes; ++y) ref_plane<L>(C, y, ref);
  double e2 = 0, r2 = 0;
  for (size_t i = 0; i < ref.size(); ++i) { const double r = 2.0 * ref[i]; e2 += (out[i] - r) * (out[i] - r); r2 += r * r; }
  return std::sqrt(e2 / r2);
}

template <int L> void test(int n, int nz, int P, int G, int pady, int avgy, int hh, int nplanes, int ndist, int npg) {
  Case<L> C; make_case<L>(C, n, nz, P, G, pady, avgy, hh, nplanes, ndist, L * 31 + n);
  printf("L=%3d n=%3d nz=%3d P=%d G=%3d h=%2d: bck %.2e / %.2e  fwd %.2e / %.2e\n", L, n, nz, P, G, hh,
         track(run_bck<L>(C, false)), track(run_bck<L>(C, true)), track(run_fwd<L>(C, npg, false)), track(run_fwd<L>(C, npg, true)));
}

int main() {
  test<40>(24, 20, 2, 24, 2, 2, 5, 3, 2, 2);
  test<48>(30, 17, 0, 17, 0, 0, 8, 3, 3, 2);
  test<64>(48, 40, 3, 46, 3, 2, 7, 4, 2, 3);
  test<80>(48, 48, 4, 56, 4, 3, 16, 3, 3, 2);
  test<96>(70, 60, 0, 60, 0, 0, 12, 2, 2, 1);
  test<128>(100, 90, 1, 92, 1, 1, 9, 2, 2, 2);
  test<160>(128, 128, 0, 128, 0, 0, 16, 3, 3, 2);
  test<192>(150, 101, 5, 111, 5, 2, 20, 2, 2, 2);
  printf("worst %.3e\n", g_worst);
  return g_worst < 1e-5 ? 0 : 1;
}
