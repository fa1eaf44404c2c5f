// Host emulation of the ESSE x transforms (esse_rows.cuh): the collapse +
// R2C rows and the C2R rows against direct DFTs in double; both thread
// orders.
#include <cstdio>
#include <cmath>
#include <vector>
#include <random>
#include <complex>
struct D3 { int x, y, z; }; static D3 threadIdx, blockDim;
static inline void __syncthreads() {}
#include <cuda_runtime.h>
static inline float __fadd_rn(float a, float b) { return a + b; }
#include "esse_rows.cuh"
using namespace irlcu;
static double g_worst = 0;
static double track(double e) { if (!(e <= g_worst)) g_worst = e; return e; }
using cd = std::complex<double>;
template <class F> void for_threads(bool rev, F f) { if (rev) for (int t = ER_NT - 1; t >= 0; --t) f(t); else for (int t = 0; t < ER_NT; ++t) f(t); }

template <int L> void test(int n, int nz, int c, unsigned seed) {
  using D = ERow<L>;
  const int nxv = n / c, nyv = n / c, nzv = nz / c, nrows = nyv * nzv;
  std::mt19937 rng(seed); std::uniform_real_distribution<float> U(0, 1);
  std::vector<float> rot((size_t)n * nz * n); for (auto &v : rot) v = U(rng);
  std::vector<float2> tw(L); for (int m = 0; m < L; ++m) tw[m] = make_float2((float)cos(-2*M_PI*m/L), (float)sin(-2*M_PI*m/L));
  // reference collapsed rows and their half spectra
  std::vector<double> row((size_t)nrows * nxv);
  for (int r = 0; r < nrows; ++r) for (int x = 0; x < nxv; ++x) { int yy = r / nzv, zz = r % nzv; double t = 0; for (int k = 0; k < c; ++k) for (int j = 0; j < c; ++j) for (int i = 0; i < c; ++i) t += rot[((size_t)(yy*c+k)*nz + zz*c+j)*n + x*c+i]; row[(size_t)r*nxv+x] = t; }
  std::vector<float2> out((size_t)D::H * nrows, make_float2(NAN, NAN));
  const int nlines = (nrows + 1) / 2;
  double e2 = 0, r2 = 0;
  for (int rev = 0; rev < 2; ++rev) {
    std::vector<float2> X(D::X_ELEMS, make_float2(NAN, NAN));
    std::vector<float2> U2((size_t)ER_LW * D::N1 * D::N2);
    for (int w0 = 0; w0 < nlines; w0 += ER_LW) {
      for_threads(rev, [&](int t) { er_fwd_a<L>(t, w0, X.data(), tw.data(), rot.data(), n, nz, c, nzv, nxv, nrows); });
      for_threads(rev, [&](int t) { for (int it = t; it < ER_LW * D::N1; it += ER_NT) er_b<L, false>(it, X.data(), &U2[(size_t)it * D::N2]); });
      for_threads(rev, [&](int t) { for (int it = t; it < ER_LW * D::N1; it += ER_NT) er_fwd_b_store<L>(it, &U2[(size_t)it * D::N2], X.data()); });
      for_threads(rev, [&](int t) { er_fwd_unpack<L>(t, w0, X.data(), out.data(), nrows); });
    }
    e2 = r2 = 0;
    for (int r = 0; r < nrows; ++r) for (int k = 0; k < D::H; ++k) { cd s = 0; for (int x = 0; x < nxv; ++x) s += row[(size_t)r*nxv+x] * std::polar(1.0, -2*M_PI*(double)x*k/L); cd g(out[(size_t)k*nrows+r].x, out[(size_t)k*nrows+r].y); e2 += std::norm(g - s); r2 += std::norm(s); }
    printf("L=%d n=%d nz=%d c=%d fwd %s rel %.2e\n", L, n, nz, c, rev ? "rev" : "fwd", track(std::sqrt(e2 / r2)));
  }
  // inverse of random half spectra (Hermitian at 0 and L/2 not required: the C2R takes the real part)
  std::vector<float2> in((size_t)D::H * nrows);
  for (auto &v : in) v = make_float2(U(rng) - 0.5f, U(rng) - 0.5f);
  for (int r = 0; r < nrows; ++r) { in[r].y = 0; in[(size_t)(L/2)*nrows + r].y = 0; }
  for (int rev = 0; rev < 2; ++rev) {
    std::vector<float2> X(D::X_ELEMS, make_float2(NAN, NAN));
    std::vector<float> g((size_t)nrows * nxv, NAN);
    std::vector<float2> U2((size_t)ER_LW * D::N1 * D::N2);
    for (int w0 = 0; w0 < nlines; w0 += ER_LW) {
      for_threads(rev, [&](int t) { er_inv_a<L>(t, w0, X.data(), tw.data(), in.data(), nrows); });
      for_threads(rev, [&](int t) { for (int it = t; it < ER_LW * D::N1; it += ER_NT) { er_b<L, true>(it, X.data(), &U2[(size_t)it * D::N2]); er_inv_b_store<L>(it, w0, &U2[(size_t)it * D::N2], g.data(), nrows, nxv, 0.25f); } });
    }
    e2 = r2 = 0;
    for (int r = 0; r < nrows; ++r) for (int x = 0; x < nxv; ++x) {
      double s = 0; for (int k = 0; k < L; ++k) { int kk = k <= L/2 ? k : L - k; cd a(in[(size_t)kk*nrows+r].x, in[(size_t)kk*nrows+r].y); if (k > L/2) a = std::conj(a); s += (a * std::polar(1.0, 2*M_PI*(double)x*k/L)).real(); }
      s *= 0.25; e2 += (g[(size_t)r*nxv+x] - s) * (g[(size_t)r*nxv+x] - s); r2 += s * s; }
    printf("L=%d n=%d nz=%d c=%d inv %s rel %.2e\n", L, n, nz, c, rev ? "rev" : "fwd", track(std::sqrt(e2 / r2)));
  }
}
int main() {
  test<32>(32, 32, 2, 1); test<32>(30, 26, 2, 2); test<64>(64, 64, 2, 3); test<64>(40, 22, 1, 4); test<128>(128, 128, 2, 5); test<128>(96, 54, 3, 6); test<256>(256, 70, 2, 7);
  printf("worst %.3e\n", g_worst);
  return g_worst < 1e-5 ? 0 : 1;
}
