// Host emulation of the ESSE y-z plane kernel (esse_yz.cuh) against a
// direct 2D DFT, kernel product and inverse in double; both thread orders.
#include <cstdio>
#include <cmath>
#include <vector>
#include <random>
#include <complex>
struct D3 { int x, y, z; }; static D3 threadIdx, blockDim;
static inline void __syncthreads() {}
#include <cuda_runtime.h>
#include "esse_yz.cuh"
using namespace irlcu;
static double g_worst = 0;
using cd = std::complex<double>;
template <class F> void for_threads(bool rev, F f) { if (rev) for (int t = EY_NT - 1; t >= 0; --t) f(t); else for (int t = 0; t < EY_NT; ++t) f(t); }

template <int L> void test(int nyv, int nzv, int nt, unsigned seed) {
  using D = EYz<L>;
  std::mt19937 rng(seed); std::uniform_real_distribution<float> U(-1, 1);
  std::vector<float2> A((size_t)nyv * nzv), Kn[2], Kp[2];
  for (auto &v : A) v = make_float2(U(rng), U(rng));
  for (int t = 0; t < 2; ++t) { Kn[t].resize(L * L); Kp[t].resize(L * L); for (auto &v : Kn[t]) v = make_float2(U(rng), U(rng)); }
  for (int t = 0; t < 2; ++t) for (int ky = 0; ky < L; ++ky) for (int kz = 0; kz < L; ++kz) Kp[t][ky * L + kz / D::N1 + D::N2 * (kz % D::N1)] = Kn[t][ky * L + kz];
  std::vector<float2> tw(L); for (int m = 0; m < L; ++m) tw[m] = make_float2((float)cos(-2*M_PI*m/L), (float)sin(-2*M_PI*m/L));
  // reference
  std::vector<cd> Ah((size_t)L * L);
  { std::vector<cd> T((size_t)nyv * L);
    for (int y = 0; y < nyv; ++y) for (int kz = 0; kz < L; ++kz) { cd s = 0; for (int z = 0; z < nzv; ++z) s += cd(A[y*nzv+z].x, A[y*nzv+z].y) * std::polar(1.0, -2*M_PI*(double)z*kz/L); T[y*L+kz] = s; }
    for (int ky = 0; ky < L; ++ky) for (int kz = 0; kz < L; ++kz) { cd s = 0; for (int y = 0; y < nyv; ++y) s += T[y*L+kz] * std::polar(1.0, -2*M_PI*(double)y*ky/L); Ah[ky*L+kz] = s; } }
  std::vector<cd> ref[2];
  for (int t = 0; t < nt; ++t) {
    std::vector<cd> P((size_t)L * L), T((size_t)L * nzv);
    for (int i = 0; i < L * L; ++i) P[i] = Ah[i] * cd(Kn[t][i].x, Kn[t][i].y);
    for (int ky = 0; ky < L; ++ky) for (int z = 0; z < nzv; ++z) { cd s = 0; for (int kz = 0; kz < L; ++kz) s += P[ky*L+kz] * std::polar(1.0, 2*M_PI*(double)z*kz/L); T[ky*nzv+z] = s; }
    ref[t].resize((size_t)nyv * nzv);
    for (int y = 0; y < nyv; ++y) for (int z = 0; z < nzv; ++z) { cd s = 0; for (int ky = 0; ky < L; ++ky) s += T[ky*nzv+z] * std::polar(1.0, 2*M_PI*(double)y*ky/L); ref[t][y*nzv+z] = s; }
  }
  for (int rev = 0; rev < 2; ++rev) {
    std::vector<float2> F(D::F_ELEMS, make_float2(NAN, NAN)), C(2 * D::C_ELEMS, make_float2(NAN, NAN));
    std::vector<float2> D0((size_t)nyv * nzv, make_float2(NAN, NAN)), D1(D0);
    for_threads(rev, [&](int t) { ey_load<L>(t, F.data(), A.data(), nyv, nzv); });
    for_threads(rev, [&](int t) { ey_z_fwd_a<L>(t, F.data(), tw.data(), nyv, nzv); });
    for_threads(rev, [&](int t) { ey_z_fwd_b<L>(t, F.data(), nyv); });
    for_threads(rev, [&](int t) { ey_y_fwd_a<L>(t, F.data(), tw.data(), nyv); });
    for (int z0 = 0; z0 < L; z0 += EY_ZC) {
      for_threads(rev, [&](int t) { ey_y_mid<L>(t, F.data(), C.data(), tw.data(), Kp[0].data(), Kp[1].data(), nt, z0); });
      for_threads(rev, [&](int t) { ey_y_inv_c<L>(t, F.data(), C.data(), nt, nyv, z0); });
    }
    for_threads(rev, [&](int t) { ey_z_inv_b<L>(t, F.data(), tw.data(), nt * nyv); });
    for_threads(rev, [&](int t) { ey_z_inv_c<L>(t, F.data(), nt * nyv, nzv); });
    for_threads(rev, [&](int t) { ey_store<L>(t, F.data(), D0.data(), D1.data(), nt, nyv, nzv); });
    for (int t = 0; t < nt; ++t) {
      double e2 = 0, r2 = 0; const auto &Dt = t ? D1 : D0;
      for (size_t i = 0; i < ref[t].size(); ++i) { cd g(Dt[i].x, Dt[i].y); e2 += std::norm(g - ref[t][i]); r2 += std::norm(ref[t][i]); }
      const double rel = std::sqrt(e2 / r2);
      if (!(rel <= g_worst)) g_worst = rel;
      printf("L=%3d nyv=%3d nzv=%3d nt=%d term %d %s: rel %.2e\n", L, nyv, nzv, nt, t, rev ? "rev" : "fwd", rel);
    }
  }
}
int main() {
  test<32>(16, 16, 2, 1); test<32>(13, 9, 1, 2);
  test<64>(32, 32, 2, 3); test<64>(20, 31, 2, 4);
  test<128>(64, 64, 2, 5); test<128>(50, 61, 1, 6);
  printf("worst %.3e\n", g_worst);
  return g_worst < 1e-5 ? 0 : 1;
}
