// k_osem.cu -- per-view OSEM projection-space kernels of libirl_b200.
//
//  * ratio epilogue (osemrecon.c:727-820): time/sensitivity scaling of the
//    calculated projection, stored-scatter add or refresh, additive scatter
//    estimate, SetNonMeasuredBinsToZero, the measured/calculated ratio with
//    its 1e-20 guard and the ViewTime scaling before backprojection;
//  * norm masks (osemrecon.c:290-295): SetMeasuredPrjBinsToOne times
//    ViewTime.
// Every operation rounds like libirl's float C code.
#include "irlcu_internal.cuh"

namespace irlcu {

// colmask bits: 1 = column measured (ratio), 2 = column set by the norm mask
__global__ void k_ratio(const float *__restrict__ calc, const float *__restrict__ calc_nosrf,
                        const int *__restrict__ views, const irlcu_view_parm *__restrict__ vp,
                        const float *__restrict__ meas_all, const float *__restrict__ scatest,
                        float *__restrict__ prjscat, const unsigned char *__restrict__ colmask, int nv,
                        int n, int nz, int use_scatest, float *__restrict__ ratio) {
  const size_t pln = (size_t)nz * n;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)nv * pln) return;
  const int bv = (int)(e / pln);
  const size_t i = e - (size_t)bv * pln;
  const int x = (int)(i % n);
  const int view = views[bv];
  const irlcu_view_parm p = vp[bv];
  const float vts = __fmul_rn(p.view_time, p.sensitivity);
  float c = __fmul_rn(calc[e], vts);
  const size_t gi = (size_t)view * pln + i;
  if (p.scat_mode == 1) {
    c = __fadd_rn(c, prjscat[gi]);
  } else if (p.scat_mode == 2) {
    prjscat[gi] = __fsub_rn(c, __fmul_rn(calc_nosrf[e], p.view_time));
  }
  if (use_scatest) c = __fadd_rn(c, scatest[gi]);
  const float m = meas_all[gi];
  // libirl passes the projection base (view 0) as the "measured" array of
  // SetNonMeasuredBinsToZero (osemrecon.c:802-803); measured data are
  // clamped at zero beforehand, so the test only matters for fidelity
  if (!(colmask[(size_t)view * n + x] & 1) || meas_all[i] < 0.f) c = 0.f;
  const float r = ((double)c > 1e-20) ? __fdiv_rn(m, c) : 0.f;
  ratio[e] = __fmul_rn(r, p.view_time);
}

int launch_ratio(const Ctx &c, const float *calc, const float *calc_nosrf, const int *dviews,
                 const irlcu_view_parm *dvp, int nv, int use_scatest, float *ratio) {
  const size_t tot = (size_t)nv * c.pln;
  k_ratio<<<(unsigned)((tot + 255) / 256), 256, 0, c.st>>>(calc, calc_nosrf, dviews, dvp, c.prj, c.scatest,
                                                            c.prjscat, c.colmask, nv, c.n, c.nz, use_scatest,
                                                            ratio);
  CU_LAUNCHED();
  return IRLCU_OK;
}

__global__ void k_norm_planes(const int *__restrict__ views, const float *__restrict__ vt,
                              const float *__restrict__ meas_all, const unsigned char *__restrict__ colmask,
                              int nv, int n, int nz, float *__restrict__ planes) {
  const size_t pln = (size_t)nz * n;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)nv * pln) return;
  const int bv = (int)(e / pln);
  const size_t i = e - (size_t)bv * pln;
  const int x = (int)(i % n);
  const int view = views[bv];
  const float m = meas_all[(size_t)view * pln + i];
  const float one = ((colmask[(size_t)view * n + x] & 2) && m >= 0.f) ? 1.f : 0.f;
  planes[e] = __fmul_rn(one, vt[bv]);
}

int launch_norm_planes(const Ctx &c, const int *dviews, const float *vt_dev, int nv,
                       const unsigned char *normcols, float *planes) {
  (void)normcols;
  const size_t tot = (size_t)nv * c.pln;
  k_norm_planes<<<(unsigned)((tot + 255) / 256), 256, 0, c.st>>>(dviews, vt_dev, c.prj, c.colmask, nv, c.n, c.nz,
                                                                  planes);
  CU_LAUNCHED();
  return IRLCU_OK;
}

}  // namespace irlcu
