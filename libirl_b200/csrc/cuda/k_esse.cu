// k_esse.cu -- ESSE effective scatter source (placeholder until the FFT
// kernels land; every call reports that the scatter model is unavailable).
#include "irlcu_internal.cuh"

namespace irlcu {

int esse_setup(Ctx &c, const irlcu_esse *e) {
  (void)c;
  (void)e;
  return set_error(IRLCU_EARG, "ESSE scatter modelling is not available in this build");
}

int launch_esse(Ctx &c, const float *rot, const int *dviews, int nv, float primary, float *src) {
  (void)c; (void)rot; (void)dviews; (void)nv; (void)primary; (void)src;
  return set_error(IRLCU_EARG, "ESSE scatter modelling is not available in this build");
}

void esse_free(Ctx &c) { (void)c; }

}  // namespace irlcu

extern "C" int irlcu_set_esse(const irlcu_esse *e) {
  if (!irlcu::g_ctx) return irlcu::set_error(IRLCU_ESTATE, "irlcu_init has not been called");
  return irlcu::esse_setup(*irlcu::g_ctx, e);
}
