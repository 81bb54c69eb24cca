// H-LU and triangular H-solve (src/hlu.jl:227-562).
#include "hm_internal.h"
#include "hm_lowrank.cuh"

namespace hm {

struct LuState {
  int dummy = 0;
};

int lu_factor(hm_handle* h) {
  (void)h;
  return fail(HM_ERR_UNSUPPORTED, "H-LU is not built yet");
}
int lu_solve_device(hm_handle* h, const double*, double*, int64_t, cudaStream_t) {
  (void)h;
  return fail(HM_ERR_UNSUPPORTED, "H-solve is not built yet");
}
int lu_perm(const hm_handle*, int64_t*) { return fail(HM_ERR_UNSUPPORTED, "H-LU is not built yet"); }
int lu_to_dense(const hm_handle*, double*) { return fail(HM_ERR_UNSUPPORTED, "H-LU is not built yet"); }
void lu_free(hm_handle* h) {
  delete h->lu;
  h->lu = nullptr;
}
int lu_copy(const hm_handle* src, hm_handle* dst) {
  (void)src;
  (void)dst;
  return HM_OK;
}

}  // namespace hm
