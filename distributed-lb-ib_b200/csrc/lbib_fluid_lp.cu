/*
 * Low-precision population storage: FP32, and FP16 / BF16 holding the
 * shifted deviation f - w_q, all with FP32 arithmetic (moments, equilibrium,
 * BGK + Guo collision).  Same AA access rules and reference boundary
 * semantics as the FP64 path (the kernels are the templates of
 * lbib_fluid_kernels.cuh); compiled with FMA contraction allowed, since these
 * forms are judged by their error against the FP64 solution, not by bits.
 * HBM bytes per fluid cell: 152 (FP32), 76 (FP16, BF16).
 */
#include "lbib_fluid_kernels.cuh"

using namespace lbib;

namespace {

template <typename T>
int lp_step(lbib_device* d) {
  FluidParamsT<T> p = make_params_t<T>(d, d->steps == 0);
  return launch_step_rows_t<T>(d, p);
}

}  // namespace

extern "C" int lbdev_lp_fluid_step(lbib_device* d) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return lp_step<float>(d);
    case LBIB_PREC_F16: return lp_step<__half>(d);
    case LBIB_PREC_BF16: return lp_step<__nv_bfloat16>(d);
    default: return -1;
  }
}

extern "C" int lbdev_lp_tile_moments(lbib_device* d) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return launch_tile_moments_t<float>(d);
    case LBIB_PREC_F16: return launch_tile_moments_t<__half>(d);
    case LBIB_PREC_BF16: return launch_tile_moments_t<__nv_bfloat16>(d);
    default: return -1;
  }
}

extern "C" int lbdev_lp_field_moments(lbib_device* d, double* rho, double* ux, double* uy, double* uz) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return launch_field_moments_t<float>(d, rho, ux, uy, uz);
    case LBIB_PREC_F16: return launch_field_moments_t<__half>(d, rho, ux, uy, uz);
    case LBIB_PREC_BF16: return launch_field_moments_t<__nv_bfloat16>(d, rho, ux, uy, uz);
    default: return -1;
  }
}

extern "C" int lbdev_lp_gather_df1(lbib_device* d, double* out) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return launch_gather_df1_t<float>(d, out);
    case LBIB_PREC_F16: return launch_gather_df1_t<__half>(d, out);
    case LBIB_PREC_BF16: return launch_gather_df1_t<__nv_bfloat16>(d, out);
    default: return -1;
  }
}

extern "C" int lbdev_lp_init(lbib_device* d, int what) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return launch_init_t<float>(d, what);
    case LBIB_PREC_F16: return launch_init_t<__half>(d, what);
    case LBIB_PREC_BF16: return launch_init_t<__nv_bfloat16>(d, what);
    default: return -1;
  }
}

extern "C" int lbdev_lp_sums(lbib_device* d, double* part, double* out) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return launch_sums_t<float>(d, part, out);
    case LBIB_PREC_F16: return launch_sums_t<__half>(d, part, out);
    case LBIB_PREC_BF16: return launch_sums_t<__nv_bfloat16>(d, part, out);
    default: return -1;
  }
}
