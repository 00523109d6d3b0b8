/*
 * FP64 fluid kernels (the drop-in path) and the dispatch of every fluid
 * launch by population precision.  Compiled with -fmad=false: the FP64
 * instantiation keeps the reference's rounding (see lbib_lattice.cuh).
 * The low-precision instantiations live in lbib_fluid_lp.cu.
 */
#include "lbib_fluid_kernels.cuh"

using namespace lbib;

extern "C" {
int lbdev_launch_fluid_bulk(lbib_device* d, const void* fluid_params);
int lbdev_lp_fluid_step(lbib_device* d);
int lbdev_lp_tile_moments(lbib_device* d);
int lbdev_lp_box_cells(lbib_device* d);
int lbdev_lp_field_moments(lbib_device* d, double* rho, double* ux, double* uy, double* uz);
int lbdev_lp_gather_df1(lbib_device* d, double* out);
int lbdev_lp_init(lbib_device* d, int what);
int lbdev_lp_sums(lbib_device* d, double* part, double* out);
}

/* One fused step.  FP64: the generic kernel over d->rows (all rows of I, or
 * only those next to the walls when the two-cell kernel takes the others).
 * In box mode (lbdev_step's overlapped step) these launches go to
 * d->fluid_stream and skip the box's tiles; the step is completed by
 * lbdev_launch_box_cells, which flips the parity. */
extern "C" int lbdev_launch_fluid_step(lbib_device* d) {
  if (LBIB_PREC_TYPE(d->prec) != LBIB_PREC_F64) {
    if (lbdev_lp_fluid_step(d)) return -2;
  } else {
    FluidParams p = make_params_t<double>(d, d->steps == 0);
    if (launch_step_rows_t<double>(d, p)) return -2;
    if (d->use_bulk && lbdev_launch_fluid_bulk(d, &p)) return -2;
  }
  if (!d->box_mode) {
    d->parity ^= 1;
    d->steps++;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* Box mode: the cells of the box's tiles (on d->stream, after the spread
 * and the bulk launches), then the step is complete. */
extern "C" int lbdev_launch_box_cells(lbib_device* d) {
  int rc;
  if (LBIB_PREC_TYPE(d->prec) != LBIB_PREC_F64) {
    rc = lbdev_lp_box_cells(d);
  } else {
    FluidParams p = make_params_t<double>(d, d->steps == 0);
    rc = launch_box_cells_t<double>(d, p);
  }
  if (rc) return -2;
  d->parity ^= 1;
  d->steps++;
  return 0;
}

extern "C" int lbdev_launch_tile_moments(lbib_device* d) {
  if (LBIB_PREC_TYPE(d->prec) != LBIB_PREC_F64) return lbdev_lp_tile_moments(d);
  return launch_tile_moments_t<double>(d);
}

extern "C" int lbdev_launch_field_moments(lbib_device* d, double* rho, double* ux, double* uy, double* uz) {
  if (LBIB_PREC_TYPE(d->prec) != LBIB_PREC_F64) return lbdev_lp_field_moments(d, rho, ux, uy, uz);
  return launch_field_moments_t<double>(d, rho, ux, uy, uz);
}

extern "C" int lbdev_launch_gather_df1(lbib_device* d, double* out) {
  if (LBIB_PREC_TYPE(d->prec) != LBIB_PREC_F64) return lbdev_lp_gather_df1(d, out);
  return launch_gather_df1_t<double>(d, out);
}

/* what = 0: populations (init_eqlbrmdistrfuncDF0 + init_df1); 1: the
 * inlet/outlet planes (init_df_inout). */
extern "C" int lbdev_launch_init(lbib_device* d, int what) {
  if (LBIB_PREC_TYPE(d->prec) != LBIB_PREC_F64) return lbdev_lp_init(d, what);
  return launch_init_t<double>(d, what);
}

extern "C" int lbdev_launch_sums(lbib_device* d, double* part, double* out) {
  if (LBIB_PREC_TYPE(d->prec) != LBIB_PREC_F64) return lbdev_lp_sums(d, part, out);
  return launch_sums_t<double>(d, part, out);
}
