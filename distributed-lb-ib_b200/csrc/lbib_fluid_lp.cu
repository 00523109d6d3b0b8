/*
 * Low-precision population storage: FP32, FP16 or BF16 deviations from a
 * fixed shift, with FP32 deviation-form arithmetic (moments, equilibrium,
 * BGK + Guo collision; Form<T> in lbib_fluid_kernels.cuh).  Same AA access
 * rules and reference boundary semantics as the FP64 path; compiled with FMA
 * contraction allowed, since these forms are judged by their error against
 * the FP64 solution, not by bits.  HBM bytes per lattice update: 152 (FP32),
 * 76 (FP16, BF16).
 *
 * Rows away from the walls (y in [3, ny-4], z in [3, min(nz-4, zin_hi)]) run
 * the word kernel of lbib_words.cuh; the cells x in {2, 3, nx-4, nx-3} of
 * those rows and the cells of forced tiles run the generic per-cell rules;
 * wall rows run the generic row kernel.  The word kernel comes in variants
 * (cells per thread, register budget) that lbdev_autotune chooses from.
 */
#include <stdint.h>
#include <stdlib.h>

#include "lbib_words.cuh"

extern "C" int lbdev_bulk_rows(const lbib_device* d, int* nrows_y, int* nrows_z);

using namespace lbib;

namespace {

template <typename T, int V, int PAR, int MINB>
__global__ void __launch_bounds__(WTPB, MINB) lbib_fluid_step_words(WordsParams<T> b) {
  const long first = (long)blockIdx.x * WTPB;
  if (b.pf > 0) words_prefetch<T, V, PAR>(b, blockIdx.x + b.pf);
  words_item<T, V, PAR>(b, first + threadIdx.x);
  /* the plane-adjacent cells x in {2, 3, nx-4, nx-3} of the rows whose first
     word this block holds, while their words are in the caches (their slots
     are theirs alone, so the order within the launch does not matter) */
  const long r0 = (first + b.gpr - 1) / b.gpr;
  long r1 = (first + WTPB + b.gpr - 1) / b.gpr;
  if (r1 > b.nrows) r1 = b.nrows;
  for (long i = threadIdx.x; i < 4 * (r1 - r0); i += WTPB) edge_cell<T, PAR>(b.p, b.nry, (int)(r0 + i / 4), (int)(i & 3));
}

/* Cells of this step's forced tiles inside the word kernel's range; a
 * persistent grid walks the tile list. */
template <typename T, int PAR>
__global__ void __launch_bounds__(64) lbib_forced_cells(FluidParamsT<T> p, const int* __restrict__ list,
                                                        const int* __restrict__ count, int zb) {
  const int n = *count;
  for (int i = blockIdx.x; i < n; i += gridDim.x) forced_cell<T, PAR>(p, list[i], threadIdx.x, zb);
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

template <typename T, int V, int MINB>
int launch_words(lbib_device* d, const FluidParamsT<T>& p) {
  WordsParams<T> b;
  b.p = p;
  int nry = 0, nrz = 0;
  if (!lbdev_bulk_rows(d, &nry, &nrz)) return 0;
  words_geometry(b, V, d->nx, nry, nrz);
  b.pf = (long)d->l2_pf * sm_count() * MINB;
  const long threads = b.nrows * b.gpr;
  const unsigned blocks = (unsigned)((threads + WTPB - 1) / WTPB);
  const int zb = 2 + nrz, c = d->cur;
  const unsigned fblocks = (unsigned)sm_count() * 8;
  if (d->parity == 0) {
    lbib_fluid_step_words<T, V, 0, MINB><<<blocks, WTPB, 0, d->stream>>>(b);
    lbib_forced_cells<T, 0><<<fblocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], zb);
  } else {
    lbib_fluid_step_words<T, V, 1, MINB><<<blocks, WTPB, 0, d->stream>>>(b);
    lbib_forced_cells<T, 1><<<fblocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], zb);
  }
  d->kernel_launches += 2;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename T>
int lp_step(lbib_device* d) {
  FluidParamsT<T> p = make_params_t<T>(d, d->steps == 0);
  if (launch_step_rows_t<T>(d, p)) return -2;
  if (!d->use_bulk) return 0;
  return with_variant<T>(d->lp_variant < 0 ? 0 : d->lp_variant,
                         [&](auto V, auto MINB) { return launch_words<T, V, MINB>(d, p); });
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

/* Word-kernel variants available for a precision (1 for FP64). */
extern "C" int lbdev_lp_variants(int prec) {
  return LBIB_PREC_TYPE(prec) == LBIB_PREC_F64 ? 1 : word_variants(prec);
}
