/*
 * Low-precision fluid kernels of the batched step (FP32 / FP16 / BF16
 * deviations, FP32 arithmetic; FMA contraction allowed, as in
 * lbib_fluid_lp.cu): instantiations of lbib_batch.cuh.
 */
#include "lbib_batch.cuh"
#include "lbib_batch_internal.h"

namespace lbib {

namespace {

template <typename T>
int rest(const BatchFluid& f) {
  const FluidParamsT<T>* P = static_cast<const FluidParamsT<T>*>(f.P);
  if (f.nrblk > 0) {
    if (f.par == 0) lbib_b_rows<T, 0><<<(unsigned)f.nrblk, 128, 0, f.stream>>>(P, f.rowyz, f.rblk, f.err);
    else lbib_b_rows<T, 1><<<(unsigned)f.nrblk, 128, 0, f.stream>>>(P, f.rowyz, f.rblk, f.err);
  }
  if (f.par == 0) lbib_b_forced<T, 0><<<f.grid_tiles, 64, 0, f.stream>>>(P, f.desc, f.list, f.count, f.tile_inst, f.err);
  else lbib_b_forced<T, 1><<<f.grid_tiles, 64, 0, f.stream>>>(P, f.desc, f.list, f.count, f.tile_inst, f.err);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename T, int V, int MINB>
int words(const BatchFluid& f, const int2* blk, long nblk) {
  if (nblk <= 0) return 0;
  const WordsParams<T>* WP = static_cast<const WordsParams<T>*>(f.WP);
  if (f.par == 0) lbib_b_words<T, V, 0, MINB><<<(unsigned)nblk, WTPB, 0, f.stream>>>(WP, blk, f.err);
  else lbib_b_words<T, V, 1, MINB><<<(unsigned)nblk, WTPB, 0, f.stream>>>(WP, blk, f.err);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename T>
int words_v(const BatchFluid& f, int v, const int2* blk, long nblk) {
  return with_variant<T>(v, [&](auto V, auto MINB) { return words<T, V, MINB>(f, blk, nblk); });
}

template <typename T>
int moments(const BatchFluid& f) {
  const FluidParamsT<T>* P = static_cast<const FluidParamsT<T>*>(f.P);
  if (f.par == 0)
    lbib_b_tile_moments<T, 0><<<f.grid_tiles, 64, 0, f.stream>>>(P, f.desc, f.list, f.count, f.tile_inst, f.Ftile, f.Utile, f.err);
  else
    lbib_b_tile_moments<T, 1><<<f.grid_tiles, 64, 0, f.stream>>>(P, f.desc, f.list, f.count, f.tile_inst, f.Ftile, f.Utile, f.err);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

int batch_fluid_rest_lp(const BatchFluid& f) {
  switch (LBIB_PREC_TYPE(f.prec)) {
    case LBIB_PREC_F32: return rest<float>(f);
    case LBIB_PREC_F16: return rest<__half>(f);
    case LBIB_PREC_BF16: return rest<__nv_bfloat16>(f);
    default: return -1;
  }
}

int batch_words_lp(const BatchFluid& f, int variant, const int2* blk, long nblk) {
  switch (LBIB_PREC_TYPE(f.prec)) {
    case LBIB_PREC_F32: return words_v<float>(f, variant, blk, nblk);
    case LBIB_PREC_F16: return words_v<__half>(f, variant, blk, nblk);
    case LBIB_PREC_BF16: return words_v<__nv_bfloat16>(f, variant, blk, nblk);
    default: return -1;
  }
}

int batch_variants_lp(int prec) { return word_variants(prec); }

int batch_variant_cells_lp(int prec, int variant) { return word_variant_cells(prec, variant); }

int batch_tile_moments_lp(const BatchFluid& f) {
  switch (LBIB_PREC_TYPE(f.prec)) {
    case LBIB_PREC_F32: return moments<float>(f);
    case LBIB_PREC_F16: return moments<__half>(f);
    case LBIB_PREC_BF16: return moments<__nv_bfloat16>(f);
    default: return -1;
  }
}

}  // namespace lbib
