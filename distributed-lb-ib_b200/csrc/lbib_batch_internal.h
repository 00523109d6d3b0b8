/*
 * Interface between the batched step's host code (lbib_batch.cu, FP64 and
 * the immersed boundary, compiled with -fmad=false) and its low-precision
 * fluid kernels (lbib_batch_lp.cu, contraction allowed).
 */
#ifndef LBIB_BATCH_INTERNAL_H
#define LBIB_BATCH_INTERNAL_H

#include <cuda_runtime_api.h>

namespace lbib {

struct BatchDesc;

/* One fluid launch set of a batch. */
struct BatchFluid {
  cudaStream_t stream;
  int prec;                /* LBIB_PREC_* storage type */
  int par;                 /* AA parity of this step */
  int B;
  const void* P;           /* FluidParamsT<T>[B] */
  const void* WP;          /* WordsParams<T>[B] */
  const BatchDesc* desc;
  const int2* rowyz;       /* generic rows (y, z), each problem's contiguous */
  const int4* rblk;        /* generic-row blocks: (problem, first row, rows, chunk) */
  long nrblk;
  const int2* xblk;        /* FP64 two-cell blocks: (problem, block) */
  long nxblk;
  const int* list;         /* touched tiles (global ids) */
  const int* count;
  const int* tile_inst;
  const double* Ftile;
  double* Utile;
  const int* err;
  int grid_tiles;          /* persistent grid for tile-list kernels */
};

/* Generic rows + forced cells (the word blocks, with the edge cells, are separate);
 * FP64: two-cell blocks + generic rows. */
int batch_fluid_rest_f64(const BatchFluid& f);
int batch_fluid_rest_lp(const BatchFluid& f);
/* Word-kernel blocks of one variant. */
int batch_words_lp(const BatchFluid& f, int variant, const int2* blk, long nblk);
int batch_variants_lp(int prec);
int batch_variant_cells_lp(int prec, int variant);   /* V of a variant */
/* Tile moments after the step (parity = the next step's). */
int batch_tile_moments_f64(const BatchFluid& f);
int batch_tile_moments_lp(const BatchFluid& f);

}  // namespace lbib

#endif
