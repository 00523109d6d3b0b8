/*
 * Batched fluid kernels: many independent problems of uneven size advanced
 * by one launch per stage.
 *
 * Every problem keeps its own populations, tables and parameters (a
 * FluidParamsT<T> per problem in device memory, whose pointers reach into
 * the batch's pools); its tiles are a slice [tile0, tile0 + ntiles) of one
 * global tile space, so one touched-tile list, one slot space and one
 * compaction serve the whole batch.  Work is enumerated across problems:
 *   rows     blocks of 128 cells over the rows the generic kernel takes,
 *            each problem's rows laid end to end;
 *   pairs    (FP64) blocks of 128 cell pairs of the two-cell kernel;
 *   words    blocks of the word kernel, (problem, block within problem);
 *            (the word blocks also step the cells x in {2, 3, nx-4, nx-3}
 *            of the rows whose first word they hold);
 *   tiles    the global touched-tile list, tile -> problem by a table.
 * A problem whose error word is set (a fiber stencil left its grid) is
 * skipped by every kernel from then on; the others continue.
 *
 * The per-cell arithmetic is the one-grid code (step_cell, x2_pair,
 * words_item, tile_moments_cell), so a problem advanced in a batch gets the same
 * numbers as the same problem on its own.
 */
#ifndef LBIB_BATCH_CUH
#define LBIB_BATCH_CUH

#include "lbib_words.cuh"

namespace lbib {

/* What the node- and tile-level kernels need of a problem. */
struct BatchDesc {
  int nx, ny, nz, ntx, nty;
  int rows, cols;          /* its one sheet */
  int bulk;                /* bulk rows run the word kernel */
  int pinned;              /* row 0 of the sheet stays put */
  long tile0, ntiles;      /* slice of the global tile space */
  long node0, S;           /* nodes [node0, node0 + S); node0 % 32 == 0 */
  double bc, sc, sc2, ds1, ds2, dt;
};

/* Copy a parameter struct into shared memory with the whole block. */
template <typename S>
__device__ __forceinline__ void block_copy(S& dst, const S* __restrict__ src) {
  static_assert(sizeof(S) % 4 == 0, "word copy");
  const uint32_t* a = reinterpret_cast<const uint32_t*>(src);
  uint32_t* b = reinterpret_cast<uint32_t*>(&dst);
  for (int i = threadIdx.x; i < (int)(sizeof(S) / 4); i += blockDim.x) b[i] = a[i];
  __syncthreads();
}

/* Generic rows: a block per 128 cells of a problem's rows, the rows of
 * problem k laid end to end (cell c of the item: row c / (nx-4), x = 2 +
 * c % (nx-4)), so small grids fill their blocks.  Item m = (problem, first
 * row in rowyz, rows of the problem, chunk). */
template <typename T, int PAR>
__global__ void __launch_bounds__(128) lbib_b_rows(const FluidParamsT<T>* __restrict__ P, const int2* __restrict__ rowyz,
                                                   const int4* __restrict__ rblk, const int* __restrict__ err) {
  __shared__ __align__(16) FluidParamsT<T> sp;
  const int4 m = rblk[blockIdx.x];
  if (err[2 * m.x]) return;
  block_copy(sp, P + m.x);
  const int w = sp.nx - 4;
  const int c = m.w * 128 + threadIdx.x;
  const int r = c / w;
  if (r >= m.z) return;
  const int2 yz = rowyz[m.y + r];
  step_cell<T, PAR>(sp, 2 + c % w, yz.x, yz.y);
}

/* Word kernel over the blocks of all problems that run it.  A block also
 * steps the plane-adjacent cells x in {2, 3, nx-4, nx-3} of the rows whose
 * first word it holds (generic per-cell rules), right after their words
 * went through the caches: a launch of their own re-read each of their
 * 2-byte populations from DRAM as a whole sector.  The slots those cells
 * read and write are theirs alone (AA), so the order within the launch
 * does not matter. */
template <typename T, int V, int PAR, int MINB>
__global__ void __launch_bounds__(WTPB, MINB) lbib_b_words(const WordsParams<T>* __restrict__ WP,
                                                           const int2* __restrict__ blk, const int* __restrict__ err) {
  __shared__ __align__(16) WordsParams<T> sb;
  const int2 m = blk[blockIdx.x];
  if (err[2 * m.x]) return;
  block_copy(sb, WP + m.x);
  const long first = (long)m.y * WTPB;
  words_item<T, V, PAR>(sb, first + threadIdx.x);
  const long r0 = fdiv((unsigned)(first + sb.gpr - 1), sb.dgpr);
  long r1 = fdiv((unsigned)(first + WTPB + sb.gpr - 1), sb.dgpr);
  if (r1 > sb.nrows) r1 = sb.nrows;
  for (long i = threadIdx.x; i < 4 * (r1 - r0); i += WTPB) edge_cell<T, PAR>(sb.p, sb.nry, (int)(r0 + i / 4), (int)(i & 3));
}

/* Cells of forced tiles in the word kernel's range, over the global list. */
template <typename T, int PAR>
__global__ void __launch_bounds__(64) lbib_b_forced(const FluidParamsT<T>* __restrict__ P,
                                                    const BatchDesc* __restrict__ D, const int* __restrict__ list,
                                                    const int* __restrict__ count, const int* __restrict__ tile_inst,
                                                    const int* __restrict__ err) {
  const int n = *count;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int tile = list[i];
    const int k = tile_inst[tile];
    if (err[2 * k] || !D[k].bulk) continue;
    const FluidParamsT<T>& p = P[k];
    const int zb = min(p.nz - 4, p.zin_hi);
    forced_cell<T, PAR>(p, (int)(tile - D[k].tile0), threadIdx.x, zb);
  }
}

/* (rho, u) of the touched tiles, over the global list. */
template <typename T, int PAR>
__global__ void lbib_b_tile_moments(const FluidParamsT<T>* __restrict__ P, const BatchDesc* __restrict__ D,
                                    const int* __restrict__ list, const int* __restrict__ count,
                                    const int* __restrict__ tile_inst, const double* __restrict__ Ftile,
                                    double* __restrict__ Utile, const int* __restrict__ err) {
  const int n = *count;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int tile = list[i];
    const int k = tile_inst[tile];
    if (err[2 * k]) continue;
    tile_moments_cell<T, PAR>(P[k], (int)(tile - D[k].tile0), i, threadIdx.x, Ftile, Utile);
  }
}

}  // namespace lbib

#endif
