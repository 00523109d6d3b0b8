/*
 * Immersed-boundary kernels of one grid: thin wrappers over the device code
 * of lbib_ib.cuh (fiber forces, node preparation, the deterministic spread
 * as a per-tile gather, interpolation and move) and their launchers.
 * Compiled with -fmad=false: every expression keeps the reference's
 * operation order.
 */
#include "lbib_ib.cuh"

using namespace lbib;

namespace {

__global__ void lbib_fiber_forces(double* __restrict__ nodes, int R, int C, double bc, double sc, double sc2,
                                  double ds1, double ds2, int bend_bug) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R * C) return;
  fiber_forces_node(nodes, R, C, bc, sc, sc2, ds1, ds2, bend_bug, i);
}

/* The sheets whose fiber forces the node preparation computes as well
 * (n = 0: none; the forces then come from lbib_fiber_forces). */
constexpr int kFuseSheets = 4;
struct SheetForces {
  int n, bend_bug;
  lbib_sheet_dev s[kFuseSheets];
};

/* A block per 32-node chunk: warp p < 4 evaluates part p of the chunk's
 * nodes (node_prep_part); warp 0 also reduces the chunk's stencil box.  A
 * fifth warp, when the block has one, computes the nodes' fiber forces for
 * the sheets `sf` names (fiber_forces_node reads neighbours' positions and
 * writes the node's own force fields only, so it runs alongside). */
__global__ void __launch_bounds__(160) lbib_node_prep(double* __restrict__ nodes, long S, int nx, int ny, int nz,
                                                      int ntx, int nty, double* __restrict__ W, int* __restrict__ st,
                                                      int* __restrict__ tile_cnt, int* __restrict__ chunk_box, int* err,
                                                      int step, SheetForces sf) {
  const long i = (long)blockIdx.x * 32 + (threadIdx.x & 31);
  const int part = threadIdx.x >> 5;
  if (part == 4) {
    if (sf.n == 0 || i >= S) return;
    int k = 0;
    while (k + 1 < sf.n && i >= sf.s[k + 1].offset) ++k;
    const lbib_sheet_dev& h = sf.s[k];
    const long li = i - h.offset;
    if (li < (long)h.rows * h.cols)
      fiber_forces_node(nodes + h.offset * 12, h.rows, h.cols, h.bc, h.sc, h.sc2, h.ds1, h.ds2, sf.bend_bug, (int)li);
    return;
  }
  int b0 = INT_MAX, b1 = INT_MIN, b2 = INT_MAX, b3 = INT_MIN, b4 = INT_MAX, b5 = INT_MIN;
  if (i < S) node_prep_part(nodes, i, part, nx, ny, nz, ntx, nty, W, st, tile_cnt, err, step, b0, b1, b2, b3, b4, b5);
  if (part == 0) chunk_box_reduce(i, S, chunk_box, b0, b1, b2, b3, b4, b5);
}

/* Tiles of columns tx in [tlo, thi) only: the slot numbering covers every
 * touched tile (so that the moment tiles of x-slabs line up), but a slab
 * lists and gathers only the tiles its own fluid cells read. */
__global__ void lbib_pair_scatter(const int* __restrict__ st, long S, int ntx, int nty, int nx, int ny, int nz,
                                  int tlo, int thi, const int* __restrict__ slot, const int* __restrict__ slot_off,
                                  int* __restrict__ slot_cursor, int2* __restrict__ ent, const int* err) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (*(volatile const int*)err) return;   /* uniform: the whole warp returns */
  pair_scatter_warp(st, i, S, ntx, nty, nx, ny, nz, tlo, thi, slot, slot_off, slot_cursor, ent);
}

/* Every listed tile: from its entries (gather_tile_ent), or, with more
 * than kListCap nodes (a crumpled sheet), by scanning the node chunks in
 * order (gather_tile_scan). */
__global__ void __launch_bounds__(64) lbib_spread_gather(const double* __restrict__ nodes, const double* __restrict__ W,
                                                         const int* __restrict__ st, const int* __restrict__ chunk_box,
                                                         long S, long nchunks, const int* __restrict__ list,
                                                         const int* __restrict__ count, const int* __restrict__ slot_off,
                                                         const int* __restrict__ slot_len,
                                                         const int* __restrict__ slot_cursor,
                                                         const int2* __restrict__ ent, int ntx, int nty, int tlo,
                                                         int thi, double* __restrict__ Ftile, const int* err) {
  __shared__ union {
    GatherSmemE e;
    ScanSmem s;
  } sm;
  if (*(volatile const int*)err) return;
  const int n = *count;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int tile = list[it], tx = tile % ntx;
    if (tx < tlo || tx >= thi) continue;   /* uniform over the block */
    const int L = slot_len[it];
    if (L <= kListCap) {
      gather_tile_ent(sm.e, nodes, W, st, it, tile, L, slot_cursor[it], ent + slot_off[it], ntx, nty, Ftile);
    } else {
      __syncthreads();   /* the union's previous contents are no longer read */
      gather_tile_scan(sm.s, nodes, W, st, chunk_box, S, 0, nchunks, it, tile, ntx, nty, Ftile);
    }
  }
}

/* Nodes [i0, i1) of the concatenated sheets.  With `box` (an overlapped
 * step's next box), the box in tiles of the moved nodes' stencils is
 * reduced into it (block reduction, then six atomics per block). */
constexpr int kMoveTPB = 64;   /* two warps, each with its staged union box */

__global__ void __launch_bounds__(kMoveTPB) lbib_move_nodes(double* __restrict__ nodes, const double* __restrict__ W,
                                                            const int* __restrict__ st, long i0, long i1, int ntx,
                                                            int nty, const int* __restrict__ slot,
                                                            const double* __restrict__ Utile, double dt,
                                                            const int* err, int* __restrict__ box, int nx, int ny,
                                                            int nz) {
  __shared__ double sU[kMoveTPB / 32][3 * kMoveCap + kMoveTiles / 2];   /* + the staged tile slots */
  const long i = i0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < i1 && !*(volatile const int*)err;
  move_warp(nodes, W, st, i, live, ntx, nty, slot, Utile, dt, sU[threadIdx.x >> 5]);
  if (!box) return;
  int b[6] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, INT_MAX, INT_MIN};
  if (live) {
    const double* m = nodes + i * 12;
    if (stencil_inside(m[0], nx) && stencil_inside(m[1], ny) && stencil_inside(m[2], nz)) {
      const int is = stencil_start(m[0]), js = stencil_start(m[1]), ks = stencil_start(m[2]);
      b[0] = is >> 2; b[1] = (is + 3) >> 2; b[2] = js >> 2; b[3] = (js + 3) >> 2; b[4] = ks >> 2; b[5] = (ks + 3) >> 2;
    }
  }
  __shared__ int red[6][4];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    int v = b[k];
    for (int o = 16; o > 0; o >>= 1) {
      const int u = __shfl_xor_sync(0xffffffffu, v, o);
      v = (k & 1) ? max(v, u) : min(v, u);
    }
    if (lane == 0) red[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    const int k = threadIdx.x;
    int v = red[k][0];
    for (int j = 1; j < (int)(blockDim.x >> 5); ++j) v = (k & 1) ? max(v, red[k][j]) : min(v, red[k][j]);
    if ((k & 1) ? v != INT_MIN : v != INT_MAX) {
      if (k & 1) atomicMax(&box[k], v);
      else atomicMin(&box[k], v);
    }
  }
}

/* The box, in tiles, of all stencils of the current node positions (one
 * block): what an overlapped fluid step leaves to the cells kernel that
 * runs after the spread.  Nodes whose stencil leaves the grid are left out
 * (the spread reports them).  No valid node: an empty box. */
__global__ void __launch_bounds__(1024) lbib_stencil_box(const double* __restrict__ nodes, long S, int nx, int ny,
                                                         int nz, int* __restrict__ box) {
  __shared__ int red[6][32];
  int b0 = INT_MAX, b1 = INT_MIN, b2 = INT_MAX, b3 = INT_MIN, b4 = INT_MAX, b5 = INT_MIN;
  for (long i0 = threadIdx.x; i0 < S; i0 += 4L * blockDim.x) {
    double x[4][3];   /* four nodes' loads in flight before any is used */
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const long i = i0 + (long)u * blockDim.x;
      const double* m = nodes + (i < S ? i : 0) * 12;
      x[u][0] = i < S ? m[0] : -1.0; x[u][1] = m[1]; x[u][2] = m[2];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (!(stencil_inside(x[u][0], nx) && stencil_inside(x[u][1], ny) && stencil_inside(x[u][2], nz))) continue;
      const int is = stencil_start(x[u][0]), js = stencil_start(x[u][1]), ks = stencil_start(x[u][2]);
      b0 = min(b0, is); b1 = max(b1, is + 3);
      b2 = min(b2, js); b3 = max(b3, js + 3);
      b4 = min(b4, ks); b5 = max(b5, ks + 3);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    b0 = min(b0, __shfl_xor_sync(0xffffffffu, b0, o)); b1 = max(b1, __shfl_xor_sync(0xffffffffu, b1, o));
    b2 = min(b2, __shfl_xor_sync(0xffffffffu, b2, o)); b3 = max(b3, __shfl_xor_sync(0xffffffffu, b3, o));
    b4 = min(b4, __shfl_xor_sync(0xffffffffu, b4, o)); b5 = max(b5, __shfl_xor_sync(0xffffffffu, b5, o));
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (lane == 0) { red[0][w] = b0; red[1][w] = b1; red[2][w] = b2; red[3][w] = b3; red[4][w] = b4; red[5][w] = b5; }
  __syncthreads();
  if (w == 0) {
    b0 = lane < nw ? red[0][lane] : INT_MAX; b1 = lane < nw ? red[1][lane] : INT_MIN;
    b2 = lane < nw ? red[2][lane] : INT_MAX; b3 = lane < nw ? red[3][lane] : INT_MIN;
    b4 = lane < nw ? red[4][lane] : INT_MAX; b5 = lane < nw ? red[5][lane] : INT_MIN;
    for (int o = 16; o > 0; o >>= 1) {
      b0 = min(b0, __shfl_xor_sync(0xffffffffu, b0, o)); b1 = max(b1, __shfl_xor_sync(0xffffffffu, b1, o));
      b2 = min(b2, __shfl_xor_sync(0xffffffffu, b2, o)); b3 = max(b3, __shfl_xor_sync(0xffffffffu, b3, o));
      b4 = min(b4, __shfl_xor_sync(0xffffffffu, b4, o)); b5 = max(b5, __shfl_xor_sync(0xffffffffu, b5, o));
    }
    if (lane == 0) {
      if (b0 > b1) { box[0] = 1; box[1] = 0; box[2] = 1; box[3] = 0; box[4] = 1; box[5] = 0; }
      else { box[0] = b0 >> 2; box[1] = b1 >> 2; box[2] = b2 >> 2; box[3] = b3 >> 2; box[4] = b4 >> 2; box[5] = b5 >> 2; }
    }
  }
}

/* Dense copy of the spread force for getters: zero, then each touched tile
 * of columns tx in [tlo, thi) (the tiles this state gathered). */
__global__ void lbib_scatter_force(const int* __restrict__ list, const int* __restrict__ count,
                                   const double* __restrict__ Ftile, int nx, int ny, int nz, int ntx, int nty, int tlo,
                                   int thi, double* __restrict__ fx, double* __restrict__ fy, double* __restrict__ fz) {
  const int n = *count;
  const int cell = threadIdx.x;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int tile = list[it];
    const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
    if (tx < tlo || tx >= thi) continue;
    const int x = tx * 4 + (cell & 3), y = ty * 4 + ((cell >> 2) & 3), z = tz * 4 + (cell >> 4);
    if (x < nx && y < ny && z < nz) {
      const long idx = ((long)z * ny + y) * nx + x;
      const double* Ft = Ftile + (long)it * 192;
      fx[idx] = Ft[cell]; fy[idx] = Ft[64 + cell]; fz[idx] = Ft[128 + cell];
    }
  }
}

}  // namespace

extern "C" int lbdev_launch_fiber_forces(lbib_device* d, int k) {
  const lbib_sheet_dev* s = &d->sh[k];
  const int n = s->rows * s->cols;
  lbib_fiber_forces<<<(n + 127) / 128, 128, 0, d->stream>>>(d->nodes + s->offset * 12, s->rows, s->cols, s->bc,
                                                            s->sc, s->sc2, s->ds1, s->ds2,
                                                            (d->compat & 1) != 0);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int lbdev_launch_stencil_box(lbib_device* d) {
  lbib_stencil_box<<<1, 1024, 0, d->stream>>>(d->nodes, d->S, d->nx, d->ny, d->nz, d->box + 6 * d->box_cur);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* The fiber forces fold into the node preparation for up to kFuseSheets
 * sheets: lbdev_launch_spread computes them when d->fuse_forces is set. */
extern "C" int lbdev_can_fuse_forces(const lbib_device* d) { return d->nsheets <= kFuseSheets; }

extern "C" int lbdev_launch_spread(lbib_device* d, int step) {
  const int c = d->cur;
  cudaStream_t st = d->stream;
  /* tile_cnt is left at zero and tile_slot[c] fully rewritten by the
     compaction, so the step needs no clearing pass */
  const long S = d->S;
  const unsigned nb = (unsigned)((S + 127) / 128);
  SheetForces sf;
  sf.n = 0;
  sf.bend_bug = (d->compat & 1) != 0;
  if (d->fuse_forces && d->nsheets <= kFuseSheets) {
    sf.n = d->nsheets;
    for (int k = 0; k < d->nsheets; ++k) sf.s[k] = d->sh[k];
  }
  lbib_node_prep<<<(unsigned)d->nchunks, sf.n ? 160 : 128, 0, st>>>(d->nodes, S, d->nx, d->ny, d->nz, d->ntx, d->nty,
                                                                    d->W, d->st, d->tile_cnt, d->chunk_box, d->err,
                                                                    step, sf);
  const unsigned nblk = (unsigned)((d->ntiles + kScanBlock - 1) / kScanBlock);
  if (d->scan_state && d->ntiles < (1L << 22) && 8 * S < (1L << 31)) {
    d->scan_tag = d->scan_tag % 255u + 1u;
    const unsigned nb1 = (unsigned)((d->ntiles + kScanBlock * kOnepassTiles - 1) / (kScanBlock * kOnepassTiles));
    lbib_compact_onepass<<<nb1, kScanBlock, 0, st>>>(d->tile_cnt, d->ntiles, (int)nb1, d->scan_state, d->scan_tag,
                                                      d->tile_list[c], d->tile_slot[c], d->slot_off, d->slot_len,
                                                      d->slot_cursor, d->tile_count[c], d->err);
    d->kernel_launches -= 2;
  } else {
    int* block_tiles = d->scan_tmp;
    int* block_pairs = d->scan_tmp + nblk + 1;
    lbib_compact_count<<<nblk, kScanBlock, 0, st>>>(d->tile_cnt, d->ntiles, block_tiles, block_pairs);
    lbib_compact_scan<<<1, kScanBlock, 0, st>>>(block_tiles, block_pairs, (int)nblk, d->tile_count[c]);
    lbib_compact_write<<<nblk, kScanBlock, 0, st>>>(d->tile_cnt, d->ntiles, block_tiles, block_pairs,
                                                    d->tile_list[c], d->tile_slot[c], d->slot_off, d->slot_len,
                                                    d->slot_cursor);
  }
  /* an x-slab lists and gathers the tiles of its own columns only */
  const int tlo = d->x_lo / 4, thi = (d->x_hi + 3) / 4;
  int2* ent = reinterpret_cast<int2*>(d->pair_node);
  lbib_pair_scatter<<<nb, 128, 0, st>>>(d->st, S, d->ntx, d->nty, d->nx, d->ny, d->nz, tlo, thi, d->tile_slot[c],
                                        d->slot_off, d->slot_cursor, ent, d->err);
  lbib_spread_gather<<<148 * 12, 64, 0, st>>>(d->nodes, d->W, d->st, d->chunk_box, S, d->nchunks, d->tile_list[c],
                                              d->tile_count[c], d->slot_off, d->slot_len, d->slot_cursor, ent,
                                              d->ntx, d->nty, tlo, thi, d->Ftile[c], d->err);
  d->kernel_launches += 6;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* moveFiberSheet over all nodes; with the pinned-row option (no reference
 * counterpart) row 0 of every sheet is left where it is: one launch per
 * sheet over its rows 1 .. rows-1. */
extern "C" int lbdev_launch_move(lbib_device* d) {
  const int c = d->cur;
  if (!(d->compat & LBIB_OPT_PIN_ROW0)) {
    const unsigned nb = (unsigned)((d->S + kMoveTPB - 1) / kMoveTPB);
    lbib_move_nodes<<<nb, kMoveTPB, 0, d->stream>>>(d->nodes, d->W, d->st, 0, d->S, d->ntx, d->nty,
                                                    d->tile_slot[c], d->Utile[c], (double)d->dt, d->err,
                                                    d->box_next, d->nx, d->ny, d->nz);
    d->kernel_launches++;
  } else {
    for (int k = 0; k < d->nsheets; ++k) {
      const long i0 = d->sh[k].offset + d->sh[k].cols, i1 = d->sh[k].offset + (long)d->sh[k].rows * d->sh[k].cols;
      const unsigned nb = (unsigned)((i1 - i0 + kMoveTPB - 1) / kMoveTPB);
      lbib_move_nodes<<<nb, kMoveTPB, 0, d->stream>>>(d->nodes, d->W, d->st, i0, i1, d->ntx, d->nty,
                                                      d->tile_slot[c], d->Utile[c], (double)d->dt, d->err, nullptr,
                                                      d->nx, d->ny, d->nz);
      d->kernel_launches++;
    }
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int lbdev_launch_scatter_force(lbib_device* d, double* fx, double* fy, double* fz) {
  const int c = d->cur;
  lbib_scatter_force<<<148 * 8, 64, 0, d->stream>>>(d->tile_list[c], d->tile_count[c], d->Ftile[c], d->nx, d->ny,
                                                     d->nz, d->ntx, d->nty, d->x_lo / 4, (d->x_hi + 3) / 4, fx, fy,
                                                     fz);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
