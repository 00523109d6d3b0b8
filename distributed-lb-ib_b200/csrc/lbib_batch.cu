/*
 * Batched step: many independent LBM-IB problems of uneven size (each with
 * its own lattice, physics and one fiber sheet) advanced together, one
 * launch per stage for the whole batch, the step captured once as a CUDA
 * graph and replayed.  No reference counterpart: the reference runs one
 * problem per process.
 *
 * Layout: per problem its populations, inlet/outlet tables and parameters
 * (a host-only lbib_device "shadow" whose pointers reach into the batch's
 * pools, so the one-grid launch helpers and getters work on it); the tiles
 * of all problems form one global tile space and the sheets one node array
 * (each problem's nodes start at a multiple of 32), so node preparation,
 * compaction, pair lists, gather and move run once for the batch.  Per
 * problem error words: a problem whose sheet leaves its grid stops, the
 * others go on.
 *
 * The FP64 kernels (IB, FP64 fluid) live here with -fmad=false, so a problem
 * in an FP64 batch gets the same bits as on its own; the low-precision fluid
 * kernels are in lbib_batch_lp.cu.
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "lbib_batch.cuh"
#include "lbib_batch_internal.h"
#include "lbib_ib.cuh"
#include "lbib_x2.cuh"

extern "C" {
int lbdev_bulk_rows(const lbib_device* d, int* nrows_y, int* nrows_z);
int lbdev_launch_init(lbib_device* d, int what);
}

using namespace lbib;

#define CK(call)                          \
  do {                                    \
    if ((call) != cudaSuccess) return -2; \
  } while (0)

/* ------------------------------------------------------------ kernels */
namespace {

__global__ void lbib_b_forces(double* __restrict__ nodes, const int* __restrict__ node_inst,
                              const BatchDesc* __restrict__ D, const int* __restrict__ err, long SP, int bend_bug) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= SP) return;
  const int k = node_inst[i];
  if (k < 0 || err[2 * k]) return;
  const BatchDesc& d = D[k];
  fiber_forces_node(nodes + d.node0 * 12, d.rows, d.cols, d.bc, d.sc, d.sc2, d.ds1, d.ds2, bend_bug,
                    (int)(i - d.node0));
}

/* step_no: the batch's device step counter (graph replays see the live
 * value), 1 for the first step. */
__global__ void lbib_b_node_prep(const double* __restrict__ nodes, const int* __restrict__ node_inst,
                                 const BatchDesc* __restrict__ D, double* __restrict__ W, int* __restrict__ st,
                                 int* __restrict__ tile_cnt, int* __restrict__ chunk_box, int* err, long SP,
                                 const int* __restrict__ step_no) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int step = *step_no;
  int b0 = INT_MAX, b1 = INT_MIN, b2 = INT_MAX, b3 = INT_MIN, b4 = INT_MAX, b5 = INT_MIN;
  const int k = i < SP ? node_inst[i] : -1;
  if (k >= 0 && !err[2 * k]) {
    const BatchDesc& d = D[k];
    node_prep_one(nodes, i, d.nx, d.ny, d.nz, d.ntx, d.nty, d.tile0, W, st, tile_cnt, err + 2 * k, step, b0, b1, b2,
                  b3, b4, b5);
  }
  chunk_box_reduce(i, SP, chunk_box, b0, b1, b2, b3, b4, b5);
}

/* Entries {chunk, lane mask} per tile, as the one-grid spread's: a warp's
 * 32 nodes belong to one problem (every problem's nodes start at a
 * multiple of 32), so the warp works with that problem's grid; warps of
 * padding nodes or of a failed problem append nothing. */
__global__ void lbib_b_pair_scatter(const int* __restrict__ st, const int* __restrict__ node_inst,
                                    const BatchDesc* __restrict__ D, const int* __restrict__ slot,
                                    const int* __restrict__ slot_off, int* __restrict__ slot_cursor,
                                    int2* __restrict__ ent, const int* err, long SP) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long i0 = i & ~31L;   /* the warp's first node: its problem is the warp's */
  const int k = i0 < SP ? node_inst[i0] : -1;
  if (k < 0 || *(volatile const int*)(err + 2 * k)) return;   /* uniform over the warp */
  const BatchDesc& d = D[k];
  const long S = i < SP && node_inst[i] == k ? i + 1 : i;   /* lanes past the problem's nodes: no node */
  pair_scatter_warp(st, i, S, d.ntx, d.nty, d.nx, d.ny, d.nz, 0, d.ntx, slot + d.tile0, slot_off, slot_cursor, ent);
}

/* Every listed tile of the batch from its entries (gather_tile_ent), or,
 * with more than kListCap nodes, by scanning its problem's node chunks in
 * order (gather_tile_scan), in one launch. */
__global__ void __launch_bounds__(64) lbib_b_gather(const double* __restrict__ nodes, const double* __restrict__ W,
                                                    const int* __restrict__ st, const int* __restrict__ chunk_box,
                                                    const int* __restrict__ list, const int* __restrict__ count,
                                                    const int* __restrict__ slot_off, const int* __restrict__ slot_len,
                                                    const int* __restrict__ slot_cursor, const int2* __restrict__ ent,
                                                    const int* __restrict__ tile_inst, const BatchDesc* __restrict__ D,
                                                    double* __restrict__ Ftile, const int* err) {
  __shared__ union {
    GatherSmemE e;
    ScanSmem s;
  } sm;
  const int n = *count;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int tile = list[it];
    const int k = tile_inst[tile];
    if (*(volatile const int*)(err + 2 * k)) continue;
    const BatchDesc& d = D[k];
    const int L = slot_len[it];
    if (L <= kListCap) {
      gather_tile_ent(sm.e, nodes, W, st, it, (int)(tile - d.tile0), L, slot_cursor[it], ent + slot_off[it], d.ntx,
                      d.nty, Ftile);
    } else {
      __syncthreads();   /* the union's previous contents are no longer read */
      const long end = d.node0 + d.S;
      gather_tile_scan(sm.s, nodes, W, st, chunk_box, end, d.node0 >> 5, (end + 31) >> 5, it, (int)(tile - d.tile0),
                       d.ntx, d.nty, Ftile);
    }
  }
}

/* The move, a warp per 32 nodes of one problem with the union box of their
 * stencils staged in shared memory (move_warp); a pinned leading row stays. */
__global__ void __launch_bounds__(64) lbib_b_move(double* __restrict__ nodes, const double* __restrict__ W,
                                                  const int* __restrict__ st, const int* __restrict__ node_inst,
                                                  const BatchDesc* __restrict__ D, const int* __restrict__ slot,
                                                  const double* __restrict__ Utile, const int* err, long SP,
                                                  int* __restrict__ step_no) {
  __shared__ double sU[2][3 * kMoveCap + kMoveTiles / 2];
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) ++*step_no;   /* the last kernel of the step; node_prep has read it */
  const long i0 = i & ~31L;
  const int k = i0 < SP ? node_inst[i0] : -1;
  if (k < 0 || *(volatile const int*)(err + 2 * k)) return;   /* uniform over the warp */
  const BatchDesc& d = D[k];
  const bool live = i < SP && node_inst[i] == k && !(d.pinned && i - d.node0 < d.cols);
  move_warp(nodes, W, st, i, live, d.ntx, d.nty, slot + d.tile0, Utile, d.dt, sU[threadIdx.x >> 5]);
}

/* FP64 rows away from the walls: the two-cell step, a block per 128 pairs of
 * a problem's (row, pair) range, the parameters in shared memory. */
template <int PAR>
__global__ void __launch_bounds__(128, 3) lbib_b_x2(const FluidParams* __restrict__ P, const int2* __restrict__ blk,
                                                    const int* __restrict__ err) {
  __shared__ __align__(16) FluidParams sp;
  const int2 m = blk[blockIdx.x];
  if (err[2 * m.x]) return;
  block_copy(sp, P + m.x);
  const int npairs = (sp.xhi - sp.xlo + 1) / 2, nry = sp.ny - 6;
  const long g = (long)m.y * 128 + threadIdx.x;
  const long row = g / npairs;
  if (row >= (long)nry * x2_rows_z(sp.nz, sp.zin_hi)) return;
  const int pr = (int)(g - row * npairs);
  x2_pair<PAR>(sp, sp.xlo + 2 * pr, 3 + (int)(row % nry), 3 + (int)(row / nry));
}

template <int PAR>
int rest_f64_t(const BatchFluid& f) {
  const FluidParams* P = static_cast<const FluidParams*>(f.P);
  if (f.nxblk > 0) lbib_b_x2<PAR><<<(unsigned)f.nxblk, 128, 0, f.stream>>>(P, f.xblk, f.err);
  if (f.nrblk > 0) lbib_b_rows<double, PAR><<<(unsigned)f.nrblk, 128, 0, f.stream>>>(P, f.rowyz, f.rblk, f.err);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

namespace lbib {

int batch_fluid_rest_f64(const BatchFluid& f) { return f.par ? rest_f64_t<1>(f) : rest_f64_t<0>(f); }

int batch_tile_moments_f64(const BatchFluid& f) {
  const FluidParamsT<double>* P = static_cast<const FluidParamsT<double>*>(f.P);
  if (f.par == 0)
    lbib_b_tile_moments<double, 0><<<f.grid_tiles, 64, 0, f.stream>>>(P, f.desc, f.list, f.count, f.tile_inst, f.Ftile,
                                                                       f.Utile, f.err);
  else
    lbib_b_tile_moments<double, 1><<<f.grid_tiles, 64, 0, f.stream>>>(P, f.desc, f.list, f.count, f.tile_inst, f.Ftile,
                                                                       f.Utile, f.err);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace lbib

/* ------------------------------------------------------------ host state */


/* The batch's large buffers (populations, in/outlet tables, force and
 * moment tiles: hundreds of MB to GBs) come from a small per-process cache:
 * a buffer freed by one batch is kept (up to a quarter of the device's
 * memory) and handed to the next batch that fits in it, because releasing
 * and mapping that much device memory costs tenths of a second per batch
 * -- a sweep screen that re-runs a few dozen points paid more for its
 * batch's cudaFree than for its steps.  Every buffer is fully written by
 * the batch's set-up before use.  A failed allocation empties the cache
 * and tries again. */
namespace {
struct CachedBuf {
  void* p;
  size_t n;
  int dev;
};
std::mutex g_cache_mu;
std::vector<CachedBuf> g_cache;          /* free buffers */
std::vector<CachedBuf> g_live;           /* buffers handed out */
size_t g_cached = 0;
constexpr size_t kCacheMin = (size_t)16 << 20;

void cache_release_all() {
  for (const CachedBuf& c : g_cache) cudaFree(c.p);
  g_cache.clear();
  g_cached = 0;
}

cudaError_t big_malloc(void** p, size_t n) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_cache_mu);
  if (n >= kCacheMin) {
    int best = -1;
    for (int i = 0; i < (int)g_cache.size(); ++i)
      if (g_cache[i].dev == dev && g_cache[i].n >= n && g_cache[i].n <= 2 * n &&
          (best < 0 || g_cache[i].n < g_cache[best].n))
        best = i;
    if (best >= 0) {
      const CachedBuf c = g_cache[best];
      g_cache.erase(g_cache.begin() + best);
      g_cached -= c.n;
      g_live.push_back(c);
      *p = c.p;
      return cudaSuccess;
    }
  }
  cudaError_t e = cudaMalloc(p, n);
  if (e != cudaSuccess && !g_cache.empty()) {
    cudaGetLastError();
    cache_release_all();
    e = cudaMalloc(p, n);
  }
  if (e == cudaSuccess) g_live.push_back({*p, n, dev});
  return e;
}

void big_free(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_cache_mu);
  for (int i = 0; i < (int)g_live.size(); ++i) {
    if (g_live[i].p != p) continue;
    const CachedBuf c = g_live[i];
    g_live.erase(g_live.begin() + i);
    size_t fr = 0, total = 0;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(c.dev);
    cudaMemGetInfo(&fr, &total);
    cudaSetDevice(cur);
    if (c.n >= kCacheMin && g_cached + c.n <= total / 4) {
      g_cache.push_back(c);
      g_cached += c.n;
    } else {
      cudaFree(c.p);
    }
    return;
  }
  cudaFree(p);
}
}  // namespace

#include "../../include/lbib.h"

#define MAXV 8

struct lbib_batch {
  int B, prec, compat;
  cudaStream_t stream;
  lbib_device** sh;              /* host-only shadows, pointers into the pools */
  lbib_problem* prob;
  BatchDesc* h_desc;
  BatchDesc* desc;
  /* pools */
  unsigned char* f;
  unsigned char* tab;
  int *tile_cnt, *tile_inst, *scan_tmp, *slot_off, *slot_len, *slot_cursor, *pair_node;
  int *tile_slot[2], *tile_list[2], *tile_count[2];
  double *Ftile[2], *Utile[2];
  double *nodes, *W;
  int *st, *node_inst, *chunk_box;
  int *err, *h_err;
  int* step_no;                  /* device step counter, 1-based */
  long NT, CAP, SP, cells;
  /* per-problem fluid parameters: [cur] with first = 0, and the first step */
  void *P[2], *P_first, *WP[2], *WP_first;
  size_t psize, wsize;
  int2* rowyz;                   /* generic rows (y, z), each problem's contiguous */
  int4* rblk;                    /* generic-row blocks */
  long nrblk;
  int2* xblk;                    /* FP64 two-cell blocks (problem, block) */
  long nxblk;
  int* variant;                  /* word-kernel variant per problem */
  int2* wblk[MAXV];              /* word blocks of each variant group */
  long nwblk[MAXV];
  long steps;
  int parity, cur;
  cudaGraph_t graph;
  cudaGraphExec_t gexec;
  int have_graph;
  long launches, pair_launches;
  int grid_tiles;
};

namespace {

int is_lp(const lbib_batch* b) { return LBIB_PREC_TYPE(b->prec) != LBIB_PREC_F64; }

size_t pop_bytes(int prec) { return lbdev_pop_bytes(prec); }

long align_up(long v, long a) { return (v + a - 1) / a * a; }

/* FluidParamsT<T> / WordsParams<T> are the same size for every T (pointers
 * and scalars); fill the typed tables through the shadows. */
template <typename T>
void fill_tables(lbib_batch* b, int c, int first, void* P, void* WP) {
  FluidParamsT<T>* p = static_cast<FluidParamsT<T>*>(P);
  WordsParams<T>* w = static_cast<WordsParams<T>*>(WP);
  for (int k = 0; k < b->B; ++k) {
    lbib_device* d = b->sh[k];
    d->cur = c;
    p[k] = make_params_t<T>(d, first);
    w[k].p = p[k];
    int nry = 0, nrz = 0;
    if (lbdev_bulk_rows(d, &nry, &nrz)) {
      const int V = is_lp(b) ? batch_variant_cells_lp(b->prec, b->variant[k]) : 2;
      words_geometry(w[k], V, d->nx, nry, nrz);
    } else {
      memset(&w[k].nry, 0, sizeof(WordsParams<T>) - offsetof(WordsParams<T>, nry));
    }
  }
}

int upload_tables(lbib_batch* b) {
  void* hp = malloc(b->psize * b->B);
  void* hw = malloc(b->wsize * b->B);
  if (!hp || !hw) { free(hp); free(hw); return -5; }
  int rc = 0;
  for (int t = 0; t < 3 && !rc; ++t) {
    const int c = t == 2 ? 1 : t, first = t == 2;
    switch (LBIB_PREC_TYPE(b->prec)) {
      case LBIB_PREC_F32: fill_tables<float>(b, c, first, hp, hw); break;
      case LBIB_PREC_F16: fill_tables<__half>(b, c, first, hp, hw); break;
      case LBIB_PREC_BF16: fill_tables<__nv_bfloat16>(b, c, first, hp, hw); break;
      default: fill_tables<double>(b, c, first, hp, hw); break;
    }
    void* dp = t == 2 ? b->P_first : b->P[t];
    void* dw = t == 2 ? b->WP_first : b->WP[t];
    if (cudaMemcpy(dp, hp, b->psize * b->B, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
    if (!rc && cudaMemcpy(dw, hw, b->wsize * b->B, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
  }
  free(hp);
  free(hw);
  return rc;
}

/* Word blocks of each variant group: (problem, block within the problem). */
int build_word_blocks(lbib_batch* b) {
  for (int v = 0; v < MAXV; ++v) { cudaFree(b->wblk[v]); b->wblk[v] = NULL; b->nwblk[v] = 0; }
  if (!is_lp(b)) return 0;
  for (int v = 0; v < batch_variants_lp(b->prec); ++v) {
    long n = 0;
    for (int k = 0; k < b->B; ++k) {
      int nry = 0, nrz = 0;
      if (b->variant[k] != v || !b->h_desc[k].bulk || !lbdev_bulk_rows(b->sh[k], &nry, &nrz)) continue;
      const int V = batch_variant_cells_lp(b->prec, v);
      const long gpr = b->sh[k]->nx / V;   /* words_geometry: rows end to end */
      n += ((long)nry * nrz * gpr + WTPB - 1) / WTPB;
    }
    if (!n) continue;
    int2* h = (int2*)malloc(sizeof(int2) * n);
    if (!h) return -5;
    long i = 0;
    for (int k = 0; k < b->B; ++k) {
      int nry = 0, nrz = 0;
      if (b->variant[k] != v || !b->h_desc[k].bulk || !lbdev_bulk_rows(b->sh[k], &nry, &nrz)) continue;
      const int V = batch_variant_cells_lp(b->prec, v);
      const long gpr = b->sh[k]->nx / V;   /* words_geometry: rows end to end */
      const long nb = ((long)nry * nrz * gpr + WTPB - 1) / WTPB;
      for (long j = 0; j < nb; ++j) h[i++] = make_int2(k, (int)j);
    }
    int rc = 0;
    if (cudaMalloc(&b->wblk[v], sizeof(int2) * n) != cudaSuccess) rc = -5;
    else if (cudaMemcpy(b->wblk[v], h, sizeof(int2) * n, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
    free(h);
    if (rc) return rc;
    b->nwblk[v] = n;
  }
  return 0;
}

/* Rows of the generic kernel (every row of I for problems without bulk
 * rows; the wall rows otherwise) and their 128-cell blocks, and the FP64
 * two-cell blocks of the bulk rows (the low-precision word blocks, which
 * also step the plane-adjacent cells, come from build_word_blocks). */
int build_rows(lbib_batch* b) {
  const int lp = is_lp(b);
  long n = 0, nr = 0, nxb = 0;
  for (int k = 0; k < b->B; ++k) {
    const lbib_device* d = b->sh[k];
    int ry = 0, rz = 0;
    const int bulk = b->h_desc[k].bulk && lbdev_bulk_rows(d, &ry, &rz);
    const long rows = (long)(d->ny - 4) * (d->nz - 4) - (bulk ? (long)ry * rz : 0);
    n += rows;
    nr += (rows * (d->nx - 4) + 127) / 128;
    if (bulk && !lp) nxb += ((long)ry * rz * ((d->nx - 4) / 2) + 127) / 128;
  }
  int2* h = (int2*)malloc(sizeof(int2) * (n ? n : 1));
  int4* rb = (int4*)malloc(sizeof(int4) * (nr ? nr : 1));
  int2* xo = (int2*)malloc(sizeof(int2) * (nxb ? nxb : 1));
  if (!h || !rb || !xo) { free(h); free(rb); free(xo); return -5; }
  long r = 0, ir = 0, ix = 0;
  for (int k = 0; k < b->B; ++k) {
    const lbib_device* d = b->sh[k];
    int ry = 0, rz = 0;
    const int bulk = b->h_desc[k].bulk && lbdev_bulk_rows(d, &ry, &rz);
    const int zb = 2 + rz;
    const long r0 = r;
    for (int z = 2; z <= d->nz - 3; ++z)
      for (int y = 2; y <= d->ny - 3; ++y) {
        const int in_bulk = bulk && y >= 3 && y <= d->ny - 4 && z >= 3 && z <= zb;
        if (!in_bulk) h[r++] = make_int2(y, z);
      }
    const long rows = r - r0;
    for (long j = 0; j < (rows * (d->nx - 4) + 127) / 128; ++j) rb[ir++] = make_int4(k, (int)r0, (int)rows, (int)j);
    if (bulk && !lp)
      for (long j = 0; j < ((long)ry * rz * ((d->nx - 4) / 2) + 127) / 128; ++j) xo[ix++] = make_int2(k, (int)j);
  }
  b->nrblk = nr;
  b->nxblk = nxb;
  int rc = 0;
  if (cudaMalloc(&b->rowyz, sizeof(int2) * (n ? n : 1)) != cudaSuccess) rc = -5;
  else if (n && cudaMemcpy(b->rowyz, h, sizeof(int2) * n, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
  if (!rc && cudaMalloc(&b->rblk, sizeof(int4) * (nr ? nr : 1)) != cudaSuccess) rc = -5;
  else if (!rc && nr && cudaMemcpy(b->rblk, rb, sizeof(int4) * nr, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
  if (!rc && cudaMalloc(&b->xblk, sizeof(int2) * (nxb ? nxb : 1)) != cudaSuccess) rc = -5;
  else if (!rc && nxb && cudaMemcpy(b->xblk, xo, sizeof(int2) * nxb, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
  free(h);
  free(rb);
  free(xo);
  return rc;
}

BatchFluid fluid_args(lbib_batch* b, int par, const void* P, const void* WP, int c) {
  BatchFluid f;
  f.stream = b->stream;
  f.prec = b->prec;
  f.par = par;
  f.B = b->B;
  f.P = P;
  f.WP = WP;
  f.desc = b->desc;
  f.rowyz = b->rowyz;
  f.rblk = b->rblk;
  f.nrblk = b->nrblk;
  f.xblk = b->xblk;
  f.nxblk = b->nxblk;
  f.list = b->tile_list[c];
  f.count = b->tile_count[c];
  f.tile_inst = b->tile_inst;
  f.Ftile = b->Ftile[c];
  f.Utile = b->Utile[c];
  f.err = b->err;
  f.grid_tiles = b->grid_tiles;
  return f;
}

constexpr int kScan = 1024;

/* One step of the batch, launched on b->stream (eagerly or into a capture). */
int batch_step(lbib_batch* b) {
  const int c = b->cur ^ 1, par = b->parity, first = b->steps == 0;
  cudaStream_t s = b->stream;
  const long SP = b->SP;
  const unsigned nb = (unsigned)((SP + 127) / 128);
  const int bend_bug = (b->compat & 1) != 0;
  lbib_b_forces<<<nb, 128, 0, s>>>(b->nodes, b->node_inst, b->desc, b->err, SP, bend_bug);
  CK(cudaMemsetAsync(b->tile_cnt, 0, sizeof(int) * b->NT, s));
  CK(cudaMemsetAsync(b->tile_slot[c], 0xff, sizeof(int) * b->NT, s));
  lbib_b_node_prep<<<nb, 128, 0, s>>>(b->nodes, b->node_inst, b->desc, b->W, b->st, b->tile_cnt, b->chunk_box, b->err,
                                      SP, b->step_no);
  const unsigned nblk = (unsigned)((b->NT + kScan - 1) / kScan);
  int* block_tiles = b->scan_tmp;
  int* block_pairs = b->scan_tmp + nblk + 1;
  lbib_compact_count<<<nblk, kScan, 0, s>>>(b->tile_cnt, b->NT, block_tiles, block_pairs);
  lbib_compact_scan<<<1, kScan, 0, s>>>(block_tiles, block_pairs, (int)nblk, b->tile_count[c]);
  lbib_compact_write<<<nblk, kScan, 0, s>>>(b->tile_cnt, b->NT, block_tiles, block_pairs, b->tile_list[c],
                                            b->tile_slot[c], b->slot_off, b->slot_len, b->slot_cursor);
  int2* ent = reinterpret_cast<int2*>(b->pair_node);
  lbib_b_pair_scatter<<<nb, 128, 0, s>>>(b->st, b->node_inst, b->desc, b->tile_slot[c], b->slot_off, b->slot_cursor,
                                         ent, b->err, SP);
  lbib_b_gather<<<b->grid_tiles, 64, 0, s>>>(b->nodes, b->W, b->st, b->chunk_box, b->tile_list[c], b->tile_count[c],
                                             b->slot_off, b->slot_len, b->slot_cursor, ent, b->tile_inst, b->desc,
                                             b->Ftile[c], b->err);
  b->launches += 8;
  /* the fused fluid step */
  const void* P = first ? b->P_first : b->P[c];
  const void* WP = first ? b->WP_first : b->WP[c];
  BatchFluid f = fluid_args(b, par, P, WP, c);
  if (is_lp(b)) {
    for (int v = 0; v < MAXV; ++v)
      if (b->nwblk[v]) {
        if (batch_words_lp(f, v, b->wblk[v], b->nwblk[v])) return -2;
        b->launches++;
      }
    if (batch_fluid_rest_lp(f)) return -2;
    b->launches += 1 + (b->nrblk > 0);
  } else {
    if (batch_fluid_rest_f64(f)) return -2;
    b->launches += (b->nxblk > 0) + (b->nrblk > 0);
  }
  /* moments of the touched tiles, read by the next step and the move */
  BatchFluid g = fluid_args(b, par ^ 1, b->P[c], b->WP[c], c);
  if ((is_lp(b) ? batch_tile_moments_lp(g) : batch_tile_moments_f64(g))) return -2;
  lbib_b_move<<<(unsigned)((SP + 63) / 64), 64, 0, s>>>(b->nodes, b->W, b->st, b->node_inst, b->desc, b->tile_slot[c],
                                                        b->Utile[c], b->err, SP, b->step_no);
  b->launches += 2;
  b->cur = c;
  b->parity ^= 1;
  b->steps++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* Keep the shadows' step state in line with the batch (for the getters). */
void sync_shadows(lbib_batch* b) {
  for (int k = 0; k < b->B; ++k) {
    lbib_device* d = b->sh[k];
    d->cur = b->cur;
    d->parity = b->parity;
    d->steps = b->steps;
    d->have_forces = b->steps > 0;
    d->have_moments = b->steps > 0;
  }
}

void free_graph(lbib_batch* b) {
  if (b->have_graph) {
    cudaGraphExecDestroy(b->gexec);
    cudaGraphDestroy(b->graph);
    b->have_graph = 0;
  }
}

/* Populations and tables of every problem back to the initial state. */
int init_state(lbib_batch* b) {
  for (int k = 0; k < b->B; ++k) {
    lbib_device* d = b->sh[k];
    d->cur = 0;
    if (lbdev_launch_init(d, 0) || lbdev_launch_init(d, 1)) return -2;
  }
  CK(cudaMemsetAsync(b->tile_slot[0], 0xff, sizeof(int) * b->NT, b->stream));
  CK(cudaMemsetAsync(b->tile_slot[1], 0xff, sizeof(int) * b->NT, b->stream));
  const int one = 1;
  CK(cudaMemcpyAsync(b->step_no, &one, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  b->steps = 0;
  b->parity = 0;
  b->cur = 0;
  sync_shadows(b);
  return 0;
}

}  // namespace

/* ------------------------------------------------------------ C ABI */

extern "C" {

static int batch_error = 0;

lbib_batch* lbib_batch_create(int n, const lbib_problem* problems, int precision, int compat) {
  batch_error = LBIB_E_ARG;
  const int t = precision & ~LBIB_PREC_SHIFT_FLOW;
  if (n < 1 || !problems || t < LBIB_PREC_F64 || t > LBIB_PREC_BF16 ||
      (precision == (LBIB_PREC_F64 | LBIB_PREC_SHIFT_FLOW)) || (compat & ~LBIB_COMPAT_ALL))
    return NULL;
  for (int k = 0; k < n; ++k) {
    const lbib_problem* p = problems + k;
    if (p->nx < 8 || p->ny < 8 || p->nz < 8 || p->nx % 4 || p->ny % 4 || p->nz % 4 || p->rows < 2 || p->cols < 2 ||
        !(p->tau > 0.5))
      return NULL;
  }
  lbib_batch* b = (lbib_batch*)calloc(1, sizeof(lbib_batch));
  if (!b) { batch_error = LBIB_E_NOMEM; return NULL; }
  b->B = n;
  b->prec = precision;
  b->compat = compat;
  int rc = 0;
  b->sh = (lbib_device**)calloc(n, sizeof(lbib_device*));
  b->prob = (lbib_problem*)malloc(sizeof(lbib_problem) * n);
  b->h_desc = (BatchDesc*)calloc(n, sizeof(BatchDesc));
  b->variant = (int*)calloc(n, sizeof(int));
  if (!b->sh || !b->prob || !b->h_desc || !b->variant) rc = -5;
  if (!rc) memcpy(b->prob, problems, sizeof(lbib_problem) * n);
  if (!rc && cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) rc = -2;
  /* sizes and offsets */
  const size_t pb = pop_bytes(precision), rb = t == LBIB_PREC_F64 ? 8 : 4;
  long foff = 0, toff = 0, tile0 = 0, cap = 0, node0 = 0;
  for (int k = 0; k < n && !rc; ++k) {
    const lbib_problem* p = problems + k;
    lbdev_config c;
    memset(&c, 0, sizeof(c));
    c.nx = p->nx; c.ny = p->ny; c.nz = p->nz; c.cube_size = 4; c.compat = compat; c.prec = precision;
    /* init_gv_constant's constants, with the problem's tau, u, Ks, Kb */
    c.tau = p->tau; c.u_l = p->u_l; c.rho_l = 1.0e0; c.Ks_l = p->Ks_l; c.Kb_l = p->Kb_l; c.g_l = 0.0;
    c.cs_l = 1.0 / (sqrt(3)); c.dt = 1;
    lbib_device* d = (lbib_device*)calloc(1, sizeof(lbib_device));
    if (!d) { rc = -5; break; }
    b->sh[k] = d;
    d->nx = p->nx; d->ny = p->ny; d->nz = p->nz; d->prec = precision;
    d->N = (long)p->nx * p->ny * p->nz;
    lbdev_set_columns(d, 0, 0);
    d->cube_size = 4;
    d->ncx = p->nx / 4; d->ncy = p->ny / 4; d->ncz = p->nz / 4;
    lbdev_set_physics(d, &c);          /* constants and boundary rows; no stream yet: no allocation */
    d->ntx = p->nx / 4; d->nty = p->ny / 4; d->ntz = p->nz / 4;
    d->ntiles = (long)d->ntx * d->nty * d->ntz;
    d->lp_variant = -1;
    BatchDesc& D = b->h_desc[k];
    D.nx = p->nx; D.ny = p->ny; D.nz = p->nz; D.ntx = d->ntx; D.nty = d->nty;
    D.rows = p->rows; D.cols = p->cols;
    D.pinned = p->pinned != 0;
    D.tile0 = tile0; D.ntiles = d->ntiles;
    D.node0 = node0; D.S = (long)p->rows * p->cols;
    D.ds1 = p->width / (p->cols - 1);
    D.ds2 = p->height / (p->rows - 1);
    /* compute_bendingforce / compute_stretchingforce, lbm_ib.c:994-996, 1164-1166, 1230 */
    D.bc = p->Kb_l / pow(D.ds2, 3);
    D.sc = p->Ks_l / (D.ds1 * D.ds1);
    D.sc2 = p->Ks_l / (D.ds2 * D.ds2);
    D.dt = 1.0;
    int ry = 0, rz = 0;
    D.bulk = lbdev_bulk_rows(d, &ry, &rz) ? 1 : 0;
    b->cells += d->N;
    foff = align_up(foff, 256);
    d->f = (void*)foff;                /* offsets for now, pointers below */
    foff += (long)(pb * 19 * d->N);
    toff = align_up(toff, 256);
    d->inlet = (void*)toff;
    toff += (long)(rb * 19 * p->ny * p->nz);
    toff = align_up(toff, 256);
    d->outlet = (void*)toff;
    toff += (long)(rb * 19 * p->ny * p->nz);
    const long c8 = 8 * D.S;
    cap += c8 < d->ntiles ? c8 : d->ntiles;
    tile0 += d->ntiles;
    node0 = align_up(node0 + D.S, 32);
  }
  b->NT = tile0;
  b->CAP = cap;
  b->SP = node0;
  /* pools */
  if (!rc && big_malloc((void**)&b->f, foff) != cudaSuccess) rc = -5;
  if (!rc && big_malloc((void**)&b->tab, toff) != cudaSuccess) rc = -5;
  const long NT = b->NT, CAP = b->CAP, SP = b->SP;
  const long nblk = (NT + kScan - 1) / kScan;
  if (!rc && cudaMalloc(&b->tile_cnt, sizeof(int) * NT) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->tile_inst, sizeof(int) * NT) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->scan_tmp, sizeof(int) * (2 * nblk + 2)) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->slot_off, sizeof(int) * CAP) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->slot_len, sizeof(int) * CAP) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->slot_cursor, sizeof(int) * CAP) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->pair_node, sizeof(int2) * 8 * SP) != cudaSuccess) rc = -5;
  for (int c = 0; c < 2 && !rc; ++c) {
    if (cudaMalloc(&b->tile_slot[c], sizeof(int) * NT) != cudaSuccess) rc = -5;
    if (!rc && cudaMalloc(&b->tile_list[c], sizeof(int) * CAP) != cudaSuccess) rc = -5;
    if (!rc && cudaMalloc(&b->tile_count[c], sizeof(int)) != cudaSuccess) rc = -5;
    if (!rc && big_malloc((void**)&b->Ftile[c], sizeof(double) * 192 * CAP) != cudaSuccess) rc = -5;
    if (!rc && big_malloc((void**)&b->Utile[c], sizeof(double) * 256 * CAP) != cudaSuccess) rc = -5;
    if (!rc && cudaMemset(b->tile_count[c], 0, sizeof(int)) != cudaSuccess) rc = -2;
  }
  if (!rc && cudaMalloc(&b->nodes, sizeof(double) * 12 * SP) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->W, sizeof(double) * 12 * SP) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->st, sizeof(int) * 3 * SP) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->node_inst, sizeof(int) * SP) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->chunk_box, sizeof(int) * 6 * (SP / 32 + 1)) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->err, sizeof(int) * 2 * n) != cudaSuccess) rc = -5;
  if (!rc && cudaMallocHost(&b->h_err, sizeof(int) * 2 * n) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->step_no, sizeof(int)) != cudaSuccess) rc = -5;
  if (!rc && cudaMemset(b->err, 0, sizeof(int) * 2 * n) != cudaSuccess) rc = -2;
  if (!rc && cudaMalloc(&b->desc, sizeof(BatchDesc) * n) != cudaSuccess) rc = -5;
  if (!rc && cudaMemcpy(b->desc, b->h_desc, sizeof(BatchDesc) * n, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
  /* shadows: offsets -> pointers, and the batch's tile buffers */
  for (int k = 0; k < n && !rc; ++k) {
    lbib_device* d = b->sh[k];
    d->f = b->f + (long)d->f;
    d->inlet = b->tab + (long)d->inlet;
    d->outlet = b->tab + (long)d->outlet;
    const long t0 = b->h_desc[k].tile0;
    for (int c = 0; c < 2; ++c) {
      d->tile_slot[c] = b->tile_slot[c] + t0;
      d->tile_list[c] = b->tile_list[c];
      d->tile_count[c] = b->tile_count[c];
      d->Ftile[c] = b->Ftile[c];
      d->Utile[c] = b->Utile[c];
    }
    d->stream = b->stream;
    d->fluid_stream = b->stream;
    d->err = b->err + 2 * k;
    d->use_bulk = b->h_desc[k].bulk;
    d->have_df1 = d->have_inout = 1;
  }
  /* tile -> problem, node -> problem, the sheets (gen_fiber_sheet + the
     init_gv shift by u_l dt, mpi/gen_fiber_sheet.c:25-68, mpi/init_gv.c:239-245) */
  if (!rc) {
    int* ti = (int*)malloc(sizeof(int) * NT);
    int* ni = (int*)malloc(sizeof(int) * SP);
    double* nd = (double*)calloc(12 * SP, sizeof(double));
    if (!ti || !ni || !nd) rc = -5;
    for (int k = 0; k < n && !rc; ++k) {
      const BatchDesc& D = b->h_desc[k];
      for (long i = 0; i < D.ntiles; ++i) ti[D.tile0 + i] = k;
    }
    for (long i = 0; i < SP && !rc; ++i) ni[i] = -1;
    for (int k = 0; k < n && !rc; ++k) {
      const BatchDesc& D = b->h_desc[k];
      const lbib_problem* p = problems + k;
      const double zdist = p->width / (p->cols - 1), ydist = p->height / (p->rows - 1);
      for (int r = 0; r < p->rows; ++r)
        for (int c = 0; c < p->cols; ++c) {
          const long i = D.node0 + (long)r * p->cols + c;
          ni[i] = k;
          double x = p->x0;
          x += p->u_l * 1;                 /* nodes[j].x += u_l * dt, dt = 1 */
          nd[i * 12 + 0] = x;
          nd[i * 12 + 1] = ydist * r + p->y0;
          nd[i * 12 + 2] = zdist * c + p->z0;
        }
    }
    if (!rc && cudaMemcpy(b->tile_inst, ti, sizeof(int) * NT, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
    if (!rc && cudaMemcpy(b->node_inst, ni, sizeof(int) * SP, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
    if (!rc && cudaMemcpy(b->nodes, nd, sizeof(double) * 12 * SP, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
    free(ti);
    free(ni);
    free(nd);
  }
  /* parameter tables (all FluidParamsT<T> have one size, as do WordsParams<T>) */
  b->psize = sizeof(FluidParamsT<double>);
  b->wsize = sizeof(WordsParams<double>);
  static_assert(sizeof(FluidParamsT<double>) == sizeof(FluidParamsT<__half>), "one table size");
  static_assert(sizeof(WordsParams<double>) == sizeof(WordsParams<__half>), "one table size");
  for (int c = 0; c < 2 && !rc; ++c) {
    if (cudaMalloc(&b->P[c], b->psize * n) != cudaSuccess) rc = -5;
    if (!rc && cudaMalloc(&b->WP[c], b->wsize * n) != cudaSuccess) rc = -5;
  }
  if (!rc && cudaMalloc(&b->P_first, b->psize * n) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&b->WP_first, b->wsize * n) != cudaSuccess) rc = -5;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  b->grid_tiles = sms * 16;
  if (!rc) rc = build_rows(b);
  if (!rc) rc = upload_tables(b);
  if (!rc) rc = build_word_blocks(b);
  if (!rc) rc = init_state(b);
  if (!rc && cudaStreamSynchronize(b->stream) != cudaSuccess) rc = -2;
  if (rc) {
    lbib_batch_free(b);
    batch_error = rc;
    return NULL;
  }
  batch_error = 0;
  return b;
}

int lbib_batch_last_error(void) { return batch_error; }

void lbib_batch_free(lbib_batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  free_graph(b);
  for (int k = 0; k < b->B && b->sh; ++k) {
    if (b->sh[k]) cudaFree(b->sh[k]->scratch);
    free(b->sh[k]);
  }
  free(b->sh);
  big_free(b->f); big_free(b->tab);
  cudaFree(b->tile_cnt); cudaFree(b->tile_inst); cudaFree(b->scan_tmp);
  cudaFree(b->slot_off); cudaFree(b->slot_len); cudaFree(b->slot_cursor); cudaFree(b->pair_node);
  for (int c = 0; c < 2; ++c) {
    cudaFree(b->tile_slot[c]); cudaFree(b->tile_list[c]); cudaFree(b->tile_count[c]);
    big_free(b->Ftile[c]); big_free(b->Utile[c]);
    cudaFree(b->P[c]); cudaFree(b->WP[c]);
  }
  cudaFree(b->P_first); cudaFree(b->WP_first);
  cudaFree(b->nodes); cudaFree(b->W); cudaFree(b->st); cudaFree(b->node_inst); cudaFree(b->chunk_box);
  cudaFree(b->err);
  cudaFree(b->step_no);
  if (b->h_err) cudaFreeHost(b->h_err);
  cudaFree(b->desc); cudaFree(b->rowyz); cudaFree(b->rblk); cudaFree(b->xblk);
  for (int v = 0; v < MAXV; ++v) cudaFree(b->wblk[v]);
  if (b->stream) cudaStreamDestroy(b->stream);
  free(b->prob); free(b->h_desc); free(b->variant);
  free(b);
}

/* Steps: the first eagerly (it reads the initial state as the reference's
 * first step does), then a captured pair of steps (odd, even) replayed. */
int lbib_batch_run(lbib_batch* b, int nsteps) {
  if (!b || nsteps < 0) return LBIB_E_ARG;
  int done = 0;
  if (b->steps == 0 && done < nsteps) {
    if (batch_step(b)) return LBIB_E_CUDA;
    ++done;
  }
  if (nsteps - done >= 2 && (b->steps & 1) == 1) {
    if (!b->have_graph) {
      const long steps = b->steps, launches = b->launches;
      const int parity = b->parity, cur = b->cur;
      if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return LBIB_E_CUDA;
      int rc = batch_step(b);
      if (!rc) rc = batch_step(b);
      cudaGraph_t g = NULL;
      const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      b->pair_launches = b->launches - launches;
      b->steps = steps; b->launches = launches; b->parity = parity; b->cur = cur;
      if (rc || e != cudaSuccess) { if (g) cudaGraphDestroy(g); return LBIB_E_CUDA; }
      if (cudaGraphInstantiate(&b->gexec, g, 0) != cudaSuccess) { cudaGraphDestroy(g); return LBIB_E_CUDA; }
      b->graph = g;
      b->have_graph = 1;
    }
    while (nsteps - done >= 2) {
      if (cudaGraphLaunch(b->gexec, b->stream) != cudaSuccess) return LBIB_E_CUDA;
      b->steps += 2;
      b->launches += b->pair_launches;
      done += 2;
    }
  }
  while (done < nsteps) {
    if (batch_step(b)) return LBIB_E_CUDA;
    ++done;
  }
  sync_shadows(b);
  return LBIB_OK;
}

int lbib_batch_synchronize(lbib_batch* b) {
  if (!b) return LBIB_E_ARG;
  return cudaStreamSynchronize(b->stream) == cudaSuccess ? LBIB_OK : LBIB_E_CUDA;
}

void* lbib_batch_stream(lbib_batch* b) { return b ? (void*)b->stream : NULL; }

long lbib_batch_cells(lbib_batch* b) { return b ? b->cells : 0; }

long lbib_batch_steps(lbib_batch* b) { return b ? b->steps : 0; }

int lbib_batch_status(lbib_batch* b, int* codes, int* failed_step) {
  if (!b) return LBIB_E_ARG;
  if (cudaMemcpyAsync(b->h_err, b->err, sizeof(int) * 2 * b->B, cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess)
    return LBIB_E_CUDA;
  int nfail = 0;
  for (int k = 0; k < b->B; ++k) {
    if (codes) codes[k] = b->h_err[2 * k];
    if (failed_step) failed_step[k] = b->h_err[2 * k + 1];
    nfail += b->h_err[2 * k] != 0;
  }
  return nfail;
}

int lbib_batch_get_sheet(lbib_batch* b, int k, double* out) {
  if (!b || k < 0 || k >= b->B || !out) return LBIB_E_ARG;
  const BatchDesc& D = b->h_desc[k];
  if (cudaMemcpyAsync(out, b->nodes + D.node0 * 12, sizeof(double) * 12 * D.S, cudaMemcpyDeviceToHost, b->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess)
    return LBIB_E_CUDA;
  return LBIB_OK;
}

int lbib_batch_get_moments(lbib_batch* b, int k, double* rho, double* ux, double* uy, double* uz) {
  if (!b || k < 0 || k >= b->B || !rho || !ux || !uy || !uz) return LBIB_E_ARG;
  return lbdev_get_moments(b->sh[k], rho, ux, uy, uz) ? LBIB_E_CUDA : LBIB_OK;
}

int lbib_batch_get_df1(lbib_batch* b, int k, double* out) {
  if (!b || k < 0 || k >= b->B || !out) return LBIB_E_ARG;
  return lbdev_get_df1(b->sh[k], out) ? LBIB_E_CUDA : LBIB_OK;
}

int lbib_batch_variants(lbib_batch* b) { return b && is_lp(b) ? batch_variants_lp(b->prec) : 1; }

int lbib_batch_set_variant(lbib_batch* b, int k, int v) {
  if (!b || k < -1 || k >= b->B || v < 0 || v >= lbib_batch_variants(b)) return LBIB_E_ARG;
  if (b->steps != 0) return LBIB_E_STATE;
  for (int i = 0; i < b->B; ++i)
    if (k < 0 || i == k) b->variant[i] = v;
  free_graph(b);
  int rc = upload_tables(b);
  if (!rc) rc = build_word_blocks(b);
  return rc ? LBIB_E_CUDA : LBIB_OK;
}

/* Per size class (problems with the same nx, ny, nz) time every word-kernel
 * variant on `steps` fluid steps of that class's word blocks alone, keep
 * the fastest for the class, and restore the initial state.  ms[c * V + v]
 * (classes in order of first appearance, up to max_ms entries) receives the
 * mean ms per step; returns the number of classes or an error code. */
int lbib_batch_autotune(lbib_batch* b, int steps, double* ms, int max_ms, int* class_of) {
  if (!b) return LBIB_E_ARG;
  if (b->steps != 0) return LBIB_E_STATE;
  const int nv = lbib_batch_variants(b);
  int* cls = (int*)malloc(sizeof(int) * b->B);
  int* rep = (int*)malloc(sizeof(int) * b->B);
  if (!cls || !rep) { free(cls); free(rep); return LBIB_E_NOMEM; }
  int ncls = 0;
  for (int k = 0; k < b->B; ++k) {
    int c = -1;
    for (int j = 0; j < ncls; ++j) {
      const lbib_problem* a = b->prob + rep[j];
      if (a->nx == b->prob[k].nx && a->ny == b->prob[k].ny && a->nz == b->prob[k].nz) { c = j; break; }
    }
    if (c < 0) { c = ncls++; rep[c] = k; }
    cls[k] = c;
    if (class_of) class_of[k] = c;
  }
  if (steps < 2) steps = 2;
  steps += steps & 1;
  int rc = 0;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = LBIB_E_CUDA;
  int* best = (int*)calloc(ncls, sizeof(int));
  float* best_ms = (float*)calloc(ncls, sizeof(float));
  for (int v = 0; v < nv && !rc && nv > 1; ++v) {
    for (int k = 0; k < b->B; ++k) b->variant[k] = v;
    if (upload_tables(b)) { rc = LBIB_E_CUDA; break; }
    for (int c = 0; c < ncls && !rc; ++c) {
      /* word blocks of class c only */
      for (int k = 0; k < b->B; ++k) b->variant[k] = cls[k] == c ? v : -1;
      if (build_word_blocks(b)) { rc = LBIB_E_CUDA; break; }
      if (!b->nwblk[v]) continue;
      float t = 0.0f;
      for (int rep2 = 0; rep2 < 2 && !rc; ++rep2) {   /* first pass warms up */
        if (cudaEventRecord(e0, b->stream) != cudaSuccess) rc = LBIB_E_CUDA;
        for (int s = 0; s < steps && !rc; ++s) {
          BatchFluid f = fluid_args(b, s & 1, b->P[0], b->WP[0], 0);
          if (batch_words_lp(f, v, b->wblk[v], b->nwblk[v])) rc = LBIB_E_CUDA;
        }
        if (!rc && cudaEventRecord(e1, b->stream) != cudaSuccess) rc = LBIB_E_CUDA;
        if (!rc && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess))
          rc = LBIB_E_CUDA;
      }
      if (rc) break;
      if (ms && c * nv + v < max_ms) ms[c * nv + v] = t / steps;
      if (v == 0 || t < best_ms[c]) { best_ms[c] = t; best[c] = v; }
    }
  }
  if (!rc) {
    for (int k = 0; k < b->B; ++k) b->variant[k] = nv > 1 ? best[cls[k]] : 0;
    free_graph(b);
    if (upload_tables(b) || build_word_blocks(b) || init_state(b)) rc = LBIB_E_CUDA;
    if (!rc && cudaStreamSynchronize(b->stream) != cudaSuccess) rc = LBIB_E_CUDA;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  free(best);
  free(best_ms);
  free(cls);
  free(rep);
  return rc ? rc : ncls;
}

long lbib_batch_kernel_launches(lbib_batch* b) { return b ? b->launches : 0; }

}  /* extern "C" */
