/*
 * Immersed-boundary device code shared by the one-grid kernels
 * (lbib_ib.cu) and the batched ones (lbib_batch.cu).
 *
 *   fiber_forces_node   compute_bendingforce + compute_stretchingforce +
 *                       compute_elasticforce (cube_pthread/lbm_ib.c:961-1318),
 *                       one node, both passes of each force in the
 *                       reference's order.
 *   node_prep_one       stencil start floor(X - 2) + 1 per axis, the twelve
 *                       delta-kernel factors 1 + cos(pi/2 r) (shared by the
 *                       spread and the interpolation of the step), the 4^3
 *                       tiles the stencil touches; chunk_box_reduce: per
 *                       32-node chunk the bounding box of its stencils.
 *   compaction kernels  touched tiles -> dense list in tile order, tile ->
 *                       slot map, and each slot's list offset
 *                       (deterministic prefix sums, three launches or one
 *                       single-pass launch); pair_scatter_warp fills the
 *                       lists with {chunk, lane mask} entries.
 *   gather_tile_ent     fiber_SpreadForce + fluid_get_SpreadForce
 *                       (lbm_ib.c:1323-1525) as a gather: one CTA per touched
 *                       tile sorts the tile's entries, writes its node list
 *                       in index order, then each thread (cell) sums the
 *                       contributions in that order -- the reference's
 *                       (sheet, row, col) order -- so the result is
 *                       deterministic and needs no atomics on forces.
 *   move_node /         moveFiberSheet (lbm_ib.c:2540-2723): u * w summed over
 *   move_warp           the 64 stencil cells in the reference's (x, y, z)
 *                       order, then X += dt U (move_warp: a warp's nodes
 *                       with their stencils' union staged in shared memory).
 * All arithmetic keeps the reference's operation order; translation units
 * that include this file are compiled with -fmad=false.
 */
#ifndef LBIB_IB_CUH
#define LBIB_IB_CUH

#include <climits>

#include "lbib_cos.h"
#include "lbib_internal.h"
#include "lbib_lattice.cuh"

namespace lbib {


/* PI as truncated in the reference, cube_pthread/lbm_ib.c:33. */
constexpr double kPi = 3.14159265358979;

__device__ __forceinline__ void set_error(int* err, int code, int step) {
  if (atomicCAS(err, 0, code) == 0) err[1] = step;
}

/* compute_bendingforce + compute_stretchingforce + compute_elasticforce for
 * node i of one R x C sheet whose records start at `nodes`. */
__device__ __forceinline__ void fiber_forces_node(double* __restrict__ nodes, int R, int C, double bc, double sc,
                                                  double sc2, double ds1, double ds2, int bend_bug, int i) {
  const int r = i / C, c = i % C;
#define P(rr, cc) (nodes + ((long)(rr) * C + (cc)) * 12)
  const double* m = P(r, c);
  double b[3], s[3];
  /* bending along the fiber (row), lbm_ib.c:1002-1052 */
  for (int d = 0; d < 3; ++d) {
    if (c == 0) {
      b[d] = bc * (-P(r, 2)[d] + 2 * P(r, 1)[d] - P(r, 0)[d]);
    } else if (c == 1) {
      b[d] = bc * (-P(r, 3)[d] + 4 * P(r, 2)[d] - 5 * P(r, 1)[d] + 2 * P(r, 0)[d]);
    } else if (c == C - 1) {
      b[d] = bc * (-P(r, c)[d] + 2 * P(r, c - 1)[d] - P(r, c - 2)[d]);
    } else if (c == C - 2) {
      const double last = (d == 0 && bend_bug) ? P(r, c)[d] : P(r, c - 2)[d];
      b[d] = bc * (2 * P(r, c + 1)[d] - 5 * P(r, c)[d] + 4 * P(r, c - 1)[d] - last);
    } else {
      b[d] = bc * (-P(r, c + 2)[d] + 4.0 * P(r, c + 1)[d] - 6.0 * P(r, c)[d] + 4.0 * P(r, c - 1)[d] - P(r, c - 2)[d]);
    }
  }
  /* bending across fibers (column), lbm_ib.c:1062-1145 */
  for (int d = 0; d < 3; ++d) {
    double v;
    if (r == 0) {
      v = bc * (-P(2, c)[d] + 2 * (P(1, c)[d]) - (P(0, c)[d]));
    } else if (r == 1) {
      v = bc * (-P(3, c)[d] + 4 * (P(2, c)[d]) - 5 * (P(1, c)[d]) + 2 * (P(0, c)[d]));
    } else if (r == R - 1) {
      v = bc * (-(P(r, c)[d]) + 2 * (P(r - 1, c)[d]) - (P(r - 2, c)[d]));
    } else if (r == R - 2) {
      v = bc * (2 * P(r + 1, c)[d] - 5 * (P(r, c)[d]) + 4 * (P(r - 1, c)[d]) - (P(r - 2, c)[d]));
    } else {
      v = bc * (-P(r + 2, c)[d] + 4.0 * (P(r + 1, c)[d]) - 6.0 * (P(r, c)[d]) + 4.0 * (P(r - 1, c)[d]) - (P(r - 2, c)[d]));
    }
    b[d] = b[d] + v;
  }
  /* stretching along the fiber (row), lbm_ib.c:1179-1221 */
  if (c == 0) {
    const double* p = P(r, 1);
    const double t0 = p[0] - m[0], t1 = p[1] - m[1], t2 = p[2] - m[2];
    const double dr = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
    s[0] = sc * ((dr - ds1) * (t0 / dr));
    s[1] = sc * ((dr - ds1) * (t1 / dr));
    s[2] = sc * ((dr - ds1) * (t2 / dr));
  } else if (c == C - 1) {
    const double* q = P(r, C - 2);
    const double t0 = m[0] - q[0], t1 = m[1] - q[1], t2 = m[2] - q[2];
    const double dl = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
    s[0] = sc * ((dl - ds1) * (t0 / dl));
    s[1] = sc * ((dl - ds1) * (t1 / dl));
    s[2] = sc * ((dl - ds1) * (t2 / dl));
  } else {
    const double* p = P(r, c + 1);
    const double* q = P(r, c - 1);
    const double r0 = p[0] - m[0], r1 = p[1] - m[1], r2 = p[2] - m[2];
    const double l0 = q[0] - m[0], l1 = q[1] - m[1], l2 = q[2] - m[2];
    const double dr = sqrt(r0 * r0 + r1 * r1 + r2 * r2);
    const double dl = sqrt(l0 * l0 + l1 * l1 + l2 * l2);
    s[0] = sc * ((dr - ds1) * (r0 / dr) + (dl - ds1) * (l0 / dl));
    s[1] = sc * ((dr - ds1) * (r1 / dr) + (dl - ds1) * (l1 / dl));
    s[2] = sc * ((dr - ds1) * (r2 / dr) + (dl - ds1) * (l2 / dl));
  }
  /* stretching across fibers (column), lbm_ib.c:1233-1278 */
  if (r == 0) {
    const double* p = P(1, c);
    const double t0 = p[0] - m[0], t1 = p[1] - m[1], t2 = p[2] - m[2];
    const double dt = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
    s[0] = s[0] + sc2 * ((dt - ds2) * (t0 / dt));
    s[1] = s[1] + sc2 * ((dt - ds2) * (t1 / dt));
    s[2] = s[2] + sc2 * ((dt - ds2) * (t2 / dt));
  } else if (r == R - 1) {
    const double* q = P(R - 2, c);
    const double t0 = m[0] - q[0], t1 = m[1] - q[1], t2 = m[2] - q[2];
    const double db = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
    s[0] = s[0] + sc2 * ((db - ds2) * (t0 / db));
    s[1] = s[1] + sc2 * ((db - ds2) * (t1 / db));
    s[2] = s[2] + sc2 * ((db - ds2) * (t2 / db));
  } else {
    const double* p = P(r + 1, c);
    const double* q = P(r - 1, c);
    const double a0 = p[0] - m[0], a1 = p[1] - m[1], a2 = p[2] - m[2];
    const double e0 = q[0] - m[0], e1 = q[1] - m[1], e2 = q[2] - m[2];
    const double dt = sqrt(a0 * a0 + a1 * a1 + a2 * a2);
    const double db = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
    s[0] = s[0] + sc2 * ((dt - ds2) * (a0 / dt) + (db - ds2) * (e0 / db));
    s[1] = s[1] + sc2 * ((dt - ds2) * (a1 / dt) + (db - ds2) * (e1 / db));
    s[2] = s[2] + sc2 * ((dt - ds2) * (a2 / dt) + (db - ds2) * (e2 / db));
  }
#undef P
  double* o = nodes + (long)i * 12;
  o[3] = b[0]; o[4] = b[1]; o[5] = b[2];
  o[6] = s[0]; o[7] = s[1]; o[8] = s[2];
  /* compute_elasticforce, lbm_ib.c:1303-1308: stretch + bend */
  o[9] = s[0] + b[0]; o[10] = s[1] + b[1]; o[11] = s[2] + b[2];
}

__device__ __forceinline__ int stencil_start(double p) { return (int)(floor(p / 1.0 - 2) + 1); }

/* The stencil of a node at coordinate p lies inside an axis of n cells:
 * start = floor(p - 2) + 1 in [0, n - 4], i.e. 1 <= p < n - 2, decided on
 * the double itself so that NaN and huge coordinates fail the test (the
 * reference stops with "out of bound" there; an int conversion first would
 * turn NaN into 0 and pass). */
__device__ __forceinline__ bool stencil_inside(double p, int n) { return p >= 1.0 && p < (double)n - 2.0; }

/* Node i: stencil start, the twelve delta-kernel factors, a count for every
 * 4^3 tile its stencil touches (tile ids offset by tile0); b0..b5 receive
 * its stencil box (left empty when the stencil leaves the grid). */
__device__ __forceinline__ void node_prep_one(const double* __restrict__ nodes, long i, int nx, int ny, int nz,
                                              int ntx, int nty, long tile0, double* __restrict__ W,
                                              int* __restrict__ st, int* __restrict__ tile_cnt, int* err, int step,
                                              int& b0, int& b1, int& b2, int& b3, int& b4, int& b5) {
  {
    const double* m = nodes + i * 12;
    const bool inside = stencil_inside(m[0], nx) && stencil_inside(m[1], ny) && stencil_inside(m[2], nz);
    const int is = inside ? stencil_start(m[0]) : 0, js = inside ? stencil_start(m[1]) : 0,
              ks = inside ? stencil_start(m[2]) : 0;
    st[i * 3 + 0] = is; st[i * 3 + 1] = js; st[i * 3 + 2] = ks;
    const double cxk = kPi / (2.0 * 1.0);
    double* w = W + i * 12;
    for (int a = 0; a < 4; ++a) {
      w[a] = 1.0e0 + lbib_cos_2phase(cxk * (1.0 * (is + a) - m[0]));
      w[4 + a] = 1.0e0 + lbib_cos_2phase(cxk * (1.0 * (js + a) - m[1]));
      w[8 + a] = 1.0e0 + lbib_cos_2phase(cxk * (1.0 * (ks + a) - m[2]));
    }
    if (!inside) {
      set_error(err, -3, step);
    } else {
      for (int tz = ks >> 2; tz <= (ks + 3) >> 2; ++tz)
        for (int ty = js >> 2; ty <= (js + 3) >> 2; ++ty)
          for (int tx = is >> 2; tx <= (is + 3) >> 2; ++tx)
            atomicAdd(&tile_cnt[tile0 + ((long)tz * nty + ty) * ntx + tx], 1);
      b0 = is; b1 = is + 3; b2 = js; b3 = js + 3; b4 = ks; b5 = ks + 3;
    }
  }
}

/* node_prep_one for the one-grid kernel, split over four threads per node:
 * part p (0..3) evaluates the three delta factors of stencil offset p (one
 * per axis); part 0 also writes the stencil start, checks the grid and
 * counts the touched tiles.  The same values as node_prep_one, with the
 * twelve dependent cosine evaluations of a node spread over four warps. */
__device__ __forceinline__ void node_prep_part(const double* __restrict__ nodes, long i, int part, int nx, int ny,
                                               int nz, int ntx, int nty, double* __restrict__ W,
                                               int* __restrict__ st, int* __restrict__ tile_cnt, int* err, int step,
                                               int& b0, int& b1, int& b2, int& b3, int& b4, int& b5) {
  const double* m = nodes + i * 12;
  const bool inside = stencil_inside(m[0], nx) && stencil_inside(m[1], ny) && stencil_inside(m[2], nz);
  const int is = inside ? stencil_start(m[0]) : 0, js = inside ? stencil_start(m[1]) : 0,
            ks = inside ? stencil_start(m[2]) : 0;
  const double cxk = kPi / (2.0 * 1.0);
  double* w = W + i * 12;
  w[part] = 1.0e0 + lbib_cos_2phase(cxk * (1.0 * (is + part) - m[0]));
  w[4 + part] = 1.0e0 + lbib_cos_2phase(cxk * (1.0 * (js + part) - m[1]));
  w[8 + part] = 1.0e0 + lbib_cos_2phase(cxk * (1.0 * (ks + part) - m[2]));
  if (part != 0) return;
  st[i * 3 + 0] = is; st[i * 3 + 1] = js; st[i * 3 + 2] = ks;
  if (!inside) {
    set_error(err, -3, step);
  } else {
    for (int tz = ks >> 2; tz <= (ks + 3) >> 2; ++tz)
      for (int ty = js >> 2; ty <= (js + 3) >> 2; ++ty)
        for (int tx = is >> 2; tx <= (is + 3) >> 2; ++tx)
          atomicAdd(&tile_cnt[((long)tz * nty + ty) * ntx + tx], 1);
    b0 = is; b1 = is + 3; b2 = js; b3 = js + 3; b4 = ks; b5 = ks + 3;
  }
}

/* The bounding box of a warp's stencils, written by lane 0 for chunk i >> 5. */
__device__ __forceinline__ void chunk_box_reduce(long i, long S, int* __restrict__ chunk_box, int b0, int b1, int b2,
                                                 int b3, int b4, int b5) {
  const int lane = threadIdx.x & 31;
  for (int o = 16; o > 0; o >>= 1) {
    b0 = min(b0, __shfl_xor_sync(0xffffffffu, b0, o));
    b1 = max(b1, __shfl_xor_sync(0xffffffffu, b1, o));
    b2 = min(b2, __shfl_xor_sync(0xffffffffu, b2, o));
    b3 = max(b3, __shfl_xor_sync(0xffffffffu, b3, o));
    b4 = min(b4, __shfl_xor_sync(0xffffffffu, b4, o));
    b5 = max(b5, __shfl_xor_sync(0xffffffffu, b5, o));
  }
  const long chunk = i >> 5;
  if (lane == 0 && chunk * 32 < S) {
    int* bx = chunk_box + chunk * 6;
    bx[0] = b0; bx[1] = b1; bx[2] = b2; bx[3] = b3; bx[4] = b4; bx[5] = b5;
  }
}

/* Deterministic compaction of the tile counts, in tile-index order:
 * per-block sums (touched tiles, node-tile pairs), a one-block scan of both,
 * then every touched tile gets its slot and the offset of its node list. */
constexpr int kScanBlock = 1024;

static __global__ void lbib_compact_count(const int* __restrict__ cnt, long n, int* __restrict__ block_tiles,
                                   int* __restrict__ block_pairs) {
  __shared__ int s[2][32];
  const long i = (long)blockIdx.x * kScanBlock + threadIdx.x;
  const int c = (i < n) ? cnt[i] : 0;
  int v = c > 0, w = c;
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, o);
    w += __shfl_xor_sync(0xffffffffu, w, o);
  }
  if ((threadIdx.x & 31) == 0) { s[0][threadIdx.x >> 5] = v; s[1][threadIdx.x >> 5] = w; }
  __syncthreads();
  if (threadIdx.x < 32) {
    int a = s[0][threadIdx.x], b = s[1][threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (threadIdx.x == 0) { block_tiles[blockIdx.x] = a; block_pairs[blockIdx.x] = b; }
  }
}

__device__ __forceinline__ void block_exclusive_scan(int* __restrict__ a, int n, int* total) {
  __shared__ int s[kScanBlock];
  int carry = 0;
  for (int base = 0; base < n; base += kScanBlock) {
    const int i = base + threadIdx.x;
    const int v = (i < n) ? a[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
      const int t = (threadIdx.x >= (unsigned)o) ? s[threadIdx.x - o] : 0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < n) a[i] = carry + s[threadIdx.x] - v;
    const int last = s[kScanBlock - 1];
    __syncthreads();
    carry += last;
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

static __global__ void lbib_compact_scan(int* __restrict__ block_tiles, int* __restrict__ block_pairs, int nblocks,
                                  int* __restrict__ total_tiles) {
  block_exclusive_scan(block_tiles, nblocks, total_tiles);
  __syncthreads();
  block_exclusive_scan(block_pairs, nblocks, nullptr);
}

static __global__ void lbib_compact_write(int* __restrict__ cnt, long n, const int* __restrict__ block_tiles,
                                   const int* __restrict__ block_pairs, int* __restrict__ list,
                                   int* __restrict__ slot, int* __restrict__ slot_off, int* __restrict__ slot_len,
                                   int* __restrict__ slot_cursor) {
  __shared__ int sv[32], sw[32];
  const long i = (long)blockIdx.x * kScanBlock + threadIdx.x;
  const int c = (i < n) ? cnt[i] : 0;
  const int v = c > 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int iv = v, iw = c;  /* inclusive warp scans */
  for (int o = 1; o < 32; o <<= 1) {
    const int tv = __shfl_up_sync(0xffffffffu, iv, o);
    const int tw = __shfl_up_sync(0xffffffffu, iw, o);
    if (lane >= o) { iv += tv; iw += tw; }
  }
  if (lane == 31) { sv[warp] = iv; sw[warp] = iw; }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int a = sv[threadIdx.x], b = sw[threadIdx.x];
    int ia = a, ib = b;
    for (int o = 1; o < 32; o <<= 1) {
      const int ta = __shfl_up_sync(0xffffffffu, ia, o);
      const int tb = __shfl_up_sync(0xffffffffu, ib, o);
      if (lane >= o) { ia += ta; ib += tb; }
    }
    sv[threadIdx.x] = ia - a;
    sw[threadIdx.x] = ib - b;
  }
  __syncthreads();
  if (v) {
    const int pos = block_tiles[blockIdx.x] + sv[warp] + iv - v;
    list[pos] = (int)i;
    slot[i] = pos;
    slot_off[pos] = block_pairs[blockIdx.x] + sw[warp] + iw - c;
    slot_len[pos] = c;
    slot_cursor[pos] = 0;
  } else if (i < n) {
    slot[i] = -1;     /* the whole map is written: no clearing pass before the step */
  }
  if (i < n && c) cnt[i] = 0;   /* counts start the next step at zero */
}

/* The same compaction in one launch: a single-pass scan with decoupled
 * look-back (Merrill & Garland, "Single-pass Parallel Prefix Scan with
 * Decoupled Look-back", 2016).  A block takes its place in tile order from
 * a ticket counter (so every block before it has started), publishes its
 * block totals, walks back over its predecessors' published totals until
 * one carries an inclusive prefix, publishes its own inclusive prefix and
 * writes its tiles' slots.  Each published word is 64 bits: an 8-bit
 * launch tag (1..255, never 0, so a zeroed or stale word never matches),
 * a 2-bit flag (1 block totals, 2 inclusive prefix), 22 bits of tiles and
 * 32 bits of pairs; the host uses it only when the tile count fits 22
 * bits.  Every wait is bounded: a walk that runs out sets err (the step
 * then fails) instead of spinning on.  state[nblk] holds the ticket,
 * which the last block resets for the next launch. */
constexpr long kLookbackSpin = 1L << 22;
constexpr int kOnepassTiles = 4;   /* tiles per thread: a block covers 4096 tiles */
constexpr int kErrLookback = -2;   /* the error word's code: LBIB_E_CUDA of include/lbib.h */

__device__ __forceinline__ unsigned long long lookback_word(unsigned tag, unsigned flag, unsigned long long t,
                                                            unsigned long long p) {
  return ((unsigned long long)tag << 56) | ((unsigned long long)flag << 54) | ((t & 0x3FFFFFull) << 32) |
         (p & 0xFFFFFFFFull);
}

static __global__ void __launch_bounds__(kScanBlock) lbib_compact_onepass(int* __restrict__ cnt, long n, int nblk,
                                                                          unsigned long long* __restrict__ state,
                                                                          unsigned tag, int* __restrict__ list,
                                                                          int* __restrict__ slot,
                                                                          int* __restrict__ slot_off,
                                                                          int* __restrict__ slot_len,
                                                                          int* __restrict__ slot_cursor,
                                                                          int* __restrict__ total, int* err) {
  __shared__ int sv[32], sw[32];
  __shared__ int s_vb, s_tt, s_tp, s_pt, s_pp;
  unsigned* ticket = reinterpret_cast<unsigned*>(state + nblk);
  if (threadIdx.x == 0) s_vb = (int)atomicAdd(ticket, 1u);
  __syncthreads();
  const int vb = s_vb;
  /* kOnepassTiles consecutive tiles per thread: fewer, fuller blocks, so
     that every block is resident at once and the look-back walks short */
  const long i0 = ((long)vb * kScanBlock + threadIdx.x) * kOnepassTiles;
  int c[kOnepassTiles], tv = 0, tw = 0;
#pragma unroll
  for (int k = 0; k < kOnepassTiles; ++k) {
    c[k] = (i0 + k < n) ? cnt[i0 + k] : 0;
    tv += c[k] > 0;
    tw += c[k];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int iv = tv, iw = tw;  /* inclusive warp scans of the threads' totals */
  for (int o = 1; o < 32; o <<= 1) {
    const int tv = __shfl_up_sync(0xffffffffu, iv, o);
    const int tw = __shfl_up_sync(0xffffffffu, iw, o);
    if (lane >= o) { iv += tv; iw += tw; }
  }
  if (lane == 31) { sv[warp] = iv; sw[warp] = iw; }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int a = sv[threadIdx.x], b = sw[threadIdx.x];
    int ia = a, ib = b;
    for (int o = 1; o < 32; o <<= 1) {
      const int ta = __shfl_up_sync(0xffffffffu, ia, o);
      const int tb = __shfl_up_sync(0xffffffffu, ib, o);
      if (lane >= o) { ia += ta; ib += tb; }
    }
    sv[threadIdx.x] = ia - a;
    sw[threadIdx.x] = ib - b;
    if (threadIdx.x == 31) { s_tt = ia; s_tp = ib; }
  }
  __syncthreads();
  if (warp == 0) {
    /* warp 0 walks back 32 predecessors at a time: lane k reads block
       j - k; the window is summed up to its nearest inclusive word once
       every word up to there has been published */
    volatile unsigned long long* vs = state;
    const unsigned long long at = (unsigned)s_tt, ap = (unsigned)s_tp;
    if (vb > 0 && lane == 0) vs[vb] = lookback_word(tag, 1u, at, ap);
    __syncwarp();
    unsigned long long et = 0, ep = 0;
    long spins = 0;
    for (int j = vb - 1; j >= 0;) {
      const int jj = j - lane;
      const unsigned long long w = jj >= 0 ? vs[jj] : lookback_word(tag, 2u, 0ull, 0ull);
      const unsigned f = (unsigned)(w >> 54) & 3u;
      const bool ready = (unsigned)(w >> 56) == tag && f != 0u;
      const unsigned incl = __ballot_sync(0xffffffffu, ready && f == 2u);
      const unsigned rdy = __ballot_sync(0xffffffffu, ready);
      const int lim = incl ? __ffs(incl) - 1 : 31;
      const unsigned need = lim == 31 ? 0xffffffffu : (1u << (lim + 1)) - 1u;
      if ((rdy & need) != need) {
        if (++spins > kLookbackSpin) {
          if (lane == 0) atomicCAS(err, 0, kErrLookback);
          break;
        }
        continue;
      }
      unsigned long long t = lane <= lim ? (w >> 32) & 0x3FFFFFull : 0ull;
      unsigned long long q = lane <= lim ? w & 0xFFFFFFFFull : 0ull;
      for (int o = 16; o > 0; o >>= 1) {
        t += __shfl_xor_sync(0xffffffffu, t, o);
        q += __shfl_xor_sync(0xffffffffu, q, o);
      }
      et += t; ep += q;
      if (incl) break;
      j -= 32;
    }
    if (lane == 0) {
      vs[vb] = lookback_word(tag, 2u, et + at, ep + ap);
      s_pt = (int)et; s_pp = (int)ep;
      if (vb == nblk - 1) {
        *total = (int)(et + at);
        *ticket = 0u;   /* every block has taken its ticket */
      }
    }
  }
  __syncthreads();
  int pos = s_pt + sv[warp] + iv - tv, off = s_pp + sw[warp] + iw - tw;
#pragma unroll
  for (int k = 0; k < kOnepassTiles; ++k) {
    const long i = i0 + k;
    if (c[k] > 0) {
      list[pos] = (int)i;
      slot[i] = pos;
      slot_off[pos] = off;
      slot_len[pos] = c[k];
      slot_cursor[pos] = 0;
      cnt[i] = 0;     /* counts start the next step at zero */
      ++pos;
      off += c[k];
    } else if (i < n) {
      slot[i] = -1;   /* the whole map is written: no clearing pass before the step */
    }
  }
}

/* The one-grid spread's lists hold entries instead of node indices: the
 * nodes of a warp (32 consecutive nodes, chunk i >> 5) that touch a tile
 * at the same stencil offset append one entry {chunk, lane mask} with one
 * atomic.  A node touches a tile at one offset only, so the masks a chunk
 * leaves in one list are disjoint; the gather merges them.  Only the
 * tiles of columns tx in [tlo, thi) are listed (an x-slab gathers the
 * force of its own columns only; the whole grid passes [0, ntx)).  The
 * eight tile offsets are walked by every lane, inactive ones included, so
 * that the warp's lanes meet at each step.  An entry's place in its list
 * depends on timing; the gather sorts the entries. */
__device__ __forceinline__ void pair_scatter_warp(const int* __restrict__ st, long i, long S, int ntx, int nty,
                                                  int nx, int ny, int nz, int tlo, int thi, const int* __restrict__ slot,
                                                  const int* __restrict__ slot_off, int* __restrict__ slot_cursor,
                                                  int2* __restrict__ ent) {
  const int lane = threadIdx.x & 31;
  int is = 0, js = 0, ks = 0;
  bool ok = i < S;
  if (ok) {
    is = st[i * 3 + 0]; js = st[i * 3 + 1]; ks = st[i * 3 + 2];
    ok = !(is < 0 || is + 3 >= nx || js < 0 || js + 3 >= ny || ks < 0 || ks + 3 >= nz);
  }
#pragma unroll
  for (int o = 0; o < 8; ++o) {
    const int tx = (is >> 2) + (o & 1), ty = (js >> 2) + ((o >> 1) & 1), tz = (ks >> 2) + (o >> 2);
    const bool here = ok && tx <= (is + 3) >> 2 && ty <= (js + 3) >> 2 && tz <= (ks + 3) >> 2 && tx >= tlo &&
                      tx < thi;
    const int s = here ? slot[((long)tz * nty + ty) * ntx + tx] : -1;
    const unsigned grp = __match_any_sync(0xffffffffu, s);
    if (!here || lane != __ffs(grp) - 1) continue;
    const int k = atomicAdd(&slot_cursor[s], 1);
    ent[slot_off[s] + k] = make_int2((int)(i >> 5), (int)grp);
  }
}

/* Longest per-tile node list sorted in shared memory; longer lists take the
 * chunk-scan path below. */
constexpr int kListCap = 1024;

/* The columns [d, d + 3] of a stencil that starts d cells from a tile's
 * origin, as a 4-bit mask of the tile's columns 0..3 (0 when |d| > 3). */
__device__ __forceinline__ unsigned span4(int d) {
  if (d >= 4 || d <= -4) return 0u;
  return d >= 0 ? (0xFu << d) & 0xFu : 0xFu >> (-d);
}

/* The 64 cells of a tile (cell = 16 z + 4 y + x) that a stencil starting at
 * (dx, dy, dz) from the tile's origin covers, as a 64-bit mask. */
__device__ __forceinline__ unsigned long long stencil_tile_mask(int dx, int dy, int dz) {
  const unsigned mx = span4(dx), my = span4(dy), mz = span4(dz);
  unsigned row = 0u;
#pragma unroll
  for (int j = 0; j < 4; ++j) row |= ((my >> j) & 1u) ? mx << (4 * j) : 0u;
  unsigned long long m = 0ull;
#pragma unroll
  for (int k = 0; k < 4; ++k) m |= ((mz >> k) & 1u) ? (unsigned long long)row << (16 * k) : 0ull;
  return m;
}

/* A staged node of the entry-list gather: its x, y and z delta weights at
 * the tile's four cell positions per axis (0 where the stencil misses the
 * position), then its force.  An odd stride of 15 doubles puts 16
 * different nodes in 16 different bank pairs. */
constexpr int kNodeRec = 15;

/* Shared memory of one entry-list gather CTA (64 threads = one 4^3 tile):
 * the list's entries as sort keys (chunk << 32 | lane mask) while the node
 * list is built, then the staged node records while they are summed. */
struct GatherSmemE {
  int ids[kListCap];                 /* the tile's nodes in index order       */
  int seg[kListCap];                 /* per entry: first node position, or -1 */
  unsigned m32[2][64];               /* per node: the cells of warp 0 / 1     */
  union {
    unsigned long long key[kListCap];
    double rec[64 * kNodeRec];
  } u;
};

/* Slot `it` (local tile `tile`) from its E entries {chunk, lane mask}: the
 * entries are sorted by chunk (bitonic, in shared memory), the masks of a
 * chunk merged, and the node list written in index order; then each of
 * the 64 threads sums its cell's contributions in node order -- the
 * reference's (sheet, row, col) order -- into Ftile[it].  The same values
 * as gather_tile. */
__device__ __forceinline__ void gather_tile_ent(GatherSmemE& sm, const double* __restrict__ nodes,
                                                const double* __restrict__ W, const int* __restrict__ st, int it,
                                                int tile, int L, int E, const int2* __restrict__ ent,
                                                int ntx, int nty, double* __restrict__ Ftile) {
  const int t = threadIdx.x;
  const double cf = 1.0 / (64.0 * 1.0 * 1.0 * 1.0);
  unsigned long long* key = sm.u.key;
  int P = 1;
  while (P < E) P <<= 1;
  __syncthreads();   /* the previous tile's data is no longer read */
  for (int k = t; k < P; k += 64) {
    unsigned long long v = ~0ull;
    if (k < E) {
      const int2 e = ent[k];
      v = ((unsigned long long)(unsigned)e.x << 32) | (unsigned)e.y;
    }
    key[k] = v;
  }
  __syncthreads();
  for (int k = 2; k <= P; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int a = t; a < P; a += 64) {
        const int b = a ^ j;
        if (b > a) {
          const unsigned long long va = key[a], vb = key[b];
          const bool up = (a & k) == 0;
          if ((va > vb) == up) { key[a] = vb; key[b] = va; }
        }
      }
      __syncthreads();
    }
  /* entries of one chunk are now adjacent: the first of each run takes the
     run's merged mask and its first position (a short serial pass) */
  if (t == 0) {
    int pos = 0;
    for (int e = 0; e < E;) {
      const unsigned ch = (unsigned)(key[e] >> 32);
      unsigned m = (unsigned)key[e];
      int f = e + 1;
      while (f < E && (unsigned)(key[f] >> 32) == ch) { m |= (unsigned)key[f]; sm.seg[f] = -1; ++f; }
      key[e] = ((unsigned long long)ch << 32) | m;
      sm.seg[e] = pos;
      pos += __popc(m);
      e = f;
    }
  }
  __syncthreads();
  for (int e = t; e < E; e += 64) {
    int pos = sm.seg[e];
    if (pos < 0) continue;
    const int base = (int)(key[e] >> 32) * 32;
    for (unsigned m = (unsigned)key[e]; m; m &= m - 1) sm.ids[pos++] = base + __ffs(m) - 1;
  }
  __syncthreads();   /* ids complete; key no longer read (aliases the node records) */
  double* rec = sm.u.rec;
  const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
  const int x0 = tx * 4, y0 = ty * 4, z0 = tz * 4;
  /* the thread's cell in a record: its x, y and z weight positions */
  const int ox = t & 3, oy = 4 + ((t >> 2) & 3), oz = 8 + (t >> 4);
  const int lane = t & 31;
  const unsigned* mw = sm.m32[t >> 5];
  double Fx = 0.0, Fy = 0.0, Fz = 0.0;
  for (int b0 = 0; b0 < L; b0 += 64) {
    const int nb = min(64, L - b0);
    if (t < nb) {
      const long nd = sm.ids[b0 + t];
      const int sx = st[nd * 3 + 0], sy = st[nd * 3 + 1], sz = st[nd * 3 + 2];
      double* r = rec + t * kNodeRec;
      const double* w = W + nd * 12;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        /* cell position c of the tile is stencil position c + (x0 - sx) */
        const int a = c + x0 - sx, b = c + y0 - sy, e = c + z0 - sz;
        r[c] = (unsigned)a < 4u ? w[a] : 0.0;
        r[4 + c] = (unsigned)b < 4u ? w[4 + b] : 0.0;
        r[8 + c] = (unsigned)e < 4u ? w[8 + e] : 0.0;
      }
      r[12] = nodes[nd * 12 + 9]; r[13] = nodes[nd * 12 + 10]; r[14] = nodes[nd * 12 + 11];
      const unsigned long long m = stencil_tile_mask(sx - x0, sy - y0, sz - z0);
      sm.m32[0][t] = (unsigned)m;
      sm.m32[1][t] = (unsigned)(m >> 32);
    }
    __syncthreads();
    /* 32 nodes at a time: the warp's 32 x 32 cover bits (node j covers
       lane l's cell) are transposed with five shuffle stages, so that
       each lane walks only the nodes that cover its cell, in node order */
    for (int j0 = 0; j0 < nb; j0 += 32) {
      unsigned x = j0 + lane < nb ? mw[j0 + lane] : 0u;
#pragma unroll
      for (int k = 16; k >= 1; k >>= 1) {
        const unsigned M = k == 16 ? 0x0000FFFFu : k == 8 ? 0x00FF00FFu : k == 4 ? 0x0F0F0F0Fu
                         : k == 2 ? 0x33333333u : 0x55555555u;
        const unsigned y = __shfl_xor_sync(0xffffffffu, x, k);
        x = (lane & k) ? (x & ~M) | ((y & ~M) >> k) : (x & M) | ((y & M) << k);
      }
      for (unsigned bits = x; bits; bits &= bits - 1u) {
        const double* r = rec + (j0 + __ffs(bits) - 1) * kNodeRec;
        const double tmp = cf * r[ox] * r[oy] * r[oz];
        Fx = Fx + r[12] * tmp;
        Fy = Fy + r[13] * tmp;
        Fz = Fz + r[14] * tmp;
      }
    }
    __syncthreads();
  }
  double* Ft = Ftile + (long)it * 192;
  Ft[t] = Fx; Ft[64 + t] = Fy; Ft[128 + t] = Fz;
}

/* Crowded tiles (more than kListCap nodes, e.g. a crumpled sheet): visit the
 * nodes chunk by chunk in global order, skipping chunks whose stencil box
 * misses the tile.  Same summation order, no list needed. */
struct ScanSmem {
  int hit[64];
  int st[32][3];
  double w[32][12];
  double fe[32][3];
};

/* Slot `it` with more than kListCap nodes: visit the node chunks
 * [c_lo, c_hi) (32 nodes each, nodes below S) in order, skipping chunks
 * whose stencil box misses the tile. */
__device__ __forceinline__ void gather_tile_scan(ScanSmem& sm, const double* __restrict__ nodes,
                                                 const double* __restrict__ W, const int* __restrict__ st,
                                                 const int* __restrict__ chunk_box, long S, long c_lo, long c_hi,
                                                 int it, int tile, int ntx, int nty, double* __restrict__ Ftile) {
  int* hit = sm.hit;
  auto& s_st = sm.st;
  auto& s_w = sm.w;
  auto& s_fe = sm.fe;
  const int cell = threadIdx.x;
  const double cf = 1.0 / (64.0 * 1.0 * 1.0 * 1.0);
  {
    const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
    const int x0 = tx * 4, y0 = ty * 4, z0 = tz * 4;
    const int gx = x0 + (cell & 3), gy = y0 + ((cell >> 2) & 3), gz = z0 + (cell >> 4);
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    for (long c0 = c_lo; c0 < c_hi; c0 += 64) {
      const long c = c0 + cell;
      int h = 0;
      if (c < c_hi) {
        const int* bx = chunk_box + c * 6;
        h = !(bx[1] < x0 || bx[0] > x0 + 3 || bx[3] < y0 || bx[2] > y0 + 3 || bx[5] < z0 || bx[4] > z0 + 3);
      }
      __syncthreads();
      hit[cell] = h;
      __syncthreads();
      for (int k = 0; k < 64; ++k) {
        if (!hit[k]) continue;
        const long base = (c0 + k) * 32;
        if (cell < 32) {
          const long nd = base + cell;
          if (nd < S) {
            s_st[cell][0] = st[nd * 3 + 0]; s_st[cell][1] = st[nd * 3 + 1]; s_st[cell][2] = st[nd * 3 + 2];
            for (int a = 0; a < 12; ++a) s_w[cell][a] = W[nd * 12 + a];
            s_fe[cell][0] = nodes[nd * 12 + 9]; s_fe[cell][1] = nodes[nd * 12 + 10]; s_fe[cell][2] = nodes[nd * 12 + 11];
          } else {
            s_st[cell][0] = INT_MIN / 2; s_st[cell][1] = INT_MIN / 2; s_st[cell][2] = INT_MIN / 2;
          }
        }
        __syncthreads();
        for (int j = 0; j < 32; ++j) {
          const int a = gx - s_st[j][0], b = gy - s_st[j][1], e = gz - s_st[j][2];
          if ((unsigned)a < 4u && (unsigned)b < 4u && (unsigned)e < 4u) {
            const double tmp = cf * s_w[j][a] * s_w[j][4 + b] * s_w[j][8 + e];
            Fx = Fx + s_fe[j][0] * tmp;
            Fy = Fy + s_fe[j][1] * tmp;
            Fz = Fz + s_fe[j][2] * tmp;
          }
        }
        __syncthreads();
      }
    }
    double* Ft = Ftile + (long)it * 192;
    Ft[cell] = Fx; Ft[64 + cell] = Fy; Ft[128 + cell] = Fz;
  }
}

/* moveFiberSheet for node i; slot maps local tiles to global slots. */
__device__ __forceinline__ void move_node(double* __restrict__ nodes, const double* __restrict__ W,
                                          const int* __restrict__ st, long i, int ntx, int nty,
                                          const int* __restrict__ slot, const double* __restrict__ Utile, double dt) {
  const double c_64 = 1.0 / (6.4e1);
  const int is = st[i * 3 + 0], js = st[i * 3 + 1], ks = st[i * 3 + 2];
  const double* w = W + i * 12;
  /* the stencil spans at most 2 tiles per axis: look their slots up first,
     so that the 64 cells' loads below do not wait on one another */
  const int tx0 = is >> 2, ty0 = js >> 2, tz0 = ks >> 2;
  int sp8[8];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int tx = tx0 + (a & 1), ty = ty0 + ((a >> 1) & 1), tz = tz0 + (a >> 2);
    const bool need = tx * 4 <= is + 3 && ty * 4 <= js + 3 && tz * 4 <= ks + 3;
    sp8[a] = need ? slot[(tz * nty + ty) * ntx + tx] : 0;
  }
  double s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
  for (int i2 = 0; i2 <= 3; i2++) {
    const int gi = is + i2;
#pragma unroll
    for (int j2 = 0; j2 <= 3; j2++) {
      const int gj = js + j2;
#pragma unroll
      for (int k2 = 0; k2 <= 3; k2++) {
        const int gk = ks + k2;
        const int sp = sp8[((gi >> 2) - tx0) | (((gj >> 2) - ty0) << 1) | (((gk >> 2) - tz0) << 2)];
        const double* U = Utile + (long)sp * 256;
        const int cell = lbib::cell_in_tile(gi, gj, gk);
        const double vx = U[64 + cell], vy = U[128 + cell], vz = U[192 + cell];
        s1 += vx * w[i2] * w[4 + j2] * w[8 + k2] * c_64;
        s2 += vy * w[i2] * w[4 + j2] * w[8 + k2] * c_64;
        s3 += vz * w[i2] * w[4 + j2] * w[8 + k2] * c_64;
      }
    }
  }
  double* m = nodes + i * 12;
  m[0] += dt * s1;
  m[1] += dt * s2;
  m[2] += dt * s3;
}


/* Cells a warp's staged move holds in shared memory: the union box of its
 * 32 nodes' stencils (along a fiber row ~5 x 20 x 5 cells); a larger
 * union (a warp straddling two rows, a crumpled sheet) takes move_node. */
constexpr int kMoveCap = 640;
constexpr int kMoveTiles = 64;   /* tiles of the union box whose slots are staged */

__device__ __forceinline__ int warp_min(int v) {
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int warp_max(int v) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

/* move_node for the 32 nodes of a warp (node i on this lane, `live` if it
 * moves), with the velocity of the union box of their stencils staged once
 * in shared memory (sU: 3 x kMoveCap doubles for this warp): the lanes
 * read each box cell's u from its moment tile with coalesced loads, then
 * every lane sums its own 64 terms from shared memory -- the same values
 * in the same order as move_node, with ~5x fewer L2 requests (neighbouring
 * nodes' stencils overlap by 3 cells of 4).  Called by all 32 lanes. */
__device__ __forceinline__ void move_warp(double* __restrict__ nodes, const double* __restrict__ W,
                                          const int* __restrict__ st, long i, bool live, int ntx, int nty,
                                          const int* __restrict__ slot, const double* __restrict__ Utile, double dt,
                                          double* __restrict__ sU) {
  const int lane = threadIdx.x & 31;
  int is = 0, js = 0, ks = 0;
  if (live) { is = st[i * 3 + 0]; js = st[i * 3 + 1]; ks = st[i * 3 + 2]; }
  const int x0 = warp_min(live ? is : INT_MAX), x1 = warp_max(live ? is + 3 : INT_MIN);
  if (x0 > x1) return;   /* no live lane */
  const int y0 = warp_min(live ? js : INT_MAX), y1 = warp_max(live ? js + 3 : INT_MIN);
  const int z0 = warp_min(live ? ks : INT_MAX), z1 = warp_max(live ? ks + 3 : INT_MIN);
  const int bx = x1 - x0 + 1, by = y1 - y0 + 1, bz = z1 - z0 + 1;
  const long vol = (long)bx * by * bz;
  const int ntiles_box = ((x1 >> 2) - (x0 >> 2) + 1) * ((y1 >> 2) - (y0 >> 2) + 1) * ((z1 >> 2) - (z0 >> 2) + 1);
  if (vol > kMoveCap || ntiles_box > kMoveTiles) {   /* uniform over the warp */
    if (live) move_node(nodes, W, st, i, ntx, nty, slot, Utile, dt);
    return;
  }
  /* the slots of the box's tiles first (at most 3 x 7 x 3 for a box that
     fits), so that the cell loads below depend on one shared-memory read */
  int* sslot = reinterpret_cast<int*>(sU + 3 * kMoveCap);
  const int tx0 = x0 >> 2, ty0 = y0 >> 2, tz0 = z0 >> 2;
  const int tbx = (x1 >> 2) - tx0 + 1, tby = (y1 >> 2) - ty0 + 1, ntb = tbx * tby * ((z1 >> 2) - tz0 + 1);
  for (int j = lane; j < ntb; j += 32) {
    const int tx = tx0 + j % tbx, ty = ty0 + (j / tbx) % tby, tz = tz0 + j / (tbx * tby);
    sslot[j] = slot[(tz * nty + ty) * ntx + tx];
  }
  __syncwarp();
  /* the box's longest axis (the fiber direction: neighbouring lanes'
     stencils are offset along it) is stored fastest, so that the lanes'
     reads below fall on consecutive words, not on one bank */
  const int f = (bx >= by && bx >= bz) ? 0 : (by >= bz ? 1 : 2);
  const int a = f == 0 ? 1 : 0, b = f == 2 ? 1 : 2;
  const int ext[3] = {bx, by, bz};
  int str[3];
  str[f] = 1; str[a] = ext[f]; str[b] = ext[f] * ext[a];
#pragma unroll 4
  for (int j = lane; j < (int)vol; j += 32) {
    int u[3];
    u[f] = j % ext[f]; u[a] = (j / ext[f]) % ext[a]; u[b] = j / (ext[f] * ext[a]);
    const int cx = x0 + u[0], cy = y0 + u[1], cz = z0 + u[2];
    /* a box corner no stencil covers may lie in an untouched tile: never read */
    const int sp = sslot[((cz >> 2) - tz0) * tbx * tby + ((cy >> 2) - ty0) * tbx + ((cx >> 2) - tx0)];
    double vx = 0.0, vy = 0.0, vz = 0.0;
    if (sp >= 0) {
      const double* U = Utile + (long)sp * 256;
      const int cell = lbib::cell_in_tile(cx, cy, cz);
      vx = U[64 + cell]; vy = U[128 + cell]; vz = U[192 + cell];
    }
    sU[j] = vx; sU[kMoveCap + j] = vy; sU[2 * kMoveCap + j] = vz;
  }
  __syncwarp();
  if (live) {
    const double c_64 = 1.0 / (6.4e1);
    const double* w = W + i * 12;
    double s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
    for (int i2 = 0; i2 <= 3; i2++) {
#pragma unroll
      for (int j2 = 0; j2 <= 3; j2++) {
#pragma unroll
        for (int k2 = 0; k2 <= 3; k2++) {
          const int c = (is + i2 - x0) * str[0] + (js + j2 - y0) * str[1] + (ks + k2 - z0) * str[2];
          const double vx = sU[c], vy = sU[kMoveCap + c], vz = sU[2 * kMoveCap + c];
          s1 += vx * w[i2] * w[4 + j2] * w[8 + k2] * c_64;
          s2 += vy * w[i2] * w[4 + j2] * w[8 + k2] * c_64;
          s3 += vz * w[i2] * w[4 + j2] * w[8 + k2] * c_64;
        }
      }
    }
    double* m = nodes + i * 12;
    m[0] += dt * s1;
    m[1] += dt * s2;
    m[2] += dt * s3;
  }
  __syncwarp();
}

}  // namespace lbib

#endif
