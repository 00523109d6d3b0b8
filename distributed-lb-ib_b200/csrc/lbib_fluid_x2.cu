/*
 * The fused D3Q19 step for rows away from the walls, two cells per thread
 * with 16-byte (double2) accesses.
 *
 * Cells: y in [3, ny-4], z in [3, min(nz-4, zin_hi)], x in [2, nx-3]; every
 * link comes from a cell of I, so the only special cells are the plane cells
 * x = 2 and x = nx-3 (fixed inlet/outlet table).  Rows next to the walls run
 * the one-cell-per-thread generic kernel of lbib_fluid.cu.
 *
 * A thread owns the pair (x, x+1), x even (nx is even, so I's x range
 * [2, nx-3] splits into pairs).  Even step: own slots, all 19 loads and
 * stores are aligned double2.  Odd step: for the 9 directions with c_x = 0
 * the source and target pairs are aligned double2 too; for the 10 with
 * c_x = +-1 they are shifted by one cell, and the thread uses two 8-byte
 * accesses (still coalesced across the warp).  Twice the bytes per memory
 * instruction of the one-cell kernel: the AA pattern alone measures 87% of
 * the HBM copy peak at one cell per thread and 96% at two.  The arithmetic
 * per cell is the generic kernel's (collide/moments in lbib_lattice.cuh).
 */
#include "lbib_internal.h"
#include "lbib_lattice.cuh"

using namespace lbib;

namespace {

constexpr int TPB = 128;

#ifndef LBIB_X2_MINB
#define LBIB_X2_MINB 3
#endif

struct X2Params {
  FluidParams p;
  int nry;       /* interior rows in y: ny - 6 */
  int npairs;    /* pairs per row: (nx - 4) / 2 */
};

/* Moments (previous step) and force of one cell, then the collision. */
__device__ __forceinline__ void relax_cell(const FluidParams& p, int x, int y, int z, bool plane, double f[19]) {
  const int tile = tile_of(x, y, z, p.ntx, p.nty);
  const int cell = cell_in_tile(x, y, z);
  double rho, ux, uy, uz;
  if (plane || p.first) {
    rho = p.rho0; ux = p.ux0; uy = 0.0; uz = 0.0;
  } else {
    const int sp = p.slot_prev[tile];
    if (sp >= 0) {
      const double* U = p.Uprev + (long)sp * 256;
      rho = U[cell]; ux = U[64 + cell]; uy = U[128 + cell]; uz = U[192 + cell];
    } else {
      moments(f, 0.0, 0.0, 0.0, p.half_dt, p.g, rho, ux, uy, uz);
    }
  }
  const int sc = p.slot_cur[tile];
  if (sc >= 0) {
    const double* Ft = p.Fcur + (long)sc * 192;
    collide<true>(f, rho, ux, uy, uz, Ft[cell], Ft[64 + cell], Ft[128 + cell], p);
  } else {
    collide<false>(f, rho, ux, uy, uz, 0.0, 0.0, 0.0, p);
  }
}

/* One cell's loads through the generic rules (plane cells, pair ends). */
template <int PAR>
__device__ __forceinline__ void load_one(const FluidParams& p, int x, int y, int z, long idx, double f[19]) {
  load_pre<PAR>(p, x, y, z, idx, (x == 2 || x == p.nx - 3) ? K_TABLE : K_FAST, f);
}

template <int PAR>
__global__ void __launch_bounds__(TPB, LBIB_X2_MINB) lbib_fluid_step_x2(X2Params b) {
  const FluidParams& p = b.p;
  const int pr = blockIdx.y * TPB + threadIdx.x;
  if (pr >= b.npairs) return;
  const int y = 3 + (int)(blockIdx.x % b.nry);
  const int z = 3 + (int)(blockIdx.x / b.nry);
  const int x = 2 + 2 * pr;
  const long idx = ((long)z * p.ny + y) * p.nx + x;
  const long N = p.N, sy = p.nx, sz = (long)p.nx * p.ny;
  const bool pa = (x == 2), pb = (x + 1 == p.nx - 3);
  double* __restrict__ F = p.f;
  double fa[19], fb[19];
  if (!pa && !pb) {
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      if (PAR == 0 || cx(q) == 0) {
        const double* src = PAR ? F + opp(q) * N + idx - link_offset(q, sy, sz) : F + q * N + idx;
        const double2 v = *reinterpret_cast<const double2*>(src);
        fa[q] = v.x; fb[q] = v.y;
      } else {
        const double* src = F + opp(q) * N + idx - link_offset(q, sy, sz);
        fa[q] = src[0]; fb[q] = src[1];
      }
    }
  } else {
    load_one<PAR>(p, x, y, z, idx, fa);
    load_one<PAR>(p, x + 1, y, z, idx + 1, fb);
  }
  relax_cell(p, x, y, z, pa, fa);
  relax_cell(p, x + 1, y, z, pb, fb);
  if (PAR == 0) {
#pragma unroll
    for (int q = 0; q < 19; ++q)
      *reinterpret_cast<double2*>(F + opp(q) * N + idx) = make_double2(fa[q], fb[q]);
  } else if (!pa && !pb) {
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      double* dst = F + q * N + idx + link_offset(q, sy, sz);
      if (cx(q) == 0) *reinterpret_cast<double2*>(dst) = make_double2(fa[q], fb[q]);
      else { dst[0] = fa[q]; dst[1] = fb[q]; }
    }
  } else {
    store_post<PAR>(p, x, y, z, idx, pa ? K_TABLE : K_FAST, fa);
    store_post<PAR>(p, x + 1, y, z, idx + 1, pb ? K_TABLE : K_FAST, fb);
  }
}

}  // namespace

/* Interior-row ranges of this kernel: y in [3, ny-4], z in
 * [3, min(nz-4, zin_hi)].  Returns 0 when there are none. */
extern "C" int lbdev_bulk_rows(const lbib_device* d, int* nrows_y, int* nrows_z) {
  *nrows_y = d->ny - 6;
  int zb = d->nz - 4;
  if (d->zin_hi < zb) zb = d->zin_hi;
  *nrows_z = zb - 2;
  return (*nrows_y > 0 && *nrows_z > 0);
}

extern "C" int lbdev_launch_fluid_bulk(lbib_device* d, const void* fluid_params) {
  X2Params b;
  b.p = *(const FluidParams*)fluid_params;
  int nrz = 0;
  if (!lbdev_bulk_rows(d, &b.nry, &nrz)) return 0;
  b.npairs = (d->nx - 4) / 2;
  dim3 grid((unsigned)((long)b.nry * nrz), (unsigned)((b.npairs + TPB - 1) / TPB));
  if (d->parity == 0) lbib_fluid_step_x2<0><<<grid, TPB, 0, d->stream>>>(b);
  else lbib_fluid_step_x2<1><<<grid, TPB, 0, d->stream>>>(b);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
