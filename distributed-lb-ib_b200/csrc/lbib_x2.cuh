/*
 * The FP64 fused D3Q19 step for rows away from the walls, two cells per
 * thread with 16-byte (double2) accesses: the device body shared by the
 * one-grid kernel (lbib_fluid_x2.cu) and the batched one (lbib_batch.cu).
 * Compile with -fmad=false: the arithmetic is the generic kernel's
 * (collide/moments in lbib_lattice.cuh), bit for bit.
 *
 * Cells: y in [3, ny-4], z in [3, min(nz-4, zin_hi)], x in [xlo, xhi] (the
 * state's columns of I); every link comes from a cell of I, so the only
 * special cells are the plane cells x = 2 and x = nx-3 (fixed inlet/outlet
 * table).  Rows next to the walls run
 * the one-cell-per-thread generic kernel.
 *
 * A thread owns the pair (x, x+1), x even (nx and the slab bounds are
 * even, so the x range splits into pairs).  Even step: own slots, all 19 loads and
 * stores are aligned double2.  Odd step: for the 9 directions with c_x = 0
 * the source and target pairs are aligned double2 too; for the 10 with
 * c_x = +-1 they are shifted by one cell, and the thread uses two 8-byte
 * accesses (still coalesced across the warp).
 */
#ifndef LBIB_X2_CUH
#define LBIB_X2_CUH

#include "lbib_lattice.cuh"

namespace lbib {

/* Rows, pairs and cells of the two-cell kernel's range. */
__host__ __device__ inline int x2_rows_z(int nz, int zin_hi) {
  const int zb = nz - 4 < zin_hi ? nz - 4 : zin_hi;
  return zb - 2;
}

/* Moments (previous step) and force of one cell, then the collision. */
__device__ __forceinline__ void x2_relax_cell(const FluidParams& p, int x, int y, int z, bool plane, double f[19]) {
  const int tile = tile_of(x, y, z, p.ntx, p.nty);
  const int cell = cell_in_tile(x, y, z);
  double rho, ux, uy, uz;
  if (plane) {
    rho = p.rho0; ux = p.ux0; uy = 0.0; uz = 0.0;
  } else if (p.first) {
    rho = p.rho0; ux = p.ux_rest; uy = 0.0; uz = 0.0;
  } else {
    const int sp = p.slot_prev[tile];
    if (sp >= 0) {
      const double* U = p.Uprev + (long)sp * 256;
      rho = U[cell]; ux = U[64 + cell]; uy = U[128 + cell]; uz = U[192 + cell];
    } else {
      moments(f, 0.0, 0.0, 0.0, p.half_dt, p.g, rho, ux, uy, uz);
    }
  }
  const int sc = p.box ? -1 : p.slot_cur[tile];   /* box mode: only unforced cells get here */
  if (sc >= 0) {
    const double* Ft = p.Fcur + (long)sc * 192;
    collide<true>(f, rho, ux, uy, uz, Ft[cell], Ft[64 + cell], Ft[128 + cell], p);
  } else {
    collide<false>(f, rho, ux, uy, uz, 0.0, 0.0, 0.0, p);
  }
}

/* The plane cell of a pair (x = 2: the inlet, x = nx-3: the outlet) takes
 * its populations from the fixed table (load_pre's K_TABLE rule); rows of
 * this kernel have z <= zin_hi, where every plane cell is a table cell. */
__device__ __forceinline__ void x2_plane_table(const FluidParams& p, int y, int z, bool pa, double fa[19],
                                               double fb[19]) {
  const double* t = pa ? p.inlet : p.outlet;
  const long P = (long)p.ny * p.nz, pi = (long)y * p.nz + z;
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const double v = t[q * P + pi];
    if (pa) fa[q] = v; else fb[q] = v;
  }
}

/* The step of the pair (x, x+1) of row (y, z); x even.  In an odd step a
 * pair holding a plane cell runs the same loads and stores as every other
 * pair -- the plane cell's pulled values are then replaced by its table, and
 * its pushes that would leave I (c_x = -1 at x = 2, +1 at x = nx-3) go to
 * its own slot opp(q) by an address select, store_post's rule -- so the warp
 * holding it does not diverge into the per-cell rules (1.89 -> 1.79 ms per
 * FP64 step at 512x256x256).  Its even-step loads keep the per-cell rules,
 * which measured faster there (even-step fluid 1.75 -> 1.67 ms). */
template <int PAR>
__device__ __forceinline__ void x2_pair(const FluidParams& p, int x, int y, int z) {
  if (p.box && in_box(p.box, x, y, z)) return;    /* both cells share a tile (x even) */
  const long idx = sidx(p, x, y, z);
  const bool pa = (x == 2), pb = (x + 1 == p.nx - 3);
  double* __restrict__ F = p.f;
  double fa[19], fb[19];
  double* __restrict__ Fi = F + idx;
  if (PAR == 0 && (pa || pb)) {
    /* even step: the per-cell rules (own slots; the plane cell's table) */
    load_pre<PAR>(p, x, y, z, idx, pa ? K_TABLE : K_FAST, fa);
    load_pre<PAR>(p, x + 1, y, z, idx + 1, pb ? K_TABLE : K_FAST, fb);
  } else {
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      if (PAR == 0 || cx(q) == 0) {
        const double* src = PAR ? Fi + p.pull[q] : Fi + q * p.N;
        const double2 v = *reinterpret_cast<const double2*>(src);
        fa[q] = v.x; fb[q] = v.y;
      } else {
        const double* src = Fi + p.pull[q];
        fa[q] = src[0]; fb[q] = src[1];
      }
    }
    if (pa || pb) x2_plane_table(p, y, z, pa, fa, fb);
  }
  x2_relax_cell(p, x, y, z, pa, fa);
  x2_relax_cell(p, x + 1, y, z, pb, fb);
  if (PAR == 0) {
#pragma unroll
    for (int q = 0; q < 19; ++q)
      *reinterpret_cast<double2*>(Fi + opp(q) * p.N) = make_double2(fa[q], fb[q]);
  } else {
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      double* dst = Fi + p.push[q];
      if (cx(q) == 0) {
        *reinterpret_cast<double2*>(dst) = make_double2(fa[q], fb[q]);
      } else {
        double* da = dst;
        double* db = dst + 1;
        if (cx(q) == -1) da = pa ? Fi + opp(q) * p.N : da;
        else db = pb ? Fi + 1 + opp(q) * p.N : db;
        *da = fa[q];
        *db = fb[q];
      }
    }
  }
}

}  // namespace lbib

#endif
