/*
 * Fluid kernels: the fused in-place D3Q19 step and the moment gathers.
 *
 * lbib_fluid_step<PAR> replaces, for one time step, the reference's
 * compute_eqlbrmdistrfuncDF1 + stream_distrfunc + bounceback_rigidwalls +
 * copy_inout_to_df2 + replace_old_DF (cube_pthread/lbm_ib.c:1673-2968):
 * each cell of I reads its 19 incoming populations once and writes its 19
 * outgoing ones once (AA pattern, one buffer).  It needs the previous step's
 * moments: cells whose 4^3 tile carried force last step read them from the
 * stored tile moments; every other cell recomputes them from its incoming
 * populations, which is exact because F(t-1) = 0 there.
 *
 * HBM roofline: 19 x 8 B read + 19 x 8 B write per fluid cell = 304 B.
 */
#include "lbib_internal.h"
#include "lbib_lattice.cuh"

using namespace lbib;

namespace {

/* Resident blocks per SM the register budget is sized for (128 threads each). */
#ifndef LBIB_FLUID_MINB
#define LBIB_FLUID_MINB 4
#endif

template <int PAR>
__global__ void __launch_bounds__(128, LBIB_FLUID_MINB) lbib_fluid_step(FluidParams p, const int2* __restrict__ rows) {
  const int x = blockIdx.y * blockDim.x + threadIdx.x + 2;
  const int2 r = rows[blockIdx.x];
  const int y = r.x;
  const int z = r.y;
  if (x > p.nx - 3) return;
  const long idx = ((long)z * p.ny + y) * p.nx + x;
  const int kind = classify(p, x, y, z);
  double f[19];
  load_pre<PAR>(p, x, y, z, idx, kind, f);
  const int tile = tile_of(x, y, z, p.ntx, p.nty);
  const int cell = cell_in_tile(x, y, z);
  double rho, ux, uy, uz;
  if (kind >= K_SEMI || p.first) {
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
  store_post<PAR>(p, x, y, z, idx, kind, f);
}

/* (rho, u)(t) of every cell of the touched tiles, after the fused step of
 * parity 1-PAR: compute_rho_and_u (lbm_ib.c:2440-2538) restricted to where
 * moveFiberSheet will read.  Cells outside M keep the initial values. */
template <int PAR>
__global__ void lbib_tile_moments(FluidParams p, const int* __restrict__ list, const int* __restrict__ count,
                                  const double* __restrict__ Ftile, double* __restrict__ Utile) {
  const int n = *count;
  const int cell = threadIdx.x;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int tile = list[i];
    const int tx = tile % p.ntx, ty = (tile / p.ntx) % p.nty, tz = tile / (p.ntx * p.nty);
    const int x = tx * 4 + (cell & 3), y = ty * 4 + ((cell >> 2) & 3), z = tz * 4 + (cell >> 4);
    double rho = p.rho0, ux = p.ux0, uy = 0.0, uz = 0.0;
    if (x >= 3 && x <= p.nx - 4 && y >= 2 && y <= p.ny - 3 && z >= 2 && z <= p.nz - 3) {
      const long idx = ((long)z * p.ny + y) * p.nx + x;
      double f[19];
      load_pre<PAR>(p, x, y, z, idx, classify(p, x, y, z), f);
      const double* Ft = Ftile + (long)i * 192;
      moments(f, Ft[cell], Ft[64 + cell], Ft[128 + cell], p.half_dt, p.g, rho, ux, uy, uz);
    }
    double* U = Utile + (long)i * 256;
    U[cell] = rho; U[64 + cell] = ux; U[128 + cell] = uy; U[192 + cell] = uz;
  }
}

/* Dense rho, u over the whole grid as the reference holds them after the
 * step: M cells from the populations (with this step's force where a tile
 * carried one), all other cells at the initial values. */
template <int PAR>
__global__ void lbib_field_moments(FluidParams p, int have_step, double* __restrict__ rho_o,
                                   double* __restrict__ ux_o, double* __restrict__ uy_o,
                                   double* __restrict__ uz_o) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  if (x >= p.nx) return;
  const long idx = ((long)z * p.ny + y) * p.nx + x;
  double rho = p.rho0, ux = p.ux0, uy = 0.0, uz = 0.0;
  if (have_step && x >= 3 && x <= p.nx - 4 && y >= 2 && y <= p.ny - 3 && z >= 2 && z <= p.nz - 3) {
    double f[19];
    load_pre<PAR>(p, x, y, z, idx, classify(p, x, y, z), f);
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    const int sc = p.slot_cur[tile_of(x, y, z, p.ntx, p.nty)];
    if (sc >= 0) {
      const int cell = cell_in_tile(x, y, z);
      const double* Ft = p.Fcur + (long)sc * 192;
      Fx = Ft[cell]; Fy = Ft[64 + cell]; Fz = Ft[128 + cell];
    }
    moments(f, Fx, Fy, Fz, p.half_dt, p.g, rho, ux, uy, uz);
  }
  rho_o[idx] = rho; ux_o[idx] = ux; uy_o[idx] = uy; uz_o[idx] = uz;
}

/* df1 as the reference holds it at the start of the next step, for cells of
 * I (natural layout [q][idx]); other cells are left untouched. */
template <int PAR>
__global__ void lbib_gather_df1(FluidParams p, double* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int y = blockIdx.y + 2, z = blockIdx.z + 2;
  if (x > p.nx - 3) return;
  const long idx = ((long)z * p.ny + y) * p.nx + x;
  double f[19];
  load_pre<PAR>(p, x, y, z, idx, classify(p, x, y, z), f);
#pragma unroll
  for (int q = 0; q < 19; ++q) out[q * p.N + idx] = f[q];
}

/* init_eqlbrmdistrfuncDF0 + init_df1 (lbm_ib.c:1528-1607, 2725-2767): the
 * equilibrium of the initial (rho_l, u_l, 0, 0), written to every cell in
 * natural order; init_df_inout (lbm_ib.c:1610-1670): the same values for the
 * inlet and outlet planes. */
__global__ void lbib_init_eq(FluidParams p, double* __restrict__ f, long count, long stride) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double ux = p.ux0, uy = 0.0, uz = 0.0, rho = p.rho0;
  const double usq = ux * ux + uy * uy + uz * uz;
  const double t6 = 1.5 * usq;
  double cu[19];
  velocity_dots(ux, uy, uz, cu);
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    double v;
    if (q == 0) v = 1.0 / 3.0 * rho * (1.0 - t6);
    else v = ((q <= 6) ? 1.0 / 18.0 : 1.0 / 36.0) * rho * (1.0 + 3.0 * cu[q] + 4.5 * (cu[q] * cu[q]) - t6);
    f[q * stride + i] = v;
  }
}

FluidParams make_params(lbib_device* d, int first) {
  FluidParams p;
  p.f = d->f; p.inlet = d->inlet; p.outlet = d->outlet;
  p.N = d->N; p.nx = d->nx; p.ny = d->ny; p.nz = d->nz;
  p.zin_hi = d->zin_hi; p.yskip_z0 = d->yskip_z0; p.first = first;
  p.rho0 = d->rho_l; p.ux0 = d->u_l;
  p.omtau = d->omtau; p.invtau = d->invtau;
  p.kw0 = d->kw[0]; p.kw1 = d->kw[1]; p.kw2 = d->kw[2];
  p.cs2 = d->cs2; p.cs4 = d->cs4; p.half_dt = d->half_dt; p.g = d->g_l;
  const int c = d->cur;
  p.slot_cur = d->tile_slot[c]; p.Fcur = d->Ftile[c];
  p.slot_prev = d->tile_slot[c ^ 1]; p.Uprev = d->Utile[c ^ 1];
  p.ntx = d->ntx; p.nty = d->nty;
  return p;
}

}  // namespace

extern "C" int lbdev_launch_fluid_bulk(lbib_device* d, const void* fluid_params);

/* One fused step: the generic kernel over d->rows (all rows of I, or only
 * the rows next to the walls when the staged kernel takes the others). */
extern "C" int lbdev_launch_fluid_step(lbib_device* d) {
  FluidParams p = make_params(d, d->steps == 0);
  if (d->nrows > 0) {
    dim3 block(128);
    dim3 grid((unsigned)d->nrows, (unsigned)((d->nx - 4 + 127) / 128));
    if (d->parity == 0) lbib_fluid_step<0><<<grid, block, 0, d->stream>>>(p, (const int2*)d->rows);
    else lbib_fluid_step<1><<<grid, block, 0, d->stream>>>(p, (const int2*)d->rows);
    d->kernel_launches++;
  }
  if (d->use_bulk && lbdev_launch_fluid_bulk(d, &p)) return -2;
  d->parity ^= 1;
  d->steps++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int lbdev_launch_tile_moments(lbib_device* d) {
  FluidParams p = make_params(d, 0);
  const int c = d->cur;
  int blocks = 148 * 16;
  if (d->parity == 0)
    lbib_tile_moments<0><<<blocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], d->Ftile[c], d->Utile[c]);
  else
    lbib_tile_moments<1><<<blocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], d->Ftile[c], d->Utile[c]);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int lbdev_launch_field_moments(lbib_device* d, double* rho, double* ux, double* uy, double* uz) {
  FluidParams p = make_params(d, 0);
  dim3 block(128);
  dim3 grid((unsigned)((d->nx + 127) / 128), (unsigned)d->ny, (unsigned)d->nz);
  const int have = d->steps > 0 && d->have_forces;
  if (d->parity == 0) lbib_field_moments<0><<<grid, block, 0, d->stream>>>(p, have, rho, ux, uy, uz);
  else lbib_field_moments<1><<<grid, block, 0, d->stream>>>(p, have, rho, ux, uy, uz);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int lbdev_launch_gather_df1(lbib_device* d, double* out) {
  FluidParams p = make_params(d, d->steps == 0);
  dim3 block(128);
  dim3 grid((unsigned)((d->nx - 4 + 127) / 128), (unsigned)(d->ny - 4), (unsigned)(d->nz - 4));
  if (d->parity == 0) lbib_gather_df1<0><<<grid, block, 0, d->stream>>>(p, out);
  else lbib_gather_df1<1><<<grid, block, 0, d->stream>>>(p, out);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int lbdev_launch_init_eq(lbib_device* d, double* f, long count, long stride) {
  FluidParams p = make_params(d, 1);
  const int block = 256;
  const long grid = (count + block - 1) / block;
  lbib_init_eq<<<(unsigned)grid, block, 0, d->stream>>>(p, f, count, stride);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
