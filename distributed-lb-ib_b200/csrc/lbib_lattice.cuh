/*
 * D3Q19 lattice, the AA in-place access rules, and the reference-faithful
 * moment / equilibrium / collision arithmetic shared by the fluid kernels.
 *
 * Compile with -fmad=false: every expression below keeps the operation order
 * of cube_pthread/lbm_ib.c, and contraction into FMA would change roundings.
 *
 * Which cells do what (reference semantics, internal axes, x = flow):
 *   I = [2, nx-3] x [2, ny-3] x [2, nz-3]  cells that collide (lbm_ib.c:1700-1712)
 *   M = [3, nx-4] x [2, ny-3] x [2, nz-3]  cells whose rho, u are updated
 *                                           (lbm_ib.c:2484-2491); rho, u stay at
 *                                           their initial values elsewhere
 *   x = 2 and x = nx-3 ("planes"): their df1 is reset every step to the fixed
 *   inlet / outlet equilibrium by copy_inout_to_df2 + replace_old_DF
 *   (lbm_ib.c:2769-2968) for z <= zin_hi.
 * A link q of cell x whose source x - c_q is outside I carries
 *   - the half-way bounce-back value f*_opp(q)(x) for cells of M
 *     (bounceback_rigidwalls, lbm_ib.c:2257-2437);
 *   - 0 where the reference never writes df2 (its calloc'd initial value):
 *     plane cells above zin_hi, and y-wall cells in the two z rows that the
 *     num_cubes_x clip skips (yskip_z0, yskip_z0+1), for links from outside
 *     in y only -- from the second step on.
 *
 * AA pattern (Bailey et al., 2009) in one buffer f[q][cell]:
 *   even step: read own slot q, write own slot opp(q);
 *   odd step:  read slot opp(q) of x - c_q, write slot q of x + c_q.
 * Bounce-back in both: a link whose source is outside I reads own slot q; an
 * odd-step push whose target is outside I goes to own slot opp(q).
 */
#ifndef LBIB_LATTICE_CUH
#define LBIB_LATTICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

namespace lbib {

/* cube_pthread/lbm_ib.c:777-833 */
__host__ __device__ constexpr int cx(int q) {
  return (q == 1 || q == 7 || q == 9 || q == 15 || q == 17) ? 1
       : (q == 2 || q == 8 || q == 10 || q == 16 || q == 18) ? -1 : 0;
}
__host__ __device__ constexpr int cy(int q) {
  return (q == 6 || q == 12 || q == 13 || q == 16 || q == 17) ? 1
       : (q == 5 || q == 11 || q == 14 || q == 15 || q == 18) ? -1 : 0;
}
__host__ __device__ constexpr int cz(int q) {
  return (q == 3 || q == 7 || q == 10 || q == 11 || q == 13) ? 1
       : (q == 4 || q == 8 || q == 9 || q == 12 || q == 14) ? -1 : 0;
}
__host__ __device__ constexpr int opp(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }

enum CellKind { K_FAST = 0, K_WALL = 1, K_SEMI = 2, K_TABLE = 3 };

struct FluidParams {
  double* f;
  const double* inlet;
  const double* outlet;
  long N;
  int nx, ny, nz;
  int zin_hi, yskip_z0, first;
  double rho0, ux0;
  double omtau, invtau, kw0, kw1, kw2, cs2, cs4, half_dt, g;
  const int* slot_cur;   /* F(t) tiles */
  const double* Fcur;
  const int* slot_prev;  /* (rho, u)(t-1) tiles */
  const double* Uprev;
  int ntx, nty;
};

__device__ __forceinline__ int classify(const FluidParams& p, int x, int y, int z) {
  if (x == 2 || x == p.nx - 3) return (z <= p.zin_hi) ? K_TABLE : K_SEMI;
  if (y == 2 || y == p.ny - 3 || z == 2 || z == p.nz - 3) return K_WALL;
  return K_FAST;
}

__device__ __forceinline__ long link_offset(int q, long sy, long sz) {
  return (long)cx(q) + (long)cy(q) * sy + (long)cz(q) * sz;
}

/* Pre-collision populations of cell (x, y, z) in I for a step of parity PAR. */
template <int PAR>
__device__ __forceinline__ void load_pre(const FluidParams& p, int x, int y, int z, long idx, int kind,
                                         double f[19]) {
  const long N = p.N;
  const double* __restrict__ F = p.f;
  if (kind == K_TABLE) {
    const double* t = (x == 2) ? p.inlet : p.outlet;
    const long P = (long)p.ny * p.nz;
    const long pi = (long)y * p.nz + z;
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = t[q * P + pi];
    return;
  }
  const long sy = p.nx, sz = (long)p.nx * p.ny;
  if (kind == K_FAST) {
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      if (PAR == 0) f[q] = F[q * N + idx];
      else f[q] = F[opp(q) * N + idx - link_offset(q, sy, sz)];
    }
    return;
  }
  const bool yskip = (kind == K_WALL) && p.yskip_z0 >= 0 && (z == p.yskip_z0 || z == p.yskip_z0 + 1);
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const int xs = x - cx(q), ys = y - cy(q), zs = z - cz(q);
    const bool yin = ys >= 2 && ys <= p.ny - 3;
    const bool zin = zs >= 2 && zs <= p.nz - 3;
    const bool xin = xs >= 2 && xs <= p.nx - 3;
    if (xin && yin && zin) {
      if (PAR == 0) f[q] = F[q * N + idx];
      else f[q] = F[opp(q) * N + idx - link_offset(q, sy, sz)];
    } else {
      const bool zero = !p.first && (kind == K_SEMI || (yskip && !yin && zin));
      f[q] = zero ? 0.0 : F[q * N + idx];
    }
  }
}

/* Post-collision populations of cell (x, y, z) in I for a step of parity PAR. */
template <int PAR>
__device__ __forceinline__ void store_post(const FluidParams& p, int x, int y, int z, long idx, int kind,
                                           const double f[19]) {
  const long N = p.N;
  double* __restrict__ F = p.f;
  if (PAR == 0) {
#pragma unroll
    for (int q = 0; q < 19; ++q) F[opp(q) * N + idx] = f[q];
    return;
  }
  const long sy = p.nx, sz = (long)p.nx * p.ny;
  if (kind == K_FAST) {
#pragma unroll
    for (int q = 0; q < 19; ++q) F[q * N + idx + link_offset(q, sy, sz)] = f[q];
    return;
  }
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const int xt = x + cx(q), yt = y + cy(q), zt = z + cz(q);
    const bool in = xt >= 2 && xt <= p.nx - 3 && yt >= 2 && yt <= p.ny - 3 && zt >= 2 && zt <= p.nz - 3;
    if (in) F[q * N + idx + link_offset(q, sy, sz)] = f[q];
    else F[opp(q) * N + idx] = f[q];
  }
}

/* compute_rho_and_u, cube_pthread/lbm_ib.c:2493-2528: sums in q order.
 * Terms with c = 0 are dropped from the momentum sums: for finite values
 * s + 0*f == s, so the result is the same number. */
__device__ __forceinline__ void moments(const double f[19], double Fx, double Fy, double Fz, double half_dt,
                                        double g, double& rho, double& ux, double& uy, double& uz) {
  double s1 = f[0];
#pragma unroll
  for (int q = 1; q < 19; ++q) s1 = s1 + f[q];
  double s2 = 0.0 * f[0];
  s2 = s2 + f[1]; s2 = s2 - f[2]; s2 = s2 + f[7]; s2 = s2 - f[8]; s2 = s2 + f[9];
  s2 = s2 - f[10]; s2 = s2 + f[15]; s2 = s2 - f[16]; s2 = s2 + f[17]; s2 = s2 - f[18];
  double s3 = 0.0 * f[0];
  s3 = s3 - f[5]; s3 = s3 + f[6]; s3 = s3 - f[11]; s3 = s3 + f[12]; s3 = s3 + f[13];
  s3 = s3 - f[14]; s3 = s3 - f[15]; s3 = s3 + f[16]; s3 = s3 + f[17]; s3 = s3 - f[18];
  double s4 = 0.0 * f[0];
  s4 = s4 + f[3]; s4 = s4 - f[4]; s4 = s4 + f[7]; s4 = s4 - f[8]; s4 = s4 - f[9];
  s4 = s4 + f[10]; s4 = s4 + f[11]; s4 = s4 - f[12]; s4 = s4 + f[13]; s4 = s4 - f[14];
  rho = s1;
  ux = (s2 + half_dt * Fx) / s1;
  uy = (s3 + half_dt * Fy) / s1;
  uz = (s4 + half_dt * (Fz + rho * g)) / s1;
}

/* c . u for each direction, as (c0*ux + c1*uy) + c2*uz evaluates with
 * c in {0, +-1}; opposite directions give exact negatives. */
__device__ __forceinline__ void velocity_dots(double ux, double uy, double uz, double cu[19]) {
  cu[0] = 0.0;
  cu[1] = ux;        cu[2] = -ux;
  cu[3] = uz;        cu[4] = -uz;
  cu[5] = -uy;       cu[6] = uy;
  cu[7] = ux + uz;   cu[8] = -cu[7];
  cu[9] = ux - uz;   cu[10] = -cu[9];
  cu[11] = uz - uy;  cu[12] = -cu[11];
  cu[13] = uy + uz;  cu[14] = -cu[13];
  cu[15] = ux - uy;  cu[16] = -cu[15];
  cu[17] = ux + uy;  cu[18] = -cu[17];
}

/* compute_eqlbrmdistrfuncDF1, cube_pthread/lbm_ib.c:1713-1807: equilibrium
 * and BGK relaxation, in place on f.  With a force the Guo term is added as
 * written there (true divisions by cs^2 and cs^4); without one that term is
 * +-0 in the reference and is skipped. */
/* Guo forcing term of direction q as lbm_ib.c:1740-1754 writes it. */
__device__ __forceinline__ double guo(int q, double ux, double uy, double uz, double Fx, double Fy, double Fzg,
                                      const FluidParams& p) {
  const double c0 = (double)cx(q), c1 = (double)cy(q), c2 = (double)cz(q);
  const double kw = (q == 0) ? p.kw0 : ((q <= 6) ? p.kw1 : p.kw2);
  const double A = (c0 - ux) * Fx + (c1 - uy) * Fy + (c2 - uz) * Fzg;
  const double B = c0 * ux + c1 * uy + c2 * uz;
  const double C = c0 * Fx + c1 * Fy + c2 * Fzg;
  return kw * (A / p.cs2 + B / p.cs4 * C);
}

struct Relax {
  double ux, uy, uz, Fx, Fy, Fzg, t6, om, it;
};

/* One opposite pair (qa, qb) with c_qa . u = cu: both equilibria share
 * 3cu, cu^2 and 1.5 u^2, and 1 + (-3cu) == 1 - 3cu exactly.  With a force
 * the Guo term is added after the relaxation, as the reference sums it. */
template <bool FORCED, int QA, int QB>
__device__ __forceinline__ void relax_pair(double* f, double cu, double wr, const Relax& r, const FluidParams& p) {
  const double a3 = 3.0 * cu;
  const double sq = 4.5 * (cu * cu);
  const double ea = wr * (1.0 + a3 + sq - r.t6);
  const double eb = wr * (1.0 + (-a3) + sq - r.t6);
  double va = f[QA] * r.om + r.it * ea;
  double vb = f[QB] * r.om + r.it * eb;
  if (FORCED) {
    va = va + guo(QA, r.ux, r.uy, r.uz, r.Fx, r.Fy, r.Fzg, p);
    vb = vb + guo(QB, r.ux, r.uy, r.uz, r.Fx, r.Fy, r.Fzg, p);
  }
  f[QA] = va;
  f[QB] = vb;
}

template <bool FORCED>
__device__ __forceinline__ void collide(double f[19], double rho, double ux, double uy, double uz,
                                        double Fx, double Fy, double Fz, const FluidParams& p) {
  Relax r;
  r.ux = ux; r.uy = uy; r.uz = uz;
  r.Fx = Fx; r.Fy = Fy; r.Fzg = FORCED ? Fz + rho * p.g : 0.0;
  r.t6 = 1.5 * (ux * ux + uy * uy + uz * uz);
  r.om = p.omtau; r.it = p.invtau;
  const double wr0 = 1.0 / 3.0 * rho;
  const double wr1 = 1.0 / 18.0 * rho;
  const double wr2 = 1.0 / 36.0 * rho;
  double v0 = f[0] * r.om + r.it * (wr0 * (1.0 - r.t6));
  if (FORCED) v0 = v0 + guo(0, ux, uy, uz, Fx, Fy, r.Fzg, p);
  f[0] = v0;
  relax_pair<FORCED, 1, 2>(f, ux, wr1, r, p);
  relax_pair<FORCED, 3, 4>(f, uz, wr1, r, p);
  relax_pair<FORCED, 6, 5>(f, uy, wr1, r, p);
  relax_pair<FORCED, 7, 8>(f, ux + uz, wr2, r, p);
  relax_pair<FORCED, 9, 10>(f, ux - uz, wr2, r, p);
  relax_pair<FORCED, 11, 12>(f, uz - uy, wr2, r, p);
  relax_pair<FORCED, 13, 14>(f, uy + uz, wr2, r, p);
  relax_pair<FORCED, 15, 16>(f, ux - uy, wr2, r, p);
  relax_pair<FORCED, 17, 18>(f, ux + uy, wr2, r, p);
}

__device__ __forceinline__ int tile_of(int x, int y, int z, int ntx, int nty) {
  return ((z >> 2) * nty + (y >> 2)) * ntx + (x >> 2);
}
__device__ __forceinline__ int cell_in_tile(int x, int y, int z) {
  return ((z & 3) << 4) | ((y & 3) << 2) | (x & 3);
}

}  // namespace lbib

#endif
