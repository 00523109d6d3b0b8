/*
 * Fluid kernels, templated on the population storage type T (double, float,
 * __half, __nv_bfloat16; arithmetic in Pop<T>::R), and their launchers.
 *
 * lbib_fluid_step<T, PAR> replaces, for one time step, the reference's
 * compute_eqlbrmdistrfuncDF1 + stream_distrfunc + bounceback_rigidwalls +
 * copy_inout_to_df2 + replace_old_DF (cube_pthread/lbm_ib.c:1673-2968):
 * each cell of I reads its 19 incoming populations once and writes its 19
 * outgoing ones once (AA pattern, one buffer).  It needs the previous step's
 * moments: cells whose 4^3 tile carried force last step read them from the
 * stored tile moments; every other cell recomputes them from its incoming
 * populations, which is exact because F(t-1) = 0 there.
 *
 * HBM roofline: 2 x 19 x sizeof(T) bytes per fluid cell (304 B for FP64,
 * 76 B for the 16-bit forms).
 *
 * lbib_fluid.cu instantiates T = double in a translation unit compiled with
 * -fmad=false (bit-faithful to the reference); lbib_fluid_lp.cu instantiates
 * the other types with contraction allowed.
 */
#ifndef LBIB_FLUID_KERNELS_CUH
#define LBIB_FLUID_KERNELS_CUH

#include "lbib_internal.h"
#include <climits>

#include "lbib_lattice.cuh"

namespace lbib {

/* Resident blocks per SM the register budget is sized for (128 threads each). */
#ifndef LBIB_FLUID_MINB
#define LBIB_FLUID_MINB 4
#endif

/* The equilibrium of the initial (rho_l, u_l, 0, 0), as
 * init_eqlbrmdistrfuncDF0 writes it (lbm_ib.c:1528-1607). */
template <typename R>
__host__ __device__ __forceinline__ R init_feq(int q, R rho, R ux) {
  const R uy = R(0), uz = R(0);
  const R usq = ux * ux + uy * uy + uz * uz;
  const R t6 = R(1.5) * usq;
  if (q == 0) return R(1.0 / 3.0) * rho * (R(1.0) - t6);
  const R cu = (R)cx(q) * ux;
  return R((q <= 6) ? 1.0 / 18.0 : 1.0 / 36.0) * rho * (R(1.0) + R(3.0) * cu + R(4.5) * (cu * cu) - t6);
}

/* Moments of a cell in the form its collision takes. */
template <typename R>
struct Mom {
  R rho, ux, uy, uz;
};

/* What the Guo term of a low-precision collision needs. */
struct LpForce {
  float ux, uy, uz, Fx, Fy, Fzg;
};

/* Guo forcing term of direction q with the FP32 constants. */
template <typename P>
__device__ __forceinline__ float lp_guo(int q, const LpForce& c, const P& p) {
  const float c0 = (float)cx(q), c1 = (float)cy(q), c2 = (float)cz(q);
  const float kw = (q == 0) ? p.fkw0 : ((q <= 6) ? p.fkw1 : p.fkw2);
  const float A = (c0 - c.ux) * c.Fx + (c1 - c.uy) * c.Fy + (c2 - c.uz) * c.Fzg;
  const float B = c0 * c.ux + c1 * c.uy + c2 * c.uz;
  const float C = c0 * c.Fx + c1 * c.Fy + c2 * c.Fzg;
  return kw * (A * p.fcs2i + B * p.fcs4i * C);
}

/* Deviation-form BGK (+ Guo) for one opposite pair (qa, qb), c_qa = -c_qb,
 * a = c_qa.u.  With P_q(u) = 3 c.u + 4.5 (c.u)^2 - 1.5 u^2 and the shift
 * s_q = w_q rho_s (1 + P_q(u_s)):
 *   feq_q - s_q = w_q (drho + rho P_q(u) - C_q),  C_q = rho_s P_q(u_s),
 * a sum of small terms (C_q is a per-direction constant), so FP32 keeps
 * the digits the deviations carry. */
template <bool FORCED, int QA, int QB, typename P>
__device__ __forceinline__ void lp_pair(float* d, float a, float itw, float drho, float rho, float t, float om,
                                        const LpForce& c, const P& p) {
  const float sq = 4.5f * a * a - t;
  const float xa = (drho - p.fC[QA]) + rho * (sq + 3.0f * a);
  const float xb = (drho - p.fC[QB]) + rho * (sq - 3.0f * a);
  float va = d[QA] * om + itw * xa;
  float vb = d[QB] * om + itw * xb;
  if (FORCED) {
    va += lp_guo(QA, c, p);
    vb += lp_guo(QB, c, p);
  }
  d[QA] = va;
  d[QB] = vb;
}

/* Form<T>: how the kernels turn populations into moments and collide.
 * FP64: absolute (rho, u) and the reference's own arithmetic.  The
 * low-precision forms: deviations d_q = f_q - s_q, drho = rho - rho_s,
 * du = u - u_s (u_s = (uxs, 0, 0)), all in FP32. */
template <typename T, bool LOW = (sizeof(T) < 8)>
struct Form;

template <typename T>
struct Form<T, false> {
  using R = double;
  using P = FluidParamsT<T>;
  static __device__ __forceinline__ void initial(const P& p, Mom<R>& m) {
    m.rho = p.rho0; m.ux = p.ux0; m.uy = 0.0; m.uz = 0.0;
  }
  /* the first step's moments of a cell x in [3, nx-4] */
  static __device__ __forceinline__ void initial_bulk(const P& p, Mom<R>& m) {
    m.rho = p.rho0; m.ux = p.ux_rest; m.uy = 0.0; m.uz = 0.0;
  }
  static __device__ __forceinline__ void from_tile(const P&, const double* U, int cell, Mom<R>& m) {
    m.rho = U[cell]; m.ux = U[64 + cell]; m.uy = U[128 + cell]; m.uz = U[192 + cell];
  }
  static __device__ __forceinline__ void moments(const R f[19], R Fx, R Fy, R Fz, const P& p, Mom<R>& m) {
    lbib::moments(f, Fx, Fy, Fz, p.half_dt, p.g, m.rho, m.ux, m.uy, m.uz);
  }
  static __device__ __forceinline__ void moments_free(const R f[19], const P& p, Mom<R>& m) {
    lbib::moments(f, 0.0, 0.0, 0.0, p.half_dt, p.g, m.rho, m.ux, m.uy, m.uz);
  }
  template <bool FORCED>
  static __device__ __forceinline__ void collide(R f[19], const Mom<R>& m, R Fx, R Fy, R Fz, const P& p) {
    lbib::collide<FORCED>(f, m.rho, m.ux, m.uy, m.uz, Fx, Fy, Fz, p);
  }
  static __device__ __forceinline__ void to_double(const Mom<R>& m, const P&, double& rho, double& ux,
                                                   double& uy, double& uz) {
    rho = m.rho; ux = m.ux; uy = m.uy; uz = m.uz;
  }
  static __device__ __forceinline__ double value(R v, int, const P&) { return v; }
  static __device__ __forceinline__ R stored_initial(int q, double rho, double ux, const P&) {
    return init_feq<double>(q, rho, ux);
  }
};

template <typename T>
struct Form<T, true> {
  using R = float;
  using P = FluidParamsT<T>;
  static __device__ __forceinline__ void initial(const P& p, Mom<R>& m) {
    m.rho = (float)(p.rho0 - p.rhos); m.ux = (float)(p.ux0 - p.uxs); m.uy = 0.0f; m.uz = 0.0f;
  }
  static __device__ __forceinline__ void initial_bulk(const P& p, Mom<R>& m) {
    m.rho = (float)(p.rho0 - p.rhos); m.ux = (float)(p.ux_rest - p.uxs); m.uy = 0.0f; m.uz = 0.0f;
  }
  static __device__ __forceinline__ void from_tile(const P& p, const double* U, int cell, Mom<R>& m) {
    m.rho = (float)(U[cell] - p.rhos); m.ux = (float)(U[64 + cell] - p.uxs);
    m.uy = (float)U[128 + cell]; m.uz = (float)U[192 + cell];
  }
  static __device__ __forceinline__ void moments(const R d[19], R Fx, R Fy, R Fz, const P& p, Mom<R>& m) {
    /* pairwise sums: short dependency chains, small magnitudes */
    const float m0 = ((d[0] + d[1]) + (d[2] + d[3])) + ((d[4] + d[5]) + (d[6] + d[7]));
    const float m1 = ((d[8] + d[9]) + (d[10] + d[11])) + ((d[12] + d[13]) + (d[14] + d[15]));
    const float drho = (m0 + m1) + ((d[16] + d[17]) + d[18]);
    const float jx = ((d[1] - d[2]) + (d[7] - d[8])) + ((d[9] - d[10]) + (d[15] - d[16])) + (d[17] - d[18]);
    const float jy = ((d[6] - d[5]) + (d[12] - d[11])) + ((d[13] - d[14]) + (d[16] - d[15])) + (d[17] - d[18]);
    const float jz = ((d[3] - d[4]) + (d[7] - d[8])) + ((d[10] - d[9]) + (d[11] - d[12])) + (d[13] - d[14]);
    const float rho = p.frs + drho;
    const float inv = __frcp_rn(rho);
    m.rho = drho;
    m.ux = (jx + p.fhdt * Fx - drho * p.fus) * inv;
    m.uy = (jy + p.fhdt * Fy) * inv;
    m.uz = (jz + p.fhdt * (Fz + rho * p.fg)) * inv;
  }
  template <bool FORCED>
  static __device__ __forceinline__ void collide(R d[19], const Mom<R>& m, R Fx, R Fy, R Fz, const P& p) {
    const float drho = m.rho, rho = p.frs + drho;
    const float ux = p.fus + m.ux, uy = m.uy, uz = m.uz;
    const float t = 1.5f * (ux * ux + uy * uy + uz * uz);
    const float om = p.fom, i1 = p.fitw1, i2 = p.fitw2;
    LpForce c;
    if (FORCED) { c.ux = ux; c.uy = uy; c.uz = uz; c.Fx = Fx; c.Fy = Fy; c.Fzg = Fz + rho * p.fg; }
    float v0 = d[0] * om + p.fitw0 * ((drho - p.fC[0]) - rho * t);
    if (FORCED) v0 += lp_guo(0, c, p);
    d[0] = v0;
    lp_pair<FORCED, 1, 2>(d, ux, i1, drho, rho, t, om, c, p);
    lp_pair<FORCED, 3, 4>(d, uz, i1, drho, rho, t, om, c, p);
    lp_pair<FORCED, 6, 5>(d, uy, i1, drho, rho, t, om, c, p);
    lp_pair<FORCED, 7, 8>(d, ux + uz, i2, drho, rho, t, om, c, p);
    lp_pair<FORCED, 9, 10>(d, ux - uz, i2, drho, rho, t, om, c, p);
    lp_pair<FORCED, 11, 12>(d, uz - uy, i2, drho, rho, t, om, c, p);
    lp_pair<FORCED, 13, 14>(d, uy + uz, i2, drho, rho, t, om, c, p);
    lp_pair<FORCED, 15, 16>(d, ux - uy, i2, drho, rho, t, om, c, p);
    lp_pair<FORCED, 17, 18>(d, ux + uy, i2, drho, rho, t, om, c, p);
  }
  /* moments without force: the unforced cells' common case */
  static __device__ __forceinline__ void moments_free(const R d[19], const P& p, Mom<R>& m) {
    const float m0 = ((d[0] + d[1]) + (d[2] + d[3])) + ((d[4] + d[5]) + (d[6] + d[7]));
    const float m1 = ((d[8] + d[9]) + (d[10] + d[11])) + ((d[12] + d[13]) + (d[14] + d[15]));
    const float drho = (m0 + m1) + ((d[16] + d[17]) + d[18]);
    const float jx = ((d[1] - d[2]) + (d[7] - d[8])) + ((d[9] - d[10]) + (d[15] - d[16])) + (d[17] - d[18]);
    const float jy = ((d[6] - d[5]) + (d[12] - d[11])) + ((d[13] - d[14]) + (d[16] - d[15])) + (d[17] - d[18]);
    const float jz = ((d[3] - d[4]) + (d[7] - d[8])) + ((d[10] - d[9]) + (d[11] - d[12])) + (d[13] - d[14]);
    const float inv = __frcp_rn(p.frs + drho);
    m.rho = drho;
    m.ux = (jx - drho * p.fus) * inv;
    m.uy = jy * inv;
    m.uz = jz * inv;
  }
  static __device__ __forceinline__ void to_double(const Mom<R>& m, const P& p, double& rho, double& ux,
                                                   double& uy, double& uz) {
    rho = p.rhos + (double)m.rho; ux = p.uxs + (double)m.ux; uy = m.uy; uz = m.uz;
  }
  static __device__ __forceinline__ double value(R v, int q, const P& p) { return (double)p.sh[q] + (double)v; }
  static __device__ __forceinline__ R stored_initial(int q, double rho, double ux, const P& p) {
    return (float)(init_feq<double>(q, rho, ux) - (double)p.sh[q]);
  }
};

/* One cell of I through the generic rules: load, moments, collision, store. */
template <typename T, int PAR>
__device__ __forceinline__ void step_cell(const FluidParamsT<T>& p, int x, int y, int z) {
  using R = typename Pop<T>::R;
  const long idx = sidx(p, x, y, z);
  const int kind = classify(p, x, y, z);
  R f[19];
  load_pre<PAR>(p, x, y, z, idx, kind, f);
  const int tile = tile_of(x, y, z, p.ntx, p.nty);
  const int cell = cell_in_tile(x, y, z);
  using F = Form<T>;
  Mom<R> m;
  if (kind >= K_SEMI) {
    F::initial(p, m);
  } else if (p.first) {
    F::initial_bulk(p, m);
  } else {
    const int sp = p.slot_prev[tile];
    if (sp >= 0) F::from_tile(p, p.Uprev + (long)sp * 256, cell, m);
    else F::moments_free(f, p, m);
  }
  /* box mode: a cell outside the box carries no force, and this step's
     tile map may still be under construction by the concurrent spread */
  const int sc = (p.box && !in_box(p.box, x, y, z)) ? -1 : p.slot_cur[tile];
  if (sc >= 0) {
    const double* Ft = p.Fcur + (long)sc * 192;
    F::template collide<true>(f, m, (R)Ft[cell], (R)Ft[64 + cell], (R)Ft[128 + cell], p);
  } else {
    F::template collide<false>(f, m, R(0), R(0), R(0), p);
  }
  store_post<PAR>(p, x, y, z, idx, kind, f);
}

template <typename T, int PAR>
__global__ void __launch_bounds__(128, LBIB_FLUID_MINB)
    lbib_fluid_step(FluidParamsT<T> p, const int2* __restrict__ rows) {
  const int x = blockIdx.y * blockDim.x + threadIdx.x + p.xlo;
  const int2 r = rows[blockIdx.x];
  if (x > p.xhi) return;
  if (p.box && in_box(p.box, x, r.x, r.y)) return;
  step_cell<T, PAR>(p, x, r.x, r.y);
}

/* Box mode: every cell of I in the tiles of the box, by the generic rules
 * (forced where this step's spread touched the tile), one CTA of 64
 * threads per tile, a persistent grid over the box. */
template <typename T, int PAR>
__global__ void __launch_bounds__(64) lbib_box_cells(FluidParamsT<T> p, int* __restrict__ reset) {
  /* the next step's box starts empty; the move fills it (it runs after us) */
  if (reset && blockIdx.x == 0 && threadIdx.x < 6) reset[threadIdx.x] = (threadIdx.x & 1) ? INT_MIN : INT_MAX;
  const int* b = p.box;
  const long lbx = (long)b[1] - b[0] + 1, lby = (long)b[3] - b[2] + 1, lbz = (long)b[5] - b[4] + 1;
  if (lbx <= 0 || lby <= 0 || lbz <= 0) return;
  const int nbx = (int)lbx, nby = (int)lby, nbz = (int)lbz;
  const long n = (long)nbx * nby * nbz;
  const int cell = threadIdx.x;
  for (long i = blockIdx.x; i < n; i += gridDim.x) {
    const int tx = b[0] + (int)(i % nbx), ty = b[2] + (int)((i / nbx) % nby), tz = b[4] + (int)(i / ((long)nbx * nby));
    const int x = tx * 4 + (cell & 3), y = ty * 4 + ((cell >> 2) & 3), z = tz * 4 + (cell >> 4);
    if (x >= p.xlo && x <= p.xhi && y >= 2 && y <= p.ny - 3 && z >= 2 && z <= p.nz - 3) step_cell<T, PAR>(p, x, y, z);
  }
}

template <typename T>
int launch_box_cells_t(lbib_device* d, const FluidParamsT<T>& p) {
  const unsigned blocks = 148 * 16;
  if (d->parity == 0) lbib_box_cells<T, 0><<<blocks, 64, 0, d->stream>>>(p, d->box_next);
  else lbib_box_cells<T, 1><<<blocks, 64, 0, d->stream>>>(p, d->box_next);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* (rho, u)(t) of cell `cell` of touched tile `tile` (slot i), after the
 * fused step of parity 1-PAR: compute_rho_and_u (lbm_ib.c:2440-2538)
 * restricted to where moveFiberSheet will read.  Cells outside M keep the
 * initial values.  Returns false for a tile outside this state's columns
 * (another slab owns it; the values are not computed). */
template <typename T, int PAR>
__device__ __forceinline__ bool tile_moment_values(const FluidParamsT<T>& p, int tile, int i, int cell,
                                                   const double* __restrict__ Ftile, double& rho, double& ux,
                                                   double& uy, double& uz) {
  using R = typename Pop<T>::R;
  const int tx = tile % p.ntx, ty = (tile / p.ntx) % p.nty, tz = tile / (p.ntx * p.nty);
  if (tx * 4 < p.olo || tx * 4 >= p.ohi) return false;
  const int x = tx * 4 + (cell & 3), y = ty * 4 + ((cell >> 2) & 3), z = tz * 4 + (cell >> 4);
  rho = p.rho0; ux = (x >= 3 && x <= p.nx - 4) ? p.ux_rest : p.ux0; uy = 0.0; uz = 0.0;
  if (x >= 3 && x <= p.nx - 4 && y >= 2 && y <= p.ny - 3 && z >= 2 && z <= p.nz - 3) {
    const long idx = sidx(p, x, y, z);
    R f[19];
    load_pre<PAR>(p, x, y, z, idx, classify(p, x, y, z), f);
    const double* Ft = Ftile + (long)i * 192;
    Mom<R> m;
    Form<T>::moments(f, (R)Ft[cell], (R)Ft[64 + cell], (R)Ft[128 + cell], p, m);
    Form<T>::to_double(m, p, rho, ux, uy, uz);
  }
  return true;
}

/* The same into slot i of Utile.  A tile outside this state's columns gets
 * -0.0, the identity of a sum, so that adding the tiles of all slabs gives
 * every value with its bits. */
template <typename T, int PAR>
__device__ __forceinline__ void tile_moments_cell(const FluidParamsT<T>& p, int tile, int i, int cell,
                                                  const double* __restrict__ Ftile, double* __restrict__ Utile) {
  double rho, ux, uy, uz;
  if (!tile_moment_values<T, PAR>(p, tile, i, cell, Ftile, rho, ux, uy, uz)) rho = ux = uy = uz = -0.0;
  double* U = Utile + (long)i * 256;
  U[cell] = rho; U[64 + cell] = ux; U[128 + cell] = uy; U[192 + cell] = uz;
}

/* Slot i of the touched-tile list: tile list[i]. */
template <typename T, int PAR>
__global__ void lbib_tile_moments(FluidParamsT<T> p, const int* __restrict__ list, const int* __restrict__ count,
                                  const double* __restrict__ Ftile, double* __restrict__ Utile) {
  const int n = *count;
  for (int i = blockIdx.x; i < n; i += gridDim.x) tile_moments_cell<T, PAR>(p, list[i], i, threadIdx.x, Ftile, Utile);
}

/* Dense rho, u over the grid as the reference holds them after the step:
 * M cells from the populations (with this step's force where a tile carried
 * one), all other cells at the initial values; this state's columns only,
 * written at their global index. */
template <typename T, int PAR>
__global__ void lbib_field_moments(FluidParamsT<T> p, int have_step, double* __restrict__ rho_o,
                                   double* __restrict__ ux_o, double* __restrict__ uy_o,
                                   double* __restrict__ uz_o) {
  using R = typename Pop<T>::R;
  const int x = blockIdx.x * blockDim.x + threadIdx.x + p.olo;
  const int y = blockIdx.y, z = blockIdx.z;
  if (x >= p.ohi) return;
  const long idx = sidx(p, x, y, z);
  double rho = p.rho0, ux = (x >= 3 && x <= p.nx - 4) ? p.ux_rest : p.ux0, uy = 0.0, uz = 0.0;
  if (have_step && x >= 3 && x <= p.nx - 4 && y >= 2 && y <= p.ny - 3 && z >= 2 && z <= p.nz - 3) {
    R f[19];
    load_pre<PAR>(p, x, y, z, idx, classify(p, x, y, z), f);
    R Fx = R(0), Fy = R(0), Fz = R(0);
    const int sc = p.slot_cur[tile_of(x, y, z, p.ntx, p.nty)];
    if (sc >= 0) {
      const int cell = cell_in_tile(x, y, z);
      const double* Ft = p.Fcur + (long)sc * 192;
      Fx = (R)Ft[cell]; Fy = (R)Ft[64 + cell]; Fz = (R)Ft[128 + cell];
    }
    Mom<R> m;
    Form<T>::moments(f, Fx, Fy, Fz, p, m);
    Form<T>::to_double(m, p, rho, ux, uy, uz);
  }
  const long g = ((long)z * p.ny + y) * p.nx + x;
  rho_o[g] = rho; ux_o[g] = ux; uy_o[g] = uy; uz_o[g] = uz;
}

/* df1 as the reference holds it at the start of the next step, for this
 * state's cells of I (natural layout [q][idx] of the global grid); other
 * cells are left untouched. */
template <typename T, int PAR>
__global__ void lbib_gather_df1(FluidParamsT<T> p, double* __restrict__ out) {
  using R = typename Pop<T>::R;
  const int x = blockIdx.x * blockDim.x + threadIdx.x + p.xlo;
  const int y = blockIdx.y + 2, z = blockIdx.z + 2;
  if (x > p.xhi) return;
  const long idx = sidx(p, x, y, z);
  R f[19];
  load_pre<PAR>(p, x, y, z, idx, classify(p, x, y, z), f);
  const long G = (long)p.nx * p.ny * p.nz, g = ((long)z * p.ny + y) * p.nx + x;
#pragma unroll
  for (int q = 0; q < 19; ++q) out[q * G + g] = Form<T>::value(f[q], q, p);
}

/* FP64 mass and momentum of the populations of I as the next step reads
 * them, one partial per (y, z) row.  Each block owns a row; its 128 threads
 * stride over x and the block sum is a fixed tree, so the result does not
 * depend on scheduling. */
template <typename T, int PAR>
__global__ void __launch_bounds__(128) lbib_row_sums(FluidParamsT<T> p, double* __restrict__ part) {
  using R = typename Pop<T>::R;
  const int y = blockIdx.x + 2, z = blockIdx.y + 2;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int x = threadIdx.x + p.xlo; x <= p.xhi; x += blockDim.x) {
    const long idx = sidx(p, x, y, z);
    R f[19];
    load_pre<PAR>(p, x, y, z, idx, classify(p, x, y, z), f);
    double m = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      const double v = Form<T>::value(f[q], q, p);
      m += v;
      if (cx(q)) jx += cx(q) > 0 ? v : -v;
      if (cy(q)) jy += cy(q) > 0 ? v : -v;
      if (cz(q)) jz += cz(q) > 0 ? v : -v;
    }
    s0 += m; s1 += jx; s2 += jy; s3 += jz;
  }
  __shared__ double sh[4][128];
  sh[0][threadIdx.x] = s0; sh[1][threadIdx.x] = s1; sh[2][threadIdx.x] = s2; sh[3][threadIdx.x] = s3;
  __syncthreads();
  for (int w = 64; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) part[((long)blockIdx.y * gridDim.x + blockIdx.x) * 4 + threadIdx.x] = sh[threadIdx.x][0];
}

/* Sum of n row partials [n][4] in a fixed order: thread t adds rows t,
 * t + 256, ... in turn, then a fixed tree. */
static __global__ void __launch_bounds__(256) lbib_sum_rows(const double* __restrict__ part, long n, double* __restrict__ out) {
  __shared__ double sh[4][256];
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (long r = threadIdx.x; r < n; r += 256)
    for (int k = 0; k < 4; ++k) s[k] += part[r * 4 + k];
  for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = sh[threadIdx.x][0];
}

/* init_df1 (lbm_ib.c:2725-2767): every cell in natural order; from rest
 * (an option) the cells x in [3, nx-4] start at u = 0. */
template <typename T>
__global__ void lbib_init_pop(FluidParamsT<T> p, T* __restrict__ f, long count) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int x = (int)(i % p.sx) + p.gx0;
  const double ux = (x >= 3 && x <= p.nx - 4) ? p.ux_rest : p.ux0;
#pragma unroll
  for (int q = 0; q < 19; ++q) f[q * count + i] = Pop<T>::put(Form<T>::stored_initial(q, p.rho0, ux, p));
}

/* init_df_inout (lbm_ib.c:1610-1670): the fixed inlet/outlet planes. */
template <typename T>
__global__ void lbib_init_table(FluidParamsT<T> p, typename Pop<T>::R* __restrict__ t, long count) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
#pragma unroll
  for (int q = 0; q < 19; ++q) t[q * count + i] = Form<T>::stored_initial(q, p.rho0, p.ux0, p);
}

template <typename T>
FluidParamsT<T> make_params_t(lbib_device* d, int first) {
  using R = typename Pop<T>::R;
  FluidParamsT<T> p;
  p.f = (T*)d->f; p.inlet = (const R*)d->inlet; p.outlet = (const R*)d->outlet;
  p.N = d->Ns; p.nx = d->nx; p.ny = d->ny; p.nz = d->nz;
  p.sx = d->sx; p.gx0 = d->gx0; p.olo = d->x_lo; p.ohi = d->x_hi;
  p.xlo = d->x_lo > 2 ? d->x_lo : 2;
  p.xhi = d->x_hi - 1 < d->nx - 3 ? d->x_hi - 1 : d->nx - 3;
  p.zin_hi = d->zin_hi; p.yskip_z0 = d->yskip_z0; p.first = first;
  p.periodic_z = (d->compat & LBIB_OPT_PERIODIC_Z) != 0;
  p.rho0 = d->rho_l; p.ux0 = d->u_l;
  p.ux_rest = (d->compat & LBIB_OPT_REST_START) ? 0.0 : d->u_l;
  p.omtau = d->omtau; p.invtau = d->invtau;
  p.kw0 = d->kw[0]; p.kw1 = d->kw[1]; p.kw2 = d->kw[2];
  p.cs2 = d->cs2; p.cs4 = d->cs4; p.half_dt = d->half_dt; p.g = d->g_l;
  const int c = d->cur;
  p.slot_cur = d->tile_slot[c]; p.Fcur = d->Ftile[c];
  p.slot_prev = d->tile_slot[c ^ 1]; p.Uprev = d->Utile[c ^ 1];
  p.ntx = d->ntx; p.nty = d->nty;
  p.box = d->box_mode ? d->box + 6 * d->box_cur : nullptr;
  lbdev_shift(d, p.sh, &p.rhos, &p.uxs);
  p.frs = (float)p.rhos; p.fus = (float)p.uxs;
  p.fom = (float)p.omtau; p.fit = (float)p.invtau; p.fhdt = (float)p.half_dt; p.fg = (float)p.g;
  p.fkw0 = (float)p.kw0; p.fkw1 = (float)p.kw1; p.fkw2 = (float)p.kw2;
  p.fcs2i = (float)(1.0 / p.cs2); p.fcs4i = (float)(1.0 / p.cs4);
  p.fitw0 = (float)(p.invtau / 3.0); p.fitw1 = (float)(p.invtau / 18.0); p.fitw2 = (float)(p.invtau / 36.0);
  for (int q = 0; q < 19; ++q) {
    const double a0 = cx(q) * p.uxs;
    p.fC[q] = (float)(p.rhos * (3.0 * a0 + 4.5 * a0 * a0 - 1.5 * p.uxs * p.uxs));
  }
  const long sy = p.sx, sz = (long)p.sx * p.ny;
  for (int q = 0; q < 19; ++q) {
    p.pull[q] = opp(q) * p.N - link_offset(q, sy, sz);
    p.push[q] = q * p.N + link_offset(q, sy, sz);
  }
  return p;
}

/* The generic kernel over d->rows. */
template <typename T>
int launch_step_rows_t(lbib_device* d, const FluidParamsT<T>& p) {
  if (d->nrows <= 0) return 0;
  dim3 block(128);
  dim3 grid((unsigned)d->nrows, (unsigned)((p.xhi - p.xlo + 1 + 127) / 128));
  if (d->parity == 0) lbib_fluid_step<T, 0><<<grid, block, 0, d->fluid_stream>>>(p, (const int2*)d->rows);
  else lbib_fluid_step<T, 1><<<grid, block, 0, d->fluid_stream>>>(p, (const int2*)d->rows);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename T>
int launch_tile_moments_t(lbib_device* d) {
  FluidParamsT<T> p = make_params_t<T>(d, 0);
  const int c = d->cur;
  const int blocks = 148 * 16;
  if (d->parity == 0)
    lbib_tile_moments<T, 0><<<blocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], d->Ftile[c], d->Utile[c]);
  else
    lbib_tile_moments<T, 1><<<blocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], d->Ftile[c], d->Utile[c]);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename T>
int launch_field_moments_t(lbib_device* d, double* rho, double* ux, double* uy, double* uz) {
  FluidParamsT<T> p = make_params_t<T>(d, 0);
  dim3 block(128);
  dim3 grid((unsigned)((p.ohi - p.olo + 127) / 128), (unsigned)d->ny, (unsigned)d->nz);
  const int have = d->steps > 0 && d->have_forces;
  if (d->parity == 0) lbib_field_moments<T, 0><<<grid, block, 0, d->stream>>>(p, have, rho, ux, uy, uz);
  else lbib_field_moments<T, 1><<<grid, block, 0, d->stream>>>(p, have, rho, ux, uy, uz);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename T>
int launch_gather_df1_t(lbib_device* d, double* out) {
  FluidParamsT<T> p = make_params_t<T>(d, d->steps == 0);
  dim3 block(128);
  dim3 grid((unsigned)((p.xhi - p.xlo + 1 + 127) / 128), (unsigned)(d->ny - 4), (unsigned)(d->nz - 4));
  if (d->parity == 0) lbib_gather_df1<T, 0><<<grid, block, 0, d->stream>>>(p, out);
  else lbib_gather_df1<T, 1><<<grid, block, 0, d->stream>>>(p, out);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* Mass and momentum sums into out[4] (device); part holds (ny-4)(nz-4)*4
 * doubles. */
template <typename T>
int launch_sums_t(lbib_device* d, double* part, double* out) {
  FluidParamsT<T> p = make_params_t<T>(d, d->steps == 0);
  dim3 grid((unsigned)(d->ny - 4), (unsigned)(d->nz - 4));
  if (d->parity == 0) lbib_row_sums<T, 0><<<grid, 128, 0, d->stream>>>(p, part);
  else lbib_row_sums<T, 1><<<grid, 128, 0, d->stream>>>(p, part);
  lbib_sum_rows<<<1, 256, 0, d->stream>>>(part, (long)(d->ny - 4) * (d->nz - 4), out);
  d->kernel_launches += 2;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <typename T>
int launch_init_t(lbib_device* d, int what) {
  using R = typename Pop<T>::R;
  FluidParamsT<T> p = make_params_t<T>(d, 1);
  const int block = 256;
  if (what == 0) {
    lbib_init_pop<T><<<(unsigned)((d->Ns + block - 1) / block), block, 0, d->stream>>>(p, (T*)d->f, d->Ns);
  } else {
    const long P = (long)d->ny * d->nz;
    lbib_init_table<T><<<(unsigned)((P + block - 1) / block), block, 0, d->stream>>>(p, (R*)d->inlet, P);
    lbib_init_table<T><<<(unsigned)((P + block - 1) / block), block, 0, d->stream>>>(p, (R*)d->outlet, P);
    d->kernel_launches++;
  }
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace lbib

#endif
