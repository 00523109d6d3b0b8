/*
 * D3Q19 lattice, the AA in-place access rules, and the reference-faithful
 * moment / equilibrium / collision arithmetic shared by the fluid kernels.
 *
 * The FP64 instantiations are compiled with -fmad=false: every expression
 * below keeps the operation order of cube_pthread/lbm_ib.c, and contraction
 * into FMA would change roundings.
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
 * Storage: a state may hold only an x-slab of the lattice (columns
 * [olo, ohi) of the global grid, plus two ghost columns on each side); all
 * coordinates in the kernels are global, and a cell's slot index is
 * ((z ny + y) sx + x - gx0) with sx the stored row length.  The whole
 * lattice is the slab [0, nx) with sx = nx, gx0 = 0.
 *
 * AA pattern (Bailey et al., 2009) in one buffer f[q][cell]:
 *   even step: read own slot q, write own slot opp(q);
 *   odd step:  read slot opp(q) of x - c_q, write slot q of x + c_q.
 * Bounce-back in both: a link whose source is outside I reads own slot q; an
 * odd-step push whose target is outside I goes to own slot opp(q).
 */
#ifndef LBIB_LATTICE_CUH
#define LBIB_LATTICE_CUH

#include <cuda_bf16.h>
#include <cuda_fp16.h>
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

/* Population storage.  R is the arithmetic type.  FP64 stores f itself.
 * The low-precision forms store the deviation d_q = f_q - s_q from a fixed
 * per-direction shift s_q (the rest weights w_q, or the equilibrium of the
 * inflow state) and do all their arithmetic on deviations in FP32, so the
 * storage bits and the FP32 mantissa are spent on the part that changes;
 * s_q == s_opp(q) for the weight shift, and the flow shift keeps the pair
 * in the parameters, so the AA phase never changes a slot's meaning. */
template <typename T> struct Pop;
template <> struct Pop<double> {
  using R = double;
  __device__ static __forceinline__ R get(double v) { return v; }
  __device__ static __forceinline__ double put(R v) { return v; }
};
template <> struct Pop<float> {
  using R = float;
  __device__ static __forceinline__ R get(float v) { return v; }
  __device__ static __forceinline__ float put(R v) { return v; }
};
template <> struct Pop<__half> {
  using R = float;
  __device__ static __forceinline__ R get(__half v) { return __half2float(v); }
  __device__ static __forceinline__ __half put(R v) { return __float2half_rn(v); }
};
template <> struct Pop<__nv_bfloat16> {
  using R = float;
  __device__ static __forceinline__ R get(__nv_bfloat16 v) { return __bfloat162float(v); }
  __device__ static __forceinline__ __nv_bfloat16 put(R v) { return __float2bfloat16_rn(v); }
};

enum CellKind { K_FAST = 0, K_WALL = 1, K_SEMI = 2, K_TABLE = 3 };

/* Everything a fluid kernel needs.  inlet/outlet hold populations in the
 * arithmetic type and in the stored representation (f for FP64, f - s_q
 * otherwise).  sh, rhos, uxs: the low-precision shift s_q and the density
 * and x velocity it carries (sum_q s_q, sum_q c_qx s_q / sum_q s_q). */
template <typename T>
struct FluidParamsT {
  using R = typename Pop<T>::R;
  T* f;
  const R* inlet;
  const R* outlet;
  long N;                /* stored cells: the slot stride */
  int nx, ny, nz;        /* the global grid */
  int sx, gx0;           /* stored row length; global x of stored column 0 */
  int olo, ohi;          /* columns this state owns: [olo, ohi) */
  int xlo, xhi;          /* columns of I it collides: [xlo, xhi] */
  int zin_hi, yskip_z0, first;
  int periodic_z;        /* option: z periodic over I (period nz - 4), walls only at y */
  double rho0, ux0;      /* moments of the plane cells and the tables (the inflow)     */
  double ux_rest;        /* initial u_x of the cells x in [3, nx-4]: ux0, 0 from rest  */
  double omtau, invtau, kw0, kw1, kw2, cs2, cs4, half_dt, g;
  const int* slot_cur;   /* F(t) tiles */
  const double* Fcur;
  const int* slot_prev;  /* (rho, u)(t-1) tiles */
  const double* Uprev;
  int ntx, nty;
  /* box mode (the fluid step overlapped with the spread): the tiles
     box[0..1] x box[2..3] x box[4..5] (inclusive, in tiles) hold every
     stencil of this step; the bulk and row kernels skip them and read no
     force, and a kernel of its own steps their cells after the spread.
     NULL: the kernels find the forced tiles through slot_cur. */
  const int* box;
  float sh[19];
  double rhos, uxs;
  /* the same constants in FP32 for the low-precision forms: rho_s, u_s,
     1 - 1/tau, 1/tau, dt/2, g, the Guo weights, 1/cs^2, 1/cs^4 */
  float frs, fus, fom, fit, fhdt, fg, fkw0, fkw1, fkw2, fcs2i, fcs4i;
  /* 1/tau times the weights, and C_q = rho_s P_q(u_s) (the shift's part of
     the deviation equilibrium) */
  float fitw0, fitw1, fitw2;
  float fC[19];
  /* element offsets from a cell's slot index for the odd step: the pull of
     direction q (slot opp(q) of x - c_q) and its push (slot q of x + c_q),
     precomputed so that a kernel forms each of its 38 addresses with one
     add */
  long pull[19], push[19];
};

/* A bounce-back link delivers this cell's own outgoing population opp(q) as
 * the incoming q; as a deviation it moves from s_opp(q) to s_q.  Before the
 * first step the slot still holds the initial population q itself. */
template <typename T>
__device__ __forceinline__ typename Pop<T>::R bounced(const FluidParamsT<T>& p, int q, typename Pop<T>::R v) {
  if constexpr (sizeof(T) == 8) return v;
  else return p.first ? v : v + (p.sh[opp(q)] - p.sh[q]);
}

/* The stored value of a population the reference holds as 0 (its calloc'd
 * df2 where nothing writes): 0, or -s_q as a deviation. */
template <typename T>
__device__ __forceinline__ typename Pop<T>::R zero_pop(const FluidParamsT<T>& p, int q) {
  if constexpr (sizeof(T) == 8) return 0.0;
  else return -p.sh[q];
}
using FluidParams = FluidParamsT<double>;

template <typename P>
__device__ __forceinline__ int classify(const P& p, int x, int y, int z) {
  if (x == 2 || x == p.nx - 3) return (z <= p.zin_hi) ? K_TABLE : K_SEMI;
  if (y == 2 || y == p.ny - 3 || z == 2 || z == p.nz - 3) return K_WALL;
  return K_FAST;
}

/* Slot index of global cell (x, y, z) in this state's storage. */
template <typename P>
__device__ __forceinline__ long sidx(const P& p, int x, int y, int z) {
  return ((long)z * p.ny + y) * p.sx + (x - p.gx0);
}

__host__ __device__ __forceinline__ long link_offset(int q, long sy, long sz) {
  return (long)cx(q) + (long)cy(q) * sy + (long)cz(q) * sz;
}

/* Ask L2 to fetch the bytes [lo, hi) of the buffer [base, end) ahead of
 * their loads (cp.async.bulk.prefetch, sm_90+): the range is widened to
 * 16-byte boundaries, as the instruction requires, and clipped to the
 * buffer.  A hint only -- no register holds the data and nothing waits on
 * it -- so a fused step can keep more DRAM traffic in flight than its
 * resident warps' loads alone. */
__device__ __forceinline__ void l2_prefetch(const void* lo, const void* hi, const void* base, const void* end) {
  uintptr_t a = (uintptr_t)lo & ~(uintptr_t)15;
  uintptr_t b = ((uintptr_t)hi + 15) & ~(uintptr_t)15;
  const uintptr_t a0 = ((uintptr_t)base + 15) & ~(uintptr_t)15, b0 = (uintptr_t)end & ~(uintptr_t)15;
  if (a < a0) a = a0;
  if (b > b0) b = b0;
  if (b > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(b - a)) : "memory");
}

/* Pre-collision populations of cell (x, y, z) in I for a step of parity PAR. */
template <int PAR, typename T>
__device__ __forceinline__ void load_pre(const FluidParamsT<T>& p, int x, int y, int z, long idx, int kind,
                                         typename Pop<T>::R f[19]) {
  using R = typename Pop<T>::R;
  const long N = p.N;
  const T* __restrict__ F = p.f;
  if (kind == K_TABLE) {
    const R* t = (x == 2) ? p.inlet : p.outlet;
    const long P = (long)p.ny * p.nz;
    const long pi = (long)y * p.nz + z;
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = t[q * P + pi];
    return;
  }
  const long sy = p.sx, sz = (long)p.sx * p.ny;
  if (kind == K_FAST) {
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = Pop<T>::get(PAR == 0 ? F[q * N + idx] : F[idx + p.pull[q]]);
    return;
  }
  const bool yskip = (kind == K_WALL) && p.yskip_z0 >= 0 && (z == p.yskip_z0 || z == p.yskip_z0 + 1);
  /* Every link's word is loaded first, from an address chosen without a
     branch (the pulled slot, or the cell's own slot q where the link's
     source lies outside I -- also where the value is then replaced by
     zero_pop), so that the 19 loads are in flight together; the rules
     are applied to the loaded values afterwards. */
  T raw[19];
  unsigned in_mask = 0u, zero_mask = 0u;
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const int xs = x - cx(q), ys = y - cy(q);
    int zs = z - cz(q);
    long wrap = 0;   /* periodic z: the source re-enters I at the other side */
    if (p.periodic_z && zs < 2) { zs += p.nz - 4; wrap = (long)(p.nz - 4) * sz; }
    if (p.periodic_z && zs > p.nz - 3) { zs -= p.nz - 4; wrap = -(long)(p.nz - 4) * sz; }
    const bool yin = ys >= 2 && ys <= p.ny - 3;
    const bool zin = zs >= 2 && zs <= p.nz - 3;
    const bool xin = xs >= 2 && xs <= p.nx - 3;
    const bool in = xin && yin && zin;
    const long a = (PAR == 0 || !in) ? q * N + idx : opp(q) * N + idx - link_offset(q, sy, sz) + wrap;
    raw[q] = F[a];
    in_mask |= (in ? 1u : 0u) << q;
    zero_mask |= ((!in && !p.first && (kind == K_SEMI || (yskip && !yin && zin))) ? 1u : 0u) << q;
  }
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const typename Pop<T>::R v = Pop<T>::get(raw[q]);
    if ((in_mask >> q) & 1u) f[q] = v;
    else f[q] = ((zero_mask >> q) & 1u) ? zero_pop(p, q) : bounced(p, q, v);
  }
}

/* Post-collision populations of cell (x, y, z) in I for a step of parity PAR. */
template <int PAR, typename T>
__device__ __forceinline__ void store_post(const FluidParamsT<T>& p, int x, int y, int z, long idx, int kind,
                                           const typename Pop<T>::R f[19]) {
  const long N = p.N;
  T* __restrict__ F = p.f;
  if (PAR == 0) {
#pragma unroll
    for (int q = 0; q < 19; ++q) F[opp(q) * N + idx] = Pop<T>::put(f[q]);
    return;
  }
  const long sy = p.sx, sz = (long)p.sx * p.ny;
  if (kind == K_FAST) {
#pragma unroll
    for (int q = 0; q < 19; ++q) F[idx + p.push[q]] = Pop<T>::put(f[q]);
    return;
  }
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const int xt = x + cx(q), yt = y + cy(q);
    int zt = z + cz(q);
    long wrap = 0;
    if (p.periodic_z && zt < 2) { zt += p.nz - 4; wrap = (long)(p.nz - 4) * sz; }
    if (p.periodic_z && zt > p.nz - 3) { zt -= p.nz - 4; wrap = -(long)(p.nz - 4) * sz; }
    const bool in = xt >= 2 && xt <= p.nx - 3 && yt >= 2 && yt <= p.ny - 3 && zt >= 2 && zt <= p.nz - 3;
    F[in ? q * N + idx + link_offset(q, sy, sz) + wrap : opp(q) * N + idx] = Pop<T>::put(f[q]);
  }
}

/* compute_rho_and_u, cube_pthread/lbm_ib.c:2493-2528: sums in q order.
 * Terms with c = 0 are dropped from the momentum sums: for finite values
 * s + 0*f == s, so the result is the same number. */
template <typename R>
__device__ __forceinline__ void moments(const R f[19], R Fx, R Fy, R Fz, R half_dt, R g, R& rho, R& ux, R& uy,
                                        R& uz) {
  R s1 = f[0];
#pragma unroll
  for (int q = 1; q < 19; ++q) s1 = s1 + f[q];
  R s2 = R(0) * f[0];
  s2 = s2 + f[1]; s2 = s2 - f[2]; s2 = s2 + f[7]; s2 = s2 - f[8]; s2 = s2 + f[9];
  s2 = s2 - f[10]; s2 = s2 + f[15]; s2 = s2 - f[16]; s2 = s2 + f[17]; s2 = s2 - f[18];
  R s3 = R(0) * f[0];
  s3 = s3 - f[5]; s3 = s3 + f[6]; s3 = s3 - f[11]; s3 = s3 + f[12]; s3 = s3 + f[13];
  s3 = s3 - f[14]; s3 = s3 - f[15]; s3 = s3 + f[16]; s3 = s3 + f[17]; s3 = s3 - f[18];
  R s4 = R(0) * f[0];
  s4 = s4 + f[3]; s4 = s4 - f[4]; s4 = s4 + f[7]; s4 = s4 - f[8]; s4 = s4 - f[9];
  s4 = s4 + f[10]; s4 = s4 + f[11]; s4 = s4 - f[12]; s4 = s4 + f[13]; s4 = s4 - f[14];
  rho = s1;
  ux = (s2 + half_dt * Fx) / s1;
  uy = (s3 + half_dt * Fy) / s1;
  uz = (s4 + half_dt * (Fz + rho * g)) / s1;
}

/* c . u for each direction, as (c0*ux + c1*uy) + c2*uz evaluates with
 * c in {0, +-1}; opposite directions give exact negatives. */
template <typename R>
__device__ __forceinline__ void velocity_dots(R ux, R uy, R uz, R cu[19]) {
  cu[0] = R(0);
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
template <typename R, typename P>
__device__ __forceinline__ R guo(int q, R ux, R uy, R uz, R Fx, R Fy, R Fzg, const P& p) {
  const R c0 = (R)cx(q), c1 = (R)cy(q), c2 = (R)cz(q);
  const R kw = (R)((q == 0) ? p.kw0 : ((q <= 6) ? p.kw1 : p.kw2));
  const R A = (c0 - ux) * Fx + (c1 - uy) * Fy + (c2 - uz) * Fzg;
  const R B = c0 * ux + c1 * uy + c2 * uz;
  const R C = c0 * Fx + c1 * Fy + c2 * Fzg;
  return kw * (A / (R)p.cs2 + B / (R)p.cs4 * C);
}

template <typename R>
struct Relax {
  R ux, uy, uz, Fx, Fy, Fzg, t6, om, it;
};

/* One opposite pair (qa, qb) with c_qa . u = cu: both equilibria share
 * 3cu, cu^2 and 1.5 u^2, and 1 + (-3cu) == 1 - 3cu exactly.  With a force
 * the Guo term is added after the relaxation, as the reference sums it. */
template <bool FORCED, int QA, int QB, typename R, typename P>
__device__ __forceinline__ void relax_pair(R* f, R cu, R wr, const Relax<R>& r, const P& p) {
  const R a3 = R(3.0) * cu;
  const R sq = R(4.5) * (cu * cu);
  const R ea = wr * (R(1.0) + a3 + sq - r.t6);
  const R eb = wr * (R(1.0) + (-a3) + sq - r.t6);
  R va = f[QA] * r.om + r.it * ea;
  R vb = f[QB] * r.om + r.it * eb;
  if (FORCED) {
    va = va + guo(QA, r.ux, r.uy, r.uz, r.Fx, r.Fy, r.Fzg, p);
    vb = vb + guo(QB, r.ux, r.uy, r.uz, r.Fx, r.Fy, r.Fzg, p);
  }
  f[QA] = va;
  f[QB] = vb;
}

template <bool FORCED, typename R, typename P>
__device__ __forceinline__ void collide(R f[19], R rho, R ux, R uy, R uz, R Fx, R Fy, R Fz, const P& p) {
  Relax<R> r;
  r.ux = ux; r.uy = uy; r.uz = uz;
  r.Fx = Fx; r.Fy = Fy; r.Fzg = FORCED ? Fz + rho * (R)p.g : R(0);
  r.t6 = R(1.5) * (ux * ux + uy * uy + uz * uz);
  r.om = (R)p.omtau; r.it = (R)p.invtau;
  const R wr0 = R(1.0 / 3.0) * rho;
  const R wr1 = R(1.0 / 18.0) * rho;
  const R wr2 = R(1.0 / 36.0) * rho;
  R v0 = f[0] * r.om + r.it * (wr0 * (R(1.0) - r.t6));
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

/* Cell (x, y, z) lies in a tile of the box (box mode). */
__device__ __forceinline__ bool in_box(const int* box, int x, int y, int z) {
  const int tx = x >> 2, ty = y >> 2, tz = z >> 2;
  return tx >= box[0] && tx <= box[1] && ty >= box[2] && ty <= box[3] && tz >= box[4] && tz <= box[5];
}

__device__ __forceinline__ int tile_of(int x, int y, int z, int ntx, int nty) {
  return ((z >> 2) * nty + (y >> 2)) * ntx + (x >> 2);
}
__device__ __forceinline__ int cell_in_tile(int x, int y, int z) {
  return ((z & 3) << 4) | ((y & 3) << 2) | (x & 3);
}

}  // namespace lbib

#endif
