/*
 * The low-precision bulk fluid step, as device code shared by the one-grid
 * kernels (lbib_fluid_lp.cu) and the batched ones (lbib_batch_lp.cu).
 *
 * A thread owns V = 8 / sizeof(T) (or 4 / sizeof(T)) consecutive cells
 * (x0 = V g) of a row away from the walls and moves every population plane
 * as one aligned word.  Even step: own slots, aligned.  Odd step, c_x = 0:
 * aligned too.  Odd step, c_x = +-1: the V values a thread needs are its own
 * word shifted by one element, the missing element coming from the
 * neighbouring lane's word (one 32-bit shuffle and a byte_perm); pushes are
 * assembled the same way before the store.  Rows are packed end to end in
 * the thread space (a warp may hold the end of one row and the start of the
 * next): the groups that collide here never are a row's first or last word,
 * so their neighbouring words are always the next lanes' of the same row,
 * or lie across a warp edge.  At a warp edge (lane 0 / 31) the
 * element crosses to another warp, and the thread that owns the pushing cell
 * reads and writes it with a scalar access -- the AA rule that a slot is
 * read and written only by the cell that pushes into it keeps that
 * race-free.  Groups whose tile carries force this step, and the cells
 * x in {2, 3, nx-4, nx-3}, are left to the generic per-cell rules
 * (forced_cell in a launch of its own; edge_cell, run by the word blocks
 * after their words for the rows whose first word they hold); their words
 * are still loaded by idle lanes so the shuffles see them, and no two
 * threads write the same element.
 */
#ifndef LBIB_WORDS_CUH
#define LBIB_WORDS_CUH

#include <stdint.h>

#include <type_traits>

#include "lbib_fluid_kernels.cuh"

namespace lbib {

constexpr int WTPB = 128;

/* Two FP32 lanes in one 64-bit register, for sm_100's packed FP32
 * add / sub / mul / fma (each lane rounds as the scalar instruction does):
 * the word kernel collides two neighbouring cells with one instruction. */
struct F2 {
  unsigned long long v;
};
__device__ __forceinline__ F2 f2(float a, float b) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ F2 f2(float a) { return f2(a, a); }
__device__ __forceinline__ void split(F2 x, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x.v)); }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
  F2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
  F2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
/* a * b + c */
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) {
  F2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

/* V populations of one plane, V cells apart by one in x, as NR = V S / 4
 * 32-bit registers (S = sizeof(T)); element e sits in register e S / 4,
 * 16-bit elements low half first. */
template <typename T, int V>
struct Word {
  static constexpr int S = (int)sizeof(T);
  static constexpr int NR = V * S / 4;
  using U = typename std::conditional<S == 2, uint16_t, uint32_t>::type;
  uint32_t r[NR];

  __device__ __forceinline__ void load(const U* a) {
    if constexpr (NR == 4) {
      const uint4 v = *reinterpret_cast<const uint4*>(a);
      r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = v.w;
    } else if constexpr (NR == 2) {
      const uint2 v = *reinterpret_cast<const uint2*>(a);
      r[0] = v.x; r[1] = v.y;
    } else {
      r[0] = *reinterpret_cast<const uint32_t*>(a);
    }
  }
  __device__ __forceinline__ void store(U* a) const {
    if constexpr (NR == 4) *reinterpret_cast<uint4*>(a) = make_uint4(r[0], r[1], r[2], r[3]);
    else if constexpr (NR == 2) *reinterpret_cast<uint2*>(a) = make_uint2(r[0], r[1]);
    else *reinterpret_cast<uint32_t*>(a) = r[0];
  }
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int i = 0; i < NR; ++i) r[i] = 0u;
  }
  /* element e as raw bits */
  __device__ __forceinline__ U elem(int e) const {
    if constexpr (S == 2) return (U)(r[e >> 1] >> (16 * (e & 1)));
    else return r[e];
  }
  /* the V values as floats */
  __device__ __forceinline__ void unpack(float* out, int stride) const {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
      if constexpr (S == 4) {
        out[i * stride] = __uint_as_float(r[i]);
      } else if constexpr (std::is_same<T, __half>::value) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&r[i]));
        out[(2 * i) * stride] = f.x; out[(2 * i + 1) * stride] = f.y;
      } else {
        const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r[i]));
        out[(2 * i) * stride] = f.x; out[(2 * i + 1) * stride] = f.y;
      }
    }
  }
  __device__ __forceinline__ void pack(const float* in, int stride) {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
      if constexpr (S == 4) {
        r[i] = __float_as_uint(in[i * stride]);
      } else if constexpr (std::is_same<T, __half>::value) {
        const __half2 h = __floats2half2_rn(in[(2 * i) * stride], in[(2 * i + 1) * stride]);
        r[i] = *reinterpret_cast<const uint32_t*>(&h);
      } else {
        const __nv_bfloat162 h = __floats2bfloat162_rn(in[(2 * i) * stride], in[(2 * i + 1) * stride]);
        r[i] = *reinterpret_cast<const uint32_t*>(&h);
      }
    }
  }
  /* [left neighbour's last element, own 0 .. V-2]; hi = the register of the
     left word that holds its last element */
  __device__ __forceinline__ Word shifted_up(uint32_t hi) const {
    Word o;
    if constexpr (S == 4) {
      o.r[0] = hi;
#pragma unroll
      for (int i = 1; i < NR; ++i) o.r[i] = r[i - 1];
    } else {
      o.r[0] = __byte_perm(hi, r[0], 0x5432);
#pragma unroll
      for (int i = 1; i < NR; ++i) o.r[i] = __byte_perm(r[i - 1], r[i], 0x5432);
    }
    return o;
  }
  /* [own 1 .. V-1, right neighbour's first element]; lo = the register of
     the right word that holds its first element */
  __device__ __forceinline__ Word shifted_down(uint32_t lo) const {
    Word o;
    if constexpr (S == 4) {
#pragma unroll
      for (int i = 0; i < NR - 1; ++i) o.r[i] = r[i + 1];
      o.r[NR - 1] = lo;
    } else {
#pragma unroll
      for (int i = 0; i < NR - 1; ++i) o.r[i] = __byte_perm(r[i], r[i + 1], 0x5432);
      o.r[NR - 1] = __byte_perm(r[NR - 1], lo, 0x5432);
    }
    return o;
  }
};

/* Division of n < 2^31 by a fixed d in [1, 2^31) with one multiply-high and
 * one add (the round-up method for invariant divisors, Granlund and
 * Montgomery 1994): l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
 * n / d = (umulhi(n, m) + n) >> l.  The kernels' thread indices are below
 * 2^31, and a 64-bit division costs tens of instructions per thread. */
struct FastDiv {
  unsigned d, m, l;
};

__host__ __forceinline__ FastDiv fast_div(unsigned d) {
  FastDiv f;
  unsigned l = 0;
  while ((1ull << l) < d) ++l;
  f.d = d;
  f.l = l;
  f.m = (unsigned)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
  return f;
}

__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv& f) { return (__umulhi(n, f.m) + n) >> f.l; }

template <typename T>
struct WordsParams {
  FluidParamsT<T> p;
  int nry;      /* bulk rows in y */
  long nrows;   /* bulk rows */
  int ngroups;  /* words per x row: nx / V */
  int gpr;      /* threads per row: ngroups (rows packed end to end) */
  int g0, g1;   /* groups whose cells all lie in [4, nx-5] */
  long pf;      /* L2 prefetch distance in blocks (0: none) */
  FastDiv dgpr, dnry;  /* division by gpr and by nry */
};

/* Where a thread's V cells sit and what it does with them. */
struct ItemCtx {
  long row;                  /* index of (0, y, z) */
  int y, z, x0;
  bool loads, active, left_active, right_active;
};

/* Groups in [g0, g1] whose tile carries no force this step are collided
 * here; forced tiles go to lbib_forced_cells. */
template <typename T, int V>
__device__ __forceinline__ bool group_here(const WordsParams<T>& b, int g, int y, int z) {
  if (!(g >= b.g0 && g <= b.g1)) return false;
  if (b.p.box) return !in_box(b.p.box, g * V, y, z);   /* V <= 4: a group is inside one tile */
  return b.p.slot_cur[tile_of(g * V, y, z, b.p.ntx, b.p.nty)] < 0;
}

/* t < 2^31 (the launchers check it).  A row's first and last words are
 * never active, so the neighbouring words' flags are the neighbouring
 * lanes' own, also across the end of a row; only lanes 0 and 31 look
 * theirs up. */
template <typename T, int V>
__device__ __forceinline__ ItemCtx item_ctx(const WordsParams<T>& b, long t) {
  ItemCtx c;
  const unsigned tu = (unsigned)t;
  const unsigned r = fdiv(tu, b.dgpr);
  const int g = (int)(tu - r * (unsigned)b.gpr);
  const bool inrow = r < (unsigned long)b.nrows;
  const unsigned rz = fdiv(r, b.dnry);
  c.y = 3 + (int)(r - rz * (unsigned)b.nry);
  c.z = 3 + (int)rz;
  c.x0 = g * V;
  c.loads = inrow && g < b.ngroups;
  c.active = inrow && group_here<T, V>(b, g, c.y, c.z);
  const int lane = threadIdx.x & 31;
  c.left_active = __shfl_up_sync(0xffffffffu, c.active, 1);
  c.right_active = __shfl_down_sync(0xffffffffu, c.active, 1);
  if (lane == 0) c.left_active = inrow && group_here<T, V>(b, g - 1, c.y, c.z);
  if (lane == 31) c.right_active = inrow && group_here<T, V>(b, g + 1, c.y, c.z);
  c.row = ((long)c.z * b.p.ny + c.y) * b.p.nx;
  return c;
}

/* Address of the word direction q reads before its shift: own slot q for
 * an even step, slot opp(q) of the row x - c_q lies in for an odd one. */
template <typename T, int PAR>
__device__ __forceinline__ const typename Word<T, 2>::U* word_src(const FluidParamsT<T>& p, const ItemCtx& c, int q) {
  using U = typename Word<T, 2>::U;
  const U* F = reinterpret_cast<const U*>(p.f);
  const long sy = p.nx, sz = (long)p.nx * p.ny;
  if (PAR == 0) return F + q * p.N + c.row + c.x0;
  (void)sy; (void)sz;
  return F + c.row + c.x0 + (p.pull[q] + cx(q));   /* the aligned word; the x shift is done in registers */
}

/* The 4-byte aligned word that holds the element a lane at a warp edge needs
 * from beyond its warp: x0 - 1 (in the high half for 16-bit storage) when
 * c_x = +1, x0 + V (low half) when c_x = -1. */
template <typename T, int V>
__device__ __forceinline__ const void* edge_src(const typename Word<T, V>::U* src, int dir) {
  if (dir > 0) return sizeof(T) == 2 ? (const void*)(src - 2) : (const void*)(src - 1);
  return (const void*)(src + V);
}

/* Form<T, true>::moments_free and collide<false> for two cells at once,
 * the same operations lane by lane. */
template <typename P>
__device__ __forceinline__ void moments_free2(const F2 d[19], const P& p, F2& drho, F2& dux, F2& duy, F2& duz) {
  const F2 m0 = ((d[0] + d[1]) + (d[2] + d[3])) + ((d[4] + d[5]) + (d[6] + d[7]));
  const F2 m1 = ((d[8] + d[9]) + (d[10] + d[11])) + ((d[12] + d[13]) + (d[14] + d[15]));
  drho = (m0 + m1) + ((d[16] + d[17]) + d[18]);
  const F2 jx = ((d[1] - d[2]) + (d[7] - d[8])) + ((d[9] - d[10]) + (d[15] - d[16])) + (d[17] - d[18]);
  const F2 jy = ((d[6] - d[5]) + (d[12] - d[11])) + ((d[13] - d[14]) + (d[16] - d[15])) + (d[17] - d[18]);
  const F2 jz = ((d[3] - d[4]) + (d[7] - d[8])) + ((d[10] - d[9]) + (d[11] - d[12])) + (d[13] - d[14]);
  float r0, r1;
  split(f2(p.frs) + drho, r0, r1);
  const F2 inv = f2(__frcp_rn(r0), __frcp_rn(r1));
  dux = fma2(drho, f2(-p.fus), jx) * inv;
  duy = jy * inv;
  duz = jz * inv;
}

template <int QA, int QB, typename P>
__device__ __forceinline__ void lp_pair2(F2* d, F2 a, F2 itw, F2 drho, F2 rho, F2 t, F2 om, const P& p) {
  const F2 sq = fma2(f2(4.5f) * a, a, f2(0.0f) - t);
  const F2 xa = fma2(rho, fma2(f2(3.0f), a, sq), drho - f2(p.fC[QA]));
  const F2 xb = fma2(rho, fma2(f2(-3.0f), a, sq), drho - f2(p.fC[QB]));
  d[QA] = fma2(d[QA], om, itw * xa);
  d[QB] = fma2(d[QB], om, itw * xb);
}

template <typename P>
__device__ __forceinline__ void collide2(F2 d[19], F2 drho, F2 dux, F2 duy, F2 duz, const P& p) {
  const F2 rho = f2(p.frs) + drho;
  const F2 ux = f2(p.fus) + dux, uy = duy, uz = duz;
  const F2 t = f2(1.5f) * fma2(ux, ux, fma2(uy, uy, uz * uz));
  const F2 om = f2(p.fom), i1 = f2(p.fitw1), i2 = f2(p.fitw2);
  d[0] = fma2(d[0], om, f2(p.fitw0) * ((drho - f2(p.fC[0])) - rho * t));
  lp_pair2<1, 2>(d, ux, i1, drho, rho, t, om, p);
  lp_pair2<3, 4>(d, uz, i1, drho, rho, t, om, p);
  lp_pair2<6, 5>(d, uy, i1, drho, rho, t, om, p);
  lp_pair2<7, 8>(d, ux + uz, i2, drho, rho, t, om, p);
  lp_pair2<9, 10>(d, ux - uz, i2, drho, rho, t, om, p);
  lp_pair2<11, 12>(d, uz - uy, i2, drho, rho, t, om, p);
  lp_pair2<13, 14>(d, uy + uz, i2, drho, rho, t, om, p);
  lp_pair2<15, 16>(d, ux - uy, i2, drho, rho, t, om, p);
  lp_pair2<17, 18>(d, ux + uy, i2, drho, rho, t, om, p);
}

/* Ask L2 for the words block blk of the flattened (bulk row, word) space
 * will load: per plane and row, the cells its threads cover plus one on
 * either side (the odd step's x shifts). */
template <typename T, int V, int PAR>
__device__ __forceinline__ void words_prefetch(const WordsParams<T>& b, long blk) {
  const long t0 = blk * WTPB, t1 = t0 + WTPB - 1;
  const long r0 = t0 / b.gpr;
  if (r0 >= b.nrows) return;
  const long r1 = t1 / b.gpr < b.nrows ? t1 / b.gpr : b.nrows - 1;
  const int nr = (int)(r1 - r0 + 1);
  const FluidParamsT<T>& p = b.p;
  const long N = p.N, sy = p.nx, sz = (long)p.nx * p.ny;
  for (int i = threadIdx.x; i < 19 * nr; i += WTPB) {
    const int q = i % 19;
    const long r = r0 + i / 19;
    const int y = 3 + (int)(r % b.nry), z = 3 + (int)(r / b.nry);
    const long gs = r == r0 ? t0 - r0 * b.gpr : 0;
    const long ge = r == r1 ? t1 - r1 * b.gpr : b.gpr - 1;
    const long row = ((long)z * p.ny + y) * p.nx;
    const T* src = PAR ? p.f + opp(q) * N + row - cy(q) * sy - cz(q) * sz : p.f + q * N + row;
    l2_prefetch(src + gs * V - 1, src + (ge + 1) * V + 1, p.f, p.f + 19 * N);
  }
}

/* Collide the V cells and store them (AA pushes assembled across lanes). */
template <typename T, int V, int PAR>
__device__ __forceinline__ void words_collide_store(const FluidParamsT<T>& p, const ItemCtx& c, int lane, float* d) {
  using Wd = Word<T, V>;
  using U = typename Wd::U;
  constexpr int NR = Wd::NR;
  if (c.active) {
    using Fm = Form<T>;
    const int tile = tile_of(c.x0, c.y, c.z, p.ntx, p.nty);
    const int c0 = cell_in_tile(c.x0, c.y, c.z);
    const int sp = p.first ? -1 : p.slot_prev[tile];
#pragma unroll
    for (int e = 0; e < V; e += 2) {
      F2 f[19];
#pragma unroll
      for (int q = 0; q < 19; ++q) f[q] = f2(d[q * V + e], d[q * V + e + 1]);
      F2 drho, dux, duy, duz;
      if (p.first || sp >= 0) {
        Mom<float> m0, m1;
        if (p.first) {
          Fm::initial_bulk(p, m0);
          m1 = m0;
        } else {
          Fm::from_tile(p, p.Uprev + (long)sp * 256, c0 + e, m0);
          Fm::from_tile(p, p.Uprev + (long)sp * 256, c0 + e + 1, m1);
        }
        drho = f2(m0.rho, m1.rho); dux = f2(m0.ux, m1.ux); duy = f2(m0.uy, m1.uy); duz = f2(m0.uz, m1.uz);
      } else {
        moments_free2(f, p, drho, dux, duy, duz);
      }
      collide2(f, drho, dux, duy, duz, p);
#pragma unroll
      for (int q = 0; q < 19; ++q) split(f[q], d[q * V + e], d[q * V + e + 1]);
    }
  }
  U* __restrict__ F = reinterpret_cast<U*>(p.f);
  const long N = p.N, sy = p.nx, sz = (long)p.nx * p.ny;
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    Wd w;
    w.pack(d + q * V, 1);
    if (PAR == 0) {
      if (c.active) w.store(F + opp(q) * N + c.row + c.x0);
    } else {
      U* dst = F + c.row + c.x0 + (p.push[q] - cx(q));   /* the aligned word the push lands in */
      if (cx(q) == 0) {
        if (c.active) w.store(dst);
      } else if (cx(q) == 1) {
        const uint32_t hi = __shfl_up_sync(0xffffffffu, w.r[NR - 1], 1);
        const Wd o = w.shifted_up(hi);
        if (c.active) {
          if (lane > 0 && c.left_active) {
            o.store(dst);
          } else {
#pragma unroll
            for (int e = 1; e < V; ++e) dst[e] = o.elem(e);
          }
          if (lane == 31 || !c.right_active) dst[V] = w.elem(V - 1);
        }
      } else {
        const uint32_t lo = __shfl_down_sync(0xffffffffu, w.r[0], 1);
        const Wd o = w.shifted_down(lo);
        if (c.active) {
          if (lane < 31 && c.right_active) {
            o.store(dst);
          } else {
#pragma unroll
            for (int e = 0; e < V - 1; ++e) dst[e] = o.elem(e);
          }
          if (lane == 0 || !c.left_active) dst[-1] = w.elem(0);
        }
      }
    }
  }
}

/* The incoming populations of direction q from the word as loaded and, at a
 * warp edge, the extra element. */
template <typename T, int V>
__device__ __forceinline__ void words_shift(Word<T, V>& w, int q, int lane, const ItemCtx& c, uint32_t edge) {
  constexpr int NR = Word<T, V>::NR;
  if (cx(q) == 1) {
    uint32_t hi = __shfl_up_sync(0xffffffffu, w.r[NR - 1], 1);
    if (lane == 0 && c.active) hi = edge;
    w = w.shifted_up(hi);
  } else if (cx(q) == -1) {
    uint32_t lo = __shfl_down_sync(0xffffffffu, w.r[0], 1);
    if (lane == 31 && c.active) lo = edge;
    w = w.shifted_down(lo);
  }
}

/* One thread's V cells of the bulk step: thread t of the flattened
 * (bulk row, word) space of b. */
template <typename T, int V, int PAR>
__device__ __forceinline__ void words_item(const WordsParams<T>& b, long t) {
  using Wd = Word<T, V>;
  const FluidParamsT<T>& p = b.p;
  const int lane = threadIdx.x & 31;
  const ItemCtx c = item_ctx<T, V>(b, t);
  float d[19 * V];  /* d[q * V + e]: population q of cell x0 + e */
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    Wd w;
    const auto* src = word_src<T, PAR>(p, c, q);
    if (c.loads) w.load(src); else w.clear();
    if (PAR == 1 && cx(q) != 0) {
      const bool edge_lane = (cx(q) == 1 ? lane == 0 : lane == 31) && c.active;
      const uint32_t edge = edge_lane ? *reinterpret_cast<const uint32_t*>(edge_src<T, V>(src, cx(q))) : 0u;
      words_shift(w, q, lane, c, edge);
    }
    w.unpack(d + q * V, 1);
  }
  words_collide_store<T, V, PAR>(p, c, lane, d);
}

/* ---- the word step with its loads staged in shared memory by TMA ----
 *
 * 16-bit storage, V = 4.  The flattened (bulk row, word) space is cut into
 * items of 128 threads: one 128-word segment of a row when a row has at
 * least 128 words (W = nx / 4), else K = 128 / W whole rows.  A persistent
 * CTA walks its items; one thread keeps STAGES items ahead of the compute
 * with 1-D bulk copies (cp.async.bulk, no multicast) of every plane's row
 * window -- the segment's cells plus 8 on either side, which covers the
 * odd step's x shifts and keeps both ends 16-byte aligned -- into shared
 * memory, completing on the stage's mbarrier.  The threads then read their
 * words from shared memory (an x-shifted word from two aligned ones), so
 * no register holds data in flight and no thread waits on DRAM; the
 * collision and the stores (pushes assembled across lanes) are the plain
 * word kernel's.  Only the slots a cell reads are used, and the AA rule
 * makes those slots read and written by that cell alone, so loading an
 * item several items ahead of the stores of this launch is safe. */
struct TmaGeom {
  int W;        /* words per row                                  */
  int segw;     /* words per item segment: min(W, 128)             */
  int K;        /* rows per item (1 when W >= 128)                 */
  int nchunk;   /* segments per row (1 when W <= 128)              */
  long nitems;
  int win;      /* elements per (plane, row) window: 4 segw + 16   */
};

__host__ __forceinline__ bool tma_geometry(TmaGeom& g, int nx, long nrows) {
  if (nx % 8) return false;
  g.W = nx / 4;
  if (g.W >= 128) {
    g.segw = 128; g.K = 1; g.nchunk = (g.W + 127) / 128;
    g.nitems = nrows * g.nchunk;
  } else {
    if (128 % g.W) return false;
    g.segw = g.W; g.K = 128 / g.W; g.nchunk = 1;
    g.nitems = (nrows + g.K - 1) / g.K;
  }
  g.win = 4 * g.segw + 16;
  return true;
}

__host__ __device__ __forceinline__ int tma_stage_bytes(const TmaGeom& g) { return 19 * g.K * g.win * 2; }

constexpr long kTmaSpin = 1L << 24;   /* mbarrier polls before a wait gives up */

__device__ __forceinline__ uint32_t cta_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

/* Item `it`: its first bulk row and the first word of its segment. */
__device__ __forceinline__ void tma_item(const TmaGeom& g, long it, long& row0, int& w0) {
  if (g.nchunk > 1) { row0 = it / g.nchunk; w0 = (int)(it - row0 * g.nchunk) * 128; }
  else { row0 = it * g.K; w0 = 0; }
}

/* Issue the bulk copies of item `it` into `stage` (one thread).  Every
 * window stays inside its plane by construction (bulk rows have whole rows
 * on either side); were one not to, the item's copies are not issued, the
 * stage's barrier is released without them and err[0] is set, so that the
 * launch reports failure instead of reading outside the buffer. */
template <typename T, int PAR>
__device__ __forceinline__ void tma_issue(const WordsParams<T>& b, const TmaGeom& g, long it, uint8_t* stage,
                                          uint64_t* full, int* err) {
  long row0;
  int w0;
  tma_item(g, it, row0, w0);
  const FluidParamsT<T>& p = b.p;
  const uint16_t* F = reinterpret_cast<const uint16_t*>(p.f);
  const long sy = p.nx, sz = (long)p.nx * p.ny;
  int nr = g.K;
  if (row0 + nr > b.nrows) nr = (int)(b.nrows - row0);
  const uint32_t bytes = (uint32_t)g.win * 2;
  bool inside = true;
  for (int k = 0; k < nr; ++k) {
    const long r = row0 + k;
    const int y = 3 + (int)(r % b.nry), z = 3 + (int)(r / b.nry);
    const long row = ((long)z * p.ny + y) * p.nx + 4L * w0 - 8;
    inside = inside && row - sz - sy >= 0 && row + sz + sy + g.win <= p.N;
  }
  if (!inside) {
    atomicExch(err, 1);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(cta_smem(full)), "r"(0u) : "memory");
    return;
  }
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(cta_smem(full)),
               "r"(bytes * 19u * (uint32_t)nr)
               : "memory");
  for (int k = 0; k < nr; ++k) {
    const long r = row0 + k;
    const int y = 3 + (int)(r % b.nry), z = 3 + (int)(r / b.nry);
    const long row = ((long)z * p.ny + y) * p.nx + 4L * w0 - 8;
#pragma unroll 1
    for (int q = 0; q < 19; ++q) {
      const uint16_t* src = PAR ? F + opp(q) * p.N + row - cy(q) * sy - cz(q) * sz : F + q * p.N + row;
      uint8_t* dst = stage + ((long)q * g.K + k) * bytes;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              cta_smem(dst)),
          "l"(src), "r"(bytes), "r"(cta_smem(full))
          : "memory");
    }
  }
}

__device__ __forceinline__ bool tma_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = cta_smem(bar);
  for (long i = 0; i < kTmaSpin; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

/* The incoming word of direction q for the thread's cells from the staged
 * window (element e0 = the thread's first cell). */
template <int PAR>
__device__ __forceinline__ Word<__half, 4> smem_word(const uint16_t* w, int e0, int q) {
  Word<__half, 4> o;
  const uint2 m = *reinterpret_cast<const uint2*>(w + e0);
  if (PAR == 0 || cx(q) == 0) {
    o.r[0] = m.x; o.r[1] = m.y;
  } else if (cx(q) == 1) {
    const uint32_t l = *reinterpret_cast<const uint32_t*>(w + e0 - 2);
    o.r[0] = __byte_perm(l, m.x, 0x5432);
    o.r[1] = __byte_perm(m.x, m.y, 0x5432);
  } else {
    const uint32_t h = *reinterpret_cast<const uint32_t*>(w + e0 + 4);
    o.r[0] = __byte_perm(m.x, m.y, 0x5432);
    o.r[1] = __byte_perm(m.y, h, 0x5432);
  }
  return o;
}

/* A cell of a forced tile inside the word kernel's range (bulk rows,
 * x in [4, nx-5]; zb = last bulk z row), by the generic per-cell rules. */
template <typename T, int PAR>
__device__ __forceinline__ void forced_cell(const FluidParamsT<T>& p, int tile, int cell, int zb) {
  const int tx = tile % p.ntx, ty = (tile / p.ntx) % p.nty, tz = tile / (p.ntx * p.nty);
  const int x = tx * 4 + (cell & 3), y = ty * 4 + ((cell >> 2) & 3), z = tz * 4 + (cell >> 4);
  if (y >= 3 && y <= p.ny - 4 && z >= 3 && z <= zb && x >= 4 && x <= p.nx - 5) step_cell<T, PAR>(p, x, y, z);
}

/* Cell k in {0..3} -> x in {2, 3, nx-4, nx-3} of bulk row r. */
template <typename T, int PAR>
__device__ __forceinline__ void edge_cell(const FluidParamsT<T>& p, int nry, int r, int k) {
  const int y = 3 + r % nry, z = 3 + r / nry;
  const int x = k < 2 ? 2 + k : p.nx - 6 + k;
  if (p.box && in_box(p.box, x, y, z)) return;
  step_cell<T, PAR>(p, x, y, z);
}

/* The word-kernel variants that the one-grid and the batched launches and
 * their autotuners choose from: {cells per thread V, resident blocks per SM
 * the registers are sized for}.  16-bit storage: {4,3} {4,4} {2,4} {2,5}
 * {2,6} {4,5} (the last spills ~64 bytes and still measured fastest at
 * 512x256x256: occupancy buys more than the spills cost); FP32: {2,3}
 * {2,4} {2,5}.  (A variant that prefetched the next rows'
 * words into shared memory with cp.async measured no faster and was
 * dropped.)  with_variant calls f(V, MINB) as integral constants. */
constexpr int kWordVariants16 = 6, kWordVariants32 = 3;

__host__ __forceinline__ int word_variants(int prec) {
  return LBIB_PREC_TYPE(prec) == LBIB_PREC_F32 ? kWordVariants32 : kWordVariants16;
}

__host__ __forceinline__ int word_variant_cells(int prec, int v) {
  return LBIB_PREC_TYPE(prec) == LBIB_PREC_F32 ? 2 : ((v <= 1 || v == 5) ? 4 : 2);
}

template <typename T, typename F>
int with_variant(int v, F&& f) {
  using std::integral_constant;
  if constexpr (sizeof(T) == 2) {
    switch (v) {
      case 1: return f(integral_constant<int, 4>{}, integral_constant<int, 4>{});
      case 2: return f(integral_constant<int, 2>{}, integral_constant<int, 4>{});
      case 3: return f(integral_constant<int, 2>{}, integral_constant<int, 5>{});
      case 4: return f(integral_constant<int, 2>{}, integral_constant<int, 6>{});
      case 5: return f(integral_constant<int, 4>{}, integral_constant<int, 5>{});
      default: return f(integral_constant<int, 4>{}, integral_constant<int, 3>{});
    }
  } else {
    switch (v) {
      case 1: return f(integral_constant<int, 2>{}, integral_constant<int, 4>{});
      case 2: return f(integral_constant<int, 2>{}, integral_constant<int, 5>{});
      default: return f(integral_constant<int, 2>{}, integral_constant<int, 3>{});
    }
  }
}

/* Bulk-row geometry of a grid for the word kernel with V cells per word. */
template <typename T>
__host__ __forceinline__ void words_geometry(WordsParams<T>& b, int V, int nx, int nry, int nrz) {
  b.nry = nry;
  b.nrows = (long)nry * nrz;
  b.ngroups = nx / V;
  b.gpr = b.ngroups;
  b.g0 = (4 + V - 1) / V;
  b.g1 = (nx - 4) / V - 1;
  b.pf = 0;
  b.dgpr = fast_div((unsigned)b.gpr);
  b.dnry = fast_div((unsigned)(nry > 0 ? nry : 1));
}

}  // namespace lbib

#endif
