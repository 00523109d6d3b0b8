/*
 * The 16-bit word step with eight cells per thread: every population plane
 * moved as one aligned 16-byte word, half the load, store, address and
 * shuffle instructions per cell of the four-cell word (lbib_words.cuh).
 *
 * A thread owns the cells x0 .. x0+7 (x0 = 8 g) of a bulk row; its two
 * halves x0 .. x0+3 and x0+4 .. x0+7 are tile columns, and each half is
 * stepped here or not on its own (act bit h): a half is stepped when its
 * cells lie in [4, nx-5] and it is neither in the box of this step's
 * stencils nor in a forced tile.  So the first and last word of a row step
 * one half each (x in [4, 7] and [nx-8, nx-5]) and the cells x in
 * {2, 3, nx-4, nx-3} are left to the generic per-cell rules, as in the
 * four-cell kernel.
 *
 * The 19 words stay packed in registers (4 x 32 bits each); the cells are
 * collided two at a time by the packed FP32 arithmetic of the four-cell
 * kernel and written back into the words, the same operations per cell.
 * Odd step, c_x = +-1: the shifted word takes one element from the
 * neighbouring lane (a shuffle and byte_perm; at a warp edge a scalar load),
 * and a push word is stored whole by the lane whose cells fill it -- its
 * own seven and the neighbour's one -- when both are stepped here and the
 * neighbour is in the warp; otherwise each lane writes the elements its own
 * stepped cells push, with 16- and 32-bit stores.  Each slot is still
 * written by exactly one thread (the AA rule: a slot is read and written
 * only by the cell that pushes into it).
 */
#ifndef LBIB_WORDS8_CUH
#define LBIB_WORDS8_CUH

#include "lbib_words.cuh"

namespace lbib {

/* A thread's eight cells and which halves of them, and of its neighbours'
 * words, are stepped here. */
struct Item8 {
  long row;            /* index of (0, y, z) */
  int y, z, x0;
  bool loads;
  unsigned act;        /* bit h: half h of this word      */
  unsigned lact, ract; /* the same for the words at x0 -/+ 8 of this row (0 if none) */
};

/* The tile column x .. x+3 (x % 4 == 0) of row (y, z) is stepped by the
 * word kernel. */
template <typename T>
__device__ __forceinline__ bool half_here8(const WordsParams<T>& b, int x, int y, int z) {
  if (x < 4 || x + 3 > b.p.nx - 5) return false;
  if (b.p.box) return !in_box(b.p.box, x, y, z);
  return b.p.slot_cur[tile_of(x, y, z, b.p.ntx, b.p.nty)] < 0;
}

template <typename T>
__device__ __forceinline__ unsigned act8(const WordsParams<T>& b, int g, int y, int z) {
  if (g < 0 || g >= b.ngroups) return 0u;
  return (half_here8(b, 8 * g, y, z) ? 1u : 0u) | (half_here8(b, 8 * g + 4, y, z) ? 2u : 0u);
}

/* Thread t of the flattened (bulk row, word) space; t < 2^31.  A row's
 * first word has no stepped low half and its last no stepped high half, so
 * the neighbouring lanes' flags are right across the end of a row too;
 * lanes 0 and 31 look their neighbours up. */
template <typename T>
__device__ __forceinline__ Item8 item8(const WordsParams<T>& b, long t) {
  Item8 c;
  const unsigned tu = (unsigned)t;
  const unsigned r = fdiv(tu, b.dgpr);
  const int g = (int)(tu - r * (unsigned)b.gpr);
  const bool inrow = r < (unsigned long)b.nrows;
  const unsigned rz = fdiv(r, b.dnry);
  c.y = 3 + (int)(r - rz * (unsigned)b.nry);
  c.z = 3 + (int)rz;
  c.x0 = 8 * g;
  c.loads = inrow && g < b.ngroups;
  c.act = inrow ? act8(b, g, c.y, c.z) : 0u;
  const int lane = threadIdx.x & 31;
  c.lact = __shfl_up_sync(0xffffffffu, c.act, 1);
  c.ract = __shfl_down_sync(0xffffffffu, c.act, 1);
  if (lane == 0) c.lact = inrow ? act8(b, g - 1, c.y, c.z) : 0u;
  if (lane == 31) c.ract = inrow ? act8(b, g + 1, c.y, c.z) : 0u;
  c.row = ((long)c.z * b.p.ny + c.y) * b.p.nx;
  return c;
}

/* Two 16-bit values (one 32-bit register) as a packed FP32 pair and back. */
template <typename T>
__device__ __forceinline__ F2 unpack2(uint32_t r) {
  if constexpr (std::is_same<T, __half>::value) {
    const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&r));
    return f2(f.x, f.y);
  } else {
    const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r));
    return f2(f.x, f.y);
  }
}

template <typename T>
__device__ __forceinline__ uint32_t pack2(F2 v) {
  float a, b;
  split(v, a, b);
  if constexpr (std::is_same<T, __half>::value) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
  } else {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
  }
}

__device__ __forceinline__ void st16(uint16_t* a, uint32_t r, int hi) { *a = (uint16_t)(r >> (16 * hi)); }
__device__ __forceinline__ void st32(uint16_t* a, uint32_t r) { *reinterpret_cast<uint32_t*>(a) = r; }
__device__ __forceinline__ void st64(uint16_t* a, uint32_t r0, uint32_t r1) {
  *reinterpret_cast<uint2*>(a) = make_uint2(r0, r1);
}

/* The stepped halves of word w at dst (16-byte aligned). */
template <typename W>
__device__ __forceinline__ void store_halves8(const W& w, uint16_t* dst, unsigned act) {
  if (act == 3u) w.store(dst);
  else if (act == 1u) st64(dst, w.r[0], w.r[1]);
  else if (act == 2u) st64(dst + 4, w.r[2], w.r[3]);
}

/* One thread's eight cells of the bulk step (16-bit storage). */
template <typename T, int PAR>
__device__ __forceinline__ void words8_item(const WordsParams<T>& b, long t) {
  using W8 = Word<T, 8>;
  static_assert(W8::NR == 4, "eight 16-bit cells per word");
  const FluidParamsT<T>& p = b.p;
  const int lane = threadIdx.x & 31;
  const Item8 c = item8<T>(b, t);
  uint16_t* __restrict__ F = reinterpret_cast<uint16_t*>(p.f);
  const long N = p.N;
  W8 w[19];
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const uint16_t* src = PAR == 0 ? F + q * N + c.row + c.x0 : F + c.row + c.x0 + (p.pull[q] + cx(q));
    if (c.loads) w[q].load(src); else w[q].clear();
    if (PAR == 1 && cx(q) == 1) {
      /* cell x0 pulls from x0 - 1: the left lane's last element */
      uint32_t hi = __shfl_up_sync(0xffffffffu, w[q].r[3], 1);
      if (lane == 0 && (c.act & 1u)) hi = *reinterpret_cast<const uint32_t*>(src - 2);
      w[q] = w[q].shifted_up(hi);
    } else if (PAR == 1 && cx(q) == -1) {
      /* cell x0 + 7 pulls from x0 + 8: the right lane's first element */
      uint32_t lo = __shfl_down_sync(0xffffffffu, w[q].r[0], 1);
      if (lane == 31 && (c.act & 2u)) lo = *reinterpret_cast<const uint32_t*>(src + 8);
      w[q] = w[q].shifted_down(lo);
    }
  }
  if (c.act) {
    using Fm = Form<T>;
    const int tile = tile_of(c.x0, c.y, c.z, p.ntx, p.nty);   /* half 1: tile + 1 */
    const int c0 = cell_in_tile(c.x0, c.y, c.z);
    const int sp0 = p.first ? -1 : p.slot_prev[tile];
    const int sp1 = p.first ? -1 : p.slot_prev[tile + 1];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int h = e >> 1;
      if (!((c.act >> h) & 1u)) continue;
      const int sp = h ? sp1 : sp0;
      const int cc = c0 + 2 * (e & 1);
      F2 f[19];
#pragma unroll
      for (int q = 0; q < 19; ++q) f[q] = unpack2<T>(w[q].r[e]);
      F2 drho, dux, duy, duz;
      if (p.first || sp >= 0) {
        Mom<float> m0, m1;
        if (p.first) {
          Fm::initial_bulk(p, m0);
          m1 = m0;
        } else {
          Fm::from_tile(p, p.Uprev + (long)sp * 256, cc, m0);
          Fm::from_tile(p, p.Uprev + (long)sp * 256, cc + 1, m1);
        }
        drho = f2(m0.rho, m1.rho); dux = f2(m0.ux, m1.ux); duy = f2(m0.uy, m1.uy); duz = f2(m0.uz, m1.uz);
      } else {
        moments_free2(f, p, drho, dux, duy, duz);
      }
      collide2(f, drho, dux, duy, duz, p);
#pragma unroll
      for (int q = 0; q < 19; ++q) w[q].r[e] = pack2<T>(f[q]);
    }
  }
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    if (PAR == 0) {
      if (c.act) store_halves8(w[q], F + opp(q) * N + c.row + c.x0, c.act);
      continue;
    }
    uint16_t* dst = F + c.row + c.x0 + (p.push[q] - cx(q));   /* the aligned word the pushes land in */
    if (cx(q) == 0) {
      if (c.act) store_halves8(w[q], dst, c.act);
    } else if (cx(q) == 1) {
      /* element k of the word at x0 is pushed by cell x0 + k - 1 */
      const uint32_t hi = __shfl_up_sync(0xffffffffu, w[q].r[3], 1);
      const W8 o = w[q].shifted_up(hi);
      const bool whole = lane > 0 && c.act == 3u && (c.lact & 2u);
      const bool right_whole = lane < 31 && c.ract == 3u && (c.act & 2u);
      if (c.act) {
        if (whole) {
          o.store(dst);
        } else {
          if (c.act & 1u) { st16(dst + 1, o.r[0], 1); st32(dst + 2, o.r[1]); st16(dst + 4, o.r[2], 0); }
          if (c.act & 2u) { st16(dst + 5, o.r[2], 1); st32(dst + 6, o.r[3]); }
        }
        if ((c.act & 2u) && !right_whole) st16(dst + 8, w[q].r[3], 1);
      }
    } else {
      /* element k of the word at x0 is pushed by cell x0 + k + 1 */
      const uint32_t lo = __shfl_down_sync(0xffffffffu, w[q].r[0], 1);
      const W8 o = w[q].shifted_down(lo);
      const bool whole = lane < 31 && c.act == 3u && (c.ract & 1u);
      const bool left_whole = lane > 0 && c.lact == 3u && (c.act & 1u);
      if (c.act) {
        if (whole) {
          o.store(dst);
        } else {
          if (c.act & 1u) { st32(dst, o.r[0]); st16(dst + 2, o.r[1], 0); }
          if (c.act & 2u) { st16(dst + 3, o.r[1], 1); st32(dst + 4, o.r[2]); st16(dst + 6, o.r[3], 0); }
        }
        if ((c.act & 1u) && !left_whole) st16(dst - 1, w[q].r[0], 0);
      }
    }
  }
}

}  // namespace lbib

#endif
