/*
 * Low-precision population storage: FP32, FP16 or BF16 deviations from a
 * fixed shift, with FP32 deviation-form arithmetic (moments, equilibrium,
 * BGK + Guo collision; Form<T> in lbib_fluid_kernels.cuh).  Same AA access
 * rules and reference boundary semantics as the FP64 path; compiled with FMA
 * contraction allowed, since these forms are judged by their error against
 * the FP64 solution, not by bits.  HBM bytes per lattice update: 152 (FP32),
 * 76 (FP16, BF16).
 *
 * Rows away from the walls (y in [3, ny-4], z in [3, min(nz-4, zin_hi)]) run
 * lbib_fluid_step_words: a thread owns V = 8 / sizeof(T) consecutive cells
 * (x0 = V g) and moves every population plane as one aligned 8-byte word.
 * Even step: own slots, aligned.  Odd step, c_x = 0: aligned too.  Odd step,
 * c_x = +-1: the V values a thread needs are its own word shifted by one
 * element, the missing element coming from the neighbouring lane's word
 * (one 64-bit shuffle); pushes are assembled the same way before the store.
 * At a warp edge (lane 0 / 31) the element crosses to another warp, and the
 * thread that owns the pushing cell reads and writes it with a scalar
 * access -- the AA rule that a slot is read and written only by the cell
 * that pushes into it keeps that race-free.  Cells x in {2, 3, nx-4, nx-3}
 * of those rows (the inlet/outlet planes and their neighbours) run the
 * generic per-cell rules in lbib_edge_cells; their words are still loaded
 * by idle lanes so the shuffles see them, and neither kernel writes an
 * element the other owns.
 */
#include <stdint.h>
#include <stdlib.h>

#include <type_traits>

#include "lbib_fluid_kernels.cuh"

extern "C" int lbdev_bulk_rows(const lbib_device* d, int* nrows_y, int* nrows_z);

using namespace lbib;

namespace {

constexpr int WTPB = 128;

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
    if constexpr (NR == 2) { const uint2 v = *reinterpret_cast<const uint2*>(a); r[0] = v.x; r[1] = v.y; }
    else r[0] = *reinterpret_cast<const uint32_t*>(a);
  }
  __device__ __forceinline__ void store(U* a) const {
    if constexpr (NR == 2) *reinterpret_cast<uint2*>(a) = make_uint2(r[0], r[1]);
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

template <typename T>
struct WordsParams {
  FluidParamsT<T> p;
  int nry;      /* bulk rows in y */
  long nrows;   /* bulk rows */
  int ngroups;  /* words per x row: nx / V */
  int gpr;      /* threads per row: ngroups rounded up to whole warps */
  int g0, g1;   /* groups whose cells all lie in [4, nx-5] */
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
  return g >= b.g0 && g <= b.g1 && b.p.slot_cur[tile_of(g * V, y, z, b.p.ntx, b.p.nty)] < 0;
}

template <typename T, int V>
__device__ __forceinline__ ItemCtx item_ctx(const WordsParams<T>& b, long t) {
  ItemCtx c;
  const long r = t / b.gpr;
  const int g = (int)(t - r * b.gpr);
  const bool inrow = r < b.nrows;
  c.y = 3 + (int)(r % b.nry);
  c.z = 3 + (int)(r / b.nry);
  c.x0 = g * V;
  c.loads = inrow && g < b.ngroups;
  c.active = inrow && group_here<T, V>(b, g, c.y, c.z);
  c.left_active = inrow && group_here<T, V>(b, g - 1, c.y, c.z);
  c.right_active = inrow && group_here<T, V>(b, g + 1, c.y, c.z);
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
  return F + opp(q) * p.N + c.row - cy(q) * sy - cz(q) * sz + c.x0;
}

/* The 4-byte aligned word that holds the element a lane at a warp edge needs
 * from beyond its warp: x0 - 1 (in the high half for 16-bit storage) when
 * c_x = +1, x0 + V (low half) when c_x = -1. */
template <typename T, int V>
__device__ __forceinline__ const void* edge_src(const typename Word<T, V>::U* src, int dir) {
  if (dir > 0) return sizeof(T) == 2 ? (const void*)(src - 2) : (const void*)(src - 1);
  return (const void*)(src + V);
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
    for (int e = 0; e < V; ++e) {
      float f[19];
#pragma unroll
      for (int q = 0; q < 19; ++q) f[q] = d[q * V + e];
      Mom<float> m;
      if (p.first) Fm::initial(p, m);
      else if (sp >= 0) Fm::from_tile(p, p.Uprev + (long)sp * 256, c0 + e, m);
      else Fm::moments_free(f, p, m);
      Fm::template collide<false>(f, m, 0.0f, 0.0f, 0.0f, p);
#pragma unroll
      for (int q = 0; q < 19; ++q) d[q * V + e] = f[q];
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
      U* dst = F + q * N + c.row + cy(q) * sy + cz(q) * sz + c.x0;
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

template <typename T, int V, int PAR, int MINB>
__global__ void __launch_bounds__(WTPB, MINB) lbib_fluid_step_words(WordsParams<T> b) {
  using Wd = Word<T, V>;
  const FluidParamsT<T>& p = b.p;
  const int lane = threadIdx.x & 31;
  const ItemCtx c = item_ctx<T, V>(b, (long)blockIdx.x * WTPB + threadIdx.x);
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

__device__ __forceinline__ void cp_async(void* smem, const void* gmem, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

/* Shared memory of the pipelined kernel, per stage: the words of the 19
 * planes, [q][thread], and the warp-edge elements [warp][10]. */
template <typename T, int V>
__host__ __device__ constexpr int pipe_stage_bytes() {
  return 19 * WTPB * Word<T, V>::NR * 4 + (WTPB / 32) * 10 * 4;
}

/* The same step as a persistent kernel: each block walks items (128
 * consecutive threads of the flattened row x word space) with a stride of
 * the grid, and while it collides one item the next item's words are
 * already on their way into shared memory (cp.async, two stages).  Each
 * thread copies and later reads only its own words, so it needs no barrier;
 * the data in flight per SM no longer depends on the registers. */
template <typename T, int V, int PAR, int MINB>
__global__ void __launch_bounds__(WTPB, MINB) lbib_fluid_step_pipe(WordsParams<T> b, long nitems) {
  using Wd = Word<T, V>;
  constexpr int NR = Wd::NR;
  extern __shared__ __align__(16) uint8_t smem[];
  const FluidParamsT<T>& p = b.p;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto words = [&](int st) { return reinterpret_cast<uint32_t*>(smem + st * pipe_stage_bytes<T, V>()); };
  auto edges = [&](int st) { return words(st) + 19 * WTPB * NR + warp * 10; };
  auto issue = [&](int st, const ItemCtx& c) {
    uint32_t* W = words(st);
    uint32_t* E = edges(st);
#pragma unroll
    for (int q = 0; q < 19; ++q)
      if (c.loads) cp_async(W + (q * WTPB + tid) * NR, word_src<T, PAR>(p, c, q), 4 * NR);
    if (PAR == 1 && c.active) {
      int k = 0;
#pragma unroll
      for (int q = 0; q < 19; ++q) {
        if (cx(q) == 0) continue;
        const bool edge_lane = cx(q) == 1 ? lane == 0 : lane == 31;
        if (edge_lane) cp_async(E + k, edge_src<T, V>(word_src<T, PAR>(p, c, q), cx(q)), 4);
        ++k;
      }
    }
  };
  long it = blockIdx.x;
  ItemCtx c = item_ctx<T, V>(b, it * WTPB + tid);
  if (it < nitems) issue(0, c);
  cp_async_commit();
  for (int k = 0; it < nitems; ++k, it += gridDim.x) {
    const long nxt = it + gridDim.x;
    const ItemCtx cn = item_ctx<T, V>(b, nxt * WTPB + tid);
    if (nxt < nitems) issue((k + 1) & 1, cn);
    cp_async_commit();
    cp_async_wait<1>();
    const uint32_t* W = words(k & 1);
    const uint32_t* E = edges(k & 1);
    float d[19 * V];
    int ke = 0;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      Wd w;
      if (c.loads) {
#pragma unroll
        for (int i = 0; i < NR; ++i) w.r[i] = W[(q * WTPB + tid) * NR + i];
      } else {
        w.clear();
      }
      if (PAR == 1 && cx(q) != 0) {
        words_shift(w, q, lane, c, E[ke]);
        ++ke;
      }
      w.unpack(d + q * V, 1);
    }
    words_collide_store<T, V, PAR>(p, c, lane, d);
    c = cn;
  }
  cp_async_wait<0>();
}

/* Cells of this step's forced tiles inside the word kernel's range (bulk
 * rows, x in [4, nx-5]), by the generic per-cell rules; zb is the last bulk
 * z row.  A persistent grid walks the tile list. */
template <typename T, int PAR>
__global__ void __launch_bounds__(64) lbib_forced_cells(FluidParamsT<T> p, const int* __restrict__ list,
                                                        const int* __restrict__ count, int zb) {
  const int n = *count;
  const int cell = threadIdx.x;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int tile = list[i];
    const int tx = tile % p.ntx, ty = (tile / p.ntx) % p.nty, tz = tile / (p.ntx * p.nty);
    const int x = tx * 4 + (cell & 3), y = ty * 4 + ((cell >> 2) & 3), z = tz * 4 + (cell >> 4);
    if (y >= 3 && y <= p.ny - 4 && z >= 3 && z <= zb && x >= 4 && x <= p.nx - 5) step_cell<T, PAR>(p, x, y, z);
  }
}

/* Cells x in {2, 3, nx-4, nx-3} of the bulk rows, by the generic rules. */
template <typename T, int PAR>
__global__ void __launch_bounds__(128) lbib_edge_cells(FluidParamsT<T> p, int nry, int nrows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 4 * nrows) return;
  const int r = i >> 2, k = i & 3;
  const int y = 3 + r % nry, z = 3 + r / nry;
  const int x = k < 2 ? 2 + k : p.nx - 6 + k;
  step_cell<T, PAR>(p, x, y, z);
}

/* Resident blocks per SM and SMs, for sizing the persistent grid. */
int sm_count();

template <typename K>
int persistent_blocks(K kernel, int smem_bytes) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, WTPB, smem_bytes);
  return sm_count() * (per_sm > 0 ? per_sm : 1);
}

template <typename T, int V, int PAR, int MINB>
int launch_pipe(lbib_device* d, const WordsParams<T>& b) {
  static int blocks = 0;
  constexpr int smem = 2 * pipe_stage_bytes<T, V>();
  if (!blocks) blocks = persistent_blocks(lbib_fluid_step_pipe<T, V, PAR, MINB>, smem);
  const long nitems = (b.nrows * b.gpr + WTPB - 1) / WTPB;
  const unsigned grid = (unsigned)(nitems < blocks ? nitems : blocks);
  lbib_fluid_step_pipe<T, V, PAR, MINB><<<grid, WTPB, smem, d->stream>>>(b, nitems);
  return 0;
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

template <typename T, int V, int MINB, int PIPE>
int launch_words(lbib_device* d, const FluidParamsT<T>& p) {
  WordsParams<T> b;
  b.p = p;
  int nrz = 0;
  if (!lbdev_bulk_rows(d, &b.nry, &nrz)) return 0;
  b.nrows = (long)b.nry * nrz;
  b.ngroups = d->nx / V;
  b.gpr = (b.ngroups + 31) / 32 * 32;
  b.g0 = (4 + V - 1) / V;
  b.g1 = (d->nx - 4) / V - 1;
  const long threads = b.nrows * b.gpr;
  const unsigned blocks = (unsigned)((threads + WTPB - 1) / WTPB);
  const unsigned eblocks = (unsigned)((4 * b.nrows + 127) / 128);
  constexpr bool pipe = PIPE != 0;
  const int zb = 2 + nrz, c = d->cur;
  const unsigned fblocks = (unsigned)sm_count() * 8;
  if (d->parity == 0) {
    if (pipe) launch_pipe<T, V, 0, MINB>(d, b);
    else lbib_fluid_step_words<T, V, 0, MINB><<<blocks, WTPB, 0, d->stream>>>(b);
    lbib_edge_cells<T, 0><<<eblocks, 128, 0, d->stream>>>(p, b.nry, (int)b.nrows);
    lbib_forced_cells<T, 0><<<fblocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], zb);
  } else {
    if (pipe) launch_pipe<T, V, 1, MINB>(d, b);
    else lbib_fluid_step_words<T, V, 1, MINB><<<blocks, WTPB, 0, d->stream>>>(b);
    lbib_edge_cells<T, 1><<<eblocks, 128, 0, d->stream>>>(p, b.nry, (int)b.nrows);
    lbib_forced_cells<T, 1><<<fblocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], zb);
  }
  d->kernel_launches += 3;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* Word-kernel variants the autotuner chooses from: cells per thread,
 * resident blocks per SM the registers are sized for, and whether the next
 * item is prefetched through shared memory. */
struct LpVariant {
  int v, minb, pipe;
};
constexpr LpVariant kVariants16[] = {{4, 3, 0}, {4, 4, 0}, {2, 4, 0}, {2, 5, 0}, {2, 6, 0}, {4, 3, 1}, {2, 5, 1}};
constexpr LpVariant kVariants32[] = {{2, 3, 0}, {2, 4, 0}, {2, 5, 0}, {2, 4, 1}};
constexpr int kN16 = sizeof(kVariants16) / sizeof(LpVariant);
constexpr int kN32 = sizeof(kVariants32) / sizeof(LpVariant);

template <typename T>
int lp_step(lbib_device* d) {
  FluidParamsT<T> p = make_params_t<T>(d, d->steps == 0);
  if (launch_step_rows_t<T>(d, p)) return -2;
  if (!d->use_bulk) return 0;
  const int i = d->lp_variant < 0 ? 0 : d->lp_variant;
  if constexpr (sizeof(T) == 2) {
    switch (i) {
      case 1: return launch_words<T, 4, 4, 0>(d, p);
      case 2: return launch_words<T, 2, 4, 0>(d, p);
      case 3: return launch_words<T, 2, 5, 0>(d, p);
      case 4: return launch_words<T, 2, 6, 0>(d, p);
      case 5: return launch_words<T, 4, 3, 1>(d, p);
      case 6: return launch_words<T, 2, 5, 1>(d, p);
      default: return launch_words<T, 4, 3, 0>(d, p);
    }
  } else {
    switch (i) {
      case 1: return launch_words<T, 2, 4, 0>(d, p);
      case 2: return launch_words<T, 2, 5, 0>(d, p);
      case 3: return launch_words<T, 2, 4, 1>(d, p);
      default: return launch_words<T, 2, 3, 0>(d, p);
    }
  }
}

}  // namespace

extern "C" int lbdev_lp_fluid_step(lbib_device* d) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return lp_step<float>(d);
    case LBIB_PREC_F16: return lp_step<__half>(d);
    case LBIB_PREC_BF16: return lp_step<__nv_bfloat16>(d);
    default: return -1;
  }
}

extern "C" int lbdev_lp_tile_moments(lbib_device* d) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return launch_tile_moments_t<float>(d);
    case LBIB_PREC_F16: return launch_tile_moments_t<__half>(d);
    case LBIB_PREC_BF16: return launch_tile_moments_t<__nv_bfloat16>(d);
    default: return -1;
  }
}

extern "C" int lbdev_lp_field_moments(lbib_device* d, double* rho, double* ux, double* uy, double* uz) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return launch_field_moments_t<float>(d, rho, ux, uy, uz);
    case LBIB_PREC_F16: return launch_field_moments_t<__half>(d, rho, ux, uy, uz);
    case LBIB_PREC_BF16: return launch_field_moments_t<__nv_bfloat16>(d, rho, ux, uy, uz);
    default: return -1;
  }
}

extern "C" int lbdev_lp_gather_df1(lbib_device* d, double* out) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return launch_gather_df1_t<float>(d, out);
    case LBIB_PREC_F16: return launch_gather_df1_t<__half>(d, out);
    case LBIB_PREC_BF16: return launch_gather_df1_t<__nv_bfloat16>(d, out);
    default: return -1;
  }
}

extern "C" int lbdev_lp_init(lbib_device* d, int what) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return launch_init_t<float>(d, what);
    case LBIB_PREC_F16: return launch_init_t<__half>(d, what);
    case LBIB_PREC_BF16: return launch_init_t<__nv_bfloat16>(d, what);
    default: return -1;
  }
}

extern "C" int lbdev_lp_sums(lbib_device* d, double* part, double* out) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return launch_sums_t<float>(d, part, out);
    case LBIB_PREC_F16: return launch_sums_t<__half>(d, part, out);
    case LBIB_PREC_BF16: return launch_sums_t<__nv_bfloat16>(d, part, out);
    default: return -1;
  }
}

/* Word-kernel variants available for a precision (1 for FP64). */
extern "C" int lbdev_lp_variants(int prec) {
  switch (LBIB_PREC_TYPE(prec)) {
    case LBIB_PREC_F32: return kN32;
    case LBIB_PREC_F16:
    case LBIB_PREC_BF16: return kN16;
    default: return 1;
  }
}
