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
 * the word kernel of lbib_words.cuh; the cells x in {2, 3, nx-4, nx-3} of
 * those rows and the cells of forced tiles run the generic per-cell rules;
 * wall rows run the generic row kernel.  The word kernel comes in variants
 * (cells per thread, register budget) that lbdev_autotune chooses from.
 */
#include <stdint.h>
#include <stdlib.h>

#include "lbib_words.cuh"
#include "lbib_words8.cuh"

extern "C" int lbdev_bulk_rows(const lbib_device* d, int* nrows_y, int* nrows_z);

using namespace lbib;

namespace {

template <typename T, int V, int PAR, int MINB>
__global__ void __launch_bounds__(WTPB, MINB) lbib_fluid_step_words(WordsParams<T> b) {
  const long first = (long)blockIdx.x * WTPB;
  if (b.pf > 0) words_prefetch<T, V, PAR>(b, blockIdx.x + b.pf);
  words_item<T, V, PAR>(b, first + threadIdx.x);
  /* the plane-adjacent cells x in {2, 3, nx-4, nx-3} of the rows whose first
     word this block holds, while their words are in the caches (their slots
     are theirs alone, so the order within the launch does not matter) */
  const long r0 = fdiv((unsigned)(first + b.gpr - 1), b.dgpr);
  long r1 = fdiv((unsigned)(first + WTPB + b.gpr - 1), b.dgpr);
  if (r1 > b.nrows) r1 = b.nrows;
  for (long i = threadIdx.x; i < 4 * (r1 - r0); i += WTPB) edge_cell<T, PAR>(b.p, b.nry, (int)(r0 + i / 4), (int)(i & 3));
}

/* The eight-cell word step (16-bit storage, lbib_words8.cuh), then the
 * plane-adjacent cells of the rows whose first word this block holds. */
template <typename T, int PAR, int MINB>
__global__ void __launch_bounds__(WTPB, MINB) lbib_fluid_step_words8(WordsParams<T> b) {
  const long first = (long)blockIdx.x * WTPB;
  words8_item<T, PAR>(b, first + threadIdx.x);
  const long r0 = fdiv((unsigned)(first + b.gpr - 1), b.dgpr);
  long r1 = fdiv((unsigned)(first + WTPB + b.gpr - 1), b.dgpr);
  if (r1 > b.nrows) r1 = b.nrows;
  for (long i = threadIdx.x; i < 4 * (r1 - r0); i += WTPB) edge_cell<T, PAR>(b.p, b.nry, (int)(r0 + i / 4), (int)(i & 3));
}

/* The word step with TMA-staged loads (lbib_words.cuh): a persistent grid
 * of CTAs, each keeping STAGES items of bulk copies in flight ahead of its
 * compute.  Errors (a window outside the buffer, an mbarrier wait that ran
 * out) go to the state's error word as LBIB_E_CUDA. */
template <typename T, int PAR, int STAGES, int MINB>
__global__ void __launch_bounds__(WTPB, MINB) lbib_fluid_step_words_tma(WordsParams<T> b, TmaGeom g, int* err) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t full[STAGES];
  __shared__ int s_bad;
  const int t = threadIdx.x, lane = t & 31;
  const int SB = tma_stage_bytes(g);
  if (t == 0) {
    for (int s = 0; s < STAGES; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(cta_smem(&full[s])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_bad = 0;
  }
  __syncthreads();
  if (t == 0)
    for (int s = 0; s < STAGES; ++s) {
      const long it = blockIdx.x + (long)s * gridDim.x;
      if (it < g.nitems) tma_issue<T, PAR>(b, g, it, smem + s * SB, &full[s], &s_bad);
    }
  const int k = t / g.segw, w = t - k * g.segw;
  int j = 0;
  bool ok = true;
  for (long it = blockIdx.x; it < g.nitems; it += gridDim.x, ++j) {
    const int s = j % STAGES;
    ok = __syncthreads_and(tma_wait(&full[s], (uint32_t)((j / STAGES) & 1)));
    if (!ok) break;
    long row0;
    int w0;
    tma_item(g, it, row0, w0);
    /* the thread's word: row row0 + k, word w0 + w */
    ItemCtx c;
    const long r = row0 + k;
    const int gw = w0 + w;
    const bool inrow = k < g.K && r < b.nrows && gw < g.W;
    const unsigned rz = fdiv((unsigned)r, b.dnry);
    c.y = 3 + (int)((unsigned)r - rz * (unsigned)b.nry);
    c.z = 3 + (int)rz;
    c.x0 = gw * 4;
    c.loads = inrow;
    c.active = inrow && group_here<T, 4>(b, gw, c.y, c.z);
    c.left_active = __shfl_up_sync(0xffffffffu, c.active, 1);
    c.right_active = __shfl_down_sync(0xffffffffu, c.active, 1);
    if (lane == 0) c.left_active = inrow && group_here<T, 4>(b, gw - 1, c.y, c.z);
    if (lane == 31) c.right_active = inrow && group_here<T, 4>(b, gw + 1, c.y, c.z);
    c.row = ((long)c.z * b.p.ny + c.y) * b.p.nx;
    float d[19 * 4];
    const uint16_t* st = reinterpret_cast<const uint16_t*>(smem + s * SB) + (long)(k < g.K ? k : 0) * g.win;
    const int e0 = 4 * w + 8;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      Word<T, 4> wd;
      if (inrow) {
        const Word<__half, 4> h = smem_word<PAR>(st + (long)q * g.K * g.win, e0, q);
        wd.r[0] = h.r[0]; wd.r[1] = h.r[1];
      } else {
        wd.clear();
      }
      wd.unpack(d + q * 4, 1);
    }
    words_collide_store<T, 4, PAR>(b.p, c, lane, d);
    __syncthreads();      /* every thread is done with stage s */
    if (t == 0) {
      const long nxt = it + (long)STAGES * gridDim.x;
      if (nxt < g.nitems) tma_issue<T, PAR>(b, g, nxt, smem + s * SB, &full[s], &s_bad);
    }
  }
  if (!ok) {
    /* a wait ran out: let the copies already issued land (bounded) before
       the CTA's shared memory is released */
    if (t == 0)
      for (int i = 0; i < STAGES; ++i) {
        const int s = (j + i) % STAGES;
        const long it = blockIdx.x + (long)(j + i) * gridDim.x;
        if (it < g.nitems) tma_wait(&full[s], (uint32_t)(((j + i) / STAGES) & 1));
      }
    __syncthreads();
  }
  /* the plane-adjacent cells x in {2, 3, nx-4, nx-3} of the rows whose
     items start at word 0, after the staged loop so that their global
     loads do not stall it: 4 K cells per such item, all threads at once */
  if (ok) {
    const long per = 4L * g.K;
    const long nmine = g.nitems > blockIdx.x ? (g.nitems - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    for (long e = t; e < nmine * per; e += WTPB) {
      const long it = blockIdx.x + (e / per) * gridDim.x;
      long row0;
      int w0;
      tma_item(g, it, row0, w0);
      const long r = row0 + (e % per) / 4;
      if (w0 == 0 && r < b.nrows) edge_cell<T, PAR>(b.p, b.nry, (int)r, (int)(e & 3));
    }
  }
  if (t == 0 && (!ok || s_bad)) atomicCAS(err, 0, -2);   /* LBIB_E_CUDA */
}

/* Cells of this step's forced tiles inside the word kernel's range; a
 * persistent grid walks the tile list. */
template <typename T, int PAR>
__global__ void __launch_bounds__(64) lbib_forced_cells(FluidParamsT<T> p, const int* __restrict__ list,
                                                        const int* __restrict__ count, int zb) {
  const int n = *count;
  for (int i = blockIdx.x; i < n; i += gridDim.x) forced_cell<T, PAR>(p, list[i], threadIdx.x, zb);
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

template <typename T, int V, int MINB>
int launch_words(lbib_device* d, const FluidParamsT<T>& p) {
  WordsParams<T> b;
  b.p = p;
  int nry = 0, nrz = 0;
  if (!lbdev_bulk_rows(d, &nry, &nrz)) return 0;
  words_geometry(b, V, d->nx, nry, nrz);
  b.pf = (long)d->l2_pf * sm_count() * MINB;
  const long threads = b.nrows * b.gpr;
  if (threads + WTPB >= (1L << 31)) return -1;   /* item_ctx divides 32-bit indices */
  const unsigned blocks = (unsigned)((threads + WTPB - 1) / WTPB);
  const int zb = 2 + nrz, c = d->cur;
  const unsigned fblocks = (unsigned)sm_count() * 8;
  /* box mode: the forced cells are among the box's, stepped after the spread */
  const bool forced = !p.box;
  if (d->parity == 0) {
    lbib_fluid_step_words<T, V, 0, MINB><<<blocks, WTPB, 0, d->fluid_stream>>>(b);
    if (forced) lbib_forced_cells<T, 0><<<fblocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], zb);
  } else {
    lbib_fluid_step_words<T, V, 1, MINB><<<blocks, WTPB, 0, d->fluid_stream>>>(b);
    if (forced) lbib_forced_cells<T, 1><<<fblocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], zb);
  }
  d->kernel_launches += forced ? 2 : 1;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* The eight-cell word step (16-bit storage) and the forced cells; the
 * four-cell kernel where a row is not a whole number of 16-byte words. */
template <typename T, int MINB>
int launch_words8(lbib_device* d, const FluidParamsT<T>& p) {
  if (d->nx % 8) return launch_words<T, 4, MINB>(d, p);
  WordsParams<T> b;
  b.p = p;
  int nry = 0, nrz = 0;
  if (!lbdev_bulk_rows(d, &nry, &nrz)) return 0;
  words_geometry(b, 8, d->nx, nry, nrz);
  const long threads = b.nrows * b.gpr;
  if (threads + WTPB >= (1L << 31)) return -1;   /* item8 divides 32-bit indices */
  const unsigned blocks = (unsigned)((threads + WTPB - 1) / WTPB);
  const int zb = 2 + nrz, c = d->cur;
  const unsigned fblocks = (unsigned)sm_count() * 8;
  const bool forced = !p.box;
  if (d->parity == 0) {
    lbib_fluid_step_words8<T, 0, MINB><<<blocks, WTPB, 0, d->fluid_stream>>>(b);
    if (forced) lbib_forced_cells<T, 0><<<fblocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], zb);
  } else {
    lbib_fluid_step_words8<T, 1, MINB><<<blocks, WTPB, 0, d->fluid_stream>>>(b);
    if (forced) lbib_forced_cells<T, 1><<<fblocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], zb);
  }
  d->kernel_launches += forced ? 2 : 1;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* The TMA-staged word step (16-bit storage) and the forced cells; the
 * plain word kernel where the row geometry does not suit it. */
template <typename T, int STAGES, int MINB>
int launch_words_tma(lbib_device* d, const FluidParamsT<T>& p) {
  WordsParams<T> b;
  b.p = p;
  int nry = 0, nrz = 0;
  if (!lbdev_bulk_rows(d, &nry, &nrz)) return 0;
  words_geometry(b, 4, d->nx, nry, nrz);
  TmaGeom g;
  if (!tma_geometry(g, d->nx, b.nrows)) return launch_words<T, 4, MINB>(d, p);
  const int smem = STAGES * tma_stage_bytes(g);
  static int attr[2] = {0, 0};
  if (smem > attr[0]) {
    if (cudaFuncSetAttribute(lbib_fluid_step_words_tma<T, 0, STAGES, MINB>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
        cudaFuncSetAttribute(lbib_fluid_step_words_tma<T, 1, STAGES, MINB>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return -2;
    attr[0] = smem;
  }
  const long cap = (long)sm_count() * MINB;
  const unsigned blocks = (unsigned)(g.nitems < cap ? g.nitems : cap);
  const int zb = 2 + nrz, c = d->cur;
  const unsigned fblocks = (unsigned)sm_count() * 8;
  const bool forced = !p.box;
  if (d->parity == 0) {
    lbib_fluid_step_words_tma<T, 0, STAGES, MINB><<<blocks, WTPB, smem, d->fluid_stream>>>(b, g, d->err);
    if (forced) lbib_forced_cells<T, 0><<<fblocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], zb);
  } else {
    lbib_fluid_step_words_tma<T, 1, STAGES, MINB><<<blocks, WTPB, smem, d->fluid_stream>>>(b, g, d->err);
    if (forced) lbib_forced_cells<T, 1><<<fblocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], zb);
  }
  d->kernel_launches += forced ? 2 : 1;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* One-grid variants beyond the word-kernel ones of lbib_words.cuh (16-bit
 * storage): {stages, resident CTAs per SM} of the TMA-staged kernel; the
 * eight-cell kernel at 4 resident CTAs per SM; and the four-cell {4, 5}
 * kernel for even steps with that eight-cell one for odd steps.  (The
 * eight-cell kernel at 3 CTAs per SM, 168 registers, and at 5, 96 registers
 * with ~450 bytes of spills, measured slower in both parities at
 * 512x256x256; its odd step gains from the halved shift work per cell, its
 * even step loses a little to the lower occupancy.) */
constexpr int kTmaVariants = 3;
constexpr int kWords8Variants = 2;

/* The box's cells of a box-mode step (after the spread). */
template <typename T>
int lp_box(lbib_device* d) {
  FluidParamsT<T> p = make_params_t<T>(d, d->steps == 0);
  return launch_box_cells_t<T>(d, p);
}

template <typename T>
int lp_step(lbib_device* d) {
  FluidParamsT<T> p = make_params_t<T>(d, d->steps == 0);
  if (launch_step_rows_t<T>(d, p)) return -2;
  if (!d->use_bulk) return 0;
  const int v = d->lp_variant < 0 ? 0 : d->lp_variant;
  if constexpr (sizeof(T) == 2) {
    const int nw = word_variants(d->prec);
    if (v == nw) return launch_words_tma<T, 2, 4>(d, p);
    if (v == nw + 1) return launch_words_tma<T, 3, 3>(d, p);
    if (v == nw + 2) return launch_words_tma<T, 2, 5>(d, p);
    const int v8 = v - nw - kTmaVariants;
    if (v8 == 0) return launch_words8<T, 4>(d, p);
    if (v8 == 1) return d->parity == 0 ? launch_words<T, 4, 5>(d, p) : launch_words8<T, 4>(d, p);
  }
  return with_variant<T>(v, [&](auto V, auto MINB) { return launch_words<T, V, MINB>(d, p); });
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

extern "C" int lbdev_lp_box_cells(lbib_device* d) {
  switch (LBIB_PREC_TYPE(d->prec)) {
    case LBIB_PREC_F32: return lp_box<float>(d);
    case LBIB_PREC_F16: return lp_box<__half>(d);
    case LBIB_PREC_BF16: return lp_box<__nv_bfloat16>(d);
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
  if (LBIB_PREC_TYPE(prec) == LBIB_PREC_F64) return 1;
  return word_variants(prec) + (LBIB_PREC_TYPE(prec) == LBIB_PREC_F32 ? 0 : kTmaVariants + kWords8Variants);
}
