/*
 * The surrogate MLP's GEMM on the 5th-generation tensor cores (sm_100a):
 * tcgen05.mma kind::f16 with BF16 operands in shared memory and the FP32
 * accumulator in tensor memory (TMEM), read back with tcgen05.ld for the
 * bias / GELU epilogue.
 *
 * C[M][N] = sum_k A(m,k) B(k,n), A(m,k) = A[m*am + k*ak], B(k,n) =
 * B[k*bk + n*bn] (element strides, so W^T and dZ^T need no copies), rows
 * and columns beyond M, N, K read as zero.  One CTA of 128 threads computes
 * a 128 x BN tile: TMEM lane i holds row m0 + i, BN FP32 columns.
 *
 * Operands are staged in K slices of 64 (four MMAs of K = 16), double
 * buffered: the threads load a slice from global memory (16-byte vectors
 * when the operand is contiguous along K, single elements otherwise) and
 * write it in the canonical K-major layout without swizzle -- 8 x 16-byte
 * "core matrices", core (kb, g) of rows 8g..8g+7 and K elements 8kb..8kb+7
 * at byte (kb * G + g) * 128, so the descriptor's stride byte offset (next
 * 8 rows) is 128 and its leading byte offset (next 8 K elements) G * 128.
 * One thread issues the MMAs of a slice and commits them to the slice's
 * mbarrier; a buffer is refilled only after that mbarrier says the MMAs
 * that read it are done.  Every wait is bounded: on a timeout the CTA
 * records an error, skips the rest and still frees its TMEM.
 */
#ifndef LBIB_MLP_TC_CUH
#define LBIB_MLP_TC_CUH

#include <stdint.h>

#include <cuda_bf16.h>

namespace lbib_tc {

constexpr int BM = 128;   /* rows per CTA = TMEM lanes                 */
constexpr int BK = 64;    /* K per stage: four MMAs of K = 16          */
constexpr int NT = 128;   /* threads per CTA                           */
constexpr long kSpin = 1L << 24;   /* try_wait polls before giving up  */

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

/* Shared-memory matrix descriptor: canonical layout, no swizzle. */
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);           /* start address        [0,14)  */
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;         /* leading byte offset  [16,30) */
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;         /* stride byte offset   [32,46) */
  d |= (uint64_t)1 << 46;                              /* descriptor version 1 [46,48) */
  return d;                                            /* base offset 0, no swizzle    */
}

/* Instruction descriptor: BF16 x BF16 -> FP32, M x N; a_mn / b_mn: the
 * operand's shared-memory tile is MN-major (core-matrix rows run along K,
 * each holding 8 consecutive M or N elements) instead of K-major. */
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N, bool a_mn = false, bool b_mn = false) {
  return (1u << 4)                      /* D format F32   [4,6)   */
         | (1u << 7)                    /* A format BF16  [7,10)  */
         | (1u << 10)                   /* B format BF16  [10,13) */
         | ((a_mn ? 1u : 0u) << 15)     /* A major        [15]    */
         | ((b_mn ? 1u : 0u) << 16)     /* B major        [16]    */
         | ((uint32_t)(N >> 3) << 17)   /* N / 8          [17,23) */
         | ((uint32_t)(M >> 4) << 24);  /* M / 16         [24,29) */
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

/* Wait for completion `parity` of the barrier; false after kSpin polls. */
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long i = 0; i < kSpin; ++i) {
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

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <int NCOL>
__device__ __forceinline__ void tmem_alloc(uint32_t* slot) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"((uint32_t)NCOL)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

template <int NCOL>
__device__ __forceinline__ void tmem_free(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"((uint32_t)NCOL) : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

/* 16 consecutive FP32 columns of this thread's TMEM lane. */
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

/* How an operand tile is staged. */
enum Stage {
  ST_K_VEC = 0,    /* contiguous along K: 16-byte vectors, K-major tile      */
  ST_MN_VEC = 1,   /* contiguous along the rows: 16-byte vectors, MN-major   */
  ST_ELEM = 2,     /* any strides: element by element, K-major tile          */
};

/* The staging mode for X(r, k) = X[r*xr + k*xk] with nr valid rows. */
__host__ __device__ inline int stage_mode(const void* X, long xr, long xk, int nr, int K) {
  const bool al = (reinterpret_cast<uintptr_t>(X) & 15) == 0;
  if (al && xk == 1 && xr % 8 == 0 && K % 8 == 0) return ST_K_VEC;
  if (al && xr == 1 && xk % 8 == 0 && nr % 8 == 0) return ST_MN_VEC;
  return ST_ELEM;
}

/* Rows [r0, r0 + R) x K elements [k0, k0 + BK) of X(r, k) = X[r*xr + k*xk]
 * into shared memory at s, as 8 x 16-byte core matrices, core (kb, g) of
 * rows 8g..8g+7 and K elements 8kb..8kb+7 at byte (kb * G + g) * 128
 * (G = R / 8).  K-major (ST_K_VEC, ST_ELEM): core row i holds row 8g+i's
 * eight K elements; MN-major (ST_MN_VEC): core row i holds K element 8kb+i
 * of the eight rows.  Either way the descriptor's leading byte offset (next
 * 8 K elements) is G * 128 and its stride byte offset (next 8 rows) 128.
 * Outside [0, nr) x [0, K): zero (r0 and nr are multiples of 8 in the
 * MN-major mode). */
template <int R>
__device__ __forceinline__ void stage_operand(__nv_bfloat16* __restrict__ s, const __nv_bfloat16* __restrict__ X,
                                              long xr, long xk, int r0, int nr, int k0, int K, int mode) {
  constexpr int G = R / 8;
  const int t = threadIdx.x;
  if (mode == ST_MN_VEC) {
    /* BK x G vectors, consecutive threads along the rows (contiguous) */
    for (int v = t; v < BK * G; v += NT) {
      const int g = v % G, k = v / G;
      const int gr = r0 + 8 * g, gk = k0 + k;
      uint4 val = make_uint4(0u, 0u, 0u, 0u);
      if (gr < nr && gk < K) val = *reinterpret_cast<const uint4*>(X + (long)gk * xk + gr);
      *reinterpret_cast<uint4*>(s + (((k >> 3) * G + g) * 64 + (k & 7) * 8)) = val;
    }
  } else if (mode == ST_K_VEC) {
    /* R x (BK / 8) vectors, eight consecutive threads per row (128
       contiguous bytes); vector (kb, r) -> core (kb, r / 8), row r % 8 */
    for (int v = t; v < R * (BK / 8); v += NT) {
      const int kb = v % (BK / 8), r = v / (BK / 8);
      const int gr = r0 + r, gk = k0 + kb * 8;
      uint4 val = make_uint4(0u, 0u, 0u, 0u);
      if (gr < nr && gk < K) val = *reinterpret_cast<const uint4*>(X + (long)gr * xr + gk);
      *reinterpret_cast<uint4*>(s + ((kb * G + (r >> 3)) * 64 + (r & 7) * 8)) = val;
    }
  } else {
    /* consecutive threads take consecutive addresses: along the rows when
       they are contiguous (a transposed operand), along K otherwise */
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);
    const bool rows_fast = xr == 1;
    for (int e = t; e < R * BK; e += NT) {
      const int r = rows_fast ? e % R : e / BK, k = rows_fast ? e / R : e % BK;
      const int gr = r0 + r, gk = k0 + k;
      const __nv_bfloat16 val = (gr < nr && gk < K) ? X[(long)gr * xr + (long)gk * xk] : zero;
      s[((k >> 3) * G + (r >> 3)) * 64 + (r & 7) * 8 + (k & 7)] = val;
    }
  }
}

}  // namespace lbib_tc

#endif
