/*
 * A small multilayer perceptron on the GPU -- the surrogate that screens
 * parameter sweeps -- with its training: BF16 weights and activations, FP32
 * accumulation on the tcgen05 tensor cores, FP32 master weights, GELU
 * hidden layers, a linear output layer, mean-squared error and Adam.  No
 * reference counterpart.
 *
 * Shapes: widths w_0 .. w_L (input, hidden..., output); layer l maps w_l to
 * w_{l+1}.  Every width is padded to a multiple of 16 inside (the padded
 * weight rows and columns are zero and stay zero: their gradients vanish);
 * the ABI sees the unpadded shapes.  Parameters, in ABI order: for each
 * layer W_l [w_{l+1}][w_l] row-major, then b_l [w_{l+1}].
 *
 * One GEMM kernel serves all products, C[M][N] = sum_k A(m,k) B(k,n), with
 * A and B read through element strides (so a transposed operand needs no
 * copy): tcgen05.mma on 128 x 64 tiles with the accumulator in TMEM
 * (mlp_gemm_tc below, device helpers in lbib_mlp_tc.cuh), the weight
 * gradients' long K split four ways with a fixed-order reduction.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/lbib.h"
#include "lbib_mlp_tc.cuh"

namespace {


/* Epilogues of the GEMM. */
enum Epi {
  EPI_STORE = 0,        /* C (fp32) = acc                                  */
  EPI_BIAS_GELU = 1,    /* Z = acc + b (fp32 out0), A = gelu(Z) (bf16 out1) */
  EPI_BIAS = 2,         /* Y = acc + b (fp32 out0)                          */
};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
  return cdf + z * pdf;
}


/* C[M][N] (row-major, ldc) = A(m,k) B(k,n), A(m,k) = A[m*am + k*ak],
 * B(k,n) = B[k*bk + n*bn], out-of-range elements read as 0, on the tcgen05
 * tensor cores (FP32 accumulator in TMEM; lbib_mlp_tc.cuh): a 128 x BN tile
 * per 128-thread CTA, K in double-buffered slices of 64.  `err` is set if an mbarrier wait
 * ran out (the tile is then not written).
 *
 * Split K (gridDim.z = S > 1, EPI_STORE only): CTA z sums the K slices
 * [z Kc, (z+1) Kc) and writes its partial tile to ws[z]; the CTA that
 * finishes a tile last (a per-tile counter) adds the S partials in z order
 * into out0 and resets the counter -- the same bits whatever the order in
 * which the CTAs run.  `aux` is the bias. */
constexpr int TC_BN = 64;
constexpr int kMaxSplit = 8;      /* split-K factors 1, 2, 4, 8             */
constexpr int kMaxTiles = 4096;   /* output tiles a split GEMM may have     */
constexpr int TC_SMEM = 2 * (lbib_tc::BM + TC_BN) * lbib_tc::BK * 2 + 64;

template <int EPI>
__global__ void __launch_bounds__(lbib_tc::NT) mlp_gemm_tc(const __nv_bfloat16* __restrict__ A, long am, long ak,
                                                         const __nv_bfloat16* __restrict__ B, long bk, long bn, int M,
                                                         int N, int K, float* __restrict__ out0,
                                                         __nv_bfloat16* __restrict__ out1, long ldc,
                                                         const float* __restrict__ aux, int* __restrict__ err,
                                                         float* __restrict__ ws, int* __restrict__ tile_cnt) {
  const float* bias = aux;
  using namespace lbib_tc;
  constexpr int BN = TC_BN;
  extern __shared__ __align__(1024) uint8_t smem[];
  __nv_bfloat16* sA = reinterpret_cast<__nv_bfloat16*>(smem);             /* [2][BM * BK] */
  __nv_bfloat16* sB = sA + 2 * BM * BK;                                    /* [2][BN * BK] */
  uint64_t* bar = reinterpret_cast<uint64_t*>(sB + 2 * BN * BK);           /* [2]          */
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  if (warp == 0) tmem_alloc<BN>(tslot);
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  /* the B operand is staged as X(n, k) = B[n*bn + k*bk] */
  const int ma = stage_mode(A, am, ak, M, K), mb = stage_mode(B, bn, bk, N, K);
  const uint32_t idesc = instr_desc_bf16(BM, BN, ma == ST_MN_VEC, mb == ST_MN_VEC);
  /* this CTA's K slices: all of them, or its share of a split */
  const int nk_all = (K + BK - 1) / BK;
  const int S = gridDim.z, per = (nk_all + S - 1) / S;
  const int kt0 = blockIdx.z * per;
  const int nk = kt0 + per <= nk_all ? per : (nk_all > kt0 ? nk_all - kt0 : 0);
  bool ok = true;
  for (int kk = 0; kk < nk; ++kk) {
    const int kt = kt0 + kk;
    const int b = kk & 1;
    if (kk >= 2 && !__syncthreads_and(mbar_wait(&bar[b], ((kk - 2) >> 1) & 1))) {
      ok = false;
      break;
    }
    __nv_bfloat16* a_s = sA + b * BM * BK;
    __nv_bfloat16* b_s = sB + b * BN * BK;
    stage_operand<BM>(a_s, A, am, ak, m0, M, kt * BK, K, ma);
    stage_operand<BN>(b_s, B, bn, bk, n0, N, kt * BK, K, mb);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < BK / 16; ++s) {
        const uint64_t da = smem_desc(smem_u32(a_s) + s * 2 * (BM / 8) * 128, (BM / 8) * 128, 128);
        const uint64_t db = smem_desc(smem_u32(b_s) + s * 2 * (BN / 8) * 128, (BN / 8) * 128, 128);
        mma_bf16(tmem, da, db, idesc, (kk > 0 || s > 0) ? 1u : 0u);
      }
      mma_commit(&bar[b]);
    }
  }
  /* the last commit covers every MMA of the tile */
  if (nk > 0) ok = __syncthreads_and(ok && mbar_wait(&bar[(nk - 1) & 1], ((nk - 1) >> 1) & 1));
  tc_fence_after();
  __shared__ int s_last;
  if (ok) {
    const int m = m0 + warp * 32 + lane;
    float* part = S > 1 ? ws + (long)blockIdx.z * M * ldc : nullptr;
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      if (nk > 0) tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      else for (int i = 0; i < 16; ++i) v[i] = 0.0f;   /* no K slice in this split */
      if (m >= M) continue;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int n = n0 + c + i;
        if (n >= N) continue;
        float x = v[i];
        if (EPI == EPI_STORE) {
          if (S > 1) part[(long)m * ldc + n] = x;
          else out0[(long)m * ldc + n] = x;
        } else {
          x += bias[n];
          out0[(long)m * ldc + n] = x;
          if (EPI == EPI_BIAS_GELU) out1[(long)m * ldc + n] = __float2bfloat16(gelu(x));
        }
      }
    }
    if (EPI == EPI_STORE && S > 1) {
      /* the last CTA of this tile adds the partials in split order */
      __threadfence();
      __syncthreads();
      if (t == 0) {
        const int tile = blockIdx.y * gridDim.x + blockIdx.x;
        s_last = atomicAdd(&tile_cnt[tile], 1) == S - 1;
        if (s_last) tile_cnt[tile] = 0;
      }
      __syncthreads();
      if (s_last) {
        __threadfence();
        for (int e = t; e < BM * BN; e += NT) {
          const int mm = m0 + e / BN, nn = n0 + e % BN;
          if (mm >= M || nn >= N) continue;
          float acc = 0.0f;
          for (int z = 0; z < S; ++z) acc += ws[(long)z * M * ldc + (long)mm * ldc + nn];
          out0[(long)mm * ldc + nn] = acc;
        }
      }
    }
  } else if (t == 0) {
    atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_free<BN>(tmem);
}

/* X (fp32, [B][w_in]) -> bf16 [B][w_pad], pad columns 0. */
__global__ void mlp_input(const float* __restrict__ X, int B, int w, int wp, __nv_bfloat16* __restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)B * wp) return;
  const int r = (int)(i / wp), c = (int)(i % wp);
  out[i] = __float2bfloat16(c < w ? X[(long)r * w + c] : 0.0f);
}

/* Mean-squared error over the unpadded outputs: dY = 2 (Y - T) / (B w)
 * (bf16, pad columns 0), and per-block loss partials. */
__global__ void mlp_mse(const float* __restrict__ Y, const float* __restrict__ T, int B, int w, int wp,
                        __nv_bfloat16* __restrict__ dY, float* __restrict__ part) {
  __shared__ float s[256];
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (i < (long)B * wp) {
    const int r = (int)(i / wp), c = (int)(i % wp);
    float d = 0.0f;
    if (c < w) {
      const float e = Y[i] - T[(long)r * w + c];
      l = e * e;
      d = 2.0f * e / ((float)B * (float)w);
    }
    dY[i] = __float2bfloat16(d);
  }
  s[threadIdx.x] = l;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

__global__ void mlp_sum(const float* __restrict__ part, int n, float scale, float* __restrict__ out) {
  __shared__ float s[256];
  float v = 0.0f;
  for (int i = threadIdx.x; i < n; i += 256) v += part[i];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0] * scale;
}

/* dZ = dA * gelu'(Z), bf16. */
__global__ void mlp_gelu_back(const float* __restrict__ dA, const float* __restrict__ Z, long n,
                              __nv_bfloat16* __restrict__ dZ) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dZ[i] = __float2bfloat16(dA[i] * gelu_grad(Z[i]));
}

/* db[n] = sum over the batch of dZ[:, n], in a fixed order: thread
 * (c, g) of a 32 x 32 block sums rows g, g + 32, ... of column 32 blockIdx.x
 * + c, then the 32 partial sums of a column are added in g order. */
__global__ void __launch_bounds__(1024) mlp_bias_grad(const __nv_bfloat16* __restrict__ dZ, int B, int w,
                                                     float* __restrict__ db) {
  __shared__ float part[32][33];
  const int c = threadIdx.x, g = threadIdx.y;
  const int n = blockIdx.x * 32 + c;
  float s = 0.0f;
  if (n < w)
    for (int r = g; r < B; r += 32) s += __bfloat162float(dZ[(long)r * w + n]);
  part[g][c] = s;
  __syncthreads();
  if (g == 0 && n < w) {
    float t = 0.0f;
    for (int k = 0; k < 32; ++k) t += part[k][c];
    db[n] = t;
  }
}

/* Adam on the fp32 master copy; refresh the bf16 weights. */
__global__ void mlp_adam(float* __restrict__ p, const float* __restrict__ gr, float* __restrict__ m,
                         float* __restrict__ v, long n, float lr, float b1, float b2, float eps, float c1, float c2,
                         __nv_bfloat16* __restrict__ wbf, const int* __restrict__ is_w) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = gr[i];
  const float mi = b1 * m[i] + (1.0f - b1) * g;
  const float vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float x = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = x;
  if (is_w[i] >= 0) wbf[is_w[i]] = __float2bfloat16(x);
}

long align16(long v) { return (v + 15) / 16 * 16; }

}  // namespace

/* ------------------------------------------------------------ state */

struct lbib_mlp {
  int L;
  int* w;               /* [L+1] widths */
  int* wp;              /* [L+1] padded */
  int max_batch;
  long np;              /* padded parameter count */
  float *p, *g, *m, *v; /* master params, grads, Adam moments (padded layout) */
  int* wmap;            /* padded param index -> bf16 weight index, or -1 */
  __nv_bfloat16* wbf;   /* bf16 weights, layer after layer, [wp_{l+1}][wp_l] */
  long* woff;           /* [L] offset of W_l in p (padded) */
  long* boff;           /* [L] offset of b_l in p */
  long* wbo;            /* [L] offset of W_l in wbf */
  __nv_bfloat16** act;  /* [L+1] bf16 activations [B][wp_l] (act[0] = input) */
  float** z;            /* [L] pre-activations fp32 [B][wp_{l+1}] */
  float* dA;            /* fp32 [B][max wp]                               */
  __nv_bfloat16* dZ;    /* bf16 [2][B][max wp]: layer l's dZ, and l-1's  */
  float* ws;            /* split-K partial tiles                          */
  long ws_elems;
  int* tile_cnt;        /* split-K arrivals per output tile (kMaxTiles)   */
  float* part;
  float* d_loss;
  int* d_err;           /* a tensor-core GEMM's mbarrier wait ran out     */
  int maxw;             /* largest padded width                           */
  long steps;
  cudaStream_t stream;  /* where the work runs: own_stream or the caller's */
  cudaStream_t own_stream;
};

namespace {

int launch_gemm(lbib_mlp* n, int epi, const __nv_bfloat16* A, long am, long ak, const __nv_bfloat16* B, long bk,
                long bn, int M, int N, int K, float* out0, __nv_bfloat16* out1, long ldc, const float* bias) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(mlp_gemm_tc<EPI_STORE>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    cudaFuncSetAttribute(mlp_gemm_tc<EPI_BIAS>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    cudaFuncSetAttribute(mlp_gemm_tc<EPI_BIAS_GELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    attr = true;
  }
  dim3 grid((unsigned)((N + TC_BN - 1) / TC_BN), (unsigned)((M + lbib_tc::BM - 1) / lbib_tc::BM), 1);
  /* a long K over few tiles (the weight gradients, K = batch) is split so
     that ~32 CTAs share it; the split depends on the shape only */
  if (epi == EPI_STORE) {
    const int tiles = (int)(grid.x * grid.y), nkt = (K + lbib_tc::BK - 1) / lbib_tc::BK;
    int sk = 1;
    while (sk * 2 <= kMaxSplit && tiles * sk < 32 && nkt >= 4 * sk * 2) sk *= 2;
    if ((long)sk * M * ldc > n->ws_elems || tiles > kMaxTiles) sk = 1;
    grid.z = (unsigned)sk;
  }
  switch (epi) {
    case EPI_BIAS_GELU:
      mlp_gemm_tc<EPI_BIAS_GELU><<<grid, lbib_tc::NT, TC_SMEM, n->stream>>>(A, am, ak, B, bk, bn, M, N, K, out0,
                                                                            out1, ldc, bias, n->d_err, n->ws,
                                                                            n->tile_cnt);
      break;
    case EPI_BIAS:
      mlp_gemm_tc<EPI_BIAS><<<grid, lbib_tc::NT, TC_SMEM, n->stream>>>(A, am, ak, B, bk, bn, M, N, K, out0, out1,
                                                                       ldc, bias, n->d_err, n->ws, n->tile_cnt);
      break;
    default:
      mlp_gemm_tc<EPI_STORE><<<grid, lbib_tc::NT, TC_SMEM, n->stream>>>(A, am, ak, B, bk, bn, M, N, K, out0, out1,
                                                                        ldc, bias, n->d_err, n->ws, n->tile_cnt);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* Forward pass of `batch` rows; the output (fp32) is z[L-1]. */
int forward(lbib_mlp* n, const float* X, int batch) {
  const unsigned nb = (unsigned)(((long)batch * n->wp[0] + 255) / 256);
  mlp_input<<<nb, 256, 0, n->stream>>>(X, batch, n->w[0], n->wp[0], n->act[0]);
  for (int l = 0; l < n->L; ++l) {
    const int in = n->wp[l], out = n->wp[l + 1];
    const __nv_bfloat16* W = n->wbf + n->wbo[l];
    const float* b = n->p + n->boff[l];
    const int epi = l + 1 < n->L ? EPI_BIAS_GELU : EPI_BIAS;
    if (launch_gemm(n, epi, n->act[l], in, 1, W, 1, in, batch, out, in, n->z[l], n->act[l + 1], out, b)) return -2;
  }
  return 0;
}

/* Gradients of the mean-squared error into n->g (padded layout). */
int backward(lbib_mlp* n, const float* T, int batch) {
  const int L = n->L;
  const long ny = (long)batch * n->wp[L];
  const unsigned nb = (unsigned)((ny + 255) / 256);
  const long zst = (long)n->max_batch * n->maxw;       /* the two dZ buffers */
  mlp_mse<<<nb, 256, 0, n->stream>>>(n->z[L - 1], T, batch, n->w[L], n->wp[L], n->dZ, n->part);
  mlp_sum<<<1, 256, 0, n->stream>>>(n->part, (int)nb, 1.0f / ((float)batch * (float)n->w[L]), n->d_loss);
  for (int l = L - 1; l >= 0; --l) {
    const int in = n->wp[l], out = n->wp[l + 1];
    __nv_bfloat16* dZ = n->dZ + ((L - 1 - l) & 1) * zst;
    __nv_bfloat16* dZ_prev = n->dZ + ((L - l) & 1) * zst;
    /* dW = dZ^T X: M = out, N = in, K = batch */
    if (launch_gemm(n, EPI_STORE, dZ, 1, out, n->act[l], in, 1, out, in, batch, n->g + n->woff[l], NULL, in, NULL))
      return -2;
    mlp_bias_grad<<<(out + 31) / 32, dim3(32, 32), 0, n->stream>>>(dZ, batch, out, n->g + n->boff[l]);
    if (l == 0) break;
    /* dZ_{l-1} = (dZ W) * gelu'(Z_{l-1}): M = batch, N = in, K = out */
    const __nv_bfloat16* W = n->wbf + n->wbo[l];
    /* the GELU derivative (erf and exp per element) is an element-wise
       kernel of its own: inside the GEMM's epilogue it ran on the GEMM's
       few CTAs and took longer than the separate launch */
    if (launch_gemm(n, EPI_STORE, dZ, out, 1, W, in, 1, batch, in, out, n->dA, NULL, in, NULL)) return -2;
    const long na = (long)batch * in;
    mlp_gelu_back<<<(unsigned)((na + 255) / 256), 256, 0, n->stream>>>(n->dA, n->z[l - 1], na, dZ_prev);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* ABI parameter index <-> padded index. */
long abi_count(const lbib_mlp* n) {
  long c = 0;
  for (int l = 0; l < n->L; ++l) c += (long)n->w[l + 1] * n->w[l] + n->w[l + 1];
  return c;
}

template <typename F>
void for_each_param(const lbib_mlp* n, F f) {
  long a = 0;
  for (int l = 0; l < n->L; ++l) {
    for (int r = 0; r < n->w[l + 1]; ++r)
      for (int c = 0; c < n->w[l]; ++c) f(a++, n->woff[l] + (long)r * n->wp[l] + c);
    for (int r = 0; r < n->w[l + 1]; ++r) f(a++, n->boff[l] + r);
  }
}

int refresh_bf16(lbib_mlp* n) {
  /* wbf from the master copy (host round trip; set-up only) */
  float* hp = (float*)malloc(sizeof(float) * n->np);
  int* map = (int*)malloc(sizeof(int) * n->np);
  long nw = n->wbo[n->L - 1] + (long)n->wp[n->L] * n->wp[n->L - 1];
  __nv_bfloat16* hw = (__nv_bfloat16*)malloc(sizeof(__nv_bfloat16) * nw);
  int rc = (!hp || !map || !hw) ? -5 : 0;
  if (!rc && cudaMemcpy(hp, n->p, sizeof(float) * n->np, cudaMemcpyDeviceToHost) != cudaSuccess) rc = -2;
  if (!rc && cudaMemcpy(map, n->wmap, sizeof(int) * n->np, cudaMemcpyDeviceToHost) != cudaSuccess) rc = -2;
  if (!rc) {
    for (long i = 0; i < nw; ++i) hw[i] = __float2bfloat16(0.0f);
    for (long i = 0; i < n->np; ++i)
      if (map[i] >= 0) hw[map[i]] = __float2bfloat16(hp[i]);
    if (cudaMemcpy(n->wbf, hw, sizeof(__nv_bfloat16) * nw, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
  }
  free(hp);
  free(map);
  free(hw);
  return rc;
}

/* splitmix64 stream for the initial weights */
double uniform01(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace

extern "C" {

lbib_mlp* lbib_mlp_create(int n_layers, const int* widths, int max_batch, unsigned long long seed) {
  if (n_layers < 1 || n_layers > 16 || !widths || max_batch < 1) return NULL;
  for (int l = 0; l <= n_layers; ++l)
    if (widths[l] < 1 || widths[l] > 4096) return NULL;
  lbib_mlp* n = (lbib_mlp*)calloc(1, sizeof(lbib_mlp));
  if (!n) return NULL;
  const int L = n_layers;
  n->L = L;
  n->max_batch = max_batch;
  n->w = (int*)calloc(L + 1, sizeof(int));
  n->wp = (int*)calloc(L + 1, sizeof(int));
  n->woff = (long*)calloc(L, sizeof(long));
  n->boff = (long*)calloc(L, sizeof(long));
  n->wbo = (long*)calloc(L, sizeof(long));
  n->act = (__nv_bfloat16**)calloc(L + 1, sizeof(void*));
  n->z = (float**)calloc(L, sizeof(void*));
  int rc = (!n->w || !n->wp || !n->woff || !n->boff || !n->wbo || !n->act || !n->z) ? -5 : 0;
  int maxw = 0;
  long np = 0, nw = 0;
  for (int l = 0; l <= L && !rc; ++l) {
    n->w[l] = widths[l];
    n->wp[l] = (int)align16(widths[l]);
    if (n->wp[l] > maxw) maxw = n->wp[l];
  }
  for (int l = 0; l < L && !rc; ++l) {
    n->woff[l] = np;
    np += (long)n->wp[l + 1] * n->wp[l];
    n->boff[l] = np;
    np += n->wp[l + 1];
    n->wbo[l] = nw;
    nw += (long)n->wp[l + 1] * n->wp[l];
  }
  n->np = np;
  n->maxw = maxw;
  if (!rc && cudaStreamCreateWithFlags(&n->own_stream, cudaStreamNonBlocking) != cudaSuccess) rc = -2;
  n->stream = n->own_stream;
  const size_t fp = sizeof(float) * np;
  if (!rc && cudaMalloc(&n->p, fp) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&n->g, fp) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&n->m, fp) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&n->v, fp) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&n->wmap, sizeof(int) * np) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&n->wbf, sizeof(__nv_bfloat16) * nw) != cudaSuccess) rc = -5;
  for (int l = 0; l <= L && !rc; ++l)
    if (cudaMalloc(&n->act[l], sizeof(__nv_bfloat16) * max_batch * n->wp[l]) != cudaSuccess) rc = -5;
  for (int l = 0; l < L && !rc; ++l)
    if (cudaMalloc(&n->z[l], sizeof(float) * max_batch * n->wp[l + 1]) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&n->dA, sizeof(float) * max_batch * maxw) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&n->dZ, sizeof(__nv_bfloat16) * 2 * max_batch * maxw) != cudaSuccess) rc = -5;
  /* split-K partials: up to kMaxSplit copies of the largest weight matrix */
  n->ws_elems = 0;
  for (int l = 0; l < L; ++l)
    if ((long)n->wp[l + 1] * n->wp[l] > n->ws_elems) n->ws_elems = (long)n->wp[l + 1] * n->wp[l];
  n->ws_elems *= kMaxSplit;
  if (!rc && cudaMalloc(&n->ws, sizeof(float) * n->ws_elems) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&n->tile_cnt, sizeof(int) * kMaxTiles) != cudaSuccess) rc = -5;
  if (!rc && cudaMemset(n->tile_cnt, 0, sizeof(int) * kMaxTiles) != cudaSuccess) rc = -2;
  if (!rc && cudaMalloc(&n->part, sizeof(float) * ((long)max_batch * maxw / 256 + 2)) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&n->d_loss, sizeof(float)) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&n->d_err, sizeof(int)) != cudaSuccess) rc = -5;
  if (!rc && cudaMemset(n->d_err, 0, sizeof(int)) != cudaSuccess) rc = -2;
  if (!rc) {
    /* He-uniform weights for the GELU layers (bound sqrt(6 / fan_in)),
       zero biases, zero padding */
    float* hp = (float*)calloc(np, sizeof(float));
    int* map = (int*)malloc(sizeof(int) * np);
    uint64_t s = seed;
    if (!hp || !map) rc = -5;
    for (long i = 0; i < np && !rc; ++i) map[i] = -1;
    for (int l = 0; l < L && !rc; ++l) {
      const double bound = sqrt(6.0 / n->w[l]);
      for (int r = 0; r < n->wp[l + 1]; ++r)
        for (int c = 0; c < n->wp[l]; ++c) {
          const long i = n->woff[l] + (long)r * n->wp[l] + c;
          map[i] = (int)(n->wbo[l] + (long)r * n->wp[l] + c);
          if (r < n->w[l + 1] && c < n->w[l]) hp[i] = (float)((2.0 * uniform01(&s) - 1.0) * bound);
        }
    }
    if (!rc && cudaMemcpy(n->p, hp, fp, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
    if (!rc && cudaMemcpy(n->wmap, map, sizeof(int) * np, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
    free(hp);
    free(map);
  }
  if (!rc && (cudaMemset(n->m, 0, fp) != cudaSuccess || cudaMemset(n->v, 0, fp) != cudaSuccess ||
              cudaMemset(n->g, 0, fp) != cudaSuccess))
    rc = -2;
  if (!rc) rc = refresh_bf16(n);
  if (rc) {
    lbib_mlp_free(n);
    return NULL;
  }
  return n;
}

void lbib_mlp_free(lbib_mlp* n) {
  if (!n) return;
  if (n->stream) cudaStreamSynchronize(n->stream);
  cudaFree(n->p); cudaFree(n->g); cudaFree(n->m); cudaFree(n->v); cudaFree(n->wmap); cudaFree(n->wbf);
  for (int l = 0; l <= n->L && n->act; ++l) cudaFree(n->act[l]);
  for (int l = 0; l < n->L && n->z; ++l) cudaFree(n->z[l]);
  cudaFree(n->dA); cudaFree(n->dZ); cudaFree(n->part); cudaFree(n->d_loss); cudaFree(n->d_err);
  cudaFree(n->ws); cudaFree(n->tile_cnt);
  if (n->own_stream) cudaStreamDestroy(n->own_stream);
  free(n->w); free(n->wp); free(n->woff); free(n->boff); free(n->wbo); free(n->act); free(n->z);
  free(n);
}

long lbib_mlp_param_count(lbib_mlp* n) { return n ? abi_count(n) : 0; }

void* lbib_mlp_stream(lbib_mlp* n) { return n ? (void*)n->stream : NULL; }

/* Run on the caller's stream (NULL is the CUDA default stream, as in every
 * CUDA call), so the caller's writes of X and T are ordered before the
 * kernels that read them and its allocator may recycle their memory as
 * soon as later work on that stream starts. */
int lbib_mlp_set_stream(lbib_mlp* n, void* stream) {
  if (!n) return LBIB_E_ARG;
  if (cudaStreamSynchronize(n->stream) != cudaSuccess) return LBIB_E_CUDA;
  n->stream = (cudaStream_t)stream;
  return LBIB_OK;
}

int lbib_mlp_get_params(lbib_mlp* n, float* out) {
  if (!n || !out) return LBIB_E_ARG;
  float* hp = (float*)malloc(sizeof(float) * n->np);
  if (!hp) return LBIB_E_NOMEM;
  int rc = cudaMemcpy(hp, n->p, sizeof(float) * n->np, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : LBIB_E_CUDA;
  if (!rc) for_each_param(n, [&](long a, long i) { out[a] = hp[i]; });
  free(hp);
  return rc;
}

int lbib_mlp_set_params(lbib_mlp* n, const float* in) {
  if (!n || !in) return LBIB_E_ARG;
  float* hp = (float*)calloc(n->np, sizeof(float));
  if (!hp) return LBIB_E_NOMEM;
  for_each_param(n, [&](long a, long i) { hp[i] = in[a]; });
  int rc = cudaMemcpy(n->p, hp, sizeof(float) * n->np, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : LBIB_E_CUDA;
  free(hp);
  if (!rc && refresh_bf16(n)) rc = LBIB_E_CUDA;
  return rc;
}

/* X [batch][w_0] fp32 and Y [batch][w_L] fp32, device pointers. */
int lbib_mlp_forward(lbib_mlp* n, const float* X, int batch, float* Y) {
  if (!n || !X || !Y || batch < 1 || batch > n->max_batch) return LBIB_E_ARG;
  if (forward(n, X, batch)) return LBIB_E_CUDA;
  const int L = n->L;
  if (cudaMemcpy2DAsync(Y, sizeof(float) * n->w[L], n->z[L - 1], sizeof(float) * n->wp[L], sizeof(float) * n->w[L],
                        batch, cudaMemcpyDeviceToDevice, n->stream) != cudaSuccess)
    return LBIB_E_CUDA;
  return lbib_mlp_synchronize(n);
}

/* Loss and gradient (ABI order, host array of lbib_mlp_param_count floats)
 * of the mean-squared error on one batch, without updating anything. */
int lbib_mlp_gradient(lbib_mlp* n, const float* X, const float* T, int batch, float* grad, float* loss) {
  if (!n || !X || !T || batch < 1 || batch > n->max_batch) return LBIB_E_ARG;
  if (forward(n, X, batch) || backward(n, T, batch)) return LBIB_E_CUDA;
  float* hg = (float*)malloc(sizeof(float) * n->np);
  if (!hg) return LBIB_E_NOMEM;
  int rc = 0;
  if (cudaMemcpyAsync(hg, n->g, sizeof(float) * n->np, cudaMemcpyDeviceToHost, n->stream) != cudaSuccess ||
      (loss && cudaMemcpyAsync(loss, n->d_loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream) != cudaSuccess) ||
      cudaStreamSynchronize(n->stream) != cudaSuccess)
    rc = LBIB_E_CUDA;
  if (!rc) rc = lbib_mlp_synchronize(n);
  if (!rc && grad) for_each_param(n, [&](long a, long i) { grad[a] = hg[i]; });
  free(hg);
  return rc;
}

/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on one batch; X, T are
 * device pointers; loss (host, may be NULL) gets the batch's loss before
 * the step.  Asynchronous unless loss is asked for. */
int lbib_mlp_train_step(lbib_mlp* n, const float* X, const float* T, int batch, float lr, float* loss) {
  if (!n || !X || !T || batch < 1 || batch > n->max_batch || !(lr > 0)) return LBIB_E_ARG;
  if (forward(n, X, batch) || backward(n, T, batch)) return LBIB_E_CUDA;
  n->steps++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = (float)(1.0 - pow(b1, (double)n->steps)), c2 = (float)(1.0 - pow(b2, (double)n->steps));
  mlp_adam<<<(unsigned)((n->np + 255) / 256), 256, 0, n->stream>>>(n->p, n->g, n->m, n->v, n->np, lr, b1, b2, 1e-8f,
                                                                    c1, c2, n->wbf, n->wmap);
  if (cudaGetLastError() != cudaSuccess) return LBIB_E_CUDA;
  if (loss) {
    if (cudaMemcpyAsync(loss, n->d_loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream) != cudaSuccess ||
        cudaStreamSynchronize(n->stream) != cudaSuccess)
      return LBIB_E_CUDA;
  }
  return LBIB_OK;
}

/* Waits for the MLP's work; LBIB_E_CUDA also when a tensor-core GEMM
 * gave up waiting on its mbarrier (its output tile was not written). */
int lbib_mlp_synchronize(lbib_mlp* n) {
  if (!n) return LBIB_E_ARG;
  int e = 0;
  if (cudaMemcpyAsync(&e, n->d_err, sizeof(int), cudaMemcpyDeviceToHost, n->stream) != cudaSuccess ||
      cudaStreamSynchronize(n->stream) != cudaSuccess)
    return LBIB_E_CUDA;
  return e ? LBIB_E_CUDA : LBIB_OK;
}

}  /* extern "C" */
