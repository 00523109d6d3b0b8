/*
 * Force spreading without any allocation: lbib_spread_force_noalloc.
 *
 * Who needs it: a host that cannot call cudaMalloc or any allocating routine
 * while it runs -- for example one that hands the library buffers from its
 * own fixed pool and forbids allocation after start-up (allocation there can
 * synchronise the device or fail under a memory cap), or one driving the
 * spread from a context where the library may not grow its footprint.  The
 * regular path (fiber_SpreadForce inside a GV) allocates its tile lists,
 * maps and weights when the sheet is uploaded.
 *
 * What it does: the same sum as the regular spread -- every node's elastic
 * force times the 4-point cosine delta kernel over its 4x4x4 stencil, each
 * cell adding its contributions in (sheet, row, col) node order with the same
 * operation order -- into dense outputs the caller provides.  Instead of
 * per-tile node lists it keeps, per 32-node chunk, the bounding box of the
 * chunk's stencils, and walks the 4^3 tiles inside the box of all stencils;
 * each tile visits the chunks whose box meets it, in order, and recomputes
 * the delta factors of their nodes in shared memory.
 *
 * Scratch: the file-scope device array lbib_noalloc_scratch below
 * (LBIB_NOALLOC_SCRATCH_INTS ints: 6 per 32-node chunk for up to
 * LBIB_NOALLOC_MAX_NODES = 2^18 nodes, 192 KiB, plus an 8-int header), which
 * every GPU that loads this library holds until the process exits.
 */
#include <cuda_runtime.h>
#include <limits.h>

#include "../../include/lbib.h"
#include "lbib_cos.h"

#define LBIB_NOALLOC_HEADER_INTS 8
#define LBIB_NOALLOC_SCRATCH_INTS (LBIB_NOALLOC_HEADER_INTS + 6 * (LBIB_NOALLOC_MAX_NODES / 32))

/* [0..5] box of all stencils (min x, max x, min y, max y, min z, max z),
 * [6] error code, [7] spare, then 6 ints per 32-node chunk. */
static __device__ __align__(256) int lbib_noalloc_scratch[LBIB_NOALLOC_SCRATCH_INTS];

namespace {

constexpr double kPiNa = 3.14159265358979;  /* the reference's truncated PI */

__device__ __forceinline__ int na_start(double p) { return (int)(floor(p / 1.0 - 2) + 1); }

/* start = floor(p - 2) + 1 in [0, n - 4] <=> 1 <= p < n - 2, tested on the
 * double so that NaN and huge coordinates are rejected before any int
 * conversion. */
__device__ __forceinline__ bool na_inside(double p, int n) { return p >= 1.0 && p < (double)n - 2.0; }

/* Everything that must start a call at a known value. */
__global__ void na_clear(int* s) {
  s[0] = INT_MAX; s[1] = INT_MIN; s[2] = INT_MAX; s[3] = INT_MIN; s[4] = INT_MAX; s[5] = INT_MIN;
  s[6] = 0; s[7] = 0;
}

/* Per node: stencil start and grid check; per 32-node chunk: the box of its
 * stencils; over all nodes: the box of all stencils. */
__global__ void na_boxes(const double* __restrict__ nodes, long S, int nx, int ny, int nz, int* s) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int b0 = INT_MAX, b1 = INT_MIN, b2 = INT_MAX, b3 = INT_MIN, b4 = INT_MAX, b5 = INT_MIN;
  if (i < S) {
    const double* m = nodes + i * 12;
    if (!(na_inside(m[0], nx) && na_inside(m[1], ny) && na_inside(m[2], nz))) {
      atomicCAS(&s[6], 0, LBIB_E_STENCIL);
    } else {
      const int is = na_start(m[0]), js = na_start(m[1]), ks = na_start(m[2]);
      b0 = is; b1 = is + 3; b2 = js; b3 = js + 3; b4 = ks; b5 = ks + 3;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    b0 = min(b0, __shfl_xor_sync(0xffffffffu, b0, o));
    b1 = max(b1, __shfl_xor_sync(0xffffffffu, b1, o));
    b2 = min(b2, __shfl_xor_sync(0xffffffffu, b2, o));
    b3 = max(b3, __shfl_xor_sync(0xffffffffu, b3, o));
    b4 = min(b4, __shfl_xor_sync(0xffffffffu, b4, o));
    b5 = max(b5, __shfl_xor_sync(0xffffffffu, b5, o));
  }
  const long chunk = i >> 5;
  if ((threadIdx.x & 31) == 0 && chunk * 32 < S) {
    int* bx = s + LBIB_NOALLOC_HEADER_INTS + chunk * 6;
    bx[0] = b0; bx[1] = b1; bx[2] = b2; bx[3] = b3; bx[4] = b4; bx[5] = b5;
    if (b0 <= b1) {
      atomicMin(&s[0], b0); atomicMax(&s[1], b1);
      atomicMin(&s[2], b2); atomicMax(&s[3], b3);
      atomicMin(&s[4], b4); atomicMax(&s[5], b5);
    }
  }
}

/* One CTA (64 threads = one 4^3 tile) per tile inside the box of all
 * stencils; chunks in node order, nodes of a chunk in order. */
__global__ void __launch_bounds__(64) na_gather(const double* __restrict__ nodes, long S, long nchunks, int nx,
                                                int ny, int nz, const int* __restrict__ s, double* __restrict__ fx,
                                                double* __restrict__ fy, double* __restrict__ fz) {
  __shared__ int hit[64];
  __shared__ int s_st[32][3];
  __shared__ double s_w[32][12];
  __shared__ double s_fe[32][3];
  if (s[6] != 0 || s[0] > s[1]) return;
  const int tx0 = s[0] >> 2, ty0 = s[2] >> 2, tz0 = s[4] >> 2;
  const int ntx = (s[1] >> 2) - tx0 + 1, nty = (s[3] >> 2) - ty0 + 1, ntz = (s[5] >> 2) - tz0 + 1;
  const long ntiles = (long)ntx * nty * ntz;
  const int cell = threadIdx.x;
  const double cf = 1.0 / (64.0 * 1.0 * 1.0 * 1.0);
  const double cxk = kPiNa / (2.0 * 1.0);
  for (long it = blockIdx.x; it < ntiles; it += gridDim.x) {
    const int tx = tx0 + (int)(it % ntx), ty = ty0 + (int)((it / ntx) % nty), tz = tz0 + (int)(it / ((long)ntx * nty));
    const int x0 = tx * 4, y0 = ty * 4, z0 = tz * 4;
    const int gx = x0 + (cell & 3), gy = y0 + ((cell >> 2) & 3), gz = z0 + (cell >> 4);
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    for (long c0 = 0; c0 < nchunks; c0 += 64) {
      const long c = c0 + cell;
      int h = 0;
      if (c < nchunks) {
        const int* bx = s + LBIB_NOALLOC_HEADER_INTS + c * 6;
        h = !(bx[1] < x0 || bx[0] > x0 + 3 || bx[3] < y0 || bx[2] > y0 + 3 || bx[5] < z0 || bx[4] > z0 + 3);
      }
      __syncthreads();
      hit[cell] = h;
      __syncthreads();
      for (int k = 0; k < 64; ++k) {
        if (!hit[k]) continue;
        const long base = (c0 + k) * 32;
        /* node j = cell / 2 of the chunk: its start and half of its 12 factors */
        const int j = cell >> 1, half = cell & 1;
        const long nd = base + j;
        if (nd < S) {
          const double* m = nodes + nd * 12;
          const int st[3] = {na_start(m[0]), na_start(m[1]), na_start(m[2])};
          if (half == 0) {
            s_st[j][0] = st[0]; s_st[j][1] = st[1]; s_st[j][2] = st[2];
            s_fe[j][0] = m[9]; s_fe[j][1] = m[10]; s_fe[j][2] = m[11];
          }
          for (int a = 6 * half; a < 6 * half + 6; ++a) {
            const int ax = a >> 2, off = a & 3;
            s_w[j][a] = 1.0e0 + lbib_cos_2phase(cxk * (1.0 * (st[ax] + off) - m[ax]));
          }
        } else if (half == 0) {
          s_st[j][0] = INT_MIN / 2; s_st[j][1] = INT_MIN / 2; s_st[j][2] = INT_MIN / 2;
        }
        __syncthreads();
        for (int q = 0; q < 32; ++q) {
          const int a = gx - s_st[q][0], b = gy - s_st[q][1], e = gz - s_st[q][2];
          if ((unsigned)a < 4u && (unsigned)b < 4u && (unsigned)e < 4u) {
            const double tmp = cf * s_w[q][a] * s_w[q][4 + b] * s_w[q][8 + e];
            Fx = Fx + s_fe[q][0] * tmp;
            Fy = Fy + s_fe[q][1] * tmp;
            Fz = Fz + s_fe[q][2] * tmp;
          }
        }
        __syncthreads();
      }
    }
    if (gx < nx && gy < ny && gz < nz) {
      const long idx = ((long)gz * ny + gy) * nx + gx;
      fx[idx] = Fx; fy[idx] = Fy; fz[idx] = Fz;
    }
  }
}

/* Device address of lbib_noalloc_scratch in the current device's context.
 * Looked up on every call (no cache): after a cudaDeviceReset, or under
 * another context on the same device ordinal, the module is loaded anew and
 * an address kept from before would point at freed memory.  The lookup
 * allocates nothing once the module is loaded (the first call on a device
 * loads it). */
int scratch_for_current_device(int** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, lbib_noalloc_scratch) != cudaSuccess || !p) return LBIB_E_CUDA;
  *out = (int*)p;
  return LBIB_OK;
}

}  // namespace

extern "C" int lbib_spread_force_noalloc(const double* nodes, long num_nodes, int nx, int ny, int nz, double* fx,
                                         double* fy, double* fz, void* stream) {
  if (!nodes || !fx || !fy || !fz || num_nodes < 1 || nx < 4 || ny < 4 || nz < 4) return LBIB_E_ARG;
  if (num_nodes > LBIB_NOALLOC_MAX_NODES) return LBIB_E_LIMIT;
  /* a launch error left by earlier, unrelated work is not this call's:
     refuse to run on it rather than report it as ours */
  if (cudaPeekAtLastError() != cudaSuccess) return LBIB_E_CUDA;
  int* s = nullptr;
  int rc = scratch_for_current_device(&s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const long N = (long)nx * ny * nz;
  const long nchunks = (num_nodes + 31) / 32;
  na_clear<<<1, 1, 0, st>>>(s);
  if (cudaGetLastError() != cudaSuccess) return LBIB_E_CUDA;
  if (cudaMemsetAsync(fx, 0, sizeof(double) * N, st) != cudaSuccess ||
      cudaMemsetAsync(fy, 0, sizeof(double) * N, st) != cudaSuccess ||
      cudaMemsetAsync(fz, 0, sizeof(double) * N, st) != cudaSuccess)
    return LBIB_E_CUDA;
  na_boxes<<<(unsigned)((num_nodes + 127) / 128), 128, 0, st>>>(nodes, num_nodes, nx, ny, nz, s);
  if (cudaGetLastError() != cudaSuccess) return LBIB_E_CUDA;
  na_gather<<<148 * 8, 64, 0, st>>>(nodes, num_nodes, nchunks, nx, ny, nz, s, fx, fy, fz);
  if (cudaGetLastError() != cudaSuccess) return LBIB_E_CUDA;
  int err = 0;
  if (cudaMemcpyAsync(&err, s + 6, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return LBIB_E_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return LBIB_E_CUDA;
  return err;
}
