/*
 * The one-grid launch of the FP64 two-cell step (lbib_x2.cuh) over the rows
 * away from the walls.  Twice the bytes per memory instruction of the
 * one-cell kernel: the AA pattern alone measures 87% of the HBM copy peak at
 * one cell per thread and 96% at two.
 */
#include "lbib_internal.h"
#include "lbib_x2.cuh"

using namespace lbib;

namespace {

constexpr int TPB = 128;

/* Resident blocks per SM each parity's kernel is compiled for (the register
 * budget): 3 x 128 threads at up to 168 registers. */
#ifndef LBIB_X2_MINB0
#define LBIB_X2_MINB0 3
#endif
#ifndef LBIB_X2_MINB1
#define LBIB_X2_MINB1 3
#endif

struct X2Params {
  FluidParams p;
  int nry;       /* interior rows in y: ny - 6 */
  int npairs;    /* pairs per row: (xhi - xlo + 1) / 2 */
  long pf;       /* L2 prefetch distance in blocks (0: none) */
};

/* Threads 0..18 ask L2 for plane q of the rows of the block pf blocks
 * later in launch order (blockIdx.x fastest): the loads it will issue. */
template <int PAR>
__device__ __forceinline__ void x2_prefetch(const X2Params& b, int q) {
  const long nrow = gridDim.x;
  const long L = (long)blockIdx.y * nrow + blockIdx.x + b.pf;
  if (L >= nrow * gridDim.y) return;
  const int row = (int)(L % nrow), pb = (int)(L / nrow);
  const int y = 3 + row % b.nry, z = 3 + row / b.nry;
  const int pr0 = pb * TPB;
  const int pr1 = pr0 + TPB < b.npairs ? pr0 + TPB : b.npairs;
  const FluidParams& p = b.p;
  const long idx = sidx(p, p.xlo + 2 * pr0, y, z);
  const double* src = PAR ? p.f + opp(q) * p.N + idx - link_offset(q, p.sx, (long)p.sx * p.ny) : p.f + q * p.N + idx;
  l2_prefetch(src, src + 2L * (pr1 - pr0), p.f, p.f + 19 * p.N);
}

template <int PAR>
__global__ void __launch_bounds__(TPB, PAR ? LBIB_X2_MINB1 : LBIB_X2_MINB0) lbib_fluid_step_x2(X2Params b) {
  if (b.pf > 0 && threadIdx.x < 19) x2_prefetch<PAR>(b, threadIdx.x);
  const int pr = blockIdx.y * TPB + threadIdx.x;
  if (pr >= b.npairs) return;
  const int y = 3 + (int)(blockIdx.x % b.nry);
  const int z = 3 + (int)(blockIdx.x / b.nry);
  x2_pair<PAR>(b.p, b.p.xlo + 2 * pr, y, z);
}

}  // namespace

/* Interior-row ranges of this kernel: y in [3, ny-4], z in
 * [3, min(nz-4, zin_hi)].  Returns 0 when there are none. */
extern "C" int lbdev_bulk_rows(const lbib_device* d, int* nrows_y, int* nrows_z) {
  *nrows_y = d->ny - 6;
  int zb = d->nz - 4;
  if (d->zin_hi < zb) zb = d->zin_hi;
  *nrows_z = zb - 2;
  return (*nrows_y > 0 && *nrows_z > 0);
}

extern "C" int lbdev_launch_fluid_bulk(lbib_device* d, const void* fluid_params) {
  X2Params b;
  b.p = *(const FluidParams*)fluid_params;
  int nrz = 0;
  if (!lbdev_bulk_rows(d, &b.nry, &nrz)) return 0;
  b.npairs = (b.p.xhi - b.p.xlo + 1) / 2;
  b.pf = 0;
  if (d->l2_pf > 0) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device);
    b.pf = (long)d->l2_pf * sms * (d->parity ? LBIB_X2_MINB1 : LBIB_X2_MINB0);
  }
  dim3 grid((unsigned)((long)b.nry * nrz), (unsigned)((b.npairs + TPB - 1) / TPB));
  if (d->parity == 0) lbib_fluid_step_x2<0><<<grid, TPB, 0, d->fluid_stream>>>(b);
  else lbib_fluid_step_x2<1><<<grid, TPB, 0, d->fluid_stream>>>(b);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}
