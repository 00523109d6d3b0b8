/*
 * x-slab decomposition of one grid over several states (one per GPU):
 * the exchange of the columns next to a slab face.  No reference
 * counterpart (the reference's pthread and MPI versions split the grid into
 * cubes inside one address space or exchange whole cube faces with MPI).
 *
 * With the AA pattern only the odd step reaches across a face, and a slot
 * of a column is read and written in the odd step by the same cell.  Slots
 * of column X with c_x = -1 are read and written by cell X + 1, those with
 * c_x = +1 by cell X - 1.  So, for a slab owning columns [lo, hi):
 *   after an even step (fill):  the ghost column lo-1 needs the c_x = -1
 *     slots of the left neighbour's column lo-1, and the ghost column hi
 *     the c_x = +1 slots of the right neighbour's column hi;
 *   after an odd step (flush):  what this slab's cells pushed into those
 *     ghost slots goes back to the neighbours' columns lo-1 and hi.
 * Only rows where both ends of the link lie in I cross: elsewhere the
 * bounce-back keeps a link inside its cell.  Each message is 5 slots x ny
 * x nz values.  The transport between slabs
 * (a copy on one GPU, NCCL send/recv, or host staging) belongs to the
 * caller: send_lo goes to the left neighbour's recv_hi, send_hi to the
 * right neighbour's recv_lo.
 */
#include <string.h>

#include "lbib_fluid_kernels.cuh"

using namespace lbib;

namespace {

/* The five directions with c_x = SIGN, in index order. */
template <int SIGN>
__device__ __forceinline__ int face_q(int j) {
  return SIGN > 0 ? (j == 0 ? 1 : j == 1 ? 7 : j == 2 ? 9 : j == 3 ? 15 : 17)
                  : (j == 0 ? 2 : j == 1 ? 8 : j == 2 ? 10 : j == 3 ? 16 : 18);
}

/* y or z offset of direction face_q(j). */
template <int SIGN>
__device__ __forceinline__ void face_cyz(int j, int& dy, int& dz) {
  const int q = face_q<SIGN>(j);
  dy = cy(q);
  dz = cz(q);
}

/* buf[j][z ny + y] <-> f[face_q(j)][(z ny + y) sx + col].  Unpacking writes
 * only the entries a step moves across the face: rows (y, z) of I whose
 * source row (y - c_y, z - c_z) is in I too.  For the other rows the
 * receiving slab's own cell has written the slot itself (a push whose
 * target is outside I goes to the cell's own opposite slot), and the
 * sender's ghost holds nothing. */
template <int SIGN, bool PACK>
__global__ void lbib_halo_copy(double* __restrict__ f, long Ns, int sx, int ny, int nz, int col,
                               double* __restrict__ buf) {
  const long P = (long)ny * nz;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const int y = (int)(i % ny), z = (int)(i / ny);
  const long idx = i * sx + col;
  const bool row_in = y >= 2 && y <= ny - 3 && z >= 2 && z <= nz - 3;
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    double* a = f + face_q<SIGN>(j) * Ns + idx;
    if (PACK) {
      buf[j * P + i] = *a;
    } else {
      int dy, dz;
      face_cyz<SIGN>(j, dy, dz);
      const int ys = y - dy, zs = z - dz;
      if (row_in && ys >= 2 && ys <= ny - 3 && zs >= 2 && zs <= nz - 3) *a = buf[j * P + i];
    }
  }
}

int halo_copy(lbib_device* d, int sign, bool pack, int x, double* buf) {
  const long P = (long)d->ny * d->nz;
  const int col = x - d->gx0;
  double* f = (double*)d->f;
  const unsigned nb = (unsigned)((P + 255) / 256);
  if (sign > 0) {
    if (pack) lbib_halo_copy<1, true><<<nb, 256, 0, d->stream>>>(f, d->Ns, d->sx, d->ny, d->nz, col, buf);
    else lbib_halo_copy<1, false><<<nb, 256, 0, d->stream>>>(f, d->Ns, d->sx, d->ny, d->nz, col, buf);
  } else {
    if (pack) lbib_halo_copy<-1, true><<<nb, 256, 0, d->stream>>>(f, d->Ns, d->sx, d->ny, d->nz, col, buf);
    else lbib_halo_copy<-1, false><<<nb, 256, 0, d->stream>>>(f, d->Ns, d->sx, d->ny, d->nz, col, buf);
  }
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

/* Buffers: halo + k * 5P, k = 0 send_lo, 1 send_hi, 2 recv_lo, 3 recv_hi. */
extern "C" int lbdev_slab_pack(lbib_device* d, int par) {
  if (!d->halo) return -4;
  const long P5 = 5L * d->ny * d->nz;
  const int lo = d->x_lo > 0, hi = d->x_hi < d->nx;
  if (par == 0) {        /* fill */
    if (lo && halo_copy(d, +1, true, d->x_lo, d->halo)) return -2;
    if (hi && halo_copy(d, -1, true, d->x_hi - 1, d->halo + P5)) return -2;
  } else {               /* flush */
    if (lo && halo_copy(d, -1, true, d->x_lo - 1, d->halo)) return -2;
    if (hi && halo_copy(d, +1, true, d->x_hi, d->halo + P5)) return -2;
  }
  return 0;
}

extern "C" int lbdev_slab_unpack(lbib_device* d, int par) {
  if (!d->halo) return -4;
  const long P5 = 5L * d->ny * d->nz;
  const int lo = d->x_lo > 0, hi = d->x_hi < d->nx;
  if (par == 0) {        /* fill */
    if (lo && halo_copy(d, -1, false, d->x_lo - 1, d->halo + 2 * P5)) return -2;
    if (hi && halo_copy(d, +1, false, d->x_hi, d->halo + 3 * P5)) return -2;
  } else {               /* flush */
    if (lo && halo_copy(d, +1, false, d->x_lo, d->halo + 2 * P5)) return -2;
    if (hi && halo_copy(d, -1, false, d->x_hi - 1, d->halo + 3 * P5)) return -2;
  }
  return 0;
}

/* This step's moment tiles (device) and their length in doubles, after the
 * tile-moment kernel; waits for the stream.  Also reads the error word:
 * returns its code (a stencil left the grid at step *failed_step). */
extern "C" int lbdev_slab_moments(lbib_device* d, double** U, long* n, int* failed_step) {
  int cnt = 0;
  if (cudaMemcpyAsync(&cnt, d->tile_count[d->cur], sizeof(int), cudaMemcpyDeviceToHost, d->stream) != cudaSuccess)
    return -2;
  if (cudaMemcpyAsync(d->h_err, d->err, sizeof(int) * 2, cudaMemcpyDeviceToHost, d->stream) != cudaSuccess) return -2;
  if (cudaStreamSynchronize(d->stream) != cudaSuccess) return -2;
  *U = d->Utile[d->cur];
  *n = (long)cnt * 256;
  if (failed_step) *failed_step = d->h_err[1];
  return d->h_err[0];
}

/* ---- direct exchange: the same columns, written into the neighbour's
 * storage (a peer device pointer, or an IPC mapping of another process's
 * buffer) by this slab's kernel -- no staging buffers and no collective.
 * The callers order the slabs' steps (a barrier after each of the two
 * exchanges); nothing here waits on another slab. */

namespace {

/* dst[face_q(j)][(z ny + y) dsx + dcol] = src[face_q(j)][(z ny + y) ssx + scol]
 * for the rows a step moves across the face (the unpack filter above). */
template <int SIGN>
__global__ void lbib_halo_push(const double* __restrict__ src, long sNs, int ssx, int scol, double* __restrict__ dst,
                               long dNs, int dsx, int dcol, int ny, int nz) {
  const long P = (long)ny * nz;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const int y = (int)(i % ny), z = (int)(i / ny);
  if (y < 2 || y > ny - 3 || z < 2 || z > nz - 3) return;
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    int dy, dz;
    face_cyz<SIGN>(j, dy, dz);
    const int ys = y - dy, zs = z - dz;
    if (ys >= 2 && ys <= ny - 3 && zs >= 2 && zs <= nz - 3) {
      const int q = face_q<SIGN>(j);
      dst[q * dNs + i * dsx + dcol] = src[q * sNs + i * ssx + scol];
    }
  }
}

int halo_push(lbib_device* d, int side, int sign, int x_src, int x_dst) {
  const long P = (long)d->ny * d->nz;
  const unsigned nb = (unsigned)((P + 255) / 256);
  const double* src = (const double*)d->f;
  const int scol = x_src - d->gx0, dcol = x_dst - d->peer_gx0[side];
  double* dst = d->peer_f[side];
  if (sign > 0)
    lbib_halo_push<1><<<nb, 256, 0, d->stream>>>(src, d->Ns, d->sx, scol, dst, d->peer_Ns[side], d->peer_sx[side],
                                                 dcol, d->ny, d->nz);
  else
    lbib_halo_push<-1><<<nb, 256, 0, d->stream>>>(src, d->Ns, d->sx, scol, dst, d->peer_Ns[side], d->peer_sx[side],
                                                  dcol, d->ny, d->nz);
  d->kernel_launches++;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

struct UTargets {
  double* U[8];
  int n;
};

/* lbib_tile_moments for this slab's tiles, each value written to every
 * slab's moment tiles (the same slot in all of them). */
template <int PAR>
__global__ void lbib_tile_moments_bcast(FluidParams p, const int* __restrict__ list, const int* __restrict__ count,
                                        const double* __restrict__ Ftile, UTargets u) {
  const int n = *count;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    double rho, ux, uy, uz;
    if (!tile_moment_values<double, PAR>(p, list[i], i, threadIdx.x, Ftile, rho, ux, uy, uz)) continue;
    for (int k = 0; k < u.n; ++k) {
      double* U = u.U[k] + (long)i * 256;
      U[threadIdx.x] = rho; U[64 + threadIdx.x] = ux; U[128 + threadIdx.x] = uy; U[192 + threadIdx.x] = uz;
    }
  }
}

}  // namespace

/* A fill (par 0) or flush (par 1) straight into the neighbours' columns:
 * the same columns and slots as lbdev_slab_pack + lbdev_slab_unpack. */
extern "C" int lbdev_slab_push(lbib_device* d, int par) {
  if (d->x_lo > 0 && !d->peer_f[0]) return -4;
  if (d->x_hi < d->nx && !d->peer_f[1]) return -4;
  const int lo = d->x_lo > 0, hi = d->x_hi < d->nx;
  if (par == 0) {        /* fill: this slab's face columns -> the neighbours' ghosts */
    if (lo && halo_push(d, 0, +1, d->x_lo, d->x_lo)) return -2;
    if (hi && halo_push(d, 1, -1, d->x_hi - 1, d->x_hi - 1)) return -2;
  } else {               /* flush: this slab's ghosts -> the neighbours' face columns */
    if (lo && halo_push(d, 0, -1, d->x_lo - 1, d->x_lo - 1)) return -2;
    if (hi && halo_push(d, 1, +1, d->x_hi, d->x_hi)) return -2;
  }
  return 0;
}

extern "C" int lbdev_slab_moments_bcast(lbib_device* d) {
  if (d->npeer_U < 1 || !d->S) return -4;
  FluidParams p = make_params_t<double>(d, 0);
  const int c = d->cur;
  UTargets u;
  u.n = d->npeer_U;
  for (int k = 0; k < u.n; ++k) u.U[k] = d->peer_U[c][k];
  const int blocks = 148 * 16;
  if (d->parity == 0)
    lbib_tile_moments_bcast<0><<<blocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], d->Ftile[c], u);
  else
    lbib_tile_moments_bcast<1><<<blocks, 64, 0, d->stream>>>(p, d->tile_list[c], d->tile_count[c], d->Ftile[c], u);
  d->kernel_launches++;
  d->have_moments = 1;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

/* ---- plumbing for the direct exchange ---------------------------------- */

extern "C" int lbdev_slab_connect(lbib_device* d, double* lo_f, long lo_Ns, int lo_sx, int lo_gx0, double* hi_f,
                                  long hi_Ns, int hi_sx, int hi_gx0, int n, double* const* U0, double* const* U1) {
  if (n < 1 || n > 8 || !U0 || !U1) return -1;
  if ((d->x_lo > 0) != (lo_f != NULL) || (d->x_hi < d->nx) != (hi_f != NULL)) return -1;
  d->peer_f[0] = lo_f; d->peer_Ns[0] = lo_Ns; d->peer_sx[0] = lo_sx; d->peer_gx0[0] = lo_gx0;
  d->peer_f[1] = hi_f; d->peer_Ns[1] = hi_Ns; d->peer_sx[1] = hi_sx; d->peer_gx0[1] = hi_gx0;
  for (int k = 0; k < n; ++k) {
    if (!U0[k] || !U1[k]) return -1;
    d->peer_U[0][k] = U0[k];
    d->peer_U[1][k] = U1[k];
  }
  d->npeer_U = n;
  return 0;
}

extern "C" int lbdev_peer_access(int device, int peer) {
  if (device == peer) return 0;
  int can = 0;
  if (cudaDeviceCanAccessPeer(&can, device, peer) != cudaSuccess || !can) return -1;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(device);
  cudaError_t e = cudaDeviceEnablePeerAccess(peer, 0);
  cudaSetDevice(cur);
  if (e == cudaErrorPeerAccessAlreadyEnabled) { cudaGetLastError(); return 0; }
  return e == cudaSuccess ? 0 : -2;
}

extern "C" int lbdev_ipc_handle(void* dev_ptr, void* handle) {
  cudaIpcMemHandle_t h;
  if (cudaIpcGetMemHandle(&h, dev_ptr) != cudaSuccess) return -2;
  memcpy(handle, &h, sizeof(h));
  return 0;
}

extern "C" int lbdev_ipc_open(const void* handle, void** dev_ptr) {
  cudaIpcMemHandle_t h;
  memcpy(&h, handle, sizeof(h));
  return cudaIpcOpenMemHandle(dev_ptr, h, cudaIpcMemLazyEnablePeerAccess) == cudaSuccess ? 0 : -2;
}

extern "C" int lbdev_ipc_close(void* dev_ptr) { return cudaIpcCloseMemHandle(dev_ptr) == cudaSuccess ? 0 : -2; }
