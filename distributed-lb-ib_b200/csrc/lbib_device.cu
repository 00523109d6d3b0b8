/*
 * GPU state of one LBM-IB problem and the order of a time step.
 *
 * A step (cube_pthread/lbm_ib.c:3124-3563, mpi/do_thread.c:50-386) is
 *   fiber forces -> spread (node prep, tile compaction, gather) -> fused
 *   fluid step -> moments on the touched tiles -> interpolate and move
 * all stream-ordered on one CUDA stream, with no host synchronisation.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lbib_internal.h"

extern "C" {
int lbdev_launch_fluid_step(lbib_device* d);
int lbdev_launch_tile_moments(lbib_device* d);
int lbdev_launch_field_moments(lbib_device* d, double* rho, double* ux, double* uy, double* uz);
int lbdev_launch_gather_df1(lbib_device* d, double* out);
int lbdev_launch_init(lbib_device* d, int what);
int lbdev_launch_sums(lbib_device* d, double* part, double* out);
int lbdev_lp_variants(int prec);
int lbdev_launch_fiber_forces(lbib_device* d, int k);
int lbdev_can_fuse_forces(const lbib_device* d);
int lbdev_launch_spread(lbib_device* d, int step);
int lbdev_launch_move(lbib_device* d);
int lbdev_launch_stencil_box(lbib_device* d);
int lbdev_launch_box_cells(lbib_device* d);
int lbdev_launch_scatter_force(lbib_device* d, double* fx, double* fy, double* fz);
}

#define CK(call)                                  \
  do {                                            \
    if ((call) != cudaSuccess) return -2;         \
  } while (0)

static void free_tiles(lbib_device* d) {
  for (int b = 0; b < 2; ++b) {
    cudaFree(d->tile_slot[b]); d->tile_slot[b] = NULL;
    cudaFree(d->tile_list[b]); d->tile_list[b] = NULL;
    cudaFree(d->tile_count[b]); d->tile_count[b] = NULL;
    cudaFree(d->Ftile[b]); d->Ftile[b] = NULL;
    cudaFree(d->Utile[b]); d->Utile[b] = NULL;
  }
  cudaFree(d->tile_cnt); d->tile_cnt = NULL;
  cudaFree(d->slot_off); d->slot_off = NULL;
  cudaFree(d->slot_len); d->slot_len = NULL;
  cudaFree(d->slot_cursor); d->slot_cursor = NULL;
  cudaFree(d->pair_node); d->pair_node = NULL;
  cudaFree(d->scan_tmp); d->scan_tmp = NULL;
  cudaFree(d->scan_state); d->scan_state = NULL;
}

static void free_sheets(lbib_device* d) {
  cudaFree(d->nodes); d->nodes = NULL;
  if (d->h_nodes) cudaFreeHost(d->h_nodes);
  d->h_nodes = NULL;
  cudaFree(d->W); d->W = NULL;
  cudaFree(d->st); d->st = NULL;
  cudaFree(d->chunk_box); d->chunk_box = NULL;
  free(d->sh); d->sh = NULL;
  d->nsheets = 0; d->S = 0; d->nchunks = 0;
}

/* Collision constants written exactly as the reference evaluates them
 * (lbm_ib.c:1722-1754): 1 - 1/tau, 1/tau, dt(1 - 1/(2 tau))/w, cs*cs, pow(cs, 4). */
static void derive_constants(lbib_device* d) {
  d->omtau = 1.0 - 1.0 / d->tau;
  d->invtau = 1.0 / d->tau;
  d->kw[0] = d->dt * (1.0 - 1.0 / (2.0 * d->tau)) / 3.0;
  d->kw[1] = d->dt * (1.0 - 1.0 / (2.0 * d->tau)) / 18.0;
  d->kw[2] = d->dt * (1.0 - 1.0 / (2.0 * d->tau)) / 36.0;
  d->cs2 = d->cs_l * d->cs_l;
  d->cs4 = pow(d->cs_l, 4);
  d->half_dt = 0.5 * d->dt;
  for (int k = 0; k < d->nsheets; ++k) {
    lbib_sheet_dev* s = &d->sh[k];
    /* compute_bendingforce / compute_stretchingforce, lbm_ib.c:994-996, 1164-1166, 1230 */
    s->bc = d->Kb_l / pow(s->ds2, 3);
    s->sc = d->Ks_l / (s->ds1 * s->ds1);
    s->sc2 = d->Ks_l / (s->ds2 * s->ds2);
  }
}

static void derive_boundaries(lbib_device* d) {
  /* copy_inout_to_df2 in the serial pthread run reaches z <= ncx*cs - 1 when
     num_cubes_x < num_cubes_z (lbm_ib.c:2800); otherwise z <= nz - 2. */
  d->zin_hi = d->nz - 2;
  if ((d->compat & 4) && d->ncx < d->ncz) d->zin_hi = d->ncx * d->cube_size - 1;
  /* the y walls skip z rows ncx*cs-2, ncx*cs-1 when num_cubes_x < num_cubes_z
     (lbm_ib.c:2378, 2414) */
  d->yskip_z0 = -1;
  if ((d->compat & 2) && d->ncx < d->ncz && !(d->compat & LBIB_OPT_PERIODIC_Z))
    d->yskip_z0 = d->ncx * d->cube_size - 2;
}

extern "C" int lbdev_bulk_rows(const lbib_device* d, int* nrows_y, int* nrows_z);

/* Bytes of one stored population value. */
extern "C" size_t lbdev_pop_bytes(int prec) {
  const int t = LBIB_PREC_TYPE(prec);
  return t == LBIB_PREC_F64 ? 8 : t == LBIB_PREC_F32 ? 4 : 2;
}

/* Shift of the low-precision forms: the rest weights w_q (rho_s = 1,
 * u_s = 0), or with LBIB_PREC_SHIFT_FLOW the equilibrium of the initial
 * state (rho_l, u_l, 0, 0), which the inflow keeps the bulk of the grid near. */
extern "C" void lbdev_shift(const lbib_device* d, float* sh, double* rhos, double* uxs) {
  if (LBIB_PREC_TYPE(d->prec) == LBIB_PREC_F64) {
    for (int q = 0; q < 19; ++q) sh[q] = 0.0f;
    *rhos = 0.0; *uxs = 0.0;
    return;
  }
  const int flow = (d->prec & LBIB_PREC_SHIFT_FLOW) != 0;
  const double rho = flow ? d->rho_l : 1.0, ux = flow ? d->u_l : 0.0;
  static const int cxq[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
  for (int q = 0; q < 19; ++q) {
    const double w = q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
    const double cu = cxq[q] * ux;
    sh[q] = (float)(w * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * ux * ux));
  }
  *rhos = rho;
  *uxs = ux;
}

/* Rows (y, z) of I that the generic fused kernel processes: all of them, or,
 * with the bulk kernels on, those they do not take (next to the walls, or
 * above zin_hi).  The bulk kernels need nx divisible by the cells they move
 * per aligned access. */
static int build_rows(lbib_device* d) {
  const char* env = getenv("LBIB_FLUID_BULK");
  int ry = 0, rz = 0;
  /* cells per aligned 8-byte word of the low-precision bulk kernel; the
     FP64 two-cell kernel wants even nx */
  const int v = LBIB_PREC_TYPE(d->prec) == LBIB_PREC_F64 ? 2 : (int)(8 / lbdev_pop_bytes(d->prec));
  d->use_bulk = !(env && env[0] == '0') && (d->nx % v == 0) && lbdev_bulk_rows(d, &ry, &rz);
  const int zb = 2 + rz;  /* last z row of the bulk kernels */
  long cap = (long)(d->ny - 4) * (d->nz - 4);
  int* h = (int*)malloc(sizeof(int) * 2 * cap);
  if (!h) return -5;
  int n = 0;
  for (int z = 2; z <= d->nz - 3; ++z)
    for (int y = 2; y <= d->ny - 3; ++y) {
      const int bulk = d->use_bulk && y >= 3 && y <= d->ny - 4 && z >= 3 && z <= zb;
      if (!bulk) { h[2 * n] = y; h[2 * n + 1] = z; ++n; }
    }
  cudaFree(d->rows);
  d->rows = NULL;
  d->nrows = n;
  int rc = 0;
  if (n > 0) {
    if (cudaMalloc(&d->rows, sizeof(int) * 2 * n) != cudaSuccess) rc = -5;
    else if (cudaMemcpy(d->rows, h, sizeof(int) * 2 * n, cudaMemcpyHostToDevice) != cudaSuccess) rc = -2;
  }
  free(h);
  return rc;
}

extern "C" int lbdev_set_physics(lbib_device* d, const lbdev_config* c) {
  d->tau = c->tau; d->u_l = c->u_l; d->rho_l = c->rho_l; d->Ks_l = c->Ks_l; d->Kb_l = c->Kb_l;
  d->g_l = c->g_l; d->cs_l = c->cs_l; d->dt = c->dt; d->compat = c->compat;
  derive_constants(d);
  derive_boundaries(d);
  return d->stream ? build_rows(d) : 0;
}

/* The columns [x_lo, x_hi) of the global grid this state holds (x_hi <= 0:
 * all of them).  A slab's bounds are multiples of 4, so every 4^3 tile lies
 * in one slab, and it is stored with two ghost columns on each side (even,
 * so the two-cell kernel's 16-byte accesses stay aligned). */
extern "C" int lbdev_set_columns(lbib_device* d, int x_lo, int x_hi) {
  if (x_hi <= 0) { x_lo = 0; x_hi = d->nx; }
  if (x_lo < 0 || x_hi > d->nx || x_hi - x_lo < 4 || x_lo % 4 || x_hi % 4) return -1;
  const int whole = x_lo == 0 && x_hi == d->nx;
  d->x_lo = x_lo; d->x_hi = x_hi;
  d->gx0 = whole ? 0 : x_lo - 2;
  d->sx = whole ? d->nx : x_hi - x_lo + 4;
  d->Ns = (long)d->sx * d->ny * d->nz;
  return 0;
}

extern "C" int lbdev_create(lbib_device** out, const lbdev_config* c) {
  *out = NULL;
  if (c->nx < 8 || c->ny < 8 || c->nz < 8 || c->cube_size < 4) return -1;
  if (c->nx % c->cube_size || c->ny % c->cube_size || c->nz % c->cube_size) return -1;
  lbib_device* d = (lbib_device*)calloc(1, sizeof(lbib_device));
  if (!d) return -5;
  d->nx = c->nx; d->ny = c->ny; d->nz = c->nz;
  d->prec = c->prec;
  d->N = (long)c->nx * c->ny * c->nz;
  /* slabs: FP64 only (the low-precision word kernel addresses whole rows) */
  if (lbdev_set_columns(d, c->x_lo, c->x_hi) ||
      ((d->x_lo > 0 || d->x_hi < d->nx) && LBIB_PREC_TYPE(c->prec) != LBIB_PREC_F64)) {
    free(d);
    return -1;
  }
  d->cube_size = c->cube_size;
  d->ncx = c->nx / c->cube_size; d->ncy = c->ny / c->cube_size; d->ncz = c->nz / c->cube_size;
  lbdev_set_physics(d, c);
  cudaGetDevice(&d->device);
  /* the state's stream gets the highest priority: in an overlapped step the
     spread's short kernels then take SMs ahead of the bulk fluid kernel,
     which runs on the low-priority side stream */
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  if (cudaStreamCreateWithPriority(&d->stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess) { free(d); return -2; }
  d->ntx = (d->nx + 3) / 4; d->nty = (d->ny + 3) / 4; d->ntz = (d->nz + 3) / 4;
  d->ntiles = (long)d->ntx * d->nty * d->ntz;
  int rc = 0;
  const size_t pop = lbdev_pop_bytes(d->prec), real = LBIB_PREC_TYPE(d->prec) == LBIB_PREC_F64 ? 8 : 4;
  if (cudaMalloc(&d->f, pop * 19 * d->Ns) != cudaSuccess) rc = -5;
  long P = (long)d->ny * d->nz;
  if (!rc && cudaMalloc(&d->inlet, real * 19 * P) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&d->outlet, real * 19 * P) != cudaSuccess) rc = -5;
  if (!rc && cudaMalloc(&d->err, sizeof(int) * 2) != cudaSuccess) rc = -5;
  if (!rc && cudaMallocHost(&d->h_err, sizeof(int) * 2) != cudaSuccess) rc = -5;
  if (!rc && cudaMemsetAsync(d->err, 0, sizeof(int) * 2, d->stream) != cudaSuccess) rc = -2;
  if (!rc && cudaMemsetAsync(d->f, 0, pop * 19 * d->Ns, d->stream) != cudaSuccess) rc = -2;
  if (!rc && (d->x_lo > 0 || d->x_hi < d->nx) &&
      cudaMalloc(&d->halo, sizeof(double) * 20 * P) != cudaSuccess) rc = -5;
  if (!rc) rc = build_rows(d);
  if (rc) { lbdev_free(d); return rc; }
  d->cur = 0;
  d->lp_variant = -1;
  const char* pf = getenv("LBIB_L2_PREFETCH");
  d->l2_pf = pf ? atoi(pf) : 0;
  d->fluid_stream = d->stream;
  /* box-mode steps for a whole grid: 1 in stream order (default), 2 with
     the fluid's bulk concurrent to the spread, 0 off (LBIB_OVERLAP) */
  const char* ov = getenv("LBIB_OVERLAP");
  d->overlap = (d->x_lo == 0 && d->x_hi == d->nx) ? (ov ? atoi(ov) : 1) : 0;
  if (d->overlap &&
      (cudaStreamCreateWithPriority(&d->side, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
       cudaEventCreateWithFlags(&d->ev_box, cudaEventDisableTiming) != cudaSuccess ||
       cudaEventCreateWithFlags(&d->ev_bulk, cudaEventDisableTiming) != cudaSuccess ||
       cudaMalloc(&d->box, sizeof(int) * 12) != cudaSuccess)) {
    lbdev_free(d);
    return -2;
  }
  *out = d;
  return 0;
}

extern "C" int lbdev_variants(const lbib_device* d) { return lbdev_lp_variants(d->prec); }

extern "C" int lbdev_set_variant(lbib_device* d, int v) {
  if (v < -1 || v >= lbdev_variants(d)) return -1;
  d->lp_variant = v;
  return 0;
}

extern "C" int lbdev_autotune(lbib_device* d, int steps, double* ms, int max_ms, int* best) {
  if (!d->have_df1 || !d->have_inout || !d->tile_slot[0]) return -4;
  if (d->steps != 0) return -4;
  if (steps < 2) steps = 2;
  steps += steps & 1;                      /* whole even/odd pairs */
  const int n = lbdev_variants(d);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int rc = 0, pick = 0;
  float best_ms = 0.0f;
  for (int v = 0; v < n && !rc; ++v) {
    d->lp_variant = v;
    for (int k = 0; k < 2 && !rc; ++k) rc = lbdev_launch_fluid_step(d);   /* warm-up */
    if (!rc && cudaEventRecord(e0, d->stream) != cudaSuccess) rc = -2;
    for (int k = 0; k < steps && !rc; ++k) rc = lbdev_launch_fluid_step(d);
    if (!rc && cudaEventRecord(e1, d->stream) != cudaSuccess) rc = -2;
    float t = 0.0f;
    if (!rc && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)) rc = -2;
    if (!rc) {
      if (ms && v < max_ms) ms[v] = t / steps;
      if (v == 0 || t < best_ms) { best_ms = t; pick = v; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  d->lp_variant = pick;
  if (best) *best = pick;
  /* the trials stepped the fluid; start again from the initial state */
  const int rc2 = lbdev_init_df1(d);
  return rc ? rc : rc2;
}

extern "C" void lbdev_free(lbib_device* d) {
  if (!d) return;
  if (d->stream) cudaStreamSynchronize(d->stream);
  free_tiles(d);
  free_sheets(d);
  cudaFree(d->f); cudaFree(d->inlet); cudaFree(d->outlet); cudaFree(d->err); cudaFree(d->rows);
  cudaFree(d->halo);
  cudaFree(d->scratch);
  for (int i = 0; i < d->nhost_reg; ++i) cudaHostUnregister(d->host_reg[i]);
  for (long i = 0; i < LBIB_PROF_EV * d->prof_cap; ++i) cudaEventDestroy(d->prof_ev[i]);
  free(d->prof_ev);
  free(d->prof_overlap);
  if (d->h_err) cudaFreeHost(d->h_err);
  if (d->side) cudaStreamDestroy(d->side);
  if (d->ev_box) cudaEventDestroy(d->ev_box);
  if (d->ev_bulk) cudaEventDestroy(d->ev_bulk);
  cudaFree(d->box);
  if (d->stream) cudaStreamDestroy(d->stream);
  free(d);
}

extern "C" int lbdev_set_sheets(lbib_device* d, int nsheets, const lbib_sheet_dev* sh, const double* nodes_host) {
  d->box_valid = 0;
  if (nsheets < 1) return -1;
  long S = 0;
  for (int k = 0; k < nsheets; ++k) {
    if (sh[k].rows < 4 || sh[k].cols < 4) return -1;
    S += (long)sh[k].rows * sh[k].cols;
  }
  CK(cudaStreamSynchronize(d->stream));
  if (S != d->S) {
    free_sheets(d);
    free_tiles(d);
    d->nchunks = (S + 31) / 32;
    CK(cudaMalloc(&d->nodes, sizeof(double) * 12 * S));
    CK(cudaMallocHost(&d->h_nodes, sizeof(double) * 12 * S));
    CK(cudaMalloc(&d->W, sizeof(double) * 12 * S));
    CK(cudaMalloc(&d->st, sizeof(int) * 3 * S));
    CK(cudaMalloc(&d->chunk_box, sizeof(int) * 6 * d->nchunks));
    /* every node touches at most 8 tiles, so 8 S slots can never overflow */
    d->cap = 8 * S < d->ntiles ? 8 * S : d->ntiles;
    for (int b = 0; b < 2; ++b) {
      CK(cudaMalloc(&d->tile_slot[b], sizeof(int) * d->ntiles));
      CK(cudaMalloc(&d->tile_list[b], sizeof(int) * d->cap));
      CK(cudaMalloc(&d->tile_count[b], sizeof(int)));
      CK(cudaMalloc(&d->Ftile[b], sizeof(double) * 192 * d->cap));
      CK(cudaMalloc(&d->Utile[b], sizeof(double) * 256 * d->cap));
      CK(cudaMemsetAsync(d->tile_slot[b], 0xff, sizeof(int) * d->ntiles, d->stream));
      CK(cudaMemsetAsync(d->tile_count[b], 0, sizeof(int), d->stream));
    }
    CK(cudaMalloc(&d->tile_cnt, sizeof(int) * d->ntiles));
    CK(cudaMemsetAsync(d->tile_cnt, 0, sizeof(int) * d->ntiles, d->stream));   /* the compaction keeps it at 0 */
    CK(cudaMalloc(&d->slot_off, sizeof(int) * d->cap));
    CK(cudaMalloc(&d->slot_len, sizeof(int) * d->cap));
    CK(cudaMalloc(&d->slot_cursor, sizeof(int) * d->cap));
    CK(cudaMalloc(&d->pair_node, sizeof(int2) * 8 * S));
    CK(cudaMalloc(&d->scan_tmp, sizeof(int) * 2 * ((d->ntiles + 1023) / 1024 + 1)));
    CK(cudaMalloc(&d->scan_state, sizeof(unsigned long long) * ((d->ntiles + 1023) / 1024 + 1)));
    CK(cudaMemsetAsync(d->scan_state, 0, sizeof(unsigned long long) * ((d->ntiles + 1023) / 1024 + 1), d->stream));
  }
  free(d->sh);
  d->sh = (lbib_sheet_dev*)malloc(sizeof(lbib_sheet_dev) * nsheets);
  memcpy(d->sh, sh, sizeof(lbib_sheet_dev) * nsheets);
  long off = 0;
  for (int k = 0; k < nsheets; ++k) {
    d->sh[k].offset = off;
    off += (long)sh[k].rows * sh[k].cols;
  }
  d->nsheets = nsheets;
  d->S = S;
  derive_constants(d);
  CK(cudaMemcpyAsync(d->nodes, nodes_host, sizeof(double) * 12 * S, cudaMemcpyHostToDevice, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  d->have_forces = 0;
  d->have_moments = 0;
  return 0;
}

extern "C" int lbdev_init_equilibrium(lbib_device* d) {
  d->have_eq = 1;
  return 0;
}

extern "C" int lbdev_init_df1(lbib_device* d) {
  d->box_valid = 0;
  if (lbdev_launch_init(d, 0)) return -2;
  d->parity = 0;
  d->steps = 0;
  d->have_df1 = 1;
  d->have_forces = 0;
  d->have_moments = 0;
  for (int b = 0; b < 2; ++b)
    if (d->tile_slot[b]) CK(cudaMemsetAsync(d->tile_slot[b], 0xff, sizeof(int) * d->ntiles, d->stream));
  return 0;
}

extern "C" int lbdev_init_inout(lbib_device* d) {
  if (lbdev_launch_init(d, 1)) return -2;
  d->have_inout = 1;
  return 0;
}

extern "C" int lbdev_stage(lbib_device* d, int which, int step_no) {
  if (!d->nodes || !d->have_df1 || !d->have_inout) return -4;
  d->box_valid = 0;   /* stage-by-stage calls may move the sheet */
  d->box_next = NULL;
  switch (which) {
    case 0:
      for (int k = 0; k < d->nsheets; ++k)
        if (lbdev_launch_fiber_forces(d, k)) return -2;
      return 0;
    case 1:
    case 2:
      return 0;  /* computed together with the bending force */
    case 3:
      d->cur ^= 1;
      d->have_forces = 1;
      d->have_moments = 0;
      return lbdev_launch_spread(d, step_no) ? -2 : 0;
    case 4:
      if (!d->have_forces) return -4;
      return lbdev_launch_fluid_step(d) ? -2 : 0;
    case 5:
    case 6:
      return 0;  /* streaming and bounce-back happen inside the fused step */
    case 7:
      d->have_moments = 1;
      return lbdev_launch_tile_moments(d) ? -2 : 0;
    case 8:
      if (!d->have_moments) return -4;
      return lbdev_launch_move(d) ? -2 : 0;
    case 9:
    case 10:
      return 0;  /* inlet/outlet copy and df2 -> df1 are part of the fused step */
    default:
      return -1;
  }
}

static int prof_grow(lbib_device* d) {
  long cap = d->prof_cap ? 2 * d->prof_cap : 256;
  cudaEvent_t* ev = (cudaEvent_t*)realloc(d->prof_ev, sizeof(cudaEvent_t) * LBIB_PROF_EV * cap);
  if (!ev) return -5;
  d->prof_ev = ev;
  char* mode = (char*)realloc(d->prof_overlap, cap);
  if (!mode) return -5;
  d->prof_overlap = mode;
  for (long i = LBIB_PROF_EV * d->prof_cap; i < LBIB_PROF_EV * cap; ++i) CK(cudaEventCreate(&d->prof_ev[i]));
  d->prof_cap = cap;
  return 0;
}

/* One full step in box mode (d->overlap, a whole grid): the box of this
 * step's stencils first; the fluid step's row and bulk kernels skip the
 * box's tiles and read no force -- they need nothing from this step's
 * forces and spread, and they lose the per-cell force-map lookups and the
 * forced collision from their code -- and the box's cells are stepped by
 * the generic rules after the spread; then the tile moments and the move.
 * Every cell is stepped once by the same per-cell arithmetic (the generic
 * rules give the two-cell kernel's bits), so the results do not change.
 * d->overlap == 2 runs the row and bulk kernels on the side stream,
 * concurrently with the forces and the spread; 1 keeps one stream (the
 * spread's kernels spread over every SM, and interleaving them with the
 * bandwidth-bound bulk kernel measured slower than running them in turn). */
static int step_overlapped(lbib_device* d, int step_no, cudaEvent_t* ev) {
  if (!d->nodes || !d->have_df1 || !d->have_inout) return -4;
  /* the box of this step's stencils: left by the previous step's move, or
     computed here (first step, positions set from the host, pinned rows --
     whose nodes the move does not visit) */
  const int pinned = (d->compat & LBIB_OPT_PIN_ROW0) != 0;
  if (!d->box_valid || pinned)
    if (lbdev_launch_stencil_box(d)) return -2;
  d->box_next = pinned ? NULL : d->box + 6 * (d->box_cur ^ 1);
  CK(cudaEventRecord(d->ev_box, d->stream));
  /* the step's buffers: the spread fills cur, the fluid reads cur ^ 1's moments */
  d->cur ^= 1;
  d->have_forces = 1;
  d->have_moments = 0;
  d->box_mode = 1;
  const int conc = d->overlap == 2;
  cudaStream_t fs = conc ? d->side : d->stream;
  int rc = 0;
  if (!conc) {
    /* the forces: in the node preparation's launch when the sheets allow */
    d->fuse_forces = lbdev_can_fuse_forces(d);
    for (int k = 0; k < d->nsheets && !rc && !d->fuse_forces; ++k) rc = lbdev_launch_fiber_forces(d, k);
    if (ev) CK(cudaEventRecord(ev[1], d->stream));
    if (!rc) rc = lbdev_launch_spread(d, step_no);
    d->fuse_forces = 0;
    if (ev) CK(cudaEventRecord(ev[2], d->stream));
    if (rc) { d->box_mode = 0; d->box_next = NULL; d->box_valid = 0; return -2; }
  }
  d->fluid_stream = fs;
  if (conc) CK(cudaStreamWaitEvent(d->side, d->ev_box, 0));
  if (ev) CK(cudaEventRecord(ev[6], fs));
  rc = lbdev_launch_fluid_step(d);
  if (ev) CK(cudaEventRecord(ev[7], fs));
  if (conc) CK(cudaEventRecord(d->ev_bulk, d->side));
  d->fluid_stream = d->stream;
  if (rc) { d->box_mode = 0; d->box_next = NULL; d->box_valid = 0; return -2; }
  if (conc) {
    for (int k = 0; k < d->nsheets && !rc; ++k) rc = lbdev_launch_fiber_forces(d, k);
    if (ev) CK(cudaEventRecord(ev[1], d->stream));
    if (!rc) rc = lbdev_launch_spread(d, step_no);
    if (ev) CK(cudaEventRecord(ev[2], d->stream));
    CK(cudaStreamWaitEvent(d->stream, d->ev_bulk, 0));
  }
  if (ev) CK(cudaEventRecord(ev[8], d->stream));
  if (!rc) rc = lbdev_launch_box_cells(d);
  d->box_mode = 0;
  if (rc) { d->box_next = NULL; d->box_valid = 0; return -2; }
  if (ev) CK(cudaEventRecord(ev[3], d->stream));
  d->have_moments = 1;
  rc = lbdev_launch_tile_moments(d) ? -2 : 0;
  if (ev) CK(cudaEventRecord(ev[4], d->stream));
  if (!rc) rc = lbdev_launch_move(d) ? -2 : 0;
  if (ev) CK(cudaEventRecord(ev[5], d->stream));
  /* the move reduced the next step's box into box_next */
  d->box_valid = !rc && d->box_next != NULL;
  if (d->box_valid) d->box_cur ^= 1;
  d->box_next = NULL;
  return rc;
}

extern "C" int lbdev_step(lbib_device* d, int step_no) {
  static const int order[] = {0, 3, 4, 7, 8};
  cudaEvent_t* ev = NULL;
  if (d->profiling) {
    if (d->prof_steps >= d->prof_cap && prof_grow(d)) return -5;
    ev = d->prof_ev + LBIB_PROF_EV * d->prof_steps;
    CK(cudaEventRecord(ev[0], d->stream));
  }
  if (d->overlap) {
    const int rc = step_overlapped(d, step_no, ev);
    if (rc) return rc;
    if (ev) d->prof_overlap[d->prof_steps++] = 1;
    return 0;
  }
  for (int i = 0; i < 5; ++i) {
    int rc = lbdev_stage(d, order[i], step_no);
    if (rc) return rc;
    if (ev) CK(cudaEventRecord(ev[i + 1], d->stream));
  }
  if (ev) d->prof_overlap[d->prof_steps++] = 0;
  return 0;
}

extern "C" int lbdev_profile_begin(lbib_device* d) {
  /* the first events are made here, not inside the profiled steps */
  if (!d->prof_cap && prof_grow(d)) return -5;
  d->profiling = 1;
  d->prof_steps = 0;
  return 0;
}

/* Sums, per stage, the event-timed milliseconds of the steps run since
 * lbdev_profile_begin, and stops profiling. */
extern "C" int lbdev_profile_end(lbib_device* d, double* stage_ms, long* steps) {
  CK(cudaStreamSynchronize(d->stream));
  for (int s = 0; s < LBIB_NSTAGE_TIMED; ++s) stage_ms[s] = 0.0;
  for (long t = 0; t < d->prof_steps; ++t) {
    cudaEvent_t* ev = d->prof_ev + LBIB_PROF_EV * t;
    for (int s = 0; s < LBIB_NSTAGE_TIMED; ++s) {
      float ms = 0.f;
      if (s == 2 && d->prof_overlap[t]) {
        /* overlapped: the bulk launches (side stream) plus the box's cells */
        float a = 0.f, b = 0.f;
        CK(cudaEventElapsedTime(&a, ev[6], ev[7]));
        CK(cudaEventElapsedTime(&b, ev[8], ev[3]));
        ms = a + b;
      } else {
        CK(cudaEventElapsedTime(&ms, ev[s], ev[s + 1]));
      }
      stage_ms[s] += ms;
    }
  }
  if (steps) *steps = d->prof_steps;
  d->profiling = 0;
  d->prof_steps = 0;
  return 0;
}

extern "C" int lbdev_check(lbib_device* d, int* failed_step) {
  CK(cudaMemcpyAsync(d->h_err, d->err, sizeof(int) * 2, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  if (failed_step) *failed_step = d->h_err[1];
  return d->h_err[0];
}

extern "C" int lbib_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

extern "C" int lbdev_sync(lbib_device* d) {
  CK(cudaStreamSynchronize(d->stream));
  return 0;
}

/* Dense scratch for the getters, allocated per call and freed after it. */
static int ensure_scratch(lbib_device* d, long doubles) {
  cudaFree(d->scratch);
  d->scratch = NULL;
  CK(cudaMalloc(&d->scratch, sizeof(double) * doubles));
  return 0;
}

/* The device address of a page-locked host array (cudaHostAlloc /
 * cudaHostRegister: mapped into the device's address space), or NULL for
 * pageable memory. */
static double* mapped_host(double* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return NULL;
  }
  return a.type == cudaMemoryTypeHost ? (double*)a.devicePointer : NULL;
}

extern "C" int lbdev_get_moments(lbib_device* d, double* rho, double* ux, double* uy, double* uz) {
  const long N = d->N;
  /* page-locked outputs: the moments kernel writes them over the link
     itself, so nothing is staged in device memory and the copy overlaps
     the computation */
  double* m[4] = {mapped_host(rho), mapped_host(ux), mapped_host(uy), mapped_host(uz)};
  if (m[0] && m[1] && m[2] && m[3]) {
    if (lbdev_launch_field_moments(d, m[0], m[1], m[2], m[3])) return -2;
    CK(cudaStreamSynchronize(d->stream));
    return 0;
  }
  if (ensure_scratch(d, 4 * N)) return -5;
  double* s = d->scratch;
  if (lbdev_launch_field_moments(d, s, s + N, s + 2 * N, s + 3 * N)) return -2;
  CK(cudaMemcpyAsync(rho, s, sizeof(double) * N, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaMemcpyAsync(ux, s + N, sizeof(double) * N, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaMemcpyAsync(uy, s + 2 * N, sizeof(double) * N, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaMemcpyAsync(uz, s + 3 * N, sizeof(double) * N, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  cudaFree(d->scratch);
  d->scratch = NULL;
  return 0;
}

extern "C" int lbdev_get_force(lbib_device* d, double* fx, double* fy, double* fz) {
  const long N = d->N;
  if (ensure_scratch(d, 3 * N)) return -5;
  double* s = d->scratch;
  CK(cudaMemsetAsync(s, 0, sizeof(double) * 3 * N, d->stream));
  if (d->have_forces && lbdev_launch_scatter_force(d, s, s + N, s + 2 * N)) return -2;
  CK(cudaMemcpyAsync(fx, s, sizeof(double) * N, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaMemcpyAsync(fy, s + N, sizeof(double) * N, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaMemcpyAsync(fz, s + 2 * N, sizeof(double) * N, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  cudaFree(d->scratch);
  d->scratch = NULL;
  return 0;
}

extern "C" int lbdev_get_df1(lbib_device* d, double* out) {
  const long N = d->N;
  if (ensure_scratch(d, 19 * N)) return -5;
  double* s = d->scratch;
  CK(cudaMemsetAsync(s, 0, sizeof(double) * 19 * N, d->stream));
  if (lbdev_launch_gather_df1(d, s)) return -2;
  CK(cudaMemcpyAsync(out, s, sizeof(double) * 19 * N, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  cudaFree(d->scratch);
  d->scratch = NULL;
  return 0;
}

/* out[4] = FP64 mass and x, y, z momentum of the populations of I. */
extern "C" int lbdev_conservation(lbib_device* d, double* out) {
  if (!d->have_df1) return -4;
  const long rows = (long)(d->ny - 4) * (d->nz - 4);
  if (ensure_scratch(d, 4 * rows + 4)) return -5;
  double* s = d->scratch;
  if (lbdev_launch_sums(d, s + 4, s)) return -2;
  CK(cudaMemcpyAsync(out, s, sizeof(double) * 4, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  cudaFree(d->scratch);
  d->scratch = NULL;
  return 0;
}

/* Sheet records to host memory; out == NULL leaves them in the pinned
 * staging buffer d->h_nodes. */
extern "C" int lbdev_get_nodes(lbib_device* d, double* out) {
  CK(cudaMemcpyAsync(d->h_nodes, d->nodes, sizeof(double) * 12 * d->S, cudaMemcpyDeviceToHost, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  if (out) memcpy(out, d->h_nodes, sizeof(double) * 12 * d->S);
  return 0;
}

extern "C" int lbdev_register_host(lbib_device* d, void* p, size_t bytes) {
  if (d->nhost_reg >= 8 || lbdev_is_registered(d, p, bytes)) return 0;
  if (cudaHostRegister(p, bytes, cudaHostRegisterDefault) != cudaSuccess) {
    cudaGetLastError();                /* not fatal: copies go through staging */
    return -2;
  }
  d->host_reg[d->nhost_reg] = p;
  d->host_reg_bytes[d->nhost_reg] = bytes;
  d->nhost_reg++;
  return 0;
}

extern "C" int lbdev_is_registered(const lbib_device* d, const void* p, size_t bytes) {
  for (int i = 0; i < d->nhost_reg; ++i)
    if (d->host_reg[i] == p && d->host_reg_bytes[i] == bytes) return 1;
  return 0;
}

extern "C" int lbdev_copy_nodes_out(lbib_device* d, long first, long n, double* host) {
  if (first < 0 || n < 0 || first + n > d->S) return -1;
  CK(cudaMemcpyAsync(host, d->nodes + 12 * first, sizeof(double) * 12 * n, cudaMemcpyDeviceToHost, d->stream));
  return 0;
}

extern "C" int lbdev_copy_nodes_in(lbib_device* d, long first, long n, const double* host) {
  d->box_valid = 0;
  if (first < 0 || n < 0 || first + n > d->S) return -1;
  CK(cudaMemcpyAsync(d->nodes + 12 * first, host, sizeof(double) * 12 * n, cudaMemcpyHostToDevice, d->stream));
  return 0;
}

extern "C" int lbdev_set_nodes(lbib_device* d, const double* in) {
  d->box_valid = 0;
  CK(cudaMemcpyAsync(d->nodes, in, sizeof(double) * 12 * d->S, cudaMemcpyHostToDevice, d->stream));
  CK(cudaStreamSynchronize(d->stream));
  return 0;
}

/* ---- restart state: everything the next step reads ------------------------
 * Written and read in this order, raw device bytes:
 *   ints   parity, cur, have_forces, have_moments, lp_variant; long steps
 *   f      [19][N] populations in the storage type
 *   inlet, outlet tables
 *   tile_count[cur], tile_slot[cur] [ntiles], tile_list[cur] [count],
 *   Ftile[cur], Utile[cur] [count] slots
 *   nodes  [S][12]
 * The caller checks that the state it loads into has the same grid,
 * precision and sheets. */
static int put(FILE* fp, const void* p, size_t n) { return fwrite(p, 1, n, fp) == n ? 0 : -7; }
static int get(FILE* fp, void* p, size_t n) { return fread(p, 1, n, fp) == n ? 0 : -7; }

static int dev_out(lbib_device* d, FILE* fp, const void* dp, size_t n, void* buf, size_t cap) {
  for (size_t o = 0; o < n; o += cap) {
    const size_t k = n - o < cap ? n - o : cap;
    CK(cudaMemcpy(buf, (const char*)dp + o, k, cudaMemcpyDeviceToHost));
    if (put(fp, buf, k)) return -7;
  }
  (void)d;
  return 0;
}

static int dev_in(lbib_device* d, FILE* fp, void* dp, size_t n, void* buf, size_t cap) {
  for (size_t o = 0; o < n; o += cap) {
    const size_t k = n - o < cap ? n - o : cap;
    if (get(fp, buf, k)) return -7;
    CK(cudaMemcpy((char*)dp + o, buf, k, cudaMemcpyHostToDevice));
  }
  (void)d;
  return 0;
}

extern "C" int lbdev_save_state(lbib_device* d, FILE* fp) {
  if (!d->nodes || !d->tile_slot[0]) return -4;
  CK(cudaStreamSynchronize(d->stream));
  const int c = d->cur;
  int count = 0;
  CK(cudaMemcpy(&count, d->tile_count[c], sizeof(int), cudaMemcpyDeviceToHost));
  const int hdr[6] = {d->parity, c, d->have_forces, d->have_moments, d->lp_variant, count};
  int rc = put(fp, hdr, sizeof(hdr));
  if (!rc) rc = put(fp, &d->steps, sizeof(d->steps));
  const size_t cap = 64u << 20;
  void* buf = malloc(cap);
  if (!buf) return -5;
  const size_t real = LBIB_PREC_TYPE(d->prec) == LBIB_PREC_F64 ? 8 : 4;
  const long P = (long)d->ny * d->nz;
  if (!rc) rc = dev_out(d, fp, d->f, lbdev_pop_bytes(d->prec) * 19 * d->Ns, buf, cap);
  if (!rc) rc = dev_out(d, fp, d->inlet, real * 19 * P, buf, cap);
  if (!rc) rc = dev_out(d, fp, d->outlet, real * 19 * P, buf, cap);
  if (!rc) rc = dev_out(d, fp, d->tile_slot[c], sizeof(int) * d->ntiles, buf, cap);
  if (!rc) rc = dev_out(d, fp, d->tile_list[c], sizeof(int) * count, buf, cap);
  if (!rc) rc = dev_out(d, fp, d->Ftile[c], sizeof(double) * 192 * count, buf, cap);
  if (!rc) rc = dev_out(d, fp, d->Utile[c], sizeof(double) * 256 * count, buf, cap);
  if (!rc) rc = dev_out(d, fp, d->nodes, sizeof(double) * 12 * d->S, buf, cap);
  free(buf);
  return rc;
}

extern "C" int lbdev_load_state(lbib_device* d, FILE* fp) {
  d->box_valid = 0;
  if (!d->nodes || !d->tile_slot[0]) return -4;
  CK(cudaStreamSynchronize(d->stream));
  int hdr[6];
  long steps = 0;
  if (get(fp, hdr, sizeof(hdr)) || get(fp, &steps, sizeof(steps))) return -7;
  const int c = hdr[1], count = hdr[5];
  if ((c & ~1) || count < 0 || count > d->cap || hdr[0] < 0 || hdr[0] > 1) return -1;
  const size_t cap = 64u << 20;
  void* buf = malloc(cap);
  if (!buf) return -5;
  const size_t real = LBIB_PREC_TYPE(d->prec) == LBIB_PREC_F64 ? 8 : 4;
  const long P = (long)d->ny * d->nz;
  int rc = dev_in(d, fp, d->f, lbdev_pop_bytes(d->prec) * 19 * d->Ns, buf, cap);
  if (!rc) rc = dev_in(d, fp, d->inlet, real * 19 * P, buf, cap);
  if (!rc) rc = dev_in(d, fp, d->outlet, real * 19 * P, buf, cap);
  if (!rc) rc = dev_in(d, fp, d->tile_slot[c], sizeof(int) * d->ntiles, buf, cap);
  if (!rc) rc = dev_in(d, fp, d->tile_list[c], sizeof(int) * count, buf, cap);
  if (!rc) rc = dev_in(d, fp, d->Ftile[c], sizeof(double) * 192 * count, buf, cap);
  if (!rc) rc = dev_in(d, fp, d->Utile[c], sizeof(double) * 256 * count, buf, cap);
  if (!rc) rc = dev_in(d, fp, d->nodes, sizeof(double) * 12 * d->S, buf, cap);
  free(buf);
  if (rc) return rc;
  CK(cudaMemcpy(d->tile_count[c], &count, sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemset(d->tile_slot[c ^ 1], 0xff, sizeof(int) * d->ntiles));
  d->parity = hdr[0];
  d->cur = c;
  d->have_forces = hdr[2];
  d->have_moments = hdr[3];
  if (hdr[4] >= -1 && hdr[4] < lbdev_variants(d)) d->lp_variant = hdr[4];
  d->steps = steps;
  d->have_df1 = d->have_inout = 1;
  return 0;
}
