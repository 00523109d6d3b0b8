/*
 * Host side of the drop-in: the reference's set-up API, step driver, stage
 * functions and dump writers (see include/lbib.h), on top of the GPU state in
 * lbib_device.cu.  Compiled as C with -ffp-contract=off so that the host-side
 * arithmetic (sheet generation, constants) rounds as the reference does.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/lbib.h"
#include "lbib_internal.h"

static __thread int g_last_error = LBIB_OK;
static int g_sticky_error = LBIB_OK;

static int set_error(int code) {
  if (code != LBIB_OK) {
    g_last_error = code;
    if (g_sticky_error == LBIB_OK) g_sticky_error = code;
  }
  return code;
}

int lbib_last_error(void) { return g_sticky_error != LBIB_OK ? g_sticky_error : g_last_error; }
void lbib_clear_error(void) { g_last_error = LBIB_OK; g_sticky_error = LBIB_OK; }

const char* lbib_error_string(int code) {
  switch (code) {
    case LBIB_OK: return "ok";
    case LBIB_E_ARG: return "invalid argument (size, NULL pointer or indivisible grid)";
    case LBIB_E_CUDA: return "a CUDA call failed";
    case LBIB_E_STENCIL: return "a fiber node's 4x4x4 stencil left the fluid grid";
    case LBIB_E_STATE: return "call out of order (no grid, sheet or initial state yet), or not for this grid (a slab / the whole grid)";
    case LBIB_E_NOMEM: return "allocation failed";
    case LBIB_E_CAPACITY: return "touched-tile capacity exceeded";
    case LBIB_E_IO: return "a dump file could not be written";
    case LBIB_E_LIMIT: return "size above the fixed maximum of the no-allocation entry point";
    default: return "unknown error";
  }
}

/* ---- set-up --------------------------------------------------------- */

/* mpi/init_gv.c:25-35 lattice velocities (also cube_pthread/lbm_ib.c:777-833) */
static const double LBIB_C[19][3] = {
    {0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 0, 1}, {0, 0, -1}, {0, -1, 0}, {0, 1, 0},
    {1, 0, 1}, {-1, 0, -1}, {1, 0, -1}, {-1, 0, 1}, {0, -1, 1}, {0, 1, -1},
    {0, 1, 1}, {0, -1, -1}, {1, -1, 0}, {-1, 1, 0}, {1, 1, 0}, {-1, -1, 0}};

void init_gv_constant(GV gv) {
  if (!gv || !gv->fluid_grid || gv->cube_size <= 0) { set_error(LBIB_E_ARG); return; }
  gv->dt = 1;
  gv->time = gv->dt;
  int dim_x = gv->fluid_grid->x_dim, dim_y = gv->fluid_grid->y_dim, dim_z = gv->fluid_grid->z_dim;
  int cs = gv->cube_size;
  gv->num_cubes_x = gv->fluid_grid->num_cubes_x = dim_x / cs;
  gv->num_cubes_y = gv->fluid_grid->num_cubes_y = dim_y / cs;
  gv->num_cubes_z = gv->fluid_grid->num_cubes_z = dim_z / cs;
  gv->ib = 2;
  gv->ie = dim_x - 3;
  gv->jb = 2;
  gv->je = dim_y - 3;
  gv->kb = 2;
  gv->ke = dim_z - 3;
  /* hard-coded physics, mpi/init_gv.c:74-97 */
  gv->Re = 1.5e2;
  gv->rho_l = 1.0e0;
  gv->u_l = 0.001;
  gv->L_l = 2.0e1;
  gv->nu_l = gv->u_l * gv->L_l / gv->Re;
  gv->tau = 0.5 * (6.0 * gv->nu_l + 1.0);
  gv->Fr = 1.0e10;
  gv->Kbhat = 0.005;
  gv->Kshat = 2.0e1;
  gv->Ksthat = 0.0e0;
  gv->cs_l = 1.0 / (sqrt(3));
  gv->g_l = gv->u_l * gv->u_l / (gv->Fr * gv->L_l);
  gv->g_l = 0.0;
  gv->Kb_l = gv->Kbhat * gv->rho_l * gv->u_l * gv->u_l * pow(gv->L_l, 4);
  gv->Ks_l = gv->Kshat * gv->rho_l * gv->u_l * gv->u_l * gv->L_l;
  memcpy(gv->c, LBIB_C, sizeof(LBIB_C));
  gv->lbib_compat = LBIB_COMPAT_ALL;
  gv->lbib_precision = LBIB_PREC_F64;
  gv->lbib_slab_lo = gv->lbib_slab_hi = 0;
}

static void fill_config(GV gv, lbdev_config* c) {
  c->nx = gv->fluid_grid->x_dim;
  c->ny = gv->fluid_grid->y_dim;
  c->nz = gv->fluid_grid->z_dim;
  c->cube_size = gv->cube_size;
  c->compat = gv->lbib_compat;
  c->prec = gv->lbib_precision;
  c->tau = gv->tau; c->u_l = gv->u_l; c->rho_l = gv->rho_l;
  c->Ks_l = gv->Ks_l; c->Kb_l = gv->Kb_l; c->g_l = gv->g_l; c->cs_l = gv->cs_l;
  c->dt = gv->dt;
  c->x_lo = gv->lbib_slab_lo; c->x_hi = gv->lbib_slab_hi;
}

void gen_fluid_grid(Fluidgrid* fluid_grid, int cube_size, int taskid, GV gv) {
  (void)taskid;
  if (!gv || !fluid_grid || cube_size <= 0) { set_error(LBIB_E_ARG); return; }
  int nx = fluid_grid->x_dim, ny = fluid_grid->y_dim, nz = fluid_grid->z_dim;
  if (nx % cube_size || ny % cube_size || nz % cube_size) { set_error(LBIB_E_ARG); return; }
  fluid_grid->num_cubes_x = nx / cube_size;
  fluid_grid->num_cubes_y = ny / cube_size;
  fluid_grid->num_cubes_z = nz / cube_size;
  gv->fluid_grid = fluid_grid;
  gv->cube_size = cube_size;
  if (gv->dev) { lbdev_free(gv->dev); gv->dev = NULL; }
  lbdev_config c;
  fill_config(gv, &c);
  int rc = lbdev_create(&gv->dev, &c);
  if (rc) set_error(rc);
}

void gen_fiber_sheet(Fibersheet* sheet) {
  if (!sheet || sheet->num_rows < 2 || sheet->num_cols < 2) { set_error(LBIB_E_ARG); return; }
  double width = sheet->width;
  double height = sheet->height;
  int num_cols = sheet->num_cols;
  int num_rows = sheet->num_rows;
  double zdist = width / (num_cols - 1);
  double ydist = height / (num_rows - 1);
  /* The rows' node arrays are consecutive pieces of one page-aligned block
     (the reference callocs each row): the block is the [rows*cols] record
     layout of the GPU copy, so that, once page-locked at upload, the sheet
     comes back from the GPU in one copy with no host-side repacking. */
  const size_t page = 4096;
  const size_t bytes = (size_t)num_rows * num_cols * sizeof(Fibernode);
  Fibernode* block = NULL;
  if (posix_memalign((void**)&block, page, (bytes + page - 1) / page * page) != 0) {
    set_error(LBIB_E_NOMEM);
    return;
  }
  memset(block, 0, (bytes + page - 1) / page * page);
  sheet->fibers = (Fiber*)calloc(num_rows, sizeof(Fiber));
  for (int row = 0; row < num_rows; ++row) {
    Fiber* fiber = sheet->fibers + row;
    fiber->nodes = block + (size_t)row * num_cols;
    fiber->num_nodes = num_cols;
    for (int col = 0; col < num_cols; ++col) {
      fiber->nodes[col].x = sheet->x_orig;
      fiber->nodes[col].y = ydist * row + sheet->y_orig;
      fiber->nodes[col].z = zdist * col + sheet->z_orig;
    }
  }
}

/* The sheet's rows lie back to back in one block (as gen_fiber_sheet makes
 * them): its first node, else NULL. */
static Fibernode* sheet_block(const Fibersheet* sh) {
  if (!sh->fibers) return NULL;
  for (int r = 1; r < sh->num_rows; ++r)
    if (sh->fibers[r].nodes != sh->fibers[0].nodes + (size_t)r * sh->num_cols) return NULL;
  return sh->fibers[0].nodes;
}

static long total_nodes(GV gv) {
  long S = 0;
  for (int k = 0; k < gv->fiber_shape->num_sheets; ++k)
    S += (long)gv->fiber_shape->sheets[k].num_rows * gv->fiber_shape->sheets[k].num_cols;
  return S;
}

/* Pack the host sheets as [S][12] Fibernode records. */
static double* pack_nodes(GV gv) {
  long S = total_nodes(gv), o = 0;
  double* buf = (double*)malloc(sizeof(double) * 12 * S);
  if (!buf) return NULL;
  for (int k = 0; k < gv->fiber_shape->num_sheets; ++k) {
    Fibersheet* sh = &gv->fiber_shape->sheets[k];
    for (int r = 0; r < sh->num_rows; ++r) {
      memcpy(buf + o * 12, sh->fibers[r].nodes, sizeof(Fibernode) * sh->num_cols);
      o += sh->num_cols;
    }
  }
  return buf;
}

static void unpack_nodes(GV gv, const double* buf) {
  long o = 0;
  for (int k = 0; k < gv->fiber_shape->num_sheets; ++k) {
    Fibersheet* sh = &gv->fiber_shape->sheets[k];
    for (int r = 0; r < sh->num_rows; ++r) {
      memcpy(sh->fibers[r].nodes, buf + o * 12, sizeof(Fibernode) * sh->num_cols);
      o += sh->num_cols;
    }
  }
}

static int upload_sheets(GV gv) {
  Fibershape* shape = gv->fiber_shape;
  if (!shape || shape->num_sheets < 1 || !gv->dev) return set_error(LBIB_E_STATE);
  lbib_sheet_dev* sh = (lbib_sheet_dev*)calloc(shape->num_sheets, sizeof(lbib_sheet_dev));
  for (int k = 0; k < shape->num_sheets; ++k) {
    Fibersheet* s = &shape->sheets[k];
    if (!s->fibers) { free(sh); return set_error(LBIB_E_STATE); }
    sh[k].rows = s->num_rows;
    sh[k].cols = s->num_cols;
    sh[k].ds1 = s->width / (s->num_cols - 1);
    sh[k].ds2 = s->height / (s->num_rows - 1);
  }
  double* buf = pack_nodes(gv);
  int rc = buf ? lbdev_set_sheets(gv->dev, shape->num_sheets, sh, buf) : LBIB_E_NOMEM;
  free(buf);
  free(sh);
  /* page-lock the sheets' blocks for direct copies (best effort) */
  for (int k = 0; !rc && k < shape->num_sheets; ++k) {
    Fibersheet* s = &shape->sheets[k];
    Fibernode* b = sheet_block(s);
    if (b) lbdev_register_host(gv->dev, b, sizeof(Fibernode) * (size_t)s->num_rows * s->num_cols);
  }
  return rc ? set_error(rc) : LBIB_OK;
}

void init_gv(GV gv) {
  if (!gv || !gv->fiber_shape || !gv->dev) { set_error(LBIB_E_STATE); return; }
  /* shift every sheet by u_l*dt, mpi/init_gv.c:239-245 */
  for (int k = 0; k < gv->fiber_shape->num_sheets; ++k) {
    Fibersheet* sh = &gv->fiber_shape->sheets[k];
    if (!sh->fibers) { set_error(LBIB_E_STATE); return; }
    for (int i = 0; i < sh->num_rows; i++)
      for (int j = 0; j < sh->num_cols; j++) sh->fibers[i].nodes[j].x += gv->u_l * gv->dt;
  }
  upload_sheets(gv);
}

void init_eqlbrmdistrfuncDF0(GV gv) {
  if (!gv || !gv->dev) { set_error(LBIB_E_STATE); return; }
  lbdev_config c;
  fill_config(gv, &c);
  lbdev_set_physics(gv->dev, &c);
  int rc = lbdev_init_equilibrium(gv->dev);
  if (rc) set_error(rc);
}

void init_df1(GV gv) {
  if (!gv || !gv->dev) { set_error(LBIB_E_STATE); return; }
  int rc = lbdev_init_df1(gv->dev);
  if (rc) set_error(rc);
}

void init_df_inout(GV gv) {
  if (!gv || !gv->dev) { set_error(LBIB_E_STATE); return; }
  int rc = lbdev_init_inout(gv->dev);
  if (rc) set_error(rc);
}

int lbib_set_params(GV gv, double tau, double u_l, double Ks_l, double Kb_l) {
  if (!gv || !(tau > 0.5) || !(Ks_l >= 0) || !(Kb_l >= 0)) return set_error(LBIB_E_ARG);
  gv->tau = tau;
  gv->u_l = u_l;
  gv->Ks_l = Ks_l;
  gv->Kb_l = Kb_l;
  if (gv->dev) {
    lbdev_config c;
    fill_config(gv, &c);
    lbdev_set_physics(gv->dev, &c);
  }
  return LBIB_OK;
}

int lbib_set_compat(GV gv, int flags) {
  if (!gv || (flags & ~LBIB_COMPAT_ALL)) return set_error(LBIB_E_ARG);
  gv->lbib_compat = flags;
  if (gv->dev) {
    lbdev_config c;
    fill_config(gv, &c);
    lbdev_set_physics(gv->dev, &c);
  }
  return LBIB_OK;
}

static int precision_ok(int p) {
  const int t = p & ~LBIB_PREC_SHIFT_FLOW;
  return t >= LBIB_PREC_F32 && t <= LBIB_PREC_BF16 ? 1 : p == LBIB_PREC_F64;
}

int lbib_set_precision(GV gv, int precision) {
  if (!gv || !precision_ok(precision)) return set_error(LBIB_E_ARG);
  if (gv->dev && gv->dev->S > 0) return set_error(LBIB_E_STATE);
  gv->lbib_precision = precision;
  if (gv->dev && gv->dev->prec != precision) {
    lbdev_free(gv->dev);
    gv->dev = NULL;
    lbdev_config c;
    fill_config(gv, &c);
    int rc = lbdev_create(&gv->dev, &c);
    if (rc) return set_error(rc);
  }
  return LBIB_OK;
}

int lbib_set_slab(GV gv, int x_lo, int x_hi) {
  if (!gv) return set_error(LBIB_E_ARG);
  if (gv->dev && gv->dev->S > 0) return set_error(LBIB_E_STATE);
  const int keep_lo = gv->lbib_slab_lo, keep_hi = gv->lbib_slab_hi;
  gv->lbib_slab_lo = x_lo;
  gv->lbib_slab_hi = x_hi;
  if (gv->dev) {
    lbdev_free(gv->dev);
    gv->dev = NULL;
    lbdev_config c;
    fill_config(gv, &c);
    int rc = lbdev_create(&gv->dev, &c);
    if (rc) {
      gv->lbib_slab_lo = keep_lo;
      gv->lbib_slab_hi = keep_hi;
      fill_config(gv, &c);
      lbdev_create(&gv->dev, &c);
      return set_error(rc);
    }
  }
  return LBIB_OK;
}

static int is_slab(GV gv) { return gv->dev && (gv->dev->x_lo > 0 || gv->dev->x_hi < gv->dev->nx); }

int lbib_slab_buffers(GV gv, double** bufs, long* len) {
  if (!gv || !bufs || !len) return set_error(LBIB_E_ARG);
  if (!is_slab(gv)) return set_error(LBIB_E_STATE);
  const long P5 = 5L * gv->dev->ny * gv->dev->nz;
  for (int k = 0; k < 4; ++k) bufs[k] = gv->dev->halo + k * P5;
  *len = P5;
  return LBIB_OK;
}

int lbib_slab_step_fluid(GV gv) {
  if (!gv) return set_error(LBIB_E_ARG);
  if (!is_slab(gv)) return set_error(LBIB_E_STATE);
  lbib_device* d = gv->dev;
  static const int order[] = {0, 3, 4};
  for (int i = 0; i < 3; ++i) {
    int rc = lbdev_stage(d, order[i], gv->time);
    if (rc) return set_error(rc);
  }
  const int par = d->parity ^ 1;      /* the step just launched */
  if (lbdev_slab_pack(d, par)) return set_error(LBIB_E_CUDA);
  return par;
}

int lbib_slab_step_moments(GV gv) {
  if (!gv) return set_error(LBIB_E_ARG);
  if (!is_slab(gv) || gv->dev->steps == 0) return set_error(LBIB_E_STATE);
  if (lbdev_slab_unpack(gv->dev, gv->dev->parity ^ 1)) return set_error(LBIB_E_CUDA);
  int rc = lbdev_stage(gv->dev, 7, gv->time);
  return rc ? set_error(rc) : LBIB_OK;
}

int lbib_slab_moments(GV gv, double** U, long* n) {
  if (!gv || !U || !n) return set_error(LBIB_E_ARG);
  if (!is_slab(gv) || !gv->dev->have_moments) return set_error(LBIB_E_STATE);
  int failed = 0;
  int e = lbdev_slab_moments(gv->dev, U, n, &failed);
  if (e) {
    if (e != LBIB_E_CUDA) gv->time = failed;
    return set_error(e);
  }
  return LBIB_OK;
}

int lbib_slab_step_move(GV gv) {
  if (!gv) return set_error(LBIB_E_ARG);
  if (!is_slab(gv)) return set_error(LBIB_E_STATE);
  int rc = lbdev_stage(gv->dev, 8, gv->time);
  if (rc) return set_error(rc);
  gv->time += gv->dt;
  return LBIB_OK;
}

int lbib_slab_storage(GV gv, double** f, long* Ns, int* sx, int* gx0, double** U0, double** U1) {
  if (!gv || !f || !Ns || !sx || !gx0 || !U0 || !U1) return set_error(LBIB_E_ARG);
  if (!is_slab(gv) || !gv->dev->Utile[0]) return set_error(LBIB_E_STATE);
  lbib_device* d = gv->dev;
  *f = (double*)d->f; *Ns = d->Ns; *sx = d->sx; *gx0 = d->gx0;
  *U0 = d->Utile[0]; *U1 = d->Utile[1];
  return LBIB_OK;
}

int lbib_slab_connect(GV gv, double* lo_f, long lo_Ns, int lo_sx, int lo_gx0, double* hi_f, long hi_Ns, int hi_sx,
                      int hi_gx0, int n, double* const* U0, double* const* U1) {
  if (!gv) return set_error(LBIB_E_ARG);
  if (!is_slab(gv)) return set_error(LBIB_E_STATE);
  return lbdev_slab_connect(gv->dev, lo_f, lo_Ns, lo_sx, lo_gx0, hi_f, hi_Ns, hi_sx, hi_gx0, n, U0, U1)
             ? set_error(LBIB_E_ARG) : LBIB_OK;
}

int lbib_slab_step_fluid_direct(GV gv) {
  if (!gv) return set_error(LBIB_E_ARG);
  if (!is_slab(gv) || gv->dev->npeer_U < 1) return set_error(LBIB_E_STATE);
  lbib_device* d = gv->dev;
  static const int order[] = {0, 3, 4};
  for (int i = 0; i < 3; ++i) {
    int rc = lbdev_stage(d, order[i], gv->time);
    if (rc) return set_error(rc);
  }
  const int par = d->parity ^ 1;
  int rc = lbdev_slab_push(d, par);
  return rc ? set_error(rc == -4 ? LBIB_E_STATE : LBIB_E_CUDA) : par;
}

int lbib_slab_step_moments_direct(GV gv) {
  if (!gv) return set_error(LBIB_E_ARG);
  if (!is_slab(gv) || gv->dev->steps == 0 || gv->dev->npeer_U < 1) return set_error(LBIB_E_STATE);
  int rc = lbdev_slab_moments_bcast(gv->dev);
  return rc ? set_error(rc == -4 ? LBIB_E_STATE : LBIB_E_CUDA) : LBIB_OK;
}

int lbib_slab_check(GV gv) {
  if (!gv || !gv->dev) return set_error(LBIB_E_STATE);
  int failed = 0;
  int e = lbdev_check(gv->dev, &failed);
  if (e) {
    if (e != LBIB_E_CUDA) gv->time = failed;
    return set_error(e);
  }
  return LBIB_OK;
}

int lbib_peer_access(int device, int peer) {
  int rc = lbdev_peer_access(device, peer);
  return rc ? set_error(rc == -1 ? LBIB_E_ARG : LBIB_E_CUDA) : LBIB_OK;
}

int lbib_ipc_handle(void* dev_ptr, void* handle) {
  if (!dev_ptr || !handle) return set_error(LBIB_E_ARG);
  return lbdev_ipc_handle(dev_ptr, handle) ? set_error(LBIB_E_CUDA) : LBIB_OK;
}

int lbib_ipc_open(const void* handle, void** dev_ptr) {
  if (!handle || !dev_ptr) return set_error(LBIB_E_ARG);
  return lbdev_ipc_open(handle, dev_ptr) ? set_error(LBIB_E_CUDA) : LBIB_OK;
}

int lbib_ipc_close(void* dev_ptr) {
  if (!dev_ptr) return set_error(LBIB_E_ARG);
  return lbdev_ipc_close(dev_ptr) ? set_error(LBIB_E_CUDA) : LBIB_OK;
}

int lbib_kernel_variants(GV gv) {
  if (!gv || !gv->dev) return set_error(LBIB_E_STATE);
  return lbdev_variants(gv->dev);
}

int lbib_set_kernel_variant(GV gv, int variant) {
  if (!gv || !gv->dev) return set_error(LBIB_E_STATE);
  return lbdev_set_variant(gv->dev, variant) ? set_error(LBIB_E_ARG) : LBIB_OK;
}

int lbib_autotune(GV gv, int steps, double* ms_per_variant, int max_variants) {
  if (!gv || !gv->dev) return set_error(LBIB_E_STATE);
  int best = 0;
  int rc = lbdev_autotune(gv->dev, steps, ms_per_variant, max_variants, &best);
  return rc ? set_error(rc) : best;
}

/* ---- restart files ---------------------------------------------------- */

/* File header: magic, layout version, the grid, precision, compat, the
 * sheets' shapes, physics and gv->time; the GPU state follows. */
#define LBIB_RESTART_MAGIC "LBIBRST1"

int lbib_save_restart(GV gv, const char* path) {
  if (!gv || !gv->dev || !gv->fiber_shape || !path) return set_error(LBIB_E_STATE);
  if (is_slab(gv)) return set_error(LBIB_E_STATE);
  FILE* fp = fopen(path, "wb");
  if (!fp) return set_error(LBIB_E_IO);
  lbib_device* d = gv->dev;
  int h[8] = {1, d->nx, d->ny, d->nz, d->prec, d->compat, gv->fiber_shape->num_sheets, gv->time};
  double phys[8] = {d->tau, d->u_l, d->rho_l, d->Ks_l, d->Kb_l, d->g_l, d->cs_l, (double)d->dt};
  int ok = fwrite(LBIB_RESTART_MAGIC, 1, 8, fp) == 8 && fwrite(h, sizeof(h), 1, fp) == 1 &&
           fwrite(phys, sizeof(phys), 1, fp) == 1;
  for (int k = 0; ok && k < gv->fiber_shape->num_sheets; ++k) {
    const int rc2[2] = {gv->fiber_shape->sheets[k].num_rows, gv->fiber_shape->sheets[k].num_cols};
    ok = fwrite(rc2, sizeof(rc2), 1, fp) == 1;
  }
  int rc = ok ? lbdev_save_state(d, fp) : LBIB_E_IO;
  if (fclose(fp) != 0 && !rc) rc = LBIB_E_IO;
  return rc ? set_error(rc) : LBIB_OK;
}

int lbib_load_restart(GV gv, const char* path) {
  if (!gv || !gv->dev || !gv->fiber_shape || !path) return set_error(LBIB_E_STATE);
  if (is_slab(gv)) return set_error(LBIB_E_STATE);
  FILE* fp = fopen(path, "rb");
  if (!fp) return set_error(LBIB_E_IO);
  lbib_device* d = gv->dev;
  char magic[8];
  int h[8];
  double phys[8];
  int rc = 0;
  if (fread(magic, 1, 8, fp) != 8 || memcmp(magic, LBIB_RESTART_MAGIC, 8) || fread(h, sizeof(h), 1, fp) != 1 ||
      fread(phys, sizeof(phys), 1, fp) != 1)
    rc = LBIB_E_IO;
  if (!rc && (h[0] != 1 || h[1] != d->nx || h[2] != d->ny || h[3] != d->nz || h[4] != d->prec ||
              h[6] != gv->fiber_shape->num_sheets))
    rc = LBIB_E_ARG;
  for (int k = 0; !rc && k < gv->fiber_shape->num_sheets; ++k) {
    int rc2[2];
    if (fread(rc2, sizeof(rc2), 1, fp) != 1) rc = LBIB_E_IO;
    else if (rc2[0] != gv->fiber_shape->sheets[k].num_rows || rc2[1] != gv->fiber_shape->sheets[k].num_cols)
      rc = LBIB_E_ARG;
  }
  if (!rc) {
    /* the saved physics and compat replace the current ones */
    gv->tau = phys[0]; gv->u_l = phys[1]; gv->rho_l = phys[2]; gv->Ks_l = phys[3]; gv->Kb_l = phys[4];
    gv->g_l = phys[5]; gv->cs_l = phys[6]; gv->dt = (int)phys[7];
    gv->lbib_compat = h[5];
    lbdev_config c;
    fill_config(gv, &c);
    rc = lbdev_set_physics(d, &c);
  }
  if (!rc) rc = lbdev_load_state(d, fp);
  fclose(fp);
  if (!rc) {
    gv->time = h[7];
    rc = lbib_sync_to_host(gv);
  }
  return rc ? set_error(rc) : LBIB_OK;
}

/* ---- the step -------------------------------------------------------- */

static int stage(LV lv, int which) {
  if (!lv || !lv->gv) return set_error(LBIB_E_ARG);
  if (lv->tid != 0) return LBIB_OK;
  GV gv = lv->gv;
  if (!gv->dev) return set_error(LBIB_E_STATE);
  int rc = lbdev_stage(gv->dev, which, gv->time);
  return rc ? set_error(rc) : LBIB_OK;
}

void compute_bendingforce(LV lv) { stage(lv, 0); }
void compute_stretchingforce(LV lv) { stage(lv, 1); }
void compute_elasticforce(LV lv) { stage(lv, 2); }
void fiber_SpreadForce(LV lv) { stage(lv, 3); }
void fluid_get_SpreadForce(LV lv) { (void)lv; }
void get_influentialdomain_fluid_grid_and_SpreadForce(LV lv) { stage(lv, 3); }
void compute_eqlbrmdistrfuncDF1(LV lv) { stage(lv, 4); }
void stream_distrfunc(LV lv) { stage(lv, 5); }
void bounceback_rigidwalls(LV lv) { stage(lv, 6); }
void compute_rho_and_u(LV lv) { stage(lv, 7); }
void fluid_SpreadVelocity(LV lv) { (void)lv; }
void fiber_get_SpreadVelocity(LV lv) { stage(lv, 8); }
void moveFiberSheet(LV lv) { stage(lv, 8); }
void copy_inout_to_df2(LV lv) { stage(lv, 9); }
void replace_old_DF(LV lv) { stage(lv, 10); }
void periodicBC(LV lv) { (void)lv; }

int lbib_stage(GV gv, int which) {
  struct lv_t lv = {0, gv};
  return stage(&lv, which);
}

static int fieldview_header_files(GV gv) {
  FILE* f = fopen("FV_nameFluid.nam", "w");
  if (!f) return set_error(LBIB_E_IO);
  fprintf(f, "u\nv\nw");
  fclose(f);
  f = fopen("FV_nameFiber.nam", "w");
  if (!f) return set_error(LBIB_E_IO);
  fprintf(f, "Afx\nAfy\nAfz");
  fclose(f);
  save_fluid_sub_grid_cord_use_fv(gv, 0, 0, 0, gv->fluid_grid->x_dim, gv->fluid_grid->y_dim, gv->fluid_grid->z_dim,
                                  "FV_gridFluid.xyz");
  return LBIB_OK;
}

static void dump_step(GV gv) {
  char f1[96], f2[96];
  int mode = gv->lbib_dump_mode;
  if (gv->dump <= 0) return;
  if ((mode & LBIB_DUMP_FIELDVIEW) && ((gv->time % gv->dump == 0) || gv->time == 1)) {
    snprintf(f1, sizeof(f1), "FV_fluid_vel_%d.f", gv->time);
    save_fluid_sub_grid_vel_use_fv(gv, 0, 0, 0, gv->fluid_grid->x_dim, gv->fluid_grid->y_dim, gv->fluid_grid->z_dim, f1);
    snprintf(f1, sizeof(f1), "FV_gridFiber%d.xyz", gv->time);
    snprintf(f2, sizeof(f2), "FV_fiber_elastic_force_%d.f", gv->time);
    save_fiber_sub_grid_cord_ef_use_fv(gv, 0, 0, gv->fiber_shape->sheets[0].num_rows - 1,
                                       gv->fiber_shape->sheets[0].num_cols - 1, f1, f2);
  }
  if ((mode & LBIB_DUMP_BINARY) && (gv->time % gv->dump == 0)) {
    /* one file per sheet, named with the fiber task's rank as mpi/do_thread.c:345 */
    for (int k = 0; k < gv->fiber_shape->num_sheets; ++k) {
      snprintf(f1, sizeof(f1), "Fiber%d_dump_step%d.bin", gv->num_fluid_tasks + k, gv->time);
      Fibersheet* sh = &gv->fiber_shape->sheets[k];
      Fibershape one = {sh, 1};
      Fibershape* keep = gv->fiber_shape;
      gv->fiber_shape = &one;
      save_fiber_sub_grid_binary(gv, 0, 0, sh->num_rows - 1, sh->num_cols - 1, f1);
      gv->fiber_shape = keep;
    }
  }
}

/* How often the step loop reads the device error word (a host sync). */
#define LBIB_CHECK_EVERY 50

void* do_thread(void* v) {
  LV lv = (LV)v;
  if (!lv || !lv->gv) { set_error(LBIB_E_ARG); return NULL; }
  if (lv->tid != 0) return NULL;
  GV gv = lv->gv;
  if (!gv->dev) { set_error(LBIB_E_STATE); return NULL; }
  int stop = gv->timesteps > 0 ? gv->timesteps : gv->TIME_STOP;
  if ((gv->lbib_dump_mode & LBIB_DUMP_FIELDVIEW) && gv->dump > 0) fieldview_header_files(gv);
  int since_check = 0;
  while (gv->time <= stop) {
    int rc = lbdev_step(gv->dev, gv->time);
    if (rc) { set_error(rc); return NULL; }
    int dumping = gv->dump > 0 && gv->lbib_dump_mode != LBIB_DUMP_NONE &&
                  ((gv->time % gv->dump == 0) || (gv->time == 1 && (gv->lbib_dump_mode & LBIB_DUMP_FIELDVIEW)));
    if (dumping || ++since_check >= LBIB_CHECK_EVERY || gv->time == stop) {
      int failed = 0;
      int e = lbdev_check(gv->dev, &failed);
      since_check = 0;
      if (e) {
        gv->time = failed;
        set_error(e);
        return NULL;
      }
    }
    if (dumping) dump_step(gv);
    gv->time += gv->dt;
  }
  return NULL;
}

int lbib_run(GV gv, int nsteps) {
  if (!gv || nsteps < 0) return set_error(LBIB_E_ARG);
  if (is_slab(gv)) return set_error(LBIB_E_STATE);
  int keep_ts = gv->timesteps;
  gv->timesteps = gv->time + nsteps - 1;
  struct lv_t lv = {0, gv};
  int before = lbib_last_error();
  do_thread(&lv);
  gv->timesteps = keep_ts;
  int after = lbib_last_error();
  return after != before ? after : LBIB_OK;
}

int lbib_synchronize(GV gv) {
  if (!gv || !gv->dev) return set_error(LBIB_E_STATE);
  return lbdev_sync(gv->dev) ? set_error(LBIB_E_CUDA) : LBIB_OK;
}

void* lbib_stream(GV gv) { return (gv && gv->dev) ? (void*)gv->dev->stream : NULL; }

long lbib_kernel_launches(GV gv) { return (gv && gv->dev) ? gv->dev->kernel_launches : 0; }

int lbib_profile_begin(GV gv) {
  if (!gv || !gv->dev) return set_error(LBIB_E_STATE);
  return lbdev_profile_begin(gv->dev) ? set_error(LBIB_E_CUDA) : LBIB_OK;
}

int lbib_profile_end(GV gv, double* stage_ms, long* steps) {
  if (!gv || !gv->dev) return set_error(LBIB_E_STATE);
  if (!stage_ms) return set_error(LBIB_E_ARG);
  int rc = lbdev_profile_end(gv->dev, stage_ms, steps);
  return rc ? set_error(rc) : LBIB_OK;
}

/* ---- host views ------------------------------------------------------- */

int lbib_sync_to_host(GV gv) {
  if (!gv || !gv->dev || !gv->fiber_shape) return set_error(LBIB_E_STATE);
  long S = total_nodes(gv);
  if (S != gv->dev->S) return set_error(LBIB_E_STATE);
  /* every sheet's block page-locked: one direct copy each */
  int direct = 1;
  for (int k = 0; direct && k < gv->fiber_shape->num_sheets; ++k) {
    const Fibersheet* sh = &gv->fiber_shape->sheets[k];
    const Fibernode* b = sheet_block(sh);
    direct = b && lbdev_is_registered(gv->dev, b, sizeof(Fibernode) * (size_t)sh->num_rows * sh->num_cols);
  }
  int rc = 0;
  if (direct) {
    long o = 0;
    for (int k = 0; !rc && k < gv->fiber_shape->num_sheets; ++k) {
      Fibersheet* sh = &gv->fiber_shape->sheets[k];
      const long n = (long)sh->num_rows * sh->num_cols;
      rc = lbdev_copy_nodes_out(gv->dev, o, n, (double*)sh->fibers[0].nodes);
      o += n;
    }
    if (!rc) rc = lbdev_sync(gv->dev);
  } else {
    rc = lbdev_get_nodes(gv->dev, NULL);    /* into the pinned staging buffer */
    if (!rc) unpack_nodes(gv, gv->dev->h_nodes);
  }
  return rc ? set_error(rc) : LBIB_OK;
}

int lbib_get_moments(GV gv, double* rho, double* ux, double* uy, double* uz) {
  if (!gv || !gv->dev) return set_error(LBIB_E_STATE);
  if (!rho || !ux || !uy || !uz) return set_error(LBIB_E_ARG);
  int rc = lbdev_get_moments(gv->dev, rho, ux, uy, uz);
  return rc ? set_error(rc) : LBIB_OK;
}

int lbib_get_force(GV gv, double* fx, double* fy, double* fz) {
  if (!gv || !gv->dev) return set_error(LBIB_E_STATE);
  if (!fx || !fy || !fz) return set_error(LBIB_E_ARG);
  int rc = lbdev_get_force(gv->dev, fx, fy, fz);
  return rc ? set_error(rc) : LBIB_OK;
}

int lbib_conservation_sums(GV gv, double* out) {
  if (!gv || !out) return set_error(LBIB_E_ARG);
  if (!gv->dev) return set_error(LBIB_E_STATE);
  int rc = lbdev_conservation(gv->dev, out);
  return rc ? set_error(rc) : LBIB_OK;
}

int lbib_get_df1(GV gv, double* out) {
  if (!gv || !gv->dev) return set_error(LBIB_E_STATE);
  if (!out) return set_error(LBIB_E_ARG);
  int rc = lbdev_get_df1(gv->dev, out);
  return rc ? set_error(rc) : LBIB_OK;
}

static long sheet_offset(GV gv, int sheet) {
  long o = 0;
  for (int k = 0; k < sheet; ++k)
    o += (long)gv->fiber_shape->sheets[k].num_rows * gv->fiber_shape->sheets[k].num_cols;
  return o;
}

int lbib_get_sheet(GV gv, int sheet, double* out) {
  if (!gv || !gv->dev || !gv->fiber_shape) return set_error(LBIB_E_STATE);
  if (!out || sheet < 0 || sheet >= gv->fiber_shape->num_sheets) return set_error(LBIB_E_ARG);
  const Fibersheet* sh = &gv->fiber_shape->sheets[sheet];
  int rc = lbdev_copy_nodes_out(gv->dev, sheet_offset(gv, sheet), (long)sh->num_rows * sh->num_cols, out);
  if (!rc) rc = lbdev_sync(gv->dev);
  return rc ? set_error(rc) : LBIB_OK;
}

int lbib_set_sheet(GV gv, int sheet, const double* in) {
  if (!gv || !gv->dev || !gv->fiber_shape) return set_error(LBIB_E_STATE);
  if (!in || sheet < 0 || sheet >= gv->fiber_shape->num_sheets) return set_error(LBIB_E_ARG);
  const Fibersheet* sh = &gv->fiber_shape->sheets[sheet];
  int rc = lbdev_copy_nodes_in(gv->dev, sheet_offset(gv, sheet), (long)sh->num_rows * sh->num_cols, in);
  if (!rc) rc = lbdev_sync(gv->dev);
  return rc ? set_error(rc) : LBIB_OK;
}

/* ---- one-call set-up for bindings ------------------------------------ */

GV lbib_case_create(int nx, int ny, int nz, int cube_size, int nsheets,
                    const int* rows, const int* cols,
                    const double* width, const double* height,
                    const double* x0, const double* y0, const double* z0,
                    double tau, double u_l, double Ks_l, double Kb_l, int compat) {
  return lbib_case_create_prec(nx, ny, nz, cube_size, nsheets, rows, cols, width, height, x0, y0, z0,
                               tau, u_l, Ks_l, Kb_l, compat, LBIB_PREC_F64);
}

static GV case_create(int nx, int ny, int nz, int cube_size, int nsheets,
                      const int* rows, const int* cols,
                      const double* width, const double* height,
                      const double* x0, const double* y0, const double* z0,
                      double tau, double u_l, double Ks_l, double Kb_l, int compat,
                      int precision, int x_lo, int x_hi);

GV lbib_case_create_prec(int nx, int ny, int nz, int cube_size, int nsheets,
                         const int* rows, const int* cols,
                         const double* width, const double* height,
                         const double* x0, const double* y0, const double* z0,
                         double tau, double u_l, double Ks_l, double Kb_l, int compat,
                         int precision) {
  return case_create(nx, ny, nz, cube_size, nsheets, rows, cols, width, height, x0, y0, z0,
                     tau, u_l, Ks_l, Kb_l, compat, precision, 0, 0);
}

GV lbib_case_create_slab(int nx, int ny, int nz, int cube_size, int nsheets,
                         const int* rows, const int* cols,
                         const double* width, const double* height,
                         const double* x0, const double* y0, const double* z0,
                         double tau, double u_l, double Ks_l, double Kb_l, int compat,
                         int x_lo, int x_hi) {
  return case_create(nx, ny, nz, cube_size, nsheets, rows, cols, width, height, x0, y0, z0,
                     tau, u_l, Ks_l, Kb_l, compat, LBIB_PREC_F64, x_lo, x_hi);
}

static GV case_create(int nx, int ny, int nz, int cube_size, int nsheets,
                      const int* rows, const int* cols,
                      const double* width, const double* height,
                      const double* x0, const double* y0, const double* z0,
                      double tau, double u_l, double Ks_l, double Kb_l, int compat,
                      int precision, int x_lo, int x_hi) {
  if (nsheets < 1 || !rows || !cols || !width || !height || !x0 || !y0 || !z0 ||
      !precision_ok(precision)) {
    set_error(LBIB_E_ARG);
    return NULL;
  }
  GV gv = (GV)calloc(1, sizeof(*gv));
  gv->fluid_grid = (Fluidgrid*)calloc(1, sizeof(Fluidgrid));
  gv->fluid_grid->x_dim = nx;
  gv->fluid_grid->y_dim = ny;
  gv->fluid_grid->z_dim = nz;
  gv->cube_size = cube_size;
  gv->fiber_shape = (Fibershape*)calloc(1, sizeof(Fibershape));
  gv->fiber_shape->num_sheets = nsheets;
  gv->fiber_shape->sheets = (Fibersheet*)calloc(nsheets, sizeof(Fibersheet));
  for (int k = 0; k < nsheets; ++k) {
    Fibersheet* s = &gv->fiber_shape->sheets[k];
    s->num_rows = rows[k]; s->num_cols = cols[k];
    s->width = width[k]; s->height = height[k];
    s->x_orig = x0[k]; s->y_orig = y0[k]; s->z_orig = z0[k];
  }
  int before = lbib_last_error();
  init_gv_constant(gv);
  gv->lbib_compat = compat;
  gv->lbib_precision = precision;
  gv->lbib_slab_lo = x_lo;
  gv->lbib_slab_hi = x_hi;
  gv->tau = tau; gv->u_l = u_l; gv->Ks_l = Ks_l; gv->Kb_l = Kb_l;
  gen_fluid_grid(gv->fluid_grid, cube_size, 0, gv);
  for (int k = 0; k < nsheets; ++k) gen_fiber_sheet(&gv->fiber_shape->sheets[k]);
  if (lbib_last_error() == before) init_gv(gv);
  if (lbib_last_error() == before) lbib_set_params(gv, tau, u_l, Ks_l, Kb_l);
  if (lbib_last_error() == before) init_eqlbrmdistrfuncDF0(gv);
  if (lbib_last_error() == before) init_df1(gv);
  if (lbib_last_error() == before) init_df_inout(gv);
  if (lbib_last_error() == before && gv->dev && lbdev_sync(gv->dev)) set_error(LBIB_E_CUDA);
  if (lbib_last_error() != before) {
    lbib_case_free(gv);
    return NULL;
  }
  return gv;
}

void lbib_free(GV gv) {
  if (!gv) return;
  if (gv->dev) { lbdev_free(gv->dev); gv->dev = NULL; }
  if (gv->fiber_shape) {
    for (int k = 0; k < gv->fiber_shape->num_sheets; ++k) {
      Fibersheet* sh = &gv->fiber_shape->sheets[k];
      if (!sh->fibers) continue;
      free(sh->fibers[0].nodes);      /* the block of all rows (gen_fiber_sheet) */
      free(sh->fibers);
      sh->fibers = NULL;
    }
  }
}

void lbib_case_free(GV gv) {
  if (!gv) return;
  lbib_free(gv);
  if (gv->fiber_shape) { free(gv->fiber_shape->sheets); free(gv->fiber_shape); }
  free(gv->fluid_grid);
  free(gv);
}

/* ---- dumps: mpi/print_info.c, cube_pthread/lbm_ib.c:331-692 ----------- */

void save_fiber_sub_grid(GV gv, int start_y, int start_z, int end_y, int end_z, char fName[]) {
  if (lbib_sync_to_host(gv)) return;
  FILE* oFile = fopen(fName, "w");
  if (!oFile) { set_error(LBIB_E_IO); return; }
  for (int k = 0; k < gv->fiber_shape->num_sheets; ++k) {
    Fiber* fiber_array = gv->fiber_shape->sheets[k].fibers;
    fprintf(oFile, "Fiber_sheets[%d] (i,j): {cord_x, cord_y, cord_z} || SF_x, SF_y, SF_z || BF_x, BF_y, BF_z || EF_x, EF_y, EF_z\n", k);
    for (int i = start_y; i <= end_y; ++i)
      for (int j = start_z; j <= end_z; ++j) {
        Fibernode* node = fiber_array[i].nodes + j;
        fprintf(oFile, "(%2d,%2d):{%.24f,%.24f,%.24f} || %.24f,%.24f,%.24f || %.24f,%.24f,%.24f || %.24f,%.24f,%.24f\n",
                i, j, node->x, node->y, node->z,
                node->stretch_force_x, node->stretch_force_y, node->stretch_force_z,
                node->bend_force_x, node->bend_force_y, node->bend_force_z,
                node->elastic_force_x, node->elastic_force_y, node->elastic_force_z);
      }
  }
  fclose(oFile);
}

/* Records {int i, int j, Fibernode} = 104 bytes, row-major, as
 * mpi/print_info.c:76-115 writes them. */
void save_fiber_sub_grid_binary(GV gv, int start_y, int start_z, int end_y, int end_z, char fName[]) {
  if (lbib_sync_to_host(gv)) return;
  FILE* oFile = fopen(fName, "wb");
  if (!oFile) { set_error(LBIB_E_IO); return; }
  const size_t rec = sizeof(int) * 2 + sizeof(Fibernode);
  long n = (long)(end_y - start_y + 1) * (end_z - start_z + 1);
  char* buffer = (char*)malloc(rec * n * gv->fiber_shape->num_sheets);
  long count = 0;
  for (int k = 0; k < gv->fiber_shape->num_sheets; ++k) {
    Fiber* fiber_array = gv->fiber_shape->sheets[k].fibers;
    for (int i = start_y; i <= end_y; ++i)
      for (int j = start_z; j <= end_z; ++j) {
        char* p = buffer + count;
        memcpy(p, &i, sizeof(int));
        memcpy(p + sizeof(int), &j, sizeof(int));
        memcpy(p + 2 * sizeof(int), fiber_array[i].nodes + j, sizeof(Fibernode));
        count += rec;
      }
  }
  fwrite(buffer, 1, count, oFile);
  free(buffer);
  fclose(oFile);
}

static int fetch_moments(GV gv, double** rho, double** ux, double** uy, double** uz) {
  long N = (long)gv->fluid_grid->x_dim * gv->fluid_grid->y_dim * gv->fluid_grid->z_dim;
  *rho = (double*)malloc(sizeof(double) * N);
  *ux = (double*)malloc(sizeof(double) * N);
  *uy = (double*)malloc(sizeof(double) * N);
  *uz = (double*)malloc(sizeof(double) * N);
  if (!*rho || !*ux || !*uy || !*uz) return set_error(LBIB_E_NOMEM);
  return lbib_get_moments(gv, *rho, *ux, *uy, *uz);
}

/* FieldView velocity file, cube_pthread/lbm_ib.c:436-507. */
void save_fluid_sub_grid_vel_use_fv(GV gv, int start_x, int start_y, int start_z, int end_x, int end_y, int end_z,
                                    char fName[]) {
  double *rho = NULL, *ux = NULL, *uy = NULL, *uz = NULL;
  if (fetch_moments(gv, &rho, &ux, &uy, &uz) == LBIB_OK) {
    FILE* oFile = fopen(fName, "w");
    if (!oFile) {
      set_error(LBIB_E_IO);
    } else {
      int nx = gv->fluid_grid->x_dim, ny = gv->fluid_grid->y_dim;
      fprintf(oFile, "%d,%d,%d,3\n", end_x - start_x, end_y - start_y, end_z - start_z);
      const double* comp[3] = {ux, uy, uz};
      for (int c = 0; c < 3; ++c)
        for (int Z = start_z; Z < end_z; Z++)
          for (int Y = start_y; Y < end_y; Y++)
            for (int X = start_x; X < end_x; X++) fprintf(oFile, "%f,", comp[c][((long)Z * ny + Y) * nx + X]);
      fclose(oFile);
    }
  }
  free(rho); free(ux); free(uy); free(uz);
}

/* FieldView grid file, cube_pthread/lbm_ib.c:510-549. */
void save_fluid_sub_grid_cord_use_fv(GV gv, int start_x, int start_y, int start_z, int end_x, int end_y, int end_z,
                                     char fName[]) {
  (void)gv;
  FILE* oFile = fopen(fName, "wb");
  if (!oFile) { set_error(LBIB_E_IO); return; }
  fprintf(oFile, "%d,%d,%d\n", end_x - start_x, end_y - start_y, end_z - start_z);
  for (int Z = start_z; Z < end_z; Z++)
    for (int Y = start_y; Y < end_y; Y++)
      for (int X = start_x; X < end_x; X++) fprintf(oFile, "%d,", X);
  for (int Z = start_z; Z < end_z; Z++)
    for (int Y = start_y; Y < end_y; Y++)
      for (int X = start_x; X < end_x; X++) fprintf(oFile, "%d,", Y);
  for (int Z = start_z; Z < end_z; Z++)
    for (int Y = start_y; Y < end_y; Y++)
      for (int X = start_x; X < end_x; X++) fprintf(oFile, "%d,", Z);
  fclose(oFile);
}

/* FieldView fiber grid and elastic-force files, cube_pthread/lbm_ib.c:650-692
 * (sheet 0, columns outer, rows inner). */
void save_fiber_sub_grid_cord_ef_use_fv(GV gv, int start_y, int start_z, int end_y, int end_z, char grid_fname[],
                                        char elastic_force_fname[]) {
  if (lbib_sync_to_host(gv)) return;
  FILE* grid_file = fopen(grid_fname, "w");
  FILE* ef_file = fopen(elastic_force_fname, "w");
  if (!grid_file || !ef_file) {
    if (grid_file) fclose(grid_file);
    if (ef_file) fclose(ef_file);
    set_error(LBIB_E_IO);
    return;
  }
  fprintf(grid_file, "%d,%d,1\n", end_y - start_y + 1, end_z - start_z + 1);
  fprintf(ef_file, "%d,%d,1,3\n", end_y - start_y + 1, end_z - start_z + 1);
  Fiber* fiber_array = gv->fiber_shape->sheets[0].fibers;
  for (int c = 0; c < 3; ++c)
    for (int j = start_z; j <= end_z; ++j)
      for (int i = start_y; i <= end_y; ++i) {
        Fibernode* node = fiber_array[i].nodes + j;
        const double pos[3] = {node->x, node->y, node->z};
        const double ef[3] = {node->elastic_force_x, node->elastic_force_y, node->elastic_force_z};
        fprintf(grid_file, "%f,", pos[c]);
        fprintf(ef_file, "%f,", ef[c]);
      }
  fclose(grid_file);
  fclose(ef_file);
}

/* Text dump of cubes, mpi/print_info.c:231-298.  rho, u, F and the
 * populations df1 = df2 (the state the next step starts from) come from the
 * GPU; dfeq is the equilibrium of the current rho, u (the GPU does not keep
 * the previous step's equilibrium). */
void save_fluid_sub_grid(GV gv, int start_x, int start_y, int start_z, int end_x, int end_y, int end_z,
                         char fName[]) {
  int nx = gv->fluid_grid->x_dim, ny = gv->fluid_grid->y_dim;
  long N = (long)nx * ny * gv->fluid_grid->z_dim;
  double *rho = NULL, *ux = NULL, *uy = NULL, *uz = NULL;
  double* df = (double*)malloc(sizeof(double) * 19 * N);
  double* F = (double*)malloc(sizeof(double) * 3 * N);
  if (!df || !F || fetch_moments(gv, &rho, &ux, &uy, &uz) || lbib_get_df1(gv, df) ||
      lbib_get_force(gv, F, F + N, F + 2 * N)) {
    free(df); free(F); free(rho); free(ux); free(uy); free(uz);
    return;
  }
  FILE* oFile = fopen(fName, "w");
  if (!oFile) {
    set_error(LBIB_E_IO);
  } else {
    int cs = gv->cube_size;
    for (int BI = start_x / cs; BI <= end_x / cs; ++BI)
      for (int BJ = start_y / cs; BJ <= end_y / cs; ++BJ)
        for (int BK = start_z / cs; BK <= end_z / cs; ++BK) {
          fprintf(oFile, "(BI,BJ,BK): {vel_x, vel_y, vel_z} || {G0, DF1, DF2}|| rho || {ElasticF_x, y, z}\n");
          for (int li = 0; li < cs; li++)
            for (int lj = 0; lj < cs; lj++)
              for (int lk = 0; lk < cs; lk++) {
                fprintf(oFile, "For cube <%d,%d,%d> Rank %d\n", BI, BJ, BK, gv->taskid);
                int X = BI * cs + li, Y = BJ * cs + lj, Z = BK * cs + lk;
                long i = ((long)Z * ny + Y) * nx + X;
                double usq = ux[i] * ux[i] + uy[i] * uy[i] + uz[i] * uz[i];
                for (int ksi = 0; ksi < 19; ksi++) {
                  const double* c = LBIB_C[ksi];
                  double cu = c[0] * ux[i] + c[1] * uy[i] + c[2] * uz[i];
                  double w = ksi == 0 ? 1.0 / 3.0 : (ksi <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
                  double feq = ksi == 0 ? w * rho[i] * (1.0 - 1.5 * usq)
                                        : w * rho[i] * (1.0 + 3.0 * cu + 4.5 * (cu * cu) - 1.5 * usq);
                  double d1 = df[ksi * N + i];
                  fprintf(oFile, "(%d,%d,%d, %2d):{%.24f,%.24f,%.24f} || {%.24f,%.24f,%.24f} || %.24f || {%.24f,%.24f,%.24f}\n",
                          X, Y, Z, ksi, ux[i], uy[i], uz[i], feq, d1, d1, rho[i], F[i], F[N + i], F[2 * N + i]);
                }
              }
        }
    fclose(oFile);
  }
  free(df); free(F); free(rho); free(ux); free(uy); free(uz);
}
