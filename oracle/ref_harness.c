/*
 * Serial / threaded driver around the reference's own pthread solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
 * reference source cube_pthread/lbm_ib.c (included below, never copied into
 * this repository) into oracle/_ref/libref.so by oracle/Makefile.  Only the
 * tests, the smoke check and the CPU-baseline legs of bench.py load it.
 *
 * What it does, and why:
 *   - Builds the reference GV exactly as cube_pthread/lbm_ib.c:main does
 *     (lbm_ib.c:3835-3912) but with P=Q=R=1 and a barrier of count 1, and
 *     calls do_thread (lbm_ib.c:3087) on the calling thread.  Serial runs are
 *     race-free and bit-reproducible; the threaded pthread layouts with P>=2
 *     are racy (spread zero/add race, lbm_ib.c:1385-1514) or corrupt wall
 *     cells (copy_inout_to_df2 loops BK < num_cubes_x, lbm_ib.c:2800).
 *   - Passes the internal (nx, ny, nz) straight to gen_fluid_grid
 *     (lbm_ib.c:924), bypassing the CLI's x/z swap (lbm_ib.c:3792-3794).
 *   - Overrides tau, u_l, Ks_l and Kb_l after init_gv (which hard-codes them,
 *     lbm_ib.c:750-773) and re-applies the two things init_gv derived from the
 *     hard-coded u_l: vel_x on every node (lbm_ib.c:837-849) and the sheet's
 *     one-step shift x += u_l*dt (lbm_ib.c:857-862).
 *   - Exposes per-kernel entry points and raw field access so the oracle's C
 *     restatement (oracle/lbib_oracle.c) and the CUDA path can be pinned
 *     against the reference itself.
 */
#include <unistd.h>
#include <limits.h>

#define main lbib_ref_cli_main
#include LBIB_REF_SOURCE
#undef main

typedef struct ref_case_t {
  GV gv;
  struct lv_t lv;
} ref_case;

/* Cell (x, y, z) of the reference's cube-tiled AoS grid. */
static Fluidnode* ref_node(GV gv, int x, int y, int z) {
  int cs = gv->cube_size;
  int cube = (x / cs) * gv->num_cubes_y * gv->num_cubes_z + (y / cs) * gv->num_cubes_z + (z / cs);
  int node = (x % cs) * cs * cs + (y % cs) * cs + (z % cs);
  return &gv->fluid_grid->sub_fluid_grid[cube].nodes[node];
}

void* ref_create(int nx, int ny, int nz, int cube_size,
                 int rows, int cols, double width, double height,
                 double x0, double y0, double z0,
                 double tau, double u_l, double Ks_l, double Kb_l) {
  ref_case* rc = (ref_case*)calloc(1, sizeof(*rc));
  GV gv = (GV)calloc(1, sizeof(*gv));
  rc->gv = gv;
  gv->fiber_shape = (Fibershape*)calloc(1, sizeof(Fibershape));
  gv->fiber_shape->num_sheets = 1;
  gv->fiber_shape->sheets = (Fibersheet*)calloc(1, sizeof(Fibersheet));
  gv->P = gv->Q = gv->R = 1;
  gv->total_threads = 1;
  gv->TIME_STOP = 0;
  gv->dump = INT_MAX;

  Fibershape* shape = gen_fiber_shape(gv, width, height, cols, rows, x0, y0, z0);
  Fluidgrid* grid = gen_fluid_grid(gv, nx, ny, nz, cube_size);
  init_gv(gv, shape, grid, cube_size);

  gv->tau = tau;
  gv->u_l = u_l;
  gv->Ks_l = Ks_l;
  gv->Kb_l = Kb_l;
  int total_cubes = gv->num_cubes_x * gv->num_cubes_y * gv->num_cubes_z;
  int per_cube = cube_size * cube_size * cube_size;
  for (int c = 0; c < total_cubes; ++c)
    for (int n = 0; n < per_cube; ++n)
      grid->sub_fluid_grid[c].nodes[n].vel_x = u_l;
  Fibersheet* sh = &shape->sheets[0];
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c) {
      sh->fibers[r].nodes[c].x = x0;
      sh->fibers[r].nodes[c].x += gv->u_l * gv->dt;
    }

  gv->lock_Fluid = (pthread_mutex_t*)malloc(sizeof(pthread_mutex_t));
  pthread_mutex_init(&gv->lock_Fluid[0], NULL);
  pthread_barrier_init(&gv->barr, NULL, 1);

  init_eqlbrmdistrfuncDF0(gv);
  init_df1(gv);
  init_df_inout(gv);
  rc->lv.tid = 0;
  rc->lv.gv = gv;
  return rc;
}

/* Run nsteps of do_thread inside workdir (the reference always writes its
 * FieldView files at time == 1, lbm_ib.c:3503-3538). */
int ref_run(void* h, int nsteps, const char* workdir) {
  ref_case* rc = (ref_case*)h;
  GV gv = rc->gv;
  char old[PATH_MAX];
  if (!getcwd(old, sizeof(old))) return -1;
  if (workdir && chdir(workdir) != 0) return -2;
  gv->TIME_STOP = gv->time + nsteps - 1;
  int saved = dup(1);
  FILE* devnull = fopen("/dev/null", "w");
  fflush(stdout);
  if (devnull) dup2(fileno(devnull), 1);
  do_thread(&rc->lv);
  fflush(stdout);
  if (devnull) { dup2(saved, 1); fclose(devnull); }
  close(saved);
  if (workdir && chdir(old) != 0) return -3;
  return 0;
}

/* The same loop with the reference's own threading: P=1 (P>=2 is racy and
 * corrupts wall cells), Q*R threads, one mutex per thread, a barrier of
 * count Q*R -- what cube_pthread/lbm_ib.c:main sets up (lbm_ib.c:3844-3935). */
int ref_run_threaded(void* h, int nsteps, int Q, int R, const char* workdir) {
  ref_case* rc = (ref_case*)h;
  GV gv = rc->gv;
  int T = Q * R;
  if (gv->num_cubes_y % Q || gv->num_cubes_z % R) return -4;
  if (gv->fiber_shape->sheets[0].num_rows < T) return -5;
  char old[PATH_MAX];
  if (!getcwd(old, sizeof(old))) return -1;
  if (workdir && chdir(workdir) != 0) return -2;
  gv->P = 1; gv->Q = Q; gv->R = R; gv->total_threads = T;
  pthread_mutex_t* locks = (pthread_mutex_t*)malloc(sizeof(pthread_mutex_t) * T);
  for (int i = 0; i < T; ++i) pthread_mutex_init(&locks[i], NULL);
  pthread_mutex_t* saved_locks = gv->lock_Fluid;
  gv->lock_Fluid = locks;
  pthread_barrier_destroy(&gv->barr);
  pthread_barrier_init(&gv->barr, NULL, T);
  gv->TIME_STOP = gv->time + nsteps - 1;
  int saved = dup(1);
  FILE* devnull = fopen("/dev/null", "w");
  fflush(stdout);
  if (devnull) dup2(fileno(devnull), 1);
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * T);
  struct lv_t* lvs = (struct lv_t*)malloc(sizeof(struct lv_t) * T);
  for (int i = 0; i < T; ++i) {
    lvs[i].tid = i; lvs[i].gv = gv;
    pthread_create(th + i, NULL, do_thread, lvs + i);
  }
  for (int i = 0; i < T; ++i) pthread_join(th[i], NULL);
  fflush(stdout);
  if (devnull) { dup2(saved, 1); fclose(devnull); }
  close(saved);
  free(th); free(lvs);
  for (int i = 0; i < T; ++i) pthread_mutex_destroy(&locks[i]);
  free(locks);
  gv->lock_Fluid = saved_locks;
  pthread_barrier_destroy(&gv->barr);
  pthread_barrier_init(&gv->barr, NULL, 1);
  gv->P = gv->Q = gv->R = 1; gv->total_threads = 1;
  if (workdir && chdir(old) != 0) return -3;
  return 0;
}

/* One reference stage on the calling thread (tid 0 of 1). */
int ref_call(void* h, int which) {
  ref_case* rc = (ref_case*)h;
  LV lv = &rc->lv;
  switch (which) {
    case 0: compute_bendingforce(lv); break;
    case 1: compute_stretchingforce(lv); break;
    case 2: compute_elasticforce(lv); break;
    case 3: get_influentialdomain_fluid_grid_and_SpreadForce(lv); break;
    case 4: compute_eqlbrmdistrfuncDF1(lv); break;
    case 5: stream_distrfunc(lv); break;
    case 6: bounceback_rigidwalls(lv); break;
    case 7: compute_rho_and_u(lv); break;
    case 8: moveFiberSheet(lv); break;
    case 9: copy_inout_to_df2(lv); break;
    case 10: replace_old_DF(lv); break;
    case 11: rc->gv->time += rc->gv->dt; break;
    default: return -1;
  }
  return 0;
}

int ref_time(void* h) { return ((ref_case*)h)->gv->time; }

/* Fields in x-fastest order: idx = (z*ny + y)*nx + x. */
void ref_get_moments(void* h, double* rho, double* ux, double* uy, double* uz) {
  GV gv = ((ref_case*)h)->gv;
  int nx = gv->fluid_grid->x_dim, ny = gv->fluid_grid->y_dim, nz = gv->fluid_grid->z_dim;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        Fluidnode* n = ref_node(gv, x, y, z);
        long i = ((long)z * ny + y) * nx + x;
        rho[i] = n->rho; ux[i] = n->vel_x; uy[i] = n->vel_y; uz[i] = n->vel_z;
      }
}

void ref_set_moments(void* h, const double* rho, const double* ux, const double* uy, const double* uz) {
  GV gv = ((ref_case*)h)->gv;
  int nx = gv->fluid_grid->x_dim, ny = gv->fluid_grid->y_dim, nz = gv->fluid_grid->z_dim;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        Fluidnode* n = ref_node(gv, x, y, z);
        long i = ((long)z * ny + y) * nx + x;
        n->rho = rho[i]; n->vel_x = ux[i]; n->vel_y = uy[i]; n->vel_z = uz[i];
      }
}

void ref_get_force(void* h, double* fx, double* fy, double* fz) {
  GV gv = ((ref_case*)h)->gv;
  int nx = gv->fluid_grid->x_dim, ny = gv->fluid_grid->y_dim, nz = gv->fluid_grid->z_dim;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        Fluidnode* n = ref_node(gv, x, y, z);
        long i = ((long)z * ny + y) * nx + x;
        fx[i] = n->elastic_force_x; fy[i] = n->elastic_force_y; fz[i] = n->elastic_force_z;
      }
}

void ref_set_force(void* h, const double* fx, const double* fy, const double* fz) {
  GV gv = ((ref_case*)h)->gv;
  int nx = gv->fluid_grid->x_dim, ny = gv->fluid_grid->y_dim, nz = gv->fluid_grid->z_dim;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        Fluidnode* n = ref_node(gv, x, y, z);
        long i = ((long)z * ny + y) * nx + x;
        n->elastic_force_x = fx[i]; n->elastic_force_y = fy[i]; n->elastic_force_z = fz[i];
      }
}

/* which: 0 = df1, 1 = df2, 2 = dfeq.  Layout [q][z][y][x]. */
void ref_get_df(void* h, int which, double* out) {
  GV gv = ((ref_case*)h)->gv;
  int nx = gv->fluid_grid->x_dim, ny = gv->fluid_grid->y_dim, nz = gv->fluid_grid->z_dim;
  long N = (long)nx * ny * nz;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        Fluidnode* n = ref_node(gv, x, y, z);
        long i = ((long)z * ny + y) * nx + x;
        const double* src = which == 0 ? n->df1 : which == 1 ? n->df2 : n->dfeq;
        for (int q = 0; q < 19; ++q) out[q * N + i] = src[q];
      }
}

void ref_set_df(void* h, int which, const double* in) {
  GV gv = ((ref_case*)h)->gv;
  int nx = gv->fluid_grid->x_dim, ny = gv->fluid_grid->y_dim, nz = gv->fluid_grid->z_dim;
  long N = (long)nx * ny * nz;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        Fluidnode* n = ref_node(gv, x, y, z);
        long i = ((long)z * ny + y) * nx + x;
        double* dst = which == 0 ? n->df1 : which == 1 ? n->df2 : n->dfeq;
        for (int q = 0; q < 19; ++q) dst[q] = in[q * N + i];
      }
}

/* Inlet (0) / outlet (1) planes, layout [q][y][z] like the reference's
 * inlet->nodes[y*dim_z + z].df_inout[k][q] (lbm_ib.c:1639-1664). */
void ref_get_inout(void* h, int which, double* out) {
  GV gv = ((ref_case*)h)->gv;
  int ny = gv->fluid_grid->y_dim, nz = gv->fluid_grid->z_dim;
  Fluidnode* plane = which == 0 ? gv->fluid_grid->inlet->nodes : gv->fluid_grid->outlet->nodes;
  for (int i = 0; i < ny * nz; ++i)
    for (int q = 0; q < 19; ++q) out[(long)q * ny * nz + i] = plane[i].df_inout[which][q];
}

/* Sheet 0 node records, 12 doubles per node in Fibernode order
 * {x, y, z, bend xyz, stretch xyz, elastic xyz}, row-major (row, col). */
void ref_get_sheet(void* h, double* out) {
  GV gv = ((ref_case*)h)->gv;
  Fibersheet* sh = &gv->fiber_shape->sheets[0];
  for (int r = 0; r < sh->num_rows; ++r)
    for (int c = 0; c < sh->num_cols; ++c)
      memcpy(out + ((long)r * sh->num_cols + c) * 12, &sh->fibers[r].nodes[c], 12 * sizeof(double));
}

void ref_set_sheet(void* h, const double* in) {
  GV gv = ((ref_case*)h)->gv;
  Fibersheet* sh = &gv->fiber_shape->sheets[0];
  for (int r = 0; r < sh->num_rows; ++r)
    for (int c = 0; c < sh->num_cols; ++c)
      memcpy(&sh->fibers[r].nodes[c], in + ((long)r * sh->num_cols + c) * 12, 12 * sizeof(double));
}

void ref_free(void* h) {
  ref_case* rc = (ref_case*)h;
  GV gv = rc->gv;
  int total_cubes = gv->num_cubes_x * gv->num_cubes_y * gv->num_cubes_z;
  for (int c = 0; c < total_cubes; ++c) free(gv->fluid_grid->sub_fluid_grid[c].nodes);
  free(gv->fluid_grid->sub_fluid_grid);
  free(gv->fluid_grid->inlet->nodes); free(gv->fluid_grid->outlet->nodes);
  free(gv->fluid_grid->inlet); free(gv->fluid_grid->outlet);
  free(gv->fluid_grid);
  Fibersheet* sh = &gv->fiber_shape->sheets[0];
  for (int r = 0; r < sh->num_rows; ++r) free(sh->fibers[r].nodes);
  free(sh->fibers);
  free(gv->fiber_shape->sheets); free(gv->fiber_shape);
  pthread_mutex_destroy(&gv->lock_Fluid[0]);
  free(gv->lock_Fluid);
  pthread_barrier_destroy(&gv->barr);
  free(gv);
  free(rc);
}
