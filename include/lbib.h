/*
 * lbib.h -- drop-in C ABI for the LBM-IB time-step loop of
 * IUPU-HPC/distributed-LB-IB, executed on one NVIDIA B200 (sm_100a).
 *
 * A host program written against the reference (mpi/main.c, or
 * cube_pthread/lbm_ib.c:main) keeps its types and call sequence:
 *
 *     init_gv_constant(gv);                      mpi/init_gv.c:49
 *     gen_fluid_grid(gv->fluid_grid, cs, 0, gv); mpi/gen_fluid_grid.c:25
 *     gen_fiber_sheet(&gv->fiber_shape->sheets[k]);   mpi/gen_fiber_sheet.c:25
 *     init_gv(gv);                               mpi/init_gv.c:117
 *     init_eqlbrmdistrfuncDF0(gv); init_df1(gv); init_df_inout(gv);
 *     do_thread(lv);                             mpi/do_thread.c:36
 *
 * and links liblbib.so instead of the reference's kernel objects.  The
 * populations, forces and sheet state then live in GPU memory; the host-side
 * Fibernode arrays are refreshed by lbib_sync_to_host() and by the dump
 * writers.  Every function keeps the reference's argument meaning.  Where the
 * reference printed and called exit(1) (a fiber stencil leaving the grid,
 * cube_pthread/lbm_ib.c:1458-1466), this library records a sticky error code
 * (lbib_last_error) and the step loop stops.
 *
 * Numerics: FP64 throughout, the same floating-point operations in the same
 * order as the reference (no contraction), so that results match the
 * reference bit for bit except through the cosine of the delta kernel, which
 * is correctly rounded here (the host C library's cosine is not).
 */
#ifndef LBIB_H
#define LBIB_H

#include <pthread.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- data model: field names of mpi/do_thread.h:96-239 ------------------ */

/* mpi/do_thread.h:96-101, cube_pthread/lbm_ib.c:54-59 */
typedef struct fiber_node_t {
  double x, y, z;
  double bend_force_x, bend_force_y, bend_force_z;
  double stretch_force_x, stretch_force_y, stretch_force_z;
  double elastic_force_x, elastic_force_y, elastic_force_z;
} Fibernode;

/* mpi/do_thread.h:104-107 */
typedef struct fiber_t {
  Fibernode* nodes;
  int num_nodes;
} Fiber;

/* mpi/do_thread.h:110-119: width along z, height along y */
typedef struct fiber_sheet_t {
  Fiber* fibers;
  double width, height;
  int num_cols, num_rows;
  double x_orig, y_orig, z_orig;
} Fibersheet;

/* mpi/do_thread.h:122-125 */
typedef struct fiber_shape_t {
  Fibersheet* sheets;
  int num_sheets;
} Fibershape;

/* mpi/do_thread.h:131-139: the reference's 824-byte AoS cell.  Only the
 * dump writers materialise it (for the cells they write); the solver keeps
 * structure-of-arrays populations in GPU memory. */
typedef struct fluid_node_t {
  double vel_x, vel_y, vel_z;
  double rho, pressure;
  double df1[19];
  double df2[19];
  double dfeq[19];
  double df_inout[2][19];
  double elastic_force_x, elastic_force_y, elastic_force_z;
} Fluidnode;

/* mpi/do_thread.h:142-145 */
typedef struct fluid_surface_t {
  Fluidnode* nodes;
} Fluidsurface;

/* mpi/do_thread.h:150-161 */
typedef struct sub_fluid_grid_t {
  int sub_coordx_start, sub_coordx_end;
  int sub_coordy_start, sub_coordy_end;
  int sub_coordz_start, sub_coordz_end;
  Fluidnode* nodes;
  bool isboundary;
  int grid_dim_x;
  int grid_dim_y;
  int grid_dim_z;
} Sub_Fluidgrid;

/* mpi/do_thread.h:166-175.  x is the flow direction (inlet at x = 1, 2,
 * outlet at x = x_dim-3, x_dim-2).  inlet/outlet/sub_fluid_grid stay NULL:
 * the populations live on the GPU. */
typedef struct fluid_grid_t {
  int x_dim;
  int y_dim;
  int z_dim;
  int num_cubes_x, num_cubes_y, num_cubes_z;
  Fluidsurface* inlet;
  Fluidsurface* outlet;
  Sub_Fluidgrid* sub_fluid_grid;
} Fluidgrid;

struct lbib_device;  /* GPU-resident state, owned by this library */

/* mpi/do_thread.h:178-239 minus the MPI message buffers, plus the pthread
 * variant's TIME_STOP/c/P/Q/R/total_threads/num_cubes_* fields
 * (cube_pthread/lbm_ib.c:126-159), plus three fields of this library. */
typedef struct gv_t {
  Fibershape* fiber_shape;
  Fluidgrid* fluid_grid;
  double tau, nu_l, u_l, rho_l, L_l, M_l, g_l, Ks_l, Kb_l, Kst_l;
  double Re, cs_l, Ma, Kn, Kshat, Ksthat, Kbhat, Mhat, Fr;
  int dt, time, timesteps, dump;
  int TIME_STOP;                   /* pthread name of the last step      */
  double c[19][3];                 /* lattice velocities (pthread GV)    */
  int ib, ie, jb, je, kb, ke;
  int tx, ty, tz;
  int threads_per_task;
  int P, Q, R, total_threads;
  int num_cubes_x, num_cubes_y, num_cubes_z;
  int cube_size;
  pthread_t* threads;
  pthread_mutex_t* lock_Fluid;
  pthread_barrier_t barr;
  int taskid;
  int num_fluid_tasks;
  /* ---- additions of this library ---- */
  struct lbib_device* dev;         /* NULL until gen_fluid_grid          */
  int lbib_compat;                 /* LBIB_COMPAT_* bits, see below      */
  int lbib_dump_mode;              /* LBIB_DUMP_* bits for do_thread     */
  int lbib_precision;              /* LBIB_PREC_* population storage     */
  int lbib_slab_lo, lbib_slab_hi;  /* x-slab held here; hi = 0: all      */
}* GV;

/* mpi/do_thread.h:242-245 */
typedef struct lv_t {
  int tid;
  GV gv;
}* LV;

/* Reference behaviours kept for parity; all are set by init_gv_constant.
 * Clearing a bit selects the corrected behaviour. */
#define LBIB_COMPAT_BEND_X_BUG    1  /* x[j] for x[j-2] at col = cols-2, cube_pthread/lbm_ib.c:1032-1035 */
#define LBIB_COMPAT_YWALL_CUBES_X 2  /* y-wall z range clipped with num_cubes_x, lbm_ib.c:2378,2414 */
#define LBIB_COMPAT_INOUT_PTHREAD 4  /* inlet/outlet copy loops BK < num_cubes_x, lbm_ib.c:2800-2882 */
#define LBIB_COMPAT_ALL           7

/* Population storage of the fluid step (no reference counterpart; the
 * reference stores FP64).  LBIB_PREC_F64 is the drop-in: results equal the
 * reference's to rounding.  The others trade accuracy for HBM traffic: they
 * store the deviation f_q - s_q from a fixed shift in FP32, FP16 or BF16
 * and do moments, equilibrium and collision on deviations in FP32 (FMA
 * contraction allowed).  The shift is the rest weights w_q, or, with
 * LBIB_PREC_SHIFT_FLOW or'ed in, the equilibrium of the initial state
 * (rho_l, u_l, 0, 0).  Forces, the moments handed to the sheets and the
 * sheets stay FP64. */
#define LBIB_PREC_F64        0
#define LBIB_PREC_F32        1
#define LBIB_PREC_F16        2
#define LBIB_PREC_BF16       3
#define LBIB_PREC_SHIFT_FLOW 16

/* What do_thread writes at time == 1 and every gv->dump steps. */
#define LBIB_DUMP_NONE      0
#define LBIB_DUMP_FIELDVIEW 1  /* FV_* files, cube_pthread/lbm_ib.c:3100-3112, 3519-3538 */
#define LBIB_DUMP_BINARY    2  /* Fiber%d_dump_step%d.bin, mpi/do_thread.c:335-352 */

/* Error codes returned by the int entry points and by lbib_last_error. */
#define LBIB_OK              0
#define LBIB_E_ARG          -1   /* bad size, NULL pointer, indivisible grid */
#define LBIB_E_CUDA         -2   /* a CUDA call failed                       */
#define LBIB_E_STENCIL      -3   /* a fiber stencil left the fluid grid      */
#define LBIB_E_STATE        -4   /* call out of order (no grid, no sheet)    */
#define LBIB_E_NOMEM        -5   /* device or host allocation failed         */
#define LBIB_E_CAPACITY     -6   /* more touched force tiles than allocated  */
#define LBIB_E_IO           -7   /* a dump file could not be written         */
#define LBIB_E_LIMIT        -8   /* a size above a fixed maximum             */

/* ---- set-up: mpi/init_gv.c, mpi/gen_*.c, mpi/init_*.c ----------------- */

/* mpi/init_gv.c:49-99: dt, time, cube counts, ib..ke and the reference's
 * hard-coded physics (Re 150, u_l 0.001, L 20, tau from nu, Kb_l, Ks_l).
 * Needs gv->fluid_grid->{x,y,z}_dim and gv->cube_size. */
void init_gv_constant(GV gv);

/* mpi/gen_fluid_grid.c:25-68: allocates the GPU state for the grid
 * described by fluid_grid (rho = rho_l, u = (u_l, 0, 0) everywhere).
 * taskid is accepted for signature compatibility; one GPU owns the grid. */
void gen_fluid_grid(Fluidgrid* fluid_grid, int cube_size, int taskid, GV gv);

/* mpi/gen_fiber_sheet.c:25-68: allocates sheet->fibers and places node
 * (row, col) at (x_orig, y_orig + row*height/(rows-1), z_orig + col*width/(cols-1)). */
void gen_fiber_sheet(Fibersheet* sheet);

/* mpi/init_gv.c:117-275: shifts every sheet by u_l*dt in x and uploads the
 * sheets to the GPU. */
void init_gv(GV gv);

/* mpi/init_eqlbrmdistrfuncDF0.c:41-120, mpi/init_df1.c:13-56,
 * mpi/init_df_inout.c:14-81: equilibrium populations, interior df1, and the
 * fixed inlet (x = ib) / outlet (x = x_dim-1) planes, all on the GPU. */
void init_eqlbrmdistrfuncDF0(GV gv);
void init_df1(GV gv);
void init_df_inout(GV gv);

/* ---- the step: mpi/do_thread.c:36-403, cube_pthread/lbm_ib.c:3087-3570 -- */

/* Runs steps while gv->time <= gv->timesteps (or TIME_STOP when timesteps
 * is 0), dumping per gv->lbib_dump_mode when time % dump == 0 (and at
 * time == 1 for FieldView, as the pthread code does).  Only tid 0 works;
 * other tids return at once, so a host that still spawns T threads stays
 * correct.  Returns NULL; check lbib_last_error(). */
void* do_thread(void* v);

/* The stages of one step, callable one by one in do_thread order.  On the
 * GPU the fluid part is one fused in-place kernel: compute_eqlbrmdistrfuncDF1
 * launches it (collision, streaming, bounce-back, inlet/outlet and the
 * df2->df1 copy together); stream_distrfunc, bounceback_rigidwalls and
 * copy_inout_to_df2 are then no-ops, and replace_old_DF closes the step.
 * Calling them out of order is undefined. */
void compute_bendingforce(LV lv);        /* mpi/compute_bendingforce.c:25      */
void compute_stretchingforce(LV lv);     /* mpi/compute_stretchingforce.c:25   */
void compute_elasticforce(LV lv);        /* mpi/compute_elasticforce.c:25      */
void fiber_SpreadForce(LV lv);           /* mpi/fiber_SpreadForce.c:64         */
void fluid_get_SpreadForce(LV lv);       /* mpi/fluid_get_SpreadForce.c:28     */
void get_influentialdomain_fluid_grid_and_SpreadForce(LV lv); /* lbm_ib.c:1323 */
void compute_eqlbrmdistrfuncDF1(LV lv);  /* mpi/compute_eqlbrmdistrfuncDF1.c:75 */
void stream_distrfunc(LV lv);            /* mpi/stream_distrfunc.c:232         */
void bounceback_rigidwalls(LV lv);       /* mpi/bounceback_rigidwalls.c:25     */
void compute_rho_and_u(LV lv);           /* mpi/compute_rho_and_u.c:27         */
void fluid_SpreadVelocity(LV lv);        /* mpi/fluid_SpreadVelocity.c:25      */
void fiber_get_SpreadVelocity(LV lv);    /* mpi/fiber_get_SpreadVelocity.c:47  */
void moveFiberSheet(LV lv);              /* cube_pthread/lbm_ib.c:2540         */
void copy_inout_to_df2(LV lv);           /* mpi/copy_inout_to_df2.c:13         */
void replace_old_DF(LV lv);              /* mpi/replace_old_DF.c:13            */
void periodicBC(LV lv);                  /* mpi/periodicBC.c:29, never called by
                                            the reference loop; a no-op here   */

/* ---- dumps: mpi/print_info.c, cube_pthread/lbm_ib.c:331-692 ------------ */
void save_fiber_sub_grid(GV gv, int start_y, int start_z, int end_y, int end_z, char fName[]);
void save_fiber_sub_grid_binary(GV gv, int start_y, int start_z, int end_y, int end_z, char fName[]);
void save_fluid_sub_grid(GV gv, int start_x, int start_y, int start_z,
                         int end_x, int end_y, int end_z, char fName[]);
void save_fluid_sub_grid_vel_use_fv(GV gv, int start_x, int start_y, int start_z,
                                    int end_x, int end_y, int end_z, char fName[]);
void save_fluid_sub_grid_cord_use_fv(GV gv, int start_x, int start_y, int start_z,
                                     int end_x, int end_y, int end_z, char fName[]);
void save_fiber_sub_grid_cord_ef_use_fv(GV gv, int start_y, int start_z, int end_y, int end_z,
                                        char grid_fname[], char elastic_force_fname[]);

/* ---- additions (no reference counterpart) ----------------------------- */

/* Overrides the physics that init_gv_constant hard-codes
 * (mpi/init_gv.c:74-97).  Call before init_gv / init_eqlbrmdistrfuncDF0:
 * it also resets the initial velocity to (u_l, 0, 0). */
int lbib_set_params(GV gv, double tau, double u_l, double Ks_l, double Kb_l);
/* The LBIB_COMPAT_* bits below, and the option bits LBIB_OPT_* (physics the
 * benchmark workloads describe and the reference does not have; their
 * parity is pinned to the CPU restatement only).  Call before init_gv;
 * lbib_case_create* take the same word as their compat argument:
 *   LBIB_OPT_PERIODIC_Z  z is periodic over the fluid interior (period
 *                        nz - 4) and only the y = 2, ny-3 walls bounce back;
 *                        the reference's periodicBC (mpi/periodicBC.c:29-134)
 *                        is never called by its step loop
 *   LBIB_OPT_REST_START  the cells x in [3, nx-4] start at u = 0 (f = f_eq
 *                        with rho = 1); the inlet/outlet planes and their
 *                        fixed tables keep the inflow (1, u_l), which then
 *                        drives the channel (the reference starts every cell
 *                        at (u_l, 0, 0), mpi/gen_fluid_grid.c:61-64)
 *   LBIB_OPT_PIN_ROW0    row 0 of every sheet stays where it is (the
 *                        reference's tethering loops are no-ops,
 *                        cube_pthread/lbm_ib.c:909-917) */
#define LBIB_OPT_PERIODIC_Z  0x100
#define LBIB_OPT_REST_START  0x200
#define LBIB_OPT_PIN_ROW0    0x400
int lbib_set_compat(GV gv, int flags);
/* Selects the population storage (LBIB_PREC_*); init_gv_constant sets F64.
 * Call before init_gv: when the grid's GPU state exists it is rebuilt in
 * the new precision (populations zeroed; run init_eqlbrmdistrfuncDF0,
 * init_df1 and init_df_inout after).  LBIB_E_STATE once sheets are
 * uploaded, LBIB_E_ARG for an unknown value. */
int lbib_set_precision(GV gv, int precision);
/* Kernel variants of the fluid step for the grid's precision (the
 * low-precision forms have several -- cells per thread, register budget,
 * prefetch -- FP64 has one), and choosing among them.  lbib_autotune times
 * every variant on `steps` fluid steps from the initial state, keeps the
 * fastest and restores the initial populations, so the run is unchanged;
 * call it after init_df1 / init_df_inout and before the first step.  It
 * returns the chosen variant (>= 0) or an error code; ms_per_variant[i]
 * (up to max_variants entries, may be NULL) gets each variant's mean ms per
 * step. */
int lbib_kernel_variants(GV gv);
int lbib_set_kernel_variant(GV gv, int variant);
int lbib_autotune(GV gv, int steps, double* ms_per_variant, int max_variants);
int lbib_last_error(void);
const char* lbib_error_string(int code);
void lbib_clear_error(void);
/* Copies sheet positions and forces back into gv->fiber_shape. */
int lbib_sync_to_host(GV gv);
/* Frees everything this library allocated for gv (GPU state, sheets,
 * fluid_grid planes); gv itself and the objects the caller made stay. */
void lbib_free(GV gv);

/* x-slab decomposition over several GPUs (no counterpart in the reference:
 * its pthread version shares one address space, its MPI version exchanges
 * whole cube faces).  Each GV holds the global columns [x_lo, x_hi) of the
 * grid (multiples of 4; FP64 storage) plus two ghost columns on each side,
 * and the whole sheet, whose forces, spread and move every slab computes
 * alike.  A step is three calls with two exchanges between them:
 *   par = lbib_slab_step_fluid(gv)  forces, spread, fused fluid step on this
 *                                   slab's cells; packs the face columns
 *                                   into send_lo / send_hi; returns the
 *                                   step's AA parity (0 or 1) or an error;
 *   exchange 1: send_lo -> left neighbour's recv_hi, send_hi -> right
 *               neighbour's recv_lo (5*ny*nz doubles each);
 *   lbib_slab_step_moments(gv)      unpacks recv_lo / recv_hi and computes
 *                                   the moment tiles of this slab's columns
 *                                   (-0.0 in the others);
 *   lbib_slab_moments(gv, &U, &n)   the moment tiles (n doubles on the
 *                                   device; waits for the stream) and the
 *                                   step's error code;
 *   exchange 2: U <- sum of U over all slabs (each value is owned by one
 *               slab and -0.0 elsewhere, so the sum keeps every bit);
 *   lbib_slab_step_move(gv)         moves the sheet; advances gv->time.
 * All device work goes on lbib_stream(gv); the exchanges must be ordered
 * after and before it.  With the slabs' results put together the run is
 * bit-identical to the whole grid on one GPU.  lbib_run refuses a slab
 * (LBIB_E_STATE), as do the restart files. */
int lbib_set_slab(GV gv, int x_lo, int x_hi);   /* like lbib_set_precision: before init_gv */
GV lbib_case_create_slab(int nx, int ny, int nz, int cube_size, int nsheets,
                         const int* rows, const int* cols,
                         const double* width, const double* height,
                         const double* x0, const double* y0, const double* z0,
                         double tau, double u_l, double Ks_l, double Kb_l, int compat,
                         int x_lo, int x_hi);
/* bufs[4] = device pointers send_lo, send_hi, recv_lo, recv_hi; *len = doubles each */
int lbib_slab_buffers(GV gv, double** bufs, long* len);
int lbib_slab_step_fluid(GV gv);
int lbib_slab_step_moments(GV gv);
int lbib_slab_moments(GV gv, double** U, long* n);
int lbib_slab_step_move(GV gv);
/* Direct exchange instead of the two buffer exchanges: each slab's kernels
 * write its face columns straight into its neighbours' populations, and its
 * moment tiles into every slab's tiles, through device pointers that reach
 * the other slabs' memory (peer access between GPUs of one process,
 * lbib_peer_access; or IPC mappings between processes, lbib_ipc_*).  Wire
 * once with lbib_slab_connect (each slab's lbib_slab_storage: populations,
 * their geometry, both moment-tile buffers; U0/U1 list all n <= 8 slabs in
 * order, this one included), then per step:
 *   lbib_slab_step_fluid_direct  -> barrier over all slabs ->
 *   lbib_slab_step_moments_direct -> barrier -> lbib_slab_check ->
 *   lbib_slab_step_move.
 * A barrier means: every slab's stream has finished (lbib_synchronize) and
 * every slab knows it; no kernel here waits on another slab. */
int lbib_slab_storage(GV gv, double** f, long* Ns, int* sx, int* gx0, double** U0, double** U1);
int lbib_slab_connect(GV gv, double* lo_f, long lo_Ns, int lo_sx, int lo_gx0, double* hi_f, long hi_Ns,
                      int hi_sx, int hi_gx0, int n, double* const* U0, double* const* U1);
int lbib_slab_step_fluid_direct(GV gv);
int lbib_slab_step_moments_direct(GV gv);
int lbib_slab_check(GV gv);        /* waits for the stream; the step's error code */
int lbib_peer_access(int device, int peer);
int lbib_ipc_handle(void* dev_ptr, void* handle);          /* handle: 64 bytes */
int lbib_ipc_open(const void* handle, void** dev_ptr);
int lbib_ipc_close(void* dev_ptr);

/* Restart files (no counterpart in the reference, which can only restart
 * from its initial state): lbib_save_restart writes everything the next
 * step reads -- populations in their storage type, inlet/outlet tables,
 * the previous step's force and moment tiles, the sheets, the step counters,
 * physics and gv->time -- so that lbib_load_restart into a GV set up with
 * the same grid, precision and sheet shapes continues the run bit for bit.
 * Errors: LBIB_E_IO (file), LBIB_E_ARG (a different grid, precision or
 * sheets), LBIB_E_STATE (no GPU state or sheets yet). */
int lbib_save_restart(GV gv, const char* path);
int lbib_load_restart(GV gv, const char* path);

/* Array access for tests, tools and bindings (x-fastest scalar fields,
 * idx = (z*y_dim + y)*x_dim + x; sheet records of 12 doubles in Fibernode
 * order, row-major).  All return LBIB_OK or an error code.
 * lbib_get_moments: when all four outputs are page-locked host memory
 * (cudaHostAlloc / cudaHostRegister), the moments kernel writes them over
 * the host link directly; pageable outputs are staged in a device buffer
 * allocated for the call.  Both give the same values. */
int lbib_get_moments(GV gv, double* rho, double* ux, double* uy, double* uz);
int lbib_get_force(GV gv, double* fx, double* fy, double* fz);
int lbib_get_df1(GV gv, double* out);            /* [19][N], cells of [2,n-3]^3 */
/* out[4] = mass and x, y, z momentum of the populations of [2,n-3]^3 as
 * the next step reads them, summed in FP64 in a fixed order (the same
 * value on every run). */
int lbib_conservation_sums(GV gv, double* out);
int lbib_get_sheet(GV gv, int sheet, double* out);
int lbib_set_sheet(GV gv, int sheet, const double* in);
int lbib_run(GV gv, int nsteps);                 /* do_thread for nsteps steps */
int lbib_device_count(void);                     /* CUDA devices visible (0 if none) */
int lbib_synchronize(GV gv);
void* lbib_stream(GV gv);                        /* the cudaStream_t used */
long lbib_kernel_launches(GV gv);                /* CUDA kernels launched so far */
/* Stage timing with CUDA events on the library's stream: between begin and
 * end every step records events around its five stages; end synchronises and
 * returns the summed milliseconds of [fiber forces, spread, fused fluid step,
 * tile moments, interpolate+move] and the number of steps timed. */
int lbib_profile_begin(GV gv);
int lbib_profile_end(GV gv, double* stage_ms, long* steps);

/* One-call set-up used by bindings: the sequence init_gv_constant,
 * gen_fluid_grid, gen_fiber_sheet (each sheet), init_gv, lbib_set_params,
 * init_eqlbrmdistrfuncDF0, init_df1, init_df_inout.  Returns a GV owned by
 * the library (free with lbib_case_free) or NULL (see lbib_last_error). */
GV lbib_case_create(int nx, int ny, int nz, int cube_size, int nsheets,
                    const int* rows, const int* cols,
                    const double* width, const double* height,
                    const double* x0, const double* y0, const double* z0,
                    double tau, double u_l, double Ks_l, double Kb_l, int compat);
/* lbib_case_create with a population storage precision (LBIB_PREC_*). */
GV lbib_case_create_prec(int nx, int ny, int nz, int cube_size, int nsheets,
                         const int* rows, const int* cols,
                         const double* width, const double* height,
                         const double* x0, const double* y0, const double* z0,
                         double tau, double u_l, double Ks_l, double Kb_l, int compat,
                         int precision);
void lbib_case_free(GV gv);
/* Calls one stage by number, in do_thread order: 0 bending, 1 stretching,
 * 2 elastic, 3 spread (fiber_SpreadForce + fluid_get_SpreadForce),
 * 4 compute_eqlbrmdistrfuncDF1, 5 stream, 6 bounce-back, 7 rho and u,
 * 8 interpolate and move, 9 inlet/outlet copy, 10 replace_old_DF. */
int lbib_stage(GV gv, int which);

/* ---- force spreading without allocation (no counterpart in the
 * reference) ------------------------------------------------------------
 *
 * For hosts that cannot allocate GPU memory while they run -- e.g. a host
 * that hands out buffers from its own fixed pool and forbids any cudaMalloc
 * after start-up, because allocation may synchronise the device or fail
 * under its memory cap.  The GV path allocates its tile lists, maps and
 * weights when a sheet is uploaded; this entry point allocates nothing.
 *
 * Computes the spread force F of fiber_SpreadForce + fluid_get_SpreadForce
 * (cube_pthread/lbm_ib.c:1323-1525) from `nodes`, num_nodes Fibernode
 * records (12 doubles each, all sheets concatenated in sheet, row, col
 * order; only x, y, z and the elastic force are read), into fx, fy, fz
 * (nx*ny*nz doubles each, x fastest), all device pointers owned by the
 * caller; the result equals the GV path's bit for bit.  Runs on `stream`
 * (a cudaStream_t, NULL for the default stream) and waits for it before
 * returning.  Returns LBIB_OK, LBIB_E_STENCIL (a stencil leaves the grid;
 * outputs zero), LBIB_E_LIMIT (num_nodes > LBIB_NOALLOC_MAX_NODES) or
 * LBIB_E_ARG / LBIB_E_CUDA.
 *
 * Its scratch (per 32-node chunk the stencil bounding box, the box of all
 * stencils and an error word) is one file-scope device array of ~192 KiB,
 * which every GPU that loads the library keeps until the process exits.
 * Every call looks up that array's device address in the current device's
 * context (the first call on a device loads the library's module there).
 * The call reads its error word back with a copy and synchronises `stream`
 * before it returns, so it must not be called while `stream` is being
 * captured into a CUDA graph.  It returns LBIB_E_CUDA without doing any work
 * if a CUDA launch error from earlier work is pending.  All calls share the
 * array: calls whose work overlaps on the GPU (other streams, other host
 * threads on the same device) race -- serialise them. */
#define LBIB_NOALLOC_MAX_NODES (1 << 18)
int lbib_spread_force_noalloc(const double* nodes, long num_nodes, int nx, int ny, int nz,
                              double* fx, double* fy, double* fz, void* stream);

/* ---- batches of independent problems (no counterpart in the reference,
 * which runs one problem per process) ------------------------------------
 *
 * Many problems of uneven size, each with its own lattice, physics and one
 * fiber sheet, advanced together: one launch per stage for the whole batch,
 * the step captured as a CUDA graph and replayed.  Each problem follows the
 * same rules and arithmetic as the GV path (an FP64 batch gives every
 * problem the bits it gets on its own); set-up mirrors init_gv_constant +
 * gen_fluid_grid + gen_fiber_sheet + init_gv + the three init_* calls with
 * the problem's tau, u_l, Ks_l, Kb_l.  A problem whose sheet leaves its grid
 * stops (lbib_batch_status reports LBIB_E_STENCIL and the step); the others
 * continue.  Sizes must be multiples of 4 (cube_size 4). */
typedef struct lbib_problem {
  int nx, ny, nz;                  /* lattice, x = flow direction            */
  double tau, u_l, Ks_l, Kb_l;
  int rows, cols;                  /* the sheet, as Fibersheet               */
  double width, height, x0, y0, z0;
  int pinned;                      /* 1: row 0 of the sheet does not move (a
                                      flap hinged at its leading edge; not in
                                      the reference, whose sheets are free) */
} lbib_problem;
typedef struct lbib_batch lbib_batch;

lbib_batch* lbib_batch_create(int n, const lbib_problem* problems, int precision, int compat);
int lbib_batch_last_error(void);                /* why lbib_batch_create failed */
void lbib_batch_free(lbib_batch* b);
int lbib_batch_run(lbib_batch* b, int nsteps);  /* asynchronous on the batch's stream */
int lbib_batch_synchronize(lbib_batch* b);
void* lbib_batch_stream(lbib_batch* b);
long lbib_batch_cells(lbib_batch* b);           /* lattice sites of all problems */
long lbib_batch_steps(lbib_batch* b);
long lbib_batch_kernel_launches(lbib_batch* b);
/* codes[k] = 0 or LBIB_E_STENCIL, failed_step[k] = the step it stopped at
 * (either may be NULL); returns the number of stopped problems. */
int lbib_batch_status(lbib_batch* b, int* codes, int* failed_step);
int lbib_batch_get_sheet(lbib_batch* b, int k, double* out);      /* rows*cols*12 */
int lbib_batch_get_moments(lbib_batch* b, int k, double* rho, double* ux, double* uy, double* uz);
int lbib_batch_get_df1(lbib_batch* b, int k, double* out);
/* Fluid word-kernel variants, set for one problem (k >= 0) or all (k = -1)
 * before the first step, or chosen per size class by timing them;
 * lbib_batch_autotune restores the initial state and returns the number of
 * classes (class_of[k], ms[class * variants + v] when non-NULL). */
int lbib_batch_variants(lbib_batch* b);
int lbib_batch_set_variant(lbib_batch* b, int k, int variant);
int lbib_batch_autotune(lbib_batch* b, int steps, double* ms, int max_ms, int* class_of);

/* ---- a small MLP trained on the GPU: the sweep surrogate (no counterpart
 * in the reference) ------------------------------------------------------
 *
 * widths[0..n_layers]: input, hidden..., output; GELU after every layer but
 * the last; BF16 weights and activations with FP32 accumulation on the
 * tensor cores; FP32 master weights; mean-squared-error loss; Adam (beta1
 * 0.9, beta2 0.999, eps 1e-8).  Parameters, in order: per layer W
 * [out][in] row-major, then b [out].  X, T, Y of forward/train/gradient are
 * device pointers to row-major FP32 [batch][width] arrays; grad and loss of
 * lbib_mlp_gradient are host memory; the work runs on the MLP's stream.
 * Returns NULL / error codes as above. */
typedef struct lbib_mlp lbib_mlp;
lbib_mlp* lbib_mlp_create(int n_layers, const int* widths, int max_batch, unsigned long long seed);
void lbib_mlp_free(lbib_mlp* n);
long lbib_mlp_param_count(lbib_mlp* n);
void* lbib_mlp_stream(lbib_mlp* n);
/* Run on the caller's CUDA stream (NULL: the CUDA default stream); the MLP
 * starts on a stream of its own.  Inputs written by the caller on another
 * stream must be ready before the MLP reads them. */
int lbib_mlp_set_stream(lbib_mlp* n, void* stream);
int lbib_mlp_get_params(lbib_mlp* n, float* out);
int lbib_mlp_set_params(lbib_mlp* n, const float* in);
int lbib_mlp_forward(lbib_mlp* n, const float* X, int batch, float* Y);
int lbib_mlp_gradient(lbib_mlp* n, const float* X, const float* T, int batch, float* grad, float* loss);
int lbib_mlp_train_step(lbib_mlp* n, const float* X, const float* T, int batch, float lr, float* loss);
int lbib_mlp_synchronize(lbib_mlp* n);

#ifdef __cplusplus
}
#endif
#endif
