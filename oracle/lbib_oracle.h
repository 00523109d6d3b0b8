/*
 * CPU restatement of the reference LBM-IB time step -- TEST INFRASTRUCTURE.
 *
 * This is the oracle: the tests, the smoke check and bench.py's CPU-baseline
 * leg use it to check (never to produce) the CUDA path's results.  The
 * product library never links it.
 *
 * Layouts: scalar fields are x-fastest, idx = (z*ny + y)*nx + x; populations
 * are [q][idx]; inlet/outlet planes are [q][y*nz + z]; a fiber node record is
 * the reference's Fibernode (12 doubles: x y z, bend xyz, stretch xyz,
 * elastic xyz), row-major over (row, col).
 */
#ifndef LBIB_ORACLE_H
#define LBIB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Reference behaviours kept for parity (all set by default).  Clearing a bit
 * selects the corrected behaviour instead. */
#define ORC_COMPAT_BEND_X_BUG     1  /* cube_pthread/lbm_ib.c:1032-1035 uses x[j] for x[j-2] */
#define ORC_COMPAT_YWALL_CUBES_X  2  /* lbm_ib.c:2378,2414 clip z against num_cubes_x */
#define ORC_COMPAT_INOUT_PTHREAD  4  /* lbm_ib.c:2800-2882 loop BK < num_cubes_x, serial */
#define ORC_COMPAT_ALL            7

/* Options with no reference counterpart (the workload definitions ask for
 * them; the reference has none of them, so their parity is unpinned beyond
 * this restatement).  They ride in the same word as the compat bits. */
#define ORC_OPT_PERIODIC_Z   0x100  /* z periodic over I, walls only at y            */
#define ORC_OPT_REST_START   0x200  /* interior starts at u = 0; inflow on the planes */
#define ORC_OPT_PIN_ROW0     0x400  /* row 0 of every sheet does not move            */

typedef struct orc_state orc_state;

orc_state* orc_create(int nx, int ny, int nz, int cube_size, int nsheets,
                      const int* rows, const int* cols,
                      const double* width, const double* height,
                      const double* x0, const double* y0, const double* z0,
                      double tau, double u_l, double Ks_l, double Kb_l,
                      int compat);
void orc_free(orc_state* s);

/* Stages of one step, in do_thread order (lbm_ib.c:3124-3563).  Those that
 * can fail return 0 or a negative error (a stencil leaving the grid). */
void orc_bending(orc_state* s);
void orc_stretching(orc_state* s);
void orc_elastic(orc_state* s);
int  orc_spread(orc_state* s);
void orc_collide(orc_state* s);
void orc_stream(orc_state* s);
void orc_bounceback(orc_state* s);
void orc_moments(orc_state* s);
int  orc_move(orc_state* s);
void orc_copy_inout(orc_state* s);
void orc_replace(orc_state* s);
int  orc_step(orc_state* s);           /* all of the above, then time += dt */
int  orc_run(orc_state* s, int nsteps);

int  orc_time(const orc_state* s);
void orc_get_moments(const orc_state* s, double* rho, double* ux, double* uy, double* uz);
void orc_set_moments(orc_state* s, const double* rho, const double* ux, const double* uy, const double* uz);
void orc_get_force(const orc_state* s, double* fx, double* fy, double* fz);
void orc_set_force(orc_state* s, const double* fx, const double* fy, const double* fz);
void orc_get_df(const orc_state* s, int which, double* out);      /* 0 df1, 1 df2, 2 dfeq */
void orc_set_df(orc_state* s, int which, const double* in);
void orc_get_inout(const orc_state* s, int which, double* out);   /* 0 inlet, 1 outlet */
void orc_get_sheet(const orc_state* s, int sheet, double* out);   /* rows*cols*12 */
void orc_set_sheet(orc_state* s, int sheet, const double* in);
void orc_set_threads(int n);
double orc_cos(double x);              /* the delta kernel's cosine of this library variant */
long orc_cos_2phase(const double* x, long n, double* out, unsigned char* slow);  /* the CUDA path's two-phase cosine */

#ifdef __cplusplus
}
#endif
#endif
