/*
 * CPU restatement of the reference LBM-IB step (IUPU-HPC/distributed-LB-IB,
 * cube_pthread/lbm_ib.c run serially) -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, and only as the checker.  The CUDA product path never calls
 * it.  It is pinned bit-for-bit against the reference itself (oracle/_ref,
 * built from the reference sources by oracle/Makefile) and against the
 * committed fixtures in tests/golden/.
 *
 * Every stage keeps the reference's floating-point expression order (it is
 * compiled with -ffp-contract=off) so that results are bit-identical to the
 * reference's serial run; each function cites the reference code it restates.
 * The layout is structure-of-arrays, not the reference's cube-tiled AoS: the
 * cube tiling only decides the iteration order, and no stage here depends on
 * that order except the force spread, whose per-cell summation order (sheet,
 * row, col) is kept.
 */
#include "lbib_oracle.h"

#include <math.h>

/* The delta kernel's cosine.  The default is the C library's cos, as the
 * reference calls it (glibc's is not correctly rounded: ~0.1% of arguments
 * in (-pi, pi] come out 1 ulp off).  Built with -DORC_CR_COS the oracle uses
 * the correctly rounded double-double cosine that the CUDA path uses, so the
 * two can be compared bit for bit; that cosine is itself checked against a
 * high-precision evaluation by tests/test_cos.py. */
#ifdef ORC_CR_COS
#include "lbib_cos.h"
#define ORC_COS(x) lbib_cos(x)
#else
#define ORC_COS(x) cos(x)
#endif
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* PI as truncated in the reference (cube_pthread/lbm_ib.c:33). */
#define ORC_PI 3.14159265358979

typedef struct {
  int rows, cols;
  double width, height, x0, y0, z0;
  double* node;  /* rows*cols*12: x y z, bend xyz, stretch xyz, elastic xyz */
} orc_sheet;

struct orc_state {
  int nx, ny, nz, cs;
  int ncx, ncy, ncz;
  long N;
  int compat;
  double tau, u_l, rho_l, Ks_l, Kb_l, g_l, cs_l;
  int dt, time;
  double c[19][3];
  double *df1, *df2, *dfeq;
  double *rho, *ux, *uy, *uz;
  double *fx, *fy, *fz;
  double *inlet, *outlet;
  int nsheets;
  orc_sheet* sheets;
};

/* Lattice velocities, cube_pthread/lbm_ib.c:777-833 (= mpi/init_gv.c:25-35). */
static const double ORC_C[19][3] = {
  {0, 0, 0},
  {1, 0, 0}, {-1, 0, 0}, {0, 0, 1}, {0, 0, -1}, {0, -1, 0}, {0, 1, 0},
  {1, 0, 1}, {-1, 0, -1}, {1, 0, -1}, {-1, 0, 1}, {0, -1, 1}, {0, 1, -1},
  {0, 1, 1}, {0, -1, -1}, {1, -1, 0}, {-1, 1, 0}, {1, 1, 0}, {-1, -1, 0}};

static inline long IDX(const orc_state* s, int x, int y, int z) {
  return ((long)z * s->ny + y) * s->nx + x;
}

static inline double* NODE(orc_sheet* sh, int r, int c) {
  return sh->node + ((long)r * sh->cols + c) * 12;
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* Equilibrium at one cell and direction, as written in
 * cube_pthread/lbm_ib.c:1548-1585 and :1727-1802 (the same expression is used
 * at set-up and in the collision). */
static inline double orc_feq(const orc_state* s, int q, double rho, double vx, double vy, double vz) {
  const double* c = s->c[q];
  double usq = vx * vx + vy * vy + vz * vz;
  if (q == 0) return 1.0 / 3.0 * rho * (1.0 - 1.5 * usq);
  double cu = c[0] * vx + c[1] * vy + c[2] * vz;
  double w = (q <= 6) ? 1.0 / 18.0 : 1.0 / 36.0;
  return w * rho * (1.0 + 3.0 * cu + 4.5 * (cu * cu) - 1.5 * usq);
}

/* Set-up: gen_fiber_shape (lbm_ib.c:866-921), gen_fluid_grid (:924-958),
 * init_gv (:705-863) with tau/u_l/Ks_l/Kb_l given instead of hard-coded,
 * init_eqlbrmdistrfuncDF0 (:1528-1607), init_df1 (:2725-2767),
 * init_df_inout (:1610-1670). */
orc_state* orc_create(int nx, int ny, int nz, int cube_size, int nsheets,
                      const int* rows, const int* cols,
                      const double* width, const double* height,
                      const double* x0, const double* y0, const double* z0,
                      double tau, double u_l, double Ks_l, double Kb_l,
                      int compat) {
  if (cube_size < 4 || nx % cube_size || ny % cube_size || nz % cube_size || nsheets < 1) return NULL;
  orc_state* s = (orc_state*)calloc(1, sizeof(*s));
  s->nx = nx; s->ny = ny; s->nz = nz; s->cs = cube_size;
  s->ncx = nx / cube_size; s->ncy = ny / cube_size; s->ncz = nz / cube_size;
  s->N = (long)nx * ny * nz;
  s->compat = compat;
  s->tau = tau; s->u_l = u_l; s->rho_l = 1.0; s->Ks_l = Ks_l; s->Kb_l = Kb_l;
  s->g_l = 0.0;
  s->cs_l = 1.0 / (sqrt(3));
  s->dt = 1; s->time = 1;
  memcpy(s->c, ORC_C, sizeof(ORC_C));
  long N = s->N;
  s->df1 = (double*)calloc(19 * N, sizeof(double));
  s->df2 = (double*)calloc(19 * N, sizeof(double));
  s->dfeq = (double*)calloc(19 * N, sizeof(double));
  s->rho = (double*)calloc(N, sizeof(double));
  s->ux = (double*)calloc(N, sizeof(double));
  s->uy = (double*)calloc(N, sizeof(double));
  s->uz = (double*)calloc(N, sizeof(double));
  s->fx = (double*)calloc(N, sizeof(double));
  s->fy = (double*)calloc(N, sizeof(double));
  s->fz = (double*)calloc(N, sizeof(double));
  s->inlet = (double*)calloc(19 * (long)ny * nz, sizeof(double));
  s->outlet = (double*)calloc(19 * (long)ny * nz, sizeof(double));

  s->nsheets = nsheets;
  s->sheets = (orc_sheet*)calloc(nsheets, sizeof(orc_sheet));
  for (int k = 0; k < nsheets; ++k) {
    orc_sheet* sh = &s->sheets[k];
    sh->rows = rows[k]; sh->cols = cols[k];
    sh->width = width[k]; sh->height = height[k];
    sh->x0 = x0[k]; sh->y0 = y0[k]; sh->z0 = z0[k];
    sh->node = (double*)calloc((long)sh->rows * sh->cols * 12, sizeof(double));
    double zdist = sh->width / (sh->cols - 1);
    double ydist = sh->height / (sh->rows - 1);
    for (int r = 0; r < sh->rows; ++r)
      for (int c = 0; c < sh->cols; ++c) {
        double* n = NODE(sh, r, c);
        n[0] = sh->x0;
        n[1] = ydist * r + sh->y0;
        n[2] = zdist * c + sh->z0;
        n[0] += s->u_l * s->dt;  /* init_gv's one-step shift, lbm_ib.c:857-862 */
      }
  }

  for (long i = 0; i < N; ++i) {
    s->rho[i] = s->rho_l; s->ux[i] = s->u_l; s->uy[i] = 0.0; s->uz[i] = 0.0;
  }
  /* rest start: the cells whose moments the step updates, x in [3, nx-4],
     start at u = 0; the plane cells x = 2, nx-3 (whose rho, u the reference
     never recomputes) and the cells the inlet/outlet tables are taken from
     keep the inflow (1, u_l), so the channel is driven from the planes */
  if (compat & ORC_OPT_REST_START)
    for (long i = 0; i < N; ++i) {
      const int x = (int)(i % nx);
      if (x >= 3 && x <= nx - 4) s->ux[i] = 0.0;
    }
  for (long i = 0; i < N; ++i)
    for (int q = 0; q < 19; ++q)
      s->dfeq[q * N + i] = orc_feq(s, q, s->rho[i], s->ux[i], s->uy[i], s->uz[i]);
  for (int z = 2; z <= nz - 3; ++z)
    for (int y = 2; y <= ny - 3; ++y)
      for (int x = 2; x <= nx - 3; ++x) {
        long i = IDX(s, x, y, z);
        for (int q = 0; q < 19; ++q) s->df1[q * N + i] = s->dfeq[q * N + i];
      }
  long P = (long)ny * nz;
  for (int y = 0; y < ny; ++y)
    for (int z = 0; z < nz; ++z) {
      long in = IDX(s, 2, y, z), out = IDX(s, nx - 1, y, z);
      for (int q = 0; q < 19; ++q) {
        s->inlet[q * P + (long)y * nz + z] = s->dfeq[q * N + in];
        s->outlet[q * P + (long)y * nz + z] = s->dfeq[q * N + out];
      }
    }
  return s;
}

void orc_free(orc_state* s) {
  if (!s) return;
  free(s->df1); free(s->df2); free(s->dfeq);
  free(s->rho); free(s->ux); free(s->uy); free(s->uz);
  free(s->fx); free(s->fy); free(s->fz);
  free(s->inlet); free(s->outlet);
  for (int k = 0; k < s->nsheets; ++k) free(s->sheets[k].node);
  free(s->sheets);
  free(s);
}

/* compute_bendingforce, cube_pthread/lbm_ib.c:961-1152 (mpi/compute_bendingforce.c:25-225).
 * Row pass assigns, column pass accumulates; Kb_l/ds2^3 in both passes as in
 * the pthread code (:996, :1062).  The x component at col = cols-2 uses
 * x[j] where x[j-2] is meant (:1032-1035) unless the compat bit is cleared. */
void orc_bending(orc_state* s) {
  for (int k = 0; k < s->nsheets; ++k) {
    orc_sheet* sh = &s->sheets[k];
    int R = sh->rows, C = sh->cols;
    double ds2 = sh->height / (R - 1);
    double bc = s->Kb_l / pow(ds2, 3);
    int bug = (s->compat & ORC_COMPAT_BEND_X_BUG) != 0;
    for (int i = 0; i < R; ++i) {
      double* n0 = NODE(sh, i, 0);
      double* n1 = NODE(sh, i, 1);
      double* n2 = NODE(sh, i, 2);
      double* n3 = NODE(sh, i, 3);
      for (int d = 0; d < 3; ++d) n0[3 + d] = bc * (-n2[d] + 2 * n1[d] - n0[d]);
      for (int d = 0; d < 3; ++d) n1[3 + d] = bc * (-n3[d] + 4 * n2[d] - 5 * n1[d] + 2 * n0[d]);
      for (int j = 2; j < C - 2; ++j) {
        double* a = NODE(sh, i, j - 2);
        double* b = NODE(sh, i, j - 1);
        double* m = NODE(sh, i, j);
        double* p = NODE(sh, i, j + 1);
        double* q = NODE(sh, i, j + 2);
        for (int d = 0; d < 3; ++d)
          m[3 + d] = bc * (-q[d] + 4.0 * p[d] - 6.0 * m[d] + 4.0 * b[d] - a[d]);
      }
      {
        int j = C - 2;
        double* a = NODE(sh, i, j - 2);
        double* b = NODE(sh, i, j - 1);
        double* m = NODE(sh, i, j);
        double* p = NODE(sh, i, j + 1);
        m[3] = bc * (2 * p[0] - 5 * m[0] + 4 * b[0] - (bug ? m[0] : a[0]));
        for (int d = 1; d < 3; ++d) m[3 + d] = bc * (2 * p[d] - 5 * m[d] + 4 * b[d] - a[d]);
      }
      {
        int j = C - 1;
        double* a = NODE(sh, i, j - 2);
        double* b = NODE(sh, i, j - 1);
        double* m = NODE(sh, i, j);
        for (int d = 0; d < 3; ++d) m[3 + d] = bc * (-m[d] + 2 * b[d] - a[d]);
      }
    }
    for (int j = 0; j < C; ++j) {
      double* f0 = NODE(sh, 0, j);
      double* f1 = NODE(sh, 1, j);
      double* f2 = NODE(sh, 2, j);
      double* f3 = NODE(sh, 3, j);
      for (int d = 0; d < 3; ++d) f0[3 + d] += bc * (-f2[d] + 2 * (f1[d]) - (f0[d]));
      for (int d = 0; d < 3; ++d) f1[3 + d] += bc * (-f3[d] + 4 * (f2[d]) - 5 * (f1[d]) + 2 * (f0[d]));
      for (int i = 2; i < R - 2; ++i) {
        double* a = NODE(sh, i - 2, j);
        double* b = NODE(sh, i - 1, j);
        double* m = NODE(sh, i, j);
        double* p = NODE(sh, i + 1, j);
        double* q = NODE(sh, i + 2, j);
        for (int d = 0; d < 3; ++d)
          m[3 + d] += bc * (-q[d] + 4.0 * (p[d]) - 6.0 * (m[d]) + 4.0 * (b[d]) - (a[d]));
      }
      {
        int i = R - 2;
        double* a = NODE(sh, i - 2, j);
        double* b = NODE(sh, i - 1, j);
        double* m = NODE(sh, i, j);
        double* p = NODE(sh, i + 1, j);
        for (int d = 0; d < 3; ++d) m[3 + d] += bc * (2 * p[d] - 5 * (m[d]) + 4 * (b[d]) - (a[d]));
      }
      {
        int i = R - 1;
        double* a = NODE(sh, i - 2, j);
        double* b = NODE(sh, i - 1, j);
        double* m = NODE(sh, i, j);
        for (int d = 0; d < 3; ++d) m[3 + d] += bc * (-(m[d]) + 2 * (b[d]) - (a[d]));
      }
    }
  }
}

/* compute_stretchingforce, cube_pthread/lbm_ib.c:1154-1282
 * (mpi/compute_stretchingforce.c:25-153).  The end nodes use the tangent
 * pointing from the neighbour at the last node (:1209-1211, :1264-1266),
 * i.e. with the opposite sign of the first node's; kept as written. */
void orc_stretching(orc_state* s) {
  for (int k = 0; k < s->nsheets; ++k) {
    orc_sheet* sh = &s->sheets[k];
    int R = sh->rows, C = sh->cols;
    double ds1 = sh->width / (C - 1);
    double ds2 = sh->height / (R - 1);
    double sc = s->Ks_l / (ds1 * ds1);
    for (int i = 0; i < R; ++i) {
      for (int j = 1; j < C - 1; ++j) {
        double* m = NODE(sh, i, j);
        double* p = NODE(sh, i, j + 1);
        double* b = NODE(sh, i, j - 1);
        double tr[3] = {p[0] - m[0], p[1] - m[1], p[2] - m[2]};
        double tl[3] = {b[0] - m[0], b[1] - m[1], b[2] - m[2]};
        double dr = sqrt(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]);
        double dl = sqrt(tl[0] * tl[0] + tl[1] * tl[1] + tl[2] * tl[2]);
        for (int d = 0; d < 3; ++d)
          m[6 + d] = sc * ((dr - ds1) * (tr[d] / dr) + (dl - ds1) * (tl[d] / dl));
      }
      {
        double* m = NODE(sh, i, 0);
        double* p = NODE(sh, i, 1);
        double tr[3] = {p[0] - m[0], p[1] - m[1], p[2] - m[2]};
        double dr = sqrt(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]);
        for (int d = 0; d < 3; ++d) m[6 + d] = sc * ((dr - ds1) * (tr[d] / dr));
      }
      {
        double* m = NODE(sh, i, C - 1);
        double* b = NODE(sh, i, C - 2);
        double tl[3] = {m[0] - b[0], m[1] - b[1], m[2] - b[2]};
        double dl = sqrt(tl[0] * tl[0] + tl[1] * tl[1] + tl[2] * tl[2]);
        for (int d = 0; d < 3; ++d) m[6 + d] = sc * ((dl - ds1) * (tl[d] / dl));
      }
    }
    double sc2 = s->Ks_l / (ds2 * ds2);
    for (int j = 0; j < C; ++j) {
      for (int i = 1; i < R - 1; ++i) {
        double* m = NODE(sh, i, j);
        double* p = NODE(sh, i + 1, j);
        double* b = NODE(sh, i - 1, j);
        double tt[3] = {p[0] - m[0], p[1] - m[1], p[2] - m[2]};
        double tb[3] = {b[0] - m[0], b[1] - m[1], b[2] - m[2]};
        double dt = sqrt(tt[0] * tt[0] + tt[1] * tt[1] + tt[2] * tt[2]);
        double db = sqrt(tb[0] * tb[0] + tb[1] * tb[1] + tb[2] * tb[2]);
        for (int d = 0; d < 3; ++d)
          m[6 + d] += sc2 * ((dt - ds2) * (tt[d] / dt) + (db - ds2) * (tb[d] / db));
      }
      {
        double* m = NODE(sh, 0, j);
        double* p = NODE(sh, 1, j);
        double tt[3] = {p[0] - m[0], p[1] - m[1], p[2] - m[2]};
        double dt = sqrt(tt[0] * tt[0] + tt[1] * tt[1] + tt[2] * tt[2]);
        for (int d = 0; d < 3; ++d) m[6 + d] += sc2 * ((dt - ds2) * (tt[d] / dt));
      }
      {
        double* m = NODE(sh, R - 1, j);
        double* b = NODE(sh, R - 2, j);
        double tb[3] = {m[0] - b[0], m[1] - b[1], m[2] - b[2]};
        double db = sqrt(tb[0] * tb[0] + tb[1] * tb[1] + tb[2] * tb[2]);
        for (int d = 0; d < 3; ++d) m[6 + d] += sc2 * ((db - ds2) * (tb[d] / db));
      }
    }
  }
}

/* compute_elasticforce, cube_pthread/lbm_ib.c:1285-1318. */
void orc_elastic(orc_state* s) {
  for (int k = 0; k < s->nsheets; ++k) {
    orc_sheet* sh = &s->sheets[k];
    long n = (long)sh->rows * sh->cols;
    for (long i = 0; i < n; ++i) {
      double* m = sh->node + i * 12;
      for (int d = 0; d < 3; ++d) m[9 + d] = m[6 + d] + m[3 + d];
    }
  }
}

/* Influential domain of a node: floor(X/dx - 2) + 1 .. +3 per axis,
 * lbm_ib.c:1423-1428 and :2603-2605. */
static inline int orc_start(double p) { return (int)(floor(p / 1.0 - 2) + 1); }

/* get_influentialdomain_fluid_grid_and_SpreadForce, lbm_ib.c:1323-1525
 * (mpi/fiber_SpreadForce.c:147-221 + mpi/fluid_get_SpreadForce.c:28-189):
 * zero F everywhere, then add every node's elastic force times the 4-point
 * cosine kernel over its 4x4x4 stencil, nodes in (sheet, row, col) order. */
int orc_spread(orc_state* s) {
  const double dx = 1.0, dy = 1.0, dz = 1.0;
  const double c_x = ORC_PI / (2.0 * dx), c_y = ORC_PI / (2.0 * dy), c_z = ORC_PI / (2.0 * dz);
  const double cf = 1.0 / (64.0 * dx * dy * dz);
  memset(s->fx, 0, s->N * sizeof(double));
  memset(s->fy, 0, s->N * sizeof(double));
  memset(s->fz, 0, s->N * sizeof(double));
  for (int k = 0; k < s->nsheets; ++k) {
    orc_sheet* sh = &s->sheets[k];
    for (int i = 0; i < sh->rows; ++i)
      for (int j = 0; j < sh->cols; ++j) {
        double* m = NODE(sh, i, j);
        int is = orc_start(m[0]), js = orc_start(m[1]), ks = orc_start(m[2]);
        for (int gi = is; gi <= is + 3; ++gi)
          for (int gj = js; gj <= js + 3; ++gj)
            for (int gk = ks; gk <= ks + 3; ++gk) {
              double rx = dx * gi - m[0];
              double ry = dy * gj - m[1];
              double rz = dz * gk - m[2];
              double tmp = cf * (1.0e0 + ORC_COS(c_x * rx)) * (1.0e0 + ORC_COS(c_y * ry)) * (1.0e0 + ORC_COS(c_z * rz));
              if (gi < 0 || gi >= s->nx || gj < 0 || gj >= s->ny || gk < 0 || gk >= s->nz) return -1;
              long c = IDX(s, gi, gj, gk);
              s->fx[c] += m[9] * tmp;
              s->fy[c] += m[10] * tmp;
              s->fz[c] += m[11] * tmp;
            }
      }
  }
  return 0;
}

/* compute_eqlbrmdistrfuncDF1, lbm_ib.c:1673-1825 (mpi/compute_eqlbrmdistrfuncDF1.c:29-230):
 * BGK collision with Guo forcing in place on df1 over [2, n-3]^3, using the
 * stored rho, u of the previous step and this step's force. */
void orc_collide(orc_state* s) {
  const double tau = s->tau, g = s->g_l, cs = s->cs_l;
  const double cs2 = cs * cs, cs4 = pow(cs, 4);
  const long N = s->N;
#pragma omp parallel for schedule(static)
  for (int z = 2; z <= s->nz - 3; ++z)
    for (int y = 2; y <= s->ny - 3; ++y)
      for (int x = 2; x <= s->nx - 3; ++x) {
        long i = IDX(s, x, y, z);
        double rho = s->rho[i], vx = s->ux[i], vy = s->uy[i], vz = s->uz[i];
        double Fx = s->fx[i], Fy = s->fy[i], Fz = s->fz[i];
        for (int q = 0; q < 19; ++q) {
          const double* c = s->c[q];
          double w = (q == 0) ? 3.0 : (q <= 6 ? 18.0 : 36.0);
          double feq = orc_feq(s, q, rho, vx, vy, vz);
          s->dfeq[q * N + i] = feq;
          s->df1[q * N + i] =
              s->df1[q * N + i] * (1.0 - 1.0 / tau) + 1.0 / tau * feq +
              s->dt * (1.0 - 1.0 / (2.0 * tau)) / w *
                  (((c[0] - vx) * Fx + (c[1] - vy) * Fy + (c[2] - vz) * (Fz + rho * g)) / (cs2) +
                   (c[0] * vx + c[1] * vy + c[2] * vz) / cs4 * (c[0] * Fx + c[1] * Fy + c[2] * (Fz + rho * g)));
        }
      }
}

/* stream_distrfunc, lbm_ib.c:1827-2254 (mpi/stream_distrfunc.c:299-338):
 * df2 at x + c_q <- df1 at x, for every source x in [2, n-3]^3. */
void orc_stream(orc_state* s) {
  const long N = s->N;
  const int periodic = (s->compat & ORC_OPT_PERIODIC_Z) != 0, nz = s->nz;
#pragma omp parallel for schedule(static)
  for (int z = 2; z <= s->nz - 3; ++z)
    for (int y = 2; y <= s->ny - 3; ++y)
      for (int x = 2; x <= s->nx - 3; ++x) {
        long i = IDX(s, x, y, z);
        for (int q = 0; q < 19; ++q) {
          int zt = z + (int)s->c[q][2];
          /* periodic option: a link leaving I in z re-enters at the other
             side (period nz - 4, the z extent of I) */
          if (periodic && zt < 2) zt += nz - 4;
          if (periodic && zt > nz - 3) zt -= nz - 4;
          long t = IDX(s, x + (int)s->c[q][0], y + (int)s->c[q][1], zt);
          s->df2[q * N + t] = s->df1[q * N + i];
        }
      }
}

/* bounceback_rigidwalls, lbm_ib.c:2257-2437 (mpi/bounceback_rigidwalls.c:25-192).
 * The per-cube start/stop rules are kept so the y-wall z range reproduces the
 * comparison with num_cubes_x (:2378, :2414). */
void orc_bounceback(orc_state* s) {
  const long N = s->N;
  const int cs = s->cs, ncx = s->ncx, ncy = s->ncy, ncz = s->ncz;
  const int xlo = 3, xhi = s->nx - 4;
#define BB(dst, src) s->df2[(dst) * N + i] = s->df1[(src) * N + i]
  if (s->compat & ORC_OPT_PERIODIC_Z) {
    /* periodic option: no z walls; the y walls over the whole z extent of I */
    for (int z = 2; z <= s->nz - 3; ++z)
      for (int x = xlo; x <= xhi; ++x) {
        long i = IDX(s, x, 2, z);
        BB(6, 5); BB(12, 11); BB(13, 14); BB(16, 15); BB(17, 18);
        i = IDX(s, x, s->ny - 3, z);
        BB(5, 6); BB(11, 12); BB(14, 13); BB(15, 16); BB(18, 17);
      }
    return;
  }
  /* z walls: z = kb and z = ke, x in [ib+1, ie-1], y in [jb, je] */
  for (int x = xlo; x <= xhi; ++x)
    for (int y = 2; y <= s->ny - 3; ++y) {
      long i = IDX(s, x, y, 2);
      BB(3, 4); BB(7, 8); BB(10, 9); BB(11, 12); BB(13, 14);
      i = IDX(s, x, y, s->nz - 3);
      BB(4, 3); BB(8, 7); BB(9, 10); BB(12, 11); BB(14, 13);
    }
  /* y walls: y = jb and y = je, x in [ib+1, ie-1], z from the cube rules */
  for (int BK = 0; BK < ncz; ++BK) {
    int zs = (BK == 0) ? 2 : 0;
    int ze = cs - 1;
    if (s->compat & ORC_COMPAT_YWALL_CUBES_X) {
      if (BK == ncx - 1) ze = cs - 3;
    } else {
      if (BK == ncz - 1) ze = cs - 3;
    }
    for (int lk = zs; lk <= ze; ++lk) {
      int z = BK * cs + lk;
      for (int x = xlo; x <= xhi; ++x) {
        long i = IDX(s, x, 2, z);
        BB(6, 5); BB(12, 11); BB(13, 14); BB(16, 15); BB(17, 18);
      }
    }
  }
  for (int BK = 0; BK < ncz; ++BK) {
    int zs = (BK == 0) ? 2 : 0;
    int ze = cs - 1;
    if (s->compat & ORC_COMPAT_YWALL_CUBES_X) {
      if (BK == ncx - 1) ze = cs - 3;
    } else {
      if (BK == ncz - 1) ze = cs - 3;
    }
    for (int lk = zs; lk <= ze; ++lk) {
      int z = BK * cs + lk;
      for (int x = xlo; x <= xhi; ++x) {
        long i = IDX(s, x, s->ny - 3, z);
        BB(5, 6); BB(11, 12); BB(14, 13); BB(15, 16); BB(18, 17);
      }
    }
  }
#undef BB
  (void)ncy;
}

/* compute_rho_and_u, lbm_ib.c:2440-2538 (mpi/compute_rho_and_u.c:27-103),
 * over x in [ib+1, ie-1], y in [jb, je], z in [kb, ke]. */
void orc_moments(orc_state* s) {
  const long N = s->N;
#pragma omp parallel for schedule(static)
  for (int z = 2; z <= s->nz - 3; ++z)
    for (int y = 2; y <= s->ny - 3; ++y)
      for (int x = 3; x <= s->nx - 4; ++x) {
        long i = IDX(s, x, y, z);
        double s1 = s->df2[i];
        double s2 = s->c[0][0] * s->df2[i];
        double s3 = s->c[0][1] * s->df2[i];
        double s4 = s->c[0][2] * s->df2[i];
        for (int q = 1; q <= 18; ++q) {
          double f = s->df2[q * N + i];
          s1 += f;
          s2 += s->c[q][0] * f;
          s3 += s->c[q][1] * f;
          s4 += s->c[q][2] * f;
        }
        s->rho[i] = s1;
        s->ux[i] = (s2 + 0.5 * s->dt * s->fx[i]) / s1;
        s->uy[i] = (s3 + 0.5 * s->dt * s->fy[i]) / s1;
        s->uz[i] = (s4 + 0.5 * s->dt * (s->fz[i] + s->rho[i] * s->g_l)) / s1;
      }
}

/* moveFiberSheet, lbm_ib.c:2540-2723 (mpi/fluid_SpreadVelocity.c:25-163 +
 * mpi/fiber_get_SpreadVelocity.c:165-237): interpolate u over the stencil
 * with u * (1+cos) * (1+cos) * (1+cos) / 64 in that order, then X += dt U. */
int orc_move(orc_state* s) {
  const double dx = 1.0, dy = 1.0, dz = 1.0;
  const double dx1 = 1.0 / dx, dy1 = 1.0 / dy, dz1 = 1.0 / dz;
  const double c_x = ORC_PI / (2.0 * dx), c_y = ORC_PI / (2.0 * dy), c_z = ORC_PI / (2.0 * dz);
  const double c_64 = 1.0 / (6.4e1);
  int err = 0;
  for (int k = 0; k < s->nsheets; ++k) {
    orc_sheet* sh = &s->sheets[k];
    long n = (long)sh->rows * sh->cols;
    /* pinned-row option: row 0 (the first cols nodes) stays where it is */
    const long a0 = (s->compat & ORC_OPT_PIN_ROW0) ? sh->cols : 0;
#pragma omp parallel for schedule(static) reduction(|: err)
    for (long a = a0; a < n; ++a) {
      double* m = sh->node + a * 12;
      double s1 = 0, s2 = 0, s3 = 0;
      int is = (int)(floor(m[0] * dx1 - 2) + 1);
      int js = (int)(floor(m[1] * dy1 - 2) + 1);
      int ks = (int)(floor(m[2] * dz1 - 2) + 1);
      for (int i2 = 0; i2 <= 3; i2++) {
        int gi = is + i2;
        double rx = dx * gi - m[0];
        for (int j2 = 0; j2 <= 3; j2++) {
          int gj = js + j2;
          double ry = dy * gj - m[1];
          for (int k2 = 0; k2 <= 3; k2++) {
            int gk = ks + k2;
            double rz = dz * gk - m[2];
            if (gi < 0 || gi >= s->nx || gj < 0 || gj >= s->ny || gk < 0 || gk >= s->nz) { err = 1; continue; }
            long c = IDX(s, gi, gj, gk);
            s1 += s->ux[c] * (1.0 + ORC_COS(c_x * rx)) * (1.0 + ORC_COS(c_y * ry)) * (1.0 + ORC_COS(c_z * rz)) * c_64;
            s2 += s->uy[c] * (1.0 + ORC_COS(c_x * rx)) * (1.0 + ORC_COS(c_y * ry)) * (1.0 + ORC_COS(c_z * rz)) * c_64;
            s3 += s->uz[c] * (1.0 + ORC_COS(c_x * rx)) * (1.0 + ORC_COS(c_y * ry)) * (1.0 + ORC_COS(c_z * rz)) * c_64;
          }
        }
      }
      m[0] += s->dt * s1;
      m[1] += s->dt * s2;
      m[2] += s->dt * s3;
    }
  }
  return err ? -1 : 0;
}

/* copy_inout_to_df2, lbm_ib.c:2769-2907 (bounds as fixed in
 * mpi/copy_inout_to_df2.c:48-140 when the compat bit is cleared).  The
 * serial pthread run visits cubes BK < min(num_cubes_x, num_cubes_z): the
 * loop bound is num_cubes_x (:2800) and cube2thread hands BK >= num_cubes_z
 * to threads that do not exist. */
void orc_copy_inout(orc_state* s) {
  const long N = s->N, P = (long)s->ny * s->nz;
  const int cs = s->cs, ncy = s->ncy, ncz = s->ncz;
  int bk_end = ncz;
  if ((s->compat & ORC_COMPAT_INOUT_PTHREAD) && s->ncx < ncz) bk_end = s->ncx;
  const int xs[4] = {2, 1, s->nx - 3, s->nx - 2};
  for (int w = 0; w < 4; ++w) {
    const double* src = w < 2 ? s->inlet : s->outlet;
    int x = xs[w];
    for (int BJ = 0; BJ < ncy; ++BJ)
      for (int BK = 0; BK < bk_end; ++BK) {
        int ys = (BJ == 0) ? 1 : 0, ye = (BJ == ncy - 1) ? cs - 2 : cs - 1;
        int zs = (BK == 0) ? 1 : 0, ze = (BK == ncz - 1) ? cs - 2 : cs - 1;
        for (int lj = ys; lj <= ye; ++lj)
          for (int lk = zs; lk <= ze; ++lk) {
            int y = BJ * cs + lj, z = BK * cs + lk;
            long i = IDX(s, x, y, z);
            for (int q = 0; q < 19; ++q) s->df2[q * N + i] = src[q * P + (long)y * s->nz + z];
          }
      }
  }
}

/* replace_old_DF, lbm_ib.c:2909-2968: df1 <- df2 on [1, n-2]^3. */
void orc_replace(orc_state* s) {
  const long N = s->N;
#pragma omp parallel for schedule(static)
  for (int z = 1; z <= s->nz - 2; ++z)
    for (int y = 1; y <= s->ny - 2; ++y)
      for (int x = 1; x <= s->nx - 2; ++x) {
        long i = IDX(s, x, y, z);
        for (int q = 0; q < 19; ++q) s->df1[q * N + i] = s->df2[q * N + i];
      }
}

/* One pass of the do_thread loop body, lbm_ib.c:3124-3563. */
int orc_step(orc_state* s) {
  orc_bending(s);
  orc_stretching(s);
  orc_elastic(s);
  if (orc_spread(s)) return -1;
  orc_collide(s);
  orc_stream(s);
  orc_bounceback(s);
  orc_moments(s);
  if (orc_move(s)) return -1;
  orc_copy_inout(s);
  orc_replace(s);
  s->time += s->dt;
  return 0;
}

int orc_run(orc_state* s, int nsteps) {
  for (int t = 0; t < nsteps; ++t)
    if (orc_step(s)) return -1;
  return 0;
}

int orc_time(const orc_state* s) { return s->time; }

/* The delta kernel's cosine as this library variant evaluates it (for tests). */
double orc_cos(double x) { return ORC_COS(x); }

/* The CUDA path's two-phase form of the same cosine, run on the host (for
 * tests; correctly rounded builds only): out[i] = lbib_cos_2phase(x[i]),
 * and, when `slow` is given, slow[i] = 1 where the quick phase left x[i] to
 * the accurate one.  Returns how many it left, or -1 in a build without the
 * correctly rounded cosine. */
long orc_cos_2phase(const double* x, long n, double* out, unsigned char* slow) {
#ifdef ORC_CR_COS
  long ns = 0;
  for (long i = 0; i < n; ++i) {
    double v;
    const int quick = lbib_cos_quick(x[i], &v);
    if (!quick) { v = lbib_cos(x[i]); ++ns; }
    out[i] = v;
    if (slow) slow[i] = (unsigned char)!quick;
  }
  return ns;
#else
  (void)x; (void)n; (void)out; (void)slow;
  return -1;
#endif
}

void orc_get_moments(const orc_state* s, double* rho, double* ux, double* uy, double* uz) {
  memcpy(rho, s->rho, s->N * sizeof(double));
  memcpy(ux, s->ux, s->N * sizeof(double));
  memcpy(uy, s->uy, s->N * sizeof(double));
  memcpy(uz, s->uz, s->N * sizeof(double));
}

void orc_set_moments(orc_state* s, const double* rho, const double* ux, const double* uy, const double* uz) {
  memcpy(s->rho, rho, s->N * sizeof(double));
  memcpy(s->ux, ux, s->N * sizeof(double));
  memcpy(s->uy, uy, s->N * sizeof(double));
  memcpy(s->uz, uz, s->N * sizeof(double));
}

void orc_get_force(const orc_state* s, double* fx, double* fy, double* fz) {
  memcpy(fx, s->fx, s->N * sizeof(double));
  memcpy(fy, s->fy, s->N * sizeof(double));
  memcpy(fz, s->fz, s->N * sizeof(double));
}

void orc_set_force(orc_state* s, const double* fx, const double* fy, const double* fz) {
  memcpy(s->fx, fx, s->N * sizeof(double));
  memcpy(s->fy, fy, s->N * sizeof(double));
  memcpy(s->fz, fz, s->N * sizeof(double));
}

void orc_get_df(const orc_state* s, int which, double* out) {
  const double* src = which == 0 ? s->df1 : which == 1 ? s->df2 : s->dfeq;
  memcpy(out, src, 19 * s->N * sizeof(double));
}

void orc_set_df(orc_state* s, int which, const double* in) {
  double* dst = which == 0 ? s->df1 : which == 1 ? s->df2 : s->dfeq;
  memcpy(dst, in, 19 * s->N * sizeof(double));
}

void orc_get_inout(const orc_state* s, int which, double* out) {
  memcpy(out, which == 0 ? s->inlet : s->outlet, 19 * (long)s->ny * s->nz * sizeof(double));
}

void orc_get_sheet(const orc_state* s, int sheet, double* out) {
  const orc_sheet* sh = &s->sheets[sheet];
  memcpy(out, sh->node, (long)sh->rows * sh->cols * 12 * sizeof(double));
}

void orc_set_sheet(orc_state* s, int sheet, const double* in) {
  orc_sheet* sh = &s->sheets[sheet];
  memcpy(sh->node, in, (long)sh->rows * sh->cols * 12 * sizeof(double));
}
