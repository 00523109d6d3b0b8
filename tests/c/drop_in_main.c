/*
 * A host program written the way the reference's mpi/main.c drives its
 * solver (flags -> init_gv_constant -> gen_fiber_sheet / gen_fluid_grid ->
 * init_gv -> init_* -> do_thread), compiled against include/lbib.h and linked
 * with liblbib.so.  Used by tests/test_abi.py (host-only mode, no GPU) and
 * tests/test_gpu_dropin.py.
 *
 *   drop_in_main -steps S -dump D -fluid_grid_xyz NX NY NZ -cube_size K
 *                -num_fibersht 1 -fibersht_width_height W H
 *                -fibersht_row_clmn R C -fibersht_xyz_0 X0 Y0 Z0
 *                [-params tau u Ks Kb] [-host_only] [-out FILE] [-fv] [-bin]
 *
 * Unlike the reference CLI the grid sizes are the internal ones (x = flow).
 * -host_only stops after the host set-up and prints constants and sheet
 * positions; otherwise the run's sheet records and rho/u fields go to FILE
 * as raw float64.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lbib.h"

static void need(int i, int argc, int n, const char* f) {
  if (i + n >= argc) { fprintf(stderr, "error: flag %s needs %d argument(s)\n", f, n); exit(2); }
}

int main(int argc, char** argv) {
  GV gv = (GV)calloc(1, sizeof(*gv));
  int host_only = 0, nsheets = 0;
  double params[4] = {0, 0, 0, 0};
  int have_params = 0;
  const char* out = NULL;
  gv->fluid_grid = (Fluidgrid*)calloc(1, sizeof(Fluidgrid));
  for (int i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "-steps")) { need(i, argc, 1, argv[i]); gv->timesteps = atoi(argv[++i]); }
    else if (!strcmp(argv[i], "-dump")) { need(i, argc, 1, argv[i]); gv->dump = atoi(argv[++i]); }
    else if (!strcmp(argv[i], "-fluid_grid_xyz")) {
      need(i, argc, 3, argv[i]);
      gv->fluid_grid->x_dim = atoi(argv[++i]);
      gv->fluid_grid->y_dim = atoi(argv[++i]);
      gv->fluid_grid->z_dim = atoi(argv[++i]);
    } else if (!strcmp(argv[i], "-cube_size")) { need(i, argc, 1, argv[i]); gv->cube_size = atoi(argv[++i]); }
    else if (!strcmp(argv[i], "-num_fibersht")) {
      need(i, argc, 1, argv[i]);
      nsheets = atoi(argv[++i]);
      gv->fiber_shape = (Fibershape*)calloc(1, sizeof(Fibershape));
      gv->fiber_shape->num_sheets = nsheets;
      gv->fiber_shape->sheets = (Fibersheet*)calloc(nsheets, sizeof(Fibersheet));
    } else if (!strcmp(argv[i], "-fibersht_width_height")) {
      for (int j = 0; j < nsheets; j++) {
        need(i, argc, 2, argv[i]);
        gv->fiber_shape->sheets[j].width = atof(argv[++i]);
        gv->fiber_shape->sheets[j].height = atof(argv[++i]);
      }
    } else if (!strcmp(argv[i], "-fibersht_row_clmn")) {
      for (int j = 0; j < nsheets; j++) {
        need(i, argc, 2, argv[i]);
        gv->fiber_shape->sheets[j].num_rows = atoi(argv[++i]);
        gv->fiber_shape->sheets[j].num_cols = atoi(argv[++i]);
      }
    } else if (!strcmp(argv[i], "-fibersht_xyz_0")) {
      for (int j = 0; j < nsheets; j++) {
        need(i, argc, 3, argv[i]);
        gv->fiber_shape->sheets[j].x_orig = atof(argv[++i]);
        gv->fiber_shape->sheets[j].y_orig = atof(argv[++i]);
        gv->fiber_shape->sheets[j].z_orig = atof(argv[++i]);
      }
    } else if (!strcmp(argv[i], "-params")) {
      need(i, argc, 4, argv[i]);
      for (int k = 0; k < 4; ++k) params[k] = atof(argv[++i]);
      have_params = 1;
    } else if (!strcmp(argv[i], "-host_only")) host_only = 1;
    else if (!strcmp(argv[i], "-out")) { need(i, argc, 1, argv[i]); out = argv[++i]; }
    else if (!strcmp(argv[i], "-fv")) gv->lbib_dump_mode |= LBIB_DUMP_FIELDVIEW;
    else if (!strcmp(argv[i], "-bin")) gv->lbib_dump_mode |= LBIB_DUMP_BINARY;
    else { fprintf(stderr, "error: unknown flag %s\n", argv[i]); return 2; }
  }
  if (!gv->fiber_shape || nsheets < 1) { fprintf(stderr, "error: -num_fibersht missing\n"); return 2; }

  /* mpi/main.c order: constants, sheets, grid, init_gv, initial state */
  init_gv_constant(gv);
  if (have_params) { gv->tau = params[0]; gv->u_l = params[1]; gv->Ks_l = params[2]; gv->Kb_l = params[3]; }
  for (int k = 0; k < nsheets; ++k) gen_fiber_sheet(&gv->fiber_shape->sheets[k]);

  if (host_only) {
    FILE* f = out ? fopen(out, "w") : stdout;
    fprintf(f, "dt %d time %d ib %d ie %d jb %d je %d kb %d ke %d\n", gv->dt, gv->time, gv->ib, gv->ie, gv->jb,
            gv->je, gv->kb, gv->ke);
    fprintf(f, "tau %.17g u_l %.17g Ks_l %.17g Kb_l %.17g cs_l %.17g\n", gv->tau, gv->u_l, gv->Ks_l, gv->Kb_l,
            gv->cs_l);
    fprintf(f, "cubes %d %d %d\n", gv->num_cubes_x, gv->num_cubes_y, gv->num_cubes_z);
    for (int k = 0; k < nsheets; ++k) {
      Fibersheet* sh = &gv->fiber_shape->sheets[k];
      for (int r = 0; r < sh->num_rows; ++r)
        for (int c = 0; c < sh->num_cols; ++c)
          fprintf(f, "node %d %d %d %.17g %.17g %.17g\n", k, r, c, sh->fibers[r].nodes[c].x,
                  sh->fibers[r].nodes[c].y, sh->fibers[r].nodes[c].z);
    }
    if (out) fclose(f);
    return lbib_last_error() == LBIB_OK ? 0 : 1;
  }

  gen_fluid_grid(gv->fluid_grid, gv->cube_size, 0, gv);
  init_gv(gv);
  init_eqlbrmdistrfuncDF0(gv);
  init_df1(gv);
  init_df_inout(gv);
  if (lbib_last_error() != LBIB_OK) {
    fprintf(stderr, "set-up failed: %s\n", lbib_error_string(lbib_last_error()));
    return 1;
  }
  /* the reference spawns threads; every tid but 0 returns at once here */
  struct lv_t lvs[2] = {{0, gv}, {1, gv}};
  do_thread(&lvs[1]);
  do_thread(&lvs[0]);
  if (lbib_last_error() != LBIB_OK) {
    fprintf(stderr, "step loop stopped at time %d: %s\n", gv->time, lbib_error_string(lbib_last_error()));
    return 1;
  }
  if (out) {
    FILE* f = fopen(out, "wb");
    lbib_sync_to_host(gv);
    for (int k = 0; k < nsheets; ++k) {
      Fibersheet* sh = &gv->fiber_shape->sheets[k];
      for (int r = 0; r < sh->num_rows; ++r) fwrite(sh->fibers[r].nodes, sizeof(Fibernode), sh->num_cols, f);
    }
    long N = (long)gv->fluid_grid->x_dim * gv->fluid_grid->y_dim * gv->fluid_grid->z_dim;
    double* buf = (double*)malloc(sizeof(double) * 4 * N);
    lbib_get_moments(gv, buf, buf + N, buf + 2 * N, buf + 3 * N);
    fwrite(buf, sizeof(double), 4 * N, f);
    free(buf);
    fclose(f);
  }
  lbib_free(gv);
  printf("time %d\n", gv->time);
  return 0;
}
