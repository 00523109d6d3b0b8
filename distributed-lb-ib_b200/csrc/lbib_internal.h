/*
 * Internal interface between the host C layer (lbib_api.c) and the CUDA
 * translation units.  Not installed; include/lbib.h is the public ABI.
 *
 * GPU data layout (one fluid grid, several sheets):
 *   f        [19][Ns] populations (FP64; FP32; FP16 or BF16 holding f - w_q),
 *            Ns = sx*ny*nz, idx = (z*ny + y)*sx + x - gx0: the whole grid
 *            (sx = nx, gx0 = 0), or an x-slab of it with ghost columns.
 *            One buffer, updated in place with the AA access pattern; `parity`
 *            says how the next fused step must read it (0: each cell's own
 *            slots in natural order; 1: the neighbours' opposite slots).
 *   inlet/outlet [19][ny*nz] fixed equilibria (reference df_inout planes).
 *   tiles    the grid is cut into 4x4x4 tiles; a step's force spread touches
 *            few of them.  For the current and the previous step the library
 *            keeps tile -> slot maps and per-slot arrays: force F(t) [slot][3][64]
 *            and moments (rho, u)(t) [slot][4][64].
 *   nodes    [S][12] Fibernode records of all sheets, concatenated.
 *   weights  [S][12] the delta-kernel factors (1 + cos(pi/2 r)) of each node's
 *            4x4x4 stencil (4 per axis), and [S][3] its start indices.
 */
#ifndef LBIB_INTERNAL_H
#define LBIB_INTERNAL_H

#include <stdio.h>

#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBIB_TILE 4
#define LBIB_TILE_CELLS 64
#define LBIB_CHUNK 32

#ifndef LBIB_PREC_F64
#define LBIB_PREC_F64 0   /* population storage precisions, as in include/lbib.h */
#define LBIB_PREC_F32 1
#define LBIB_PREC_F16 2
#define LBIB_PREC_BF16 3
#define LBIB_PREC_SHIFT_FLOW 16
#endif
#define LBIB_PREC_TYPE(p) ((p) & 15)

#ifndef LBIB_OPT_PERIODIC_Z
#define LBIB_OPT_PERIODIC_Z 0x100  /* option bits of the compat word, as in include/lbib.h */
#define LBIB_OPT_REST_START 0x200
#define LBIB_OPT_PIN_ROW0   0x400
#endif

typedef struct lbib_sheet_dev {
  int rows, cols;
  long offset;                   /* first node in the concatenated arrays */
  double bc;                     /* Kb_l / ds2^3                  (bending)    */
  double sc, sc2;                /* Ks_l / ds1^2, Ks_l / ds2^2    (stretching) */
  double ds1, ds2;               /* width/(cols-1), height/(rows-1)            */
} lbib_sheet_dev;

typedef struct lbib_device {
  int nx, ny, nz;
  long N;                        /* cells of the global grid                 */
  /* the x-slab this state holds: global columns [x_lo, x_hi), stored with
     two ghost columns on each side (the whole grid: [0, nx), no ghosts) */
  int x_lo, x_hi;
  int sx, gx0;                   /* stored row length; global x of column 0  */
  long Ns;                       /* stored cells: sx * ny * nz               */
  double* halo;                  /* slab exchange buffers [4][5][ny*nz]:     */
                                 /* send_lo, send_hi, recv_lo, recv_hi       */
  /* direct exchange: the neighbours' populations (peer or IPC-mapped device
     pointers, with their storage geometry) and every slab's moment tiles */
  double* peer_f[2];             /* left, right neighbour (NULL: none)       */
  long peer_Ns[2];
  int peer_sx[2], peer_gx0[2];
  double* peer_U[2][8];          /* [buffer][slab], this slab's own included */
  int npeer_U;
  int cube_size, ncx, ncy, ncz;
  int compat;
  int zin_hi;                    /* last z row the inlet/outlet copy reaches  */
  int yskip_z0;                  /* y walls skip rows z0, z0+1 (or -1)        */
  /* physics and the collision constants, computed on the host exactly as the
     reference writes them */
  double tau, u_l, rho_l, Ks_l, Kb_l, g_l, cs_l;
  int dt;
  double omtau, invtau, kw[3], cs2, cs4, half_dt;
  /* populations: [19][N] of the storage type of `prec`; inlet/outlet in
     its arithmetic type (double for FP64, float otherwise) */
  int prec;
  void* f;
  void* inlet;
  void* outlet;
  int parity;
  long steps;                    /* fused steps since init_df1               */
  int use_bulk;                  /* bulk kernel for rows away from walls     */
  int lp_variant;                /* low-precision word-kernel variant, -1 = default */
  int l2_pf;                     /* bulk kernels: L2 prefetch distance, in waves of
                                    resident blocks (0: none)                  */
  int* rows;                     /* device int2 (y, z) rows of the generic kernel */
  int nrows;
  int have_eq, have_df1, have_inout;
  /* force / moment tiles, double buffered by step */
  int ntx, nty, ntz;
  long ntiles;
  long cap;                      /* slots per buffer                          */
  int* tile_cnt;                 /* [ntiles] nodes whose stencil touches it   */
  int* slot_off;                 /* [cap] start of the slot's node list       */
  int* slot_len;                 /* [cap] length of the slot's node list      */
  int* slot_cursor;              /* [cap] fill cursor                         */
  int* pair_node;                /* [8 S] int2 entry lists of the touched tiles */
  int* tile_slot[2];             /* [ntiles] slot or -1                       */
  int* tile_list[2];             /* [cap] touched tiles in index order        */
  int* tile_count[2];            /* [1]                                       */
  int* scan_tmp;                 /* block sums for the compaction             */
  unsigned long long* scan_state; /* one-pass compaction: per-block words + ticket */
  unsigned scan_tag;             /* the one-pass compaction's launch tag (1..255) */
  double* Ftile[2];              /* [cap][3][64]                              */
  double* Utile[2];              /* [cap][4][64]                              */
  int cur;                       /* buffers of the step in progress / last    */
  int have_forces;               /* Ftile[cur] holds this step's spread       */
  int have_moments;              /* Utile[cur] holds this step's moments      */
  /* sheets */
  int nsheets;
  long S;
  lbib_sheet_dev* sh;            /* host array [nsheets]                      */
  double* nodes;                 /* [S][12]                                   */
  double* h_nodes;               /* [S][12] pinned host staging for syncs     */
  double* W;                     /* [S][12]                                   */
  int* st;                       /* [S][3]                                    */
  int* chunk_box;                /* [nchunks][6]                              */
  long nchunks;
  /* errors and plumbing */
  int* err;                      /* [2]: code, step                           */
  int* h_err;                    /* pinned mirror                             */
  double* scratch;               /* dense field scratch for getters           */
  void* host_reg[8];             /* host blocks page-locked for direct copies */
  size_t host_reg_bytes[8];
  int nhost_reg;
  cudaStream_t stream;
  /* the fluid step overlapped with the spread (one-grid steps): the row and
     bulk kernels run on fluid_stream, skipping the tiles of the box of this
     step's stencils (box[6], in tiles, computed at the start of the step);
     the box's cells run on `stream` after the spread */
  cudaStream_t fluid_stream;     /* == stream unless a step is overlapped     */
  cudaStream_t side;
  cudaEvent_t ev_box, ev_bulk;
  int* box;                      /* [2][6]: this step's box and the next's    */
  int box_cur;                   /* which of the two this step uses           */
  int box_valid;                 /* box[box_cur] holds the current positions' */
  int* box_next;                 /* the move accumulates the next box here    */
  int box_mode;                  /* 1 inside an overlapped step               */
  int overlap;                   /* overlapped steps allowed (LBIB_OVERLAP)   */
  int fuse_forces;               /* the spread's node preparation also computes the fiber forces */
  int device;
  long kernel_launches;          /* kernels this state has launched           */
  /* optional stage timing: events around the five stages of each step */
  int profiling;
  cudaEvent_t* prof_ev;          /* [prof_cap][LBIB_PROF_EV]                  */
  char* prof_overlap;            /* [prof_cap] the step was overlapped        */
  long prof_steps, prof_cap;
} lbib_device;

#define LBIB_NSTAGE_TIMED 5      /* forces, spread, fluid, moments, move */
#define LBIB_PROF_EV 9           /* events per profiled step                 */

typedef struct lbdev_config {
  int nx, ny, nz, cube_size, compat, prec;
  int x_lo, x_hi;                /* slab columns; x_hi = 0: the whole grid */
  double tau, u_l, rho_l, Ks_l, Kb_l, g_l, cs_l;
  int dt;
} lbdev_config;

int  lbdev_create(lbib_device** out, const lbdev_config* cfg);
/* Columns [x_lo, x_hi) of the grid held by d (x_hi <= 0: all); sets the
 * storage geometry, allocates nothing. */
int  lbdev_set_columns(lbib_device* d, int x_lo, int x_hi);
/* Slab exchange (FP64 slabs): after a fused step of parity `par`, pack the
 * columns the neighbours need into send_lo / send_hi; after the transport,
 * unpack recv_lo / recv_hi into this slab's columns. */
int  lbdev_slab_pack(lbib_device* d, int par);
int  lbdev_slab_unpack(lbib_device* d, int par);
int  lbdev_slab_moments(lbib_device* d, double** U, long* n, int* failed_step);
/* Direct exchange (lbdev_slab_connect first): after a fused step of parity
 * `par`, write the face columns straight into the neighbours' storage;
 * the moment tiles of this slab's columns into every slab's tiles. */
int  lbdev_slab_push(lbib_device* d, int par);
int  lbdev_slab_moments_bcast(lbib_device* d);
int  lbdev_slab_connect(lbib_device* d, double* lo_f, long lo_Ns, int lo_sx, int lo_gx0, double* hi_f,
                        long hi_Ns, int hi_sx, int hi_gx0, int n, double* const* U0, double* const* U1);
int  lbdev_peer_access(int device, int peer);
int  lbdev_ipc_handle(void* dev_ptr, void* handle);     /* 64 bytes */
int  lbdev_ipc_open(const void* handle, void** dev_ptr);
int  lbdev_ipc_close(void* dev_ptr);
size_t lbdev_pop_bytes(int prec);
/* The low-precision shift s_q and the (rho, u_x) it carries. */
void lbdev_shift(const lbib_device* d, float* sh, double* rhos, double* uxs);
void lbdev_free(lbib_device* d);
int  lbdev_set_physics(lbib_device* d, const lbdev_config* cfg);
int  lbdev_set_sheets(lbib_device* d, int nsheets, const lbib_sheet_dev* sh, const double* nodes_host);
int  lbdev_init_equilibrium(lbib_device* d);   /* init_eqlbrmdistrfuncDF0 */
int  lbdev_init_df1(lbib_device* d);           /* init_df1 */
int  lbdev_init_inout(lbib_device* d);         /* init_df_inout */
int  lbdev_stage(lbib_device* d, int which, int step_no);
int  lbdev_step(lbib_device* d, int step_no);
int  lbdev_check(lbib_device* d, int* failed_step);  /* syncs, reads error word */
int  lbdev_get_moments(lbib_device* d, double* rho, double* ux, double* uy, double* uz);
int  lbdev_get_force(lbib_device* d, double* fx, double* fy, double* fz);
int  lbdev_get_df1(lbib_device* d, double* out);
int  lbdev_conservation(lbib_device* d, double* out);
int  lbdev_get_nodes(lbib_device* d, double* out);
int  lbdev_set_nodes(lbib_device* d, const double* in);
int  lbdev_sync(lbib_device* d);
/* Page-lock a host block the library owns (a sheet's node records) so that
 * copies go to it directly; best effort, undone by lbdev_free. */
int  lbdev_register_host(lbib_device* d, void* p, size_t bytes);
int  lbdev_is_registered(const lbib_device* d, const void* p, size_t bytes);
/* Node records [first, first+n) to host memory, asynchronous on the stream. */
int  lbdev_copy_nodes_out(lbib_device* d, long first, long n, double* host);
int  lbdev_copy_nodes_in(lbib_device* d, long first, long n, const double* host);
int  lbdev_variants(const lbib_device* d);     /* kernel variants for this precision */
int  lbdev_set_variant(lbib_device* d, int v);
/* Times every variant on fluid steps from the initial state, keeps the
 * fastest, and restores the initial populations; only before the first
 * step.  ms[i] = mean ms per step of variant i (ms may be NULL). */
int  lbdev_autotune(lbib_device* d, int steps, double* ms, int max_ms, int* best);
/* Restart state (raw device bytes of everything the next step reads). */
int  lbdev_save_state(lbib_device* d, FILE* fp);
int  lbdev_load_state(lbib_device* d, FILE* fp);
int  lbdev_profile_begin(lbib_device* d);
int  lbdev_profile_end(lbib_device* d, double* stage_ms, long* steps);

#ifdef __cplusplus
}
#endif
#endif
