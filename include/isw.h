/* isw: B200 (sm_100a) dynamical core for the stacked-layer TRiSK shallow-water step and FCT tracer transport.
 *
 * C ABI. Every function returns ISW_OK (0) or an error status and never throws; isw_last_error() gives the message of
 * the calling thread's last failure. Device arrays are plain pointers to the caller's CUDA memory (FP64, C-contiguous,
 * layer-major x[k * n + i] as the reference lays them out); `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream). Handles are not thread-safe; different handles may be used from different threads on
 * different streams. Host arrays passed to the create functions are copied; device arrays passed to step functions are
 * borrowed for the call only (all work is queued on `stream`; nothing is allocated during a step).
 *
 * Reference interfaces replaced (paths in goofyboson/insilica-world-v2):
 *   isw_grid_create            src/insilica/gpu.py:55-83     DeviceGrid(grid)            (+ d2_stencil, gpu.py:86-108)
 *   isw_layers_create          src/insilica/layers.py:36-92  Layers(dg, layers, b, ...)
 *   isw_layers_step            src/insilica/layers.py:185-212 Layers.step(h, u, dt, nfast, Fm)
 *   isw_layers_step_air        the same with theta: the air branch (layers.py:134-136, 152-166, 187-192, 203-206)
 *   isw_layers_update_gfast    src/insilica/layers.py:104-109 Layers.update_gfast(h, theta)
 *   isw_layers_exchange        src/insilica/layers.py:214-232 Layers.exchange(wx, h, u, M, psi, theta, seq)
 *   isw_layers_set_option      the attributes Layers.sig / .tide / .cbot / .cd_bot (layers.py:36-40, 139-149), set by
 *                              ocean.py:88-90, 159, 245 and tides.py:64-69
 *   isw_layers_substeps        src/insilica/layers.py:99-102 Layers.substeps(h, dt)
 *   isw_layers_lap             src/insilica/layers.py:123-127 Layers._lap(u, out)   (used by lap_max, :111-121)
 *   isw_layers_vmix_heat       src/insilica/world.py:317-318  core.k['vmix_heat'](grid, block, args) after the sea
 *                              coupling (kernel kernels/layers.cu:596-621)
 *   isw_layers_mask            src/insilica/layers.py:94-97   Layers.mask(a, rows) (kernel kernels/layers.cu:495-499),
 *                              called by ocean.py:125
 *   isw_layers_status          none: the status word of the one-stack batch a Layers steps through
 *   isw_transport_create       src/insilica/transport.py:19-30 Transport(dg, layers, beta, tracers)
 *   isw_transport_mass_after   src/insilica/transport.py:32-35 Transport.mass_after(M0, Fm, M1)
 *   isw_transport_step_many    src/insilica/transport.py:40-71 Transport.step_many(M0, M1, Fm, tracers, order)
 *   isw_dsum                   src/insilica/gpu.py:111-126   dsum(x, y)
 *   isw_batch_*                src/insilica/ensemble.py:8-29 Ensemble.step, with each member's world.py:290-301 tick
 *                              (Layers.step, Transport.mass_after, Transport.step_many, copyto(M, M1)) in one launch
 *   isw_mesh_build / _get      src/insilica/grid/__init__.py:86-103 make(n, order): icosa.py build_grid :227-277 with
 *                              lloyd_scvt :194-223, edge_list :280-287, hilbert_order :309-338, reorder :341-353;
 *                              trisk.py build_trisk :15-113 and gather_tables :116-142
 */
#ifndef ISW_H
#define ISW_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ISW_OK = 0,
  ISW_EINVAL = 1,        /* bad argument: null handle or pointer, size or shape mismatch, out-of-range index table */
  ISW_ECUDA = 2,         /* a CUDA runtime call failed (the message names it) */
  ISW_ENOMEM = 3,        /* device or host allocation failed at create time */
  ISW_EUNSUPPORTED = 4,  /* a combination this build does not run: air layers or option branches in the mixed form or
                          * in a batch (they step in the FP64 form, call by call) */
  ISW_ETIMEOUT = 5,      /* a bounded device-side wait gave up (persistent kernels); the context stays usable */
  ISW_ENOTFINITE = 6     /* a step left a NaN or Inf thickness (batched steps), or substeps met a non-finite column */
};

/* Precision forms. ISW_FP64: plain FP64, the reference's FP64 path bit for bit (1e-12 where exp() enters). ISW_MIXED:
 * momentum, the TRiSK operators, the slow tendencies and the FCT curvature corrections in FP32; thicknesses, masses, the
 * layer fluxes, the fast loop's sub-step sum and the final wind update in FP64 (state arrays stay FP64). A mixed Layers
 * handle steps through the batched kernels (isw_layers_step uses a private one-stack batch); a mixed Transport handle's
 * per-call isw_transport_step_many runs the FP64 arithmetic, and the mixed FCT runs inside isw_batch_step. */
enum { ISW_FP64 = 0, ISW_MIXED = 1 };

typedef struct isw_grid isw_grid;
typedef struct isw_layers isw_layers;
typedef struct isw_transport isw_transport;
typedef struct isw_mesh isw_mesh;
typedef struct isw_batch isw_batch;

/* A host grid: the reference Grid's arrays (names as in src/insilica/grid/trisk.py and icosa.py). Sizes: N cells, E
 * edges, NV vertices; tables int32 (pads -1), signs and slots int8, geometry FP64. deg, dist, eKi, eKj feed the
 * 3rd-order transport stencil (gpu.py:86-108). */
typedef struct isw_grid_host {
  int n, N, E, NV;
  const int32_t *eI, *eJ;                 /* E */
  const int32_t *nbr, *cellEdge, *cellEdgeAsc; /* N x 6 */
  const int8_t *cellSign;                 /* N x 6 */
  const int32_t *ev1, *ev2;               /* E */
  const int32_t *vEdge, *vCell;           /* NV x 3 */
  const int8_t *vEdgeSign, *vSlot;        /* NV x 3 */
  const int32_t *eoeStart;                /* E + 1 */
  const int32_t *eoe;                     /* eoeStart[E] */
  const double *le, *de;                  /* E */
  const double *areaCell;                 /* N */
  const double *areaV, *fV;               /* NV */
  const double *kite;                     /* N x 6 */
  const double *w;                        /* eoeStart[E] */
  const uint8_t *deg;                     /* N */
  const double *dist;                     /* N x 6 */
  const uint8_t *eKi, *eKj;               /* E */
} isw_grid_host;

/* Layers options (reference layers.py:36-37): Boussinesq or air layers, with the option branches below and the per-step
 * fields of isw_layers_set_option. Air layers and option branches run in the FP64 form, call by call; the mixed form and
 * batches take Boussinesq layers without options (ISW_EUNSUPPORTED otherwise). */
typedef struct isw_layers_params {
  int L;                                  /* 1 .. 8 */
  double grav;
  const double *gprime;                   /* L - 1 values (host) */
  const double *drag, *stress;            /* L values each (host) */
  double nu4, floor_, rotation, div_damp, thin, vmix, vmix_cd;
  const double *b;                        /* N topography (host) or NULL for none */
  int precision;                          /* ISW_FP64 or ISW_MIXED */
  /* air layers (reference Layers(air=...)): h is mass per area (kg/m^2), each layer carries a potential temperature;
   * cp, kappa, rd the air's constants, p0 the reference pressure of theta (Pa). air = 0: Boussinesq layers. */
  int air;
  double cp, kappa, rd, p0;
  double thin_wind;                       /* air: below this thickness the exchange gives a layer its neighbours' wind */
  /* option branches of Boussinesq layers (reference layers.py:36-40): wall (E host values, 0 = a closed edge, or NULL),
   * shelf (a layer squeezed below it takes the thinner cell's thickness at an edge and fades its pressure force; 0 off),
   * shelf_bed != 0: only layers resting on the sea floor count as squeezed. FP64 form. */
  const double *wall;
  double shelf;
  int shelf_bed;
  /* FP64 Boussinesq layers without options step through a private one-stack batch (tiled fast loop, one graph per
   * step; bit-identical results); percall != 0 keeps the per-call kernels (two grid-wide passes per fast sub-step). */
  int percall;
} isw_layers_params;

/* Per-step fields of the option branches (reference attributes Layers.sig / .zm, .tide, .cbot, .cd_bot set by the ocean
 * and the tides): array is a device array the caller keeps filled (borrowed until replaced or cleared with NULL).
 *   ISW_OPT_SIG     L x N buoyancy sigma_k = g (rho_k - rho_0) / rho_0 per cell (the layers' mid-heights zm are kept
 *                   by the core); replaces the fixed g'
 *   ISW_OPT_TIDE    N tide-generating potential (m^2/s^2)
 *   ISW_OPT_CBOT    E internal-tide drag of the bottom layer (m/s per edge)
 *   ISW_OPT_CD_BOT  value: the bottom layer's quadratic drag coefficient (array unused) */
enum { ISW_OPT_SIG = 1, ISW_OPT_TIDE = 2, ISW_OPT_CBOT = 3, ISW_OPT_CD_BOT = 4 };

const char *isw_last_error(void);
int isw_version(void);

int isw_grid_create(const isw_grid_host *g, int device, isw_grid **out);
/* Destroy a grid only after every Layers and Transport handle made on it is destroyed. */
int isw_grid_destroy(isw_grid *g);

int isw_layers_create(isw_grid *g, const isw_layers_params *p, isw_layers **out);
int isw_layers_destroy(isw_layers *s);
/* One time-split RK3 step in place on h (L x N), u (L x E); Fm (L x E, or NULL) receives l dt F of the final stage. */
int isw_layers_step(isw_layers *s, double *h, double *u, double *Fm, double dt, int nfast, void *stream);
/* One step of air layers (reference Layers.step(h, u, dt, nfast, Fm, theta), layers.py:185-206 with the air branch of
 * _stage, :134-136 and :152-166): theta (L x N) is read and, with the interfacial stress's heating, updated in place. */
int isw_layers_step_air(isw_layers *s, double *h, double *u, double *Fm, double *theta, double dt, int nfast, void *stream);
/* Between-step exchange (reference Layers.exchange, layers.py:214-232): thickness wx (L - 1 x N, positive upward across
 * the interface below layer k) moves between layers with the tracer psi and momentum, conservatively; M (L x N) the
 * layers' mass; theta (air layers, or NULL) takes the heat of the momentum mixing and of the last step's nabla^4 loss;
 * seq != 0 moves the tracer in the order water passes through the column. FP64 form. */
int isw_layers_exchange(isw_layers *s, const double *wx, double *h, double *u, double *M, double *psi, double *theta, int seq,
                        void *stream);
/* Set one per-step field of the option branches (ISW_OPT_*); cached step graphs are dropped. Set options before adding
 * the Layers to a batch (a batch reads them when its stacks change). FP64 form. */
int isw_layers_set_option(isw_layers *s, int option, const double *array, double value);
/* Air layers: the fast mode's coefficient per cell from the state (reference Layers.update_gfast, layers.py:104-109). */
int isw_layers_update_gfast(isw_layers *s, const double *h, const double *theta, void *stream);
/* max(1, ceil(dt sqrt(max_i Gc_i sum_k h_k) / (0.5 d_min))): synchronises `stream`. */
int isw_layers_substeps(isw_layers *s, const double *h, double dt, int *out, void *stream);
/* out (L x E) = the edge vector Laplacian of u (L x E). */
int isw_layers_lap(isw_layers *s, const double *u, double *out, void *stream);
/* The heat of kinetic energy removed at the edges returned to the layers' potential temperature (the reference's
 * kernel-table entry core.k['vmix_heat'], called by world.py:317-318 after the sea coupling with the sea's dissipation):
 * diss (E, J/m^2 per edge) gives each cell half of l_e d_e diss_e; each layer k of the column warms by q / (mu pibar_k)
 * with pibar_k the layer's mass-mean Exner function from h (L x N, mass per area). theta (L x N) updated in place; grav,
 * cp, kappa, p0 are the caller's (the world passes its gravity, core.cpa, core.kap and P0). Any precision form. */
int isw_layers_vmix_heat(isw_layers *s, const double *h, const double *diss, double *theta, double grav, double cp,
                         double kappa, double p0, void *stream);
/* Zero the wall edges (wall[e] == 0) of the first `rows` rows (1..8) of an edge field a (rows x E); no-op without walls. */
int isw_layers_mask(isw_layers *s, double *a, int rows, void *stream);
/* The status word of the one-stack batch that isw_layers_step uses (as isw_batch_status; ISW_OK when the handle steps
 * call by call). While it holds ISW_ETIMEOUT or ISW_ENOTFINITE, isw_layers_step refuses with that status. */
int isw_layers_status(isw_layers *s, void *stream, int reset);
/* Replace the bottom height b (N values, a DEVICE pointer, copied on `stream`) the layers rest on: the reference's
 * Layers.b (layers.py:55), which it fixes at construction; here a served request's layers are reused for the next
 * request of the same kind with that request's own terrain. */
int isw_layers_set_bottom(isw_layers *s, const double *b, void *stream);

int isw_transport_create(isw_grid *g, int L, double beta, int tracers, int precision, isw_transport **out);
int isw_transport_destroy(isw_transport *t);
/* M1 (L x N) = M0 moved by the volume fluxes Fm (L x E). */
int isw_transport_mass_after(isw_transport *t, const double *M0, const double *Fm, double *M1, void *stream);
/* Move each of the ntr tracers (device pointers to L x N arrays, given in a host array) in place by Fm; order 1 or 3. */
int isw_transport_step_many(isw_transport *t, const double *M0, const double *M1, const double *Fm, double *const *tracers,
                            int ntr, int order, void *stream);

/* Deterministic sum of x[0..n) (or of x * y): the reference's fixed tree; synchronises `stream`, writes *out. */
int isw_dsum(const double *x, const double *y, long long n, double *out, void *stream);
/* The same sum (bit-identical to isw_dsum) for callers that cannot allocate device memory at the call: no counterpart in
 * the reference. It allocates nothing: its pass scratch is a fixed file-scope device array, so n is limited to
 * 134217728 values (larger n is rejected with ISW_EINVAL). *out is a DEVICE pointer, written on `stream` without
 * synchronising. The first call on each device looks up the array's device address (make it before any stream
 * capture); calls share the array, so calls that overlap on the GPU race and must be serialised. */
int isw_dsum_static(const double *x, const double *y, long long n, double *out, void *stream);

/* Batched step: stacks (a Layers handle with its state h, u, Fm, and optionally a Transport with M, M1 and tracers)
 * registered once, then advanced together by isw_batch_step as ONE CUDA graph per step (one kernel per phase over every
 * stack; the barotropic sub-steps in shared-memory tiles, one cooperative kernel per stage): the RK3 step, the receiving
 * masses M1, the FCT step of every tracer, and M <- M1. Stacks may use different grids, layer counts and precision
 * forms: each phase is one kernel per form present, and in a batch holding both forms the fast-loop tiles serve the mixed
 * stacks while the FP64 ones take the grid-wide sub-steps. Each stack's result is bit-identical to stepping it alone.
 * Registered pointers are borrowed until removed. */
int isw_batch_create(int device, isw_batch **out);
int isw_batch_destroy(isw_batch *b);
int isw_batch_add(isw_batch *b, isw_layers *layers, isw_transport *tr, double *h, double *u, double *Fm, double *M, double *M1,
                  double *const *tracers, int ntr, double dt, int nfast, int *slot);
/* The same for air layers (a Layers created with air != 0), which also carry their potential temperature theta (L x N,
 * FP64, updated in place by the interfacial stress's heat): the batched step runs the air branch (reference
 * layers.py:134-136, 152-166, 187-206) in the FP64 form, grid-wide (no tiles), with the stress's heat returned to theta
 * before the transport reads the tracers (theta may be one of them, as in world.py:291-301). Bit-identical to
 * isw_layers_step_air followed by the transport calls. A batch holding air stacks does not pipeline. */
int isw_batch_add_air(isw_batch *b, isw_layers *layers, isw_transport *tr, double *h, double *u, double *Fm, double *theta,
                      double *M, double *M1, double *const *tracers, int ntr, double dt, int nfast, int *slot);
int isw_batch_remove(isw_batch *b, int slot);
int isw_batch_step(isw_batch *b, void *stream);
/* Tuning (the autotuner's knobs; results are the same under every setting). The barotropic fast loop runs in
 * shared-memory tiles (tiles_enabled != 0, the default) exchanging every k sub-steps, k the largest up to tile_k (1..8,
 * default 8) whose tiles fit in shared memory, or as grid-wide passes. layout: 0 choose, 1 shared (one cooperative launch,
 * every stack cut in proportion to its cells so the tiles fill the SMs), 2 packed (tiles of about tile_cells owned cells,
 * 64..4096, 0 = by blocks per SM; stacks packed into cooperative launches of at most SMs x blocks-per-SM tiles).
 * blocks_per_sm: 0 choose, 1 (1024-thread tiles) or 2 (512-thread tiles). */
int isw_batch_config(isw_batch *b, int tiles_enabled, int tile_k, int layout, int tile_cells, int blocks_per_sm);
/* How the untiled stacks run their grid-wide sub-steps. ISW_GRID_SPLIT (the default): two kernel launches per
 * sub-step, a cell pass and an edge pass. ISW_GRID_PERSISTENT: one cooperative launch per stage and precision form whose
 * co-resident blocks run every sub-step, meeting at a bounded grid barrier after each cell pass and each edge pass.
 * Results are bit-identical either way. This core's own layout choice: no counterpart in the reference (whose
 * Layers.step launches two kernels per sub-step, layers.py:168-175). */
enum { ISW_GRID_SPLIT = 0, ISW_GRID_PERSISTENT = 1 };
int isw_batch_grid_loop(isw_batch *b, int mode);
/* The fast-loop layout of the stacks on grids of one level (an ensemble or a serving mix holds several): mode 0 follows
 * the batch's configuration (the default), 1 keeps them untiled (grid-wide sub-steps), 2 tiles them in the packed layout
 * with about tile_cells owned cells per tile (0: the batch's) and an exchange interval of at most tile_k (0: the
 * batch's); the packed layout must be allowed by isw_batch_config (tiles on). Results are the same under every layout.
 * This core's layout choice: no counterpart in the reference. */
int isw_batch_level_layout(isw_batch *b, int level, int mode, int tile_cells, int tile_k);
/* Pipelined steps (on != 0): each isw_batch_step queues a step's dynamics beside the previous step's transport (two
 * branches of one graph, the step's layer fluxes Fm double-buffered), so the registered masses M and tracers lag the
 * dynamics by one step until isw_batch_flush, which completes the last step's transport and puts its Fm in the
 * registered arrays; the state is then bit-identical to stepping in the plain order. Adding or removing stacks,
 * configuring or switching the mode flushes first. Off by default. */
int isw_batch_pipeline(isw_batch *b, int on);
int isw_batch_flush(isw_batch *b, void *stream);
/* The batch's layout: registered stacks, fast-loop tiles, the exchange interval in use, the largest tile's shared memory
 * (bytes), the cooperative launches per stage, tile blocks per SM (0 when untiled). */
int isw_batch_info(isw_batch *b, int *stacks, int *tiles, int *tile_k, long long *smem_bytes, int *groups, int *blocks_per_sm);
/* The batch's device status word: ISW_OK, ISW_ETIMEOUT after a grid barrier's bounded wait ran out, or ISW_ENOTFINITE
 * after a step left a NaN or Inf thickness (checked for every cell and layer at the end of each step). The kernel that
 * records a failure also writes it to a mapped host word, and isw_batch_step refuses to run (returning that status)
 * until the word is cleared, so later steps never run on a half-updated state. Synchronises `stream`; reset != 0
 * clears the word (restore the state first). */
int isw_batch_status(isw_batch *b, void *stream, int reset);
/* Failure-detection test: one step in which block 0 never arrives at the first grid barrier, so every other block's
 * bounded wait runs out after timeout_ns (1 ms .. 2 s) and the status word becomes ISW_ETIMEOUT. Test use only. */
int isw_batch_fault_test(isw_batch *b, long long timeout_ns, void *stream);

/* Build the level-n mesh (N = 10 4^n + 2 cells) on the host: icosphere, Lloyd smoothing to 1e-11 rad (at most max_iters
 * iterations; on CUDA device `device`, or on host cores when device < 0), geometry, edge list, Hilbert renumbering when
 * hilbert != 0, TRiSK weights and gather tables. pos_v1 (N x 3, or NULL) supplies the smoothed positions in the
 * icosphere's numbering instead of running Lloyd. */
int isw_mesh_build(int n, int hilbert, int max_iters, int device, const double *pos_v1, isw_mesh **out);
/* A mesh array by its reference name ("eI", "cellEdge", "w", "pos", ...). kind: 0 float64, 1 int32, 2 int8, 3 uint8,
 * 4 float64 3-vectors (count = vectors), 5 int64 scalar, 6 float64 scalar. The data stays owned by the mesh. */
int isw_mesh_get(const isw_mesh *m, const char *name, const void **data, int64_t *count, int *kind);
int isw_mesh_destroy(isw_mesh *m);

#ifdef __cplusplus
}
#endif
#endif
