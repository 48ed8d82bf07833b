/*
 * nuvort_gpu.h -- C ABI of libnuvort_gpu.so, the B200 (sm_100a) filament-velocity
 * path of the NuVort quantised-vortex code.
 *
 * The reference (a Fortran 90 program) has no plugin or FFI layer: its hot path is a
 * set of argument-less module procedures called in order from the time loop in
 * src/run.f90:24-65, communicating through the module globals f(:), pcount, t, dt and
 * the run.in parameters (src/cdata.f90:19-127).  Each stage call below replaces one of
 * those procedures and keeps its semantics; the filament state lives on the GPU between
 * calls.  A Fortran caller binds these with ISO_C_BINDING (see fortran/nuvort_gpu.f90).
 *
 * Conventions
 *   - Every function returns an int status: NV_OK (0) or a negative NV_ERR_* code.
 *     nv_last_error() returns a message for the calling thread's last failure.
 *     The reference prints and calls `stop` instead (fatal_error, src/cdata.f90:245-255).
 *   - Slots are 1-based and system-local exactly as in the reference: infront==0 marks an
 *     empty slot; pcount counts slots, empty ones included.
 *   - Host arrays of 3-vectors are point-major, the memory layout of a Fortran
 *     real(c_double) :: a(3,pcount) array: a[3*(k-1)+c] holds f(k)%x(c+1).
 *   - A handle holds nsys independent filament systems (an ensemble).  A handle is used by
 *     one host thread at a time and owns one CUDA stream; it is not reentrant.
 *   - The library owns all device memory.  Host pointers are read or written only during
 *     the call that receives them.
 */
#ifndef NUVORT_GPU_H
#define NUVORT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
enum {
  NV_OK = 0,
  NV_ERR_ARG = -1,         /* invalid argument */
  NV_ERR_CUDA = -2,        /* CUDA runtime failure */
  NV_ERR_CAPACITY = -3,    /* pinsert needed a slot beyond the system's capacity */
  NV_ERR_SINGULAR = -4,    /* tree walk met dist<epsilon (src/tree.f90:289-295) */
  NV_ERR_TREE_DEPTH = -5,  /* octree deeper than NV_TREE_MAX_DEPTH levels, its node buffer
                              exhausted, or a walk longer than the tree (a malformed tree) */
  NV_ERR_NAN = -6,         /* NaN position (NAN_finder, src/general.f90:172-190) */
  NV_ERR_EMPTY = -7,       /* no live points left (src/line.f90:25-27) */
  NV_ERR_TIMESTEP = -8,    /* dt fails timestep_check (src/initial.f90:169-180) */
  NV_ERR_UNSUPPORTED = -9, /* option combination outside this library (e.g. solid walls in
                              mixed precision) */
  NV_ERR_STATE = -10,      /* call out of order (e.g. tree search with no tree built) */
  NV_ERR_QUEUE = -11,      /* serial topology resolver overflowed its work queue */
  NV_ERR_IO = -12,         /* run.in (or a snapshot/restart file) could not be opened or read */
  NV_ERR_TIMEOUT = -13     /* a bounded device-side wait gave up (the context stays usable) */
};

/* ---- option values (the run.in strings of src/cdata.f90:131-241) -------------------- */
enum { NV_VEL_LIA = 0, NV_VEL_BS = 1, NV_VEL_TREE = 2 };               /* velocity */
enum { NV_BC_PERIODIC = 0, NV_BC_OPEN = 1, NV_BC_SOLID = 2 };          /* boundary_x/y/z */
/* normal_velocity, the fields of get_normal_velocity (src/normal_fluid.f90:83-118): 'zero',
 * 'xflow', 'shear_xflow' (A sin(2 pi z/L_z + omega t) along x), 'ychannel' (A (1-(2y/L_y)^2)
 * along x), 'channel' (the 10-term duct series), 'noisey_xflow' (A times a noise sample that
 * advances once per pmotion; samples from nv_set_normal_fluid_noise), 'laizetDNS' and
 * 'turbDNS' (trilinear interpolation on a stored grid, nv_set_normal_fluid_grid).  'uniform'
 * is an extension (a constant vector norm_vel_vec) that the reference lacks. */
enum {
  NV_NF_ZERO = 0, NV_NF_XFLOW = 1, NV_NF_UNIFORM = 2, NV_NF_SHEAR_XFLOW = 3, NV_NF_CHANNEL = 4,
  NV_NF_YCHANNEL = 5, NV_NF_NOISEY_XFLOW = 6, NV_NF_LAIZET_DNS = 7, NV_NF_TURB_DNS = 8
};
/* precision of the non-local sum: FP64 reproduces the reference's arithmetic; MIXED runs the
 * far field in FP32 with compensated accumulation and keeps the near field in FP64. */
enum { NV_PREC_FP64 = 0, NV_PREC_MIXED = 1 };
/* non-local evaluation inside a handle: follow `velocity`, or (batched ensembles) pick the
 * direct sum below a point-count crossover and the tree above it. */
enum { NV_SCHED_AS_SET = 0, NV_SCHED_CROSSOVER = 1 };

#define NV_TREE_MAX_DEPTH 42

/* ---- parameters: one record per system; field names are the run.in keys ------------- */
typedef struct nv_params {
  int32_t nsteps;                 /* nsteps                                  cdata.f90:155 */
  int32_t shots;                  /* shots                                   cdata.f90:158 */
  int32_t recon_shots;            /* recon_shots (default 1)                 cdata.f90:161 */
  int32_t velocity;               /* NV_VEL_*                                cdata.f90:181 */
  int32_t boundary[3];            /* NV_BC_* for x,y,z (default periodic)    cdata.f90:184 */
  int32_t normal_velocity;        /* NV_NF_*                                 cdata.f90:196 */
  int32_t tree_extra_correction;  /* logical, default true                  cdata.f90:194 */
  int32_t nan_test;               /* NAN_test, default true                 cdata.f90:218 */
  int32_t overide_timestep_check; /* default false                           cdata.f90:222 */
  int32_t precision;              /* NV_PREC_* (extension)                               */
  double dt;                      /* dt                                      cdata.f90:167 */
  double delta;                   /* delta                                   cdata.f90:170 */
  double quant_circ;              /* default 9.97e-4                         cdata.f90:173 */
  double corea;                   /* default 8.244023e-9                     cdata.f90:176 */
  double box_size[3];             /* box_size                                cdata.f90:178 */
  double tree_theta;              /* 0 = no tree, brute pclose               cdata.f90:190 */
  double norm_vel_xflow;          /* default 0.5                             cdata.f90:202 */
  double norm_vel_vec[3];         /* NV_NF_UNIFORM vector (extension)                    */
  double alpha[2];                /* mutual friction alpha, alpha'           cdata.f90:204 */
  double super_velocity[3];       /* imposed superflow                       cdata.f90:206 */
  double normal_fluid_cutoff;     /* default 1e8                             cdata.f90:198 */
  double t_zero_normal_fluid;     /* default 1e8                             cdata.f90:200 */
  double norm_shear_omega;        /* shear_xflow frequency, default 0        cdata.f90:232 */
} nv_params;

/* Host view of one system's filament state (the fields of type(qvort), cdata.f90:19-29,
 * that the hot path reads or writes).  Optional pointers may be NULL. */
typedef struct nv_host_state {
  int32_t pcount;     /* slots described by the arrays                           */
  double *x;          /* [3*pcount] positions (required)                         */
  double *u, *u1, *u2;/* [3*pcount] velocity and the two older velocities (opt.) */
  double *ghosti;     /* [3*pcount] ghost of the point in front (optional)       */
  double *ghostb;     /* [3*pcount] ghost of the point behind (optional)         */
  int32_t *infront;   /* [pcount] 1-based, 0 = empty (required)                  */
  int32_t *behind;    /* [pcount] (required)                                     */
  int32_t *closest;   /* [pcount] reconnection candidate (optional)              */
  double *closestd;   /* [pcount] its distance (optional)                        */
  /* solid walls (optional; NULL: no pinned points): a point pinned in front (pinnedi, its
   * infront is itself: the segment ends in the wall) or behind (pinnedb), and the wall it is
   * pinned to, wpinned(1:3) in -1, 0, +1 (src/cdata.f90:27-28) */
  int32_t *wpinned;   /* [3*pcount]                                              */
  int32_t *pinnedi;   /* [pcount] logical 0/1                                    */
  int32_t *pinnedb;   /* [pcount] logical 0/1                                    */
} nv_host_state;

/* Topology events, logged in the order the reference's serial sweeps make them. */
enum { NV_EV_INSERT = 1, NV_EV_RECON = 2, NV_EV_REMOVE = 3, NV_EV_LOOPKILL = 4, NV_EV_WALL = 5,
       NV_EV_CLEAR = 6 };
typedef struct nv_event {
  int32_t itime; /* step number (the reference's itime)                                  */
  int32_t kind;  /* NV_EV_*                                                              */
  int32_t i;     /* INSERT: point i; RECON: point i; REMOVE: point i; LOOPKILL: start p;
                    WALL: the point wall_recon cleared (src/reconnection.f90:66-150);
                    CLEAR: point i pinned behind, cleared with the point in front of it
                    when that one is pinned in front (line.f90:125-127,
                    reconnection.f90:71-75)                                             */
  int32_t j;     /* INSERT: new slot; RECON: partner j; REMOVE: removed slot;
                    LOOPKILL: points cleared; WALL: points cleared (1-3); CLEAR: points
                    cleared (2, or 1 for a point pinned at both ends)                   */
} nv_event;

typedef struct nv_counters {
  int32_t pcount;        /* slots in use                                        */
  int32_t live;          /* slots with infront>0 (kept on the device)           */
  int32_t recon_count;   /* reconnections so far         (recon_count)          */
  int32_t remove_count;  /* premove removals so far      (remove_count)         */
  int32_t insert_count;  /* pinsert insertions so far                           */
  int32_t loop_kills;    /* loops cleared by loop_killer                        */
  int64_t tree_eval;     /* accepted tree interactions in the last velocity pass */
  int64_t tree_tests;    /* opening tests (nodes visited) in the last velocity pass */
  int32_t itime;         /* last completed step                                 */
  int32_t n_events;      /* events so far (the log keeps the first ones to fit)  */
  double t;              /* simulation time                                     */
  uint64_t event_hash;   /* order-sensitive digest of every event so far: equal
                            for two runs exactly when their event sequences agree
                            (up to 64-bit collisions), whether or not the log kept
                            them all                                            */
  int32_t wall_recon_count; /* wall_recon cuts so far (wall_recon_count)         */
  int32_t reserved;
} nv_counters;

/* One octree node (type node, src/tree.f90:20-32) as dumped in preorder by nv_tree_dump:
 * children in the reference's fbl..btr order, empty (pcount==0) children omitted. */
typedef struct nv_tree_node {
  double pos[3];      /* corner posx, posy, posz                              */
  double width;
  double cent[3];     /* centx, centy, centz                                  */
  double circ[3];
  int32_t pcount;
  int32_t depth;      /* root = 0                                             */
  int32_t leaf;       /* the member slot when pcount==1, else 0               */
  int32_t first_next; /* parray(1)%infront at construction (tree.f90:221,282) */
} nv_tree_node;

typedef struct nv_handle nv_handle;

/* ---- set-up ------------------------------------------------------------------------ */
/* Fill *p with the reference defaults of src/cdata.f90:76-127. */
int nv_params_default(nv_params *p);
/* Read a run.in file into *p (fields not named in the file keep their values), with the
 * semantics of read_run_file, src/cdata.f90:131-241: `key value` lines split at the first
 * blank, unknown keys ignored, and a value that fails to parse ends the read silently. */
int nv_read_run_file(const char *path, nv_params *p);
/* Check one system's parameters as init_setup does (src/initial.f90:14-146). */
int nv_check_params(const nv_params *p);

/* Create a handle for nsys systems.  params[s] holds system s's parameters and
 * capacity[s] its maximum slot count (pinsert appends beyond pcount up to it).
 * All systems share params[0].precision.  device selects the CUDA device. */
int nv_create(const nv_params *params, int32_t nsys, const int32_t *capacity,
              int32_t device, nv_handle **out);
int nv_destroy(nv_handle *h);

/* Copy one system's state to the device (replaces f(:), pcount); the clock and counters
 * are kept.  The links are checked before anything is written: a link outside 0..pcount, or
 * infront/behind disagreeing on an empty slot, returns NV_ERR_ARG and leaves the system's
 * device state exactly as it was. */
int nv_upload(nv_handle *h, int32_t sys, const nv_host_state *st);
/* Copy one system's state back.  Arrays must hold at least `cap` slots; st->pcount
 * receives the system's pcount (NV_ERR_ARG if it exceeds cap). */
int nv_download(nv_handle *h, int32_t sys, nv_host_state *st, int32_t cap);
int nv_set_clock(nv_handle *h, int32_t sys, double t, int32_t itime);
int nv_counters_get(nv_handle *h, int32_t sys, nv_counters *c);
/* Copy up to cap logged events of system sys; *n receives the number copied.  The log holds
 * T events (all systems); when more have happened (n_events of the counters is larger),
 * it is incomplete and event_hash is the record to compare. */
int nv_events_get(nv_handle *h, int32_t sys, nv_event *buf, int32_t cap, int32_t *n);

/* ---- stages: one call per reference procedure, applied to every system -------------- */
int nv_ghostp(nv_handle *h);            /* ghostp            src/boundary.f90:10-19      */
int nv_construct_tree(nv_handle *h);    /* construct_tree    src/tree.f90:38-157         */
int nv_pmotion(nv_handle *h);           /* pmotion           src/timestep.f90:16-45      */
int nv_pinsert(nv_handle *h);           /* pinsert           src/line.f90:18-96          */
int nv_pclose(nv_handle *h);            /* pclose_tree (tree_theta>0, src/tree.f90:190-244)
                                           or pclose (src/line.f90:135-160)             */
int nv_precon(nv_handle *h);            /* precon            src/reconnection.f90:11-61  */
int nv_wall_recon(nv_handle *h);        /* wall_recon        src/reconnection.f90:66-150 */
int nv_premove(nv_handle *h);           /* premove           src/line.f90:102-130        */
int nv_enforce_boundary(nv_handle *h);  /* enforce_boundary  src/boundary.f90:91-138     */
int nv_empty_tree(nv_handle *h);        /* empty_tree        src/tree.f90:160-186        */
int nv_end_step(nv_handle *h);          /* t=t+dt, NAN_finder: src/run.f90:49,64         */

/* Run nsteps whole time steps (the sequence of src/run.f90:26-64) on the device; the
 * step is captured once in a CUDA graph and replayed. */
int nv_step(nv_handle *h, int32_t nsteps);

/* One calc_velocity pass for every slot of system sys at the current positions
 * (ghostp, construct_tree when velocity is Tree, then src/timestep.f90:49-141).
 * u3 receives [3*pcount] velocities (0 for empty slots).  Nothing is moved. */
int nv_calc_velocity(nv_handle *h, int32_t sys, double *u3);

/* Dump system sys's current octree in preorder; *n receives the node count (records
 * beyond cap are not written).  Replaces reading vtree (src/tree.f90:34). */
int nv_tree_dump(nv_handle *h, int32_t sys, nv_tree_node *buf, int32_t cap, int32_t *n);

/* The reference's direct Biot-Savart velocity (calc_velocity with velocity 'BS',
 * src/timestep.f90:74-98 and :123-140, plain FP64) at n listed slots of system sys,
 * whatever scheme the system itself uses: the FP64 direct-sum yardstick for tree and
 * mixed-precision errors on large systems.  u3 receives [3*n] velocities in list order. */
int nv_calc_velocity_direct_at(nv_handle *h, int32_t sys, const int32_t *targets, int32_t n,
                               double *u3);

/* Cumulative device time (ms) per stage since creation: ms[0] ghosts, [1] tree build,
 * [2] velocity, [3] AB3 update, [4] topology, [5] whole steps, and the parts of [4]:
 * [6] pinsert, [7] pclose, [8] precon, [9] premove.  n = entries wanted (at most 10). */
int nv_stage_times(nv_handle *h, double *ms, int32_t n);
/* Mixed precision: interactions closer than factor*delta (leaves of the tree walk, segment
 * pairs of the direct sum) are evaluated in FP64; the rest in FP32, except interactions that
 * are ill-conditioned in FP32 (checked per interaction), which also run in FP64.  Default 2. */
int nv_set_near_factor(nv_handle *h, double factor);
/* Mixed precision: a far term runs in FP64 instead of FP32 when FP32 would lose digits:
 * |r||e| + r.e < angle |r||e| (the segment subtends nearly 180 degrees at the target),
 * |r x circ|^2 < line |circ|^2 min(|r|^2,|e|^2) (the target near the segment's line) or
 * |e|^2 < end max(|r|^2,|circ|^2) (near its far end), r, e: target to the segment's ends.
 * Defaults 0.1, 1e-3, 1e-2 (mixed vs FP64 velocity within 1e-7 RMS on the benchmark
 * tangles); smaller values trade accuracy for speed (angle 0 turns that guard off).  line
 * must be at least 1e-9: it also keeps the FP32 term away from its singularity (a target on
 * the segment). */
int nv_set_fp32_guards(nv_handle *h, double angle, double line, double end);
/* pinsert places the insertions of new points that the sweep reaches again by a fixed-point
 * iteration (default 6 rounds); a system that has not converged runs the serial sweep.
 * Both give the reference's result.  n = 0 runs the serial sweep for every system (0..64). */
int nv_set_insert_iterations(nv_handle *h, int32_t n);
/* The tree walks take each root's opening test from a parallel estimate of the root's centre
 * (the exact centre is a sequential sum over all slots, computed meanwhile on a side stream);
 * tests within the estimate's error bound are redone once the exact centre is known.
 * scale (>= 1, default 1) multiplies that bound; a very large scale sends every root test
 * through the exact path, for testing. */
int nv_set_root_band(nv_handle *h, double scale);
/* Split of the tree walks' work, so that a small system still fills the GPU.  Mixed
 * precision: the central image's walks (the deepest) are split over `parts` groups of the
 * root's children (1, 2, 4 or 8), each a work item of its own; the groups' sums are added in
 * group order.  Plain FP64: parts > 1 gives each target two threads, one summing the
 * unshifted image and one the 26 shifted ones, added in the reference's order (the result
 * is the same bit for bit); 1 keeps one thread per target.  0 (the default) picks the split
 * from the number of work items and the SM count. */
int nv_set_walk_parts(nv_handle *h, int32_t parts);
/* Event margins: how close the topology tests came to deciding the other way.  While on,
 * each system keeps the smallest |value - threshold| / threshold of pinsert's segment length
 * against delta (line.f90:41), premove's distance against .99 delta (line.f90:115), precon's
 * closestd against delta/2 (reconnection.f90:24) and precon's tangent dot product against 0.9
 * (reconnection.f90:34).  The pinsert margin covers exactly the lengths the reference
 * measures; the others cover every value the device evaluates, which includes every value
 * the reference evaluates, so they are never above the reference's.  nv_set_event_margins
 * switches them on (1) or off (0) and resets them; out[4] of nv_event_margins_get receives
 * them, 1e300 where no test ran. */
int nv_set_event_margins(nv_handle *h, int32_t on);
int nv_event_margins_get(nv_handle *h, int32_t sys, double *out);
/* One tangle over several GPUs (one process and handle per GPU, each holding the whole
 * state): nv_step_velocity runs a step up to and including the velocity pass,
 * nv_step_finish the rest (AB3 update, topology, wrap, clock), the two together exactly
 * nv_step(1).  With nv_set_walk_range a tree-walk system's velocity pass computes only the
 * targets at walk positions lo <= q < hi (the walk order: the live points in Morton order at
 * positions 1 .. live, then the empty slots).  The ends fall on warp boundaries: lo - 1 a
 * multiple of 32, and hi - 1 one too or hi = cap + 1 (the mixed walk's 32 targets of a warp
 * share their FP32 partial sums' flush points, which a warp cut in two would change); other
 * ends are refused with NV_ERR_ARG.  nv_velocity_pack copies the velocities of
 * positions lo .. lo+count-1 into a device buffer [count][3] and nv_velocity_unpack writes
 * them back, so that ranks split the positions, exchange their parts between the two halves
 * (an all-gather), and every rank continues with the full velocity field: the same step,
 * bit for bit, as one GPU's.  Default range: all positions. */
int nv_set_walk_range(nv_handle *h, int32_t sys, int32_t lo, int32_t hi);
int nv_velocity_pack(nv_handle *h, int32_t sys, int32_t lo, int32_t count, double *d_buf);
int nv_velocity_unpack(nv_handle *h, int32_t sys, int32_t lo, int32_t count, const double *d_buf);
int nv_step_velocity(nv_handle *h);
int nv_step_finish(nv_handle *h);
/* Data of the normal-fluid fields that the reference reads from files.  noisey_xflow: the n
 * multipliers of noise_file (src/normal_fluid.f90:156-162; the reference reads 100000), used
 * one per step from the first, wrapping after the last (randomise_normal_fluid, :340-348).
 * laizetDNS / turbDNS: the velocity grid as the reference reads it (setup_laizet :164-190,
 * setup_turbDNS :192-216): u holds the three components one after another, each nx*ny*nz
 * values in Fortran order (x fastest); laizetDNS needs nx,ny,nz = 128,129,84 and the 129
 * values of yp.dat (its u is halved as setup_laizet does), turbDNS 256,256,256 (yp NULL).
 * Point positions below the first grid node, which the reference reads out of its array,
 * wrap on the periodic axes and clamp on laizet's y axis. */
int nv_set_normal_fluid_noise(nv_handle *h, int32_t sys, const double *noise, int32_t n);
int nv_set_normal_fluid_grid(nv_handle *h, int32_t sys, const double *u, int32_t nx, int32_t ny, int32_t nz,
                             const double *yp);
/* Split of the plain FP64 direct sum's work.  64: one thread per target, each summing its
 * terms as it computes them.  1, 2, 4 or 8: a block of 128 threads per that many targets;
 * three warps compute the terms tile by tile and one lane per (target, component) adds them
 * in the reference's order, so a small system still fills the GPU (the result is the same
 * bit for bit).  0 (the default) takes 64 when the direct-sum systems' slots give at least
 * two blocks of 64 per SM, else the largest split with about four blocks per SM. */
int nv_set_direct_split(nv_handle *h, int32_t targets_per_block);
/* How pclose (systems with tree_theta 0, src/line.f90:135-160) finds each point's nearest
 * live non-neighbour: 0 (the default) from a cell list of the live points, rebuilt on every
 * reconnection step, searching rings of cells around the point until no unsearched cell can
 * hold a closer one; 1 by scanning every slot, as the reference does.  Both give the
 * reference's closest and closestd bit for bit (ties to the lowest slot). */
int nv_set_pclose_method(nv_handle *h, int32_t method);

/* Turn per-step stage timing on (default) or off.  With timing on, nv_step waits for each
 * step and adds its device time per stage to nv_stage_times; off, steps are queued back to
 * back. */
int nv_set_timing(nv_handle *h, int32_t on);
/* Number of kernel launches one step replays (kernel nodes of the step's CUDA graph,
 * library scan kernels included).  Captures the graph if needed. */
int nv_step_launches(nv_handle *h, int32_t *n);
/* Measure this device's FP64 fused-multiply-add rate (TFLOP/s, 2 flops per FMA) with a
 * short throughput kernel: the denominator of the FP64 CUDA-core roofline. */
int nv_measure_fp64_peak(int32_t device, double *tflops);
/* The same for FP32 FMAs (the far-field arithmetic of the mixed-precision path). */
int nv_measure_fp32_peak(int32_t device, double *tflops);

/* ---- velocity pass without library allocations ------------------------------------------
 * No counterpart in the reference: the Fortran program has no device memory at all.
 *
 * nv_calc_velocity_bs_static computes calc_velocity with velocity 'BS' in plain FP64 (the
 * same kernels and the same results as nv_calc_velocity on a BS system) for ONE system
 * whose filament state the caller already keeps in device memory, and it allocates
 * nothing: no cudaMalloc, no cudaFree, no handle.  It is meant for callers that must own
 * every device allocation themselves -- for example a CUDA Fortran or OpenACC host that
 * keeps f(:) in its own device arrays or memory pool and budgets that memory, or a time
 * loop that cannot afford the device-wide synchronisation that cudaMalloc/cudaFree imply.
 * All scratch (ghosts, segment records, work list, constants, error word) lives in one
 * static device array sized for NV_STATIC_MAX_SLOTS slots, about 5.6 MB, which every GPU
 * that loads this library holds until the process exits.
 *   p        parameters of the system (velocity must be NV_VEL_BS)
 *   pcount   slots, 1..NV_STATIC_MAX_SLOTS (larger systems: NV_ERR_CAPACITY)
 *   d_x3     device [3*pcount] positions, point-major as the host arrays above
 *   d_infront, d_behind   device [pcount] 1-based links, 0 = empty slot
 *   t        simulation time (mutual friction cut-offs)
 *   d_u3     device [3*pcount] output velocities (0 for empty slots)
 *   stream   a cudaStream_t (NULL = the default stream); the call waits for it to finish
 * Each call looks up the array's device address in the current context (so a device reset
 * between calls is safe), waits for `stream` to finish its work and then reads the device
 * error word back to the host before it returns; none of that is allowed while a stream is
 * being captured, so no call may be made during a stream capture.  A call that fails
 * (NV_ERR_ARG for links outside 0..pcount or infront/behind disagreeing on an empty slot,
 * NV_ERR_TIMEOUT for a device wait that gave up) leaves d_u3 unwritten.  Every call uses the
 * same array and leaves its contents behind; calls whose work overlaps on the GPU (two host
 * threads, or two streams) race on it and must be serialised by the caller. */
#define NV_STATIC_MAX_SLOTS 32768
int nv_calc_velocity_bs_static(const nv_params *p, int32_t pcount, const double *d_x3,
                               const int32_t *d_infront, const int32_t *d_behind, double t,
                               double *d_u3, void *stream);

/* ---- diagnostics, snapshots and restart files (src/diagnostic.f90, src/output.f90) ----- */
/* One row of data/ts.log (print_info, src/output.f90:20-44) and the values behind it.  The
 * velocity and curvature figures come from the last nv_calculate_diagnostics, avg_sep and
 * total_length from the last pinsert, the counters from the system's state. */
typedef struct nv_ts_row {
  int32_t itime;             /* step of the row (ts.log prints itime/shots)                    */
  int32_t live;              /* count(f(:)%infront>0)                                          */
  int32_t recon_count;
  int32_t wall_recon_count;  /* wall_recon cuts so far (wall_recon_count)                      */
  int32_t remove_count;
  int32_t reserved;
  int64_t tree_eval;         /* accepted tree interactions of the last velocity pass (the
                                reference's counter is a default integer and wraps past 2^31) */
  double t;
  double delta;
  double avg_sep;            /* pinsert's average separation (ts.log prints avg_sep/delta)      */
  double total_length;       /* pinsert's summed segment length                                */
  double maxu, maxdu;        /* velocity_info: max |u|, max |u1 - u2| over every slot            */
  double mean_u_sup, mean_u_mf; /* velocity_info: sums of |u_sup|, |u_mf| over every slot / live */
  double kappa_bar, kappa_min, kappa_max; /* curv_info (kappa_min: huge(0.) if no curvature > 0) */
} nv_ts_row;

/* calculate_diagnostics (src/diagnostic.f90:9-74) for every system: ghostp, then
 * velocity_info, curv_info and stretching_rate as device reductions; the per-point curvature
 * and stretching are kept for snapshots.  The reference calls it when mod(itime,shots)==0;
 * the caller decides when.  Sums run in a fixed parallel order (within ~1e-13 relative of the
 * reference's sequential sums); maxima and minima are exact. */
int nv_calculate_diagnostics(nv_handle *h);
/* The ts.log row of system sys (NV_ERR_STATE before the first nv_calculate_diagnostics). */
int nv_ts_row_get(nv_handle *h, int32_t sys, nv_ts_row *row);
/* The row as print_info writes it to data/ts.log, format
 * (i6.4,f13.7,i10.1,i13.1,i13.1,f7.4,f13.6,f13.5,f13.5,f10.2,i13.1,i13.1) with itime/shots,
 * t, live, recon_count, wall_recon_count, avg_sep/delta, total_length, maxu, maxdu,
 * kappa_bar, remove_count, tree_eval; no newline.  cap: size of buf. */
int nv_format_ts_row(const nv_ts_row *row, int32_t shots, char *buf, int32_t cap);

/* Every field of type(qvort) (src/cdata.f90:19-31), for file I/O: point-major 3-vectors as
 * in nv_host_state. */
typedef struct nv_full_state {
  int32_t pcount;
  double *x, *u, *u1, *u2, *u_mf, *u_sup;  /* [3*pcount]                               */
  double *curv, *stretch;                  /* [pcount]                                 */
  double *ghosti, *ghostb;                 /* [3*pcount]                               */
  int32_t *infront, *behind, *closest;     /* [pcount]                                 */
  double *closestd;                        /* [pcount]                                 */
  int32_t *wpinned;                        /* [3*pcount] (NULL: zero)                  */
  int32_t *pinnedi, *pinnedb;              /* [pcount] logical 0/1 (NULL: .false.)     */
} nv_full_state;

/* Every field of system sys (u_sup and u_mf of its last velocity pass, curv and stretch of
 * its last diagnostics); arrays of at least cap slots; st->pcount receives pcount. */
int nv_download_full(nv_handle *h, int32_t sys, nv_full_state *st, int32_t cap);
/* nv_upload plus u_sup, u_mf, curv and stretch (NULL: zero). */
int nv_upload_full(nv_handle *h, int32_t sys, const nv_full_state *st);

/* printf (src/output.f90:47-70): the stream file data/var%04d.log that the MATLAB tools read
 * (bin/vortex/vortex_load.m): t, pcount, x(1..3), infront, u(1..3), u_mf(1..3), curv,
 * stretch, each over all pcount slots, little-endian, no record markers. */
int nv_write_snapshot(nv_handle *h, int32_t sys, const char *path);
/* data_dump (src/output.f90:85-94): data/var.dat as gfortran's unformatted sequential write
 * of pcount, recon_count, itime, t and f, each a record framed by 4-byte length markers; f
 * holds pcount type(qvort) records of 248 bytes (reals 8, integers and logicals 4).  Files
 * whose f record would exceed 2^31-1 bytes (8.6M points) are refused (NV_ERR_UNSUPPORTED). */
int nv_write_dump(nv_handle *h, int32_t sys, const char *path);
/* data_restore (src/initial.f90:151-166): reads a var.dat into system sys (state, t, itime,
 * recon_count); the next step is itime+1.  NV_ERR_IO if the file cannot be read or is not such
 * a file, NV_ERR_CAPACITY if its pcount exceeds the system's capacity, NV_ERR_ARG if it holds
 * pinned points and the system has no solid wall. */
int nv_restore_dump(nv_handle *h, int32_t sys, const char *path);
/* The same formats between host arrays and files, without a handle or a GPU. */
int nv_snapshot_write_file(const nv_full_state *st, double t, const char *path);
int nv_dump_write_file(const nv_full_state *st, int32_t recon_count, int32_t itime, double t, const char *path);
/* Reads a var.dat: *pcount_out receives its pcount; the arrays of st (NULL to skip one) are
 * filled when they hold at least cap >= pcount slots (else NV_ERR_ARG after setting the count). */
int nv_dump_read_file(const char *path, nv_full_state *st, int32_t cap, int32_t *pcount_out, int32_t *recon_count,
                      int32_t *itime, double *t);

/* nv_upload / nv_download for `count` distinct systems sys[i] with states st[i] (nv_download_many:
 * arrays of cap[i] slots): the same results as count single calls, with every system's
 * copies and kernels in flight together and one wait.  Each optional array is given for every
 * listed system or for none.  A rejected link check changes no system.  Systems with solid
 * walls, or pinned arrays, go through the single calls one by one.  With page-locked host
 * arrays (nv_host_register) the copies run asynchronously at full bandwidth. */
int nv_upload_many(nv_handle *h, int32_t count, const int32_t *sys, const nv_host_state *st);
int nv_download_many(nv_handle *h, int32_t count, const int32_t *sys, nv_host_state *st, const int32_t *cap);
/* Every system of the handle at once with the host arrays packed: system s's rows follow
 * system s-1's, from row pcounts[0] + ... + pcounts[s-1] (links system-local, 1-based, as in
 * nv_upload); all->pcount is the total.  One copy per array each way.  nv_download_packed
 * fills pcounts[nsys] and all->pcount (arrays of cap_rows rows).  Systems with solid walls
 * and pinned arrays are refused (NV_ERR_UNSUPPORTED): use the per-system calls. */
int nv_upload_packed(nv_handle *h, const nv_host_state *all, const int32_t *pcounts);
int nv_download_packed(nv_handle *h, nv_host_state *all, int64_t cap_rows, int32_t *pcounts);
/* Page-locks (cudaHostRegister) or releases a host range, e.g. the caller's f(:) arrays. */
int nv_host_register(void *p, size_t bytes);
int nv_host_unregister(void *p);

/* Diagnostic counters of system sys for the last step, for profiling the topology stages:
 * [0] pinsert candidates, [1] insertions, [2] steps that needed the serial pinsert sweep
 * (cumulative), [3] precon candidates, [4] premove candidates, [5] insertions made by new
 * points that the sweep reached again, [6] fixed-point iterations the parallel pinsert took
 * to place them (a system that has not converged after the last one runs the serial sweep),
 * [7] premove visits on the live state: extra slots << 32 | candidates, and for the mixed
 * tree walk of the last velocity evaluation: [8] terms evaluated in FP64 (near leaves and
 * terms FP32 would evaluate badly), [9] opening tests decided in FP64 (FP32 too close to
 * call), [10] terms evaluated in FP32, [11] unused.  n = entries wanted (<= 12). */
int nv_diagnostics(nv_handle *h, int32_t sys, int64_t *out, int32_t n);

/* Block until the handle's stream is idle and report any device-side error. */
int nv_sync(nv_handle *h);

const char *nv_last_error(void);
const char *nv_version(void);

#ifdef __cplusplus
}
#endif
#endif /* NUVORT_GPU_H */
