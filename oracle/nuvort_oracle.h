/*
 * nuvort_oracle.h -- CPU oracle for the NuVort filament-velocity path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a line-by-line C++ restatement of the reference
 * Fortran routines (src/timestep.f90, src/tree.f90, src/derivatives.f90, src/general.f90,
 * src/boundary.f90, src/line.f90, src/reconnection.f90, src/normal_fluid.f90,
 * src/initial.f90, src/run.f90).  Only tests, the smoke check and the CPU-baseline leg of
 * the benchmark may load it, and only as the checker.  The product (libnuvort_gpu.so)
 * never calls it.
 *
 * Parity status: UNPINNED.  The reference ships no tests, golden vectors or known-answer
 * fixtures, and it cannot be compiled here (no Fortran compiler).  The restatement is
 * checked against the one analytic answer the reference prints (the ring self-velocity
 * of src/initial_cond.f90:16) and against invariants; see oracle/README.md.
 *
 * The API mirrors include/nuvort_gpu.h (same parameter, state, event and counter
 * records) for a single system, so tests feed both sides identical inputs.
 */
#ifndef NUVORT_ORACLE_H
#define NUVORT_ORACLE_H

#include "../include/nuvort_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_handle or_handle;

/* One octree node in preorder (children in the reference's fbl..btr order), empty
 * (pcount==0) children omitted.  Matches the GPU library's nv_tree_node. */
typedef struct or_tree_node {
  double pos[3];    /* corner posx,posy,posz                                  */
  double width;
  double cent[3];   /* centx,centy,centz                                      */
  double circ[3];
  int32_t pcount;
  int32_t depth;    /* root = 0                                               */
  int32_t leaf;     /* the member slot when pcount==1, else 0                 */
  int32_t first_next; /* parray(1)%infront snapshot (src/tree.f90:221,282)  */
} or_tree_node;

int or_create(const nv_params *p, or_handle **out);
int or_destroy(or_handle *h);
int or_upload(or_handle *h, const nv_host_state *st);
int or_download(or_handle *h, nv_host_state *st, int32_t cap);
int or_set_clock(or_handle *h, double t, int32_t itime);
int or_counters_get(or_handle *h, nv_counters *c);
int or_events_get(or_handle *h, nv_event *buf, int32_t cap, int32_t *n);

int or_ghostp(or_handle *h);
int or_construct_tree(or_handle *h);
int or_pmotion(or_handle *h);
int or_pinsert(or_handle *h);
int or_pclose(or_handle *h);
int or_precon(or_handle *h);
int or_wall_recon(or_handle *h);
/* Event margins, as nv_set_event_margins / nv_event_margins_get define them. */
int or_set_event_margins(or_handle *h, int32_t on);
int or_event_margins_get(or_handle *h, double *out);
int or_premove(or_handle *h);
int or_enforce_boundary(or_handle *h);
int or_empty_tree(or_handle *h);
int or_end_step(or_handle *h);
int or_step(or_handle *h, int32_t nsteps);

/* calc_velocity for every slot (ghostp and construct_tree first, as nv_calc_velocity). */
int or_calc_velocity(or_handle *h, double *u3);
/* calc_velocity for the listed slots only, with the given velocity scheme (NV_VEL_*),
 * at the current positions; ghosts (and the tree, for NV_VEL_TREE) are rebuilt first.
 * Used as the FP64 direct-sum error oracle on subsamples and for the CPU baseline. */
int or_calc_velocity_targets(or_handle *h, int32_t velocity, const int32_t *targets,
                             int32_t n, double *u3);
/* Data of the file-based normal fluids, as nv_set_normal_fluid_noise / _grid take it. */
int or_set_normal_fluid_noise(or_handle *h, const double *noise, int32_t n);
int or_set_normal_fluid_grid(or_handle *h, const double *u, int32_t nx, int32_t ny, int32_t nz, const double *yp);
/* calculate_diagnostics (src/diagnostic.f90:9-74) and the values print_info writes
 * (src/output.f90:20-44), with sequential sums as the reference's sum intrinsic makes them. */
int or_calculate_diagnostics(or_handle *h);
int or_ts_row_get(or_handle *h, nv_ts_row *row);
/* Every kept field of f(:), and the upload of one (u_sup, u_mf, curv, stretch included). */
int or_download_full(or_handle *h, nv_full_state *st, int32_t cap);
int or_upload_full(or_handle *h, const nv_full_state *st);
/* printf (src/output.f90:47-70) and data_dump (src/output.f90:85-94) files. */
int or_write_snapshot(or_handle *h, const char *path);
int or_write_dump(or_handle *h, const char *path);
/* Dump the current tree (built by or_construct_tree) in preorder. */
int or_tree_dump(or_handle *h, or_tree_node *buf, int32_t cap, int32_t *n);

void or_set_threads(int32_t n);
int32_t or_get_threads(void);
const char *or_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
