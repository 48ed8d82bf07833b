// handle.cuh -- host-side definition of nv_handle and the kernel launchers.
#pragma once

#include <string>
#include <vector>

#include "common.cuh"
#include "mixed.cuh"

struct TreeBuffers;  // tree.cu
struct TopoBuffers;  // topo.cu

enum { ST_GHOST = 0, ST_TREE, ST_VELOCITY, ST_AB3, ST_TOPO, ST_STEP, ST_INSERT, ST_CLOSE, ST_RECON, ST_REMOVE, ST_COUNT };

struct nv_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // concurrent branch of the tree build (walk order, root sums)
  cudaStream_t side2 = nullptr;  // second branch (sums of the large shallow nodes)
  cudaEvent_t fork2_ev = nullptr, join2_ev = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr, sort_ev = nullptr;
  int nsys = 0;
  int precision = NV_PREC_FP64;
  std::vector<nv_params> params;
  std::vector<SysConst> sc;
  std::vector<int> cap, base;
  long long T = 0;  // slots including one dummy per system
  int max_cap = 0;

  // device state
  SysConst *d_sc = nullptr;
  SysDyn *d_dyn = nullptr;
  double *x = nullptr, *u = nullptr, *u1 = nullptr, *u2 = nullptr;
  double *gi = nullptr, *gb = nullptr, *closestd = nullptr;
  int *nxt = nullptr, *prv = nullptr, *closest = nullptr, *sys_of = nullptr;
  double4 *seg = nullptr;   // FP64 segment records, 2 per slot
  float4 *seg32 = nullptr;  // FP32 segment records, 3 per slot (mixed precision)
  double *partial = nullptr; // per-image partial sums [image][component][slot] (mixed precision)
  std::vector<void *> nf_buffers;  // normal-fluid noise and grid data (nv_set_normal_fluid_*)
  double *usm = nullptr;     // f(:)%u_sup, f(:)%u_mf of the last velocity pass [6][T]
  int *pin = nullptr;        // solid walls: pinned record per slot [T] (pin_* in common.cuh)
  double *umir = nullptr;    // solid walls: the tree's mirror sums per slot [3][T]
  bool any_solid = false, any_mirror = false;  // a system with solid walls (with tree walks)
  double *cs = nullptr;      // f(:)%curv, f(:)%stretch of the last diagnostics [2][T]
  struct DiagRec *d_drec = nullptr;  // per system: the last diagnostics' reductions
  double *stage = nullptr;   // nv_upload / nv_download staging: host arrays as they are, 3 x (largest capacity + 1) doubles
  double *bstage = nullptr;  // nv_upload_many / nv_download_many staging: every listed system's array at once, 3T doubles
  int4 *d_btab = nullptr;    // their per-system table (base, rows, n, offset), nsys entries
  int *d_bcheck = nullptr;   // their link checks, two ints per system
  int *d_upck = nullptr;     // nv_upload checks: [0] link errors (1 out of range, 2 empty-slot mismatch), [1] live slots
  int4 *d_work_img = nullptr;  // (system, image, first slot) items of the mixed direct sum
  int n_work_img = 0;
  int4 *d_work_timg = nullptr; // same for the mixed tree walk
  int n_work_timg = 0;
  double near_factor = 2.0;    // near field: pairs closer than near_factor*delta run in FP64
  Fp32Guards guards;
  double root_band_scale = 1.0;  // scale of the root centre estimate's error bound
  int ins_iters = 6;  // fixed-point iterations of the parallel pinsert; 0: serial sweep only
  int tree_sys0 = 0;           // first system that walks the tree (its theta0 builds the mixed nodes)
  int walk_parts = 0;          // central image of the mixed tree walk split over this many root-child groups (0: automatic)
  int walk_parts_used = 1;     // the split the work list was built with
  unsigned links_epoch = 0;    // bumped by every stage that relinks points (pinsert, precon, premove, upload)
  unsigned *d_err = nullptr;
  DevEvent *d_events = nullptr;
  int *d_event_count = nullptr;
  int event_cap = 0;

  // work lists: blocks of target slots, (system, first global slot)
  int2 *d_work_direct = nullptr;
  int n_work_direct = 0;
  int2 *d_work_tree = nullptr;
  int n_work_tree = 0;
  int2 *d_work_lia = nullptr;
  int n_work_lia = 0;
  int direct_tb = 64;  // targets per block of the direct sum and of the FP64 tree walk (which assumes 64)
  int pclose_method = 0;  // nv_set_pclose_method: 0 cell list, 1 every slot (brute force)
  int direct_split = 0;  // nv_set_direct_split: 0 automatic, 64 one thread per target, 1/2/4/8 split kernel
  int direct_g = 64;     // targets per block of the direct sum in use
  int2 *d_work_split = nullptr;  // (system, first slot) items of direct_g slots for the split kernel
  int n_work_split = 0;
  bool any_tree = false, any_direct = false, any_lia = false;

  TreeBuffers *tree = nullptr;
  TopoBuffers *topo = nullptr;

  // CUDA graph of one whole step
  cudaGraphExec_t graph_exec = nullptr;
  bool graph_valid = false;
  int step_kernels = 0;

  // stage timing
  bool timing = true;
  cudaEvent_t ev[2 * ST_COUNT] = {};
  double stage_ms[ST_COUNT] = {};
  cudaError_t timing_error = cudaSuccess;

  // host mirrors
  std::vector<SysDyn> h_dyn;
};

// launchers (each enqueues on h->stream)
void launch_begin_step(nv_handle *h);
void launch_ghost(nv_handle *h);
void launch_velocity(nv_handle *h);
void launch_ab3(nv_handle *h);
void launch_wrap(nv_handle *h, int mode);  // bit 1 wrap, bit 2 NaN check
void launch_end_step(nv_handle *h);

// direct sum (direct.cu)
int direct_targets_per_block(const nv_handle *h, long long slots);
void launch_direct(nv_handle *h);
void launch_direct_targets(nv_handle *h, int sys, const int *d_targets, int n, double *d_u3);
// mixed precision (mixed.cu)
void launch_direct_mixed(nv_handle *h);
void launch_mixed_combine(nv_handle *h, int which);
void launch_tree_walk_mixed(nv_handle *h);
const int *tree_iperm(nv_handle *h);  // slot -> walk position of the last tree build (or null)
const int *tree_perm(nv_handle *h);   // walk position (global: base + q) -> slot
// tree (tree.cu)
constexpr int kMaxWalkParts = 8;  // the central image's walk splits over at most the root's 8 children
int n_sms_host();                  // SMs of the current device
void tree_alloc(nv_handle *h);
void tree_free(nv_handle *h);
void launch_tree_build(nv_handle *h);
void launch_tree_walk(nv_handle *h);
void launch_closest_tree(nv_handle *h);
void join_root_sums(nv_handle *h);     // the main stream waits for the roots' exact sums
void launch_walk_fixup(nv_handle *h);  // deferred root tests of the last tree walk
int tree_dump(nv_handle *h, int sys, void *buf, int cap, int *n);
// diagnostics (diag.cu): ghosts, per-point curvature and stretching, per-system reductions
int diag_launch(nv_handle *h);
// topology (topo.cu)
void topo_alloc(nv_handle *h);
void topo_free(nv_handle *h);
void launch_pinsert(nv_handle *h);
void launch_pclose(nv_handle *h, bool only_brute);
void launch_precon(nv_handle *h);
void launch_premove(nv_handle *h);
// solid walls (solid.cu): the serial topology stages of the systems with solid walls
void launch_solid_pinsert(nv_handle *h);
void launch_solid_precon(nv_handle *h);
void launch_wall_recon(nv_handle *h);
void launch_solid_premove(nv_handle *h);

int set_error(int code, const std::string &msg);
// status code and message for a non-zero device error word (DERR_* bits)
int status_from_device_bits(unsigned bits, std::string &msg);
SysConst sysconst_for(const nv_params &p, int base, int cap);
void launch_ghost_raw(cudaStream_t st, const SysConst *sc, const SysDyn *dyn, const int *sys_of, const double *x,
                      const int *nxt, const int *prv, double *gi, double *gb, double4 *seg, long long T,
                      unsigned *err);
void launch_direct_raw(cudaStream_t st, const SysConst *sc, const SysDyn *dyn, const int2 *work, int nwork,
                       const double *x, const double *gi, const double *gb, const int *nxt, const int *prv,
                       const double4 *seg, double *u, long long T, unsigned *err);
int check_cuda(cudaError_t e, const char *what);
#define NV_CUDA(call)                                   \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return check_cuda(_e, #call); \
  } while (0)

inline int grid_for(long long n, int tb) { return (int)((n + tb - 1) / tb); }
