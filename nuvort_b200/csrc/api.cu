// api.cu -- the extern "C" boundary of libnuvort_gpu (include/nuvort_gpu.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "handle.cuh"

namespace {
thread_local std::string g_err;
}

SysConst sysconst_for(const nv_params &p, int base, int cap);

int set_error(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

int check_cuda(cudaError_t e, const char *what) {
  return set_error(NV_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

const char *kVersion = "nuvort_b200 0.1.0 (sm_100a)";

// ---- host state <-> device slots (nv_upload / nv_download) -----------------------------------
// The host arrays (point k of 1..n at row k-1, components interleaved, links 1-based within
// the system) are copied as they are into the staging buffer; these kernels move them to and
// from the system's slots base+1..base+cap (structure of arrays, global links).
__global__ void k_put_rows(double *__restrict__ dev, long long T, int base, int rows, int n, int comps,
                           const double *__restrict__ host) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;  // slot within the system, 0 = dummy
  if (k >= rows) return;
  for (int c = 0; c < comps; ++c)
    dev[c * T + base + k] = host && k >= 1 && k <= n ? host[(long long)comps * (k - 1) + c] : 0.0;
}

// links already checked by k_upload_check
__global__ void k_put_links(int *__restrict__ dev, int base, int rows, int n, const int *__restrict__ host) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= rows) return;
  const int v = host && k >= 1 && k <= n ? host[k - 1] : 0;
  dev[base + k] = v ? base + v : 0;
}

// The staged host links (infront, behind and, if given, closest: n each), before any of them
// reaches the system's slots: every link in 0..n, and an empty slot carries an empty link
// pair.  Counts the live slots.
__global__ void k_upload_check(const int *__restrict__ inf, const int *__restrict__ beh,
                               const int *__restrict__ clo, int n, int *__restrict__ check) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = k < n;
  bool live = false;
  if (in) {
    const int a = inf[k], b = beh[k], c = clo ? clo[k] : 0;
    if (a < 0 || a > n || b < 0 || b > n || c < 0 || c > n) atomicOr(&check[0], 1);
    if ((a == 0) != (b == 0)) atomicOr(&check[0], 2);
    live = a > 0;
  }
  const unsigned bl = __ballot_sync(0xffffffffu, live);
  if ((threadIdx.x & 31) == 0 && bl) atomicAdd(&check[1], __popc(bl));
}

// Pinned records from the staged host arrays (wpinned [3n], pinnedi [n], pinnedb [n]; null:
// not pinned) into the system's slots, empty beyond n.
__global__ void k_put_pin(int *__restrict__ pin, int base, int rows, int n, const int *__restrict__ wp,
                          const int *__restrict__ pi, const int *__restrict__ pb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= rows) return;
  int v = 0;
  if (k >= 1 && k <= n) {
    int w[3] = {0, 0, 0};
    if (wp)
      for (int c = 0; c < 3; ++c) w[c] = wp[3 * (k - 1) + c];
    v = pin_encode(pi && pi[k - 1], pb && pb[k - 1], w);
  }
  pin[base + k] = v;
}

__global__ void k_get_pin(const int *__restrict__ pin, int base, int n, int *__restrict__ wp, int *__restrict__ pi,
                          int *__restrict__ pb) {
  const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k > n) return;
  const int v = pin ? pin[base + k] : 0;
  if (wp)
    for (int c = 0; c < 3; ++c) wp[3 * (k - 1) + c] = pin_w(v, c);
  if (pi) pi[k - 1] = pin_i(v);
  if (pb) pb[k - 1] = pin_b(v);
}

__global__ void k_get_rows(const double *__restrict__ dev, long long T, int base, int n, int comps,
                           double *__restrict__ host) {
  const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k > n) return;
  for (int c = 0; c < comps; ++c) host[(long long)comps * (k - 1) + c] = dev[c * T + base + k];
}

__global__ void k_get_links(const int *__restrict__ dev, int base, int n, int *__restrict__ host) {
  const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k > n) return;
  const int v = dev[base + k];
  host[k - 1] = v ? v - base : 0;
}

// ---- batched transfers: one launch per array over every listed system ---------------------
// tab[i] = (base, rows = cap + 1, n, offset of the system's rows in the staging buffer);
// blockIdx.y is the system, blockIdx.x covers its rows.
__global__ void k_upload_check_many(const int4 *__restrict__ tab, const int *__restrict__ inf,
                                    const int *__restrict__ beh, const int *__restrict__ clo,
                                    int *__restrict__ check) {
  const int4 t = tab[blockIdx.y];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool live = false;
  if (k < t.z) {
    const int a = inf[t.w + k], b = beh[t.w + k], c = clo ? clo[t.w + k] : 0;
    if (a < 0 || a > t.z || b < 0 || b > t.z || c < 0 || c > t.z) atomicOr(&check[2 * blockIdx.y], 1);
    if ((a == 0) != (b == 0)) atomicOr(&check[2 * blockIdx.y], 2);
    live = a > 0;
  }
  const unsigned bl = __ballot_sync(0xffffffffu, live);
  if ((threadIdx.x & 31) == 0 && bl) atomicAdd(&check[2 * blockIdx.y + 1], __popc(bl));
}
__global__ void k_put_links_many(int *__restrict__ dev, const int4 *__restrict__ tab, const int *__restrict__ host) {
  const int4 t = tab[blockIdx.y];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= t.y) return;
  const int v = host && k >= 1 && k <= t.z ? host[t.w + k - 1] : 0;
  dev[t.x + k] = v ? t.x + v : 0;
}
__global__ void k_put_rows_many(double *__restrict__ dev, long long T, const int4 *__restrict__ tab, int comps,
                                const double *__restrict__ host) {
  const int4 t = tab[blockIdx.y];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= t.y) return;
  for (int c = 0; c < comps; ++c)
    dev[c * T + t.x + k] = host && k >= 1 && k <= t.z ? host[(long long)comps * (t.w + k - 1) + c] : 0.0;
}
__global__ void k_get_rows_many(const double *__restrict__ dev, long long T, const int4 *__restrict__ tab, int comps,
                                double *__restrict__ host) {
  const int4 t = tab[blockIdx.y];
  const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k > t.z) return;
  for (int c = 0; c < comps; ++c) host[(long long)comps * (t.w + k - 1) + c] = dev[c * T + t.x + k];
}
__global__ void k_get_links_many(const int *__restrict__ dev, const int4 *__restrict__ tab, int *__restrict__ host) {
  const int4 t = tab[blockIdx.y];
  const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k > t.z) return;
  const int v = dev[t.x + k];
  host[t.w + k - 1] = v ? v - t.x : 0;
}

// velocities of walk positions [lo, hi) of system s to / from a packed buffer [count][3]
__global__ void k_vel_pack(const double *__restrict__ U, long long T, const int *__restrict__ perm, int base, int lo,
                           int count, double *__restrict__ buf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int g = perm[base + lo + i];
  for (int c = 0; c < 3; ++c) buf[3 * (long long)i + c] = U[c * T + g];
}
__global__ void k_vel_unpack(double *__restrict__ U, long long T, const int *__restrict__ perm, int base, int lo,
                             int count, const double *__restrict__ buf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int g = perm[base + lo + i];
  for (int c = 0; c < 3; ++c) U[c * T + g] = buf[3 * (long long)i + c];
}

int err_code_from_bits(unsigned bits, std::string &msg) {
  if (bits & DERR_SINGULAR) { msg = "tree_walk: singularity in BS (tree) velocity field (dist<epsilon)"; return NV_ERR_SINGULAR; }
  if (bits & DERR_TREE_DEPTH) { msg = "octree deeper than NV_TREE_MAX_DEPTH levels (coincident points?)"; return NV_ERR_TREE_DEPTH; }
  if (bits & DERR_TREE_NODES) { msg = "octree node buffer exhausted"; return NV_ERR_TREE_DEPTH; }
  if (bits & DERR_WALK) { msg = "tree walk visited more nodes than the octree holds (a malformed tree)"; return NV_ERR_TREE_DEPTH; }
  if (bits & DERR_NAN) { msg = "there is a NAN in the (filament) f%x array"; return NV_ERR_NAN; }
  if (bits & DERR_EMPTY) { msg = "pinsert: vortex line length is 0, run over"; return NV_ERR_EMPTY; }
  if (bits & DERR_CAPACITY) { msg = "pinsert: system capacity exhausted"; return NV_ERR_CAPACITY; }
  if (bits & DERR_QUEUE) { msg = "topology resolver work queue overflow"; return NV_ERR_QUEUE; }
  if (bits & DERR_TIMEOUT) { msg = "device wait gave up (bounded spin exceeded)"; return NV_ERR_TIMEOUT; }
  msg = "unknown device error";
  return NV_ERR_CUDA;
}

}  // namespace

int status_from_device_bits(unsigned bits, std::string &msg) { return err_code_from_bits(bits, msg); }

namespace {

// Synchronise the handle's stream and turn the device error word into a status.
int finish(nv_handle *h) {
  NV_CUDA(cudaStreamSynchronize(h->stream));
  NV_CUDA(cudaGetLastError());
  unsigned bits = 0;
  NV_CUDA(cudaMemcpy(&bits, h->d_err, sizeof bits, cudaMemcpyDeviceToHost));
  if (bits) {
    std::string msg;
    int code = err_code_from_bits(bits, msg);
    return set_error(code, msg);
  }
  return NV_OK;
}

int set_device(nv_handle *h) {
  NV_CUDA(cudaSetDevice(h->device));
  return NV_OK;
}

// A normal fluid that needs data the caller has not given (nv_set_normal_fluid_*).
int nf_missing(const nv_handle *h) {
  for (int s = 0; s < h->nsys; ++s) {
    const SysConst &c = h->sc[s];
    if (!c.mf_on) continue;
    if (c.nf_kind == NV_NF_NOISEY_XFLOW && !c.nf_noise)
      return set_error(NV_ERR_STATE, "noisey_xflow needs its noise samples (nv_set_normal_fluid_noise)");
    if ((c.nf_kind == NV_NF_LAIZET_DNS || c.nf_kind == NV_NF_TURB_DNS) && !c.nf_grid)
      return set_error(NV_ERR_STATE, "laizetDNS/turbDNS need their grid (nv_set_normal_fluid_grid)");
  }
  return NV_OK;
}


SysConst make_sysconst(const nv_params &p, int base, int cap) {
  SysConst s;
  std::memset(&s, 0, sizeof s);
  s.dt = p.dt;
  s.delta = p.delta;
  s.quant_circ = p.quant_circ;
  s.corea = p.corea;
  for (int c = 0; c < 3; ++c) s.box[c] = p.box_size[c];
  s.tree_theta = p.tree_theta;
  s.beta_pref = p.quant_circ / (4.0 * NV_PI);
  s.log_pref = 1.1 / p.corea;
  s.two_pi = 2 * NV_PI;
  s.alpha[0] = p.alpha[0];
  s.alpha[1] = p.alpha[1];
  // get_normal_velocity (normal_fluid.f90:92-117): uniform fields, plus super_velocity.
  double vn[3] = {0, 0, 0};
  if (p.normal_velocity == NV_NF_XFLOW) vn[0] = p.norm_vel_xflow;
  if (p.normal_velocity == NV_NF_UNIFORM)
    for (int c = 0; c < 3; ++c) vn[c] = p.norm_vel_vec[c];
  for (int c = 0; c < 3; ++c) s.vn[c] = vn[c] + p.super_velocity[c];
  for (int c = 0; c < 3; ++c) s.super_velocity[c] = p.super_velocity[c];
  s.normal_fluid_cutoff = p.normal_fluid_cutoff;
  s.t_zero_normal_fluid = p.t_zero_normal_fluid;
  s.nf_kind = p.normal_velocity;
  s.nf_a = p.norm_vel_xflow;
  s.nf_omega = p.norm_shear_omega;
  s.bsize = std::max(p.box_size[0], std::max(p.box_size[1], p.box_size[2]));
  // create_periodic_loop_array (boundary.f90:143-175): i,j,k in -1..1, k fastest.
  int n = 0;
  for (int i = -1; i <= 1; ++i)
    for (int j = -1; j <= 1; ++j)
      for (int k = -1; k <= 1; ++k) {
        double ii, jj, kk;
        if (p.boundary[0] == NV_BC_PERIODIC) ii = i * p.box_size[0];
        else { if (i != 0) continue; ii = 0; }
        if (p.boundary[1] == NV_BC_PERIODIC) jj = j * p.box_size[1];
        else { if (j != 0) continue; jj = 0; }
        if (p.boundary[2] == NV_BC_PERIODIC) kk = k * p.box_size[2];
        else { if (k != 0) continue; kk = 0; }
        if (ii == 0 && jj == 0 && kk == 0) continue;
        s.shift[n][0] = ii;
        s.shift[n][1] = jj;
        s.shift[n][2] = kk;
        ++n;
      }
  s.n_shift = n;
  // create_mirror_loop_array (boundary.f90:180-212): the reflections -1..1 on the solid axes,
  // k fastest, without (0,0,0)
  int nm = 0;
  for (int i = -1; i <= 1; ++i)
    for (int j = -1; j <= 1; ++j)
      for (int k = -1; k <= 1; ++k) {
        const int r[3] = {i, j, k};
        bool ok = true;
        for (int c = 0; c < 3; ++c)
          if (p.boundary[c] != NV_BC_SOLID && r[c] != 0) ok = false;
        if (!ok || (i == 0 && j == 0 && k == 0)) continue;
        for (int c = 0; c < 3; ++c) s.mirror[nm][c] = r[c];
        ++nm;
      }
  s.n_mirror = nm;
  for (int c = 0; c < 3; ++c) s.solid[c] = p.boundary[c] == NV_BC_SOLID;
  s.velocity = p.velocity;
  for (int c = 0; c < 3; ++c) s.periodic[c] = p.boundary[c] == NV_BC_PERIODIC;
  s.tree_extra_correction = p.tree_extra_correction != 0;
  s.mf_on = (std::fabs(p.alpha[0]) > NV_EPS) || (std::fabs(p.alpha[1]) > NV_EPS);
  s.recon_shots = p.recon_shots > 0 ? p.recon_shots : 1;
  s.nan_test = p.nan_test != 0;
  s.use_tree = p.tree_theta > 0;
  s.sched_tree = p.velocity == NV_VEL_TREE;
  s.base = base;
  s.cap = cap;
  s.walk_lo = 1;
  s.walk_hi = cap + 1;
  return s;
}

template <class T>
int dalloc(T **p, size_t n) {
  NV_CUDA(cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T)));
  NV_CUDA(cudaMemset(*p, 0, std::max<size_t>(n, 1) * sizeof(T)));
  return NV_OK;
}

void build_worklist(nv_handle *h, int which, std::vector<int2> &w) {
  w.clear();
  const int tb = h->direct_tb;
  for (int s = 0; s < h->nsys; ++s) {
    const SysConst &sc = h->sc[s];
    int kind = sc.velocity == NV_VEL_LIA ? 0 : (sc.sched_tree ? 2 : 1);
    if (kind != which) continue;
    for (int k = 1; k <= h->cap[s]; k += tb) w.push_back(make_int2(s, sc.base + k));
  }
}

int upload_worklist(int2 **dptr, int *n, const std::vector<int2> &w) {
  if (*dptr) cudaFree(*dptr);
  *dptr = nullptr;
  *n = (int)w.size();
  if (w.empty()) return NV_OK;
  NV_CUDA(cudaMalloc((void **)dptr, w.size() * sizeof(int2)));
  NV_CUDA(cudaMemcpy(*dptr, w.data(), w.size() * sizeof(int2), cudaMemcpyHostToDevice));
  return NV_OK;
}

int upload_worklist4(int4 **dptr, int *n, const std::vector<int4> &w) {
  if (*dptr) cudaFree(*dptr);
  *dptr = nullptr;
  *n = (int)w.size();
  if (w.empty()) return NV_OK;
  NV_CUDA(cudaMalloc((void **)dptr, w.size() * sizeof(int4)));
  NV_CUDA(cudaMemcpy(*dptr, w.data(), w.size() * sizeof(int4), cudaMemcpyHostToDevice));
  return NV_OK;
}

// (system, image, first slot, part) items over every image of every system of one kind.
// With parts > 1 the central image (the deepest walks) is listed once per part, each part
// walking a group of the root's children; all central items come first.
void build_image_worklist(nv_handle *h, int which, int tb, std::vector<int4> &w, int parts = 1) {
  w.clear();
  for (int pass = 0; pass < 2; ++pass)
    for (int s = 0; s < h->nsys; ++s) {
      const SysConst &sc = h->sc[s];
      int kind = sc.velocity == NV_VEL_LIA ? 0 : (sc.sched_tree ? 2 : 1);
      if (kind != which) continue;
      for (int m = pass == 0 ? 0 : 1; m <= (pass == 0 ? 0 : sc.n_shift); ++m)
        for (int part = 0; part < (m == 0 ? parts : 1); ++part)
          for (int k = 1; k <= h->cap[s]; k += tb) w.push_back(make_int4(s, m, sc.base + k, part));
    }
}

// Central-image split of the mixed tree walk: enough central blocks to fill the GPU about
// four times over (the central walks are the longest, and a few hundred of them leave most
// SMs idle), at most one part per root child.
int auto_walk_parts(const nv_handle *h) {
  long long central = 0;
  for (int s = 0; s < h->nsys; ++s)
    if (h->sc[s].sched_tree && h->sc[s].velocity != NV_VEL_LIA) central += (h->cap[s] + 127) / 128;
  if (central == 0) return 1;
  const long long resident = 8LL * n_sms_host();
  int p = 1;
  while (p < kMaxWalkParts && central * p < 4 * resident) p *= 2;
  return p;
}

int rebuild_worklists(nv_handle *h) {
  std::vector<int2> w;
  int rc;
  if (h->precision == NV_PREC_MIXED) {
    std::vector<int4> w4;
    build_image_worklist(h, 1, 128, w4);
    if ((rc = upload_worklist4(&h->d_work_img, &h->n_work_img, w4)) != NV_OK) return rc;
    h->walk_parts_used = h->walk_parts > 0 ? h->walk_parts : auto_walk_parts(h);
    build_image_worklist(h, 2, 128, w4, h->walk_parts_used);
    if ((rc = upload_worklist4(&h->d_work_timg, &h->n_work_timg, w4)) != NV_OK) return rc;
  }
  for (int s = 0; s < h->nsys; ++s)
    if (h->sc[s].sched_tree) {
      h->tree_sys0 = s;
      break;
    }
  build_worklist(h, 0, w);
  if ((rc = upload_worklist(&h->d_work_lia, &h->n_work_lia, w)) != NV_OK) return rc;
  h->any_lia = !w.empty();
  build_worklist(h, 1, w);
  if ((rc = upload_worklist(&h->d_work_direct, &h->n_work_direct, w)) != NV_OK) return rc;
  h->any_direct = !w.empty();
  {  // the split direct sum for few targets: items of direct_g slots
    long long slots = 0;
    for (int s = 0; s < h->nsys; ++s)
      if (h->sc[s].velocity == NV_VEL_BS) slots += h->cap[s];
    h->direct_g = h->any_direct ? direct_targets_per_block(h, slots) : 64;
    w.clear();
    if (h->direct_g < 64)
      for (int s = 0; s < h->nsys; ++s)
        if (h->sc[s].velocity == NV_VEL_BS)
          for (int k = 1; k <= h->cap[s]; k += h->direct_g) w.push_back(make_int2(s, h->sc[s].base + k));
    if ((rc = upload_worklist(&h->d_work_split, &h->n_work_split, w)) != NV_OK) return rc;
  }
  build_worklist(h, 2, w);
  if ((rc = upload_worklist(&h->d_work_tree, &h->n_work_tree, w)) != NV_OK) return rc;
  h->any_tree = !w.empty();
  return NV_OK;
}

// the host copy of one system's dynamic state (after the stream's work so far)
int pull_dyn_one(nv_handle *h, int sys) {
  NV_CUDA(cudaMemcpyAsync(&h->h_dyn[sys], h->d_dyn + sys, sizeof(SysDyn), cudaMemcpyDeviceToHost, h->stream));
  NV_CUDA(cudaStreamSynchronize(h->stream));
  return NV_OK;
}

bool any_use_tree(nv_handle *h) {
  for (auto &s : h->sc)
    if (s.use_tree) return true;
  return false;
}

// During stream capture a plain cudaEventRecord only orders streams; the External flag
// makes it an event-record node of the graph, whose timestamps cudaEventElapsedTime reads.
void record(nv_handle *h, cudaEvent_t ev) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(h->stream, &cs);
  if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(ev, h->stream, cudaEventRecordExternal);
  else cudaEventRecord(ev, h->stream);
}
void time_begin(nv_handle *h, int st) {
  if (h->timing) record(h, h->ev[2 * st]);
}
void time_end(nv_handle *h, int st) {
  if (h->timing) record(h, h->ev[2 * st + 1]);
}

// The body of one time step, src/run.f90:26-64 (diagnostics and output excluded), with
// stage timing events.
void enqueue_step(nv_handle *h) {
  launch_begin_step(h);
  time_begin(h, ST_GHOST);
  launch_ghost(h);
  time_end(h, ST_GHOST);
  time_begin(h, ST_TREE);
  if (any_use_tree(h) || h->any_tree) launch_tree_build(h);
  time_end(h, ST_TREE);
  time_begin(h, ST_VELOCITY);
  launch_velocity(h);
  time_end(h, ST_VELOCITY);
  time_begin(h, ST_AB3);
  launch_ab3(h);
  time_end(h, ST_AB3);
  time_begin(h, ST_TOPO);
  time_begin(h, ST_INSERT);
  launch_pinsert(h);
  time_end(h, ST_INSERT);
  time_begin(h, ST_CLOSE);
  launch_pclose(h, false);  // each system checks mod(itime, recon_shots) on the device
  time_end(h, ST_CLOSE);
  time_begin(h, ST_RECON);
  launch_precon(h);
  launch_wall_recon(h);  // systems with solid walls; the others have no pinned points
  time_end(h, ST_RECON);
  time_begin(h, ST_REMOVE);
  launch_premove(h);
  time_end(h, ST_REMOVE);
  launch_wrap(h, 3);
  launch_end_step(h);
  time_end(h, ST_TOPO);
}

int capture_step(nv_handle *h) {
  if (h->graph_valid) return NV_OK;
  NV_CUDA(cudaGetLastError());
  cudaGraph_t graph = nullptr;
  const bool timing = h->timing;
  h->timing = true;  // the graph always records the stage events
  NV_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  enqueue_step(h);
  h->timing = timing;
  cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
  if (e != cudaSuccess) return check_cuda(e, "cudaStreamEndCapture");
  NV_CUDA(cudaGetLastError());
  size_t n = 0;
  NV_CUDA(cudaGraphGetNodes(graph, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  if (n) NV_CUDA(cudaGraphGetNodes(graph, nodes.data(), &n));
  int kernels = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    NV_CUDA(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) ++kernels;
  }
  h->step_kernels = kernels;
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  e = cudaGraphInstantiate(&h->graph_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return check_cuda(e, "cudaGraphInstantiate");
  NV_CUDA(cudaGetLastError());
  h->graph_valid = true;
  return NV_OK;
}

// Stage times of the step just replayed (the graph's event-record nodes).  A failed query
// only drops the timing sample; it is cleared so that it cannot surface as a step error.
void accumulate_stage_times(nv_handle *h) {
  const int st[] = {ST_GHOST, ST_TREE, ST_VELOCITY, ST_AB3, ST_TOPO, ST_INSERT, ST_CLOSE, ST_RECON, ST_REMOVE};
  for (int s : st) {
    float ms = 0;
    cudaError_t e = cudaEventElapsedTime(&ms, h->ev[2 * s], h->ev[2 * s + 1]);
    if (e == cudaSuccess) h->stage_ms[s] += ms;
    else h->timing_error = e;
  }
  float ms = 0;
  cudaError_t e = cudaEventElapsedTime(&ms, h->ev[2 * ST_GHOST], h->ev[2 * ST_TOPO + 1]);
  if (e == cudaSuccess) h->stage_ms[ST_STEP] += ms;
  else h->timing_error = e;
  cudaGetLastError();
}

}  // namespace

// Restart bookkeeping for data_restore (io.cpp): the clock and recon_count of a dump.
int set_restart_counters(nv_handle *h, int sys, double t, int itime, int recon_count) {
  if (!h || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "bad system");
  int rc = set_device(h);
  if (rc || (rc = pull_dyn_one(h, sys))) return rc;
  h->h_dyn[sys].t = t;
  h->h_dyn[sys].itime = itime;
  h->h_dyn[sys].recon_count = recon_count;
  NV_CUDA(cudaMemcpy(h->d_dyn + sys, &h->h_dyn[sys], sizeof(SysDyn), cudaMemcpyHostToDevice));
  return NV_OK;
}

int sys_capacity(nv_handle *h, int sys) { return (h && sys >= 0 && sys < h->nsys) ? h->cap[sys] : -1; }

// Per-system constants for callers outside this file (the static-scratch entry point).
SysConst sysconst_for(const nv_params &p, int base, int cap) { return make_sysconst(p, base, cap); }

// ---- batched transfers ------------------------------------------------------------------
namespace {
int ensure_batch(nv_handle *h) {
  if (h->bstage) return NV_OK;
  int rc;
  if ((rc = dalloc(&h->bstage, 3 * (size_t)h->T)) || (rc = dalloc(&h->d_btab, (size_t)h->nsys)) ||
      (rc = dalloc(&h->d_bcheck, 2 * (size_t)h->nsys)))
    return rc;
  return NV_OK;
}
// every listed state gives the optional array or none does
template <class F>
bool all_or_none(int count, const nv_host_state *st, F field) {
  int given = 0;
  for (int i = 0; i < count; ++i) given += field(st[i]) != nullptr;
  return given == 0 || given == count;
}
bool fields_consistent(int count, const nv_host_state *st) {
  return all_or_none(count, st, [](const nv_host_state &s) { return (const void *)s.u; }) &&
         all_or_none(count, st, [](const nv_host_state &s) { return (const void *)s.u1; }) &&
         all_or_none(count, st, [](const nv_host_state &s) { return (const void *)s.u2; }) &&
         all_or_none(count, st, [](const nv_host_state &s) { return (const void *)s.ghosti; }) &&
         all_or_none(count, st, [](const nv_host_state &s) { return (const void *)s.ghostb; }) &&
         all_or_none(count, st, [](const nv_host_state &s) { return (const void *)s.closest; }) &&
         all_or_none(count, st, [](const nv_host_state &s) { return (const void *)s.closestd; });
}
int batch_args(nv_handle *h, int count, const int32_t *sys, const void *st, const char *who) {
  if (!h || count < 0 || (count > 0 && (!sys || !st))) return set_error(NV_ERR_ARG, std::string(who) + ": bad arguments");
  std::vector<char> seen(h->nsys, 0);
  for (int i = 0; i < count; ++i) {
    if (sys[i] < 0 || sys[i] >= h->nsys || seen[sys[i]])
      return set_error(NV_ERR_ARG, std::string(who) + ": systems must be distinct and in range");
    seen[sys[i]] = 1;
  }
  return NV_OK;
}
}  // namespace

extern "C" {

const char *nv_last_error(void) { return g_err.c_str(); }
const char *nv_version(void) { return kVersion; }

int nv_params_default(nv_params *p) {
  if (!p) return set_error(NV_ERR_ARG, "null params");
  std::memset(p, 0, sizeof *p);
  p->shots = 1;
  p->recon_shots = 1;
  p->velocity = NV_VEL_BS;
  p->boundary[0] = p->boundary[1] = p->boundary[2] = NV_BC_PERIODIC;
  p->normal_velocity = NV_NF_ZERO;
  p->tree_extra_correction = 1;
  p->nan_test = 1;
  p->overide_timestep_check = 0;
  p->precision = NV_PREC_FP64;
  p->quant_circ = 9.97E-4;
  p->corea = 8.244023E-9;
  p->tree_theta = 0.0;
  p->norm_vel_xflow = 0.5;
  p->normal_fluid_cutoff = 1E8;
  p->t_zero_normal_fluid = 1E8;
  p->norm_shear_omega = 0.;
  return NV_OK;
}

// init_setup checks (initial.f90:21-25,37-81,131-141) and timestep_check (:169-180).
int nv_check_params(const nv_params *p) {
  if (!p) return set_error(NV_ERR_ARG, "null params");
  if (p->delta < NV_EPS) return set_error(NV_ERR_ARG, "delta must be set in run.in");
  if (!(std::min(p->box_size[0], std::min(p->box_size[1], p->box_size[2])) > 0.))
    return set_error(NV_ERR_ARG, "box size is less than or equal zero");
  for (int c = 0; c < 3; ++c) {
    if (p->boundary[c] != NV_BC_PERIODIC && p->boundary[c] != NV_BC_OPEN && p->boundary[c] != NV_BC_SOLID)
      return set_error(NV_ERR_ARG, "incorrect boundary parameter");
    if (p->boundary[c] == NV_BC_SOLID && p->precision == NV_PREC_MIXED)
      return set_error(NV_ERR_UNSUPPORTED, "solid boundaries run in the plain FP64 precision only");
  }
  if (p->velocity != NV_VEL_LIA && p->velocity != NV_VEL_BS && p->velocity != NV_VEL_TREE)
    return set_error(NV_ERR_ARG, "correct value for \"velocity\" in run.in has not been set");
  if (p->normal_velocity < NV_NF_ZERO || p->normal_velocity > NV_NF_TURB_DNS)
    return set_error(NV_ERR_ARG, "correct parameter for normal_veloctity not set");
  if (p->tree_theta > 0)
    for (int c = 0; c < 3; ++c)
      if (p->boundary[c] == NV_BC_OPEN)
        return set_error(NV_ERR_ARG, "tree approximation cannot run with open boundaries in its current form");
  if (p->precision != NV_PREC_FP64 && p->precision != NV_PREC_MIXED)
    return set_error(NV_ERR_ARG, "unknown precision");
  if (!p->overide_timestep_check) {
    const double delta_min = p->delta / 2.;
    const double dt_max = std::fabs(((delta_min) * (delta_min)) / (p->quant_circ * std::log(delta_min / (NV_PI * p->corea))));
    if (!(p->dt < dt_max)) return set_error(NV_ERR_TIMESTEP, "dt is too large (timestep_check)");
  }
  return NV_OK;
}

int nv_create(const nv_params *params, int32_t nsys, const int32_t *capacity, int32_t device, nv_handle **out) {
  if (!params || !capacity || !out || nsys < 1) return set_error(NV_ERR_ARG, "nv_create: bad arguments");
  *out = nullptr;
  for (int s = 0; s < nsys; ++s) {
    int rc = nv_check_params(&params[s]);
    if (rc != NV_OK) return rc;
    if (capacity[s] < 1) return set_error(NV_ERR_ARG, "nv_create: capacity must be >= 1");
    if (params[s].precision != params[0].precision)
      return set_error(NV_ERR_ARG, "nv_create: all systems of a handle share one precision");
    if (params[0].precision == NV_PREC_MIXED && params[s].velocity == NV_VEL_TREE)
      for (int q = 0; q < s; ++q)
        if (params[q].velocity == NV_VEL_TREE &&
            (params[q].tree_theta != params[s].tree_theta ||
             params[q].tree_extra_correction != params[s].tree_extra_correction))
          return set_error(NV_ERR_ARG, "nv_create: mixed-precision tree systems of a handle share tree_theta");
  }
  auto *h = new nv_handle();
  h->device = device;
  h->nsys = nsys;
  h->precision = params[0].precision;
  h->params.assign(params, params + nsys);
  h->cap.assign(capacity, capacity + nsys);
  long long off = 0;
  for (int s = 0; s < nsys; ++s) {
    h->base.push_back((int)off);
    off += (long long)capacity[s] + 1;
    h->max_cap = std::max(h->max_cap, (int)capacity[s]);
  }
  if (off >= (1LL << 31) - 1) {
    delete h;
    return set_error(NV_ERR_ARG, "nv_create: total capacity exceeds 2^31 slots");
  }
  h->T = off;
  for (int s = 0; s < nsys; ++s) h->sc.push_back(make_sysconst(params[s], h->base[s], capacity[s]));
  int rc = NV_OK;
  auto bail = [&](int code) {
    nv_destroy(h);
    return code;
  };
  if ((rc = set_device(h)) != NV_OK) return bail(rc);
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->join_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->sort_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->side2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->fork2_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->join2_ev, cudaEventDisableTiming) != cudaSuccess)
    return bail(set_error(NV_ERR_CUDA, "stream creation failed"));
  const long long T = h->T;
  if ((rc = dalloc(&h->d_sc, nsys)) || (rc = dalloc(&h->d_dyn, nsys)) || (rc = dalloc(&h->x, 3 * T)) ||
      (rc = dalloc(&h->u, 3 * T)) || (rc = dalloc(&h->u1, 3 * T)) || (rc = dalloc(&h->u2, 3 * T)) ||
      (rc = dalloc(&h->gi, 3 * T)) || (rc = dalloc(&h->gb, 3 * T)) || (rc = dalloc(&h->closestd, T)) ||
      (rc = dalloc(&h->nxt, T)) || (rc = dalloc(&h->prv, T)) || (rc = dalloc(&h->closest, T)) ||
      (rc = dalloc(&h->sys_of, T)) || (rc = dalloc(&h->seg, 2 * T)) || (rc = dalloc(&h->d_err, 1)) ||
      (rc = dalloc(&h->d_event_count, 1)) || (rc = dalloc(&h->d_upck, 2)) || (rc = dalloc(&h->usm, 6 * T)) ||
      (rc = dalloc(&h->cs, 2 * T)) || (rc = dalloc(&h->d_drec, nsys)))
    return bail(rc);
  for (auto &c : h->sc) {  // the velocity passes keep u_sup and u_mf there
    c.usm = h->usm;
    c.usm_T = T;
    h->any_solid |= c.solid[0] || c.solid[1] || c.solid[2];
  }
  if (h->any_solid) {  // pinned records and the tree's mirror sums of the solid-wall systems
    if ((rc = dalloc(&h->pin, T)) || (rc = dalloc(&h->umir, 3 * T))) return bail(rc);
    for (auto &c : h->sc)
      if (c.solid[0] || c.solid[1] || c.solid[2]) {
        c.pin = h->pin;
        c.umir = h->umir;
        h->any_mirror |= c.sched_tree && c.n_mirror > 0;
      }
  }
  {
    int maxcap = 0;
    for (int s = 0; s < nsys; ++s) maxcap = std::max(maxcap, h->cap[s]);
    if ((rc = dalloc(&h->stage, 3 * ((size_t)maxcap + 1)))) return bail(rc);
  }
  if (h->precision == NV_PREC_MIXED) {
    if ((rc = dalloc(&h->seg32, 3 * T))) return bail(rc);
    const int nimg = 27 + kMaxWalkParts - 1;  // the images, then the central image's extra parts
    if ((rc = dalloc(&h->partial, (size_t)nimg * 3 * T))) return bail(rc);
  }
  h->event_cap = (int)std::min<long long>(std::max<long long>(1 << 16, T), 1 << 24);
  if ((rc = dalloc(&h->d_events, h->event_cap))) return bail(rc);
  if (cudaMemcpy(h->d_sc, h->sc.data(), nsys * sizeof(SysConst), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(set_error(NV_ERR_CUDA, "upload of system constants failed"));
  std::vector<int> sys_of(T);
  for (int s = 0; s < nsys; ++s)
    for (int k = 0; k <= capacity[s]; ++k) sys_of[h->base[s] + k] = s;
  if (cudaMemcpy(h->sys_of, sys_of.data(), T * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(set_error(NV_ERR_CUDA, "upload of slot map failed"));
  h->h_dyn.assign(nsys, SysDyn{});
  for (auto &d : h->h_dyn) {
    std::memset(&d, 0, sizeof d);
    d.noise_counter = 1;
  }
  if (cudaMemcpy(h->d_dyn, h->h_dyn.data(), nsys * sizeof(SysDyn), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(set_error(NV_ERR_CUDA, "upload of system state failed"));
  if ((rc = rebuild_worklists(h))) return bail(rc);
  for (auto &e : h->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return bail(set_error(NV_ERR_CUDA, "event creation failed"));
  tree_alloc(h);
  topo_alloc(h);
  if (cudaGetLastError() != cudaSuccess) return bail(set_error(NV_ERR_CUDA, "allocation failed"));
  *out = h;
  return NV_OK;
}

int nv_destroy(nv_handle *h) {
  if (!h) return NV_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  tree_free(h);
  topo_free(h);
  for (void *p : h->nf_buffers) cudaFree(p);
  void *ptrs[] = {h->bstage, h->d_btab, h->d_bcheck, h->pin, h->umir, h->usm, h->cs, h->d_drec, h->partial, h->stage, h->d_upck, h->d_sc, h->d_dyn, h->x, h->u, h->u1, h->u2, h->gi, h->gb, h->closestd, h->nxt, h->prv,
                  h->closest, h->sys_of, h->seg, h->seg32, h->d_err, h->d_events, h->d_event_count,
                  h->d_work_direct, h->d_work_tree, h->d_work_lia, h->d_work_img, h->d_work_timg, h->d_work_split};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (auto &e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->fork_ev) cudaEventDestroy(h->fork_ev);
  if (h->join_ev) cudaEventDestroy(h->join_ev);
  if (h->sort_ev) cudaEventDestroy(h->sort_ev);
  if (h->fork2_ev) cudaEventDestroy(h->fork2_ev);
  if (h->join2_ev) cudaEventDestroy(h->join2_ev);
  if (h->side2) cudaStreamDestroy(h->side2);
  if (h->side) cudaStreamDestroy(h->side);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return NV_OK;
}

int nv_upload(nv_handle *h, int32_t sys, const nv_host_state *st) {
  if (!h || !st || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_upload: bad arguments");
  if (!st->x || !st->infront || !st->behind) return set_error(NV_ERR_ARG, "nv_upload: x, infront, behind are required");
  const int n = st->pcount, cap = h->cap[sys], base = h->base[sys];
  if (n < 0 || n > cap) return set_error(NV_ERR_ARG, "nv_upload: pcount exceeds the system's capacity");
  const SysConst &scs = h->sc[sys];
  if (!(scs.solid[0] || scs.solid[1] || scs.solid[2]))
    for (int k = 0; k < n; ++k)
      if ((st->pinnedi && st->pinnedi[k]) || (st->pinnedb && st->pinnedb[k]))
        return set_error(NV_ERR_ARG, "nv_upload: pinned points need a solid boundary (system left unchanged)");
  int rc = set_device(h);
  if (rc) return rc;
  const long long T = h->T;
  const int rows = cap + 1;  // the system's dummy slot and all its slots
  cudaStream_t sm = h->stream;
  // The links are staged and checked first, so that a rejected upload leaves the system as
  // it was: infront, behind and closest side by side in the staging buffer (3n ints fit in
  // its 3(cap+1) doubles).
  int *stage_i = reinterpret_cast<int *>(h->stage);
  int *s_inf = stage_i, *s_beh = stage_i + n, *s_clo = st->closest ? stage_i + 2 * (size_t)n : nullptr;
  NV_CUDA(cudaMemsetAsync(h->d_upck, 0, 2 * sizeof(int), sm));
  if (n > 0) {
    NV_CUDA(cudaMemcpyAsync(s_inf, st->infront, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, sm));
    NV_CUDA(cudaMemcpyAsync(s_beh, st->behind, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, sm));
    if (s_clo) NV_CUDA(cudaMemcpyAsync(s_clo, st->closest, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, sm));
    k_upload_check<<<grid_for(n, 256), 256, 0, sm>>>(s_inf, s_beh, s_clo, n, h->d_upck);
  }
  int check[2] = {0, 0};
  NV_CUDA(cudaMemcpyAsync(check, h->d_upck, sizeof check, cudaMemcpyDeviceToHost, sm));
  NV_CUDA(cudaStreamSynchronize(sm));
  if (check[0] & 1) return set_error(NV_ERR_ARG, "nv_upload: link out of range (system left unchanged)");
  if (check[0] & 2)
    return set_error(NV_ERR_ARG, "nv_upload: infront/behind disagree on an empty slot (system left unchanged)");
  ++h->links_epoch;
  k_put_links<<<grid_for(rows, 256), 256, 0, sm>>>(h->nxt, base, rows, n, n > 0 ? s_inf : nullptr);
  k_put_links<<<grid_for(rows, 256), 256, 0, sm>>>(h->prv, base, rows, n, n > 0 ? s_beh : nullptr);
  k_put_links<<<grid_for(rows, 256), 256, 0, sm>>>(h->closest, base, rows, n, n > 0 ? s_clo : nullptr);
  // each double array goes to the staging buffer in one copy and from there to the slots (in
  // stream order, so the buffer is reused array after array, after the links above)
  auto put = [&](double *dev, const double *src, int comps) -> int {
    if (src && n > 0)
      NV_CUDA(cudaMemcpyAsync(h->stage, src, (size_t)comps * n * sizeof(double), cudaMemcpyHostToDevice, sm));
    k_put_rows<<<grid_for(rows, 256), 256, 0, sm>>>(dev, T, base, rows, n, comps, src ? h->stage : nullptr);
    return NV_OK;
  };
  if ((rc = put(h->x, st->x, 3)) || (rc = put(h->u, st->u, 3)) || (rc = put(h->u1, st->u1, 3)) ||
      (rc = put(h->u2, st->u2, 3)) || (rc = put(h->gi, st->ghosti, 3)) || (rc = put(h->gb, st->ghostb, 3)) ||
      (rc = put(h->closestd, st->closestd, 1)))
    return rc;
  // the new f(:) carries no u_sup, u_mf, curv or stretch yet (nv_upload_full sets them)
  k_put_rows<<<grid_for(rows, 256), 256, 0, sm>>>(h->usm, T, base, rows, n, 6, nullptr);
  k_put_rows<<<grid_for(rows, 256), 256, 0, sm>>>(h->cs, T, base, rows, n, 2, nullptr);
  if (h->pin) {  // pinned records (the staging buffer holds 5n ints)
    const int *wp = nullptr, *pi = nullptr, *pb = nullptr;
    if (n > 0 && st->wpinned) {
      NV_CUDA(cudaMemcpyAsync(stage_i, st->wpinned, 3 * (size_t)n * sizeof(int), cudaMemcpyHostToDevice, sm));
      wp = stage_i;
    }
    if (n > 0 && st->pinnedi) {
      NV_CUDA(cudaMemcpyAsync(stage_i + 3 * (size_t)n, st->pinnedi, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, sm));
      pi = stage_i + 3 * (size_t)n;
    }
    if (n > 0 && st->pinnedb) {
      NV_CUDA(cudaMemcpyAsync(stage_i + 4 * (size_t)n, st->pinnedb, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, sm));
      pb = stage_i + 4 * (size_t)n;
    }
    k_put_pin<<<grid_for(rows, 256), 256, 0, sm>>>(h->pin, base, rows, n, wp, pi, pb);
  }
  SysDyn &d = h->h_dyn[sys];
  // keep the clock and counters; replace the slot count (pull_dyn_one waits for the copies)
  rc = pull_dyn_one(h, sys);
  if (rc) return rc;
  d.pcount = n;
  d.nlive = check[1];
  NV_CUDA(cudaMemcpy(h->d_dyn + sys, &d, sizeof(SysDyn), cudaMemcpyHostToDevice));
  unsigned zero = 0;
  NV_CUDA(cudaMemcpy(h->d_err, &zero, sizeof zero, cudaMemcpyHostToDevice));
  return NV_OK;
}

int nv_download(nv_handle *h, int32_t sys, nv_host_state *st, int32_t cap) {
  if (!h || !st || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_download: bad arguments");
  int rc = set_device(h);
  if (rc) return rc;
  if ((rc = pull_dyn_one(h, sys))) return rc;
  const int n = h->h_dyn[sys].pcount, base = h->base[sys];
  st->pcount = n;
  if (n > cap) return set_error(NV_ERR_ARG, "nv_download: arrays hold fewer slots than pcount");
  const long long T = h->T;
  cudaStream_t sm = h->stream;
  // slots -> staging buffer in the host layout -> one copy (to pageable memory the copy
  // returns once it is done, so the buffer is free for the next array)
  auto get = [&](const double *dev, double *dst, int comps) -> int {
    if (!dst || n == 0) return NV_OK;
    k_get_rows<<<grid_for(n, 256), 256, 0, sm>>>(dev, T, base, n, comps, h->stage);
    NV_CUDA(cudaMemcpyAsync(dst, h->stage, (size_t)comps * n * sizeof(double), cudaMemcpyDeviceToHost, sm));
    return NV_OK;
  };
  int *stage_i = reinterpret_cast<int *>(h->stage);
  auto get_link = [&](const int *dev, int *dst) -> int {
    if (!dst || n == 0) return NV_OK;
    k_get_links<<<grid_for(n, 256), 256, 0, sm>>>(dev, base, n, stage_i);
    NV_CUDA(cudaMemcpyAsync(dst, stage_i, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, sm));
    return NV_OK;
  };
  if ((rc = get(h->x, st->x, 3)) || (rc = get(h->u, st->u, 3)) || (rc = get(h->u1, st->u1, 3)) ||
      (rc = get(h->u2, st->u2, 3)) || (rc = get(h->gi, st->ghosti, 3)) || (rc = get(h->gb, st->ghostb, 3)) ||
      (rc = get_link(h->nxt, st->infront)) || (rc = get_link(h->prv, st->behind)) ||
      (rc = get_link(h->closest, st->closest)) || (rc = get(h->closestd, st->closestd, 1)))
    return rc;
  if (n > 0 && (st->wpinned || st->pinnedi || st->pinnedb)) {  // pinned records, one int array at a time
    int *out[3] = {st->wpinned, st->pinnedi, st->pinnedb};
    const int per[3] = {3, 1, 1};
    for (int q = 0; q < 3; ++q) {
      if (!out[q]) continue;
      k_get_pin<<<grid_for(n, 256), 256, 0, sm>>>(h->pin, base, n, q == 0 ? stage_i : nullptr, q == 1 ? stage_i : nullptr,
                                                 q == 2 ? stage_i : nullptr);
      NV_CUDA(cudaMemcpyAsync(out[q], stage_i, (size_t)per[q] * n * sizeof(int), cudaMemcpyDeviceToHost, sm));
    }
  }
  NV_CUDA(cudaStreamSynchronize(sm));
  return NV_OK;
}


}  // extern "C"

// The batched transfers of count systems sys[i] (n[i] points each), whatever the host layout:
// `stage(kind, dst)` copies host array `kind` of every listed system into the staging buffer
// at the packed offsets (system i's rows from row off[i] = n[0] + ... + n[i-1]); kinds 0-2 are
// infront, behind, closest, 3-9 x, u, u1, u2, ghosti, ghostb, closestd.
namespace {
enum { kInf, kBeh, kClo, kX, kU, kU1, kU2, kGi, kGb, kCd, kKinds };
const int kComps[kKinds] = {1, 1, 1, 3, 3, 3, 3, 3, 3, 1};

template <class Stage>
int upload_batch(nv_handle *h, int count, const int32_t *sys, const int *n, const bool given[kKinds], Stage stage,
                 const char *who) {
  int rc;
  if ((rc = set_device(h)) || (rc = ensure_batch(h))) return rc;
  cudaStream_t sm = h->stream;
  const long long T = h->T;
  std::vector<int4> tab(count);
  long long N = 0;
  int maxrows = 1;
  for (int i = 0; i < count; ++i) {
    tab[i] = make_int4(h->base[sys[i]], h->cap[sys[i]] + 1, n[i], (int)N);
    N += n[i];
    maxrows = std::max(maxrows, h->cap[sys[i]] + 1);
  }
  NV_CUDA(cudaMemcpyAsync(h->d_btab, tab.data(), count * sizeof(int4), cudaMemcpyHostToDevice, sm));
  const dim3 grid(grid_for(maxrows, 256), count);
  // links: staged and checked for every system before any system changes
  int *si = reinterpret_cast<int *>(h->bstage);
  int *s_inf = si, *s_beh = si + N, *s_clo = si + 2 * N;
  if ((rc = stage(kInf, s_inf)) || (rc = stage(kBeh, s_beh)) || (given[kClo] && (rc = stage(kClo, s_clo)))) return rc;
  NV_CUDA(cudaMemsetAsync(h->d_bcheck, 0, 2 * count * sizeof(int), sm));
  k_upload_check_many<<<grid, 256, 0, sm>>>(h->d_btab, s_inf, s_beh, given[kClo] ? s_clo : nullptr, h->d_bcheck);
  std::vector<int> check(2 * count);
  NV_CUDA(cudaMemcpyAsync(check.data(), h->d_bcheck, 2 * count * sizeof(int), cudaMemcpyDeviceToHost, sm));
  NV_CUDA(cudaStreamSynchronize(sm));
  for (int i = 0; i < count; ++i) {
    if (check[2 * i] & 1)
      return set_error(NV_ERR_ARG, std::string(who) + ": link out of range in system " + std::to_string(sys[i]) +
                                       " (no system changed)");
    if (check[2 * i] & 2)
      return set_error(NV_ERR_ARG, std::string(who) + ": infront/behind disagree on an empty slot in system " +
                                       std::to_string(sys[i]) + " (no system changed)");
  }
  ++h->links_epoch;
  k_put_links_many<<<grid, 256, 0, sm>>>(h->nxt, h->d_btab, s_inf);
  k_put_links_many<<<grid, 256, 0, sm>>>(h->prv, h->d_btab, s_beh);
  k_put_links_many<<<grid, 256, 0, sm>>>(h->closest, h->d_btab, given[kClo] ? s_clo : nullptr);
  // each double array of every system into the staging buffer, then one launch to the slots
  // (in stream order, so the buffer is reused array after array)
  double *dev[kKinds] = {nullptr, nullptr, nullptr, h->x, h->u, h->u1, h->u2, h->gi, h->gb, h->closestd};
  for (int kind = kX; kind < kKinds; ++kind) {
    if (given[kind] && (rc = stage(kind, h->bstage))) return rc;
    k_put_rows_many<<<grid, 256, 0, sm>>>(dev[kind], T, h->d_btab, kComps[kind], given[kind] ? h->bstage : nullptr);
  }
  k_put_rows_many<<<grid, 256, 0, sm>>>(h->usm, T, h->d_btab, 6, nullptr);
  k_put_rows_many<<<grid, 256, 0, sm>>>(h->cs, T, h->d_btab, 2, nullptr);
  // the clocks and counters stay; the slot counts are replaced
  NV_CUDA(cudaMemcpyAsync(h->h_dyn.data(), h->d_dyn, h->nsys * sizeof(SysDyn), cudaMemcpyDeviceToHost, sm));
  NV_CUDA(cudaStreamSynchronize(sm));
  for (int i = 0; i < count; ++i) {
    SysDyn &d = h->h_dyn[sys[i]];
    d.pcount = n[i];
    d.nlive = check[2 * i + 1];
  }
  NV_CUDA(cudaMemcpyAsync(h->d_dyn, h->h_dyn.data(), h->nsys * sizeof(SysDyn), cudaMemcpyHostToDevice, sm));
  NV_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(unsigned), sm));
  NV_CUDA(cudaStreamSynchronize(sm));
  return NV_OK;
}

// `fetch(kind, src, tab)` copies array `kind` of every listed system from the staging buffer
// (packed offsets tab[i].w) to the host.  n_out[i] receives each system's pcount first;
// `fits(i, n)` refuses a system whose arrays are too small.
template <class Fits, class Fetch>
int download_batch(nv_handle *h, int count, const int32_t *sys, const bool want[kKinds], int *n_out, Fits fits,
                   Fetch fetch) {
  int rc;
  if ((rc = set_device(h)) || (rc = ensure_batch(h))) return rc;
  cudaStream_t sm = h->stream;
  const long long T = h->T;
  NV_CUDA(cudaMemcpyAsync(h->h_dyn.data(), h->d_dyn, h->nsys * sizeof(SysDyn), cudaMemcpyDeviceToHost, sm));
  NV_CUDA(cudaStreamSynchronize(sm));
  std::vector<int4> tab(count);
  long long N = 0;
  int maxn = 1;
  for (int i = 0; i < count; ++i) {
    const int s = sys[i], n = h->h_dyn[s].pcount;
    n_out[i] = n;
    if ((rc = fits(i, n))) return rc;
    tab[i] = make_int4(h->base[s], h->cap[s] + 1, n, (int)N);
    N += n;
    maxn = std::max(maxn, n);
  }
  NV_CUDA(cudaMemcpyAsync(h->d_btab, tab.data(), count * sizeof(int4), cudaMemcpyHostToDevice, sm));
  const dim3 grid(grid_for(maxn, 256), count);
  // one launch per array over every system into the staging buffer, then the copies out
  // (stream order keeps the buffer from being overwritten before its copies are done)
  const double *dev[kKinds] = {nullptr, nullptr, nullptr, h->x, h->u, h->u1, h->u2, h->gi, h->gb, h->closestd};
  const int *devl[3] = {h->nxt, h->prv, h->closest};
  for (int kind = 0; kind < kKinds; ++kind) {
    if (!want[kind]) continue;
    if (kind <= kClo) k_get_links_many<<<grid, 256, 0, sm>>>(devl[kind], h->d_btab, reinterpret_cast<int *>(h->bstage));
    else k_get_rows_many<<<grid, 256, 0, sm>>>(dev[kind], T, h->d_btab, kComps[kind], h->bstage);
    if ((rc = fetch(kind, tab))) return rc;
  }
  NV_CUDA(cudaStreamSynchronize(sm));
  return NV_OK;
}

void *field_of(const nv_host_state &s, int kind) {
  switch (kind) {
    case kInf: return s.infront;
    case kBeh: return s.behind;
    case kClo: return s.closest;
    case kX: return s.x;
    case kU: return s.u;
    case kU1: return s.u1;
    case kU2: return s.u2;
    case kGi: return s.ghosti;
    case kGb: return s.ghostb;
    default: return s.closestd;
  }
}
size_t elem_bytes(int kind) { return kind <= kClo ? sizeof(int) : sizeof(double); }
}  // namespace

extern "C" {

int nv_upload_many(nv_handle *h, int32_t count, const int32_t *sys, const nv_host_state *st) {
  int rc = batch_args(h, count, sys, st, "nv_upload_many");
  if (rc) return rc;
  bool one_by_one = false;  // systems with solid walls go through nv_upload one at a time
  for (int i = 0; i < count; ++i) {
    const nv_host_state &s = st[i];
    if (!s.x || !s.infront || !s.behind) return set_error(NV_ERR_ARG, "nv_upload_many: x, infront, behind are required");
    if (s.pcount < 0 || s.pcount > h->cap[sys[i]])
      return set_error(NV_ERR_ARG, "nv_upload_many: pcount exceeds a system's capacity");
    if (h->sc[sys[i]].pin || s.wpinned || s.pinnedi || s.pinnedb) one_by_one = true;
  }
  if (one_by_one) {
    for (int i = 0; i < count; ++i)
      if ((rc = nv_upload(h, sys[i], &st[i]))) return rc;
    return NV_OK;
  }
  if (!fields_consistent(count, st))
    return set_error(NV_ERR_ARG, "nv_upload_many: each optional array must be given for every listed system or none");
  if (count == 0) return NV_OK;
  std::vector<int> n(count), off(count);
  for (int i = 0, o = 0; i < count; ++i) {
    n[i] = st[i].pcount;
    off[i] = o;
    o += n[i];
  }
  bool given[kKinds];
  for (int kind = 0; kind < kKinds; ++kind) given[kind] = field_of(st[0], kind) != nullptr;
  cudaStream_t sm = h->stream;
  auto stage = [&](int kind, void *dst) -> int {
    const int c = kComps[kind];
    const size_t e = elem_bytes(kind);
    for (int i = 0; i < count; ++i)
      if (n[i])
        NV_CUDA(cudaMemcpyAsync(static_cast<char *>(dst) + (size_t)c * off[i] * e, field_of(st[i], kind),
                                (size_t)c * n[i] * e, cudaMemcpyHostToDevice, sm));
    return NV_OK;
  };
  return upload_batch(h, count, sys, n.data(), given, stage, "nv_upload_many");
}

int nv_download_many(nv_handle *h, int32_t count, const int32_t *sys, nv_host_state *st, const int32_t *cap) {
  int rc = batch_args(h, count, sys, st, "nv_download_many");
  if (rc) return rc;
  if (count > 0 && !cap) return set_error(NV_ERR_ARG, "nv_download_many: bad arguments");
  bool one_by_one = false;  // pinned records go through nv_download one system at a time
  for (int i = 0; i < count; ++i)
    if (st[i].wpinned || st[i].pinnedi || st[i].pinnedb) one_by_one = true;
  if (one_by_one) {
    for (int i = 0; i < count; ++i)
      if ((rc = nv_download(h, sys[i], &st[i], cap[i]))) return rc;
    return NV_OK;
  }
  if (!fields_consistent(count, st) ||
      !all_or_none(count, st, [](const nv_host_state &s) { return (const void *)s.x; }) ||
      !all_or_none(count, st, [](const nv_host_state &s) { return (const void *)s.infront; }) ||
      !all_or_none(count, st, [](const nv_host_state &s) { return (const void *)s.behind; }))
    return set_error(NV_ERR_ARG, "nv_download_many: each array must be asked for every listed system or none");
  if (count == 0) return NV_OK;
  bool want[kKinds];
  for (int kind = 0; kind < kKinds; ++kind) want[kind] = field_of(st[0], kind) != nullptr;
  std::vector<int> n(count);
  cudaStream_t sm = h->stream;
  auto fits = [&](int i, int pc) -> int {
    st[i].pcount = pc;
    return pc > cap[i] ? set_error(NV_ERR_ARG, "nv_download_many: arrays hold fewer slots than pcount") : NV_OK;
  };
  auto fetch = [&](int kind, const std::vector<int4> &tab) -> int {
    const int c = kComps[kind];
    const size_t e = elem_bytes(kind);
    for (int i = 0; i < count; ++i)
      if (tab[i].z)
        NV_CUDA(cudaMemcpyAsync(field_of(st[i], kind), reinterpret_cast<char *>(h->bstage) + (size_t)c * tab[i].w * e,
                                (size_t)c * tab[i].z * e, cudaMemcpyDeviceToHost, sm));
    return NV_OK;
  };
  return download_batch(h, count, sys, want, n.data(), fits, fetch);
}

int nv_upload_packed(nv_handle *h, const nv_host_state *all, const int32_t *pcounts) {
  if (!h || !all || !pcounts) return set_error(NV_ERR_ARG, "nv_upload_packed: bad arguments");
  if (!all->x || !all->infront || !all->behind) return set_error(NV_ERR_ARG, "nv_upload_packed: x, infront, behind are required");
  if (all->wpinned || all->pinnedi || all->pinnedb) return set_error(NV_ERR_UNSUPPORTED, "nv_upload_packed: no pinned records (use nv_upload)");
  long long tot = 0;
  std::vector<int32_t> sys(h->nsys);
  std::vector<int> n(h->nsys);
  for (int s = 0; s < h->nsys; ++s) {
    if (h->sc[s].pin) return set_error(NV_ERR_UNSUPPORTED, "nv_upload_packed: a system has solid walls (use nv_upload)");
    if (pcounts[s] < 0 || pcounts[s] > h->cap[s]) return set_error(NV_ERR_ARG, "nv_upload_packed: pcount exceeds a system's capacity");
    sys[s] = s;
    n[s] = pcounts[s];
    tot += pcounts[s];
  }
  if (tot != all->pcount) return set_error(NV_ERR_ARG, "nv_upload_packed: all->pcount must be the sum of pcounts");
  bool given[kKinds];
  for (int kind = 0; kind < kKinds; ++kind) given[kind] = field_of(*all, kind) != nullptr;
  cudaStream_t sm = h->stream;
  auto stage = [&](int kind, void *dst) -> int {  // the packed host array is the staging layout
    if (tot) NV_CUDA(cudaMemcpyAsync(dst, field_of(*all, kind), (size_t)kComps[kind] * tot * elem_bytes(kind),
                                     cudaMemcpyHostToDevice, sm));
    return NV_OK;
  };
  return upload_batch(h, h->nsys, sys.data(), n.data(), given, stage, "nv_upload_packed");
}

int nv_download_packed(nv_handle *h, nv_host_state *all, int64_t cap_rows, int32_t *pcounts) {
  if (!h || !all || !pcounts) return set_error(NV_ERR_ARG, "nv_download_packed: bad arguments");
  if (all->wpinned || all->pinnedi || all->pinnedb) return set_error(NV_ERR_UNSUPPORTED, "nv_download_packed: no pinned records (use nv_download)");
  std::vector<int32_t> sys(h->nsys);
  for (int s = 0; s < h->nsys; ++s) sys[s] = s;
  bool want[kKinds];
  for (int kind = 0; kind < kKinds; ++kind) want[kind] = field_of(*all, kind) != nullptr;
  long long tot = 0;
  auto fits = [&](int i, int pc) -> int {
    tot += pc;
    return tot > cap_rows ? set_error(NV_ERR_ARG, "nv_download_packed: arrays hold fewer rows than the systems' points") : NV_OK;
  };
  cudaStream_t sm = h->stream;
  auto fetch = [&](int kind, const std::vector<int4> &) -> int {
    if (tot) NV_CUDA(cudaMemcpyAsync(field_of(*all, kind), h->bstage, (size_t)kComps[kind] * tot * elem_bytes(kind),
                                     cudaMemcpyDeviceToHost, sm));
    return NV_OK;
  };
  int rc = download_batch(h, h->nsys, sys.data(), want, pcounts, fits, fetch);
  if (rc == NV_OK) all->pcount = (int32_t)tot;
  return rc;
}

int nv_host_register(void *p, size_t bytes) {
  if (!p || bytes == 0) return set_error(NV_ERR_ARG, "nv_host_register: bad arguments");
  NV_CUDA(cudaHostRegister(p, bytes, cudaHostRegisterDefault));
  return NV_OK;
}
int nv_host_unregister(void *p) {
  if (!p) return set_error(NV_ERR_ARG, "nv_host_unregister: bad arguments");
  NV_CUDA(cudaHostUnregister(p));
  return NV_OK;
}

int nv_upload_full(nv_handle *h, int32_t sys, const nv_full_state *st) {
  if (!h || !st || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_upload_full: bad arguments");
  nv_host_state hs;
  std::memset(&hs, 0, sizeof hs);
  hs.pcount = st->pcount;
  hs.x = st->x;
  hs.u = st->u;
  hs.u1 = st->u1;
  hs.u2 = st->u2;
  hs.ghosti = st->ghosti;
  hs.ghostb = st->ghostb;
  hs.infront = st->infront;
  hs.behind = st->behind;
  hs.closest = st->closest;
  hs.closestd = st->closestd;
  hs.wpinned = st->wpinned;
  hs.pinnedi = st->pinnedi;
  hs.pinnedb = st->pinnedb;
  int rc = nv_upload(h, sys, &hs);  // checks the links before writing anything
  if (rc) return rc;
  const int n = st->pcount, base = h->base[sys], rows = h->cap[sys] + 1;
  const long long T = h->T;
  cudaStream_t sm = h->stream;
  auto put = [&](double *dev, const double *src, int comps) -> int {
    if (src && n > 0)
      NV_CUDA(cudaMemcpyAsync(h->stage, src, (size_t)comps * n * sizeof(double), cudaMemcpyHostToDevice, sm));
    k_put_rows<<<grid_for(rows, 256), 256, 0, sm>>>(dev, T, base, rows, n, comps, src ? h->stage : nullptr);
    return NV_OK;
  };
  if ((rc = put(h->usm, st->u_sup, 3)) || (rc = put(h->usm + 3 * T, st->u_mf, 3)) || (rc = put(h->cs, st->curv, 1)) ||
      (rc = put(h->cs + T, st->stretch, 1)))
    return rc;
  NV_CUDA(cudaStreamSynchronize(sm));
  return NV_OK;
}

int nv_download_full(nv_handle *h, int32_t sys, nv_full_state *st, int32_t cap) {
  if (!h || !st || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_download_full: bad arguments");
  nv_host_state hs;
  std::memset(&hs, 0, sizeof hs);
  hs.x = st->x;
  hs.u = st->u;
  hs.u1 = st->u1;
  hs.u2 = st->u2;
  hs.ghosti = st->ghosti;
  hs.ghostb = st->ghostb;
  hs.infront = st->infront;
  hs.behind = st->behind;
  hs.closest = st->closest;
  hs.closestd = st->closestd;
  hs.wpinned = st->wpinned;
  hs.pinnedi = st->pinnedi;
  hs.pinnedb = st->pinnedb;
  int rc = nv_download(h, sys, &hs, cap);
  st->pcount = hs.pcount;
  if (rc) return rc;
  const int n = hs.pcount, base = h->base[sys];
  const long long T = h->T;
  cudaStream_t sm = h->stream;
  auto get = [&](const double *dev, double *dst, int comps) -> int {
    if (!dst || n == 0) return NV_OK;
    k_get_rows<<<grid_for(n, 256), 256, 0, sm>>>(dev, T, base, n, comps, h->stage);
    NV_CUDA(cudaMemcpyAsync(dst, h->stage, (size_t)comps * n * sizeof(double), cudaMemcpyDeviceToHost, sm));
    return NV_OK;
  };
  if ((rc = get(h->usm, st->u_sup, 3)) || (rc = get(h->usm + 3 * T, st->u_mf, 3)) || (rc = get(h->cs, st->curv, 1)) ||
      (rc = get(h->cs + T, st->stretch, 1)))
    return rc;
  NV_CUDA(cudaStreamSynchronize(sm));
  return NV_OK;
}

int nv_calculate_diagnostics(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc || (rc = diag_launch(h))) return rc;
  return finish(h);
}

int nv_ts_row_get(nv_handle *h, int32_t sys, nv_ts_row *row) {
  if (!h || !row || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_ts_row_get: bad arguments");
  int rc = set_device(h);
  if (rc || (rc = pull_dyn_one(h, sys))) return rc;
  DiagRec r;
  NV_CUDA(cudaMemcpy(&r, h->d_drec + sys, sizeof r, cudaMemcpyDeviceToHost));
  if (!r.valid) return set_error(NV_ERR_STATE, "nv_ts_row_get: no diagnostics yet (call nv_calculate_diagnostics)");
  const SysDyn &d = h->h_dyn[sys];
  std::memset(row, 0, sizeof *row);
  row->itime = d.itime;
  row->live = r.live;
  row->recon_count = d.recon_count;
  row->wall_recon_count = d.wall_recon_count;
  row->remove_count = d.remove_count;
  row->tree_eval = (int64_t)d.tree_eval;
  row->t = d.t;
  row->delta = h->params[sys].delta;
  row->avg_sep = d.avg_sep;
  row->total_length = d.total_length;
  row->maxu = r.maxu;
  row->maxdu = r.maxdu;
  row->mean_u_sup = r.sum_usup / r.live;  // velocity_info: sum over f(:) / count(infront>0)
  row->mean_u_mf = r.sum_umf / r.live;
  row->kappa_bar = r.sum_curv / r.live;   // curv_info
  row->kappa_min = r.kappa_min;
  row->kappa_max = r.kappa_max;
  return NV_OK;
}

int nv_set_clock(nv_handle *h, int32_t sys, double t, int32_t itime) {
  if (!h || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_set_clock: bad arguments");
  int rc = set_device(h);
  if (rc || (rc = pull_dyn_one(h, sys))) return rc;
  h->h_dyn[sys].t = t;
  h->h_dyn[sys].itime = itime;
  NV_CUDA(cudaMemcpy(h->d_dyn + sys, &h->h_dyn[sys], sizeof(SysDyn), cudaMemcpyHostToDevice));
  return NV_OK;
}

int nv_counters_get(nv_handle *h, int32_t sys, nv_counters *c) {
  if (!h || !c || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_counters_get: bad arguments");
  int rc = set_device(h);
  if (rc || (rc = pull_dyn_one(h, sys))) return rc;
  const SysDyn &d = h->h_dyn[sys];
  c->pcount = d.pcount;
  c->live = d.nlive;
  c->recon_count = d.recon_count;
  c->remove_count = d.remove_count;
  c->insert_count = d.insert_count;
  c->loop_kills = d.loop_kills;
  c->tree_eval = (int64_t)d.tree_eval;
  c->tree_tests = (int64_t)d.tree_tests;
  c->itime = d.itime;
  c->n_events = d.event_seq;
  c->t = d.t;
  c->event_hash = d.ev_hash;
  c->wall_recon_count = d.wall_recon_count;
  c->reserved = 0;
  return NV_OK;
}

int nv_events_get(nv_handle *h, int32_t sys, nv_event *buf, int32_t cap, int32_t *n) {
  if (!h || !n || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_events_get: bad arguments");
  int rc = set_device(h);
  if (rc) return rc;
  int total = 0;
  NV_CUDA(cudaMemcpy(&total, h->d_event_count, sizeof(int), cudaMemcpyDeviceToHost));
  total = std::min(total, h->event_cap);
  std::vector<DevEvent> ev(total);
  if (total) NV_CUDA(cudaMemcpy(ev.data(), h->d_events, total * sizeof(DevEvent), cudaMemcpyDeviceToHost));
  std::vector<DevEvent> mine;
  for (auto &e : ev)
    if (e.sys == sys) mine.push_back(e);
  std::sort(mine.begin(), mine.end(), [](const DevEvent &a, const DevEvent &b) { return a.seq < b.seq; });
  const int base = h->base[sys];
  int m = 0;
  for (auto &e : mine) {
    if (m >= cap) break;
    if (buf) {
      buf[m].itime = e.itime;
      buf[m].kind = e.kind;
      buf[m].i = e.i ? e.i - base : 0;
      const bool count = e.kind == NV_EV_LOOPKILL || e.kind == NV_EV_WALL || e.kind == NV_EV_CLEAR;
      buf[m].j = count ? e.j : (e.j ? e.j - base : 0);
    }
    ++m;
  }
  *n = m;
  return NV_OK;
}

// ---- stages ---------------------------------------------------------------------------
int nv_ghostp(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  launch_ghost(h);
  return finish(h);
}
int nv_construct_tree(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  launch_tree_build(h);
  join_root_sums(h);
  return finish(h);
}
int nv_pmotion(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  if (nf_missing(h)) return NV_ERR_STATE;
  int rc = set_device(h);
  if (rc) return rc;
  launch_velocity(h);
  launch_ab3(h);
  return finish(h);
}
int nv_pinsert(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  launch_pinsert(h);
  return finish(h);
}
int nv_pclose(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  launch_pclose(h, false);
  return finish(h);
}
int nv_precon(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  launch_precon(h);
  return finish(h);
}
int nv_wall_recon(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  launch_wall_recon(h);
  return finish(h);
}
int nv_premove(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  launch_premove(h);
  return finish(h);
}
int nv_enforce_boundary(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  launch_wrap(h, 1);
  return finish(h);
}
int nv_empty_tree(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  return NV_OK;  // the device tree is rebuilt in place by the next construct_tree
}
int nv_end_step(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  launch_wrap(h, 2);
  launch_end_step(h);
  return finish(h);
}

int nv_step(nv_handle *h, int32_t nsteps) {
  if (!h || nsteps < 0) return set_error(NV_ERR_ARG, "nv_step: bad arguments");
  if (nf_missing(h)) return NV_ERR_STATE;
  int rc = set_device(h);
  if (rc || (rc = capture_step(h))) return rc;
  for (int k = 0; k < nsteps; ++k) {
    NV_CUDA(cudaGraphLaunch(h->graph_exec, h->stream));
    if (h->timing) {
      if ((rc = finish(h))) return rc;
      accumulate_stage_times(h);
    }
  }
  return finish(h);
}

int nv_set_near_factor(nv_handle *h, double factor) {
  if (!h || !(factor >= 0)) return set_error(NV_ERR_ARG, "nv_set_near_factor: bad arguments");
  h->near_factor = factor;
  h->graph_valid = false;  // the factor is a launch argument of the captured kernels
  return NV_OK;
}

int nv_set_fp32_guards(nv_handle *h, double angle, double line, double end) {
  if (!h || !(angle >= 0 && angle <= 2) || !(line >= 1e-9 && line <= 1) || !(end >= 0 && end <= 1))
    return set_error(NV_ERR_ARG, "nv_set_fp32_guards: angle in [0,2], line in [1e-9,1] (it also keeps the "
                                 "FP32 term away from its singularity, a target on the segment), end in [0,1]");
  h->guards.angle = (float)angle;
  h->guards.line = (float)line;
  h->guards.end = (float)end;
  h->graph_valid = false;  // launch arguments of the captured kernels
  return NV_OK;
}

int nv_set_root_band(nv_handle *h, double scale) {
  if (!h || !(scale >= 1.0)) return set_error(NV_ERR_ARG, "nv_set_root_band: scale must be >= 1");
  h->root_band_scale = scale;
  h->graph_valid = false;  // a launch argument of the captured step
  return NV_OK;
}

int nv_set_walk_range(nv_handle *h, int32_t sys, int32_t lo, int32_t hi) {
  if (!h || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_set_walk_range: bad arguments");
  SysConst &c = h->sc[sys];
  if (!c.sched_tree || c.velocity == NV_VEL_LIA || c.pin)
    return set_error(NV_ERR_UNSUPPORTED, "nv_set_walk_range: tree-walk systems without solid walls only");
  if (lo < 1 || hi < lo || hi > c.cap + 1) return set_error(NV_ERR_ARG, "nv_set_walk_range: need 1 <= lo <= hi <= cap + 1");
  if ((lo - 1) % 32 != 0 || ((hi - 1) % 32 != 0 && hi != c.cap + 1))
    return set_error(NV_ERR_ARG, "nv_set_walk_range: lo - 1 and hi - 1 must be multiples of 32 (or hi = cap + 1)");
  int rc = set_device(h);
  if (rc) return rc;
  c.walk_lo = lo;
  c.walk_hi = hi;
  NV_CUDA(cudaMemcpy(h->d_sc + sys, &c, sizeof(SysConst), cudaMemcpyHostToDevice));
  return NV_OK;
}

int nv_velocity_pack(nv_handle *h, int32_t sys, int32_t lo, int32_t count, double *d_buf) {
  if (!h || sys < 0 || sys >= h->nsys || lo < 1 || count < 0 || lo + count > h->cap[sys] + 1 || (count && !d_buf))
    return set_error(NV_ERR_ARG, "nv_velocity_pack: bad arguments");
  const int *perm = tree_perm(h);
  if (!perm) return set_error(NV_ERR_STATE, "nv_velocity_pack: no walk order (no tree built)");
  int rc = set_device(h);
  if (rc) return rc;
  if (count) k_vel_pack<<<grid_for(count, 256), 256, 0, h->stream>>>(h->u, h->T, perm, h->base[sys], lo, count, d_buf);
  return finish(h);
}

int nv_velocity_unpack(nv_handle *h, int32_t sys, int32_t lo, int32_t count, const double *d_buf) {
  if (!h || sys < 0 || sys >= h->nsys || lo < 1 || count < 0 || lo + count > h->cap[sys] + 1 || (count && !d_buf))
    return set_error(NV_ERR_ARG, "nv_velocity_unpack: bad arguments");
  const int *perm = tree_perm(h);
  if (!perm) return set_error(NV_ERR_STATE, "nv_velocity_unpack: no walk order (no tree built)");
  int rc = set_device(h);
  if (rc) return rc;
  if (count) k_vel_unpack<<<grid_for(count, 256), 256, 0, h->stream>>>(h->u, h->T, perm, h->base[sys], lo, count, d_buf);
  return finish(h);
}

int nv_step_velocity(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  if (nf_missing(h)) return NV_ERR_STATE;
  int rc = set_device(h);
  if (rc) return rc;
  launch_begin_step(h);
  launch_ghost(h);
  if (any_use_tree(h) || h->any_tree) launch_tree_build(h);
  launch_velocity(h);
  return finish(h);
}

int nv_step_finish(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  launch_ab3(h);
  launch_pinsert(h);
  launch_pclose(h, false);
  launch_precon(h);
  launch_wall_recon(h);
  launch_premove(h);
  launch_wrap(h, 3);
  launch_end_step(h);
  return finish(h);
}

int nv_set_walk_parts(nv_handle *h, int32_t parts) {
  if (!h || parts < 0 || parts > kMaxWalkParts || (parts & (parts - 1)))
    return set_error(NV_ERR_ARG, "nv_set_walk_parts: parts must be 0 (automatic), 1, 2, 4 or 8");
  int rc = set_device(h);
  if (rc) return rc;
  h->walk_parts = parts;
  if ((rc = rebuild_worklists(h))) return rc;
  h->graph_valid = false;  // the work list is a launch argument of the captured walk
  return NV_OK;
}

int nv_set_event_margins(nv_handle *h, int32_t on) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  for (int s = 0; s < h->nsys; ++s) {
    if ((rc = pull_dyn_one(h, s))) return rc;
    SysDyn &d = h->h_dyn[s];
    d.margin_on = on ? 1 : 0;
    for (double &v : d.margin) v = 1e300;
    NV_CUDA(cudaMemcpy(h->d_dyn + s, &d, sizeof(SysDyn), cudaMemcpyHostToDevice));
  }
  return NV_OK;
}

int nv_event_margins_get(nv_handle *h, int32_t sys, double *out) {
  if (!h || !out || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_event_margins_get: bad arguments");
  int rc = set_device(h);
  if (rc || (rc = pull_dyn_one(h, sys))) return rc;
  for (int k = 0; k < 4; ++k) out[k] = h->h_dyn[sys].margin[k];
  return NV_OK;
}

int nv_set_direct_split(nv_handle *h, int32_t targets_per_block) {
  const int g = targets_per_block;
  if (!h || !(g == 0 || g == 1 || g == 2 || g == 4 || g == 8 || g == 64))
    return set_error(NV_ERR_ARG, "nv_set_direct_split: targets_per_block must be 0 (automatic), 1, 2, 4, 8 or 64");
  int rc = set_device(h);
  if (rc) return rc;
  h->direct_split = g;
  if ((rc = rebuild_worklists(h))) return rc;
  h->graph_valid = false;  // the work list is a launch argument of the captured direct sum
  return NV_OK;
}

int nv_set_pclose_method(nv_handle *h, int32_t method) {
  if (!h || (method != 0 && method != 1))
    return set_error(NV_ERR_ARG, "nv_set_pclose_method: method must be 0 (cell list) or 1 (every slot)");
  h->pclose_method = method;
  h->graph_valid = false;  // the captured step holds the chosen kernels
  return NV_OK;
}

// Normal-fluid data: copy to the device, point the system's constants at it.
namespace {
int nf_upload(nv_handle *h, const double *src, size_t n, const double **dst) {
  void *p = nullptr;
  NV_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(double)));
  h->nf_buffers.push_back(p);
  NV_CUDA(cudaMemcpy(p, src, n * sizeof(double), cudaMemcpyHostToDevice));
  *dst = static_cast<const double *>(p);
  return NV_OK;
}
int sc_refresh(nv_handle *h, int sys) {
  NV_CUDA(cudaMemcpy(h->d_sc + sys, &h->sc[sys], sizeof(SysConst), cudaMemcpyHostToDevice));
  h->graph_valid = false;
  return NV_OK;
}
}  // namespace

int nv_set_normal_fluid_noise(nv_handle *h, int32_t sys, const double *noise, int32_t n) {
  if (!h || sys < 0 || sys >= h->nsys || !noise || n < 1)
    return set_error(NV_ERR_ARG, "nv_set_normal_fluid_noise: bad arguments");
  int rc = set_device(h);
  if (rc || (rc = nf_upload(h, noise, (size_t)n, &h->sc[sys].nf_noise))) return rc;
  h->sc[sys].nf_noise_n = n;
  return sc_refresh(h, sys);
}

int nv_set_normal_fluid_grid(nv_handle *h, int32_t sys, const double *u, int32_t nx, int32_t ny, int32_t nz,
                             const double *yp) {
  if (!h || sys < 0 || sys >= h->nsys || !u) return set_error(NV_ERR_ARG, "nv_set_normal_fluid_grid: bad arguments");
  SysConst &sc = h->sc[sys];
  const bool laizet = sc.nf_kind == NV_NF_LAIZET_DNS;
  if (!laizet && sc.nf_kind != NV_NF_TURB_DNS)
    return set_error(NV_ERR_STATE, "nv_set_normal_fluid_grid: the system's normal_velocity is not laizetDNS or turbDNS");
  if (laizet ? (nx != 128 || ny != 129 || nz != 84 || !yp) : (nx != 256 || ny != 256 || nz != 256))
    return set_error(NV_ERR_ARG, "nv_set_normal_fluid_grid: laizetDNS takes 128x129x84 and yp, turbDNS 256^3");
  int rc = set_device(h);
  if (rc) return rc;
  const size_t nn = (size_t)nx * ny * nz;
  std::vector<double> g(u, u + 3 * nn);
  if (laizet)
    for (auto &v : g) v = v / 2.;  // laizet_u=laizet_u/2. (normal_fluid.f90:178)
  std::vector<double> ax[3];
  const double pi = NV_PI;
  ax[0].resize(nx);
  ax[1].resize(ny);
  ax[2].resize(nz);
  if (laizet) {  // setup_laizet (normal_fluid.f90:183-189)
    for (int i = 1; i <= nx; ++i) ax[0][i - 1] = (i - 1) * (1. / 128) * 4 * pi - 2 * pi;
    for (int j = 0; j < ny; ++j) ax[1][j] = yp[j];
    for (int i = 1; i <= nz; ++i) ax[2][i - 1] = (i - 1) * (1. / 84) * 4 * pi / 3 - 4 * pi / 6;
    sc.nf_step[0] = (1. / 128) * 4 * pi;
    sc.nf_step[1] = 0.;
    sc.nf_step[2] = (1. / 84) * 4 * pi / 3;
  } else {  // setup_turbDNS (normal_fluid.f90:203-214)
    for (int a = 0; a < 3; ++a) {
      for (int i = 1; i <= 256; ++i) ax[a][i - 1] = (i - 1) * (1. / 256) * sc.box[a] - sc.box[a] / 2.;
      sc.nf_step[a] = (1. / 256) * sc.box[a];
    }
  }
  if ((rc = nf_upload(h, g.data(), g.size(), &sc.nf_grid))) return rc;
  for (int a = 0; a < 3; ++a) {
    if ((rc = nf_upload(h, ax[a].data(), ax[a].size(), &sc.nf_axis[a]))) return rc;
    sc.nf_n[a] = (int)ax[a].size();
  }
  return sc_refresh(h, sys);
}

int nv_set_insert_iterations(nv_handle *h, int32_t n) {
  if (!h || n < 0 || n > 64) return set_error(NV_ERR_ARG, "nv_set_insert_iterations: n must be 0..64");
  h->ins_iters = n;
  h->graph_valid = false;  // the iteration count shapes the captured step
  return NV_OK;
}

int nv_set_timing(nv_handle *h, int32_t on) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  h->timing = on != 0;
  return NV_OK;
}

int nv_step_launches(nv_handle *h, int32_t *n) {
  if (!h || !n) return set_error(NV_ERR_ARG, "nv_step_launches: bad arguments");
  int rc = set_device(h);
  if (rc || (rc = capture_step(h))) return rc;
  *n = h->step_kernels;
  return NV_OK;
}

int nv_calc_velocity(nv_handle *h, int32_t sys, double *u3) {
  if (!h || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_calc_velocity: bad arguments");
  if (nf_missing(h)) return NV_ERR_STATE;
  int rc = set_device(h);
  if (rc) return rc;
  time_begin(h, ST_GHOST);
  launch_ghost(h);
  time_end(h, ST_GHOST);
  time_begin(h, ST_TREE);
  if (h->any_tree) launch_tree_build(h);
  time_end(h, ST_TREE);
  time_begin(h, ST_VELOCITY);
  launch_velocity(h);
  time_end(h, ST_VELOCITY);
  if ((rc = finish(h))) return rc;
  if (h->timing) {
    const int st[] = {ST_GHOST, ST_TREE, ST_VELOCITY};
    for (int s : st) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, h->ev[2 * s], h->ev[2 * s + 1]) == cudaSuccess) h->stage_ms[s] += ms;
    }
  }
  if (!u3) return NV_OK;
  nv_host_state hs;
  std::memset(&hs, 0, sizeof hs);
  std::vector<int> inf(h->cap[sys]), beh(h->cap[sys]);
  hs.u = u3;
  hs.infront = inf.data();
  hs.behind = beh.data();
  if ((rc = nv_download(h, sys, &hs, h->cap[sys]))) return rc;
  for (int k = 0; k < hs.pcount; ++k)
    if (inf[k] == 0) u3[3 * k] = u3[3 * k + 1] = u3[3 * k + 2] = 0.0;
  return NV_OK;
}

int nv_calc_velocity_direct_at(nv_handle *h, int32_t sys, const int32_t *targets, int32_t n, double *u3) {
  if (!h || !targets || !u3 || sys < 0 || sys >= h->nsys || n < 0)
    return set_error(NV_ERR_ARG, "nv_calc_velocity_direct_at: bad arguments");
  int rc = set_device(h);
  if (rc || (rc = pull_dyn_one(h, sys))) return rc;
  std::vector<int> g(n);
  for (int k = 0; k < n; ++k) {
    if (targets[k] < 1 || targets[k] > h->h_dyn[sys].pcount)
      return set_error(NV_ERR_ARG, "nv_calc_velocity_direct_at: target slot out of range");
    g[k] = h->base[sys] + targets[k];
  }
  int *dt = nullptr;
  double *du = nullptr;
  NV_CUDA(cudaMalloc(&dt, std::max(n, 1) * sizeof(int)));
  NV_CUDA(cudaMalloc(&du, std::max(n, 1) * 3 * sizeof(double)));
  cudaMemcpy(dt, g.data(), n * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemset(du, 0, std::max(n, 1) * 3 * sizeof(double));
  launch_ghost(h);
  launch_direct_targets(h, sys, dt, n, du);
  rc = finish(h);
  if (rc == NV_OK) {
    cudaError_t e = cudaMemcpy(u3, du, n * 3 * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = check_cuda(e, "nv_calc_velocity_direct_at copy");
  }
  cudaFree(dt);
  cudaFree(du);
  return rc;
}

int nv_stage_times(nv_handle *h, double *ms, int32_t n) {
  if (!h || !ms) return set_error(NV_ERR_ARG, "nv_stage_times: bad arguments");
  if (h->timing_error != cudaSuccess)
    return check_cuda(h->timing_error, "stage timing (cudaEventElapsedTime)");
  for (int k = 0; k < n && k < ST_COUNT; ++k) ms[k] = h->stage_ms[k];
  return NV_OK;
}

int nv_tree_dump(nv_handle *h, int32_t sys, nv_tree_node *buf, int32_t cap, int32_t *n) {
  if (!h || !n || sys < 0 || sys >= h->nsys) return set_error(NV_ERR_ARG, "nv_tree_dump: bad arguments");
  int rc = set_device(h);
  if (rc) return rc;
  return tree_dump(h, sys, buf, cap, n);
}

int nv_diagnostics(nv_handle *h, int32_t sys, int64_t *out, int32_t n) {
  if (!h || !out || sys < 0 || sys >= h->nsys || n < 0 || n > 12) return set_error(NV_ERR_ARG, "nv_diagnostics: bad arguments");
  int rc = set_device(h);
  if (rc || (rc = pull_dyn_one(h, sys))) return rc;
  for (int k = 0; k < n; ++k) out[k] = h->h_dyn[sys].diag[k];
  return NV_OK;
}

int nv_sync(nv_handle *h) {
  if (!h) return set_error(NV_ERR_ARG, "null handle");
  int rc = set_device(h);
  if (rc) return rc;
  return finish(h);
}

}  // extern "C"
