// noalloc.cu -- nv_calc_velocity_bs_static: the plain FP64 direct-sum velocity pass for one
// system whose state already sits in caller-owned device memory, with every scratch array
// (ghosts, segment records, work list, per-system constants, error word) carved out of one
// fixed static device array instead of memory the library allocates.
//
// The array is a file-scope __device__ symbol, so it exists on every GPU that loads the
// library, from module load until the process exits.  Host code cannot use the symbol's
// name as a device address; the first call on each device context looks the address up with
// cudaGetSymbolAddress (with that device current) and later calls in the same context reuse
// it.  A device reset creates a new context (and reloads the module), so the address is
// looked up again there.
#include <cstring>
#include <mutex>
#include <string>

#include "handle.cuh"

namespace {

constexpr int kS = NV_STATIC_MAX_SLOTS + 1;  // slots 0..max; slot 0 is the empty dummy
constexpr int kW = (NV_STATIC_MAX_SLOTS + 63) / 64;  // 64-target blocks of the direct sum

constexpr size_t align256(size_t n) { return (n + 255) & ~size_t(255); }
constexpr size_t kOffSc = 0;
constexpr size_t kOffDyn = kOffSc + align256(sizeof(SysConst));
constexpr size_t kOffErr = kOffDyn + align256(sizeof(SysDyn));
constexpr size_t kOffSysOf = kOffErr + 256;
constexpr size_t kOffWork = kOffSysOf + align256(sizeof(int) * kS);
constexpr size_t kOffX = kOffWork + align256(sizeof(int2) * kW);
constexpr size_t kOffGi = kOffX + align256(sizeof(double) * 3 * kS);
constexpr size_t kOffGb = kOffGi + align256(sizeof(double) * 3 * kS);
constexpr size_t kOffU = kOffGb + align256(sizeof(double) * 3 * kS);
constexpr size_t kOffNxt = kOffU + align256(sizeof(double) * 3 * kS);
constexpr size_t kOffPrv = kOffNxt + align256(sizeof(int) * kS);
constexpr size_t kOffSeg = kOffPrv + align256(sizeof(int) * kS);
constexpr size_t kBytes = kOffSeg + align256(sizeof(double4) * 2 * kS);

// The scratch of every call (about 5.6 MB for 32768 slots).
static __device__ __align__(256) unsigned char g_scratch[kBytes];

constexpr unsigned kErrLink = 1u << 8;  // a link outside 0..pcount

// Per device: the context the address was looked up in (its process-unique id) and the
// address.  A context id of 0 means "not set up".
struct ScratchAddr {
  unsigned long long ctx_id;
  unsigned char *ptr;
};
ScratchAddr g_addr[64] = {};
std::mutex g_setup;

// The id of the calling thread's current context (cuCtxGetCurrent + cuCtxGetId, reached
// through the runtime's driver entry points so that the library needs no -lcuda).
typedef int (*CtxGetCurrentFn)(void **);
typedef int (*CtxGetIdFn)(void *, unsigned long long *);
int current_context_id(unsigned long long *id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
    NV_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1));
    NV_CUDA(cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2));
    if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
      return set_error(NV_ERR_CUDA, "nv_calc_velocity_bs_static: driver context queries unavailable");
    get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    get_id = reinterpret_cast<CtxGetIdFn>(f2);
  }
  void *ctx = nullptr;
  if (get_current(&ctx) != 0) return set_error(NV_ERR_CUDA, "nv_calc_velocity_bs_static: cuCtxGetCurrent failed");
  if (!ctx) {  // no context current on this thread yet: the runtime's primary one
    int dev = 0;
    NV_CUDA(cudaGetDevice(&dev));
    NV_CUDA(cudaSetDevice(dev));  // initialises and binds the device's primary context
    if (get_current(&ctx) != 0 || !ctx)
      return set_error(NV_ERR_CUDA, "nv_calc_velocity_bs_static: no current CUDA context");
  }
  if (get_id(ctx, id) != 0 || *id == 0) return set_error(NV_ERR_CUDA, "nv_calc_velocity_bs_static: cuCtxGetId failed");
  return NV_OK;
}

// Device address of g_scratch in the current device's context: looked up once per context.
int scratch_base(unsigned char **out) {
  int dev = 0;
  NV_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(NV_ERR_ARG, "nv_calc_velocity_bs_static: device index above 63");
  unsigned long long ctx = 0;
  int rc = current_context_id(&ctx);
  if (rc != NV_OK) return rc;
  std::lock_guard<std::mutex> lock(g_setup);
  if (g_addr[dev].ctx_id != ctx) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return check_cuda(e, "cudaGetSymbolAddress(static scratch)");
    g_addr[dev] = ScratchAddr{ctx, static_cast<unsigned char *>(p)};
  }
  *out = g_addr[dev].ptr;
  return NV_OK;
}

// Caller's point-major arrays -> SoA scratch (1-based slots, slot 0 empty).
__global__ void k_static_pack(const double *__restrict__ x3, const int32_t *__restrict__ inf,
                              const int32_t *__restrict__ beh, int n, double *__restrict__ X, int *__restrict__ nxt,
                              int *__restrict__ prv, unsigned *err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > n) return;
  if (k == 0) {
    X[0] = X[kS] = X[2 * kS] = 0.0;
    nxt[0] = prv[0] = 0;
    return;
  }
  const int a = inf[k - 1], b = beh[k - 1];
  if (a < 0 || a > n || b < 0 || b > n || (a == 0) != (b == 0)) atomicOr(err, kErrLink);
  nxt[k] = (a < 0 || a > n) ? 0 : a;
  prv[k] = (b < 0 || b > n) ? 0 : b;
  for (int c = 0; c < 3; ++c) X[c * kS + k] = x3[3 * (k - 1) + c];
}

// SoA velocities -> the caller's point-major output (0 for empty slots).  After any device
// error (bad links, a wait that gave up) the output is left untouched: U would hold another
// call's velocities.
__global__ void k_static_unpack(const double *__restrict__ U, const int *__restrict__ nxt, int n, double *__restrict__ u3,
                                const unsigned *__restrict__ err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (k > n || *err) return;
  const bool live = nxt[k] != 0;
  for (int c = 0; c < 3; ++c) u3[3 * (k - 1) + c] = live ? U[c * kS + k] : 0.0;
}

}  // namespace

extern "C" int nv_calc_velocity_bs_static(const nv_params *p, int32_t pcount, const double *d_x3,
                                          const int32_t *d_infront, const int32_t *d_behind, double t,
                                          double *d_u3, void *stream) {
  if (!p || !d_x3 || !d_infront || !d_behind || !d_u3)
    return set_error(NV_ERR_ARG, "nv_calc_velocity_bs_static: null argument");
  if (pcount < 1 || pcount > NV_STATIC_MAX_SLOTS)
    return set_error(NV_ERR_CAPACITY, "nv_calc_velocity_bs_static: pcount must be 1.." +
                                          std::to_string(NV_STATIC_MAX_SLOTS) + " (size of the static scratch)");
  if (p->velocity != NV_VEL_BS)
    return set_error(NV_ERR_ARG, "nv_calc_velocity_bs_static: only velocity BS (the direct sum) is provided");
  int rc = nv_check_params(p);
  if (rc != NV_OK) return rc;
  for (int c = 0; c < 3; ++c)
    if (p->boundary[c] == NV_BC_SOLID)
      return set_error(NV_ERR_UNSUPPORTED, "nv_calc_velocity_bs_static: solid boundaries need pinned records");
  unsigned char *base = nullptr;
  if ((rc = scratch_base(&base)) != NV_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  SysConst *d_sc = reinterpret_cast<SysConst *>(base + kOffSc);
  SysDyn *d_dyn = reinterpret_cast<SysDyn *>(base + kOffDyn);
  unsigned *d_err = reinterpret_cast<unsigned *>(base + kOffErr);
  int *sys_of = reinterpret_cast<int *>(base + kOffSysOf);
  int2 *work = reinterpret_cast<int2 *>(base + kOffWork);
  double *X = reinterpret_cast<double *>(base + kOffX);
  double *GI = reinterpret_cast<double *>(base + kOffGi);
  double *GB = reinterpret_cast<double *>(base + kOffGb);
  double *U = reinterpret_cast<double *>(base + kOffU);
  int *nxt = reinterpret_cast<int *>(base + kOffNxt);
  int *prv = reinterpret_cast<int *>(base + kOffPrv);
  double4 *seg = reinterpret_cast<double4 *>(base + kOffSeg);

  // Host-side records of this call (stack memory; the copies are staged before returning).
  const SysConst sc = sysconst_for(*p, 0, pcount);
  SysDyn dyn;
  std::memset(&dyn, 0, sizeof dyn);
  dyn.pcount = pcount;
  dyn.t = t;
  int2 wl[kW];
  const int nwork = (pcount + 63) / 64;
  for (int b = 0; b < nwork; ++b) wl[b] = make_int2(0, 1 + 64 * b);
  NV_CUDA(cudaMemcpyAsync(d_sc, &sc, sizeof sc, cudaMemcpyHostToDevice, st));
  NV_CUDA(cudaMemcpyAsync(d_dyn, &dyn, sizeof dyn, cudaMemcpyHostToDevice, st));
  NV_CUDA(cudaMemcpyAsync(work, wl, nwork * sizeof(int2), cudaMemcpyHostToDevice, st));
  // the array keeps the previous call's contents: clear what must start at zero
  NV_CUDA(cudaMemsetAsync(d_err, 0, sizeof(unsigned), st));
  NV_CUDA(cudaMemsetAsync(sys_of, 0, sizeof(int) * kS, st));
  k_static_pack<<<grid_for(pcount + 1, 256), 256, 0, st>>>(d_x3, d_infront, d_behind, pcount, X, nxt, prv, d_err);
  launch_ghost_raw(st, d_sc, d_dyn, sys_of, X, nxt, prv, GI, GB, seg, kS, d_err);
  launch_direct_raw(st, d_sc, d_dyn, work, nwork, X, GI, GB, nxt, prv, seg, U, kS, d_err);
  k_static_unpack<<<grid_for(pcount, 256), 256, 0, st>>>(U, nxt, pcount, d_u3, d_err);
  NV_CUDA(cudaGetLastError());
  NV_CUDA(cudaStreamSynchronize(st));
  unsigned bits = 0;
  NV_CUDA(cudaMemcpy(&bits, d_err, sizeof bits, cudaMemcpyDeviceToHost));
  if (bits & kErrLink)
    return set_error(NV_ERR_ARG, "nv_calc_velocity_bs_static: infront/behind out of range or disagreeing on an "
                                 "empty slot (output left unwritten)");
  if (bits) {
    std::string msg;
    const int code = status_from_device_bits(bits, msg);
    return set_error(code, "nv_calc_velocity_bs_static: " + msg + " (output left unwritten)");
  }
  return NV_OK;
}
