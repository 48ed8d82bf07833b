// diag.cu -- calculate_diagnostics (src/diagnostic.f90:9-74) on the device.
//
// The reference calls it every `shots` steps: ghostp, then velocity_info (max |u|, max
// |u1 - u2|, mean |u_sup| and |u_mf|), curv_info (curvature |s''| per point, its mean, min
// over positive values and max) and stretching_rate (u . s'' per point).  Here one kernel
// computes the per-point curvature and stretching (kept for snapshots), and one block per
// system reduces them with the velocity norms.  Maxima and minima are exact; the sums run in
// a fixed order (per thread by stride, then a tree over the block) where the reference adds
// one point after another, so they agree with it to ~1e-13 relative.
#include <cfloat>
#include <cstdio>
#include <cstring>

#include "handle.cuh"

namespace {

constexpr int kDiagThreads = 256;

// curv_info's curvature (general.f90:53-61) and stretching_rate's u . s'' (diagnostic.f90:
// 60-74); 0 for empty slots.
__global__ void k_diag_slots(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                             const int *__restrict__ sys_of, const double *__restrict__ X,
                             const double *__restrict__ GI, const double *__restrict__ GB,
                             const double *__restrict__ U, const int *__restrict__ nxt, double *__restrict__ cs,
                             long long T) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T) return;
  const int s = sys_of[g];
  const int k = (int)(g - scs[s].base);
  if (k < 1 || k > dyn[s].pcount) return;
  double curv = 0., stretch = 0.;
  if (nxt[g] != 0) {
    double x[3], gi[3], gb[3], u[3], fdd[3];
    load3(X, T, (int)g, x);
    load3(GI, T, (int)g, gi);
    load3(GB, T, (int)g, gb);
    load3(U, T, (int)g, u);
    deriv2(x, gi, gb, fdd);
    curv = e_sqrt(dot3(fdd, fdd));
    stretch = dot3(u, fdd);
  }
  cs[g] = curv;
  cs[T + g] = stretch;
}

__device__ __forceinline__ double norm3(const double *__restrict__ a, long long T, long long g) {
  return e_sqrt(e_add(e_add(e_sq(a[g]), e_sq(a[T + g])), e_sq(a[2 * T + g])));
}

// One block per system: velocity_info and the reductions of curv_info over slots 1..pcount.
__global__ void __launch_bounds__(kDiagThreads) k_diag_reduce(const SysConst *__restrict__ scs,
                                                              const SysDyn *__restrict__ dyn, int nsys,
                                                              const double *__restrict__ U,
                                                              const double *__restrict__ U1,
                                                              const double *__restrict__ U2,
                                                              const double *__restrict__ usm,
                                                              const double *__restrict__ cs,
                                                              const int *__restrict__ nxt, DiagRec *rec,
                                                              long long T) {
  __shared__ double smax_u[kDiagThreads], smax_du[kDiagThreads], ssup[kDiagThreads], smf[kDiagThreads];
  __shared__ double scurv[kDiagThreads], skmax[kDiagThreads], skmin[kDiagThreads];
  __shared__ int slive[kDiagThreads];
  const int s = blockIdx.x;
  if (s >= nsys) return;
  const int base = scs[s].base, pc = dyn[s].pcount;
  const int t = threadIdx.x;
  double mu = -DBL_MAX, mdu = -DBL_MAX, sup = 0., smf_ = 0., sc_ = 0., kmax = -DBL_MAX, kmin = DBL_MAX;
  int live = 0;
  for (int k = 1 + t; k <= pc; k += kDiagThreads) {
    const long long g = base + k;
    mu = fmax(mu, norm3(U, T, g));
    const double d0 = e_sub(U1[g], U2[g]), d1 = e_sub(U1[T + g], U2[T + g]), d2 = e_sub(U1[2 * T + g], U2[2 * T + g]);
    mdu = fmax(mdu, e_sqrt(e_add(e_add(e_sq(d0), e_sq(d1)), e_sq(d2))));
    sup = e_add(sup, norm3(usm, T, g));
    smf_ = e_add(smf_, norm3(usm + 3 * T, T, g));
    const double c = cs[g];
    sc_ = e_add(sc_, c);
    kmax = fmax(kmax, c);
    if (c > 0.) kmin = fmin(kmin, c);
    live += nxt[g] > 0;
  }
  smax_u[t] = mu;
  smax_du[t] = mdu;
  ssup[t] = sup;
  smf[t] = smf_;
  scurv[t] = sc_;
  skmax[t] = kmax;
  skmin[t] = kmin;
  slive[t] = live;
  __syncthreads();
  for (int w = kDiagThreads / 2; w > 0; w >>= 1) {
    if (t < w) {
      smax_u[t] = fmax(smax_u[t], smax_u[t + w]);
      smax_du[t] = fmax(smax_du[t], smax_du[t + w]);
      ssup[t] = e_add(ssup[t], ssup[t + w]);
      smf[t] = e_add(smf[t], smf[t + w]);
      scurv[t] = e_add(scurv[t], scurv[t + w]);
      skmax[t] = fmax(skmax[t], skmax[t + w]);
      skmin[t] = fmin(skmin[t], skmin[t + w]);
      slive[t] += slive[t + w];
    }
    __syncthreads();
  }
  if (t == 0) {
    DiagRec r;
    r.maxu = smax_u[0];
    r.maxdu = smax_du[0];
    r.sum_usup = ssup[0];
    r.sum_umf = smf[0];
    r.sum_curv = scurv[0];
    r.kappa_max = skmax[0];
    r.kappa_min = skmin[0];  // minval over an empty mask: huge(0.), as Fortran gives
    r.live = slive[0];
    r.valid = 1;
    rec[s] = r;
  }
}

}  // namespace

int diag_launch(nv_handle *h) {
  launch_ghost(h);  // calculate_diagnostics refreshes the ghosts first (diagnostic.f90:13)
  k_diag_slots<<<grid_for(h->T, 256), 256, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->gi, h->gb, h->u,
                                                          h->nxt, h->cs, h->T);
  k_diag_reduce<<<h->nsys, kDiagThreads, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, h->u, h->u1, h->u2, h->usm,
                                                         h->cs, h->nxt, h->d_drec, h->T);
  return cudaGetLastError() == cudaSuccess ? NV_OK : set_error(NV_ERR_CUDA, "diagnostics launch failed");
}
