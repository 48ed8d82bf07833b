// basic.cu -- per-slot stages: ghosts, local-only velocity, AB3 update, periodic wrap,
// and the per-step clock.  All are HBM-bound streaming kernels, one thread per slot,
// launched over every slot of every system (empty slots and slots beyond a system's
// pcount return at once).
#include "handle.cuh"

namespace {

constexpr int TB = 256;

__device__ __forceinline__ bool slot_of(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                                        const int *__restrict__ sys_of, long long g, int &s) {
  s = sys_of[g];
  const int k = (int)(g - scs[s].base);
  return k >= 1 && k <= dyn[s].pcount;
}

__global__ void k_begin_step(SysDyn *dyn, int nsys, const unsigned *err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || *err) return;
  dyn[s].itime += 1;
}

// ghostp (boundary.f90:10-19) + get_ghost_p (:26-84); also packs the segment records
// (x_j, gi_j - x_j, c_j) that the direct sums stage in shared memory: FP64 (2 x 32 B)
// and, for mixed precision, FP32 (3 x 16 B: position hi, position lo, segment).
__global__ void k_ghost(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                        const int *__restrict__ sys_of, const double *__restrict__ X,
                        const int *__restrict__ nxt, const int *__restrict__ prv,
                        double *__restrict__ GI, double *__restrict__ GB, double4 *__restrict__ seg,
                        float4 *__restrict__ seg32, long long T, const unsigned *err) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T || *err) return;
  int s;
  const bool in = slot_of(scs, dyn, sys_of, g, s);
  const int n = in ? nxt[g] : 0;
  if (n == 0) {
    seg[2 * g] = make_double4(0, 0, 0, 0);
    seg[2 * g + 1] = make_double4(0, 0, 0, 0);
    if (seg32) {
      seg32[3 * g] = make_float4(0, 0, 0, 0);
      seg32[3 * g + 1] = make_float4(0, 0, 0, 0);
      seg32[3 * g + 2] = make_float4(0, 0, 0, 0);
    }
    return;
  }
  const SysConst &sc = scs[s];
  const int b = prv[g];
  const int pin = sc.pin ? sc.pin[g] : 0;
  double x[3], xi[3], xb[3], gi[3], gb[3];
  load3(X, T, (int)g, x);
  load3(X, T, n, xi);
  load3(X, T, b, xb);
  ghosts_of(sc, pin, x, xi, xb, gi, gb);
  store3(GI, T, (int)g, gi);
  store3(GB, T, (int)g, gb);
  double d[3] = {e_sub(gi[0], x[0]), e_sub(gi[1], x[1]), e_sub(gi[2], x[2])};
  const double c = e_add(e_add(e_sq(d[0]), e_sq(d[1])), e_sq(d[2]));
  // a segment pinned in front goes into the wall: no Biot-Savart source (timestep.f90:161,187)
  seg[2 * g] = make_double4(x[0], x[1], x[2], pin_i(pin) ? 0.0 : 1.0);
  seg[2 * g + 1] = make_double4(d[0], d[1], d[2], c);
  if (seg32) {  // FP32 record: position split hi + lo (x = hi + lo to ~1e-16), segment vector
    const float h0 = (float)x[0], h1 = (float)x[1], h2 = (float)x[2];
    seg32[3 * g] = make_float4(h0, h1, h2, 1.0f);
    seg32[3 * g + 1] = make_float4((float)(x[0] - (double)h0), (float)(x[1] - (double)h1), (float)(x[2] - (double)h2), 0.0f);
    seg32[3 * g + 2] = make_float4((float)d[0], (float)d[1], (float)d[2], (float)c);
  }
}

// calc_velocity with velocity 'LIA' (timestep.f90:60-73): local term + MF only.
__global__ void k_velocity_lia(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                               const int2 *__restrict__ work, const double *__restrict__ X,
                               const double *__restrict__ GI, const double *__restrict__ GB,
                               const int *__restrict__ nxt, double *__restrict__ U, long long T,
                               const unsigned *err) {
  if (*err) return;
  const int2 w = work[blockIdx.x];
  const SysConst &sc = scs[w.x];
  const int g = w.y + threadIdx.x;
  const int k = g - sc.base;
  if (k > dyn[w.x].pcount || k > sc.cap || nxt[g] == 0) return;
  double x[3], gi[3], gb[3], u[3], fdot[3];
  load3(X, T, g, x);
  load3(GI, T, g, gi);
  load3(GB, T, g, gb);
  local_velocity(sc, x, gi, gb, u, fdot);
  mf_epilogue(sc, dyn[w.x], x, fdot, u, g);
  store3(U, T, g, u);
}

// Second loop of pmotion (timestep.f90:28-43): Euler / AB2 / AB3 by exact zero tests on
// the stored velocities, then u2 <- u1, u1 <- u.
__global__ void k_ab3(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                      const int *__restrict__ sys_of, const int *__restrict__ nxt, double *__restrict__ X,
                      const double *__restrict__ U, double *__restrict__ U1, double *__restrict__ U2,
                      long long T, const unsigned *err) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T || *err) return;
  int s;
  if (!slot_of(scs, dyn, sys_of, g, s) || nxt[g] == 0) return;
  const double dt = scs[s].dt;
  double x[3], u[3], u1[3], u2[3];
  load3(X, T, (int)g, x);
  load3(U, T, (int)g, u);
  load3(U1, T, (int)g, u1);
  load3(U2, T, (int)g, u2);
  const double m1 = fmax(fabs(u1[0]), fmax(fabs(u1[1]), fabs(u1[2])));
  const double m2 = fmax(fabs(u2[0]), fmax(fabs(u2[1]), fabs(u2[2])));
  if (m1 == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c] = e_add(x[c], e_mul(dt, u[c]));
  } else if (m2 == 0) {
    const double a = e_mul(3.0 / 2.0, dt), b = e_mul(1.0 / 2.0, dt);
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c] = e_sub(e_add(x[c], e_mul(a, u[c])), e_mul(b, u1[c]));
  } else {
    const double a = e_mul(23.0 / 12.0, dt), b = e_mul(4.0 / 3.0, dt), e = e_mul(5.0 / 12.0, dt);
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c] = e_add(e_sub(e_add(x[c], e_mul(a, u[c])), e_mul(b, u1[c])), e_mul(e, u2[c]));
  }
  store3(X, T, (int)g, x);
  store3(U2, T, (int)g, u1);
  store3(U1, T, (int)g, u);
}

// enforce_boundary (boundary.f90:91-138, periodic part) followed by NAN_finder
// (general.f90:172-190) over every slot 1..pcount.
__global__ void k_wrap(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                       const int *__restrict__ sys_of, const int *__restrict__ nxt, double *__restrict__ X,
                       long long T, unsigned *err, int mode) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T || *err) return;
  int s;
  if (!slot_of(scs, dyn, sys_of, g, s)) return;
  const SysConst &sc = scs[s];
  double x[3];
  load3(X, T, (int)g, x);
  if ((mode & 1) && nxt[g] != 0) {
    bool moved = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (!sc.periodic[c]) continue;
      const double L = sc.box[c];
      if (x[c] > (L / 2.0)) { x[c] = e_sub(x[c], L); moved = true; }
      else if (x[c] < (-L / 2.0)) { x[c] = e_add(x[c], L); moved = true; }
    }
    // a pinned point is set back on its wall (boundary.f90:123-136): the axis of the first
    // largest |wpinned| component, at +-0.499999999 of the box
    const int pin = sc.pin ? sc.pin[g] : 0;
    if (pin_i(pin) || pin_b(pin)) {
      int pc = 0;
      for (int c = 1; c < 3; ++c)
        if (abs(pin_w(pin, c)) > abs(pin_w(pin, pc))) pc = c;
      const int w = pin_w(pin, pc);
      if (w > 0) { x[pc] = e_mul(0.499999999, sc.box[pc]); moved = true; }
      else if (w < 0) { x[pc] = e_mul(-0.499999999, sc.box[pc]); moved = true; }
    }
    if (moved) store3(X, T, (int)g, x);
  }
  if ((mode & 2) && sc.nan_test && (isnan(x[0]) || isnan(x[1]) || isnan(x[2]))) set_err(err, DERR_NAN);
}

// randomise_normal_fluid (normal_fluid.f90:340-348), at the end of pmotion: the next noise
// sample, wrapping after the last.
__global__ void k_nf_advance(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, const unsigned *err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || *err || scs[s].nf_kind != NV_NF_NOISEY_XFLOW) return;
  int c = dyn[s].noise_counter + 1;
  if (c > scs[s].nf_noise_n) c = 1;
  dyn[s].noise_counter = c;
}

__global__ void k_end_step(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, const unsigned *err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || *err) return;
  dyn[s].t = dyn[s].t + scs[s].dt;
}

}  // namespace

void launch_begin_step(nv_handle *h) {
  k_begin_step<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(h->d_dyn, h->nsys, h->d_err);
}

void launch_ghost(nv_handle *h) {
  k_ghost<<<grid_for(h->T, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->nxt, h->prv,
                                                     h->gi, h->gb, h->seg, h->seg32, h->T, h->d_err);
}

void launch_velocity(nv_handle *h) {
  if (h->any_lia)
    k_velocity_lia<<<h->n_work_lia, h->direct_tb, 0, h->stream>>>(h->d_sc, h->d_dyn, h->d_work_lia, h->x,
                                                                  h->gi, h->gb, h->nxt, h->u, h->T, h->d_err);
  if (h->precision == NV_PREC_MIXED) {
    if (h->any_direct) {
      launch_direct_mixed(h);
      launch_mixed_combine(h, 1);
    }
    if (h->any_tree) {
      launch_tree_walk_mixed(h);
      launch_walk_fixup(h);
      launch_mixed_combine(h, 2);
    }
    join_root_sums(h);
    return;
  }
  if (h->any_direct) launch_direct(h);
  if (h->any_tree) {
    launch_tree_walk(h);
    launch_walk_fixup(h);
  }
  join_root_sums(h);
}

void launch_ab3(nv_handle *h) {
  k_ab3<<<grid_for(h->T, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->nxt, h->x, h->u, h->u1,
                                                   h->u2, h->T, h->d_err);
  bool noise = false;
  for (auto &s : h->sc) noise |= s.nf_kind == NV_NF_NOISEY_XFLOW;
  if (noise) k_nf_advance<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, h->d_err);
}

// mode bit 1: periodic wrap; bit 2: NaN check.
void launch_wrap(nv_handle *h, int mode) {
  k_wrap<<<grid_for(h->T, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->nxt, h->x, h->T,
                                                    h->d_err, mode);
}

void launch_end_step(nv_handle *h) {
  k_end_step<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, h->d_err);
}

// Ghost/segment pass on explicitly given buffers (used by the static-scratch entry point).
void launch_ghost_raw(cudaStream_t st, const SysConst *sc, const SysDyn *dyn, const int *sys_of, const double *x,
                      const int *nxt, const int *prv, double *gi, double *gb, double4 *seg, long long T,
                      unsigned *err) {
  k_ghost<<<grid_for(T, TB), TB, 0, st>>>(sc, dyn, sys_of, x, nxt, prv, gi, gb, seg, nullptr, T, err);
}
