// common.cuh -- shared device-side definitions of libnuvort_gpu.
//
// Device layout (one handle, nsys systems):
//   * Global slot index g.  System s owns slots [base_s, base_s + cap_s]; slot base_s is
//     an unused dummy (the reference's slot 0), slot base_s + k is the reference's f(k).
//     System 0's dummy is global slot 0, so a link value 0 means "empty" in every system.
//   * Links (infront/behind/closest) hold GLOBAL slot indices; the host converts to and
//     from the reference's 1-based system-local numbering at upload/download.  The map is
//     monotone inside a system, so "lowest j" tie-breaks are unchanged.
//   * FP64 per-slot arrays are SoA: component c of slot g is a[c * T + g].
//   * seg: the Biot-Savart segment of each slot, packed for staged tile loads.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/nuvort_gpu.h"

#define NV_PI 3.14159265358979324
#define NV_EPS 2.220446049250313e-16  // epsilon(0.) for real(8)

// Device error word bits (OR-ed by kernels, read by the host after launches).
enum : unsigned {
  DERR_SINGULAR = 1u << 0,
  DERR_TREE_DEPTH = 1u << 1,
  DERR_NAN = 1u << 2,
  DERR_EMPTY = 1u << 3,
  DERR_CAPACITY = 1u << 4,
  DERR_QUEUE = 1u << 5,
  DERR_TIMEOUT = 1u << 6,
  DERR_TREE_NODES = 1u << 7,
  DERR_WALK = 1u << 8,  // a tree walk visited more nodes than the tree holds
};

struct SysConst {
  double dt, delta, quant_circ, corea;
  double box[3];
  double tree_theta;
  double beta_pref;   // quant_circ/(4.*pi)       timestep.f90:79
  double log_pref;    // 1.1/corea                timestep.f90:79
  double two_pi;      // 2*pi                     timestep.f90:168
  double alpha[2];
  double vn[3];       // get_normal_velocity(x) for the uniform cases, +super_velocity
  double super_velocity[3];
  double normal_fluid_cutoff, t_zero_normal_fluid;
  double bsize;       // maxval(box_size)         tree.f90:45
  double shift[26][3];
  int velocity;
  int periodic[3];
  int tree_extra_correction;
  int mf_on;          // (|alpha(1)|>eps .or. |alpha(2)|>eps)   timestep.f90:126
  int n_shift;
  int recon_shots;
  int nan_test;
  int use_tree;       // tree_theta>0 (run.f90:29,37)
  int base, cap;
  int sched_tree;     // non-local sum by the tree walk (velocity==Tree)
  // f(:)%u_sup and f(:)%u_mf (timestep.f90:123,137) of the handle's slots: [6][usm_T],
  // components 0-2 u_sup, 3-5 u_mf; null where they are not kept
  double *usm;
  long long usm_T;
  // position-dependent normal fluid (normal_fluid.f90:83-118); vn above serves zero / xflow /
  // uniform
  int nf_kind;                 // NV_NF_*
  double nf_a, nf_omega;       // norm_vel_xflow, norm_shear_omega
  const double *nf_noise;      // noisey_xflow samples
  int nf_noise_n;
  const double *nf_grid;       // laizetDNS / turbDNS: u [3][nz][ny][nx]
  const double *nf_axis[3];    // xp, yp, zp
  int nf_n[3];
  double nf_step[3];           // grid spacing of the interpolation weights (y of laizet: 0, from yp)
  // solid walls (boundary.f90:26-42,180-212; timestep.f90:201-234): pinned flags per slot
  // (global index; see pin_*), the mirror images' reflections in create_mirror_loop_array
  // order, the tree's mirror sums per slot; all null / 0 for a system without solid walls
  const int *pin;
  double *umir;
  int n_mirror;
  int mirror[26][3];
  int solid[3];
  // the tree walks compute targets at walk positions walk_lo <= q < walk_hi only (the walk
  // order: the system's dummy slot, its live points in Morton order, its empty slots); all
  // by default, a range when one tangle's velocity is split over several GPUs
  int walk_lo, walk_hi;
};

// Pinned-point record of a slot: bit 0 pinnedi, bit 1 pinnedb, bits 2-7 wpinned(1..3), two
// bits each (0, +1, or 3 for -1).  0 for every point away from a solid wall.
__host__ __device__ __forceinline__ bool pin_i(int p) { return p & 1; }
__host__ __device__ __forceinline__ bool pin_b(int p) { return p & 2; }
__host__ __device__ __forceinline__ int pin_w(int p, int c) {
  const int v = (p >> (2 + 2 * c)) & 3;
  return v == 3 ? -1 : v;
}
__host__ __device__ __forceinline__ int pin_encode(int pinnedi, int pinnedb, const int w[3]) {
  int p = (pinnedi ? 1 : 0) | (pinnedb ? 2 : 0);
  for (int c = 0; c < 3; ++c) p |= ((w[c] < 0 ? 3 : w[c] > 0 ? 1 : 0) << (2 + 2 * c));
  return p;
}

struct SysDyn {
  int pcount;
  int itime;
  double t;
  int recon_count, remove_count, insert_count, loop_kills;
  unsigned long long tree_eval;
  unsigned long long tree_tests;
  int event_seq;
  unsigned long long ev_hash;  // sum of event_digest over this system's events
  int live;          // pinsert: the system has a live point (src/line.f90:25-27)
  int nlive;         // live slots: set by nv_upload, kept by the topology stages' events
  int old_pcount;
  int ins_fallback;  // pinsert needs the serial sweep this step
  int ins_conv;      // pinsert's fixed-point iteration has converged
  int ins_mismatch;  // positions where the iteration's H and H' differ
  int noise_counter; // noisey_xflow: 1-based sample in use (xflow_noise_counter)
  int wall_recon_count;  // wall_recon cuts (reconnection.f90:91)
  long long diag[12];  // see nv_diagnostics
  double total_length;  // pinsert: sum of the segment lengths it measured (line.f90:39)
  double avg_sep;       // pinsert: total_length / (old_pcount - empty slots) (line.f90:95)
  // Event margins while margin_on: the smallest |value - threshold| / threshold of the
  // topology tests since they were switched on -- [0] pinsert's length > delta, [1] premove's
  // distance < .99 delta, [2] precon's closestd < delta/2, [3] precon's tangent dot > 0.9.
  int margin_on;
  double margin[4];
};

// Lowers margin[k] of d to |value - thr| / thr while the margins are on (the IEEE order of
// non-negative doubles is that of their bit patterns; most values lose to the plain read).
__device__ __forceinline__ void margin_note_abs(SysDyn &d, int k, double absdiff, double thr) {
  const double v = absdiff / thr;
  if (v < *(volatile double *)&d.margin[k])
    atomicMin((unsigned long long *)&d.margin[k], (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void margin_note(SysDyn &d, int k, double value, double thr) {
  if (d.margin_on) margin_note_abs(d, k, fabs(value - thr), thr);
}

// Reductions of calculate_diagnostics (diagnostic.f90:9-74) per system.
struct DiagRec {
  double maxu, maxdu;         // velocity_info
  double sum_usup, sum_umf;   // sums of |u_sup|, |u_mf| over every slot
  double sum_curv, kappa_max, kappa_min;  // curv_info (kappa_min over curvatures > 0; 0 if none)
  int live;                   // count(f(:)%infront>0)
  int valid;                  // set by a diagnostics pass
};

// Order-sensitive digest of one event (system-local slots; a loop kill's j is its count):
// the per-system sum over all events is equal for two runs whose event sequences agree,
// and differs otherwise except for 64-bit collisions.  splitmix64 finaliser as the mixer.
__device__ __forceinline__ unsigned long long digest_mix(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ unsigned long long event_digest(int seq, int itime, int kind, int i, int j) {
  unsigned long long h = digest_mix((unsigned long long)(unsigned)seq);
  h = digest_mix(h ^ (((unsigned long long)(unsigned)i << 32) | (unsigned)j));
  return digest_mix(h ^ (((unsigned long long)(unsigned)itime << 8) | (unsigned)kind));
}

// One logged topology event (system-local numbering is restored on the host).
struct DevEvent {
  int sys, seq, itime, kind, i, j;
};

// ---- exact IEEE FP64 operations (no FMA contraction), matching one rounding per op ----
__device__ __forceinline__ double e_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double e_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double e_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double e_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double e_sqrt(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ double e_sq(double a) { return __dmul_rn(a, a); }

// p + 2|r| (r L/2 - p): the cartesian reflection of one coordinate in the wall r (-1, 0, +1)
// of an axis of length L, in the reference's order (timestep.f90:221-222, boundary.f90:35)
__device__ __forceinline__ double reflect1(double p, int r, double L) {
  return e_add(p, e_mul((double)(2 * (r < 0 ? -r : r)), e_sub(e_mul(e_mul(0.5, (double)r), L), p)));
}

// dist_gen (derivatives.f90:40-47)
__device__ __forceinline__ double dist_gen(const double a[3], const double b[3]) {
  return e_sqrt(e_add(e_add(e_sq(e_sub(a[0], b[0])), e_sq(e_sub(a[1], b[1]))), e_sq(e_sub(a[2], b[2]))));
}
__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  return e_add(e_add(e_mul(a[0], b[0]), e_mul(a[1], b[1])), e_mul(a[2], b[2]));
}
// cross_product (general.f90:152-159)
__device__ __forceinline__ void cross3(const double a[3], const double b[3], double c[3]) {
  c[0] = e_sub(e_mul(a[1], b[2]), e_mul(a[2], b[1]));
  c[1] = e_sub(e_mul(a[2], b[0]), e_mul(a[0], b[2]));
  c[2] = e_sub(e_mul(a[0], b[1]), e_mul(a[1], b[0]));
}

__device__ __forceinline__ void load3(const double *__restrict__ a, long long T, int g, double v[3]) {
  v[0] = a[g];
  v[1] = a[T + g];
  v[2] = a[2 * T + g];
}
__device__ __forceinline__ void store3(double *__restrict__ a, long long T, int g, const double v[3]) {
  a[g] = v[0];
  a[T + g] = v[1];
  a[2 * T + g] = v[2];
}

// get_ghost_p (boundary.f90:26-84, non-pinned branch): neighbour positions unwrapped
// across periodic faces relative to x.
__device__ __forceinline__ void ghost_adjust(const SysConst &sc, const double x[3], double g[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!sc.periodic[c]) continue;
    const double L = sc.box[c];
    const double h = L / 2.0;
    if (e_sub(x[c], g[c]) > h) g[c] = e_add(g[c], L);
    else if (e_sub(x[c], g[c]) < -h) g[c] = e_sub(g[c], L);
  }
}

// get_ghost_p (boundary.f90:26-84) from the neighbours' positions xi = x(infront), xb =
// x(behind): a point pinned in front (pinnedi, the segment into the wall) takes its behind
// point and that point's reflection in its wall as the point in front; pinned behind, the
// mirror image; both then unwrapped across the periodic faces.
__device__ __forceinline__ void ghosts_of(const SysConst &sc, int pin, const double x[3], const double xi[3],
                                          const double xb[3], double gi[3], double gb[3]) {
  for (int c = 0; c < 3; ++c) {
    if (pin_i(pin)) {
      gb[c] = xb[c];
      gi[c] = reflect1(xb[c], pin_w(pin, c), sc.box[c]);
    } else if (pin_b(pin)) {
      gi[c] = xi[c];
      gb[c] = reflect1(xi[c], pin_w(pin, c), sc.box[c]);
    } else {
      gi[c] = xi[c];
      gb[c] = xb[c];
    }
  }
  ghost_adjust(sc, x, gi);
  ghost_adjust(sc, x, gb);
}

// get_deriv_1 / get_deriv_2 (derivatives.f90:11-36)
__device__ __forceinline__ void deriv1(const double x[3], const double gi[3], const double gb[3],
                                       double s[3]) {
  const double disti = dist_gen(x, gi), distb = dist_gen(x, gb);
  const double den = e_mul(e_mul(2.0, distb), disti);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double v = e_sub(e_add(e_mul(distb, gi[c]), e_mul(e_sub(disti, distb), x[c])), e_mul(disti, gb[c]));
    s[c] = e_div(v, den);
  }
}
__device__ __forceinline__ void deriv2(const double x[3], const double gi[3], const double gb[3],
                                       double s[3]) {
  const double disti = dist_gen(x, gi), distb = dist_gen(x, gb);
  const double d1 = e_mul(disti, e_add(disti, distb));
  const double d2 = e_mul(disti, distb);
  const double d3 = e_mul(distb, e_add(disti, distb));
#pragma unroll
  for (int c = 0; c < 3; ++c)
    s[c] = e_mul(2.0, e_add(e_sub(e_div(gi[c], d1), e_div(x[c], d2)), e_div(gb[c], d3)));
}

// new point of an insertion (line.f90:62-79)
__device__ __forceinline__ void new_point(const double x[3], const double gi[3], const double gb[3], double disti,
                                          double xn[3]) {
  double fdd[3];
  deriv2(x, gi, gb, fdd);
  double curv = e_sqrt(dot3(fdd, fdd));
  const double mid[3] = {e_mul(0.5, e_add(x[0], gi[0])), e_mul(0.5, e_add(x[1], gi[1])), e_mul(0.5, e_add(x[2], gi[2]))};
  for (int c = 0; c < 3; ++c) xn[c] = mid[c];
  if (curv > 1E-5) {
    curv = e_div(1.0, curv);
    const double disc = e_sub(e_mul(curv, curv), e_mul(0.25, e_mul(disti, disti)));
    if (disc > 0.) {
      const double sfac = e_mul(e_sub(e_sqrt(disc), curv), curv);
      for (int c = 0; c < 3; ++c) xn[c] = e_add(mid[c], e_mul(sfac, fdd[c]));
    }
  }
}

// A system with solid walls carries pinned records; its topology stages run as the exact
// serial sweeps of solid.cu and the parallel ones skip it.
__device__ __forceinline__ bool walled(const SysConst &sc) { return sc.pin != nullptr; }
__device__ __forceinline__ bool pinned_at(const SysConst &sc, int g) {
  return sc.pin && (sc.pin[g] & 3);
}

// Local part of calc_velocity (timestep.f90:60-80,102-105): u = beta s' x s''.
__device__ __forceinline__ void local_velocity(const SysConst &sc, const double x[3],
                                               const double gi[3], const double gb[3], double u[3],
                                               double fdot[3]) {
  double fddot[3], cr[3];
  deriv1(x, gi, gb, fdot);
  deriv2(x, gi, gb, fddot);
  double beta;
  if (sc.velocity == NV_VEL_LIA) {
    double curv = e_sqrt(dot3(fddot, fddot));
    if (curv < NV_EPS) curv = NV_EPS;
    else curv = e_div(1.0, curv);
    beta = e_mul(sc.beta_pref, log(e_div(e_mul(4.6, curv), sc.corea)));
  } else {
    beta = e_mul(sc.beta_pref, log(e_mul(sc.log_pref, e_sqrt(e_mul(dist_gen(x, gi), dist_gen(x, gb))))));
  }
  cross3(fdot, fddot, cr);
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = e_mul(beta, cr[c]);
}

// Grid node of a coordinate for the DNS interpolation (laizet_interp / turbDNS_interp,
// normal_fluid.f90:225-338): n = minloc(|x - axis|) (the first on a tie); if x lies above it
// the pair is (n, n+1), else (n-1, n); n+1 past the last node wraps to the first on a
// periodic axis.  Positions below the first node (the reference then reads index 0, outside
// its array) wrap to the last node on a periodic axis, clamp on a closed one.
__device__ __forceinline__ void grid_pair(const double *__restrict__ ax, int n, double x, bool periodic, int &lo,
                                          int &hi) {
  int best = 0;
  double bd = fabs(x - ax[0]);
  for (int i = 1; i < n; ++i) {
    const double d = fabs(x - ax[i]);
    if (d < bd) {
      bd = d;
      best = i;
    }
  }
  if (x > ax[best]) {
    lo = best;
    hi = best + 1;
  } else {
    lo = best - 1;
    hi = best;
  }
  if (lo < 0) lo = periodic ? n - 1 : 0;
  if (hi >= n) hi = periodic ? 0 : n - 1;
}

// get_normal_velocity (normal_fluid.f90:83-118) at x and time t, +super_velocity; un must be
// the field the caller uses when t < t_zero_normal_fluid.
__device__ __forceinline__ void normal_velocity(const SysConst &sc, int noise_counter, const double x[3], double t,
                                                double un[3]) {
  switch (sc.nf_kind) {
    case NV_NF_SHEAR_XFLOW:  // :98-99
      un[0] = e_mul(sc.nf_a, sin(e_add(e_div(e_mul(2 * NV_PI, x[2]), sc.box[2]), e_mul(t, sc.nf_omega))));
      un[1] = un[2] = 0.0;
      break;
    case NV_NF_YCHANNEL: {  // :100-101
      const double q = e_div(e_mul(2.0, x[1]), sc.box[1]);
      un[0] = e_mul(sc.nf_a, e_sub(1.0, e_mul(q, q)));
      un[1] = un[2] = 0.0;
      break;
    }
    case NV_NF_CHANNEL: {  // :102-108
      double cossum = 0.0;
      for (int ii = 1; ii <= 10; ++ii) {
        const double ak = e_mul((double)(2 * ii - 1), e_div(NV_PI, 2.0));
        const double sgn = (ii & 1) ? -1.0 : 1.0;  // (-1)**ii
        const double ak3 = e_mul(e_mul(ak, ak), ak);
        const double ch = cosh(e_div(e_mul(e_mul(ak, 2.0), x[1]), sc.box[1]));
        const double co = cos(e_div(e_mul(e_mul(ak, 2.0), x[2]), sc.box[2]));
        cossum = e_add(cossum, e_div(e_mul(e_mul(4.0, e_div(sgn, ak3)), e_mul(ch, co)), cosh(ak)));
      }
      const double q = e_div(e_mul(2.0, x[2]), sc.box[2]);
      un[0] = e_mul(e_mul(sc.nf_a, e_add(e_sub(1.0, e_mul(q, q)), cossum)), 1.2);
      un[1] = un[2] = 0.0;
      break;
    }
    case NV_NF_NOISEY_XFLOW:  // :96-97 with the sample of this step (no samples: no flow)
      un[0] = sc.nf_noise ? e_mul(sc.nf_noise[noise_counter - 1], sc.nf_a) : 0.0;
      un[1] = un[2] = 0.0;
      break;
    case NV_NF_LAIZET_DNS:
    case NV_NF_TURB_DNS: {  // :225-338 trilinear interpolation (no grid: no flow)
      if (!sc.nf_grid) {
        un[0] = un[1] = un[2] = 0.0;
        break;
      }
      const bool turb = sc.nf_kind == NV_NF_TURB_DNS;
      int lo[3], hi[3];
      for (int a = 0; a < 3; ++a) grid_pair(sc.nf_axis[a], sc.nf_n[a], x[a], turb || a != 1, lo[a], hi[a]);
      const double xd = e_div(e_sub(x[0], sc.nf_axis[0][lo[0]]), sc.nf_step[0]);
      const double yd = turb ? e_div(e_sub(x[1], sc.nf_axis[1][lo[1]]), sc.nf_step[1])
                             : e_div(e_sub(x[1], sc.nf_axis[1][lo[1]]), e_sub(sc.nf_axis[1][hi[1]], sc.nf_axis[1][lo[1]]));
      const double zd = e_div(e_sub(x[2], sc.nf_axis[2][lo[2]]), sc.nf_step[2]);
      const long long nx = sc.nf_n[0], nxy = (long long)sc.nf_n[0] * sc.nf_n[1], nn = nxy * sc.nf_n[2];
      auto at = [&](int i, int j, int k, int c) { return sc.nf_grid[c * nn + k * nxy + j * nx + i]; };
      for (int c = 0; c < 3; ++c) {
        const double c00 = e_add(e_mul(at(lo[0], lo[1], lo[2], c), e_sub(1.0, xd)), e_mul(at(hi[0], lo[1], lo[2], c), xd));
        const double c10 = e_add(e_mul(at(lo[0], hi[1], lo[2], c), e_sub(1.0, xd)), e_mul(at(hi[0], hi[1], lo[2], c), xd));
        const double c01 = e_add(e_mul(at(lo[0], lo[1], hi[2], c), e_sub(1.0, xd)), e_mul(at(hi[0], lo[1], hi[2], c), xd));
        const double c11 = e_add(e_mul(at(lo[0], hi[1], hi[2], c), e_sub(1.0, xd)), e_mul(at(hi[0], hi[1], hi[2], c), xd));
        const double c0 = e_add(e_mul(c00, e_sub(1.0, yd)), e_mul(c10, yd));
        const double c1 = e_add(e_mul(c01, e_sub(1.0, yd)), e_mul(c11, yd));
        un[c] = e_add(e_mul(c0, e_sub(1.0, zd)), e_mul(c1, zd));
      }
      break;
    }
    default:  // zero, xflow, uniform: a constant field
      for (int c = 0; c < 3; ++c) un[c] = e_sub(sc.vn[c], sc.super_velocity[c]);
  }
  for (int c = 0; c < 3; ++c) un[c] = e_add(un[c], sc.super_velocity[c]);  // :117
}

// Mutual friction and imposed flow (timestep.f90:123-140); u holds u_sup on entry, x is the
// point's position (the normal fluid's argument).  For the velocity pass of a step (slot
// g >= 0) u_sup and u_mf are kept as the reference stores them in f(g) (u_mf only when it is
// computed); g < 0 keeps nothing.
__device__ __forceinline__ void mf_epilogue(const SysConst &sc, const SysDyn &dy, const double x[3],
                                            const double fdot[3], double u[3], long long g = -1) {
  const double t = dy.t;
  const bool keep = sc.usm && g >= 0;
  if (keep)
#pragma unroll
    for (int c = 0; c < 3; ++c) sc.usm[c * sc.usm_T + g] = u[c];
  if (sc.mf_on && t < sc.normal_fluid_cutoff) {
    double un[3], w[3], c1[3], c2[3], umf[3];
    if (t < sc.t_zero_normal_fluid) {
      if (sc.nf_kind <= NV_NF_UNIFORM) {
#pragma unroll
        for (int c = 0; c < 3; ++c) un[c] = sc.vn[c];
      } else {
        normal_velocity(sc, dy.noise_counter, x, t, un);
      }
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) un[c] = 0.0;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) w[c] = e_sub(un[c], u[c]);
    cross3(fdot, w, c1);
    cross3(fdot, c1, c2);
#pragma unroll
    for (int c = 0; c < 3; ++c) umf[c] = e_sub(e_mul(sc.alpha[0], c1[c]), e_mul(sc.alpha[1], c2[c]));
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], umf[c]);
    if (keep)
#pragma unroll
      for (int c = 0; c < 3; ++c) sc.usm[(3 + c) * sc.usm_T + g] = umf[c];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], sc.super_velocity[c]);
}

// One desingularised segment term (timestep.f90:162-170 / 188-196), reference order:
//   u_bs = (r x d) * quant_circ / ((2 pi)(4ac - b^2)) * ((2c+b)/sqrt(a+b+c) - b/sqrt(a)).
// Returns false when the reference skips the term (4ac-b^2 == 0 exactly).
__device__ __forceinline__ bool bs_term_exact(const double r[3], const double d[3], double a,
                                              double c, double qc, double two_pi, double out[3]) {
  const double b = e_mul(2.0, dot3(r, d));
  const double D = e_sub(e_mul(e_mul(4.0, a), c), e_mul(b, b));
  if (D == 0.0) return false;
  double cr[3];
  cross3(r, d, cr);
  const double den = e_mul(two_pi, D);
  const double fac = e_sub(e_div(e_add(e_mul(2.0, c), b), e_sqrt(e_add(e_add(a, b), c))), e_div(b, e_sqrt(a)));
#pragma unroll
  for (int k = 0; k < 3; ++k) out[k] = e_mul(e_div(e_mul(cr[k], qc), den), fac);
  return true;
}

__device__ __forceinline__ void set_err(unsigned *err, unsigned bit) { atomicOr(err, bit); }

// biot_savart_mirror's test (timestep.f90:214-217) of whether target g skips its own image
// in mirror m: the sum of wpinned(g) - reflect is zero and the sum of wpinned(g) is below 2
// (component sums, as the reference writes them).
__device__ __forceinline__ bool mirror_skips_own(const SysConst &sc, int pin_g, int m) {
  int d = 0, w = 0;
  for (int c = 0; c < 3; ++c) {
    d += pin_w(pin_g, c) - sc.mirror[m][c];
    w += pin_w(pin_g, c);
  }
  return d == 0 && w < 2;
}

// One term of biot_savart_mirror (timestep.f90:201-234): segment j (x_j to ghosti_j) reflected
// in mirror m, its orientation reversed (from the reflected ghost to the reflected point), at
// target g (position xi, pinned record pin_g, behind pi); false when the reference skips it.
__device__ __forceinline__ bool mirror_term(const SysConst &sc, int m, const double *__restrict__ X,
                                            const double *__restrict__ GI, const int *__restrict__ nxt, long long T,
                                            int j, int g, int pi, int pin_g, bool skip_own, const double xi[3],
                                            double out[3]) {
  if (nxt[j] == 0 || pin_i(sc.pin[j])) return false;
  if (skip_own && ((pin_b(pin_g) && j == g) || (pin_i(pin_g) && j == pi))) return false;
  double sgi[3], s[3];
  for (int c = 0; c < 3; ++c) {
    sgi[c] = reflect1(X[c * T + j], sc.mirror[m][c], sc.box[c]);
    s[c] = reflect1(GI[c * T + j], sc.mirror[m][c], sc.box[c]);
  }
  const double a = e_add(e_add(e_sq(e_sub(xi[0], s[0])), e_sq(e_sub(xi[1], s[1]))), e_sq(e_sub(xi[2], s[2])));
  const double r[3] = {e_sub(s[0], xi[0]), e_sub(s[1], xi[1]), e_sub(s[2], xi[2])};
  const double d[3] = {e_sub(sgi[0], s[0]), e_sub(sgi[1], s[1]), e_sub(sgi[2], s[2])};
  const double c = e_add(e_add(e_sq(e_sub(s[0], sgi[0])), e_sq(e_sub(s[1], sgi[1]))), e_sq(e_sub(s[2], sgi[2])));
  return bs_term_exact(r, d, a, c, sc.quant_circ, sc.two_pi, out);
}
