// topo.cu -- topology stages: pinsert, pclose (brute), precon, premove, loop_killer.
//
// The reference runs pinsert, precon and premove as serial sweeps in ascending slot order
// (src/line.f90:30, src/reconnection.f90:180, src/line.f90:107), where an event can change
// what later slots see.  Here each stage is
//   1. a parallel pass over all slots that marks the slots whose test can pass on the
//      current state (or, for pinsert, whose stale-ghost test passes);
//   2. a stable compaction of the marks into an ascending list per system (prefix sum);
//   3. one thread per system that walks the marked slots in ascending order (a two-level
//      bitmap; slots an earlier event in the same sweep has touched are marked on the way,
//      since their test must be re-evaluated) and applies the reference's exact tests and
//      updates.  pinsert has a parallel form for the common case (see below).
// A slot that is neither marked nor touched has a test that is false in the serial sweep
// too, so the events are the reference's, event for event and in the same order.
#include <cub/cub.cuh>

#include "handle.cuh"

struct TopoBuffers {
  int *flag_a = nullptr, *pos_a = nullptr, *list_a = nullptr;
  int *flag_b = nullptr, *pos_b = nullptr, *list_b = nullptr;
  int *flag_c = nullptr, *pos_c = nullptr, *list_c = nullptr;
  int *dec = nullptr;       // per slot: bit0 stale test, bit1 fresh test, bit2 inserts, bit3 case A
  int *newslot = nullptr;   // per slot: the slot its insertion fills
  double *xnew = nullptr;   // per slot: new point position [3][T]
  unsigned *l0 = nullptr, *l1 = nullptr;  // sweep bitmaps
  unsigned *touched = nullptr;             // per-system touched-slot bitmaps too big for smem
  long long touched_words = 0;             // words per system
  int smem_words = 0;                      // bitmap words the sweep keeps in shared memory
  void *cub_tmp = nullptr;
  size_t cub_bytes = 0;
};

namespace {

constexpr int TB = 256;

// Two-level bitmap of the slots a serial sweep must still visit: bit g of l0 marks slot g,
// bit w of l1 marks l0 word w as possibly non-empty.  The sweep takes the lowest marked
// slot above the last one visited; events mark slots further ahead (there is no capacity
// limit, unlike a fixed-size queue).
struct Sweep {
  unsigned *l0, *l1;
  long long T;
  __device__ void mark(int g) const {
    atomicOr(&l0[g >> 5], 1u << (g & 31));
    atomicOr(&l1[g >> 10], 1u << ((g >> 5) & 31));
  }
  __device__ void unmark(int g) const { atomicAnd(&l0[g >> 5], ~(1u << (g & 31))); }
  // lowest marked slot >= from and <= last, or INT_MAX
  __device__ int next(int from, int last) const {
    if (from > last) return INT_MAX;
    int w = from >> 5;
    unsigned bits = l0[w] & (~0u << (from & 31));
    for (;;) {
      if (bits) {
        const int g = (w << 5) + __ffs(bits) - 1;
        return g <= last ? g : INT_MAX;
      }
      // next non-empty l0 word after w, located through l1
      int w1 = (w + 1) >> 5;
      unsigned b1 = ((w + 1) & 31) ? (l1[w1] & (~0u << ((w + 1) & 31))) : l1[w1];
      const int wlast = last >> 5;
      for (;;) {
        if (b1) break;
        ++w1;
        if ((w1 << 5) > wlast) return INT_MAX;
        b1 = l1[w1];
      }
      w = (w1 << 5) + __ffs(b1) - 1;
      if (w > wlast) return INT_MAX;
      bits = l0[w];
      if (!bits) {  // stale summary bit: clear it and keep looking
        atomicAnd(&l1[w >> 5], ~(1u << (w & 31)));
      }
    }
  }
};

// l0/l1 from a 0/1 flag per slot (one thread per l0 word, then one per l1 word).
__global__ void k_bits_l0(const int *__restrict__ flag, unsigned *l0, long long T) {
  const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (w * 32 >= T + 32) return;
  unsigned b = 0;
  for (int k = 0; k < 32; ++k) {
    const long long g = w * 32 + k;
    if (g < T && flag[g]) b |= 1u << k;
  }
  l0[w] = b;
}
__global__ void k_bits_l1(const unsigned *__restrict__ l0, unsigned *l1, long long nw0) {
  const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (w * 32 >= nw0 + 32) return;
  unsigned b = 0;
  for (int k = 0; k < 32; ++k) {
    const long long q = w * 32 + k;
    if (q < nw0 && l0[q]) b |= 1u << k;
  }
  l1[w] = b;
}

__device__ __forceinline__ bool recon_step(const SysConst &sc, const SysDyn &d) {
  return (d.itime % sc.recon_shots) == 0;
}

__device__ void log_event(SysDyn &d, int s, int kind, int i, int j, DevEvent *ev, int *ev_count, int ev_cap) {
  const int seq = d.event_seq++;
  const int slot = atomicAdd(ev_count, 1);
  if (slot < ev_cap) ev[slot] = DevEvent{s, seq, d.itime, kind, i, j};
}

struct State {
  double *X, *U, *U1, *U2, *GI, *GB, *CD;
  int *nxt, *prv, *cl;
  long long T;
};

__device__ void clear_particle(const State &S, int g) {  // general.f90:10-20
  const long long T = S.T;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    S.X[c * T + g] = 0; S.U[c * T + g] = 0; S.U1[c * T + g] = 0; S.U2[c * T + g] = 0;
    S.GI[c * T + g] = 0; S.GB[c * T + g] = 0;
  }
  S.nxt[g] = 0; S.prv[g] = 0; S.cl[g] = 0; S.CD[g] = 0;
}

// loop_killer (reconnection.f90:155-182).  Only "fewer than 4 points" matters, so the
// count stops after three hops; the result equals the reference's full walk.
__device__ void loop_killer(const State &S, SysDyn &d, int s, int particle, int pcount, DevEvent *ev,
                            int *ev_count, int ev_cap) {
  int counter = 1, nx = particle;
  const int hops = pcount < 3 ? pcount : 3;
  for (int it = 0; it < hops; ++it) {
    nx = S.nxt[nx];
    if (nx == particle) break;
    counter++;
  }
  if (counter < 4) {
    log_event(d, s, NV_EV_LOOPKILL, particle, counter, ev, ev_count, ev_cap);
    d.loop_kills++;
    nx = particle;
    for (int it = 0; it < pcount; ++it) {
      const int sn = S.nxt[nx];
      clear_particle(S, nx);
      nx = sn;
      if (nx == particle) break;
    }
  }
}

__device__ __forceinline__ void get_ghost_p(const SysConst &sc, const State &S, int g, double gi[3], double gb[3]) {
  double x[3];
  load3(S.X, S.T, g, x);
  load3(S.X, S.T, S.nxt[g], gi);
  load3(S.X, S.T, S.prv[g], gb);
  ghost_adjust(sc, x, gi);
  ghost_adjust(sc, x, gb);
}
__device__ __forceinline__ void refresh_ghosts(const SysConst &sc, const State &S, int g) {
  double gi[3], gb[3];
  get_ghost_p(sc, S, g, gi, gb);
  store3(S.GI, S.T, g, gi);
  store3(S.GB, S.T, g, gb);
}

// ---- pass 1 kernels: marks ----------------------------------------------------------------
// precon marks: live slot with delta/2 > closestd > epsilon(1.) (reconnection.f90:185).
__global__ void k_mark_recon(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn, const int *__restrict__ sys_of,
                             const double *__restrict__ CD, const int *__restrict__ nxt, int *fa, long long T,
                             const unsigned *err) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g > T) return;
  int a = 0;
  if (g < T && !*err) {
    const int s = sys_of[g];
    const SysConst &sc = scs[s];
    const int k = (int)(g - sc.base);
    if (k >= 1 && k <= dyn[s].pcount && recon_step(sc, dyn[s]) && nxt[g] != 0) {
      const double cd = CD[g];
      a = (cd < sc.delta / 2.) && (cd > NV_EPS);
    }
  }
  fa[g] = a;
}

// premove marks: live slot with |x_i - x_{i+2}| < .99 delta (line.f90:113-115).
__global__ void k_mark_remove(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn, const int *__restrict__ sys_of,
                              const double *__restrict__ X, const int *__restrict__ nxt, int *fa, long long T,
                              const unsigned *err) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g > T) return;
  int a = 0;
  if (g < T && !*err) {
    const int s = sys_of[g];
    const SysConst &sc = scs[s];
    const int k = (int)(g - sc.base);
    if (k >= 1 && k <= dyn[s].pcount && recon_step(sc, dyn[s]) && nxt[g] != 0) {
      double x[3], y[3];
      load3(X, T, (int)g, x);
      load3(X, T, nxt[nxt[g]], y);
      a = dist_gen(x, y) < e_mul(.99, sc.delta);
    }
  }
  fa[g] = a;
}

__global__ void k_scatter(const int *__restrict__ flag, const int *__restrict__ pos, int *__restrict__ list, long long T) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < T && flag[g]) list[pos[g]] = (int)g;
}

__global__ void k_zero_live(SysDyn *dyn, int nsys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nsys) dyn[s].live = 0;
}

// ---- pass 3: serial resolvers, one thread per system ---------------------------------------

// pinsert (line.f90:18-96).
__global__ void k_insert_resolve(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, State S, Sweep sw,
                                 const int *__restrict__ pos_b, const int *__restrict__ list_b, unsigned *err,
                                 DevEvent *ev, int *ev_count, int ev_cap, int only_fallback) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || *err) return;
  if (only_fallback && !dyn[s].ins_fallback) return;
  const SysConst &sc = scs[s];
  SysDyn d = dyn[s];
  if (d.live == 0) {
    atomicOr(err, DERR_EMPTY);
    return;
  }
  const int base = sc.base;
  const int old_last = base + d.pcount;  // loop bound old_pcount (line.f90:28-30)
  int pc = d.pcount;
  int ei = pos_b[base], ee = pos_b[base + sc.cap + 1];
  int last = base;
  const long long T = S.T;
  for (;;) {
    const int i = sw.next(last + 1, old_last);
    if (i == INT_MAX) break;
    last = i;
    sw.unmark(i);
    if (S.nxt[i] == 0) continue;
    double x[3], gi[3], gb[3];
    load3(S.X, T, i, x);
    load3(S.GI, T, i, gi);
    load3(S.GB, T, i, gb);
    const double disti = dist_gen(x, gi);
    if (!(disti > sc.delta)) continue;
    int par_new;
    if (ei < ee) {
      par_new = list_b[ei++];
    } else {
      if (pc + 1 > sc.cap) {
        atomicOr(err, DERR_CAPACITY);
        break;
      }
      par_new = base + (++pc);
    }
    double fdd[3], xn[3];
    deriv2(x, gi, gb, fdd);
    double curv = e_sqrt(dot3(fdd, fdd));
    double mid[3] = {e_mul(0.5, e_add(x[0], gi[0])), e_mul(0.5, e_add(x[1], gi[1])), e_mul(0.5, e_add(x[2], gi[2]))};
    if (curv > 1E-5) {
      curv = e_div(1.0, curv);
      const double disc = e_sub(e_mul(curv, curv), e_mul(0.25, e_mul(disti, disti)));
      if (disc > 0.) {
        const double sfac = e_mul(e_sub(e_sqrt(disc), curv), curv);
        for (int c = 0; c < 3; ++c) xn[c] = e_add(mid[c], e_mul(sfac, fdd[c]));
      } else {
        for (int c = 0; c < 3; ++c) xn[c] = mid[c];
      }
    } else {
      for (int c = 0; c < 3; ++c) xn[c] = mid[c];
    }
    const int nx = S.nxt[i];
    double ui[3], un[3], zero[3] = {0, 0, 0};
    load3(S.U, T, i, ui);
    load3(S.U, T, nx, un);
    for (int c = 0; c < 3; ++c) un[c] = e_mul(0.5, e_add(ui[c], un[c]));
    store3(S.X, T, par_new, xn);
    store3(S.U, T, par_new, un);
    store3(S.U1, T, par_new, zero);
    store3(S.U2, T, par_new, zero);
    S.prv[par_new] = i;
    S.nxt[par_new] = nx;
    refresh_ghosts(sc, S, par_new);
    S.prv[nx] = par_new;
    refresh_ghosts(sc, S, nx);
    S.nxt[i] = par_new;
    refresh_ghosts(sc, S, i);
    log_event(d, s, NV_EV_INSERT, i, par_new, ev, ev_count, ev_cap);
    d.insert_count++;
    // slots whose test changed and that the sweep has not reached yet
    if (nx > i && nx <= old_last) sw.mark(nx);
    if (par_new > i && par_new <= old_last) sw.mark(par_new);
  }
  d.pcount = pc;
  dyn[s] = d;
}

// precon (reconnection.f90:11-61).
__device__ void norm_tanf(const State &S, int g, double t[3]) {  // general.f90:106-117
  double x[3], gi[3], gb[3];
  load3(S.X, S.T, g, x);
  load3(S.GI, S.T, g, gi);
  load3(S.GB, S.T, g, gb);
  deriv1(x, gi, gb, t);
  const double len = e_sqrt(e_add(e_add(e_sq(t[0]), e_sq(t[1])), e_sq(t[2])));
  for (int c = 0; c < 3; ++c) t[c] = e_div(t[c], len);
}

__global__ void k_recon_resolve(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, State S,
                                const int *__restrict__ pos_a, const int *__restrict__ list_a, unsigned *err,
                                DevEvent *ev, int *ev_count, int ev_cap) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  SysDyn d = dyn[s];
  if (!recon_step(sc, d)) return;
  const int base = sc.base;
  const int li = pos_a[base], le = pos_a[base + sc.cap + 1];
  d.diag[3] = le - li;
  const long long T = S.T;
  for (int idx = li; idx < le; ++idx) {
    const int i = list_a[idx];
    if (S.nxt[i] == 0) continue;
    const int pari = S.nxt[i], parb = S.prv[i];
    const int j = S.cl[i];
    if (j == pari || j == parb || j == 0) continue;
    if (S.nxt[j] == 0) continue;
    const int parjb = S.prv[j];
    double t1[3], t2[3];
    norm_tanf(S, i, t1);
    norm_tanf(S, j, t2);
    const double dot_val = dot3(t1, t2);
    if (dot_val > 0.9) continue;
    double xi[3], gii[3], gbi[3], xj[3], gij[3], gbj[3], xpi[3], xpj[3];
    load3(S.X, T, i, xi);
    load3(S.GI, T, i, gii);
    load3(S.GB, T, i, gbi);
    load3(S.X, T, j, xj);
    load3(S.GI, T, j, gij);
    load3(S.GB, T, j, gbj);
    load3(S.X, T, pari, xpi);
    load3(S.X, T, parjb, xpj);
    const double l_before = e_add(e_add(e_add(dist_gen(xi, gii), dist_gen(xi, gbi)), dist_gen(xj, gij)), dist_gen(xj, gbj));
    const double l_after = e_add(e_add(e_add(dist_gen(xi, gbi), dist_gen(xi, xj)), dist_gen(xj, gij)), dist_gen(xpi, xpj));
    if (l_after <= l_before) {
      d.recon_count++;
      log_event(d, s, NV_EV_RECON, i, j, ev, ev_count, ev_cap);
      S.nxt[parjb] = pari;
      S.prv[pari] = parjb;
      S.nxt[i] = j;
      S.prv[j] = i;
      loop_killer(S, d, s, pari, d.pcount, ev, ev_count, ev_cap);
      loop_killer(S, d, s, i, d.pcount, ev, ev_count, ev_cap);
    }
  }
  dyn[s] = d;
}

// pclose (line.f90:135-160): exact nearest non-neighbour, non-periodic distance, strict <
// so ties keep the lowest j.  One thread per target slot.
__global__ void k_pclose_brute(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                               const int *__restrict__ sys_of, const double *__restrict__ X,
                               const int *__restrict__ nxt, const int *__restrict__ prv, int *__restrict__ cl,
                               double *__restrict__ CD, long long T, const unsigned *err) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T || *err) return;
  const int s = sys_of[g];
  const SysConst &sc = scs[s];
  if (sc.use_tree || !recon_step(sc, dyn[s])) return;
  const int pc = dyn[s].pcount;
  const int k = (int)(g - sc.base);
  if (k < 1 || k > pc || nxt[g] == 0) return;
  const int ni = nxt[g], pi = prv[g];
  double xi[3];
  load3(X, T, (int)g, xi);
  double best = 100.;
  double best2 = 1e300;
  int bj = cl[g];
  for (int j = sc.base + 1; j <= sc.base + pc; ++j) {
    if (nxt[j] == 0 || j == g || j == ni || j == pi) continue;
    double xj[3];
    load3(X, T, j, xj);
    const double d2 = e_add(e_add(e_sq(e_sub(xi[0], xj[0])), e_sq(e_sub(xi[1], xj[1]))), e_sq(e_sub(xi[2], xj[2])));
    if (d2 > best2) continue;  // sqrt is monotone: cannot be strictly closer
    const double dist = e_sqrt(d2);
    if (dist < best) {
      best = dist;
      best2 = d2;
      bj = j;
    }
  }
  cl[g] = bj;
  CD[g] = best;
}


// ---- parallel pinsert ---------------------------------------------------------------------
// In the serial sweep (line.f90:30-93) slot k is tested against its step-start ghost unless
// its predecessor p = behind(k) < k inserted earlier in the same sweep: that insertion
// refreshed k's ghosts from the current positions (line.f90:88-89).  So each live slot has
// two candidate outcomes, a stale test and a fresh test; when they agree the outcome is
// known, and only slots where they differ depend on their predecessor's outcome.
// New points that the sweep reaches later (placed in a free slot above their creator) are
// tested again by the reference; when any such point would insert, the step falls back to
// the serial resolver.

// bit0 stale test, bit1 fresh test (ghost of the current infront position); list = either.
__global__ void k_ins_mark(const SysConst *__restrict__ scs, SysDyn *__restrict__ dyn, const int *__restrict__ sys_of,
                           const double *__restrict__ X, const double *__restrict__ GI, const int *__restrict__ nxt,
                           int *fa, int *fb, int *dec, long long T, const unsigned *err) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g > T) return;
  int a = 0, b = 0, dv = 0;
  if (g < T && !*err) {
    const int s = sys_of[g];
    const SysConst &sc = scs[s];
    const int k = (int)(g - sc.base);
    if (k >= 1 && k <= dyn[s].pcount) {
      if (nxt[g] == 0) {
        b = 1;
      } else {
        double x[3], gi[3], gf[3];
        load3(X, T, (int)g, x);
        load3(GI, T, (int)g, gi);
        load3(X, T, nxt[g], gf);
        ghost_adjust(sc, x, gf);
        const int st = dist_gen(x, gi) > sc.delta, fr = dist_gen(x, gf) > sc.delta;
        dv = st | (fr << 1);
        a = st | fr;
        dyn[s].live = 1;
      }
    }
  }
  fa[g] = a;
  fb[g] = b;
  if (g < T) dec[g] = dv;
}

// Outcomes: known where the two tests agree (decided here, in parallel); where they differ
// the outcome is the fresh test if the predecessor p = behind(k) < k inserts, else the stale
// one -- those "ambiguous" slots are marked for an ordered pass.
__global__ void k_ins_decide_easy(const int *__restrict__ list_a, const int *__restrict__ n_ptr, int *dec, int *famb,
                                  const unsigned *err) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= *n_ptr || *err) return;
  const int k = list_a[e];
  const int dv = dec[k];
  const int st = dv & 1, fr = (dv >> 1) & 1;
  if (st == fr) dec[k] = dv | (st << 2);
  else famb[k] = 1;
}

// Ambiguous slots in ascending order, one thread per system (their predecessors' outcomes
// are final: decided in parallel, or earlier in this pass).
__global__ void k_ins_decide_amb(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, const int *__restrict__ prv,
                                 const int *__restrict__ pos_m, const int *__restrict__ list_m,
                                 const int *__restrict__ pos_a, int *dec, const unsigned *err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  dyn[s].ins_fallback = 0;
  dyn[s].diag[0] = pos_a[sc.base + sc.cap + 1] - pos_a[sc.base];
  const int mi = pos_m[sc.base], me = pos_m[sc.base + sc.cap + 1];
  for (int idx = mi; idx < me; ++idx) {
    const int k = list_m[idx];
    const int dv = dec[k];
    const int p = prv[k];
    const bool caseA = p < k && (dec[p] & 4);
    const int d = caseA ? (dv >> 1) & 1 : dv & 1;
    dec[k] = dv | (d << 2);
  }
}

// Case A (ghosts refreshed by the predecessor's insertion) and the insertion flags.
__global__ void k_ins_decide_case(const int *__restrict__ list_a, const int *__restrict__ n_ptr,
                                  const int *__restrict__ prv, int *dec, int *fc, const unsigned *err) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= *n_ptr || *err) return;
  const int k = list_a[e];
  const int dv = dec[k];
  const int p = prv[k];
  const bool caseA = p < k && (dec[p] & 4);
  if (caseA) dec[k] = dv | 8;
  fc[k] = (dv >> 2) & 1;
}

__global__ void k_zero_flags(int *f, long long n) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g <= n) f[g] = 0;
}

// New points along chains of consecutive insertions: a chain starts at an inserting slot
// whose ghosts were not refreshed (case B) and continues to infront(k) while that slot
// inserts in case A (its ghosts then hold the current infront position and the new point
// just placed behind it).  One thread per chain head.
__global__ void k_ins_points(const SysConst *__restrict__ scs, SysDyn *dyn, const int *__restrict__ sys_of, State S,
                             const int *__restrict__ pos_c, const int *__restrict__ list_c, const int *__restrict__ pos_b,
                             const int *__restrict__ list_b, const int *__restrict__ dec, int *newslot, double *xnew,
                             const int *__restrict__ nev_total, unsigned *err) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= *nev_total || *err) return;
  int k = list_c[e];
  if (dec[k] & 8) return;  // not a chain head
  const int s = sys_of[k];
  const SysConst &sc = scs[s];
  const int base = sc.base;
  const int ev0 = pos_c[base], fb0 = pos_b[base], nfree = pos_b[base + sc.cap + 1] - fb0;
  const int pc = dyn[s].pcount;
  const long long T = S.T;
  const int old_last = base + pc;
  double gbk[3];
  bool fresh = false;
  for (;;) {
    const int rank = pos_c[k] - ev0;
    const int slot = rank < nfree ? list_b[fb0 + rank] : base + pc + 1 + (rank - nfree);
    if (slot > base + sc.cap) {
      atomicOr(err, DERR_CAPACITY);
      return;
    }
    newslot[k] = slot;
    double x[3], gi[3], gb[3];
    load3(S.X, T, k, x);
    const int nx = S.nxt[k];
    if (fresh) {  // ghosts refreshed by the predecessor's insertion (get_ghost_p, line.f90:89)
      load3(S.X, T, nx, gi);
      ghost_adjust(sc, x, gi);
      for (int c = 0; c < 3; ++c) gb[c] = gbk[c];
      ghost_adjust(sc, x, gb);
    } else {
      load3(S.GI, T, k, gi);
      load3(S.GB, T, k, gb);
    }
    const double disti = dist_gen(x, gi);
    double fdd[3], xn[3];
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
    for (int c = 0; c < 3; ++c) xnew[c * T + k] = xn[c];
    // a new point the sweep reaches later is tested again (its ghost: infront of k)
    if (slot > k && slot <= old_last) {
      double gn[3];
      load3(S.X, T, nx, gn);
      ghost_adjust(sc, xn, gn);
      const double dn = dist_gen(xn, gn);
      if (dn > sc.delta) {
        if (atomicExch(&dyn[s].ins_fallback, 1) == 0) {
          dyn[s].diag[5] = k - base;
          dyn[s].diag[6] = slot - base;
          dyn[s].diag[7] = __double_as_longlong(dn);
        }
      }
    }
    // continue the chain: infront(k) inserts with ghosts refreshed by this insertion
    if (nx > k && (dec[nx] & 8)) {
      for (int c = 0; c < 3; ++c) gbk[c] = xn[c];
      fresh = true;
      k = nx;
      continue;
    }
    break;
  }
}

// Apply every insertion (links, new point state) and log the events in sweep order.
__global__ void k_ins_apply(const SysConst *__restrict__ scs, SysDyn *dyn, const int *__restrict__ sys_of, State S,
                            const int *__restrict__ pos_c, const int *__restrict__ list_c, const int *__restrict__ newslot,
                            const double *__restrict__ xnew, const int *__restrict__ nev_total, DevEvent *ev,
                            int *ev_count, int ev_cap, const unsigned *err) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= *nev_total || *err) return;
  const int k = list_c[e];
  const int s = sys_of[k];
  if (dyn[s].ins_fallback) return;
  const SysConst &sc = scs[s];
  const long long T = S.T;
  const int slot = newslot[k];
  const int nx = S.nxt[k];
  double ui[3], un[3], xn[3], zero[3] = {0, 0, 0};
  load3(S.U, T, k, ui);
  load3(S.U, T, nx, un);
  for (int c = 0; c < 3; ++c) {
    un[c] = e_mul(0.5, e_add(ui[c], un[c]));
    xn[c] = xnew[c * T + k];
  }
  store3(S.X, T, slot, xn);
  store3(S.U, T, slot, un);
  store3(S.U1, T, slot, zero);
  store3(S.U2, T, slot, zero);
  S.cl[slot] = 0;
  S.CD[slot] = 0;
  S.prv[slot] = k;
  S.nxt[slot] = nx;
  S.prv[nx] = slot;
  S.nxt[k] = slot;
  const int rank = pos_c[k] - pos_c[sc.base];
  const int seq = dyn[s].event_seq + rank;
  const int at = atomicAdd(ev_count, 1);
  if (at < ev_cap) ev[at] = DevEvent{s, seq, dyn[s].itime, NV_EV_INSERT, k, slot};
}

// Ghosts of every slot an insertion touched, from the final links and positions (each
// touched slot's last refresh in the serial sweep sees exactly this state).
__global__ void k_ins_ghosts(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                             const int *__restrict__ sys_of, State S, const int *__restrict__ list_c,
                             const int *__restrict__ newslot, const int *__restrict__ nev_total, const unsigned *err) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= *nev_total || *err) return;
  const int k = list_c[e];
  const int s = sys_of[k];
  if (dyn[s].ins_fallback) return;
  const SysConst &sc = scs[s];
  const int slot = newslot[k];
  refresh_ghosts(sc, S, k);
  refresh_ghosts(sc, S, slot);
  refresh_ghosts(sc, S, S.nxt[slot]);
}

// Counters: pcount grows by the insertions beyond the free slots.
__global__ void k_ins_finish(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, const int *__restrict__ pos_c,
                             const int *__restrict__ pos_b, unsigned *err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  SysDyn &d = dyn[s];
  if (d.live == 0) {
    atomicOr(err, DERR_EMPTY);
    return;
  }
  const int nev = pos_c[sc.base + sc.cap + 1] - pos_c[sc.base];
  d.diag[1] = nev;
  if (d.ins_fallback) {
    d.diag[2] += 1;
    return;
  }
  const int nfree = pos_b[sc.base + sc.cap + 1] - pos_b[sc.base];
  d.event_seq += nev;
  d.insert_count += nev;
  if (nev > nfree) d.pcount += nev - nfree;
}


// ---- precon sweep, warp-prefetched --------------------------------------------------------
// The reference's sweep (reconnection.f90:180-221) is kept exactly: candidates in ascending
// order, each decided on the state left by the events before it.  A warp loads 32
// candidates at a time and decides each on the current state in parallel; lane 0 then walks
// them in order.  A candidate's decision reads the links of i and of its partner j only
// (nxt/prv of both; x and ghosts do not change in precon, and a cleared neighbour means a
// cleared i or j), so the parallel decision stands unless an event earlier in the sweep
// wrote the links of i or j -- tracked in a per-system bitmap of touched slots (shared
// memory when it fits).  Touched candidates are decided again by lane 0 on the live state.

struct ReconIn {
  int i, pari, parb, j, nj, parjb;
  int yes;  // 1: reconnect, 0: no, -1: skip (reconnection.f90:181-190)
  double dot_val, l_before, l_after;
};

__device__ ReconIn recon_decide(const State &S, int i, double half_delta, int cl_i) {
  ReconIn r;
  r.i = i;
  r.pari = S.nxt[i];
  r.parb = S.prv[i];
  r.j = cl_i;
  r.nj = 0;
  r.parjb = 0;
  r.yes = -1;
  r.dot_val = r.l_before = r.l_after = 0;
  if (r.pari == 0) return r;
  const int j = r.j;
  if (j == r.pari || j == r.parb || j == 0) return r;
  r.nj = S.nxt[j];
  if (r.nj == 0) return r;
  r.parjb = S.prv[j];
  double t1[3], t2[3];
  norm_tanf(S, i, t1);
  norm_tanf(S, j, t2);
  r.dot_val = dot3(t1, t2);
  if (r.dot_val > 0.9) {
    r.yes = 0;
    return r;
  }
  const long long T = S.T;
  double xi[3], gii[3], gbi[3], xj[3], gij[3], gbj[3], xpi[3], xpj[3];
  load3(S.X, T, i, xi);
  load3(S.GI, T, i, gii);
  load3(S.GB, T, i, gbi);
  load3(S.X, T, j, xj);
  load3(S.GI, T, j, gij);
  load3(S.GB, T, j, gbj);
  load3(S.X, T, r.pari, xpi);
  load3(S.X, T, r.parjb, xpj);
  r.l_before = e_add(e_add(e_add(dist_gen(xi, gii), dist_gen(xi, gbi)), dist_gen(xj, gij)), dist_gen(xj, gbj));
  r.l_after = e_add(e_add(e_add(dist_gen(xi, gbi), dist_gen(xi, xj)), dist_gen(xj, gij)), dist_gen(xpi, xpj));
  r.yes = r.l_after <= r.l_before ? 1 : 0;
  (void)half_delta;
  return r;
}

__device__ __forceinline__ bool bit_get(const unsigned *b, int k) { return (b[k >> 5] >> (k & 31)) & 1u; }
__device__ __forceinline__ void bit_set(unsigned *b, int k) { b[k >> 5] |= 1u << (k & 31); }

// Slots whose links an event of the current chunk wrote: bit set in `bits` and recorded
// in `list` so that the bits can be cleared when the chunk ends (the next chunk's parallel
// decisions are taken on the state that already includes them).
struct Touched {
  unsigned *bits;
  int *list;
  int n;
  int base;
  __device__ void add(int g) {
    if (g <= base) return;
    const int k = g - base;
    if (!bit_get(bits, k)) {
      bit_set(bits, k);
      list[n++] = k;
    }
  }
  __device__ bool has(int g) const { return g > base && bit_get(bits, g - base); }
};
constexpr int kTouchedPerChunk = 32 * 10;  // 4 relinked + up to 6 cleared slots per event

// Events of one chunk, staged in shared memory by lane 0 and written with one atomic.
struct EventStage {
  DevEvent *buf;
  int n;
  __device__ void add(SysDyn &d, int s, int kind, int i, int j) {
    buf[n++] = DevEvent{s, d.event_seq++, d.itime, kind, i, j};
  }
};
__device__ void flush_events(EventStage &es, int lane, DevEvent *ev, int *ev_count, int ev_cap) {
  int n = __shfl_sync(0xffffffffu, es.n, 0);
  if (n == 0) return;
  int at = 0;
  if (lane == 0) at = atomicAdd(ev_count, n);
  at = __shfl_sync(0xffffffffu, at, 0);
  for (int q = lane; q < n; q += 32)
    if (at + q < ev_cap) ev[at + q] = es.buf[q];
  __syncwarp();
  if (lane == 0) es.n = 0;
  __syncwarp();
}

__device__ void loop_killer_stage(const State &S, SysDyn &d, int s, int particle, int pcount, EventStage &es,
                                  Touched &tc) {
  int counter = 1, nx = particle;
  const int hops = pcount < 3 ? pcount : 3;
  for (int it = 0; it < hops; ++it) {
    nx = S.nxt[nx];
    if (nx == particle) break;
    counter++;
  }
  if (counter < 4) {
    es.add(d, s, NV_EV_LOOPKILL, particle, counter);
    d.loop_kills++;
    nx = particle;
    for (int it = 0; it < pcount; ++it) {
      const int sn = S.nxt[nx];
      tc.add(nx);
      clear_particle(S, nx);
      nx = sn;
      if (nx == particle) break;
    }
  }
}

__global__ void __launch_bounds__(32) k_recon_sweep(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, State S,
                                                    const int *__restrict__ pos_a, const int *__restrict__ list_a,
                                                    unsigned *gbits, long long gbits_words_per_sys, int smem_words,
                                                    unsigned *err, DevEvent *ev, int *ev_count, int ev_cap) {
  extern __shared__ unsigned sbits[];
  __shared__ int tlist[kTouchedPerChunk];
  __shared__ DevEvent ebuf[96];
  const int s = blockIdx.x;
  const int lane = threadIdx.x;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  if (!recon_step(sc, dyn[s])) return;
  const int base = sc.base;
  const int nwords = (sc.cap + 1 + 31) / 32;
  unsigned *bits = nwords <= smem_words ? sbits : gbits + (long long)s * gbits_words_per_sys;
  for (int w = lane; w < nwords; w += 32) bits[w] = 0;
  Touched tc{bits, tlist, 0, base};
  EventStage es{ebuf, 0};
  const int li = pos_a[base], le = pos_a[base + sc.cap + 1];
  SysDyn d = dyn[s];  // lane 0's copy is the live one
  if (lane == 0) d.diag[3] = le - li;
  __syncwarp();
  const double half_delta = sc.delta / 2.;
  for (int k0 = li; k0 < le; k0 += 32) {
    const int k = k0 + lane;
    ReconIn in;
    in.yes = -1;
    in.i = 0;
    if (k < le) {
      const int i = list_a[k];
      in = recon_decide(S, i, half_delta, S.cl[i]);
    }
    __syncwarp();
    const int n = min(32, le - k0);
    for (int l = 0; l < n; ++l) {
      int i = __shfl_sync(0xffffffffu, in.i, l);
      int yes = __shfl_sync(0xffffffffu, in.yes, l);
      int pari = __shfl_sync(0xffffffffu, in.pari, l);
      int j = __shfl_sync(0xffffffffu, in.j, l);
      int parjb = __shfl_sync(0xffffffffu, in.parjb, l);
      if (lane == 0) {
        if (tc.has(i) || tc.has(j)) {
          // an earlier event wrote the links of i or j: decide again on the live state
          if (S.nxt[i] == 0) {
            yes = -1;
          } else {
            const ReconIn r = recon_decide(S, i, half_delta, S.cl[i]);
            yes = r.yes;
            pari = r.pari;
            parjb = r.parjb;
          }
        }
        if (yes == 1) {
          d.recon_count++;
          es.add(d, s, NV_EV_RECON, i, j);
          S.nxt[parjb] = pari;
          S.prv[pari] = parjb;
          S.nxt[i] = j;
          S.prv[j] = i;
          tc.add(i);
          tc.add(j);
          tc.add(pari);
          tc.add(parjb);
          loop_killer_stage(S, d, s, pari, d.pcount, es, tc);
          loop_killer_stage(S, d, s, i, d.pcount, es, tc);
        }
      }
    }
    // the chunk's writes are now visible to the next chunk's parallel decisions
    __threadfence_block();
    const int nt = __shfl_sync(0xffffffffu, tc.n, 0);
    __syncwarp();
    for (int q = lane; q < nt; q += 32) {
      const int kk = tlist[q];
      atomicAnd(&bits[kk >> 5], ~(1u << (kk & 31)));
    }
    if (lane == 0) tc.n = 0;
    flush_events(es, lane, ev, ev_count, ev_cap);
  }
  if (lane == 0) dyn[s] = d;
}


// ---- premove sweep, warp-prefetched --------------------------------------------------------
// line.f90:107-129 in ascending slot order.  A candidate's test reads infront(i),
// infront(infront(i)) and their positions; it is re-evaluated on the live state when an
// event of the current chunk touched i or infront(i).  A removal at i changes the test of
// p = behind(i); when p > i and p is not a candidate it is visited later as an extra slot
// (the two-level bitmap).
__global__ void __launch_bounds__(32) k_remove_sweep(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, State S,
                                                     const int *__restrict__ pos_a, const int *__restrict__ list_a,
                                                     const int *__restrict__ cand, Sweep sw, unsigned *gbits,
                                                     long long gbits_words_per_sys, int smem_words, unsigned *err,
                                                     DevEvent *ev, int *ev_count, int ev_cap) {
  extern __shared__ unsigned sbits[];
  __shared__ int tlist[kTouchedPerChunk];
  __shared__ DevEvent ebuf[96];
  const int s = blockIdx.x;
  const int lane = threadIdx.x;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  if (!recon_step(sc, dyn[s])) return;
  const int base = sc.base;
  const int nwords = (sc.cap + 1 + 31) / 32;
  unsigned *bits = nwords <= smem_words ? sbits : gbits + (long long)s * gbits_words_per_sys;
  for (int w = lane; w < nwords; w += 32) bits[w] = 0;
  Touched tc{bits, tlist, 0, base};
  EventStage es{ebuf, 0};
  const int li = pos_a[base], le = pos_a[base + sc.cap + 1];
  SysDyn d = dyn[s];
  const int lastslot = base + d.pcount;
  const double thr = e_mul(.99, sc.delta);
  const long long T = S.T;
  int extras = 0, last = base;  // lane 0: pending extra visits, last slot visited
  if (lane == 0) d.diag[4] = le - li;
  __syncwarp();
  // one visit of slot i on the live state (lane 0)
  auto visit = [&](int i) {
    if (S.nxt[i] == 0) return;
    const int infront = S.nxt[i];
    const int tinfront = S.nxt[infront];
    double xi[3], xt[3];
    load3(S.X, T, i, xi);
    load3(S.X, T, tinfront, xt);
    if (!(dist_gen(xi, xt) < thr)) return;
    S.prv[tinfront] = i;
    S.nxt[i] = tinfront;
    tc.add(i);
    tc.add(infront);
    tc.add(tinfront);
    clear_particle(S, infront);
    es.add(d, s, NV_EV_REMOVE, i, infront);
    loop_killer_stage(S, d, s, i, d.pcount, es, tc);
    d.remove_count++;
    const int p = S.prv[i];
    if (p > i && p <= lastslot && !cand[p]) {
      sw.mark(p);
      ++extras;
    }
  };
  auto run_extras = [&](int upto) {  // extra slots in (last, upto]
    while (extras > 0) {
      const int e = sw.next(last + 1, upto);
      if (e == INT_MAX) break;
      sw.unmark(e);
      --extras;
      last = e;
      visit(e);
    }
  };
  for (int k0 = li; k0 < le; k0 += 32) {
    const int k = k0 + lane;
    int i = 0, inf = 0, yes = 0;
    if (k < le) {
      i = list_a[k];
      inf = S.nxt[i];
      if (inf) {
        const int tinf = S.nxt[inf];
        double xi[3], xt[3];
        load3(S.X, T, i, xi);
        load3(S.X, T, tinf, xt);
        yes = dist_gen(xi, xt) < thr;
      }
    }
    __syncwarp();
    const int n = min(32, le - k0);
    for (int l = 0; l < n; ++l) {
      const int il = __shfl_sync(0xffffffffu, i, l);
      const int infl = __shfl_sync(0xffffffffu, inf, l);
      const int yl = __shfl_sync(0xffffffffu, yes, l);
      if (lane == 0) {
        run_extras(il - 1);
        last = il;
        if (tc.has(il) || tc.has(infl) || yl) visit(il);
      }
    }
    __threadfence_block();
    const int nt = __shfl_sync(0xffffffffu, tc.n, 0);
    __syncwarp();
    for (int q = lane; q < nt; q += 32) {
      const int kk = tlist[q];
      atomicAnd(&bits[kk >> 5], ~(1u << (kk & 31)));
    }
    if (lane == 0) tc.n = 0;
    flush_events(es, lane, ev, ev_count, ev_cap);
  }
  if (lane == 0) run_extras(lastslot);
  flush_events(es, lane, ev, ev_count, ev_cap);
  if (lane == 0) dyn[s] = d;
}

State make_state(nv_handle *h) {
  return State{h->x, h->u, h->u1, h->u2, h->gi, h->gb, h->closestd, h->nxt, h->prv, h->closest, h->T};
}

void compact(nv_handle *h, int *flag, int *pos, int *list) {
  TopoBuffers *tb = h->topo;
  size_t bytes = tb->cub_bytes;
  cub::DeviceScan::ExclusiveSum(tb->cub_tmp, bytes, flag, pos, (int)(h->T + 1), h->stream);
  k_scatter<<<grid_for(h->T, TB), TB, 0, h->stream>>>(flag, pos, list, h->T);
}

int resolver_grid(nv_handle *h) { return grid_for(h->nsys, 32); }

// Sweep bitmaps from a flag array.
Sweep make_sweep(nv_handle *h, const int *flag) {
  TopoBuffers *tb = h->topo;
  const long long T = h->T;
  const long long nw0 = T / 32 + 1;
  k_bits_l0<<<grid_for(nw0, 256), 256, 0, h->stream>>>(flag, tb->l0, T);
  k_bits_l1<<<grid_for(nw0 / 32 + 1, 256), 256, 0, h->stream>>>(tb->l0, tb->l1, nw0);
  return Sweep{tb->l0, tb->l1, T};
}

}  // namespace

void topo_alloc(nv_handle *h) {
  auto *tb = new TopoBuffers();
  const size_t n = (size_t)h->T + 1;
  cudaMalloc(&tb->flag_a, n * sizeof(int));
  cudaMalloc(&tb->pos_a, n * sizeof(int));
  cudaMalloc(&tb->list_a, n * sizeof(int));
  cudaMalloc(&tb->flag_b, n * sizeof(int));
  cudaMalloc(&tb->pos_b, n * sizeof(int));
  cudaMalloc(&tb->list_b, n * sizeof(int));
  cudaMalloc(&tb->flag_c, n * sizeof(int));
  cudaMalloc(&tb->pos_c, n * sizeof(int));
  cudaMalloc(&tb->list_c, n * sizeof(int));
  cudaMalloc(&tb->dec, n * sizeof(int));
  cudaMalloc(&tb->newslot, n * sizeof(int));
  cudaMalloc(&tb->xnew, 3 * n * sizeof(double));
  cudaMalloc(&tb->l0, (n / 32 + 2) * sizeof(unsigned));
  {
    // touched-slot bitmaps: shared memory up to the device's opt-in limit, else global
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int maxwords = (h->max_cap + 1 + 31) / 32;
    tb->smem_words = std::min(maxwords, std::max(0, optin - 4096) / 4);
    if (tb->smem_words < maxwords) {
      tb->touched_words = maxwords;
      cudaMalloc(&tb->touched, (size_t)h->nsys * maxwords * sizeof(unsigned));
    }
    const int smem = tb->smem_words * (int)sizeof(unsigned);
    cudaFuncSetAttribute(k_recon_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_remove_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  }
  cudaMalloc(&tb->l1, (n / 1024 + 2) * sizeof(unsigned));
  cub::DeviceScan::ExclusiveSum(nullptr, tb->cub_bytes, tb->flag_a, tb->pos_a, (int)n);
  cudaMalloc(&tb->cub_tmp, std::max<size_t>(tb->cub_bytes, 16));
  h->topo = tb;
}

void topo_free(nv_handle *h) {
  TopoBuffers *tb = h->topo;
  if (!tb) return;
  cudaFree(tb->flag_a); cudaFree(tb->pos_a); cudaFree(tb->list_a);
  cudaFree(tb->flag_b); cudaFree(tb->pos_b); cudaFree(tb->list_b);
  cudaFree(tb->flag_c); cudaFree(tb->pos_c); cudaFree(tb->list_c);
  cudaFree(tb->dec); cudaFree(tb->newslot); cudaFree(tb->xnew);
  cudaFree(tb->l0); cudaFree(tb->l1);
  if (tb->touched) cudaFree(tb->touched);
  cudaFree(tb->cub_tmp);
  delete tb;
  h->topo = nullptr;
}

void launch_pinsert(nv_handle *h) {
  TopoBuffers *tb = h->topo;
  const long long T = h->T;
  k_zero_live<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(h->d_dyn, h->nsys);
  k_ins_mark<<<grid_for(T + 1, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->gi, h->nxt,
                                                         tb->flag_a, tb->flag_b, tb->dec, T, h->d_err);
  compact(h, tb->flag_a, tb->pos_a, tb->list_a);  // candidates (either test passes)
  compact(h, tb->flag_b, tb->pos_b, tb->list_b);  // free slots
  k_zero_flags<<<grid_for(T + 1, TB), TB, 0, h->stream>>>(tb->flag_c, T);
  const int *ncand = tb->pos_a + T;
  k_ins_decide_easy<<<grid_for(T, 128), 128, 0, h->stream>>>(tb->list_a, ncand, tb->dec, tb->flag_c, h->d_err);
  compact(h, tb->flag_c, tb->pos_c, tb->list_c);  // ambiguous slots
  k_ins_decide_amb<<<resolver_grid(h), 32, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, h->prv, tb->pos_c, tb->list_c,
                                                           tb->pos_a, tb->dec, h->d_err);
  k_zero_flags<<<grid_for(T + 1, TB), TB, 0, h->stream>>>(tb->flag_c, T);
  k_ins_decide_case<<<grid_for(T, 128), 128, 0, h->stream>>>(tb->list_a, ncand, h->prv, tb->dec, tb->flag_c,
                                                             h->d_err);
  compact(h, tb->flag_c, tb->pos_c, tb->list_c);  // insertions, in sweep order
  const State S = make_state(h);
  // the number of insertions (pos_c[T]) is known only on the device: launch over every
  // slot, threads beyond the count return at once
  const int grid = grid_for(T, 128);
  const int *nev = tb->pos_c + T;
  k_ins_points<<<grid, 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, S, tb->pos_c, tb->list_c, tb->pos_b,
                                            tb->list_b, tb->dec, tb->newslot, tb->xnew, nev, h->d_err);
  k_ins_apply<<<grid, 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, S, tb->pos_c, tb->list_c, tb->newslot,
                                           tb->xnew, nev, h->d_events, h->d_event_count, h->event_cap, h->d_err);
  k_ins_ghosts<<<grid, 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, S, tb->list_c, tb->newslot, nev, h->d_err);
  k_ins_finish<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, tb->pos_c, tb->pos_b,
                                                              h->d_err);
  const Sweep sw = make_sweep(h, tb->flag_a);
  k_insert_resolve<<<resolver_grid(h), 32, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, S, sw, tb->pos_b, tb->list_b,
                                                           h->d_err, h->d_events, h->d_event_count, h->event_cap, 1);
}

void launch_pclose(nv_handle *h, bool only_brute) {
  bool any_brute = false, any_tree = false;
  for (auto &s : h->sc) (s.use_tree ? any_tree : any_brute) = true;
  if (any_brute)
    k_pclose_brute<<<grid_for(h->T, 128), 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->nxt, h->prv,
                                                               h->closest, h->closestd, h->T, h->d_err);
  if (any_tree && !only_brute) launch_closest_tree(h);
}

void launch_precon(nv_handle *h) {
  TopoBuffers *tb = h->topo;
  k_mark_recon<<<grid_for(h->T + 1, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->closestd, h->nxt,
                                                              tb->flag_a, h->T, h->d_err);
  compact(h, tb->flag_a, tb->pos_a, tb->list_a);
  const size_t smem = (size_t)tb->smem_words * sizeof(unsigned);
  k_recon_sweep<<<h->nsys, 32, smem, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, make_state(h), tb->pos_a, tb->list_a,
                                                  tb->touched, tb->touched_words, tb->smem_words, h->d_err,
                                                  h->d_events, h->d_event_count, h->event_cap);
}

void launch_premove(nv_handle *h) {
  TopoBuffers *tb = h->topo;
  k_mark_remove<<<grid_for(h->T + 1, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->nxt,
                                                               tb->flag_a, h->T, h->d_err);
  compact(h, tb->flag_a, tb->pos_a, tb->list_a);
  // extra visits start empty: bitmaps from an all-zero flag array
  k_zero_flags<<<grid_for(h->T + 1, TB), TB, 0, h->stream>>>(tb->flag_b, h->T);
  const Sweep sw = make_sweep(h, tb->flag_b);
  const size_t smem = (size_t)tb->smem_words * sizeof(unsigned);
  k_remove_sweep<<<h->nsys, 32, smem, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, make_state(h), tb->pos_a, tb->list_a,
                                                   tb->flag_a, sw, tb->touched, tb->touched_words, tb->smem_words,
                                                   h->d_err, h->d_events, h->d_event_count, h->event_cap);
}
