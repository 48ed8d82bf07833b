// solid.cu -- the topology stages of systems with solid walls, as exact serial sweeps.
//
// Points pinned to a wall (pinnedi: the segment in front ends in the wall, infront is the
// point itself; pinnedb: the same behind) change every topology stage of the reference:
// pinsert and premove skip them and clean up pairs of wall points (src/line.f90:36,109-127),
// loop_killer stops at them (src/reconnection.f90:164), and wall_recon (:66-150) cuts a
// filament that reaches a wall into two pinned ends.  Solid-wall runs are small (the
// reference's lattice example has a few thousand points), so here each of those stages is
// one thread per solid-wall system walking the slots in the reference's order on the live
// device state, statement for statement; the parallel stages of topo.cu skip these systems.
// Events go to the same log and digest as the parallel stages'.
#include "handle.cuh"

namespace {

struct SolidState {
  double *X, *U, *U1, *U2, *GI, *GB, *CD;
  int *nxt, *prv, *cl, *pin;
  long long T;
  DevEvent *ev;
  int *ev_count;
  int ev_cap;
};

__device__ bool solid_system(const SysConst &sc) { return sc.solid[0] || sc.solid[1] || sc.solid[2]; }

// clear_particle (general.f90:10-20): u_mf, u_sup, curv and stretch are kept, as there.
__device__ void clear_slot(const SolidState &S, int g) {
  for (int c = 0; c < 3; ++c) {
    S.X[c * S.T + g] = 0; S.U[c * S.T + g] = 0; S.U1[c * S.T + g] = 0; S.U2[c * S.T + g] = 0;
    S.GI[c * S.T + g] = 0; S.GB[c * S.T + g] = 0;
  }
  S.nxt[g] = 0; S.prv[g] = 0; S.cl[g] = 0; S.CD[g] = 0; S.pin[g] = 0;
}

// get_ghost_p (boundary.f90:26-84) of slot g on the current state
__device__ void refresh(const SysConst &sc, const SolidState &S, int g) {
  double x[3], xi[3], xb[3], gi[3], gb[3];
  load3(S.X, S.T, g, x);
  load3(S.X, S.T, S.nxt[g], xi);
  load3(S.X, S.T, S.prv[g], xb);
  ghosts_of(sc, S.pin[g], x, xi, xb, gi, gb);
  store3(S.GI, S.T, g, gi);
  store3(S.GB, S.T, g, gb);
}

// One logged event; j is a count for loop kills, wall cuts and wall-pair clean-ups.
__device__ void log_event(const SolidState &S, SysDyn &d, int s, int base, int kind, int i, int j) {
  const bool count = kind == NV_EV_LOOPKILL || kind == NV_EV_WALL || kind == NV_EV_CLEAR;
  const int seq = d.event_seq++;
  d.ev_hash += event_digest(seq, d.itime, kind, i - base, count ? j : j - base);
  const int a = atomicAdd(S.ev_count, 1);
  if (a < S.ev_cap) S.ev[a] = DevEvent{s, seq, d.itime, kind, i, j};
}

__device__ int live_count(const SolidState &S, int base, int pc) {
  int n = 0;
  for (int k = 1; k <= pc; ++k) n += S.nxt[base + k] > 0;
  return n;
}

// loop_killer (reconnection.f90:155-182): a loop that meets a pinned point is left alone.
__device__ void loop_killer(const SolidState &S, SysDyn &d, int s, int base, int particle) {
  const int pc = d.pcount;
  int counter = 1, next = particle;
  for (int it = 1; it <= pc; ++it) {
    if (pin_i(S.pin[next]) || pin_b(S.pin[next])) return;
    next = S.nxt[next];
    if (next == particle) break;
    counter = counter + 1;
  }
  if (counter < 4) {
    log_event(S, d, s, base, NV_EV_LOOPKILL, particle, counter);
    d.loop_kills += 1;
    d.nlive -= counter;
    next = particle;
    for (int it = 1; it <= pc; ++it) {
      const int store_next = S.nxt[next];
      clear_slot(S, next);
      next = store_next;
      if (next == particle) break;
    }
  }
}

// pinsert (line.f90:18-96) for one system.
__global__ void k_solid_pinsert(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, SolidState S, unsigned *err) {
  const int s = blockIdx.x;
  if (s >= nsys || threadIdx.x != 0 || *err || !solid_system(scs[s])) return;
  const SysConst &sc = scs[s];
  SysDyn &d = dyn[s];
  const int base = sc.base;
  const long long T = S.T;
  if (live_count(S, base, d.pcount) == 0) {
    atomicOr(err, DERR_EMPTY);
    return;
  }
  const int old_pcount = d.pcount;
  d.old_pcount = old_pcount;
  double total_length = 0.0;
  int free_at = 1;  // no slot below the first empty one empties during the sweep
  for (int i = 1; i <= old_pcount; ++i) {
    const int g = base + i;
    if (S.nxt[g] == 0) continue;
    if (pin_i(S.pin[g])) continue;
    double x[3], gi[3], gb[3];
    load3(S.X, T, g, x);
    load3(S.GI, T, g, gi);
    load3(S.GB, T, g, gb);
    const double disti = dist_gen(x, gi);
    total_length = e_add(total_length, disti);
    margin_note(d, 0, disti, sc.delta);
    if (!(disti > sc.delta)) continue;
    // the first empty slot (minloc(f(:)%infront)), else the array grows by one
    while (free_at <= d.pcount && S.nxt[base + free_at] != 0) ++free_at;
    int pn;
    if (free_at <= d.pcount) {
      pn = base + free_at;
    } else {
      if (d.pcount + 1 > sc.cap) {
        atomicOr(err, DERR_CAPACITY);
        return;
      }
      d.pcount += 1;
      pn = base + d.pcount;
      clear_slot(S, pn);
    }
    // the new point (line.f90:62-84)
    double xn[3];
    new_point(x, gi, gb, disti, xn);
    const int nx = S.nxt[g];
    for (int c = 0; c < 3; ++c) {
      S.X[c * T + pn] = xn[c];
      S.U[c * T + pn] = e_mul(0.5, e_add(S.U[c * T + g], S.U[c * T + nx]));
      S.U1[c * T + pn] = 0.0;
      S.U2[c * T + pn] = 0.0;
    }
    S.pin[pn] = 0;  // the pinned conditions zeroed (line.f90:82-84)
    S.prv[pn] = g;
    S.nxt[pn] = nx;
    refresh(sc, S, pn);
    S.prv[nx] = pn;
    refresh(sc, S, nx);
    S.nxt[g] = pn;
    refresh(sc, S, g);
    log_event(S, d, s, base, NV_EV_INSERT, g, pn);
    d.insert_count += 1;
    d.nlive += 1;
  }
  int empty = 0;
  for (int k = 1; k <= d.pcount; ++k) empty += S.nxt[base + k] == 0;
  d.total_length = total_length;
  d.avg_sep = total_length / (double)(old_pcount - empty);
}

// Two wall points next to each other, i pinned behind and its point in front pinned in
// front, are cleared together (line.f90:125-127, reconnection.f90:71-75).
__device__ bool clear_wall_pair(const SolidState &S, SysDyn &d, int s, int base, int g) {
  if (!pin_b(S.pin[g])) return false;
  const int nx = S.nxt[g];
  if (!pin_i(S.pin[nx])) return false;
  const int n = nx == g ? 1 : 2;
  log_event(S, d, s, base, NV_EV_CLEAR, g, n);
  clear_slot(S, nx);
  clear_slot(S, g);
  d.nlive -= n;
  return true;
}

// precon (reconnection.f90:11-61) for one system; pinned points never reach it as i or j
// (pclose gives them closestd = 100 and skips them as candidates).
__global__ void k_solid_precon(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, SolidState S,
                               const unsigned *err) {
  const int s = blockIdx.x;
  if (s >= nsys || threadIdx.x != 0 || *err || !solid_system(scs[s])) return;
  const SysConst &sc = scs[s];
  SysDyn &d = dyn[s];
  if ((d.itime % sc.recon_shots) != 0) return;
  const int base = sc.base;
  const long long T = S.T;
  for (int i = 1; i <= d.pcount; ++i) {
    const int g = base + i;
    if (S.nxt[g] == 0) continue;
    const int pari = S.nxt[g], parb = S.prv[g];
    const double cd = S.CD[g];
    if (cd > NV_EPS) margin_note(d, 2, cd, sc.delta / 2.);
    if (!((cd < sc.delta / 2.) && (cd > NV_EPS))) continue;
    const int j = S.cl[g];
    if (j == pari || j == parb || j == 0) continue;
    if (S.nxt[j] == 0) continue;
    const int parjb = S.prv[j];
    double t1[3], t2[3], x[3], gi_[3], gb_[3];
    for (int q = 0; q < 2; ++q) {  // norm_tanf (general.f90:106-117)
      double *t = q ? t2 : t1;
      const int p = q ? j : g;
      load3(S.X, T, p, x);
      load3(S.GI, T, p, gi_);
      load3(S.GB, T, p, gb_);
      deriv1(x, gi_, gb_, t);
      const double len = e_sqrt(e_add(e_add(e_sq(t[0]), e_sq(t[1])), e_sq(t[2])));
      for (int c = 0; c < 3; ++c) t[c] = e_div(t[c], len);
    }
    const double dot_val = dot3(t1, t2);
    margin_note(d, 3, dot_val, 0.9);
    if (dot_val > 0.9) continue;
    double xi[3], gii[3], gbi[3], xj[3], gij[3], gbj[3], xpi[3], xpj[3];
    load3(S.X, T, g, xi);
    load3(S.GI, T, g, gii);
    load3(S.GB, T, g, gbi);
    load3(S.X, T, j, xj);
    load3(S.GI, T, j, gij);
    load3(S.GB, T, j, gbj);
    load3(S.X, T, pari, xpi);
    load3(S.X, T, parjb, xpj);
    const double l_before =
        e_add(e_add(e_add(dist_gen(xi, gii), dist_gen(xi, gbi)), dist_gen(xj, gij)), dist_gen(xj, gbj));
    const double l_after =
        e_add(e_add(e_add(dist_gen(xi, gbi), dist_gen(xi, xj)), dist_gen(xj, gij)), dist_gen(xpi, xpj));
    if (!(l_after <= l_before)) continue;
    d.recon_count += 1;
    log_event(S, d, s, base, NV_EV_RECON, g, j);
    S.nxt[parjb] = pari;
    S.prv[pari] = parjb;
    S.nxt[g] = j;
    S.prv[j] = g;
    loop_killer(S, d, s, base, pari);
    loop_killer(S, d, s, base, g);
  }
}

// wall_recon (reconnection.f90:66-150) for one system: a point within delta/2 of a solid
// wall is removed and the filament cut there, its neighbours pinned to that wall.
__global__ void k_solid_wall_recon(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, SolidState S,
                                   const unsigned *err) {
  const int s = blockIdx.x;
  if (s >= nsys || threadIdx.x != 0 || *err || !solid_system(scs[s])) return;
  const SysConst &sc = scs[s];
  SysDyn &d = dyn[s];
  if ((d.itime % sc.recon_shots) != 0) return;
  const int base = sc.base;
  const long long T = S.T;
  for (int i = 1; i <= d.pcount; ++i) {
    const int g = base + i;
    if (S.nxt[g] == 0) continue;
    // a cleared pair: the reference goes on to test the cleared i at x = 0, inside every
    // wall while delta < box, so nothing more happens to it
    if (clear_wall_pair(S, d, s, base, g)) continue;
    if (pin_i(S.pin[g]) || pin_b(S.pin[g])) continue;
    for (int a = 0; a < 3; ++a) {  // x, y, z walls in turn, each on the state the last left
      if (!sc.solid[a]) continue;
      const double xa = S.X[a * T + g];
      const double lim = e_mul(0.5, e_sub(sc.box[a], sc.delta));
      int side = 0;
      if (xa > lim) side = 1;
      else if (xa < -lim) side = -1;
      if (side == 0) continue;
      const int pari = S.nxt[g], parb = S.prv[g];
      int w[3] = {0, 0, 0};
      w[a] = side;
      S.pin[pari] = pin_encode(pin_i(S.pin[pari]), 1, w);
      S.prv[pari] = pari;
      S.pin[parb] = pin_encode(1, pin_b(S.pin[parb]), w);
      S.nxt[parb] = parb;
      clear_slot(S, g);
      int cleared = 1;
      if (pin_i(S.pin[pari]) && pin_b(S.pin[pari])) {
        clear_slot(S, pari);
        ++cleared;
      }
      if (pin_i(S.pin[parb]) && pin_b(S.pin[parb])) {
        clear_slot(S, parb);
        ++cleared;
      }
      log_event(S, d, s, base, NV_EV_WALL, g, cleared);
      d.wall_recon_count += 1;
      d.nlive -= cleared;
    }
  }
}

// premove (line.f90:103-129) for one system.
__global__ void k_solid_premove(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, SolidState S,
                                const unsigned *err) {
  const int s = blockIdx.x;
  if (s >= nsys || threadIdx.x != 0 || *err || !solid_system(scs[s])) return;
  const SysConst &sc = scs[s];
  SysDyn &d = dyn[s];
  if ((d.itime % sc.recon_shots) != 0) return;
  const int base = sc.base;
  const long long T = S.T;
  const double thr = e_mul(.99, sc.delta);
  for (int i = 1; i <= d.pcount; ++i) {
    const int g = base + i;
    if (S.nxt[g] == 0) continue;
    if (pin_i(S.pin[g])) continue;
    const int infront = S.nxt[g];
    if (pin_i(S.pin[infront])) continue;
    const int tinfront = S.nxt[infront];
    double xi[3], xt[3];
    load3(S.X, T, g, xi);
    load3(S.X, T, tinfront, xt);
    const double dii = dist_gen(xi, xt);
    margin_note(d, 1, dii, thr);
    if (dii < thr) {
      S.prv[tinfront] = g;
      S.nxt[g] = tinfront;
      clear_slot(S, infront);
      log_event(S, d, s, base, NV_EV_REMOVE, g, infront);
      d.nlive -= 1;
      loop_killer(S, d, s, base, g);
      d.remove_count += 1;
    }
    clear_wall_pair(S, d, s, base, g);
  }
}

}  // namespace

static SolidState solid_state(nv_handle *h) {
  return SolidState{h->x,   h->u,   h->u1,      h->u2,  h->gi,        h->gb,           h->closestd,
                    h->nxt, h->prv, h->closest, h->pin, h->T,         h->d_events,     h->d_event_count,
                    h->event_cap};
}

void launch_solid_pinsert(nv_handle *h) {
  if (!h->any_solid) return;
  k_solid_pinsert<<<h->nsys, 32, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, solid_state(h), h->d_err);
}
void launch_solid_precon(nv_handle *h) {
  if (!h->any_solid) return;
  k_solid_precon<<<h->nsys, 32, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, solid_state(h), h->d_err);
}
void launch_wall_recon(nv_handle *h) {
  if (!h->any_solid) return;
  ++h->links_epoch;
  k_solid_wall_recon<<<h->nsys, 32, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, solid_state(h), h->d_err);
}
void launch_solid_premove(nv_handle *h) {
  if (!h->any_solid) return;
  k_solid_premove<<<h->nsys, 32, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, solid_state(h), h->d_err);
}
