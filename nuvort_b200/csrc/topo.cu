// topo.cu -- topology stages: pinsert, pclose (brute), precon, premove, loop_killer.
//
// The reference runs pinsert, precon and premove as serial sweeps in ascending slot order
// (src/line.f90:30, src/reconnection.f90:180, src/line.f90:107), where an event can change
// what later slots see.  Here each stage is
//   1. a parallel pass over all slots that marks the slots whose test can pass on the
//      current state (or, for pinsert, whose stale-ghost test passes);
//   2. a stable compaction of the marks into an ascending list per system (prefix sum);
//   3. one warp per system that walks the marked slots in ascending order, 32 at a time:
//      the lanes decide their candidates on the state at the start of the chunk in
//      parallel, lane 0 applies the events in order and decides again, on the live state,
//      every candidate whose inputs an earlier event of the chunk wrote (a shared-memory set
//      of touched slots).  Slots that an event makes testable and that the sweep reaches
//      later are visited as extra slots (a two-level bitmap).  pinsert has a fully
//      parallel form for the common case (see below) and sweeps only when that cannot apply.
// A slot that is neither marked nor touched has a test that is false in the serial sweep
// too, so the events are the reference's, event for event and in the same order.
#include <cmath>
#include <cstring>
#include <vector>

#include <cub/cub.cuh>

#include "handle.cuh"

struct TopoBuffers {
  int *flag_a = nullptr, *pos_a = nullptr, *list_a = nullptr;
  int *flag_b = nullptr, *pos_b = nullptr, *list_b = nullptr;
  int *flag_c = nullptr, *pos_c = nullptr, *list_c = nullptr;
  int *dec = nullptr;       // per slot: bit0 stale test, bit1 fresh test, bit2 inserts, bit3 case A
  int *newslot = nullptr;   // per slot: the slot its insertion fills
  double *xnew = nullptr;   // per insertion position: new point position [3][T]
  double *unew = nullptr;   // per insertion position: new point velocity [3][T]
  int *segnx = nullptr;     // per insertion position: infront of the original slot
  int *fh[2] = {nullptr, nullptr};  // higher-order insertion positions, H and H'
  int *pos_h = nullptr;     // exclusive prefix sum of H
  unsigned *l0 = nullptr, *l1 = nullptr;  // sweep bitmaps
  // pinsert's measured segment lengths (total_length, line.f90:39): per slot the stale and
  // the fresh distance, the one the sweep used, and per inserting slot the distance its new
  // point measured when the sweep reached it (-1: not reached)
  double *len_st = nullptr, *len_fr = nullptr, *seglen = nullptr, *dn_new = nullptr;
  int total_parts = 1;                          // blocks per system summing the lengths
  double *psum = nullptr, *pnear = nullptr;     // per (system, part): their sum and nearest to delta
  void *cub_tmp = nullptr;
  size_t cub_bytes = 0;
  // cell list of the closest-point search of the systems without a tree (pclose)
  struct CellGrid *grid = nullptr;  // per system; nc = 0 for tree systems
  long long n_cells = 0;            // cells of all systems
  int *cell_of = nullptr;           // per slot: its cell, -1 if not listed
  int *cell_cnt = nullptr;          // per cell: members (counted, then used as a fill cursor)
  int *cell_start = nullptr;        // per cell: first entry in cell_items (exclusive sum, n_cells + 1)
  int *cell_items = nullptr;        // slots grouped by cell
  bool any_cells = false;
};

// A system's cell grid over its box [-L/2, L/2)^3 (points outside are clamped to the edge
// cells): nc[a] cells of width L[a]/nc[a] >= wmin along axis a, cells numbered from base.
struct CellGrid {
  double inv_w[3], half[3];
  double wmin;
  int nc[3];
  long long base;
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

struct State {
  double *X, *U, *U1, *U2, *GI, *GB, *CD;
  int *nxt, *prv, *cl;
  long long T;
  double *seglen;  // pinsert: the length each visited slot measured
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
__global__ void k_mark_recon(const SysConst *__restrict__ scs, SysDyn *dyn, const int *__restrict__ sys_of,
                             const double *__restrict__ CD, const int *__restrict__ nxt, int *fa, long long T,
                             const unsigned *err) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g > T) return;
  int a = 0;
  if (g < T && !*err) {
    const int s = sys_of[g];
    const SysConst &sc = scs[s];
    const int k = (int)(g - sc.base);
    if (k >= 1 && k <= dyn[s].pcount && recon_step(sc, dyn[s]) && nxt[g] != 0 && !walled(sc)) {
      const double cd = CD[g];
      a = (cd < sc.delta / 2.) && (cd > NV_EPS);
      if (cd > NV_EPS) margin_note(dyn[s], 2, cd, sc.delta / 2.);
    }
  }
  fa[g] = a;
}

// premove marks: live slot with |x_i - x_{i+2}| < .99 delta (line.f90:113-115).
__global__ void k_mark_remove(const SysConst *__restrict__ scs, SysDyn *dyn, const int *__restrict__ sys_of,
                              const double *__restrict__ X, const int *__restrict__ nxt, int *fa, long long T,
                              const unsigned *err) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g > T) return;
  int a = 0;
  if (g < T && !*err) {
    const int s = sys_of[g];
    const SysConst &sc = scs[s];
    const int k = (int)(g - sc.base);
    if (k >= 1 && k <= dyn[s].pcount && recon_step(sc, dyn[s]) && nxt[g] != 0 && !walled(sc)) {
      double x[3], y[3];
      load3(X, T, (int)g, x);
      load3(X, T, nxt[nxt[g]], y);
      const double dii = dist_gen(x, y);
      a = dii < e_mul(.99, sc.delta);
      margin_note(dyn[s], 1, dii, e_mul(.99, sc.delta));
    }
  }
  fa[g] = a;
}

__global__ void k_scatter(const int *__restrict__ flag, const int *__restrict__ pos, int *__restrict__ list, long long T) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < T && flag[g]) list[pos[g]] = (int)g;
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

// ---- pclose on a cell list -------------------------------------------------------------------
// The reference's pclose (line.f90:135-160) is the exact nearest live non-neighbour by the
// non-periodic distance, the first j in ascending order among equal distances (strict <), and
// it leaves closest alone when no j comes below 100.  The cell list finds the same point: the
// target searches rings of cells around its own (Chebyshev ring r), keeps the minimum of
// (distance, slot) -- the lowest slot among equal distances, whatever the visiting order -- and
// stops once that distance is below r * wmin: every point outside rings 0..r lies in a cell at
// least r+1 cells away along some axis, so at least r whole cell widths away.  (A point within
// rounding of a cell face may be filed one cell off; the stop test keeps a relative margin of
// 1e-10, far above that rounding.)
__device__ __forceinline__ int cell_coord(const CellGrid &G, int a, double x) {
  const double f = (x + G.half[a]) * G.inv_w[a];
  int c = f < 0. ? 0 : (int)f;
  return c >= G.nc[a] ? G.nc[a] - 1 : c;
}

__global__ void k_cell_count(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                             const int *__restrict__ sys_of, const CellGrid *__restrict__ grid,
                             const double *__restrict__ X, const int *__restrict__ nxt, int *__restrict__ cell_of,
                             int *__restrict__ cnt, long long T, const unsigned *err) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T) return;
  int c = -1;
  const int s = sys_of[g];
  const SysConst &sc = scs[s];
  const CellGrid &G = grid[s];
  const int k = (int)(g - sc.base);
  if (!*err && G.nc[0] > 0 && recon_step(sc, dyn[s]) && k >= 1 && k <= dyn[s].pcount && nxt[g] != 0 &&
      pinned_at(sc, (int)g)) {
    c = -2;  // a pinned point: neither a target nor a candidate (line.f90:142-149)
  } else if (!*err && G.nc[0] > 0 && recon_step(sc, dyn[s]) && k >= 1 && k <= dyn[s].pcount && nxt[g] != 0) {
    double x[3];
    load3(X, T, (int)g, x);
    c = (int)(G.base + ((long long)cell_coord(G, 2, x[2]) * G.nc[1] + cell_coord(G, 1, x[1])) * G.nc[0] +
              cell_coord(G, 0, x[0]));
    atomicAdd(&cnt[c], 1);
  }
  cell_of[g] = c;
}

// Files each listed slot into its cell (the order inside a cell does not matter: the search
// takes the minimum of (distance, slot)).
__global__ void k_cell_fill(const int *__restrict__ cell_of, const int *__restrict__ start, int *__restrict__ cnt,
                            int *__restrict__ items, long long T) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T) return;
  const int c = cell_of[g];
  if (c < 0) return;
  items[start[c] + atomicSub(&cnt[c], 1) - 1] = (int)g;
}

__global__ void k_pclose_cells(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                               const int *__restrict__ sys_of, const CellGrid *__restrict__ grid,
                               const double *__restrict__ X, const int *__restrict__ nxt, const int *__restrict__ prv,
                               const int *__restrict__ cell_of, const int *__restrict__ start,
                               const int *__restrict__ items, int *__restrict__ cl, double *__restrict__ CD,
                               long long T) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T) return;
  if (cell_of[g] == -2) CD[g] = 100.;  // pinned: closestd=100 and no search
  if (cell_of[g] < 0) return;  // listed: live unpinned slot of a cell-list system on a recon step
  const int s = sys_of[g];
  const CellGrid &G = grid[s];
  const int ni = nxt[g], pi = prv[g];
  double xi[3];
  load3(X, T, (int)g, xi);
  const int cx = cell_coord(G, 0, xi[0]), cy = cell_coord(G, 1, xi[1]), cz = cell_coord(G, 2, xi[2]);
  const int rmax = max(max(G.nc[0], G.nc[1]), G.nc[2]) - 1;
  bool found = false;
  double best = 100.;
  int bj = cl[g];
  for (int r = 0; r <= rmax; ++r) {
    for (int dz = -r; dz <= r; ++dz) {
      const int z = cz + dz;
      if (z < 0 || z >= G.nc[2]) continue;
      for (int dy = -r; dy <= r; ++dy) {
        const int y = cy + dy;
        if (y < 0 || y >= G.nc[1]) continue;
        const bool shell = dz == -r || dz == r || dy == -r || dy == r;
        for (int dx = -r; dx <= r; dx += (shell || r == 0) ? 1 : 2 * r) {  // interior rows: the two end cells
          const int x = cx + dx;
          if (x < 0 || x >= G.nc[0]) continue;
          const long long c = G.base + ((long long)z * G.nc[1] + y) * G.nc[0] + x;
          for (int e = start[c]; e < start[c + 1]; ++e) {
            const int j = items[e];
            if (j == g || j == ni || j == pi) continue;
            double xj[3];
            load3(X, T, j, xj);
            const double d2 =
                e_add(e_add(e_sq(e_sub(xi[0], xj[0])), e_sq(e_sub(xi[1], xj[1]))), e_sq(e_sub(xi[2], xj[2])));
            const double dist = e_sqrt(d2);
            if (found ? (dist < best || (dist == best && j < bj)) : dist < best) {
              best = dist;
              bj = j;
              found = true;
            }
          }
        }
      }
    }
    if (found && best < (double)r * G.wmin * (1. - 1e-10)) break;
  }
  cl[g] = bj;
  CD[g] = best;
}

// pclose (line.f90:135-160): exact nearest non-neighbour, non-periodic distance, strict <
// so ties keep the lowest j.  One thread per target slot, every slot scanned: kept as the
// method to compare the cell list with (nv_set_pclose_method).
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
  if (pinned_at(sc, (int)g)) {  // pinned points are not tested (line.f90:142-144)
    CD[g] = 100.;
    return;
  }
  const int ni = nxt[g], pi = prv[g];
  double xi[3];
  load3(X, T, (int)g, xi);
  double best = 100.;
  double best2 = 1e300;
  int bj = cl[g];
  for (int j = sc.base + 1; j <= sc.base + pc; ++j) {
    if (nxt[j] == 0 || j == g || j == ni || j == pi || pinned_at(sc, j)) continue;
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


// g as seen from x: the nearest periodic image (get_ghost_p's adjustment)
__device__ __forceinline__ void ghost_of(const SysConst &sc, const double x[3], const double g[3], double out[3]) {
  for (int c = 0; c < 3; ++c) out[c] = g[c];
  ghost_adjust(sc, x, out);
}

// ---- parallel pinsert ---------------------------------------------------------------------
// In the serial sweep (line.f90:30-93) slot k is tested against its step-start ghost unless
// its predecessor p = behind(k) < k inserted earlier in the same sweep: that insertion
// refreshed k's ghosts from the current positions (line.f90:88-89).  So each live slot has
// two candidate outcomes, a stale test and a fresh test; when they agree the outcome is
// known, and only slots where they differ depend on their predecessor's outcome.
// New points that the sweep reaches later (placed in a free slot above their creator) are
// tested again by the reference and may insert in turn; k_ins_chain resolves those
// higher-order insertions by a fixed-point iteration over their positions.

// bit0 stale test, bit1 fresh test (ghost of the current infront position); list = either.
__global__ void k_ins_mark(const SysConst *__restrict__ scs, SysDyn *__restrict__ dyn, const int *__restrict__ sys_of,
                           const double *__restrict__ X, const double *__restrict__ GI, const int *__restrict__ nxt,
                           int *fa, int *fb, int *dec, double *len_st, double *len_fr, long long T,
                           const unsigned *err) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g > T) return;
  int a = 0, b = 0, dv = 0;
  double lst = 0., lfr = 0.;
  if (g < T && !*err) {
    const int s = sys_of[g];
    const SysConst &sc = scs[s];
    const int k = (int)(g - sc.base);
    if (k >= 1 && k <= dyn[s].pcount && !walled(sc)) {
      if (nxt[g] == 0) {
        b = 1;
      } else {
        double x[3], gi[3], gf[3];
        load3(X, T, (int)g, x);
        load3(GI, T, (int)g, gi);
        load3(X, T, nxt[g], gf);
        ghost_adjust(sc, x, gf);
        lst = dist_gen(x, gi);
        lfr = dist_gen(x, gf);
        const int st = lst > sc.delta, fr = lfr > sc.delta;
        dv = st | (fr << 1);
        a = st | fr;
        dyn[s].live = 1;
      }
    }
  }
  fa[g] = a;
  fb[g] = b;
  if (g < T) {
    dec[g] = dv;
    len_st[g] = lst;
    len_fr[g] = lfr;
  }
}

// The length each live slot's test measured (line.f90:38-39): with the ghosts its
// predecessor's insertion refreshed when that predecessor lies below it and inserts (the
// same rule as its decision), else with the step-start ghosts; 0 for empty slots.  New points
// the sweep reaches are written when the insertions are applied.
__global__ void k_ins_len(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                          const int *__restrict__ sys_of, const int *__restrict__ nxt, const int *__restrict__ prv,
                          const int *__restrict__ dec, const double *__restrict__ len_st,
                          const double *__restrict__ len_fr, double *__restrict__ seglen, long long T) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T) return;
  double v = 0.;
  const int s = sys_of[g];
  const int k = (int)(g - scs[s].base);
  if (k >= 1 && k <= dyn[s].pcount && nxt[g] != 0) {
    const int p = prv[g];
    v = (p < g && (dec[p] & 4)) ? len_fr[g] : len_st[g];
  }
  seglen[g] = v;
}

// total_length and avg_sep of the pinsert just made (line.f90:39,95): the measured lengths
// summed in a fixed order -- block (s, p) sums part p of system s's slots (per thread by
// stride, then a tree over the block), and k_ins_total adds the parts in order (the reference
// adds them one after another, which agrees to ~1e-13 relative) -- divided by old_pcount minus
// the empty slots left among the pcount slots.  Many blocks per large system: one block
// summing a million lengths takes milliseconds.
constexpr int kTotalThreads = 256;
__global__ void __launch_bounds__(kTotalThreads) k_ins_part(const SysConst *__restrict__ scs, const SysDyn *dyn,
                                                            int nsys, int parts, const double *__restrict__ seglen,
                                                            double *__restrict__ psum, double *__restrict__ pnear,
                                                            const unsigned *err) {
  __shared__ double sum_[kTotalThreads], near_[kTotalThreads];
  const int s = blockIdx.x / parts, p = blockIdx.x % parts;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  if (walled(sc)) return;  // the serial sweep of solid.cu sums its own lengths
  const int pc = dyn[s].pcount;
  const bool margins = dyn[s].margin_on;
  const int per = (pc + parts - 1) / parts;
  const int k0 = 1 + p * per, k1 = min(pc, k0 + per - 1);
  double acc = 0., near = 1e300;  // near: the smallest |length - delta| (event margins)
  for (int k = k0 + threadIdx.x; k <= k1; k += kTotalThreads) {
    const double l = seglen[sc.base + k];
    acc += l;
    if (margins && l > 0.) near = fmin(near, fabs(l - sc.delta));  // the lengths the tests measured
  }
  sum_[threadIdx.x] = acc;
  near_[threadIdx.x] = near;
  __syncthreads();
  for (int w = kTotalThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sum_[threadIdx.x] += sum_[threadIdx.x + w];
      near_[threadIdx.x] = fmin(near_[threadIdx.x], near_[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    psum[blockIdx.x] = sum_[0];
    pnear[blockIdx.x] = near_[0];
  }
}

__global__ void k_ins_total(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, int parts,
                            const double *__restrict__ psum, const double *__restrict__ pnear, const unsigned *err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  if (walled(sc)) return;
  SysDyn &d = dyn[s];
  double tot = 0., near = 1e300;
  for (int p = 0; p < parts; ++p) {
    tot += psum[s * parts + p];
    near = fmin(near, pnear[s * parts + p]);
  }
  d.total_length = tot;
  const int empty = d.pcount - d.nlive;
  d.avg_sep = tot / (double)(d.old_pcount - empty);
  if (d.margin_on && near < 1e300) margin_note_abs(d, 0, near, sc.delta);
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

// Ambiguous slots.  The outcome of ambiguous k is its fresh test when p = behind(k) < k
// inserts, else its stale test; p's outcome is final unless p is ambiguous too.  So the
// ambiguous slots form chains k -> infront(k) (while infront(k) > k is ambiguous), each
// starting at a slot whose predecessor is decided or lies above it.  One thread per
// ambiguous slot; the chain heads walk their chains.
__global__ void k_ins_decide_amb(const int *__restrict__ list_m, const int *__restrict__ n_ptr,
                                 const int *__restrict__ nxt, const int *__restrict__ prv,
                                 const int *__restrict__ famb, int *dec, const unsigned *err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *n_ptr || *err) return;
  int k = list_m[t];
  const int p = prv[k];
  if (p < k && famb[p]) return;  // inside a chain: its head decides it
  int refreshed = p < k && (dec[p] & 4);
  for (;;) {
    const int dv = dec[k];
    const int d = refreshed ? (dv >> 1) & 1 : dv & 1;
    dec[k] = dv | (d << 2);
    const int nx = nxt[k];
    if (!(nx > k && famb[nx])) break;
    refreshed = d;
    k = nx;
  }
}

// Per-system state of a pinsert: flags of the fixed-point iteration, live marker.
__global__ void k_ins_begin(SysDyn *dyn, int nsys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  dyn[s].live = 0;
  dyn[s].old_pcount = dyn[s].pcount;
  dyn[s].ins_fallback = 0;
  dyn[s].ins_conv = 0;
  dyn[s].ins_mismatch = 0;
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

// New points along chains of consecutive insertions, with the insertions of new points the
// sweep reaches again.  A chain starts at an inserting slot whose ghosts were not refreshed
// (case B) and continues to infront(k) while that slot inserts in case A (its ghosts then
// hold the current infront position and the newest point placed behind it).
//
// The insertion at k puts e1 between k and nx = infront(k).  When e1's slot lies above k
// (and within the step-start pcount) the sweep visits e1 at that position and tests it
// against nx; if it inserts, e2 goes between e1 and nx, and so on: a sub-chain e1, e2, ...
// whose points are fixed by positions alone (e_m's ghosts are nx and e_{m-1}, or k).  The
// one quantity that couples different chains is the slot of each new point, the free slot
// of the insertion's rank in sweep order, where the sweep order merges the original
// insertions (at their slots) with these higher-order ones (at the new points' slots).
// Given a set H of higher-order positions, pos_c + pos_h give every rank; the walk then
// yields the higher-order positions H' it implies.  Each event depends only on events at
// lower positions, so once H' = H every event is the serial sweep's (by induction over the
// sweep position).  The walk is repeated from H = {} a fixed number of times; a system
// that has not converged by then runs the serial sweep.
__global__ void k_ins_chain(const SysConst *__restrict__ scs, SysDyn *dyn, const int *__restrict__ sys_of, State S,
                            const int *__restrict__ pos_c, const int *__restrict__ list_c,
                            const int *__restrict__ pos_b, const int *__restrict__ list_b, const int *__restrict__ dec,
                            const int *__restrict__ pos_h, int *fout, int *newslot, int *segnx, double *xnew,
                            double *unew, double *dn_new, const int *__restrict__ nev_total, unsigned *err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *nev_total || *err) return;
  int k = list_c[t];
  if (dec[k] & 8) return;  // not a chain head
  const int s = sys_of[k];
  if (dyn[s].ins_conv || dyn[s].ins_fallback) return;
  const SysConst &sc = scs[s];
  const int base = sc.base;
  const int ev0 = pos_c[base], h0 = pos_h[base];
  const int fb0 = pos_b[base], nfree = pos_b[base + sc.cap + 1] - fb0;
  const int pc = dyn[s].pcount;
  const long long T = S.T;
  const int old_last = base + pc;
  // slot of the insertion with sweep rank r: the free slots in ascending order, then pcount+1..
  auto slot_of = [&](int g) -> int {
    const int r = (pos_c[g] - ev0) + (pos_h[g] - h0);
    const int slot = r < nfree ? list_b[fb0 + r] : base + pc + 1 + (r - nfree);
    if (slot > base + sc.cap) {  // possibly an artefact of a not yet consistent H:
      dyn[s].ins_fallback = 1;    // the serial sweep decides (and reports a real overflow)
      return -1;
    }
    return slot;
  };
  auto put = [&](int g, int slot, int nx, const double xn[3], const double un[3]) {
    newslot[g] = slot;
    segnx[g] = nx;
    for (int c = 0; c < 3; ++c) {
      xnew[c * T + g] = xn[c];
      unew[c * T + g] = un[c];
    }
  };
  double gbk[3];
  bool fresh = false;
  for (;;) {
    const int slot = slot_of(k);
    if (slot < 0) return;
    double x[3], gi[3], gb[3], xnx[3], uk[3], unx[3], xn[3], un[3];
    load3(S.X, T, k, x);
    const int nx = S.nxt[k];
    load3(S.X, T, nx, xnx);
    if (fresh) {  // ghosts refreshed by the predecessor's insertion (get_ghost_p, line.f90:89)
      ghost_of(sc, x, xnx, gi);
      ghost_of(sc, x, gbk, gb);
    } else {
      load3(S.GI, T, k, gi);
      load3(S.GB, T, k, gb);
    }
    new_point(x, gi, gb, dist_gen(x, gi), xn);
    load3(S.U, T, k, uk);
    load3(S.U, T, nx, unx);
    for (int c = 0; c < 3; ++c) un[c] = e_mul(0.5, e_add(uk[c], unx[c]));
    put(k, slot, nx, xn, un);
    // the sub-chain of new points the sweep reaches again
    double last[3], xe[3], ue[3], xprev[3];
    for (int c = 0; c < 3; ++c) {
      last[c] = xn[c];
      xe[c] = xn[c];
      ue[c] = un[c];
      xprev[c] = x[c];
    }
    int at = k, e = slot;
    for (;;) {
      if (!(e > at && e <= old_last)) {  // the sweep never reaches at's new point
        dn_new[at] = -1.0;
        break;
      }
      double gie[3], gbe[3], xq[3], uq[3];
      ghost_of(sc, xe, xnx, gie);
      const double dn = dist_gen(xe, gie);
      dn_new[at] = dn;  // the length the new point e measures when the sweep reaches it
      if (!(dn > sc.delta)) break;
      fout[e] = 1;
      const int q = slot_of(e);
      if (q < 0) return;
      ghost_of(sc, xe, xprev, gbe);
      new_point(xe, gie, gbe, dn, xq);
      for (int c = 0; c < 3; ++c) uq[c] = e_mul(0.5, e_add(ue[c], unx[c]));
      put(e, q, nx, xq, uq);
      if (e < nx)  // inserted before the sweep reaches nx: nx's behind ghost
        for (int c = 0; c < 3; ++c) last[c] = xq[c];
      for (int c = 0; c < 3; ++c) {
        xprev[c] = xe[c];
        xe[c] = xq[c];
        ue[c] = uq[c];
      }
      at = e;
      e = q;
    }
    // continue the chain: infront(k) inserts with ghosts refreshed by this insertion
    if (nx > k && (dec[nx] & 8)) {
      for (int c = 0; c < 3; ++c) gbk[c] = last[c];
      fresh = true;
      k = nx;
      continue;
    }
    break;
  }
}

// Every system takes the serial sweep (no fixed-point rounds).
__global__ void k_ins_all_serial(SysDyn *dyn, int nsys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nsys) dyn[s].ins_fallback = 1;
}

// Zero the output flags of the systems still iterating.
__global__ void k_ins_zero_open(const SysDyn *__restrict__ dyn, const int *__restrict__ sys_of, int *f, long long T) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T) return;
  if (!dyn[sys_of[g]].ins_conv) f[g] = 0;
}

// Count, per system still iterating, the positions where H and H' differ.
__global__ void k_ins_compare(SysDyn *dyn, const int *__restrict__ sys_of, const int *__restrict__ fin,
                              const int *__restrict__ fout, long long T) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T || fin[g] == fout[g]) return;
  const int s = sys_of[g];
  if (!dyn[s].ins_conv) atomicAdd(&dyn[s].ins_mismatch, 1);
}

// A system whose H' equals H has converged (iteration `it`, counted from 1).
__global__ void k_ins_converge(SysDyn *dyn, int nsys, int it, int last) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  SysDyn &d = dyn[s];
  if (d.ins_conv || d.ins_fallback) return;
  if (d.ins_mismatch == 0) {
    d.ins_conv = 1;
    d.diag[6] = it;
  } else if (last) {
    d.ins_fallback = 1;
    d.diag[6] = it;
  }
  d.ins_mismatch = 0;
}

// Apply every insertion (links, new point state) and log the events in sweep order: one
// thread per original insertion, following its sub-chain.
__global__ void k_ins_apply(const SysConst *__restrict__ scs, SysDyn *dyn, const int *__restrict__ sys_of, State S,
                            const int *__restrict__ pos_c, const int *__restrict__ list_c,
                            const int *__restrict__ pos_h, const int *__restrict__ fh,
                            const int *__restrict__ newslot, const int *__restrict__ segnx,
                            const double *__restrict__ xnew, const double *__restrict__ unew,
                            const double *__restrict__ dn_new, const int *__restrict__ nev_total, DevEvent *ev,
                            int *ev_count, int ev_cap, unsigned *err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *nev_total || *err) return;
  const int k = list_c[t];
  const int s = sys_of[k];
  if (dyn[s].ins_fallback) return;
  const SysConst &sc = scs[s];
  const long long T = S.T;
  const int ev0 = pos_c[sc.base], h0 = pos_h[sc.base];
  const int seq0 = dyn[s].event_seq, itime = dyn[s].itime;
  const int nx = segnx[k];
  const double zero[3] = {0, 0, 0};
  int g = k;
  for (int hops = 0;; ++hops) {
    if (hops > sc.cap) {  // a sub-chain is shorter than the free slots; guard only
      atomicOr(err, DERR_QUEUE);
      return;
    }
    const int q = newslot[g];
    double xn[3], un[3];
    for (int c = 0; c < 3; ++c) {
      xn[c] = xnew[c * T + g];
      un[c] = unew[c * T + g];
    }
    store3(S.X, T, q, xn);
    store3(S.U, T, q, un);
    store3(S.U1, T, q, zero);
    store3(S.U2, T, q, zero);
    S.cl[q] = 0;
    S.CD[q] = 0;
    S.prv[q] = g;
    S.nxt[g] = q;
    if (dn_new[g] >= 0.) S.seglen[q] = dn_new[g];
    const int seq = seq0 + (pos_c[g] - ev0) + (pos_h[g] - h0);
    const int a = atomicAdd(ev_count, 1);
    if (a < ev_cap) ev[a] = DevEvent{s, seq, itime, NV_EV_INSERT, g, q};
    atomicAdd(&dyn[s].ev_hash, event_digest(seq, itime, NV_EV_INSERT, g - sc.base, q - sc.base));
    if (fh[q]) {  // the sweep reaches q and it inserts
      g = q;
      continue;
    }
    S.nxt[q] = nx;
    S.prv[nx] = q;
    break;
  }
}

// Ghosts of every slot an insertion touched, from the final links and positions (each
// touched slot's last refresh in the serial sweep sees exactly this state).
__global__ void k_ins_ghosts(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                             const int *__restrict__ sys_of, State S, const int *__restrict__ list_c,
                             const int *__restrict__ fh, const int *__restrict__ newslot,
                             const int *__restrict__ nev_total, unsigned *err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *nev_total || *err) return;
  const int k = list_c[t];
  const int s = sys_of[k];
  if (dyn[s].ins_fallback) return;
  const SysConst &sc = scs[s];
  refresh_ghosts(sc, S, k);
  int q = newslot[k];
  for (int hops = 0;; ++hops) {
    if (hops > sc.cap) {
      atomicOr(err, DERR_QUEUE);
      return;
    }
    refresh_ghosts(sc, S, q);
    if (!fh[q]) break;
    q = newslot[q];
  }
  refresh_ghosts(sc, S, S.nxt[q]);
}

// Counters: pcount grows by the insertions beyond the free slots.
__global__ void k_ins_finish(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, const int *__restrict__ pos_a,
                             const int *__restrict__ pos_c, const int *__restrict__ pos_h,
                             const int *__restrict__ pos_b, unsigned *err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  if (walled(sc)) return;
  SysDyn &d = dyn[s];
  if (d.live == 0) {
    atomicOr(err, DERR_EMPTY);
    return;
  }
  const int end = sc.base + sc.cap + 1;
  d.diag[0] = pos_a[end] - pos_a[sc.base];
  const int nhigh = pos_h[end] - pos_h[sc.base];
  const int nev = pos_c[end] - pos_c[sc.base] + nhigh;
  d.diag[1] = nev;
  d.diag[5] = nhigh;
  if (d.ins_fallback) return;
  const int nfree = pos_b[end] - pos_b[sc.base];
  d.event_seq += nev;
  d.insert_count += nev;
  d.nlive += nev;
  if (nev > nfree) d.pcount += nev - nfree;
}


// ---- precon sweep, warp-prefetched --------------------------------------------------------
// The reference's sweep (reconnection.f90:180-221) is kept exactly: candidates in ascending
// order, each decided on the state left by the events before it.  A warp loads 32
// candidates at a time and decides each on the current state in parallel; lane 0 then walks
// them in order.  A candidate's decision reads the links of i and of its partner j only
// (nxt/prv of both; x and ghosts do not change in precon, and a cleared neighbour means a
// cleared i or j), so the parallel decision stands unless an event earlier in the sweep
// wrote the links of i or j -- tracked in a shared-memory set of touched slots.  Touched
// candidates are decided again by lane 0 on the live state.

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

// Slots written by the events of the current chunk, as an open-addressing hash set in
// shared memory (keys are global slot indices, 0 = empty; the per-system dummy slot is
// never recorded).  After kLimit slots the set is full and every slot counts as touched
// until the chunk ends, so the remaining candidates are decided on the live state.
template <int kBits, int kLimit>
struct SlotSet {
  static constexpr int kCap = 1 << kBits;
  static_assert(2 * kLimit <= kCap, "load factor above one half");
  int *keys;
  int n;
  int full;
  int base;
  unsigned char *fl = nullptr;  // optional per-entry flags (what was written)
  __device__ static int home(int g) { return (int)(((unsigned)g * 0x9E3779B1u) >> (32 - kBits)); }
  // table index of g, or -1
  __device__ int find(int g) const {
    for (int h = home(g);; h = (h + 1) & (kCap - 1)) {
      const int k = keys[h];
      if (k == g) return h;
      if (k == 0) return -1;
    }
  }
  // table index of g after recording it, or -1 once the set is full
  __device__ int add(int g) {
    if (g <= base || full) return -1;
    int h = home(g);
    for (;; h = (h + 1) & (kCap - 1)) {
      const int k = keys[h];
      if (k == g) return h;
      if (k == 0) break;
    }
    if (n == kLimit) {
      full = 1;
      return -1;
    }
    keys[h] = g;
    if (fl) fl[h] = 0;
    ++n;
    return h;
  }
  // record g with flag bits f (the flags array must be set)
  __device__ void add(int g, unsigned f) {
    const int h = add(g);
    if (h >= 0) fl[h] |= (unsigned char)f;
  }
  __device__ bool has(int g) const { return full || (g > base && find(g) >= 0); }
  // g recorded with any of the flag bits f
  __device__ bool has(int g, unsigned f) const {
    if (full) return true;
    if (g <= base) return false;
    const int h = find(g);
    return h >= 0 && (fl[h] & f);
  }
  // warp-collective: empty the set for the next chunk (lane 0 holds n and full)
  __device__ void reset(int lane) {
    __syncwarp();
    const int used = __shfl_sync(0xffffffffu, n | full, 0);
    if (used) {
      for (int q = lane; q < kCap; q += 32) keys[q] = 0;
    }
    n = 0;
    full = 0;
    __syncwarp();
  }
};
constexpr int kTouchedPerChunk = 32 * 10;  // 4 relinked + up to 6 cleared slots per event
using Touched = SlotSet<10, kTouchedPerChunk>;

// A sweep's running event number and counters, in registers of the thread that applies
// the events; written back to the system's SysDyn when the sweep ends.
struct Tally {
  int seq, itime, pcount, base;
  int recon, remove, insert, kills, cleared;  // cleared: points the loop kills cleared
  unsigned long long hash;
  __device__ static Tally of(const SysDyn &d, int base) {
    return Tally{d.event_seq, d.itime, d.pcount, base, 0, 0, 0, 0, 0, 0ull};
  }
  __device__ void store(SysDyn &d) const {
    d.event_seq = seq;
    d.ev_hash += hash;
    d.recon_count += recon;
    d.remove_count += remove;
    d.insert_count += insert;
    d.loop_kills += kills;
    d.nlive += insert - remove - cleared;
  }
};

// Events of one chunk, staged in shared memory by lane 0 and written with one atomic.  A
// chunk with more events than the stage holds spills the stage from lane 0.
constexpr int kEventStage = 96;
struct EventStage {
  DevEvent *buf;
  int n;
  DevEvent *ev;
  int *ev_count;
  int ev_cap;
  __device__ void spill() {
    const int at = atomicAdd(ev_count, n);
    for (int q = 0; q < n; ++q)
      if (at + q < ev_cap) ev[at + q] = buf[q];
    n = 0;
  }
  __device__ void add(Tally &t, int s, int kind, int i, int j) {
    if (n == kEventStage) spill();
    t.hash += event_digest(t.seq, t.itime, kind, i - t.base, kind == NV_EV_LOOPKILL ? j : j - t.base);
    buf[n++] = DevEvent{s, t.seq++, t.itime, kind, i, j};
  }
};
__device__ void flush_events(EventStage &es, int lane) {
  const int n = __shfl_sync(0xffffffffu, es.n, 0);
  if (n == 0) return;
  int at = 0;
  if (lane == 0) at = atomicAdd(es.ev_count, n);
  at = __shfl_sync(0xffffffffu, at, 0);
  for (int q = lane; q < n; q += 32)
    if (at + q < es.ev_cap) es.ev[at + q] = es.buf[q];
  __syncwarp();
  if (lane == 0) es.n = 0;
  __syncwarp();
}

// loop_killer (reconnection.f90:155-182).  Only "fewer than 4 points" matters, so the
// count stops after three hops; the result equals the reference's full walk.
template <class Set, class OnClear>
__device__ void loop_killer_stage(const State &S, Tally &d, int s, int particle, int pcount, EventStage &es,
                                  Set &tc, OnClear on_clear) {
  int counter = 1, nx = particle;
  const int hops = pcount < 3 ? pcount : 3;
  for (int it = 0; it < hops; ++it) {
    nx = S.nxt[nx];
    if (nx == particle) break;
    counter++;
  }
  if (counter < 4) {
    es.add(d, s, NV_EV_LOOPKILL, particle, counter);
    d.kills++;
    d.cleared += counter;
    nx = particle;
    for (int it = 0; it < pcount; ++it) {
      const int sn = S.nxt[nx];
      if (tc.fl) tc.add(nx, 3u);
      else tc.add(nx);
      on_clear(nx);
      clear_particle(S, nx);
      nx = sn;
      if (nx == particle) break;
    }
  }
}
template <class Set>
__device__ void loop_killer_stage(const State &S, Tally &d, int s, int particle, int pcount, EventStage &es,
                                  Set &tc) {
  loop_killer_stage(S, d, s, particle, pcount, es, tc, [](int) {});
}

// loop_killer's count (up to three hops) on links read from a small override table first
// (the links an event just rewrote and links prefetched before it), global memory after.
template <int N>
__device__ int loop_count(const State &S, int particle, int pcount, const int (&key)[N], const int (&val)[N]) {
  int counter = 1, nx = particle;
  const int hops = pcount < 3 ? pcount : 3;
  for (int it = 0; it < hops; ++it) {
    int nn = -1;
#pragma unroll
    for (int q = 0; q < N; ++q)
      if (nn < 0 && key[q] == nx) nn = val[q];
    nx = nn >= 0 ? nn : S.nxt[nx];
    if (nx == particle) break;
    counter++;
  }
  return counter;
}

// ---- sweeps by rounds of kRound candidates -------------------------------------------------
// A block of kRound threads loads kRound candidates at once and decides each on the state at
// the start of the round; warp 0 then walks them in ascending order, lane 0 applying the
// events.  Lane 0 stops only at candidates whose prefetched test passes or whose inputs an
// earlier event of the round wrote (the "need" bits, recomputed by the whole warp against
// the shared-memory touched set after every event, for the candidates the sweep has not
// reached yet); every other candidate's test fails in the serial sweep too.
constexpr int kRound = 256;
// precon's rounds are larger: its candidates are many (every close pair), its events few, and
// a round's fixed cost (the prefetch's chain of dependent loads) is paid once per round
constexpr int kReconRound = 512;
constexpr int kReconWords = kReconRound / 32;
constexpr int kExtraHeap = 1024;  // pending extra slots of the premove sweep held in shared memory
constexpr int kRoundWords = kRound / 32;
using RoundTouched = SlotSet<11, 1024>;

// first candidate above pos whose bit is set in a | b (words of 32), or n
__device__ __forceinline__ int next_marked(const unsigned *a, const unsigned *b, int pos, int n) {
  for (int l = pos + 1; l < n;) {
    const int wd = l >> 5;
    const unsigned bits = (a[wd] | b[wd]) & (~0u << (l & 31));
    if (bits) {
      const int r = (wd << 5) + __ffs(bits) - 1;
      return r < n ? r : n;
    }
    l = (wd + 1) << 5;
  }
  return n;
}

// Slot -> index of a candidate of the current round that reads that slot's links (one
// entry per slot a candidate reads; duplicates allowed), so that an event can mark exactly
// the candidates it affects.  Built by the whole block at the start of a round.
constexpr int kMapBits = 11;
constexpr int kMapCap = 1 << kMapBits;  // up to 4 entries per candidate at half load
struct CandMap {
  int *key;
  int *idx;
  __device__ static int home(int g) { return (int)(((unsigned)g * 0x9E3779B1u) >> (32 - kMapBits)); }
  __device__ void insert(int g, int q) const {
    if (g <= 0) return;
    for (int h = home(g);; h = (h + 1) & (kMapCap - 1)) {
      if (atomicCAS(&key[h], 0, g) == 0) {
        idx[h] = q;
        return;
      }
    }
  }
  // set the need bit of every candidate q > bound recorded under slot g
  __device__ void mark(int g, int bound, unsigned *need) const {
    if (g <= 0) return;
    for (int h = home(g);; h = (h + 1) & (kMapCap - 1)) {
      const int k = key[h];
      if (k == 0) return;
      if (k == g) {
        const int q = idx[h];
        if (q > bound) need[q >> 5] |= 1u << (q & 31);
      }
    }
  }
};

struct ReconRec {
  int i, yes, pari, j, parjb, nj, a1, a2, a3, b2;
};

__global__ void __launch_bounds__(kReconRound) k_recon_sweep(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys,
                                                        State S, const int *__restrict__ pos_a,
                                                        const int *__restrict__ list_a, unsigned *err, DevEvent *ev,
                                                        int *ev_count, int ev_cap) {
  __shared__ int tkeys[RoundTouched::kCap];
  __shared__ int mkey[kMapCap], midx[kMapCap];
  __shared__ DevEvent ebuf[kEventStage];
  __shared__ ReconRec rec[kReconRound];
  __shared__ unsigned ymask[kReconWords], nmask[kReconWords];
  __shared__ int s_used;
  const int s = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  if (!recon_step(sc, dyn[s]) || walled(sc)) return;
  const int base = sc.base;
  for (int q = tid; q < RoundTouched::kCap; q += kReconRound) tkeys[q] = 0;
  for (int q = tid; q < kMapCap; q += kReconRound) mkey[q] = 0;
  RoundTouched tc{tkeys, 0, 0, base};
  const CandMap map{mkey, midx};
  EventStage es{ebuf, 0, ev, ev_count, ev_cap};
  const int li = pos_a[base], le = pos_a[base + sc.cap + 1];
  Tally d = Tally::of(dyn[s], base);  // thread 0 applies the events
  const double half_delta = sc.delta / 2.;
  __syncthreads();
  for (int c0 = li; c0 < le; c0 += kReconRound) {
    const int n = min(kReconRound, le - c0);
    ReconRec r{0, -1, 0, 0, 0, 0, 0, 0, 0, 0};
    if (tid < n) {
      const int i = list_a[c0 + tid];
      const ReconIn in = recon_decide(S, i, half_delta, S.cl[i]);
      if (in.yes >= 0) margin_note(dyn[s], 3, in.dot_val, 0.9);
      r.i = i;
      r.yes = in.yes;
      r.pari = in.pari;
      r.j = in.j;
      r.parjb = in.parjb;
      r.nj = in.nj;
      if (in.yes == 1) {  // the links the two loop_killer walks follow
        r.a1 = S.nxt[in.pari];
        r.b2 = S.nxt[in.nj];
        r.a2 = S.nxt[r.a1];
        r.a3 = S.nxt[r.a2];
      }
      // the decision reads the links of i and j
      map.insert(i, tid);
      if (in.j != i) map.insert(in.j, tid);
    }
    rec[tid] = r;
    const unsigned yb = __ballot_sync(0xffffffffu, r.yes == 1);
    if (lane == 0) {
      ymask[wid] = yb;
      nmask[wid] = 0;
    }
    __syncthreads();
    if (tid == 0) {
      int bound = -1;
      auto on_clear = [&](int g) { map.mark(g, bound, nmask); };
      for (int pos = -1;;) {
        const int l = next_marked(ymask, nmask, pos, n);
        if (l >= n) break;
        bound = l;
        const ReconRec &c = rec[l];
        int i = c.i, j = c.j, yes = c.yes, pari = c.pari, parjb = c.parjb;
        bool live = (nmask[l >> 5] >> (l & 31)) & 1u;
        if (live) {  // an earlier event of the round wrote the links of i or j
          if (S.nxt[i] == 0) {
            yes = -1;
          } else {
            const ReconIn q = recon_decide(S, i, half_delta, S.cl[i]);
            if (q.yes >= 0) margin_note(dyn[s], 3, q.dot_val, 0.9);
            yes = q.yes;
            pari = q.pari;
            parjb = q.parjb;
          }
        }
        if (yes == 1) {
          live = live || tc.has(pari) || tc.has(c.a1) || tc.has(c.a2) || tc.has(c.nj);
          d.recon++;
          es.add(d, s, NV_EV_RECON, i, j);
          S.nxt[parjb] = pari;
          S.prv[pari] = parjb;
          S.nxt[i] = j;
          S.prv[j] = i;
          tc.add(i);
          tc.add(j);
          tc.add(pari);
          tc.add(parjb);
          map.mark(i, l, nmask);
          map.mark(j, l, nmask);
          map.mark(pari, l, nmask);
          map.mark(parjb, l, nmask);
          if (live) {
            loop_killer_stage(S, d, s, pari, d.pcount, es, tc, on_clear);
            loop_killer_stage(S, d, s, i, d.pcount, es, tc, on_clear);
          } else {
            const int key[7] = {parjb, i, pari, c.a1, c.a2, j, c.nj};
            const int val[7] = {pari, j, c.a1, c.a2, c.a3, c.nj, c.b2};
            bool killed = false;
            if (loop_count(S, pari, d.pcount, key, val) < 4) {
              loop_killer_stage(S, d, s, pari, d.pcount, es, tc, on_clear);
              killed = true;
            }
            if (killed || loop_count(S, i, d.pcount, key, val) < 4)
              loop_killer_stage(S, d, s, i, d.pcount, es, tc, on_clear);
          }
        }
        pos = l;
      }
      if (es.n) es.spill();
      s_used = tc.n | tc.full;
      tc.n = 0;
      tc.full = 0;
      __threadfence_block();  // the round's writes are visible to the next round's loads
    }
    __syncthreads();
    if (s_used)
      for (int q = tid; q < RoundTouched::kCap; q += kReconRound) tkeys[q] = 0;
    for (int q = tid; q < kMapCap; q += kReconRound) mkey[q] = 0;
    __syncthreads();
  }
  if (tid == 0) {
    d.store(dyn[s]);
    dyn[s].diag[3] = le - li;
  }
}


// ---- premove sweep ---------------------------------------------------------------------------
// line.f90:107-129 in ascending slot order, by rounds.  A candidate's test reads infront(i),
// infront(infront(i)) and their positions; it is taken again on the live state when an
// event of the round wrote i's or infront's infront link (or cleared them).  A removal at i
// changes the test of p = behind(i); when p > i and p is not a candidate it is visited
// later as an extra slot, in slot order between the candidates (a min-heap in shared
// memory, the two-level bitmap past it).
struct RemoveRec {
  int i, inf, yes, tinf, c1, c2, pv, pcand;
};

__global__ void __launch_bounds__(kRound) k_remove_sweep(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys,
                                                         State S, const int *__restrict__ pos_a,
                                                         const int *__restrict__ list_a, const int *__restrict__ cand,
                                                         Sweep sw, unsigned *err, DevEvent *ev, int *ev_count,
                                                         int ev_cap) {
  __shared__ int tkeys[RoundTouched::kCap];
  __shared__ unsigned char tflags[RoundTouched::kCap];
  __shared__ int mkey[kMapCap], midx[kMapCap];
  __shared__ DevEvent ebuf[kEventStage];
  __shared__ RemoveRec rec[kRound];
  __shared__ unsigned ymask[kRoundWords], nmask[kRoundWords];
  __shared__ int heap[kExtraHeap];  // pending extra slots (a min-heap); the bitmap past it
  __shared__ int s_used;
  const int s = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  if (!recon_step(sc, dyn[s]) || walled(sc)) return;
  const int base = sc.base;
  for (int q = tid; q < RoundTouched::kCap; q += kRound) tkeys[q] = 0;
  for (int q = tid; q < kMapCap; q += kRound) mkey[q] = 0;
  // flag 1: the slot's infront link was written (or the slot cleared); flag 2: its behind link
  RoundTouched tc{tkeys, 0, 0, base, tflags};
  const CandMap map{mkey, midx};
  EventStage es{ebuf, 0, ev, ev_count, ev_cap};
  const int li = pos_a[base], le = pos_a[base + sc.cap + 1];
  Tally d = Tally::of(dyn[s], base);  // thread 0 applies the events
  const int lastslot = base + d.pcount;
  const double thr = e_mul(.99, sc.delta);
  const long long T = S.T;
  int last = base;               // thread 0: last slot visited
  int bound = -1;                // thread 0: candidates above this index are not reached yet
  long long n_live = 0, n_extra = 0;  // visits on the live state: candidates, extra slots
  int hsize = 0, bm_extras = 0;  // pending extras in the heap / in the bitmap (heap full)
  int popped = 0;                // last extra taken from the heap (a duplicate pops next to it)
  auto push_extra = [&](int p) {
    if (hsize < kExtraHeap) {
      int c = hsize++;
      while (c > 0) {
        const int par = (c - 1) >> 1;
        if (heap[par] <= p) break;
        heap[c] = heap[par];
        c = par;
      }
      heap[c] = p;
    } else {
      sw.mark(p);
      ++bm_extras;
    }
  };
  auto pop_heap = [&]() {
    const int v = heap[--hsize];
    int c = 0;
    for (;;) {
      int ch = 2 * c + 1;
      if (ch >= hsize) break;
      if (ch + 1 < hsize && heap[ch + 1] < heap[ch]) ++ch;
      if (heap[ch] >= v) break;
      heap[c] = heap[ch];
      c = ch;
    }
    if (hsize > 0) heap[c] = v;
  };
  // lowest pending extra slot in (last, upto], taken off the pending set, or INT_MAX
  auto take_extra = [&](int upto) -> int {
    for (;;) {
      int e = INT_MAX;
      bool from_heap = false;
      if (hsize > 0 && heap[0] <= upto) {
        e = heap[0];
        from_heap = true;
      }
      if (bm_extras > 0) {
        const int b2 = sw.next(last + 1, min(upto, e == INT_MAX ? upto : e - 1));
        if (b2 != INT_MAX) {
          sw.unmark(b2);
          --bm_extras;
          return b2;
        }
      }
      if (!from_heap) return INT_MAX;
      pop_heap();
      if (e == popped) continue;  // the same slot marked twice
      popped = e;
      return e;
    }
  };
  auto on_clear = [&](int g) { map.mark(g, bound, nmask); };
  // one visit of slot i on the live state (thread 0)
  auto visit = [&](int i) {
    if (S.nxt[i] == 0) return;
    const int infront = S.nxt[i];
    const int tinfront = S.nxt[infront];
    double xi[3], xt[3];
    load3(S.X, T, i, xi);
    load3(S.X, T, tinfront, xt);
    const double dii = dist_gen(xi, xt);
    margin_note(dyn[s], 1, dii, thr);
    if (!(dii < thr)) return;
    S.prv[tinfront] = i;
    S.nxt[i] = tinfront;
    tc.add(i, 1u);
    tc.add(infront, 3u);
    tc.add(tinfront, 2u);
    map.mark(i, bound, nmask);
    map.mark(infront, bound, nmask);
    clear_particle(S, infront);
    es.add(d, s, NV_EV_REMOVE, i, infront);
    loop_killer_stage(S, d, s, i, d.pcount, es, tc, on_clear);
    d.remove++;
    const int p = S.prv[i];
    if (p > i && p <= lastslot && !cand[p]) push_extra(p);
  };
  // a removal decided on the prefetched links (i, infront and the walk's links untouched)
  auto remove_fast = [&](const RemoveRec &c) {
    const int i = c.i, infront = c.inf, tinfront = c.tinf;
    int p = c.pv, pc = c.pcand;
    if (tc.has(i, 2u)) {  // an earlier event of the round wrote i's behind link
      p = S.prv[i];
      pc = p > i && p <= lastslot ? cand[p] : 1;
    }
    S.prv[tinfront] = i;
    S.nxt[i] = tinfront;
    tc.add(i, 1u);
    tc.add(infront, 3u);
    tc.add(tinfront, 2u);
    map.mark(i, bound, nmask);
    map.mark(infront, bound, nmask);
    clear_particle(S, infront);
    es.add(d, s, NV_EV_REMOVE, i, infront);
    const int key[4] = {i, infront, tinfront, c.c1};  // infront is cleared: no infront link
    const int val[4] = {tinfront, 0, c.c1, c.c2};
    if (loop_count(S, i, d.pcount, key, val) < 4) {
      loop_killer_stage(S, d, s, i, d.pcount, es, tc, on_clear);
      p = S.prv[i];
      pc = p > i && p <= lastslot ? cand[p] : 1;
    }
    d.remove++;
    if (p > i && p <= lastslot && !pc) push_extra(p);
  };
  __syncthreads();
  for (int c0 = li; c0 < le; c0 += kRound) {
    const int n = min(kRound, le - c0);
    RemoveRec r{0, 0, 0, 0, 0, 0, 0, 1};
    if (tid < n) {
      r.i = list_a[c0 + tid];
      r.inf = S.nxt[r.i];
      if (r.inf) {
        r.tinf = S.nxt[r.inf];
        double xi[3], xt[3];
        load3(S.X, T, r.i, xi);
        load3(S.X, T, r.tinf, xt);
        const double dii = dist_gen(xi, xt);
        margin_note(dyn[s], 1, dii, thr);
        r.yes = dii < thr;
        if (r.yes) {
          r.pv = S.prv[r.i];
          r.c1 = S.nxt[r.tinf];
          if (r.pv > r.i && r.pv <= lastslot) r.pcand = cand[r.pv];
          r.c2 = S.nxt[r.c1];
        }
      }
      // the test reads the infront links of i and infront(i)
      map.insert(r.i, tid);
      if (r.inf != r.i) map.insert(r.inf, tid);
    }
    rec[tid] = r;
    const unsigned yb = __ballot_sync(0xffffffffu, r.yes != 0);
    if (lane == 0) {
      ymask[wid] = yb;
      nmask[wid] = 0;
    }
    __syncthreads();
    if (tid == 0) {
      for (int pos = -1;;) {
        const int l = next_marked(ymask, nmask, pos, n);
        // the sweep position of the next candidate; past the round: the next round's first
        const int kl = l < n ? rec[l].i : c0 + n < le ? list_a[c0 + n] : lastslot + 1;
        const int e = hsize > 0 || bm_extras > 0 ? take_extra(min(kl - 1, lastslot)) : INT_MAX;
        if (e != INT_MAX) {  // an extra slot below the next candidate
          last = e;
          bound = pos;
          ++n_extra;
          visit(e);
          continue;
        }
        if (l >= n) break;
        last = kl;
        bound = l;
        const RemoveRec &c = rec[l];
        if (((nmask[l >> 5] >> (l & 31)) & 1u) || tc.has(c.tinf, 1u) || tc.has(c.c1, 1u)) {
          ++n_live;  // an earlier event wrote links the test or the loop_killer walk reads
          visit(kl);
        } else {
          remove_fast(c);
        }
        pos = l;
      }
      if (es.n) es.spill();
      s_used = tc.n | tc.full;
      tc.n = 0;
      tc.full = 0;
      __threadfence_block();
    }
    __syncthreads();
    if (s_used)
      for (int q = tid; q < RoundTouched::kCap; q += kRound) tkeys[q] = 0;
    for (int q = tid; q < kMapCap; q += kRound) mkey[q] = 0;
    __syncthreads();
  }
  if (tid == 0) {
    // extra slots above the last candidate
    bound = kRound;
    for (;;) {
      const int e = take_extra(lastslot);
      if (e == INT_MAX) break;
      last = e;
      ++n_extra;
      visit(e);
    }
    if (es.n) es.spill();
    d.store(dyn[s]);
    dyn[s].diag[4] = le - li;
    dyn[s].diag[7] = (n_extra << 32) | n_live;
  }
}

// ---- pinsert sweep, warp-prefetched --------------------------------------------------------
// The reference's serial sweep (line.f90:30-93), used for a system whose step has an
// insertion the parallel form cannot place: a new point put in a free slot that the sweep
// reaches later and that inserts again.  Candidates (the slots whose stale or fresh test
// passes) are taken 32 at a time; each lane decides its candidate on the state at the start
// of the chunk and precomputes the new point, its velocity and the neighbour positions the
// ghost refreshes need.  Lane 0 then applies the insertions in slot order.  What an
// insertion writes -- the ghosts and links of i, infront(i) and the new point -- is mirrored
// in a shared-memory table, so a later candidate of the same chunk whose slot or infront
// slot was written reads its current ghosts and links from there instead of global memory.
// New points that the sweep still reaches (free slots above their creator, up to the
// step-start pcount) are visited as extra slots through the two-level bitmap, on the live
// state; so are chunks whose table fills up.
struct InsIn {
  int k, nx, pk, nn, yes;
  double x[3], gi[3], gb[3], xn[3], un[3], xnx[3], xpk[3], xnn[3];
};

__device__ InsIn ins_prefetch(const SysConst &sc, const State &S, int k) {
  InsIn r;
  r.k = k;
  r.yes = 0;
  r.nx = S.nxt[k];
  if (r.nx == 0) return r;
  const long long T = S.T;
  load3(S.X, T, k, r.x);
  load3(S.GI, T, k, r.gi);
  load3(S.GB, T, k, r.gb);
  r.pk = S.prv[k];
  r.nn = S.nxt[r.nx];
  load3(S.X, T, r.nx, r.xnx);
  load3(S.X, T, r.pk, r.xpk);
  load3(S.X, T, r.nn, r.xnn);
  double uk[3], unx[3];
  load3(S.U, T, k, uk);
  load3(S.U, T, r.nx, unx);
  for (int c = 0; c < 3; ++c) r.un[c] = e_mul(0.5, e_add(uk[c], unx[c]));
  const double disti = dist_gen(r.x, r.gi);
  if (disti > sc.delta) {
    r.yes = 1;
    new_point(r.x, r.gi, r.gb, disti, r.xn);
  }
  return r;
}

// the table of written slots: ghosts and links as they now stand in global memory
struct InsTable {
  static constexpr int kBits = 9;
  static constexpr int kLimit = 240;
  using Set = SlotSet<kBits, kLimit>;
  double *gi, *gb;  // [kCap][3]
  int *nxt, *prv;
};

__global__ void __launch_bounds__(32) k_insert_sweep(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, State S,
                                                     const int *__restrict__ pos_a, const int *__restrict__ list_a,
                                                     const int *__restrict__ pos_b, const int *__restrict__ list_b,
                                                     Sweep sw, unsigned *err, DevEvent *ev, int *ev_count,
                                                     int ev_cap) {
  using Set = InsTable::Set;
  __shared__ int tkeys[Set::kCap];
  __shared__ double tgi[Set::kCap * 3], tgb[Set::kCap * 3];
  __shared__ int tnxt[Set::kCap], tprv[Set::kCap];
  __shared__ int fslot[32];
  __shared__ DevEvent ebuf[kEventStage];
  const int s = blockIdx.x;
  const int lane = threadIdx.x;
  if (s >= nsys || *err) return;
  const SysConst &sc = scs[s];
  if (!dyn[s].ins_fallback || walled(sc)) return;
  const int base = sc.base;
  for (int q = lane; q < Set::kCap; q += 32) tkeys[q] = 0;
  Set tc{tkeys, 0, 0, base};
  EventStage es{ebuf, 0, ev, ev_count, ev_cap};
  Tally d = Tally::of(dyn[s], base);  // lane 0's copy is the live one
  const int old_last = base + d.pcount;  // loop bound old_pcount (line.f90:28-30)
  const int li = pos_a[base], le = pos_a[base + sc.cap + 1];
  const int ee = pos_b[base + sc.cap + 1];
  const long long T = S.T;
  int ei = pos_b[base], pc = d.pcount, extras = 0, last = base, fs0 = 0;
  bool stop = false;
  __syncwarp();

  // mirror of slot g's ghosts and links (lane 0)
  auto put = [&](int g, const double gi[3], const double gb[3], int nx, int pv) {
    const int h = tc.add(g);
    if (h < 0) return;
    for (int c = 0; c < 3; ++c) {
      tgi[3 * h + c] = gi[c];
      tgb[3 * h + c] = gb[c];
    }
    tnxt[h] = nx;
    tprv[h] = pv;
  };
  // the next free slot (line.f90:36-50): the step-start free slots in ascending order, then
  // pcount + 1
  auto take_slot = [&](int &slot) -> bool {
    if (ei < ee) {
      const int q = ei - fs0;
      slot = (q >= 0 && q < 32) ? fslot[q] : list_b[ei];
      ++ei;
      return true;
    }
    if (pc + 1 > sc.cap) {
      atomicOr(err, DERR_CAPACITY);
      return false;
    }
    slot = base + (++pc);
    return true;
  };
  auto after_insert = [&](int i, int p) {
    es.add(d, s, NV_EV_INSERT, i, p);
    d.insert++;
    if (p > i && p <= old_last) {  // the sweep reaches the new point later
      sw.mark(p);
      ++extras;
    }
  };
  // one visit of slot i on the live state: the reference's statements in order (lane 0)
  auto visit_live = [&](int i) -> bool {
    const int nx = S.nxt[i];
    if (nx == 0) return true;
    double x[3], gi[3], gb[3];
    load3(S.X, T, i, x);
    load3(S.GI, T, i, gi);
    load3(S.GB, T, i, gb);
    const double disti = dist_gen(x, gi);
    S.seglen[i] = disti;
    if (!(disti > sc.delta)) return true;
    int p;
    if (!take_slot(p)) return false;
    double xn[3], ui[3], un[3];
    const double zero[3] = {0, 0, 0};
    new_point(x, gi, gb, disti, xn);
    load3(S.U, T, i, ui);
    load3(S.U, T, nx, un);
    for (int c = 0; c < 3; ++c) un[c] = e_mul(0.5, e_add(ui[c], un[c]));
    store3(S.X, T, p, xn);
    store3(S.U, T, p, un);
    store3(S.U1, T, p, zero);
    store3(S.U2, T, p, zero);
    S.prv[p] = i;
    S.nxt[p] = nx;
    double a[3], b[3];
    get_ghost_p(sc, S, p, a, b);
    store3(S.GI, T, p, a);
    store3(S.GB, T, p, b);
    put(p, a, b, nx, i);
    S.prv[nx] = p;
    get_ghost_p(sc, S, nx, a, b);
    store3(S.GI, T, nx, a);
    store3(S.GB, T, nx, b);
    put(nx, a, b, S.nxt[nx], p);
    S.nxt[i] = p;
    get_ghost_p(sc, S, i, a, b);
    store3(S.GI, T, i, a);
    store3(S.GB, T, i, b);
    put(i, a, b, p, S.prv[i]);
    after_insert(i, p);
    return true;
  };
  auto run_extras = [&](int upto) -> bool {  // extra slots in (last, upto]
    while (extras > 0) {
      const int e = sw.next(last + 1, upto);
      if (e == INT_MAX) break;
      sw.unmark(e);
      --extras;
      last = e;
      if (!visit_live(e)) return false;
    }
    return true;
  };

  for (int k0 = li; k0 < le; k0 += 32) {
    const int k = k0 + lane;
    InsIn in;
    in.k = 0;
    in.yes = 0;
    in.nx = 0;
    if (k < le) in = ins_prefetch(sc, S, list_a[k]);
    fs0 = __shfl_sync(0xffffffffu, ei, 0);
    if (fs0 + lane < ee) fslot[lane] = list_b[fs0 + lane];
    __syncwarp();
    const int n = min(32, le - k0);
    for (int l = 0; l < n; ++l) {
      // lane 0 takes candidate l from its lane (shuffles, all lanes take part)
      const int kl = __shfl_sync(0xffffffffu, in.k, l);
      const int nx = __shfl_sync(0xffffffffu, in.nx, l);
      const int pk = __shfl_sync(0xffffffffu, in.pk, l);
      const int nn = __shfl_sync(0xffffffffu, in.nn, l);
      int yes = __shfl_sync(0xffffffffu, in.yes, l);
      double x[3], gi[3], gb[3], xn[3], un[3], xnx[3], xpk[3], xnn[3];
      for (int c = 0; c < 3; ++c) {
        x[c] = __shfl_sync(0xffffffffu, in.x[c], l);
        gi[c] = __shfl_sync(0xffffffffu, in.gi[c], l);
        gb[c] = __shfl_sync(0xffffffffu, in.gb[c], l);
        xn[c] = __shfl_sync(0xffffffffu, in.xn[c], l);
        un[c] = __shfl_sync(0xffffffffu, in.un[c], l);
        xnx[c] = __shfl_sync(0xffffffffu, in.xnx[c], l);
        xpk[c] = __shfl_sync(0xffffffffu, in.xpk[c], l);
        xnn[c] = __shfl_sync(0xffffffffu, in.xnn[c], l);
      }
      if (lane != 0 || stop) continue;
      if (kl > old_last) {
        stop = true;
        continue;
      }
      if (!run_extras(kl - 1)) {
        stop = true;
        continue;
      }
      last = kl;
      if (nx == 0) continue;  // free at the chunk start; pinsert frees nothing
      const int hk = tc.full ? -1 : tc.find(kl);
      const int hx = tc.full ? -1 : tc.find(nx);
      if (tc.full || nx == kl || (hk >= 0 && tnxt[hk] != nx)) {
        if (!visit_live(kl)) stop = true;
        continue;
      }
      int pv = pk;
      if (hk >= 0) {  // written earlier in this chunk: its ghosts and behind link from the table
        for (int c = 0; c < 3; ++c) {
          gi[c] = tgi[3 * hk + c];
          gb[c] = tgb[3 * hk + c];
        }
        pv = tprv[hk];
        const double disti = dist_gen(x, gi);
        yes = disti > sc.delta;
        if (yes) new_point(x, gi, gb, disti, xn);
      }
      if (!yes) continue;
      int p;
      if (!take_slot(p)) {
        stop = true;
        continue;
      }
      // the three ghost refreshes of line.f90:86-91 from known positions
      double gip[3], gbp[3], gix[3], gbx[3], gik[3], gbk[3];
      ghost_of(sc, xn, xnx, gip);
      ghost_of(sc, xn, x, gbp);
      int nnx = nn;
      if (hx >= 0) {
        for (int c = 0; c < 3; ++c) gix[c] = tgi[3 * hx + c];
        nnx = tnxt[hx];
      } else {
        ghost_of(sc, xnx, xnn, gix);
      }
      ghost_of(sc, xnx, xn, gbx);
      ghost_of(sc, x, xn, gik);
      if (hk >= 0) {
        for (int c = 0; c < 3; ++c) gbk[c] = gb[c];
      } else {
        ghost_of(sc, x, xpk, gbk);
      }
      const double zero[3] = {0, 0, 0};
      store3(S.X, T, p, xn);
      store3(S.U, T, p, un);
      store3(S.U1, T, p, zero);
      store3(S.U2, T, p, zero);
      S.prv[p] = kl;
      S.nxt[p] = nx;
      store3(S.GI, T, p, gip);
      store3(S.GB, T, p, gbp);
      S.prv[nx] = p;
      store3(S.GI, T, nx, gix);
      store3(S.GB, T, nx, gbx);
      S.nxt[kl] = p;
      store3(S.GI, T, kl, gik);
      store3(S.GB, T, kl, gbk);
      put(p, gip, gbp, nx, kl);
      put(nx, gix, gbx, nnx, p);
      put(kl, gik, gbk, p, pv);
      after_insert(kl, p);
    }
    stop = __shfl_sync(0xffffffffu, stop, 0);
    // the chunk's writes are now visible to the next chunk's prefetch
    __threadfence_block();
    tc.reset(lane);
    flush_events(es, lane);
    if (stop) break;
  }
  if (lane == 0 && !stop) run_extras(old_last);
  flush_events(es, lane);
  if (lane == 0) {
    d.store(dyn[s]);
    dyn[s].pcount = pc;
    dyn[s].diag[2] += 1;
  }
}

State make_state(nv_handle *h) {
  return State{h->x,  h->u,       h->u1, h->u2, h->gi, h->gb, h->closestd, h->nxt, h->prv, h->closest, h->T,
               h->topo->seglen};
}

void compact(nv_handle *h, int *flag, int *pos, int *list) {
  TopoBuffers *tb = h->topo;
  size_t bytes = tb->cub_bytes;
  cub::DeviceScan::ExclusiveSum(tb->cub_tmp, bytes, flag, pos, (int)(h->T + 1), h->stream);
  k_scatter<<<grid_for(h->T, TB), TB, 0, h->stream>>>(flag, pos, list, h->T);
}


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
  cudaMalloc(&tb->unew, 3 * n * sizeof(double));
  cudaMalloc(&tb->segnx, n * sizeof(int));
  cudaMalloc(&tb->fh[0], n * sizeof(int));
  cudaMalloc(&tb->fh[1], n * sizeof(int));
  cudaMalloc(&tb->pos_h, n * sizeof(int));
  cudaMalloc(&tb->l0, (n / 32 + 2) * sizeof(unsigned));
  cudaMalloc(&tb->l1, (n / 1024 + 2) * sizeof(unsigned));
  cudaMalloc(&tb->len_st, n * sizeof(double));
  cudaMalloc(&tb->len_fr, n * sizeof(double));
  cudaMalloc(&tb->seglen, n * sizeof(double));
  cudaMalloc(&tb->dn_new, n * sizeof(double));
  cudaMemset(tb->seglen, 0, n * sizeof(double));
  {
    int maxcap = 1;
    for (int s = 0; s < h->nsys; ++s) maxcap = std::max(maxcap, h->cap[s]);
    tb->total_parts = std::min(64, (maxcap + 16383) / 16384);
    cudaMalloc(&tb->psum, (size_t)h->nsys * tb->total_parts * sizeof(double));
    cudaMalloc(&tb->pnear, (size_t)h->nsys * tb->total_parts * sizeof(double));
  }
  // cell grids of the systems without a tree: about two slots per cell at full capacity,
  // cells at least as wide as delta/2 and at most 256 per axis
  std::vector<CellGrid> grids(h->nsys);
  long long cells = 0;
  for (int s = 0; s < h->nsys; ++s) {
    CellGrid &G = grids[s];
    std::memset(&G, 0, sizeof G);
    const SysConst &sc = h->sc[s];
    if (sc.use_tree) continue;
    const double vol = sc.box[0] * sc.box[1] * sc.box[2];
    const double w = std::max(std::cbrt(vol * 2.0 / std::max(h->cap[s], 1)), 0.5 * sc.delta);
    G.wmin = 1e300;
    for (int a = 0; a < 3; ++a) {
      G.nc[a] = (int)std::min(256.0, std::max(1.0, std::floor(sc.box[a] / w)));
      G.inv_w[a] = G.nc[a] / sc.box[a];
      G.half[a] = sc.box[a] / 2;
      G.wmin = std::min(G.wmin, sc.box[a] / G.nc[a]);
    }
    G.base = cells;
    cells += (long long)G.nc[0] * G.nc[1] * G.nc[2];
  }
  tb->n_cells = cells;
  tb->any_cells = cells > 0 && cells < (1LL << 30);
  size_t scan_n = n;
  if (tb->any_cells) {
    cudaMalloc(&tb->grid, h->nsys * sizeof(CellGrid));
    cudaMemcpy(tb->grid, grids.data(), h->nsys * sizeof(CellGrid), cudaMemcpyHostToDevice);
    cudaMalloc(&tb->cell_of, n * sizeof(int));
    cudaMalloc(&tb->cell_cnt, (cells + 1) * sizeof(int));
    cudaMalloc(&tb->cell_start, (cells + 1) * sizeof(int));
    cudaMalloc(&tb->cell_items, n * sizeof(int));
    scan_n = std::max(scan_n, (size_t)cells + 1);
  }
  cub::DeviceScan::ExclusiveSum(nullptr, tb->cub_bytes, tb->flag_a, tb->pos_a, (int)scan_n);
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
  cudaFree(tb->unew); cudaFree(tb->segnx); cudaFree(tb->fh[0]); cudaFree(tb->fh[1]); cudaFree(tb->pos_h);
  cudaFree(tb->l0); cudaFree(tb->l1);
  cudaFree(tb->len_st); cudaFree(tb->len_fr); cudaFree(tb->seglen); cudaFree(tb->dn_new);
  cudaFree(tb->psum); cudaFree(tb->pnear);
  cudaFree(tb->grid); cudaFree(tb->cell_of); cudaFree(tb->cell_cnt); cudaFree(tb->cell_start);
  cudaFree(tb->cell_items);
  cudaFree(tb->cub_tmp);
  delete tb;
  h->topo = nullptr;
}

void launch_pinsert(nv_handle *h) {
  ++h->links_epoch;
  TopoBuffers *tb = h->topo;
  const long long T = h->T;
  k_ins_begin<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(h->d_dyn, h->nsys);
  k_ins_mark<<<grid_for(T + 1, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->gi, h->nxt,
                                                         tb->flag_a, tb->flag_b, tb->dec, tb->len_st, tb->len_fr, T,
                                                         h->d_err);
  compact(h, tb->flag_a, tb->pos_a, tb->list_a);  // candidates (either test passes)
  compact(h, tb->flag_b, tb->pos_b, tb->list_b);  // free slots
  k_zero_flags<<<grid_for(T + 1, TB), TB, 0, h->stream>>>(tb->flag_c, T);
  const int *ncand = tb->pos_a + T;
  k_ins_decide_easy<<<grid_for(T, 128), 128, 0, h->stream>>>(tb->list_a, ncand, tb->dec, tb->flag_c, h->d_err);
  compact(h, tb->flag_c, tb->pos_c, tb->list_c);  // ambiguous slots
  k_ins_decide_amb<<<grid_for(T, 128), 128, 0, h->stream>>>(tb->list_c, tb->pos_c + T, h->nxt, h->prv, tb->flag_c,
                                                            tb->dec, h->d_err);
  k_zero_flags<<<grid_for(T + 1, TB), TB, 0, h->stream>>>(tb->flag_c, T);
  k_ins_decide_case<<<grid_for(T, 128), 128, 0, h->stream>>>(tb->list_a, ncand, h->prv, tb->dec, tb->flag_c,
                                                             h->d_err);
  compact(h, tb->flag_c, tb->pos_c, tb->list_c);  // insertions, in sweep order
  k_ins_len<<<grid_for(T, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->nxt, h->prv, tb->dec, tb->len_st,
                                                   tb->len_fr, tb->seglen, T);
  const State S = make_state(h);
  // the number of insertions (pos_c[T]) is known only on the device: launch over every
  // slot, threads beyond the count return at once
  const int grid = grid_for(T, 128);
  const int *nev = tb->pos_c + T;
  const int iters = h->ins_iters;
  k_zero_flags<<<grid_for(T + 1, TB), TB, 0, h->stream>>>(tb->fh[0], T);
  if (iters == 0) {
    k_ins_all_serial<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(h->d_dyn, h->nsys);
    size_t bytes = tb->cub_bytes;
    cub::DeviceScan::ExclusiveSum(tb->cub_tmp, bytes, tb->fh[0], tb->pos_h, (int)(T + 1), h->stream);
  }
  for (int it = 0; it < iters; ++it) {
    int *fin = tb->fh[it & 1], *fout = tb->fh[(it + 1) & 1];
    k_ins_zero_open<<<grid_for(T, TB), TB, 0, h->stream>>>(h->d_dyn, h->sys_of, fout, T);
    size_t bytes = tb->cub_bytes;
    cub::DeviceScan::ExclusiveSum(tb->cub_tmp, bytes, fin, tb->pos_h, (int)(T + 1), h->stream);
    k_ins_chain<<<grid, 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, S, tb->pos_c, tb->list_c, tb->pos_b,
                                             tb->list_b, tb->dec, tb->pos_h, fout, tb->newslot, tb->segnx, tb->xnew,
                                             tb->unew, tb->dn_new, nev, h->d_err);
    k_ins_compare<<<grid_for(T, TB), TB, 0, h->stream>>>(h->d_dyn, h->sys_of, fin, fout, T);
    k_ins_converge<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(h->d_dyn, h->nsys, it + 1, it + 1 == iters);
  }
  const int *fh = tb->fh[iters > 0 ? (iters - 1) & 1 : 0];  // pos_h is its prefix sum
  k_ins_apply<<<grid, 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, S, tb->pos_c, tb->list_c, tb->pos_h, fh,
                                           tb->newslot, tb->segnx, tb->xnew, tb->unew, tb->dn_new, nev, h->d_events,
                                           h->d_event_count, h->event_cap, h->d_err);
  k_ins_ghosts<<<grid, 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, S, tb->list_c, fh, tb->newslot, nev,
                                            h->d_err);
  k_ins_finish<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, tb->pos_a, tb->pos_c,
                                                              tb->pos_h, tb->pos_b, h->d_err);
  // systems with an insertion the parallel form cannot place: the sweep (extra visits start
  // empty: bitmaps from an all-zero flag array; flag_b is free once the free slots are listed)
  k_zero_flags<<<grid_for(T + 1, TB), TB, 0, h->stream>>>(tb->flag_b, T);
  const Sweep sw = make_sweep(h, tb->flag_b);
  k_insert_sweep<<<h->nsys, 32, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, S, tb->pos_a, tb->list_a, tb->pos_b,
                                                tb->list_b, sw, h->d_err, h->d_events, h->d_event_count,
                                                h->event_cap);
  k_ins_part<<<h->nsys * tb->total_parts, kTotalThreads, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, tb->total_parts,
                                                                         tb->seglen, tb->psum, tb->pnear, h->d_err);
  k_ins_total<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, tb->total_parts, tb->psum,
                                                             tb->pnear, h->d_err);
  launch_solid_pinsert(h);
}

void launch_pclose(nv_handle *h, bool only_brute) {
  bool any_brute = false, any_tree = false;
  for (auto &s : h->sc) (s.use_tree ? any_tree : any_brute) = true;
  TopoBuffers *tb = h->topo;
  if (any_brute && (h->pclose_method == 1 || !tb->any_cells)) {
    k_pclose_brute<<<grid_for(h->T, 128), 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->nxt, h->prv,
                                                               h->closest, h->closestd, h->T, h->d_err);
  } else if (any_brute) {
    const long long T = h->T;
    cudaMemsetAsync(tb->cell_cnt, 0, (tb->n_cells + 1) * sizeof(int), h->stream);
    k_cell_count<<<grid_for(T, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, tb->grid, h->x, h->nxt,
                                                        tb->cell_of, tb->cell_cnt, T, h->d_err);
    size_t bytes = tb->cub_bytes;
    cub::DeviceScan::ExclusiveSum(tb->cub_tmp, bytes, tb->cell_cnt, tb->cell_start, (int)(tb->n_cells + 1),
                                  h->stream);
    k_cell_fill<<<grid_for(T, TB), TB, 0, h->stream>>>(tb->cell_of, tb->cell_start, tb->cell_cnt, tb->cell_items, T);
    k_pclose_cells<<<grid_for(T, 128), 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, tb->grid, h->x, h->nxt,
                                                            h->prv, tb->cell_of, tb->cell_start, tb->cell_items,
                                                            h->closest, h->closestd, T);
  }
  if (any_tree && !only_brute) launch_closest_tree(h);
}

void launch_precon(nv_handle *h) {
  ++h->links_epoch;
  TopoBuffers *tb = h->topo;
  k_mark_recon<<<grid_for(h->T + 1, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->closestd, h->nxt,
                                                              tb->flag_a, h->T, h->d_err);
  compact(h, tb->flag_a, tb->pos_a, tb->list_a);
  k_recon_sweep<<<h->nsys, kReconRound, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, make_state(h), tb->pos_a, tb->list_a,
                                               h->d_err, h->d_events, h->d_event_count, h->event_cap);
  launch_solid_precon(h);
}

void launch_premove(nv_handle *h) {
  ++h->links_epoch;
  TopoBuffers *tb = h->topo;
  k_mark_remove<<<grid_for(h->T + 1, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->nxt,
                                                               tb->flag_a, h->T, h->d_err);
  compact(h, tb->flag_a, tb->pos_a, tb->list_a);
  // extra visits start empty: bitmaps from an all-zero flag array
  k_zero_flags<<<grid_for(h->T + 1, TB), TB, 0, h->stream>>>(tb->flag_b, h->T);
  const Sweep sw = make_sweep(h, tb->flag_b);
  k_remove_sweep<<<h->nsys, kRound, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, make_state(h), tb->pos_a, tb->list_a,
                                                tb->flag_a, sw, h->d_err, h->d_events, h->d_event_count,
                                                h->event_cap);
  launch_solid_premove(h);
}
