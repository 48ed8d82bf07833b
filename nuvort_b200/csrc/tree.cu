// tree.cu -- Barnes-Hut octree on the device: build, velocity walk, closest-point walk.
//
// Build (construct_tree/build_tree/new_tree, src/tree.f90:38-157), top-down, one level per
// pass, all systems of the handle at once:
//   * Node k's members are kept as a contiguous list of slots in ascending slot order.
//     Splitting a node is a stable 8-way partition of that list by octant, so every child's
//     list is again in ascending slot order -- the order in which the reference sums a
//     node's centre and circulation (tree.f90:124-143), reproduced exactly.
//   * The octant of a point is decided by the reference's own membership test against the
//     child's corner, computed with the same FP64 additions (child corner = parent corner
//     (+ width/2)); a point that fails its child's upper bound (rounding can make a child's
//     far face differ by an ulp from the parent's) belongs to no child, as in the reference.
//   * Octant digit = 4*[y upper] + 2*[z upper] + [x upper]: the child order fbl, fbr, ftl,
//     ftr, bbl, bbr, btl, btr of tree.f90:71-93.  Only non-empty children are stored;
//     siblings are contiguous, so a preorder walk follows first_child / skip links.
//   * The root holds every slot (pcount includes empty slots, tree.f90:48), its centre is
//     the mean over live slots and its circulation is zero (tree.f90:50-54).
// Walks: one thread per target point, stackless preorder over first_child/skip, with the
// reference's opening test and arithmetic (tree_walk tree.f90:250-316, closest_tree
// :206-244) in the same order, so the accumulated velocity is the reference's bit for bit.
#include <cub/cub.cuh>

#include "handle.cuh"
#include "mixed.cuh"

constexpr int kMaxLevels = NV_TREE_MAX_DEPTH;
constexpr int kEnd = -1;
constexpr int kBigNode = 2048;  // nodes with more members are split by a whole block
constexpr int kBlockSumNode = 8192;  // nodes with more members are summed by a whole block
constexpr int kCtrBig = kMaxLevels + 6;  // ctr[kCtrBig]: entries of the block-summed node list
constexpr int kCtrBigSnap = kMaxLevels + 7;  // entries listed when the early block sums start
constexpr int kSnapLevel = 1;  // the early block sums: the big nodes of depth 1, listed by the root's split
// ctr[kCtrSplit + b]: entries of the level lists of nodes to split, by level % 3 = b:
// [+0..+2] nodes above kBigNode members (split by a block), [+3..+5] the others with >= 2
constexpr int kCtrSplit = kMaxLevels + 8;
constexpr int kCtrSize = kMaxLevels + 16;
constexpr int kDeferCap = 1 << 20;  // deferred root tests listed per velocity pass
constexpr int kFlush = 16;      // FP32 far-field terms summed before promotion to FP64
static_assert((kFlush & (kFlush - 1)) == 0, "the walk tests the flush by a mask");

struct TreeBuffers {
  int max_nodes = 0;
  long long max_members = 0;
  double4 *nA = nullptr;  // cent.xyz, width
  double4 *nB = nullptr;  // circ.xyz, geo_dist
  double4 *nP = nullptr;  // corner posx,posy,posz
  int4 *nI = nullptr;     // pcount, first_child, skip, first_next
  int2 *nR = nullptr;     // member range start, member count
  int *nDepth = nullptr;
  int *nLeaf = nullptr;
  int *nSib = nullptr;    // next sibling, or kEnd for a last child (and roots)
  int *members = nullptr;
  // roots: a parallel estimate of the centre with a bound on its distance to the exact
  // (sequential) one, so the walks need not wait for the exact sum; (target, image) pairs
  // whose root test the bound cannot settle are listed and redone once the exact sum is in
  // the roots' split as one stable radix sort of the live slots by (system, octant)
  unsigned *rkey[2] = {nullptr, nullptr};
  int *rval[2] = {nullptr, nullptr};
  int *root_cnt = nullptr;  // per system: members per octant
  int *root_mb = nullptr;   // per system: first member entry of the children
  void *rsort_tmp = nullptr;
  size_t rsort_bytes = 0;
  int rkey_bits = 0;
  double4 *root_apx = nullptr;  // per system: centre estimate, bound
  double *root_part = nullptr;  // per system and part: partial sums of x, y, z, |x|, |y|, |z|
  int root_parts = 1;
  int2 *defer = nullptr;        // (slot, image) pairs, image -1: the whole target (FP64 walk)
  int *defer_n = nullptr;
  int *bigl = nullptr;    // non-root nodes with more than kBlockSumNode members
  int max_big = 0;
  int *split_blk[3] = {nullptr, nullptr, nullptr};  // nodes of a level split by a block, by level % 3
  int *split_wrp[3] = {nullptr, nullptr, nullptr};  // nodes of a level split by a warp
  int max_blk = 0, max_wrp = 0;
  int *ctr = nullptr;     // [0] n_nodes [1] n_members [2 + L] first node of level L
  int *flag = nullptr, *pos = nullptr;
  void *cub_tmp = nullptr;
  size_t cub_bytes = 0;
  // walk order: each system's slots sorted by Morton code of the position (live slots first)
  unsigned long long *okey[2] = {nullptr, nullptr};
  int *oval[2] = {nullptr, nullptr};
  int *perm = nullptr;  // = oval[1]: position base+q of system s -> slot
  int *iperm = nullptr; // slot -> its position in the walk order (inverse of perm)
  void *sort_tmp = nullptr;
  size_t sort_bytes = 0;
  int key_bits = 0;
  bool built = false;
  MixedNodes mx;
  unsigned prep_epoch = ~0u;  // the handle's links epoch when the mixed records took prv
};

namespace {

constexpr int TB = 256;

__global__ void k_live_flags(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                             const int *__restrict__ sys_of, const int *__restrict__ nxt, int *flag, long long T,
                             int *ctr) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g > T) return;
  int f = 0;
  if (g < T) {
    const int s = sys_of[g];
    const SysConst &sc = scs[s];
    const int k = (int)(g - sc.base);
    f = (sc.use_tree || sc.sched_tree) && k >= 1 && k <= dyn[s].pcount && nxt[g] != 0;
  }
  flag[g] = f;
  if (g == 0)
    for (int b = 0; b < 6; ++b) ctr[kCtrSplit + b] = 0;
}

__global__ void k_scatter_live(const int *__restrict__ flag, const int *__restrict__ pos, int *__restrict__ members,
                               long long T) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < T && flag[g]) members[pos[g]] = (int)g;
}


// Root of every system (construct_tree, tree.f90:38-59).
__global__ void k_roots(const SysConst *__restrict__ scs, SysDyn *dyn, int nsys, const int *__restrict__ nxt,
                        const int *__restrict__ pos, TreeBuffers tb, long long T) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) {
    tb.ctr[0] = nsys;
    tb.ctr[2] = 0;
    tb.ctr[3] = nsys;
    tb.ctr[1] = pos[T];
    tb.ctr[kCtrBig] = 0;
  }
  if (s >= nsys) return;
  const SysConst &sc = scs[s];
  const int pc = (sc.use_tree || sc.sched_tree) ? dyn[s].pcount : 0;
  const double h = -sc.bsize / 2.0;
  tb.nP[s] = make_double4(h, h, h, 0);
  tb.nA[s] = make_double4(0, 0, 0, sc.bsize);
  tb.nB[s] = make_double4(0, 0, 0, 0);
  tb.nI[s] = make_int4(pc, kEnd, kEnd, pc >= 1 ? nxt[sc.base + 1] : 0);
  tb.nR[s] = make_int2(pos[sc.base], pos[sc.base + sc.cap + 1] - pos[sc.base]);
  tb.nDepth[s] = 0;
  tb.nSib[s] = kEnd;
  for (int d = 0; d < 8; ++d) tb.root_cnt[8 * s + d] = 0;
  tb.nLeaf[s] = pc == 1 ? sc.base + 1 : 0;
  dyn[s].tree_eval = 0;
  dyn[s].tree_tests = 0;
  dyn[s].diag[8] = dyn[s].diag[9] = dyn[s].diag[10] = 0;
}

// Sort keys of the walk order: (system, class, Morton code of the position on a 1024^3 grid
// of the box); class 0 is the dummy slot, 1 live slots, 2 the rest.  The order only decides
// which lanes walk together; every target's result is independent of it.
__device__ __forceinline__ unsigned spread3(unsigned v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__global__ void k_order_keys(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                             const int *__restrict__ sys_of, const double *__restrict__ X,
                             const int *__restrict__ nxt, unsigned long long *key, int *val, long long T) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= T) return;
  const int s = sys_of[g];
  const SysConst &sc = scs[s];
  const int k = (int)(g - sc.base);
  unsigned long long inner;
  if (k == 0) {
    inner = 0;
  } else if (k <= dyn[s].pcount && nxt[g] != 0) {
    unsigned q[3];
    for (int c = 0; c < 3; ++c) {
      const double f = (X[c * T + g] / sc.bsize + 0.5) * 1024.0;
      q[c] = f <= 0. ? 0u : f >= 1023. ? 1023u : (unsigned)f;
    }
    inner = (1ull << 32) | (spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2));
  } else {
    inner = (2ull << 32) | (unsigned)k;
  }
  key[g] = ((unsigned long long)s << 34) | inner;
  val[g] = (int)g;
}

__global__ void k_inv_perm(const int *__restrict__ perm, int *__restrict__ iperm, long long T) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < T) iperm[perm[i]] = (int)i;
}

__global__ void k_iota(int *v, long long n) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < n) v[g] = (int)g;
}

// Octant of x in node (corner P, half-width h), or 8 when x lies in no child.
__device__ __forceinline__ int octant(const double x[3], const double4 P, double h) {
  const double p[3] = {P.x, P.y, P.z};
  int up[3];
  bool in = true;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double mid = e_add(p[c], h);  // child corner posx+(width/2)      tree.f90:74
    if (x[c] >= mid) {
      up[c] = 1;
      in = in && (x[c] < e_add(mid, h));  // x < posx+width of the upper child
    } else {
      up[c] = 0;
      in = in && (x[c] >= p[c]);  // lower child: posx <= x < posx+width (= mid)
    }
  }
  return in ? (4 * up[1] + 2 * up[2] + up[0]) : 8;
}

__device__ __forceinline__ double4 ldg4(const double4 *p) {
  const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
  const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ void load_x(const double *__restrict__ X, long long T, int g, double x[3]) {
  x[0] = __ldg(X + g);
  x[1] = __ldg(X + T + g);
  x[2] = __ldg(X + 2 * T + g);
}

// Create the non-empty children of node p (counts cnt[0..7]); returns first child id via
// *id0 and member base via *mb0 (or -1 on overflow).  Called by one thread.
// What a node's split reserves: child ids, member slots, entries of the next level's block
// and warp split lists, entries of the block-summed node list.
struct SplitNeeds {
  int nchild, kept, nblk, nwrp, nbig;
};
__device__ SplitNeeds split_needs(const int cnt[8]) {
  SplitNeeds n{0, 0, 0, 0, 0};
#pragma unroll
  for (int d = 0; d < 8; ++d) {
    n.nchild += cnt[d] != 0;
    n.kept += cnt[d];
    if (cnt[d] >= 2) {
      if (cnt[d] > kBigNode) ++n.nblk;
      else ++n.nwrp;
    }
    if (cnt[d] > kBlockSumNode) ++n.nbig;
  }
  return n;
}

// The children of node p at reserved offsets (id0, mb0, qb, qw, qg); false when they do not
// fit the buffers (error set).
__device__ bool write_children(TreeBuffers &tb, int p, const int cnt[8], const SplitNeeds &n, int id0, int mb0,
                               int qb, int qw, int qg, unsigned *err) {
  if (id0 + n.nchild > tb.max_nodes || (long long)mb0 + n.kept > tb.max_members || qb + n.nblk > tb.max_blk ||
      qw + n.nwrp > tb.max_wrp || qg + n.nbig > tb.max_big) {
    atomicOr(err, DERR_TREE_NODES);
    return false;
  }
  const int4 Ip = tb.nI[p];
  const int depth = tb.nDepth[p] + 1;
  const int lb = depth % 3;
  const double4 P = tb.nP[p];
  const double h = tb.nA[p].w / 2.0;
  int off = 0, k = 0, kb = 0, kw = 0, kg = 0;
#pragma unroll
  for (int d = 0; d < 8; ++d) {
    if (!cnt[d]) continue;
    const int id = id0 + k;
    const bool last = (k == n.nchild - 1);
    const double cx = (d & 1) ? e_add(P.x, h) : P.x;
    const double cz = (d & 2) ? e_add(P.z, h) : P.z;
    const double cy = (d & 4) ? e_add(P.y, h) : P.y;
    tb.nP[id] = make_double4(cx, cy, cz, 0);
    tb.nA[id] = make_double4(0, 0, 0, h);
    tb.nI[id] = make_int4(cnt[d], kEnd, last ? Ip.z : id + 1, 0);
    tb.nR[id] = make_int2(mb0 + off, cnt[d]);
    tb.nDepth[id] = depth;
    tb.nSib[id] = last ? kEnd : id + 1;
    if (cnt[d] >= 2) {  // the child's level list of nodes still to split
      if (cnt[d] > kBigNode) tb.split_blk[lb][qb + kb++] = id;
      else tb.split_wrp[lb][qw + kw++] = id;
    }
    if (cnt[d] > kBlockSumNode) tb.bigl[qg + kg++] = id;
    off += cnt[d];
    ++k;
  }
  tb.nI[p].y = id0;
  return true;
}

__device__ void make_children(TreeBuffers &tb, int p, const int cnt[8], int *id0_out, int *mb0_out, unsigned *err) {
  int mask = 0, kept = 0;
#pragma unroll
  for (int d = 0; d < 8; ++d) {
    if (cnt[d]) mask |= 1 << d;
    kept += cnt[d];
  }
  const int nchild = __popc(mask);
  int4 Ip = tb.nI[p];
  if (nchild == 0) {
    *id0_out = -1;
    *mb0_out = -1;
    return;
  }
  // one reservation per counter for the whole node (node ids, member slots, split-list and
  // big-node entries), the atomics issued together rather than one per child
  const int depth = tb.nDepth[p] + 1;
  const int lb = depth % 3;
  int nblk = 0, nwrp = 0, nbig = 0;
#pragma unroll
  for (int d = 0; d < 8; ++d) {
    if (cnt[d] >= 2) {
      if (cnt[d] > kBigNode) ++nblk;
      else ++nwrp;
    }
    if (cnt[d] > kBlockSumNode) ++nbig;
  }
  const int id0 = atomicAdd(&tb.ctr[0], nchild);
  const int mb0 = atomicAdd(&tb.ctr[1], kept);
  const int qb = nblk ? atomicAdd(&tb.ctr[kCtrSplit + lb], nblk) : 0;
  const int qw = nwrp ? atomicAdd(&tb.ctr[kCtrSplit + 3 + lb], nwrp) : 0;
  const int qg = nbig ? atomicAdd(&tb.ctr[kCtrBig], nbig) : 0;
  if (id0 + nchild > tb.max_nodes || (long long)mb0 + kept > tb.max_members || qb + nblk > tb.max_blk ||
      qw + nwrp > tb.max_wrp || qg + nbig > tb.max_big) {
    atomicOr(err, DERR_TREE_NODES);
    *id0_out = -1;
    *mb0_out = -1;
    return;
  }
  const double4 P = tb.nP[p];
  const double h = tb.nA[p].w / 2.0;
  int off = 0, k = 0, kb = 0, kw = 0, kg = 0;
#pragma unroll
  for (int d = 0; d < 8; ++d) {
    if (!cnt[d]) continue;
    const int id = id0 + k;
    const bool last = (k == nchild - 1);
    const double cx = (d & 1) ? e_add(P.x, h) : P.x;
    const double cz = (d & 2) ? e_add(P.z, h) : P.z;
    const double cy = (d & 4) ? e_add(P.y, h) : P.y;
    tb.nP[id] = make_double4(cx, cy, cz, 0);
    tb.nA[id] = make_double4(0, 0, 0, h);
    tb.nI[id] = make_int4(cnt[d], kEnd, last ? Ip.z : id + 1, 0);
    tb.nR[id] = make_int2(mb0 + off, cnt[d]);
    tb.nDepth[id] = depth;
    tb.nSib[id] = last ? kEnd : id + 1;
    if (cnt[d] >= 2) {  // the child's level list of nodes still to split
      if (cnt[d] > kBigNode) tb.split_blk[lb][qb + kb++] = id;
      else tb.split_wrp[lb][qw + kw++] = id;
    }
    if (cnt[d] > kBlockSumNode) tb.bigl[qg + kg++] = id;
    off += cnt[d];
    ++k;
  }
  tb.nI[p].y = id0;
  *id0_out = id0;
  *mb0_out = mb0;
}

// The roots' split (build_tree at the root, tree.f90:66-94) for every system at once: the
// live slots, in slot order, are sorted stably by (system, octant digit; 8 for a point in
// no child), which lists each child's members in slot order, as the warp and block splits
// do node by node.
__global__ void k_root_digits(const double *__restrict__ X, long long T, TreeBuffers tb,
                              const int *__restrict__ sys_of, const int *__restrict__ pos,
                              const SysConst *__restrict__ scs) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= T) return;
  const int n_live = pos[T];
  if (q >= n_live) {
    tb.rkey[0][q] = 0xFFFFFFFFu;
    tb.rval[0][q] = 0;
    return;
  }
  const int g = tb.members[q];
  const int s = sys_of[g];
  int d = 8;
  // a point pinned in front (its segment goes into the wall) counts in the root's centre but
  // belongs to no child (new_tree, tree.f90:128)
  if (tb.nI[s].x >= 2 && !(scs[s].pin && pin_i(scs[s].pin[g]))) {
    double x[3];
    load_x(X, T, g, x);
    d = octant(x, tb.nP[s], tb.nA[s].w / 2.0);
    if (d < 8) {  // one atomic per (system, octant) per warp: 8 counters take all the slots
      const int key = 8 * s + d;
      const unsigned peers = __match_any_sync(__activemask(), key);
      if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&tb.root_cnt[key], __popc(peers));
    }
  }
  tb.rkey[0][q] = ((unsigned)s << 4) | (unsigned)d;
  tb.rval[0][q] = g;
}

__global__ void k_root_children(TreeBuffers tb, int nsys, unsigned *err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  tb.root_mb[s] = -1;
  if (tb.nI[s].x < 2) return;
  int cnt[8];
  for (int d = 0; d < 8; ++d) cnt[d] = tb.root_cnt[8 * s + d];
  int id0 = -1, mb0 = -1;
  make_children(tb, s, cnt, &id0, &mb0, err);
  tb.root_mb[s] = mb0;
}

__global__ void k_root_scatter(TreeBuffers tb, const int *__restrict__ pos, long long T) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= T || p >= pos[T]) return;
  const unsigned key = tb.rkey[1][p];
  const int s = (int)(key >> 4), d = (int)(key & 15u);
  const int mb = tb.root_mb[s];
  if (d < 8 && mb >= 0) tb.members[mb + (int)(p - tb.nR[s].x)] = tb.rval[1][p];
}

// Split node p (at most kBigNode members) with one warp: count the members per octant, make
// the children, then write each member to its child's list in member order (stable).  Each
// lane takes kUnroll members per pass (k0 + 32 u + lane), their loads in flight together.
constexpr int kUnroll = 4;
constexpr int kSplitThreads = 512;

// Octants (8: outside every child, or past `end`) and slots of members k0 + 32 u + lane of
// the list mem[0 .. end).
__device__ __forceinline__ void octants_of(const double *__restrict__ X, long long T, const int *mem, int k0, int end,
                                           int lane, const double4 &P, double h, int d[kUnroll], int slot[kUnroll]) {
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    const int k = k0 + 32 * u + lane;
    slot[u] = k < end ? mem[k] : -1;
  }
  double x[kUnroll][3];
#pragma unroll
  for (int u = 0; u < kUnroll; ++u)
    if (slot[u] >= 0) load_x(X, T, slot[u], x[u]);
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) d[u] = slot[u] >= 0 ? octant(x[u], P, h) : 8;
}

// Members k0 .. of a pass ranked in member order: the stable position of each in its child's
// list (base_off + run + the lanes before it with the same octant), -1 for none.
__device__ __forceinline__ void rank_and_write(TreeBuffers &tb, int mb0, const int base_off[8], int run[8],
                                               const int d[kUnroll], const int slot[kUnroll], int lane) {
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) {
    int mypos = -1;
#pragma unroll
    for (int dd = 0; dd < 8; ++dd) {
      const unsigned b = __ballot_sync(0xffffffffu, d[u] == dd);
      if (d[u] == dd) mypos = mb0 + base_off[dd] + run[dd] + __popc(b & lt);
      run[dd] += __popc(b);
    }
    if (mypos >= 0) tb.members[mypos] = slot[u];
  }
}

// Node p's member count per octant (the warp's lanes over its member list).
__device__ void warp_count(const double *__restrict__ X, long long T, const TreeBuffers &tb, int p, int lane,
                           int cnt[8]) {
  const int2 R = tb.nR[p];
  const double4 P = tb.nP[p];
  const double h = tb.nA[p].w / 2.0;
  for (int k0 = 0; k0 < R.y; k0 += 32 * kUnroll) {
    int d[kUnroll], slot[kUnroll];
    octants_of(X, T, tb.members + R.x, k0, R.y, lane, P, h, d, slot);
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int dd = 0; dd < 8; ++dd) cnt[dd] += __popc(__ballot_sync(0xffffffffu, d[u] == dd));
  }
}

// Node p's members into its children's lists (stable: slot order kept), from member slot mb0.
__device__ void warp_scatter(const double *__restrict__ X, long long T, TreeBuffers &tb, int p, int lane,
                             const int cnt[8], int mb0) {
  const int2 R = tb.nR[p];
  const double4 P = tb.nP[p];
  const double h = tb.nA[p].w / 2.0;
  int base_off[8], run[8];
  {
    int off = 0;
#pragma unroll
    for (int dd = 0; dd < 8; ++dd) {
      base_off[dd] = off;
      off += cnt[dd];
      run[dd] = 0;
    }
  }
  for (int k0 = 0; k0 < R.y; k0 += 32 * kUnroll) {
    int d[kUnroll], slot[kUnroll];
    octants_of(X, T, tb.members + R.x, k0, R.y, lane, P, h, d, slot);
    rank_and_write(tb, mb0, base_off, run, d, slot, lane);
  }
}

// The counters a split reserves from, for children at list level lb.
__device__ __forceinline__ int *split_ctr(TreeBuffers &tb, int c, int lb) {
  return c == 0 ? &tb.ctr[0]
       : c == 1 ? &tb.ctr[1]
       : c == 2 ? &tb.ctr[kCtrSplit + lb]
       : c == 3 ? &tb.ctr[kCtrSplit + 3 + lb]
                : &tb.ctr[kCtrBig];
}

// Node p split by the whole warp: count, lane 0 reserves and writes the children, scatter.
__device__ void warp_split_one(const double *__restrict__ X, long long T, TreeBuffers &tb, int p, int lane, int lb,
                               unsigned *err) {
  int cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  warp_count(X, T, tb, p, lane, cnt);
  const SplitNeeds nd = split_needs(cnt);
  int mb0 = -1;
  if (lane == 0 && nd.nchild > 0) {
    const int v[5] = {nd.nchild, nd.kept, nd.nblk, nd.nwrp, nd.nbig};
    int base[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) base[c] = v[c] ? atomicAdd(split_ctr(tb, c, lb), v[c]) : 0;
    if (write_children(tb, p, cnt, nd, base[0], base[1], base[2], base[3], base[4], err)) mb0 = base[1];
  }
  mb0 = __shfl_sync(0xffffffffu, mb0, 0);
  if (mb0 >= 0) warp_scatter(X, T, tb, p, lane, cnt, mb0);
}

// Nodes with at most kLaneNode members, when a level lists many (the deep levels), are split
// by one lane each: the lane counts its node's members per octant (digits kept, 4 bits a
// member), the warp makes one reservation per counter for its lanes' nodes, and each lane
// writes its children and scatters its members in member order.
constexpr int kLaneNode = 16;

__device__ void lane_split(const double *__restrict__ X, long long T, TreeBuffers &tb, int p, int2 R, int lane,
                           int lb, unsigned *err) {
  const bool mine = p >= 0;
  int cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long digs = 0;
  if (mine) {
    const double4 P = tb.nP[p];
    const double h = tb.nA[p].w / 2.0;
    unsigned long long cp = 0;  // eight counts of 5 bits
    for (int k = 0; k < R.y; ++k) {
      double x[3];
      load_x(X, T, tb.members[R.x + k], x);
      const int d = octant(x, P, h);
      digs |= (unsigned long long)d << (4 * k);
      if (d < 8) cp += 1ull << (5 * d);
    }
#pragma unroll
    for (int dd = 0; dd < 8; ++dd) cnt[dd] = (int)((cp >> (5 * dd)) & 31u);
  }
  const SplitNeeds nd = mine ? split_needs(cnt) : SplitNeeds{0, 0, 0, 0, 0};
  const int v[5] = {nd.nchild, nd.kept, nd.nblk, nd.nwrp, nd.nbig};
  int off[5], base[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) {  // exclusive prefix over the lanes, the total in lane 31
    int x = v[c];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    off[c] = x - v[c];
    base[c] = 0;
    if (lane == 31 && x) base[c] = atomicAdd(split_ctr(tb, c, lb), x);
    base[c] = __shfl_sync(0xffffffffu, base[c], 31);
  }
  if (!mine || nd.nchild == 0) return;
  const int mb0 = base[1] + off[1];
  if (!write_children(tb, p, cnt, nd, base[0] + off[0], mb0, base[2] + off[2], base[3] + off[3], base[4] + off[4],
                      err))
    return;
  unsigned long long op = 0, run = 0;  // children's list offsets and fill, 5 bits each
  int o = 0;
#pragma unroll
  for (int dd = 0; dd < 8; ++dd) {
    op |= (unsigned long long)o << (5 * dd);
    o += cnt[dd];
  }
  for (int k = 0; k < R.y; ++k) {
    const int d = (int)((digs >> (4 * k)) & 15u);
    if (d < 8) {
      const int at = (int)(((op >> (5 * d)) & 31u) + ((run >> (5 * d)) & 31u));
      run += 1ull << (5 * d);
      tb.members[mb0 + at] = tb.members[R.x + k];
    }
  }
}

// Split node p (more than kBigNode members) with a whole block: each warp takes a contiguous
// slice of the member list and the slices' counts are prefix-summed, so the partition stays
// stable.
__device__ void split_node_block(const double *__restrict__ X, long long T, TreeBuffers &tb, int p,
                                 unsigned *err) {
  __shared__ int wcnt[32][8];
  __shared__ int s_id0, s_mb0, s_cnt[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int2 R = tb.nR[p];
  const double4 P = tb.nP[p];
  const double h = tb.nA[p].w / 2.0;
  const int per = (R.y + nw - 1) / nw;
  const int s0 = w * per, s1 = min(R.y, s0 + per);
  int cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int k0 = s0; k0 < s1; k0 += 32 * kUnroll) {
    int d[kUnroll], slot[kUnroll];
    octants_of(X, T, tb.members + R.x, k0, s1, lane, P, h, d, slot);
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int dd = 0; dd < 8; ++dd) cnt[dd] += __popc(__ballot_sync(0xffffffffu, d[u] == dd));
  }
  if (lane == 0)
#pragma unroll
    for (int dd = 0; dd < 8; ++dd) wcnt[w][dd] = cnt[dd];
  __syncthreads();
  if (threadIdx.x < 8) {
    int tot = 0;
    for (int ww = 0; ww < nw; ++ww) {
      const int c = wcnt[ww][threadIdx.x];
      wcnt[ww][threadIdx.x] = tot;  // exclusive prefix over warps
      tot += c;
    }
    s_cnt[threadIdx.x] = tot;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int c[8];
    for (int dd = 0; dd < 8; ++dd) c[dd] = s_cnt[dd];
    int id0, mb0;
    make_children(tb, p, c, &id0, &mb0, err);
    s_id0 = id0;
    s_mb0 = mb0;
  }
  __syncthreads();
  const int mb0 = s_mb0;
  if (s_id0 >= 0) {
    int base_off[8], run[8];
    int off = 0;
#pragma unroll
    for (int dd = 0; dd < 8; ++dd) {
      base_off[dd] = off + wcnt[w][dd];
      off += s_cnt[dd];
      run[dd] = 0;
    }
    for (int k0 = s0; k0 < s1; k0 += 32 * kUnroll) {
      int d[kUnroll], slot[kUnroll];
      octants_of(X, T, tb.members + R.x, k0, s1, lane, P, h, d, slot);
      rank_and_write(tb, mb0, base_off, run, d, slot, lane);
    }
  }
}

// One level of the build: the listed big nodes by blocks, then the other listed nodes by
// warps.  One block of kSplitThreads per SM, with registers for the loads of several
// members (or nodes) per lane in flight at once.  The children's lists (level + 1) fill as nodes split; the list of level + 2 is
// idle during this level (read at level - 1, filled at level + 1) and is emptied here.
__global__ void __launch_bounds__(kSplitThreads, 1) k_split_level(const double *__restrict__ X, long long T, TreeBuffers tb,
                                                      int level, unsigned *err) {
  const int b = level % 3, b2 = (level + 2) % 3;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    tb.ctr[kCtrSplit + b2] = 0;
    tb.ctr[kCtrSplit + 3 + b2] = 0;
  }
  const int nbl = min(tb.ctr[kCtrSplit + b], tb.max_blk);
  for (int bq = blockIdx.x; bq < nbl; bq += gridDim.x) {
    const int p = tb.split_blk[b][bq];
    if (tb.nDepth[p] >= kMaxLevels) {
      if (threadIdx.x == 0) atomicOr(err, DERR_TREE_DEPTH);
      continue;
    }
    split_node_block(X, T, tb, p, err);
    __syncthreads();
  }
  // The other listed nodes by warps.  Where they outnumber the warps twice over (the small,
  // numerous nodes of the deep levels) a warp takes an equal share of them, up to 32: each
  // lane splits its own when it has at most kLaneNode members, and the warp the larger ones
  // one at a time; elsewhere a warp splits one node at a time.
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int nwl = min(tb.ctr[kCtrSplit + 3 + b], tb.max_wrp);
  const int lb = (level + 1) % 3;  // the children's level lists
  if (nwl >= 2 * nwarps) {
    const int per = min(32, (nwl + nwarps - 1) / nwarps);  // nodes per warp: every warp busy
    for (int wq0 = warp * per; wq0 < nwl; wq0 += nwarps * per) {
      int p = lane < per && wq0 + lane < nwl ? tb.split_wrp[b][wq0 + lane] : -1;
      if (p >= 0 && tb.nDepth[p] >= kMaxLevels) {
        atomicOr(err, DERR_TREE_DEPTH);
        p = -1;
      }
      const int2 R = p >= 0 ? tb.nR[p] : make_int2(0, 0);
      const bool small = p >= 0 && R.y <= kLaneNode;
      lane_split(X, T, tb, small ? p : -1, R, lane, lb, err);
      for (unsigned big = __ballot_sync(0xffffffffu, p >= 0 && !small); big; big &= big - 1) {
        const int pp = __shfl_sync(0xffffffffu, p, __ffs(big) - 1);
        warp_split_one(X, T, tb, pp, lane, lb, err);
      }
    }
  } else {
    for (int wq = warp; wq < nwl; wq += nwarps) {
      const int p = tb.split_wrp[b][wq];
      if (tb.nDepth[p] >= kMaxLevels) {
        if (lane == 0) atomicOr(err, DERR_TREE_DEPTH);
        continue;
      }
      warp_split_one(X, T, tb, p, lane, lb, err);
    }
  }
}

// Centre and circulation of every node: sequential sums in ascending slot order
// (new_tree, tree.f90:124-152; the root's masked mean, tree.f90:50-54), plus the
// geometric distance of the opening test's correction (tree.f90:267-269).
constexpr int kSmallNode = 16;  // nodes up to this many members are summed by one thread

__device__ __forceinline__ void finish_node(TreeBuffers &tb, int id, bool root, double cx, double cy, double cz,
                                            double qx, double qy, double qz, const int *__restrict__ nxt,
                                            unsigned *err) {
  const int2 R = tb.nR[id];
  int4 I = tb.nI[id];
  const double4 P = tb.nP[id];
  const double w = tb.nA[id].w;
  if (R.y != 0) {
    cx = e_div(cx, (double)R.y);
    cy = e_div(cy, (double)R.y);
    cz = e_div(cz, (double)R.y);
  }
  const double hw = w / 2.;
  const double geo = e_sqrt(e_add(e_add(e_sq(e_sub(cx, e_add(P.x, hw))), e_sq(e_sub(cy, e_add(P.y, hw)))),
                                   e_sq(e_sub(cz, e_add(P.z, hw)))));
  // the centre only: the width (nA.w) is not written, since the split of this node may be
  // reading it at the same time (the depth-1 nodes are summed beside the level-1 split)
  double *a = reinterpret_cast<double *>(&tb.nA[id]);
  a[0] = cx;
  a[1] = cy;
  a[2] = cz;
  tb.nB[id] = make_double4(qx, qy, qz, geo);
  if (!root) {
    const int first = R.y > 0 ? tb.members[R.x] : 0;
    I.w = first ? nxt[first] : 0;
    tb.nI[id].w = I.w;  // the node's other links belong to the splits
    tb.nLeaf[id] = I.x == 1 ? first : 0;
    if (tb.nDepth[id] >= kMaxLevels && I.x > 1) atomicOr(err, DERR_TREE_DEPTH);
  }
}

// Nodes with at most kSmallNode members (most of them leaves): one thread each.
__global__ void k_node_sums_small(const double *__restrict__ X, const double *__restrict__ GI,
                                  const int *__restrict__ nxt, long long T, TreeBuffers tb, int nsys, unsigned *err) {
  const int n = tb.ctr[0];
  for (int id = nsys + blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x) {
    const int2 R = tb.nR[id];
    if (R.y > kSmallNode) continue;
    const bool root = false;
    double cx = 0, cy = 0, cz = 0, qx = 0, qy = 0, qz = 0;
    for (int k = 0; k < R.y; ++k) {
      const int g = tb.members[R.x + k];
      const double x0 = __ldg(X + g), x1 = __ldg(X + T + g), x2 = __ldg(X + 2 * T + g);
      cx = e_add(cx, x0);
      cy = e_add(cy, x1);
      cz = e_add(cz, x2);
      if (!root) {
        qx = e_sub(e_add(qx, __ldg(GI + g)), x0);
        qy = e_sub(e_add(qy, __ldg(GI + T + g)), x1);
        qz = e_sub(e_add(qz, __ldg(GI + 2 * T + g)), x2);
      }
    }
    finish_node(tb, id, root, cx, cy, cz, qx, qy, qz, nxt, err);
  }
}

// Sequential sums of one node by one warp: the warp gathers 32 members' coordinates and
// ghosts (coalesced member reads) into shared memory; lanes 0-2 then add the three centre
// components and lanes 3-5 the three circulation components, each in ascending member order
// -- the reference loop's sequence of roundings.  A lane first moves its 32 operands into
// registers and then runs the dependent additions unrolled, so the chain proceeds at the
// latency of the additions alone; the next tile's loads are issued before them.
constexpr int kTilePad = 33;  // row stride: lanes 0-5 reading one column hit distinct banks

__device__ __forceinline__ void warp_node_sums(const double *__restrict__ X, const double *__restrict__ GI,
                                               long long T, const int *__restrict__ mem, int count, bool circ,
                                               double (*buf)[kTilePad], int lane, double &acc) {
  acc = 0;
  double v[6];
  auto gather = [&](int k0) {
    const int k = k0 + lane;
    if (k < count) {
      const int g = mem[k];
      v[0] = __ldg(X + g);
      v[1] = __ldg(X + T + g);
      v[2] = __ldg(X + 2 * T + g);
      if (circ) {
        v[3] = __ldg(GI + g);
        v[4] = __ldg(GI + T + g);
        v[5] = __ldg(GI + 2 * T + g);
      }
    }
  };
  gather(0);
  for (int k0 = 0; k0 < count; k0 += 32) {
    __syncwarp();
    if (k0 + lane < count) {
#pragma unroll
      for (int c = 0; c < 3; ++c) buf[c][lane] = v[c];
      if (circ)
#pragma unroll
        for (int c = 3; c < 6; ++c) buf[c][lane] = v[c];
    }
    __syncwarp();
    if (k0 + 32 < count) gather(k0 + 32);
    const int cnt = min(32, count - k0);
    // centre lanes 0-2: acc + x; circulation lanes 3-5: (acc + gi) - x.  With circulations
    // the centre lanes subtract +0 (which returns its operand, -0 included), so that the six
    // chains run as one instruction stream instead of two divergent ones in turn
    const int ncomp = circ ? 6 : 3;
    const bool sub = lane >= 3;
    const double *a = buf[lane < 6 ? lane : 0], *bq = buf[sub && lane < 6 ? lane - 3 : 0];
    if (lane < ncomp) {
      if (!circ) {
        for (int l = 0; l < cnt; ++l) acc = e_add(acc, a[l]);
      } else if (cnt == 32) {
        double r[32], q[32];
#pragma unroll
        for (int l = 0; l < 32; ++l) {
          r[l] = a[l];
          const double x = bq[l];
          q[l] = sub ? x : 0.0;
        }
#pragma unroll
        for (int l = 0; l < 32; ++l) acc = e_sub(e_add(acc, r[l]), q[l]);
      } else {
        for (int l = 0; l < cnt; ++l) {
          const double x = bq[l];
          acc = e_sub(e_add(acc, a[l]), sub ? x : 0.0);
        }
      }
    }
  }
}

// Nodes (roots excepted) with kSmallNode < members <= kBlockSumNode: one warp each.
__global__ void __launch_bounds__(128) k_node_sums_big(const double *__restrict__ X, const double *__restrict__ GI,
                                                       const int *__restrict__ nxt, long long T, TreeBuffers tb,
                                                       int nsys, unsigned *err) {
  __shared__ double sm[4][6][kTilePad];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int n = tb.ctr[0];
  // The warp's nodes are ids nsys + warp + j nwarps (consecutive ids, often one level's
  // nodes of similar size, go to different warps); their records are read 32 at a time and
  // the ones in this kernel's size range summed in turn.
  for (long long j0 = 0; nsys + warp + j0 * nwarps < n; j0 += 32) {
    const long long idl = nsys + warp + (j0 + lane) * nwarps;
    const int2 Rl = idl < n ? tb.nR[idl] : make_int2(0, 0);
    for (unsigned m = __ballot_sync(0xffffffffu, Rl.y > kSmallNode && Rl.y <= kBlockSumNode); m; m &= m - 1) {
      const int l = __ffs(m) - 1;
      const int2 R = make_int2(__shfl_sync(0xffffffffu, Rl.x, l), __shfl_sync(0xffffffffu, Rl.y, l));
      double acc;
      warp_node_sums(X, GI, T, tb.members + R.x, R.y, true, sm[wl], lane, acc);
      const double cx = __shfl_sync(0xffffffffu, acc, 0), cy = __shfl_sync(0xffffffffu, acc, 1),
                   cz = __shfl_sync(0xffffffffu, acc, 2), qx = __shfl_sync(0xffffffffu, acc, 3),
                   qy = __shfl_sync(0xffffffffu, acc, 4), qz = __shfl_sync(0xffffffffu, acc, 5);
      if (lane == 0) finish_node(tb, (int)(nsys + warp + (j0 + l) * nwarps), false, cx, cy, cz, qx, qy, qz, nxt, err);
    }
  }
}

// Sequential sums of one large node by a block: warps 1.. stream member tiles into a ring of
// kSumDepth shared-memory tiles with 8-byte cp.async copies, kSumDepth - 1 tiles ahead of
// warp 0, whose lanes 0-2 (centre) and 3-5 (circulation) add each tile in member order.
constexpr int kSumTile = 512, kSumDepth = 4, kSumThreads = 256;
constexpr int kSumRow = kSumTile + 1;  // padded: lanes 0-5 reading one column hit distinct banks
constexpr size_t kSumSmem = (size_t)kSumDepth * 6 * kSumRow * sizeof(double);

__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_depth() {
  asm volatile("cp.async.wait_group %0;" ::"n"(kSumDepth - 2) : "memory");
}

__device__ void block_node_sums(const double *__restrict__ X, const double *__restrict__ GI, long long T,
                                const int *__restrict__ mem, int count, bool circ, double *sm, double &acc) {
  const int tid = threadIdx.x, lane = tid & 31;
  const bool producer = tid >= 32;
  const int ptid = tid - 32, np = kSumThreads - 32;
  const int ntiles = (count + kSumTile - 1) / kSumTile;
  const int ncomp = circ ? 6 : 3;
  auto issue = [&](int t) {  // producers: copies of tile t into its ring slot
    if (t < ntiles) {
      double *slot = sm + (size_t)(t % kSumDepth) * 6 * kSumRow;
      for (int e = ptid; e < kSumTile; e += np) {
        const int k = t * kSumTile + e;
        if (k >= count) break;
        const int g = mem[k];
        cp_async8(slot + e, X + g);
        cp_async8(slot + kSumRow + e, X + T + g);
        cp_async8(slot + 2 * kSumRow + e, X + 2 * T + g);
        if (circ) {
          cp_async8(slot + 3 * kSumRow + e, GI + g);
          cp_async8(slot + 4 * kSumRow + e, GI + T + g);
          cp_async8(slot + 5 * kSumRow + e, GI + 2 * T + g);
        }
      }
    }
    cp_async_commit();  // one group per tile, empty or not, so that the wait counts line up
  };
  acc = 0;
  if (producer) {
    for (int t = 0; t < kSumDepth - 1; ++t) issue(t);
    cp_async_wait_depth();  // tile 0 has landed
  }
  __syncthreads();
  for (int t = 0; t < ntiles; ++t) {
    if (producer) {
      issue(t + kSumDepth - 1);  // into the slot consumed in the previous round
      cp_async_wait_depth();     // tile t + 1 has landed
    } else if (lane < ncomp) {
      const double *slot = sm + (size_t)(t % kSumDepth) * 6 * kSumRow;
      // as in warp_node_sums: with circulations the centre lanes subtract +0, one stream
      const bool sub = lane >= 3;
      const double *a = slot + lane * kSumRow;
      const double *b = slot + (sub ? lane - 3 : 0) * kSumRow;
      const int cnt = min(kSumTile, count - t * kSumTile);
      if (!circ) {
        if (cnt == kSumTile) {
          for (int e0 = 0; e0 < kSumTile; e0 += 32) {
            double r[32];
#pragma unroll
            for (int l = 0; l < 32; ++l) r[l] = a[e0 + l];
#pragma unroll
            for (int l = 0; l < 32; ++l) acc = e_add(acc, r[l]);
          }
        } else {
          for (int l = 0; l < cnt; ++l) acc = e_add(acc, a[l]);
        }
      } else if (cnt == kSumTile) {
        for (int e0 = 0; e0 < kSumTile; e0 += 32) {
          double r[32], q[32];
#pragma unroll
          for (int l = 0; l < 32; ++l) {
            r[l] = a[e0 + l];
            const double x = b[e0 + l];
            q[l] = sub ? x : 0.0;
          }
#pragma unroll
          for (int l = 0; l < 32; ++l) acc = e_sub(e_add(acc, r[l]), q[l]);
        }
      } else {
        for (int l = 0; l < cnt; ++l) {
          const double x = b[l];
          acc = e_sub(e_add(acc, a[l]), sub ? x : 0.0);
        }
      }
    }
    __syncthreads();
  }
  if (producer) asm volatile("cp.async.wait_all;" ::: "memory");
}

// Non-root nodes with more than kBlockSumNode members (listed by the splits): one block each.
__global__ void __launch_bounds__(kSumThreads) k_node_sums_block(const double *__restrict__ X,
                                                                  const double *__restrict__ GI,
                                                                  const int *__restrict__ nxt, long long T,
                                                                  TreeBuffers tb, int part, unsigned *err) {
  // part 0: the big depth-1 nodes, listed by the roots' split (their member lists final),
  // summed beside the level splits (which read their width and write their first child,
  // fields the sums leave alone); part 1, after the levels: every other big node
  extern __shared__ double sm_dyn[];
  const int snap = tb.ctr[kCtrBigSnap];
  const int nbig = part == 0 ? snap : min(tb.ctr[kCtrBig], tb.max_big);
  for (int b = blockIdx.x; b < nbig; b += gridDim.x) {
    const int id = tb.bigl[b];
    const bool early = b < snap && tb.nDepth[id] <= kSnapLevel;
    if (early != (part == 0)) continue;  // block-uniform
    const int2 R = tb.nR[id];
    double acc;
    block_node_sums(X, GI, T, tb.members + R.x, R.y, true, sm_dyn, acc);
    const double cx = __shfl_sync(0xffffffffu, acc, 0), cy = __shfl_sync(0xffffffffu, acc, 1),
                 cz = __shfl_sync(0xffffffffu, acc, 2), qx = __shfl_sync(0xffffffffu, acc, 3),
                 qy = __shfl_sync(0xffffffffu, acc, 4), qz = __shfl_sync(0xffffffffu, acc, 5);
    if (threadIdx.x == 0) finish_node(tb, id, false, cx, cy, cz, qx, qy, qz, nxt, err);
    __syncthreads();
  }
}

__global__ void k_big_snapshot(TreeBuffers tb) {
  if (threadIdx.x == 0 && blockIdx.x == 0) tb.ctr[kCtrBigSnap] = min(tb.ctr[kCtrBig], tb.max_big);
}

// Roots: the masked mean over live slots (tree.f90:50-54), circulation zero.  One block per
// system; launched beside the level splits (it reads only the root's member list, which
// the splits do not change).
__global__ void __launch_bounds__(kSumThreads) k_root_sums(const double *__restrict__ X, long long T,
                                                            TreeBuffers tb, int nsys, const int *__restrict__ nxt,
                                                            unsigned *err) {
  extern __shared__ double sm_dyn[];
  const int id = blockIdx.x;
  if (id >= nsys) return;
  const int2 R = tb.nR[id];
  double acc;
  block_node_sums(X, nullptr, T, tb.members + R.x, R.y, false, sm_dyn, acc);
  const double cx = __shfl_sync(0xffffffffu, acc, 0), cy = __shfl_sync(0xffffffffu, acc, 1),
               cz = __shfl_sync(0xffffffffu, acc, 2);
  if (threadIdx.x == 0) finish_node(tb, id, true, cx, cy, cz, 0.0, 0.0, 0.0, nxt, err);
}

// Estimate of each root's centre (the mean over live slots, tree.f90:50-52) by a blocked
// sum over `parts` blocks per system (k_root_partial, then k_root_approx adding the parts in
// order), and a bound on its distance to the reference's sequential sum: a sum of N
// terms in FP64 is within (N-1) u sum|x| of the exact one in either order, so the two means
// differ by at most 2 u (sum|x| + sum|y| + sum|z|) plus the roundings of the divisions.
__global__ void __launch_bounds__(256) k_root_partial(const double *__restrict__ X, long long T, TreeBuffers tb,
                                                      int nsys, int parts) {
  __shared__ double red[6][8];
  const int s = blockIdx.x / parts, part = blockIdx.x % parts;
  if (s >= nsys) return;
  const int2 R = tb.nR[s];
  const int per = (R.y + parts - 1) / parts;
  const int k0 = part * per, k1 = min(R.y, k0 + per);
  const int *mem = tb.members + R.x;
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int k = k0 + (int)threadIdx.x; k < k1; k += blockDim.x) {
    const int g = mem[k];
    for (int c = 0; c < 3; ++c) {
      const double v = __ldg(X + c * T + g);
      a[c] += v;
      a[3 + c] += fabs(v);
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int c = 0; c < 6; ++c) {
    double v = a[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[c][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
    tb.root_part[(long long)blockIdx.x * 6 + threadIdx.x] = t;
  }
}

__global__ void k_root_approx(TreeBuffers tb, int nsys, int parts, double band_scale) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  double t[6] = {0, 0, 0, 0, 0, 0};
  for (int q = 0; q < parts; ++q)
    for (int c = 0; c < 6; ++c) t[c] += tb.root_part[((long long)s * parts + q) * 6 + c];
  const int n = tb.nR[s].y;
  const double dn = n > 0 ? (double)n : 1.0;
  const double cx = t[0] / dn, cy = t[1] / dn, cz = t[2] / dn;
  const double u = 1.2e-16;
  const double bound =
      band_scale * (2.0 * u * (t[3] + t[4] + t[5]) + 8.0 * u * (fabs(cx) + fabs(cy) + fabs(cz)) + 1e-300);
  tb.root_apx[s] = n > 0 ? make_double4(cx, cy, cz, bound) : make_double4(0, 0, 0, 0);
}

// The opening test of root `root` (tree.f90:264-278) for target xi and image shift s from
// the centre estimate: 0 the root is opened, 1 it is accepted (its circulation is zero, so
// the image adds nothing), 2 the estimate cannot tell.  The root's box is centred on the
// origin (corner -bsize/2, width bsize), so geo = |centre|.
__device__ __forceinline__ int root_decision(const TreeBuffers &tb, const SysConst &sc, int root, const double xi[3],
                                             const double s[3]) {
  const int4 I = tb.nI[root];
  if (I.x <= 1) return 2;  // empty or single-slot root: the exact path handles it
  if (sc.tree_extra_correction && sc.tree_theta > 1.1547) return 2;  // dist <= geo branch
  const double4 R = tb.root_apx[root];
  const double d0 = xi[0] - (R.x + s[0]), d1 = xi[1] - (R.y + s[1]), d2 = xi[2] - (R.z + s[2]);
  const double dist = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  const double thr = sc.bsize / sc.tree_theta;
  double margin = dist - thr, pert = R.w;
  if (sc.tree_extra_correction) {
    margin -= sqrt(R.x * R.x + R.y * R.y + R.z * R.z);
    pert *= 2.0;
  }
  pert += 1e-12 * (dist + thr);
  if (margin > pert) return 1;
  if (margin < -pert) return 0;
  return 2;
}

__device__ __forceinline__ void defer_push(const TreeBuffers &tb, int g, int m, unsigned *err) {
  const int q = atomicAdd(tb.defer_n, 1);
  if (q < kDeferCap) tb.defer[q] = make_int2(g, m);
  else atomicOr(err, DERR_QUEUE);
}

// tree_walk (tree.f90:250-316) for one image; accumulates into acc in preorder.
// `start` is the root, or the root's first child when the root is already known to be
// opened (its test then counted by the caller).
__device__ __forceinline__ void walk_fp64(const TreeBuffers &tb, int start, const SysConst &sc, const double xi[3],
                                          int gi_, int pi_, const int *__restrict__ prv, const double s[3], bool unshifted,
                                          double acc[3], unsigned long long &evals, unsigned long long &tests,
                                          bool &singular, bool &overrun) {
  const double qc = sc.quant_circ, two_pi = sc.two_pi, theta0 = sc.tree_theta;
  const bool corr = sc.tree_extra_correction;
  int node = start;
  int left = tb.ctr[0];  // a walk of a well-formed tree visits each node at most once
  while (node != kEnd) {
    if (--left < 0) {
      overrun = true;
      break;
    }
    const double4 A = ldg4(&tb.nA[node]);
    const int4 I = __ldg(&tb.nI[node]);
    if (I.x == 0) {
      node = I.z;
      continue;
    }
    ++tests;
    const double cs[3] = {e_add(A.x, s[0]), e_add(A.y, s[1]), e_add(A.z, s[2])};
    const double dist = e_sqrt(e_add(e_add(e_sq(e_sub(xi[0], cs[0])), e_sq(e_sub(xi[1], cs[1]))), e_sq(e_sub(xi[2], cs[2]))));
    const double4 B = ldg4(&tb.nB[node]);
    double theta;
    if (corr) {
      const double dg = e_sub(dist, B.w);
      theta = dg > 0. ? e_div(A.w, dg) : e_div(A.w, dist);
    } else {
      theta = e_div(A.w, dist);
    }
    if (I.x == 1 || theta < theta0) {
      node = I.z;
      if (I.x == 1) {
        const int j = __ldg(prv + I.w);
        if (unshifted && (j == gi_ || j == pi_)) continue;
        if (dist < NV_EPS) {
          singular = true;
          continue;
        }
      }
      const double vect[3] = {e_sub(cs[0], xi[0]), e_sub(cs[1], xi[1]), e_sub(cs[2], xi[2])};
      const double circ[3] = {B.x, B.y, B.z};
      const double a = e_mul(dist, dist);
      const double b = e_mul(2.0, dot3(vect, circ));
      const double c = dot3(circ, circ);
      const double D = e_sub(e_mul(e_mul(4.0, a), c), e_mul(b, b));
      if (D < NV_EPS) continue;
      double cr[3];
      cross3(vect, circ, cr);
      const double den = e_mul(two_pi, D);
      const double fac = e_sub(e_div(e_add(e_mul(2.0, c), b), e_sqrt(e_add(e_add(a, b), c))), e_div(b, e_sqrt(a)));
#pragma unroll
      for (int k = 0; k < 3; ++k) acc[k] = e_add(acc[k], e_mul(e_div(e_mul(cr[k], qc), den), fac));
      ++evals;
    } else {
      node = I.y != kEnd ? I.y : I.z;
    }
  }
}

// Local term, the unshifted image's tree sum ub0, the shifted images' sum ubs, mutual
// friction, in the reference's order of additions (timestep.f90:79-140).
__device__ void fp64_epilogue(const SysConst &sc, const SysDyn &dy, int g, const double *__restrict__ X,
                              const double *__restrict__ GI, const double *__restrict__ GB, double *__restrict__ U,
                              long long T, const double ub0[3], const double ubs[3]) {
  double xi[3], gi[3], gb[3], u[3], fdot[3];
  load3(X, T, g, xi);
  load3(GI, T, g, gi);
  load3(GB, T, g, gb);
  local_velocity(sc, xi, gi, gb, u, fdot);
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], ub0[c]);
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], ubs[c]);
  if (sc.n_mirror)  // the mirrored trees' sum, walked before (k_tree_walk_mirror)
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], sc.umir[c * T + g]);
  mf_epilogue(sc, dy, xi, fdot, u, g);
  store3(U, T, g, u);
}

// tree_walk_mirror (tree.f90:321-392) for every mirror of target g, in mirror order, into
// acc: each node's centre and centre + circulation reflected in the wall; theta = width/dist
// (the reference computes the corrected angle and then overwrites it with this one); a leaf
// whose segment goes into the wall, and the target's own image as biot_savart_mirror skips
// it, add nothing; the accept test includes the root (its circulation is zero, so an accepted
// root adds nothing either).
__device__ void walk_mirror(const TreeBuffers &tb, int root, const SysConst &sc, const double xi[3], int g, int pi_,
                            int pin_g, const int *__restrict__ prv, double acc[3], unsigned long long &evals,
                            unsigned long long &tests, bool &singular, bool &overrun) {
  const double qc = sc.quant_circ, two_pi = sc.two_pi, theta0 = sc.tree_theta;
  for (int m = 0; m < sc.n_mirror; ++m) {
    const bool own = mirror_skips_own(sc, pin_g, m);
    int node = root;
    int left = tb.ctr[0];
    while (node != kEnd) {
      if (--left < 0) {
        overrun = true;
        break;
      }
      const double4 A = ldg4(&tb.nA[node]);
      const int4 I = __ldg(&tb.nI[node]);
      if (I.x == 0) {
        node = I.z;
        continue;
      }
      ++tests;
      const double4 B = ldg4(&tb.nB[node]);
      const double cent[3] = {A.x, A.y, A.z}, circ[3] = {B.x, B.y, B.z};
      double s[3], sgi[3];
      for (int c = 0; c < 3; ++c) {
        s[c] = reflect1(e_add(cent[c], circ[c]), sc.mirror[m][c], sc.box[c]);
        sgi[c] = reflect1(cent[c], sc.mirror[m][c], sc.box[c]);
      }
      const double dist = e_sqrt(e_add(e_add(e_sq(e_sub(xi[0], s[0])), e_sq(e_sub(xi[1], s[1]))), e_sq(e_sub(xi[2], s[2]))));
      const double theta = e_div(A.w, dist);
      if (I.x == 1 || theta < theta0) {
        node = (node == root) ? kEnd : I.z;
        if (I.x == 1) {
          const int j = __ldg(prv + I.w);
          if (pin_i(sc.pin[j])) continue;
          if (own && ((pin_b(pin_g) && g == j) || (pin_i(pin_g) && j == pi_))) continue;
          if (dist < NV_EPS) {
            singular = true;
            continue;
          }
        }
        const double vect[3] = {e_sub(s[0], xi[0]), e_sub(s[1], xi[1]), e_sub(s[2], xi[2])};
        const double dv[3] = {e_sub(sgi[0], s[0]), e_sub(sgi[1], s[1]), e_sub(sgi[2], s[2])};
        const double a = e_mul(dist, dist);
        const double b = e_mul(2.0, dot3(vect, dv));
        const double c = e_add(e_add(e_sq(e_sub(s[0], sgi[0])), e_sq(e_sub(s[1], sgi[1]))), e_sq(e_sub(s[2], sgi[2])));
        const double D = e_sub(e_mul(e_mul(4.0, a), c), e_mul(b, b));
        if (D < NV_EPS) continue;
        double cr[3];
        cross3(vect, dv, cr);
        const double den = e_mul(two_pi, D);
        const double fac = e_sub(e_div(e_add(e_mul(2.0, c), b), e_sqrt(e_add(e_add(a, b), c))), e_div(b, e_sqrt(a)));
#pragma unroll
        for (int k = 0; k < 3; ++k) acc[k] = e_add(acc[k], e_mul(e_div(e_mul(cr[k], qc), den), fac));
        ++evals;
      } else {
        node = I.y != kEnd ? I.y : (node == root ? kEnd : I.z);
      }
    }
  }
}

// The mirror sums of every live target of the tree systems with solid walls (one thread
// each), written to umir for the FP64 walk's epilogue.  Runs after the roots' exact centres.
__global__ void k_tree_walk_mirror(const SysConst *__restrict__ scs, SysDyn *dyn, const int2 *__restrict__ work,
                                   const double *__restrict__ X, const int *__restrict__ nxt,
                                   const int *__restrict__ prv, long long T, TreeBuffers tb, unsigned *err) {
  const int2 w = work[blockIdx.x];
  const SysConst &sc = scs[w.x];
  if (!sc.n_mirror) return;
  const int g = w.y + threadIdx.x;
  const int k = g - sc.base;
  unsigned long long evals = 0, tests = 0;
  bool singular = false, overrun = false;
  if (!*err && k >= 1 && k <= dyn[w.x].pcount && k <= sc.cap && nxt[g] != 0) {
    double xi[3], acc[3] = {0, 0, 0};
    load3(X, T, g, xi);
    walk_mirror(tb, w.x, sc, xi, g, prv[g], sc.pin[g], prv, acc, evals, tests, singular, overrun);
    for (int c = 0; c < 3; ++c) sc.umir[c * T + g] = acc[c];
  }
  if (singular) atomicOr(err, DERR_SINGULAR);
  if (overrun) atomicOr(err, DERR_WALK);
  if (evals) atomicAdd(&dyn[w.x].tree_eval, evals);
  if (tests) atomicAdd(&dyn[w.x].tree_tests, tests);
}

// The tree sums of target g (timestep.f90:49-141 with tree_walk): over the unshifted image
// into ub0, then over the 26 shifts in order into ubs.  part 0 does both and the epilogue;
// part 1 only ub0, part 2 only ubs (the epilogue then runs where both are known) -- each
// sum is the same chain of additions either way.  With `decided` the root's tests come from
// the centre estimate: a target for which any of them is too close to call is deferred
// whole (nothing counted; part 2 leaves the push to part 1), to be redone exactly.  Returns
// false for a deferred target.
__device__ bool fp64_target(const SysConst &sc, const SysDyn &dy, int sys, int g, const double *__restrict__ X,
                            const double *__restrict__ GI, const double *__restrict__ GB,
                            const int *__restrict__ prv, double *__restrict__ U, long long T, const TreeBuffers &tb,
                            bool decided, int part, double ub0[3], double ubs[3], unsigned long long &evals,
                            unsigned long long &tests, unsigned *err) {
  double xi[3];
  load3(X, T, g, xi);
  const double zero[3] = {0, 0, 0};
  int start[27];
  const int first = tb.nI[sys].y;
  unsigned long long t0 = 0;
  for (int m = 0; m <= sc.n_shift; ++m) {
    start[m] = sys;
    if (!decided) continue;
    const int d = root_decision(tb, sc, sys, xi, m == 0 ? zero : sc.shift[m - 1]);
    if (d == 2) {
      if (part != 2) defer_push(tb, g, -1, err);
      return false;
    }
    start[m] = d == 1 ? kEnd : first;  // accepted: adds nothing; opened: walk the children
    ++t0;
  }
  if (part != 2) tests += t0;  // the root tests are counted once
  const int pi_ = prv[g];
  bool singular = false, overrun = false;
#pragma unroll
  for (int c = 0; c < 3; ++c) ub0[c] = ubs[c] = 0.;
  if (part != 2) walk_fp64(tb, start[0], sc, xi, g, pi_, prv, zero, true, ub0, evals, tests, singular, overrun);
  if (part != 1)
    for (int m = 0; m < sc.n_shift; ++m)
      walk_fp64(tb, start[m + 1], sc, xi, g, pi_, prv, sc.shift[m], false, ubs, evals, tests, singular, overrun);
  if (singular) atomicOr(err, DERR_SINGULAR);
  if (overrun) atomicOr(err, DERR_WALK);
  if (part == 0) fp64_epilogue(sc, dy, g, X, GI, GB, U, T, ub0, ubs);
  return true;
}

// Plain FP64 tree walk, 64 targets per block.  With `split`, two threads per target (128
// per block): warps 0-1 sum the unshifted image (the deepest walk), warps 2-3 the 26 shifted
// ones, and the second thread adds the two sums in the reference's order once both are
// done -- for small systems, whose few blocks would leave most SMs idle.  Without, one
// thread per target does it all (64 per block).
__global__ void __launch_bounds__(128) k_tree_walk_fp64(const SysConst *__restrict__ scs, SysDyn *dyn,
                                                        const int2 *__restrict__ work, const double *__restrict__ X,
                                                        const double *__restrict__ GI, const double *__restrict__ GB,
                                                        const int *__restrict__ nxt, const int *__restrict__ prv,
                                                        double *__restrict__ U, long long T, TreeBuffers tb,
                                                        int split, unsigned *err) {
  __shared__ double s_ub0[3][64];
  const int2 w = work[blockIdx.x];
  const SysConst &sc = scs[w.x];
  const int t = threadIdx.x & 63, part = split ? 1 + (threadIdx.x >> 6) : 0;
  const int q = w.y + t - sc.base;  // position in the system's walk order
  const int g = q >= 1 && q <= sc.cap ? tb.perm[sc.base + q] : sc.base;
  const int k = g - sc.base;
  unsigned long long evals = 0, tests = 0;
  double ub0[3] = {0, 0, 0}, ubs[3] = {0, 0, 0};
  bool done = false;
  if (!*err && k >= 1 && k <= dyn[w.x].pcount && nxt[g] != 0 && q >= sc.walk_lo && q < sc.walk_hi)
    done = fp64_target(sc, dyn[w.x], w.x, g, X, GI, GB, prv, U, T, tb, true, part, ub0, ubs, evals, tests, err);
  if (part == 1)
    for (int c = 0; c < 3; ++c) s_ub0[c][t] = ub0[c];
  __syncthreads();
  if (part == 2 && done) {
    for (int c = 0; c < 3; ++c) ub0[c] = s_ub0[c][t];
    fp64_epilogue(sc, dyn[w.x], g, X, GI, GB, U, T, ub0, ubs);
  }
  // tree_eval (tree.f90:308): one atomic per warp
  unsigned long long tot = evals, tt = tests;
  for (int o = 16; o > 0; o >>= 1) {
    tot += __shfl_down_sync(0xffffffffu, tot, o);
    tt += __shfl_down_sync(0xffffffffu, tt, o);
  }
  if ((threadIdx.x & 31) == 0 && tot) atomicAdd(&dyn[w.x].tree_eval, tot);
  if ((threadIdx.x & 31) == 0 && tt) atomicAdd(&dyn[w.x].tree_tests, tt);
}

// The deferred root tests, after the exact root sums: FP64 targets again whole (image -1),
// mixed (target, image) pairs as that image's partial sum from the exact FP64 walk.
__global__ void k_walk_fixup(const SysConst *__restrict__ scs, SysDyn *dyn, const int *__restrict__ sys_of,
                             const double *__restrict__ X, const double *__restrict__ GI,
                             const double *__restrict__ GB, const int *__restrict__ prv, double *__restrict__ U,
                             double *__restrict__ partial, long long T, TreeBuffers tb, unsigned *err) {
  const int n = min(*tb.defer_n, kDeferCap);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int2 d = tb.defer[e];
    const int g = d.x, s = sys_of[g];
    const SysConst &sc = scs[s];
    unsigned long long evals = 0, tests = 0;
    if (d.y < 0) {
      double ub0[3], ubs[3];
      fp64_target(sc, dyn[s], s, g, X, GI, GB, prv, U, T, tb, false, 0, ub0, ubs, evals, tests, err);
    } else {
      const int m = d.y;
      double xi[3], acc[3] = {0, 0, 0};
      const double zero[3] = {0, 0, 0};
      load3(X, T, g, xi);
      bool singular = false, overrun = false;
      walk_fp64(tb, s, sc, xi, g, prv[g], prv, m == 0 ? zero : sc.shift[m - 1], m == 0, acc, evals, tests,
                singular, overrun);
      if (singular) atomicOr(err, DERR_SINGULAR);
      if (overrun) atomicOr(err, DERR_WALK);
      const long long o = (long long)m * 3 * T + g;
      partial[o] = acc[0];
      partial[o + T] = acc[1];
      partial[o + 2 * T] = acc[2];
    }
    if (evals) atomicAdd(&dyn[s].tree_eval, evals);
    if (tests) atomicAdd(&dyn[s].tree_tests, tests);
  }
}

// Squared distance from x to the cell [P, P + w]^3 (0 inside).
__device__ __forceinline__ double cube_dist2(const double x[3], const double4 P, double w) {
  const double p[3] = {P.x, P.y, P.z};
  double d2 = 0.;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double lo = p[c] - x[c], hi = x[c] - (p[c] + w);
    const double d = fmax(fmax(lo, hi), 0.);
    d2 += d * d;
  }
  return d2;
}

// An upper bound on the distance the closest-point walk settles on: the distance of a leaf
// that walk accepts and counts, or 100.  A node whose cell holds the target is opened by the
// walk (its centroid lies in the same cell, so width/dist >= 1/sqrt(3) > .5), so every child
// of such a node is reached; a child that is a single point is accepted, and below such a
// child the walk's own opening test decides what is reached.  Any accepted leaf's distance,
// formed as the walk forms it, is at least the walk's final closestd.  The search follows
// the cells that hold the target down from the root, takes the nearest counted leaf child on
// the way, and then walks, with the reference's opening test, the subtree of the deepest
// node on that path that holds at least kBoundNode points (a few dozen visits): warps whose
// targets all get a bound near their final closestd prune the rest of their walks alike.
constexpr int kBoundNode = 16;

__device__ double closest_bound(const TreeBuffers &tb, const SysConst &sc, int root, const double xi[3], int g,
                                int ni, int pi_, const int *__restrict__ prv) {
  double best = 100.;
  auto counted = [&](int j) { return j != g && j != ni && j != pi_ && !pinned_at(sc, j); };
  auto dist_to = [&](const double4 &A) {
    return e_sqrt(e_add(e_add(e_sq(e_sub(xi[0], A.x)), e_sq(e_sub(xi[1], A.y))), e_sq(e_sub(xi[2], A.z))));
  };
  {  // the root's cell must hold the target too (it always does between enforce_boundary calls)
    const double4 P = ldg4(&tb.nP[root]);
    const double w = tb.nA[root].w;
    if (!(xi[0] >= P.x && xi[0] < P.x + w && xi[1] >= P.y && xi[1] < P.y + w && xi[2] >= P.z && xi[2] < P.z + w))
      return best;
  }
  int node = root, deep = root;
  for (int depth = 0; depth <= kMaxLevels && node != kEnd; ++depth) {
    const int4 I = __ldg(&tb.nI[node]);
    if (I.x <= 1 || I.y == kEnd) break;
    if (I.x >= kBoundNode) deep = node;
    const int stop = I.z;  // the node after the last child's subtree
    int next = kEnd;
    for (int c = I.y; c != kEnd && c != stop;) {
      const int4 Ic = __ldg(&tb.nI[c]);
      if (Ic.x == 1) {
        if (counted(__ldg(prv + Ic.w))) best = fmin(best, dist_to(ldg4(&tb.nA[c])));
      } else if (Ic.x > 1 && next == kEnd) {
        const double4 P = ldg4(&tb.nP[c]);
        const double w = tb.nA[c].w;
        if (xi[0] >= P.x && xi[0] < P.x + w && xi[1] >= P.y && xi[1] < P.y + w && xi[2] >= P.z && xi[2] < P.z + w)
          next = c;
      }
      c = Ic.z;
    }
    node = next;
  }
  // the walk below `deep` (opened: it holds the target), with the reference's opening test
  const int4 Id = __ldg(&tb.nI[deep]);
  if (Id.x <= 1) return best;
  int left = tb.ctr[0];  // (a malformed tree only loosens the bound; the main walk reports it)
  for (int n = Id.y; n != kEnd && n != Id.z && --left >= 0;) {
    const int4 I = __ldg(&tb.nI[n]);
    if (I.x == 0) {
      n = I.z;
      continue;
    }
    const double4 A = ldg4(&tb.nA[n]);
    const double dist = dist_to(A);
    if (I.x == 1 || e_div(A.w, dist) < .5) {
      if (I.x == 1 && counted(__ldg(prv + I.w))) best = fmin(best, dist);
      n = I.z;
    } else {
      n = I.y != kEnd ? I.y : I.z;
    }
  }
  return best;
}

// pclose_tree + closest_tree (tree.f90:190-244): theta = width/dist < .5, no shift, no
// correction; the candidate is prv(first member's infront at build time) with the links of
// now (after pinsert).  Subtrees whose cells lie farther than min(cd, closest_bound) are
// skipped: they hold no leaf or node that could still change closest or closestd.
template <bool kPrefetch>
__global__ void k_closest_tree(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                               const int *__restrict__ sys_of, const double *__restrict__ X,
                               const int *__restrict__ nxt, const int *__restrict__ prv, int *__restrict__ cl,
                               double *__restrict__ CD, long long T, TreeBuffers tb, unsigned *err) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T || *err) return;
  const long long g = tb.perm[t];  // the walk order: neighbouring threads, neighbouring targets
  const int s = sys_of[g];
  const SysConst &sc = scs[s];
  if (!sc.use_tree || (dyn[s].itime % sc.recon_shots) != 0) return;
  const int k = (int)(g - sc.base);
  if (k < 1 || k > dyn[s].pcount) return;
  double cd = 100.;
  const int ni = nxt[g];
  if (ni == 0) {
    CD[g] = cd;
    return;
  }
  if (pinned_at(sc, (int)g)) {  // pinned points are not tested (tree.f90:198-199)
    CD[g] = cd;
    return;
  }
  const int pi_ = prv[g];
  int best = cl[g];
  double xi[3];
  load3(X, T, (int)g, xi);
  // The reference forms dist = sqrt(d2) and theta = width/dist at every node.  Both are
  // correctly rounded, so theta < .5 and dist < cd can differ from d2 > 4 width^2 and
  // d2 < cd^2 only when d2 lies within a few ulps of the bound: outside a 1e-12 band the
  // squared comparison decides, inside it the reference's own expressions do.
  constexpr double kBand = 1e-12;
  double cd2 = cd * cd;
  // slack of the subtree skip below: covers the rounding of the centroids (sums of up to
  // 2^24 positions) and of the distances
  const double margin = 1e-8 * sc.bsize;
  const double bound = closest_bound(tb, sc, s, xi, (int)g, ni, pi_, prv);
  int node = s;
  double4 A = ldg4(&tb.nA[node]);
  int4 I = __ldg(&tb.nI[node]);
  int left = tb.ctr[0];  // a walk of a well-formed tree visits each node at most once
  for (;;) {
    if (--left < 0) {
      atomicOr(err, DERR_WALK);
      break;
    }
    // kPrefetch (few targets, latency-bound): the records of both possible successors (next
    // in preorder past the subtree, first child) are requested before this node is decided,
    // so their loads overlap the test; with a full GPU the extra loads cost more than that
    const int nz = I.z, ny = I.y;
    double4 Az = make_double4(0, 0, 0, 0), Ay = Az;
    int4 Iz = make_int4(0, kEnd, kEnd, 0), Iy = Iz;
    if (kPrefetch && nz != kEnd) {
      Az = ldg4(&tb.nA[nz]);
      Iz = __ldg(&tb.nI[nz]);
    }
    if (kPrefetch && ny != kEnd) {
      Ay = ldg4(&tb.nA[ny]);
      Iy = __ldg(&tb.nI[ny]);
    }
    bool down = false;  // to the first child; else past the subtree
    if (I.x != 0) {
      const double d2 = e_add(e_add(e_sq(e_sub(xi[0], A.x)), e_sq(e_sub(xi[1], A.y))), e_sq(e_sub(xi[2], A.z)));
      bool acc = I.x == 1;
      if (!acc) {
        const double w4 = 4.0 * A.w * A.w;
        if (d2 > w4 * (1 + kBand)) acc = true;
        else if (d2 >= w4 * (1 - kBand)) acc = e_div(A.w, e_sqrt(d2)) < .5;
      }
      if (acc) {
        bool closer;
        if (d2 < cd2 * (1 - kBand)) closer = true;
        else if (d2 > cd2 * (1 + kBand)) closer = false;
        else closer = e_sqrt(d2) < cd;
        if (closer) {
          const int j = prv[I.w];
          if (I.x > 1) {
            best = 0;
          } else if (j != (int)g && ni != j && pi_ != j && !pinned_at(sc, j)) {  // pinned j: nothing
            best = j;
            cd = e_sqrt(d2);
            cd2 = cd * cd;
          }
        }
      } else if (ny != kEnd &&
                 !(node != s && cube_dist2(xi, ldg4(&tb.nP[node]), A.w) >
                               (fmin(cd, bound) + margin) * (fmin(cd, bound) + margin))) {
        down = true;
      }
      // (an opened node whose cell lies farther than cd: every member of this node lies in
      // its cell -- the splits drop points outside the children's cells -- so every
      // centroid in its subtree is farther than cd: none is closer, now or later (cd only
      // shrinks), and none changes best or cd.  Its subtree is skipped.)
    }
    const int next = down ? ny : nz;
    if (next == kEnd) break;
    if (kPrefetch) {
      A = down ? Ay : Az;
      I = down ? Iy : Iz;
    } else {
      A = ldg4(&tb.nA[next]);
      I = __ldg(&tb.nI[next]);
    }
    node = next;
  }
  cl[g] = best;
  CD[g] = cd;
}

// Mixed-precision node records: FP64 centre with the squared acceptance distance, FP32
// circulation.  The opening test of tree_walk (tree.f90:266-278) accepts a node when
//   dist - geo > 0 and width/(dist - geo) < theta0   <=>  dist > geo + width/theta0, or
//   dist - geo <= 0 and width/dist < theta0          <=>  geo >= dist > width/theta0,
// (without the correction: dist > width/theta0); comparing squared distances in FP64 gives
// the same decisions except at exact ties.  The second branch needs geo > width/theta0,
// impossible for theta0 <= 2/sqrt(3) (geo <= sqrt(3)/2 width), so it is tested only above.
// Roots are skipped: their exact centre may still be summing (the walks take the roots'
// tests from the centre estimate).
// Relative half-width of the band around the opening threshold inside which the mixed
// walk's FP32 test defers to the FP64 one (the FP32 |r|^2 is within ~1e-6 of its value).
constexpr float kTestBand = 1e-5f;

__global__ void k_node_prep(TreeBuffers tb, int nsys, double theta0, int corr, float line_guard,
                            const int *__restrict__ prv) {
  const int n = tb.ctr[0];
  for (int id = nsys + blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x) {
    const double4 A = tb.nA[id], B = tb.nB[id];
    const double t0 = A.w / theta0;
    const double t1 = corr ? B.w + t0 : t0;
    tb.mx.C[id] = make_double4(A.x, A.y, A.z, t1 * t1);
    const float qx = (float)B.x, qy = (float)B.y, qz = (float)B.z;
    tb.mx.G[id] = make_double2(corr ? B.w * B.w : -1.0, t0 * t0);
    const float hx = (float)A.x, hy = (float)A.y, hz = (float)A.z;
    const int4 I = tb.nI[id];
    WalkNode wn;
    wn.a = make_float4(hx, hy, hz, (float)(t1 * t1));
    const float q2 = qx * qx + qy * qy + qz * qz;
    wn.b = make_float4((float)(A.x - hx), (float)(A.y - hy), (float)(A.z - hz), q2);
    wn.c = make_float4(qx, qy, qz, line_guard * q2);
    wn.d = make_int4(I.x, I.y, tb.nSib[id], I.x == 1 ? prv[I.w] : I.w);
    tb.mx.W[id] = wn;
  }
}

// A leaf's record holds prv of its member, the start of the leaf's segment, for the walk's
// own-segment test; this refreshes it when points were relinked after the build.
__global__ void k_leaf_links(TreeBuffers tb, int nsys, const int *__restrict__ prv) {
  const int n = tb.ctr[0];
  for (int id = nsys + blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x) {
    const int4 I = tb.nI[id];
    if (I.x == 1) tb.mx.W[id].d.w = prv[I.w];
  }
}

// Mixed tree walk: one lane per (target, image), a warp walking together.  A warp holds 32
// targets that are close in space (consecutive in the Morton walk order) against one image
// and traverses the union of their walks: a stack of (node, lane mask) entries, where an
// entry stands for a node and its following siblings and the mask holds the lanes whose
// walk reaches them.  The stack lives in registers, entry d in lane d % 32.  Each node's
// 64-byte record is read once per warp (broadcast); each lane takes the reference's opening
// decision for itself, so a lane accepts exactly the nodes its own walk (tree.f90:250-316)
// accepts, in the same preorder.
//
// The opening test compares |r|^2 with t1^2.  r is formed in FP32 from the high and low
// parts of the centre and of the image-shifted target (|r_FP32 - r| <~ 2^-23 |r|), so
// |r|^2 in FP32 is within 1e-6 of its value; outside a 1e-5 band around t1^2 the FP32
// comparison gives the FP64 answer, inside it the FP64 test runs.  Far interactions in FP32;
// accepted leaves within the near radius and ill-conditioned far terms in FP64.  Writes
// the image's partial sum.
constexpr int kWalkStack = 64;  // two register entries per lane; the build stops at depth 42

// Large systems (kSplit false, the GPU full of long walks): the FP64 accumulators live in
// shared memory and 9 blocks fit on an SM; small ones (split central image, a short tail):
// accumulators in registers, 8 blocks (both measured faster than the other choice).
template <bool kSplit>
__global__ void __launch_bounds__(128, kSplit ? 8 : 9) k_tree_walk_mixed(const SysConst *__restrict__ scs, SysDyn *dyn,
                                                            const int4 *__restrict__ work,
                                                            const double *__restrict__ X,
                                                            const int *__restrict__ nxt, const int *__restrict__ prv,
                                                            double *__restrict__ partial, long long T, TreeBuffers tb,
                                                            double near_factor, Fp32Guards gd, int parts,
                                                            unsigned *err) {
  const int lane = threadIdx.x & 31;
  const int4 w = work[blockIdx.x];  // system, image, first position, part of a split central image
  const SysConst &sc = scs[w.x];
  const int m = w.y, part = w.w;
  const int q = w.z + threadIdx.x - sc.base;  // position in the system's walk order
  const int g = q >= 1 && q <= sc.cap ? tb.perm[sc.base + q] : sc.base;
  const int k = g - sc.base;
  unsigned evals = 0, tests = 0, n64 = 0, nband = 0;
  // A walk range's ends fall on warp boundaries (nv_set_walk_range): a warp walks all its
  // targets or none, and the warp's visits (the union of its lanes' walks), which set where
  // the FP32 partials are flushed, are the same as without a range.
  const bool valid = !*err && k >= 1 && k <= dyn[w.x].pcount && nxt[g] != 0 && q >= sc.walk_lo && q < sc.walk_hi;
  const unsigned live = __ballot_sync(0xffffffffu, valid);
  float xh[3] = {0, 0, 0}, xl[3] = {0, 0, 0};  // target - shift, FP32 high and low parts
  int pi_ = 0;
  if (valid) {
    double xs[3];
    load3(X, T, g, xs);
    if (m > 0)
      for (int c = 0; c < 3; ++c) xs[c] -= sc.shift[m - 1][c];
    for (int c = 0; c < 3; ++c) {
      xh[c] = (float)xs[c];
      xl[c] = (float)(xs[c] - (double)xh[c]);
    }
    pi_ = prv[g];
  }
  const float near2 = (float)(near_factor * sc.delta * near_factor * sc.delta);
  const double gq64 = sc.quant_circ / (4.0 * NV_PI);
  const float gq = (float)gq64;
  const bool second = sc.tree_extra_correction && sc.tree_theta > 1.1547;
  // FP32 partial over at most kFlush far interactions: a lane adds at most one term per
  // node visit and the warp promotes every lane's partial to FP64 after kFlush visits
  float fx = 0, fy = 0, fz = 0;
  int since_flush = 0;  // warp-uniform
  // FP64: near field plus the flushed FP32 partials (touched only at a flush or an FP64 term)
  __shared__ double s_acc[kSplit ? 1 : 3][128];
  double r_acc0 = 0., r_acc1 = 0., r_acc2 = 0.;
  double &nx = kSplit ? r_acc0 : s_acc[0][threadIdx.x];
  double &ny = kSplit ? r_acc1 : s_acc[kSplit ? 0 : 1][threadIdx.x];
  double &nz = kSplit ? r_acc2 : s_acc[kSplit ? 0 : 2][threadIdx.x];
  nx = ny = nz = 0.;
  bool singular = false;
  // r and |r|^2 in FP64 as the FP64 walk forms them: (centre + shift) - target
  auto exact_r = [&](int cur, double r[3]) -> double {
    const double4 C = ldg4(&tb.mx.C[cur]);
    double xi[3];
    load3(X, T, g, xi);
    const double s0 = m > 0 ? sc.shift[m - 1][0] : 0., s1 = m > 0 ? sc.shift[m - 1][1] : 0.,
                 s2 = m > 0 ? sc.shift[m - 1][2] : 0.;
    r[0] = e_sub(e_add(C.x, s0), xi[0]);
    r[1] = e_sub(e_add(C.y, s1), xi[1]);
    r[2] = e_sub(e_add(C.z, s2), xi[2]);
    return e_add(e_add(e_sq(r[0]), e_sq(r[1])), e_sq(r[2]));
  };
  // FP64 evaluation of an accepted node: the reference's singularity check and skip decision
  // in its own arithmetic (tree.f90:289-303), the value from the cancellation-free form
  auto exact_term = [&](int cur) {
    double r[3];
    const double d2 = exact_r(cur, r);
    const double dist = e_sqrt(d2);
    if (dist < NV_EPS) {
      singular = true;
      return;
    }
    const double4 B = ldg4(&tb.nB[cur]);
    const double circ[3] = {B.x, B.y, B.z};
    const double a = e_mul(dist, dist);
    const double b = e_mul(2.0, dot3(r, circ));
    const double c = dot3(circ, circ);
    const double D = e_sub(e_mul(e_mul(4.0, a), c), e_mul(b, b));
    if (D < NV_EPS) return;
    double tm[3];
    term64_stable(r, circ, d2, gq64, tm);
    nx += tm[0];
    ny += tm[1];
    nz += tm[2];
    ++evals;
    ++n64;
  };
  // the root's test from the centre estimate: accepted (nothing to add), opened (the walk
  // starts at its children) or deferred until the exact centre is known
  int rd = 1;
  if (valid) {
    double xi[3];
    const double zero[3] = {0, 0, 0};
    load3(X, T, g, xi);
    rd = root_decision(tb, sc, w.x, xi, m > 0 ? sc.shift[m - 1] : zero);
    if (part == 0) {  // the parts of a split central image share one root test
      if (rd == 2) defer_push(tb, g, m, err);
      else ++tests;
    }
  }
  const unsigned open0 = __ballot_sync(0xffffffffu, valid && rd == 0);
  const int first = tb.nI[w.x].y;
  // The root's children are nodes first .. first+nc-1.  A part of a split central image
  // walks children lo .. hi-1 of them (ids below lim); every other item walks them all.
  int start = first, lim = INT_MAX;
  if (kSplit && m == 0 && first != kEnd) {
    int nc = 0;
    for (int d = 0; d < 8; ++d) nc += tb.root_cnt[8 * w.x + d] != 0;
    const int lo = part * 8 / parts, hi = min((part + 1) * 8 / parts, nc);
    start = lo < nc ? first + lo : kEnd;
    lim = first + hi;
  }
  (void)live;
  // (cur, mask): the node the warp is at and the lanes whose walk reaches it, warp-uniform.
  // The stack holds the pending next siblings of the nodes opened on the way down: entry d
  // (node, mask) in lane d % 32, register pair 0 for d < 32, 1 above.
  int sn0 = 0, sn1 = 0;
  unsigned sm0 = 0, sm1 = 0;
  int top = -1;
  int cur = start;
  unsigned mask = open0;
  bool more = open0 && start != kEnd;
  // (no visit budget here, unlike the FP64 walks: even a check per flush cost 3% of the
  // walk; the warp visits each node of the tree the build makes at most once)
  while (more) {
    const WalkNode *wn = tb.mx.W + cur;
    // the whole 64-byte record at once: one load latency per node instead of a chain
    const int4 D = __ldg(&wn->d);
    const float4 A = __ldg(&wn->a), B = __ldg(&wn->b), Q = __ldg(&wn->c);
    // the next sibling, none past the last root child of this item's group (the root's
    // children are the only nodes with ids in [first, lim))
    const int sib = kSplit && D.z >= lim && cur >= first && cur < lim ? kEnd : D.z;
    bool open = false;
    if ((mask >> lane) & 1u) {  // (every node below a root has members)
      ++tests;
      const float rx = (A.x - xh[0]) + (B.x - xl[0]);
      const float ry = (A.y - xh[1]) + (B.y - xl[1]);
      const float rz = (A.z - xh[2]) + (B.z - xl[2]);
      const float d2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
      bool acc;
      if (D.x == 1) {
        acc = true;
      } else if (!second && d2 > A.w * (1.f + kTestBand)) {
        acc = true;
      } else if (!second && d2 < A.w * (1.f - kTestBand)) {
        acc = false;
      } else {  // near the threshold (or the second criterion): the FP64 test
        ++nband;
        double r[3];
        const double d2e = exact_r(cur, r);
        acc = d2e > tb.mx.C[cur].w;
        if (!acc && second) {
          const double2 G = tb.mx.G[cur];
          acc = d2e <= G.x && d2e > G.y;
        }
      }
      if (!acc) {
        open = true;
      } else {
        bool done = false;
        if (D.x == 1) {
          if (m == 0)  // the target's own segments are skipped in the central image
            done = D.w == g || D.w == pi_;  // D.w: prv of the leaf's member
          if (!done && d2 < near2) {
            exact_term(cur);  // near leaf: the reference arithmetic in FP64
            done = true;
          }
        }
        if (!done) {
          // the reference skips 4ac-b^2 < epsilon (tree.f90:303); 4ac-b^2 = 4|r x circ|^2
          const float cx = fmaf(ry, Q.z, -rz * Q.y), cy = fmaf(rz, Q.x, -rx * Q.z), cz = fmaf(rx, Q.y, -ry * Q.x);
          const float cr2 = fmaf(cx, cx, fmaf(cy, cy, cz * cz));
          if (!(4.f * cr2 < (float)NV_EPS)) {
            const float ex = rx + Q.x, ey = ry + Q.y, ez = rz + Q.z;
            const float ee = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
            const float re = fmaf(rx, ex, fmaf(ry, ey, rz * ez));
            // ia = 1/|r|, ib = 1/|r + circ|; pp = |r||r + circ|
            const float ia = rsqrtf(d2), ib = rsqrtf(ee);
            const float pp = (d2 * ia) * (ee * ib);
            if (cr2 < Q.w * fminf(d2, ee) || ee < gd.end * fmaxf(d2, B.w) || pp + re < gd.angle * pp) {
              // the target lies near the segment's line or near its far end (or the optional
              // angle guard): FP32 would cancel digits there
              exact_term(cur);
            } else {
              // (|r| + |e|) / (pp (pp + r.e)) = (ia + ib) / (pp + r.e), e = r + circ, with
              // pp + r.e = |r x circ|^2 / (pp - r.e) when r.e < 0 (no cancellation either way)
              const bool obtuse = re < 0.f;
              const float num = gq * (ia + ib) * (obtuse ? pp - re : 1.f);
              const float f = __fdividef(num, obtuse ? cr2 : pp + re);  // MUFU reciprocal
              fx = fmaf(f, cx, fx);
              fy = fmaf(f, cy, fy);
              fz = fmaf(f, cz, fz);
              ++evals;
            }
          }
        }
      }
    }
    const unsigned omask = __ballot_sync(0xffffffffu, open);
    if (omask && D.y != kEnd) {  // the lanes that open cur walk its children first
      if (sib != kEnd) {         // and come back to cur's next sibling afterwards
        ++top;
        if (top >= kWalkStack) {  // deeper than any tree the build makes; guard only
          if (lane == 0) atomicOr(err, DERR_TREE_DEPTH);
          break;
        }
        if (lane == (top & 31)) {
          if (top >= 32) {
            sn1 = sib;
            sm1 = mask;
          } else {
            sn0 = sib;
            sm0 = mask;
          }
        }
      }
      cur = D.y;
      mask = omask;
    } else if (sib != kEnd) {
      cur = sib;
    } else if (top >= 0) {
      const int src = top & 31;
      const bool hi = top >= 32;
      cur = __shfl_sync(0xffffffffu, hi ? sn1 : sn0, src);
      mask = __shfl_sync(0xffffffffu, hi ? sm1 : sm0, src);
      --top;
    } else {
      more = false;
    }
    if (++since_flush == kFlush) {  // at most kFlush FP32 terms per partial
      nx += (double)fx;
      ny += (double)fy;
      nz += (double)fz;
      fx = fy = fz = 0.f;
      since_flush = 0;
    }
  }
  if (singular) atomicOr(err, DERR_SINGULAR);
  if (valid) {
    const int slot = m == 0 && part > 0 ? 26 + part : m;  // extra parts after the 27 images
    const long long o = (long long)slot * 3 * T + g;
    partial[o] = (double)fx + nx;
    partial[o + T] = (double)fy + ny;
    partial[o + 2 * T] = (double)fz + nz;
  }
  unsigned long long tot = evals, tt = tests, t64 = n64, tb_ = nband;
  for (int o = 16; o > 0; o >>= 1) {
    tot += __shfl_down_sync(0xffffffffu, tot, o);
    tt += __shfl_down_sync(0xffffffffu, tt, o);
    t64 += __shfl_down_sync(0xffffffffu, t64, o);
    tb_ += __shfl_down_sync(0xffffffffu, tb_, o);
  }
  if (lane == 0 && tot) atomicAdd(&dyn[w.x].tree_eval, tot);
  if (lane == 0 && tt) atomicAdd(&dyn[w.x].tree_tests, tt);
  if (lane == 0 && t64) atomicAdd((unsigned long long *)&dyn[w.x].diag[8], t64);
  if (lane == 0 && tb_) atomicAdd((unsigned long long *)&dyn[w.x].diag[9], tb_);
  if (lane == 0 && tot > t64) atomicAdd((unsigned long long *)&dyn[w.x].diag[10], tot - t64);
}

int n_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

}  // namespace

int n_sms_host() { return n_sms(); }
const int *tree_iperm(nv_handle *h) { return h->tree ? h->tree->iperm : nullptr; }
const int *tree_perm(nv_handle *h) { return h->tree ? h->tree->perm : nullptr; }

void tree_alloc(nv_handle *h) {
  bool need = false;
  for (auto &s : h->sc) need = need || s.use_tree || s.sched_tree;
  if (!need) return;
  auto *tb = new TreeBuffers();
  const long long T = h->T;
  tb->max_nodes = (int)std::min<long long>(3 * T + h->nsys + 1024, (1LL << 31) - 1);
  tb->max_members = 24 * T + 1024;
  cudaMalloc(&tb->nA, (size_t)tb->max_nodes * sizeof(double4));
  cudaMalloc(&tb->nB, (size_t)tb->max_nodes * sizeof(double4));
  cudaMalloc(&tb->nP, (size_t)tb->max_nodes * sizeof(double4));
  cudaMalloc(&tb->nI, (size_t)tb->max_nodes * sizeof(int4));
  cudaMalloc(&tb->nR, (size_t)tb->max_nodes * sizeof(int2));
  cudaMalloc(&tb->nDepth, (size_t)tb->max_nodes * sizeof(int));
  cudaMalloc(&tb->nSib, (size_t)tb->max_nodes * sizeof(int));
  cudaMalloc(&tb->nLeaf, (size_t)tb->max_nodes * sizeof(int));
  cudaMalloc(&tb->members, (size_t)tb->max_members * sizeof(int));
  // each level holds at most T / (kBlockSumNode + 1) nodes above the block threshold
  tb->max_big = (int)std::min<long long>((long long)kMaxLevels * (T / (kBlockSumNode + 1) + 1) + 64, 1 << 30);
  cudaMalloc(&tb->bigl, (size_t)tb->max_big * sizeof(int));
  cudaMalloc(&tb->root_apx, (size_t)h->nsys * sizeof(double4));
  for (int b = 0; b < 2; ++b) {
    cudaMalloc(&tb->rkey[b], (size_t)T * sizeof(unsigned));
    cudaMalloc(&tb->rval[b], (size_t)T * sizeof(int));
  }
  cudaMalloc(&tb->root_cnt, (size_t)h->nsys * 8 * sizeof(int));
  cudaMalloc(&tb->root_mb, (size_t)h->nsys * sizeof(int));
  {
    int sb = 1;
    while ((1LL << sb) < h->nsys) ++sb;
    tb->rkey_bits = std::min(32, 4 + sb);
    cub::DeviceRadixSort::SortPairs(nullptr, tb->rsort_bytes, tb->rkey[0], tb->rkey[1], tb->rval[0], tb->rval[1],
                                    (int)T, 0, tb->rkey_bits);
    cudaMalloc(&tb->rsort_tmp, std::max<size_t>(tb->rsort_bytes, 16));
  }
  tb->root_parts = std::max(1, std::min(64, 4096 / h->nsys));
  cudaMalloc(&tb->root_part, (size_t)h->nsys * tb->root_parts * 6 * sizeof(double));
  cudaMalloc(&tb->defer, (size_t)kDeferCap * sizeof(int2));
  cudaMalloc(&tb->defer_n, sizeof(int));
  cudaMemset(tb->defer_n, 0, sizeof(int));
  cudaFuncSetAttribute(k_root_sums, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSumSmem);
  cudaFuncSetAttribute(k_node_sums_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSumSmem);
  if (h->precision == NV_PREC_MIXED) {
    cudaMalloc(&tb->mx.C, (size_t)tb->max_nodes * sizeof(double4));
    cudaMalloc(&tb->mx.W, (size_t)tb->max_nodes * sizeof(WalkNode));
    cudaMalloc(&tb->mx.G, (size_t)tb->max_nodes * sizeof(double2));
  }
  cudaMalloc(&tb->ctr, kCtrSize * sizeof(int));
  cudaMemset(tb->ctr, 0, kCtrSize * sizeof(int));
  tb->max_blk = (int)(T / (kBigNode + 1) + h->nsys + 64);
  tb->max_wrp = (int)(T / 2 + h->nsys + 64);
  for (int b = 0; b < 3; ++b) {
    cudaMalloc(&tb->split_blk[b], (size_t)tb->max_blk * sizeof(int));
    cudaMalloc(&tb->split_wrp[b], (size_t)tb->max_wrp * sizeof(int));
  }
  cudaMalloc(&tb->flag, (T + 1) * sizeof(int));
  cudaMalloc(&tb->pos, (T + 1) * sizeof(int));
  cub::DeviceScan::ExclusiveSum(nullptr, tb->cub_bytes, tb->flag, tb->pos, (int)(T + 1));
  cudaMalloc(&tb->cub_tmp, std::max<size_t>(tb->cub_bytes, 16));
  for (int b = 0; b < 2; ++b) {
    cudaMalloc(&tb->okey[b], (size_t)T * sizeof(unsigned long long));
    cudaMalloc(&tb->oval[b], (size_t)T * sizeof(int));
  }
  tb->perm = tb->oval[1];
  cudaMalloc(&tb->iperm, (size_t)T * sizeof(int));
  k_iota<<<grid_for(T, TB), TB, 0, h->stream>>>(tb->perm, T);  // a permutation before the first build
  int sb = 1;
  while ((1LL << sb) < h->nsys) ++sb;
  tb->key_bits = 34 + sb;
  cub::DeviceRadixSort::SortPairs(nullptr, tb->sort_bytes, tb->okey[0], tb->okey[1], tb->oval[0], tb->oval[1], (int)T,
                                  0, tb->key_bits);
  cudaMalloc(&tb->sort_tmp, std::max<size_t>(tb->sort_bytes, 16));
  h->tree = tb;
}

void tree_free(nv_handle *h) {
  TreeBuffers *tb = h->tree;
  if (!tb) return;
  void *ptrs[] = {tb->nA, tb->nB, tb->nP, tb->nI, tb->nR, tb->nDepth, tb->nLeaf, tb->nSib, tb->members, tb->bigl, tb->root_apx, tb->root_part, tb->defer, tb->defer_n,
                  tb->rkey[0], tb->rkey[1], tb->rval[0], tb->rval[1], tb->root_cnt, tb->root_mb, tb->rsort_tmp, tb->ctr,
                  tb->flag, tb->pos, tb->cub_tmp, tb->mx.C, tb->mx.W, tb->mx.G, tb->okey[0], tb->okey[1],
                  tb->oval[0], tb->oval[1], tb->iperm, tb->sort_tmp, tb->split_blk[0], tb->split_blk[1],
                  tb->split_blk[2], tb->split_wrp[0], tb->split_wrp[1], tb->split_wrp[2]};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete tb;
  h->tree = nullptr;
}

void launch_tree_build(nv_handle *h) {
  TreeBuffers *tb = h->tree;
  if (!tb) return;
  const long long T = h->T;
  k_live_flags<<<grid_for(T + 1, TB), TB, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->nxt, tb->flag, T,
                                                         tb->ctr);
  size_t bytes = tb->cub_bytes;
  cub::DeviceScan::ExclusiveSum(tb->cub_tmp, bytes, tb->flag, tb->pos, (int)(T + 1), h->stream);
  k_scatter_live<<<grid_for(T, TB), TB, 0, h->stream>>>(tb->flag, tb->pos, tb->members, T);
  k_roots<<<grid_for(h->nsys, 64), 64, 0, h->stream>>>(h->d_sc, h->d_dyn, h->nsys, h->nxt, tb->pos, *tb, T);
  // the walk order and the roots' exact sums (one long sequential chain per system) run
  // on the side stream; the walks wait for the order, the fix-up of deferred root tests
  // and the closest-point walk for the sums
  cudaEventRecord(h->fork_ev, h->stream);
  cudaStreamWaitEvent(h->side, h->fork_ev, 0);
  k_order_keys<<<grid_for(T, TB), TB, 0, h->side>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->nxt, tb->okey[0],
                                                    tb->oval[0], T);
  {
    size_t sb = tb->sort_bytes;
    cub::DeviceRadixSort::SortPairs(tb->sort_tmp, sb, tb->okey[0], tb->okey[1], tb->oval[0], tb->oval[1], (int)T, 0,
                                    tb->key_bits, h->side);
  }
  k_inv_perm<<<grid_for(T, TB), TB, 0, h->side>>>(tb->perm, tb->iperm, T);
  cudaEventRecord(h->sort_ev, h->side);
  k_root_sums<<<h->nsys, kSumThreads, kSumSmem, h->side>>>(h->x, T, *tb, h->nsys, h->nxt, h->d_err);
  cudaEventRecord(h->join_ev, h->side);
  const int sms = n_sms();
  k_root_digits<<<grid_for(T, TB), TB, 0, h->stream>>>(h->x, T, *tb, h->sys_of, tb->pos, h->d_sc);
  {
    size_t sb = tb->rsort_bytes;
    cub::DeviceRadixSort::SortPairs(tb->rsort_tmp, sb, tb->rkey[0], tb->rkey[1], tb->rval[0], tb->rval[1], (int)T, 0,
                                    tb->rkey_bits, h->stream);
  }
  k_root_children<<<grid_for(h->nsys, 64), 64, 0, h->stream>>>(*tb, h->nsys, h->d_err);
  k_root_scatter<<<grid_for(T, TB), TB, 0, h->stream>>>(*tb, tb->pos, T);
  // the big depth-1 nodes' sums (the longest sequential chains after the roots') start as soon
  // as the roots' split has listed them and written their member lists, beside the levels
  k_big_snapshot<<<1, 32, 0, h->stream>>>(*tb);
  cudaEventRecord(h->fork2_ev, h->stream);
  cudaStreamWaitEvent(h->side2, h->fork2_ev, 0);
  k_node_sums_block<<<sms, kSumThreads, kSumSmem, h->side2>>>(h->x, h->gi, h->nxt, T, *tb, 0, h->d_err);
  cudaEventRecord(h->join2_ev, h->side2);
  for (int L = 1; L < kMaxLevels; ++L)
    k_split_level<<<sms, kSplitThreads, 0, h->stream>>>(h->x, T, *tb, L, h->d_err);
  k_node_sums_block<<<sms, kSumThreads, kSumSmem, h->stream>>>(h->x, h->gi, h->nxt, T, *tb, 1, h->d_err);
  k_node_sums_big<<<sms * 8, 128, 0, h->stream>>>(h->x, h->gi, h->nxt, T, *tb, h->nsys, h->d_err);
  k_node_sums_small<<<sms * 8, 128, 0, h->stream>>>(h->x, h->gi, h->nxt, T, *tb, h->nsys, h->d_err);
  k_root_partial<<<h->nsys * tb->root_parts, 256, 0, h->stream>>>(h->x, T, *tb, h->nsys, tb->root_parts);
  k_root_approx<<<grid_for(h->nsys, 128), 128, 0, h->stream>>>(*tb, h->nsys, tb->root_parts, h->root_band_scale);
  cudaStreamWaitEvent(h->stream, h->sort_ev, 0);
  cudaStreamWaitEvent(h->stream, h->join2_ev, 0);
  if (h->precision == NV_PREC_MIXED) {
    // theta0 and the correction flag are per system; a handle's systems share them when
    // any of them walks the tree (checked at creation)
    k_node_prep<<<sms * 4, 256, 0, h->stream>>>(*tb, h->nsys, h->sc[h->tree_sys0].tree_theta,
                                                h->sc[h->tree_sys0].tree_extra_correction, h->guards.line, h->prv);
    tb->prep_epoch = h->links_epoch;
  }
  tb->built = true;
}

void join_root_sums(nv_handle *h) {
  if (h->tree) cudaStreamWaitEvent(h->stream, h->join_ev, 0);
}

void launch_walk_fixup(nv_handle *h) {
  TreeBuffers *tb = h->tree;
  if (!tb) return;
  join_root_sums(h);
  k_walk_fixup<<<n_sms(), 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->gi, h->gb, h->prv, h->u,
                                               h->partial, h->T, *tb, h->d_err);
}

void launch_tree_walk(nv_handle *h) {
  TreeBuffers *tb = h->tree;
  if (!tb || h->n_work_tree == 0) return;
  if (h->any_mirror) {  // solid walls: the mirrored trees first, on the roots' exact centres
    join_root_sums(h);
    k_tree_walk_mirror<<<h->n_work_tree, 64, 0, h->stream>>>(h->d_sc, h->d_dyn, h->d_work_tree, h->x, h->nxt, h->prv,
                                                             h->T, *tb, h->d_err);
  }
  cudaMemsetAsync(tb->defer_n, 0, sizeof(int), h->stream);
  // two threads per target while the one-thread blocks would fill the GPU less than ~4
  // times (automatic), or as nv_set_walk_parts asks
  const int split = h->walk_parts == 0 ? h->n_work_tree < 32 * n_sms() : h->walk_parts > 1;
  k_tree_walk_fp64<<<h->n_work_tree, split ? 128 : 64, 0, h->stream>>>(
      h->d_sc, h->d_dyn, h->d_work_tree, h->x, h->gi, h->gb, h->nxt, h->prv, h->u, h->T, *tb, split, h->d_err);
}

void launch_tree_walk_mixed(nv_handle *h) {
  TreeBuffers *tb = h->tree;
  if (!tb || h->n_work_timg == 0) return;
  if (tb->prep_epoch != h->links_epoch) {  // relinked since the build
    k_leaf_links<<<n_sms() * 4, 256, 0, h->stream>>>(*tb, h->nsys, h->prv);
    tb->prep_epoch = h->links_epoch;
  }
  cudaMemsetAsync(tb->defer_n, 0, sizeof(int), h->stream);
  auto walk = h->walk_parts_used > 1 ? k_tree_walk_mixed<true> : k_tree_walk_mixed<false>;
  walk<<<h->n_work_timg, 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->d_work_timg, h->x, h->nxt, h->prv, h->partial,
                                              h->T, *tb, h->near_factor, h->guards, h->walk_parts_used, h->d_err);
}

void launch_closest_tree(nv_handle *h) {
  TreeBuffers *tb = h->tree;
  if (!tb) return;
  join_root_sums(h);
  // successor prefetch while the targets fill the GPU less than ~8 blocks per SM
  auto walk = h->T < 8LL * 128 * n_sms() ? k_closest_tree<true> : k_closest_tree<false>;
  walk<<<grid_for(h->T, 128), 128, 0, h->stream>>>(h->d_sc, h->d_dyn, h->sys_of, h->x, h->nxt, h->prv, h->closest,
                                                   h->closestd, h->T, *tb, h->d_err);
}

// Preorder dump of system `sys`'s tree (host side: download nodes, follow first_child/skip).
int tree_dump(nv_handle *h, int sys, void *buf, int cap, int *n) {
  TreeBuffers *tb = h->tree;
  if (!tb || !tb->built) return set_error(NV_ERR_STATE, "no tree has been built");
  cudaStreamSynchronize(h->stream);
  int nn = 0;
  NV_CUDA(cudaMemcpy(&nn, tb->ctr, sizeof(int), cudaMemcpyDeviceToHost));
  std::vector<double4> A(nn), B(nn), P(nn);
  std::vector<int4> I(nn);
  std::vector<int> D(nn), Lf(nn);
  NV_CUDA(cudaMemcpy(A.data(), tb->nA, nn * sizeof(double4), cudaMemcpyDeviceToHost));
  NV_CUDA(cudaMemcpy(B.data(), tb->nB, nn * sizeof(double4), cudaMemcpyDeviceToHost));
  NV_CUDA(cudaMemcpy(P.data(), tb->nP, nn * sizeof(double4), cudaMemcpyDeviceToHost));
  NV_CUDA(cudaMemcpy(I.data(), tb->nI, nn * sizeof(int4), cudaMemcpyDeviceToHost));
  NV_CUDA(cudaMemcpy(D.data(), tb->nDepth, nn * sizeof(int), cudaMemcpyDeviceToHost));
  NV_CUDA(cudaMemcpy(Lf.data(), tb->nLeaf, nn * sizeof(int), cudaMemcpyDeviceToHost));
  struct Rec {
    double pos[3], width, cent[3], circ[3];
    int32_t pcount, depth, leaf, first_next;
  };
  Rec *out = static_cast<Rec *>(buf);
  const int base = h->base[sys];
  int m = 0;
  for (int node = sys; node != kEnd;) {
    if (out && m < cap) {
      Rec &r = out[m];
      r.pos[0] = P[node].x; r.pos[1] = P[node].y; r.pos[2] = P[node].z;
      r.width = A[node].w;
      r.cent[0] = A[node].x; r.cent[1] = A[node].y; r.cent[2] = A[node].z;
      r.circ[0] = B[node].x; r.circ[1] = B[node].y; r.circ[2] = B[node].z;
      r.pcount = I[node].x;
      r.depth = D[node];
      r.leaf = Lf[node] ? Lf[node] - base : 0;
      r.first_next = I[node].w ? I[node].w - base : 0;
    }
    ++m;
    node = (I[node].x > 1 && I[node].y != kEnd) ? I[node].y : I[node].z;
  }
  *n = m;
  return NV_OK;
}
