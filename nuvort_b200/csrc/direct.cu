// direct.cu -- the direct Biot-Savart sum over all segments and their periodic images.
//
// Plain FP64 kernel (k_direct_fp64): one thread per target point, the segment records of
// the target's system streamed through shared memory in tiles by 1-D bulk copies
// (cp.async.bulk + mbarrier, double-buffered).  The summation order is the reference's:
//   u_bs = sum_j ascending (unshifted)                   timestep.f90:83-85
//   u_bs' = sum_images (in periodic_loop_array order) sum_j ascending   :88-92
// with every operation rounded once (no FMA), so the result is bit-identical to the
// reference arithmetic except for the ulp-level difference of the device log() in the
// local term.  The image loop is outside the tile loop for that reason: each image
// re-streams the tiles (from L2; the kernel is FP64-pipe bound, not memory bound).
#include <vector>

#include "handle.cuh"
#include "tma.cuh"

namespace {

constexpr int kDirectTJ = 128;  // segments per staged tile (64 B each)

template <int TJ>
__global__ void __launch_bounds__(64) k_direct_fp64(
    const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn, const int2 *__restrict__ work,
    const double *__restrict__ X, const double *__restrict__ GI, const double *__restrict__ GB,
    const int *__restrict__ nxt, const int *__restrict__ prv, const double4 *__restrict__ seg,
    double *__restrict__ U, long long T, unsigned *err, const int *__restrict__ targets = nullptr, int ntargets = 0,
    double *__restrict__ Uout = nullptr) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double4 *tiles = reinterpret_cast<double4 *>(smem_raw);  // [2][2*TJ]
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_abort;

  const int2 w = work[blockIdx.x];
  const SysConst &sc = scs[w.x];
  const int base = sc.base;
  const int pc = dyn[w.x].pcount;
  const int tid = threadIdx.x;
  int g;
  bool active;
  if (targets) {  // listed targets (k-th thread of block b takes targets[64 b + k])
    const int idx = w.y + tid;
    g = idx < ntargets ? targets[idx] : base;
    active = idx < ntargets && g > base && g - base <= pc && nxt[g] != 0;
  } else {
    if (w.y - base > pc) return;  // block-uniform: every target beyond pcount
    g = w.y + tid;
    active = (g - base <= pc) && (g - base <= sc.cap) && nxt[g] != 0;
  }

  // One thread reads the sticky error word so that the whole block agrees on it.
  if (tid == 0) {
    s_abort = (*err != 0);
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (s_abort) return;

  double xi[3] = {0, 0, 0};
  int pi = -1;
  if (active) {
    load3(X, T, g, xi);
    pi = prv[g];
  }
  const int nt = (pc + TJ - 1) / TJ;
  const int Q = (1 + sc.n_shift) * nt;
  const double qc = sc.quant_circ, two_pi = sc.two_pi;

  auto issue = [&](int q) {
    const int t = q % nt;
    const int n = min(TJ, pc - t * TJ);
    const int buf = q & 1;
    mbar_expect_tx(&bar[buf], (unsigned)(n * 64));
    bulk_g2s(tiles + buf * 2 * TJ, seg + 2 * (long long)(base + 1 + t * TJ), (unsigned)(n * 64), &bar[buf]);
  };
  int issued = 0;
  if (tid == 0) {
    if (Q > 0) issue(0);
    if (Q > 1) issue(1);
  }
  issued = Q < 2 ? Q : 2;

  double ub0[3] = {0, 0, 0}, ubs[3] = {0, 0, 0};
  int consumed = 0;
  for (int q = 0; q < Q; ++q) {
    const int buf = q & 1;
    const bool ok = mbar_wait(&bar[buf], (unsigned)((q >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(err, DERR_TIMEOUT);
      break;
    }
    consumed = q + 1;
    const int m = q / nt, t = q % nt;
    const int n = min(TJ, pc - t * TJ);
    const int j0 = base + 1 + t * TJ;
    const double4 *tl = tiles + buf * 2 * TJ;
    if (active) {
      if (m == 0) {
#pragma unroll 2
        for (int jj = 0; jj < n; ++jj) {
          const double4 A = tl[2 * jj], B = tl[2 * jj + 1];
          const int gj = j0 + jj;
          if (A.w == 0.0 || gj == g || gj == pi) continue;
          const double r[3] = {e_sub(A.x, xi[0]), e_sub(A.y, xi[1]), e_sub(A.z, xi[2])};
          const double d[3] = {B.x, B.y, B.z};
          const double a = e_add(e_add(e_sq(r[0]), e_sq(r[1])), e_sq(r[2]));
          double tm[3];
          if (bs_term_exact(r, d, a, B.w, qc, two_pi, tm)) {
            ub0[0] = e_add(ub0[0], tm[0]);
            ub0[1] = e_add(ub0[1], tm[1]);
            ub0[2] = e_add(ub0[2], tm[2]);
          }
        }
      } else {
        const double s0 = sc.shift[m - 1][0], s1 = sc.shift[m - 1][1], s2 = sc.shift[m - 1][2];
#pragma unroll 2
        for (int jj = 0; jj < n; ++jj) {
          const double4 A = tl[2 * jj], B = tl[2 * jj + 1];
          const int gj = j0 + jj;
          if (A.w == 0.0 || gj == pi) continue;
          const double r[3] = {e_sub(e_add(A.x, s0), xi[0]), e_sub(e_add(A.y, s1), xi[1]), e_sub(e_add(A.z, s2), xi[2])};
          const double d[3] = {B.x, B.y, B.z};
          const double a = e_add(e_add(e_sq(r[0]), e_sq(r[1])), e_sq(r[2]));
          double tm[3];
          if (bs_term_exact(r, d, a, B.w, qc, two_pi, tm)) {
            ubs[0] = e_add(ubs[0], tm[0]);
            ubs[1] = e_add(ubs[1], tm[1]);
            ubs[2] = e_add(ubs[2], tm[2]);
          }
        }
      }
    }
    __syncthreads();
    if (q + 2 < Q) {
      if (tid == 0) issue(q + 2);
      issued = q + 3;
    }
  }
  // A give-up leaves copies in flight: wait for them (bounded) before shared memory is
  // released.
  if (tid == 0)
    for (int q = consumed; q < issued; ++q) mbar_wait(&bar[q & 1], (unsigned)((q >> 1) & 1));
  if (!active) return;

  // solid walls: the mirror images, in mirror order, each over j ascending (timestep.f90:94-98)
  double um[3] = {0, 0, 0};
  if (sc.n_mirror) {
    const int pin_g = sc.pin[g];
    for (int m = 0; m < sc.n_mirror; ++m) {
      const bool own = mirror_skips_own(sc, pin_g, m);
      for (int j = base + 1; j <= base + pc; ++j) {
        double tm[3];
        if (mirror_term(sc, m, X, GI, nxt, T, j, g, pi, pin_g, own, xi, tm))
          for (int c = 0; c < 3; ++c) um[c] = e_add(um[c], tm[c]);
      }
    }
  }

  double gi[3], gb[3], u[3], fdot[3];
  load3(GI, T, g, gi);
  load3(GB, T, g, gb);
  local_velocity(sc, xi, gi, gb, u, fdot);
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], ub0[c]);
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], ubs[c]);
  if (sc.n_mirror)
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], um[c]);
  mf_epilogue(sc, dyn[w.x], xi, fdot, u, targets ? -1 : g);
  if (targets) {
    const int idx = w.y + tid;
    for (int c = 0; c < 3; ++c) Uout[3 * (long long)idx + c] = u[c];
    return;
  }
  store3(U, T, g, u);
}

// Few targets (a small system, or a short list of targets): the same sums with the work of
// each target spread over a block.  A block takes G targets; three warps compute the terms
// of a step -- one tile of segments of one image, 192 terms -- into shared memory while warp
// 0 adds the previous step's terms, one lane per (target, component), in slot order: the
// additions are the reference's, in the reference's order, only the terms are computed
// elsewhere.  A skipped term (empty slot, excluded neighbour, 4ac-b^2 == 0) is stored as
// +0.0: the accumulators start at +0.0 and a round-to-nearest sum is never -0.0 unless both
// operands are, so adding +0.0 leaves them bit for bit unchanged, exactly as skipping does.
constexpr int kSplitTerms = 192;  // terms per step: two per computing thread

template <int G>
__global__ void __launch_bounds__(128) k_direct_fp64_split(
    const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn, const int2 *__restrict__ work,
    const double *__restrict__ X, const double *__restrict__ GI, const double *__restrict__ GB,
    const int *__restrict__ nxt, const int *__restrict__ prv, const double4 *__restrict__ seg,
    double *__restrict__ U, long long T, const unsigned *err, const int *__restrict__ targets, int ntargets,
    double *__restrict__ Uout) {
  constexpr int TJ = kSplitTerms / G;  // segments per step
  constexpr int LD = TJ + 1;           // padded row: the adding lanes read different banks
  __shared__ double s_terms[2][3 * G][LD];
  __shared__ double s_x[G][3];
  __shared__ double s_sum[G][3][3];
  __shared__ int s_g[G], s_p[G], s_act[G], s_pin[G];
  __shared__ int s_abort;

  const int2 w = work[blockIdx.x];
  const SysConst &sc = scs[w.x];
  const int base = sc.base;
  const int pc = dyn[w.x].pcount;
  const int tid = threadIdx.x;
  if (!targets && w.y - base > pc) return;  // block-uniform: every target beyond pcount
  if (tid == 0) s_abort = (*err != 0);
  if (tid < G) {
    int g;
    bool act;
    if (targets) {
      const int idx = w.y + tid;
      g = idx < ntargets ? targets[idx] : base;
      act = idx < ntargets && g > base && g - base <= pc && nxt[g] != 0;
    } else {
      g = w.y + tid;
      act = g - base <= pc && g - base <= sc.cap && nxt[g] != 0;
    }
    s_g[tid] = g;
    s_act[tid] = act;
    s_p[tid] = act ? prv[g] : -1;
    s_pin[tid] = act && sc.pin ? sc.pin[g] : 0;
    double xi[3] = {0, 0, 0};
    if (act) load3(X, T, g, xi);
    for (int c = 0; c < 3; ++c) s_x[tid][c] = xi[c];
  }
  __syncthreads();
  if (s_abort) return;

  const int nt = (pc + TJ - 1) / TJ;
  const int Q = (1 + sc.n_shift + sc.n_mirror) * nt;  // unshifted, shifted, then mirror images
  const double qc = sc.quant_circ, two_pi = sc.two_pi;
  double acc0 = 0.0, accs = 0.0, accm = 0.0;  // adding lanes: unshifted, shifted, mirror sums
  for (int q = 0; q <= Q; ++q) {
    if (tid >= 32) {
      if (q < Q) {  // terms of step q
        const int m = q / nt, t = q % nt;
        const int n = min(TJ, pc - t * TJ);
        double(*out)[LD] = s_terms[q & 1];
        double s0 = 0, s1 = 0, s2 = 0;
        if (m > 0) {
          s0 = sc.shift[m - 1][0];
          s1 = sc.shift[m - 1][1];
          s2 = sc.shift[m - 1][2];
        }
#pragma unroll
        for (int r = 0; r < kSplitTerms / 96; ++r) {
          const int e = (tid - 32) + 96 * r;
          const int tq = e / TJ, jj = e % TJ;
          if (jj >= n) continue;
          const int gj = base + 1 + t * TJ + jj;
          double tm[3] = {0.0, 0.0, 0.0};
          if (m > sc.n_shift) {  // mirror image m - 1 - n_shift
            const int mm = m - 1 - sc.n_shift;
            if (!s_act[tq] || !mirror_term(sc, mm, X, GI, nxt, T, gj, s_g[tq], s_p[tq], s_pin[tq],
                                           mirror_skips_own(sc, s_pin[tq], mm), s_x[tq], tm))
              tm[0] = tm[1] = tm[2] = 0.0;
          } else if (s_act[tq] && gj != s_p[tq] && (m > 0 || gj != s_g[tq])) {
            const double4 A = seg[2 * (long long)gj], B = seg[2 * (long long)gj + 1];
            if (A.w != 0.0) {
              double rr[3];
              if (m == 0) {
                rr[0] = e_sub(A.x, s_x[tq][0]);
                rr[1] = e_sub(A.y, s_x[tq][1]);
                rr[2] = e_sub(A.z, s_x[tq][2]);
              } else {
                rr[0] = e_sub(e_add(A.x, s0), s_x[tq][0]);
                rr[1] = e_sub(e_add(A.y, s1), s_x[tq][1]);
                rr[2] = e_sub(e_add(A.z, s2), s_x[tq][2]);
              }
              const double d[3] = {B.x, B.y, B.z};
              const double a = e_add(e_add(e_sq(rr[0]), e_sq(rr[1])), e_sq(rr[2]));
              if (!bs_term_exact(rr, d, a, B.w, qc, two_pi, tm)) tm[0] = tm[1] = tm[2] = 0.0;
            }
          }
          out[3 * tq + 0][jj] = tm[0];
          out[3 * tq + 1][jj] = tm[1];
          out[3 * tq + 2][jj] = tm[2];
        }
      }
    } else if (q >= 1 && tid < 3 * G) {  // add the terms of step q-1, in slot order
      const int m = (q - 1) / nt, t = (q - 1) % nt;
      const int n = min(TJ, pc - t * TJ);
      const double *row = s_terms[(q - 1) & 1][tid];
      double acc = m == 0 ? acc0 : m <= sc.n_shift ? accs : accm;
#pragma unroll 8
      for (int jj = 0; jj < n; ++jj) acc = e_add(acc, row[jj]);
      if (m == 0) acc0 = acc;
      else if (m <= sc.n_shift) accs = acc;
      else accm = acc;
    }
    __syncthreads();
  }
  if (tid < 3 * G) {
    s_sum[tid / 3][tid % 3][0] = acc0;
    s_sum[tid / 3][tid % 3][1] = accs;
    s_sum[tid / 3][tid % 3][2] = accm;
  }
  __syncthreads();
  if (tid >= G || !s_act[tid]) return;
  const int g = s_g[tid];
  double xi[3] = {s_x[tid][0], s_x[tid][1], s_x[tid][2]};
  double gi[3], gb[3], u[3], fdot[3];
  load3(GI, T, g, gi);
  load3(GB, T, g, gb);
  local_velocity(sc, xi, gi, gb, u, fdot);
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], s_sum[tid][c][0]);
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], s_sum[tid][c][1]);
  if (sc.n_mirror)
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], s_sum[tid][c][2]);
  mf_epilogue(sc, dyn[w.x], xi, fdot, u, targets ? -1 : g);
  if (targets) {
    const int idx = w.y + tid;
    for (int c = 0; c < 3; ++c) Uout[3 * (long long)idx + c] = u[c];
    return;
  }
  store3(U, T, g, u);
}

template <int G>
void launch_split(cudaStream_t st, const nv_handle *h, const int2 *work, int nwork, const int *targets, int ntargets,
                  double *Uout) {
  k_direct_fp64_split<G><<<nwork, 128, 0, st>>>(h->d_sc, h->d_dyn, work, h->x, h->gi, h->gb, h->nxt, h->prv,
                                                   h->seg, h->u, h->T, h->d_err, targets, ntargets, Uout);
}

void launch_split_g(int G, cudaStream_t st, const nv_handle *h, const int2 *work, int nwork, const int *targets,
                    int ntargets, double *Uout) {
  switch (G) {
    case 1: launch_split<1>(st, h, work, nwork, targets, ntargets, Uout); break;
    case 2: launch_split<2>(st, h, work, nwork, targets, ntargets, Uout); break;
    case 4: launch_split<4>(st, h, work, nwork, targets, ntargets, Uout); break;
    default: launch_split<8>(st, h, work, nwork, targets, ntargets, Uout); break;
  }
}

}  // namespace

// Targets per block of the split direct sum for n target slots: the largest of 8, 4, 2, 1
// that still gives about four blocks per SM (1 when even that is not reached).
int direct_split_g(long long n) {
  const long long want = 4LL * n_sms_host();
  int G = 8;
  while (G > 1 && n / G < want) G /= 2;
  return G;
}

// Direct-sum targets per block in use: 64 (one thread per target, k_direct_fp64) when the
// direct systems' slots fill the GPU with at least two blocks of 64 per SM, else the split
// kernel's G.  direct_split (nv_set_direct_split) overrides the choice.
int direct_targets_per_block(const nv_handle *h, long long slots) {
  if (h->direct_split > 0) return h->direct_split;
  if (slots >= 2LL * 64 * n_sms_host()) return 64;
  return direct_split_g(slots);
}

void launch_direct(nv_handle *h) {
  if (h->n_work_direct == 0) return;
  if (h->direct_g < 64) {
    launch_split_g(h->direct_g, h->stream, h, h->d_work_split, h->n_work_split, nullptr, 0, nullptr);
    return;
  }
  const size_t smem = 2 * 2 * kDirectTJ * sizeof(double4);
  k_direct_fp64<kDirectTJ><<<h->n_work_direct, 64, smem, h->stream>>>(
      h->d_sc, h->d_dyn, h->d_work_direct, h->x, h->gi, h->gb, h->nxt, h->prv, h->seg, h->u, h->T, h->d_err);
}

// Direct sum on explicitly given buffers (used by the static-scratch entry point).
void launch_direct_raw(cudaStream_t st, const SysConst *sc, const SysDyn *dyn, const int2 *work, int nwork,
                       const double *x, const double *gi, const double *gb, const int *nxt, const int *prv,
                       const double4 *seg, double *u, long long T, unsigned *err) {
  if (nwork == 0) return;
  const size_t smem = 2 * 2 * kDirectTJ * sizeof(double4);
  k_direct_fp64<kDirectTJ><<<nwork, 64, smem, st>>>(sc, dyn, work, x, gi, gb, nxt, prv, seg, u, T, err);
}

// FP64 direct-sum velocity (the reference's BS scheme, whatever the system's own scheme) at
// listed target slots; u3 is a device buffer of 3*n doubles (point-major, listed order).
void launch_direct_targets(nv_handle *h, int sys, const int *d_targets, int n, double *d_u3) {
  if (n <= 0) return;
  const int G = direct_targets_per_block(h, n);
  std::vector<int2> w;
  for (int b = 0; b < (n + G - 1) / G; ++b) w.push_back(make_int2(sys, G * b));
  int2 *dw = nullptr;
  cudaMallocAsync((void **)&dw, w.size() * sizeof(int2), h->stream);
  cudaMemcpyAsync(dw, w.data(), w.size() * sizeof(int2), cudaMemcpyHostToDevice, h->stream);
  if (G < 64) {
    launch_split_g(G, h->stream, h, dw, (int)w.size(), d_targets, n, d_u3);
  } else {
    const size_t smem = 2 * 2 * kDirectTJ * sizeof(double4);
    k_direct_fp64<kDirectTJ><<<(int)w.size(), 64, smem, h->stream>>>(h->d_sc, h->d_dyn, dw, h->x, h->gi, h->gb,
                                                                     h->nxt, h->prv, h->seg, h->u, h->T, h->d_err,
                                                                     d_targets, n, d_u3);
  }
  cudaFreeAsync(dw, h->stream);
}
