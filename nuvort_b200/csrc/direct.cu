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

  double gi[3], gb[3], u[3], fdot[3];
  load3(GI, T, g, gi);
  load3(GB, T, g, gb);
  local_velocity(sc, xi, gi, gb, u, fdot);
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], ub0[c]);
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c] = e_add(u[c], ubs[c]);
  mf_epilogue(sc, dyn[w.x].t, fdot, u);
  if (targets) {
    const int idx = w.y + tid;
    for (int c = 0; c < 3; ++c) Uout[3 * (long long)idx + c] = u[c];
    return;
  }
  store3(U, T, g, u);
}

}  // namespace

void launch_direct(nv_handle *h) {
  if (h->n_work_direct == 0) return;
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
  std::vector<int2> w;
  for (int b = 0; b < (n + 63) / 64; ++b) w.push_back(make_int2(sys, 64 * b));
  int2 *dw = nullptr;
  cudaMallocAsync((void **)&dw, w.size() * sizeof(int2), h->stream);
  cudaMemcpyAsync(dw, w.data(), w.size() * sizeof(int2), cudaMemcpyHostToDevice, h->stream);
  const size_t smem = 2 * 2 * kDirectTJ * sizeof(double4);
  k_direct_fp64<kDirectTJ><<<(int)w.size(), 64, smem, h->stream>>>(h->d_sc, h->d_dyn, dw, h->x, h->gi, h->gb, h->nxt,
                                                                   h->prv, h->seg, h->u, h->T, h->d_err, d_targets, n,
                                                                   d_u3);
  cudaFreeAsync(dw, h->stream);
}
