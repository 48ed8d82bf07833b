// mixed.cu -- mixed-precision direct sum and the FP64 epilogue shared with the mixed tree walk.
//
// k_direct_mixed: one thread per (target, periodic image); the target's system's segments
// stream through shared memory in tiles by 1-D bulk copies (48-byte FP32 records: position
// hi, position lo, segment vector).  r = x_j - x_i is formed from the hi/lo split, so it is
// exact to ~1e-16 before rounding to FP32.  Each tile is summed in FP32 and the tile sums are
// added with Kahan compensation; pairs closer than near_radius are evaluated in FP64 with the
// reference expression from the FP64 segment records.  Per-image partial sums go to a buffer;
// k_mixed_combine adds them per target in FP64, in image order, to the FP64 local term and
// mutual friction (timestep.f90:79-140).
#include "handle.cuh"
#include "mixed.cuh"
#include "tma.cuh"

namespace {

constexpr int kTJ = 128;  // segments per staged tile (48 B each)
constexpr int kTB = 128;  // targets per block

template <int TJ>
__global__ void __launch_bounds__(kTB) k_direct_mixed(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                                                      const int4 *__restrict__ work, const double *__restrict__ X,
                                                      const int *__restrict__ nxt, const int *__restrict__ prv,
                                                      const float4 *__restrict__ seg32, const double4 *__restrict__ seg64,
                                                      double *__restrict__ partial, long long T, double near_factor, Fp32Guards gd,
                                                      unsigned *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float4 *tiles = reinterpret_cast<float4 *>(smem_raw);  // [2][3*TJ]
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_abort;

  const int4 w = work[blockIdx.x];  // system, image, first slot
  const SysConst &sc = scs[w.x];
  const int base = sc.base, m = w.y;
  const int pc = dyn[w.x].pcount;
  if (w.z - base > pc) return;  // block-uniform
  const int tid = threadIdx.x;
  const int g = w.z + tid;
  const bool active = (g - base <= pc) && (g - base <= sc.cap) && nxt[g] != 0;
  if (tid == 0) {
    s_abort = (*err != 0);
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (s_abort) return;

  // target, moved by minus the image shift: r = (x_j + s) - x_i = x_j - (x_i - s)
  double xi[3] = {0, 0, 0}, s[3] = {0, 0, 0};
  if (m > 0)
    for (int c = 0; c < 3; ++c) s[c] = sc.shift[m - 1][c];
  int pi_ = -1;
  if (active) {
    load3(X, T, g, xi);
    pi_ = prv[g];
  }
  float th[3], tl[3];
  for (int c = 0; c < 3; ++c) {
    const double t = xi[c] - s[c];
    th[c] = (float)t;
    tl[c] = (float)(t - (double)th[c]);
  }
  const double gq64 = sc.quant_circ / (4.0 * NV_PI);
  const float gq = (float)gq64;
  const double nr = near_factor * sc.delta;
  const float near2 = (float)(nr * nr);

  const int nt = (pc + TJ - 1) / TJ;
  auto issue = [&](int t) {
    const int n = min(TJ, pc - t * TJ);
    const int buf = t & 1;
    mbar_expect_tx(&bar[buf], (unsigned)(n * 48));
    bulk_g2s(tiles + buf * 3 * TJ, seg32 + 3 * (long long)(base + 1 + t * TJ), (unsigned)(n * 48), &bar[buf]);
  };
  if (tid == 0) {
    if (nt > 0) issue(0);
    if (nt > 1) issue(1);
  }
  int issued = nt < 2 ? nt : 2, consumed = 0;
  float hx = 0, hy = 0, hz = 0, cx = 0, cy = 0, cz = 0;  // Kahan sums over tiles
  double nx = 0, ny = 0, nz = 0;                          // FP64 near field
  for (int t = 0; t < nt; ++t) {
    const int buf = t & 1;
    const bool ok = mbar_wait(&bar[buf], (unsigned)((t >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(err, DERR_TIMEOUT);
      break;
    }
    consumed = t + 1;
    const int n = min(TJ, pc - t * TJ);
    const int j0 = base + 1 + t * TJ;
    const float4 *tl4 = tiles + buf * 3 * TJ;
    if (active) {
      // FP32 partial sums over sub-tiles of 32 segments, each added with Kahan compensation
      for (int q0 = 0; q0 < n; q0 += 32) {
        const int q1 = min(n, q0 + 32);
        float ux = 0, uy = 0, uz = 0;
#pragma unroll 4
        for (int jj = q0; jj < q1; ++jj) {
          const float4 H = tl4[3 * jj], L = tl4[3 * jj + 1], D = tl4[3 * jj + 2];
          const int gj = j0 + jj;
          if (H.w == 0.f || gj == pi_ || (m == 0 && gj == g)) continue;
          const float rx = (H.x - th[0]) + (L.x - tl[0]);
          const float ry = (H.y - th[1]) + (L.y - tl[1]);
          const float rz = (H.z - th[2]) + (L.z - tl[2]);
          const float a = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
          if (a >= near2) {
            // FP32 unless the pair is ill-conditioned in FP32: the segment subtends more than
            // 120 degrees, the target lies near its line (typically the next-but-one segment
            // along the target's own filament), or near its far end
            const float ex = rx + D.x, ey = ry + D.y, ez = rz + D.z;
            const float ee = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
            const float crx = fmaf(ry, D.z, -rz * D.y), cry = fmaf(rz, D.x, -rx * D.z), crz = fmaf(rx, D.y, -ry * D.x);
            const float cr2 = fmaf(crx, crx, fmaf(cry, cry, crz * crz));
            const float re = fmaf(rx, ex, fmaf(ry, ey, rz * ez));
            const float r1 = a * rsqrtf(a), r2 = ee * rsqrtf(ee);
            const float pp = r1 * r2;
            if (!(cr2 < gd.line * D.w * fminf(a, ee) || ee < gd.end * fmaxf(a, D.w) || pp + re < gd.angle * pp)) {
              // pp + r.e = |r x d|^2 / (pp - r.e) when r.e < 0: no cancellation either way
              const bool obtuse = re < 0.f;
              const float num = gq * (r1 + r2) * (obtuse ? pp - re : 1.f);
              const float f = __fdividef(num, pp * (obtuse ? cr2 : pp + re));  // MUFU reciprocal
              ux = fmaf(f, crx, ux);
              uy = fmaf(f, cry, uy);
              uz = fmaf(f, crz, uz);
              continue;
            }
          }
          {
            // near field and ill-conditioned pairs in FP64 from the FP64 segment records: the
            // reference's skip decision (4ac - b^2 == 0, timestep.f90:166,192) in its own
            // arithmetic, the value from the cancellation-free form
            const double4 A = seg64[2 * (long long)gj], B = seg64[2 * (long long)gj + 1];
            double r[3];
            if (m == 0) {
              r[0] = e_sub(A.x, xi[0]); r[1] = e_sub(A.y, xi[1]); r[2] = e_sub(A.z, xi[2]);
            } else {
              r[0] = e_sub(e_add(A.x, s[0]), xi[0]);
              r[1] = e_sub(e_add(A.y, s[1]), xi[1]);
              r[2] = e_sub(e_add(A.z, s[2]), xi[2]);
            }
            const double d[3] = {B.x, B.y, B.z};
            const double aa = e_add(e_add(e_sq(r[0]), e_sq(r[1])), e_sq(r[2]));
            const double bb = e_mul(2.0, dot3(r, d));
            if (e_sub(e_mul(e_mul(4.0, aa), B.w), e_mul(bb, bb)) != 0.0) {
              double tm[3];
              term64_stable(r, d, aa, gq64, tm);
              nx += tm[0];
              ny += tm[1];
              nz += tm[2];
            }
          }
        }
        kahan_add(hx, cx, ux);
        kahan_add(hy, cy, uy);
        kahan_add(hz, cz, uz);
      }
    }
    __syncthreads();
    if (t + 2 < nt) {
      if (tid == 0) issue(t + 2);
      issued = t + 3;
    }
  }
  if (tid == 0)
    for (int q = consumed; q < issued; ++q) mbar_wait(&bar[q & 1], (unsigned)((q >> 1) & 1));
  if (!active) return;
  const long long o = (long long)m * 3 * T + g;
  partial[o] = ((double)hx - (double)cx) + nx;
  partial[o + T] = ((double)hy - (double)cy) + ny;
  partial[o + 2 * T] = ((double)hz - (double)cz) + nz;
}

// Per target: u = local + partial[image 0] + sum_{images 1..n} partial[image], then MF and
// the imposed flow, all in FP64 (timestep.f90:79-92,123-140).
__global__ void k_mixed_combine(const SysConst *__restrict__ scs, const SysDyn *__restrict__ dyn,
                                const int2 *__restrict__ work, const double *__restrict__ X,
                                const double *__restrict__ GI, const double *__restrict__ GB,
                                const int *__restrict__ nxt, const double *__restrict__ partial,
                                double *__restrict__ U, long long T, int extra, const int *__restrict__ iperm,
                                const unsigned *err) {
  if (*err) return;
  const int2 w = work[blockIdx.x];
  const SysConst &sc = scs[w.x];
  const int g = w.y + threadIdx.x;
  const int k = g - sc.base;
  if (k > dyn[w.x].pcount || k > sc.cap || nxt[g] == 0) return;
  if (iperm && (sc.walk_lo > 1 || sc.walk_hi <= sc.cap)) {  // a walk range: its targets only
    const int q = iperm[g] - sc.base;
    if (q < sc.walk_lo || q >= sc.walk_hi) return;
  }
  double xi[3], gi[3], gb[3], u[3], fdot[3];
  load3(X, T, g, xi);
  load3(GI, T, g, gi);
  load3(GB, T, g, gb);
  local_velocity(sc, xi, gi, gb, u, fdot);
  double b0[3], bs[3] = {0, 0, 0};
  for (int c = 0; c < 3; ++c) b0[c] = partial[(long long)c * T + g];
  for (int e = 1; e <= extra; ++e)  // the central image's other parts, in part order
    for (int c = 0; c < 3; ++c) b0[c] += partial[((long long)(26 + e) * 3 + c) * T + g];
  for (int m = 1; m <= sc.n_shift; ++m)
    for (int c = 0; c < 3; ++c) bs[c] += partial[((long long)m * 3 + c) * T + g];
  for (int c = 0; c < 3; ++c) u[c] = e_add(e_add(u[c], b0[c]), bs[c]);
  mf_epilogue(sc, dyn[w.x], xi, fdot, u, g);
  store3(U, T, g, u);
}

}  // namespace

void launch_direct_mixed(nv_handle *h) {
  if (h->n_work_img == 0) return;
  const size_t smem = 2 * 3 * kTJ * sizeof(float4);
  k_direct_mixed<kTJ><<<h->n_work_img, kTB, smem, h->stream>>>(
      h->d_sc, h->d_dyn, h->d_work_img, h->x, h->nxt, h->prv, h->seg32, h->seg, h->partial, h->T, h->near_factor, h->guards,
      h->d_err);
}

// which: 1 = direct-sum systems, 2 = tree systems
void launch_mixed_combine(nv_handle *h, int which) {
  const int2 *wl = which == 1 ? h->d_work_direct : h->d_work_tree;
  const int n = which == 1 ? h->n_work_direct : h->n_work_tree;
  if (n == 0) return;
  const int extra = which == 2 ? h->walk_parts_used - 1 : 0;
  k_mixed_combine<<<n, h->direct_tb, 0, h->stream>>>(h->d_sc, h->d_dyn, wl, h->x, h->gi, h->gb, h->nxt, h->partial,
                                                     h->u, h->T, extra, which == 2 ? tree_iperm(h) : nullptr,
                                                     h->d_err);
}

int mixed_tiles_per_block() { return kTB; }
