// nuvort_oracle.cpp -- CPU oracle (test infrastructure only; see nuvort_oracle.h).
//
// A line-by-line restatement of the reference Fortran.  Every expression keeps the
// Fortran left-to-right evaluation order, and the file is compiled with
// -ffp-contract=off -fno-fast-math so that, like gfortran -O2 on x86-64 (no FMA without
// -march), each operation rounds once.  All reals are float64 (the reference builds with
// -fdefault-real-8, src/Makefile:4).  Slots are 1-based; index 0 is an unused dummy.
#include "nuvort_oracle.h"

#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Constants of src/cdata.f90:65-71, evaluated in float64.
const double pi = 3.14159265358979324;
const double one_half = 1.0 / 2.0;
const double three_twos = 3.0 / 2.0;
const double twenty_three_twelve = 23.0 / 12.0;
const double four_thirds = 4.0 / 3.0;
const double five_twelths = 5.0 / 12.0;
const double eps = 2.220446049250313e-16;  // epsilon(0.) for real(8)

thread_local std::string g_err;
thread_local long long tests_tls = 0;  // opening tests of the calling thread

struct Pt {  // type(qvort), src/cdata.f90:19-29
  double x[3], u[3], u1[3], u2[3], u_mf[3], u_sup[3];
  double curv, stretch;
  double ghosti[3], ghostb[3];
  int infront, behind, closest;
  double closestd;
  int wpinned[3];          // the wall a pinned point sits on (-1, 0 or 1 per axis)
  bool pinnedi, pinnedb;   // the segment in front / behind goes into that wall
};

struct Node {  // type node, src/tree.f90:20-32
  double posx, posy, posz, width;
  int pcount;
  Node *child[8];  // fbl, fbr, ftl, ftr, bbl, bbr, btl, btr
  double centx, centy, centz;
  double vec_cent[3];  // (centx, centy, centz), set with them
  double circ[3];
  int first;       // slot of parray(1)
  int first_next;  // parray(1)%infront at construction
  int depth;
};

inline double sq(double a) { return a * a; }

inline double dist_gen(const double *a, const double *b) {  // derivatives.f90:40-47
  return std::sqrt(sq(a[0] - b[0]) + sq(a[1] - b[1]) + sq(a[2] - b[2]));
}
inline double dist_gen_sq(const double *a, const double *b) {  // general.f90:64-71
  return sq(a[0] - b[0]) + sq(a[1] - b[1]) + sq(a[2] - b[2]);
}
inline void cross_product(const double *a, const double *b, double *c) {  // general.f90:152
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
inline double dot3(const double *a, const double *b) {  // dot_product of 3-vectors
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

struct Sys {
  nv_params p{};
  int pcount = 0;
  std::vector<Pt> f;  // f[0] unused
  double t = 0.0;
  int itime = 0;
  int recon_count = 0, remove_count = 0, insert_count = 0, loop_kills = 0;
  long long tree_eval = 0;
  long long tree_tests = 0;
  double total_length = 0.0, avg_sep = 0.0;
  // calculate_diagnostics (diagnostic.f90:9-74)
  double maxu = 0.0, maxdu = 0.0, mean_u_sup = 0.0, mean_u_mf = 0.0;
  double kappa_bar = 0.0, kappa_min = 0.0, kappa_max = 0.0;
  int diag_live = 0;
  bool diag_valid = false;
  std::vector<std::array<double, 3>> shifts;  // periodic_loop_array
  std::vector<std::array<int, 3>> mirrors;    // mirror_loop_array
  int wall_recon_count = 0;
  // event margins (the library's nv_event_margins_get): smallest |value - thr| / thr of
  // pinsert's length, premove's distance, precon's closestd and tangent dot, over the values
  // the routines below evaluate
  bool margin_on = false;
  double margin[4] = {1e300, 1e300, 1e300, 1e300};
  void note(int k, double value, double thr) {
    if (!margin_on) return;
    const double v = std::fabs(value - thr) / thr;
    if (v < margin[k]) margin[k] = v;
  }
  Node *vtree = nullptr;
  std::vector<std::unique_ptr<Node>> pool;
  std::vector<nv_event> events;
  int depth_error = 0;
  int singular_error = 0;

  // ---- boundary.f90:143-175 create_periodic_loop_array --------------------------------
  void make_shifts() {
    shifts.clear();
    for (int i = -1; i <= 1; ++i)
      for (int j = -1; j <= 1; ++j)
        for (int k = -1; k <= 1; ++k) {
          double ii, jj, kk;
          if (p.boundary[0] == NV_BC_PERIODIC) ii = i * p.box_size[0];
          else { if (i != 0) continue; ii = 0; }
          if (p.boundary[1] == NV_BC_PERIODIC) jj = j * p.box_size[1];
          else { if (j != 0) continue; jj = 0; }
          if (p.boundary[2] == NV_BC_PERIODIC) kk = k * p.box_size[2];
          else { if (k != 0) continue; kk = 0; }
          if (ii == 0 && jj == 0 && kk == 0) continue;
          shifts.push_back({ii, jj, kk});
        }
  }

  // ---- boundary.f90:180-212 create_mirror_loop_array --------------------------------------
  void make_mirrors() {
    mirrors.clear();
    for (int i = -1; i <= 1; ++i)
      for (int j = -1; j <= 1; ++j)
        for (int k = -1; k <= 1; ++k) {
          int ii, jj, kk;
          if (p.boundary[0] == NV_BC_SOLID) ii = i;
          else { if (i != 0) continue; ii = 0; }
          if (p.boundary[1] == NV_BC_SOLID) jj = j;
          else { if (j != 0) continue; jj = 0; }
          if (p.boundary[2] == NV_BC_SOLID) kk = k;
          else { if (k != 0) continue; kk = 0; }
          if (ii == 0 && jj == 0 && kk == 0) continue;
          mirrors.push_back({ii, jj, kk});
        }
  }
  // v + 2|r|(0.5 r L - v) per component: the reflection of v in the walls r names
  void reflect(const double *v, const int *r, double *out) const {
    for (int c = 0; c < 3; ++c)
      out[c] = v[c] + 2 * std::abs(r[c]) * (0.5 * r[c] * p.box_size[c] - v[c]);
  }

  void ensure_size(int n) {
    if ((int)f.size() < n + 1) {
      Pt z;
      std::memset(&z, 0, sizeof z);
      f.resize(n + 1, z);
    }
  }

  void clear_particle(int i) {  // general.f90:10-20
    Pt &q = f[i];
    for (int c = 0; c < 3; ++c) {
      q.x[c] = 0; q.u[c] = 0; q.u1[c] = 0; q.u2[c] = 0; q.ghosti[c] = 0; q.ghostb[c] = 0;
    }
    q.infront = 0; q.behind = 0; q.closest = 0; q.closestd = 0;
    q.pinnedi = false; q.pinnedb = false;
    q.wpinned[0] = q.wpinned[1] = q.wpinned[2] = 0;
  }

  // ---- boundary.f90:26-84 get_ghost_p ------------------------------------------------------
  void get_ghost_p(int i, double *gi, double *gb) {
    if (f[i].pinnedi) {
      for (int c = 0; c < 3; ++c) gb[c] = f[f[i].behind].x[c];
      reflect(f[f[i].behind].x, f[i].wpinned, gi);
    } else if (f[i].pinnedb) {
      for (int c = 0; c < 3; ++c) gi[c] = f[f[i].infront].x[c];
      reflect(f[f[i].infront].x, f[i].wpinned, gb);
    } else {
      for (int c = 0; c < 3; ++c) {
        gi[c] = f[f[i].infront].x[c];
        gb[c] = f[f[i].behind].x[c];
      }
    }
    for (int c = 0; c < 3; ++c) {
      if (p.boundary[c] != NV_BC_PERIODIC) continue;
      const double L = p.box_size[c];
      if ((f[i].x[c] - gi[c]) > (L / 2.0)) gi[c] = gi[c] + L;
      else if ((f[i].x[c] - gi[c]) < (-L / 2.0)) gi[c] = gi[c] - L;
      if ((f[i].x[c] - gb[c]) > (L / 2.0)) gb[c] = gb[c] + L;
      else if ((f[i].x[c] - gb[c]) < (-L / 2.0)) gb[c] = gb[c] - L;
    }
  }

  void ghostp() {  // boundary.f90:10-19
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= pcount; ++i) {
      if (f[i].infront == 0) continue;
      get_ghost_p(i, f[i].ghosti, f[i].ghostb);
    }
  }

  void enforce_boundary() {  // boundary.f90:91-138
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= pcount; ++i) {
      if (f[i].infront == 0) continue;
      for (int c = 0; c < 3; ++c) {
        if (p.boundary[c] != NV_BC_PERIODIC) continue;
        const double L = p.box_size[c];
        if (f[i].x[c] > (L / 2.0)) f[i].x[c] = f[i].x[c] - L;
        else if (f[i].x[c] < (-L / 2.0)) f[i].x[c] = f[i].x[c] + L;
      }
      if (f[i].pinnedi || f[i].pinnedb) {  // back onto the wall: maxloc(abs(wpinned)), first on ties
        int pc = 0;
        for (int c = 1; c < 3; ++c)
          if (std::abs(f[i].wpinned[c]) > std::abs(f[i].wpinned[pc])) pc = c;
        if (f[i].wpinned[pc] > 0) f[i].x[pc] = 0.499999999 * p.box_size[pc];
        else if (f[i].wpinned[pc] < 0) f[i].x[pc] = -0.499999999 * p.box_size[pc];
      }
    }
  }

  // ---- derivatives.f90:11-36 -----------------------------------------------------------
  void get_deriv_1(int i, double *s) const {
    const Pt &q = f[i];
    double disti = dist_gen(q.x, q.ghosti), distb = dist_gen(q.x, q.ghostb);
    for (int c = 0; c < 3; ++c)
      s[c] = distb * q.ghosti[c] + (disti - distb) * q.x[c] - disti * q.ghostb[c];
    const double den = 2.0 * distb * disti;
    for (int c = 0; c < 3; ++c) s[c] = s[c] / den;
  }
  void get_deriv_2(int i, double *s) const {
    const Pt &q = f[i];
    double disti = dist_gen(q.x, q.ghosti), distb = dist_gen(q.x, q.ghostb);
    for (int c = 0; c < 3; ++c)
      s[c] = 2.0 * (q.ghosti[c] / (disti * (disti + distb)) - q.x[c] / (disti * distb) +
                    q.ghostb[c] / (distb * (disti + distb)));
  }
  void norm_tanf(int i, double *t) const {  // general.f90:106-117
    get_deriv_1(i, t);
    double length = std::sqrt(sq(t[0]) + sq(t[1]) + sq(t[2]));
    for (int c = 0; c < 3; ++c) t[c] = t[c] / length;
  }

  // ---- timestep.f90:151-172 biot_savart --------------------------------------------------
  void biot_savart(int i, double *u) const {
    const Pt &qi = f[i];
    for (int j = 1; j <= pcount; ++j) {
      const Pt &qj = f[j];
      if (qj.infront == 0 || i == j || qi.behind == j) continue;
      if (qj.pinnedi) continue;  // the segment into the wall
      double r[3], d[3];
      for (int c = 0; c < 3; ++c) { r[c] = qj.x[c] - qi.x[c]; d[c] = qj.ghosti[c] - qj.x[c]; }
      double a_bs = dist_gen_sq(qj.x, qi.x);
      double b_bs = 2.0 * dot3(r, d);
      double c_bs = dist_gen_sq(qj.ghosti, qj.x);
      if (4 * a_bs * c_bs - b_bs * b_bs == 0) continue;
      double ub[3];
      cross_product(r, d, ub);
      const double den = (2 * pi) * (4 * a_bs * c_bs - b_bs * b_bs);
      const double fac = (2 * c_bs + b_bs) / std::sqrt(a_bs + b_bs + c_bs) - (b_bs / std::sqrt(a_bs));
      for (int c = 0; c < 3; ++c) {
        ub[c] = ub[c] * p.quant_circ / den;
        ub[c] = ub[c] * fac;
        u[c] = u[c] + ub[c];
      }
    }
  }
  // ---- timestep.f90:175-198 biot_savart_shift ---------------------------------------------
  void biot_savart_shift(int i, double *u, const double *shift) const {
    const Pt &qi = f[i];
    for (int j = 1; j <= pcount; ++j) {
      const Pt &qj = f[j];
      if (qj.infront == 0 || qi.behind == j) continue;
      if (qj.pinnedi) continue;
      double xs[3], r[3], d[3];
      for (int c = 0; c < 3; ++c) {
        xs[c] = qj.x[c] + shift[c];
        r[c] = xs[c] - qi.x[c];
        d[c] = qj.ghosti[c] - qj.x[c];
      }
      double a_bs = dist_gen_sq(qi.x, xs);
      double b_bs = 2.0 * dot3(r, d);
      double c_bs = dist_gen_sq(qj.ghosti, qj.x);
      if (4 * a_bs * c_bs - b_bs * b_bs == 0) continue;
      double ub[3];
      cross_product(r, d, ub);
      const double den = (2 * pi) * (4 * a_bs * c_bs - b_bs * b_bs);
      const double fac = (2 * c_bs + b_bs) / std::sqrt(a_bs + b_bs + c_bs) - (b_bs / std::sqrt(a_bs));
      for (int c = 0; c < 3; ++c) {
        ub[c] = ub[c] * p.quant_circ / den;
        ub[c] = ub[c] * fac;
        u[c] = u[c] + ub[c];
      }
    }
  }

  // the own-image skip of the mirror sums (timestep.f90:215-218, tree.f90:365-368)
  bool own_image_skipped(int i, int j, const int *reflect) const {
    const Pt &qi = f[i];
    const int d = (qi.wpinned[0] - reflect[0]) + (qi.wpinned[1] - reflect[1]) + (qi.wpinned[2] - reflect[2]);
    if (d == 0 && (qi.wpinned[0] + qi.wpinned[1] + qi.wpinned[2]) < 2) {
      if (qi.pinnedb && i == j) return true;
      if (qi.pinnedi && j == qi.behind) return true;
    }
    return false;
  }
  // ---- timestep.f90:201-234 biot_savart_mirror ----------------------------------------------
  void biot_savart_mirror(int i, double *u, const int *reflect_) const {
    const Pt &qi = f[i];
    for (int j = 1; j <= pcount; ++j) {
      const Pt &qj = f[j];
      if (qj.infront == 0 || qj.pinnedi) continue;
      if (own_image_skipped(i, j, reflect_)) continue;
      double s_gi_img[3], s_img[3], r[3], d[3];
      reflect(qj.x, reflect_, s_gi_img);
      reflect(qj.ghosti, reflect_, s_img);
      for (int c = 0; c < 3; ++c) { r[c] = s_img[c] - qi.x[c]; d[c] = s_gi_img[c] - s_img[c]; }
      double a_bs = dist_gen_sq(qi.x, s_img);
      double b_bs = 2.0 * dot3(r, d);
      double c_bs = dist_gen_sq(s_img, s_gi_img);
      if (4 * a_bs * c_bs - b_bs * b_bs == 0) continue;
      double ub[3];
      cross_product(r, d, ub);
      const double den = (2 * pi) * (4 * a_bs * c_bs - b_bs * b_bs);
      const double fac = (2 * c_bs + b_bs) / std::sqrt(a_bs + b_bs + c_bs) - (b_bs / std::sqrt(a_bs));
      for (int c = 0; c < 3; ++c) {
        ub[c] = ub[c] * p.quant_circ / den;
        ub[c] = ub[c] * fac;
        u[c] = u[c] + ub[c];
      }
    }
  }

  // ---- tree.f90:321-396 tree_walk_mirror -----------------------------------------------------
  // theta is width/dist whatever tree_extra_correction says: the reference computes the
  // corrected value and then overwrites it (tree.f90:354).
  void tree_walk_mirror(int i, const Node *n, const int *reflect_, double *u, long long &evals,
                        int &singular) const {
    if (n->pcount == 0) return;
    ++tests_tls;
    const Pt &qi = f[i];
    double s_img[3], s_gi_img[3], sc_[3];
    for (int c = 0; c < 3; ++c) sc_[c] = n->vec_cent[c] + n->circ[c];
    reflect(n->vec_cent, reflect_, s_gi_img);
    reflect(sc_, reflect_, s_img);
    const double dist = dist_gen(qi.x, s_img);
    const double theta = n->width / dist;
    if (n->pcount == 1 || theta < p.tree_theta) {
      if (n->pcount == 1) {
        const int j = f[n->first_next].behind;
        if (f[j].pinnedi) return;
        if (own_image_skipped(i, j, reflect_)) return;
        if (dist < eps) { singular = 1; return; }
      }
      double r[3], d[3];
      for (int c = 0; c < 3; ++c) { r[c] = s_img[c] - qi.x[c]; d[c] = s_gi_img[c] - s_img[c]; }
      double a_bs = dist * dist;
      double b_bs = 2.0 * dot3(r, d);
      double c_bs = dist_gen_sq(s_img, s_gi_img);
      if (4 * a_bs * c_bs - b_bs * b_bs < eps) return;
      double ub[3];
      cross_product(r, d, ub);
      const double den = (2 * pi) * (4 * a_bs * c_bs - b_bs * b_bs);
      const double fac = (2 * c_bs + b_bs) / std::sqrt(a_bs + b_bs + c_bs) - (b_bs / std::sqrt(a_bs));
      for (int c = 0; c < 3; ++c) {
        ub[c] = ub[c] * p.quant_circ / den;
        ub[c] = ub[c] * fac;
        u[c] = u[c] + ub[c];
      }
      ++evals;
    } else {
      for (int k = 0; k < 8; ++k) tree_walk_mirror(i, n->child[k], reflect_, u, evals, singular);
    }
  }

  // ---- tree.f90:250-316 tree_walk --------------------------------------------------------
  void tree_walk(int i, const Node *n, const double *shift, double *u, long long &evals,
                 int &singular) const {
    if (n->pcount == 0) return;
    ++tests_tls;
    const Pt &qi = f[i];
    const double cs[3] = {n->centx + shift[0], n->centy + shift[1], n->centz + shift[2]};
    double dist = std::sqrt(sq(qi.x[0] - cs[0]) + sq(qi.x[1] - cs[1]) + sq(qi.x[2] - cs[2]));
    double theta;
    if (p.tree_extra_correction) {
      double geo = std::sqrt(sq(n->centx - (n->posx + n->width / 2.0)) +
                             sq(n->centy - (n->posy + n->width / 2.0)) +
                             sq(n->centz - (n->posz + n->width / 2.0)));
      if (dist - geo > 0.0) theta = n->width / (dist - geo);
      else theta = n->width / dist;
    } else {
      theta = n->width / dist;
    }
    if (n->pcount == 1 || theta < p.tree_theta) {
      if (n->pcount == 1) {
        const int j = f[n->first_next].behind;
        const double ms = std::fmax(std::fabs(shift[0]), std::fmax(std::fabs(shift[1]), std::fabs(shift[2])));
        if (ms < eps) {
          if (j == i) return;
          if (j == qi.behind) return;
        }
        if (dist < eps) { singular = 1; return; }
      }
      double vect[3] = {cs[0] - qi.x[0], cs[1] - qi.x[1], cs[2] - qi.x[2]};
      double a_bs = dist * dist;
      double b_bs = 2.0 * dot3(vect, n->circ);
      double c_bs = dot3(n->circ, n->circ);
      if (4 * a_bs * c_bs - b_bs * b_bs < eps) return;
      double ub[3];
      cross_product(vect, n->circ, ub);
      const double den = (2 * pi) * (4 * a_bs * c_bs - b_bs * b_bs);
      const double fac = (2 * c_bs + b_bs) / std::sqrt(a_bs + b_bs + c_bs) - (b_bs / std::sqrt(a_bs));
      for (int c = 0; c < 3; ++c) {
        ub[c] = ub[c] * p.quant_circ / den;
        ub[c] = ub[c] * fac;
        u[c] = u[c] + ub[c];
      }
      ++evals;
    } else {
      for (int k = 0; k < 8; ++k) tree_walk(i, n->child[k], shift, u, evals, singular);
    }
  }

  // ---- normal_fluid.f90:83-118 get_normal_velocity -------------------------------------
  // noisey_xflow samples (load_noise :156-162) and the counter randomise_normal_fluid advances
  std::vector<double> xflow_noise;
  int xflow_noise_counter = 1;
  // laizetDNS / turbDNS grid (setup_laizet :164-190, setup_turbDNS :192-216), Fortran order
  std::vector<double> laizet_u, xp, yp, zp;
  int gn[3] = {0, 0, 0};

  double grid_u(int i, int j, int k, int c) const {  // laizet_u(i,j,k,c), 1-based
    return laizet_u[(size_t)(i - 1) + (size_t)gn[0] * ((j - 1) + (size_t)gn[1] * ((k - 1) + (size_t)gn[2] * (c - 1)))];
  }
  // nearest node by minloc(abs(x-axis)) (first on a tie), then the bracketing pair; the index
  // the reference would take below the first node (0, outside its array) wraps on a periodic
  // axis and clamps on a closed one, as the library does
  static void pair_of(const std::vector<double> &ax, double x, bool periodic, int &n, int &nn) {
    const int m = (int)ax.size();
    n = 1;
    for (int i = 2; i <= m; ++i)
      if (std::fabs(x - ax[i - 1]) < std::fabs(x - ax[n - 1])) n = i;
    if (x > ax[n - 1]) {
      nn = n + 1;
    } else {
      n = n - 1;
      nn = n + 1;
    }
    if (n < 1) n = periodic ? m : 1;
    if (nn > m) nn = periodic ? 1 : m;
  }
  void dns_interp(const double *x, double *u, bool turb) const {  // :225-338
    int nx, nnx, ny, nny, nz, nnz;
    pair_of(xp, x[0], true, nx, nnx);
    pair_of(yp, x[1], turb, ny, nny);
    pair_of(zp, x[2], true, nz, nnz);
    double xd, yd, zd;
    if (turb) {
      xd = (x[0] - xp[nx - 1]) / ((1. / 256) * p.box_size[0]);
      yd = (x[1] - yp[ny - 1]) / ((1. / 256) * p.box_size[1]);
      zd = (x[2] - zp[nz - 1]) / ((1. / 256) * p.box_size[2]);
    } else {
      xd = (x[0] - xp[nx - 1]) / ((1. / 128) * 4 * pi);
      yd = (x[1] - yp[ny - 1]) / (yp[nny - 1] - yp[ny - 1]);
      zd = (x[2] - zp[nz - 1]) / ((1. / 84) * 4 * pi / 3);
    }
    for (int c = 1; c <= 3; ++c) {
      const double c00 = grid_u(nx, ny, nz, c) * (1 - xd) + grid_u(nnx, ny, nz, c) * xd;
      const double c10 = grid_u(nx, nny, nz, c) * (1 - xd) + grid_u(nnx, nny, nz, c) * xd;
      const double c01 = grid_u(nx, ny, nnz, c) * (1 - xd) + grid_u(nnx, ny, nnz, c) * xd;
      const double c11 = grid_u(nx, nny, nnz, c) * (1 - xd) + grid_u(nnx, nny, nnz, c) * xd;
      const double c0 = c00 * (1 - yd) + c10 * yd;
      const double c1 = c01 * (1 - yd) + c11 * yd;
      u[c - 1] = c0 * (1 - zd) + c1 * zd;
    }
  }
  void get_normal_velocity(const double *x, double *u) const {
    u[0] = u[1] = u[2] = 0.0;
    switch (p.normal_velocity) {
      case NV_NF_XFLOW:
        u[0] = p.norm_vel_xflow;
        break;
      case NV_NF_UNIFORM:  // the library's extension
        u[0] = p.norm_vel_vec[0]; u[1] = p.norm_vel_vec[1]; u[2] = p.norm_vel_vec[2];
        break;
      case NV_NF_NOISEY_XFLOW:
        u[0] = xflow_noise.empty() ? 0.0 : xflow_noise[xflow_noise_counter - 1] * p.norm_vel_xflow;
        break;
      case NV_NF_SHEAR_XFLOW:
        u[0] = p.norm_vel_xflow * std::sin(2 * pi * x[2] / p.box_size[2] + t * p.norm_shear_omega);
        break;
      case NV_NF_YCHANNEL:
        u[0] = p.norm_vel_xflow * (1. - sq(2. * x[1] / p.box_size[1]));
        break;
      case NV_NF_CHANNEL: {
        double cossum = 0.0;
        for (int ii = 1; ii <= 10; ++ii) {
          const double ak = (2 * ii - 1) * (pi / 2);
          const double m1 = (ii % 2) ? -1.0 : 1.0;  // (-1)**ii
          cossum = cossum + 4 * (m1 / (ak * ak * ak)) *
                                (std::cosh(ak * 2 * x[1] / p.box_size[1]) * std::cos(ak * 2 * x[2] / p.box_size[2])) /
                                std::cosh(ak);
        }
        u[0] = p.norm_vel_xflow * (1. - sq(2 * x[2] / p.box_size[2]) + cossum) * 1.2;
        break;
      }
      case NV_NF_LAIZET_DNS:
      case NV_NF_TURB_DNS:
        if (!laizet_u.empty()) dns_interp(x, u, p.normal_velocity == NV_NF_TURB_DNS);
        break;
      default:
        break;
    }
    for (int c = 0; c < 3; ++c) u[c] = u[c] + p.super_velocity[c];
  }
  void randomise_normal_fluid() {  // :340-348
    if (p.normal_velocity == NV_NF_NOISEY_XFLOW && !xflow_noise.empty()) {
      xflow_noise_counter = xflow_noise_counter + 1;
      if (xflow_noise_counter > (int)xflow_noise.size()) xflow_noise_counter = 1;
    }
  }

  // ---- timestep.f90:49-141 calc_velocity --------------------------------------------------
  void calc_velocity(double *u, int i, int velocity, long long &evals, int &singular) {
    Pt &qi = f[i];
    double f_dot[3], f_ddot[3], cr[3], u_bs[3];
    get_deriv_1(i, f_dot);
    get_deriv_2(i, f_ddot);
    if (velocity == NV_VEL_LIA) {
      double curv = std::sqrt(dot3(f_ddot, f_ddot));
      if (curv < eps) curv = eps;
      else curv = 1.0 / curv;
      const double beta = (p.quant_circ / (4.0 * pi)) * std::log(4.6 * curv / p.corea);
      cross_product(f_dot, f_ddot, cr);
      for (int c = 0; c < 3; ++c) u[c] = beta * cr[c];
    } else {
      const double beta = (p.quant_circ / (4.0 * pi)) *
          std::log((1.1 / p.corea) * std::sqrt(dist_gen(qi.x, qi.ghosti) * dist_gen(qi.x, qi.ghostb)));
      cross_product(f_dot, f_ddot, cr);
      for (int c = 0; c < 3; ++c) u[c] = beta * cr[c];
      u_bs[0] = u_bs[1] = u_bs[2] = 0.0;
      if (velocity == NV_VEL_BS) {
        biot_savart(i, u_bs);
        for (int c = 0; c < 3; ++c) u[c] = u[c] + u_bs[c];
        u_bs[0] = u_bs[1] = u_bs[2] = 0.0;
        for (const auto &s : shifts) biot_savart_shift(i, u_bs, s.data());
        for (int c = 0; c < 3; ++c) u[c] = u[c] + u_bs[c];
        double u_mir[3] = {0.0, 0.0, 0.0};
        for (const auto &m : mirrors) biot_savart_mirror(i, u_mir, m.data());
        for (int c = 0; c < 3; ++c) u[c] = u[c] + u_mir[c];
      } else {
        const double zero[3] = {0.0, 0.0, 0.0};
        tree_walk(i, vtree, zero, u_bs, evals, singular);
        for (int c = 0; c < 3; ++c) u[c] = u[c] + u_bs[c];
        u_bs[0] = u_bs[1] = u_bs[2] = 0.0;
        for (const auto &s : shifts) tree_walk(i, vtree, s.data(), u_bs, evals, singular);
        for (int c = 0; c < 3; ++c) u[c] = u[c] + u_bs[c];
        double u_mir[3] = {0.0, 0.0, 0.0};
        for (const auto &m : mirrors) tree_walk_mirror(i, vtree, m.data(), u_mir, evals, singular);
        for (int c = 0; c < 3; ++c) u[c] = u[c] + u_mir[c];
      }
    }
    for (int c = 0; c < 3; ++c) qi.u_sup[c] = u[c];
    if (std::fabs(p.alpha[0]) > eps || std::fabs(p.alpha[1]) > eps) {
      if (t < p.normal_fluid_cutoff) {
        double u_norm[3], w[3], c1[3], c2[3], u_mf[3];
        if (t < p.t_zero_normal_fluid) get_normal_velocity(qi.x, u_norm);
        else u_norm[0] = u_norm[1] = u_norm[2] = 0.0;
        for (int c = 0; c < 3; ++c) w[c] = u_norm[c] - u[c];
        cross_product(f_dot, w, c1);
        cross_product(f_dot, c1, c2);
        for (int c = 0; c < 3; ++c) u_mf[c] = p.alpha[0] * c1[c] - p.alpha[1] * c2[c];
        for (int c = 0; c < 3; ++c) { u[c] = u[c] + u_mf[c]; qi.u_mf[c] = u_mf[c]; }
      }
    }
    for (int c = 0; c < 3; ++c) u[c] = u[c] + p.super_velocity[c];
  }

  // ---- timestep.f90:16-45 pmotion ----------------------------------------------------------
  int pmotion() {
    long long evals = 0, tests = 0;
    int singular = 0;
    const int velocity = p.velocity;
#pragma omp parallel reduction(+ : evals, tests) reduction(| : singular)
    {
      tests_tls = 0;
#pragma omp for schedule(dynamic, 16)
      for (int i = 1; i <= pcount; ++i) {
        if (f[i].infront == 0) continue;
        double u[3];
        calc_velocity(u, i, velocity, evals, singular);
        for (int c = 0; c < 3; ++c) f[i].u[c] = u[c];
      }
      tests += tests_tls;
    }
    tree_eval += evals;
    tree_tests += tests;
    if (singular) { singular_error = 1; return NV_ERR_SINGULAR; }
    const double dt = p.dt;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= pcount; ++i) {
      Pt &q = f[i];
      if (q.infront == 0) continue;
      const double m1 = std::fmax(std::fabs(q.u1[0]), std::fmax(std::fabs(q.u1[1]), std::fabs(q.u1[2])));
      const double m2 = std::fmax(std::fabs(q.u2[0]), std::fmax(std::fabs(q.u2[1]), std::fabs(q.u2[2])));
      if (m1 == 0) {
        for (int c = 0; c < 3; ++c) q.x[c] = q.x[c] + dt * q.u[c];
      } else if (m2 == 0) {
        for (int c = 0; c < 3; ++c)
          q.x[c] = q.x[c] + three_twos * dt * q.u[c] - one_half * dt * q.u1[c];
      } else {
        for (int c = 0; c < 3; ++c)
          q.x[c] = q.x[c] + twenty_three_twelve * dt * q.u[c] - four_thirds * dt * q.u1[c] +
                   five_twelths * dt * q.u2[c];
      }
      for (int c = 0; c < 3; ++c) { q.u2[c] = q.u1[c]; q.u1[c] = q.u[c]; }
    }
    randomise_normal_fluid();  // timestep.f90:44
    return NV_OK;
  }

  // ---- tree.f90:38-157 construct_tree / build_tree / new_tree ------------------------------
  Node *alloc_node() {
    pool.emplace_back(new Node());
    Node *n = pool.back().get();
    std::memset(n, 0, sizeof *n);
    return n;
  }
  void new_tree(Node *&out, double posx, double posy, double posz, double width,
                const std::vector<int> &parray, int depth) {
    Node *n = alloc_node();
    out = n;
    n->posx = posx; n->posy = posy; n->posz = posz; n->width = width; n->depth = depth;
    n->centx = 0.0; n->centy = 0.0; n->centz = 0.0;
    n->circ[0] = n->circ[1] = n->circ[2] = 0.0;
    std::vector<int> mine;
    int counter = 0;
    for (int k : parray) {
      const Pt &q = f[k];
      if (q.infront == 0) continue;
      if (q.pinnedi) continue;  // the segment into the wall is not part of the tree
      if ((q.x[0] >= posx) && (q.x[0] < (posx + width)) && (q.x[1] >= posy) &&
          (q.x[1] < (posy + width)) && (q.x[2] >= posz) && (q.x[2] < (posz + width))) {
        counter = counter + 1;
        mine.push_back(k);
        n->centx = n->centx + q.x[0];
        n->centy = n->centy + q.x[1];
        n->centz = n->centz + q.x[2];
        n->circ[0] = n->circ[0] + q.ghosti[0] - q.x[0];
        n->circ[1] = n->circ[1] + q.ghosti[1] - q.x[1];
        n->circ[2] = n->circ[2] + q.ghosti[2] - q.x[2];
      }
    }
    if (counter != 0) {
      n->centx = n->centx / counter;
      n->centy = n->centy / counter;
      n->centz = n->centz / counter;
    }
    n->vec_cent[0] = n->centx; n->vec_cent[1] = n->centy; n->vec_cent[2] = n->centz;
    n->pcount = counter;
    if (counter > 0) { n->first = mine[0]; n->first_next = f[mine[0]].infront; }
    build_tree(n, mine);
  }
  void build_tree(Node *n, const std::vector<int> &parray) {
    if (n->pcount > 1) {
      if (n->depth >= NV_TREE_MAX_DEPTH) { depth_error = 1; n->pcount = 1; return; }
      const double h = n->width / 2;
      const double w = n->width / 2.0;
      const int d = n->depth + 1;
      new_tree(n->child[0], n->posx, n->posy, n->posz, w, parray, d);
      new_tree(n->child[1], n->posx + h, n->posy, n->posz, w, parray, d);
      new_tree(n->child[2], n->posx, n->posy, n->posz + h, w, parray, d);
      new_tree(n->child[3], n->posx + h, n->posy, n->posz + h, w, parray, d);
      new_tree(n->child[4], n->posx, n->posy + h, n->posz, w, parray, d);
      new_tree(n->child[5], n->posx + h, n->posy + h, n->posz, w, parray, d);
      new_tree(n->child[6], n->posx, n->posy + h, n->posz + h, w, parray, d);
      new_tree(n->child[7], n->posx + h, n->posy + h, n->posz + h, w, parray, d);
    }
  }
  int construct_tree() {
    empty_tree();
    const double bsize = std::fmax(p.box_size[0], std::fmax(p.box_size[1], p.box_size[2]));
    Node *r = alloc_node();
    vtree = r;
    r->posx = -bsize / 2.0; r->posy = -bsize / 2.0; r->posz = -bsize / 2.0;
    r->width = bsize;
    r->pcount = pcount;
    r->depth = 0;
    double sx = 0, sy = 0, sz = 0;
    int cnt = 0;
    for (int i = 1; i <= pcount; ++i) {
      if (f[i].infront > 0) { sx = sx + f[i].x[0]; sy = sy + f[i].x[1]; sz = sz + f[i].x[2]; ++cnt; }
    }
    r->centx = sx / cnt; r->centy = sy / cnt; r->centz = sz / cnt;
    r->vec_cent[0] = r->centx; r->vec_cent[1] = r->centy; r->vec_cent[2] = r->centz;
    r->circ[0] = r->circ[1] = r->circ[2] = 0.0;
    r->first = 1;
    r->first_next = pcount >= 1 ? f[1].infront : 0;
    std::vector<int> all(pcount);
    for (int i = 0; i < pcount; ++i) all[i] = i + 1;
    depth_error = 0;
    build_tree(r, all);
    return depth_error ? NV_ERR_TREE_DEPTH : NV_OK;
  }
  void empty_tree() {
    vtree = nullptr;
    pool.clear();
  }
  void dump(const Node *n, std::vector<or_tree_node> &out) const {
    if (n->pcount == 0) return;
    or_tree_node r;
    r.pos[0] = n->posx; r.pos[1] = n->posy; r.pos[2] = n->posz; r.width = n->width;
    r.cent[0] = n->centx; r.cent[1] = n->centy; r.cent[2] = n->centz;
    for (int c = 0; c < 3; ++c) r.circ[c] = n->circ[c];
    r.pcount = n->pcount; r.depth = n->depth;
    r.leaf = n->pcount == 1 ? n->first : 0;
    r.first_next = n->first_next;
    out.push_back(r);
    if (n->pcount > 1 && n->child[0])
      for (int k = 0; k < 8; ++k) dump(n->child[k], out);
  }

  // ---- tree.f90:190-244 pclose_tree / closest_tree -----------------------------------------
  void closest_tree(int i, const Node *n) {
    if (f[i].infront == 0) return;
    if (n->pcount == 0) return;
    double dist = std::sqrt(sq(f[i].x[0] - n->centx) + sq(f[i].x[1] - n->centy) + sq(f[i].x[2] - n->centz));
    double theta = n->width / dist;
    if (n->pcount == 1 || theta < .5) {
      if (dist < f[i].closestd) {
        const int j = f[n->first_next].behind;
        if (n->pcount > 1) {
          f[i].closest = 0;
        } else if ((i != j) && (f[i].infront != j) && (f[i].behind != j)) {
          if (f[j].pinnedi || f[j].pinnedb) {
            // pinned: nothing
          } else {
            f[i].closest = j;
            f[i].closestd = dist;
          }
        }
      }
    } else {
      for (int k = 0; k < 8; ++k) closest_tree(i, n->child[k]);
    }
  }
  void pclose_tree() {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 1; i <= pcount; ++i) {
      f[i].closestd = 100.0;
      if (f[i].infront == 0) continue;
      if (f[i].pinnedi || f[i].pinnedb) continue;
      closest_tree(i, vtree);
    }
  }
  // ---- line.f90:135-160 pclose ----------------------------------------------------------------
  void pclose() {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 1; i <= pcount; ++i) {
      if (f[i].infront == 0) continue;
      f[i].closestd = 100.0;
      if (f[i].pinnedi || f[i].pinnedb) continue;
      for (int j = 1; j <= pcount; ++j) {
        if (f[j].infront == 0) continue;
        if ((i != j) && (f[i].infront != j) && (f[i].behind != j) && !f[j].pinnedi && !f[j].pinnedb) {
          const double dist = dist_gen(f[i].x, f[j].x);
          if (dist < f[i].closestd) { f[i].closest = j; f[i].closestd = dist; }
        }
      }
    }
  }

  // ---- reconnection.f90:155-182 loop_killer -------------------------------------------------
  void loop_killer(int particle) {
    int counter = 1;
    int next = particle;
    for (int i = 1; i <= pcount; ++i) {
      if (f[next].pinnedi || f[next].pinnedb) return;
      next = f[next].infront;
      if (next == particle) break;
      counter = counter + 1;
    }
    if (counter < 4) {
      events.push_back(nv_event{itime, NV_EV_LOOPKILL, particle, counter});
      ++loop_kills;
      next = particle;
      for (int i = 1; i <= pcount; ++i) {
        const int store_next = f[next].infront;
        clear_particle(next);
        next = store_next;
        if (next == particle) break;
      }
    }
  }

  // ---- diagnostic.f90:9-74 calculate_diagnostics ------------------------------------------
  void calculate_diagnostics() {
    ghostp();
    // velocity_info (:22-34): maxval/sum over every slot of f(:), divided by the live count
    int live = 0;
    for (int i = 1; i <= pcount; ++i) live += f[i].infront > 0;
    double mu = -1.7976931348623157e308, mdu = -1.7976931348623157e308, ssup = 0.0, smf = 0.0;
    for (int i = 1; i <= pcount; ++i) {
      const Pt &q = f[i];
      const double a = std::sqrt(q.u[0] * q.u[0] + q.u[1] * q.u[1] + q.u[2] * q.u[2]);
      if (a > mu) mu = a;
      const double b = std::sqrt((q.u1[0] - q.u2[0]) * (q.u1[0] - q.u2[0]) + (q.u1[1] - q.u2[1]) * (q.u1[1] - q.u2[1]) +
                                 (q.u1[2] - q.u2[2]) * (q.u1[2] - q.u2[2]));
      if (b > mdu) mdu = b;
    }
    for (int i = 1; i <= pcount; ++i)
      ssup = ssup + std::sqrt(f[i].u_sup[0] * f[i].u_sup[0] + f[i].u_sup[1] * f[i].u_sup[1] +
                              f[i].u_sup[2] * f[i].u_sup[2]);
    for (int i = 1; i <= pcount; ++i)
      smf = smf + std::sqrt(f[i].u_mf[0] * f[i].u_mf[0] + f[i].u_mf[1] * f[i].u_mf[1] + f[i].u_mf[2] * f[i].u_mf[2]);
    maxu = mu;
    maxdu = mdu;
    mean_u_sup = ssup / live;
    mean_u_mf = smf / live;
    // curv_info (:37-57): curvature (general.f90:53-61) per point, 0 for empty slots
    double sum = 0.0, kmax = -1.7976931348623157e308, kmin = 1.7976931348623157e308;
    for (int i = 1; i <= pcount; ++i) {
      double curvi = 0.0;
      if (f[i].infront != 0) {
        double fddot[3];
        get_deriv_2(i, fddot);
        curvi = std::sqrt(dot3(fddot, fddot));
      }
      f[i].curv = curvi;
    }
    for (int i = 1; i <= pcount; ++i) sum = sum + f[i].curv;
    for (int i = 1; i <= pcount; ++i) {
      if (f[i].curv > kmax) kmax = f[i].curv;
      if (f[i].curv > 0.0 && f[i].curv < kmin) kmin = f[i].curv;
    }
    kappa_bar = sum / live;
    kappa_max = kmax;
    kappa_min = kmin;
    // stretching_rate (:60-74): u . s''
    for (int i = 1; i <= pcount; ++i) {
      if (f[i].infront == 0) {
        f[i].stretch = 0.0;
      } else {
        double s_ddot[3];
        get_deriv_2(i, s_ddot);
        f[i].stretch = dot3(f[i].u, s_ddot);
      }
    }
    diag_live = live;
    diag_valid = true;
  }

  // ---- line.f90:18-96 pinsert -----------------------------------------------------------------
  int pinsert() {
    int live = 0;
    for (int i = 1; i <= pcount; ++i) live += f[i].infront > 0;
    if (live == 0) return NV_ERR_EMPTY;
    const int old_pcount = pcount;
    total_length = 0.0;
    for (int i = 1; i <= old_pcount; ++i) {
      if (f[i].infront == 0) continue;
      if (f[i].pinnedi) continue;
      const double disti = dist_gen(f[i].x, f[i].ghosti);
      total_length = total_length + disti;
      note(0, disti, p.delta);
      if (disti > p.delta) {
        int par_new = 0;
        for (int k = 1; k <= pcount; ++k) if (f[k].infront == 0) { par_new = k; break; }
        if (par_new == 0) {
          ensure_size(pcount + 1);
          par_new = pcount + 1;
          pcount = pcount + 1;
          clear_particle(par_new);
        }
        double f_ddot[3];
        get_deriv_2(i, f_ddot);
        double curv = std::sqrt(dot3(f_ddot, f_ddot));
        Pt &qn = f[par_new];
        if (curv > 1E-5) {
          curv = 1.0 / curv;
          if (curv * curv - 0.25 * (disti * disti) > 0.0) {
            const double s = (std::sqrt(curv * curv - 0.25 * (disti * disti)) - curv) * curv;
            for (int c = 0; c < 3; ++c)
              qn.x[c] = 0.5 * (f[i].x[c] + f[i].ghosti[c]) + s * f_ddot[c];
          } else {
            for (int c = 0; c < 3; ++c) qn.x[c] = 0.5 * (f[i].x[c] + f[i].ghosti[c]);
          }
        } else {
          for (int c = 0; c < 3; ++c) qn.x[c] = 0.5 * (f[i].x[c] + f[i].ghosti[c]);
        }
        for (int c = 0; c < 3; ++c) qn.u[c] = 0.5 * (f[i].u[c] + f[f[i].infront].u[c]);
        for (int c = 0; c < 3; ++c) { qn.u1[c] = 0.0; qn.u2[c] = 0.0; }
        qn.pinnedi = false; qn.pinnedb = false;
        qn.wpinned[0] = qn.wpinned[1] = qn.wpinned[2] = 0;
        qn.behind = i;
        qn.infront = f[i].infront;
        get_ghost_p(par_new, qn.ghosti, qn.ghostb);
        const int nx = f[i].infront;
        f[nx].behind = par_new;
        get_ghost_p(nx, f[nx].ghosti, f[nx].ghostb);
        f[i].infront = par_new;
        get_ghost_p(i, f[i].ghosti, f[i].ghostb);
        events.push_back(nv_event{itime, NV_EV_INSERT, i, par_new});
        ++insert_count;
      }
    }
    int empty = 0;
    for (int i = 1; i <= pcount; ++i) empty += f[i].infront == 0;
    avg_sep = total_length / (old_pcount - empty);
    return NV_OK;
  }

  // ---- line.f90:102-130 premove ---------------------------------------------------------------
  void premove() {
    for (int i = 1; i <= pcount; ++i) {
      if (f[i].infront == 0) continue;
      if (f[i].pinnedi) continue;
      const int infront = f[i].infront;
      if (f[infront].pinnedi) continue;
      const double distii = dist_gen(f[i].x, f[f[infront].infront].x);
      note(1, distii, .99 * p.delta);
      if (distii < .99 * p.delta) {
        const int tinfront = f[f[i].infront].infront;
        f[tinfront].behind = i;
        f[i].infront = tinfront;
        clear_particle(infront);
        events.push_back(nv_event{itime, NV_EV_REMOVE, i, infront});
        loop_killer(i);
        remove_count = remove_count + 1;
      }
      clear_wall_pair(i);
    }
  }
  // two wall points next to each other cleared together (line.f90:125-127,
  // reconnection.f90:71-75); logged as one event with the number of points cleared
  bool clear_wall_pair(int i) {
    if (!f[i].pinnedb) return false;  // (a cleared i is not pinned: f(0) is never read)
    const int nx = f[i].infront;
    if (!f[nx].pinnedi) return false;
    events.push_back(nv_event{itime, NV_EV_CLEAR, i, nx == i ? 1 : 2});
    clear_particle(nx);
    clear_particle(i);
    return true;
  }

  // ---- reconnection.f90:66-150 wall_recon ------------------------------------------------------
  void wall_recon() {
    for (int i = 1; i <= pcount; ++i) {
      if (f[i].infront == 0) continue;
      clear_wall_pair(i);
      if (f[i].pinnedi || f[i].pinnedb) continue;
      for (int a = 0; a < 3; ++a) {  // the x, y and z blocks in turn
        if (p.boundary[a] != NV_BC_SOLID) continue;
        int side = 0;
        if (f[i].x[a] > 0.5 * (p.box_size[a] - p.delta)) side = 1;
        else if (f[i].x[a] < -0.5 * (p.box_size[a] - p.delta)) side = -1;
        if (side == 0) continue;
        const int pari = f[i].infront, parb = f[i].behind;
        f[pari].pinnedb = true; f[pari].behind = pari;
        for (int c = 0; c < 3; ++c) f[pari].wpinned[c] = c == a ? side : 0;
        f[parb].pinnedi = true; f[parb].infront = parb;
        for (int c = 0; c < 3; ++c) f[parb].wpinned[c] = c == a ? side : 0;
        clear_particle(i);
        int cleared = 1;
        if (f[pari].pinnedi && f[pari].pinnedb) { clear_particle(pari); ++cleared; }
        if (f[parb].pinnedi && f[parb].pinnedb) { clear_particle(parb); ++cleared; }
        events.push_back(nv_event{itime, NV_EV_WALL, i, cleared});
        wall_recon_count = wall_recon_count + 1;
      }
    }
  }

  // ---- reconnection.f90:11-61 precon ----------------------------------------------------------
  void precon() {
    for (int i = 1; i <= pcount; ++i) {
      if (f[i].infront == 0) continue;
      const int pari = f[i].infront, parb = f[i].behind;
      if (f[i].closestd > eps) note(2, f[i].closestd, p.delta / 2.0);
      if ((f[i].closestd < p.delta / 2.0) && (f[i].closestd > eps)) {
        const int j = f[i].closest;
        if (j == pari) continue;
        if (j == parb) continue;
        if (j == 0) continue;
        if (f[j].infront == 0) continue;
        const int parjb = f[j].behind;
        double t1[3], t2[3];
        norm_tanf(i, t1);
        norm_tanf(j, t2);
        const double dot_val = dot3(t1, t2);
        note(3, dot_val, 0.9);
        if (dot_val > 0.9) {
          // parallel: no reconnection
        } else {
          const double l_before = dist_gen(f[i].x, f[i].ghosti) + dist_gen(f[i].x, f[i].ghostb) +
                                  dist_gen(f[j].x, f[j].ghosti) + dist_gen(f[j].x, f[j].ghostb);
          const double l_after = dist_gen(f[i].x, f[i].ghostb) + dist_gen(f[i].x, f[j].x) +
                                 dist_gen(f[j].x, f[j].ghosti) + dist_gen(f[pari].x, f[parjb].x);
          if (l_after <= l_before) {
            recon_count = recon_count + 1;
            events.push_back(nv_event{itime, NV_EV_RECON, i, j});
            f[parjb].infront = pari;
            f[pari].behind = parjb;
            f[i].infront = j;
            f[j].behind = i;
            loop_killer(pari);
            loop_killer(i);
          }
        }
      }
    }
  }

  int nan_finder() const {  // general.f90:172-190
    for (int i = 1; i <= pcount; ++i)
      for (int c = 0; c < 3; ++c)
        if (std::isnan(f[i].x[c])) return NV_ERR_NAN;
    return NV_OK;
  }

  // ---- run.f90:24-65, one iteration ----------------------------------------------------------
  int one_step() {
    itime = itime + 1;
    ghostp();
    int rc;
    if (p.tree_theta > 0) { if ((rc = construct_tree()) != NV_OK) return rc; }
    if ((rc = pmotion()) != NV_OK) return rc;
    if ((rc = pinsert()) != NV_OK) return rc;
    if (itime % p.recon_shots == 0) {
      if (p.tree_theta > 0) pclose_tree();
      else pclose();
      precon();
      wall_recon();
      premove();
    }
    enforce_boundary();
    t = t + p.dt;
    if (p.tree_theta > 0) empty_tree();
    if (p.nan_test) { if ((rc = nan_finder()) != NV_OK) return rc; }
    return NV_OK;
  }
};

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

}  // namespace

struct or_handle {
  Sys s;
};

extern "C" {

int or_create(const nv_params *p, or_handle **out) {
  if (!p || !out) return fail(NV_ERR_ARG, "null argument");
  auto *h = new or_handle();
  h->s.p = *p;
  h->s.make_shifts();
  h->s.make_mirrors();
  h->s.ensure_size(0);
  *out = h;
  return NV_OK;
}

int or_destroy(or_handle *h) {
  delete h;
  return NV_OK;
}

int or_upload(or_handle *h, const nv_host_state *st) {
  if (!h || !st || !st->x || !st->infront || !st->behind || st->pcount < 0)
    return fail(NV_ERR_ARG, "upload: missing x/infront/behind");
  Sys &s = h->s;
  s.pcount = st->pcount;
  s.f.clear();
  s.ensure_size(s.pcount);
  for (int k = 1; k <= s.pcount; ++k) {
    Pt &q = s.f[k];
    for (int c = 0; c < 3; ++c) {
      const int o = 3 * (k - 1) + c;
      q.x[c] = st->x[o];
      q.u[c] = st->u ? st->u[o] : 0.0;
      q.u1[c] = st->u1 ? st->u1[o] : 0.0;
      q.u2[c] = st->u2 ? st->u2[o] : 0.0;
      q.ghosti[c] = st->ghosti ? st->ghosti[o] : 0.0;
      q.ghostb[c] = st->ghostb ? st->ghostb[o] : 0.0;
    }
    q.infront = st->infront[k - 1];
    q.behind = st->behind[k - 1];
    q.closest = st->closest ? st->closest[k - 1] : 0;
    q.closestd = st->closestd ? st->closestd[k - 1] : 0.0;
    for (int c = 0; c < 3; ++c) q.wpinned[c] = st->wpinned ? st->wpinned[3 * (k - 1) + c] : 0;
    q.pinnedi = st->pinnedi && st->pinnedi[k - 1];
    q.pinnedb = st->pinnedb && st->pinnedb[k - 1];
  }
  s.events.clear();
  return NV_OK;
}

int or_download(or_handle *h, nv_host_state *st, int32_t cap) {
  if (!h || !st) return fail(NV_ERR_ARG, "null argument");
  Sys &s = h->s;
  if (s.pcount > cap) return fail(NV_ERR_ARG, "download: capacity too small");
  st->pcount = s.pcount;
  for (int k = 1; k <= s.pcount; ++k) {
    const Pt &q = s.f[k];
    for (int c = 0; c < 3; ++c) {
      const int o = 3 * (k - 1) + c;
      if (st->x) st->x[o] = q.x[c];
      if (st->u) st->u[o] = q.u[c];
      if (st->u1) st->u1[o] = q.u1[c];
      if (st->u2) st->u2[o] = q.u2[c];
      if (st->ghosti) st->ghosti[o] = q.ghosti[c];
      if (st->ghostb) st->ghostb[o] = q.ghostb[c];
    }
    if (st->infront) st->infront[k - 1] = q.infront;
    if (st->behind) st->behind[k - 1] = q.behind;
    if (st->closest) st->closest[k - 1] = q.closest;
    if (st->closestd) st->closestd[k - 1] = q.closestd;
    for (int c = 0; c < 3; ++c)
      if (st->wpinned) st->wpinned[3 * (k - 1) + c] = q.wpinned[c];
    if (st->pinnedi) st->pinnedi[k - 1] = q.pinnedi;
    if (st->pinnedb) st->pinnedb[k - 1] = q.pinnedb;
  }
  return NV_OK;
}

int or_set_clock(or_handle *h, double t, int32_t itime) {
  h->s.t = t;
  h->s.itime = itime;
  return NV_OK;
}

int or_counters_get(or_handle *h, nv_counters *c) {
  const Sys &s = h->s;
  c->pcount = s.pcount;
  int live = 0;
  for (int i = 1; i <= s.pcount; ++i) live += s.f[i].infront > 0;
  c->live = live;
  c->recon_count = s.recon_count;
  c->remove_count = s.remove_count;
  c->insert_count = s.insert_count;
  c->loop_kills = s.loop_kills;
  c->wall_recon_count = s.wall_recon_count;
  c->tree_eval = s.tree_eval;
  c->tree_tests = s.tree_tests;
  c->itime = s.itime;
  c->n_events = (int32_t)s.events.size();
  c->t = s.t;
  return NV_OK;
}

int or_set_normal_fluid_noise(or_handle *h, const double *noise, int32_t n) {
  if (!h || !noise || n < 1) return fail(NV_ERR_ARG, "bad noise");
  h->s.xflow_noise.assign(noise, noise + n);
  h->s.xflow_noise_counter = 1;
  return NV_OK;
}

int or_set_normal_fluid_grid(or_handle *h, const double *u, int32_t nx, int32_t ny, int32_t nz, const double *yp) {
  Sys &s = h->s;
  const bool laizet = s.p.normal_velocity == NV_NF_LAIZET_DNS;
  const size_t nn = (size_t)nx * ny * nz;
  s.laizet_u.assign(u, u + 3 * nn);
  if (laizet)
    for (auto &v : s.laizet_u) v = v / 2.;  // setup_laizet: laizet_u=laizet_u/2.
  s.gn[0] = nx; s.gn[1] = ny; s.gn[2] = nz;
  s.xp.resize(nx); s.yp.resize(ny); s.zp.resize(nz);
  if (laizet) {
    for (int i = 1; i <= nx; ++i) s.xp[i - 1] = (i - 1) * (1. / 128) * 4 * pi - 2 * pi;
    for (int j = 0; j < ny; ++j) s.yp[j] = yp[j];
    for (int i = 1; i <= nz; ++i) s.zp[i - 1] = (i - 1) * (1. / 84) * 4 * pi / 3 - 4 * pi / 6;
  } else {
    for (int i = 1; i <= nx; ++i) s.xp[i - 1] = (i - 1) * (1. / 256) * s.p.box_size[0] - s.p.box_size[0] / 2.;
    for (int i = 1; i <= ny; ++i) s.yp[i - 1] = (i - 1) * (1. / 256) * s.p.box_size[1] - s.p.box_size[1] / 2.;
    for (int i = 1; i <= nz; ++i) s.zp[i - 1] = (i - 1) * (1. / 256) * s.p.box_size[2] - s.p.box_size[2] / 2.;
  }
  return NV_OK;
}

int or_calculate_diagnostics(or_handle *h) {
  h->s.calculate_diagnostics();
  return NV_OK;
}

int or_ts_row_get(or_handle *h, nv_ts_row *row) {  // the values print_info writes (output.f90:20-44)
  const Sys &s = h->s;
  if (!s.diag_valid) return fail(NV_ERR_STATE, "no diagnostics yet");
  std::memset(row, 0, sizeof *row);
  row->itime = s.itime;
  row->live = s.diag_live;
  row->recon_count = s.recon_count;
  row->wall_recon_count = s.wall_recon_count;
  row->remove_count = s.remove_count;
  row->tree_eval = s.tree_eval;
  row->t = s.t;
  row->delta = s.p.delta;
  row->avg_sep = s.avg_sep;
  row->total_length = s.total_length;
  row->maxu = s.maxu;
  row->maxdu = s.maxdu;
  row->mean_u_sup = s.mean_u_sup;
  row->mean_u_mf = s.mean_u_mf;
  row->kappa_bar = s.kappa_bar;
  row->kappa_min = s.kappa_min;
  row->kappa_max = s.kappa_max;
  return NV_OK;
}

int or_download_full(or_handle *h, nv_full_state *st, int32_t cap) {
  if (!h || !st) return fail(NV_ERR_ARG, "null argument");
  const Sys &s = h->s;
  if (s.pcount > cap) return fail(NV_ERR_ARG, "download: capacity too small");
  st->pcount = s.pcount;
  for (int k = 1; k <= s.pcount; ++k) {
    const Pt &q = s.f[k];
    for (int c = 0; c < 3; ++c) {
      const int o = 3 * (k - 1) + c;
      if (st->x) st->x[o] = q.x[c];
      if (st->u) st->u[o] = q.u[c];
      if (st->u1) st->u1[o] = q.u1[c];
      if (st->u2) st->u2[o] = q.u2[c];
      if (st->u_mf) st->u_mf[o] = q.u_mf[c];
      if (st->u_sup) st->u_sup[o] = q.u_sup[c];
      if (st->ghosti) st->ghosti[o] = q.ghosti[c];
      if (st->ghostb) st->ghostb[o] = q.ghostb[c];
    }
    if (st->curv) st->curv[k - 1] = q.curv;
    if (st->stretch) st->stretch[k - 1] = q.stretch;
    if (st->infront) st->infront[k - 1] = q.infront;
    if (st->behind) st->behind[k - 1] = q.behind;
    if (st->closest) st->closest[k - 1] = q.closest;
    if (st->closestd) st->closestd[k - 1] = q.closestd;
    for (int c = 0; c < 3; ++c)
      if (st->wpinned) st->wpinned[3 * (k - 1) + c] = q.wpinned[c];
    if (st->pinnedi) st->pinnedi[k - 1] = q.pinnedi;
    if (st->pinnedb) st->pinnedb[k - 1] = q.pinnedb;
  }
  return NV_OK;
}

int or_upload_full(or_handle *h, const nv_full_state *st) {
  nv_host_state hs{st->pcount, st->x, st->u, st->u1, st->u2, st->ghosti, st->ghostb,
                   st->infront, st->behind, st->closest, st->closestd, st->wpinned, st->pinnedi, st->pinnedb};
  int rc = or_upload(h, &hs);
  if (rc) return rc;
  for (int k = 1; k <= st->pcount; ++k) {
    Pt &q = h->s.f[k];
    for (int c = 0; c < 3; ++c) {
      q.u_mf[c] = st->u_mf ? st->u_mf[3 * (k - 1) + c] : 0.0;
      q.u_sup[c] = st->u_sup ? st->u_sup[3 * (k - 1) + c] : 0.0;
    }
    q.curv = st->curv ? st->curv[k - 1] : 0.0;
    q.stretch = st->stretch ? st->stretch[k - 1] : 0.0;
  }
  return NV_OK;
}

// printf (output.f90:47-70): the unformatted stream file, one write per statement.
int or_write_snapshot(or_handle *h, const char *path) {
  const Sys &s = h->s;
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return fail(NV_ERR_IO, "cannot open file");
  const int32_t pc = s.pcount;
  std::fwrite(&s.t, sizeof(double), 1, fp);                                        // write(98) t
  std::fwrite(&pc, sizeof(int32_t), 1, fp);                                        // write(98) pcount
  for (int c = 0; c < 3; ++c)                                                      // f(:)%x(1..3)
    for (int i = 1; i <= pc; ++i) std::fwrite(&s.f[i].x[c], sizeof(double), 1, fp);
  for (int i = 1; i <= pc; ++i) std::fwrite(&s.f[i].infront, sizeof(int32_t), 1, fp);  // f(:)%infront
  for (int c = 0; c < 3; ++c)                                                      // f(:)%u(1..3)
    for (int i = 1; i <= pc; ++i) std::fwrite(&s.f[i].u[c], sizeof(double), 1, fp);
  for (int c = 0; c < 3; ++c)                                                      // f(:)%u_mf(1..3)
    for (int i = 1; i <= pc; ++i) std::fwrite(&s.f[i].u_mf[c], sizeof(double), 1, fp);
  for (int i = 1; i <= pc; ++i) std::fwrite(&s.f[i].curv, sizeof(double), 1, fp);     // f(:)%curv
  for (int i = 1; i <= pc; ++i) std::fwrite(&s.f[i].stretch, sizeof(double), 1, fp);  // f(:)%stretch
  std::fclose(fp);
  return NV_OK;
}

// data_dump (output.f90:85-94) as gfortran writes it: each write statement one sequential
// record, a 4-byte byte count before and after; f element after element, component after
// component (type qvort, cdata.f90:19-29; real(8), integer(4), logical(4)).
int or_write_dump(or_handle *h, const char *path) {
  const Sys &s = h->s;
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return fail(NV_ERR_IO, "cannot open file");
  auto rec_int = [&](int32_t v) {
    const int32_t m = 4;
    std::fwrite(&m, 4, 1, fp); std::fwrite(&v, 4, 1, fp); std::fwrite(&m, 4, 1, fp);
  };
  rec_int(s.pcount);       // write(53) pcount
  rec_int(s.recon_count);  // write(53) recon_count
  rec_int(s.itime);        // write(53) itime
  {
    const int32_t m = 8;  // write(53) t
    std::fwrite(&m, 4, 1, fp); std::fwrite(&s.t, 8, 1, fp); std::fwrite(&m, 4, 1, fp);
  }
  const int32_t m = 248 * s.pcount;  // write(53) f
  std::fwrite(&m, 4, 1, fp);
  for (int i = 1; i <= s.pcount; ++i) {
    const Pt &q = s.f[i];
    std::fwrite(q.x, 8, 3, fp); std::fwrite(q.u, 8, 3, fp); std::fwrite(q.u1, 8, 3, fp);
    std::fwrite(q.u2, 8, 3, fp); std::fwrite(q.u_mf, 8, 3, fp); std::fwrite(q.u_sup, 8, 3, fp);
    std::fwrite(&q.curv, 8, 1, fp); std::fwrite(&q.stretch, 8, 1, fp);
    std::fwrite(q.ghosti, 8, 3, fp); std::fwrite(q.ghostb, 8, 3, fp);
    std::fwrite(&q.infront, 4, 1, fp); std::fwrite(&q.behind, 4, 1, fp); std::fwrite(&q.closest, 4, 1, fp);
    std::fwrite(&q.closestd, 8, 1, fp);
    const int32_t pin[5] = {q.wpinned[0], q.wpinned[1], q.wpinned[2], q.pinnedi ? 1 : 0, q.pinnedb ? 1 : 0};
    std::fwrite(pin, 4, 5, fp);  // wpinned(3), pinnedi, pinnedb (gfortran .true. is 1)
  }
  std::fwrite(&m, 4, 1, fp);
  std::fclose(fp);
  return NV_OK;
}

int or_events_get(or_handle *h, nv_event *buf, int32_t cap, int32_t *n) {
  const auto &ev = h->s.events;
  int m = (int)ev.size() < cap ? (int)ev.size() : cap;
  for (int k = 0; k < m; ++k) buf[k] = ev[k];
  *n = m;
  return NV_OK;
}

int or_ghostp(or_handle *h) { h->s.ghostp(); return NV_OK; }
int or_construct_tree(or_handle *h) {
  int rc = h->s.construct_tree();
  return rc == NV_OK ? rc : fail(rc, "tree deeper than NV_TREE_MAX_DEPTH");
}
int or_pmotion(or_handle *h) {
  if (h->s.p.velocity == NV_VEL_TREE && !h->s.vtree) return fail(NV_ERR_STATE, "no tree");
  h->s.tree_eval = 0;
  h->s.tree_tests = 0;
  int rc = h->s.pmotion();
  return rc == NV_OK ? rc : fail(rc, "singularity in BS (tree) velocity field");
}
int or_pinsert(or_handle *h) {
  int rc = h->s.pinsert();
  return rc == NV_OK ? rc : fail(rc, "vortex line length is 0, run over");
}
int or_pclose(or_handle *h) {
  if (h->s.p.tree_theta > 0) {
    if (!h->s.vtree) return fail(NV_ERR_STATE, "no tree");
    h->s.pclose_tree();
  } else {
    h->s.pclose();
  }
  return NV_OK;
}
int or_precon(or_handle *h) { h->s.precon(); return NV_OK; }
int or_wall_recon(or_handle *h) { h->s.wall_recon(); return NV_OK; }
int or_set_event_margins(or_handle *h, int32_t on) {
  h->s.margin_on = on != 0;
  for (double &v : h->s.margin) v = 1e300;
  return NV_OK;
}
int or_event_margins_get(or_handle *h, double *out) {
  for (int k = 0; k < 4; ++k) out[k] = h->s.margin[k];
  return NV_OK;
}
int or_premove(or_handle *h) { h->s.premove(); return NV_OK; }
int or_enforce_boundary(or_handle *h) { h->s.enforce_boundary(); return NV_OK; }
int or_empty_tree(or_handle *h) { h->s.empty_tree(); return NV_OK; }
int or_end_step(or_handle *h) {
  h->s.t = h->s.t + h->s.p.dt;
  if (h->s.p.nan_test && h->s.nan_finder() != NV_OK) return fail(NV_ERR_NAN, "NaN in f%x");
  return NV_OK;
}

int or_step(or_handle *h, int32_t nsteps) {
  for (int k = 0; k < nsteps; ++k) {
    h->s.tree_eval = 0;
    h->s.tree_tests = 0;
    int rc = h->s.one_step();
    if (rc != NV_OK) return fail(rc, "step failed");
  }
  return NV_OK;
}

int or_calc_velocity_targets(or_handle *h, int32_t velocity, const int32_t *targets,
                             int32_t n, double *u3) {
  Sys &s = h->s;
  s.ghostp();
  if (velocity == NV_VEL_TREE) {
    int rc = s.construct_tree();
    if (rc != NV_OK) return fail(rc, "tree deeper than NV_TREE_MAX_DEPTH");
  }
  long long evals = 0, tests = 0;
  int singular = 0;
#pragma omp parallel reduction(+ : evals, tests) reduction(| : singular)
  {
    tests_tls = 0;
#pragma omp for schedule(dynamic, 4)
    for (int k = 0; k < n; ++k) {
      const int i = targets[k];
      double u[3] = {0.0, 0.0, 0.0};
      if (i >= 1 && i <= s.pcount && s.f[i].infront != 0) s.calc_velocity(u, i, velocity, evals, singular);
      for (int c = 0; c < 3; ++c) u3[3 * k + c] = u[c];
    }
    tests += tests_tls;
  }
  s.tree_eval = evals;
  s.tree_tests = tests;
  if (singular) return fail(NV_ERR_SINGULAR, "singularity in BS (tree) velocity field");
  return NV_OK;
}

int or_calc_velocity(or_handle *h, double *u3) {
  std::vector<int32_t> all(h->s.pcount);
  for (int i = 0; i < h->s.pcount; ++i) all[i] = i + 1;
  return or_calc_velocity_targets(h, h->s.p.velocity, all.data(), h->s.pcount, u3);
}

int or_tree_dump(or_handle *h, or_tree_node *buf, int32_t cap, int32_t *n) {
  if (!h->s.vtree) return fail(NV_ERR_STATE, "no tree");
  std::vector<or_tree_node> out;
  h->s.dump(h->s.vtree, out);
  int m = (int)out.size() < cap ? (int)out.size() : cap;
  for (int k = 0; k < m; ++k) buf[k] = out[k];
  *n = (int32_t)out.size();
  return NV_OK;
}

void or_set_threads(int32_t n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
int32_t or_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
const char *or_last_error(void) { return g_err.c_str(); }

}  // extern "C"
