// io.cpp -- the reference's snapshot and restart files, written and read on the host.
//
//   * printf (src/output.f90:47-70): data/var%04d.log, an unformatted stream file (no record
//     markers): t, pcount, then per field the values of all pcount slots -- x(1), x(2), x(3),
//     infront, u(1..3), u_mf(1..3), curv, stretch -- the layout bin/vortex/vortex_load.m reads.
//   * data_dump (src/output.f90:85-94) / data_restore (src/initial.f90:151-166): data/var.dat,
//     gfortran unformatted sequential records pcount, recon_count, itime, t, f, each framed by
//     a 4-byte length marker before and after.  f is the array of type(qvort) (src/cdata.f90:
//     19-29) written element after element, each element component after component with no
//     padding: x, u, u1, u2, u_mf, u_sup (3 reals each), curv, stretch, ghosti, ghostb (3
//     reals each), infront, behind, closest (integers), closestd, wpinned(3) (integers),
//     pinnedi, pinnedb (logicals) -- 248 bytes with the reference's -fdefault-real-8 build.
// The host is little-endian, as the files are on the machines that write them.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nuvort_gpu.h"

int set_error(int code, const std::string &msg);
int set_restart_counters(nv_handle *h, int sys, double t, int itime, int recon_count);
int sys_capacity(nv_handle *h, int sys);

namespace {

constexpr long long kQvortBytes = 248;  // one type(qvort) element in the file
constexpr long long kMaxRecord = 2147483647LL;

struct File {
  FILE *f = nullptr;
  explicit File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

template <class T>
void put(std::vector<unsigned char> &b, T v) {
  const unsigned char *p = reinterpret_cast<const unsigned char *>(&v);
  b.insert(b.end(), p, p + sizeof v);
}
template <class T>
T get(const unsigned char *p) {
  T v;
  std::memcpy(&v, p, sizeof v);
  return v;
}

double comp(const double *a, int k, int c) { return a ? a[3 * k + c] : 0.0; }
double val(const double *a, int k) { return a ? a[k] : 0.0; }
int ival(const int32_t *a, int k) { return a ? a[k] : 0; }

// One sequential record: marker, payload, marker.
bool write_record(FILE *f, const std::vector<unsigned char> &payload) {
  const int32_t m = (int32_t)payload.size();
  return std::fwrite(&m, 4, 1, f) == 1 && (payload.empty() || std::fwrite(payload.data(), 1, payload.size(), f) ==
                                                                   payload.size()) &&
         std::fwrite(&m, 4, 1, f) == 1;
}

// Reads one sequential record; false at a short read or a marker mismatch.
bool read_record(FILE *f, std::vector<unsigned char> &payload) {
  int32_t m1 = 0, m2 = 0;
  if (std::fread(&m1, 4, 1, f) != 1 || m1 < 0) return false;
  payload.resize((size_t)m1);
  if (m1 > 0 && std::fread(payload.data(), 1, (size_t)m1, f) != (size_t)m1) return false;
  return std::fread(&m2, 4, 1, f) == 1 && m2 == m1;
}

// Fortran edit descriptors as gfortran writes them: a field that does not fit is w asterisks;
// Fw.d writes NaN and Infinity (Inf when w < 8) right-justified.
std::string fit(const std::string &s, int w) { return (int)s.size() > w ? std::string(w, '*') : s; }
std::string f_edit(double v, int w, int d) {
  char b[64];
  if (std::isnan(v)) {
    std::snprintf(b, sizeof b, "%*s", w, "NaN");
  } else if (std::isinf(v)) {
    const char *word = w >= 9 || (w == 8 && v > 0) ? "Infinity" : "Inf";
    std::snprintf(b, sizeof b, "%*s%s", w - (int)std::strlen(word) - (v < 0), v < 0 ? "-" : "", word);
  } else {
    std::snprintf(b, sizeof b, "%*.*f", w, d, v);
  }
  return fit(b, w);
}
std::string i_edit(long long v, int w, int m) {
  char b[64];
  std::snprintf(b, sizeof b, "%*.*lld", w, m, v);
  return fit(b, w);
}

}  // namespace

extern "C" {

// print_info's ts.log row (src/output.f90:38-40), format
// (i6.4,f13.7,i10.1,i13.1,i13.1,f7.4,f13.6,f13.5,f13.5,f10.2,i13.1,i13.1).
int nv_format_ts_row(const nv_ts_row *row, int32_t shots, char *buf, int32_t cap) {
  if (!row || !buf || cap < 1 || shots < 1) return set_error(NV_ERR_ARG, "nv_format_ts_row: bad arguments");
  const std::string line = i_edit(row->itime / shots, 6, 4) + f_edit(row->t, 13, 7) + i_edit(row->live, 10, 1) +
                           i_edit(row->recon_count, 13, 1) + i_edit(row->wall_recon_count, 13, 1) +
                           f_edit(row->avg_sep / row->delta, 7, 4) + f_edit(row->total_length, 13, 6) +
                           f_edit(row->maxu, 13, 5) + f_edit(row->maxdu, 13, 5) + f_edit(row->kappa_bar, 10, 2) +
                           i_edit(row->remove_count, 13, 1) + i_edit(row->tree_eval, 13, 1);
  if ((int)line.size() + 1 > cap) return set_error(NV_ERR_ARG, "nv_format_ts_row: buffer too small");
  std::memcpy(buf, line.c_str(), line.size() + 1);
  return NV_OK;
}

int nv_snapshot_write_file(const nv_full_state *st, double t, const char *path) {
  if (!st || !path || st->pcount < 0) return set_error(NV_ERR_ARG, "nv_snapshot_write_file: bad arguments");
  const int n = st->pcount;
  std::vector<unsigned char> b;
  b.reserve(12 + (size_t)n * (13 * 8 + 4));
  put(b, t);
  put(b, (int32_t)n);
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < n; ++k) put(b, comp(st->x, k, c));
  for (int k = 0; k < n; ++k) put(b, (int32_t)ival(st->infront, k));
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < n; ++k) put(b, comp(st->u, k, c));
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < n; ++k) put(b, comp(st->u_mf, k, c));
  for (int k = 0; k < n; ++k) put(b, val(st->curv, k));
  for (int k = 0; k < n; ++k) put(b, val(st->stretch, k));
  File f(path, "wb");
  if (!f.f) return set_error(NV_ERR_IO, std::string("cannot open ") + path);
  if (std::fwrite(b.data(), 1, b.size(), f.f) != b.size()) return set_error(NV_ERR_IO, std::string("short write: ") + path);
  return NV_OK;
}

int nv_dump_write_file(const nv_full_state *st, int32_t recon_count, int32_t itime, double t, const char *path) {
  if (!st || !path || st->pcount < 0) return set_error(NV_ERR_ARG, "nv_dump_write_file: bad arguments");
  const int n = st->pcount;
  if ((long long)n * kQvortBytes > kMaxRecord)
    return set_error(NV_ERR_UNSUPPORTED, "nv_dump_write_file: f record above 2^31-1 bytes (gfortran subrecords)");
  File f(path, "wb");
  if (!f.f) return set_error(NV_ERR_IO, std::string("cannot open ") + path);
  std::vector<unsigned char> b;
  bool ok = true;
  b.clear(); put(b, (int32_t)n); ok = ok && write_record(f.f, b);
  b.clear(); put(b, recon_count); ok = ok && write_record(f.f, b);
  b.clear(); put(b, itime); ok = ok && write_record(f.f, b);
  b.clear(); put(b, t); ok = ok && write_record(f.f, b);
  b.clear();
  b.reserve((size_t)n * kQvortBytes);
  for (int k = 0; k < n; ++k) {
    const double *v3[] = {st->x, st->u, st->u1, st->u2, st->u_mf, st->u_sup};
    for (const double *a : v3)
      for (int c = 0; c < 3; ++c) put(b, comp(a, k, c));
    put(b, val(st->curv, k));
    put(b, val(st->stretch, k));
    for (int c = 0; c < 3; ++c) put(b, comp(st->ghosti, k, c));
    for (int c = 0; c < 3; ++c) put(b, comp(st->ghostb, k, c));
    put(b, (int32_t)ival(st->infront, k));
    put(b, (int32_t)ival(st->behind, k));
    put(b, (int32_t)ival(st->closest, k));
    put(b, val(st->closestd, k));
    for (int c = 0; c < 3; ++c) put(b, (int32_t)(st->wpinned ? st->wpinned[3 * k + c] : 0));
    put(b, (int32_t)ival(st->pinnedi, k));  // logical: .true. is 1, .false. 0
    put(b, (int32_t)ival(st->pinnedb, k));
  }
  ok = ok && write_record(f.f, b);
  if (!ok) return set_error(NV_ERR_IO, std::string("short write: ") + path);
  return NV_OK;
}

int nv_dump_read_file(const char *path, nv_full_state *st, int32_t cap, int32_t *pcount_out, int32_t *recon_count,
                      int32_t *itime, double *t) {
  if (!path || !pcount_out) return set_error(NV_ERR_ARG, "nv_dump_read_file: bad arguments");
  File f(path, "rb");
  if (!f.f) return set_error(NV_ERR_IO, std::string("cannot open ") + path);
  std::vector<unsigned char> r[5];
  for (auto &x : r)
    if (!read_record(f.f, x)) return set_error(NV_ERR_IO, std::string("not a var.dat record sequence: ") + path);
  if (r[0].size() != 4 || r[1].size() != 4 || r[2].size() != 4 || r[3].size() != 8)
    return set_error(NV_ERR_IO, std::string("unexpected record sizes in ") + path);
  const int n = get<int32_t>(r[0].data());
  if (n < 0 || (long long)r[4].size() != (long long)n * kQvortBytes)
    return set_error(NV_ERR_IO, std::string("f record does not hold pcount type(qvort) elements: ") + path);
  *pcount_out = n;
  if (recon_count) *recon_count = get<int32_t>(r[1].data());
  if (itime) *itime = get<int32_t>(r[2].data());
  if (t) *t = get<double>(r[3].data());
  if (!st) return NV_OK;
  st->pcount = n;
  if (n > cap) return set_error(NV_ERR_ARG, "nv_dump_read_file: arrays hold fewer slots than the file's pcount");
  const unsigned char *p = r[4].data();
  for (int k = 0; k < n; ++k, p += kQvortBytes) {
    const unsigned char *q = p;
    double *v3[] = {st->x, st->u, st->u1, st->u2, st->u_mf, st->u_sup};
    for (double *a : v3) {
      for (int c = 0; c < 3; ++c)
        if (a) a[3 * k + c] = get<double>(q + 8 * c);
      q += 24;
    }
    if (st->curv) st->curv[k] = get<double>(q);
    if (st->stretch) st->stretch[k] = get<double>(q + 8);
    q += 16;
    for (int c = 0; c < 3; ++c)
      if (st->ghosti) st->ghosti[3 * k + c] = get<double>(q + 8 * c);
    q += 24;
    for (int c = 0; c < 3; ++c)
      if (st->ghostb) st->ghostb[3 * k + c] = get<double>(q + 8 * c);
    q += 24;
    if (st->infront) st->infront[k] = get<int32_t>(q);
    if (st->behind) st->behind[k] = get<int32_t>(q + 4);
    if (st->closest) st->closest[k] = get<int32_t>(q + 8);
    q += 12;
    if (st->closestd) st->closestd[k] = get<double>(q);
    q += 8;
    for (int c = 0; c < 3; ++c)
      if (st->wpinned) st->wpinned[3 * k + c] = get<int32_t>(q + 4 * c);
    if (st->pinnedi) st->pinnedi[k] = get<int32_t>(q + 12) != 0;
    if (st->pinnedb) st->pinnedb[k] = get<int32_t>(q + 16) != 0;
  }
  return NV_OK;
}

}  // extern "C"

namespace {

// Host arrays for one system's full state.
struct FullArrays {
  std::vector<double> x, u, u1, u2, umf, usup, curv, stretch, gi, gb, cd;
  std::vector<int32_t> inf, beh, cl, wp, pi, pb;
  nv_full_state st;
  explicit FullArrays(int cap) {
    const size_t n3 = 3 * (size_t)cap, n = (size_t)cap;
    x.resize(n3); u.resize(n3); u1.resize(n3); u2.resize(n3); umf.resize(n3); usup.resize(n3);
    gi.resize(n3); gb.resize(n3); curv.resize(n); stretch.resize(n); cd.resize(n);
    inf.resize(n); beh.resize(n); cl.resize(n); wp.resize(n3); pi.resize(n); pb.resize(n);
    st = nv_full_state{0,          x.data(),  u.data(),  u1.data(), u2.data(),  umf.data(), usup.data(), curv.data(),
                       stretch.data(), gi.data(), gb.data(), inf.data(), beh.data(), cl.data(),  cd.data(),
                       wp.data(),  pi.data(), pb.data()};
  }
};

// The system's current pcount (the number of slots a download returns).
int pcount_of(nv_handle *h, int sys, int *n) {
  nv_counters c;
  int rc = nv_counters_get(h, sys, &c);
  if (rc == NV_OK) *n = c.pcount;
  return rc;
}

}  // namespace

extern "C" {

int nv_write_snapshot(nv_handle *h, int32_t sys, const char *path) {
  if (!h || !path) return set_error(NV_ERR_ARG, "nv_write_snapshot: bad arguments");
  int n = 0, rc = pcount_of(h, sys, &n);
  if (rc) return rc;
  FullArrays a(n);
  if ((rc = nv_download_full(h, sys, &a.st, n))) return rc;
  nv_counters c;
  if ((rc = nv_counters_get(h, sys, &c))) return rc;
  return nv_snapshot_write_file(&a.st, c.t, path);
}

int nv_write_dump(nv_handle *h, int32_t sys, const char *path) {
  if (!h || !path) return set_error(NV_ERR_ARG, "nv_write_dump: bad arguments");
  int n = 0, rc = pcount_of(h, sys, &n);
  if (rc) return rc;
  FullArrays a(n);
  if ((rc = nv_download_full(h, sys, &a.st, n))) return rc;
  nv_counters c;
  if ((rc = nv_counters_get(h, sys, &c))) return rc;
  return nv_dump_write_file(&a.st, c.recon_count, c.itime, c.t, path);
}

int nv_restore_dump(nv_handle *h, int32_t sys, const char *path) {
  if (!h || !path) return set_error(NV_ERR_ARG, "nv_restore_dump: bad arguments");
  int32_t n = 0, recon = 0, itime = 0;
  double t = 0;
  int rc = nv_dump_read_file(path, nullptr, 0, &n, &recon, &itime, &t);
  if (rc) return rc;
  const int cap = sys_capacity(h, sys);
  if (cap < 0) return set_error(NV_ERR_ARG, "nv_restore_dump: bad system");
  if (n > cap) return set_error(NV_ERR_CAPACITY, "nv_restore_dump: the file's pcount exceeds the system's capacity");
  FullArrays a(n);
  if ((rc = nv_dump_read_file(path, &a.st, n, &n, &recon, &itime, &t))) return rc;
  if ((rc = nv_upload_full(h, sys, &a.st))) return rc;
  return set_restart_counters(h, sys, t, itime, recon);
}

}  // extern "C"
