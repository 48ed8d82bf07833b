// runin.cpp -- nv_read_run_file: the run.in reader of src/cdata.f90:131-241.
//
// Semantics kept from the reference:
//   * each line is read into a 100-character buffer (longer lines are cut);
//   * the label is the text before the first blank, the value list the text after it;
//   * unknown labels are ignored;
//   * values are read list-directed: blank- or comma-separated items, '/' ends the list;
//   * the loop runs while the last read succeeded, so a value that fails to parse (or a
//     list with too few items, which is an end-of-record condition) silently ends the
//     whole read, after assigning the items that were read.
// Keys this library does not use (initial-condition and output keys) are still parsed, so
// that a malformed one ends the read exactly where the reference's would.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nuvort_gpu.h"

int set_error(int code, const std::string &msg);

namespace {

// List-directed items of one value string.
std::vector<std::string> items(const std::string &s, bool &quoted_err) {
  std::vector<std::string> out;
  quoted_err = false;
  size_t i = 0;
  const size_t n = s.size();
  while (i < n) {
    while (i < n && (s[i] == ' ' || s[i] == '\t')) ++i;
    if (i >= n) break;
    if (s[i] == '/') break;
    if (s[i] == ',') { ++i; continue; }
    if (s[i] == '\'' || s[i] == '"') {
      const char q = s[i++];
      std::string v;
      while (i < n && s[i] != q) v += s[i++];
      if (i >= n) { quoted_err = true; break; }
      ++i;
      out.push_back(v);
      continue;
    }
    std::string v;
    while (i < n && s[i] != ' ' && s[i] != '\t' && s[i] != ',' && s[i] != '/') v += s[i++];
    out.push_back(v);
  }
  return out;
}

bool parse_int(const std::string &t, int32_t &v) {
  if (t.empty()) return false;
  size_t i = 0;
  if (t[0] == '+' || t[0] == '-') i = 1;
  if (i >= t.size()) return false;
  for (size_t k = i; k < t.size(); ++k)
    if (!std::isdigit((unsigned char)t[k])) return false;
  v = (int32_t)std::strtol(t.c_str(), nullptr, 10);
  return true;
}

bool parse_real(const std::string &t0, double &v) {
  if (t0.empty()) return false;
  std::string t = t0;
  for (auto &c : t)
    if (c == 'd' || c == 'D' || c == 'q' || c == 'Q') c = 'e';
  // Fortran also accepts a signed exponent without a letter (1.0+5): insert the 'e'.
  for (size_t k = 1; k < t.size(); ++k)
    if ((t[k] == '+' || t[k] == '-') && t[k - 1] != 'e' && t[k - 1] != 'E') {
      t.insert(k, "e");
      break;
    }
  char *end = nullptr;
  v = std::strtod(t.c_str(), &end);
  return end && *end == '\0' && end != t.c_str();
}

bool parse_logical(const std::string &t, int32_t &v) {
  size_t i = 0;
  if (i < t.size() && t[i] == '.') ++i;
  if (i >= t.size()) return false;
  const char c = (char)std::toupper((unsigned char)t[i]);
  if (c == 'T') { v = 1; return true; }
  if (c == 'F') { v = 0; return true; }
  return false;
}

enum Kind { K_INT, K_REAL, K_LOGICAL, K_STRING };

}  // namespace

extern "C" int nv_read_run_file(const char *path, nv_params *p) {
  if (!path || !p) return set_error(NV_ERR_ARG, "nv_read_run_file: null argument");
  FILE *fh = std::fopen(path, "r");
  if (!fh) return set_error(NV_ERR_IO, std::string("cannot open ") + path);
  char line[4096];
  bool ok = true;
  while (ok && std::fgets(line, sizeof line, fh)) {
    std::string buffer(line);
    while (!buffer.empty() && (buffer.back() == '\n' || buffer.back() == '\r')) buffer.pop_back();
    if (buffer.size() > 100) buffer.resize(100);
    buffer.resize(100, ' ');
    const size_t pos = buffer.find(' ');
    const std::string label = pos == std::string::npos ? std::string() : buffer.substr(0, pos);
    const std::string rest = pos == std::string::npos ? std::string() : buffer.substr(pos + 1);
    bool qerr = false;
    const std::vector<std::string> it = items(rest, qerr);
    auto need = [&](size_t k) { return !qerr && it.size() >= k; };
    auto read_ints = [&](int32_t *dst, size_t n) {
      for (size_t k = 0; k < n; ++k) {
        if (!need(k + 1)) return false;
        int32_t v;
        if (!parse_int(it[k], v)) return false;
        if (dst) dst[k] = v;
      }
      return true;
    };
    auto read_reals = [&](double *dst, size_t n) {
      for (size_t k = 0; k < n; ++k) {
        if (!need(k + 1)) return false;
        double v;
        if (!parse_real(it[k], v)) return false;
        if (dst) dst[k] = v;
      }
      return true;
    };
    auto read_logical = [&](int32_t *dst) {
      if (!need(1)) return false;
      int32_t v;
      if (!parse_logical(it[0], v)) return false;
      if (dst) *dst = v;
      return true;
    };
    auto read_string = [&](std::string &dst) {
      if (!need(1)) return false;
      dst = it[0];
      return true;
    };
    std::string sv;
    int32_t idummy;
    double rdummy[3];
    if (label == "nsteps") ok = read_ints(&p->nsteps, 1);
    else if (label == "shots") ok = read_ints(&p->shots, 1);
    else if (label == "recon_shots") ok = read_ints(&p->recon_shots, 1);
    else if (label == "pcount") ok = read_ints(&idummy, 1);
    else if (label == "dt") ok = read_reals(&p->dt, 1);
    else if (label == "delta") ok = read_reals(&p->delta, 1);
    else if (label == "quant_circ") ok = read_reals(&p->quant_circ, 1);
    else if (label == "corea") ok = read_reals(&p->corea, 1);
    else if (label == "box_size") ok = read_reals(p->box_size, 3);
    else if (label == "velocity") {
      ok = read_string(sv);
      if (ok) p->velocity = sv == "LIA" ? NV_VEL_LIA : sv == "BS" ? NV_VEL_BS : sv == "Tree" ? NV_VEL_TREE : -1;
    } else if (label == "boundary_x" || label == "boundary_y" || label == "boundary_z") {
      ok = read_string(sv);
      if (ok)
        p->boundary[label[9] - 'x'] = sv == "periodic" ? NV_BC_PERIODIC : sv == "open" ? NV_BC_OPEN
                                      : sv == "solid"  ? NV_BC_SOLID
                                                       : -1;
    } else if (label == "tree_theta") ok = read_reals(&p->tree_theta, 1);
    else if (label == "tree_print") ok = read_logical(&idummy);
    else if (label == "tree_extra_correction") ok = read_logical(&p->tree_extra_correction);
    else if (label == "normal_velocity") {
      ok = read_string(sv);
      if (ok)
        p->normal_velocity = sv == "zero" ? NV_NF_ZERO : sv == "xflow" ? NV_NF_XFLOW : sv == "uniform" ? NV_NF_UNIFORM
                           : sv == "shear_xflow"  ? NV_NF_SHEAR_XFLOW
                           : sv == "channel"      ? NV_NF_CHANNEL
                           : sv == "ychannel"     ? NV_NF_YCHANNEL
                           : sv == "noisey_xflow" ? NV_NF_NOISEY_XFLOW
                           : sv == "laizetDNS"    ? NV_NF_LAIZET_DNS
                           : sv == "turbDNS"      ? NV_NF_TURB_DNS
                                                  : 100;
    } else if (label == "normal_fluid_cutoff") ok = read_reals(&p->normal_fluid_cutoff, 1);
    else if (label == "t_zero_normal_fluid") ok = read_reals(&p->t_zero_normal_fluid, 1);
    else if (label == "norm_vel_xflow") ok = read_reals(&p->norm_vel_xflow, 1);
    else if (label == "norm_shear_omega") ok = read_reals(&p->norm_shear_omega, 1);
    else if (label == "noise_file") ok = read_string(sv);  // the caller loads it: nv_set_normal_fluid_noise
    else if (label == "alpha") ok = read_reals(p->alpha, 2);
    else if (label == "super_velocity") ok = read_reals(p->super_velocity, 3);
    else if (label == "initf") ok = read_string(sv);
    else if (label == "scaling_factor") ok = read_reals(rdummy, 1);
    else if (label == "loop_translate") ok = read_reals(rdummy, 3);
    else if (label == "rotation_factor") ok = read_reals(rdummy, 1);
    else if (label == "line_count") ok = read_ints(&idummy, 1);
    else if (label == "NAN_test") ok = read_logical(&p->nan_test);
    else if (label == "max_warn_count") ok = read_ints(&idummy, 1);
    else if (label == "overide_timestep_check") ok = read_logical(&p->overide_timestep_check);
    else if (label == "serial_run") ok = read_logical(&idummy);
    else if (label == "qvort_nproc") ok = read_ints(&idummy, 1);
    else if (label == "wave_amp") ok = read_reals(rdummy, 1);
    else if (label == "noise_file") ok = read_string(sv);
    else if (label == "norm_shear_omega") ok = read_reals(rdummy, 1);
    else if (label == "lattice_ratio") ok = read_reals(rdummy, 1);
    // extension keys of this library
    else if (label == "norm_vel_vec") ok = read_reals(p->norm_vel_vec, 3);
    else if (label == "precision") {
      ok = read_string(sv);
      if (ok) p->precision = sv == "mixed" ? NV_PREC_MIXED : sv == "fp64" ? NV_PREC_FP64 : -1;
    }
  }
  std::fclose(fh);
  return NV_OK;
}
