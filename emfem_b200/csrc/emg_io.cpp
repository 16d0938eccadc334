// Survey files: the .emd reader and the .rsp writer of the reference
// (read_emd, save_rsp: src/em_io.cc:202-287, 316-399), so a caller that
// keeps the reference's file layout can feed this library and compare its
// responses with the observations.
//
// .emd: every line loses what follows '#' and is trimmed (parse_string,
// src/em_utils.cc:34-58); the remaining whitespace-separated tokens are, in
// order: n_freqs, the frequencies; n_tx, 7 values per transmitter; n_rx,
// x y z per receiver; n_obs, then per observation otype fidx tidx ridx and
// re im err_re err_im.  Observations of the AP types are stored as the
// reference keeps them: (log re, im in radians), errors (err_re/100)^2 and
// (err_im in radians)^2; the others as (re, im), errors squared.
//
// .rsp: the reference's exact layout and printf formats; AP observations
// and responses are written back as (exp real, imag in degrees).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "emg_io.h"

namespace emg {

namespace {

constexpr double kPi = 3.14159265358979323846;  // em_defs.h:16
constexpr double kRtod = 180.0 / kPi;           // em_defs.h:20
constexpr double kDtor = kPi / 180.0;           // em_defs.h:21

bool is_ap(int t) {
  switch (t) {
  case 212: case 222:                                   // R_XY_AP, R_YX_AP
  case 112: case 122: case 132: case 142: case 152: case 162:  // F_*_AP
    return true;
  }
  return false;
}

// comment removal and trimming of one line (parse_string)
std::string strip(const std::string &s) {
  std::string l = s;
  size_t pos = l.find('#');
  if (pos != std::string::npos) l.erase(pos);
  pos = l.find_first_not_of(" \t\r");
  if (pos == std::string::npos) return std::string();
  l.erase(0, pos);
  pos = l.find_last_not_of(" \t\r");
  l.erase(pos + 1);
  return l + "\n";
}

}  // namespace

bool read_emd(const std::string &path, Survey &s, std::string &err) {
  std::ifstream ifs(path);
  if (!ifs.good()) {
    err = "Unable to open file " + path + ".";
    return false;
  }
  std::stringstream ss;
  std::string line;
  while (std::getline(ifs, line)) ss << strip(line);
  auto fail = [&](const char *what) {
    err = std::string("malformed .emd file ") + path + ": " + what;
    return false;
  };
  long n = 0;
  if (!(ss >> n) || n < 0) return fail("frequency count");
  s.freqs.resize(n);
  for (auto &f : s.freqs)
    if (!(ss >> f)) return fail("frequencies");
  if (!(ss >> n) || n < 0) return fail("transmitter count");
  s.tx.resize(n * kTxSize);
  for (auto &v : s.tx)
    if (!(ss >> v)) return fail("transmitters");
  if (!(ss >> n) || n < 0) return fail("receiver count");
  s.rx.resize(n * 3);
  for (auto &v : s.rx)
    if (!(ss >> v)) return fail("receivers");
  if (!(ss >> n) || n < 0) return fail("observation count");
  s.otype.resize(n);
  s.fidx.resize(n);
  s.tidx.resize(n);
  s.ridx.resize(n);
  s.obs.resize(n);
  s.obserr.resize(n);
  for (long i = 0; i < n; ++i) {
    double re, im, err_re, err_im;
    if (!(ss >> s.otype[i] >> s.fidx[i] >> s.tidx[i] >> s.ridx[i] >> re >> im >> err_re >> err_im))
      return fail("observations");
    if (is_ap(s.otype[i])) {
      err_re = err_re / 100.0;
      err_im = err_im * kDtor;
      s.obs[i] = std::complex<double>(std::log(re), im * kDtor);
    } else {
      s.obs[i] = std::complex<double>(re, im);
    }
    s.obserr[i] = std::complex<double>(err_re * err_re, err_im * err_im);
  }
  return true;
}

bool write_rsp(const std::string &path, const Survey &s, const std::complex<double> *rsp, std::string &err) {
  FILE *fp = std::fopen(path.c_str(), "w");
  if (!fp) {
    err = "Unable to open file " + path + " for writing.";
    return false;
  }
  std::fprintf(fp, "# frequencies\n");
  std::fprintf(fp, "%d\n", (int)s.freqs.size());
  for (double f : s.freqs) std::fprintf(fp, "%.4E\n", f);
  const int ntx = (int)s.tx.size() / kTxSize;
  std::fprintf(fp, "# transmiters\n");
  std::fprintf(fp, "%d\n", ntx);
  for (int i = 0; i < ntx; ++i) {
    for (int j = 0; j < kTxSize; ++j) std::fprintf(fp, "% .4E ", s.tx[(size_t)i * kTxSize + j]);
    std::fprintf(fp, "\n");
  }
  const int nrx = (int)s.rx.size() / 3;
  std::fprintf(fp, "# recievers\n");
  std::fprintf(fp, "%d\n", nrx);
  for (int i = 0; i < nrx; ++i)
    std::fprintf(fp, "% .4E % .4E % .4E\n", s.rx[3 * (size_t)i], s.rx[3 * (size_t)i + 1], s.rx[3 * (size_t)i + 2]);
  std::fprintf(fp, "# observations\n");
  std::fprintf(fp, "%d\n", (int)s.obs.size());
  std::fprintf(fp, "#%6s %6s %5s %7s %13s %13s %13s %13s\n", "otype", "fidx", "tidx", "ridx", "amp", "phase", "amp`",
               "phase`");
  for (size_t i = 0; i < s.obs.size(); ++i) {
    if (is_ap(s.otype[i])) {
      const std::complex<double> o(std::exp(s.obs[i].real()), s.obs[i].imag() * kRtod);
      const std::complex<double> r(std::exp(rsp[i].real()), rsp[i].imag() * kRtod);
      std::fprintf(fp, "% 7d % 6d % 5d % 7d % 13.6E % 13.3f % 13.6E % 13.3f\n", s.otype[i], s.fidx[i], s.tidx[i],
                   s.ridx[i], o.real(), o.imag(), r.real(), r.imag());
    } else {
      std::fprintf(fp, "% 7d % 6d % 5d % 7d % 13.6E % 13.6E % 13.6E % 13.6E\n", s.otype[i], s.fidx[i], s.tidx[i],
                   s.ridx[i], s.obs[i].real(), s.obs[i].imag(), rsp[i].real(), rsp[i].imag());
    }
  }
  const bool ok = std::fclose(fp) == 0;
  if (!ok) err = "error closing " + path + ".";
  return ok;
}

// Mesh::save_vtk (src/em_mesh.cc:183-248): legacy ASCII unstructured grid
// with the tets, then cell data "subdomain" (0 on one process), "tet_attr"
// and the caller's arrays in name order (the reference keeps them in a
// std::map).
bool write_vtk(const std::string &path, int nv, const double *pts, int nt, const int *tets, const int *attr,
               const std::vector<std::pair<std::string, const double *>> &arrays, std::string &err) {
  FILE *fp = std::fopen(path.c_str(), "w");
  if (!fp) {
    err = "Unable to open file " + path + " for writing.";
    return false;
  }
  std::fprintf(fp, "# vtk DataFile Version 2.0\n");
  std::fprintf(fp, "Unstructured Grid\n");
  std::fprintf(fp, "ASCII\n");
  std::fprintf(fp, "DATASET UNSTRUCTURED_GRID\n");
  std::fprintf(fp, "POINTS %d double\n", nv);
  for (int i = 0; i < nv; ++i)
    std::fprintf(fp, "%.17g %.17g %.17g\n", pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2]);
  std::fprintf(fp, "\n");
  std::fprintf(fp, "CELLS %d %d\n", nt, nt * (4 + 1));
  for (int i = 0; i < nt; ++i) {
    std::fprintf(fp, "%d", 4);
    for (int j = 0; j < 4; ++j) std::fprintf(fp, " %4d", tets[4 * (size_t)i + j]);
    std::fprintf(fp, "\n");
  }
  std::fprintf(fp, "\n");
  std::fprintf(fp, "CELL_TYPES %d\n", nt);
  for (int i = 0; i < nt; ++i) std::fprintf(fp, "%d\n", 10);
  std::fprintf(fp, "\n");
  std::fprintf(fp, "CELL_DATA %d\n", nt);
  std::fprintf(fp, "SCALARS subdomain double 1\n");
  std::fprintf(fp, "LOOKUP_TABLE default\n");
  for (int i = 0; i < nt; ++i) std::fprintf(fp, "%.15g\n", 0.0);
  std::fprintf(fp, "\n");
  std::fprintf(fp, "SCALARS tet_attr double 1\n");
  std::fprintf(fp, "LOOKUP_TABLE default\n");
  for (int i = 0; i < nt; ++i) std::fprintf(fp, "%.15g\n", (double)attr[i]);
  std::fprintf(fp, "\n");
  std::vector<std::pair<std::string, const double *>> sorted(arrays);
  std::stable_sort(sorted.begin(), sorted.end(),
                   [](const std::pair<std::string, const double *> &a, const std::pair<std::string, const double *> &b) {
                     return a.first < b.first;
                   });
  for (size_t k = 0; k < sorted.size(); ++k) {
    if (k > 0 && sorted[k].first == sorted[k - 1].first) continue;  // a map keeps one array per name
    std::fprintf(fp, "SCALARS %s double 1\n", sorted[k].first.c_str());
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < nt; ++i) std::fprintf(fp, "%.15g\n", sorted[k].second[i]);
    std::fprintf(fp, "\n");
  }
  const bool ok = std::fclose(fp) == 0;
  if (!ok) err = "error closing " + path + ".";
  return ok;
}

}  // namespace emg
