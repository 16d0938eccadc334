// Survey files (.emd in, .rsp out) in the reference's layout (emg_io.cpp).
#pragma once

#include <complex>
#include <string>
#include <utility>
#include <vector>

namespace emg {

constexpr int kTxSize = 7;  // TX_SIZE, src/em_defs.h:25

struct Survey {
  std::vector<double> freqs, tx, rx;  // tx: kTxSize per transmitter, rx: x y z per receiver
  std::vector<int> otype, fidx, tidx, ridx;
  std::vector<std::complex<double>> obs, obserr;
};

bool read_emd(const std::string &path, Survey &s, std::string &err);
bool write_rsp(const std::string &path, const Survey &s, const std::complex<double> *rsp, std::string &err);
bool write_vtk(const std::string &path, int nv, const double *pts, int nt, const int *tets, const int *attr,
               const std::vector<std::pair<std::string, const double *>> &arrays, std::string &err);

}  // namespace emg
