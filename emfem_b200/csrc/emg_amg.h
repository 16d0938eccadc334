// Host AMG hierarchy (emg_amg.cpp).
#pragma once

#include <cstdint>
#include <vector>

#include "emg_internal.h"

namespace emg {

struct AmgParams {
  double theta = 0.25;
  int pmax = 4;
  int max_coarse = 200;
  int max_levels = 25;
  uint64_t seed = 12345;
  // systems AMG, unknown approach: row i carries function i % num_functions
  // on the finest level; strength and interpolation only couple rows of the
  // same function (the coarse operators still couple them through R A P)
  int num_functions = 1;
};

struct HostLevel {
  HCsr A;     // level operator (two parts)
  HCsr P, R;  // interpolation and restriction (single part)
};

struct HostAmg {
  std::vector<HostLevel> lv;  // all levels but the coarsest
  HCsr coarse;                // coarsest operator (two parts)
};

HCsr transpose(const HCsr &A);
HCsr spgemm(const HCsr &A, const HCsr &B);
HCsr galerkin(const HCsr &R, const HCsr &A, const HCsr &P);
// builds the hierarchy of A (taken by value: pass an rvalue to avoid a copy)
void amg_build(HCsr A, double w_ref, const AmgParams &prm, HostAmg &out);
void coarse_inverse(const HCsr &A, double w, std::vector<double> &X);

}  // namespace emg
