// Nodal AMG hierarchy setup on the device (emg_amg_gpu.cu).
#pragma once

#include <vector>

#include "emg_amg.h"
#include "emg_internal.h"

namespace emg {

// device CSR in FP64 with one or two value parts (vm empty: one part; a
// pattern-only matrix has no vc either)
struct GCsr {
  int n = 0, m = 0;
  long nnz = 0;
  DBuf<int> rp, ci;
  DBuf<double> vc, vm;
};

struct GpuLevel {
  GCsr A, P, R;
};

// A^T (rows in increasing column order, values of the first part only)
void gcsr_transpose(const GCsr &A, GCsr &T, cudaStream_t s);
// C = R A P for both value parts of A (rows in increasing column order)
void gcsr_galerkin(const GCsr &R, const GCsr &A, const GCsr &P, GCsr &C, cudaStream_t s);
// the hierarchy of A with the host build's algorithms (amg_build); the last
// operator is returned in `coarse`
void amg_build_gpu(GCsr A, double w_ref, const AmgParams &prm, std::vector<GpuLevel> &lv, GCsr &coarse,
                   cudaStream_t s);
void gcsr_to_host(const GCsr &d, HCsr &h, cudaStream_t s);
// nodal subspace operator sp (0 G, 1-3 Pi_x/y/z, 4 the vector space without
// couplings) from the device nodal assembly (assemble_nodal_device); fold_w
// >= 0 folds the two parts into one for that w
void nodal_operator_gpu(Context &c, const DBuf<double> &parts, int sp, GCsr &out, double fold_w);
void gcsr_from_host(const HCsr &h, GCsr &d, cudaStream_t s);

}  // namespace emg
