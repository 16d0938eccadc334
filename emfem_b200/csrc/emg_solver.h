// Solver engine: AMS preconditioner, batched FCG, batched FGMRES.
#pragma once

#include <functional>
#include <map>
#include <utility>
#include <string>
#include <vector>

#include "emg_amg.h"
#include "emg_internal.h"
#include "emg_linalg.h"

namespace emg {

// Cache of instantiated CUDA graphs keyed by an argument pair; owns the execs.
struct GraphCache {
  std::map<std::pair<const void *, void *>, cudaGraphExec_t> exec;
  std::map<std::pair<const void *, void *>, int> seen;
  std::map<std::pair<const void *, void *>, long> kernels;  // kernel nodes per graph
  GraphCache() = default;
  GraphCache(const GraphCache &) = delete;
  GraphCache &operator=(const GraphCache &) = delete;
  GraphCache(GraphCache &&o) noexcept : exec(std::move(o.exec)), seen(std::move(o.seen)), kernels(std::move(o.kernels)) {
    o.exec.clear();
  }
  GraphCache &operator=(GraphCache &&o) noexcept {
    if (this != &o) {
      clear();
      exec = std::move(o.exec);
      seen = std::move(o.seen);
      kernels = std::move(o.kernels);
      o.exec.clear();
    }
    return *this;
  }
  ~GraphCache() { clear(); }
  void clear() {
    for (auto &kv : exec) cudaGraphExecDestroy(kv.second);
    exec.clear();
    seen.clear();
    kernels.clear();
  }
};

// AMS (Hiptmair-Xu auxiliary space preconditioner, as hypre's AMS applies it)
// for B(w) = C + w Ms on K real columns with per-column w.
template <typename T>
struct Ams {
  struct Level {
    DCsr<T> A, P, R;
    long nnzA = 0, nnzP = 0, nnzR = 0;
  };
  struct Sub {
    std::vector<Level> lv;       // operator levels (last has no P/R)
    HCsr coarse;                 // coarsest operator (host, two parts)
    int nc = 0;
    DBuf<double> cinv;           // n_distinct_omega x nc x nc
    std::vector<double> cinv_w;  // omegas the inverses were built for
  };
  DCsr<T> B;                       // values only: pattern is the context's
  const int *brp = nullptr, *bci = nullptr;
  long nnzB = 0;
  bool two = true;  // two value parts (batched) or combined (one frequency)
  Sub sub[4];
  DBuf<T> tangent;
  // G^T B (vertex x edge): curl part (boundary elements only) and mass part
  const int *grp = nullptr, *gci = nullptr;
  long nnzG = 0;
  DBuf<T> gvc, gvm;
  DBuf<T> gtmp;                    // G^T b (nv x K)
  int ne = 0, nv = 0;
  const int *edges = nullptr, *inc_rp = nullptr, *inc = nullptr;
  std::string cycle = "034515430";
  int relax_times = 1;
  double relax_w = 1.0;
  int amg_relax_times = 1;
  int cheb = 1;                    // 1: degree-2 Chebyshev smoothing, 0: l1-Jacobi
  bool use_graphs = true;          // replay each application as one CUDA graph
  bool split_gradient = false;     // last '1' of the cycle returned as potential gphi()
  GraphCache graphs;
  // per-call state
  int K = 0;
  DBuf<double> omega;              // K
  DBuf<int> cslot;                 // K, coarse-inverse index per column
  std::vector<double> h_omega;
  // workspace
  DBuf<T> er, ex2, ed;
  std::vector<DBuf<T>> wb[4], wx[4], wr[4], wx2[4], wd[4];

  void set_columns(const std::vector<double> &col_omega, cudaStream_t s);
  void apply(const T *b, T *x, cudaStream_t s);
  void apply_eager(const T *b, T *x, cudaStream_t s);
  const T *gphi() const { return wx[0][0].p; }  // gradient potential (split form)
  void spmm_B(int mode, const T *x, const T *b, T *y, cudaStream_t s);
  size_t device_bytes() const;

  void vcycle(int sp, int l, cudaStream_t s);
  // one smoothing application on operator A (edge B when A == nullptr);
  // returns the buffer holding the result (cur, or oth after a swap)
  T *smooth(const DCsr<T> *A, long nnz, int n, T *cur, T *oth, const T *b, T *rbuf, T *dbuf, bool zero_guess,
            const char *bin, cudaStream_t s);
  void ensure_workspace(cudaStream_t s);
  int ws_K = 0;
};

// Builds the AMS data for the context's mesh and operators.
//   per_frequency = true: the reference's flow -- B = C + w Ms combined for
//   one w, hierarchies from B(w) (create_pc per frequency);
//   per_frequency = false: two-part operators, hierarchies from w_ref, valid
//   for every frequency of a block.
template <typename T>
void ams_setup(Context &c, Ams<T> &ams, bool per_frequency, double w, double w_ref);

// batched FCG on B(w_c) with AMS, K real columns; returns per-column iteration
// counts; x starts at zero.  Columns converge independently to
// ||r_c|| <= rtol ||b_c|| (unpreconditioned norm, src/em_la.cc:120).
template <typename T>
struct Fcg {
  int K = 0;
  int mmax = 1;
  DBuf<T> r, z, p;
  std::vector<DBuf<T>> P, S;  // previous directions and B-products (ring)
  DBuf<double> dots, eta, eord, alpha, beta, rn, bn;
  DBuf<T *> ptrs;
  std::vector<int> its;
  long total_its = 0;
  int verbose = 0;
  int solve(Ams<T> &ams, const T *b, T *x, double rtol, int maxit, cudaStream_t s);
  // generic form: pc(r, z) applies the preconditioner, opB(p, s) the operator;
  // n rows, K columns
  int solve_with(int n, int Kc, const std::function<void(const T *, T *)> &pc,
                 const std::function<void(const T *, T *)> &opB, const T *b, T *x, double rtol, int maxit,
                 cudaStream_t s);
};

struct SolveStats {
  int outer_its = 0;
  long inner_its = 0;
  std::vector<double> true_res;  // per column
  std::vector<int> col_its;
  std::vector<int> converged;
  double seconds = 0;
};

// Batched FGMRES(restart) on k complex columns (FP64):
//   real_form = true: the reference's real 2n system [[C,-M],[-M,-C]] with
//   real inner products (matshell_mult_a, src/em_la.cc:65-87);
//   real_form = false: (C + i w Ms) z = conj(s) with complex inner products.
// precond(v, z): z = P v on n x k complex (interleaved) device vectors.
struct Fgmres {
  int n = 0, k = 0, restart = 30;
  DBuf<double> V, Z, w, r, h, hn, scale, y, omega, nrm;
  int solve(Context &c, const double *b, double *x, bool use_guess, double rtol, int maxit, bool real_form,
            const std::function<void(const double *, double *)> &precond, SolveStats &st);
};

}  // namespace emg
