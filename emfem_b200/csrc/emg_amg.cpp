// Nodal AMG hierarchy setup for the AMS subspace operators (host C++).
//
// Replaces the BoomerAMG setup that hypre's AMS performs for G^T B G and
// Pi_d^T B Pi_d (invoked by PCSetUp, src/em_la.cc:156-157).  The method
// follows the published algorithms, not hypre's source:
//   * classical strength of connection, theta = 0.25 (hypre's default);
//   * PMIS coarsening (De Sterck, Yang & Heys 2006) with a deterministic
//     per-point random tie breaker, the parallel relative of the HMIS
//     coarsening hypre's AMS defaults select;
//   * direct interpolation with separate scaling of negative and positive
//     couplings, truncated to Pmax = 4 entries per row with row-sum
//     preservation (hypre: interp 6 = ext+i, which this does not restate);
//   * Galerkin coarse operators R A P with R = P^T.
// Every operator carries two value parts, A(w) = Ac + w Am.  Interpolation
// is computed once from Ac + w_ref Am; the Galerkin products are formed for
// both parts, so one hierarchy serves every frequency of a block solve.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "emg_amg.h"

namespace emg {

static inline double combined(const HCsr &A, long k, double w) {
  return A.vm.empty() ? A.vc[k] : A.vc[k] + w * A.vm[k];
}

// j couples with i in the AMG sense: j != i and, for a system, the same
// function (fn empty: scalar problem)
static inline bool same_fn(const std::vector<int> &fn, int i, int j) { return fn.empty() || fn[i] == fn[j]; }

// j strongly influences i  <=>  -a_ij >= theta * max_{k != i} (-a_ik)
static void strength(const HCsr &A, double w, double theta, const std::vector<int> &fn, std::vector<int> &srp,
                     std::vector<int> &sci) {
  const int n = A.n;
  std::vector<int> cnt(n + 1, 0);
  std::vector<double> mx(n, 0.0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double m = 0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] != i && same_fn(fn, i, A.ci[k])) m = std::max(m, -combined(A, k, w));
    mx[i] = m;
    int c = 0;
    if (m > 0)
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if (A.ci[k] != i && same_fn(fn, i, A.ci[k]) && -combined(A, k, w) >= theta * m) ++c;
    cnt[i + 1] = c;
  }
  for (int i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
  srp = cnt;
  sci.resize(srp[n]);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double m = mx[i];
    int p = srp[i];
    if (m > 0)
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if (A.ci[k] != i && same_fn(fn, i, A.ci[k]) && -combined(A, k, w) >= theta * m) sci[p++] = A.ci[k];
  }
}

static inline double hash_unit(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

// PMIS: cf[i] = 1 (C) or -1 (F)
static void pmis(int n, const std::vector<int> &srp, const std::vector<int> &sci, uint64_t seed,
                 std::vector<int> &cf) {
  // transpose of S (the order inside a row of S^T does not matter below)
  std::vector<int> trp(n + 1, 0), tci(sci.size());
  const long ns = (long)sci.size();
#pragma omp parallel for schedule(static)
  for (long k = 0; k < ns; ++k) {
#pragma omp atomic
    trp[sci[k] + 1]++;
  }
  for (int i = 0; i < n; ++i) trp[i + 1] += trp[i];
  {
    std::vector<int> pos(trp.begin(), trp.end() - 1);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
      for (int k = srp[i]; k < srp[i + 1]; ++k) {
        int p;
#pragma omp atomic capture
        p = pos[sci[k]]++;
        tci[p] = i;
      }
  }
  std::vector<double> lam(n);
  cf.assign(n, 0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    int infl = trp[i + 1] - trp[i];
    lam[i] = infl + hash_unit(seed * 1000003ull + (uint64_t)i);
    if (infl == 0) cf[i] = -1;  // influences nobody: F (no interpolation if S_i empty)
  }
  std::vector<int> und;
  for (int i = 0; i < n; ++i)
    if (cf[i] == 0) und.push_back(i);
  std::vector<char> newc(n, 0);
  while (!und.empty()) {
    // independent set: local maxima of the measure among undecided neighbours
#pragma omp parallel for schedule(static)
    for (size_t u = 0; u < und.size(); ++u) {
      int i = und[u];
      bool best = true;
      for (int k = srp[i]; k < srp[i + 1] && best; ++k) {
        int j = sci[k];
        if (cf[j] == 0 && lam[j] > lam[i]) best = false;
      }
      for (int k = trp[i]; k < trp[i + 1] && best; ++k) {
        int j = tci[k];
        if (cf[j] == 0 && lam[j] > lam[i]) best = false;
      }
      newc[i] = best;
    }
    const long nu = (long)und.size();
#pragma omp parallel for schedule(static)
    for (long u = 0; u < nu; ++u)
      if (newc[und[u]]) cf[und[u]] = 1;
    // points that strongly depend on a new C point become F (every writer
    // stores the same -1 into a still-undecided point)
#pragma omp parallel for schedule(static)
    for (long u = 0; u < nu; ++u) {
      const int i = und[u];
      if (!newc[i]) continue;
      newc[i] = 0;
      for (int k = trp[i]; k < trp[i + 1]; ++k) {
        const int j = tci[k];
        int cj;
#pragma omp atomic read
        cj = cf[j];
        if (cj == 0) {
#pragma omp atomic write
          cf[j] = -1;
        }
      }
    }
    std::vector<int> next;
    next.reserve(und.size());
    for (int i : und)
      if (cf[i] == 0) next.push_back(i);
    if (next.size() == und.size()) {  // cannot happen with distinct measures; guard anyway
      for (int i : next) cf[i] = 1;
      next.clear();
    }
    und.swap(next);
  }
}

static void direct_interp(const HCsr &A, double w, const std::vector<int> &fn, const std::vector<int> &srp,
                          const std::vector<int> &sci, const std::vector<int> &cf, int pmax, HCsr &P) {
  const int n = A.n;
  std::vector<int> cidx(n, -1);
  int nc = 0;
  for (int i = 0; i < n; ++i)
    if (cf[i] == 1) cidx[i] = nc++;
  P.n = n;
  P.m = nc;
  // row i of P into `row` (sorted by coarse column); `strong` is a zeroed
  // marker array of n entries, returned zeroed
  auto make_row = [&](int i, std::vector<char> &strong, std::vector<std::pair<int, double>> &row) {
    row.clear();
    if (cf[i] == 1) {
      row.push_back({cidx[i], 1.0});
      return;
    }
    for (int k = srp[i]; k < srp[i + 1]; ++k) strong[sci[k]] = 1;
    double diag = 0, sn = 0, sp = 0, cn = 0, cp = 0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int j = A.ci[k];
      double a = combined(A, k, w);
      if (j == i) { diag = a; continue; }
      if (!same_fn(fn, i, j)) continue;
      if (a < 0) sn += a; else sp += a;
      if (cf[j] == 1 && strong[j]) { if (a < 0) cn += a; else cp += a; }
    }
    double alpha = cn != 0 ? sn / cn : 0.0;
    double beta = cp != 0 ? sp / cp : 0.0;
    if (cp == 0) diag += sp;
    if (diag != 0) {
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        int j = A.ci[k];
        if (j == i || cf[j] != 1 || !strong[j]) continue;
        double a = combined(A, k, w);
        row.push_back({cidx[j], -(a < 0 ? alpha : beta) * a / diag});
      }
    }
    for (int k = srp[i]; k < srp[i + 1]; ++k) strong[sci[k]] = 0;
    if ((int)row.size() > pmax) {
      double tot = 0, kept = 0;
      for (auto &p : row) tot += p.second;
      // largest |w| first; equal magnitudes: the lower coarse column (the
      // earlier entry of the row) first, so that the choice is deterministic
      std::partial_sort(row.begin(), row.begin() + pmax, row.end(),
                        [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
                          const double fa = std::fabs(a.second), fb = std::fabs(b.second);
                          return fa > fb || (fa == fb && a.first < b.first);
                        });
      row.resize(pmax);
      for (auto &p : row) kept += p.second;
      if (kept != 0)
        for (auto &p : row) p.second *= tot / kept;
    }
    std::sort(row.begin(), row.end());
  };
  // two passes over the rows (sizes, then entries) with per-thread scratch:
  // no per-row allocation; each row is computed the same way both times
  P.rp.assign(n + 1, 0);
#pragma omp parallel
  {
    std::vector<char> strong(n, 0);
    std::vector<std::pair<int, double>> row;
#pragma omp for schedule(dynamic, 1024)
    for (int i = 0; i < n; ++i) {
      make_row(i, strong, row);
      P.rp[i + 1] = (int)row.size();
    }
  }
  for (int i = 0; i < n; ++i) P.rp[i + 1] += P.rp[i];
  P.ci.resize(P.rp[n]);
  P.vc.resize(P.rp[n]);
  P.vm.clear();
#pragma omp parallel
  {
    std::vector<char> strong(n, 0);
    std::vector<std::pair<int, double>> row;
#pragma omp for schedule(dynamic, 1024)
    for (int i = 0; i < n; ++i) {
      make_row(i, strong, row);
      for (size_t k = 0; k < row.size(); ++k) {
        P.ci[P.rp[i] + k] = row[k].first;
        P.vc[P.rp[i] + k] = row[k].second;
      }
    }
  }
}

// A^T with the entries of every row in increasing column order of A (the
// order a serial row-by-row scatter gives): rows of A are split into one
// contiguous chunk per thread, and each thread scatters its chunk behind the
// entries of the chunks before it.
HCsr transpose(const HCsr &A) {
  HCsr T;
  T.n = A.m;
  T.m = A.n;
  const long nnz = A.nnz();
  const bool two = !A.vm.empty();
  T.rp.assign(T.n + 1, 0);
  T.ci.resize(nnz);
  T.vc.resize(nnz);
  if (two) T.vm.resize(nnz);
#ifdef _OPENMP
  const int nth = std::max(1, std::min(omp_get_max_threads(), (int)(nnz / 65536) + 1));
#else
  const int nth = 1;
#endif
  std::vector<std::vector<int>> cnt(nth, std::vector<int>(T.n, 0));
  auto chunk = [&](int t, int &r0, int &r1) {
    r0 = (int)((long)A.n * t / nth);
    r1 = (int)((long)A.n * (t + 1) / nth);
  };
#pragma omp parallel for num_threads(nth) schedule(static, 1)
  for (int t = 0; t < nth; ++t) {
    int r0, r1;
    chunk(t, r0, r1);
    for (long k = A.rp[r0]; k < A.rp[r1]; ++k) cnt[t][A.ci[k]]++;
  }
  for (int c = 0; c < T.n; ++c) {
    int tot = 0;
    for (int t = 0; t < nth; ++t) {
      const int v = cnt[t][c];
      cnt[t][c] = tot;  // offset of thread t inside row c
      tot += v;
    }
    T.rp[c + 1] = T.rp[c] + tot;
  }
#pragma omp parallel for num_threads(nth) schedule(static, 1)
  for (int t = 0; t < nth; ++t) {
    int r0, r1;
    chunk(t, r0, r1);
    std::vector<int> &pos = cnt[t];
    for (int i = r0; i < r1; ++i)
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        const int c = A.ci[k];
        const int p = T.rp[c] + pos[c]++;
        T.ci[p] = i;
        T.vc[p] = A.vc[k];
        if (two) T.vm[p] = A.vm[k];
      }
  }
  return T;
}

// C = A * B, A with one or two parts, B single part.  Rows in parallel.
HCsr spgemm(const HCsr &A, const HCsr &B) {
  HCsr C;
  C.n = A.n;
  C.m = B.m;
  const bool two = !A.vm.empty();
  std::vector<int> cnt(A.n + 1, 0);
#pragma omp parallel
  {
    std::vector<int> mark(B.m, -1);
#pragma omp for schedule(dynamic, 256)
    for (int i = 0; i < A.n; ++i) {
      int c = 0;
      for (int ka = A.rp[i]; ka < A.rp[i + 1]; ++ka) {
        int j = A.ci[ka];
        for (int kb = B.rp[j]; kb < B.rp[j + 1]; ++kb)
          if (mark[B.ci[kb]] != i) { mark[B.ci[kb]] = i; ++c; }
      }
      cnt[i + 1] = c;
    }
  }
  C.rp.assign(A.n + 1, 0);
  for (int i = 0; i < A.n; ++i) C.rp[i + 1] = C.rp[i] + cnt[i + 1];
  C.ci.resize(C.rp[A.n]);
  C.vc.resize(C.rp[A.n]);
  if (two) C.vm.resize(C.rp[A.n]);
#pragma omp parallel
  {
    std::vector<int> mark(B.m, -1);
    std::vector<double> ac(B.m), am(two ? B.m : 0);
    std::vector<int> cols;
#pragma omp for schedule(dynamic, 256)
    for (int i = 0; i < A.n; ++i) {
      cols.clear();
      for (int ka = A.rp[i]; ka < A.rp[i + 1]; ++ka) {
        int j = A.ci[ka];
        double vc = A.vc[ka], vm = two ? A.vm[ka] : 0.0;
        for (int kb = B.rp[j]; kb < B.rp[j + 1]; ++kb) {
          int c = B.ci[kb];
          double b = B.vc[kb];
          if (mark[c] != i) {
            mark[c] = i;
            ac[c] = 0;
            if (two) am[c] = 0;
            cols.push_back(c);
          }
          ac[c] += vc * b;
          if (two) am[c] += vm * b;
        }
      }
      std::sort(cols.begin(), cols.end());
      int p = C.rp[i];
      for (int c : cols) {
        C.ci[p] = c;
        C.vc[p] = ac[c];
        if (two) C.vm[p] = am[c];
        ++p;
      }
    }
  }
  return C;
}

// Galerkin product C = R A P in one pass per coarse row (R, P single part,
// A one or two parts): no intermediate A P, both value parts together.
HCsr galerkin(const HCsr &R, const HCsr &A, const HCsr &P) {
  HCsr C;
  C.n = R.n;
  C.m = P.m;
  const bool two = !A.vm.empty();
  // one pass: each thread appends its rows to its own arena (columns sorted,
  // values summed in the order R's, A's and P's entries are met); the rows
  // are then copied into place
  struct Arena {
    std::vector<int> ci;
    std::vector<double> vc, vm;
  };
#ifdef _OPENMP
  const int nth = omp_get_max_threads();
#else
  const int nth = 1;
#endif
  std::vector<Arena> arena(nth);
  std::vector<int> owner(C.n), start(C.n), len(C.n);
#pragma omp parallel num_threads(nth)
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num();
#else
    const int tid = 0;
#endif
    Arena &ar = arena[tid];
    std::vector<int> mark(P.m, -1);
    std::vector<double> ac(P.m), am(two ? P.m : 0);
    std::vector<int> cols;
#pragma omp for schedule(dynamic, 64)
    for (int I = 0; I < C.n; ++I) {
      cols.clear();
      for (int kr = R.rp[I]; kr < R.rp[I + 1]; ++kr) {
        const int i = R.ci[kr];
        const double r = R.vc[kr];
        for (int ka = A.rp[i]; ka < A.rp[i + 1]; ++ka) {
          const int k = A.ci[ka];
          const double rc = r * A.vc[ka], rm = two ? r * A.vm[ka] : 0.0;
          for (int kp = P.rp[k]; kp < P.rp[k + 1]; ++kp) {
            const int J = P.ci[kp];
            if (mark[J] != I) {
              mark[J] = I;
              ac[J] = 0;
              if (two) am[J] = 0;
              cols.push_back(J);
            }
            ac[J] += rc * P.vc[kp];
            if (two) am[J] += rm * P.vc[kp];
          }
        }
      }
      std::sort(cols.begin(), cols.end());
      owner[I] = tid;
      start[I] = (int)ar.ci.size();
      len[I] = (int)cols.size();
      for (int J : cols) {
        ar.ci.push_back(J);
        ar.vc.push_back(ac[J]);
        if (two) ar.vm.push_back(am[J]);
      }
    }
  }
  C.rp.assign(C.n + 1, 0);
  for (int I = 0; I < C.n; ++I) C.rp[I + 1] = C.rp[I] + len[I];
  C.ci.resize(C.rp[C.n]);
  C.vc.resize(C.rp[C.n]);
  if (two) C.vm.resize(C.rp[C.n]);
#pragma omp parallel for schedule(static)
  for (int I = 0; I < C.n; ++I) {
    const Arena &ar = arena[owner[I]];
    std::copy(ar.ci.begin() + start[I], ar.ci.begin() + start[I] + len[I], C.ci.begin() + C.rp[I]);
    std::copy(ar.vc.begin() + start[I], ar.vc.begin() + start[I] + len[I], C.vc.begin() + C.rp[I]);
    if (two) std::copy(ar.vm.begin() + start[I], ar.vm.begin() + start[I] + len[I], C.vm.begin() + C.rp[I]);
  }
  return C;
}

void amg_build(HCsr A, double w_ref, const AmgParams &prm, HostAmg &out) {
  out.lv.clear();
  std::vector<int> fn;
  if (prm.num_functions > 1) {
    fn.resize(A.n);
    for (int i = 0; i < A.n; ++i) fn[i] = i % prm.num_functions;
  }
  for (int l = 0;; ++l) {
    if (A.n <= prm.max_coarse || l + 1 >= prm.max_levels) break;
    std::vector<int> srp, sci, cf;
    strength(A, w_ref, prm.theta, fn, srp, sci);
    pmis(A.n, srp, sci, prm.seed + (uint64_t)l, cf);
    HCsr P;
    direct_interp(A, w_ref, fn, srp, sci, cf, prm.pmax, P);
    if (P.m == 0 || P.m > 0.95 * A.n) break;
    if (!fn.empty()) {  // a coarse point keeps its function
      std::vector<int> fc;
      fc.reserve(P.m);
      for (int i = 0; i < A.n; ++i)
        if (cf[i] == 1) fc.push_back(fn[i]);
      fn.swap(fc);
    }
    HCsr R = transpose(P);
    HCsr RAP = galerkin(R, A, P);
    HostLevel L;
    L.A = std::move(A);
    L.P = std::move(P);
    L.R = std::move(R);
    out.lv.push_back(std::move(L));
    A = std::move(RAP);
  }
  out.coarse = std::move(A);
}

// Generalized inverse of Ac + w Am (semidefinite Cholesky; pivots that collapse
// to rounding level are pinned, which solves the consistent singular systems
// of the gradient space whose null space holds the constants).
void coarse_inverse(const HCsr &A, double w, std::vector<double> &X) {
  const int n = A.n;
  std::vector<double> L((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) L[(size_t)i * n + A.ci[k]] = combined(A, k, w);
  // symmetrize against rounding
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j) {
      double v = 0.5 * (L[(size_t)i * n + j] + L[(size_t)j * n + i]);
      L[(size_t)i * n + j] = L[(size_t)j * n + i] = v;
    }
  std::vector<char> live(n, 1);
  for (int j = 0; j < n; ++j) {
    double a = L[(size_t)j * n + j];
    double s = a;
    for (int k = 0; k < j; ++k) s -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
    if (!(s > 1e-12 * std::fabs(a))) {
      live[j] = 0;
      for (int i = j; i < n; ++i) L[(size_t)i * n + j] = 0.0;
      continue;
    }
    s = std::sqrt(s);
    L[(size_t)j * n + j] = s;
    for (int i = j + 1; i < n; ++i) {
      double v = L[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) v -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
      L[(size_t)i * n + j] = v / s;
    }
  }
  X.assign((size_t)n * n, 0.0);
  std::vector<double> y(n);
  for (int c = 0; c < n; ++c) {
    for (int i = 0; i < n; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) v -= L[(size_t)i * n + k] * y[k];
      y[i] = live[i] ? v / L[(size_t)i * n + i] : 0.0;
    }
    for (int i = n - 1; i >= 0; --i) {
      double v = y[i];
      for (int k = i + 1; k < n; ++k) v -= L[(size_t)k * n + i] * y[k];
      y[i] = live[i] ? v / L[(size_t)i * n + i] : 0.0;
    }
    for (int i = 0; i < n; ++i) X[(size_t)i * n + c] = y[i];
  }
}

}  // namespace emg
