// Host AMG checks (built and run by test_amg_host_cpu.py): on a Kuhn-grid
// Laplacian with two value parts, with one and with three functions per
// vertex (weakly coupled), the hierarchy from amg_build must satisfy
//   * R = P^T exactly; P has at most pmax entries per row; every coarse
//     column J has exactly one identity row (its C point);
//   * each Galerkin operator equals R (A P) formed by two sparse products to
//     1e-13 of its largest entry, and is symmetric;
//   * with three functions, P never interpolates across functions.
// Prints "ok" or the first failure.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "emg_amg.h"

using namespace emg;

static HCsr grid(int N, int nf) {
  const int n = N * N * N;
  const int off[14][3] = {{1, 0, 0},  {-1, 0, 0},  {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}, {1, 1, 0},
                          {-1, -1, 0}, {0, 1, 1}, {0, -1, -1}, {1, 0, 1}, {-1, 0, -1}, {1, 1, 1}, {-1, -1, -1}};
  HCsr A;
  A.n = A.m = n * nf;
  A.rp.assign(n * nf + 1, 0);
  for (int v = 0; v < n; ++v) {
    const int i = v % N, j = (v / N) % N, k = v / (N * N);
    std::vector<int> nb;
    for (auto &o : off) {
      const int a = i + o[0], b = j + o[1], c = k + o[2];
      if (a < 0 || b < 0 || c < 0 || a >= N || b >= N || c >= N) continue;
      nb.push_back((c * N + b) * N + a);
    }
    nb.push_back(v);
    std::sort(nb.begin(), nb.end());
    for (int f = 0; f < nf; ++f) {
      for (int u : nb)
        for (int g = 0; g < nf; ++g) {
          if (g != f && u != v) continue;  // cross-function couplings only on the diagonal block
          double c = u == v ? (g == f ? (double)(nb.size() - 1) + 1.3 : -0.6) : -1.0;
          A.ci.push_back(u * nf + g);
          A.vc.push_back(c);
          A.vm.push_back(u == v && g == f ? 1.0 : (u == v ? 0.0 : 0.1));
        }
      A.rp[v * nf + f + 1] = (int)A.ci.size();
    }
  }
  return A;
}

static double maxabs(const std::vector<double> &a) {
  double m = 0;
  for (double x : a) m = std::max(m, std::fabs(x));
  return m;
}

static int fail(const char *what, int level) {
  printf("FAIL %s at level %d\n", what, level);
  return 1;
}

static int check(int N, int nf) {
  HCsr A0 = grid(N, nf);
  AmgParams p;
  p.num_functions = nf;
  p.max_coarse = 50;
  HostAmg h;
  amg_build(A0, 1.0, p, h);
  if (h.lv.size() < 2) return fail("too few levels", 0);
  std::vector<int> fn(A0.n);
  for (int i = 0; i < A0.n; ++i) fn[i] = i % nf;
  for (size_t l = 0; l < h.lv.size(); ++l) {
    const HostLevel &L = h.lv[l];
    const HCsr &P = L.P, &R = L.R, &A = L.A;
    // R = P^T
    HCsr PT = transpose(P);
    if (PT.rp != R.rp || PT.ci != R.ci || PT.vc != R.vc) return fail("R != P^T", (int)l);
    // P structure; C points from identity rows
    std::vector<int> cpt(P.m, -1);
    for (int i = 0; i < P.n; ++i) {
      const int len = P.rp[i + 1] - P.rp[i];
      if (len > p.pmax) return fail("row of P longer than pmax", (int)l);
      if (len == 1 && P.vc[P.rp[i]] == 1.0) {
        const int J = P.ci[P.rp[i]];
        if (cpt[J] >= 0) {
          // an F point interpolating from one C point with weight 1 is allowed;
          // keep the first identity row whose index maps to J's C point
          continue;
        }
        cpt[J] = i;
      }
    }
    for (int J = 0; J < P.m; ++J)
      if (cpt[J] < 0) return fail("coarse column without identity row", (int)l);
    if (nf > 1)
      for (int i = 0; i < P.n; ++i)
        for (int k = P.rp[i]; k < P.rp[i + 1]; ++k)
          if (fn[cpt[P.ci[k]]] != fn[i]) return fail("interpolation across functions", (int)l);
    // Galerkin product against two sparse products
    const HCsr &C = l + 1 < h.lv.size() ? h.lv[l + 1].A : h.coarse;
    HCsr AP = spgemm(A, P);
    HCsr APc = AP;
    APc.vm.clear();
    HCsr RAPc = spgemm(R, APc);
    HCsr APm = AP;
    APm.vc = AP.vm;
    APm.vm.clear();
    HCsr RAPm = spgemm(R, APm);
    if (RAPc.rp != C.rp || RAPc.ci != C.ci) return fail("Galerkin pattern", (int)l);
    const double sc = maxabs(C.vc), sm = maxabs(C.vm);
    for (size_t k = 0; k < C.vc.size(); ++k) {
      if (std::fabs(C.vc[k] - RAPc.vc[k]) > 1e-13 * sc) return fail("Galerkin values (part 1)", (int)l);
      if (std::fabs(C.vm[k] - RAPm.vc[k]) > 1e-13 * sm) return fail("Galerkin values (part 2)", (int)l);
    }
    // symmetry of the coarse operator
    HCsr CT = transpose(C);
    if (CT.rp != C.rp || CT.ci != C.ci) return fail("coarse pattern not symmetric", (int)l);
    for (size_t k = 0; k < C.vc.size(); ++k)
      if (std::fabs(C.vc[k] - CT.vc[k]) > 1e-13 * sc) return fail("coarse operator not symmetric", (int)l);
    // functions of the coarse unknowns, for the next level
    std::vector<int> fc(P.m);
    for (int J = 0; J < P.m; ++J) fc[J] = fn[cpt[J]];
    fn.swap(fc);
  }
  return 0;
}

int main() {
  if (check(18, 1) || check(12, 3)) return 1;
  printf("ok\n");
  return 0;
}
