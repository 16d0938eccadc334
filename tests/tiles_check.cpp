// Row tiling of a CSR pattern (emg_tiles.cpp, host side of the tiled SpMM),
// built and run by test_tiles_host_cpu.py.  For banded random patterns and
// several shared-memory budgets: every tile's column list is strictly
// ascending and no longer than the budget, every nonzero's local index points
// at its own column, the chosen R is the largest power of two <= r_max whose
// busiest tile fits, and an impossible budget is refused.
#include <algorithm>
#include <cstdio>
#include <random>
#include <set>
#include <vector>

#include "emg_tiles.h"

using namespace emg;

static int busiest(int n, const std::vector<int> &rp, const std::vector<int> &ci, int R) {
  int w = 0;
  for (int t = 0; t * R < n; ++t) {
    std::set<int> s(ci.begin() + rp[t * R], ci.begin() + rp[std::min(n, (t + 1) * R)]);
    w = std::max(w, (int)s.size());
  }
  return w;
}

int main() {
  std::mt19937 rng(3);
  const int n = 20011;
  std::vector<int> rp(n + 1, 0), ci;
  for (int i = 0; i < n; ++i) {
    std::set<int> s;
    const int deg = 5 + (int)(rng() % 20);
    for (int d = 0; d < deg; ++d) {
      const int j = i + (int)(rng() % 401) - 200;
      if (j >= 0 && j < n) s.insert(j);
    }
    s.insert(i);
    ci.insert(ci.end(), s.begin(), s.end());
    rp[i + 1] = (int)ci.size();
  }
  for (int lim : {4096, 700, 300, 150}) {
    int R = 0, umax = 0;
    std::vector<int> urp, ucol;
    std::vector<unsigned short> lci;
    const bool ok = tile_rows(n, rp, ci, lim, 128, R, umax, urp, ucol, lci);
    int expect_R = 0;
    for (int r = 128; r >= 8; r /= 2)
      if (busiest(n, rp, ci, r) <= lim) {
        expect_R = r;
        break;
      }
    if (!ok) {
      if (expect_R) { printf("FAIL refused a fitting budget %d\n", lim); return 1; }
      continue;
    }
    if (R != expect_R) { printf("FAIL R=%d expected %d (budget %d)\n", R, expect_R, lim); return 1; }
    const int nt = (int)urp.size() - 1;
    if (nt != (n + R - 1) / R || (int)lci.size() != rp[n]) { printf("FAIL sizes\n"); return 1; }
    for (int t = 0; t < nt; ++t) {
      if (urp[t + 1] - urp[t] > umax || umax > lim) { printf("FAIL list longer than budget\n"); return 1; }
      for (int u = urp[t] + 1; u < urp[t + 1]; ++u)
        if (ucol[u] <= ucol[u - 1]) { printf("FAIL list not ascending\n"); return 1; }
      for (int k = rp[t * R]; k < rp[std::min(n, (t + 1) * R)]; ++k)
        if (lci[k] >= urp[t + 1] - urp[t] || ucol[urp[t] + lci[k]] != ci[k]) { printf("FAIL local index\n"); return 1; }
    }
  }
  int R, umax;
  std::vector<int> urp, ucol;
  std::vector<unsigned short> lci;
  if (tile_rows(n, rp, ci, 10, 128, R, umax, urp, ucol, lci)) { printf("FAIL accepted an impossible budget\n"); return 1; }
  printf("ok\n");
  return 0;
}
