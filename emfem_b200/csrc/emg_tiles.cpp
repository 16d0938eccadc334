// Row tiling of a CSR pattern with per-tile column lists (host side of the
// tiled SpMM, emg_linalg.cuh: spmm_tiled_kernel).

#include <algorithm>
#include <vector>

#include "emg_tiles.h"

namespace emg {

bool tile_rows(int n, const std::vector<int> &rp, const std::vector<int> &ci, int umax_limit, int r_max, int &R_out,
               int &umax_out, std::vector<int> &urp, std::vector<int> &ucol, std::vector<unsigned short> &lci) {
  if (n <= 0 || umax_limit < 1) return false;
  umax_limit = std::min(umax_limit, 65536);  // local indices are 16-bit
  for (int R = r_max; R >= 8; R /= 2) {
    const int nt = (n + R - 1) / R;
    std::vector<int> cnt(nt + 1, 0);
    int worst = 0;
#pragma omp parallel
    {
      std::vector<int> cols;
#pragma omp for schedule(dynamic, 64) reduction(max : worst)
      for (int t = 0; t < nt; ++t) {
        cols.assign(ci.begin() + rp[t * R], ci.begin() + rp[std::min(n, (t + 1) * R)]);
        std::sort(cols.begin(), cols.end());
        const int u = (int)(std::unique(cols.begin(), cols.end()) - cols.begin());
        cnt[t + 1] = u;
        worst = std::max(worst, u);
      }
    }
    if (worst > umax_limit) continue;
    for (int t = 0; t < nt; ++t) cnt[t + 1] += cnt[t];
    ucol.assign(cnt[nt], 0);
    lci.assign(rp[n], 0);
#pragma omp parallel
    {
      std::vector<int> cols;
#pragma omp for schedule(dynamic, 64)
      for (int t = 0; t < nt; ++t) {
        const int kb = rp[t * R], ke = rp[std::min(n, (t + 1) * R)];
        cols.assign(ci.begin() + kb, ci.begin() + ke);
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        std::copy(cols.begin(), cols.end(), ucol.begin() + cnt[t]);
        for (int k = kb; k < ke; ++k)
          lci[k] = (unsigned short)(std::lower_bound(cols.begin(), cols.end(), ci[k]) - cols.begin());
      }
    }
    urp.swap(cnt);
    R_out = R;
    umax_out = std::max(worst, 1);
    return true;
  }
  return false;
}

}  // namespace emg
