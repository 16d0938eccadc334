// Row tiling of a CSR pattern for the tiled SpMM (host, emg_tiles.cpp).
#pragma once

#include <vector>

namespace emg {

// Tiles of R consecutive rows (R the largest power of two <= r_max, >= 8,
// whose busiest tile has at most umax_limit distinct columns): tile t's
// distinct columns, ascending, are ucol[urp[t] .. urp[t+1]) and lci[k] is
// nonzero k's position in its tile's list.  umax_out = the largest list.
// Returns false when no R qualifies.
bool tile_rows(int n, const std::vector<int> &rp, const std::vector<int> &ci, int umax_limit, int r_max, int &R_out,
               int &umax_out, std::vector<int> &urp, std::vector<int> &ucol, std::vector<unsigned short> &lci);

}  // namespace emg
