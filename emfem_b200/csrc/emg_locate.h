// Point location index (emg_locate.cpp): find_cell_around_point
// (src/em_mesh.cc:527-566) without the per-query O(T) bitmap.
#pragma once

#include <vector>

namespace emg {

// sign (-1, 0, 1) of orient3d(a, b, c, d) = det[a-d; b-d; c-d], exact (the
// sign of TetGen's robust predicate, which the containment test reads)
int orient3d_sign(const double *a, const double *b, const double *c, const double *d);

struct PointIndex {
  int nv = 0, nt = 0;
  std::vector<double> pts;
  std::vector<int> tets, nbr, v2t;
  double lo[3], hi[3], h[3], hmin = 0;
  int dim[3] = {1, 1, 1};
  std::vector<int> cell_start, cell_vertex;  // vertices bucketed by grid cell
  PointIndex(int nv, const double *pts, int nt, const int *tets, const int *nbr);
  int closest_vertex(const double *p) const;
  bool contains(int t, const double *p) const;
  int find(const double *p) const;  // tet index, or -1 when no tet contains p
 private:
  void cell_coords(const double *p, int c[3]) const;
  long cell_id(const double *p) const;
};

}  // namespace emg
