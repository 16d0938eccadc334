// Point location: find_cell_around_point (src/em_mesh.cc:527-566) with a
// reusable index.
//
// The reference starts from the tet stored for the vertex closest to the
// point (vertex_to_tet keeps the last tet listed for each vertex,
// src/em_mesh.cc:510-515) and walks the neighbour graph breadth-first until a
// tet contains the point, clearing an O(T) bitmap per query.  Here the
// closest vertex comes from a uniform grid of the vertices (exact nearest
// neighbour, ties to the lowest vertex index) and the visited set is a
// per-query hash set, so a query costs the walk it makes and nothing more.
// The walk and the containment test are the reference's, with the exact
// orientation sign of its predicate, so every point gets the same tet, ties
// on shared faces included.

#include <algorithm>
#include <cmath>
#include <queue>
#include <unordered_set>
#include <vector>

#include "emg_locate.h"

namespace emg {

namespace {

// Exact sign of a sum of products of doubles with floating-point expansions
// (Shewchuk, "Adaptive precision floating-point arithmetic and fast robust
// geometric predicates", Discrete Comput. Geom. 18, 1997): a value is an
// unevaluated sum of doubles of increasing magnitude that do not overlap, so
// its sign is the sign of its largest nonzero term.  Round to nearest; no
// FMA contraction in the error-free transformations (fma is called only
// where its single rounding is the point: the product's error term).
struct Expansion {
  double t[160];
  int n = 0;
  // e += b exactly (grow-expansion with zero elimination)
  void add(double b) {
    int m = 0;
    double q = b;
    for (int i = 0; i < n; ++i) {
      const double x = q + t[i];
      const double bv = x - q, av = x - bv;
      const double err = (q - av) + (t[i] - bv);
      q = x;
      if (err != 0.0) t[m++] = err;
    }
    if (q != 0.0 || m == 0) t[m++] = q;
    n = m;
  }
  // e += sign * p * q * r exactly: p q = hi + lo (two-product), then each
  // part times r is again a two-product, four terms in all
  void add_product3(double sign, double p, double q, double r) {
    const double hi = p * q, lo = std::fma(p, q, -hi);
    const double a = hi * r, ae = std::fma(hi, r, -a);
    const double b = lo * r, be = std::fma(lo, r, -b);
    add(sign * be);
    add(sign * b);
    add(sign * ae);
    add(sign * a);
  }
  int sign() const {
    for (int i = n - 1; i >= 0; --i)
      if (t[i] != 0.0) return t[i] > 0.0 ? 1 : -1;
    return 0;
  }
};

// sign of det3 of rows p, q, r, added to e with the given sign
void add_det3(Expansion &e, double sign, const double *p, const double *q, const double *r) {
  e.add_product3(sign, p[0], q[1], r[2]);
  e.add_product3(-sign, p[0], q[2], r[1]);
  e.add_product3(-sign, p[1], q[0], r[2]);
  e.add_product3(sign, p[1], q[2], r[0]);
  e.add_product3(sign, p[2], q[0], r[1]);
  e.add_product3(-sign, p[2], q[1], r[0]);
}

// exact sign of det[a-d; b-d; c-d] = det4 of the rows (x, y, z, 1) of a, b,
// c, d = det3(a,b,c) - det3(a,b,d) + det3(a,c,d) - det3(b,c,d), evaluated on
// the input coordinates themselves (the differences a - d would round)
int orient3d_exact(const double *a, const double *b, const double *c, const double *d) {
  Expansion e;
  add_det3(e, 1.0, a, b, c);
  add_det3(e, -1.0, a, b, d);
  add_det3(e, 1.0, a, c, d);
  add_det3(e, -1.0, b, c, d);
  return e.sign();
}

// orient3d(a,b,c,d) = det[a-d; b-d; c-d] (TetGen's robust predicate, whose
// sign is exact): a floating-point filter (error bound 1e-14 of the
// permanent, above the 7.8e-16 that bounds the rounding of this evaluation),
// then the exact sign from orient3d_exact
double orient3d(const double *a, const double *b, const double *c, const double *d) {
  const double adx = a[0] - d[0], bdx = b[0] - d[0], cdx = c[0] - d[0];
  const double ady = a[1] - d[1], bdy = b[1] - d[1], cdy = c[1] - d[1];
  const double adz = a[2] - d[2], bdz = b[2] - d[2], cdz = c[2] - d[2];
  const double det = adx * (bdy * cdz - bdz * cdy) + bdx * (cdy * adz - cdz * ady) + cdx * (ady * bdz - adz * bdy);
  const double perm = (std::fabs(bdy * cdz) + std::fabs(bdz * cdy)) * std::fabs(adx) +
                      (std::fabs(cdy * adz) + std::fabs(cdz * ady)) * std::fabs(bdx) +
                      (std::fabs(ady * bdz) + std::fabs(adz * bdy)) * std::fabs(cdx);
  if (std::fabs(det) > 1e-14 * perm) return det;
  return (double)orient3d_exact(a, b, c, d);
}

}  // namespace

int orient3d_sign(const double *a, const double *b, const double *c, const double *d) {
  const double v = orient3d(a, b, c, d);
  return v > 0.0 ? 1 : (v < 0.0 ? -1 : 0);
}

PointIndex::PointIndex(int nv_, const double *pts_, int nt_, const int *tets_, const int *nbr_)
    : nv(nv_), nt(nt_), pts(pts_, pts_ + 3 * (size_t)nv_), tets(tets_, tets_ + 4 * (size_t)nt_),
      nbr(nbr_, nbr_ + 4 * (size_t)nt_), v2t(nv_, 0) {
  for (int t = 0; t < nt; ++t)
    for (int k = 0; k < 4; ++k) v2t[tets[4 * (size_t)t + k]] = t;
  for (int d = 0; d < 3; ++d) {
    lo[d] = 1e300;
    hi[d] = -1e300;
  }
  for (int v = 0; v < nv; ++v)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], pts[3 * (size_t)v + d]);
      hi[d] = std::max(hi[d], pts[3 * (size_t)v + d]);
    }
  // about two vertices per cell on a box of the vertices' extents
  const double target = std::max(1.0, nv / 2.0);
  double ext[3], vol = 1;
  for (int d = 0; d < 3; ++d) {
    ext[d] = std::max(hi[d] - lo[d], 1e-300);
    vol *= ext[d];
  }
  const double side = std::cbrt(vol / target);
  hmin = 1e300;
  long ncell = 1;
  for (int d = 0; d < 3; ++d) {
    dim[d] = (int)std::min(1024.0, std::max(1.0, std::floor(ext[d] / side)));
    h[d] = ext[d] / dim[d];
    hmin = std::min(hmin, h[d]);
    ncell *= dim[d];
  }
  cell_start.assign(ncell + 1, 0);
  std::vector<long> cell_of(nv);
  for (int v = 0; v < nv; ++v) {
    cell_of[v] = cell_id(&pts[3 * (size_t)v]);
    cell_start[cell_of[v] + 1]++;
  }
  for (long c = 0; c < ncell; ++c) cell_start[c + 1] += cell_start[c];
  cell_vertex.resize(nv);
  std::vector<int> pos(cell_start.begin(), cell_start.end() - 1);
  for (int v = 0; v < nv; ++v) cell_vertex[pos[cell_of[v]]++] = v;  // ascending v inside a cell
}

void PointIndex::cell_coords(const double *p, int c[3]) const {
  for (int d = 0; d < 3; ++d) {
    double x = (p[d] - lo[d]) / h[d];
    int i = x < 0 ? 0 : (x >= dim[d] ? dim[d] - 1 : (int)x);
    c[d] = i;
  }
}

long PointIndex::cell_id(const double *p) const {
  int c[3];
  cell_coords(p, c);
  return ((long)c[2] * dim[1] + c[1]) * dim[0] + c[0];
}

// nearest vertex, ties to the lowest index (squared distances as
// (dx*dx + dy*dy) + dz*dz, the same expression for every candidate)
int PointIndex::closest_vertex(const double *p) const {
  int c0[3];
  cell_coords(p, c0);
  double best = 1e300;
  int bv = -1;
  const int rmax = std::max(dim[0], std::max(dim[1], dim[2]));
  for (int r = 0; r <= rmax; ++r) {
    for (int k = c0[2] - r; k <= c0[2] + r; ++k) {
      if (k < 0 || k >= dim[2]) continue;
      for (int j = c0[1] - r; j <= c0[1] + r; ++j) {
        if (j < 0 || j >= dim[1]) continue;
        for (int i = c0[0] - r; i <= c0[0] + r; ++i) {
          if (i < 0 || i >= dim[0]) continue;
          // only the shell of Chebyshev radius r
          if (std::max(std::abs(i - c0[0]), std::max(std::abs(j - c0[1]), std::abs(k - c0[2]))) != r) continue;
          const long c = ((long)k * dim[1] + j) * dim[0] + i;
          for (int q = cell_start[c]; q < cell_start[c + 1]; ++q) {
            const int v = cell_vertex[q];
            const double *x = &pts[3 * (size_t)v];
            const double dd = (p[0] - x[0]) * (p[0] - x[0]) + (p[1] - x[1]) * (p[1] - x[1]) + (p[2] - x[2]) * (p[2] - x[2]);
            if (dd < best || (dd == best && v < bv)) {
              best = dd;
              bv = v;
            }
          }
        }
      }
    }
    // every cell beyond this shell is at least r * hmin from the point's
    // projection onto the grid box, hence from the point itself; one shell
    // of slack covers vertices that rounding put into a neighbouring cell
    const double bound = (r > 0 ? r - 1 : 0) * hmin;
    if (bv >= 0 && best < bound * bound) break;
  }
  return bv;
}

bool PointIndex::contains(int t, const double *p) const {
  const double *v[4];
  for (int k = 0; k < 4; ++k) v[k] = &pts[3 * (size_t)tets[4 * (size_t)t + k]];
  const double d0 = orient3d(v[0], v[1], v[3], p);
  const double d1 = orient3d(v[1], v[2], v[3], p);
  const double d2 = orient3d(v[1], v[0], v[2], p);
  const double d3 = orient3d(v[0], v[3], v[2], p);
  return d0 >= 0.0 && d1 >= 0.0 && d2 >= 0.0 && d3 >= 0.0;
}

int PointIndex::find(const double *p) const {
  const int v = closest_vertex(p);
  if (v < 0) return -1;
  std::unordered_set<int> touched;
  std::queue<int> q;
  q.push(v2t[v]);
  while (!q.empty()) {
    const int t = q.front();
    q.pop();
    if (!touched.insert(t).second) continue;
    if (contains(t, p)) return t;
    for (int i = 0; i < 4; ++i) {
      const int n = nbr[4 * (size_t)t + i];
      if (n >= 0 && !touched.count(n)) q.push(n);
    }
  }
  return -1;
}

}  // namespace emg
