// Shared device helpers for element kernels.
//
// Canonical tet: the kernels see every tet with its four vertices sorted by
// global id.  Canonical local edge k joins sorted vertices (p,q) from
// kEdgeP/kEdgeQ with p<q, so it runs from the lower to the higher global
// vertex id -- the orientation of edgelist after build_edge_info
// (src/em_mesh.cc:448-461) and of the reference's Whitney basis
// phi = l_a grad l_b - l_b grad l_a with a = edgelist[e][0]
// (src/em_fe.cc:176-180, src/em_mesh.h:156-172).  Every index below is a
// compile-time constant, so element matrices stay in registers.
#pragma once

#include <cuda_runtime.h>

namespace emg {

__host__ __device__ constexpr int kEdgeP(int k) { return k < 3 ? 0 : (k < 5 ? 1 : 2); }
__host__ __device__ constexpr int kEdgeQ(int k) { return k < 3 ? k + 1 : (k < 5 ? k - 1 : 3); }
// face f (opposite sorted vertex f) contains canonical edges not touching f
__host__ __device__ constexpr bool kEdgeOnFace(int k, int f) { return kEdgeP(k) != f && kEdgeQ(k) != f; }

// packed symmetric 4x4 index
__host__ __device__ constexpr int sym_idx(int p, int q) {
  return p <= q ? p * (7 - p) / 2 + q : q * (7 - q) / 2 + p;
}

struct TetGeom {
  double x[4][3];   // sorted vertices
  double gr[4][3];  // gradients of the barycentric coordinates
  double vol;       // signed volume of the tet in its input orientation
  int ge[6];        // canonical global edges
  int v[4];         // sorted vertex ids
};

// Loads a canonical tet: ctet (sorted vertex ids), cedge (canonical global
// edges) and cpar (+1/-1 parity of the sort) come from canonicalize_kernel.
__device__ __forceinline__ void load_tet_geom(const double *__restrict__ pts, const int *__restrict__ ctet,
                                              const int *__restrict__ cedge, const signed char *__restrict__ cpar,
                                              int t, TetGeom &g) {
  int4 v = __ldg(reinterpret_cast<const int4 *>(ctet) + t);
  g.v[0] = v.x; g.v[1] = v.y; g.v[2] = v.z; g.v[3] = v.w;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int d = 0; d < 3; ++d) g.x[p][d] = __ldg(pts + 3 * (long)g.v[p] + d);
#pragma unroll
  for (int k = 0; k < 6; ++k) g.ge[k] = __ldg(cedge + 6 * (long)t + k);
  double e1[3], e2[3], e3[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    e1[d] = g.x[1][d] - g.x[0][d];
    e2[d] = g.x[2][d] - g.x[0][d];
    e3[d] = g.x[3][d] - g.x[0][d];
  }
  double c23[3] = {e2[1] * e3[2] - e2[2] * e3[1], e2[2] * e3[0] - e2[0] * e3[2], e2[0] * e3[1] - e2[1] * e3[0]};
  double c31[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2], e3[0] * e1[1] - e3[1] * e1[0]};
  double c12[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  double det = e1[0] * c23[0] + e1[1] * c23[1] + e1[2] * c23[2];
  double inv = 1.0 / det;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    g.gr[1][d] = c23[d] * inv;
    g.gr[2][d] = c31[d] * inv;
    g.gr[3][d] = c12[d] * inv;
    g.gr[0][d] = -(g.gr[1][d] + g.gr[2][d] + g.gr[3][d]);
  }
  g.vol = (double)__ldg(cpar + t) * det / 6.0;
}

// barycentric coordinate of sorted vertex p at point y
__device__ __forceinline__ double lambda_at(const TetGeom &g, int p, const double y[3]) {
  // lambda_p(y) = 1/4-free form: lambda_p(x_p) = 1 and linear
  return 1.0 + g.gr[p][0] * (y[0] - g.x[p][0]) + g.gr[p][1] * (y[1] - g.x[p][1]) + g.gr[p][2] * (y[2] - g.x[p][2]);
}

}  // namespace emg
