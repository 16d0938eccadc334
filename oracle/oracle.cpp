// EMFEM CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 FP64 restatement of the reference's per-frequency forward
// solve, used by the test-suite as the parity checker and by bench.py as the
// timed CPU baseline.  Nothing in the emfem_b200 product links, loads or calls
// this file.
//
// Parity status: the reference ships no tests, fixtures or golden vectors and
// cannot be compiled here (PETSc, hypre, TetGen, Metis, Eigen and MPI are
// absent), so the restatement is pinned by known-answer tests instead:
// closed-form Whitney element matrices, quadrature sums, curl(grad)=0,
// symmetry/SPD of the assembled operators and the exact 1-D layered
// plane-wave solution.  The PETSc/hypre solver internals (FGMRES, FCG, AMS,
// BoomerAMG) are restated from their published methods; their iteration
// counts are not pinned ("parity unpinned"), only the converged answers are.
//
// Every function cites the reference file:line it restates.

#include <algorithm>
#include <cassert>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <queue>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

#include <chrono>
static double wall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static const double PI = 3.14159265358979323846;   // em_defs.h:16
static const double MU = 4 * PI * 1E-7;            // em_defs.h:17
static const double DTOR = PI / 180.0;             // em_defs.h:21
static const double EPS = 1.0E-6;                  // em_defs.h:23
static const cplx II(0.0, 1.0);                    // em_defs.h:18

extern "C" {

struct OrcMesh {
  int nv, nt, ne;
  const double *pts;        // 3*nv
  const int *tets;          // 4*nt
  const int *attr;          // nt
  const int *edges;         // 2*ne (sorted endpoints)
  const int *tet2edge;      // 6*nt
  const int *nbr;           // 4*nt
  const int *non;           // 4*nt
  const unsigned char *ebdr;// ne
};

struct OrcModel {
  int aniso_form;  // em_defs.h:37
  int nrho, ncol;
  const double *rho;  // nrho*ncol row-major
};

}  // extern "C"

// ---------------------------------------------------------------------------
// small dense helpers (replace Eigen)
// ---------------------------------------------------------------------------
struct V3 {
  double x[3];
  double &operator[](int i) { return x[i]; }
  double operator[](int i) const { return x[i]; }
};
static inline V3 mk(double a, double b, double c) { V3 v; v[0] = a; v[1] = b; v[2] = c; return v; }
static inline V3 sub(const V3 &a, const V3 &b) { return mk(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
static inline double dot(const V3 &a, const V3 &b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline V3 cross(const V3 &a, const V3 &b) {
  return mk(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
static inline double norm(const V3 &a) { return std::sqrt(dot(a, a)); }

struct Z3 { cplx x[3]; };

// 4x4 inverse and determinant by cofactor expansion.
static double det4(const double m[16]) {
  double inv0 = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
  double inv4 = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
  double inv8 = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
  double inv12 = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
  return m[0] * inv0 + m[1] * inv4 + m[2] * inv8 + m[3] * inv12;
}
static void inv4(const double m[16], double out[16]) {
  double inv[16];
  inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
  inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
  inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
  inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
  inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
  inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
  inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
  inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
  inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
  inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
  inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
  inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
  inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
  inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
  inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
  inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
  double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
  for (int i = 0; i < 16; ++i) out[i] = inv[i] / det;
}

// ---------------------------------------------------------------------------
// TetAccessor (em_mesh.h:129-283)
// ---------------------------------------------------------------------------
struct Tet {
  const OrcMesh *m;
  int t;
  V3 vertex(int v) const {
    const double *p = m->pts + 3 * (size_t)m->tets[4 * (size_t)t + v];
    return mk(p[0], p[1], p[2]);
  }
  int vertex_index(int v) const { return m->tets[4 * (size_t)t + v]; }
  int edge_index(int e) const { return m->tet2edge[6 * (size_t)t + e]; }
  // em_mesh.h:156-172
  int edge_end_point(int e, int ep) const {
    int ge = m->tet2edge[6 * (size_t)t + e];
    for (int v = 0; v < 4; ++v)
      if (m->edges[2 * (size_t)ge + ep] == m->tets[4 * (size_t)t + v]) return v;
    assert(false);
    return -1;
  }
  bool edge_on_boundary(int e) const { return m->ebdr[edge_index(e)] != 0; }
  int neighbor(int f) const { return m->nbr[4 * (size_t)t + f]; }
  int neighbor_of_neighbor(int f) const { return m->non[4 * (size_t)t + f]; }
  int attribute() const { return m->attr[t]; }
  // jac = [[1 1 1 1],[v0 v1 v2 v3]] as in em_fe.cc:139-142 (row-major here)
  void jac(double J[16]) const {
    for (int i = 0; i < 4; ++i) {
      V3 p = vertex(i);
      J[0 * 4 + i] = 1.0;
      J[1 * 4 + i] = p[0];
      J[2 * 4 + i] = p[1];
      J[3 * 4 + i] = p[2];
    }
  }
  // em_mesh.h:196-206
  double volume() const { double J[16]; jac(J); return det4(J) / 6.0; }
  // em_mesh.h:232-254 (circumradius of the tetrahedron)
  double diameter() const {
    V3 v[4];
    for (int i = 0; i < 4; ++i) v[i] = vertex(i);
    double a = norm(sub(v[1], v[2])), b = norm(sub(v[0], v[2])), c = norm(sub(v[0], v[1]));
    double aa = norm(sub(v[0], v[3])), bb = norm(sub(v[1], v[3])), cc = norm(sub(v[2], v[3]));
    double la = a * aa, lb = b * bb, lc = c * cc;
    double s = 0.5 * (la + lb + lc);
    return std::sqrt(s * (s - la) * (s - lb) * (s - lc)) / (6.0 * volume());
  }
  // em_mesh.h:256-274 (circumradius of face f)
  double face_diameter(int f) const {
    V3 v[3];
    for (int i = 0; i < 3; ++i) v[i] = vertex((f + i + 1) % 4);
    double a = norm(sub(v[1], v[2])), b = norm(sub(v[0], v[2])), c = norm(sub(v[0], v[1]));
    double area = 0.25 * std::sqrt((a + b + c) * (b + c - a) * (c + a - b) * (a + b - c));
    return a * b * c / (4.0 * area);
  }
};

// Exact sign of det[a-d; b-d; c-d]: TetGen's orient3d (a robust predicate
// whose sign is exact; it is a third-party source absent here) restated with
// floating-point expansions (Shewchuk 1997: error-free two-sum and
// two-product, grow-expansion).  The determinant is the 4x4 one of the rows
// (x, y, z, 1), i.e. the signed sum of the 24 products x_i y_j z_k over
// distinct rows i, j, k with the sign of the permutation (i, j, k, l).
static void expansion_grow(std::vector<double> &e, double b) {
  std::vector<double> h;
  double q = b;
  for (double ei : e) {
    const double s = q + ei;
    const double bb = s - q;
    const double err = (q - (s - bb)) + (ei - bb);
    q = s;
    if (err != 0.0) h.push_back(err);
  }
  if (q != 0.0 || h.empty()) h.push_back(q);
  e.swap(h);
}

static int orient3d_exact_sign(const V3 &a, const V3 &b, const V3 &c, const V3 &d) {
  const V3 *r[4] = {&a, &b, &c, &d};
  std::vector<double> e;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        if (i == j || i == k || j == k) continue;
        const int l = 6 - i - j - k;
        // parity of the permutation (i, j, k, l) by counting inversions
        const int p[4] = {i, j, k, l};
        int inv = 0;
        for (int u = 0; u < 4; ++u)
          for (int v = u + 1; v < 4; ++v) inv += p[u] > p[v];
        const double sg = (inv & 1) ? -1.0 : 1.0;
        const double x = (*r[i])[0], y = (*r[j])[1], z = (*r[k])[2];
        const double hi = x * y, lo = std::fma(x, y, -hi);
        const double t1 = hi * z, t1e = std::fma(hi, z, -t1);
        const double t2 = lo * z, t2e = std::fma(lo, z, -t2);
        expansion_grow(e, sg * t2e);
        expansion_grow(e, sg * t2);
        expansion_grow(e, sg * t1e);
        expansion_grow(e, sg * t1);
      }
  for (int i = (int)e.size() - 1; i >= 0; --i)
    if (e[i] != 0.0) return e[i] > 0.0 ? 1 : -1;
  return 0;
}

// orient3d(a,b,c,d) = det[a-d; b-d; c-d]: a floating-point filter, then the
// exact sign
static double orient3d(const V3 &a, const V3 &b, const V3 &c, const V3 &d) {
  double adx = a[0] - d[0], bdx = b[0] - d[0], cdx = c[0] - d[0];
  double ady = a[1] - d[1], bdy = b[1] - d[1], cdy = c[1] - d[1];
  double adz = a[2] - d[2], bdz = b[2] - d[2], cdz = c[2] - d[2];
  double det = adx * (bdy * cdz - bdz * cdy) + bdx * (cdy * adz - cdz * ady) + cdx * (ady * bdz - adz * bdy);
  double perm = (std::fabs(bdy * cdz) + std::fabs(bdz * cdy)) * std::fabs(adx) +
                (std::fabs(cdy * adz) + std::fabs(cdz * ady)) * std::fabs(bdx) +
                (std::fabs(ady * bdz) + std::fabs(adz * bdy)) * std::fabs(cdx);
  if (std::fabs(det) > 1e-14 * perm) return det;
  return (double)orient3d_exact_sign(a, b, c, d);
}

// em_mesh.h:208-230
static bool contains_point(const Tet &tet, const V3 &p) {
  V3 v[4];
  for (int i = 0; i < 4; ++i) v[i] = tet.vertex(i);
  double d[4];
  d[0] = orient3d(v[0], v[1], v[3], p);
  d[1] = orient3d(v[1], v[2], v[3], p);
  d[2] = orient3d(v[1], v[0], v[2], p);
  d[3] = orient3d(v[0], v[3], v[2], p);
  int gt = 0;
  for (int i = 0; i < 4; ++i) gt += d[i] >= 0.0;
  return gt == 4;
}

// ---------------------------------------------------------------------------
// FEValues (em_fe.cc:156-285)
// ---------------------------------------------------------------------------
struct FEV {
  Tet tet;
  double a[4], b[4], c[4], d[4];
  int ev[6][2], fv[4][3], fe[4][3];
  void reinit(const Tet &t) {
    tet = t;
    // generate_meta_info em_fe.cc:238-268
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 2; ++j) ev[i][j] = tet.edge_end_point(i, j);
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 3; ++j) fv[i][j] = (i + j + 1) % 4;
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 6; ++k)
          if ((fv[i][j] == ev[k][0] && fv[i][(j + 1) % 3] == ev[k][1]) ||
              (fv[i][j] == ev[k][1] && fv[i][(j + 1) % 3] == ev[k][0]))
            fe[i][j] = k;
    // calculate_coefs em_fe.cc:270-285: rows of the inverse Jacobian
    double J[16], Ji[16];
    tet.jac(J);
    inv4(J, Ji);
    for (int i = 0; i < 4; ++i) {
      a[i] = Ji[i * 4 + 0];
      b[i] = Ji[i * 4 + 1];
      c[i] = Ji[i * 4 + 2];
      d[i] = Ji[i * 4 + 3];
    }
  }
  double value_q(int n, const V3 &p) const { return a[n] + p[0] * b[n] + p[1] * c[n] + p[2] * d[n]; }
  V3 grad_q(int n) const { return mk(b[n], c[n], d[n]); }
  // em_fe.cc:176-180
  V3 value_nedelec(int e, const V3 &p) const {
    double l0 = value_q(ev[e][0], p), l1 = value_q(ev[e][1], p);
    V3 g0 = grad_q(ev[e][0]), g1 = grad_q(ev[e][1]);
    return mk(l0 * g1[0] - l1 * g0[0], l0 * g1[1] - l1 * g0[1], l0 * g1[2] - l1 * g0[2]);
  }
  // em_fe.cc:182-185
  V3 curl_nedelec(int e) const {
    V3 cr = cross(grad_q(ev[e][0]), grad_q(ev[e][1]));
    return mk(2 * cr[0], 2 * cr[1], 2 * cr[2]);
  }
  // em_fe.cc:207-210
  V3 face_normal(int f) const {
    V3 n = mk(-b[f], -c[f], -d[f]);
    double l = norm(n);
    return mk(n[0] / l, n[1] / l, n[2] / l);
  }
};

// em_fe.cc:82-128 (p=2) and em_fe.cc:130-154
static void cell_quadrature(const Tet &tet, V3 q[4], double jxw[4]) {
  const double A = 0.585410196624969, B = 0.138196601125011;
  const double ref[4][3] = {{A, B, B}, {B, A, B}, {B, B, A}, {B, B, B}};
  double J[16];
  tet.jac(J);
  double dj = det4(J);
  for (int i = 0; i < 4; ++i) {
    double nc[4] = {1 - ref[i][0] - ref[i][1] - ref[i][2], ref[i][0], ref[i][1], ref[i][2]};
    for (int r = 0; r < 3; ++r) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += J[(r + 1) * 4 + k] * nc[k];
      q[i][r] = s;
    }
    jxw[i] = dj * (1.0 / 24.0);
  }
}

// em_fe.cc:6-44 (p=2) and em_fe.cc:46-80
static void face_quadrature(const Tet &tet, int f, V3 q[3], double jxw[3]) {
  const double ref[3][3] = {{2.0 / 3, 1.0 / 6, 1.0 / 6}, {1.0 / 6, 2.0 / 3, 1.0 / 6}, {1.0 / 6, 1.0 / 6, 2.0 / 3}};
  double J[16], Ji[16];
  tet.jac(J);
  inv4(J, Ji);
  double dj = det4(J);
  V3 row = mk(Ji[f * 4 + 1] * dj * 6, Ji[f * 4 + 2] * dj * 6, Ji[f * 4 + 3] * dj * 6);
  double s = norm(row);
  for (int i = 0; i < 3; ++i) {
    double nc[4];
    nc[f] = 0.0;
    for (int j = 0; j < 3; ++j) nc[(f + j + 1) % 4] = ref[i][j];
    for (int r = 0; r < 3; ++r) {
      double v = 0;
      for (int k = 0; k < 4; ++k) v += J[(r + 1) * 4 + k] * nc[k];
      q[i][r] = v;
    }
    jxw[i] = s * (1.0 / 6.0);
  }
}

// em_fwd.cc:14-72
static void cell_sigma(const OrcModel *md, int idx, double s[9]) {
  for (int i = 0; i < 9; ++i) s[i] = 0;
  const double *r = md->rho + (size_t)idx * md->ncol;
  switch (md->aniso_form) {
  case 0: s[0] = s[4] = s[8] = 1.0 / r[0]; break;
  case 1: s[0] = s[4] = 1.0 / r[0]; s[8] = 1.0 / r[1]; break;
  case 2: s[0] = 1.0 / r[0]; s[4] = 1.0 / r[1]; s[8] = 1.0 / r[2]; break;
  case 3: {
    double sd[9] = {1.0 / r[0], 0, 0, 0, 1.0 / r[1], 0, 0, 0, 1.0 / r[2]};
    double X[9] = {1, 0, 0, 0, std::cos(r[3] * DTOR), std::sin(r[3] * DTOR), 0, -std::sin(r[3] * DTOR), std::cos(r[3] * DTOR)};
    double Y[9] = {std::cos(r[4] * DTOR), 0, -std::sin(r[4] * DTOR), 0, 1, 0, std::sin(r[4] * DTOR), 0, std::cos(r[4] * DTOR)};
    double Z[9] = {std::cos(r[5] * DTOR), std::sin(r[5] * DTOR), 0, -std::sin(r[5] * DTOR), std::cos(r[5] * DTOR), 0, 0, 0, 1};
    auto mul = [](const double *A, const double *B, double *C) {
      double T[9];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double v = 0;
          for (int k = 0; k < 3; ++k) v += A[i * 3 + k] * B[k * 3 + j];
          T[i * 3 + j] = v;
        }
      std::memcpy(C, T, sizeof(T));
    };
    double R[9], Rt[9], T[9];
    mul(Z, Y, R);
    mul(R, X, R);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) Rt[i * 3 + j] = R[j * 3 + i];
    mul(R, sd, T);
    mul(T, Rt, s);
    break;
  }
  default: break;
  }
}

static V3 matvec3(const double s[9], const V3 &v) {
  return mk(s[0] * v[0] + s[1] * v[1] + s[2] * v[2], s[3] * v[0] + s[4] * v[1] + s[5] * v[2],
            s[6] * v[0] + s[7] * v[1] + s[8] * v[2]);
}

// element matrices as in em_fwd.cc:356-375 (before boundary zeroing)
static void element_matrices(const Tet &cell, const FEV &fv, const double sig[9], double omega,
                             double c[36], double m[36]) {
  V3 q[4];
  double jxw[4];
  cell_quadrature(cell, q, jxw);
  for (int i = 0; i < 36; ++i) c[i] = m[i] = 0;
  for (int i = 0; i < 6; ++i) {
    for (int j = 0; j <= i; ++j) {
      for (int k = 0; k < 4; ++k) {
        c[i * 6 + j] += (1.0 / MU) * dot(fv.curl_nedelec(i), fv.curl_nedelec(j)) * jxw[k];
        m[i * 6 + j] += omega * dot(fv.value_nedelec(i, q[k]), matvec3(sig, fv.value_nedelec(j, q[k]))) * jxw[k];
      }
      if (i != j) {
        c[j * 6 + i] = c[i * 6 + j];
        m[j * 6 + i] = m[i * 6 + j];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// sparse matrices
// ---------------------------------------------------------------------------
struct Csr {
  int n = 0, m = 0;
  std::vector<int> rp, ci;
  std::vector<double> v;
};

static void spmv(const Csr &A, const double *x, double *y) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A.n; ++i) {
    double s = 0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) s += A.v[k] * x[A.ci[k]];
    y[i] = s;
  }
}

static Csr transpose(const Csr &A) {
  Csr T;
  T.n = A.m;
  T.m = A.n;
  T.rp.assign(T.n + 1, 0);
  for (int k = 0; k < A.rp[A.n]; ++k) T.rp[A.ci[k] + 1]++;
  for (int i = 0; i < T.n; ++i) T.rp[i + 1] += T.rp[i];
  T.ci.resize(A.rp[A.n]);
  T.v.resize(A.rp[A.n]);
  std::vector<int> pos(T.rp.begin(), T.rp.end() - 1);
  for (int i = 0; i < A.n; ++i)
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int p = pos[A.ci[k]]++;
      T.ci[p] = i;
      T.v[p] = A.v[k];
    }
  return T;
}

// C = A*B with a dense accumulator per row (Gustavson); columns sorted.
static Csr spgemm(const Csr &A, const Csr &B) {
  Csr C;
  C.n = A.n;
  C.m = B.m;
  C.rp.assign(C.n + 1, 0);
  std::vector<int> mark(B.m, -1);
  std::vector<double> acc(B.m, 0.0);
  std::vector<int> cols;
  for (int i = 0; i < A.n; ++i) {
    cols.clear();
    for (int ka = A.rp[i]; ka < A.rp[i + 1]; ++ka) {
      int j = A.ci[ka];
      double av = A.v[ka];
      for (int kb = B.rp[j]; kb < B.rp[j + 1]; ++kb) {
        int c = B.ci[kb];
        if (mark[c] != i) {
          mark[c] = i;
          acc[c] = 0;
          cols.push_back(c);
        }
        acc[c] += av * B.v[kb];
      }
    }
    std::sort(cols.begin(), cols.end());
    for (int c : cols) {
      C.ci.push_back(c);
      C.v.push_back(acc[c]);
    }
    C.rp[i + 1] = (int)C.ci.size();
  }
  return C;
}

// ---------------------------------------------------------------------------
// sparsity pattern (em_fwd.cc:191-246), single rank: every tet owned
// ---------------------------------------------------------------------------
static void sparsity(const OrcMesh *m, std::vector<int> &rp, std::vector<int> &ci) {
  std::vector<std::vector<int>> pat(m->ne);
  for (int t = 0; t < m->nt; ++t) {
    int idx[6];
    for (int i = 0; i < 6; ++i) idx[i] = m->tet2edge[6 * (size_t)t + i];
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) pat[idx[i]].push_back(idx[j]);
  }
  rp.assign(m->ne + 1, 0);
  ci.clear();
  for (int i = 0; i < m->ne; ++i) {
    std::sort(pat[i].begin(), pat[i].end());
    pat[i].erase(std::unique(pat[i].begin(), pat[i].end()), pat[i].end());
    rp[i] = (int)ci.size();
    ci.insert(ci.end(), pat[i].begin(), pat[i].end());
    std::vector<int>().swap(pat[i]);
  }
  rp[m->ne] = (int)ci.size();
}

static int find_slot(const int *rp, const int *ci, int r, int c) {
  const int *b = ci + rp[r], *e = ci + rp[r + 1];
  const int *p = std::lower_bound(b, e, c);
  assert(p != e && *p == c);
  return (int)(p - ci);
}

// ---------------------------------------------------------------------------
// assembly (em_fwd.cc:318-400)
// ---------------------------------------------------------------------------
static void assemble(const OrcMesh *m, const OrcModel *md, double omega, const int *rp, const int *ci,
                     double *C, double *M, unsigned char *bdr_cell) {
  size_t nnz = rp[m->ne];
  std::fill(C, C + nnz, 0.0);
  std::fill(M, M + nnz, 0.0);
  for (int t = 0; t < m->nt; ++t) {
    Tet cell{m, t};
    double sig[9];
    cell_sigma(md, cell.attribute(), sig);
    FEV fv;
    fv.reinit(cell);
    double c[36], mm[36];
    element_matrices(cell, fv, sig, omega, c, mm);
    if (bdr_cell) bdr_cell[t] = 0;
    for (int i = 0; i < 6; ++i) {
      if (cell.edge_on_boundary(i)) {
        for (int j = 0; j < 6; ++j) {
          if (j != i) c[i * 6 + j] = c[j * 6 + i] = 0.0;
          mm[i * 6 + j] = mm[j * 6 + i] = 0.0;
        }
        if (bdr_cell) bdr_cell[t] = 1;
      }
    }
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) {
        int s = find_slot(rp, ci, cell.edge_index(i), cell.edge_index(j));
        C[s] += c[i * 6 + j];
        M[s] += mm[i * 6 + j];
      }
  }
}

// ---------------------------------------------------------------------------
// 1-D layered plane wave (em_pw.h:6-139)
// ---------------------------------------------------------------------------
struct PlaneWave {
  int nlay;
  double omega;
  std::vector<double> ztop, lsig;
  std::vector<cplx> a, b, c, d;
  void initialize(const double *zt, const double *ls, int n, double freq) {
    nlay = n;
    ztop.assign(zt, zt + n);
    lsig.assign(ls, ls + n);
    omega = 2 * PI * freq;
    std::vector<cplx> kk(nlay + 1), Rp(nlay + 1, 0.0), expmgh(nlay + 1, 0.0);
    for (int i = 1; i <= nlay; ++i) kk[i] = std::sqrt(-II * omega * MU * lsig[i - 1]);
    kk[0] = std::sqrt(-II * omega * MU * lsig[0]);
    for (int i = 1; i <= nlay - 1; ++i) expmgh[i] = std::exp(-kk[i] * (ztop[i] - ztop[i - 1]));
    for (int i = nlay - 1; i >= 1; --i) {
      cplx gmogp = (-II * omega * MU * (lsig[i - 1] - lsig[i])) / std::pow(kk[i] + kk[i + 1], 2);
      cplx rjexp = Rp[i + 1] * expmgh[i + 1];
      Rp[i] = (gmogp + rjexp) / (1.0 + gmogp * rjexp) * expmgh[i];
    }
    a.assign(nlay + 1, 0.0);
    b.assign(nlay + 1, 0.0);
    c.assign(nlay + 1, 0.0);
    d.assign(nlay + 1, 0.0);
    a[0] = 1.0;
    c[0] = 1.0;
    for (int i = 1; i <= nlay; ++i) {
      cplx Atop = a[i - 1] + b[i - 1] * expmgh[i - 1];
      b[i] = Atop / (1.0 + Rp[i] * expmgh[i]);
      a[i] = b[i] * Rp[i];
      Atop = c[i - 1] + d[i - 1] * expmgh[i - 1];
      d[i] = Atop / (1.0 - Rp[i] * expmgh[i]);
      c[i] = -d[i] * Rp[i];
    }
  }
  void field(double z, cplx eh[4]) const {
    int ilay = 0;
    for (int i = nlay - 1; i >= 0; --i)
      if (z >= ztop[i]) { ilay = i; break; }
    cplx kk = std::sqrt(-II * omega * MU * lsig[ilay]);
    cplx expp = 0.0, exppdz = 0.0;
    cplx expm = std::exp(-kk * (z - ztop[ilay]));
    cplx expmdz = -kk * expm;
    if (ilay != nlay - 1) {
      expp = std::exp(kk * (z - ztop[ilay + 1]));
      exppdz = kk * expp;
    }
    eh[0] = a[ilay + 1] * expp + b[ilay + 1] * expm;
    eh[1] = (a[ilay + 1] * exppdz + b[ilay + 1] * expmdz) / (II * MU * omega);
    eh[2] = (c[ilay + 1] * exppdz + d[ilay + 1] * expmdz) / lsig[ilay];
    eh[3] = c[ilay + 1] * expp + d[ilay + 1] * expm;
    for (int i = 0; i < 4; ++i)
      if (std::abs(eh[i]) < 1E-80) eh[i] = 0.0;
  }
  // em_pw.h:108-119
  void efield(const V3 &p, int mode, cplx ep[3]) const {
    cplx eh[4];
    ep[0] = ep[1] = ep[2] = 0.0;
    field(p[2], eh);
    if (mode == -1) ep[0] = std::conj(eh[0]);
    else if (mode == -2) ep[1] = std::conj(eh[2]);
  }
  void hfield(const V3 &p, int mode, cplx hp[3]) const {
    cplx eh[4];
    hp[0] = hp[1] = hp[2] = 0.0;
    field(p[2], eh);
    if (mode == -1) hp[1] = std::conj(eh[1]);
    else if (mode == -2) hp[0] = std::conj(eh[3]);
  }
};

// ---------------------------------------------------------------------------
// point location (em_mesh.cc:504-566)
// ---------------------------------------------------------------------------
static int closest_vertex(const OrcMesh *m, const V3 &p) {
  int best = 0;
  double bd = 1e300;
  for (int v = 0; v < m->nv; ++v) {
    const double *q = m->pts + 3 * (size_t)v;
    double d = (p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) + (p[2] - q[2]) * (p[2] - q[2]);
    if (d < bd) { bd = d; best = v; }
  }
  return best;
}

static int find_cell(const OrcMesh *m, const std::vector<int> &v2t, const V3 &p) {
  std::vector<char> touched(m->nt, 0);
  std::queue<int> q;
  q.push(v2t[closest_vertex(m, p)]);
  while (!q.empty()) {
    int t = q.front();
    q.pop();
    if (touched[t]) continue;
    touched[t] = 1;
    Tet tet{m, t};
    if (contains_point(tet, p)) return t;
    for (int i = 0; i < 4; ++i) {
      int n = tet.neighbor(i);
      if (n >= 0 && !touched[n]) q.push(n);
    }
  }
  return -1;
}

static std::vector<int> vertex_to_tet(const OrcMesh *m) {
  std::vector<int> v2t(m->nv, 0);
  for (int t = 0; t < m->nt; ++t)
    for (int v = 0; v < 4; ++v) v2t[m->tets[4 * (size_t)t + v]] = t;
  return v2t;
}

// ---------------------------------------------------------------------------
// Krylov solvers and AMS (restated from the published methods; see header)
// ---------------------------------------------------------------------------
struct AmgLevel {
  Csr A, P, R;  // P: n x nc ; R = P^T
  std::vector<double> dense;  // coarsest: Cholesky factor (row-major)
  int nc = 0;
};

struct Amg {
  std::vector<AmgLevel> lv;
  double theta = 0.25;
  int pmax = 4, max_coarse = 64, max_levels = 25;
};

// classical strength: j strongly influences i if -a_ij >= theta*max_k(-a_ik)
// (for a_ii > 0; hypre's default measure).
static void strength(const Csr &A, double theta, std::vector<std::vector<int>> &S) {
  S.assign(A.n, {});
  for (int i = 0; i < A.n; ++i) {
    double mx = 0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] != i) mx = std::max(mx, -A.v[k]);
    if (mx <= 0) continue;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] != i && -A.v[k] >= theta * mx) S[i].push_back(A.ci[k]);
  }
}

// Ruge-Stueben first pass (the form HMIS reduces to on a single process).
static void rs_coarsen(int n, const std::vector<std::vector<int>> &S, std::vector<int> &cf) {
  std::vector<std::vector<int>> ST(n);
  for (int i = 0; i < n; ++i)
    for (int j : S[i]) ST[j].push_back(i);
  std::vector<int> lam(n);
  cf.assign(n, 0);  // 0 undecided, 1 C, -1 F
  std::priority_queue<std::pair<int, int>> pq;
  for (int i = 0; i < n; ++i) {
    lam[i] = (int)ST[i].size();
    if (S[i].empty() && ST[i].empty()) cf[i] = -1;  // isolated: F without interpolation
    else pq.push({lam[i], -i});
  }
  while (!pq.empty()) {
    auto top = pq.top();
    pq.pop();
    int i = -top.second;
    if (cf[i] != 0 || top.first != lam[i]) continue;
    cf[i] = 1;
    for (int j : ST[i]) {
      if (cf[j] != 0) continue;
      cf[j] = -1;
      for (int k : S[j])
        if (cf[k] == 0) { lam[k]++; pq.push({lam[k], -k}); }
    }
    for (int j : S[i])
      if (cf[j] == 0) { lam[j]--; pq.push({lam[j], -j}); }
  }
  for (int i = 0; i < n; ++i)
    if (cf[i] == 0) cf[i] = 1;
}

// direct interpolation with separate positive/negative scaling and Pmax
// truncation.
static Csr direct_interp(const Csr &A, const std::vector<std::vector<int>> &S, const std::vector<int> &cf,
                         int pmax, int &nc) {
  int n = A.n;
  std::vector<int> cidx(n, -1);
  nc = 0;
  for (int i = 0; i < n; ++i)
    if (cf[i] == 1) cidx[i] = nc++;
  Csr P;
  P.n = n;
  P.m = nc;
  P.rp.assign(n + 1, 0);
  std::vector<char> strong(n, 0);
  for (int i = 0; i < n; ++i) {
    if (cf[i] == 1) {
      P.ci.push_back(cidx[i]);
      P.v.push_back(1.0);
      P.rp[i + 1] = (int)P.ci.size();
      continue;
    }
    for (int j : S[i]) strong[j] = 1;
    double diag = 0, sn = 0, sp = 0, cn = 0, cp = 0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int j = A.ci[k];
      double a = A.v[k];
      if (j == i) { diag = a; continue; }
      if (a < 0) sn += a; else sp += a;
      if (cf[j] == 1 && strong[j]) { if (a < 0) cn += a; else cp += a; }
    }
    double alpha = cn != 0 ? sn / cn : 0.0;
    double beta = cp != 0 ? sp / cp : 0.0;
    if (cp == 0) diag += sp;  // lump positive couplings into the diagonal
    std::vector<std::pair<double, int>> w;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int j = A.ci[k];
      if (j == i || cf[j] != 1 || !strong[j]) continue;
      double a = A.v[k];
      double wij = -(a < 0 ? alpha : beta) * a / diag;
      w.push_back({wij, cidx[j]});
    }
    for (int j : S[i]) strong[j] = 0;
    if ((int)w.size() > pmax) {
      double tot = 0, kept = 0;
      for (auto &p : w) tot += p.first;
      std::sort(w.begin(), w.end(), [](const std::pair<double, int> &x, const std::pair<double, int> &y) {
        return std::fabs(x.first) > std::fabs(y.first);
      });
      w.resize(pmax);
      for (auto &p : w) kept += p.first;
      if (kept != 0)
        for (auto &p : w) p.first *= tot / kept;
    }
    std::sort(w.begin(), w.end(), [](const std::pair<double, int> &x, const std::pair<double, int> &y) {
      return x.second < y.second;
    });
    for (auto &p : w) {
      P.ci.push_back(p.second);
      P.v.push_back(p.first);
    }
    P.rp[i + 1] = (int)P.ci.size();
  }
  return P;
}

static void dense_cholesky(const Csr &A, std::vector<double> &L) {
  int n = A.n;
  L.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) L[(size_t)i * n + A.ci[k]] = A.v[k];
  // Semidefinite-aware: the gradient-space operator G^T B G keeps the
  // constants in its null space, so a pivot that collapses to rounding level
  // is dropped (its unknown is pinned to zero), which solves the consistent
  // singular system.
  for (int j = 0; j < n; ++j) {
    double a = L[(size_t)j * n + j];
    double s = a;
    for (int k = 0; k < j; ++k) s -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
    if (!(s > 1e-12 * std::fabs(a))) {
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
}

static void dense_solve(const std::vector<double> &L, int n, const double *b, double *x) {
  for (int i = 0; i < n; ++i) {
    double v = b[i];
    for (int k = 0; k < i; ++k) v -= L[(size_t)i * n + k] * x[k];
    x[i] = L[(size_t)i * n + i] != 0 ? v / L[(size_t)i * n + i] : 0.0;
  }
  for (int i = n - 1; i >= 0; --i) {
    double v = x[i];
    for (int k = i + 1; k < n; ++k) v -= L[(size_t)k * n + i] * x[k];
    x[i] = L[(size_t)i * n + i] != 0 ? v / L[(size_t)i * n + i] : 0.0;
  }
}

static void amg_setup(Amg &amg, const Csr &A0) {
  amg.lv.clear();
  amg.lv.push_back(AmgLevel());
  amg.lv[0].A = A0;
  for (int l = 0;; ++l) {
    AmgLevel &L = amg.lv[l];
    if (L.A.n <= amg.max_coarse || l + 1 >= amg.max_levels) {
      dense_cholesky(L.A, L.dense);
      break;
    }
    std::vector<std::vector<int>> S;
    strength(L.A, amg.theta, S);
    std::vector<int> cf;
    rs_coarsen(L.A.n, S, cf);
    int nc;
    Csr P = direct_interp(L.A, S, cf, amg.pmax, nc);
    if (nc == 0 || nc >= L.A.n) {
      dense_cholesky(L.A, L.dense);
      break;
    }
    L.P = P;
    L.R = transpose(P);
    L.nc = nc;
    AmgLevel next;
    next.A = spgemm(L.R, spgemm(L.A, L.P));
    amg.lv.push_back(std::move(next));
  }
}

// symmetric Gauss-Seidel sweep (hypre relax type 6 on one process)
static void sgs(const Csr &A, const double *b, double *x) {
  for (int pass = 0; pass < 2; ++pass) {
    for (int ii = 0; ii < A.n; ++ii) {
      int i = pass == 0 ? ii : A.n - 1 - ii;
      double s = b[i], d = 0;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        if (A.ci[k] == i) d = A.v[k];
        else s -= A.v[k] * x[A.ci[k]];
      }
      if (d != 0) x[i] = s / d;
    }
  }
}

static void amg_vcycle(const Amg &amg, int l, const double *b, double *x) {
  const AmgLevel &L = amg.lv[l];
  int n = L.A.n;
  if (!L.dense.empty()) {
    dense_solve(L.dense, n, b, x);
    return;
  }
  std::fill(x, x + n, 0.0);
  sgs(L.A, b, x);
  std::vector<double> r(n), rc(L.nc), ec(L.nc, 0.0), e(n);
  spmv(L.A, x, r.data());
  for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
  spmv(L.R, r.data(), rc.data());
  amg_vcycle(amg, l + 1, rc.data(), ec.data());
  spmv(L.P, ec.data(), e.data());
  for (int i = 0; i < n; ++i) x[i] += e[i];
  sgs(L.A, b, x);
}

struct Ams {
  Csr B, G, Pi[3], GT, PiT[3];
  Amg amgG, amgPi[3];
  std::string cycle = "034515430";  // hypre AMS cycle type 13
};

// setup_ams (em_la.cc:230-295) plus the AMS construction of hypre.
static void ams_setup(Ams &ams, const OrcMesh *m, const Csr &B) {
  ams.B = B;
  Csr &G = ams.G;
  G.n = m->ne;
  G.m = m->nv;
  G.rp.resize(m->ne + 1);
  G.ci.resize(2 * (size_t)m->ne);
  G.v.resize(2 * (size_t)m->ne);
  for (int e = 0; e < m->ne; ++e) {
    G.rp[e] = 2 * e;
    G.ci[2 * e] = m->edges[2 * e];
    G.ci[2 * e + 1] = m->edges[2 * e + 1];
    G.v[2 * e] = -1;
    G.v[2 * e + 1] = 1;
  }
  G.rp[m->ne] = 2 * m->ne;
  for (int d = 0; d < 3; ++d) {
    Csr &P = ams.Pi[d];
    P = G;
    for (int e = 0; e < m->ne; ++e) {
      double t = m->pts[3 * (size_t)m->edges[2 * e + 1] + d] - m->pts[3 * (size_t)m->edges[2 * e] + d];
      P.v[2 * e] = 0.5 * t;
      P.v[2 * e + 1] = 0.5 * t;
    }
  }
  ams.GT = transpose(G);
  amg_setup(ams.amgG, spgemm(ams.GT, spgemm(B, G)));
  for (int d = 0; d < 3; ++d) {
    ams.PiT[d] = transpose(ams.Pi[d]);
    amg_setup(ams.amgPi[d], spgemm(ams.PiT[d], spgemm(B, ams.Pi[d])));
  }
}

static void ams_apply(const Ams &ams, const double *b, double *x) {
  int n = ams.B.n;
  std::fill(x, x + n, 0.0);
  std::vector<double> r(n), e(n);
  for (char c : ams.cycle) {
    if (c == '0') {
      sgs(ams.B, b, x);
      continue;
    }
    const Csr *P, *PT;
    const Amg *amg;
    if (c == '1') { P = &ams.G; PT = &ams.GT; amg = &ams.amgG; }
    else { int d = c - '3'; P = &ams.Pi[d]; PT = &ams.PiT[d]; amg = &ams.amgPi[d]; }
    spmv(ams.B, x, r.data());
    for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
    std::vector<double> rs(PT->n), es(PT->n, 0.0);
    spmv(*PT, r.data(), rs.data());
    amg_vcycle(*amg, 0, rs.data(), es.data());
    spmv(*P, es.data(), e.data());
    for (int i = 0; i < n; ++i) x[i] += e[i];
  }
}

static double vdot(const double *a, const double *b, int n) {
  double s = 0;
#pragma omp parallel for reduction(+ : s)
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

// flexible CG with standard truncation (PETSc KSPFCG, mmax=30), zero initial
// guess, unpreconditioned residual norm, rtol relative to ||b||.
static int fcg(const Csr &A, const Ams &pc, const double *b, double *x, double rtol, int maxit, int mmax) {
  int n = A.n;
  std::vector<double> r(b, b + n), z(n);
  std::vector<std::vector<double>> P, S;
  std::vector<double> eta;
  std::fill(x, x + n, 0.0);
  double bn = std::sqrt(vdot(b, b, n));
  if (bn == 0) return 0;
  int it;
  for (it = 0; it < maxit; ++it) {
    ams_apply(pc, r.data(), z.data());
    std::vector<double> p(z);
    for (size_t j = 0; j < P.size(); ++j) {
      double beta = vdot(z.data(), S[j].data(), n) / eta[j];
      for (int i = 0; i < n; ++i) p[i] -= beta * P[j][i];
    }
    std::vector<double> s(n);
    spmv(A, p.data(), s.data());
    double et = vdot(p.data(), s.data(), n);
    double alpha = vdot(p.data(), r.data(), n) / et;
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * s[i];
    }
    P.push_back(std::move(p));
    S.push_back(std::move(s));
    eta.push_back(et);
    if ((int)P.size() > mmax) {
      P.erase(P.begin());
      S.erase(S.begin());
      eta.erase(eta.begin());
    }
    double rn = std::sqrt(vdot(r.data(), r.data(), n));
    if (rn <= rtol * bn) return it + 1;
  }
  return it;
}

struct Solver {
  const OrcMesh *m;
  Csr C, M, B;
  Ams ams;
  double inner_rtol = 1e-2;
  int inner_maxit = 100, inner_mmax = 30;
  long inner_its = 0;
};

// matshell_mult_a (em_la.cc:65-87): y = [C xr - M xi ; -M xr - C xi]
static void mult_a(const Solver &s, const double *x, double *y) {
  int n = s.C.n;
  std::vector<double> w(n);
  spmv(s.C, x, y);
  spmv(s.M, x + n, w.data());
  for (int i = 0; i < n; ++i) y[i] -= w[i];
  spmv(s.M, x, y + n);
  for (int i = 0; i < n; ++i) y[n + i] = -y[n + i];
  spmv(s.C, x + n, w.data());
  for (int i = 0; i < n; ++i) y[n + i] -= w[i];
}

// pc_apply_b (em_la.cc:208-228)
static void pc_apply(Solver &s, const double *b, double *x) {
  int n = s.C.n;
  s.inner_its += fcg(s.B, s.ams, b, x, s.inner_rtol, s.inner_maxit, s.inner_mmax);
  s.inner_its += fcg(s.B, s.ams, b + n, x + n, s.inner_rtol, s.inner_maxit, s.inner_mmax);
}

// FGMRES(restart) with classical Gram-Schmidt (PETSc KSPFGMRES defaults),
// zero initial guess (em_la.cc:49), convergence on the residual estimate.
static int fgmres(Solver &s, const double *b, double *x, double rtol, int maxit, int restart,
                  double *final_true_res) {
  int N = 2 * s.C.n;
  std::fill(x, x + N, 0.0);
  double bn = std::sqrt(vdot(b, b, N));
  int total = 0;
  if (bn == 0) { *final_true_res = 0; return 0; }
  std::vector<double> r(N), w(N);
  while (total < maxit) {
    mult_a(s, x, r.data());
    for (int i = 0; i < N; ++i) r[i] = b[i] - r[i];
    double beta = std::sqrt(vdot(r.data(), r.data(), N));
    if (beta <= rtol * bn) break;
    std::vector<std::vector<double>> V(1, std::vector<double>(N)), Z;
    for (int i = 0; i < N; ++i) V[0][i] = r[i] / beta;
    std::vector<double> H((restart + 1) * restart, 0.0), cs(restart), sn(restart), g(restart + 1, 0.0);
    g[0] = beta;
    int j;
    bool conv = false;
    for (j = 0; j < restart && total < maxit; ++j, ++total) {
      Z.push_back(std::vector<double>(N));
      pc_apply(s, V[j].data(), Z[j].data());
      mult_a(s, Z[j].data(), w.data());
      for (int i = 0; i <= j; ++i) H[i * restart + j] = vdot(w.data(), V[i].data(), N);
      for (int i = 0; i <= j; ++i) {
        double h = H[i * restart + j];
        for (int k = 0; k < N; ++k) w[k] -= h * V[i][k];
      }
      double hn = std::sqrt(vdot(w.data(), w.data(), N));
      H[(j + 1) * restart + j] = hn;
      V.push_back(std::vector<double>(N));
      for (int k = 0; k < N; ++k) V[j + 1][k] = hn > 0 ? w[k] / hn : 0.0;
      for (int i = 0; i < j; ++i) {
        double a = H[i * restart + j], bb = H[(i + 1) * restart + j];
        H[i * restart + j] = cs[i] * a + sn[i] * bb;
        H[(i + 1) * restart + j] = -sn[i] * a + cs[i] * bb;
      }
      double a = H[j * restart + j], bb = H[(j + 1) * restart + j];
      double den = std::sqrt(a * a + bb * bb);
      cs[j] = den > 0 ? a / den : 1.0;
      sn[j] = den > 0 ? bb / den : 0.0;
      H[j * restart + j] = den;
      H[(j + 1) * restart + j] = 0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      if (std::fabs(g[j + 1]) <= rtol * bn) { ++j; ++total; conv = true; break; }
    }
    std::vector<double> y(j);
    for (int i = j - 1; i >= 0; --i) {
      double v = g[i];
      for (int k = i + 1; k < j; ++k) v -= H[i * restart + k] * y[k];
      y[i] = v / H[i * restart + i];
    }
    for (int i = 0; i < j; ++i)
      for (int k = 0; k < N; ++k) x[k] += y[i] * Z[i][k];
    if (conv) break;
  }
  mult_a(s, x, r.data());
  for (int i = 0; i < N; ++i) r[i] = b[i] - r[i];
  *final_true_res = std::sqrt(vdot(r.data(), r.data(), N)) / bn;
  return total;
}

// ---------------------------------------------------------------------------
// error estimator (em_fwd.cc:963-1180)
// ---------------------------------------------------------------------------
static void fn_value(const FEV &fv, const V3 &p, const double *re, const double *im, cplx e[3]) {
  e[0] = e[1] = e[2] = 0.0;
  for (int i = 0; i < 6; ++i) {
    int id = fv.tet.edge_index(i);
    cplx v(re[id], im[id]);
    V3 b = fv.value_nedelec(i, p);
    for (int k = 0; k < 3; ++k) e[k] += v * b[k];
  }
}
static void fn_curl(const FEV &fv, const double *re, const double *im, cplx e[3]) {
  e[0] = e[1] = e[2] = 0.0;
  for (int i = 0; i < 6; ++i) {
    int id = fv.tet.edge_index(i);
    cplx v(re[id], im[id]);
    V3 b = fv.curl_nedelec(i);
    for (int k = 0; k < 3; ++k) e[k] += v * b[k];
  }
}
static void zsig(const double s[9], const cplx e[3], cplx o[3]) {
  for (int i = 0; i < 3; ++i) o[i] = s[i * 3 + 0] * e[0] + s[i * 3 + 1] * e[1] + s[i * 3 + 2] * e[2];
}

// ===========================================================================
// C ABI (ctypes)
// ===========================================================================
extern "C" {

int orc_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

void orc_cell_sigma(const OrcModel *md, int idx, double *s9) { cell_sigma(md, idx, s9); }

// FEValues::reinit coefficients: abcd rows (16) and local edge endpoints (12).
void orc_fe_coefs(const OrcMesh *m, int t, double *abcd, int *ev) {
  FEV fv;
  fv.reinit(Tet{m, t});
  for (int i = 0; i < 4; ++i) {
    abcd[i * 4 + 0] = fv.a[i];
    abcd[i * 4 + 1] = fv.b[i];
    abcd[i * 4 + 2] = fv.c[i];
    abcd[i * 4 + 3] = fv.d[i];
  }
  for (int e = 0; e < 6; ++e) { ev[2 * e] = fv.ev[e][0]; ev[2 * e + 1] = fv.ev[e][1]; }
}

void orc_cell_quadrature(const OrcMesh *m, int t, double *q12, double *jxw4) {
  V3 q[4];
  cell_quadrature(Tet{m, t}, q, jxw4);
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 3; ++k) q12[i * 3 + k] = q[i][k];
}

void orc_face_quadrature(const OrcMesh *m, int t, int f, double *q9, double *jxw3) {
  V3 q[3];
  face_quadrature(Tet{m, t}, f, q, jxw3);
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) q9[i * 3 + k] = q[i][k];
}

void orc_element_matrices(const OrcMesh *m, const OrcModel *md, int t, double omega, double *c36, double *m36) {
  Tet cell{m, t};
  FEV fv;
  fv.reinit(cell);
  double sig[9];
  cell_sigma(md, cell.attribute(), sig);
  element_matrices(cell, fv, sig, omega, c36, m36);
}

void orc_tet_geometry(const OrcMesh *m, int t, double *vol, double *diam, double *fdiam4) {
  Tet tet{m, t};
  *vol = tet.volume();
  *diam = tet.diameter();
  for (int f = 0; f < 4; ++f) fdiam4[f] = tet.face_diameter(f);
}

// make_sparsity_patterns; returns nnz, or -(needed nnz) when cap is too small.
long orc_sparsity(const OrcMesh *m, int *rp, int *ci, long cap) {
  std::vector<int> r, c;
  sparsity(m, r, c);
  if ((long)c.size() > cap) return -(long)c.size();
  std::copy(r.begin(), r.end(), rp);
  std::copy(c.begin(), c.end(), ci);
  return (long)c.size();
}

void orc_assemble(const OrcMesh *m, const OrcModel *md, double freq, const int *rp, const int *ci,
                  double *C, double *M, unsigned char *bdr_cell) {
  assemble(m, md, 2 * PI * freq, rp, ci, C, M, bdr_cell);
}

void orc_matshell_mult(int n, const int *rp, const int *ci, const double *C, const double *M,
                       const double *x, double *y) {
  Csr Cc, Mc;
  Cc.n = Cc.m = Mc.n = Mc.m = n;
  Cc.rp.assign(rp, rp + n + 1);
  Cc.ci.assign(ci, ci + rp[n]);
  Mc.rp = Cc.rp;
  Mc.ci = Cc.ci;
  Cc.v.assign(C, C + rp[n]);
  Mc.v.assign(M, M + rp[n]);
  Solver s;
  s.C = Cc;
  s.M = Mc;
  mult_a(s, x, y);
}

void orc_plane_wave(int nlay, const double *ztop, const double *lsig, double freq, int nz, const double *z,
                    double *eh_out /* nz*4 complex */) {
  PlaneWave pw;
  pw.initialize(ztop, lsig, nlay, freq);
  for (int i = 0; i < nz; ++i) {
    cplx eh[4];
    pw.field(z[i], eh);
    for (int k = 0; k < 4; ++k) {
      eh_out[(i * 4 + k) * 2] = eh[k].real();
      eh_out[(i * 4 + k) * 2 + 1] = eh[k].imag();
    }
  }
}

int orc_find_cell(const OrcMesh *m, int np, const double *p, int *tet_out) {
  std::vector<int> v2t = vertex_to_tet(m);
  int bad = 0;
  for (int i = 0; i < np; ++i) {
    tet_out[i] = find_cell(m, v2t, mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]));
    bad += tet_out[i] < 0;
  }
  return bad;
}

// generate_layered_model (em_fwd.cc:74-133) and update_background_model
// (em_fwd.cc:135-159): layered columns below the four top corners.
// Output: corners (4x3), nlay[4], ztop/lsig (4 x maxl).
int orc_background_model(const OrcMesh *m, const OrcModel *md, int maxl, double *corners, int *nlay,
                         double *ztop, double *lsig) {
  std::vector<int> v2t = vertex_to_tet(m);
  V3 p = mk(-1e15, -1e15, -1e15);
  V3 tl, br;
  {
    const double *q = m->pts + 3 * (size_t)closest_vertex(m, p);
    tl = mk(q[0], q[1], q[2]);
    p = mk(1e15, 1e15, 1e15);
    q = m->pts + 3 * (size_t)closest_vertex(m, p);
    br = mk(q[0], q[1], q[2]);
  }
  V3 cs[4] = {mk(tl[0], tl[1], tl[2]), mk(br[0], tl[1], tl[2]), mk(br[0], br[1], tl[2]), mk(tl[0], br[1], tl[2])};
  for (int c = 0; c < 4; ++c) {
    for (int k = 0; k < 3; ++k) corners[c * 3 + k] = cs[c][k];
    std::vector<double> z, sg;
    V3 fp = cs[c];
    while (fp[2] < br[2]) {
      int v = closest_vertex(m, fp);
      int t = find_cell(m, v2t, mk(fp[0], fp[1], fp[2] + EPS));
      if (t < 0) return -1;
      Tet cell{m, t};
      double s[9];
      cell_sigma(md, cell.attribute(), s);
      z.push_back(fp[2]);
      sg.push_back((s[0] + s[4] + s[8]) / 3.0);
      int i;
      for (i = 0; i < 4; ++i) {
        V3 cv = cell.vertex(i);
        if (cell.vertex_index(i) != v && std::fabs(cv[0] - cs[c][0]) < EPS && std::fabs(cv[1] - cs[c][1]) < EPS) {
          fp = cv;
          break;
        }
      }
      if (i == 4) return -2;
    }
    int n = 0;
    ztop[c * maxl + 0] = z[0];
    lsig[c * maxl + 0] = sg[0];
    n = 1;
    for (size_t i = 0; i + 1 < z.size(); ++i)
      if (sg[i] != sg[i + 1]) {
        if (n >= maxl) return -3;
        ztop[c * maxl + n] = z[i + 1];
        lsig[c * maxl + n] = sg[i + 1];
        ++n;
      }
    nlay[c] = n;
  }
  return 0;
}

// calculate_boundary_values (em_fwd.cc:402-486) + assemble_rhs_mt
// (em_fwd.cc:488-580).  bdr_cell flags come from orc_assemble.
void orc_rhs_mt(const OrcMesh *m, const OrcModel *md, double freq, int mode, const double *corners,
                const int *nlay, const double *ztop, const double *lsig, int maxl, const unsigned char *bdr_cell,
                double *s_re, double *s_im) {
  double omega = 2 * PI * freq;
  PlaneWave pwf[4];
  for (int c = 0; c < 4; ++c) pwf[c].initialize(ztop + c * maxl, lsig + c * maxl, nlay[c], freq);
  V3 tc[4];
  for (int c = 0; c < 4; ++c) tc[c] = mk(corners[c * 3], corners[c * 3 + 1], corners[c * 3 + 2]);
  std::vector<char> have(m->ne, 0);
  std::vector<cplx> bv(m->ne, 0.0);
  for (int t = 0; t < m->nt; ++t) {
    if (!bdr_cell[t]) continue;
    Tet cell{m, t};
    FEV fv;
    fv.reinit(cell);
    for (int i = 0; i < 6; ++i) {
      if (!cell.edge_on_boundary(i)) continue;
      V3 p0 = cell.vertex(cell.edge_end_point(i, 0)), p1 = cell.vertex(cell.edge_end_point(i, 1));
      V3 ec = mk((p0[0] + p1[0]) / 2.0, (p0[1] + p1[1]) / 2.0, (p0[2] + p1[2]) / 2.0);
      V3 ed = sub(p1, p0);
      double co[4];
      if (std::fabs(ec[0] - tc[0][0]) < EPS) {
        double w = (1.0 - std::cos(PI * (ec[1] - tc[0][1]) / (tc[2][1] - tc[0][1]))) / 2.0;
        co[0] = 1.0 - w; co[1] = 0.0; co[2] = 0.0; co[3] = w;
      } else if (std::fabs(ec[1] - tc[0][1]) < EPS) {
        double w = (1.0 - std::cos(PI * (ec[0] - tc[0][0]) / (tc[2][0] - tc[0][0]))) / 2.0;
        co[0] = 1.0 - w; co[1] = w; co[2] = 0.0; co[3] = 0.0;
      } else if (std::fabs(ec[0] - tc[2][0]) < EPS) {
        double w = (1.0 - std::cos(PI * (ec[1] - tc[0][1]) / (tc[2][1] - tc[0][1]))) / 2.0;
        co[0] = 0.0; co[1] = 1.0 - w; co[2] = w; co[3] = 0.0;
      } else if (std::fabs(ec[1] - tc[2][1]) < EPS) {
        double w = (1.0 - std::cos(PI * (ec[0] - tc[0][0]) / (tc[2][0] - tc[0][0]))) / 2.0;
        co[0] = 0.0; co[1] = 0.0; co[2] = w; co[3] = 1.0 - w;
      } else {
        double area = (tc[2][0] - tc[0][0]) * (tc[2][1] - tc[0][1]);
        co[0] = ((tc[2][0] - ec[0]) * (tc[2][1] - ec[1])) / area;
        co[1] = ((ec[0] - tc[3][0]) * (tc[3][1] - ec[1])) / area;
        co[2] = ((ec[0] - tc[0][0]) * (ec[1] - tc[0][1])) / area;
        co[3] = ((tc[1][0] - ec[0]) * (ec[1] - tc[1][1])) / area;
      }
      cplx ep[3] = {0.0, 0.0, 0.0};
      for (int c = 0; c < 4; ++c) {
        cplx e4[3];
        pwf[c].efield(ec, mode, e4);
        for (int k = 0; k < 3; ++k) ep[k] += co[c] * e4[k];
      }
      V3 phi = fv.value_nedelec(i, ec);
      cplx num = ed[0] * ep[0] + ed[1] * ep[1] + ed[2] * ep[2];
      cplx dof = num / dot(ed, phi);
      int gi = cell.edge_index(i);
      if (!have[gi]) {
        have[gi] = 1;
        bv[gi] = std::abs(dof) > 1E-13 ? dof : cplx(0.0);
      }
    }
  }
  std::fill(s_re, s_re + m->ne, 0.0);
  std::fill(s_im, s_im + m->ne, 0.0);
  for (int t = 0; t < m->nt; ++t) {
    if (!bdr_cell[t]) continue;
    Tet cell{m, t};
    FEV fv;
    fv.reinit(cell);
    double sig[9];
    cell_sigma(md, cell.attribute(), sig);
    double c[36], mm[36];
    element_matrices(cell, fv, sig, omega, c, mm);
    double br[6] = {0}, bi[6] = {0};
    for (int i = 0; i < 6; ++i) {
      if (!cell.edge_on_boundary(i)) continue;
      double vr = bv[cell.edge_index(i)].real(), vi = bv[cell.edge_index(i)].imag();
      br[i] = vr * c[i * 6 + i];
      bi[i] = -vi * c[i * 6 + i];
      for (int j = 0; j < 6; ++j) {
        if (!cell.edge_on_boundary(j)) {
          br[j] -= c[j * 6 + i] * vr;
          bi[j] += mm[j * 6 + i] * vr;
          br[j] += mm[j * 6 + i] * vi;
          bi[j] += c[j * 6 + i] * vi;
        }
      }
    }
    for (int i = 0; i < 6; ++i) {
      s_re[cell.edge_index(i)] += br[i];
      s_im[cell.edge_index(i)] += bi[i];
    }
  }
}

// divide_line_source + assemble_rhs_csem (em_fwd.cc:582-671); tx_tet holds
// the cell of every dipole (point location is host mesh work).
int orc_rhs_csem(const OrcMesh *m, double freq, const double *tx, int n_div, double *s_re, double *s_im) {
  double omega = 2 * PI * freq;
  std::vector<double> cx, cy, cz, wt;
  V3 center = mk(tx[0], tx[1], tx[2]);
  V3 dir = mk(std::cos(tx[3] * DTOR) * std::cos(tx[4] * DTOR), std::sin(tx[3] * DTOR) * std::cos(tx[4] * DTOR),
              std::sin(tx[4] * DTOR));
  double current = tx[5], length = tx[6];
  std::vector<V3> pts;
  std::vector<double> w;
  if (std::fabs(tx[6]) <= 0.1) {
    pts.push_back(center);
    w.push_back(1.0);
  } else {
    V3 A = mk(center[0] - dir[0] * length / 2, center[1] - dir[1] * length / 2, center[2] - dir[2] * length / 2);
    for (int i = 0; i < n_div; ++i) {
      V3 B = mk(A[0] + dir[0] * length / n_div, A[1] + dir[1] * length / n_div, A[2] + dir[2] * length / n_div);
      pts.push_back(mk((A[0] + B[0]) / 2, (A[1] + B[1]) / 2, (A[2] + B[2]) / 2));
      w.push_back(1.0 / n_div);
      A = B;
    }
  }
  std::fill(s_re, s_re + m->ne, 0.0);
  std::fill(s_im, s_im + m->ne, 0.0);
  std::vector<int> v2t = vertex_to_tet(m);
  for (size_t j = 0; j < pts.size(); ++j) {
    int t = find_cell(m, v2t, pts[j]);
    if (t < 0) return -1;
    Tet cell{m, t};
    FEV fv;
    fv.reinit(cell);
    for (int i = 0; i < 6; ++i)
      s_im[cell.edge_index(i)] += omega * current * dot(fv.value_nedelec(i, pts[j]), dir) * w[j];
  }
  return 0;
}

// assemble_rhs_dual (em_fwd.cc:673-717)
int orc_rhs_dual(const OrcMesh *m, int nrx, const double *rx, double *s_re, double *s_im) {
  std::fill(s_re, s_re + m->ne, 0.0);
  std::fill(s_im, s_im + m->ne, 0.0);
  std::vector<int> v2t = vertex_to_tet(m);
  for (int r = 0; r < nrx; ++r) {
    V3 p = mk(rx[3 * r], rx[3 * r + 1], rx[3 * r + 2]);
    int t = find_cell(m, v2t, p);
    if (t < 0) return -1 - r;
    Tet cell{m, t};
    FEV fv;
    fv.reinit(cell);
    for (int j = 0; j < 6; ++j) {
      V3 v = fv.value_nedelec(j, p);
      s_re[cell.edge_index(j)] += v[0] + v[1] + v[2];
      s_im[cell.edge_index(j)] += v[0] + v[1] + v[2];
    }
  }
  return 0;
}

// Real-form FGMRES(FCG(AMS)) solve of one right-hand side.  C and M are the
// assembled matrices (M already scaled by omega).  Returns outer iterations;
// stats = {true relative residual, inner iterations, setup seconds unused}.
int orc_solve(const OrcMesh *m, int n, const int *rp, const int *ci, const double *C, const double *M,
              const double *s_re, const double *s_im, double rtol, int maxit, double *e_re, double *e_im,
              double *stats) {
  Solver s;
  s.m = m;
  s.C.n = s.C.m = n;
  s.C.rp.assign(rp, rp + n + 1);
  s.C.ci.assign(ci, ci + rp[n]);
  s.C.v.assign(C, C + rp[n]);
  s.M = s.C;
  s.M.v.assign(M, M + rp[n]);
  s.B = s.C;  // create_pc (em_la.cc:122-128): B = C + M
  for (size_t k = 0; k < s.B.v.size(); ++k) s.B.v[k] += M[k];
  double t0 = wall();
  ams_setup(s.ams, m, s.B);
  double t1 = wall();
  std::vector<double> b(2 * n), x(2 * n);
  std::copy(s_re, s_re + n, b.begin());
  std::copy(s_im, s_im + n, b.begin() + n);
  double tr;
  int its = fgmres(s, b.data(), x.data(), rtol, maxit, 30, &tr);
  std::copy(x.begin(), x.begin() + n, e_re);
  std::copy(x.begin() + n, x.end(), e_im);
  if (stats) {
    stats[0] = tr;
    stats[1] = (double)s.inner_its;
    stats[2] = t1 - t0;       // AMS setup seconds
    stats[3] = wall() - t1;   // FGMRES seconds
  }
  return its;
}

// estimate_error (em_fwd.cc:1102-1166) before the Allreduce: per-solution
// per-tet indicators eta[s][t] (volume + face terms).
void orc_estimate(const OrcMesh *m, const OrcModel *md, double freq, int nsol, const double *const *sre,
                  const double *const *sim, double *eta) {
  double omega = 2 * PI * freq;
  size_t T = m->nt;
  std::vector<double> fe((size_t)nsol * T * 4, -1.0);
  for (int s = 0; s < nsol; ++s) std::fill(eta + s * T, eta + (s + 1) * T, 0.0);
  for (int t = 0; t < m->nt; ++t) {
    Tet cell{m, t};
    // integrate_over_cell em_fwd.cc:1005-1043
    {
      double sig[9];
      cell_sigma(md, cell.attribute(), sig);
      V3 q[4];
      double jxw[4];
      cell_quadrature(cell, q, jxw);
      FEV fv;
      fv.reinit(cell);
      double diam = cell.diameter();
      for (int s = 0; s < nsol; ++s) {
        double res = 0;
        for (int k = 0; k < 4; ++k) {
          cplx e[3], se[3];
          fn_value(fv, q[k], sre[s], sim[s], e);
          zsig(sig, e, se);
          double sq = 0;
          for (int c = 0; c < 3; ++c) sq += std::norm(II * omega * se[c]);
          res += sq * jxw[k];
        }
        eta[s * T + t] += res * diam * diam;
      }
    }
    for (int f = 0; f < 4; ++f) {
      if (cell.neighbor(f) < 0)
        for (int s = 0; s < nsol; ++s) fe[(s * T + t) * 4 + f] = 0.0;
      if (fe[(0 * T + t) * 4 + f] >= 0.0) continue;
      // integrate_over_face em_fwd.cc:1045-1100
      int n = cell.neighbor(f), non = cell.neighbor_of_neighbor(f);
      Tet cn{m, n};
      double sig[9], sign[9];
      cell_sigma(md, cell.attribute(), sig);
      cell_sigma(md, cn.attribute(), sign);
      FEV fv, fvn;
      fv.reinit(cell);
      fvn.reinit(cn);
      V3 fnrm = fv.face_normal(f);
      V3 q[3];
      double jxw[3];
      face_quadrature(cell, f, q, jxw);
      double fd = cell.face_diameter(f);
      for (int s = 0; s < nsol; ++s) {
        double dotj = 0, crossh = 0;
        for (int k = 0; k < 3; ++k) {
          cplx e[3], en[3], se[3], sen[3];
          fn_value(fv, q[k], sre[s], sim[s], e);
          fn_value(fvn, q[k], sre[s], sim[s], en);
          zsig(sig, e, se);
          zsig(sign, en, sen);
          cplx j = (se[0] - sen[0]) * fnrm[0] + (se[1] - sen[1]) * fnrm[1] + (se[2] - sen[2]) * fnrm[2];
          dotj += std::norm(j) * jxw[k];
          cplx ce[3], cen[3];
          fn_curl(fv, sre[s], sim[s], ce);
          fn_curl(fvn, sre[s], sim[s], cen);
          cplx d[3] = {ce[0] - cen[0], ce[1] - cen[1], ce[2] - cen[2]};
          cplx x0 = d[1] * fnrm[2] - d[2] * fnrm[1];
          cplx x1 = d[2] * fnrm[0] - d[0] * fnrm[2];
          cplx x2 = d[0] * fnrm[1] - d[1] * fnrm[0];
          crossh += (std::norm(x0) + std::norm(x1) + std::norm(x2)) * jxw[k];
        }
        double v = (dotj + crossh) * fd / 2.0;
        fe[(s * T + t) * 4 + f] = v;
        fe[(s * T + n) * 4 + non] = v;
      }
    }
    for (int s = 0; s < nsol; ++s)
      for (int f = 0; f < 4; ++f) eta[s * T + t] += fe[(s * T + t) * 4 + f];
  }
}


// Eigen::VectorXd::sum() (the total of refine_fixed_fraction,
// src/em_fwd.cc:1192) in the order Eigen evaluates it when the reference is
// built for x86-64 without -march flags, where Eigen vectorises with SSE2
// packets of two doubles: two packet accumulators advance over pairs of
// packets, then they are added, a leftover whole packet is added, the two
// lanes are summed, and an odd last element comes last.  The threshold, and
// so the flag set, can move by one ulp of the total with another order.
static double orc_eigen_sse2_sum(const double *x, int n) {
  if (n < 2) return n == 1 ? x[0] : 0.0;
  const int n1 = n / 2 * 2;  // elements in whole packets
  const int n2 = n / 4 * 4;  // elements in whole packet pairs
  double a0 = x[0], a1 = x[1];
  if (n1 > 2) {
    double b0 = x[2], b1 = x[3];
    for (int i = 4; i < n2; i += 4) {
      a0 += x[i];
      a1 += x[i + 1];
      b0 += x[i + 2];
      b1 += x[i + 3];
    }
    a0 += b0;
    a1 += b1;
    if (n1 > n2) {
      a0 += x[n2];
      a1 += x[n2 + 1];
    }
  }
  double r = a0 + a1;
  for (int i = n1; i < n; ++i) r += x[i];
  return r;
}

// refine_fixed_fraction (em_fwd.cc:1182-1215)
void orc_refine_fixed_fraction(int n, const double *err, double fraction, unsigned char *flag) {
  const double total = orc_eigen_sse2_sum(err, n);
  std::vector<double> s(err, err + n);
  std::sort(s.begin(), s.end(), std::greater<double>());
  double sum = 0, thr = 0;
  for (int i = 0; i < n; ++i) {
    if (sum < fraction * total) sum += s[i];
    else { thr = s[i]; break; }
  }
  for (int i = 0; i < n; ++i)
    if (err[i] > thr) flag[i] = 1;
}

// refine_fixed_number (em_fwd.cc:1217-1240)
void orc_refine_fixed_number(int n, const double *err, double fraction, unsigned char *flag) {
  int k = (int)(n * fraction);
  std::vector<double> s(err, err + n);
  std::nth_element(s.begin(), s.begin() + k, s.end(), std::greater<double>());
  double thr = s[k];
  for (int i = 0; i < n; ++i)
    if (err[i] > thr) flag[i] = 1;
}

// interpolate_fields (em_fwd.cc:719-744): E and H at point p inside tet t.
void orc_interpolate_fields(const OrcMesh *m, int t, const double *p, double freq, const double *re,
                            const double *im, double *eh /* 6 complex: E then H */) {
  Tet cell{m, t};
  FEV fv;
  fv.reinit(cell);
  V3 pp = mk(p[0], p[1], p[2]);
  cplx es[3] = {0.0, 0.0, 0.0}, hs[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < 6; ++i) {
    int id = cell.edge_index(i);
    cplx v(re[id], im[id]);
    V3 b = fv.value_nedelec(i, pp), c = fv.curl_nedelec(i);
    for (int k = 0; k < 3; ++k) {
      es[k] += v * b[k];
      hs[k] += -1.0 / (II * 2.0 * PI * freq * MU) * v * c[k];
    }
  }
  for (int k = 0; k < 3; ++k) {
    eh[2 * k] = es[k].real();
    eh[2 * k + 1] = es[k].imag();
    eh[6 + 2 * k] = hs[k].real();
    eh[6 + 2 * k + 1] = hs[k].imag();
  }
}

// calculate_response_mt (em_fwd.cc:747-800): tensor impedance and tipper
// entries from the fields of the two polarisations at one receiver.
// f: e_xy[3], h_xy[3], e_yx[3], h_yx[3] (complex, interleaved).  Types as
// the reference's ObsType (em_defs.h:50-73); 212/222 (apparent resistivity
// and phase, declared but refused by the reference) are derived from the
// Z_XY / Z_YX entries as the reference's AP pair (em_io.cc:248-262): log of
// rho_a = |Z|^2 / (w mu) and the phase of conj(Z) in radians.  Returns 0,
// or -1 for a type the path does not compute.
int orc_response_mt(double freq, const double *f, int otype, double *out) {
  cplx e_xy[3], h_xy[3], e_yx[3], h_yx[3];
  for (int k = 0; k < 3; ++k) {
    e_xy[k] = cplx(f[2 * k], f[2 * k + 1]);
    h_xy[k] = cplx(f[6 + 2 * k], f[6 + 2 * k + 1]);
    e_yx[k] = cplx(f[12 + 2 * k], f[12 + 2 * k + 1]);
    h_yx[k] = cplx(f[18 + 2 * k], f[18 + 2 * k + 1]);
  }
  const cplx det = h_xy[0] * h_yx[1] - h_yx[0] * h_xy[1];
  cplx r;
  switch (otype) {
  case 311: r = (e_xy[0] * h_yx[1] - e_yx[0] * h_xy[1]) / det; break;
  case 321: r = (e_yx[0] * h_xy[0] - e_xy[0] * h_yx[0]) / det; break;
  case 331: r = (e_xy[1] * h_yx[1] - e_yx[1] * h_xy[1]) / det; break;
  case 341: r = (e_yx[1] * h_xy[0] - e_xy[1] * h_yx[0]) / det; break;
  case 351: r = (h_xy[2] * h_yx[1] - h_yx[2] * h_xy[1]) / det; break;
  case 361: r = (h_yx[2] * h_xy[0] - h_xy[2] * h_yx[0]) / det; break;
  case 212:
  case 222: {
    const cplx z = otype == 212 ? (e_yx[0] * h_xy[0] - e_xy[0] * h_yx[0]) / det
                                : (e_xy[1] * h_yx[1] - e_yx[1] * h_xy[1]) / det;
    const double w = 2.0 * PI * freq;
    r = cplx(std::log(std::norm(z) / (w * MU)), std::atan2(-z.imag(), z.real()));
    break;
  }
  default: return -1;
  }
  out[0] = r.real();
  out[1] = r.imag();
  return 0;
}

// calculate_response_csem (em_fwd.cc:802-871): field components (RI) or
// their complex logarithms (AP).  f: e[3], h[3] (complex, interleaved).
int orc_response_csem(const double *f, int otype, double *out) {
  const int comp = otype / 10 % 10;  // 1..6: Ex, Ey, Ez, Hx, Hy, Hz
  const int kind = otype % 10;       // 1: RI, 2: AP
  if (otype / 100 != 1 || comp < 1 || comp > 6 || (kind != 1 && kind != 2)) return -1;
  cplx v(f[2 * (comp - 1)], f[2 * (comp - 1) + 1]);
  if (kind == 2) v = std::log(v);
  out[0] = v.real();
  out[1] = v.imag();
  return 0;
}

}  // extern "C"
