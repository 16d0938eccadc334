// Element-matrix generation and scatter into the precomputed CSR pattern.
//
// Replaces the tet loop of assemble_matrix (src/em_fwd.cc:343-392): one
// thread computes the closed-form Whitney element matrices of one tet (the
// 4-point rule of em_fe.cc:82-128 is exact for these integrands, so the
// closed form equals the reference up to rounding), stages them in shared
// memory, and the warp then scatters its 32 tets' 36+36 entries with
// coalesced reads of the tet->slot map and FP64 atomic adds.
//
// C is omega-independent and the mass part is stored without omega (Ms);
// the reference's M is omega * Ms (src/em_fwd.cc:336,365).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>

#include "emg_internal.h"
#include "emg_kernels.cuh"

namespace emg {

// get_cell_attribute (src/em_fwd.cc:14-72) once per attribute.
void sigma_table(int aniso_form, int nrho, int ncol, const double *rho, std::vector<double> &out) {
  out.assign((size_t)nrho * 9, 0.0);
  for (int i = 0; i < nrho; ++i) {
    const double *r = rho + (size_t)i * ncol;
    double *s = &out[(size_t)i * 9];
    switch (aniso_form) {
    case EMG_ISOTROPIC: s[0] = s[4] = s[8] = 1.0 / r[0]; break;
    case EMG_VERTICAL: s[0] = s[4] = 1.0 / r[0]; s[8] = 1.0 / r[1]; break;
    case EMG_TRIAXIAL: s[0] = 1.0 / r[0]; s[4] = 1.0 / r[1]; s[8] = 1.0 / r[2]; break;
    case EMG_ARBITRARY: {
      // sigma = Rz Ry Rx diag(1/rho) Rx^T Ry^T Rz^T, angles in degrees
      double cx = std::cos(r[3] * DTOR), sx = std::sin(r[3] * DTOR);
      double cy = std::cos(r[4] * DTOR), sy = std::sin(r[4] * DTOR);
      double cz = std::cos(r[5] * DTOR), sz = std::sin(r[5] * DTOR);
      double X[9] = {1, 0, 0, 0, cx, sx, 0, -sx, cx};
      double Y[9] = {cy, 0, -sy, 0, 1, 0, sy, 0, cy};
      double Z[9] = {cz, sz, 0, -sz, cz, 0, 0, 0, 1};
      double ZY[9], R[9];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double v = 0;
          for (int k = 0; k < 3; ++k) v += Z[a * 3 + k] * Y[k * 3 + b];
          ZY[a * 3 + b] = v;
        }
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double v = 0;
          for (int k = 0; k < 3; ++k) v += ZY[a * 3 + k] * X[k * 3 + b];
          R[a * 3 + b] = v;
        }
      double d[3] = {1.0 / r[0], 1.0 / r[1], 1.0 / r[2]};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double v = 0;
          for (int k = 0; k < 3; ++k) v += R[a * 3 + k] * d[k] * R[b * 3 + k];
          s[a * 3 + b] = v;
        }
      break;
    }
    default: fail(EMG_ERR_USER, "Unsupported anisotropy form %d.", aniso_form);
    }
  }
}

// ---------------------------------------------------------------------------
// host: CSR pattern = make_sparsity_patterns (src/em_fwd.cc:191-246)
// row e: sorted unique edges sharing a tet with e (diagonal included)
// ---------------------------------------------------------------------------
void build_sparsity(Context &c) {
  const int ne = c.ne, nt = c.nt;
  std::vector<int> e2t_rp(ne + 1, 0), e2t;
  for (int t = 0; t < nt; ++t)
    for (int i = 0; i < 6; ++i) e2t_rp[c.h_t2e[6 * (size_t)t + i] + 1]++;
  for (int e = 0; e < ne; ++e) e2t_rp[e + 1] += e2t_rp[e];
  e2t.resize(e2t_rp[ne]);
  {
    std::vector<int> pos(e2t_rp.begin(), e2t_rp.end() - 1);
    for (int t = 0; t < nt; ++t)
      for (int i = 0; i < 6; ++i) e2t[pos[c.h_t2e[6 * (size_t)t + i]]++] = t;
  }
  std::vector<int> cnt(ne + 1, 0);
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 4096)
    for (int e = 0; e < ne; ++e) {
      buf.clear();
      for (int k = e2t_rp[e]; k < e2t_rp[e + 1]; ++k)
        for (int i = 0; i < 6; ++i) buf.push_back(c.h_t2e[6 * (size_t)e2t[k] + i]);
      std::sort(buf.begin(), buf.end());
      cnt[e + 1] = (int)(std::unique(buf.begin(), buf.end()) - buf.begin());
    }
  }
  c.h_rp.assign(ne + 1, 0);
  for (int e = 0; e < ne; ++e) c.h_rp[e + 1] = c.h_rp[e] + cnt[e + 1];
  c.nnz = c.h_rp[ne];
  c.h_ci.resize(c.nnz);
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 4096)
    for (int e = 0; e < ne; ++e) {
      buf.clear();
      for (int k = e2t_rp[e]; k < e2t_rp[e + 1]; ++k)
        for (int i = 0; i < 6; ++i) buf.push_back(c.h_t2e[6 * (size_t)e2t[k] + i]);
      std::sort(buf.begin(), buf.end());
      int u = (int)(std::unique(buf.begin(), buf.end()) - buf.begin());
      std::copy(buf.begin(), buf.begin() + u, c.h_ci.begin() + c.h_rp[e]);
    }
  }
  c.rp.upload(c.h_rp, c.stream);
  c.ci.upload(c.h_ci, c.stream);
}

// vertex adjacency (pattern of G^T B G and Pi^T B Pi) and vertex->edge incidence
void build_vertex_pattern(Context &c) {
  const int nv = c.nv, ne = c.ne;
  std::vector<int> deg(nv + 1, 0);
  for (int e = 0; e < ne; ++e) {
    deg[c.h_edges[2 * e] + 1]++;
    deg[c.h_edges[2 * e + 1] + 1]++;
  }
  std::vector<int> inc_rp(nv + 1, 0);
  for (int v = 0; v < nv; ++v) inc_rp[v + 1] = inc_rp[v] + deg[v + 1];
  std::vector<int> inc(inc_rp[nv]);
  {
    std::vector<int> pos(inc_rp.begin(), inc_rp.end() - 1);
    for (int e = 0; e < ne; ++e) {
      inc[pos[c.h_edges[2 * e]]++] = 2 * e + 0;
      inc[pos[c.h_edges[2 * e + 1]]++] = 2 * e + 1;
    }
  }
  c.h_vrp.assign(nv + 1, 0);
  for (int v = 0; v < nv; ++v) c.h_vrp[v + 1] = c.h_vrp[v] + 1 + (inc_rp[v + 1] - inc_rp[v]);
  c.h_vci.resize(c.h_vrp[nv]);
#pragma omp parallel for schedule(static)
  for (int v = 0; v < nv; ++v) {
    int *out = &c.h_vci[c.h_vrp[v]];
    int k = 0;
    out[k++] = v;
    for (int j = inc_rp[v]; j < inc_rp[v + 1]; ++j) {
      int e = inc[j] >> 1, ep = inc[j] & 1;
      out[k++] = c.h_edges[2 * e + (1 - ep)];
    }
    std::sort(out, out + k);
  }
  c.vrp.upload(c.h_vrp, c.stream);
  c.vci.upload(c.h_vci, c.stream);
  c.vinc_rp.upload(inc_rp, c.stream);
  c.vinc.upload(inc, c.stream);
}

// ---------------------------------------------------------------------------
// device kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ int find_col(const int *__restrict__ ci, int b, int e, int col) {
  // rows are short (<= ~40): binary search
  int lo = b, hi = e - 1;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(ci + mid) < col) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// slot[t*36 + k*6 + l] = CSR slot of (cedge[t][k], cedge[t][l])
__global__ void slot_map_kernel(int nt, const int *__restrict__ cedge, const int *__restrict__ rp,
                                const int *__restrict__ ci, int *__restrict__ slot) {
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)nt * 36) return;
  int t = (int)(idx / 36), ent = (int)(idx % 36);
  int row = __ldg(cedge + 6 * (long)t + ent / 6), col = __ldg(cedge + 6 * (long)t + ent % 6);
  slot[idx] = find_col(ci, __ldg(rp + row), __ldg(rp + row + 1), col);
}

// vslot[t*16 + p*4 + q] = slot of (ctet[t][p], ctet[t][q]) in the vertex pattern
__global__ void vslot_map_kernel(int nt, const int *__restrict__ tets, const int *__restrict__ rp,
                                 const int *__restrict__ ci, int *__restrict__ slot) {
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)nt * 16) return;
  int t = (int)(idx / 16), ent = (int)(idx % 16);
  int row = __ldg(tets + 4 * (long)t + ent / 4), col = __ldg(tets + 4 * (long)t + ent % 4);
  slot[idx] = find_col(ci, __ldg(rp + row), __ldg(rp + row + 1), col);
}

void build_slot_maps(Context &c) {
  c.slot.alloc((size_t)c.nt * 36);
  long n36 = (long)c.nt * 36;
  slot_map_kernel<<<(unsigned)((n36 + 255) / 256), 256, 0, c.stream>>>(c.nt, c.cedge.p, c.rp.p, c.ci.p, c.slot.p);
  EMG_LAUNCH_CHECK();
  c.vslot.alloc((size_t)c.nt * 16);
  long n16 = (long)c.nt * 16;
  vslot_map_kernel<<<(unsigned)((n16 + 255) / 256), 256, 0, c.stream>>>(c.nt, c.ctet.p, c.vrp.p, c.vci.p, c.vslot.p);
  EMG_LAUNCH_CHECK();
}

// canonical tets: sorted vertex ids, canonical global edges, sort parity
__global__ void canonicalize_kernel(int nt, const int *__restrict__ tets, const int *__restrict__ t2e,
                                    const int *__restrict__ edges, int *__restrict__ ctet,
                                    int *__restrict__ cedge, signed char *__restrict__ cpar,
                                    int *__restrict__ bad) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  int v[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = __ldg(tets + 4 * (long)t + i);
  int par = 1;
  // sorting network on 4 keys, counting swaps for the parity
#define EMG_CSWAP(a, b) if (v[a] > v[b]) { int tmp_ = v[a]; v[a] = v[b]; v[b] = tmp_; par = -par; }
  EMG_CSWAP(0, 1) EMG_CSWAP(2, 3) EMG_CSWAP(0, 2) EMG_CSWAP(1, 3) EMG_CSWAP(1, 2)
#undef EMG_CSWAP
#pragma unroll
  for (int i = 0; i < 4; ++i) ctet[4 * (long)t + i] = v[i];
  cpar[t] = (signed char)par;
  int le[6], la[6], lb[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    le[i] = __ldg(t2e + 6 * (long)t + i);
    la[i] = __ldg(edges + 2 * (long)le[i]);
    lb[i] = __ldg(edges + 2 * (long)le[i] + 1);
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    int a = v[kEdgeP(k)], b = v[kEdgeQ(k)];
    int ge = -1;
#pragma unroll
    for (int i = 0; i < 6; ++i)
      if (la[i] == a && lb[i] == b) ge = le[i];
    if (ge < 0) atomicExch(bad, t + 1);
    cedge[6 * (long)t + k] = ge < 0 ? 0 : ge;
  }
}

void canonicalize(Context &c) {
  c.ctet.alloc((size_t)c.nt * 4);
  c.cedge.alloc((size_t)c.nt * 6);
  c.cpar.alloc((size_t)c.nt);
  DBuf<int> bad(1);
  bad.zero(c.stream);
  canonicalize_kernel<<<(unsigned)((c.nt + 255) / 256), 256, 0, c.stream>>>(c.nt, c.tets.p, c.t2e.p, c.edges.p,
                                                                            c.ctet.p, c.cedge.p, c.cpar.p, bad.p);
  EMG_LAUNCH_CHECK();
  int hb = 0;
  bad.download(&hb, 1, c.stream);
  EMG_CUDA(cudaStreamSynchronize(c.stream));
  if (hb) fail(EMG_ERR_USER, "tet %d: tet2edgelist does not match tetrahedronlist/edgelist", hb - 1);
}

struct ElemIn {
  const double *pts;
  const int *ctet, *cedge, *attr;
  const signed char *cpar;
  const unsigned char *ebdr;
  const double *sig;
};

// Element matrices of tet t in canonical order: c (curl-curl / mu) and ms
// (mass without omega), boundary rows/columns zeroed as
// src/em_fwd.cc:377-388.  Returns whether the tet touches a boundary edge.
//   c_kl  = V/mu curl(phi_k).curl(phi_l),  curl(phi_k) = 2 grad l_p x grad l_q
//   ms_kl = V/20 [(1+d_pr) S_qs - (1+d_ps) S_qr - (1+d_qr) S_ps + (1+d_qs) S_pr]
// for k=(p,q), l=(r,s), S_ab = grad l_a . sigma grad l_b (int l_a l_b = V(1+d_ab)/20).
__device__ __forceinline__ bool element_matrices(const ElemIn &in, int t, double c[36], double ms[36],
                                                 TetGeom &g) {
  load_tet_geom(in.pts, in.ctet, in.cedge, in.cpar, t, g);
  const double *sg = in.sig + 9 * (long)__ldg(in.attr + t);
  double s[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) s[k] = __ldg(sg + k);
  double S[10];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = p; q < 4; ++q) {
      double sq0 = s[0] * g.gr[q][0] + s[1] * g.gr[q][1] + s[2] * g.gr[q][2];
      double sq1 = s[3] * g.gr[q][0] + s[4] * g.gr[q][1] + s[5] * g.gr[q][2];
      double sq2 = s[6] * g.gr[q][0] + s[7] * g.gr[q][1] + s[8] * g.gr[q][2];
      S[sym_idx(p, q)] = g.gr[p][0] * sq0 + g.gr[p][1] * sq1 + g.gr[p][2] * sq2;
    }
  double cu[6][3];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int a = kEdgeP(k), b = kEdgeQ(k);
    cu[k][0] = 2.0 * (g.gr[a][1] * g.gr[b][2] - g.gr[a][2] * g.gr[b][1]);
    cu[k][1] = 2.0 * (g.gr[a][2] * g.gr[b][0] - g.gr[a][0] * g.gr[b][2]);
    cu[k][2] = 2.0 * (g.gr[a][0] * g.gr[b][1] - g.gr[a][1] * g.gr[b][0]);
  }
  const double vc = g.vol / MU, vm = g.vol / 20.0;
  bool bd[6];
  bool any = false;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    bd[k] = __ldg(in.ebdr + g.ge[k]) != 0;
    any |= bd[k];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
#pragma unroll
    for (int l = 0; l <= k; ++l) {
      const int p = kEdgeP(k), q = kEdgeQ(k), r = kEdgeP(l), u = kEdgeQ(l);
      double ckl = vc * (cu[k][0] * cu[l][0] + cu[k][1] * cu[l][1] + cu[k][2] * cu[l][2]);
      double mkl = vm * ((1.0 + (p == r)) * S[sym_idx(q, u)] - (1.0 + (p == u)) * S[sym_idx(q, r)] -
                         (1.0 + (q == r)) * S[sym_idx(p, u)] + (1.0 + (q == u)) * S[sym_idx(p, r)]);
      if (bd[k] || bd[l]) {
        if (k != l) ckl = 0.0;
        mkl = 0.0;
      }
      c[k * 6 + l] = ckl;
      c[l * 6 + k] = ckl;
      ms[k * 6 + l] = mkl;
      ms[l * 6 + k] = mkl;
    }
  }
  return any;
}

constexpr int ASM_THREADS = 64;

__global__ void __launch_bounds__(ASM_THREADS) assemble_edge_kernel(ElemIn in, int nt, const int *__restrict__ slot,
                                                                  double *__restrict__ Cv, double *__restrict__ Mv,
                                                                  unsigned char *__restrict__ bdr_cell) {
  __shared__ double sc[ASM_THREADS * 36];
  __shared__ double sm[ASM_THREADS * 36];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t = blockIdx.x * ASM_THREADS + tid;
  if (t < nt) {
    double c[36], m[36];
    TetGeom g;
    bool bd = element_matrices(in, t, c, m, g);
    bdr_cell[t] = bd ? 1 : 0;
#pragma unroll
    for (int k = 0; k < 36; ++k) {
      sc[tid * 36 + k] = c[k];
      sm[tid * 36 + k] = m[k];
    }
  }
  __syncwarp();
  // warp-cooperative scatter over the (tet, entry) pairs of the warp's 32
  // tets: slot-map reads are coalesced, shared reads conflict-free
  const int t0 = blockIdx.x * ASM_THREADS + warp * 32;
  const int nvalid = min(32, nt - t0);
  const double *wc = sc + warp * 32 * 36;
  const double *wm = sm + warp * 32 * 36;
  const int *ws = slot + (long)t0 * 36;
#pragma unroll 4
  for (int r = 0; r < 36; ++r) {
    int p = r * 32 + lane;
    if (p < nvalid * 36) {
      int s = __ldg(ws + p);
      atomicAdd(Cv + s, wc[p]);
      atomicAdd(Mv + s, wm[p]);
    }
  }
}

ElemIn elem_in(Context &c) {
  return ElemIn{c.pts.p, c.ctet.p, c.cedge.p, c.attr.p, c.cpar.p, c.ebdr.p, c.sigma_tab.p};
}

void assemble_edge(Context &c) {
  c.Cv.alloc(c.nnz);
  c.Msv.alloc(c.nnz);
  c.bdr_cell.alloc(c.nt);
  c.Cv.zero(c.stream);
  c.Msv.zero(c.stream);
  unsigned blocks = (unsigned)((c.nt + ASM_THREADS - 1) / ASM_THREADS);
  assemble_edge_kernel<<<blocks, ASM_THREADS, 0, c.stream>>>(elem_in(c), c.nt, c.slot.p, c.Cv.p, c.Msv.p,
                                                              c.bdr_cell.p);
  EMG_LAUNCH_CHECK();
}

// Nodal subspace operators Q^T K Q for Q = G_e (gradient: -1 at the lower,
// +1 at the higher vertex, src/em_la.cc:254-270) and Pi_{x,y,z},e (0.5 t_e[d]
// at both endpoints, t_e = x(v1) - x(v0): the Nedelec interpolation AMS
// builds from G and the vertex coordinates), K = c and ms.  Summing element
// contributions equals G^T B G etc. of the assembled B because the boundary
// zeroing is element-local.
struct NodalOut {
  double *v[8];
};

__global__ void __launch_bounds__(128) assemble_nodal_kernel(ElemIn in, int nt, const int *__restrict__ vslot,
                                                              NodalOut out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double c[36], m[36];
  TetGeom g;
  const bool touches_bdr = element_matrices(in, t, c, m, g);
  int vs[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) vs[k] = __ldg(vslot + 16 * (long)t + k);
#pragma unroll
  for (int sp = 0; sp < 4; ++sp) {
    double Q[6][4];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const int a = kEdgeP(k), b = kEdgeQ(k);
#pragma unroll
      for (int p = 0; p < 4; ++p) Q[k][p] = 0.0;
      if (sp == 0) {
        Q[k][a] = -1.0;
        Q[k][b] = 1.0;
      } else {
        double w = 0.5 * (g.x[b][sp - 1] - g.x[a][sp - 1]);
        Q[k][a] = w;
        Q[k][b] = w;
      }
    }
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      // curl(grad) = 0: G_e^T c G_e vanishes exactly unless boundary zeroing
      // broke the element matrix; skipping it keeps rounding noise (~1e-16
      // |C|) out of the gradient space, where w sigma_air Ms is ~1e-10 |C|
      if (sp == 0 && part == 0 && !touches_bdr) continue;
      const double *K = part == 0 ? c : m;
      double KQ[6][4];
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          double v = 0;
#pragma unroll
          for (int j = 0; j < 6; ++j) v += K[i * 6 + j] * Q[j][q];
          KQ[i][q] = v;
        }
      double *o = out.v[sp * 2 + part];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          double v = 0;
#pragma unroll
          for (int i = 0; i < 6; ++i) v += Q[i][p] * KQ[i][q];
          atomicAdd(o + vs[p * 4 + q], v);
        }
    }
  }
}

void assemble_nodal_device(Context &c, DBuf<double> &buf) {
  long vnnz = c.h_vrp[c.nv];
  buf.alloc((size_t)vnnz * 8);
  buf.zero(c.stream);
  NodalOut o;
  for (int k = 0; k < 8; ++k) o.v[k] = buf.p + (size_t)k * vnnz;
  assemble_nodal_kernel<<<(unsigned)((c.nt + 127) / 128), 128, 0, c.stream>>>(elem_in(c), c.nt, c.vslot.p, o);
  EMG_LAUNCH_CHECK();
}

void assemble_nodal(Context &c, HCsr out[4]) {
  long vnnz = c.h_vrp[c.nv];
  DBuf<double> buf;
  assemble_nodal_device(c, buf);
  // each part straight into its operator (no staging copy of all eight)
  for (int sp = 0; sp < 4; ++sp) {
    out[sp].n = out[sp].m = c.nv;
    out[sp].rp = c.h_vrp;
    out[sp].ci = c.h_vci;
    out[sp].vc.resize(vnnz);
    out[sp].vm.resize(vnnz);
    buf.download_at(out[sp].vc.data(), (size_t)(2 * sp) * vnnz, vnnz, c.stream);
    buf.download_at(out[sp].vm.data(), (size_t)(2 * sp + 1) * vnnz, vnnz, c.stream);
  }
  EMG_CUDA(cudaStreamSynchronize(c.stream));
}

// The vector nodal space of AMS (hypre's Pi space, cycle character '2'):
// Pi = [Pi_x Pi_y Pi_z] interpolates a vertex vector field (3 values per
// vertex) onto the edges, and Pi^T K Pi couples the three components.  The
// nine 4x4 element blocks Q_d1^T K Q_d2 are summed into nine vertex-pattern
// arrays per value part; the host interleaves them as row 3 v + d1, column
// 3 u + d2.
struct PiOut {
  double *v[18];  // (d1 * 3 + d2) * 2 + part
};

__global__ void __launch_bounds__(128) assemble_pivec_kernel(ElemIn in, int nt, const int *__restrict__ vslot,
                                                              PiOut out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double c[36], m[36];
  TetGeom g;
  element_matrices(in, t, c, m, g);
  int vs[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) vs[k] = __ldg(vslot + 16 * (long)t + k);
  // w[k][d]: Pi_d weight of edge k at both of its endpoints
  double w[6][3];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int a = kEdgeP(k), b = kEdgeQ(k);
#pragma unroll
    for (int d = 0; d < 3; ++d) w[k][d] = 0.5 * (g.x[b][d] - g.x[a][d]);
  }
#pragma unroll
  for (int part = 0; part < 2; ++part) {
    const double *K = part == 0 ? c : m;
#pragma unroll 1
    for (int d2 = 0; d2 < 3; ++d2) {
      // KQ = K Q_d2 (6 x 4)
      double KQ[6][4];
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) KQ[i][q] = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const int a = kEdgeP(j), b = kEdgeQ(j);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          const double v = K[i * 6 + j] * w[j][d2];
          KQ[i][a] += v;
          KQ[i][b] += v;
        }
      }
#pragma unroll 1
      for (int d1 = 0; d1 < 3; ++d1) {
        double B[4][4];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) B[p][q] = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          const int a = kEdgeP(i), b = kEdgeQ(i);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const double v = w[i][d1] * KQ[i][q];
            B[a][q] += v;
            B[b][q] += v;
          }
        }
        double *o = out.v[(d1 * 3 + d2) * 2 + part];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) atomicAdd(o + vs[p * 4 + q], B[p][q]);
      }
    }
  }
}

void assemble_pi_vector(Context &c, HCsr &out, bool coupled) {
  const long vnnz = c.h_vrp[c.nv];
  DBuf<double> buf((size_t)vnnz * 18);
  buf.zero(c.stream);
  PiOut o;
  for (int k = 0; k < 18; ++k) o.v[k] = buf.p + (size_t)k * vnnz;
  assemble_pivec_kernel<<<(unsigned)((c.nt + 127) / 128), 128, 0, c.stream>>>(elem_in(c), c.nt, c.vslot.p, o);
  EMG_LAUNCH_CHECK();
  std::vector<double> h((size_t)vnnz * 18);
  buf.download(h.data(), h.size(), c.stream);
  EMG_CUDA(cudaStreamSynchronize(c.stream));
  const int nv = c.nv;
  out.n = out.m = 3 * nv;
  out.rp.assign(3 * (size_t)nv + 1, 0);
  const int nb = coupled ? 3 : 1;  // column blocks per row: all three components, or its own
  for (int v = 0; v < nv; ++v)
    for (int d = 0; d < 3; ++d) out.rp[3 * v + d + 1] = nb * (c.h_vrp[v + 1] - c.h_vrp[v]);
  for (int i = 0; i < 3 * nv; ++i) out.rp[i + 1] += out.rp[i];
  out.ci.resize(out.rp[3 * nv]);
  out.vc.resize(out.rp[3 * nv]);
  out.vm.resize(out.rp[3 * nv]);
#pragma omp parallel for schedule(static)
  for (int v = 0; v < nv; ++v)
    for (int d1 = 0; d1 < 3; ++d1) {
      long p = out.rp[3 * v + d1];
      for (int k = c.h_vrp[v]; k < c.h_vrp[v + 1]; ++k)
        for (int d2 = 0; d2 < 3; ++d2) {
          if (!coupled && d2 != d1) continue;
          out.ci[p] = 3 * c.h_vci[k] + d2;
          out.vc[p] = h[(size_t)((d1 * 3 + d2) * 2) * vnnz + k];
          out.vm[p] = h[(size_t)((d1 * 3 + d2) * 2 + 1) * vnnz + k];
          ++p;
        }
    }
}

// ---------------------------------------------------------------------------
// G^T B as a vertex x edge operator.  The gradient-space residual of AMS,
// G^T (b - B x), is formed as G^T b - (G^T B) x: G^T C vanishes exactly on
// every element without a boundary edge (curl grad = 0), so the product keeps
// no trace of the curl-curl scale that swamps w sigma Ms in the air when
// B x is evaluated in FP32.
// ---------------------------------------------------------------------------
void build_gtb_pattern(Context &c) {
  c.tiles.clear();
  const int nv = c.nv, nt = c.nt;
  std::vector<int> v2t_rp(nv + 1, 0), v2t;
  for (int t = 0; t < nt; ++t)
    for (int i = 0; i < 4; ++i) v2t_rp[c.h_tets[4 * (size_t)t + i] + 1]++;
  for (int v = 0; v < nv; ++v) v2t_rp[v + 1] += v2t_rp[v];
  v2t.resize(v2t_rp[nv]);
  {
    std::vector<int> pos(v2t_rp.begin(), v2t_rp.end() - 1);
    for (int t = 0; t < nt; ++t)
      for (int i = 0; i < 4; ++i) v2t[pos[c.h_tets[4 * (size_t)t + i]]++] = t;
  }
  std::vector<int> cnt(nv + 1, 0);
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 4096)
    for (int v = 0; v < nv; ++v) {
      buf.clear();
      for (int k = v2t_rp[v]; k < v2t_rp[v + 1]; ++k)
        for (int i = 0; i < 6; ++i) buf.push_back(c.h_t2e[6 * (size_t)v2t[k] + i]);
      std::sort(buf.begin(), buf.end());
      cnt[v + 1] = (int)(std::unique(buf.begin(), buf.end()) - buf.begin());
    }
  }
  c.h_grp.assign(nv + 1, 0);
  for (int v = 0; v < nv; ++v) c.h_grp[v + 1] = c.h_grp[v] + cnt[v + 1];
  c.h_gci.resize(c.h_grp[nv]);
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 4096)
    for (int v = 0; v < nv; ++v) {
      buf.clear();
      for (int k = v2t_rp[v]; k < v2t_rp[v + 1]; ++k)
        for (int i = 0; i < 6; ++i) buf.push_back(c.h_t2e[6 * (size_t)v2t[k] + i]);
      std::sort(buf.begin(), buf.end());
      int u = (int)(std::unique(buf.begin(), buf.end()) - buf.begin());
      std::copy(buf.begin(), buf.begin() + u, c.h_gci.begin() + c.h_grp[v]);
    }
  }
  c.grp.upload(c.h_grp, c.stream);
  c.gci.upload(c.h_gci, c.stream);
}

// gslot[t*24 + p*6 + k] = slot of (ctet[t][p], cedge[t][k]) in the G^T B pattern
__global__ void gslot_map_kernel(int nt, const int *__restrict__ ctet, const int *__restrict__ cedge,
                                 const int *__restrict__ rp, const int *__restrict__ ci, int *__restrict__ slot) {
  long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)nt * 24) return;
  int t = (int)(idx / 24), ent = (int)(idx % 24);
  int row = __ldg(ctet + 4 * (long)t + ent / 6), col = __ldg(cedge + 6 * (long)t + ent % 6);
  slot[idx] = find_col(ci, __ldg(rp + row), __ldg(rp + row + 1), col);
}

__global__ void __launch_bounds__(128) assemble_gtb_kernel(ElemIn in, int nt, const int *__restrict__ gslot,
                                                            double *__restrict__ gc, double *__restrict__ gm) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double c[36], m[36];
  TetGeom g;
  const bool touches_bdr = element_matrices(in, t, c, m, g);
  // (G_e^T K)[p][k] = sum over local edges j=(a,b): (-1 if p==a, +1 if p==b) K[j][k]
#pragma unroll
  for (int p = 0; p < 4; ++p) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      double vm = 0, vc = 0;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const double sgn = (kEdgeP(j) == p) ? -1.0 : ((kEdgeQ(j) == p) ? 1.0 : 0.0);
        if (sgn != 0.0) {
          vm += sgn * m[j * 6 + k];
          vc += sgn * c[j * 6 + k];
        }
      }
      const int sl = __ldg(gslot + 24 * (long)t + p * 6 + k);
      atomicAdd(gm + sl, vm);
      if (touches_bdr) atomicAdd(gc + sl, vc);
    }
  }
}

void assemble_gtb(Context &c, DBuf<double> &gc, DBuf<double> &gm) {
  if (c.h_grp.empty()) build_gtb_pattern(c);
  if (!c.gslot.p) {
    c.gslot.alloc((size_t)c.nt * 24);
    long n24 = (long)c.nt * 24;
    gslot_map_kernel<<<(unsigned)((n24 + 255) / 256), 256, 0, c.stream>>>(c.nt, c.ctet.p, c.cedge.p, c.grp.p, c.gci.p,
                                                                          c.gslot.p);
    EMG_LAUNCH_CHECK();
  }
  long nnz = c.h_grp[c.nv];
  gc.alloc(nnz);
  gm.alloc(nnz);
  gc.zero(c.stream);
  gm.zero(c.stream);
  assemble_gtb_kernel<<<(unsigned)((c.nt + 127) / 128), 128, 0, c.stream>>>(elem_in(c), c.nt, c.gslot.p, gc.p, gm.p);
  EMG_LAUNCH_CHECK();
}

}  // namespace emg
