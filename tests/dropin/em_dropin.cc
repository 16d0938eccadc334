/*
 * Replacement bodies of the reference's hot-path functions over the
 * emfem_b200 C ABI: what a maintainer puts into src/em_la.cc and
 * src/em_fwd.cc (the signatures are the reference's, src/em_la.h:8-20 and
 * src/em_fwd.h:10-51).  Compiled here against the PETSc stand-in of this
 * folder; with PETSc the same code compiles against <petsc.h>.  Every emg_*
 * failure becomes SETERRQ(..., EM_ERR_USER, emg_last_error()).
 */
#include "em_dropin.h"

#include <algorithm>
#include <cmath>
#include <vector>

#define EMG_CALL(ctx, x)                                                       \
  do {                                                                         \
    int rc__ = (x);                                                            \
    if (rc__ != EMG_OK) SETERRQ((ctx)->world_comm, EM_ERR_USER, "%s", emg_last_error()); \
  } while (0)

static int slot_of(EMContext *ctx, const PETScBlockVector &e) {
  if (&e == &ctx->dual_e) return EMG_SOL_DUAL;
  if (&e == &ctx->csem_e) return EMG_SOL_CSEM;
  return &e == &ctx->mt_e[XY_POLAR] ? EMG_SOL_MT_XY : EMG_SOL_MT_YX;
}

// create_linear_system (src/em_fwd.cc:248-295): pattern, operators and the
// named solution vectors live on the device; the host Vecs are views
PetscErrorCode create_linear_system(EMContext *ctx, int tidx) {
  PetscFunctionBegin;
  EMG_CALL(ctx, emg_create_linear_system(ctx->emg, tidx));
  PetscFunctionReturn(0);
}

PetscErrorCode destroy_linear_system(EMContext *ctx) {
  PetscFunctionBegin;
  EMG_CALL(ctx, emg_destroy_linear_system(ctx->emg));
  PetscFunctionReturn(0);
}

// assemble_matrix (src/em_fwd.cc:318-400)
PetscErrorCode assemble_matrix(EMContext *ctx, int fidx) {
  PetscFunctionBegin;
  EMG_CALL(ctx, emg_assemble_matrix(ctx->emg, fidx));
  PetscFunctionReturn(0);
}

// assemble_rhs_csem (src/em_fwd.cc:616-671): dipole cells from the
// reference's point location on the context's mesh, RHS into ctx->s
PetscErrorCode assemble_rhs_csem(EMContext *ctx, int fidx, int tidx) {
  PetscScalar *sr, *si;
  const double *t = &ctx->tx[7 * (size_t)tidx];
  std::vector<double> pts;
  if (t[6] <= 0.1 && t[6] >= -0.1) {
    pts.assign(t, t + 3);
  } else {
    // divide_line_source (src/em_fwd.cc:582-614) midpoints
    const double dtor = 3.14159265358979323846 / 180.0;
    const double d[3] = {std::cos(t[3] * dtor) * std::cos(t[4] * dtor), std::sin(t[3] * dtor) * std::cos(t[4] * dtor),
                         std::sin(t[4] * dtor)};
    const int nd = (int)ctx->n_tx_divisions;
    double a[3] = {t[0] - d[0] * t[6] / 2, t[1] - d[1] * t[6] / 2, t[2] - d[2] * t[6] / 2};
    for (int i = 0; i < nd; ++i) {
      double b[3] = {a[0] + d[0] * t[6] / nd, a[1] + d[1] * t[6] / nd, a[2] + d[2] * t[6] / nd};
      for (int q = 0; q < 3; ++q) pts.push_back((a[q] + b[q]) / 2);
      for (int q = 0; q < 3; ++q) a[q] = b[q];
    }
  }
  std::vector<int> cells(pts.size() / 3);
  PetscFunctionBegin;
  EMG_CALL(ctx, emg_find_cell_around_point(ctx->emg, (int)cells.size(), pts.data(), cells.data()));
  PetscCall(VecGetArray(ctx->s.re, &sr));
  PetscCall(VecGetArray(ctx->s.im, &si));
  int rc = emg_assemble_rhs_csem(ctx->emg, fidx, t, cells.data(), sr, si);
  PetscCall(VecRestoreArray(ctx->s.re, &sr));
  PetscCall(VecRestoreArray(ctx->s.im, &si));
  EMG_CALL(ctx, rc);
  PetscFunctionReturn(0);
}

// assemble_rhs_dual (src/em_fwd.cc:673-717)
PetscErrorCode assemble_rhs_dual(EMContext *ctx) {
  PetscScalar *sr, *si;
  const int nrx = (int)(ctx->rx.size() / 3);
  std::vector<int> cells(nrx);
  PetscFunctionBegin;
  EMG_CALL(ctx, emg_find_cell_around_point(ctx->emg, nrx, ctx->rx.data(), cells.data()));
  PetscCall(VecGetArray(ctx->s.re, &sr));
  PetscCall(VecGetArray(ctx->s.im, &si));
  int rc = emg_assemble_rhs_dual(ctx->emg, nrx, ctx->rx.data(), cells.data(), sr, si);
  PetscCall(VecRestoreArray(ctx->s.re, &sr));
  PetscCall(VecRestoreArray(ctx->s.im, &si));
  EMG_CALL(ctx, rc);
  PetscFunctionReturn(0);
}

// create_pc / destroy_pc (src/em_la.cc:113-206): B = C + M and the AMS
PetscErrorCode create_pc(EMContext *ctx) {
  PetscFunctionBegin;
  EMG_CALL(ctx, emg_create_pc(ctx->emg));
  PetscFunctionReturn(0);
}

PetscErrorCode destroy_pc(EMContext *ctx) {
  PetscFunctionBegin;
  EMG_CALL(ctx, emg_destroy_pc(ctx->emg));
  PetscFunctionReturn(0);
}

// the [re; im] VecNest blocks as one array of 2n, as the C ABI takes them
static PetscErrorCode nest_gather(Vec v, std::vector<double> &out) {
  Vec r, i;
  const PetscScalar *a, *b;
  PetscInt n;
  PetscCall(VecNestGetSubVec(v, 0, &r));
  PetscCall(VecNestGetSubVec(v, 1, &i));
  PetscCall(VecGetSize(r, &n));
  out.resize(2 * (size_t)n);
  PetscCall(VecGetArrayRead(r, &a));
  PetscCall(VecGetArrayRead(i, &b));
  std::copy(a, a + n, out.begin());
  std::copy(b, b + n, out.begin() + n);
  PetscCall(VecRestoreArrayRead(r, &a));
  PetscCall(VecRestoreArrayRead(i, &b));
  return 0;
}

static PetscErrorCode nest_scatter(const std::vector<double> &in, Vec v) {
  Vec r, i;
  PetscScalar *a, *b;
  PetscInt n;
  PetscCall(VecNestGetSubVec(v, 0, &r));
  PetscCall(VecNestGetSubVec(v, 1, &i));
  PetscCall(VecGetSize(r, &n));
  PetscCall(VecGetArray(r, &a));
  PetscCall(VecGetArray(i, &b));
  std::copy(in.begin(), in.begin() + n, a);
  std::copy(in.begin() + n, in.begin() + 2 * n, b);
  PetscCall(VecRestoreArray(r, &a));
  PetscCall(VecRestoreArray(i, &b));
  return 0;
}

// matshell_mult_a (src/em_la.cc:65-87): y = [C xr - M xi; -M xr - C xi]
PetscErrorCode matshell_mult_a(Mat A, Vec x, Vec y) {
  EMContext *ctx;
  std::vector<double> xv, yv;
  PetscFunctionBegin;
  PetscCall(MatShellGetContext(A, &ctx));
  PetscCall(nest_gather(x, xv));
  yv.resize(xv.size());
  EMG_CALL(ctx, emg_matshell_mult_a(ctx->emg, xv.data(), yv.data()));
  PetscCall(nest_scatter(yv, y));
  PetscFunctionReturn(0);
}

// pc_apply_b (src/em_la.cc:208-228): both halves through FCG(AMS)
PetscErrorCode pc_apply_b(PC pc, Vec b, Vec x) {
  EMContext *ctx;
  std::vector<double> bv, xv;
  PetscFunctionBegin;
  PetscCall(PCShellGetContext(pc, (void **)&ctx));
  PetscCall(nest_gather(b, bv));
  xv.resize(bv.size());
  EMG_CALL(ctx, emg_pc_apply_b(ctx->emg, bv.data(), xv.data()));
  PetscCall(nest_scatter(xv, x));
  PetscFunctionReturn(0);
}

// solve_linear_system (src/em_la.cc:35-63)
PetscErrorCode solve_linear_system(EMContext *ctx, const PETScBlockVector &s, PETScBlockVector &e, PetscInt max_it,
                                   PetscReal rtol) {
  const PetscScalar *sr, *si;
  PetscScalar *er, *ei;
  emg_solve_info info;
  PetscFunctionBegin;
  const int slot = slot_of(ctx, e);
  PetscCall(VecGetArrayRead(s.re, &sr));
  PetscCall(VecGetArrayRead(s.im, &si));
  int rc = emg_solve_linear_system(ctx->emg, slot, sr, si, (int)max_it, rtol, &info);
  PetscCall(VecRestoreArrayRead(s.re, &sr));
  PetscCall(VecRestoreArrayRead(s.im, &si));
  // like the reference, a solve that reaches max_it is not an error
  if (rc != EMG_OK && rc != EMG_DIVERGED_ITS) SETERRQ(ctx->world_comm, EM_ERR_USER, "%s", emg_last_error());
  PetscCall(VecGetArray(e.re, &er));
  PetscCall(VecGetArray(e.im, &ei));
  rc = emg_get_solution(ctx->emg, slot, er, ei);
  PetscCall(VecRestoreArray(e.re, &er));
  PetscCall(VecRestoreArray(e.im, &ei));
  EMG_CALL(ctx, rc);
  PetscFunctionReturn(0);
}

// estimate_error (src/em_fwd.cc:1102-1180): ctx->mt_error[XY/YX] or csem_error
PetscErrorCode estimate_error(EMContext *ctx, int fidx, int tidx) {
  PetscFunctionBegin;
  const long nt = ctx->n_tets;
  std::vector<double> err((tidx < 0 ? 2 : 1) * (size_t)nt);
  EMG_CALL(ctx, emg_estimate_error(ctx->emg, fidx, tidx, err.data(), nullptr));
  if (tidx < 0) {
    ctx->mt_error[XY_POLAR].v.assign(err.begin(), err.begin() + nt);
    ctx->mt_error[YX_POLAR].v.assign(err.begin() + nt, err.end());
  } else {
    ctx->csem_error.v = err;
  }
  PetscFunctionReturn(0);
}

// refine_fixed_fraction / refine_fixed_number (src/em_fwd.cc:1182-1240)
static PetscErrorCode mark(const Eigen::VectorXd &error, std::vector<bool> &flag, double fraction, bool by_fraction) {
  PetscFunctionBegin;
  if ((long)flag.size() != error.size()) SETERRQ(PETSC_COMM_SELF, EM_ERR_USER, "flag size mismatch");
  std::vector<unsigned char> f(flag.begin(), flag.end());
  int rc = by_fraction ? emg_refine_fixed_fraction((int)error.size(), error.data(), fraction, f.data())
                       : emg_refine_fixed_number((int)error.size(), error.data(), fraction, f.data());
  if (rc != EMG_OK) SETERRQ(PETSC_COMM_SELF, EM_ERR_USER, "%s", emg_last_error());
  for (size_t i = 0; i < f.size(); ++i) flag[i] = f[i] != 0;
  PetscFunctionReturn(0);
}

PetscErrorCode refine_fixed_fraction(const Eigen::VectorXd &error, std::vector<bool> &flag, double fraction) {
  return mark(error, flag, fraction, true);
}

PetscErrorCode refine_fixed_number(const Eigen::VectorXd &error, std::vector<bool> &flag, double fraction) {
  return mark(error, flag, fraction, false);
}
