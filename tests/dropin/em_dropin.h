/*
 * The reference's hot-path declarations (src/em_la.h:8-20, src/em_fwd.h:10-51)
 * and the EMContext fields they touch (src/em_ctx.h:15-64, src/em_defs.h),
 * with one added member: the emfem_b200 context.  Eigen and the mesh classes
 * are reduced to what the drop-in bodies use.  Test infrastructure.
 */
#ifndef EMG_TEST_EM_DROPIN_H
#define EMG_TEST_EM_DROPIN_H

#include <map>
#include <vector>

#include "emfem_b200.h"
#include "petsc.h"

namespace Eigen {
// the part of Eigen::VectorXd the error vectors and marking use
struct VectorXd {
  std::vector<double> v;
  long size() const { return (long)v.size(); }
  void resize(long n) { v.assign((size_t)n, 0.0); }
  double *data() { return v.data(); }
  const double *data() const { return v.data(); }
  double &operator[](long i) { return v[(size_t)i]; }
  double operator[](long i) const { return v[(size_t)i]; }
};
}  // namespace Eigen

struct PETScBlockVector {
  Vec re, im;
};
enum PolarType { XY_POLAR = -1, YX_POLAR = -2 };
#define EM_ERR_USER -1

struct EMContext {
  MPI_Comm world_comm = 0, group_comm = 0;
  std::vector<double> freqs;
  std::vector<double> tx;          // TX_SIZE values per transmitter
  std::vector<double> rx;          // 3 per receiver (Point in the reference)
  PETScBlockVector s, csem_e, dual_e;
  std::map<int, PETScBlockVector> mt_e;
  Mat A = nullptr;                 // MatShell whose context is this EMContext
  KSP A_ksp = nullptr, B_ksp = nullptr;
  Eigen::VectorXd csem_error;
  std::map<int, Eigen::VectorXd> mt_error;
  PetscReal e_rtol = 1e-8, dual_rtol = 1e-6;
  PetscInt K_max_it = 100, n_tx_divisions = 20;
  PetscInt n_edges = 0, n_tets = 0;
  emg_context *emg = nullptr;      // added: the device context
};

PetscErrorCode create_linear_system(EMContext *, int);
PetscErrorCode destroy_linear_system(EMContext *);
PetscErrorCode assemble_matrix(EMContext *, int);
PetscErrorCode assemble_rhs_csem(EMContext *, int, int);
PetscErrorCode assemble_rhs_dual(EMContext *);
PetscErrorCode create_pc(EMContext *);
PetscErrorCode destroy_pc(EMContext *);
PetscErrorCode pc_apply_b(PC, Vec, Vec);
PetscErrorCode matshell_mult_a(Mat, Vec, Vec);
PetscErrorCode solve_linear_system(EMContext *, const PETScBlockVector &, PETScBlockVector &, PetscInt, PetscReal);
PetscErrorCode estimate_error(EMContext *, int, int);
PetscErrorCode refine_fixed_fraction(const Eigen::VectorXd &, std::vector<bool> &, double);
PetscErrorCode refine_fixed_number(const Eigen::VectorXd &, std::vector<bool> &, double);

#endif
