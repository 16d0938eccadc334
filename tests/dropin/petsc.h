/*
 * Minimal stand-in for the part of PETSc's API that the drop-in bodies of
 * em_la.cc / em_fwd.cc use, so that they compile and run in a test without
 * PETSc.  Sequential only: a Vec is a host array, MPI_Comm an int.  Test
 * infrastructure; the real build includes PETSc's own header instead.
 */
#ifndef EMG_TEST_PETSC_STUB_H
#define EMG_TEST_PETSC_STUB_H

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <vector>

typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscReal;
typedef double PetscScalar;
typedef int MPI_Comm;
enum PetscBool { PETSC_FALSE = 0, PETSC_TRUE = 1 };
#define PETSC_COMM_SELF 0
#define PETSC_COMM_WORLD 0

struct _p_Vec {
  std::vector<PetscScalar> a;
  _p_Vec *sub[2] = {nullptr, nullptr};  // VecNest of two blocks (not owned)
};
typedef _p_Vec *Vec;
struct _p_Mat {
  void *ctx;
};
typedef _p_Mat *Mat;
struct _p_PC {
  void *ctx;
};
typedef _p_PC *PC;
struct _p_KSP {
  PC pc;
};
typedef _p_KSP *KSP;
typedef void *PetscViewer;

/* error handling: PetscCall returns the nonzero code, SETERRQ prints and returns */
#define PetscFunctionBegin
#define PetscFunctionReturn(x) return (x)
#define PetscCall(x)                       \
  do {                                     \
    PetscErrorCode ierr__ = (x);           \
    if (ierr__) return ierr__;             \
  } while (0)
inline PetscErrorCode petsc_stub_error(MPI_Comm, PetscErrorCode code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::fprintf(stderr, "[PETSc stub] error %d: ", code);
  std::vfprintf(stderr, fmt, ap);
  std::fprintf(stderr, "\n");
  va_end(ap);
  return code;
}
#define SETERRQ(comm, code, ...) return petsc_stub_error(comm, code, __VA_ARGS__)

inline PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt n, Vec *v) {
  *v = new _p_Vec();
  (*v)->a.assign((size_t)n, 0.0);
  return 0;
}
inline PetscErrorCode VecDestroy(Vec *v) {
  delete *v;
  *v = nullptr;
  return 0;
}
inline PetscErrorCode VecGetSize(Vec v, PetscInt *n) {
  *n = (PetscInt)v->a.size();
  return 0;
}
inline PetscErrorCode VecGetArray(Vec v, PetscScalar **p) {
  *p = v->a.data();
  return 0;
}
inline PetscErrorCode VecRestoreArray(Vec, PetscScalar **p) {
  *p = nullptr;
  return 0;
}
inline PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **p) {
  *p = v->a.data();
  return 0;
}
inline PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar **p) {
  *p = nullptr;
  return 0;
}
inline PetscErrorCode VecZeroEntries(Vec v) {
  for (auto &x : v->a) x = 0.0;
  return 0;
}
inline PetscErrorCode VecCreateNest(MPI_Comm, PetscInt nb, void *, Vec *blocks, Vec *v) {
  if (nb != 2) return 1;
  *v = new _p_Vec();
  (*v)->sub[0] = blocks[0];
  (*v)->sub[1] = blocks[1];
  return 0;
}
inline PetscErrorCode VecNestGetSubVec(Vec v, PetscInt i, Vec *s) {
  if (i < 0 || i > 1 || !v->sub[i]) return 1;
  *s = v->sub[i];
  return 0;
}
inline PetscErrorCode MatShellGetContext(Mat m, void *ctx) {
  *(void **)ctx = m->ctx;
  return 0;
}
inline PetscErrorCode PCShellGetContext(PC pc, void *ctx) {
  *(void **)ctx = pc->ctx;
  return 0;
}

#endif
