// ORACLE — TEST INFRASTRUCTURE ONLY.
// Single-process stand-in for the PETSc API surface that Free CFD's sources
// use (PETSc 3.0/3.1 era signatures).  Vec is a dense std::vector<double>:
// VecSetValues / VecGetValues / VecSet / VecAXPY behave as PETSc's do on one
// rank, so the residual the reference assembles into its rhs Vec can be read
// back.  Mat records nothing unless the harness switches capture on (then
// MatSetValues accumulates the entries of the rows it asks for).  The KSP
// solve is not available: the harness never calls it.
#ifndef FCFD_REF_STUB_PETSCKSP_H
#define FCFD_REF_STUB_PETSCKSP_H

#include <cstddef>
#include <map>
#include <stdexcept>
#include <utility>
#include <vector>

#include "mpi.h"

typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscTruth;
typedef int PetscBool;
typedef const char *KSPType;
typedef int (*KSPOrthogFn)(void *, int);

#define PETSC_COMM_WORLD MPI_COMM_WORLD
#define PETSC_TRUE 1
#define PETSC_FALSE 0
#define PETSC_NULL 0
#define PETSC_DECIDE (-1)
#define PETSC_DEFAULT (-2)
#define KSPFGMRES "fgmres"
#define KSPGMRES "gmres"

enum InsertMode { INSERT_VALUES = 1, ADD_VALUES = 2 };
enum MatStructure { SAME_NONZERO_PATTERN = 0, DIFFERENT_NONZERO_PATTERN = 1 };
enum MatAssemblyType { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 };

struct FcfdRefVec { std::vector<double> v; };
struct FcfdRefMat {
  // Optional capture: entries (row, col) of rows in [cap_lo, cap_hi).
  std::map<std::pair<int, int>, double> entries;
};
struct FcfdRefKsp {
  int iterations;
  double rnorm;
  FcfdRefKsp() : iterations(0), rnorm(0.) {}
};
typedef FcfdRefVec *Vec;
typedef FcfdRefMat *Mat;
typedef FcfdRefKsp *KSP;
typedef FcfdRefKsp *PC;

// Matrix capture switch and row window (set by the harness; defined there).
extern int fcfd_ref_mat_capture;
extern int fcfd_ref_mat_cap_lo, fcfd_ref_mat_cap_hi;

extern int (*PetscErrorPrintf)(const char[], ...);

static inline PetscErrorCode PetscInitialize(int *, char ***, const char *, const char *) { return 0; }
static inline PetscErrorCode PetscFinalize() { return 0; }

static inline PetscErrorCode VecCreateMPI(MPI_Comm, PetscInt nlocal, PetscInt, Vec *v) {
  *v = new FcfdRefVec;
  (*v)->v.assign((size_t)nlocal, 0.);
  return 0;
}
static inline PetscErrorCode VecSetFromOptions(Vec) { return 0; }
static inline PetscErrorCode VecDuplicate(Vec a, Vec *b) {
  *b = new FcfdRefVec;
  (*b)->v.assign(a->v.size(), 0.);
  return 0;
}
static inline PetscErrorCode VecSet(Vec a, PetscScalar s) {
  for (size_t i = 0; i < a->v.size(); ++i) a->v[i] = s;
  return 0;
}
static inline PetscErrorCode VecSetValues(Vec a, PetscInt n, const PetscInt *idx, const PetscScalar *y, InsertMode m) {
  for (PetscInt i = 0; i < n; ++i) {
    if (m == ADD_VALUES) a->v.at((size_t)idx[i]) += y[i];
    else a->v.at((size_t)idx[i]) = y[i];
  }
  return 0;
}
static inline PetscErrorCode VecGetValues(Vec a, PetscInt n, const PetscInt *idx, PetscScalar *y) {
  for (PetscInt i = 0; i < n; ++i) y[i] = a->v.at((size_t)idx[i]);
  return 0;
}
static inline PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
static inline PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
static inline PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x) {
  for (size_t i = 0; i < y->v.size(); ++i) y->v[i] += a * x->v[i];
  return 0;
}
static inline PetscErrorCode VecDestroy(Vec v) {
  delete v;
  return 0;
}

static inline PetscErrorCode MatCreateMPIAIJ(MPI_Comm, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, const PetscInt *,
                                             PetscInt, const PetscInt *, Mat *A) {
  *A = new FcfdRefMat;
  return 0;
}
static inline PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt *rows, PetscInt n, const PetscInt *cols,
                                          const PetscScalar *v, InsertMode mode) {
  if (!fcfd_ref_mat_capture) return 0;
  for (PetscInt i = 0; i < m; ++i) {
    if (rows[i] < fcfd_ref_mat_cap_lo || rows[i] >= fcfd_ref_mat_cap_hi) continue;
    for (PetscInt j = 0; j < n; ++j) {
      double &e = A->entries[std::make_pair((int)rows[i], (int)cols[j])];
      if (mode == ADD_VALUES) e += v[i * n + j];
      else e = v[i * n + j];
    }
  }
  return 0;
}
static inline PetscErrorCode MatZeroEntries(Mat A) {
  A->entries.clear();
  return 0;
}
static inline PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
static inline PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType) { return 0; }
static inline PetscErrorCode MatDestroy(Mat A) {
  delete A;
  return 0;
}

static inline PetscErrorCode KSPCreate(MPI_Comm, KSP *k) {
  *k = new FcfdRefKsp;
  return 0;
}
static inline PetscErrorCode KSPSetOperators(KSP, Mat, Mat, MatStructure) { return 0; }
static inline PetscErrorCode KSPSetTolerances(KSP, PetscReal, PetscReal, PetscReal, PetscInt) { return 0; }
static inline PetscErrorCode KSPSetInitialGuessKnoll(KSP, PetscTruth) { return 0; }
static inline PetscErrorCode KSPSetType(KSP, KSPType) { return 0; }
static inline PetscErrorCode KSPGMRESSetRestart(KSP, PetscInt) { return 0; }
static inline PetscErrorCode KSPGMRESModifiedGramSchmidtOrthogonalization(void *, int) { return 0; }
static inline PetscErrorCode KSPGMRESSetOrthogonalization(KSP, KSPOrthogFn) { return 0; }
static inline PetscErrorCode KSPSetFromOptions(KSP) { return 0; }
static inline PetscErrorCode KSPSolve(KSP, Vec, Vec) {
  throw std::runtime_error("the single-process reference build has no linear solver");
}
static inline PetscErrorCode KSPGetIterationNumber(KSP k, PetscInt *n) {
  *n = k->iterations;
  return 0;
}
static inline PetscErrorCode KSPGetResidualNorm(KSP k, PetscReal *r) {
  *r = k->rnorm;
  return 0;
}
static inline PetscErrorCode KSPDestroy(KSP k) {
  delete k;
  return 0;
}
static inline PetscErrorCode PCDestroy(PC) { return 0; }

#endif
