// petscsys.h -- TEST INFRASTRUCTURE ONLY: the PETSc/MPI system layer that the
// reference's stepper and measurer use, for the oracle's reference build.
// Single node; ranks are processes sharing an arena (shim_runtime.h).
#pragma once

#include <math.h>

#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "shim_runtime.h"

typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscInt;
typedef int PetscMPIInt;
typedef int PetscErrorCode;
typedef int PetscClassId;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef enum { INSERT_VALUES = 1, ADD_VALUES = 2 } InsertMode;

#define PETSC_DECIDE (-1)
#define PETSC_MAX_PATH_LEN 4096

// ---- MPI ---------------------------------------------------------------------
struct lgvshim_comm {
  int id;
};
typedef lgvshim_comm MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
inline constexpr MPI_Comm MPI_COMM_WORLD{0};
#define PETSC_COMM_WORLD MPI_COMM_WORLD
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPIU_SCALAR 2
#define MPIU_REAL 2
#define MPIU_BOOL 3
#define MPI_SUM 0

inline size_t lgvshim_type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_INT: return sizeof(int);
    case MPI_DOUBLE: return sizeof(double);
    case MPIU_BOOL: return sizeof(PetscBool);
  }
  lgvshim::fail("unsupported MPI datatype");
}

inline int MPI_Comm_rank(MPI_Comm, int *r) {
  *r = lgvshim::g_rank;
  return 0;
}
inline int MPI_Comm_size(MPI_Comm, int *s) {
  *s = lgvshim::g_size;
  return 0;
}

// Sum over ranks in rank order (double or int).
inline void lgvshim_sum(const void *send, void *recv, int n, MPI_Datatype t, bool to_me) {
  const size_t es = lgvshim_type_size(t);
  if (t != MPI_DOUBLE && t != MPI_INT) lgvshim::fail("MPI_SUM on an unsupported datatype");
  std::vector<char> acc((size_t)n * es, 0);
  lgvshim::exchange(send, (size_t)n * es, [&](const char *src, size_t r) {
    if (!to_me) return;
    for (int i = 0; i < n; ++i) {
      if (t == MPI_DOUBLE) {
        double a, b;
        std::memcpy(&b, src + i * es, es);
        if (r == 0) a = b;
        else {
          std::memcpy(&a, acc.data() + i * es, es);
          a = a + b;
        }
        std::memcpy(acc.data() + i * es, &a, es);
      } else {
        int a, b;
        std::memcpy(&b, src + i * es, es);
        if (r == 0) a = b;
        else {
          std::memcpy(&a, acc.data() + i * es, es);
          a = a + b;
        }
        std::memcpy(acc.data() + i * es, &a, es);
      }
    }
  });
  if (to_me) std::memcpy(recv, acc.data(), (size_t)n * es);
}

inline int MPI_Reduce(const void *send, void *recv, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm) {
  if (op != MPI_SUM) lgvshim::fail("only MPI_SUM is supported");
  lgvshim_sum(send, recv, n, t, lgvshim::g_rank == root);
  return 0;
}
inline int MPI_Allreduce(const void *send, void *recv, int n, MPI_Datatype t, MPI_Op op, MPI_Comm) {
  if (op != MPI_SUM) lgvshim::fail("only MPI_SUM is supported");
  lgvshim_sum(send, recv, n, t, true);
  return 0;
}
inline int MPI_Bcast(void *buf, int n, MPI_Datatype t, int root, MPI_Comm) {
  const size_t bytes = (size_t)n * lgvshim_type_size(t);
  lgvshim::exchange(buf, bytes, [&](const char *src, size_t r) {
    if ((int)r == root && lgvshim::g_rank != root) std::memcpy(buf, src, bytes);
  });
  return 0;
}
inline int MPI_Barrier(MPI_Comm) {
  lgvshim::barrier();
  return 0;
}

// ---- PETSc system -------------------------------------------------------------
#define PetscCall(call)                         \
  do {                                          \
    PetscErrorCode lgvshim_ierr_ = (call);      \
    if (lgvshim_ierr_) return lgvshim_ierr_;    \
  } while (0)
#define PetscCallVoid(call)                     \
  do {                                          \
    PetscErrorCode lgvshim_ierr_ = (call);      \
    if (lgvshim_ierr_) return;                  \
  } while (0)
#define CHKERRQ(ierr)      \
  do {                     \
    if (ierr) return ierr; \
  } while (0)

// Only rank 0 prints, as PetscPrintf on PETSC_COMM_WORLD does.
inline PetscErrorCode PetscPrintf(MPI_Comm, const char *fmt, ...) {
  if (lgvshim::g_rank != 0) return 0;
  va_list ap;
  va_start(ap, fmt);
  std::vfprintf(stdout, fmt, ap);
  va_end(ap);
  return 0;
}
// The one-argument form ModelA::write uses when built without HDF5.
inline PetscErrorCode PetscPrintf(const char *fmt, ...) {
  if (lgvshim::g_rank != 0) return 0;
  va_list ap;
  va_start(ap, fmt);
  std::vfprintf(stdout, fmt, ap);
  va_end(ap);
  return 0;
}

inline PetscErrorCode PetscInitialize(int *, char ***, const char *, const char *) { return 0; }
inline PetscErrorCode PetscFinalize() { return 0; }

typedef int PetscLogEvent;
inline PetscErrorCode PetscLogEventRegister(const char *name, PetscClassId, PetscLogEvent *e) {
  *e = lgvshim::event_register(name);
  return 0;
}
inline PetscErrorCode PetscLogEventBegin(PetscLogEvent e, const void *, const void *, const void *, const void *) {
  lgvshim::event_begin(e);
  return 0;
}
inline PetscErrorCode PetscLogEventEnd(PetscLogEvent e, const void *, const void *, const void *, const void *) {
  lgvshim::event_end(e);
  return 0;
}

typedef struct lgvshim_object *PetscObject;

// PETSc built with complex support gives C++ mixed complex/integer arithmetic
// (the integer converted to PetscReal); the measurer's FFT normalisation
// divides a std::complex<double> by a size_t (measurer.h:39).
#define LGVSHIM_COMPLEX_INT_OPS(T)                                                                                    \
  inline std::complex<double> operator/(const std::complex<double> &a, const T &b) { return a / (PetscReal)b; }     \
  inline std::complex<double> operator*(const std::complex<double> &a, const T &b) { return a * (PetscReal)b; }     \
  inline std::complex<double> operator*(const T &a, const std::complex<double> &b) { return (PetscReal)a * b; }     \
  inline std::complex<double> operator+(const std::complex<double> &a, const T &b) { return a + (PetscReal)b; }     \
  inline std::complex<double> operator-(const std::complex<double> &a, const T &b) { return a - (PetscReal)b; }
LGVSHIM_COMPLEX_INT_OPS(int)
LGVSHIM_COMPLEX_INT_OPS(long)
LGVSHIM_COMPLEX_INT_OPS(unsigned long)
inline PetscErrorCode PetscObjectSetName(PetscObject, const char *) { return 0; }
