// petscvec.h -- TEST INFRASTRUCTURE ONLY: PETSc vectors for the oracle's
// reference build.  A global vector lives in the shared arena (every rank sees
// all of it and owns a z-slab); a local vector is private and carries ghosts.
#pragma once

#include <vector>

#include "petscsys.h"

struct _p_DM;

struct _p_Vec {
  double *a = nullptr;      // storage (the whole lattice for a global vector)
  size_t n = 0;             // doubles in `a`
  size_t lo = 0, hi = 0;    // owned range of `a` in doubles
  bool local = false;
  _p_DM *dm = nullptr;
  std::vector<double> own;  // storage when not in the shared arena
};
typedef _p_Vec *Vec;

inline Vec lgvshim_new_global(_p_DM *dm, size_t n, size_t lo, size_t hi) {
  Vec v = new _p_Vec();
  v->a = lgvshim::alloc_global(n, v->own);
  v->n = n;
  v->lo = lo;
  v->hi = hi;
  v->dm = dm;
  return v;
}
inline Vec lgvshim_new_local(_p_DM *dm, size_t n) {
  Vec v = new _p_Vec();
  v->own.assign(n, 0.0);
  v->a = v->own.data();
  v->n = n;
  v->lo = 0;
  v->hi = n;
  v->local = true;
  v->dm = dm;
  return v;
}

inline PetscErrorCode VecDuplicate(Vec x, Vec *y) {
  *y = x->local ? lgvshim_new_local(x->dm, x->n) : lgvshim_new_global(x->dm, x->n, x->lo, x->hi);
  return 0;
}
inline PetscErrorCode VecCopy(Vec x, Vec y) {
  if (x->n != y->n || x->lo != y->lo || x->hi != y->hi) lgvshim::fail("VecCopy: layouts differ");
  std::memcpy(y->a + y->lo, x->a + x->lo, (x->hi - x->lo) * sizeof(double));
  return 0;
}
inline PetscErrorCode VecSet(Vec x, PetscScalar v) {
  for (size_t i = x->lo; i < x->hi; ++i) x->a[i] = v;
  return 0;
}
inline PetscErrorCode VecDestroy(Vec *x) {
  delete *x;  // arena storage is not reclaimed
  *x = nullptr;
  return 0;
}
inline PetscErrorCode VecGetLocalSize(Vec x, int *n) {
  *n = (int)(x->hi - x->lo);
  return 0;
}
inline PetscErrorCode VecGetArray(Vec x, PetscScalar **p) {
  *p = x->a + x->lo;
  return 0;
}
inline PetscErrorCode VecRestoreArray(Vec, PetscScalar **p) {
  *p = nullptr;
  return 0;
}
