// petscdmda.h -- TEST INFRASTRUCTURE ONLY: the structured-grid (DMDA) calls of
// the reference's stepper and measurer, for the oracle's reference build.
// 3-D, periodic in every direction, any stencil width; the process grid is
// 1 x 1 x R (z-slabs, the first P % R ranks own one extra plane).
#pragma once

#include <map>
#include <vector>

#include "petscvec.h"

typedef enum { DM_BOUNDARY_NONE, DM_BOUNDARY_GHOSTED, DM_BOUNDARY_MIRROR, DM_BOUNDARY_PERIODIC } DMBoundaryType;
typedef enum { DMDA_STENCIL_STAR, DMDA_STENCIL_BOX } DMDAStencilType;

struct _p_DM {
  int M = 0, N = 0, P = 0;  // x, y, z extents
  int dof = 0, s = 0;
  int zs = 0, ze = 0;       // owned planes [zs, ze)
  std::vector<Vec> pool;    // DMGetLocalVector work vectors
  std::map<void *, std::vector<std::vector<void *>>> tables;  // live DMDAVecGetArray* index tables

  size_t site_bytes() const { return (size_t)dof * sizeof(double); }
  size_t local_doubles() const { return (size_t)(M + 2 * s) * (N + 2 * s) * (ze - zs + 2 * s) * dof; }
  size_t global_doubles() const { return (size_t)M * N * P * dof; }
};
typedef _p_DM *DM;

inline int lgvshim_wrap(int a, int n) { return ((a % n) + n) % n; }

inline PetscErrorCode DMDACreate3d(MPI_Comm, DMBoundaryType bx, DMBoundaryType by, DMBoundaryType bz,
                                   DMDAStencilType, PetscInt M, PetscInt N, PetscInt P, PetscInt, PetscInt,
                                   PetscInt, PetscInt dof, PetscInt s, const PetscInt *, const PetscInt *,
                                   const PetscInt *, DM *da) {
  if (bx != DM_BOUNDARY_PERIODIC || by != DM_BOUNDARY_PERIODIC || bz != DM_BOUNDARY_PERIODIC)
    lgvshim::fail("DMDACreate3d: only periodic boundaries are provided");
  const int R = lgvshim::g_size, r = lgvshim::g_rank;
  if (P < R) lgvshim::fail("DMDACreate3d: more ranks than z planes");
  DM d = new _p_DM();
  d->M = M;
  d->N = N;
  d->P = P;
  d->dof = dof;
  d->s = s;
  int z = 0;
  for (int q = 0; q < r; ++q) z += P / R + (q < P % R ? 1 : 0);
  d->zs = z;
  d->ze = z + P / R + (r < P % R ? 1 : 0);
  if (s > d->ze - d->zs && R > 1) lgvshim::fail("DMDACreate3d: stencil wider than a slab");
  *da = d;
  return 0;
}
inline PetscErrorCode DMSetFromOptions(DM) { return 0; }
inline PetscErrorCode DMSetUp(DM) { return 0; }
inline PetscErrorCode DMDestroy(DM *da) {
  for (Vec v : (*da)->pool) delete v;
  delete *da;
  *da = nullptr;
  return 0;
}

inline PetscErrorCode DMDAGetCorners(DM da, PetscInt *xs, PetscInt *ys, PetscInt *zs, PetscInt *m, PetscInt *n,
                                     PetscInt *p) {
  if (xs) *xs = 0;
  if (ys) *ys = 0;
  if (zs) *zs = da->zs;
  if (m) *m = da->M;
  if (n) *n = da->N;
  if (p) *p = da->ze - da->zs;
  return 0;
}

inline PetscErrorCode DMCreateGlobalVector(DM da, Vec *v) {
  const size_t plane = (size_t)da->M * da->N * da->dof;
  *v = lgvshim_new_global(da, da->global_doubles(), plane * da->zs, plane * da->ze);
  return 0;
}
inline PetscErrorCode DMCreateLocalVector(DM da, Vec *v) {
  *v = lgvshim_new_local(da, da->local_doubles());
  return 0;
}
inline PetscErrorCode DMGetLocalVector(DM da, Vec *v) {
  if (!da->pool.empty()) {
    *v = da->pool.back();
    da->pool.pop_back();
    return 0;
  }
  return DMCreateLocalVector(da, v);
}
inline PetscErrorCode DMRestoreLocalVector(DM da, Vec *v) {
  da->pool.push_back(*v);
  *v = nullptr;
  return 0;
}

// Offset of local-box site (i, j, k) (global indices, ghosts included) in doubles.
inline size_t lgvshim_local_off(DM da, int i, int j, int k) {
  const size_t gx = da->M + 2 * da->s, gy = da->N + 2 * da->s;
  return (((size_t)(k - da->zs + da->s) * gy + (j + da->s)) * gx + (i + da->s)) * da->dof;
}
inline size_t lgvshim_global_off(DM da, int i, int j, int k) {
  return (((size_t)k * da->N + j) * da->M + i) * da->dof;
}

// Fill the local box (owned sites and ghosts) from the global vector with the
// periodic wrap.  Every rank must have finished writing its slab before the
// copy, and must not write again until all copies are done: two barriers.
inline PetscErrorCode DMGlobalToLocalBegin(DM da, Vec g, InsertMode mode, Vec l) {
  if (mode != INSERT_VALUES || g->local || !l->local) lgvshim::fail("DMGlobalToLocal: unsupported arguments");
  lgvshim::barrier();
  const int s = da->s;
  const size_t sb = da->site_bytes(), row = (size_t)da->M * sb;
  for (int k = da->zs - s; k < da->ze + s; ++k) {
    const int kw = lgvshim_wrap(k, da->P);
    for (int j = -s; j < da->N + s; ++j) {
      const int jw = lgvshim_wrap(j, da->N);
      std::memcpy(l->a + lgvshim_local_off(da, 0, j, k), g->a + lgvshim_global_off(da, 0, jw, kw), row);
      for (int i = -s; i < 0; ++i)
        std::memcpy(l->a + lgvshim_local_off(da, i, j, k), g->a + lgvshim_global_off(da, i + da->M, jw, kw), sb);
      for (int i = da->M; i < da->M + s; ++i)
        std::memcpy(l->a + lgvshim_local_off(da, i, j, k), g->a + lgvshim_global_off(da, i - da->M, jw, kw), sb);
    }
  }
  return 0;
}
inline PetscErrorCode DMGlobalToLocalEnd(DM, Vec, InsertMode, Vec) {
  lgvshim::barrier();
  return 0;
}

// Add the local box into the global vector, ghosts onto the sites they wrap
// to.  Owned planes first, then the planes below and above the slab (owned by
// the neighbouring ranks), with a barrier between phases so no two ranks add
// into one plane at once.
inline void lgvshim_add_planes(DM da, Vec l, Vec g, int k0, int k1) {
  const int s = da->s;
  for (int k = k0; k < k1; ++k) {
    const int kw = lgvshim_wrap(k, da->P);
    for (int j = -s; j < da->N + s; ++j) {
      const int jw = lgvshim_wrap(j, da->N);
      for (int i = -s; i < da->M + s; ++i) {
        const int iw = lgvshim_wrap(i, da->M);
        const double *src = l->a + lgvshim_local_off(da, i, j, k);
        double *dst = g->a + lgvshim_global_off(da, iw, jw, kw);
        for (int c = 0; c < da->dof; ++c) dst[c] += src[c];
      }
    }
  }
}
inline PetscErrorCode DMLocalToGlobal(DM da, Vec l, InsertMode mode, Vec g) {
  if (mode != ADD_VALUES || !l->local || g->local) lgvshim::fail("DMLocalToGlobal: only ADD_VALUES is provided");
  const int s = da->s;
  if (lgvshim::g_size == 1) {
    lgvshim_add_planes(da, l, g, da->zs - s, da->ze + s);
    return 0;
  }
  lgvshim_add_planes(da, l, g, da->zs, da->ze);
  lgvshim::barrier();
  lgvshim_add_planes(da, l, g, da->zs - s, da->zs);
  lgvshim::barrier();
  lgvshim_add_planes(da, l, g, da->ze, da->ze + s);
  lgvshim::barrier();
  return 0;
}

// Index tables for a[k][j][i] (site structs) or a[k][j][i][c] (DOF form), in
// global indices: the owned slab of a global vector, the ghosted box of a
// local one.
inline void *lgvshim_tables(DM da, Vec v, bool dof_form) {
  int i0, j0, k0, ni, nj, nk;
  if (v->local) {
    i0 = -da->s, j0 = -da->s, k0 = da->zs - da->s;
    ni = da->M + 2 * da->s, nj = da->N + 2 * da->s, nk = da->ze - da->zs + 2 * da->s;
  } else {
    i0 = 0, j0 = 0, k0 = da->zs;
    ni = da->M, nj = da->N, nk = da->ze - da->zs;
  }
  char *base = v->local ? (char *)v->a : (char *)(v->a + lgvshim_global_off(da, 0, 0, da->zs));
  const size_t sb = da->site_bytes();
  std::vector<std::vector<void *>> t;
  if (dof_form) {
    std::vector<void *> sites((size_t)nk * nj * ni);
    for (size_t q = 0; q < sites.size(); ++q) sites[q] = base + q * sb;
    std::vector<void *> rows((size_t)nk * nj);
    t.push_back(std::move(sites));
    for (size_t q = 0; q < rows.size(); ++q) rows[q] = (void *)(&t[0][q * ni] - i0);
    std::vector<void *> planes(nk);
    t.push_back(std::move(rows));
    for (int q = 0; q < nk; ++q) planes[q] = (void *)(&t[1][(size_t)q * nj] - j0);
    t.push_back(std::move(planes));
  } else {
    std::vector<void *> rows((size_t)nk * nj);
    for (size_t q = 0; q < rows.size(); ++q) rows[q] = base + (q * ni - (ptrdiff_t)i0) * sb;
    std::vector<void *> planes(nk);
    t.push_back(std::move(rows));
    for (int q = 0; q < nk; ++q) planes[q] = (void *)(&t[0][(size_t)q * nj] - j0);
    t.push_back(std::move(planes));
  }
  void *top = (void *)(&t.back()[0] - k0);
  da->tables[top] = std::move(t);
  return top;
}
inline PetscErrorCode lgvshim_untable(DM da, void *arrayp) {
  void *top = *(void **)arrayp;
  da->tables.erase(top);
  *(void **)arrayp = nullptr;
  return 0;
}

inline PetscErrorCode DMDAVecGetArray(DM da, Vec v, void *arrayp) {
  *(void **)arrayp = lgvshim_tables(da, v, false);
  return 0;
}
inline PetscErrorCode DMDAVecRestoreArray(DM da, Vec, void *arrayp) { return lgvshim_untable(da, arrayp); }
inline PetscErrorCode DMDAVecGetArrayRead(DM da, Vec v, void *arrayp) { return DMDAVecGetArray(da, v, arrayp); }
inline PetscErrorCode DMDAVecRestoreArrayRead(DM da, Vec v, void *arrayp) { return DMDAVecRestoreArray(da, v, arrayp); }
inline PetscErrorCode DMDAVecGetArrayDOF(DM da, Vec v, void *arrayp) {
  *(void **)arrayp = lgvshim_tables(da, v, true);
  return 0;
}
inline PetscErrorCode DMDAVecRestoreArrayDOF(DM da, Vec, void *arrayp) { return lgvshim_untable(da, arrayp); }
