// shim_runtime.h -- TEST INFRASTRUCTURE ONLY.
//
// A single-node stand-in for the parts of PETSc and MPI that the reference
// stepper and measurer call (Stepper.cxx, ModelA.h, NoiseGenerator.h,
// measurer.cxx), so that those translation units compile unmodified and run as
// the oracle's reference build.  The surface is the one listed by the calls in
// those files: DMDA 3-D periodic with stencil width 1, global/local vectors,
// DMGlobalToLocal (INSERT_VALUES), DMLocalToGlobal (ADD_VALUES), DMDA array
// access with ghost-offset indexing, VecSet/VecCopy/VecDuplicate, MPI
// reductions and broadcasts, PetscPrintf and the PetscLogEvent timers.
//
// Ranks are processes.  The driver (ref_stepper_main.cpp) maps one shared
// arena, then forks; every rank sees the same global vectors in that arena,
// owns a z-slab of them as DMDACreate3d would with a 1 x 1 x R process grid
// (the first N % R ranks own one extra plane), keeps its local (ghosted)
// vectors private, and meets the others at process-shared barriers.  With one
// rank nothing is shared or forked.  Reductions add the ranks' contributions
// in rank order.
#pragma once

#include <pthread.h>
#include <sys/mman.h>

#include <chrono>
#include <cstdarg>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

namespace lgvshim {

// ---- ranks and the shared arena ---------------------------------------------
struct Shared {
  pthread_barrier_t barrier;
  size_t arena_bytes;   // bytes after the header for global vectors
  size_t slot_bytes;    // bytes per rank in the reduction slots
  size_t arena_used;    // bump pointer (only rank 0's copy is authoritative; all ranks allocate alike)
};

inline int g_rank = 0;
inline int g_size = 1;
inline Shared *g_shared = nullptr;  // null with one rank
inline char *g_arena = nullptr;     // global vectors
inline char *g_slots = nullptr;     // reduction slots, slot_bytes per rank
inline size_t g_arena_off = 0;      // this rank's bump pointer

[[noreturn]] inline void fail(const char *what) {
  std::fprintf(stderr, "shim(rank %d): %s\n", g_rank, what);
  std::fflush(stderr);
  std::_Exit(70);
}

// Map the arena before forking.  arena_bytes: room for every global vector the
// run creates; slot_bytes: the largest reduction payload.
inline void setup_shared(int size, size_t arena_bytes, size_t slot_bytes) {
  g_size = size;
  if (size == 1) return;
  const size_t hdr = (sizeof(Shared) + 4095) / 4096 * 4096;
  const size_t total = hdr + arena_bytes + slot_bytes * (size_t)size;
  void *p = mmap(nullptr, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  if (p == MAP_FAILED) fail("mmap of the shared arena failed");
  g_shared = (Shared *)p;
  g_shared->arena_bytes = arena_bytes;
  g_shared->slot_bytes = slot_bytes;
  pthread_barrierattr_t at;
  pthread_barrierattr_init(&at);
  pthread_barrierattr_setpshared(&at, PTHREAD_PROCESS_SHARED);
  if (pthread_barrier_init(&g_shared->barrier, &at, (unsigned)size)) fail("pthread_barrier_init failed");
  g_arena = (char *)p + hdr;
  g_slots = g_arena + arena_bytes;
}

inline void barrier() {
  if (g_size == 1) return;
  pthread_barrier_wait(&g_shared->barrier);
}

// Storage of a global vector: shared when there are several ranks.
inline double *alloc_global(size_t n, std::vector<double> &own) {
  if (g_size == 1) {
    own.assign(n, 0.0);
    return own.data();
  }
  const size_t bytes = (n * sizeof(double) + 255) / 256 * 256;
  if (g_arena_off + bytes > g_shared->arena_bytes) fail("shared arena exhausted (too many global vectors)");
  double *p = (double *)(g_arena + g_arena_off);
  g_arena_off += bytes;
  return p;
}

// Reduction in rank order: every rank deposits n doubles, then `combine`
// reads all deposits.  Two barriers keep the slots stable.
template <class F>
inline void exchange(const void *src, size_t bytes, F combine) {
  if (g_size == 1) {
    combine((const char *)src, (size_t)0);
    return;
  }
  if (bytes > g_shared->slot_bytes) fail("reduction payload larger than the slot");
  std::memcpy(g_slots + (size_t)g_rank * g_shared->slot_bytes, src, bytes);
  barrier();
  for (int r = 0; r < g_size; ++r) combine(g_slots + (size_t)r * g_shared->slot_bytes, (size_t)r);
  barrier();
}

// ---- event timers (PetscLogEvent) ------------------------------------------
struct EventTimer {
  std::string name;
  double seconds = 0;
  long count = 0;
  std::chrono::steady_clock::time_point t0;
  int depth = 0;
};
inline std::vector<EventTimer> g_events;

inline int event_register(const char *name) {
  for (size_t i = 0; i < g_events.size(); ++i)
    if (g_events[i].name == name) return (int)i;
  g_events.push_back(EventTimer{name});
  return (int)g_events.size() - 1;
}
inline void event_begin(int e) {
  if (e < 0 || (size_t)e >= g_events.size()) return;
  EventTimer &t = g_events[e];
  if (t.depth++ == 0) t.t0 = std::chrono::steady_clock::now();
}
inline void event_end(int e) {
  if (e < 0 || (size_t)e >= g_events.size()) return;
  EventTimer &t = g_events[e];
  if (--t.depth == 0) {
    t.seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t.t0).count();
    t.count++;
  }
}

}  // namespace lgvshim
