// Plumbing shared by the facade headers: the C ABI of libm3lb.so, a registry
// of live solver handles (so a global fence can wait for all of them) and
// the facade's error policy.
//
// Errors: the C ABI returns status codes and never aborts.  The facade keeps
// the reference's behaviour for setup errors (print the reason, abort:
// src/solver/FluidSolver.hpp:204-209) so that call sites need no new error
// handling.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <set>

#include "m3lb.h"

namespace m3lb_facade {

struct Registry {
  std::mutex mu;
  std::set<m3lb_solver*> live;
  std::set<m3lb_scalar*> live_scalar;
};
inline Registry& registry() {
  static Registry r;
  return r;
}
inline void add(m3lb_solver* h) {
  std::lock_guard<std::mutex> g(registry().mu);
  registry().live.insert(h);
}
inline void remove(m3lb_solver* h) {
  std::lock_guard<std::mutex> g(registry().mu);
  registry().live.erase(h);
}
inline void add(m3lb_scalar* h) {
  std::lock_guard<std::mutex> g(registry().mu);
  registry().live_scalar.insert(h);
}
inline void remove(m3lb_scalar* h) {
  std::lock_guard<std::mutex> g(registry().mu);
  registry().live_scalar.erase(h);
}

inline void check(int rc, const char* what) {
  if (rc != M3LB_OK) {
    std::fprintf(stderr, "m3lb: %s failed (%d): %s\n", what, rc, m3lb_last_error());
    std::abort();
  }
}

inline void fence_all() {
  std::lock_guard<std::mutex> g(registry().mu);
  for (m3lb_solver* h : registry().live) check(m3lb_sync(h), "fence");
  for (m3lb_scalar* h : registry().live_scalar) check(m3lb_scalar_sync(h), "fence");
}

}  // namespace m3lb_facade
