// A per-device cache of one device address that stays valid only inside the
// CUDA context it was looked up in.
//
// A __device__ array lives in the module that a context loaded, so its
// address belongs to that context: after cudaDeviceReset the primary context
// is created anew and the module may load elsewhere, and a caller that makes
// a non-primary context current sees the module of that context.  The cache
// therefore keeps, per device index, the ID of the context the address was
// looked up in (cuCtxGetId: unique for the life of the process, never reused)
// and looks the address up again whenever the current context's ID differs.
// Plain C++ with no CUDA types, so the decision logic is also compiled and
// checked on a host without a GPU.
#pragma once
#include <mutex>

namespace m3lb {

template <int NDEV>
class CtxAddrCache {
 public:
  // The address for device `dev` under the context with ID `ctx`: the cached
  // one when it was looked up under that same context, else lookup(&addr)
  // (returning 0 on success) is called and its result stored for `ctx`.
  // ctx == 0 means "context unknown": the address is looked up and not kept.
  // Returns 0, the lookup's nonzero status, or -1 for a device index out of
  // range.
  template <class Lookup>
  int get(int dev, unsigned long long ctx, Lookup lookup, void** out) {
    if (dev < 0 || dev >= NDEV) return -1;
    std::lock_guard<std::mutex> lk(mu_);
    Entry& e = e_[dev];
    if (ctx != 0 && e.addr && e.ctx == ctx) {
      *out = e.addr;
      return 0;
    }
    void* p = nullptr;
    const int rc = lookup(&p);
    if (rc) return rc;
    if (ctx != 0) {
      e.ctx = ctx;
      e.addr = p;
    }
    *out = p;
    return 0;
  }

 private:
  struct Entry {
    unsigned long long ctx = 0;
    void* addr = nullptr;
  };
  std::mutex mu_;
  Entry e_[NDEV];
};

}  // namespace m3lb
