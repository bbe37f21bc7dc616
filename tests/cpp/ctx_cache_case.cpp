// Host-only check of the per-context address cache behind
// m3lb_reduce_static (m3lb_b200/csrc/ctx_cache.h): an address is looked up
// once per (device, context), looked up again when the device's current
// context changes (a new context after cudaDeviceReset has a new ID), never
// kept when the context is unknown, and a failed lookup is reported and not
// cached.  Prints "ok" and exits 0 when every check holds.
#include <cstdio>

#include "ctx_cache.h"

static int fails = 0;
#define CHECK(c)                                                \
  do {                                                          \
    if (!(c)) {                                                 \
      std::printf("FAIL line %d: %s\n", __LINE__, #c);          \
      ++fails;                                                  \
    }                                                           \
  } while (0)

int main() {
  m3lb::CtxAddrCache<4> cache;
  int lookups = 0;
  char mod_a[1], mod_b[1], mod_c[1];
  void* next = mod_a;  // what the next lookup returns
  auto lookup = [&](void** p) {
    ++lookups;
    *p = next;
    return 0;
  };
  void* got = nullptr;

  CHECK(cache.get(0, 11, lookup, &got) == 0 && got == mod_a && lookups == 1);
  CHECK(cache.get(0, 11, lookup, &got) == 0 && got == mod_a && lookups == 1);  // cached
  next = mod_b;  // the device was reset: new context ID, module elsewhere
  CHECK(cache.get(0, 12, lookup, &got) == 0 && got == mod_b && lookups == 2);
  CHECK(cache.get(0, 12, lookup, &got) == 0 && got == mod_b && lookups == 2);
  next = mod_c;  // another device keeps its own entry
  CHECK(cache.get(1, 12, lookup, &got) == 0 && got == mod_c && lookups == 3);
  CHECK(cache.get(0, 12, lookup, &got) == 0 && got == mod_b && lookups == 3);
  // unknown context: looked up every time, never stored
  CHECK(cache.get(2, 0, lookup, &got) == 0 && got == mod_c && lookups == 4);
  CHECK(cache.get(2, 0, lookup, &got) == 0 && lookups == 5);
  // a failing lookup is returned and leaves the entry as it was
  auto bad = [&](void** p) {
    ++lookups;
    *p = nullptr;
    return 7;
  };
  CHECK(cache.get(0, 13, bad, &got) == 7 && lookups == 6);
  CHECK(cache.get(0, 12, lookup, &got) == 0 && got == mod_b && lookups == 6);
  // device index out of range
  CHECK(cache.get(4, 12, lookup, &got) == -1 && cache.get(-1, 12, lookup, &got) == -1);
  CHECK(lookups == 6);
  if (fails) return 1;
  std::printf("ok\n");
  return 0;
}
