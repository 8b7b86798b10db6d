// Host-only checks of the per-context address cache behind
// s1b_goldstein_noalloc (no GPU: contexts are stand-in handles and ids).
#include <cstdio>

#include "s1b_ctx_cache.h"

static int failures = 0;
#define CHECK(cond)                                              \
  do {                                                           \
    if (!(cond)) {                                               \
      std::printf("FAILED line %d: %s\n", __LINE__, #cond);      \
      ++failures;                                                \
    }                                                            \
  } while (0)

int main() {
  char ctx_a, ctx_b, ctx_c, addr1, addr2, addr3;
  void *v = nullptr;
  {
    ContextKeyedCache<4> c;
    CHECK(!c.find(&ctx_a, 1, &v));
    c.put(&ctx_a, 1, &addr1);
    CHECK(c.find(&ctx_a, 1, &v) && v == &addr1);
    // a second context on the same device keeps its own address
    CHECK(!c.find(&ctx_b, 2, &v));
    c.put(&ctx_b, 2, &addr2);
    CHECK(c.find(&ctx_b, 2, &v) && v == &addr2);
    CHECK(c.find(&ctx_a, 1, &v) && v == &addr1);
    // the handle of a destroyed context reused by a new one (new id): a miss,
    // and the new address replaces the stale entry
    CHECK(!c.find(&ctx_a, 3, &v));
    c.put(&ctx_a, 3, &addr3);
    CHECK(c.find(&ctx_a, 3, &v) && v == &addr3);
    CHECK(!c.find(&ctx_a, 1, &v));
    CHECK(c.find(&ctx_b, 2, &v) && v == &addr2);
  }
  {
    // more contexts than slots: the oldest entries are evicted, never a
    // wrong address returned
    ContextKeyedCache<2> c;
    c.put(&ctx_a, 1, &addr1);
    c.put(&ctx_b, 2, &addr2);
    c.put(&ctx_c, 3, &addr3);
    CHECK(c.find(&ctx_c, 3, &v) && v == &addr3);
    int hits = c.find(&ctx_a, 1, &v) + c.find(&ctx_b, 2, &v);
    CHECK(hits == 1);
    if (c.find(&ctx_a, 1, &v)) CHECK(v == &addr1);
    if (c.find(&ctx_b, 2, &v)) CHECK(v == &addr2);
  }
  std::printf(failures ? "ctx cache: %d failures\n" : "ctx cache ok%.0d\n", failures);
  return failures ? 1 : 0;
}
