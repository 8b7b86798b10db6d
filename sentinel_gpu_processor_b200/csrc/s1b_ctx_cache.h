// Per-context cache of one device address (host code, no CUDA types).
//
// The device address of a module symbol belongs to a CUDA context, not to a
// device: a context made current by a host application (a non-primary
// driver context), or a primary context rebuilt after cudaDeviceReset, can
// place the module at another address.  Entries are therefore keyed on the
// context handle together with the context's unique id (cuCtxGetId), since a
// destroyed context's handle can be handed out again for a new one.
#ifndef S1B_CTX_CACHE_H
#define S1B_CTX_CACHE_H

#include <stdint.h>

#include <mutex>

template <int N>
class ContextKeyedCache {
 public:
  // True, with *value set, when (ctx, id) holds an entry.
  bool find(const void *ctx, uint64_t id, void **value) {
    std::lock_guard<std::mutex> lock(mu_);
    for (int i = 0; i < N; ++i)
      if (e_[i].used && e_[i].ctx == ctx && e_[i].id == id) {
        *value = e_[i].value;
        return true;
      }
    return false;
  }

  // Store value for (ctx, id).  An entry with the same handle (a context
  // that was destroyed, its handle reused) is replaced; otherwise a free
  // slot is taken, or the oldest entry is evicted.
  void put(const void *ctx, uint64_t id, void *value) {
    std::lock_guard<std::mutex> lock(mu_);
    int slot = -1;
    for (int i = 0; i < N && slot < 0; ++i)
      if (e_[i].used && e_[i].ctx == ctx) slot = i;
    for (int i = 0; i < N && slot < 0; ++i)
      if (!e_[i].used) slot = i;
    if (slot < 0) {
      slot = next_;
      next_ = (next_ + 1) % N;
    }
    e_[slot] = Entry{ctx, id, value, true};
  }

 private:
  struct Entry {
    const void *ctx;
    uint64_t id;
    void *value;
    bool used;
  };
  Entry e_[N] = {};
  int next_ = 0;
  std::mutex mu_;
};

#endif
