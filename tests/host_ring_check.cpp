// Randomised check of the streaming service's host ring (host_ring.h):
// ranges held at once never overlap and stay inside the ring, releases in any
// order free the space, and a range of up to half the ring always fits once
// the ring is empty.  Built and run by tests/test_host_ring.py.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <thread>
#include <vector>

#include "host_ring.h"

using rodv::HostRing;

struct Held {
  uint64_t pos, n;
};

static bool overlaps(const Held& a, const Held& b) {
  return a.pos < b.pos + b.n && b.pos < a.pos + a.n;
}

int main() {
  const uint64_t cap = 1000;
  HostRing ring(cap);
  std::mt19937_64 rng(7);
  std::vector<Held> held;
  for (int it = 0; it < 20000; ++it) {
    const bool take = held.empty() || (rng() % 3 != 0 && held.size() < 12);
    if (take) {
      const uint64_t n = 1 + rng() % (cap / 2);
      // acquire blocks when the ring is full: free the oldest ranges (in a
      // random order) until the range fits, as the service's worker would
      std::atomic<uint64_t> got{HostRing::kNone};
      std::thread t([&] { got = ring.acquire(n); });
      while (true) {
        std::this_thread::yield();
        if (got.load() != HostRing::kNone) break;
        if (held.empty()) continue;  // an empty ring must take it
        const size_t k = rng() % held.size();
        ring.release(held[k].pos);
        held.erase(held.begin() + (long)k);
      }
      t.join();
      const uint64_t pos = got.load();
      const Held h{pos, n};
      if (pos + n > cap) {
        std::printf("FAIL range [%llu, %llu) outside the ring\n", (unsigned long long)pos,
                    (unsigned long long)(pos + n));
        return 1;
      }
      for (const Held& o : held)
        if (overlaps(o, h)) {
          std::printf("FAIL overlap\n");
          return 1;
        }
      held.push_back(h);
    } else {
      const size_t k = rng() % held.size();
      ring.release(held[k].pos);
      held.erase(held.begin() + (long)k);
    }
    if (ring.held() < held.size()) {
      std::printf("FAIL ring holds fewer ranges than were handed out\n");
      return 1;
    }
  }
  for (const Held& h : held) ring.release(h.pos);
  if (ring.held() != 0) {
    std::printf("FAIL ranges left after every release\n");
    return 1;
  }
  ring.stop();
  if (ring.acquire(10) != HostRing::kNone) {
    std::printf("FAIL acquire after stop\n");
    return 1;
  }
  std::printf("OK\n");
  return 0;
}
