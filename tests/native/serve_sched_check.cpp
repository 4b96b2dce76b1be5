// Property check of the serving loop's slot ring and wave policy
// (xmp_b200/csrc/serve_sched.h), compiled with the host compiler alone.
// Exit status 0 and "ok" on stdout when every property holds.
#include "serve_sched.h"
#include <cstdio>
#include <deque>
#include <random>
#include <vector>

using xmpb::serve::SlotRing;
using xmpb::serve::WavePolicy;

#define CHECK(c)                                                        \
  do {                                                                  \
    if (!(c)) {                                                         \
      std::printf("FAIL line %d: %s\n", __LINE__, #c);                  \
      return 1;                                                         \
    }                                                                   \
  } while (0)

struct Live {
  uint32_t first, n, taken;
};

int main() {
  // fixed cases
  {
    SlotRing r(1000, 128);  // capacity rounds down to 896
    CHECK(r.capacity() == 896);
    uint32_t f, t;
    CHECK(!r.alloc(0, &f, &t));
    CHECK(!r.alloc(897, &f, &t));
    CHECK(r.alloc(1, &f, &t) && f == 0 && t == 128);
    CHECK(r.alloc(700, &f, &t) && f == 128 && t == 768);
    CHECK(r.used() == 896 && r.largest_free() == 0);
    CHECK(!r.alloc(1, &f, &t));
    r.release(128);
    CHECK(r.largest_free() == 128);
    CHECK(r.alloc(100, &f, &t) && f == 0 && t == 128);  // the freed head, wrapping
    r.release(768);
    r.release(128);
    CHECK(r.used() == 0 && r.largest_free() == 896);
    CHECK(r.alloc(896, &f, &t) && f == 0);  // empty ring restarts at slot 0
  }
  // random alloc / in-order release: live ranges never overlap and stay in bounds
  std::mt19937 rng(12345);
  for (int trial = 0; trial < 200; trial++) {
    const uint32_t gran = 1u << (rng() % 8);
    const uint32_t cap = gran * (1 + rng() % 64);
    SlotRing r(cap, gran);
    std::deque<Live> live;
    std::vector<int> owner(cap, -1);
    for (int step = 0; step < 2000; step++) {
      if (!live.empty() && (rng() % 3 == 0)) {
        Live l = live.front();
        live.pop_front();
        for (uint32_t s = l.first; s < l.first + l.n; s++) owner[s] = -1;
        r.release(l.taken);
        continue;
      }
      const uint32_t n = 1 + rng() % (cap + gran);
      const uint32_t lf = r.largest_free();
      uint32_t f = 0, t = 0;
      bool ok = r.alloc(n, &f, &t);
      // alloc succeeds exactly when n (rounded to the granule) fits the largest free run
      uint32_t rounded = (n + gran - 1) / gran * gran;
      CHECK(ok == (rounded <= lf));
      if (!ok) continue;
      CHECK(f % gran == 0);
      CHECK(f + rounded <= cap);
      CHECK(t >= rounded);
      for (uint32_t s = f; s < f + rounded; s++) {
        CHECK(owner[s] == -1);
        owner[s] = step;
      }
      CHECK(r.used() <= cap);
      live.push_back(Live{f, rounded, t});
    }
    while (!live.empty()) {
      r.release(live.front().taken);
      live.pop_front();
    }
    CHECK(r.used() == 0);
  }
  // wave policy
  {
    WavePolicy p;
    p.max_wave_ops = 100;
    CHECK(!p.should_launch(0, 4));   // nothing pending
    CHECK(p.should_launch(1, 1));    // an idle stream: at once
    CHECK(!p.should_launch(500, 0)); // every stream busy: keep merging
  }
  std::printf("ok\n");
  return 0;
}
