// Unit test of the byte-budgeted LRU policy used by the server (host only).
#include <cstdio>
#include <string>
#include <vector>

#include "../../raptr_b200/csrc/lru_budget.h"

static int failures = 0;
#define CHECK(c)                                            \
  do {                                                      \
    if (!(c)) {                                             \
      std::printf("FAIL line %d: %s\n", __LINE__, #c);      \
      failures++;                                           \
    }                                                       \
  } while (0)

int main() {
  raptr::LruBudget<std::string> c(100);
  bool fits = false;
  CHECK(c.victims(100, &fits).empty() && fits);
  CHECK(c.victims(101, &fits).empty() && !fits);
  c.put("a", 40);
  c.put("b", 30);
  c.put("c", 20);
  CHECK(c.used() == 90);
  // room for 10 more without eviction
  CHECK(c.victims(10, &fits).empty() && fits);
  // 35 more: evict the least recently used first (a)
  std::vector<std::string> v = c.victims(35, &fits);
  CHECK(fits && v.size() == 1 && v[0] == "a");
  // touching a makes b the oldest, and b alone makes room
  c.touch("a");
  v = c.victims(35, &fits);
  CHECK(fits && v.size() == 1 && v[0] == "b");
  // pinned entries are never chosen
  c.pin("b");
  v = c.victims(35, &fits);
  CHECK(fits && v.size() == 2 && v[0] == "c" && v[1] == "a");
  c.pin("c");
  v = c.victims(35, &fits);
  CHECK(fits && v.size() == 1 && v[0] == "a");
  v = c.victims(75, &fits);  // even without a, 50 + 75 > 100
  CHECK(!fits && v.size() == 1 && v[0] == "a");
  c.unpin("b");
  c.unpin("c");
  CHECK(c.pins("b") == 0 && c.pins("c") == 0);
  // resize, erase
  c.put("c", 50);
  CHECK(c.used() == 120 && c.bytes("c") == 50);
  c.erase("a");
  CHECK(c.used() == 80 && !c.contains("a"));
  v = c.victims(0, &fits);
  CHECK(fits && v.empty());

  // admission: an oversized request fails without evicting idle entries
  raptr::LruBudget<std::string> d(100);
  d.put("idle", 60);
  std::vector<std::string> vic;
  CHECK(raptr::decide_admission(d, 120, false, &vic) == raptr::Admission::kFail && vic.empty());
  CHECK(d.contains("idle") && d.used() == 60);
  // ... and waits while other work runs
  CHECK(raptr::decide_admission(d, 120, true, &vic) == raptr::Admission::kWait && vic.empty());
  // a request that fits after evicting the idle entry is admitted
  CHECK(raptr::decide_admission(d, 70, false, &vic) == raptr::Admission::kAdmit && vic.size() == 1 &&
        vic[0] == "idle");
  // one that fits as is evicts nothing
  CHECK(raptr::decide_admission(d, 40, false, &vic) == raptr::Admission::kAdmit && vic.empty());
  // a pinned entry in the way: wait if work runs, else fail
  d.pin("idle");
  CHECK(raptr::decide_admission(d, 70, true, &vic) == raptr::Admission::kWait);
  CHECK(raptr::decide_admission(d, 70, false, &vic) == raptr::Admission::kFail && vic.empty());
  std::printf("failures %d\n", failures);
  return failures == 0 ? 0 : 1;
}
