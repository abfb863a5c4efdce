// Unit checks of the serving loop's batch planning and admission rules
// (serve_plan.h), compiled and run by tests/test_serve_plan.py on the CPU.
#include <cstdio>
#include <cstdlib>

#include "serve_plan.h"

using namespace sc;

static int failures = 0;
#define CHECK(c)                                              \
  do {                                                        \
    if (!(c)) {                                               \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
      ++failures;                                             \
    }                                                         \
  } while (0)

static PlanKey omp(int64_t dict) {
  PlanKey k;
  k.dict = dict;
  return k;
}
static PlanKey lasso(int64_t dict, int mode, int L) {
  PlanKey k;
  k.dict = dict;
  k.algo = 1;
  k.mode = mode;
  k.L = L;
  k.path = 4 * L;
  return k;
}

int main() {
  // empty queue: nothing to do
  CHECK(plan_batch({}, 100).empty());
  // the oldest request decides the key; same-key requests join in order
  {
    std::vector<PlanItem> q = {{omp(1), 10}, {omp(2), 5}, {omp(1), 20}, {lasso(1, 2, 64), 7},
                               {omp(1), 30}};
    auto t = plan_batch(q, 1000);
    CHECK(t.size() == 3 && t[0] == 0 && t[1] == 2 && t[2] == 4);
  }
  // the signal cap skips requests that would overflow it, keeps later ones
  {
    std::vector<PlanItem> q = {{omp(1), 60}, {omp(1), 50}, {omp(1), 40}};
    auto t = plan_batch(q, 100);
    CHECK(t.size() == 2 && t[0] == 0 && t[1] == 2);
  }
  // the oldest request is taken even when it alone exceeds the cap
  {
    std::vector<PlanItem> q = {{omp(1), 500}, {omp(1), 1}};
    auto t = plan_batch(q, 100);
    CHECK(t.size() == 1 && t[0] == 0);
  }
  // Lasso requests merge only with equal mode, pos, L, path and precision
  {
    PlanKey a = lasso(3, 2, 64), b = lasso(3, 2, 64), c = lasso(3, 1, 64), d = lasso(3, 2, 32);
    PlanKey e = lasso(3, 2, 64);
    e.precision = 1;
    PlanKey f = lasso(3, 2, 64);
    f.path = 1024;
    CHECK(a == b);
    CHECK(!(a == c) && !(a == d) && !(a == e) && !(a == f));
    std::vector<PlanItem> q = {{a, 1}, {c, 1}, {d, 1}, {b, 1}, {e, 1}};
    auto t = plan_batch(q, 1000);
    CHECK(t.size() == 2 && t[0] == 0 && t[1] == 3);
  }
  // batch bytes grow with the signals and include the BF16 split in tc mode
  CHECK(batch_bytes(64, 256, 64, 10, 1000, false) < batch_bytes(64, 256, 64, 10, 2000, false));
  CHECK(batch_bytes(64, 256, 64, 10, 1000, false) < batch_bytes(64, 256, 64, 10, 1000, true));
  // admission: dictionaries + every slot's holdings (the own slot at its
  // high-water mark) within the budget
  {
    std::vector<size_t> res = {100, 200, 0};
    CHECK(admit(50, res, 2, 650, 1000));   // 50 + 100 + 200 + 650 = 1000
    CHECK(!admit(50, res, 2, 651, 1000));
    CHECK(admit(50, res, 0, 80, 1000));    // own slot keeps its 100
    CHECK(!admit(50, res, 0, 751, 1000));  // 50 + 751 + 200 > 1000
  }
  // nearest-rank percentiles
  {
    std::vector<double> v;
    for (int i = 100; i >= 1; --i) v.push_back(i);
    CHECK(percentile(v, 50) == 50);
    CHECK(percentile(v, 99) == 99);
    CHECK(percentile(v, 100) == 100);
    CHECK(percentile({}, 99) == 0);
    CHECK(percentile({7}, 99) == 7);
  }
  if (failures) return 1;
  // the pool warm-up: every slot's largest batch, within the budget's room
  CHECK(pool_target(100, 3, 1000, 200) == 300);
  CHECK(pool_target(400, 3, 1000, 200) == 800);
  CHECK(pool_target(400, 3, 100, 200) == 0);
  std::printf("serve_plan: all checks passed\n");
  return 0;
}
