// Batch planning and device-memory admission of the serving loop: plain host
// code without CUDA, so that it can be unit-tested on a machine without a GPU.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace sc {

// Requests can share one launch when they code against the same dictionary
// with the same algorithm and options; L / eps / lambda may differ per
// request (per-signal vectors), the Lasso's L (its slab stride and path
// length) may not.
struct PlanKey {
  int64_t dict = 0;
  int algo = 0;       // 0 OMP, 1 Lasso
  int mode = 0;       // Lasso constraint mode
  int pos = 0;
  int L = 0;          // Lasso: clamped L; OMP: 0 (per signal)
  int path = 0;       // Lasso: length of the homotopy path (its iteration cap)
  int precision = 0;
  int refine = 0;
  bool operator==(const PlanKey& o) const {
    return dict == o.dict && algo == o.algo && mode == o.mode && pos == o.pos && L == o.L &&
           path == o.path && precision == o.precision && refine == o.refine;
  }
};

struct PlanItem {
  PlanKey key;
  int64_t n = 0;  // signals
};

// The next batch: the oldest queued request and every later request with the
// same key, in queue order, while the signal total stays within max_signals
// (the oldest request is always taken, whatever its size).  Returns queue
// positions.
inline std::vector<size_t> plan_batch(const std::vector<PlanItem>& queue, int64_t max_signals) {
  std::vector<size_t> take;
  if (queue.empty()) return take;
  const PlanKey k0 = queue.front().key;
  int64_t total = queue.front().n;
  take.push_back(0);
  for (size_t i = 1; i < queue.size(); ++i) {
    if (!(queue[i].key == k0)) continue;
    if (total + queue[i].n > max_signals) continue;
    total += queue[i].n;
    take.push_back(i);
  }
  return take;
}

// Device bytes a batch of n signals holds: X, D^T X, the per-signal slabs,
// the CSC output, per-signal parameters, the BF16 split of X (tc) and the
// small per-signal vectors of the pipeline.
inline size_t batch_bytes(int m, int Kp, int mp, int L, int64_t n, bool tc) {
  const size_t per = (size_t)m * 4 + (size_t)Kp * 4 + (size_t)L * 8 /* slabs */ +
                     (size_t)L * 8 /* CSC */ + 8 + 16 /* parameters */ +
                     (tc ? (size_t)mp * 4 : 0) + 64;
  return per * (size_t)std::max<int64_t>(n, 1) + ((size_t)1 << 20);
}

// What the stream-ordered pool should hold for the slots, given the largest
// batch workspace over the resident dictionaries (`need`): every slot's
// largest batch, within what the budget leaves after the dictionaries.
inline size_t pool_target(size_t need, size_t slots, size_t budget, size_t dict_bytes) {
  const size_t room = budget > dict_bytes ? budget - dict_bytes : 0;
  return std::min(need * slots, room);
}

// Admission: the resident dictionaries plus what every slot holds must stay
// within the budget.  A slot's workspaces only grow, so slot s holding
// `reserved[s]` bytes and needing `need` ends up holding the larger of both.
inline bool admit(size_t dict_bytes, const std::vector<size_t>& reserved, size_t s, size_t need,
                  size_t budget) {
  size_t total = dict_bytes;
  for (size_t i = 0; i < reserved.size(); ++i)
    total += i == s ? std::max(reserved[i], need) : reserved[i];
  return total <= budget;
}

// Latency percentile (nearest rank) of an unsorted sample, in its unit.
inline double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double r = q / 100.0 * (double)v.size();
  size_t k = (size_t)std::max(1.0, std::ceil(r));
  k = std::min(k, v.size());
  return v[k - 1];
}

}  // namespace sc
