// Byte-budgeted LRU bookkeeping for cached system matrices (host only, no
// CUDA): which entries to evict so that a new allocation fits the budget.
// Entries in use (pinned) are never chosen.  Plain C++ so that the policy is
// tested on its own.
#pragma once

#include <cstdint>
#include <list>
#include <map>
#include <vector>

namespace raptr {

template <class Key>
class LruBudget {
 public:
  explicit LruBudget(int64_t budget) : budget_(budget) {}

  int64_t budget() const { return budget_; }
  int64_t used() const { return used_; }
  bool contains(const Key& k) const { return index_.count(k) != 0; }
  int64_t bytes(const Key& k) const {
    auto it = index_.find(k);
    return it == index_.end() ? 0 : it->second->bytes;
  }

  // Records (or resizes) an entry and marks it most recently used.
  void put(const Key& k, int64_t bytes) {
    auto it = index_.find(k);
    if (it != index_.end()) {
      used_ += bytes - it->second->bytes;
      it->second->bytes = bytes;
      order_.splice(order_.end(), order_, it->second);
      return;
    }
    order_.push_back(Node{k, bytes, 0});
    index_[k] = std::prev(order_.end());
    used_ += bytes;
  }

  void touch(const Key& k) {
    auto it = index_.find(k);
    if (it != index_.end()) order_.splice(order_.end(), order_, it->second);
  }

  void pin(const Key& k) {
    auto it = index_.find(k);
    if (it != index_.end()) it->second->pins++;
  }
  void unpin(const Key& k) {
    auto it = index_.find(k);
    if (it != index_.end() && it->second->pins > 0) it->second->pins--;
  }
  int pins(const Key& k) const {
    auto it = index_.find(k);
    return it == index_.end() ? 0 : it->second->pins;
  }

  void erase(const Key& k) {
    auto it = index_.find(k);
    if (it == index_.end()) return;
    used_ -= it->second->bytes;
    order_.erase(it->second);
    index_.erase(it);
  }

  // Least recently used unpinned entries whose removal brings used() +
  // extra within the budget, oldest first; empty when nothing needs to go.
  // *fits tells whether the budget can be met at all.
  std::vector<Key> victims(int64_t extra, bool* fits) const {
    std::vector<Key> out;
    int64_t u = used_;
    for (auto it = order_.begin(); it != order_.end() && u + extra > budget_; ++it) {
      if (it->pins > 0) continue;
      out.push_back(it->key);
      u -= it->bytes;
    }
    if (fits) *fits = u + extra <= budget_;
    return out;
  }

 private:
  struct Node {
    Key key;
    int64_t bytes;
    int pins;
  };
  int64_t budget_;
  int64_t used_ = 0;
  std::list<Node> order_;  // front = least recently used
  std::map<Key, typename std::list<Node>::iterator> index_;
};

// Admission of a request whose matrix is not resident: `need` bytes (the
// matrix estimate plus the request's state) on top of what is in use.
//   kAdmit: fits after evicting `victims` (possibly none);
//   kWait:  cannot fit while other work holds memory -- retry later;
//   kFail:  cannot fit even with every unpinned entry evicted and nothing
//           else running -- fail it, and evict nothing.
enum class Admission { kAdmit, kWait, kFail };

template <class Key>
Admission decide_admission(const LruBudget<Key>& cache, int64_t need, bool running, std::vector<Key>* victims) {
  bool fits = false;
  std::vector<Key> v = cache.victims(need, &fits);
  victims->clear();
  if (fits) {
    *victims = std::move(v);
    return Admission::kAdmit;
  }
  return running ? Admission::kWait : Admission::kFail;
}

}  // namespace raptr
