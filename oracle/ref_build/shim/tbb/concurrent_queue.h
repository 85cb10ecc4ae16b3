// Minimal stand-in for oneTBB's concurrent_queue, written for building the
// reference ParaCOSM sources without TBB installed. It only provides what the
// reference calls (push, try_pop, empty, clear); a mutex guards a std::deque.
// Test infrastructure only: used to compile the reference as the checker.
#pragma once
#include <deque>
#include <mutex>
#include <utility>
namespace tbb {
template <typename T>
class concurrent_queue {
 public:
  void push(const T& v) { std::lock_guard<std::mutex> g(mu_); q_.push_back(v); }
  void push(T&& v) { std::lock_guard<std::mutex> g(mu_); q_.push_back(std::move(v)); }
  template <typename... A> void emplace(A&&... a) {
    std::lock_guard<std::mutex> g(mu_); q_.emplace_back(std::forward<A>(a)...);
  }
  bool try_pop(T& out) {
    std::lock_guard<std::mutex> g(mu_);
    if (q_.empty()) return false;
    out = std::move(q_.front()); q_.pop_front(); return true;
  }
  bool empty() const { std::lock_guard<std::mutex> g(mu_); return q_.empty(); }
  void clear() { std::lock_guard<std::mutex> g(mu_); q_.clear(); }
 private:
  mutable std::mutex mu_;
  std::deque<T> q_;
};
}  // namespace tbb
