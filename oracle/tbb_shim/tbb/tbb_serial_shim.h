// Stand-in for the handful of oneTBB facilities the reference CPU path uses. TBB is not installed in this image. Every construct runs in program
// order on the calling thread, which reproduces the reference's canonical
// single-thread output order (ascending cell ids in the critical lists).
// Test infrastructure only: used to compile the reference checker.
#pragma once
#include <algorithm>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>
#include <cstddef>
#include <utility>

namespace tbb {

template <typename Value>
class blocked_range {
 public:
  blocked_range(Value b, Value e, std::size_t grain = 1) : b_(b), e_(e), grain_(grain) {}
  Value begin() const { return b_; }
  Value end() const { return e_; }
  std::size_t grainsize() const { return grain_; }
  bool empty() const { return !(b_ < e_); }

 private:
  Value b_, e_;
  std::size_t grain_;
};

template <typename Range, typename Body>
void parallel_for(const Range& r, const Body& body) {
  if (!r.empty()) body(r);
}

template <typename Index, typename Func>
void parallel_for(Index first, Index last, const Func& f) {
  for (Index i = first; i < last; ++i) f(i);
}

template <typename... Fs>
void parallel_invoke(Fs&&... fs) {
  (fs(), ...);
}

template <typename It, typename Cmp>
void parallel_sort(It first, It last, const Cmp& cmp) {
  std::sort(first, last, cmp);
}

template <typename It>
void parallel_sort(It first, It last) {
  std::sort(first, last);
}

// One slot per calling thread. Serial TBB constructs only ever touch the
// first slot (so the reference's per-thread lists concatenate in program
// order), while the reference also calls local() from ATen's parallel_for,
// which does run on several OpenMP threads.
template <typename T>
class enumerable_thread_specific {
 public:
  T& local() {
    std::lock_guard<std::mutex> g(m_);
    auto id = std::this_thread::get_id();
    for (std::size_t i = 0; i < ids_.size(); ++i)
      if (ids_[i] == id) return slots_[i];
    ids_.push_back(id);
    slots_.emplace_back();
    return slots_.back();
  }
  typename std::deque<T>::iterator begin() { return slots_.begin(); }
  typename std::deque<T>::iterator end() { return slots_.end(); }
  typename std::deque<T>::const_iterator begin() const { return slots_.begin(); }
  typename std::deque<T>::const_iterator end() const { return slots_.end(); }

 private:
  std::mutex m_;
  std::vector<std::thread::id> ids_;
  std::deque<T> slots_;
};

class global_control {
 public:
  enum parameter { max_allowed_parallelism, thread_stack_size };
  global_control(parameter, std::size_t) {}
};

}  // namespace tbb
