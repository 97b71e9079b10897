// Serial stand-in for the handful of oneTBB facilities the reference CPU path
// uses. TBB is not installed in this image. Every construct runs in program
// order on the calling thread, which reproduces the reference's canonical
// single-thread output order (ascending cell ids in the critical lists).
// Test infrastructure only: used to compile the reference checker.
#pragma once
#include <algorithm>
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

template <typename T>
class enumerable_thread_specific {
 public:
  T& local() { return slot_; }
  T* begin() { return &slot_; }
  T* end() { return &slot_ + 1; }
  const T* begin() const { return &slot_; }
  const T* end() const { return &slot_ + 1; }

 private:
  T slot_{};
};

class global_control {
 public:
  enum parameter { max_allowed_parallelism, thread_stack_size };
  global_control(parameter, std::size_t) {}
};

}  // namespace tbb
