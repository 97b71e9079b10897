// Parallel stand-in for the oneTBB facilities the reference CPU path uses
// (TBB is not installed in this image), for timing the reference on all host
// cores while keeping its single-thread output order. Test infrastructure
// only: used to compile the timed reference CPU baseline.
//
//  * parallel_for(blocked_range) splits the range into one contiguous chunk
//    per thread, in order; enumerable_thread_specific::local() called inside
//    chunk t returns slot t, and the slots iterate in chunk order, so
//    per-thread lists concatenate in ascending order exactly as one thread
//    would build them (cpu/critical_points.hxx:21-64).
//  * parallel_invoke runs its functions on separate threads (TBB may run them
//    concurrently, so the reference makes them independent).
//  * parallel_sort is the libstdc++ parallel sort; every comparator the
//    reference sorts with is a strict total order (unique ids break ties), so
//    the sorted result does not depend on the algorithm.
//  * global_control caps the threads of all three.
// local() outside such a chunk (from ATen's own parallel_for threads, which
// use their slot only as scratch) gets a slot per OS thread after the chunk
// slots.
#pragma once
#include <omp.h>

#include <algorithm>
#include <cstddef>
#include <deque>
#include <memory>
#include <mutex>
#include <parallel/algorithm>
#include <thread>
#include <tuple>
#include <utility>
#include <vector>

namespace tbb {

namespace shim {
inline int& max_threads() {
  static int n = 0;  // 0: no cap
  return n;
}
inline int threads() {
  int n = omp_get_max_threads();
  const int cap = max_threads();
  if (cap > 0 && cap < n) n = cap;
  return n < 1 ? 1 : n;
}
inline int& chunk_slot() {
  static thread_local int s = -1;  // chunk index of the running parallel_for body, -1 outside
  return s;
}
}  // namespace shim

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
  if (r.empty()) return;
  const long long b = (long long)r.begin(), e = (long long)r.end(), n = e - b;
  int T = shim::threads();
  if ((long long)T > n) T = (int)n;
#pragma omp parallel for num_threads(T) schedule(static, 1)
  for (int t = 0; t < T; ++t) {
    const long long lo = b + n * t / T, hi = b + n * (t + 1) / T;
    const int prev = shim::chunk_slot();
    shim::chunk_slot() = t;
    body(Range((decltype(r.begin()))lo, (decltype(r.begin()))hi, r.grainsize()));
    shim::chunk_slot() = prev;
  }
}

template <typename Index, typename Func>
void parallel_for(Index first, Index last, const Func& f) {
  const long long n = (long long)last - (long long)first;
  if (n <= 0) return;
  const int T = shim::threads();
#pragma omp parallel for num_threads(T) schedule(static)
  for (long long i = 0; i < n; ++i) f((Index)(first + i));
}

template <typename... Fs>
void parallel_invoke(Fs&&... fs) {
  if (shim::threads() <= 1) {
    (fs(), ...);
    return;
  }
  std::vector<std::thread> pool;
  auto launch = [&](auto& f) { pool.emplace_back([&f]() { f(); }); };
  (launch(fs), ...);
  for (auto& t : pool) t.join();
}

template <typename It, typename Cmp>
void parallel_sort(It first, It last, const Cmp& cmp) {
  const int T = shim::threads();
  if (T <= 1)
    std::sort(first, last, cmp);
  else
    __gnu_parallel::sort(first, last, cmp, __gnu_parallel::default_parallel_tag(T));
}

template <typename It>
void parallel_sort(It first, It last) {
  parallel_sort(first, last, std::less<typename std::iterator_traits<It>::value_type>());
}

template <typename T>
class enumerable_thread_specific {
 public:
  T& local() {
    std::lock_guard<std::mutex> g(m_);
    const int s = shim::chunk_slot();
    if (s >= 0) {
      if ((std::size_t)s >= chunk_.size()) chunk_.resize(s + 1);
      if (!chunk_[s]) chunk_[s].reset(new T());
      return *chunk_[s];
    }
    auto id = std::this_thread::get_id();
    for (std::size_t i = 0; i < ids_.size(); ++i)
      if (ids_[i] == id) return *other_[i];
    ids_.push_back(id);
    other_.emplace_back(new T());
    return *other_.back();
  }
  // chunk slots in chunk order, then the other threads' slots
  template <typename F>
  void for_each(F&& f) {
    for (auto& p : chunk_)
      if (p) f(*p);
    for (auto& p : other_) f(*p);
  }
  class iterator {
   public:
    iterator(std::vector<T*>* v, std::size_t i) : v_(v), i_(i) {}
    T& operator*() const { return *(*v_)[i_]; }
    T* operator->() const { return (*v_)[i_]; }
    iterator& operator++() {
      ++i_;
      return *this;
    }
    bool operator!=(const iterator& o) const { return i_ != o.i_; }
    bool operator==(const iterator& o) const { return i_ == o.i_; }

   private:
    std::vector<T*>* v_;
    std::size_t i_;
  };
  iterator begin() {
    snapshot();
    return iterator(&order_, 0);
  }
  iterator end() { return iterator(&order_, order_.size()); }
  iterator begin() const { return const_cast<enumerable_thread_specific*>(this)->begin(); }
  iterator end() const { return const_cast<enumerable_thread_specific*>(this)->end(); }

 private:
  void snapshot() {
    order_.clear();
    for (auto& p : chunk_)
      if (p) order_.push_back(p.get());
    for (auto& p : other_) order_.push_back(p.get());
  }
  std::mutex m_;
  std::vector<std::unique_ptr<T>> chunk_;
  std::vector<std::thread::id> ids_;
  std::vector<std::unique_ptr<T>> other_;
  std::vector<T*> order_;
};

class global_control {
 public:
  enum parameter { max_allowed_parallelism, thread_stack_size };
  global_control(parameter p, std::size_t v) : p_(p), prev_(shim::max_threads()) {
    if (p == max_allowed_parallelism) shim::max_threads() = (int)v;
  }
  ~global_control() {
    if (p_ == max_allowed_parallelism) shim::max_threads() = prev_;
  }

 private:
  parameter p_;
  int prev_;
};

}  // namespace tbb
