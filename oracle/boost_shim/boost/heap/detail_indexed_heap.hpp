// Boost.Heap API shim (test infrastructure for the oracle only).
//
// The reference's CPU solvers (PrunedDP++, D-PrunedDP++, TrimCDP-multi-core-CPU,
// D-TrimCDP-multi-core-CPU) include <boost/heap/fibonacci_heap.hpp> and
// <boost/heap/pairing_heap.hpp> from Boost 1.85.0 (reference README.md:12).  Boost
// is not installed in this image, so this header restates the part of the
// published Boost.Heap interface those solvers use: a mutable priority queue whose
// push() returns a stable handle, with top(), pop(), update(handle, value),
// size() and empty().  Like Boost.Heap it is a max-heap with respect to the
// comparator (default std::less<T>; boost::heap::compare<C> overrides it), so
// top() is the element x for which cmp(x, y) is false for every other y.
//
// Implementation: an array-backed binary heap of pointers to heap-allocated nodes;
// each node records its current array position so that update() can sift in either
// direction.  Boost uses a Fibonacci / pairing heap; only the ORDER of equal keys
// can differ, which changes which of several equal-cost trees a solver returns,
// never a cost.
#pragma once
#include <cstddef>
#include <functional>
#include <utility>
#include <vector>

namespace boost {
namespace heap {

template <class C>
struct compare {
  typedef C type;
};

namespace shim_detail {

template <class T, class... Opts>
struct pick_compare {
  typedef std::less<T> type;
};
template <class T, class C, class... Rest>
struct pick_compare<T, boost::heap::compare<C>, Rest...> {
  typedef C type;
};
template <class T, class Other, class... Rest>
struct pick_compare<T, Other, Rest...> {
  typedef typename pick_compare<T, Rest...>::type type;
};

template <class T, class Cmp>
class indexed_heap {
  struct node {
    T value;
    std::size_t pos;
  };

 public:
  typedef T value_type;
  typedef std::size_t size_type;

  class handle_type {
   public:
    handle_type() : n_(nullptr) {}
    explicit handle_type(node* n) : n_(n) {}
    T& operator*() const { return n_->value; }
    node* n_;
  };

  indexed_heap() = default;
  indexed_heap(const indexed_heap&) = delete;
  indexed_heap& operator=(const indexed_heap&) = delete;
  ~indexed_heap() { clear(); }

  handle_type push(const T& v) {
    node* n = new node{v, a_.size()};
    a_.push_back(n);
    up(n->pos);
    return handle_type(n);
  }
  const T& top() const { return a_[0]->value; }
  void pop() {
    node* n = a_[0];
    node* last = a_.back();
    a_.pop_back();
    if (!a_.empty()) {
      a_[0] = last;
      last->pos = 0;
      down(0);
    }
    delete n;
  }
  void update(handle_type h, const T& v) {
    h.n_->value = v;
    up(h.n_->pos);
    down(h.n_->pos);
  }
  void update(handle_type h) {
    up(h.n_->pos);
    down(h.n_->pos);
  }
  void increase(handle_type h, const T& v) { update(h, v); }
  void decrease(handle_type h, const T& v) { update(h, v); }
  size_type size() const { return a_.size(); }
  bool empty() const { return a_.empty(); }
  void clear() {
    for (node* n : a_) delete n;
    a_.clear();
  }

 private:
  // max-heap w.r.t. cmp_: parent is never "less" than a child.
  bool less_(std::size_t i, std::size_t j) const { return cmp_(a_[i]->value, a_[j]->value); }
  void swap_(std::size_t i, std::size_t j) {
    std::swap(a_[i], a_[j]);
    a_[i]->pos = i;
    a_[j]->pos = j;
  }
  void up(std::size_t i) {
    while (i > 0) {
      std::size_t p = (i - 1) / 2;
      if (!less_(p, i)) break;
      swap_(p, i);
      i = p;
    }
  }
  void down(std::size_t i) {
    const std::size_t n = a_.size();
    for (;;) {
      std::size_t l = 2 * i + 1, r = l + 1, m = i;
      if (l < n && less_(m, l)) m = l;
      if (r < n && less_(m, r)) m = r;
      if (m == i) break;
      swap_(i, m);
      i = m;
    }
  }

  std::vector<node*> a_;
  Cmp cmp_;
};

}  // namespace shim_detail
}  // namespace heap
}  // namespace boost
