// Boost.Heap fibonacci_heap API shim; see detail_indexed_heap.hpp.
#pragma once
#include "detail_indexed_heap.hpp"
namespace boost {
namespace heap {
template <class T, class... Opts>
class fibonacci_heap
    : public shim_detail::indexed_heap<T, typename shim_detail::pick_compare<T, Opts...>::type> {};
}  // namespace heap
}  // namespace boost
