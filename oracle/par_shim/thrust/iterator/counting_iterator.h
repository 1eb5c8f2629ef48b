// TEST INFRASTRUCTURE ONLY -- never linked into the product.
//
// Two stand-ins that let the reference's std::par build (par/ppc.cxx) compile with g++ and
// run on every host core, as the CPU baseline: a counting iterator in place of thrust's, and
// for_each_n with std::execution::par_unseq over it as an OpenMP loop (the libstdc++ here
// has no TBB back end, so the standard one would run serially).  Build recipe:
// oracle/Makefile, target _ref/ppc_par.
#pragma once
#include <cstddef>
#include <execution>
#include <iterator>

namespace thrust {

template <class T>
struct counting_iterator {
  using iterator_category = std::random_access_iterator_tag;
  using value_type = T;
  using difference_type = std::ptrdiff_t;
  using pointer = const T*;
  using reference = T;
  T v;
  explicit counting_iterator(T x = 0) : v(x) {}
  T operator*() const { return v; }
  T operator[](difference_type k) const { return (T)(v + k); }
  counting_iterator& operator++() { ++v; return *this; }
  counting_iterator operator++(int) { counting_iterator t = *this; ++v; return t; }
  counting_iterator& operator+=(difference_type k) { v = (T)(v + k); return *this; }
  counting_iterator operator+(difference_type k) const { return counting_iterator((T)(v + k)); }
  difference_type operator-(const counting_iterator& o) const { return (difference_type)v - (difference_type)o.v; }
  bool operator==(const counting_iterator& o) const { return v == o.v; }
  bool operator!=(const counting_iterator& o) const { return v != o.v; }
};

}  // namespace thrust

namespace std {

// more specialised than the standard overload, so par_unseq over a counting iterator lands here
template <class T, class Size, class F>
thrust::counting_iterator<T> for_each_n(const execution::parallel_unsequenced_policy&,
                                        thrust::counting_iterator<T> first, Size n, F f) {
  const long long m = (long long)n;
#pragma omp parallel for schedule(dynamic, 16)
  for (long long i = 0; i < m; i++) f((T)(first.v + i));
  return thrust::counting_iterator<T>((T)(first.v + m));
}

}  // namespace std
