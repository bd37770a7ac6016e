// TEST INFRASTRUCTURE ONLY — a minimal stand-in for the Boost header of this name, written
// for this project: just the names the reference uses, with the same meaning.
#pragma once
#include <cstddef>
#include <iterator>
#include <type_traits>
#include <utility>

namespace boost {
template <class F, class It>
class transform_iterator {
  public:
    using iterator_category = std::input_iterator_tag;
    using value_type = std::decay_t<decltype(std::declval<const F&>()(*std::declval<It>()))>;
    using difference_type = std::ptrdiff_t;
    using pointer = void;
    using reference = value_type;
    transform_iterator() = default;
    transform_iterator(It it, F f) : it_(it), f_(f) {}
    reference operator*() const { return f_(*it_); }
    transform_iterator& operator++() { ++it_; return *this; }
    transform_iterator operator++(int) { auto t = *this; ++it_; return t; }
    difference_type operator-(const transform_iterator& o) const { return it_ - o.it_; }
    bool operator==(const transform_iterator& o) const { return it_ == o.it_; }
    bool operator!=(const transform_iterator& o) const { return it_ != o.it_; }

  private:
    It it_{};
    F f_{};
};
template <class It, class F>
transform_iterator<F, It> make_transform_iterator(It it, F f) {
    return transform_iterator<F, It>(it, f);
}
}  // namespace boost
