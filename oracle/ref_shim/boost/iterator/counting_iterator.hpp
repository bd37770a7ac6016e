// TEST INFRASTRUCTURE ONLY — a minimal stand-in for the Boost header of this name, written
// for this project: just the names the reference uses, with the same meaning.
#pragma once
#include <cstddef>
#include <iterator>

namespace boost {
template <class I>
class counting_iterator {
  public:
    using iterator_category = std::random_access_iterator_tag;
    using value_type = I;
    using difference_type = std::ptrdiff_t;
    using pointer = const I*;
    using reference = const I&;
    counting_iterator() = default;
    explicit counting_iterator(I v) : v_(v) {}
    reference operator*() const { return v_; }
    counting_iterator& operator++() { ++v_; return *this; }
    counting_iterator operator++(int) { auto t = *this; ++v_; return t; }
    counting_iterator& operator--() { --v_; return *this; }
    counting_iterator& operator+=(difference_type d) { v_ = I(v_ + d); return *this; }
    counting_iterator operator+(difference_type d) const { return counting_iterator(I(v_ + d)); }
    difference_type operator-(const counting_iterator& o) const { return difference_type(v_) - difference_type(o.v_); }
    bool operator==(const counting_iterator& o) const { return v_ == o.v_; }
    bool operator!=(const counting_iterator& o) const { return v_ != o.v_; }
    bool operator<(const counting_iterator& o) const { return v_ < o.v_; }

  private:
    I v_{};
};
template <class I>
counting_iterator<I> make_counting_iterator(I v) {
    return counting_iterator<I>(v);
}
}  // namespace boost
