// TEST INFRASTRUCTURE ONLY — a minimal stand-in for the Boost header of this name, written
// for this project: just the names the reference uses, with the same meaning.
// flat_set: a sorted vector of unique keys.
#pragma once
#include <algorithm>
#include <functional>
#include <initializer_list>
#include <utility>
#include <vector>

namespace boost {
namespace container {
template <class T, class Cmp = std::less<T>>
class flat_set {
    std::vector<T> v_;
    Cmp c_{};

  public:
    using value_type = T;
    using key_type = T;
    using size_type = std::size_t;
    using iterator = typename std::vector<T>::const_iterator;
    using const_iterator = typename std::vector<T>::const_iterator;
    using const_reverse_iterator = typename std::vector<T>::const_reverse_iterator;
    using reference = const T&;
    using const_reference = const T&;
    flat_set() = default;
    flat_set(std::initializer_list<T> il) { for (const auto& x : il) insert(x); }
    template <class It>
    flat_set(It b, It e) { for (; b != e; ++b) insert(*b); }
    const_iterator begin() const { return v_.begin(); }
    const_iterator end() const { return v_.end(); }
    const_iterator cbegin() const { return v_.cbegin(); }
    const_iterator cend() const { return v_.cend(); }
    const_reverse_iterator rbegin() const { return v_.rbegin(); }
    const_reverse_iterator rend() const { return v_.rend(); }
    size_type size() const { return v_.size(); }
    bool empty() const { return v_.empty(); }
    void clear() { v_.clear(); }
    void reserve(size_type n) { v_.reserve(n); }
    const T& operator[](size_type i) const { return v_[i]; }
    const T* data() const { return v_.data(); }
    const_iterator lower_bound(const T& x) const { return std::lower_bound(v_.begin(), v_.end(), x, c_); }
    const_iterator find(const T& x) const {
        auto it = lower_bound(x);
        return (it != v_.end() && !c_(x, *it)) ? it : v_.end();
    }
    size_type count(const T& x) const { return find(x) != v_.end() ? 1 : 0; }
    bool contains(const T& x) const { return find(x) != v_.end(); }
    std::pair<const_iterator, bool> insert(const T& x) {
        auto it = std::lower_bound(v_.begin(), v_.end(), x, c_);
        if (it != v_.end() && !c_(x, *it)) return {it, false};
        auto p = v_.insert(it, x);
        return {p, true};
    }
    template <class It>
    void insert(It b, It e) { for (; b != e; ++b) insert(*b); }
    template <class... A>
    std::pair<const_iterator, bool> emplace(A&&... a) { return insert(T(std::forward<A>(a)...)); }
    size_type erase(const T& x) {
        auto it = find(x);
        if (it == v_.end()) return 0;
        v_.erase(it);
        return 1;
    }
    const_iterator erase(const_iterator it) { return v_.erase(it); }
    bool operator==(const flat_set& o) const { return v_ == o.v_; }
    bool operator!=(const flat_set& o) const { return v_ != o.v_; }
    bool operator<(const flat_set& o) const { return v_ < o.v_; }
};
}  // namespace container
}  // namespace boost
