// TEST INFRASTRUCTURE ONLY — a minimal stand-in for the Boost header of this name, written
// for this project: just the names the reference uses, with the same meaning.
#pragma once
#include <utility>

namespace boost {
namespace placeholders {
struct arg1_t {};
static constexpr arg1_t _1{};
}  // namespace placeholders

// bind(f, _1): a copyable, default-constructible unary forwarder.
template <class F>
struct unary_binder {
    F f{};
    template <class A>
    auto operator()(A&& a) const -> decltype(f(std::forward<A>(a))) {
        return f(std::forward<A>(a));
    }
};
template <class F>
unary_binder<F> bind(F f, placeholders::arg1_t) {
    return unary_binder<F>{f};
}
}  // namespace boost
