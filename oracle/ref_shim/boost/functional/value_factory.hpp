// TEST INFRASTRUCTURE ONLY — a minimal stand-in for the Boost header of this name, written
// for this project: just the names the reference uses, with the same meaning.
#pragma once
#include <utility>

namespace boost {
template <class T>
struct value_factory {
    using result_type = T;
    template <class... A>
    T operator()(A&&... a) const {
        return T(std::forward<A>(a)...);
    }
};
}  // namespace boost
