// TEST INFRASTRUCTURE ONLY — a minimal stand-in for the Boost header of this name, written
// for this project: just the names the reference uses, with the same meaning.
// Component ids numbered in order of first discovery over vertices 0..n-1; returns the count.
#pragma once
#include <cstddef>
#include <vector>

#include "adjacency_list.hpp"

namespace boost {
template <class O, class V, class D, class VP, class EP, class Out>
std::size_t connected_components(const adjacency_list<O, V, D, VP, EP>& g, Out comp) {
    const std::size_t n = g.adj.size();
    std::vector<char> seen(n, 0);
    std::vector<std::size_t> stack;
    std::size_t c = 0;
    for (std::size_t s = 0; s < n; ++s) {
        if (seen[s]) continue;
        seen[s] = 1;
        stack.push_back(s);
        while (!stack.empty()) {
            std::size_t u = stack.back();
            stack.pop_back();
            comp[u] = c;
            for (std::size_t w : g.adj[u])
                if (!seen[w]) {
                    seen[w] = 1;
                    stack.push_back(w);
                }
        }
        ++c;
    }
    return c;
}
}  // namespace boost
