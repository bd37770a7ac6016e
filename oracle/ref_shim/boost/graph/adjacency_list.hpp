// TEST INFRASTRUCTURE ONLY — a minimal stand-in for the Boost header of this name, written
// for this project: just the names the reference uses, with the same meaning.
// An undirected graph over vertices 0..n-1 (n grows with the largest vertex added).
#pragma once
#include <cstddef>
#include <utility>
#include <vector>

namespace boost {
struct vecS {};
struct undirectedS {};
struct vertex_index_t {};
struct edge_index_t {};
template <class Tag, class T>
struct property {};

template <class OutS = vecS, class VertS = vecS, class Dir = undirectedS, class VP = void, class EP = void>
class adjacency_list {
  public:
    std::vector<std::vector<std::size_t>> adj;
    void touch(std::size_t v) {
        if (v >= adj.size()) adj.resize(v + 1);
    }
};

template <class O, class V, class D, class VP, class EP>
std::pair<int, bool> add_edge(std::size_t u, std::size_t v, adjacency_list<O, V, D, VP, EP>& g) {
    g.touch(u);
    g.touch(v);
    g.adj[u].push_back(v);
    g.adj[v].push_back(u);
    return {0, true};
}

template <class O, class V, class D, class VP, class EP>
std::size_t num_vertices(const adjacency_list<O, V, D, VP, EP>& g) {
    return g.adj.size();
}
}  // namespace boost
