// rcm.cpp -- reverse Cuthill-McKee ordering and symmetric permutation.
//
// Ordering rule (restated by the oracle in oracle/sell_rcm_oracle.py, bit-exact):
//   * graph = off-diagonal pattern of the (structurally symmetric) CSR; degree = its size;
//   * components are taken in order of their lowest unvisited node index;
//   * start node: the component's minimum-(degree, index) node, then George-Liu
//     pseudo-peripheral search (move to the minimum-(degree, index) node of the last BFS
//     level while the eccentricity grows);
//   * Cuthill-McKee BFS appends each node's unvisited neighbours sorted by (degree, index);
//   * the concatenated order is reversed.  perm[new] = old.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.hpp"

namespace xplus {

namespace {
struct Graph {
    int n;
    std::vector<int> ptr, adj, deg;
};

Graph make_graph(int n, const int* row_ptr, const int* col_idx) {
    Graph G;
    G.n = n;
    G.ptr.assign(static_cast<size_t>(n) + 1, 0);
    G.deg.assign(static_cast<size_t>(n), 0);
    for (int i = 0; i < n; ++i) {
        int d = 0;
        for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) d += (col_idx[k] != i);
        G.deg[static_cast<size_t>(i)] = d;
        G.ptr[static_cast<size_t>(i) + 1] = G.ptr[static_cast<size_t>(i)] + d;
    }
    G.adj.resize(static_cast<size_t>(G.ptr[static_cast<size_t>(n)]));
    for (int i = 0; i < n; ++i) {
        int w = G.ptr[static_cast<size_t>(i)];
        for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
            if (col_idx[k] != i) G.adj[static_cast<size_t>(w++)] = col_idx[k];
    }
    return G;
}

// BFS level structure from root over nodes with mark == 0 (mark is restored on exit).
// Returns the number of levels; last level nodes in `last`.
int bfs_levels(const Graph& G, int root, std::vector<int>& mark, std::vector<int>& order,
               std::vector<int>& last) {
    order.clear();
    order.push_back(root);
    mark[static_cast<size_t>(root)] = 2;
    size_t level_begin = 0;
    int levels = 0;
    while (level_begin < order.size()) {
        const size_t level_end = order.size();
        ++levels;
        for (size_t q = level_begin; q < level_end; ++q) {
            const int v = order[q];
            for (int k = G.ptr[static_cast<size_t>(v)]; k < G.ptr[static_cast<size_t>(v) + 1]; ++k) {
                const int u = G.adj[static_cast<size_t>(k)];
                if (mark[static_cast<size_t>(u)] == 0) {
                    mark[static_cast<size_t>(u)] = 2;
                    order.push_back(u);
                }
            }
        }
        if (order.size() == level_end) {
            last.assign(order.begin() + static_cast<long>(level_begin), order.begin() + static_cast<long>(level_end));
        }
        level_begin = level_end;
    }
    for (int v : order) mark[static_cast<size_t>(v)] = 0;
    return levels;
}

inline bool less_deg(const Graph& G, int a, int b) {
    const int da = G.deg[static_cast<size_t>(a)], db = G.deg[static_cast<size_t>(b)];
    return da < db || (da == db && a < b);
}
}  // namespace

void rcm_order(int n, const int* row_ptr, const int* col_idx, int* perm) {
    const Graph G = make_graph(n, row_ptr, col_idx);
    std::vector<int> mark(static_cast<size_t>(n), 0);  // 0 unvisited, 1 placed, 2 in BFS
    std::vector<int> order, last, result;
    result.reserve(static_cast<size_t>(n));
    std::vector<int> nbrs;
    for (int seed = 0; seed < n; ++seed) {
        if (mark[static_cast<size_t>(seed)] != 0) continue;
        // component of seed; its minimum-(degree, index) node
        bfs_levels(G, seed, mark, order, last);
        int v = order[0];
        for (int u : order)
            if (less_deg(G, u, v)) v = u;
        // George-Liu pseudo-peripheral node
        int ecc = bfs_levels(G, v, mark, order, last);
        while (true) {
            int u = last[0];
            for (int w : last)
                if (less_deg(G, w, u)) u = w;
            std::vector<int> order2, last2;
            const int ecc_u = bfs_levels(G, u, mark, order2, last2);
            if (ecc_u > ecc) {
                v = u;
                ecc = ecc_u;
                last.swap(last2);
            } else {
                break;
            }
        }
        // Cuthill-McKee from v
        size_t head = result.size();
        result.push_back(v);
        mark[static_cast<size_t>(v)] = 1;
        while (head < result.size()) {
            const int x = result[head++];
            nbrs.clear();
            for (int k = G.ptr[static_cast<size_t>(x)]; k < G.ptr[static_cast<size_t>(x) + 1]; ++k) {
                const int u = G.adj[static_cast<size_t>(k)];
                if (mark[static_cast<size_t>(u)] == 0) {
                    mark[static_cast<size_t>(u)] = 1;
                    nbrs.push_back(u);
                }
            }
            std::sort(nbrs.begin(), nbrs.end(), [&](int a, int b) { return less_deg(G, a, b); });
            result.insert(result.end(), nbrs.begin(), nbrs.end());
        }
    }
    for (int i = 0; i < n; ++i) perm[i] = result[static_cast<size_t>(n - 1 - i)];
}

void permute_symmetric(int n, const int* row_ptr, const int* col_idx, const double* values,
                       const int* perm, std::vector<int>& orp, std::vector<int>& oci,
                       std::vector<double>& ov) {
    std::vector<int> iperm(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) iperm[static_cast<size_t>(perm[i])] = i;
    orp.assign(static_cast<size_t>(n) + 1, 0);
    for (int i = 0; i < n; ++i) orp[static_cast<size_t>(i) + 1] = orp[static_cast<size_t>(i)] + (row_ptr[perm[i] + 1] - row_ptr[perm[i]]);
    oci.resize(static_cast<size_t>(orp[static_cast<size_t>(n)]));
    ov.resize(static_cast<size_t>(orp[static_cast<size_t>(n)]));
    std::vector<std::pair<int, double>> tmp;
    for (int i = 0; i < n; ++i) {
        const int old = perm[i];
        tmp.clear();
        for (int k = row_ptr[old]; k < row_ptr[old + 1]; ++k)
            tmp.emplace_back(iperm[static_cast<size_t>(col_idx[k])], values[k]);
        std::stable_sort(tmp.begin(), tmp.end(), [](const std::pair<int, double>& a, const std::pair<int, double>& b) { return a.first < b.first; });
        int w = orp[static_cast<size_t>(i)];
        for (auto& e : tmp) {
            oci[static_cast<size_t>(w)] = e.first;
            ov[static_cast<size_t>(w)] = e.second;
            ++w;
        }
    }
}

}  // namespace xplus

using namespace xplus;

extern "C" {

int xplus_rcm(int n, const int* row_ptr, const int* col_idx, int* perm) {
    return guarded([&] {
        require(n > 0 && row_ptr && col_idx && perm, XPLUS_ERR_ARG, "invalid argument");
        validate_csr(n, row_ptr, col_idx, row_ptr[n]);
        rcm_order(n, row_ptr, col_idx, perm);
    });
}

int xplus_permute_symmetric(int n, const int* row_ptr, const int* col_idx, const double* values,
                            const int* perm, int* out_row_ptr, int* out_col_idx,
                            double* out_values) {
    return guarded([&] {
        require(n > 0 && row_ptr && col_idx && values && perm && out_row_ptr && out_col_idx &&
                    out_values, XPLUS_ERR_ARG, "invalid argument");
        validate_csr(n, row_ptr, col_idx, row_ptr[n]);
        std::vector<char> seen(static_cast<size_t>(n), 0);
        for (int i = 0; i < n; ++i) {
            require(perm[i] >= 0 && perm[i] < n && !seen[static_cast<size_t>(perm[i])], XPLUS_ERR_ARG,
                    "perm is not a permutation");
            seen[static_cast<size_t>(perm[i])] = 1;
        }
        std::vector<int> orp, oci;
        std::vector<double> ov;
        permute_symmetric(n, row_ptr, col_idx, values, perm, orp, oci, ov);
        std::memcpy(out_row_ptr, orp.data(), orp.size() * sizeof(int));
        std::memcpy(out_col_idx, oci.data(), oci.size() * sizeof(int));
        std::memcpy(out_values, ov.data(), ov.size() * sizeof(double));
    });
}

}  // extern "C"
