// Symmetric fill- and bandwidth-reducing orderings of a sparsity pattern (host side), shared
// by the cusolverRF-style analysis (src/cusolverRF.jl:70-95, where cusolverSp computes the
// :AMD / :MDQ / :RCM orderings) and the reordered ILU(0) / IC(0) preconditioners.
#include <algorithm>
#include <functional>
#include <iterator>
#include <set>
#include <vector>

#include "ordering.cuh"

namespace bpf {

// ------------------------------------------------------------------------------------
// orderings
// ------------------------------------------------------------------------------------
void sym_adjacency(int n, const std::vector<int> &rp, const std::vector<int> &ci,
                          std::vector<std::vector<int>> &adj) {
    adj.assign(n, {});
    for (int i = 0; i < n; i++)
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            int j = ci[k];
            if (j == i) continue;
            adj[i].push_back(j);
            adj[j].push_back(i);
        }
    for (auto &a : adj) {
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
    }
}

// Minimum degree on the explicit elimination graph: eliminate a node of least current
// degree (smallest index on ties), turning its neighbourhood into a clique.  The queue is a
// binary heap of (degree, node) with lazy deletion (an entry whose degree is no longer the
// node's is skipped when it surfaces), so the node taken is the smallest current (degree,
// node) pair; the clique is formed with a marker array on unsorted adjacency lists.
std::vector<int> order_min_degree(int n, const std::vector<int> &rp, const std::vector<int> &ci) {
    std::vector<std::vector<int>> adj;
    sym_adjacency(n, rp, ci, adj);
    using Key = std::pair<int, int>;
    std::vector<Key> heap;
    heap.reserve(2 * (size_t)n);
    std::vector<int> deg(n);
    for (int v = 0; v < n; v++) {
        deg[v] = (int)adj[v].size();
        heap.push_back({deg[v], v});
    }
    std::make_heap(heap.begin(), heap.end(), std::greater<Key>());
    std::vector<char> gone(n, 0);
    std::vector<int> mark(n, -1), order, nb;
    order.reserve(n);
    int stamp = 0;
    while (!heap.empty()) {
        std::pop_heap(heap.begin(), heap.end(), std::greater<Key>());
        const Key t = heap.back();
        heap.pop_back();
        const int v = t.second;
        if (gone[v] || t.first != deg[v]) continue;
        gone[v] = 1;
        order.push_back(v);
        nb.swap(adj[v]);
        for (int u : nb) {
            // adj[u] <- adj[u] U nb \ {u, v}
            std::vector<int> &a = adj[u];
            const int s = stamp++;
            size_t w = 0;
            for (size_t r = 0; r < a.size(); r++) {
                const int x = a[r];
                if (x == v) continue;
                mark[x] = s;
                a[w++] = x;
            }
            a.resize(w);
            mark[u] = s;
            for (int x : nb)
                if (mark[x] != s) {
                    mark[x] = s;
                    a.push_back(x);
                }
            if ((int)a.size() != deg[u]) {
                deg[u] = (int)a.size();
                heap.push_back({deg[u], u});
                std::push_heap(heap.begin(), heap.end(), std::greater<Key>());
            }
        }
        std::vector<int>().swap(nb);
    }
    return order;
}

static std::vector<int> bfs_levels(int s, const std::vector<std::vector<int>> &adj,
                                   std::vector<int> &lev, const std::vector<char> &done) {
    std::vector<int> q{s};
    lev.assign(adj.size(), -1);
    lev[s] = 0;
    for (size_t h = 0; h < q.size(); h++) {
        int v = q[h];
        for (int u : adj[v])
            if (lev[u] < 0 && !done[u]) {
                lev[u] = lev[v] + 1;
                q.push_back(u);
            }
    }
    return q;
}

// Reverse Cuthill-McKee from a pseudo-peripheral start node of each component.
std::vector<int> order_rcm(int n, const std::vector<int> &rp, const std::vector<int> &ci) {
    std::vector<std::vector<int>> adj;
    sym_adjacency(n, rp, ci, adj);
    std::vector<char> done(n, 0);
    std::vector<int> order, lev;
    order.reserve(n);
    for (int seed = 0; seed < n; seed++) {
        if (done[seed]) continue;
        // pseudo-peripheral node (George-Liu)
        int s = seed, ecc = -1;
        for (int it = 0; it < 8; it++) {
            std::vector<int> comp = bfs_levels(s, adj, lev, done);
            int e = lev[comp.back()];
            if (e <= ecc) break;
            ecc = e;
            int best = comp.back();
            for (int v : comp)
                if (lev[v] == e && adj[v].size() < adj[best].size()) best = v;
            s = best;
        }
        std::vector<int> q{s};
        done[s] = 1;
        for (size_t h = 0; h < q.size(); h++) {
            int v = q[h];
            std::vector<int> nb;
            for (int u : adj[v])
                if (!done[u]) nb.push_back(u);
            std::sort(nb.begin(), nb.end(), [&](int a, int b) {
                return adj[a].size() < adj[b].size() || (adj[a].size() == adj[b].size() && a < b);
            });
            for (int u : nb) {
                done[u] = 1;
                q.push_back(u);
            }
        }
        order.insert(order.end(), q.begin(), q.end());
    }
    std::reverse(order.begin(), order.end());
    return order;
}

int permute_pattern(int n, const std::vector<int> &arp, const std::vector<int> &aci,
                    const std::vector<int> &perm, std::vector<int> &rp, std::vector<int> &ci,
                    std::vector<int> &amap, std::vector<int> &diag) {
    const int nnz = arp[n];
    std::vector<int> pinv(n);
    for (int i = 0; i < n; i++) pinv[perm[i]] = i;
    rp.assign(n + 1, 0);
    for (int i = 0; i < n; i++) rp[i + 1] = rp[i] + (arp[perm[i] + 1] - arp[perm[i]]);
    ci.resize(nnz);
    amap.resize(nnz);
    diag.assign(n, -1);
    std::vector<std::pair<int, int>> row;
    for (int i = 0; i < n; i++) {
        const int r = perm[i];
        row.clear();
        for (int k = arp[r]; k < arp[r + 1]; k++) row.push_back({pinv[aci[k]], k});
        std::sort(row.begin(), row.end());
        for (size_t t = 0; t < row.size(); t++) {
            ci[rp[i] + t] = row[t].first;
            amap[row[t].second] = rp[i] + (int)t;
            if (row[t].first == i) diag[i] = rp[i] + (int)t;
        }
        if (diag[i] < 0) return r;
    }
    return -1;
}

}  // namespace bpf
