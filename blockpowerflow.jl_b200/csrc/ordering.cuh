// Symmetric orderings of a square sparsity pattern (host side).  Each returns `order` with
// order[k] = the original index placed at position k.
#pragma once

#include <vector>

namespace bpf {

// Adjacency of the symmetrized pattern A + A^T without the diagonal, sorted and unique.
void sym_adjacency(int n, const std::vector<int> &rp, const std::vector<int> &ci,
                   std::vector<std::vector<int>> &adj);
// Minimum degree on the explicit elimination graph (the :AMD / :MDQ criterion).
std::vector<int> order_min_degree(int n, const std::vector<int> &rp, const std::vector<int> &ci);
// Reverse Cuthill-McKee from a pseudo-peripheral start node of each component.
std::vector<int> order_rcm(int n, const std::vector<int> &rp, const std::vector<int> &ci);

}  // namespace bpf
