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
// Pattern of A_hat = A(perm, perm): row i of A_hat is A's row perm[i], columns renumbered by
// the inverse permutation and sorted; amap[k] = position of A's entry k in A_hat; diag[i] =
// position of A_hat(i, i).  Returns the first row (of A) without a diagonal entry, or -1.
int permute_pattern(int n, const std::vector<int> &arp, const std::vector<int> &aci,
                    const std::vector<int> &perm, std::vector<int> &rp, std::vector<int> &ci,
                    std::vector<int> &amap, std::vector<int> &diag);

}  // namespace bpf
