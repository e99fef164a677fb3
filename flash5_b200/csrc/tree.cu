// tree.cu -- the tree part of a regrid on the host (what PARAMESH's
// amr_refine_derefine does before gr_updateRefinement moves the data): the
// marked leaves are split, refinement spreads until every leaf's neighbours
// (diagonals included) are within one level, and a parent's children are
// removed when all of them are unrefined leaves marked for derefinement and
// no neighbour's child touching the parent stays refined.  Nodes are keyed
// by (level, x, y, z) and kept in hash sets; the result is ordered by level
// and then Morton index, as the Python grid builder orders nodes.
#include <stdint.h>
#include <algorithm>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include "../../include/flash_hy.h"

namespace {

struct Tree {
  int ndim, L, nblk[3], per[3];
  std::unordered_set<uint64_t> leaves, inner;

  static uint64_t key(int l, int x, int y, int z) {
    return ((uint64_t)l << 57) | ((uint64_t)x << 38) | ((uint64_t)y << 19) | (uint64_t)z;
  }
  static void unkey(uint64_t k, int &l, int c[3]) {
    l = (int)(k >> 57);
    c[0] = (int)((k >> 38) & 0x7ffff);
    c[1] = (int)((k >> 19) & 0x7ffff);
    c[2] = (int)(k & 0x7ffff);
  }
  int ext(int l, int d) const { return d < ndim ? nblk[d] << (l - 1) : 1; }
  void children(int l, const int c[3], uint64_t out[8]) const {
    for (int o = 0; o < (1 << ndim); ++o)
      out[o] = key(l + 1, 2 * c[0] + (o & 1), ndim > 1 ? 2 * c[1] + ((o >> 1) & 1) : 0,
                   ndim > 2 ? 2 * c[2] + ((o >> 2) & 1) : 0);
  }
  bool neighbor(int l, const int c[3], const int o[3], int p[3]) const {
    for (int d = 0; d < 3; ++d) {
      int v = c[d] + (d < ndim ? o[d] : 0);
      if (d < ndim && (v < 0 || v >= ext(l, d))) {
        if (!per[d]) return false;
        v = ((v % ext(l, d)) + ext(l, d)) % ext(l, d);
      }
      p[d] = v;
    }
    return true;
  }
  void split(uint64_t k) {
    int l, c[3];
    unkey(k, l, c);
    leaves.erase(k);
    inner.insert(k);
    uint64_t ch[8];
    children(l, c, ch);
    for (int o = 0; o < (1 << ndim); ++o) leaves.insert(ch[o]);
  }
  // does the neighbour p (level l, offset o from the block) have a child
  // touching the block that is in set S?
  bool touching_child_in(int l, const int p[3], const int o[3], const std::unordered_set<uint64_t> &S,
                         const std::unordered_set<uint64_t> *exclude = nullptr) const {
    uint64_t ch[8];
    children(l, p, ch);
    for (int q = 0; q < (1 << ndim); ++q) {
      int cl, cc[3];
      unkey(ch[q], cl, cc);
      bool touch = true;
      for (int d = 0; d < ndim; ++d) {
        const int co = cc[d] - 2 * p[d];
        if ((o[d] == 1 && co != 0) || (o[d] == -1 && co != 1)) touch = false;
      }
      if (touch && S.count(ch[q]) && !(exclude && exclude->count(ch[q]))) return true;
    }
    return false;
  }
  template <class F> void for_offsets(F f) const {
    for (int z = -1; z <= (ndim > 2 ? 1 : -1); ++z)
      for (int y = -1; y <= (ndim > 1 ? 1 : -1); ++y)
        for (int x = -1; x <= 1; ++x) {
          const int o[3] = {x, ndim > 1 ? y : 0, ndim > 2 ? z : 0};
          if (!o[0] && !o[1] && !o[2]) continue;
          if (f(o)) return;
        }
  }
  void balance() {
    bool changed = true;
    while (changed) {
      changed = false;
      std::vector<uint64_t> todo;
      for (uint64_t k : leaves) {
        int l, c[3];
        unkey(k, l, c);
        if (l >= L) continue;
        bool need = false;
        for_offsets([&](const int o[3]) {
          int p[3];
          if (!neighbor(l, c, o, p) || !inner.count(key(l, p[0], p[1], p[2]))) return false;
          need = touching_child_in(l, p, o, inner);
          return need;
        });
        if (need) todo.push_back(k);
      }
      for (uint64_t k : todo)
        if (leaves.count(k)) { split(k); changed = true; }
    }
  }
};

uint64_t morton(const int c[3]) {
  uint64_t k = 0;
  for (int bit = 0; bit < 16; ++bit)
    for (int d = 0; d < 3; ++d) k |= (uint64_t)((c[d] >> bit) & 1) << (3 * bit + d);
  return k;
}

}  // namespace

extern "C" int flash_hy_refine_tree(const flash_hy_grid_desc *g, const unsigned char *refine,
                                    const unsigned char *derefine, int min_level, int cap, int *new_n,
                                    int *new_levels, int *new_coords, int *new_parent, int *src, int *how) {
  if (!g || !refine || !derefine || !new_n || g->ndim < 2 || g->ndim > 3 || g->max_level < 1 ||
      g->max_level > 16 || !g->block_level || !g->block_coords)
    return FLASH_HY_ERR_BAD_ARG;
  Tree t;
  t.ndim = g->ndim;
  t.L = g->max_level;
  for (int d = 0; d < 3; ++d) {
    t.nblk[d] = d < g->ndim ? g->nblk_l1[d] : 1;
    t.per[d] = d < g->ndim && g->bc[2 * d] == FLASH_HY_BC_PERIODIC;
  }
  std::unordered_map<uint64_t, int> old_of;
  old_of.reserve((size_t)g->nblocks * 2);
  for (int b = 0; b < g->nblocks; ++b) {
    const int *c = &g->block_coords[3 * b];
    old_of[Tree::key(g->block_level[b], c[0], g->ndim > 1 ? c[1] : 0, g->ndim > 2 ? c[2] : 0)] = b;
  }
  std::vector<char> old_leaf(g->nblocks, 1);
  for (int b = 0; b < g->nblocks; ++b) {
    const int l = g->block_level[b];
    if (l > 1) {
      const int *c = &g->block_coords[3 * b];
      auto it = old_of.find(Tree::key(l - 1, c[0] / 2, g->ndim > 1 ? c[1] / 2 : 0, g->ndim > 2 ? c[2] / 2 : 0));
      if (it == old_of.end()) return FLASH_HY_ERR_BAD_ARG;
      old_leaf[it->second] = 0;
    }
  }
  std::unordered_set<uint64_t> old_leaves, old_inner, dmark;
  for (auto &kv : old_of) {
    (old_leaf[kv.second] ? old_leaves : old_inner).insert(kv.first);
    if (old_leaf[kv.second] && derefine[kv.second]) dmark.insert(kv.first);
  }
  t.leaves = old_leaves;
  t.inner = old_inner;
  for (int b = 0; b < g->nblocks; ++b)
    if (refine[b] && old_leaf[b] && g->block_level[b] < t.L) {
      const int *c = &g->block_coords[3 * b];
      t.split(Tree::key(g->block_level[b], c[0], g->ndim > 1 ? c[1] : 0, g->ndim > 2 ? c[2] : 0));
    }
  t.balance();
  // derefinement
  std::unordered_set<uint64_t> cand;
  for (uint64_t k : old_inner) {
    int l, c[3];
    Tree::unkey(k, l, c);
    if (l < min_level) continue;
    uint64_t ch[8];
    t.children(l, c, ch);
    bool all = true;
    for (int o = 0; o < (1 << t.ndim) && all; ++o) all = t.leaves.count(ch[o]) && dmark.count(ch[o]);
    if (all) cand.insert(k);
  }
  bool changed = true;
  while (changed) {
    changed = false;
    std::vector<uint64_t> drop;
    for (uint64_t k : cand) {
      int l, c[3];
      Tree::unkey(k, l, c);
      bool blocked = false;
      t.for_offsets([&](const int o[3]) {
        int p[3];
        if (!t.neighbor(l, c, o, p) || !t.inner.count(Tree::key(l, p[0], p[1], p[2]))) return false;
        // a touching child of the neighbour that stays refined (not a candidate)
        blocked = t.touching_child_in(l, p, o, t.inner, &cand);
        return blocked;
      });
      if (blocked) drop.push_back(k);
    }
    for (uint64_t k : drop) { cand.erase(k); changed = true; }
  }
  for (uint64_t k : cand) {
    int l, c[3];
    Tree::unkey(k, l, c);
    uint64_t ch[8];
    t.children(l, c, ch);
    for (int o = 0; o < (1 << t.ndim); ++o) t.leaves.erase(ch[o]);
    t.inner.erase(k);
    t.leaves.insert(k);
  }
  // ordered node list
  struct Node { int l; uint64_t m; uint64_t k; };
  std::vector<Node> nodes;
  nodes.reserve(t.leaves.size() + t.inner.size());
  for (const auto *S : {&t.leaves, &t.inner})
    for (uint64_t k : *S) {
      int l, c[3];
      Tree::unkey(k, l, c);
      nodes.push_back({l, morton(c), k});
    }
  std::sort(nodes.begin(), nodes.end(), [](const Node &a, const Node &b) { return a.l != b.l ? a.l < b.l : a.m < b.m; });
  const int n = (int)nodes.size();
  *new_n = n;
  if (n > cap || !new_levels || !new_coords || !new_parent || !src || !how) return FLASH_HY_ERR_BAD_ARG;
  std::unordered_map<uint64_t, int> new_of;
  new_of.reserve((size_t)n * 2);
  for (int q = 0; q < n; ++q) new_of[nodes[q].k] = q;
  for (int q = 0; q < n; ++q) {
    int l, c[3];
    Tree::unkey(nodes[q].k, l, c);
    new_levels[q] = l;
    new_coords[3 * q] = c[0]; new_coords[3 * q + 1] = c[1]; new_coords[3 * q + 2] = c[2];
    new_parent[q] = l > 1 ? new_of.at(Tree::key(l - 1, c[0] / 2, c[1] / 2, c[2] / 2)) : -1;
    auto it = old_of.find(nodes[q].k);
    if (it != old_of.end()) {
      src[q] = it->second;
      how[q] = (old_inner.count(nodes[q].k) && t.leaves.count(nodes[q].k)) ? 2 : 0;
    } else {
      auto pit = old_of.find(Tree::key(l - 1, c[0] / 2, c[1] / 2, c[2] / 2));
      if (pit == old_of.end() || !old_leaves.count(pit->first)) return FLASH_HY_ERR_BAD_ARG;
      src[q] = pit->second;
      how[q] = 1;
    }
  }
  return 0;
}
