// The compile step on the host: node and element order, DOF numbering, the stdBrick batch
// (maps, parameter sets, padding), lumped masses and the optional element coloring.
//
// The arrays it produces must equal the reference's compile_model output value for value
// (src/compile/batches.cpp:54-393), because every device vector is indexed by them and results
// are compared equation by equation. So each step keeps the reference's rules:
//   RCM            src/compile/renumber.cpp:58-177 (node graph from elements and equalDOF
//                  ties; George-Liu start; neighbours by degree then index; reversed per
//                  component)
//   element order  renumber.cpp:198-215 (smallest internal node index, stable)
//   numbering      src/compile/dof_numbering.cpp:269-485 (union-find with the smallest DOF id as
//                  root; a group with a fixed DOF is fixed; equations in DOF id order)
//   batch          batches.cpp:110-228 (parameter sets per (group, region) in first-use order;
//                  value[k * padded + e]; padding -1 / 0)
//   lumped mass    batches.cpp:204-224 and 231-261 (element masses in batch order, then nodal
//                  masses)
//   coloring       batches.cpp:21-50 (greedy in batch order)
// Models with exact constraints (rigid links, embedded nodes), beams and other elements are
// outside this path and are refused.
#include <algorithm>
#include <map>
#include <numeric>
#include <tuple>
#include <unordered_map>

#include "brick_gp.cuh"
#include "host.hpp"

namespace fx {
namespace {

using Index = int32_t;

struct Graph {
  std::vector<Index> start, adj;
  Index degree(Index v) const { return start[v + 1] - start[v]; }
};

Graph node_graph(const fx_model& m, const std::unordered_map<int32_t, Index>& idx) {
  const Index N = static_cast<Index>(m.tags.size());
  std::vector<std::vector<Index>> nbr(static_cast<size_t>(N));
  for (const auto& g : m.groups) {
    const size_t ne = g.tags.size();
    for (size_t e = 0; e < ne; ++e)
      for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b)
          if (a != b) nbr[idx.at(g.conn[e * 8 + a])].push_back(idx.at(g.conn[e * 8 + b]));
  }
  for (size_t r = 0; r < m.eqd_retained.size(); ++r) {
    const Index a = idx.at(m.eqd_retained[r]), b = idx.at(m.eqd_constrained[r]);
    nbr[a].push_back(b);
    nbr[b].push_back(a);
  }
  Graph G;
  G.start.assign(static_cast<size_t>(N) + 1, 0);
  for (Index v = 0; v < N; ++v) {
    auto& l = nbr[v];
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
    G.start[v + 1] = G.start[v] + static_cast<Index>(l.size());
  }
  G.adj.reserve(static_cast<size_t>(G.start[N]));
  for (auto& l : nbr) G.adj.insert(G.adj.end(), l.begin(), l.end());
  return G;
}

// Breadth-first levels from root over the nodes not yet numbered; the last level and the depth.
std::vector<Index> last_level(const Graph& G, Index root, const std::vector<char>& done, int& depth) {
  std::vector<Index> level{root}, last = level;
  std::vector<char> seen(done);
  seen[root] = 1;
  depth = 0;
  while (!level.empty()) {
    last = level;
    std::vector<Index> next;
    for (Index v : level)
      for (Index k = G.start[v]; k < G.start[v + 1]; ++k)
        if (!seen[G.adj[k]]) {
          seen[G.adj[k]] = 1;
          next.push_back(G.adj[k]);
        }
    if (!next.empty()) ++depth;
    level = std::move(next);
  }
  return last;
}

std::vector<Index> rcm_order(const Graph& G) {
  const Index N = static_cast<Index>(G.start.size()) - 1;
  auto lighter = [&](Index a, Index b) { return G.degree(a) != G.degree(b) ? G.degree(a) < G.degree(b) : a < b; };
  std::vector<char> done(static_cast<size_t>(N), 0);
  std::vector<Index> order;
  order.reserve(static_cast<size_t>(N));
  for (Index s = 0; s < N; ++s) {
    if (done[s]) continue;
    // lightest node of s's component (degree, then index)
    Index best = s;
    {
      std::vector<Index> stack{s};
      std::vector<char> seen(done);
      seen[s] = 1;
      while (!stack.empty()) {
        const Index v = stack.back();
        stack.pop_back();
        if (lighter(v, best)) best = v;
        for (Index k = G.start[v]; k < G.start[v + 1]; ++k)
          if (!seen[G.adj[k]]) {
            seen[G.adj[k]] = 1;
            stack.push_back(G.adj[k]);
          }
      }
    }
    // pseudo-peripheral root: follow the lightest node of the last level while depth grows
    Index root = best;
    int depth = -1;
    for (int it = 0; it < 32; ++it) {
      int d;
      const auto last = last_level(G, root, done, d);
      if (d <= depth) break;
      depth = d;
      root = *std::min_element(last.begin(), last.end(), lighter);
    }
    const size_t first = order.size();
    order.push_back(root);
    done[root] = 1;
    for (size_t head = first; head < order.size(); ++head) {
      const Index v = order[head];
      std::vector<Index> next;
      for (Index k = G.start[v]; k < G.start[v + 1]; ++k)
        if (!done[G.adj[k]]) {
          done[G.adj[k]] = 1;
          next.push_back(G.adj[k]);
        }
      std::sort(next.begin(), next.end(), lighter);
      for (Index w : next) order.push_back(w);
    }
    std::reverse(order.begin() + static_cast<std::ptrdiff_t>(first), order.end());
  }
  return order;
}

struct UnionFind {
  std::vector<Index> parent;
  explicit UnionFind(Index n) : parent(static_cast<size_t>(n)) { std::iota(parent.begin(), parent.end(), 0); }
  Index find(Index a) {
    while (parent[a] != a) {
      parent[a] = parent[parent[a]];
      a = parent[a];
    }
    return a;
  }
  void join(Index a, Index b) {
    a = find(a);
    b = find(b);
    if (a == b) return;
    if (b < a) std::swap(a, b);
    parent[b] = a;
  }
};

Index round_up(Index n, int w) {
  w = std::max(w, 1);
  return (n + w - 1) / w * w;
}

}  // namespace

void compile_model(const fx_model& m, int renumbering, int simd_width, bool coloring, fx_compiled& c) {
  const Index N = static_cast<Index>(m.tags.size());
  std::unordered_map<int32_t, Index> idx;  // model index of each node tag
  idx.reserve(static_cast<size_t>(N));
  for (Index i = 0; i < N; ++i) {
    if (!idx.emplace(m.tags[i], i).second) throw Error(FX_E_INVALID, "duplicate node tag " + std::to_string(m.tags[i]));
  }
  for (const auto& g : m.groups)
    for (int32_t t : g.conn)
      if (!idx.count(t)) throw Error(FX_E_INVALID, "element refers to missing node " + std::to_string(t));

  // ---- node order and element order
  if (renumbering == FX_RENUMBER_RCM) {
    c.node_order = rcm_order(node_graph(m, idx));
  } else {
    c.node_order.resize(static_cast<size_t>(N));
    std::iota(c.node_order.begin(), c.node_order.end(), 0);
  }
  c.node_rank.assign(static_cast<size_t>(N), 0);
  for (Index i = 0; i < N; ++i) c.node_rank[c.node_order[i]] = i;
  std::vector<Index> key;
  std::vector<std::pair<Index, Index>> where;  // global element -> (group, index)
  for (size_t gi = 0; gi < m.groups.size(); ++gi) {
    const auto& g = m.groups[gi];
    for (size_t e = 0; e < g.tags.size(); ++e) {
      Index k = INT32_MAX;
      for (int a = 0; a < 8; ++a) k = std::min(k, c.node_rank[idx.at(g.conn[e * 8 + a])]);
      key.push_back(k);
      where.emplace_back(static_cast<Index>(gi), static_cast<Index>(e));
    }
  }
  c.element_order.resize(key.size());
  std::iota(c.element_order.begin(), c.element_order.end(), 0);
  if (renumbering == FX_RENUMBER_RCM)
    std::stable_sort(c.element_order.begin(), c.element_order.end(), [&](Index a, Index b) { return key[a] < key[b]; });

  // ---- DOF numbering
  c.num_nodes = N;
  c.node_model_index = c.node_order;
  c.node_tag.resize(static_cast<size_t>(N));
  c.dof_offset.assign(static_cast<size_t>(N) + 1, 0);
  std::unordered_map<int32_t, Index> internal;
  internal.reserve(static_cast<size_t>(N));
  for (Index i = 0; i < N; ++i) {
    c.node_tag[i] = m.tags[c.node_order[i]];
    internal[c.node_tag[i]] = i;
    c.dof_offset[i + 1] = c.dof_offset[i] + 3;
  }
  const Index ndof = c.dof_offset[N];
  auto dof_id = [&](int32_t tag, int32_t dof1) {
    const auto it = internal.find(tag);
    if (it == internal.end()) throw Error(FX_E_INVALID, "constraint names missing node " + std::to_string(tag));
    if (dof1 < 1 || dof1 > 3) throw Error(FX_E_INVALID, "DOF out of range at node " + std::to_string(tag));
    return c.dof_offset[it->second] + (dof1 - 1);
  };
  {
    // one equalDOF command (retained node) per constrained node, as the reference requires
    std::unordered_map<int32_t, int32_t> retained_of;
    for (size_t r = 0; r < m.eqd_retained.size(); ++r) {
      const auto [it, fresh] = retained_of.emplace(m.eqd_constrained[r], m.eqd_retained[r]);
      if (!fresh && it->second != m.eqd_retained[r])
        throw Error(FX_E_INVALID, "node " + std::to_string(m.eqd_constrained[r]) +
                                      " is constrained by more than one equalDOF command");
    }
  }
  UnionFind uf(ndof);
  for (size_t r = 0; r < m.eqd_retained.size(); ++r)
    uf.join(dof_id(m.eqd_retained[r], m.eqd_dof[r]), dof_id(m.eqd_constrained[r], m.eqd_dof[r]));
  std::vector<char> fixed_root(static_cast<size_t>(ndof), 0);
  for (size_t r = 0; r < m.fix_node.size(); ++r) fixed_root[uf.find(dof_id(m.fix_node[r], m.fix_dof[r]))] = 1;
  c.eq.assign(static_cast<size_t>(ndof), -1);
  std::vector<Index> eq_of_root(static_cast<size_t>(ndof), -1);
  Index next = 0;
  for (Index a = 0; a < ndof; ++a) {
    const Index root = uf.find(a);
    if (fixed_root[root]) continue;
    if (eq_of_root[root] < 0) eq_of_root[root] = next++;
    c.eq[a] = eq_of_root[root];
  }
  c.num_equations = next;

  c.coords.resize(static_cast<size_t>(3) * N);
  for (Index i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) c.coords[static_cast<size_t>(k) * N + i] = m.coords[static_cast<size_t>(c.node_order[i]) * 3 + k];
  c.eq_dof.assign(static_cast<size_t>(next), -1);
  for (Index i = 0; i < N; ++i)
    for (int d = 0; d < 3; ++d) {
      const Index q = c.eq[c.dof_offset[i] + d];
      if (q >= 0) c.eq_dof[q] = d;
    }

  // ---- the stdBrick batch
  std::unordered_map<int32_t, int32_t> region_of;  // element tag -> last Rayleigh region naming it
  for (size_t r = 0; r < m.regions.size(); ++r)
    for (int32_t t : m.regions[r].elements) region_of[t] = static_cast<int32_t>(r);
  const Index count = static_cast<Index>(c.element_order.size());
  const Index P = round_up(count, simd_width);
  c.count = count;
  c.padded = P;
  c.b_tag.assign(static_cast<size_t>(P), -1);
  c.b_node.assign(static_cast<size_t>(8) * P, -1);
  c.b_eq.assign(static_cast<size_t>(24) * P, -1);
  c.b_param.assign(static_cast<size_t>(P), 0);
  c.params.clear();
  c.lumped_mass.assign(static_cast<size_t>(next), 0.0);
  c.lumped_alpha_mass.assign(static_cast<size_t>(next), 0.0);
  c.nodal_mass.assign(static_cast<size_t>(next), 0.0);
  c.nodal_alpha_mass.assign(static_cast<size_t>(next), 0.0);
  std::map<std::pair<int32_t, int32_t>, int32_t> param_of;  // (group, region) -> parameter set
  for (Index e = 0; e < count; ++e) {
    const auto [gi, ei] = where[c.element_order[e]];
    const Group& g = m.groups[gi];
    const int32_t tag = g.tags[ei];
    c.b_tag[e] = tag;
    const auto rit = region_of.find(tag);
    const int32_t region = rit == region_of.end() ? -1 : rit->second;
    const auto [pit, fresh] = param_of.emplace(std::make_pair(gi, region), static_cast<int32_t>(c.params.size()));
    if (fresh) {
      fx_param_set ps{};
      ps.kind = g.mat.kind;
      ps.mass_type = g.lumped ? 1 : 0;
      ps.E = g.mat.E;
      ps.nu = g.mat.nu;
      ps.rho = g.mat.rho;
      for (int q = 0; q < 3; ++q) ps.b[q] = g.b[q];
      if (region >= 0) {
        const Region& r = m.regions[region];
        ps.alphaM = r.alphaM;
        ps.betaK = r.betaK;
        ps.betaKinit = r.betaKinit;
        ps.betaKcomm = r.betaKcomm;
      }
      ps.sigma_y = g.mat.sigma_y;
      ps.H = g.mat.H;
      ps.hk = g.mat.hk;
      c.params.push_back(ps);
    }
    c.b_param[e] = pit->second;
    double xl[3][8];
    for (int a = 0; a < 8; ++a) {
      const Index n = internal.at(g.conn[static_cast<size_t>(ei) * 8 + a]);
      c.b_node[static_cast<size_t>(a) * P + e] = n;
      for (int d = 0; d < 3; ++d) {
        c.b_eq[static_cast<size_t>(3 * a + d) * P + e] = c.eq[c.dof_offset[n] + d];
        xl[d][a] = c.coords[static_cast<size_t>(d) * N + n];
      }
    }
    const fx_param_set& ps = c.params[pit->second];
    ParamGP pg{};
    pg.rho = ps.rho;
    double mj[8];
    lumped_mass(pg, xl, mj);
    for (int k = 0; k < 24; ++k) {
      const Index q = c.b_eq[static_cast<size_t>(k) * P + e];
      if (q < 0) continue;
      c.lumped_mass[q] += mj[k / 3];
      c.lumped_alpha_mass[q] += ps.alphaM * mj[k / 3];
    }
  }
  if (coloring) {
    std::vector<Index> color_of(static_cast<size_t>(count), -1);
    std::vector<std::vector<Index>> used(static_cast<size_t>(next));
    Index ncolors = 0;
    std::vector<char> taken;
    for (Index e = 0; e < count; ++e) {
      taken.assign(static_cast<size_t>(ncolors) + 1, 0);
      for (int k = 0; k < 24; ++k) {
        const Index q = c.b_eq[static_cast<size_t>(k) * P + e];
        if (q < 0) continue;
        for (Index col : used[q]) taken[col] = 1;
      }
      Index col = 0;
      while (taken[col]) ++col;
      color_of[e] = col;
      ncolors = std::max(ncolors, col + 1);
      for (int k = 0; k < 24; ++k) {
        const Index q = c.b_eq[static_cast<size_t>(k) * P + e];
        if (q >= 0 && std::find(used[q].begin(), used[q].end(), col) == used[q].end()) used[q].push_back(col);
      }
    }
    c.color_start.assign(static_cast<size_t>(ncolors) + 1, 0);
    for (Index col : color_of) ++c.color_start[col + 1];
    for (Index k = 0; k < ncolors; ++k) c.color_start[k + 1] += c.color_start[k];
    c.color_elements.resize(static_cast<size_t>(count));
    std::vector<Index> fill(c.color_start.begin(), c.color_start.end() - 1);
    for (Index e = 0; e < count; ++e) c.color_elements[fill[color_of[e]]++] = e;
  }

  // ---- nodal masses, damped by the alphaM of their node's last region
  std::unordered_map<int32_t, int32_t> node_region;
  if (!m.mass_node.empty() && !m.regions.empty()) {
    std::unordered_map<int32_t, std::pair<size_t, size_t>> element_at;
    for (size_t g = 0; g < m.groups.size(); ++g)
      for (size_t e = 0; e < m.groups[g].tags.size(); ++e) element_at[m.groups[g].tags[e]] = {g, e};
    for (size_t r = 0; r < m.regions.size(); ++r)
      for (int32_t t : m.regions[r].elements) {
        const auto [g, e] = element_at.at(t);
        for (int a = 0; a < 8; ++a) node_region[m.groups[g].conn[e * 8 + a]] = static_cast<int32_t>(r);
      }
  }
  for (size_t r = 0; r < m.mass_node.size(); ++r) {
    const Index q = c.eq[dof_id(m.mass_node[r], m.mass_dof[r])];
    if (q < 0) continue;
    c.lumped_mass[q] += m.mass_value[r];
    c.nodal_mass[q] += m.mass_value[r];
    const auto it = node_region.find(m.mass_node[r]);
    if (it != node_region.end()) {
      const double am = m.regions[it->second].alphaM * m.mass_value[r];
      c.nodal_alpha_mass[q] += am;
      c.lumped_alpha_mass[q] += am;
    }
  }
}

}  // namespace fx
