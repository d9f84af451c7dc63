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
//                  masses; SSPbrick: density times each node's volume weight, ssp_brick.hpp)
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
#include "ssp_brick.cuh"

namespace fx {
namespace {

using Index = int32_t;

// ---- node order: reverse Cuthill-McKee
//
// Rules the numbering follows, so that it equals the reference's node by node
// (src/compile/renumber.cpp:58-177):
//   R1 the graph joins the nodes at two different corner positions of one element, and the two
//      nodes of each equalDOF pair (in both directions); a node's degree counts its distinct
//      neighbours;
//   R2 "lighter" compares nodes by degree, then by model index;
//   R3 components are numbered one after another, in the order of their lowest model index;
//   R4 a component's root comes from its lightest node by the George-Liu walk: level the
//      component from the current root and, while the number of levels grows (at most 32
//      levelings), move the root to the lightest node of the last level;
//   R5 from the root, breadth first, each node's neighbours not yet reached are appended
//      lightest first; the component's sequence is then reversed.
// Elements follow by the smallest rank among their nodes, ties in model order.

// Adjacency in compressed rows, built by counting: row v lists v's neighbours ascending.
class NodeAdjacency {
 public:
  NodeAdjacency(const fx_model& m, const std::unordered_map<int32_t, Index>& idx) {
    const Index N = static_cast<Index>(m.tags.size());
    std::vector<Index> corner;  // model index per element corner, group after group
    for (const auto& g : m.groups)
      for (int32_t t : g.conn) corner.push_back(idx.at(t));
    std::vector<Index> tie_a(m.eqd_retained.size()), tie_b(m.eqd_retained.size());
    for (size_t r = 0; r < tie_a.size(); ++r) {
      tie_a[r] = idx.at(m.eqd_retained[r]);
      tie_b[r] = idx.at(m.eqd_constrained[r]);
    }
    // pass 1: row lengths with repeats; pass 2: fill; then each row sorted and compacted
    std::vector<int64_t> cap(static_cast<size_t>(N) + 1, 0);
    for (Index v : corner) cap[v + 1] += 7;
    for (size_t r = 0; r < tie_a.size(); ++r) ++cap[tie_a[r] + 1], ++cap[tie_b[r] + 1];
    for (Index v = 0; v < N; ++v) cap[v + 1] += cap[v];
    std::vector<Index> raw(static_cast<size_t>(cap[N]));
    std::vector<int64_t> fill(cap.begin(), cap.end() - 1);
    for (size_t e = 0; e + 8 <= corner.size(); e += 8)
      for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j)
          if (i != j) raw[fill[corner[e + i]]++] = corner[e + j];
    for (size_t r = 0; r < tie_a.size(); ++r) {
      raw[fill[tie_a[r]]++] = tie_b[r];
      raw[fill[tie_b[r]]++] = tie_a[r];
    }
    row_.assign(static_cast<size_t>(N) + 1, 0);
    col_.reserve(raw.size() / 2);
    for (Index v = 0; v < N; ++v) {
      auto* lo = raw.data() + cap[v];
      auto* hi = raw.data() + cap[v + 1];
      std::sort(lo, hi);
      hi = std::unique(lo, hi);
      col_.insert(col_.end(), lo, hi);
      row_[v + 1] = static_cast<Index>(col_.size());
    }
  }
  Index nodes() const { return static_cast<Index>(row_.size()) - 1; }
  Index degree(Index v) const { return row_[v + 1] - row_[v]; }
  const Index* begin(Index v) const { return col_.data() + row_[v]; }
  const Index* end(Index v) const { return col_.data() + row_[v + 1]; }
  bool lighter(Index a, Index b) const {
    const Index da = degree(a), db = degree(b);
    return da != db ? da < db : a < b;
  }

 private:
  std::vector<Index> row_, col_;
};

// Breadth-first traversals over the nodes not numbered yet. A node's mark is kNumbered once it
// has a number, and equals the pass counter while the current traversal has reached it.
class LevelWalker {
 public:
  explicit LevelWalker(const NodeAdjacency& g) : g_(g), mark_(static_cast<size_t>(g.nodes()), 0) {}

  // Visits everything reachable from root; `seq` holds the nodes in visiting order, level after
  // level. With `lightest_first`, each node's newly reached neighbours enter lightest first (R5).
  // Returns the number of levels.
  int walk(Index root, bool lightest_first) {
    ++pass_;
    seq.clear();
    seq.push_back(root);
    mark_[root] = pass_;
    size_t level_begin = 0;
    int levels = 0;
    last_level = 0;
    while (level_begin < seq.size()) {
      const size_t level_end = seq.size();
      ++levels;
      last_level = level_begin;
      for (size_t h = level_begin; h < level_end; ++h) {
        const size_t grown = seq.size();
        for (const Index* w = g_.begin(seq[h]); w != g_.end(seq[h]); ++w)
          if (mark_[*w] != kNumbered && mark_[*w] != pass_) {
            mark_[*w] = pass_;
            seq.push_back(*w);
          }
        if (lightest_first)
          std::sort(seq.begin() + static_cast<std::ptrdiff_t>(grown), seq.end(),
                    [this](Index a, Index b) { return g_.lighter(a, b); });
      }
      level_begin = level_end;
    }
    return levels;
  }

  bool numbered(Index v) const { return mark_[v] == kNumbered; }
  void number_visited() {
    for (Index v : seq) mark_[v] = kNumbered;
  }
  Index lightest(size_t from) const {
    Index best = seq[from];
    for (size_t i = from + 1; i < seq.size(); ++i)
      if (g_.lighter(seq[i], best)) best = seq[i];
    return best;
  }

  std::vector<Index> seq;
  size_t last_level = 0;  // where the last level starts in seq

 private:
  static constexpr int32_t kNumbered = -1;
  const NodeAdjacency& g_;
  std::vector<int32_t> mark_;
  int32_t pass_ = 0;
};

std::vector<Index> rcm_node_order(const fx_model& m, const std::unordered_map<int32_t, Index>& idx) {
  const NodeAdjacency g(m, idx);
  LevelWalker walker(g);
  std::vector<Index> order;
  order.reserve(static_cast<size_t>(g.nodes()));
  for (Index s = 0; s < g.nodes(); ++s) {  // R3
    if (walker.numbered(s)) continue;
    walker.walk(s, false);
    Index root = walker.lightest(0);  // R4: the component's lightest node
    int levels = 0;
    for (int round = 0; round < 32; ++round) {
      const int l = walker.walk(root, false);
      if (l <= levels) break;
      levels = l;
      root = walker.lightest(walker.last_level);
    }
    walker.walk(root, true);  // R5
    walker.number_visited();
    order.insert(order.end(), walker.seq.rbegin(), walker.seq.rend());
  }
  return order;
}

// Element order: ascending key (the smallest node rank of the element), equal keys in model
// order; a counting sort over the key range, stable by construction.
std::vector<Index> order_by_key(const std::vector<Index>& key, Index key_range) {
  std::vector<Index> first(static_cast<size_t>(key_range) + 1, 0);
  for (Index k : key) ++first[k + 1];
  for (Index k = 0; k < key_range; ++k) first[k + 1] += first[k];
  std::vector<Index> out(key.size());
  for (size_t e = 0; e < key.size(); ++e) out[first[key[e]]++] = static_cast<Index>(e);
  return out;
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
    c.node_order = rcm_node_order(m, idx);
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
  if (renumbering == FX_RENUMBER_RCM) {
    c.element_order = order_by_key(key, N);
  } else {
    c.element_order.resize(key.size());
    std::iota(c.element_order.begin(), c.element_order.end(), 0);
  }

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
      ps.element = g.mat.element;
      ps.mass_type = (g.lumped || g.mat.element == FX_ELEM_SSPBRICK) ? 1 : 0;  // SSPbrick always lumps
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
    if (ps.element == FX_ELEM_SSPBRICK) {  // density times each node's volume weight
      double nv[8];
      ssp::node_volumes(xl, nv);
      for (int j = 0; j < 8; ++j) mj[j] = ps.rho * nv[j];
    } else {
      lumped_mass(pg, xl, mj);
    }
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
