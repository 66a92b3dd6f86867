#include "gfa.h"

#include <algorithm>
#include <map>
#include <stdexcept>

namespace poa {

BuildGraph::BuildGraph(const HostParams &p) : sigma(int(p.alphabet.size())) {
  add_node(p.encode('N'));
  add_node(p.encode('N'));
}

int32_t BuildGraph::add_node(int b) {
  const int32_t id = n();
  base.push_back(b);
  parent.push_back(id);
  coverage.push_back(0);
  in_id.emplace_back();
  in_w.emplace_back();
  out_id.emplace_back();
  out_w.emplace_back();
  aligned.insert(aligned.end(), size_t(sigma), -1);
  aligned[size_t(id) * size_t(sigma) + size_t(b)] = id;
  return id;
}

// graph.rs:62-79: one observation of an edge (self edges ignored)
void BuildGraph::add_edge(int32_t from, int32_t to) {
  if (from == to) return;
  auto &oi = out_id[size_t(from)];
  auto it = std::find(oi.begin(), oi.end(), to);
  if (it != oi.end()) {
    out_w[size_t(from)][size_t(it - oi.begin())] += 1;
  } else {
    oi.push_back(to);
    out_w[size_t(from)].push_back(1);
  }
  auto &ii = in_id[size_t(to)];
  auto jt = std::find(ii.begin(), ii.end(), from);
  if (jt != ii.end()) {
    in_w[size_t(to)][size_t(jt - ii.begin())] += 1;
  } else {
    ii.push_back(from);
    in_w[size_t(to)].push_back(1);
  }
  coverage[size_t(to)] += 1;
}

bool BuildGraph::has_edge(int32_t from, int32_t to) const {
  const auto &oi = out_id[size_t(from)];
  return std::find(oi.begin(), oi.end(), to) != oi.end();
}

// graph.rs:82-122 with every item an existing node: edges along the items,
// then to the sink; the path keeps the ids >= 2.
void BuildGraph::add_path_nodes(int32_t seq_id, const std::vector<int32_t> &ids) {
  int32_t prev = -1;
  std::vector<int32_t> path;
  for (int32_t id : ids) {
    if (prev >= 0) add_edge(prev, id);
    prev = id;
    if (id >= 2) path.push_back(id);
  }
  add_edge(prev >= 0 ? prev : 0, 1);
  path_seq.push_back(seq_id);
  paths.push_back(std::move(path));
}

int64_t BuildGraph::edges() const {
  int64_t e = 0;
  for (auto &v : in_id) e += int64_t(v.size());
  return e;
}

void BuildGraph::toposort(std::vector<int32_t> &rank_of, std::vector<int32_t> &order) const {
  const int32_t nn = n();
  std::vector<int64_t> degree(static_cast<size_t>(nn));
  std::vector<int32_t> stack;
  for (int32_t id = 0; id < nn; ++id) {
    degree[size_t(id)] = int64_t(in_id[size_t(id)].size());
    if (degree[size_t(id)] == 0) stack.push_back(id);
  }
  rank_of.assign(size_t(nn), 0);
  order.clear();
  while (!stack.empty()) {
    const int32_t id = stack.back();
    stack.pop_back();
    rank_of[size_t(id)] = int32_t(order.size());
    order.push_back(id);
    for (int32_t next : out_id[size_t(id)]) {
      if (degree[size_t(next)] == 0) throw std::runtime_error("invalid graph column dependencies");
      if (--degree[size_t(next)] == 0) stack.push_back(next);
    }
  }
  if (int32_t(order.size()) != nn) throw std::runtime_error("graph contains a cycle (possibly between alignment columns)");
}

namespace {

std::vector<std::string> split(const std::string &s, char sep) {
  std::vector<std::string> out;
  size_t a = 0;
  for (;;) {
    const size_t b = s.find(sep, a);
    out.push_back(s.substr(a, b == std::string::npos ? std::string::npos : b - a));
    if (b == std::string::npos) break;
    a = b + 1;
  }
  return out;
}

}  // namespace

BuildGraph read_gfa(const HostParams &p, const char *text, size_t len, std::vector<GfaRecord> &records) {
  struct PathLine {
    std::string name;
    std::vector<std::string> segs;
  };
  std::vector<std::string> seg_names, seg_seqs;
  std::map<std::string, size_t> seg_index;
  std::vector<std::pair<std::string, std::string>> links;
  std::vector<PathLine> plines;
  const std::string all(text, len);
  for (std::string line : split(all, '\n')) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty() || line[0] == '#') continue;
    const auto f = split(line, '\t');
    if (f[0] == "S") {
      if (f.size() < 3) throw std::runtime_error("malformed GFA segment line");
      if (f[2].empty() || f[2] == "*") throw std::runtime_error("GFA segment " + f[1] + " has no sequence");
      if (seg_index.count(f[1])) throw std::runtime_error("duplicate GFA segment " + f[1]);
      seg_index[f[1]] = seg_names.size();
      seg_names.push_back(f[1]);
      seg_seqs.push_back(f[2]);
    } else if (f[0] == "L") {
      if (f.size() < 6) throw std::runtime_error("malformed GFA link line");
      if (f[2] != "+" || f[4] != "+") throw std::runtime_error("unsupported GFA link orientation");
      if (f[5] != "0M" && f[5] != "*") throw std::runtime_error("unsupported GFA link overlap " + f[5]);
      links.emplace_back(f[1], f[3]);
    } else if (f[0] == "P") {
      if (f.size() < 3) throw std::runtime_error("malformed GFA path line");
      PathLine pl{f[1], {}};
      if (f[2] != "*") {
        for (const auto &e : split(f[2], ',')) {
          if (e.size() < 2) throw std::runtime_error("malformed GFA path " + f[1]);
          if (e.back() == '-') throw std::runtime_error("unsupported GFA path orientation in " + f[1]);
          if (e.back() != '+') throw std::runtime_error("malformed GFA path " + f[1]);
          pl.segs.push_back(e.substr(0, e.size() - 1));
        }
      }
      plines.push_back(std::move(pl));
    }
  }
  BuildGraph g(p);
  std::vector<std::vector<int32_t>> seg_nodes(seg_names.size());
  for (size_t k = 0; k < seg_names.size(); ++k)
    for (char c : seg_seqs[k]) seg_nodes[k].push_back(g.add_node(p.encode(uint8_t(c))));
  auto seg_of = [&](const std::string &name, const std::string &what) {
    auto it = seg_index.find(name);
    if (it == seg_index.end()) throw std::runtime_error("GFA " + what + " references unknown segment " + name);
    return it->second;
  };
  std::vector<std::pair<int32_t, int32_t>> link_nodes;
  for (const auto &l : links) {
    const size_t a = seg_of(l.first, "link"), b = seg_of(l.second, "link");
    if (a == b) throw std::runtime_error("GFA link from segment " + l.first + " to itself forms a cycle");
    link_nodes.emplace_back(seg_nodes[a].back(), seg_nodes[b].front());
  }
  records.clear();
  for (size_t k = 0; k < plines.size(); ++k) {
    const auto &pl = plines[k];
    std::vector<int32_t> ids{0};
    std::vector<char> seen(size_t(g.n()), 0);
    std::string seq;
    for (const auto &sn : pl.segs) {
      const size_t sg = seg_of(sn, "path " + pl.name);
      for (int32_t id : seg_nodes[sg]) {
        if (seen[size_t(id)]) throw std::runtime_error("GFA path " + pl.name + " revisits segment " + sn);
        seen[size_t(id)] = 1;
        ids.push_back(id);
      }
      seq += seg_seqs[sg];
    }
    g.add_path_nodes(int32_t(k), ids);
    records.push_back({pl.name, seq});
  }
  for (const auto &nodes : seg_nodes)
    for (size_t k = 1; k < nodes.size(); ++k)
      if (!g.has_edge(nodes[k - 1], nodes[k])) g.add_edge(nodes[k - 1], nodes[k]);
  for (const auto &ln : link_nodes)
    if (!g.has_edge(ln.first, ln.second)) g.add_edge(ln.first, ln.second);
  for (int32_t id = 2; id < g.n(); ++id)
    if (g.in_id[size_t(id)].empty()) g.add_edge(0, id);
  for (int32_t id = 2; id < g.n(); ++id)
    if (g.out_id[size_t(id)].empty()) g.add_edge(id, 1);
  return g;
}

}  // namespace poa
