#include "host_graph.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>

namespace poa {

HostParams HostParams::from(const poa_params *p) {
  HostParams r;
  r.match_score = p->match_score;
  r.mismatch = p->mismatch;
  r.gap_open = p->gap_open;
  r.gap_ext = p->gap_ext;
  r.b = p->b;
  r.f = p->f;
  r.adaptive = p->adaptive != 0;
  r.seeding = p->seeding != 0;
  r.k = p->k;
  r.w = p->w;
  r.progressive = p->progressive != 0;
  r.result = p->result;
  r.threads = p->threads;
  r.win_band = p->win_band;
  r.win_max = p->win_max;
  r.mm_filter_ratio = p->mm_filter_ratio;
  r.max_occ = p->max_occ;
  r.tr_dist = p->tr_dist;
  r.verbose = p->verbose;
  r.is_rna = p->is_rna != 0;
  const int n = p->alphabet_len > 0 ? p->alphabet_len : 0;
  if (n && p->alphabet) r.alphabet.assign(p->alphabet, p->alphabet + n);
  if (n && p->matrix) r.matrix.assign(p->matrix, p->matrix + int64_t(n) * n);
  return r;
}

int HostParams::encode(uint8_t c) const {
  if (c >= 'a' && c <= 'z') c = uint8_t(c - 32);
  if (alphabet.size() <= 5 && c == 'U') c = 'T';
  for (size_t i = 0; i < alphabet.size(); ++i)
    if (alphabet[i] == c) return int(i);
  for (size_t i = 0; i < alphabet.size(); ++i)
    if (alphabet[i] == 'N') return int(i);
  return int(alphabet.size()) - 1;
}

uint8_t HostParams::decode(int code) const {
  const uint8_t c = alphabet[size_t(code)];
  return (is_rna && alphabet.size() <= 5 && c == 'T') ? uint8_t('U') : c;
}

std::string HostParams::validate() const {
  const size_t n = alphabet.size();
  if (n == 0 || n > 256 || matrix.size() != n * n) return "invalid scoring matrix dimensions";
  if (threads == 0) return "thread count must be positive";
  if (!(k >= 1 && k <= 31) || !(w >= 1 && w < 32768)) return "k must be 1..31 and minimizer window must be 1..32767";
  if (gap_open > 0 || gap_ext > 0) return "gap penalties must be zero or negative";
  if (result < 0 || result > 2 || verbose < 0 || verbose > 2) return "result format and verbosity must be 0..2";
  if (!std::isfinite(mm_filter_ratio) || mm_filter_ratio < 0.0 || mm_filter_ratio > 1.0)
    return "minimizer filter ratio must be between 0 and 1";
  if (win_max == 0) return "window maximum must be positive";
  return std::string();
}

uint64_t HostParams::largest() const {
  uint64_t m = 0;
  for (int32_t x : matrix) m = std::max<uint64_t>(m, uint64_t(std::llabs(int64_t(x))));
  const int64_t opening = int64_t(gap_open) + int64_t(gap_ext);
  m = std::max<uint64_t>(m, uint64_t(std::llabs(opening)));
  m = std::max<uint64_t>(m, uint64_t(std::llabs(int64_t(gap_ext))));
  return m;
}

HostGraph HostGraph::parse(const int32_t *rec) {
  HostGraph g;
  g.n = rec[0];
  const int64_t in_e = rec[1], out_e = rec[2];
  const int n_paths = rec[3];
  const int path_used = rec[4];
  g.n_rank = rec[5];
  g.sigma = rec[6];
  const int n = g.n;
  const int32_t *p = rec + 7;
  auto take = [&](std::vector<int32_t> &v, int64_t cnt) {
    v.assign(p, p + cnt);
    p += cnt;
  };
  take(g.base, n);
  take(g.parent, n);
  take(g.rank, n);
  take(g.coverage, n);
  take(g.aligned, int64_t(n) * g.sigma);
  take(g.rank_to_node, g.n_rank);
  std::vector<int32_t> icnt, ocnt;
  take(icnt, n);
  take(ocnt, n);
  g.in_off.assign(size_t(n) + 1, 0);
  g.out_off.assign(size_t(n) + 1, 0);
  for (int i = 0; i < n; ++i) {
    g.in_off[i + 1] = g.in_off[i] + icnt[i];
    g.out_off[i + 1] = g.out_off[i] + ocnt[i];
  }
  g.in_id.resize(size_t(in_e));
  g.in_w.resize(size_t(in_e));
  for (int64_t k = 0; k < in_e; ++k) {
    g.in_id[k] = p[2 * k];
    g.in_w[k] = p[2 * k + 1];
  }
  p += 2 * in_e;
  g.out_id.resize(size_t(out_e));
  g.out_w.resize(size_t(out_e));
  for (int64_t k = 0; k < out_e; ++k) {
    g.out_id[k] = p[2 * k];
    g.out_w[k] = p[2 * k + 1];
  }
  p += 2 * out_e;
  take(g.path_seq, n_paths);
  g.path_off.resize(size_t(n_paths) + 1);
  for (int i = 0; i <= n_paths; ++i) g.path_off[i] = p[i];
  p += n_paths + 1;
  take(g.path_items, path_used);
  return g;
}

// Heaviest incoming edge over a FIFO Kahn walk from the source; ties go to
// the higher accumulated score, then the lower incoming index. Coverage of a
// node is max(coverage, sum of outgoing weights).
void HostGraph::consensus(const HostParams &p, std::vector<uint8_t> &seq, std::vector<int64_t> &ids,
                          std::vector<int64_t> &cov) const {
  std::vector<int64_t> degree(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) degree[i] = in_off[i + 1] - in_off[i];
  std::deque<int> queue{0};
  std::vector<int> previous(size_t(n), -1);
  std::vector<uint64_t> score(size_t(n), 0);
  while (!queue.empty()) {
    const int id = queue.front();
    queue.pop_front();
    if (id != 0) {
      int64_t best = -1;
      for (int64_t k = in_off[id]; k < in_off[id + 1]; ++k) {
        if (best < 0) {
          best = k;
          continue;
        }
        const int32_t wb = in_w[best], wk = in_w[k];
        const uint64_t sb = score[in_id[best]], sk = score[in_id[k]];
        // replace on a strictly heavier edge or, at equal weight, a strictly
        // higher score; the earlier index wins full ties.
        if (wk > wb || (wk == wb && sk > sb)) best = k;
      }
      if (best >= 0) {
        previous[id] = in_id[best];
        score[id] = score[in_id[best]] + uint64_t(in_w[best]);
      }
    }
    if (id == 1) break;
    for (int64_t k = out_off[id]; k < out_off[id + 1]; ++k) {
      const int next = out_id[k];
      if (--degree[next] == 0) queue.push_back(next);
    }
  }
  ids.clear();
  for (int cur = previous[1]; cur >= 0 && cur != 0; cur = previous[cur]) ids.push_back(cur);
  std::reverse(ids.begin(), ids.end());
  seq.clear();
  cov.clear();
  for (int64_t i : ids) {
    seq.push_back(p.decode(base[i]));
    int64_t s = 0;
    for (int64_t k = out_off[i]; k < out_off[i + 1]; ++k) s += out_w[k];
    cov.push_back(std::max<int64_t>(coverage[i], s));
  }
}

bool HostGraph::grouped_ranks(std::vector<int32_t> &node_rank, std::vector<int32_t> &order,
                              std::string &err) const {
  std::vector<int64_t> degree(size_t(n), 0);
  std::vector<int> stack;
  node_rank.assign(size_t(n), 0);
  order.clear();
  for (int id = 0; id < n; ++id) {
    if (parent[id] != id) continue;
    int64_t d = 0;
    for (int c = 0; c < sigma; ++c) {
      const int a = aligned[int64_t(id) * sigma + c];
      if (a >= 0) d += in_off[a + 1] - in_off[a];
    }
    degree[id] = d;
    if (d == 0) stack.push_back(id);
  }
  int64_t visited = 0;
  while (!stack.empty()) {
    const int id = stack.back();
    stack.pop_back();
    const int r = int(order.size());
    order.push_back(id);
    for (int c = 0; c < sigma; ++c) {
      const int member = aligned[int64_t(id) * sigma + c];
      if (member < 0) continue;
      node_rank[member] = r;
      ++visited;
      for (int64_t k = out_off[member]; k < out_off[member + 1]; ++k) {
        const int next = parent[out_id[k]];
        if (degree[next] == 0) {
          err = "invalid graph column dependencies";
          return false;
        }
        if (--degree[next] == 0) stack.push_back(next);
      }
    }
  }
  if (visited != n) {
    err = "graph contains a cycle (possibly between alignment columns)";
    return false;
  }
  return true;
}

bool HostGraph::msa(const HostParams &p, const std::vector<std::string> &names,
                    const std::vector<std::string> &comments, std::string &out, std::string &err) const {
  out.clear();
  const int n_paths = int(path_seq.size());
  if (n_paths == 0) return true;
  std::vector<int32_t> node_rank, order;
  if (!grouped_ranks(node_rank, order, err)) return false;
  const size_t width = order.size() >= 2 ? order.size() - 2 : 0;
  for (int pi = 0; pi < n_paths; ++pi) {
    const int sid = path_seq[pi];
    if (sid < 0 || size_t(sid) >= names.size()) {
      err = "unknown sequence ID in graph path";
      return false;
    }
    std::string row(width, '-');
    for (int64_t k = path_off[pi]; k < path_off[pi + 1]; ++k) {
      const int id = path_items[k];
      const size_t r = size_t(node_rank[parent[id]]);
      if (r == 0 || r > width) {
        err = "graph path is outside MSA columns";
        return false;
      }
      row[r - 1] = char(p.decode(base[id]));
    }
    out += '>';
    out += names[size_t(sid)];
    out += ' ';
    out += comments[size_t(sid)];
    out += '\n';
    out += row;
    out += '\n';
  }
  return true;
}

bool HostGraph::gfa(const HostParams &p, const std::vector<std::string> &names, std::string &out,
                    std::string &err) const {
  out.clear();
  const int n_paths = int(path_seq.size());
  if (n <= 2 && n_paths == 0) return true;
  out = "H\tVN:Z:1.0\n";
  std::vector<int64_t> degree(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) degree[i] = in_off[i + 1] - in_off[i];
  std::deque<int> queue{0};
  char buf[64];
  while (!queue.empty()) {
    const int id = queue.front();
    queue.pop_front();
    if (id == 1) break;
    if (id >= 2) {
      int len = snprintf(buf, sizeof buf, "S\t%d\t%c\n", id - 1, char(p.decode(base[id])));
      out.append(buf, size_t(len));
      for (int64_t k = in_off[id]; k < in_off[id + 1]; ++k) {
        const int prev = in_id[k];
        if (prev != 0) {
          len = snprintf(buf, sizeof buf, "L\t%d\t+\t%d\t+\t0M\n", prev - 1, id - 1);
          out.append(buf, size_t(len));
        }
      }
    }
    for (int64_t k = out_off[id]; k < out_off[id + 1]; ++k) {
      const int next = out_id[k];
      if (--degree[next] == 0) queue.push_back(next);
    }
  }
  for (int pi = 0; pi < n_paths; ++pi) {
    const int sid = path_seq[pi];
    if (sid < 0 || size_t(sid) >= names.size()) {
      err = "unknown sequence ID in graph path";
      return false;
    }
    out += "P\t";
    out += names[size_t(sid)];
    out += '\t';
    if (path_off[pi] == path_off[pi + 1]) out += '*';
    for (int64_t k = path_off[pi]; k < path_off[pi + 1]; ++k) {
      if (k > path_off[pi]) out += ',';
      const int len = snprintf(buf, sizeof buf, "%d+", path_items[k] - 1);
      out.append(buf, size_t(len));
    }
    out += "\t*\n";
  }
  return true;
}

}  // namespace poa

namespace poa {

// graph.rs:125-178 with grouped = false, as the device toposort: in-degrees
// from the incoming lists, zero-degree nodes pushed in id order, successors
// in outgoing order.
int32_t HostGraph::lifo_order() {
  std::vector<int32_t> deg(static_cast<size_t>(n)), stack;
  stack.reserve(size_t(n));
  for (int id = 0; id < n; ++id) {
    deg[size_t(id)] = int32_t(in_off[size_t(id) + 1] - in_off[size_t(id)]);
    if (deg[size_t(id)] == 0) stack.push_back(id);
  }
  rank.assign(size_t(n), 0);
  rank_to_node.clear();
  while (!stack.empty()) {
    const int id = stack.back();
    stack.pop_back();
    rank[size_t(id)] = int32_t(rank_to_node.size());
    rank_to_node.push_back(id);
    for (int64_t k = out_off[size_t(id)]; k < out_off[size_t(id) + 1]; ++k) {
      const int next = out_id[size_t(k)];
      if (deg[size_t(next)] == 0) {
        n_rank = int(rank_to_node.size());
        return 13;  // column dependencies (graph.rs:164-166)
      }
      if (--deg[size_t(next)] == 0) stack.push_back(next);
    }
  }
  n_rank = int(rank_to_node.size());
  return n_rank == n ? 0 : 12;  // cycle (graph.rs:174-176)
}

}  // namespace poa
