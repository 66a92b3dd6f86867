// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of minipoa-rs's partial-order-alignment path, used as the
// checker for the GPU library and as the timed CPU baseline. Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load it. Each
// function cites the reference file:line it restates (paths are within the
// minipoa-rs project).
//
// Parity pinning: the reference crate cannot be built here (src/io.rs is
// missing and there is no Rust toolchain), so this restatement is pinned by the
// reference's own known-answer and property tests, restated under tests/.
#include "oracle.h"

#include <immintrin.h>

#include <algorithm>
#include <map>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <optional>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace orc {

using i64 = int64_t;
using i32 = int32_t;
using usize = uint64_t;

constexpr i64 NEG = -(i64(1) << 50);  // align.rs:16
constexpr usize WIDTH = 8;            // align.rs:17
constexpr uint8_t MATCH = 1, DELETE = 2, INSERT = 4, ALL = 7;  // align.rs:20-23
constexpr i32 NEG32 = -(1 << 29);                               // align.rs:216
constexpr uint64_t SCORE_LIMIT = uint64_t(1) << 26;             // align.rs:217
constexpr i32 SHIFT_FILL = NEG32 - 2 * i32(SCORE_LIMIT);        // align.rs:220

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

static thread_local std::string g_error;
static thread_local uint64_t g_cells = 0;

// lib.rs:47-138
struct Params {
  i32 match_score = 2, mismatch = -4, gap_open = -4, gap_ext = -2;
  usize b = 100, f = 40;
  bool adaptive = false, seeding = false;
  usize k = 19, w = 10;
  bool progressive = false;
  usize threads = 1, win_band = 500, win_max = 10000;
  double mm_filter_ratio = 0.25;
  usize max_occ = 0, tr_dist = 1000;
  uint8_t result = 0, verbose = 0;
  std::vector<uint8_t> alphabet;
  std::vector<i32> matrix;
  bool is_rna = false;

  static Params from(const orc_params *p) {
    Params r;
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
    r.result = uint8_t(p->result);
    r.threads = p->threads;
    r.win_band = p->win_band;
    r.win_max = p->win_max;
    r.mm_filter_ratio = p->mm_filter_ratio;
    r.max_occ = p->max_occ;
    r.tr_dist = p->tr_dist;
    r.verbose = uint8_t(p->verbose);
    r.is_rna = p->is_rna != 0;
    if (p->alphabet_len > 0 && p->alphabet) r.alphabet.assign(p->alphabet, p->alphabet + p->alphabet_len);
    usize n2 = usize(std::max(p->alphabet_len, 0)) * usize(std::max(p->alphabet_len, 0));
    if (n2 && p->matrix) r.matrix.assign(p->matrix, p->matrix + n2);
    return r;
  }
  // lib.rs:110-126
  usize encode(uint8_t base) const {
    if (base >= 'a' && base <= 'z') base = uint8_t(base - 32);
    if (alphabet.size() <= 5 && base == 'U') base = 'T';
    for (usize i = 0; i < alphabet.size(); ++i)
      if (alphabet[i] == base) return i;
    for (usize i = 0; i < alphabet.size(); ++i)
      if (alphabet[i] == 'N') return i;
    return alphabet.size() - 1;
  }
  // lib.rs:127-134
  uint8_t decode(usize base) const {
    uint8_t c = alphabet[base];
    if (is_rna && alphabet.size() <= 5 && c == 'T') return 'U';
    return c;
  }
  // lib.rs:135-137
  i32 score(usize a, usize b) const { return matrix[a * alphabet.size() + b]; }
  // lib.rs:149-173
  void validate() const {
    usize n = alphabet.size();
    if (n == 0 || n > 256 || matrix.size() != n * n) throw Error("invalid scoring matrix dimensions");
    if (threads == 0) throw Error("thread count must be positive");
    if (!(k >= 1 && k <= 31) || !(w >= 1 && w < 32768))
      throw Error("k must be 1..31 and minimizer window must be 1..32767");
    if (gap_open > 0 || gap_ext > 0) throw Error("gap penalties must be zero or negative");
    if (result > 2 || verbose > 2) throw Error("result format and verbosity must be 0..2");
    if (!(mm_filter_ratio == mm_filter_ratio) || mm_filter_ratio < 0.0 || mm_filter_ratio > 1.0 ||
        mm_filter_ratio == 1.0 / 0.0)
      throw Error("minimizer filter ratio must be between 0 and 1");
    if (win_max == 0) throw Error("window maximum must be positive");
  }
};

constexpr i64 NONE = -1;

// lib.rs:140-145
struct AlignedBase {
  i64 node;  // NONE = None
  usize base;
  i64 aligned;
};

// graph.rs:6-18
struct Node {
  usize id = 0, rank = 0, parent = 0, base = 0;
  std::vector<usize> incoming, in_weights, outgoing, out_weights;
  std::vector<i64> aligned;
  usize coverage = 0;
};

// graph.rs:20-27
struct Graph {
  std::vector<Node> nodes;
  std::vector<usize> rank;
  std::vector<std::pair<usize, std::vector<usize>>> paths;
  usize alphabet_size = 0;

  // graph.rs:30-40
  explicit Graph(const Params &p) : alphabet_size(p.alphabet.size()) {
    add_node(p.encode('N'));
    add_node(p.encode('N'));
  }
  Graph() = default;

  // graph.rs:42-59
  usize add_node(usize base) {
    usize id = nodes.size();
    Node n;
    n.id = id;
    n.parent = id;
    n.base = base;
    n.aligned.assign(alphabet_size, NONE);
    n.aligned[base] = i64(id);
    nodes.push_back(std::move(n));
    return id;
  }

  // graph.rs:62-79
  void add_edge(usize from, usize to) {
    if (from == to) return;
    auto &out = nodes[from].outgoing;
    auto it = std::find(out.begin(), out.end(), to);
    if (it != out.end()) {
      nodes[from].out_weights[usize(it - out.begin())] += 1;
    } else {
      out.push_back(to);
      nodes[from].out_weights.push_back(1);
    }
    auto &in = nodes[to].incoming;
    auto jt = std::find(in.begin(), in.end(), from);
    if (jt != in.end()) {
      nodes[to].in_weights[usize(jt - in.begin())] += 1;
    } else {
      in.push_back(from);
      nodes[to].in_weights.push_back(1);
    }
    nodes[to].coverage += 1;
  }

  // graph.rs:82-122
  void add_path(usize seq_id, const std::vector<AlignedBase> &alignment) {
    for (auto &item : alignment) {
      if (item.base >= alphabet_size) throw Error("alignment base outside alphabet");
      if ((item.node != NONE && usize(item.node) >= nodes.size()) ||
          (item.aligned != NONE && usize(item.aligned) >= nodes.size()))
        throw Error("alignment references an unknown node");
    }
    std::optional<usize> previous;
    std::vector<usize> path;
    path.reserve(alignment.size());
    for (auto &item : alignment) {
      usize id;
      if (item.node != NONE) {
        id = usize(item.node);
      } else if (item.aligned != NONE) {
        usize parent = nodes[usize(item.aligned)].parent;
        if (nodes[parent].aligned[item.base] != NONE) {
          id = usize(nodes[parent].aligned[item.base]);
        } else {
          id = add_node(item.base);
          nodes[id].parent = parent;
          nodes[parent].aligned[item.base] = i64(id);
        }
      } else {
        id = add_node(item.base);
      }
      if (previous) add_edge(*previous, id);
      previous = id;
      if (id >= 2) path.push_back(id);
    }
    add_edge(previous ? *previous : 0, 1);
    paths.emplace_back(seq_id, std::move(path));
  }

  // graph.rs:125-178
  void toposort(bool grouped) {
    std::vector<usize> degree(nodes.size(), 0);
    std::vector<usize> stack;
    for (auto &n : nodes) {
      if (grouped && n.parent != n.id) continue;
      if (grouped) {
        usize s = 0;
        for (i64 a : n.aligned)
          if (a != NONE) s += nodes[usize(a)].incoming.size();
        degree[n.id] = s;
      } else {
        degree[n.id] = n.incoming.size();
      }
      if (degree[n.id] == 0) stack.push_back(n.id);
    }
    rank.clear();
    usize visited = 0;
    while (!stack.empty()) {
      usize id = stack.back();
      stack.pop_back();
      usize r = rank.size();
      rank.push_back(id);
      usize single = id;
      const usize *mem_begin = &single, *mem_end = &single + 1;
      std::vector<usize> members;
      if (grouped) {
        for (i64 a : nodes[id].aligned)
          if (a != NONE) members.push_back(usize(a));
        mem_begin = members.data();
        mem_end = members.data() + members.size();
      }
      for (const usize *mp = mem_begin; mp != mem_end; ++mp) {
        usize member = *mp;
        nodes[member].rank = r;
        visited += 1;
        for (usize next : nodes[member].outgoing) {
          usize nx = grouped ? nodes[next].parent : next;
          if (degree[nx] == 0) throw Error("invalid graph column dependencies");
          degree[nx] -= 1;
          if (degree[nx] == 0) stack.push_back(nx);
        }
      }
    }
    if (visited != nodes.size()) throw Error("graph contains a cycle (possibly between alignment columns)");
  }

  // graph.rs:181-237
  void consensus(const Params &p, std::vector<uint8_t> &seq, std::vector<usize> &ids,
                 std::vector<usize> &coverage) const {
    std::vector<usize> degree(nodes.size());
    for (usize i = 0; i < nodes.size(); ++i) degree[i] = nodes[i].incoming.size();
    std::deque<usize> queue{0};
    std::vector<i64> previous(nodes.size(), NONE);
    std::vector<usize> score(nodes.size(), 0);
    while (!queue.empty()) {
      usize id = queue.front();
      queue.pop_front();
      const Node &node = nodes[id];
      if (id != 0) {
        // max_by keeps the LAST maximum under the comparator
        // (weight, score, then reversed index), i.e. heaviest edge, then the
        // higher accumulated score, then the lowest index.
        i64 best = -1;
        for (usize k = 0; k < node.incoming.size(); ++k) {
          if (best < 0) {
            best = i64(k);
            continue;
          }
          usize a = node.incoming[usize(best)], b = node.incoming[k];
          usize ai = usize(best), bi = k;
          // compare(best, k): Ordering of best relative to k
          int c;
          if (node.in_weights[ai] != node.in_weights[bi])
            c = node.in_weights[ai] < node.in_weights[bi] ? -1 : 1;
          else if (score[a] != score[b])
            c = score[a] < score[b] ? -1 : 1;
          else
            c = bi < ai ? -1 : (bi > ai ? 1 : 0);
          if (c <= 0) best = i64(k);  // max_by returns the last of equal maxima
        }
        if (best >= 0) {
          usize pp = node.incoming[usize(best)];
          previous[id] = i64(pp);
          score[id] = score[pp] + node.in_weights[usize(best)];
        }
      }
      if (id == 1) break;
      for (usize next : node.outgoing) {
        degree[next] -= 1;
        if (degree[next] == 0) queue.push_back(next);
      }
    }
    ids.clear();
    i64 cur = previous[1];
    while (cur != NONE) {
      if (cur == 0) break;
      ids.push_back(usize(cur));
      cur = previous[usize(cur)];
    }
    std::reverse(ids.begin(), ids.end());
    seq.clear();
    coverage.clear();
    for (usize i : ids) {
      seq.push_back(p.decode(nodes[i].base));
      usize s = 0;
      for (usize w : nodes[i].out_weights) s += w;
      coverage.push_back(std::max(nodes[i].coverage, s));
    }
  }

  // graph.rs:239-253
  std::string msa(const Params &p, const std::vector<std::string> &names, const std::vector<std::string> &comments) {
    if (paths.empty()) return std::string();
    auto saved_rank = rank;
    std::vector<usize> node_ranks(nodes.size());
    for (usize i = 0; i < nodes.size(); ++i) node_ranks[i] = nodes[i].rank;
    std::string result;
    std::string err;
    try {
      toposort(true);
      result = msa_grouped(p, names, comments);
    } catch (const Error &e) {
      err = e.what();
    }
    rank = saved_rank;
    for (usize i = 0; i < nodes.size(); ++i) nodes[i].rank = node_ranks[i];
    if (!err.empty()) throw Error(err);
    return result;
  }

  // graph.rs:255-279
  std::string msa_grouped(const Params &p, const std::vector<std::string> &names,
                          const std::vector<std::string> &comments) const {
    std::string out;
    usize width = rank.size() >= 2 ? rank.size() - 2 : 0;
    for (auto &pr : paths) {
      usize sid = pr.first;
      if (sid >= names.size()) throw Error("unknown sequence ID in graph path");
      std::string row(width, '-');
      for (usize id : pr.second) {
        usize r = nodes[nodes[id].parent].rank;
        if (r == 0 || r > width) throw Error("graph path is outside MSA columns");
        row[r - 1] = char(p.decode(nodes[id].base));
      }
      out += ">";
      out += names[sid];
      out += " ";
      out += comments[sid];
      out += "\n";
      out += row;
      out += "\n";
    }
    return out;
  }

  // graph.rs:281-331
  std::string gfa(const Params &p, const std::vector<std::string> &names) const {
    if (nodes.size() <= 2 && paths.empty()) return std::string();
    std::string out = "H\tVN:Z:1.0\n";
    std::vector<usize> degree(nodes.size());
    for (usize i = 0; i < nodes.size(); ++i) degree[i] = nodes[i].incoming.size();
    std::deque<usize> queue{0};
    while (!queue.empty()) {
      usize id = queue.front();
      queue.pop_front();
      if (id == 1) break;
      const Node &node = nodes[id];
      if (id >= 2) {
        out += "S\t" + std::to_string(id - 1) + "\t";
        out += char(p.decode(node.base));
        out += "\n";
        for (usize prev : node.incoming)
          if (prev != 0) out += "L\t" + std::to_string(prev - 1) + "\t+\t" + std::to_string(id - 1) + "\t+\t0M\n";
      }
      for (usize next : node.outgoing) {
        degree[next] -= 1;
        if (degree[next] == 0) queue.push_back(next);
      }
    }
    for (auto &pr : paths) {
      if (pr.first >= names.size()) throw Error("unknown sequence ID in graph path");
      out += "P\t" + names[pr.first] + "\t";
      if (pr.second.empty()) out += "*";
      for (usize i = 0; i < pr.second.size(); ++i) {
        if (i > 0) out += ",";
        out += std::to_string(pr.second[i] - 1) + "+";
      }
      out += "\t*\n";
    }
    return out;
  }
};

// ---------------------------------------------------------------------------
// DP matrices and the traceback (align.rs:25-77, 228-353, 1164-1347)

// align.rs:25-77
struct Row {
  usize start = 0;
  std::vector<i64> m, d, ins;
  bool contains(usize j) const { return j >= start && j - start < m.size(); }
  i64 M(usize j) const { return contains(j) ? m[j - start] : NEG; }
  i64 D(usize j) const { return contains(j) ? d[j - start] : NEG; }
  i64 I(usize j) const { return contains(j) ? ins[j - start] : NEG; }
};

struct I64Matrix {
  const std::vector<Row> &rows;
  bool contains_at(usize r, usize c) const { return rows[r].contains(c); }
  i64 m_at(usize r, usize c) const { return rows[r].M(c); }
  i64 d_at(usize r, usize c) const { return rows[r].D(c); }
  i64 i_at(usize r, usize c) const { return rows[r].I(c); }
  i64 negative() const { return NEG; }
};

// align.rs:228-274, 302-334
struct FastRow {
  usize start = 0, len = 0, m_offset = 0, d_offset = 0, i_offset = 0;
};

struct FastMatrix {
  std::vector<i32> &data;
  std::vector<FastRow> rows;
  usize cursor = 0;

  FastRow allocate(usize start, usize stop) {
    if (stop < start) throw Error("invalid alignment band");
    usize len = stop - start;
    usize size = len * 3 + WIDTH * 2;
    usize end = cursor + size;
    if (end > data.size()) data.resize(end, NEG32);
    FastRow row{start, len, cursor + WIDTH, cursor + WIDTH * 2 + len, cursor + WIDTH * 2 + len * 2};
    std::fill(data.begin() + i64(cursor), data.begin() + i64(row.d_offset + len), NEG32);
    cursor = end;
    return row;
  }
  bool contains_at(usize r, usize c) const {
    const FastRow &row = rows[r];
    return c >= row.start && c - row.start < row.len;
  }
  i64 m_at(usize r, usize c) const {
    const FastRow &row = rows[r];
    return contains_at(r, c) ? i64(data[row.m_offset + c - row.start]) : i64(NEG32);
  }
  i64 d_at(usize r, usize c) const {
    const FastRow &row = rows[r];
    return contains_at(r, c) ? i64(data[row.d_offset + c - row.start]) : i64(NEG32);
  }
  i64 i_at(usize r, usize c) const {
    const FastRow &row = rows[r];
    return contains_at(r, c) ? i64(data[row.i_offset + c - row.start]) : i64(NEG32);
  }
  i64 negative() const { return i64(NEG32); }
};

// align.rs:1316-1347
static void push_diagonal(std::vector<AlignedBase> &result, const Graph &graph, usize i, usize n, usize j, usize m,
                          usize query_base, usize node_id, usize node_base) {
  if (i == n - 1 && j != m - 1) {
    result.push_back({NONE, query_base, NONE});
  } else if (node_base == query_base) {
    result.push_back({i64(node_id), graph.nodes[node_id].base, NONE});
  } else {
    usize parent = graph.nodes[node_id].parent;
    result.push_back({graph.nodes[parent].aligned[query_base], query_base, i64(parent)});
  }
}

// align.rs:1164-1313
template <class Mx>
static std::vector<AlignedBase> traceback(const Params &params, const Graph &graph, usize beg, usize n,
                                          const std::vector<usize> &seq, usize m, const std::vector<i64> &head,
                                          const Mx &rows, i64 gap_open, i64 gap_ext) {
  usize i = n - 1, j = m - 1;
  uint8_t op = ALL;
  std::vector<AlignedBase> result;
  result.reserve(m);
  usize steps = 0;
  const usize unknown = params.encode('N');
  while (i > 0 || j > 0) {
    steps += 1;
    if (steps > n + m) throw Error("alignment traceback failed to advance");
    if (!rows.contains_at(i, j) || rows.m_at(i, j) <= rows.negative() / 2)
      throw Error("alignment traceback left active band");
    const Node &node = graph.nodes[graph.rank[beg + i]];
    usize base = (i == n - 1) ? unknown : node.base;
    i64 score = i64(params.score(base, seq[j]));
    auto choose = [&](uint8_t state, i64 penalty, usize previous_j) -> i64 {
      i64 best = -1;
      usize weight = 0;
      for (usize k = 0; k < node.incoming.size(); ++k) {
        usize r = graph.nodes[node.incoming[k]].rank;
        if (r < beg || r >= beg + i) continue;
        usize p = r - beg;
        if (head[p] == NEG || !rows.contains_at(p, previous_j)) continue;
        i64 source = state == DELETE ? rows.d_at(p, previous_j) : rows.m_at(p, previous_j);
        i64 target = state == MATCH ? rows.m_at(i, j) : rows.d_at(i, j);
        if (target == source + penalty && (best < 0 || node.in_weights[k] > weight)) {
          best = i64(k);
          weight = node.in_weights[k];
        }
      }
      return best;
    };
    i64 preferred = -1;
    if ((op & MATCH) && j > 0 && base == seq[j]) preferred = choose(MATCH, score, j - 1);
    if (preferred >= 0) {
      usize total = 0;
      for (usize w : node.in_weights) total += w;
      if (!(node.in_weights[usize(preferred)] >= total / 10)) preferred = -1;
    }
    if (preferred >= 0) {
      push_diagonal(result, graph, i, n, j, m, seq[j], node.id, base);
      i = graph.nodes[node.incoming[usize(preferred)]].rank - beg;
      j -= 1;
      op = ALL;
      continue;
    }
    if ((op & DELETE) && (op == DELETE || rows.m_at(i, j) == rows.d_at(i, j))) {
      i64 k = choose(INSERT, gap_open, j);
      if (k >= 0) {
        i = graph.nodes[node.incoming[usize(k)]].rank - beg;
        op = params.gap_open == 0 ? ALL : uint8_t(MATCH | INSERT);
        continue;
      }
      k = choose(DELETE, gap_ext, j);
      if (k >= 0) {
        i = graph.nodes[node.incoming[usize(k)]].rank - beg;
        op = DELETE;
        continue;
      }
    }
    if ((op & INSERT) && j > 0 && rows.contains_at(i, j - 1) && (op == INSERT || rows.m_at(i, j) == rows.i_at(i, j))) {
      if (rows.i_at(i, j) == rows.m_at(i, j - 1) + gap_open) {
        result.push_back({NONE, seq[j], NONE});
        j -= 1;
        op = params.gap_open == 0 ? ALL : uint8_t(MATCH | DELETE);
        continue;
      }
      if (rows.i_at(i, j) == rows.i_at(i, j - 1) + gap_ext) {
        result.push_back({NONE, seq[j], NONE});
        j -= 1;
        op = INSERT;
        continue;
      }
    }
    if ((op & MATCH) && j > 0) {
      i64 k = choose(MATCH, score, j - 1);
      if (k >= 0) {
        push_diagonal(result, graph, i, n, j, m, seq[j], node.id, base);
        i = graph.nodes[node.incoming[usize(k)]].rank - beg;
        j -= 1;
        op = ALL;
        continue;
      }
    }
    throw Error("alignment traceback has no predecessor at graph row " + std::to_string(i) + ", query column " +
                std::to_string(j));
  }
  usize start = graph.rank[beg];
  result.push_back({i64(start), graph.nodes[start].base, NONE});
  std::reverse(result.begin(), result.end());
  result.pop_back();
  return result;
}

// ---------------------------------------------------------------------------
// Shared setup of both kernels (align.rs:598-687 and 922-1011)

struct Setup {
  usize beg = 0, end = 0, n = 0, m = 0, unknown = 0, padded = 0;
  std::vector<usize> seq;
  bool adaptive = false;
  i64 band = 0;
  std::vector<i64> head, tail, support;
};

static Setup setup(const Params &params, const Graph &graph, usize beg_id, usize end_id, const uint8_t *query,
                   usize qlen, bool adaptive, usize band_b) {
  Setup s;
  if (beg_id >= graph.nodes.size() || end_id >= graph.nodes.size()) throw Error("alignment anchor is not in graph");
  s.beg = graph.nodes[beg_id].rank;
  s.end = graph.nodes[end_id].rank;
  if (s.end <= s.beg || s.end >= graph.rank.size()) throw Error("alignment anchors are not topologically ordered");
  s.n = s.end - s.beg + 1;
  s.m = qlen + 2;
  if (s.n > usize(INT32_MAX) || s.m > usize(INT32_MAX)) throw Error("alignment exceeds coordinate limits");
  s.unknown = params.encode('N');
  s.padded = (s.m / WIDTH + 1) * WIDTH;
  s.seq.reserve(s.padded);
  s.seq.push_back(s.unknown);
  for (usize i = 0; i < qlen; ++i) s.seq.push_back(params.encode(query[i]));
  s.seq.resize(s.padded, s.unknown);
  s.adaptive = adaptive || params.adaptive;
  usize add = params.f == 0 ? 0 : s.m / params.f;
  usize band = band_b + add < band_b ? UINT64_MAX : band_b + add;  // saturating_add
  s.band = i64(std::min<usize>(band, usize(INT32_MAX)));
  const usize n = s.n, beg = s.beg, end = s.end;
  s.head.assign(n, NEG);
  s.tail.assign(n, NEG);
  s.support.assign(n, 0);
  s.head[0] = 0;
  for (usize i = 1; i < n; ++i) {
    const Node &node = graph.nodes[graph.rank[beg + i]];
    bool have = false;
    usize bp = 0, bw = 0;
    for (usize k = 0; k < node.incoming.size(); ++k) {
      usize r = graph.nodes[node.incoming[k]].rank;
      if (r < beg || r >= beg + i) continue;
      usize p = r - beg;
      if (s.head[p] == NEG) continue;
      if (!have || node.in_weights[k] > bw || (node.in_weights[k] == bw && s.support[p] > s.support[bp])) {
        have = true;
        bp = p;
        bw = node.in_weights[k];
      }
    }
    if (have) {
      s.head[i] = s.head[bp] + 1;
      s.support[i] = s.support[bp] + i64(bw);
    }
  }
  s.tail[n - 1] = 1;
  for (usize ii = n - 1; ii-- > 0;) {
    usize i = ii;
    const Node &node = graph.nodes[graph.rank[beg + i]];
    bool have = false;
    usize bs = 0, bw = 0;
    for (usize k = 0; k < node.outgoing.size(); ++k) {
      usize r = graph.nodes[node.outgoing[k]].rank;
      if (r <= beg + i || r > end) continue;
      usize sx = r - beg;
      if (s.tail[sx] == NEG) continue;
      if (!have || node.out_weights[k] > bw || (node.out_weights[k] == bw && s.support[sx] > s.support[bs])) {
        have = true;
        bs = sx;
        bw = node.out_weights[k];
      }
    }
    if (have) {
      s.tail[i] = s.tail[bs] + 1;
      s.support[i] = s.support[bs] + i64(bw);
    }
  }
  if (s.head[n - 1] == NEG) throw Error("no graph path connects alignment anchors");
  return s;
}

struct Adaptive {
  std::vector<i64> peak, streak, peak_left, peak_right, offset_left, offset_right, extra;
  Adaptive(usize n, usize m)
      : peak(n, 0), streak(n, 0), peak_left(n, i64(m)), peak_right(n, 0), offset_left(n, 0), offset_right(n, 0),
        extra(n, 0) {}
};

// align.rs:711-734 / 1017-1040: band bounds of row i, 8-rounded.
static void row_band(const Params &params, const Setup &s, const Adaptive &a, usize i, usize &start, usize &stop) {
  const i64 m = i64(s.m);
  i64 left, right;
  if (params.f == 0) {
    left = 0;
    right = m;
  } else if (s.adaptive) {
    i64 x = std::min(std::min(a.peak_left[i], s.head[i] + a.offset_left[i]), m - s.tail[i]);
    i64 y = std::max(std::max(a.peak_right[i], s.head[i] + a.offset_right[i]), m - s.tail[i]);
    left = std::max<i64>(x - s.band - a.extra[i], 0);
    right = std::min<i64>(y + s.band + a.extra[i], m);
  } else {
    left = std::max<i64>(std::min(s.head[i], m - s.tail[i]) - s.band, 0);
    right = std::min<i64>(std::max(s.head[i], m - s.tail[i]) + s.band, m);
  }
  if (left > right || right < 0) throw Error("alignment band does not intersect graph path");
  start = usize(left) / WIDTH * WIDTH;
  stop = (usize(right) / WIDTH + 1) * WIDTH;
}

// align.rs:829-897 / 1087-1147: band state update after row i with its argmax.
static void adaptive_update(const Graph &graph, const Setup &s, Adaptive &a, usize i, i64 maximum) {
  const usize beg = s.beg, end = s.end;
  const Node &node = graph.nodes[graph.rank[beg + i]];
  a.peak[i] = maximum;
  i64 max_streak = 0;
  bool is_match = false;
  if (node.base == s.seq[usize(maximum)]) {
    for (usize pred : node.incoming) {
      usize r = graph.nodes[pred].rank;
      if (r < beg || r >= beg + i) continue;
      usize p = r - beg;
      if (s.head[p] == NEG) continue;
      max_streak = std::max(max_streak, a.streak[p]);
      if (a.peak[p] + 1 == maximum) {
        a.streak[i] = std::max(a.streak[i], a.streak[p] + 1);
        is_match = true;
      }
    }
  }
  if (!is_match && max_streak < 30) a.extra[i] = std::min(a.extra[i] + max_streak + 1, 5 * s.band);
  if (a.streak[i] >= 30) {
    a.offset_left[i] = maximum - s.head[i];
    a.offset_right[i] = maximum - s.head[i];
    a.extra[i] = 0;
    for (usize succ : node.outgoing) {
      usize r = graph.nodes[succ].rank;
      if (r > beg + i && r <= end) {
        usize sx = r - beg;
        a.offset_left[sx] = a.offset_left[i];
        a.offset_right[sx] = a.offset_right[i];
      }
    }
  }
  for (usize succ : node.outgoing) {
    usize r = graph.nodes[succ].rank;
    if (r <= beg + i || r > end) continue;
    usize sx = r - beg;
    a.offset_left[sx] = std::min(a.offset_left[sx], a.offset_left[i]);
    a.offset_right[sx] = std::max(a.offset_right[sx], a.offset_right[i]);
    a.peak_left[sx] = std::min(a.peak_left[sx], maximum);
    a.peak_right[sx] = std::max(a.peak_right[sx], maximum + 1);
    a.extra[sx] = a.extra[i] != 0 ? std::max(a.extra[sx], a.extra[i]) : 0;
  }
}

// ---------------------------------------------------------------------------
// i32 kernel, serial restatement of poa_simd_arena (align.rs:588-911). The
// SIMD code's per-lane arithmetic is reproduced element by element: M/D start
// at NEG32, the predecessor loop runs over the 8-aligned band overlap reading
// the NEG32 pad left of a predecessor row, and the insertion scan starts each
// row at carry NEG32.

static void avx2_row_preds(std::vector<i32> &data, const FastRow &row, const FastRow &prev, i32 open, i32 ext);
static void avx2_row_scan(std::vector<i32> &data, const FastRow &row, const i32 *profile, i32 open, i32 ext);
static i32 avx2_row_max(const i32 *scores, usize len);

static std::vector<AlignedBase> poa_i32(const Params &params, const Graph &graph, usize beg_id, usize end_id,
                                        const uint8_t *query, usize qlen, bool adaptive, usize band_b, bool avx2) {
  static thread_local std::vector<i32> arena;  // align.rs:222-226 (DP_ARENA)
  Setup s = setup(params, graph, beg_id, end_id, query, qlen, adaptive, band_b);
  const usize n = s.n, m = s.m, beg = s.beg, padded = s.padded;
  Adaptive a(n, m);
  const usize alphabet = params.alphabet.size();
  std::vector<i32> profiles(alphabet * padded);
  for (usize base = 0; base < alphabet; ++base)
    for (usize c = 0; c < padded; ++c) profiles[base * padded + c] = params.score(base, s.seq[c]);
  const i32 gap_ext = params.gap_ext;
  const i32 gap_open = params.gap_open + gap_ext;
  FastMatrix mx{arena, std::vector<FastRow>(n), 0};
  for (usize i = 0; i < n; ++i) {
    if (s.head[i] == NEG || s.tail[i] == NEG) continue;
    usize start, stop;
    row_band(params, s, a, i, start, stop);
    FastRow row = mx.allocate(start, stop);
    mx.rows[i] = row;
    g_cells += row.len;
    std::vector<i32> &D = mx.data;
    if (i == 0) {
      if (start != 0) throw Error("alignment band excludes source");
      D[row.m_offset] = params.score(s.unknown, s.unknown);
      D[row.i_offset] = NEG32;
      for (usize j = 1; j < row.len; ++j) {
        i32 ins = std::max(D[row.i_offset + j - 1] + gap_ext, D[row.m_offset + j - 1] + gap_open);
        D[row.i_offset + j] = ins;
        D[row.m_offset + j] = std::max(D[row.m_offset + j], ins);
      }
      continue;
    }
    const Node &node = graph.nodes[graph.rank[beg + i]];
    for (usize pred : node.incoming) {
      usize r = graph.nodes[pred].rank;
      if (r < beg || r >= beg + i) continue;
      usize p = r - beg;
      if (s.head[p] == NEG) continue;
      const FastRow prev = mx.rows[p];
      if (avx2) {
        avx2_row_preds(D, row, prev, gap_open, gap_ext);
        continue;
      }
      usize ov_start = std::max(start, prev.start);
      usize ov_stop = std::min(stop, prev.start + prev.len);
      for (usize j = ov_start; j < ov_stop; ++j) {
        usize local = j - start, prior = j - prev.start;
        i32 diagonal = D[prev.m_offset + prior - 1];  // reads the NEG32 pad when prior == 0
        i32 pm = D[prev.m_offset + prior];
        i32 pd = D[prev.d_offset + prior];
        D[row.m_offset + local] = std::max(D[row.m_offset + local], diagonal);
        D[row.d_offset + local] = std::max(std::max(D[row.d_offset + local], pd + gap_ext), pm + gap_open);
      }
    }
    usize base = (i == n - 1) ? s.unknown : node.base;
    const i32 *profile = &profiles[base * padded];
    if (avx2) {
      avx2_row_scan(D, row, profile + start, gap_open, gap_ext);
    } else {
      i32 carry = NEG32;
      for (usize local = 0; local < row.len; ++local) {
        i32 md = std::max(D[row.m_offset + local] + profile[start + local], D[row.d_offset + local]);
        D[row.i_offset + local] = carry;
        D[row.m_offset + local] = std::max(md, carry);
        carry = std::max(carry + gap_ext, md + gap_open);
      }
    }
    if (params.f != 0 && s.adaptive) {
      const i32 *scores = &D[row.m_offset];
      i32 maximum_score;
      if (avx2) {
        maximum_score = avx2_row_max(scores, row.len);
      } else {
        maximum_score = NEG32;
        for (usize c = 0; c < row.len; ++c) maximum_score = std::max(maximum_score, scores[c]);
      }
      usize argmax = 0;
      while (scores[argmax] != maximum_score) ++argmax;
      adaptive_update(graph, s, a, i, i64(start + argmax));
    }
  }
  return traceback(params, graph, beg, n, s.seq, m, s.head, mx, i64(gap_open), i64(gap_ext));
}

// ---------------------------------------------------------------------------
// i64 kernel (align.rs:913-1162)

static std::vector<AlignedBase> poa_i64(const Params &params, const Graph &graph, usize beg_id, usize end_id,
                                        const uint8_t *query, usize qlen, bool adaptive, usize band_b) {
  Setup s = setup(params, graph, beg_id, end_id, query, qlen, adaptive, band_b);
  const usize n = s.n, m = s.m, beg = s.beg;
  Adaptive a(n, m);
  const i64 gap_ext = params.gap_ext;
  const i64 gap_open = i64(params.gap_open) + gap_ext;
  std::vector<Row> rows(n);
  for (usize i = 0; i < n; ++i) {
    if (s.head[i] == NEG || s.tail[i] == NEG) continue;
    usize start, stop;
    row_band(params, s, a, i, start, stop);
    Row row;
    row.start = start;
    row.m.assign(stop - start, NEG);
    row.d.assign(stop - start, NEG);
    row.ins.assign(stop - start, NEG);
    g_cells += stop - start;
    if (i == 0) {
      if (!row.contains(0)) throw Error("alignment band excludes source");
      row.m[0] = i64(params.score(s.unknown, s.unknown));
      for (usize j = 1; j < row.m.size(); ++j) {
        row.ins[j] = std::max(row.ins[j - 1] + gap_ext, row.m[j - 1] + gap_open);
        row.m[j] = std::max(row.m[j], row.ins[j]);
      }
      rows[i] = std::move(row);
      continue;
    }
    const Node &node = graph.nodes[graph.rank[beg + i]];
    usize base = (i == n - 1) ? s.unknown : node.base;
    for (usize j = start, local = 0; j < stop; ++j, ++local) {
      usize block = j / WIDTH * WIDTH;
      i64 diagonal = NEG, deletion = NEG;
      for (usize pred : node.incoming) {
        usize r = graph.nodes[pred].rank;
        if (r < beg || r >= beg + i) continue;
        usize p = r - beg;
        if (s.head[p] == NEG) continue;
        const Row &prev = rows[p];
        if (!prev.contains(block)) continue;
        if (j > 0) diagonal = std::max(diagonal, prev.M(j - 1));
        deletion = std::max(std::max(deletion, prev.D(j) + gap_ext), prev.M(j) + gap_open);
      }
      row.d[local] = deletion;
      i64 md = std::max(diagonal + i64(params.score(base, s.seq[j])), deletion);
      row.m[local] = std::max(md, row.ins[local]);
      if (local + 1 < row.m.size()) row.ins[local + 1] = std::max(row.ins[local] + gap_ext, md + gap_open);
    }
    if (params.f != 0 && s.adaptive) {
      usize argmax = 0;
      for (usize j = 1; j < row.m.size(); ++j)
        if (row.m[j] > row.m[argmax]) argmax = j;
      adaptive_update(graph, s, a, i, i64(start + argmax));
    }
    rows[i] = std::move(row);
  }
  I64Matrix mx{rows};
  return traceback(params, graph, beg, n, s.seq, m, s.head, mx, gap_open, gap_ext);
}

// ---------------------------------------------------------------------------
// AVX2 8-lane i32 kernel pieces (the timed CPU baseline). They mirror the
// reference's wide::i32x8 organisation (align.rs:459-491, 755-845).

// Lanes shifted up by 1, 2 or 4 with SHIFT_FILL in the vacated low lanes.
__attribute__((target("avx2"))) static inline __m256i shift1(__m256i v, __m256i fill) {
  return _mm256_blend_epi32(_mm256_permutevar8x32_epi32(v, _mm256_setr_epi32(0, 0, 1, 2, 3, 4, 5, 6)), fill, 0x01);
}
__attribute__((target("avx2"))) static inline __m256i shift2(__m256i v, __m256i fill) {
  return _mm256_blend_epi32(_mm256_permutevar8x32_epi32(v, _mm256_setr_epi32(0, 0, 0, 1, 2, 3, 4, 5)), fill, 0x03);
}
__attribute__((target("avx2"))) static inline __m256i shift4(__m256i v, __m256i fill) {
  return _mm256_blend_epi32(_mm256_permutevar8x32_epi32(v, _mm256_setr_epi32(0, 0, 0, 0, 0, 1, 2, 3)), fill, 0x0F);
}

// Three shift stages give the within-block max-plus prefix; the carried-in
// insertion state is added as a broadcast (align.rs:459-491).
__attribute__((target("avx2"))) static inline __m256i insertion_prefix_v(__m256i md, __m256i carryv, i32 open,
                                                                         i32 ext) {
  const __m256i fill = _mm256_set1_epi32(SHIFT_FILL);
  __m256i v = _mm256_add_epi32(md, _mm256_set1_epi32(open));
  v = _mm256_max_epi32(v, _mm256_add_epi32(shift1(v, fill), _mm256_set1_epi32(ext)));
  v = _mm256_max_epi32(v, _mm256_add_epi32(shift2(v, fill), _mm256_set1_epi32(ext * 2)));
  v = _mm256_max_epi32(v, _mm256_add_epi32(shift4(v, fill), _mm256_set1_epi32(ext * 4)));
  const __m256i ramp = _mm256_setr_epi32(ext, ext * 2, ext * 3, ext * 4, ext * 5, ext * 6, ext * 7, ext * 8);
  return _mm256_max_epi32(v, _mm256_add_epi32(carryv, ramp));
}

__attribute__((target("avx2"))) static inline __m256i insertion_prefix(__m256i md, i32 carry, i32 open, i32 ext) {
  return insertion_prefix_v(md, _mm256_set1_epi32(carry), open, ext);
}

__attribute__((target("avx2"))) static void avx2_row_preds(std::vector<i32> &data, const FastRow &row,
                                                           const FastRow &prev, i32 open, i32 ext) {
  usize ov_start = std::max(row.start, prev.start);
  usize ov_stop = std::min(row.start + row.len, prev.start + prev.len);
  const __m256i vext = _mm256_set1_epi32(ext), vopen = _mm256_set1_epi32(open);
  i32 *d = data.data();
  for (usize j = ov_start; j < ov_stop; j += WIDTH) {
    usize local = j - row.start, prior = j - prev.start;
    __m256i diag = _mm256_loadu_si256((const __m256i *)(d + prev.m_offset + prior - 1));
    __m256i pm = _mm256_loadu_si256((const __m256i *)(d + prev.m_offset + prior));
    __m256i pd = _mm256_loadu_si256((const __m256i *)(d + prev.d_offset + prior));
    __m256i *mp = (__m256i *)(d + row.m_offset + local);
    __m256i *dp = (__m256i *)(d + row.d_offset + local);
    __m256i mv = _mm256_max_epi32(_mm256_loadu_si256(mp), diag);
    __m256i dv = _mm256_max_epi32(_mm256_max_epi32(_mm256_loadu_si256(dp), _mm256_add_epi32(pd, vext)),
                                  _mm256_add_epi32(pm, vopen));
    _mm256_storeu_si256(mp, mv);
    _mm256_storeu_si256(dp, dv);
  }
}

__attribute__((target("avx2"))) static void avx2_row_scan(std::vector<i32> &data, const FastRow &row,
                                                          const i32 *profile, i32 open, i32 ext) {
  i32 *d = data.data();
  __m256i carryv = _mm256_set1_epi32(NEG32);
  const __m256i up1 = _mm256_setr_epi32(0, 0, 1, 2, 3, 4, 5, 6);
  const __m256i last = _mm256_set1_epi32(7);
  for (usize local = 0; local < row.len; local += WIDTH) {
    __m256i diag = _mm256_add_epi32(_mm256_loadu_si256((const __m256i *)(d + row.m_offset + local)),
                                    _mm256_loadu_si256((const __m256i *)(profile + local)));
    __m256i md = _mm256_max_epi32(diag, _mm256_loadu_si256((const __m256i *)(d + row.d_offset + local)));
    __m256i next = insertion_prefix_v(md, carryv, open, ext);
    // current I = [carry, next[0..6]]; the next carry is next[7] broadcast
    __m256i cur = _mm256_blend_epi32(_mm256_permutevar8x32_epi32(next, up1), carryv, 0x01);
    _mm256_storeu_si256((__m256i *)(d + row.i_offset + local), cur);
    _mm256_storeu_si256((__m256i *)(d + row.m_offset + local), _mm256_max_epi32(md, cur));
    carryv = _mm256_permutevar8x32_epi32(next, last);
  }
}

__attribute__((target("avx2"))) static i32 avx2_row_max(const i32 *scores, usize len) {
  __m256i best = _mm256_set1_epi32(NEG32);
  for (usize c = 0; c + WIDTH <= len; c += WIDTH)
    best = _mm256_max_epi32(best, _mm256_loadu_si256((const __m256i *)(scores + c)));
  alignas(32) i32 a[8];
  _mm256_store_si256((__m256i *)a, best);
  return *std::max_element(a, a + 8);
}

// ---------------------------------------------------------------------------
// align.rs:493-529
static bool i32_scores_safe(const Params &params, const Graph &graph, usize beg_id, usize end_id, usize query_len,
                            int kernel) {
  if (kernel == ORC_FORCE_I64 || beg_id >= graph.nodes.size() || end_id >= graph.nodes.size()) return false;
  usize rb = graph.nodes[beg_id].rank, re = graph.nodes[end_id].rank;
  if (re < rb) return false;
  unsigned __int128 steps = (unsigned __int128)(re - rb) + query_len + WIDTH * 2 + 4;
  i64 opening = i64(params.gap_open) + i64(params.gap_ext);
  uint64_t largest = 0;
  for (i32 x : params.matrix) largest = std::max<uint64_t>(largest, uint64_t(std::llabs(i64(x))));
  largest = std::max<uint64_t>(largest, uint64_t(std::llabs(opening)));
  largest = std::max<uint64_t>(largest, uint64_t(std::llabs(i64(params.gap_ext))));
  unsigned __int128 bound = (unsigned __int128)largest * steps;
  return bound <= SCORE_LIMIT;
}

// align.rs:531-545
static std::vector<AlignedBase> poa_inner(const Params &params, const Graph &graph, usize beg_id, usize end_id,
                                          const uint8_t *q, usize qlen, bool adaptive, usize band_b, int kernel) {
  if (kernel == ORC_I32_ONLY) return poa_i32(params, graph, beg_id, end_id, q, qlen, adaptive, band_b, false);
  if (kernel == ORC_I64_ONLY) return poa_i64(params, graph, beg_id, end_id, q, qlen, adaptive, band_b);
  if (i32_scores_safe(params, graph, beg_id, end_id, qlen, kernel))
    return poa_i32(params, graph, beg_id, end_id, q, qlen, adaptive, band_b, kernel == ORC_AUTO_AVX2);
  return poa_i64(params, graph, beg_id, end_id, q, qlen, adaptive, band_b);
}

// align.rs:192-211
static std::vector<AlignedBase> poa(const Params &params, const Graph &graph, usize beg_id, usize end_id,
                                    const uint8_t *q, usize qlen, bool adaptive, usize band_b, int kernel) {
  try {
    return poa_inner(params, graph, beg_id, end_id, q, qlen, adaptive, band_b, kernel);
  } catch (const Error &) {
    if (params.f == 0) throw;
    Params full = params;
    full.f = 0;
    return poa_inner(full, graph, beg_id, end_id, q, qlen, false, band_b, kernel);
  }
}

// align.rs:81-98 (unseeded). Seeded windows are not restated here.
static std::vector<AlignedBase> align(const Params &params, const Graph &graph, const uint8_t *q, usize qlen,
                                      int kernel) {
  if (graph.nodes.size() <= 2) {
    std::vector<AlignedBase> r;
    r.reserve(qlen + 1);
    r.push_back({0, params.encode('N'), NONE});
    for (usize i = 0; i < qlen; ++i) r.push_back({NONE, params.encode(q[i]), NONE});
    return r;
  }
  if (params.seeding) throw Error("seeded windows are not available in this build");
  return poa(params, graph, 0, 1, q, qlen, params.adaptive, params.b, kernel);
}

// lib.rs:184-204. With progressive (-p) the reads go in the guide order
// (minimizer::guide_order, src/minimizer.rs:505-578), which depends on the
// minimizer sketches: the caller passes it (`order`, n entries), as the
// GPU path computes it, so both align the reads in the same order; paths
// keep each read's own index.
static void extend_graph(const Params &params, Graph &graph, usize n, const uint8_t *const *seqs, const int64_t *lens,
                         usize existing, int kernel, const int64_t *order = nullptr) {
  if (params.progressive && existing == 0 && !order)
    throw Error("progressive guide order needs the order (the sketches are the library's)");
  for (usize k = existing; k < n; ++k) {
    const usize id = (order && existing == 0) ? usize(order[k]) : k;
    auto path = align(params, graph, seqs[id], usize(lens[id]), kernel);
    graph.add_path(id, path);
    graph.toposort(false);
  }
}

// GFA input. The reference's reader (io::read_gfa, declared by src/lib.rs:7
// and called at lib.rs:214-218) is absent from its source tree (src/io.rs is
// missing), so this restates the behaviour its tests pin:
// tests/io_cli.rs:375-399 (multi-base segments, paths become records and
// graph paths, round trip through Graph::gfa), :401-408 (links without
// paths still build a graph), :410-431 (rejected inputs: duplicate
// segments, unknown references, reverse orientations, self links, cycles,
// non-zero overlaps, segments without sequence), :564-581 (extension of a
// GFA graph), :584-610 (empty paths; a path revisiting a node fails with
// "revisits"). The construction order, which edge weights and tie-breaks
// depend on: nodes per segment base in S-line order; then each path in
// P-line order through add_path from the source; then the segment-internal
// and L-line edges that no path created (add_edge, weight 1); then edges
// from the source to every node without an incoming edge and from every
// node without an outgoing edge to the sink (node order); then the LIFO
// toposort (graph.rs:125-178), which rejects cycles.
struct Record {
  std::string name, comment, seq;
};

static std::vector<std::string> split(const std::string &s, char sep) {
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

static Graph read_gfa(const Params &p, const std::string &text, std::vector<Record> &recs) {
  struct Link {
    std::string from, to;
  };
  struct PathLine {
    std::string name;
    std::vector<std::string> segs;
  };
  std::vector<std::string> seg_names, seg_seqs;
  std::map<std::string, usize> seg_index;
  std::vector<Link> links;
  std::vector<PathLine> plines;
  for (std::string line : split(text, '\n')) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty() || line[0] == '#') continue;
    const auto f = split(line, '\t');
    if (f[0] == "S") {
      if (f.size() < 3) throw Error("malformed GFA segment line");
      if (f[2].empty() || f[2] == "*") throw Error("GFA segment " + f[1] + " has no sequence");
      if (seg_index.count(f[1])) throw Error("duplicate GFA segment " + f[1]);
      seg_index[f[1]] = seg_names.size();
      seg_names.push_back(f[1]);
      seg_seqs.push_back(f[2]);
    } else if (f[0] == "L") {
      if (f.size() < 6) throw Error("malformed GFA link line");
      if (f[2] != "+" || f[4] != "+") throw Error("unsupported GFA link orientation");
      if (f[5] != "0M" && f[5] != "*") throw Error("unsupported GFA link overlap " + f[5]);
      links.push_back({f[1], f[3]});
    } else if (f[0] == "P") {
      if (f.size() < 3) throw Error("malformed GFA path line");
      PathLine pl{f[1], {}};
      if (f[2] != "*") {
        for (const auto &e : split(f[2], ',')) {
          if (e.size() < 2) throw Error("malformed GFA path " + f[1]);
          if (e.back() == '-') throw Error("unsupported GFA path orientation in " + f[1]);
          if (e.back() != '+') throw Error("malformed GFA path " + f[1]);
          pl.segs.push_back(e.substr(0, e.size() - 1));
        }
      }
      plines.push_back(std::move(pl));
    }
  }
  Graph g(p);
  std::vector<std::vector<usize>> seg_nodes(seg_names.size());
  for (usize k = 0; k < seg_names.size(); ++k)
    for (char c : seg_seqs[k]) seg_nodes[k].push_back(g.add_node(p.encode(uint8_t(c))));
  auto seg_of = [&](const std::string &name, const std::string &what) -> usize {
    auto it = seg_index.find(name);
    if (it == seg_index.end()) throw Error("GFA " + what + " references unknown segment " + name);
    return it->second;
  };
  std::vector<std::pair<usize, usize>> link_nodes;
  for (const auto &l : links) {
    const usize a = seg_of(l.from, "link"), b = seg_of(l.to, "link");
    if (a == b) throw Error("GFA link from segment " + l.from + " to itself forms a cycle");
    link_nodes.push_back({seg_nodes[a].back(), seg_nodes[b].front()});
  }
  recs.clear();
  for (usize k = 0; k < plines.size(); ++k) {
    const auto &pl = plines[k];
    std::vector<AlignedBase> items{{0, g.nodes[0].base, NONE}};
    std::vector<char> seen(g.nodes.size(), 0);
    std::string seq;
    for (const auto &sn : pl.segs) {
      const usize sg = seg_of(sn, "path " + pl.name);
      for (usize id : seg_nodes[sg]) {
        if (seen[id]) throw Error("GFA path " + pl.name + " revisits segment " + sn);
        seen[id] = 1;
        items.push_back({i64(id), g.nodes[id].base, NONE});
      }
      seq += seg_seqs[sg];
    }
    g.add_path(k, items);
    recs.push_back({pl.name, "", seq});
  }
  auto has_edge = [&](usize a, usize b) {
    const auto &out = g.nodes[a].outgoing;
    return std::find(out.begin(), out.end(), b) != out.end();
  };
  for (const auto &nodes : seg_nodes)
    for (usize k = 1; k < nodes.size(); ++k)
      if (!has_edge(nodes[k - 1], nodes[k])) g.add_edge(nodes[k - 1], nodes[k]);
  for (const auto &ln : link_nodes)
    if (!has_edge(ln.first, ln.second)) g.add_edge(ln.first, ln.second);
  for (usize id = 2; id < g.nodes.size(); ++id)
    if (g.nodes[id].incoming.empty()) g.add_edge(0, id);
  for (usize id = 2; id < g.nodes.size(); ++id)
    if (g.nodes[id].outgoing.empty()) g.add_edge(id, 1);
  g.toposort(false);
  return g;
}

}  // namespace orc

// ---------------------------------------------------------------------------
// C ABI

using namespace orc;

namespace {
template <class F>
int guard(F &&f) {
  try {
    f();
    g_error.clear();
    return 0;
  } catch (const std::exception &e) {
    g_error = e.what();
    return 1;
  }
}
orc_item *items_out(const std::vector<AlignedBase> &v) {
  orc_item *o = (orc_item *)std::malloc(sizeof(orc_item) * (v.size() + 1));
  for (size_t i = 0; i < v.size(); ++i) o[i] = {v[i].node, int64_t(v[i].base), v[i].aligned};
  return o;
}
char *str_out(const std::string &s) {
  char *o = (char *)std::malloc(s.size() + 1);
  std::memcpy(o, s.data(), s.size());
  o[s.size()] = 0;
  return o;
}
inline uint64_t fnv1a(const std::string &s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}
}  // namespace

extern "C" {

const char *orc_last_error(void) { return g_error.c_str(); }
void orc_free(void *p) { std::free(p); }

void *orc_graph_new(const orc_params *p) {
  Params pp = Params::from(p);
  return new Graph(pp);
}
void orc_graph_free(void *g) { delete (Graph *)g; }
void *orc_graph_clone(const void *g) { return new Graph(*(const Graph *)g); }

int orc_params_validate(const orc_params *p) {
  return guard([&] { Params::from(p).validate(); });
}
int64_t orc_encode(const orc_params *p, uint8_t c) { return int64_t(Params::from(p).encode(c)); }

int orc_align_sequences(const orc_params *p, int64_t n, const uint8_t *const *seqs, const int64_t *lens, int kernel,
                        void **out_graph) {
  *out_graph = nullptr;
  return guard([&] {
    Params pp = Params::from(p);
    pp.validate();
    auto *g = new Graph(pp);
    try {
      extend_graph(pp, *g, usize(n), seqs, lens, 0, kernel);
    } catch (...) {
      delete g;
      throw;
    }
    *out_graph = g;
  });
}

int orc_align_sequences_in_order(const orc_params *p, int64_t n, const uint8_t *const *seqs, const int64_t *lens,
                                 const int64_t *order, int kernel, void **out_graph) {
  *out_graph = nullptr;
  return guard([&] {
    Params pp = Params::from(p);
    pp.validate();
    auto *g = new Graph(pp);
    try {
      extend_graph(pp, *g, usize(n), seqs, lens, 0, kernel, order);
    } catch (...) {
      delete g;
      throw;
    }
    *out_graph = g;
  });
}

int orc_extend_graph(const orc_params *p, void *g, int64_t n, const uint8_t *const *seqs, const int64_t *lens,
                     int64_t existing, int kernel) {
  return guard([&] {
    Params pp = Params::from(p);
    extend_graph(pp, *(Graph *)g, usize(n), seqs, lens, usize(existing), kernel);
  });
}

int orc_align(const orc_params *p, const void *g, const uint8_t *q, int64_t len, int kernel, orc_item **out,
              int64_t *out_len) {
  *out = nullptr;
  *out_len = 0;
  return guard([&] {
    Params pp = Params::from(p);
    auto v = align(pp, *(const Graph *)g, q, usize(len), kernel);
    *out = items_out(v);
    *out_len = int64_t(v.size());
  });
}

int orc_poa(const orc_params *p, const void *g, int64_t beg_id, int64_t end_id, const uint8_t *q, int64_t len,
            int adaptive, uint64_t band_b, int kernel, int retry, orc_item **out, int64_t *out_len) {
  *out = nullptr;
  *out_len = 0;
  return guard([&] {
    Params pp = Params::from(p);
    const Graph &gr = *(const Graph *)g;
    auto v = retry ? poa(pp, gr, usize(beg_id), usize(end_id), q, usize(len), adaptive != 0, band_b, kernel)
                   : poa_inner(pp, gr, usize(beg_id), usize(end_id), q, usize(len), adaptive != 0, band_b, kernel);
    *out = items_out(v);
    *out_len = int64_t(v.size());
  });
}

int orc_i32_scores_safe(const orc_params *p, const void *g, int64_t beg_id, int64_t end_id, int64_t qlen) {
  Params pp = Params::from(p);
  return i32_scores_safe(pp, *(const Graph *)g, usize(beg_id), usize(end_id), usize(qlen), ORC_AUTO_SERIAL) ? 1 : 0;
}

int orc_add_path(const orc_params *p, void *g, int64_t seq_id, const orc_item *items, int64_t n) {
  (void)p;
  return guard([&] {
    std::vector<AlignedBase> v(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
      if (items[i].base < 0) throw Error("alignment base outside alphabet");
      v[size_t(i)] = {items[i].node, usize(items[i].base), items[i].aligned};
    }
    ((Graph *)g)->add_path(usize(seq_id), v);
  });
}

int64_t orc_add_node(void *g, int64_t base) { return int64_t(((Graph *)g)->add_node(usize(base))); }
void orc_add_edge(void *g, int64_t from, int64_t to) { ((Graph *)g)->add_edge(usize(from), usize(to)); }

int orc_toposort(void *g, int grouped) {
  return guard([&] { ((Graph *)g)->toposort(grouped != 0); });
}

int orc_consensus(const orc_params *p, const void *g, uint8_t **seq, int64_t **ids, int64_t **coverage,
                  int64_t *len) {
  return guard([&] {
    Params pp = Params::from(p);
    std::vector<uint8_t> s;
    std::vector<usize> id, cov;
    ((const Graph *)g)->consensus(pp, s, id, cov);
    *len = int64_t(s.size());
    *seq = (uint8_t *)std::malloc(s.size() + 1);
    std::memcpy(*seq, s.data(), s.size());
    (*seq)[s.size()] = 0;
    *ids = (int64_t *)std::malloc(sizeof(int64_t) * (id.size() + 1));
    *coverage = (int64_t *)std::malloc(sizeof(int64_t) * (cov.size() + 1));
    for (size_t i = 0; i < id.size(); ++i) {
      (*ids)[i] = int64_t(id[i]);
      (*coverage)[i] = int64_t(cov[i]);
    }
  });
}

int orc_msa(const orc_params *p, void *g, int64_t n, const char *const *names, const char *const *comments,
            char **out, int64_t *out_len) {
  return guard([&] {
    Params pp = Params::from(p);
    std::vector<std::string> nm(names, names + n), cm(comments, comments + n);
    std::string s = ((Graph *)g)->msa(pp, nm, cm);
    *out = str_out(s);
    *out_len = int64_t(s.size());
  });
}

int orc_gfa(const orc_params *p, const void *g, int64_t n, const char *const *names, char **out, int64_t *out_len) {
  return guard([&] {
    Params pp = Params::from(p);
    std::vector<std::string> nm(names, names + n);
    std::string s = ((const Graph *)g)->gfa(pp, nm);
    *out = str_out(s);
    *out_len = int64_t(s.size());
  });
}

int64_t orc_graph_nodes(const void *g) { return int64_t(((const Graph *)g)->nodes.size()); }
int64_t orc_graph_paths(const void *g) { return int64_t(((const Graph *)g)->paths.size()); }
void orc_graph_node_fields(const void *g, int64_t *out) {
  const Graph &gr = *(const Graph *)g;
  for (size_t i = 0; i < gr.nodes.size(); ++i) {
    out[4 * i + 0] = int64_t(gr.nodes[i].base);
    out[4 * i + 1] = int64_t(gr.nodes[i].parent);
    out[4 * i + 2] = int64_t(gr.nodes[i].rank);
    out[4 * i + 3] = int64_t(gr.nodes[i].coverage);
  }
}
int64_t orc_graph_edge_total(const void *g) {
  const Graph &gr = *(const Graph *)g;
  int64_t t = 0;
  for (auto &n : gr.nodes) t += int64_t(n.incoming.size());
  return t;
}
void orc_graph_edges(const void *g, int64_t *in_cnt, int64_t *out_cnt, int64_t *in_pairs, int64_t *out_pairs) {
  const Graph &gr = *(const Graph *)g;
  size_t a = 0, b = 0;
  for (size_t i = 0; i < gr.nodes.size(); ++i) {
    const Node &n = gr.nodes[i];
    in_cnt[i] = int64_t(n.incoming.size());
    out_cnt[i] = int64_t(n.outgoing.size());
    for (size_t k = 0; k < n.incoming.size(); ++k) {
      in_pairs[a++] = int64_t(n.incoming[k]);
      in_pairs[a++] = int64_t(n.in_weights[k]);
    }
    for (size_t k = 0; k < n.outgoing.size(); ++k) {
      out_pairs[b++] = int64_t(n.outgoing[k]);
      out_pairs[b++] = int64_t(n.out_weights[k]);
    }
  }
}
void orc_graph_rank(const void *g, int64_t *out) {
  const Graph &gr = *(const Graph *)g;
  for (size_t i = 0; i < gr.rank.size(); ++i) out[i] = int64_t(gr.rank[i]);
}
int64_t orc_graph_rank_len(const void *g) { return int64_t(((const Graph *)g)->rank.size()); }
void orc_graph_aligned(const void *g, int64_t *out) {
  const Graph &gr = *(const Graph *)g;
  size_t a = 0;
  for (auto &n : gr.nodes)
    for (i64 x : n.aligned) out[a++] = x;
}
int64_t orc_graph_path_total(const void *g) {
  const Graph &gr = *(const Graph *)g;
  int64_t t = 0;
  for (auto &p : gr.paths) t += int64_t(p.second.size());
  return t;
}
void orc_graph_path_data(const void *g, int64_t *seq_ids, int64_t *lens, int64_t *ids) {
  const Graph &gr = *(const Graph *)g;
  size_t a = 0;
  for (size_t i = 0; i < gr.paths.size(); ++i) {
    seq_ids[i] = int64_t(gr.paths[i].first);
    lens[i] = int64_t(gr.paths[i].second.size());
    for (usize id : gr.paths[i].second) ids[a++] = int64_t(id);
  }
}

uint64_t orc_cells(void) { return g_cells; }
void orc_reset_cells(void) { g_cells = 0; }

int orc_batch_run(const orc_params *p, int64_t n_sets, const int64_t *set_off, const uint8_t *const *seqs,
                  const int64_t *lens, int kernel, int threads, int out_format, uint64_t *hashes, uint64_t *cells) {
  Params pp = Params::from(p);
  std::atomic<int64_t> next{0};
  std::atomic<uint64_t> total{0};
  std::atomic<int> failed{0};
  std::string first_error;
  std::vector<std::thread> pool;
  if (threads < 1) threads = 1;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&] {
      uint64_t local = 0;
      for (;;) {
        int64_t s = next.fetch_add(1);
        if (s >= n_sets) break;
        uint64_t before = g_cells;
        try {
          Graph g(pp);
          int64_t a = set_off[s], b = set_off[s + 1];
          extend_graph(pp, g, usize(b - a), seqs + a, lens + a, 0, kernel);
          std::string o;
          if (out_format == 0) {
            std::vector<uint8_t> sq;
            std::vector<usize> ids, cov;
            g.consensus(pp, sq, ids, cov);
            o = ">consensus sequence\n" + std::string(sq.begin(), sq.end()) + "\n";
          } else if (out_format == 2) {
            std::vector<std::string> names;
            for (int64_t r = 0; r < b - a; ++r) names.push_back("read" + std::to_string(r));
            o = g.gfa(pp, names);
          }
          if (hashes) hashes[s] = fnv1a(o);
        } catch (const std::exception &e) {
          failed.store(1);
          if (hashes) hashes[s] = 0;
        }
        local += g_cells - before;
      }
      total += local;
    });
  }
  for (auto &th : pool) th.join();
  if (cells) *cells = total.load();
  if (failed.load()) {
    g_error = "a read set failed";
    return 1;
  }
  return 0;
}

int orc_avx2_available(void) { return __builtin_cpu_supports("avx2") ? 1 : 0; }

// FNV-1a of a byte string: the hash orc_batch_run reports per set, so a
// caller can compare another implementation's output text with it.
uint64_t orc_fnv1a(const uint8_t *data, int64_t len) {
  return fnv1a(std::string(reinterpret_cast<const char *>(data), size_t(len)));
}

__attribute__((target("avx2"))) void orc_avx2_prefix(const int32_t *md8, int32_t carry, int32_t open, int32_t ext,
                                                     int32_t *out8) {
  __m256i v = insertion_prefix(_mm256_loadu_si256((const __m256i *)md8), carry, open, ext);
  _mm256_storeu_si256((__m256i *)out8, v);
}

// GFA text -> graph (io::read_gfa as restated above). Records come back as
// "name\tsequence\n" lines.
int orc_read_gfa(const orc_params *p, const char *text, int64_t len, void **out_graph, char **records,
                 int64_t *records_len) {
  *out_graph = nullptr;
  *records = nullptr;
  *records_len = 0;
  return guard([&] {
    Params pp = Params::from(p);
    pp.validate();
    std::vector<Record> recs;
    auto *g = new Graph(read_gfa(pp, std::string(text, size_t(len)), recs));
    std::string r;
    for (auto &x : recs) r += x.name + "\t" + x.seq + "\n";
    *records = str_out(r);
    *records_len = int64_t(r.size());
    *out_graph = g;
  });
}

}  // extern "C"
