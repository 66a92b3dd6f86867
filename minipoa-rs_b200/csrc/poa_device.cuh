// Device-side partial-order alignment for sm_100a.
//
// One warp owns one alignment job at a time. The DP row of a graph node is
// computed by the warp across query columns (32-column chunks, one column per
// lane); the query-direction affine gap is a warp-shuffle max-plus prefix
// scan. The serial parts of the read loop (band-guide passes, traceback,
// read-into-graph fusion, LIFO toposort) run on lane 0 against the job's
// device-resident graph, so no graph crosses PCIe between reads.
//
// Semantics restated from minipoa-rs: src/align.rs (poa, poa_inner, both DP
// kernels, traceback, push_diagonal), src/graph.rs (add_node, add_edge,
// add_path, toposort) and src/lib.rs (extend_graph). Integer arithmetic is
// the reference's: int32 with NEG32 sentinels where the score guard allows,
// int64 with NEG = -2^50 otherwise.
#pragma once
#include <cstdint>

namespace poa {

constexpr int32_t NEG32 = -(1 << 29);               // align.rs:216
constexpr int64_t NEG64 = -(int64_t(1) << 50);      // align.rs:16
constexpr uint64_t SCORE_LIMIT = uint64_t(1) << 26; // align.rs:217
constexpr int OP_MATCH = 1, OP_DELETE = 2, OP_INSERT = 4, OP_ALL = 7;  // align.rs:20-23
constexpr int CHUNK = 4;                             // edge-list entries per chunk
constexpr unsigned FULL = 0xffffffffu;

// Status codes of device routines. 1..13 map one-to-one onto the reference's
// error strings (formatted on the host); 100+ are resource conditions that are
// never alignment errors and never trigger the full-DP retry.
enum Status : int32_t {
  ST_OK = 0,
  ST_ANCHOR_NOT_IN_GRAPH = 1,   // align.rs:598-600
  ST_ANCHORS_NOT_ORDERED = 2,   // align.rs:603-605
  ST_COORD_LIMITS = 3,          // align.rs:608-610
  ST_NO_PATH = 4,               // align.rs:678-680
  ST_BAND_NO_INTERSECT = 5,     // align.rs:730-732
  ST_BAND_EXCLUDES_SOURCE = 6,  // align.rs:738-740
  ST_TB_NO_ADVANCE = 7,         // align.rs:1184-1186
  ST_TB_LEFT_BAND = 8,          // align.rs:1191-1193
  ST_TB_NO_PRED = 9,            // align.rs:1300-1302
  ST_BASE_OUTSIDE = 10,         // graph.rs:84-86
  ST_UNKNOWN_NODE = 11,         // graph.rs:87-91
  ST_CYCLE = 12,                // graph.rs:174-176
  ST_COLUMN_DEPS = 13,          // graph.rs:164-166
  ST_ARENA_FULL = 100,
  ST_GRAPH_FULL = 101,
  ST_SEEDING_UNSUPPORTED = 102,
};

__host__ __device__ inline bool is_alignment_error(int32_t s) { return s > 0 && s < 100; }

// Scoring and band parameters shared by every job of a launch.
struct DevParams {
  const int32_t *matrix;  // sigma * sigma
  const uint8_t *encode;  // 256-entry Params::encode table
  int32_t sigma;
  int32_t unknown;        // encode('N')
  int32_t gap_open_raw;   // Params::gap_open (the zero-open traceback rule)
  int32_t gap_ext;        // E
  int32_t gap_open;       // O = gap_open + gap_ext (align.rs:621-622)
  int32_t adaptive;
  int32_t kernel;         // 0 = score-guard dispatch, 1 = i32 only, 2 = i64 only
  int32_t seeding;
  uint64_t b, f;
  uint64_t largest;       // max(|matrix|, |O|, |E|) of i32_scores_safe
};

// One alignment job: a graph resident in device memory plus its reads.
// Edge lists are chains of CHUNK-entry chunks appended in insertion order,
// which every tie-break of the reference depends on.
struct Job {
  // capacities (host-set)
  int32_t node_cap, chunk_cap, path_cap, max_paths;
  // live sizes (device-updated)
  int32_t n_nodes, n_chunks, n_edges, n_paths, path_used, n_rank;
  // node arrays [node_cap]
  uint8_t *base;
  int32_t *parent, *rank, *coverage;
  int32_t *aligned;  // [node_cap * sigma], -1 = None
  int32_t *in_head, *in_tail, *in_cnt, *out_head, *out_tail, *out_cnt;
  int32_t *rank_to_node;  // Graph::rank
  // edge chunks [chunk_cap]
  int32_t *chunk_id, *chunk_w;  // [chunk_cap * CHUNK]
  int32_t *chunk_next;
  // paths
  int32_t *path_items;  // [path_cap]
  int32_t *path_off;    // [max_paths + 1]
  int32_t *path_seq;    // [max_paths]
  // reads of this job (batch-shared buffer)
  const uint8_t *reads;
  const int64_t *read_off;
  const int32_t *read_len;
  int32_t n_reads, next_read;
  // outcome
  int32_t status, err_i, err_j, n_items;
  uint64_t cells;     // DP cells of completed reads (retries included)
  uint64_t dp_bytes;  // DP state bytes stored for those cells (M, D, I)
};

// Work counted by one alignment: 8-aligned band cells and the bytes of DP
// state they stored.
struct Work {
  uint64_t cells, dp_bytes;
};

// Per-read scratch carved from the front of a warp slot's arena.
struct Scratch {
  int64_t *head, *tail, *support, *row_off, *wsum;
  int64_t *peak, *streak, *peak_left, *peak_right, *offset_left, *offset_right, *extra;
  int32_t *row_start, *row_len, *pred_start, *pred_cnt, *succ_start, *succ_cnt;
  int2 *pred;      // (row, weight) in incoming order, band-guide filtered
  int32_t *succ;   // successor rows in outgoing order, range filtered
  int32_t *seq;    // encoded, padded query
  int4 *items;     // alignment result (node, base, aligned, -)
  char *dp;        // DP matrix cells
  int64_t dp_bytes;
};

__device__ __forceinline__ int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

// Carves scratch for n rows, e edges and a padded query of `padded` columns.
// Returns false when the arena is too small for the scratch itself.
__device__ inline bool carve_scratch(char *arena, int64_t bytes, int n, int e, int64_t padded, int64_t n_items,
                                     Scratch &s) {
  int64_t o = 0;
  auto take = [&](int64_t sz) {
    int64_t at = o;
    o = align_up(o + sz, 128);
    return arena + at;
  };
  const int64_t N = n;
  s.head = (int64_t *)take(N * 8);
  s.tail = (int64_t *)take(N * 8);
  s.support = (int64_t *)take(N * 8);
  s.row_off = (int64_t *)take(N * 8);
  s.wsum = (int64_t *)take(N * 8);
  s.peak = (int64_t *)take(N * 8);
  s.streak = (int64_t *)take(N * 8);
  s.peak_left = (int64_t *)take(N * 8);
  s.peak_right = (int64_t *)take(N * 8);
  s.offset_left = (int64_t *)take(N * 8);
  s.offset_right = (int64_t *)take(N * 8);
  s.extra = (int64_t *)take(N * 8);
  s.row_start = (int32_t *)take(N * 4);
  s.row_len = (int32_t *)take(N * 4);
  s.pred_start = (int32_t *)take(N * 4);
  s.pred_cnt = (int32_t *)take(N * 4);
  s.succ_start = (int32_t *)take(N * 4);
  s.succ_cnt = (int32_t *)take(N * 4);
  s.pred = (int2 *)take(int64_t(e + 1) * 8);
  s.succ = (int32_t *)take(int64_t(e + 1) * 4);
  s.seq = (int32_t *)take((padded + 32) * 4);
  s.items = (int4 *)take((n_items + 1) * 16);
  s.dp = arena + o;
  s.dp_bytes = bytes - o;
  return s.dp_bytes >= 0;
}

// ---------------------------------------------------------------------------
// Graph primitives (lane 0). graph.rs:42-79

__device__ inline int32_t add_node(Job *J, int sigma, int base) {
  const int id = J->n_nodes++;
  J->base[id] = uint8_t(base);
  J->parent[id] = id;
  J->rank[id] = 0;
  J->coverage[id] = 0;
  for (int c = 0; c < sigma; ++c) J->aligned[int64_t(id) * sigma + c] = -1;
  J->aligned[int64_t(id) * sigma + base] = id;
  J->in_cnt[id] = 0;
  J->out_cnt[id] = 0;
  J->in_head[id] = J->in_tail[id] = -1;
  J->out_head[id] = J->out_tail[id] = -1;
  return id;
}

__device__ inline void list_append(Job *J, int32_t *head, int32_t *tail, int32_t *cnt, int node, int id) {
  const int c = cnt[node];
  const int slot = c % CHUNK;
  int ch;
  if (slot == 0) {
    ch = J->n_chunks++;
    J->chunk_next[ch] = -1;
    if (c == 0)
      head[node] = ch;
    else
      J->chunk_next[tail[node]] = ch;
    tail[node] = ch;
  } else {
    ch = tail[node];
  }
  J->chunk_id[int64_t(ch) * CHUNK + slot] = id;
  J->chunk_w[int64_t(ch) * CHUNK + slot] = 1;
  cnt[node] = c + 1;
}

// Increments the weight of `id` in a node's list; false when absent.
__device__ inline bool list_bump(Job *J, const int32_t *head, const int32_t *cnt, int node, int id) {
  const int n = cnt[node];
  int ch = head[node];
  for (int k = 0; k < n; ch = J->chunk_next[ch]) {
    for (int s = 0; s < CHUNK && k < n; ++s, ++k) {
      if (J->chunk_id[int64_t(ch) * CHUNK + s] == id) {
        J->chunk_w[int64_t(ch) * CHUNK + s] += 1;
        return true;
      }
    }
  }
  return false;
}

__device__ inline void add_edge(Job *J, int from, int to) {
  if (from == to) return;
  if (!list_bump(J, J->out_head, J->out_cnt, from, to)) list_append(J, J->out_head, J->out_tail, J->out_cnt, from, to);
  if (!list_bump(J, J->in_head, J->in_cnt, to, from)) {
    list_append(J, J->in_head, J->in_tail, J->in_cnt, to, from);
    J->n_edges += 1;
  }
  J->coverage[to] += 1;
}

// Visits (id, weight) of a node's list in insertion order.
template <class F>
__device__ inline void for_list(const Job *J, const int32_t *head, const int32_t *cnt, int node, F &&f) {
  const int n = cnt[node];
  int ch = head[node];
  for (int k = 0; k < n; ch = J->chunk_next[ch]) {
    const int64_t b = int64_t(ch) * CHUNK;
    for (int s = 0; s < CHUNK && k < n; ++s, ++k) f(J->chunk_id[b + s], J->chunk_w[b + s]);
  }
}

// graph.rs:82-122 (lane 0). Capacity is checked before any change.
__device__ inline int32_t add_path(Job *J, const DevParams &P, int seq_id, const int4 *items, int n) {
  for (int t = 0; t < n; ++t) {
    const int4 it = items[t];
    if (it.y < 0 || it.y >= P.sigma) return ST_BASE_OUTSIDE;
    if ((it.x >= 0 && it.x >= J->n_nodes) || (it.z >= 0 && it.z >= J->n_nodes)) return ST_UNKNOWN_NODE;
  }
  if (J->n_nodes + n > J->node_cap || J->n_chunks + 2 * (n + 1) > J->chunk_cap ||
      J->path_used + n > J->path_cap || J->n_paths + 1 > J->max_paths)
    return ST_GRAPH_FULL;
  int previous = -1;
  for (int t = 0; t < n; ++t) {
    const int4 it = items[t];
    int id;
    if (it.x >= 0) {
      id = it.x;
    } else if (it.z >= 0) {
      const int parent = J->parent[it.z];
      const int a = J->aligned[int64_t(parent) * P.sigma + it.y];
      if (a >= 0) {
        id = a;
      } else {
        id = add_node(J, P.sigma, it.y);
        J->parent[id] = parent;
        J->aligned[int64_t(parent) * P.sigma + it.y] = id;
      }
    } else {
      id = add_node(J, P.sigma, it.y);
    }
    if (previous >= 0) add_edge(J, previous, id);
    previous = id;
    if (id >= 2) J->path_items[J->path_used++] = id;
  }
  add_edge(J, previous >= 0 ? previous : 0, 1);
  J->path_seq[J->n_paths] = seq_id;
  J->path_off[J->n_paths + 1] = J->path_used;
  J->n_paths += 1;
  return ST_OK;
}

// graph.rs:125-178 with grouped = false (lane 0); LIFO Kahn over
// incoming-list degrees, successors pushed in outgoing order.
__device__ inline int32_t toposort(Job *J, int32_t *deg, int32_t *stack) {
  const int N = J->n_nodes;
  int sp = 0;
  for (int id = 0; id < N; ++id) {
    deg[id] = J->in_cnt[id];
    if (deg[id] == 0) stack[sp++] = id;
  }
  int r = 0, visited = 0;
  int32_t st = ST_OK;
  while (sp > 0 && st == ST_OK) {
    const int id = stack[--sp];
    J->rank_to_node[r] = id;
    J->rank[id] = r;
    ++r;
    ++visited;
    for_list(J, J->out_head, J->out_cnt, id, [&](int next, int) {
      if (st != ST_OK) return;
      if (deg[next] == 0) {
        st = ST_COLUMN_DEPS;
        return;
      }
      if (--deg[next] == 0) stack[sp++] = next;
    });
  }
  J->n_rank = r;
  if (st != ST_OK) return st;
  if (visited != N) return ST_CYCLE;
  return ST_OK;
}

// ---------------------------------------------------------------------------
// Alignment (align.rs)

template <typename S>
struct ScoreTraits;
template <>
struct ScoreTraits<int32_t> {
  static constexpr int32_t NEGV = NEG32;
  static constexpr int32_t LOWEST = INT32_MIN;
};
template <>
struct ScoreTraits<int64_t> {
  static constexpr int64_t NEGV = NEG64;
  static constexpr int64_t LOWEST = INT64_MIN;
};

__device__ __forceinline__ int32_t shfl_up_s(int32_t v, int d) { return __shfl_up_sync(FULL, v, d); }
__device__ __forceinline__ int64_t shfl_up_s(int64_t v, int d) {
  return (int64_t)__shfl_up_sync(FULL, (long long)v, d);
}
__device__ __forceinline__ int32_t shfl_s(int32_t v, int l) { return __shfl_sync(FULL, v, l); }
__device__ __forceinline__ int64_t shfl_s(int64_t v, int l) { return (int64_t)__shfl_sync(FULL, (long long)v, l); }
__device__ __forceinline__ int32_t shfl_xor_s(int32_t v, int d) { return __shfl_xor_sync(FULL, v, d); }
__device__ __forceinline__ int64_t shfl_xor_s(int64_t v, int d) {
  return (int64_t)__shfl_xor_sync(FULL, (long long)v, d);
}
template <typename T>
__device__ __forceinline__ T maxs(T a, T b) {
  return a > b ? a : b;
}
template <typename T>
__device__ __forceinline__ T mins(T a, T b) {
  return a < b ? a : b;
}

// Band-guide passes of align.rs:623-680 (lane 0). Builds each row's filtered
// predecessor list (incoming order, in-range, head != NEG), its total
// incoming weight, and its range-filtered successor list.
__device__ inline int32_t guides(const Job *J, Scratch &s, int beg, int end, int n) {
  for (int i = 0; i < n; ++i) {
    s.head[i] = NEG64;
    s.tail[i] = NEG64;
    s.support[i] = 0;
  }
  s.head[0] = 0;
  s.pred_start[0] = 0;
  s.pred_cnt[0] = 0;
  {
    int64_t w0 = 0;
    for_list(J, J->in_head, J->in_cnt, J->rank_to_node[beg], [&](int, int w) { w0 += w; });
    s.wsum[0] = w0;
  }
  int pc = 0;
  for (int i = 1; i < n; ++i) {
    const int node = J->rank_to_node[beg + i];
    const int ps = pc;
    bool have = false;
    int bp = 0, bw = 0;
    int64_t wsum = 0;
    for_list(J, J->in_head, J->in_cnt, node, [&](int pred, int w) {
      wsum += w;
      const int r = J->rank[pred];
      if (r < beg || r >= beg + i) return;
      const int p = r - beg;
      if (s.head[p] == NEG64) return;
      s.pred[pc++] = make_int2(p, w);
      if (!have || w > bw || (w == bw && s.support[p] > s.support[bp])) {
        have = true;
        bp = p;
        bw = w;
      }
    });
    s.pred_start[i] = ps;
    s.pred_cnt[i] = pc - ps;
    s.wsum[i] = wsum;
    if (have) {
      s.head[i] = s.head[bp] + 1;
      s.support[i] = s.support[bp] + bw;
    }
  }
  s.tail[n - 1] = 1;
  int sc = 0;
  s.succ_start[n - 1] = 0;
  s.succ_cnt[n - 1] = 0;
  {
    // successors of the last row are outside (beg, end] by definition
  }
  for (int i = n - 2; i >= 0; --i) {
    const int node = J->rank_to_node[beg + i];
    const int ss = sc;
    bool have = false;
    int bs = 0, bw = 0;
    for_list(J, J->out_head, J->out_cnt, node, [&](int succ, int w) {
      const int r = J->rank[succ];
      if (r <= beg + i || r > end) return;
      const int sx = r - beg;
      s.succ[sc++] = sx;
      if (s.tail[sx] == NEG64) return;
      if (!have || w > bw || (w == bw && s.support[sx] > s.support[bs])) {
        have = true;
        bs = sx;
        bw = w;
      }
    });
    s.succ_start[i] = ss;
    s.succ_cnt[i] = sc - ss;
    if (have) {
      s.tail[i] = s.tail[bs] + 1;
      s.support[i] = s.support[bs] + bw;
    }
  }
  if (s.head[n - 1] == NEG64) return ST_NO_PATH;
  return ST_OK;
}

// align.rs:829-897 (lane 0): band state after row i peaked at `maximum`.
__device__ inline void adaptive_update(const Job *J, Scratch &s, int beg, int i, int64_t maximum, int64_t band) {
  const int node = J->rank_to_node[beg + i];
  s.peak[i] = maximum;
  int64_t max_streak = 0;
  bool is_match = false;
  if (int(J->base[node]) == s.seq[maximum]) {
    for (int t = 0; t < s.pred_cnt[i]; ++t) {
      const int p = s.pred[s.pred_start[i] + t].x;
      max_streak = maxs(max_streak, s.streak[p]);
      if (s.peak[p] + 1 == maximum) {
        s.streak[i] = maxs(s.streak[i], s.streak[p] + 1);
        is_match = true;
      }
    }
  }
  if (!is_match && max_streak < 30) s.extra[i] = mins(s.extra[i] + max_streak + 1, 5 * band);
  const int ss = s.succ_start[i], sn = s.succ_cnt[i];
  if (s.streak[i] >= 30) {
    s.offset_left[i] = maximum - s.head[i];
    s.offset_right[i] = maximum - s.head[i];
    s.extra[i] = 0;
    for (int t = 0; t < sn; ++t) {
      const int sx = s.succ[ss + t];
      s.offset_left[sx] = s.offset_left[i];
      s.offset_right[sx] = s.offset_right[i];
    }
  }
  for (int t = 0; t < sn; ++t) {
    const int sx = s.succ[ss + t];
    s.offset_left[sx] = mins(s.offset_left[sx], s.offset_left[i]);
    s.offset_right[sx] = maxs(s.offset_right[sx], s.offset_right[i]);
    s.peak_left[sx] = mins(s.peak_left[sx], maximum);
    s.peak_right[sx] = maxs(s.peak_right[sx], maximum + 1);
    s.extra[sx] = s.extra[i] != 0 ? maxs(s.extra[sx], s.extra[i]) : 0;
  }
}

// Traceback of align.rs:1164-1347 (lane 0), reading the stored DP states.
// Writes the path (source first, sink entry dropped) to s.items.
template <typename S>
__device__ int32_t traceback(Job *J, const DevParams &P, Scratch &s, const S *A, int beg, int n, int64_t m,
                             int *n_out) {
  constexpr S NEGV = ScoreTraits<S>::NEGV;
  const int64_t neg_half = int64_t(NEGV) / 2;
  auto contains = [&](int r, int64_t c) -> bool {
    const int st = s.row_start[r];
    return c >= st && c - st < s.row_len[r];
  };
  auto Mv = [&](int r, int64_t c) -> int64_t {
    return contains(r, c) ? int64_t(A[s.row_off[r] + (c - s.row_start[r])]) : int64_t(NEGV);
  };
  auto Dv = [&](int r, int64_t c) -> int64_t {
    return contains(r, c) ? int64_t(A[s.row_off[r] + s.row_len[r] + (c - s.row_start[r])]) : int64_t(NEGV);
  };
  auto Iv = [&](int r, int64_t c) -> int64_t {
    return contains(r, c) ? int64_t(A[s.row_off[r] + 2 * int64_t(s.row_len[r]) + (c - s.row_start[r])])
                          : int64_t(NEGV);
  };
  const int64_t O = P.gap_open, E = P.gap_ext;
  int i = n - 1;
  int64_t j = m - 1;
  int op = OP_ALL;
  int nres = 0;
  int64_t steps = 0;
  int4 *res = s.items;
  while (i > 0 || j > 0) {
    steps += 1;
    if (steps > int64_t(n) + m) return ST_TB_NO_ADVANCE;
    if (!contains(i, j) || Mv(i, j) <= neg_half) return ST_TB_LEFT_BAND;
    const int node = J->rank_to_node[beg + i];
    const int nb = J->base[node];
    const int base = (i == n - 1) ? P.unknown : nb;
    const int qb = s.seq[j];
    const int64_t score = P.matrix[base * P.sigma + qb];
    const int pb = s.pred_start[i], pc = s.pred_cnt[i];
    // choose(): first max-weight predecessor whose stored state explains
    // (state, penalty) at column pj (align.rs:1201-1225).
    auto choose = [&](int state, int64_t penalty, int64_t pj, int &bp_out, int &bw_out) -> bool {
      bool found = false;
      int bp = -1, bw = 0;
      const int64_t target = state == OP_MATCH ? Mv(i, j) : Dv(i, j);
      for (int t = 0; t < pc; ++t) {
        const int2 e = s.pred[pb + t];
        if (!contains(e.x, pj)) continue;
        const int64_t source = state == OP_DELETE ? Dv(e.x, pj) : Mv(e.x, pj);
        if (target == source + penalty && (!found || e.y > bw)) {
          found = true;
          bp = e.x;
          bw = e.y;
        }
      }
      bp_out = bp;
      bw_out = bw;
      return found;
    };
    auto push_diagonal = [&]() {
      if (i == n - 1 && j != m - 1) {
        res[nres++] = make_int4(-1, qb, -1, 0);
      } else if (base == qb) {
        res[nres++] = make_int4(node, nb, -1, 0);
      } else {
        const int parent = J->parent[node];
        res[nres++] = make_int4(J->aligned[int64_t(parent) * P.sigma + qb], qb, parent, 0);
      }
    };
    int kp, kw;
    bool preferred = false;
    if ((op & OP_MATCH) && j > 0 && base == qb) preferred = choose(OP_MATCH, score, j - 1, kp, kw);
    if (preferred && !(int64_t(kw) >= s.wsum[i] / 10)) preferred = false;
    if (preferred) {
      push_diagonal();
      i = kp;
      j -= 1;
      op = OP_ALL;
      continue;
    }
    if ((op & OP_DELETE) && (op == OP_DELETE || Mv(i, j) == Dv(i, j))) {
      if (choose(OP_INSERT, O, j, kp, kw)) {
        i = kp;
        op = P.gap_open_raw == 0 ? OP_ALL : (OP_MATCH | OP_INSERT);
        continue;
      }
      if (choose(OP_DELETE, E, j, kp, kw)) {
        i = kp;
        op = OP_DELETE;
        continue;
      }
    }
    if ((op & OP_INSERT) && j > 0 && contains(i, j - 1) && (op == OP_INSERT || Mv(i, j) == Iv(i, j))) {
      if (Iv(i, j) == Mv(i, j - 1) + O) {
        res[nres++] = make_int4(-1, qb, -1, 0);
        j -= 1;
        op = P.gap_open_raw == 0 ? OP_ALL : (OP_MATCH | OP_DELETE);
        continue;
      }
      if (Iv(i, j) == Iv(i, j - 1) + E) {
        res[nres++] = make_int4(-1, qb, -1, 0);
        j -= 1;
        op = OP_INSERT;
        continue;
      }
    }
    if ((op & OP_MATCH) && j > 0) {
      if (choose(OP_MATCH, score, j - 1, kp, kw)) {
        push_diagonal();
        i = kp;
        j -= 1;
        op = OP_ALL;
        continue;
      }
    }
    J->err_i = i;
    J->err_j = int32_t(j);
    return ST_TB_NO_PRED;
  }
  // result = reverse(pushed + [source]) without its last element.
  for (int a = 0, b = nres - 1; a < b; ++a, --b) {
    const int4 t = res[a];
    res[a] = res[b];
    res[b] = t;
  }
  for (int k = nres - 1; k >= 1; --k) res[k] = res[k - 1];
  if (nres > 0) {
    const int src = J->rank_to_node[beg];
    res[0] = make_int4(src, J->base[src], -1, 0);
  }
  *n_out = nres;
  return ST_OK;
}

// align.rs:493-529
__device__ inline bool i32_scores_safe(const Job *J, const DevParams &P, int beg_id, int end_id, int64_t qlen) {
  if (P.kernel == 2) return false;
  if (beg_id >= J->n_nodes || end_id >= J->n_nodes) return false;
  const int rb = J->rank[beg_id], re = J->rank[end_id];
  if (re < rb) return false;
  const uint64_t steps = uint64_t(re - rb) + uint64_t(qlen) + 8 * 2 + 4;
  if (P.largest == 0) return true;
  return steps <= SCORE_LIMIT / P.largest;
}

// One DP kernel invocation (poa_simd_arena, align.rs:588-911, or
// poa_scalar_i64, align.rs:913-1162) by a whole warp.
template <typename S>
__device__ int32_t poa_kernel(Job *J, const DevParams &P, char *arena, int64_t arena_bytes, int beg_id, int end_id,
                              const uint8_t *query, int qlen, bool adaptive_arg, uint64_t band_b, uint64_t f,
                              Scratch &s, int *n_items, Work *cells) {
  constexpr S NEGV = ScoreTraits<S>::NEGV;
  const int lane = threadIdx.x & 31;
  if (beg_id >= J->n_nodes || end_id >= J->n_nodes) return ST_ANCHOR_NOT_IN_GRAPH;
  const int beg = J->rank[beg_id], end = J->rank[end_id];
  if (end <= beg || end >= J->n_rank) return ST_ANCHORS_NOT_ORDERED;
  const int n = end - beg + 1;
  const int64_t m = int64_t(qlen) + 2;
  if (m > INT32_MAX) return ST_COORD_LIMITS;
  const int64_t padded = (m / 8 + 1) * 8;
  if (!carve_scratch(arena, arena_bytes, n, J->n_edges, padded, m + 1, s)) return ST_ARENA_FULL;
  for (int64_t c = lane; c < padded; c += 32)
    s.seq[c] = (c == 0 || c > qlen) ? P.unknown : int(P.encode[query[c - 1]]);
  const bool adaptive = adaptive_arg || P.adaptive;
  uint64_t bandu = band_b + (f == 0 ? 0 : uint64_t(m) / f);
  if (bandu < band_b) bandu = UINT64_MAX;
  const int64_t band = int64_t(bandu < uint64_t(INT32_MAX) ? bandu : uint64_t(INT32_MAX));
  const S E = S(P.gap_ext), O = S(P.gap_open);
  int32_t st = ST_OK;
  __syncwarp();
  if (lane == 0) st = guides(J, s, beg, end, n);
  st = __shfl_sync(FULL, st, 0);
  if (st != ST_OK) return st;
  for (int i = lane; i < n; i += 32) {
    s.peak[i] = 0;
    s.streak[i] = 0;
    s.peak_left[i] = m;
    s.peak_right[i] = 0;
    s.offset_left[i] = 0;
    s.offset_right[i] = 0;
    s.extra[i] = 0;
  }
  __syncwarp();
  S *A = reinterpret_cast<S *>(s.dp);
  const int64_t cap = s.dp_bytes / int64_t(sizeof(S));
  int64_t cursor = 0;
  uint64_t row_cells = 0;
  const bool do_adapt = f != 0 && adaptive;
  for (int i = 0; i < n; ++i) {
    const int64_t hi = s.head[i], ti = s.tail[i];
    if (hi == NEG64 || ti == NEG64) {
      if (lane == 0) {
        s.row_start[i] = 0;
        s.row_len[i] = 0;
        s.row_off[i] = 0;
      }
      __syncwarp();
      continue;
    }
    int64_t left, right;
    if (f == 0) {
      left = 0;
      right = m;
    } else if (adaptive) {
      const int64_t x = mins(mins(s.peak_left[i], hi + s.offset_left[i]), m - ti);
      const int64_t y = maxs(maxs(s.peak_right[i], hi + s.offset_right[i]), m - ti);
      left = maxs<int64_t>(x - band - s.extra[i], 0);
      right = mins<int64_t>(y + band + s.extra[i], m);
    } else {
      left = maxs<int64_t>(mins(hi, m - ti) - band, 0);
      right = mins<int64_t>(maxs(hi, m - ti) + band, m);
    }
    if (left > right || right < 0) return ST_BAND_NO_INTERSECT;
    const int start = int(left / 8 * 8);
    const int stop = int((right / 8 + 1) * 8);
    const int len = stop - start;
    if (cursor + 3 * int64_t(len) > cap) return ST_ARENA_FULL;
    const int64_t off = cursor;
    cursor += 3 * int64_t(len);
    row_cells += uint64_t(len);
    if (lane == 0) {
      s.row_start[i] = start;
      s.row_len[i] = len;
      s.row_off[i] = off;
    }
    S *R = A + off;
    if (i == 0) {
      if (start != 0) return ST_BAND_EXCLUDES_SOURCE;
      if (lane == 0) {
        for (int c = 0; c < len; ++c) {
          R[c] = NEGV;
          R[len + c] = NEGV;
        }
        R[0] = S(P.matrix[P.unknown * P.sigma + P.unknown]);
        R[2 * len] = NEGV;
        for (int c = 1; c < len; ++c) {
          const S ins = maxs<S>(R[2 * len + c - 1] + E, R[c - 1] + O);
          R[2 * len + c] = ins;
          R[c] = maxs<S>(R[c], ins);
        }
      }
      __syncwarp();
      continue;
    }
    const int node = J->rank_to_node[beg + i];
    const int base = (i == n - 1) ? P.unknown : int(J->base[node]);
    const int32_t *mrow = P.matrix + base * P.sigma;
    const int pb = s.pred_start[i], pc = s.pred_cnt[i];
    S carry = NEGV;
    S bestv = ScoreTraits<S>::LOWEST;
    int bestj = INT32_MAX;
    for (int c0 = start; c0 < stop; c0 += 32) {
      const int j = c0 + lane;
      const bool valid = j < stop;
      S M = NEGV, D = NEGV;
      if (valid) {
        for (int t = 0; t < pc; ++t) {
          const int p = s.pred[pb + t].x;
          const int ps = s.row_start[p], pl = s.row_len[p];
          if (j >= ps && j < ps + pl) {
            const S *Q = A + s.row_off[p];
            const int k = j - ps;
            const S mp = Q[k], dp = Q[pl + k];
            const S dg = k > 0 ? Q[k - 1] : NEGV;
            M = maxs(M, dg);
            D = maxs(D, maxs<S>(dp + E, mp + O));
          }
        }
      }
      const S prof = valid ? S(mrow[s.seq[j]]) : S(0);
      const S md = maxs<S>(M + prof, D);
      S x = md + O;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const S y = shfl_up_s(x, d);
        if (lane >= d) x = maxs<S>(x, y + S(d) * E);
      }
      x = maxs<S>(x, carry + S(lane + 1) * E);
      S I = shfl_up_s(x, 1);
      if (lane == 0) I = carry;
      const S Mf = maxs(md, I);
      if (valid) {
        const int c = j - start;
        R[c] = Mf;
        R[len + c] = D;
        R[2 * len + c] = I;
        if (Mf > bestv) {
          bestv = Mf;
          bestj = j;
        }
      }
      carry = shfl_s(x, 31);
    }
    __syncwarp();
    if (do_adapt) {
      S v = bestv;
      int jj = bestj;
#pragma unroll
      for (int d = 16; d; d >>= 1) {
        const S ov = shfl_xor_s(v, d);
        const int oj = __shfl_xor_sync(FULL, jj, d);
        if (ov > v || (ov == v && oj < jj)) {
          v = ov;
          jj = oj;
        }
      }
      if (lane == 0) adaptive_update(J, s, beg, i, int64_t(jj), band);
      __syncwarp();
    }
  }
  cells->cells += row_cells;
  cells->dp_bytes += row_cells * 3 * sizeof(S);
  if (lane == 0) st = traceback<S>(J, P, s, A, beg, n, m, n_items);
  st = __shfl_sync(FULL, st, 0);
  *n_items = __shfl_sync(FULL, *n_items, 0);
  return st;
}

// poa_inner (align.rs:531-545): score-guard dispatch.
__device__ inline int32_t poa_inner(Job *J, const DevParams &P, char *arena, int64_t bytes, int beg_id, int end_id,
                                    const uint8_t *q, int qlen, bool adaptive, uint64_t band_b, uint64_t f,
                                    Scratch &s, int *n_items, Work *cells) {
  const bool use32 = P.kernel == 1 || (P.kernel == 0 && i32_scores_safe(J, P, beg_id, end_id, qlen));
  if (use32)
    return poa_kernel<int32_t>(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive, band_b, f, s, n_items, cells);
  return poa_kernel<int64_t>(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive, band_b, f, s, n_items, cells);
}

// poa (align.rs:192-211): on an alignment error with f != 0, retry with the
// full matrix (f = 0, static band).
__device__ inline int32_t poa_retry(Job *J, const DevParams &P, char *arena, int64_t bytes, int beg_id, int end_id,
                                    const uint8_t *q, int qlen, bool adaptive, uint64_t band_b, Scratch &s,
                                    int *n_items, Work *cells) {
  int32_t st = poa_inner(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive, band_b, P.f, s, n_items, cells);
  if (is_alignment_error(st) && P.f != 0)
    st = poa_inner(J, P, arena, bytes, beg_id, end_id, q, qlen, false, band_b, 0, s, n_items, cells);
  return st;
}

// align::align (align.rs:81-98) for unseeded parameters; writes s.items.
__device__ inline int32_t align_query(Job *J, const DevParams &P, char *arena, int64_t bytes, const uint8_t *q,
                                      int qlen, Scratch &s, int *n_items, Work *cells) {
  const int lane = threadIdx.x & 31;
  if (J->n_nodes <= 2) {
    if (!carve_scratch(arena, bytes, 2, 0, (int64_t(qlen) + 2) / 8 * 8 + 8, int64_t(qlen) + 3, s))
      return ST_ARENA_FULL;
    if (lane == 0) s.items[0] = make_int4(0, P.unknown, -1, 0);
    for (int c = lane; c < qlen; c += 32) s.items[c + 1] = make_int4(-1, int(P.encode[q[c]]), -1, 0);
    *n_items = qlen + 1;
    __syncwarp();
    return ST_OK;
  }
  if (P.seeding) return ST_SEEDING_UNSUPPORTED;
  return poa_retry(J, P, arena, bytes, 0, 1, q, qlen, P.adaptive != 0, P.b, s, n_items, cells);
}

// One step of extend_graph (lib.rs:199-201): align, add_path, toposort(false).
// Capacity is checked before the DP so a full graph stops cleanly.
__device__ inline int32_t extend_one(Job *J, const DevParams &P, char *arena, int64_t bytes, const uint8_t *q,
                                     int qlen, int r) {
  const int lane = threadIdx.x & 31;
  if (J->n_nodes + qlen + 2 > J->node_cap || J->n_chunks + 2 * (qlen + 3) > J->chunk_cap ||
      J->path_used + qlen + 1 > J->path_cap || J->n_paths + 1 > J->max_paths)
    return ST_GRAPH_FULL;
  // toposort scratch (degree + stack) reuses the arena once the alignment is
  // consumed; it must fit before the graph is touched.
  const int64_t nodes_after = int64_t(J->n_nodes) + qlen + 2;
  if (nodes_after * 8 > bytes) return ST_ARENA_FULL;
  Scratch s;
  int n_items = 0;
  Work cells{};
  int32_t st = align_query(J, P, arena, bytes, q, qlen, s, &n_items, &cells);
  if (st != ST_OK) return st;
  if (lane == 0) {
    // toposort runs after add_path has consumed s.items, so its scratch may
    // overwrite the front of the arena.
    st = add_path(J, P, r, s.items, n_items);
    if (st == ST_OK) {
      int32_t *deg = reinterpret_cast<int32_t *>(arena);
      int32_t *stack = deg + nodes_after;
      st = toposort(J, deg, stack);
    }
    if (st == ST_OK) {
      J->cells += cells.cells;
      J->dp_bytes += cells.dp_bytes;
      J->next_read = r + 1;
    }
  }
  st = __shfl_sync(FULL, st, 0);
  __syncwarp();
  return st;
}

}  // namespace poa
