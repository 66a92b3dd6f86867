// Device-side partial-order alignment for sm_100a.
//
// One warp owns one alignment job at a time. A DP row (one graph node) is a
// blocked register tile: each lane owns a run of consecutive query columns,
// scans it serially, and one warp-shuffle max-plus scan over the lane
// aggregates carries the query-direction affine gap across lanes.
// Predecessor rows are read from a per-warp shared-memory ring of recent
// rows. The band guides gather their lists warp-parallel; the serial parts
// of the read loop (guide passes, traceback, read-into-graph fusion) run on
// lane 0 against the job's device-resident graph, so no graph crosses PCIe
// between reads.
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
  int32_t relaxed_order;  // read loops may keep a spliced order between reads
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
  int32_t order_exact;  // 1 when rank is the reference's LIFO toposort order
  uint64_t cells;       // DP cells of completed reads (retries included)
  uint64_t dp_bytes;    // DP state bytes stored for those cells (M, D, I)
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
  int2 *pred;          // (row, weight) in incoming order; row = -1 once head is NEG
  int2 *succ;          // (row, weight) in outgoing order, range filtered
  int32_t *row_base;   // base code a row scores with (N for the last row)
  int4 *pmeta;         // per pred entry: (row, band start, band length, -)
  int64_t *pmeta_off;  // per pred entry: the predecessor row's arena offset
  int32_t *seq;        // encoded, padded query
  int4 *items;         // alignment result (node, base, aligned, resolved id)
  char *dp;            // DP matrix cells
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
  s.succ = (int2 *)take(int64_t(e + 1) * 8);
  s.row_base = (int32_t *)take(N * 4);
  s.pmeta = (int4 *)take(int64_t(e + 1) * 16);
  s.pmeta_off = (int64_t *)take(int64_t(e + 1) * 8);
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

// graph.rs:82-122 (lane 0). Capacity is checked before any change. The
// resolved node id of each item is written to its .w field.
__device__ inline int32_t add_path(Job *J, const DevParams &P, int seq_id, int4 *items, int n) {
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
    items[t].w = id;
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

// Band-guide passes of align.rs:623-680, by the whole warp. Lanes gather
// every row's in-range predecessor list (incoming order) and successor list
// (outgoing order) in parallel, with the total incoming weight; lane 0 then
// runs the serial head / tail / support passes over the compact lists.
// Predecessors whose head stays NEG are marked row = -1: the DP, the adaptive
// update and the traceback skip them, as the reference's head filter does.
// (head or tail, support) of the last GRING rows live in a shared-memory
// ring so the serial passes read their neighbours without an L2 round trip.
constexpr int GRING = 64;
__device__ inline int32_t guides(const Job *J, Scratch &s, int beg, int end, int n, int64_t *ring_v,
                                 int64_t *ring_s) {
  const int lane = threadIdx.x & 31;
  int pbase = 0, sbase = 0;
  for (int i0 = 0; i0 < n; i0 += 32) {
    const int i = i0 + lane;
    int cin = 0, cout = 0;
    int64_t wsum = 0;
    int node = -1;
    if (i < n) {
      node = J->rank_to_node[beg + i];
      for_list(J, J->in_head, J->in_cnt, node, [&](int pred, int w) {
        wsum += w;
        const int r = J->rank[pred];
        if (r >= beg && r < beg + i) ++cin;
      });
      for_list(J, J->out_head, J->out_cnt, node, [&](int succ, int) {
        const int r = J->rank[succ];
        if (r > beg + i && r <= end) ++cout;
      });
    }
    int pin = cin, pout = cout;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int a = __shfl_up_sync(FULL, pin, d);
      const int b = __shfl_up_sync(FULL, pout, d);
      if (lane >= d) {
        pin += a;
        pout += b;
      }
    }
    if (i < n) {
      const int ps = pbase + pin - cin, ss = sbase + pout - cout;
      s.pred_start[i] = ps;
      s.pred_cnt[i] = cin;
      s.succ_start[i] = ss;
      s.succ_cnt[i] = cout;
      s.wsum[i] = wsum;
      int k = ps;
      for_list(J, J->in_head, J->in_cnt, node, [&](int pred, int w) {
        const int r = J->rank[pred];
        if (r >= beg && r < beg + i) s.pred[k++] = make_int2(r - beg, w);
      });
      k = ss;
      for_list(J, J->out_head, J->out_cnt, node, [&](int succ, int w) {
        const int r = J->rank[succ];
        if (r > beg + i && r <= end) s.succ[k++] = make_int2(r - beg, w);
      });
      s.head[i] = NEG64;
      s.tail[i] = NEG64;
      s.support[i] = 0;
    }
    pbase += __shfl_sync(FULL, pin, 31);
    sbase += __shfl_sync(FULL, pout, 31);
  }
  __syncwarp();
  int32_t st = ST_OK;
  if (lane == 0) {
    int64_t *rv = ring_v, *rs = ring_s;
    s.head[0] = 0;
    if (rv) {
      rv[0] = 0;
      rs[0] = 0;
    }
    for (int i = 1; i < n; ++i) {
      bool have = false;
      int bw = 0;
      int64_t bsup = 0, bhead = 0;
      const int pb = s.pred_start[i], pc = s.pred_cnt[i];
      for (int t = 0; t < pc; ++t) {
        const int2 e = s.pred[pb + t];
        const bool near = rv && i - e.x < GRING;
        const int64_t hp = near ? rv[e.x & (GRING - 1)] : s.head[e.x];
        if (hp == NEG64) {
          s.pred[pb + t].x = -1;
          continue;
        }
        const int64_t sp = near ? rs[e.x & (GRING - 1)] : s.support[e.x];
        if (!have || e.y > bw || (e.y == bw && sp > bsup)) {
          have = true;
          bw = e.y;
          bsup = sp;
          bhead = hp;
        }
      }
      const int64_t hi = have ? bhead + 1 : NEG64;
      const int64_t si = have ? bsup + bw : 0;
      if (have) {
        s.head[i] = hi;
        s.support[i] = si;
      }
      if (rv) {
        rv[i & (GRING - 1)] = hi;
        rs[i & (GRING - 1)] = si;
      }
    }
    s.tail[n - 1] = 1;
    if (rv) rv[(n - 1) & (GRING - 1)] = 1;  // rs keeps the forward support of the last row
    for (int i = n - 2; i >= 0; --i) {
      bool have = false;
      int bw = 0;
      int64_t bsup = 0, btail = 0;
      const int sb = s.succ_start[i], sn = s.succ_cnt[i];
      for (int t = 0; t < sn; ++t) {
        const int2 e = s.succ[sb + t];
        const bool near = rv && e.x - i < GRING;
        const int64_t ts = near ? rv[e.x & (GRING - 1)] : s.tail[e.x];
        if (ts == NEG64) continue;
        const int64_t ss = near ? rs[e.x & (GRING - 1)] : s.support[e.x];
        if (!have || e.y > bw || (e.y == bw && ss > bsup)) {
          have = true;
          bw = e.y;
          bsup = ss;
          btail = ts;
        }
      }
      const int64_t ti = have ? btail + 1 : NEG64;
      const int64_t si = have ? bsup + bw : 0;
      if (have) {
        s.tail[i] = ti;
        s.support[i] = si;
      }
      if (rv) {
        rv[i & (GRING - 1)] = ti;
        rs[i & (GRING - 1)] = si;
      }
    }
    if (s.head[n - 1] == NEG64) st = ST_NO_PATH;
  }
  st = __shfl_sync(FULL, st, 0);
  __syncwarp();
  return st;
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
      if (p < 0) continue;
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
      const int sx = s.succ[ss + t].x;
      s.offset_left[sx] = s.offset_left[i];
      s.offset_right[sx] = s.offset_right[i];
    }
  }
  for (int t = 0; t < sn; ++t) {
    const int sx = s.succ[ss + t].x;
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
        if (e.x < 0 || !contains(e.x, pj)) continue;
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

// Per-warp shared memory: the M and D states of the last RING_ROWS rows,
// indexed by absolute query column modulo RING_W, so predecessor rows are
// read from shared memory instead of L2/HBM (a slot is valid for row r only
// while ring_row[r % RING_ROWS] == r); the scoring matrix; the guide rings.
constexpr int RING_ROWS = 4;
constexpr int RING_W = 512;
constexpr int SMEM_MATRIX = 512;  // sigma^2 entries kept in shared memory (sigma <= 22)
struct WarpSmem {
  int32_t ring_m[RING_ROWS][RING_W];
  int32_t ring_d[RING_ROWS][RING_W];
  int32_t ring_row[RING_ROWS];
  int32_t matrix[SMEM_MATRIX];
  int64_t gring_v[GRING];  // guide passes: head (forward) or tail (backward)
  int64_t gring_s[GRING];  // guide passes: support
};

// One int32 DP row of at most 32*C columns (align.rs:751-828) as a blocked
// register tile: lane l owns columns [start + C*l, start + C*l + C). The
// predecessors (band, arena row and ring slot held by the lanes of `vmask`)
// are folded into M and D; each lane scans its block serially, one warp
// max-plus scan over the lane aggregates (shift C*E per lane) gives every
// lane its carried-in insertion state, and a per-lane fixup finishes I and
// M. All identities are exact in integers: I[j+1] = max(I[j] + E, md[j] + O)
// with I[start] = NEG32.
template <int C>
__device__ __forceinline__ void dp_row_blocked(int lane, int start, int len, int32_t *R, const int32_t *seq,
                                               const int32_t *mrow, int32_t E, int32_t O, unsigned vmask,
                                               int my_ps, int my_pl, int my_slot, const int32_t *my_g,
                                               WarpSmem *sm, int out_slot, bool adapt, int32_t &bestv,
                                               int &bestj) {
  const int stop = start + len;
  const int j0 = start + C * lane;
  int32_t Mx[C], Dx[C];
#pragma unroll
  for (int k = 0; k < C; ++k) {
    Mx[k] = NEG32;
    Dx[k] = NEG32;
  }
  while (vmask) {
    const int t = __ffs(vmask) - 1;
    vmask &= vmask - 1;
    const int ps = __shfl_sync(FULL, my_ps, t);
    const int pl = __shfl_sync(FULL, my_pl, t);
    const int slot = __shfl_sync(FULL, my_slot, t);
    const int32_t *g = reinterpret_cast<const int32_t *>(__shfl_sync(FULL, (long long)my_g, t));
    if (slot >= 0) {
      const int32_t *rm = sm->ring_m[slot];
      const int32_t *rd = sm->ring_d[slot];
      int32_t prev = (j0 > ps && j0 - 1 < ps + pl) ? rm[(j0 - 1) & (RING_W - 1)] : NEG32;
#pragma unroll
      for (int k = 0; k < C; ++k) {
        const int j = j0 + k;
        const bool in = unsigned(j - ps) < unsigned(pl);
        const int32_t mp = rm[j & (RING_W - 1)], dp = rd[j & (RING_W - 1)];
        if (in) {
          Mx[k] = maxs(Mx[k], prev);
          Dx[k] = maxs(Dx[k], maxs(dp + E, mp + O));
        }
        prev = in ? mp : NEG32;
      }
    } else {
      int32_t prev = (j0 > ps && j0 - 1 < ps + pl) ? g[j0 - 1 - ps] : NEG32;
#pragma unroll
      for (int k = 0; k < C; ++k) {
        const int j = j0 + k;
        const bool in = unsigned(j - ps) < unsigned(pl);
        int32_t mp = NEG32, dp = NEG32;
        if (in) {
          mp = g[j - ps];
          dp = g[pl + j - ps];
          Mx[k] = maxs(Mx[k], prev);
          Dx[k] = maxs(Dx[k], maxs(dp + E, mp + O));
        }
        prev = mp;
      }
    }
  }
  // md and the in-block scan x[k] = max over k' <= k of md[k'] + O + (k-k')E
  int32_t X[C];
#pragma unroll
  for (int k = 0; k < C; ++k) {
    const int j = j0 + k;
    const int32_t prof = j < stop ? mrow[seq[j]] : 0;
    Mx[k] = maxs(Mx[k] + prof, Dx[k]);  // Mx now holds md
    X[k] = Mx[k] + O;
    if (k > 0) X[k] = maxs(X[k], X[k - 1] + E);
  }
  // lane aggregates: y_l = max over k < start + C(l+1) of md[k] + O + shift
  int32_t y = X[C - 1];
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int32_t v = __shfl_up_sync(FULL, y, d);
    if (lane >= d) y = maxs(y, v + d * C * E);
  }
  int32_t cin = __shfl_up_sync(FULL, y, 1);
  cin = lane == 0 ? NEG32 : maxs(cin, NEG32 + C * lane * E);
  __syncwarp();  // every predecessor read of the ring precedes this row's writes
  if (j0 < stop) {
    const int o = C * lane;
#pragma unroll
    for (int k0 = 0; k0 < C; k0 += 4) {
      if (j0 + k0 < stop) {
        int32_t iv[4], mv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int k = k0 + q;
          iv[q] = k == 0 ? cin : maxs(X[k - 1], cin + k * E);
          mv[q] = maxs(Mx[k], iv[q]);
          const int j = j0 + k;
          sm->ring_m[out_slot][j & (RING_W - 1)] = mv[q];
          sm->ring_d[out_slot][j & (RING_W - 1)] = Dx[k];
          if (adapt && mv[q] > bestv) {
            bestv = mv[q];
            bestj = j;
          }
        }
        *reinterpret_cast<int4 *>(R + o + k0) = make_int4(mv[0], mv[1], mv[2], mv[3]);
        *reinterpret_cast<int4 *>(R + len + o + k0) = make_int4(Dx[k0], Dx[k0 + 1], Dx[k0 + 2], Dx[k0 + 3]);
        *reinterpret_cast<int4 *>(R + 2 * len + o + k0) = make_int4(iv[0], iv[1], iv[2], iv[3]);
      }
    }
  }
}

// Dispatches one int32 row to the blocked tile of the right width.
__device__ __forceinline__ void dp_row_fast(int lane, int start, int len, int32_t *R, const int32_t *seq,
                                            const int32_t *mrow, int32_t E, int32_t O, unsigned vmask, int ps,
                                            int pl, int slot, const int32_t *g, WarpSmem *sm, int out_slot,
                                            bool adapt, int32_t &bv, int &bj) {
  if (len <= 128)
    dp_row_blocked<4>(lane, start, len, R, seq, mrow, E, O, vmask, ps, pl, slot, g, sm, out_slot, adapt, bv, bj);
  else if (len <= 256)
    dp_row_blocked<8>(lane, start, len, R, seq, mrow, E, O, vmask, ps, pl, slot, g, sm, out_slot, adapt, bv, bj);
  else
    dp_row_blocked<16>(lane, start, len, R, seq, mrow, E, O, vmask, ps, pl, slot, g, sm, out_slot, adapt, bv, bj);
}

// One row by the generic interleaved loop (int64 kernel, rows wider than
// RING_W, or more than 32 predecessors): 32-column chunks, predecessor rows
// from the arena, a warp-shuffle scan per chunk with a serial carry.
template <typename S>
__device__ __forceinline__ void dp_row_generic(int lane, int start, int len, S *R, const S *A, const Scratch &s,
                                               int pb, int pc, const int32_t *mrow, S E, S O, bool adapt, S &bestv,
                                               int &bestj) {
  constexpr S NEGV = ScoreTraits<S>::NEGV;
  const int stop = start + len;
  S carry = NEGV;
  for (int c0 = start; c0 < stop; c0 += 32) {
    const int j = c0 + lane;
    const bool valid = j < stop;
    S M = NEGV, D = NEGV;
    if (valid) {
      for (int t = 0; t < pc; ++t) {
        const int p = s.pred[pb + t].x;
        if (p < 0) continue;
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
      if (adapt && Mf > bestv) {
        bestv = Mf;
        bestj = j;
      }
    }
    carry = shfl_s(x, 31);
  }
}

// Row 0 (align.rs:737-750), serial on lane 0.
template <typename S>
__device__ __forceinline__ void dp_row0(S *R, int len, S s00, S E, S O) {
  constexpr S NEGV = ScoreTraits<S>::NEGV;
  for (int c = 0; c < len; ++c) {
    R[c] = NEGV;
    R[len + c] = NEGV;
  }
  R[0] = s00;
  R[2 * len] = NEGV;
  for (int c = 1; c < len; ++c) {
    const S ins = maxs<S>(R[2 * len + c - 1] + E, R[c - 1] + O);
    R[2 * len + c] = ins;
    R[c] = maxs<S>(R[c], ins);
  }
}

// One DP kernel invocation (poa_simd_arena, align.rs:588-911, or
// poa_scalar_i64, align.rs:913-1162) by a whole warp.
template <typename S>
__device__ int32_t poa_kernel(Job *J, const DevParams &P, char *arena, int64_t arena_bytes, int beg_id, int end_id,
                              const uint8_t *query, int qlen, bool adaptive_arg, uint64_t band_b, uint64_t f,
                              Scratch &s, int *n_items, Work *cells, WarpSmem *sm) {
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
  const S s00 = S(P.matrix[P.unknown * P.sigma + P.unknown]);
  __syncwarp();
  int32_t st = guides(J, s, beg, end, n, sm ? sm->gring_v : nullptr, sm ? sm->gring_s : nullptr);
  if (st != ST_OK) return st;
  const bool do_adapt = f != 0 && adaptive;
  if (do_adapt) {
    for (int i = lane; i < n; i += 32) {
      s.peak[i] = 0;
      s.streak[i] = 0;
      s.peak_left[i] = m;
      s.peak_right[i] = 0;
      s.offset_left[i] = 0;
      s.offset_right[i] = 0;
      s.extra[i] = 0;
    }
  }
  S *A = reinterpret_cast<S *>(s.dp);
  const int64_t cap = s.dp_bytes / int64_t(sizeof(S));
  uint64_t row_cells = 0;
  constexpr bool kFastType = sizeof(S) == 4;
  const bool smem_matrix = P.sigma * P.sigma <= SMEM_MATRIX;
  if (sm) {
    if (lane < RING_ROWS) sm->ring_row[lane] = -1;
    if (smem_matrix)
      for (int k = lane; k < P.sigma * P.sigma; k += 32) sm->matrix[k] = P.matrix[k];
  }
  __syncwarp();
  if (!do_adapt) {
    // Static band (align.rs:711-734 with f == 0 or without adaptive band):
    // every row's band is fixed once the guides are known, so the warp plans
    // all rows at once (band, base code, arena offset). The first failing row
    // in row order gives the reference's status.
    int64_t tot = 0;
    int err_code = ST_OK;
    uint64_t err_cells = 0;
    for (int i0 = 0; i0 < n; i0 += 32) {
      const int i = i0 + lane;
      int start = 0, len = 0, code = ST_OK;
      if (i < n) {
        const int64_t hi = s.head[i], ti = s.tail[i];
        if (hi != NEG64 && ti != NEG64) {
          int64_t left, right;
          if (f == 0) {
            left = 0;
            right = m;
          } else {
            left = maxs<int64_t>(mins(hi, m - ti) - band, 0);
            right = mins<int64_t>(maxs(hi, m - ti) + band, m);
          }
          if (left > right || right < 0) {
            code = ST_BAND_NO_INTERSECT;
          } else {
            start = int(left / 8 * 8);
            len = int((right / 8 + 1) * 8) - start;
            if (i == 0 && start != 0) code = ST_BAND_EXCLUDES_SOURCE;
          }
        }
        s.row_base[i] = (i == n - 1) ? P.unknown : int(J->base[J->rank_to_node[beg + i]]);
      }
      const int64_t own = 3 * int64_t(len);
      int64_t inc = own;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int64_t v = shfl_up_s(inc, d);
        if (lane >= d) inc += v;
      }
      if (i < n) {
        s.row_start[i] = start;
        s.row_len[i] = len;
        s.row_off[i] = tot + inc - own;
      }
      const unsigned bad = __ballot_sync(FULL, code != ST_OK);
      if (bad && err_code == ST_OK) {
        const int l = __ffs(bad) - 1;
        err_code = __shfl_sync(FULL, code, l);
        // rows the reference allocates before it stops (row 0 is allocated
        // before its source check)
        const int64_t before = shfl_s(int64_t(inc - own), l) / 3;
        const int flen = __shfl_sync(FULL, len, l);
        err_cells = row_cells + uint64_t(before) + (err_code == ST_BAND_EXCLUDES_SOURCE ? uint64_t(flen) : 0);
      }
      const int64_t group = shfl_s(inc, 31);
      row_cells += uint64_t(group / 3);
      tot += group;
    }
    if (err_code != ST_OK) {
      cells->cells += err_cells;
      cells->dp_bytes += err_cells * 3 * sizeof(S);
      return err_code;
    }
    if (tot > cap) return ST_ARENA_FULL;
    __syncwarp();
    const int etot = s.pred_start[n - 1] + s.pred_cnt[n - 1];
    for (int e = lane; e < etot; e += 32) {
      const int p = s.pred[e].x;
      if (p >= 0) {
        s.pmeta[e] = make_int4(p, s.row_start[p], s.row_len[p], 0);
        s.pmeta_off[e] = s.row_off[p];
      } else {
        s.pmeta[e] = make_int4(-1, 0, 0, 0);
        s.pmeta_off[e] = 0;
      }
    }
    __syncwarp();
    if (s.row_len[0] > 0 && lane == 0) dp_row0<S>(A + s.row_off[0], s.row_len[0], s00, E, O);
    __syncwarp();
    // rows 1..n-1, software-pipelined: row i+2's descriptor and row i+1's
    // predecessor metadata are loaded while row i computes
    auto desc = [&](int r) { return make_int4(s.row_start[r], s.row_len[r], s.pred_start[r], s.pred_cnt[r]); };
    int4 d1 = n > 1 ? desc(1) : make_int4(0, 0, 0, 0);
    int4 d2 = n > 2 ? desc(2) : make_int4(0, 0, 0, 0);
    int64_t o1 = n > 1 ? s.row_off[1] : 0, o2 = n > 2 ? s.row_off[2] : 0;
    int b1 = n > 1 ? s.row_base[1] : 0, b2 = n > 2 ? s.row_base[2] : 0;
    int4 m1 = make_int4(-1, 0, 0, 0);
    int64_t mo1 = 0;
    if (n > 1 && lane < d1.w) {
      m1 = s.pmeta[d1.z + lane];
      mo1 = s.pmeta_off[d1.z + lane];
    }
    for (int i = 1; i < n; ++i) {
      const int4 d = d1;
      const int64_t off = o1;
      const int base = b1;
      const int4 mt = m1;
      const int64_t mo = mo1;
      d1 = d2;
      o1 = o2;
      b1 = b2;
      m1 = make_int4(-1, 0, 0, 0);
      mo1 = 0;
      if (i + 1 < n && lane < d1.w) {
        m1 = s.pmeta[d1.z + lane];
        mo1 = s.pmeta_off[d1.z + lane];
      }
      if (i + 2 < n) {
        d2 = desc(i + 2);
        o2 = s.row_off[i + 2];
        b2 = s.row_base[i + 2];
      }
      const int start = d.x, len = d.y, pb = d.z, pc = d.w;
      if (len == 0) continue;
      S *R = A + off;
      if (kFastType && sm && len <= RING_W && pc <= 32) {
        const int p = mt.x;
        const bool ok = p >= 0 && mt.z > 0;
        const int sl = p >= 0 ? p % RING_ROWS : 0;
        const int my_slot = (ok && sm->ring_row[sl] == p) ? sl : -1;
        const int32_t *my_g = reinterpret_cast<const int32_t *>(A) + mo;
        const unsigned vmask = __ballot_sync(FULL, ok);
        const int32_t *mrow = smem_matrix ? sm->matrix + base * P.sigma : P.matrix + base * P.sigma;
        int32_t bv = INT32_MIN;
        int bj = INT32_MAX;
        dp_row_fast(lane, start, len, reinterpret_cast<int32_t *>(R), s.seq, mrow, int32_t(E), int32_t(O), vmask,
                    mt.y, mt.z, my_slot, my_g, sm, i % RING_ROWS, false, bv, bj);
        __syncwarp();
        if (lane == 0) sm->ring_row[i % RING_ROWS] = i;
        __syncwarp();
        continue;
      }
      if (sm && lane == 0) sm->ring_row[i % RING_ROWS] = -1;
      S bv = ScoreTraits<S>::LOWEST;
      int bj = INT32_MAX;
      dp_row_generic<S>(lane, start, len, R, A, s, pb, pc, P.matrix + base * P.sigma, E, O, false, bv, bj);
      __syncwarp();
    }
  } else {
    // Adaptive band (align.rs:711-729, 829-897): row i's band follows its
    // predecessors' peaks, so rows are planned one at a time.
    int64_t cursor = 0;
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
      const int64_t x = mins(mins(s.peak_left[i], hi + s.offset_left[i]), m - ti);
      const int64_t y = maxs(maxs(s.peak_right[i], hi + s.offset_right[i]), m - ti);
      const int64_t left = maxs<int64_t>(x - band - s.extra[i], 0);
      const int64_t right = mins<int64_t>(y + band + s.extra[i], m);
      if (left > right || right < 0) {
        cells->cells += row_cells;
        cells->dp_bytes += row_cells * 3 * sizeof(S);
        return ST_BAND_NO_INTERSECT;
      }
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
        if (start != 0) {
          cells->cells += row_cells;
          cells->dp_bytes += row_cells * 3 * sizeof(S);
          return ST_BAND_EXCLUDES_SOURCE;
        }
        if (lane == 0) dp_row0<S>(R, len, s00, E, O);
        __syncwarp();
        continue;
      }
      const int node = J->rank_to_node[beg + i];
      const int base = (i == n - 1) ? P.unknown : int(J->base[node]);
      const int pb = s.pred_start[i], pc = s.pred_cnt[i];
      S bestv = ScoreTraits<S>::LOWEST;
      int bestj = INT32_MAX;
      if (kFastType && sm && len <= RING_W && pc <= 32) {
        int my_ps = 0, my_pl = 0, my_slot = -1;
        const int32_t *my_g = nullptr;
        bool ok = false;
        if (lane < pc) {
          const int p = s.pred[pb + lane].x;
          if (p >= 0) {
            my_ps = s.row_start[p];
            my_pl = s.row_len[p];
            my_g = reinterpret_cast<const int32_t *>(A) + s.row_off[p];
            const int sl = p % RING_ROWS;
            my_slot = sm->ring_row[sl] == p ? sl : -1;
            ok = my_pl > 0;
          }
        }
        const unsigned vmask = __ballot_sync(FULL, ok);
        const int32_t *mrow = smem_matrix ? sm->matrix + base * P.sigma : P.matrix + base * P.sigma;
        int32_t bv = INT32_MIN;
        int bj = INT32_MAX;
        dp_row_fast(lane, start, len, reinterpret_cast<int32_t *>(R), s.seq, mrow, int32_t(E), int32_t(O), vmask,
                    my_ps, my_pl, my_slot, my_g, sm, i % RING_ROWS, true, bv, bj);
        __syncwarp();
        if (lane == 0) sm->ring_row[i % RING_ROWS] = i;
        bestv = S(bv);
        bestj = bj;
      } else {
        if (sm && lane == 0) sm->ring_row[i % RING_ROWS] = -1;
        dp_row_generic<S>(lane, start, len, R, A, s, pb, pc, P.matrix + base * P.sigma, E, O, true, bestv, bestj);
      }
      __syncwarp();
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
                                    Scratch &s, int *n_items, Work *cells, WarpSmem *sm) {
  const bool use32 = P.kernel == 1 || (P.kernel == 0 && i32_scores_safe(J, P, beg_id, end_id, qlen));
  if (use32)
    return poa_kernel<int32_t>(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive, band_b, f, s, n_items, cells,
                               sm);
  return poa_kernel<int64_t>(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive, band_b, f, s, n_items, cells,
                             sm);
}

// poa (align.rs:192-211): on an alignment error with f != 0, retry with the
// full matrix (f = 0, static band).
__device__ inline int32_t poa_retry(Job *J, const DevParams &P, char *arena, int64_t bytes, int beg_id, int end_id,
                                    const uint8_t *q, int qlen, bool adaptive, uint64_t band_b, Scratch &s,
                                    int *n_items, Work *cells, WarpSmem *sm) {
  int32_t st = poa_inner(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive, band_b, P.f, s, n_items, cells, sm);
  if (is_alignment_error(st) && P.f != 0)
    st = poa_inner(J, P, arena, bytes, beg_id, end_id, q, qlen, false, band_b, 0, s, n_items, cells, sm);
  return st;
}

// align::align (align.rs:81-98) for unseeded parameters; writes s.items.
__device__ inline int32_t align_query(Job *J, const DevParams &P, char *arena, int64_t bytes, const uint8_t *q,
                                      int qlen, Scratch &s, int *n_items, Work *cells, WarpSmem *sm) {
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
  return poa_retry(J, P, arena, bytes, 0, 1, q, qlen, P.adaptive != 0, P.b, s, n_items, cells, sm);
}

// Splices a read's new nodes into the current topological order (warp-wide):
// each run of consecutive new nodes on the path is placed right after the
// pre-existing path node before it. The result is a valid topological order
// when consecutive pre-existing path nodes keep increasing ranks; otherwise
// nothing is changed and false is returned (the caller then runs the LIFO
// toposort of graph.rs:125-178). With a static band and no seeding the rank
// order does not change any alignment: band guides, DP states and traceback
// choices depend only on the predecessor / successor lists in insertion order.
__device__ inline bool reorder_incremental(Job *J, const int4 *items, int n_items, int n_old, char *buf,
                                           int64_t buf_bytes) {
  const int lane = threadIdx.x & 31;
  const int n_new = J->n_nodes;
  if (J->n_rank != n_old || n_items <= 0) return false;
  if (int64_t(4) * (2 * int64_t(n_old) + n_new) > buf_bytes) return false;
  int32_t *add = reinterpret_cast<int32_t *>(buf);
  int32_t *first = add + n_old;
  int32_t *nr2n = first + n_old;
  for (int r = lane; r < n_old; r += 32) add[r] = 0;
  __syncwarp();
  long long carry = -1;  // last pre-existing path item as (index << 32 | rank)
  bool bad = false;
  for (int t0 = 0; t0 < n_items; t0 += 32) {
    const int t = t0 + lane;
    const int id = t < n_items ? items[t].w : -1;
    const bool old = t < n_items && id >= 0 && id < n_old;
    const int rk = old ? J->rank[id] : 0;
    long long inc = old ? ((long long)t << 32) | (unsigned)rk : -1;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const long long v = __shfl_up_sync(FULL, inc, d);
      if (lane >= d) inc = inc > v ? inc : v;
    }
    long long prev = __shfl_up_sync(FULL, inc, 1);
    if (lane == 0) prev = -1;
    prev = prev > carry ? prev : carry;
    if (old && prev >= 0) {
      const int pt = int(prev >> 32), pr = int(prev & 0xffffffffLL);
      if (pr >= rk) bad = true;
      if (t - pt - 1 > 0) {
        add[pr] = t - pt - 1;
        first[pr] = items[pt + 1].w;
      }
    }
    const long long last = __shfl_sync(FULL, inc, 31);
    carry = last > carry ? last : carry;
  }
  if (__any_sync(FULL, bad) || carry < 0) return false;
  if (lane == 0) {
    const int pt = int(carry >> 32), pr = int(carry & 0xffffffffLL);
    if (n_items - pt - 1 > 0) {
      add[pr] = n_items - pt - 1;
      first[pr] = items[pt + 1].w;
    }
  }
  __syncwarp();
  int shift = 0;
  for (int r0 = 0; r0 < n_old; r0 += 32) {
    const int r = r0 + lane;
    const int a = r < n_old ? add[r] : 0;
    int inc = a;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int v = __shfl_up_sync(FULL, inc, d);
      if (lane >= d) inc += v;
    }
    if (r < n_old) {
      const int node = J->rank_to_node[r];
      const int nr = r + shift + inc - a;
      nr2n[nr] = node;
      J->rank[node] = nr;
      for (int k = 0; k < a; ++k) {
        const int id = first[r] + k;
        nr2n[nr + 1 + k] = id;
        J->rank[id] = nr + 1 + k;
      }
    }
    shift += __shfl_sync(FULL, inc, 31);
  }
  __syncwarp();
  for (int r = lane; r < n_new; r += 32) J->rank_to_node[r] = nr2n[r];
  if (lane == 0) J->n_rank = n_new;
  __syncwarp();
  return true;
}

// The exact LIFO order (graph.rs:125-178) when the current one came from
// reorder_incremental (lane 0; the arena holds the degree and stack arrays).
__device__ inline int32_t finalize_order(Job *J, char *arena, int64_t bytes) {
  if (J->order_exact) return ST_OK;
  if (int64_t(J->n_nodes) * 8 > bytes) return ST_ARENA_FULL;
  int32_t *deg = reinterpret_cast<int32_t *>(arena);
  const int32_t st = toposort(J, deg, deg + J->n_nodes);
  if (st == ST_OK) J->order_exact = 1;
  return st;
}

// One step of extend_graph (lib.rs:199-201): align, add_path, toposort(false).
// Capacity is checked before the DP so a full graph stops cleanly.
__device__ inline int32_t extend_one(Job *J, const DevParams &P, char *arena, int64_t bytes, const uint8_t *q,
                                     int qlen, int r, WarpSmem *sm) {
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
  int32_t st = align_query(J, P, arena, bytes, q, qlen, s, &n_items, &cells, sm);
  if (st != ST_OK) return st;
  const int n_old = J->n_nodes;
  if (lane == 0) st = add_path(J, P, r, s.items, n_items);
  st = __shfl_sync(FULL, st, 0);
  __syncwarp();
  if (st != ST_OK) return st;
  // order-free reads (static band, no seeding) keep a spliced order; the
  // others, and any splice that would break the order, use the LIFO toposort
  const bool order_free = P.relaxed_order && !P.seeding && !(P.adaptive && P.f != 0);
  bool spliced = false;
  if (order_free) spliced = reorder_incremental(J, s.items, n_items, n_old, s.dp, s.dp_bytes);
  if (lane == 0) {
    if (spliced) {
      J->order_exact = 0;
    } else {
      // toposort runs after add_path has consumed s.items, so its scratch may
      // overwrite the front of the arena.
      int32_t *deg = reinterpret_cast<int32_t *>(arena);
      int32_t *stack = deg + nodes_after;
      st = toposort(J, deg, stack);
      J->order_exact = 1;
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
