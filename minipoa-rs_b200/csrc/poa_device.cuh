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
  ST_OUT_TOO_SMALL = 103,  // a caller's output buffer holds fewer items than the path
  ST_WAVE_STALL = 104,     // internal: a row-wavefront step found no row able to advance
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
  int32_t row_wave;       // static-band int32 rows: 0 one at a time, 1 wavefront where suited, 2 wavefront
  int32_t byte_prof;      // sigma <= 8 and every score fits a signed byte (dp_wave's packed profile)
  int32_t giant_alone;    // batched runs: a giant's block keeps only the giant and its helpers
  int32_t wide_rows;      // batched runs: the kernel form with bands up to 2048 columns in striped segments
  int32_t teams;          // batched runs: one 4-warp block per job (a job and its three helpers)
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
  int32_t seq_base;  // sequence id of read 0 (reads extending an imported graph follow its records)
  const int32_t *read_id;  // when set, the sequence id of each read (reads in guide order, -p)
  // outcome
  int32_t status, err_i, err_j, n_items;
  int32_t order_exact;  // 1 when rank is the reference's LIFO toposort order
  int32_t giant;        // batched runs: a job far above the average size (gets its SM to itself)
  char *arena;          // when set, the job's own DP arena (serving); else the warp slot's
  int64_t arena_bytes;
  int32_t *done_flag;   // when set (host-mapped memory), raised once the job leaves the kernel
  uint64_t cells;       // DP cells of completed reads (retries included)
  uint64_t dp_bytes;    // DP state bytes stored for those cells (M, D, I)
  uint64_t pred_cells;  // predecessor-cell updates of those reads (band overlaps)
  uint64_t far_preds;   // predecessor rows read from the arena (left the ring)
  uint64_t rows_g4;     // rows of the 4-stripe tile (385-512 columns)
  uint64_t rows_generic;  // rows of the generic row (wider bands, many predecessors, i64)
  int32_t coop;         // 1 once a read of the job ran cooperative rows
  int32_t wave_reads;   // reads whose static-band DP ran as a row wavefront
  uint64_t phase[4];    // profiling builds (POA_PHASE_CYCLES): warp cycles in band guides,
                        // DP rows, traceback, graph update (add_path + rank order)
};

// Work counted by one alignment: 8-aligned band cells, the bytes of DP
// state they stored, the predecessor-cell updates (the sum over rows of each
// in-band predecessor's band overlap, the reference's predecessor loop
// trip count) and which row paths ran.
struct Work {
  uint64_t cells, dp_bytes, pred_cells, far_preds, rows_g4, rows_generic;
  int32_t coop, wave;
  uint64_t phase[4];
};

// Warp cycle counters of the read loop's phases, compiled in for profiling
// builds only (-DPOA_PHASE_CYCLES); otherwise the reads are constant zero.
#ifdef POA_PHASE_CYCLES
__device__ __forceinline__ uint64_t phase_clock() { return clock64(); }
#else
__device__ __forceinline__ uint64_t phase_clock() { return 0; }
#endif

// Per-read scratch carved from the front of a warp slot's arena.
struct Scratch {
  int64_t *head, *tail, *support, *support_b, *row_off, *wsum;
  int64_t *peak, *streak, *peak_left, *peak_right, *offset_left, *offset_right, *extra;
  int32_t *row_start, *row_len, *pred_start, *pred_cnt, *succ_start, *succ_cnt;
  int2 *pred;          // (row, weight) in incoming order; row = -1 once head is NEG
  int2 *succ;          // (row, weight) in outgoing order, range filtered
  int32_t *row_base;   // base code a row scores with (N for the last row)
  int4 *pmeta;         // per pred entry: (row, band start, band length, -)
  int64_t *pmeta_off;  // per pred entry: the predecessor row's arena offset
  int4 *tb;            // traceback, two per pred entry: the predecessor row's descriptor (see fill_tb)
  int4 *planc;         // static band, per row: (band start, band length, pred_start, pred_cnt | base << 24)
  int4 *pent;          // static band, per pred entry: where the predecessor's states are (see plan_rows)
  int32_t *nf;         // static band, per row: rows before it that did not go through the ring
  int4 *wrec;          // row wavefront, per row: an 80-byte record (see plan_wave)
  int32_t *seq;        // encoded, padded query
  uint8_t *seq8;       // the same, one byte per column (when it does not fit shared memory)
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
  s.support_b = (int64_t *)take(N * 8);
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
  s.tb = (int4 *)take(int64_t(e + 1) * 32);
  s.planc = (int4 *)take(N * 16);
  s.pent = (int4 *)take(int64_t(e + 1) * 16);
  s.nf = (int32_t *)take(N * 4);
  s.wrec = (int4 *)take(N * 80);
  s.seq = (int32_t *)take((padded + 32) * 4);
  s.seq8 = (uint8_t *)take(padded + 32);
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

// add_path (graph.rs:82-122) by the whole warp, one item per lane. It covers
// the case every alignment path is in: the items name pairwise distinct
// nodes. That holds when no pre-existing node is named twice (checked with
// `mark`, n_nodes zeroed words of scratch, or, without scratch, by strictly
// increasing ranks), no item names the sink, and no two items create the
// same column sibling (same parent and base); those facts are checked first,
// and when one fails nothing has been changed and false is returned, so the
// caller runs the serial add_path. With distinct nodes every node gains at
// most one incoming and one outgoing edge, so the edges are independent and
// each lane appends its own; new node ids are handed out in path order by a
// prefix count, as the serial loop does. Edge-list chunks may be numbered in
// another order than the serial loop numbers them; chunk numbers are storage
// only, the lists keep their insertion order. Invalid items and capacity
// give the serial function's status (true is returned, graph unchanged).
__device__ inline bool add_path_warp(Job *J, const DevParams &P, int seq_id, int4 *items, int n, int32_t *status,
                                     int32_t *mark = nullptr) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int n_old = J->n_nodes;
  *status = ST_OK;
  for (int t0 = 0; t0 < n; t0 += 32) {
    const int t = t0 + lane;
    int code = ST_OK;
    if (t < n) {
      const int4 it = items[t];
      if (it.y < 0 || it.y >= P.sigma)
        code = ST_BASE_OUTSIDE;
      else if ((it.x >= 0 && it.x >= n_old) || (it.z >= 0 && it.z >= n_old))
        code = ST_UNKNOWN_NODE;
    }
    const unsigned bad = __ballot_sync(FULL, code != ST_OK);
    if (bad) {
      *status = __shfl_sync(FULL, code, __ffs(bad) - 1);
      return true;
    }
  }
  if (n_old + n > J->node_cap || J->n_chunks + 2 * (n + 1) > J->chunk_cap || J->path_used + n > J->path_cap ||
      J->n_paths + 1 > J->max_paths) {
    *status = ST_GRAPH_FULL;
    return true;
  }
  // resolve: .w = node id (existing), -1 (new node), -(parent + 2) (new
  // column sibling, whose (parent, base) slot of `aligned` is claimed)
  bool ok = true;
  int rank_carry = -1;
  if (mark) {
    for (int v = lane; v < n_old; v += 32) mark[v] = 0;
    __syncwarp();
  }
  for (int t0 = 0; t0 < n; t0 += 32) {
    const int t = t0 + lane;
    int w = -1, rk = -1;
    bool fail = false;
    if (t < n) {
      const int4 it = items[t];
      if (it.x >= 0) {
        w = it.x;
      } else if (it.z >= 0) {
        const int parent = J->parent[it.z];
        int32_t *slot = &J->aligned[int64_t(parent) * P.sigma + it.y];
        const int a = *slot;
        if (a >= 0) {
          w = a;
        } else {
          w = -(parent + 2);
          fail = atomicMin(slot, INT32_MIN + t) != -1;  // another item claimed it first
        }
      }
      if (w >= 0) {
        if (mark)
          fail = fail || atomicExch(&mark[w], 1) != 0;  // named twice
        else
          rk = J->rank[w];
        fail = fail || w == 1;
      }
      items[t].w = w;
    }
    int pm = rk;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int v = __shfl_up_sync(FULL, pm, d);
      if (lane >= d) pm = max(pm, v);
    }
    int before = __shfl_up_sync(FULL, pm, 1);
    if (lane == 0) before = -1;
    before = max(before, rank_carry);
    if (!mark && w >= 0 && rk <= before) fail = true;
    rank_carry = max(rank_carry, __shfl_sync(FULL, pm, 31));
    if (__any_sync(FULL, fail)) ok = false;
  }
  __syncwarp();
  if (!ok) {
    for (int t = lane; t < n; t += 32) {
      const int4 it = items[t];
      if (it.w <= -2) atomicExch(&J->aligned[int64_t(-(it.w + 2)) * P.sigma + it.y], -1);
    }
    __syncwarp();
    return false;
  }
  // nodes, in path order
  const int path_base = J->path_used;
  int new_carry = 0, path_carry = 0;
  for (int t0 = 0; t0 < n; t0 += 32) {
    const int t = t0 + lane;
    int4 it = make_int4(0, 0, 0, 0);
    if (t < n) it = items[t];
    const bool fresh = t < n && it.w < 0;
    const unsigned fm = __ballot_sync(FULL, fresh);
    int id = it.w;
    if (fresh) {
      id = n_old + new_carry + __popc(fm & lt);
      const int parent = it.w <= -2 ? -(it.w + 2) : id;
      J->base[id] = uint8_t(it.y);
      J->parent[id] = parent;
      J->rank[id] = 0;
      J->coverage[id] = 0;
      for (int c = 0; c < P.sigma; ++c) J->aligned[int64_t(id) * P.sigma + c] = c == it.y ? id : -1;
      J->in_cnt[id] = 0;
      J->out_cnt[id] = 0;
      J->in_head[id] = J->in_tail[id] = -1;
      J->out_head[id] = J->out_tail[id] = -1;
      if (it.w <= -2) J->aligned[int64_t(parent) * P.sigma + it.y] = id;
      items[t].w = id;
    }
    const bool on_path = t < n && id >= 2;
    const unsigned pmask = __ballot_sync(FULL, on_path);
    if (on_path) J->path_items[path_base + path_carry + __popc(pmask & lt)] = id;
    new_carry += __popc(fm);
    path_carry += __popc(pmask);
  }
  __syncwarp();
  // edges k = 1..K: items[k-1] -> items[k], and the last item (or the
  // source) -> sink
  const int K = n > 0 ? n : 1;
  int chunk_carry = J->n_chunks, in_added = 0;
  for (int k0 = 1; k0 <= K; k0 += 32) {
    const int k = k0 + lane;
    const bool live = k <= K;
    int from = 0, to = 1;
    if (live) {
      from = n > 0 ? items[k - 1].w : 0;
      to = k < n ? items[k].w : 1;
    }
    const bool act = live && from != to;
    bool out_new = false, in_new = false;
    if (act) {
      // a list of a pre-existing node cannot hold a new node yet
      const bool both_old = from < n_old && to < n_old;
      out_new = !(both_old && list_bump(J, J->out_head, J->out_cnt, from, to));
      in_new = !(both_old && list_bump(J, J->in_head, J->in_cnt, to, from));
    }
    const int oc = out_new ? J->out_cnt[from] : 1, ic = in_new ? J->in_cnt[to] : 1;
    const int need = int(out_new && oc % CHUNK == 0) + int(in_new && ic % CHUNK == 0);
    int inc = need;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int v = __shfl_up_sync(FULL, inc, d);
      if (lane >= d) inc += v;
    }
    int ch = chunk_carry + inc - need;
    auto append = [&](int32_t *head, int32_t *tail, int32_t *cnt, int node, int id, int c) {
      const int slot = c % CHUNK;
      int chunk;
      if (slot == 0) {
        chunk = ch++;
        J->chunk_next[chunk] = -1;
        if (c == 0)
          head[node] = chunk;
        else
          J->chunk_next[tail[node]] = chunk;
        tail[node] = chunk;
      } else {
        chunk = tail[node];
      }
      J->chunk_id[int64_t(chunk) * CHUNK + slot] = id;
      J->chunk_w[int64_t(chunk) * CHUNK + slot] = 1;
      cnt[node] = c + 1;
    };
    if (out_new) append(J->out_head, J->out_tail, J->out_cnt, from, to, oc);
    if (in_new) append(J->in_head, J->in_tail, J->in_cnt, to, from, ic);
    if (act) J->coverage[to] += 1;
    chunk_carry += __shfl_sync(FULL, inc, 31);
    in_added += __popc(__ballot_sync(FULL, in_new));
  }
  __syncwarp();
  if (lane == 0) {
    J->n_nodes = n_old + new_carry;
    J->path_used = path_base + path_carry;
    J->n_chunks = chunk_carry;
    J->n_edges += in_added;
    J->path_seq[J->n_paths] = seq_id;
    J->path_off[J->n_paths + 1] = J->path_used;
    J->n_paths += 1;
  }
  __syncwarp();
  return true;
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
constexpr int GRING = 32;
__device__ inline int32_t guides(const Job *J, Scratch &s, int beg, int end, int n, int64_t *ring_v,
                                 int64_t *ring_s, int64_t *ring_b, Work *w) {
  const int lane = threadIdx.x & 31;
  const uint64_t tg0 = phase_clock();
  int pbase = 0, sbase = 0;
  for (int i0 = 0; i0 < n; i0 += 32) {
    const int i = i0 + lane;
    int cin = 0, cout = 0;
    int64_t wsum = 0;
    int node = -1;
    // the first chunk of each list (CHUNK entries) is read as vectors; longer
    // lists are walked again below
    int4 in_id = make_int4(0, 0, 0, 0), in_w = in_id, out_id = in_id, out_w = in_id;
    int in_n = 0, out_n = 0, in_r[CHUNK] = {0, 0, 0, 0}, out_r[CHUNK] = {0, 0, 0, 0};
    if (i < n) {
      node = J->rank_to_node[beg + i];
      in_n = J->in_cnt[node];
      out_n = J->out_cnt[node];
      const int ih = J->in_head[node], oh = J->out_head[node];
      if (in_n > 0) {
        in_id = *reinterpret_cast<const int4 *>(J->chunk_id + int64_t(ih) * CHUNK);
        in_w = *reinterpret_cast<const int4 *>(J->chunk_w + int64_t(ih) * CHUNK);
      }
      if (out_n > 0) {
        out_id = *reinterpret_cast<const int4 *>(J->chunk_id + int64_t(oh) * CHUNK);
        out_w = *reinterpret_cast<const int4 *>(J->chunk_w + int64_t(oh) * CHUNK);
      }
      const int iid[CHUNK] = {in_id.x, in_id.y, in_id.z, in_id.w};
      const int iw[CHUNK] = {in_w.x, in_w.y, in_w.z, in_w.w};
      const int oid[CHUNK] = {out_id.x, out_id.y, out_id.z, out_id.w};
#pragma unroll
      for (int k = 0; k < CHUNK; ++k) {
        if (k < in_n) in_r[k] = J->rank[iid[k]];
        if (k < out_n) out_r[k] = J->rank[oid[k]];
      }
#pragma unroll
      for (int k = 0; k < CHUNK; ++k) {
        if (k < in_n) {
          wsum += iw[k];
          if (in_r[k] >= beg && in_r[k] < beg + i) ++cin;
        }
        if (k < out_n && out_r[k] > beg + i && out_r[k] <= end) ++cout;
      }
      if (in_n > CHUNK || out_n > CHUNK) {
        int k = 0;
        for_list(J, J->in_head, J->in_cnt, node, [&](int pred, int w) {
          if (k++ < CHUNK) return;
          wsum += w;
          const int r = J->rank[pred];
          if (r >= beg && r < beg + i) ++cin;
        });
        k = 0;
        for_list(J, J->out_head, J->out_cnt, node, [&](int succ, int) {
          if (k++ < CHUNK) return;
          const int r = J->rank[succ];
          if (r > beg + i && r <= end) ++cout;
        });
      }
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
      int kp = ps, ks = ss;
      const int iw[CHUNK] = {in_w.x, in_w.y, in_w.z, in_w.w};
      const int ow[CHUNK] = {out_w.x, out_w.y, out_w.z, out_w.w};
#pragma unroll
      for (int k = 0; k < CHUNK; ++k) {
        if (k < in_n && in_r[k] >= beg && in_r[k] < beg + i) s.pred[kp++] = make_int2(in_r[k] - beg, iw[k]);
        if (k < out_n && out_r[k] > beg + i && out_r[k] <= end) s.succ[ks++] = make_int2(out_r[k] - beg, ow[k]);
      }
      if (in_n > CHUNK || out_n > CHUNK) {
        int k = 0;
        for_list(J, J->in_head, J->in_cnt, node, [&](int pred, int w) {
          if (k++ < CHUNK) return;
          const int r = J->rank[pred];
          if (r >= beg && r < beg + i) s.pred[kp++] = make_int2(r - beg, w);
        });
        k = 0;
        for_list(J, J->out_head, J->out_cnt, node, [&](int succ, int w) {
          if (k++ < CHUNK) return;
          const int r = J->rank[succ];
          if (r > beg + i && r <= end) s.succ[ks++] = make_int2(r - beg, w);
        });
      }
      s.head[i] = NEG64;
      s.tail[i] = NEG64;
      s.support[i] = 0;
    }
    pbase += __shfl_sync(FULL, pin, 31);
    sbase += __shfl_sync(FULL, pout, 31);
  }
  __syncwarp();
  // The serial passes run on every lane in lockstep (each lane computes the
  // same values and writes the same words, so it only ever reads its own
  // writes). Lane l holds the list start, count and first two entries of row
  // i0 + l of the current 32-row block, loaded one block ahead, and the rows
  // read them by shuffle; (head or tail, support) of the last GRING rows sit
  // in a shared-memory ring.
  //
  // The forward pass (head, predecessors) and the backward pass (tail,
  // successors) advance together, one row each per step, so the warp has two
  // independent dependency chains to overlap. The backward pass does not
  // depend on the forward one: the reference starts it from the sink's
  // forward support, but every backward support is that value plus the
  // weights along a path to the sink, so its comparisons (larger support
  // wins a tie of weights) are the same from 0, and only head and tail leave
  // this function. The two passes keep separate support arrays and rings
  // (the backward ring sits in the DP ring's shared memory, unused until the
  // DP).
  struct Lists {
    int start, cnt;
    int2 e0, e1;
  };
  auto load = [&](const int32_t *st, const int32_t *ct, const int2 *ent, int r, bool ok) {
    Lists L{0, 0, make_int2(-1, 0), make_int2(-1, 0)};
    if (ok) {
      L.start = st[r];
      L.cnt = ct[r];
      if (L.cnt > 0) L.e0 = ent[L.start];
      if (L.cnt > 1) L.e1 = ent[L.start + 1];
    }
    return L;
  };
  struct Pass {
    bool forward;
    int64_t *val, *sup, *rv, *rsu;
    const int32_t *st, *ct;
    int2 *ent;
    Lists cur, nxt;
    int lb, lc;
    int2 f0, f1;
    int last;
    int64_t last_v, last_s, my_v, my_s;
    bool my_set;
  };
  const int count = n - 1;  // rows 1..n-1 forward, n-2..0 backward
  auto row_of = [&](const Pass &p, int q) { return p.forward ? 1 + q : n - 2 - q; };
  auto begin = [&](Pass &p) {
    p.nxt = load(p.st, p.ct, p.ent, row_of(p, lane), lane < count);
    // the row computed last (row 0 forward, row n-1 backward, to begin
    // with): most rows' best candidate is that row, read from registers
    p.last = p.forward ? 0 : n - 1;
    p.last_v = p.rv[p.last & (GRING - 1)];
    p.last_s = p.rsu[p.last & (GRING - 1)];
  };
  auto block = [&](Pass &p, int q0) {
    p.cur = p.nxt;
    p.nxt = load(p.st, p.ct, p.ent, row_of(p, q0 + 32 + lane), q0 + 32 + lane < count);
    p.lb = __shfl_sync(FULL, p.cur.start, 0);
    p.lc = __shfl_sync(FULL, p.cur.cnt, 0);
    p.f0 = make_int2(__shfl_sync(FULL, p.cur.e0.x, 0), __shfl_sync(FULL, p.cur.e0.y, 0));
    p.f1 = make_int2(__shfl_sync(FULL, p.cur.e1.x, 0), __shfl_sync(FULL, p.cur.e1.y, 0));
    // the block's results stay in the lanes (lane k: row k of the block)
    // and are stored once at its end
    p.my_v = p.my_s = 0;
    p.my_set = false;
  };
  auto block_end = [&](Pass &p, int q0) {
    if (p.my_set) {
      const int i = row_of(p, q0 + lane);
      p.val[i] = p.my_v;
      p.sup[i] = p.my_s;
    }
  };
  // One row of a pass: the first predecessor (successor) of largest weight,
  // ties to the larger support, among those whose value is set. Rows with at
  // most two candidates (nearly all) read both candidates' values before
  // choosing, and the next row's list entries are taken by shuffle while
  // this row computes.
  auto step = [&](Pass &p, int q0, int k, int lim) {
    const bool forward = p.forward;
    const int i = row_of(p, q0 + k);
    const int pb = p.lb, pc = p.lc;
    const int2 e0 = p.f0, e1 = p.f1;
    const int kn = k + 1 < lim ? k + 1 : k;  // the next row's entries, fetched early
    p.lb = __shfl_sync(FULL, p.cur.start, kn);
    p.lc = __shfl_sync(FULL, p.cur.cnt, kn);
    p.f0 = make_int2(__shfl_sync(FULL, p.cur.e0.x, kn), __shfl_sync(FULL, p.cur.e0.y, kn));
    p.f1 = make_int2(__shfl_sync(FULL, p.cur.e1.x, kn), __shfl_sync(FULL, p.cur.e1.y, kn));
    auto get = [&](int x, int64_t &v, int64_t &sp) {
      if (x == p.last) {
        v = p.last_v;
        sp = p.last_s;
        return;
      }
      const bool near = (forward ? i - x : x - i) < GRING;
      v = near ? p.rv[x & (GRING - 1)] : p.val[x];
      sp = near ? p.rsu[x & (GRING - 1)] : p.sup[x];
    };
    bool have = false;
    int bw = 0;
    int64_t bsup = 0, bval = 0;
    auto consider = [&](const int2 &e, int64_t v, int64_t sp, int t) {
      if (v == NEG64) {
        if (forward) p.ent[pb + t].x = -1;
        return;
      }
      if (!have || e.y > bw || (e.y == bw && sp > bsup)) {
        have = true;
        bw = e.y;
        bsup = sp;
        bval = v;
      }
    };
    if (pc <= 2) {
      int64_t v0 = NEG64, s0 = 0, v1 = NEG64, s1 = 0;
      if (pc >= 1) get(e0.x, v0, s0);
      if (pc >= 2) get(e1.x, v1, s1);
      if (pc >= 1) consider(e0, v0, s0, 0);
      if (pc >= 2) consider(e1, v1, s1, 1);
    } else {
      for (int t = 0; t < pc; ++t) {
        const int2 e = t == 0 ? e0 : (t == 1 ? e1 : p.ent[pb + t]);
        int64_t v, sp;
        get(e.x, v, sp);
        consider(e, v, sp, t);
      }
    }
    const int64_t vi = have ? bval + 1 : NEG64;
    const int64_t si = have ? bsup + bw : 0;
    if (lane == k) {
      p.my_v = vi;
      p.my_s = si;
      p.my_set = have;
    }
    p.rv[i & (GRING - 1)] = vi;
    p.rsu[i & (GRING - 1)] = si;
    p.last = i;
    p.last_v = vi;
    p.last_s = si;
  };
  Pass F{true, s.head, s.support, ring_v, ring_s, s.pred_start, s.pred_cnt, s.pred};
  Pass B{false, s.tail, s.support_b, ring_b, ring_b + GRING, s.succ_start, s.succ_cnt, s.succ};
  const uint64_t tg1 = phase_clock();
  // forward from the source (head 0), backward from the sink (tail 1)
  s.head[0] = 0;
  ring_v[0] = 0;
  ring_s[0] = 0;
  s.tail[n - 1] = 1;
  s.support_b[n - 1] = 0;
  ring_b[(n - 1) & (GRING - 1)] = 1;
  ring_b[GRING + ((n - 1) & (GRING - 1))] = 0;
  begin(F);
  begin(B);
  for (int q0 = 0; q0 < count; q0 += 32) {
    block(F, q0);
    block(B, q0);
    const int lim = min(32, count - q0);
    for (int k = 0; k < lim; ++k) {
      step(F, q0, k, lim);
      step(B, q0, k, lim);
    }
    block_end(F, q0);
    block_end(B, q0);
    __syncwarp();  // later blocks read these rows back from memory
  }
  __syncwarp();
  (void)w;
  (void)tg0;
  (void)tg1;
  return s.head[n - 1] == NEG64 ? ST_NO_PATH : ST_OK;
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

// Per predecessor entry of every row, the descriptor a traceback step needs
// to move to that predecessor (warp-wide, after the DP): tb[2e] = (row, band
// start, band length, edge weight), tb[2e + 1] = (arena offset low 32 bits,
// arena offset bits 32-47 | base code << 16 | preferred << 24, the row's
// predecessor list start, its count). `preferred` is the reference's
// preferred-match weight test of the entry's edge, weight >= (sum of the row's
// incoming weights) / 10 (align.rs:1227-1228). An entry whose predecessor is
// out of range or skipped has row -1.
__device__ inline int fill_tb(Scratch &s, int n) {
  const int lane = threadIdx.x & 31;
  int wmax = 0;
  for (int i = lane; i < n; i += 32) {
    const int pb = s.pred_start[i], pc = s.pred_cnt[i];
    const int64_t ws10 = s.wsum[i] / 10;
    for (int t = 0; t < pc; ++t) {
      const int2 pr = s.pred[pb + t];
      wmax = max(wmax, pr.y);
      int4 a = make_int4(-1, 0, 0, pr.y), b = make_int4(0, 0, 0, 0);
      if (pr.x >= 0) {
        const int p = pr.x;
        const uint64_t off = uint64_t(s.row_off[p]);
        a = make_int4(p, s.row_start[p], s.row_len[p], pr.y);
        b = make_int4(int(off & 0xffffffffu),
                      int(((off >> 32) & 0xffffu) | (uint32_t(s.row_base[p]) << 16) | (int64_t(pr.y) >= ws10 ? 1u << 24 : 0u)),
                      s.pred_start[p], s.pred_cnt[p]);
      }
      s.tb[2 * (pb + t)] = a;
      s.tb[2 * (pb + t) + 1] = b;
    }
  }
  __syncwarp();
  return int(__reduce_max_sync(FULL, unsigned(wmax)));
}

// Traceback of align.rs:1164-1347 by the whole warp, reading the stored DP
// states. Each step is the reference's decision sequence (preferred match,
// deletion open / extend, insertion open / extend, match); lane t examines
// predecessor t of the current row in parallel, and the reference's choose()
// -- the first predecessor of largest weight among those whose state explains
// the cell -- becomes a ballot plus a max-reduction over the lanes.
//
// A step costs one memory round trip: lane t holds predecessor t's
// descriptor (fill_tb) in registers, so the states of the current cell and of
// every predecessor cell are loaded at once, together with the descriptors of
// the first two predecessors of each predecessor -- the next row's entries
// whichever predecessor the step moves to; they reach their lanes by shuffle.
// Steps are recorded as (row, column, kind) and resolved into AlignedBase
// items (push_diagonal, align.rs:1316-1347) by a parallel pass at the end,
// which also reverses them and prepends the source.
template <typename S>
__device__ int32_t traceback(Job *J, const DevParams &P, Scratch &s, const S *A, int beg, int n, int64_t m,
                             const int32_t *mat, const uint8_t *q8, int *n_out, Work *w = nullptr) {
  constexpr S NEGV = ScoreTraits<S>::NEGV;
  const int lane = threadIdx.x & 31;
  const int64_t neg_half = int64_t(NEGV) / 2;
  const int64_t O = P.gap_open, E = P.gap_ext;
  constexpr int KIND_INS = 0, KIND_DIAG = 1;
  const int4 none = make_int4(-1, 0, 0, 0), zero = make_int4(0, 0, 0, 0);
  const bool small_w = fill_tb(s, n) < (1 << 26);
  int i = n - 1;
  int j = int(m - 1);
  int op = OP_ALL;
  int nres = 0;
  int64_t steps = 0;
  int4 *res = s.items;
  // the current row and this lane's predecessor entry of it (lanes < pc)
  int rs = s.row_start[i], rl = s.row_len[i], pb = s.pred_start[i], pc = s.pred_cnt[i], rb = s.row_base[i];
  int64_t ro = s.row_off[i];
  int4 ea = none, eb = zero;
  if (lane < pc) {
    ea = s.tb[2 * (pb + lane)];
    eb = s.tb[2 * (pb + lane) + 1];
  }
  auto at = [&](int64_t off, int start, int len, int plane, int c) -> int64_t {
    return (c >= start && c - start < len) ? int64_t(A[off + int64_t(plane) * len + (c - start)]) : int64_t(NEGV);
  };
  auto eoff = [](const int4 &b) { return int64_t(uint64_t(uint32_t(b.x)) | (uint64_t(uint32_t(b.y) & 0xffffu) << 32)); };
  int32_t st = ST_OK;
  while (i > 0 || j > 0) {
    const uint64_t ts0 = phase_clock();
    steps += 1;
    if (steps > int64_t(n) + m) {
      st = ST_TB_NO_ADVANCE;
      break;
    }
    if (!(j >= rs && j - rs < rl)) {
      st = ST_TB_LEFT_BAND;
      break;
    }
    // one round of loads: the current cell (and its left neighbour), every
    // predecessor cell, and the predecessors' first two entries; each lane
    // also loads the descriptor of row i - 1 - lane for the L2 prefetch below
    const int pf_r = i - 1 - lane;
    int64_t pf_o = 0;
    int pf_s = 0, pf_l = 0;
    if (pf_r >= 0) {
      pf_o = s.row_off[pf_r];
      pf_s = s.row_start[pf_r];
      pf_l = s.row_len[pf_r];
    }
    const int64_t Mij = at(ro, rs, rl, 0, j), Dij = at(ro, rs, rl, 1, j), Iij = at(ro, rs, rl, 2, j);
    const int64_t Mim = at(ro, rs, rl, 0, j - 1), Iim = at(ro, rs, rl, 2, j - 1);
    int64_t Mpm = NEGV, Mpj = NEGV, Dpj = NEGV;
    int4 n0a = none, n0b = zero, n1a = none, n1b = zero;
    const bool mine = lane < pc && ea.x >= 0;
    if (mine) {
      const int64_t po = eoff(eb);
      Mpm = at(po, ea.y, ea.z, 0, j - 1);
      Mpj = at(po, ea.y, ea.z, 0, j);
      Dpj = at(po, ea.y, ea.z, 1, j);
      if (eb.w > 0) {
        n0a = s.tb[2 * eb.z];
        n0b = s.tb[2 * eb.z + 1];
      }
      if (eb.w > 1) {
        n1a = s.tb[2 * (eb.z + 1)];
        n1b = s.tb[2 * (eb.z + 1) + 1];
      }
    }
    if (Mij <= neg_half) {
      st = ST_TB_LEFT_BAND;
      break;
    }
    // The path reaches the rows just below this one within the next steps,
    // near this column; their states were written a whole read ago and have
    // usually left L2, so each lane brings one row's M, D and I around the
    // column it will likely be reached at back into L2 (descriptors loaded
    // with this step's states, so issuing costs no wait).
    if (pf_r >= 0) {
      const int c0 = max(j - 8 - lane, pf_s), c1 = min(j + 1, pf_s + pf_l - 1);
      if (c0 <= c1) {
        const S *base = A + pf_o;
#pragma unroll
        for (int plane = 0; plane < 3; ++plane) {
          asm volatile("prefetch.global.L2 [%0];" ::"l"(base + int64_t(plane) * pf_l + (c0 - pf_s)));
          asm volatile("prefetch.global.L2 [%0];" ::"l"(base + int64_t(plane) * pf_l + (c1 - pf_s)));
        }
      }
    }
    const uint64_t ts1 = phase_clock();
    const int qb = q8[j];
    const int64_t score = mat[rb * P.sigma + qb];
    // per-predecessor flags; best lane and weight per kind (chunk 0 from the
    // registers, further chunks of 32 from memory)
    int m_lane = -1, m_w = 0, o_lane = -1, o_w = 0, x_lane = -1, x_w = 0;
    int m_chunk = 0, o_chunk = 0, x_chunk = 0;
    // one reduction per kind: the key holds a valid bit, the weight and
    // 31 - lane, so the largest key is the largest weight and, among equal
    // weights, the first predecessor (weights below 2^26, checked once per
    // traceback; otherwise a ballot, a maximum and a second ballot)
    auto best = [&](bool f, int w, int t0, int &bl, int &bw, int &bc) {
      int l, mx;
      if (small_w) {
        const unsigned key = f ? (0x80000000u | (unsigned(w) << 5) | unsigned(31 - lane)) : 0u;
        const unsigned k = __reduce_max_sync(FULL, key);
        if (!k) return;
        l = 31 - int(k & 31u);
        mx = int((k >> 5) & 0x3ffffffu);
      } else {
        const unsigned msk = __ballot_sync(FULL, f);
        if (!msk) return;
        mx = int(__reduce_max_sync(FULL, f ? unsigned(w) : 0u));
        l = __ffs(__ballot_sync(FULL, f && w == mx)) - 1;
      }
      if (bl < 0 || mx > bw) {
        bl = l;
        bw = mx;
        bc = t0;
      }
    };
    auto flags = [&](const int4 &a, int64_t pm, int64_t pj, int64_t dj, bool &fm, bool &fo, bool &fx) {
      const bool c1 = j - 1 >= a.y && j - 1 - a.y < a.z, c0 = j >= a.y && j - a.y < a.z;
      fm = j > 0 && c1 && Mij == pm + score;
      fo = c0 && Dij == pj + O;
      fx = c0 && Dij == dj + E;
    };
    {
      bool fm = false, fo = false, fx = false;
      if (mine) flags(ea, Mpm, Mpj, Dpj, fm, fo, fx);
      best(fm, ea.w, 0, m_lane, m_w, m_chunk);
      best(fo, ea.w, 0, o_lane, o_w, o_chunk);
      best(fx, ea.w, 0, x_lane, x_w, x_chunk);
    }
    for (int t0 = 32; t0 < pc; t0 += 32) {  // rows with more than 32 predecessors
      const int t = t0 + lane;
      int4 qa = none, qbd = zero;
      if (t < pc) {
        qa = s.tb[2 * (pb + t)];
        qbd = s.tb[2 * (pb + t) + 1];
      }
      bool fm = false, fo = false, fx = false;
      if (qa.x >= 0) {
        const int64_t po = eoff(qbd);
        flags(qa, at(po, qa.y, qa.z, 0, j - 1), at(po, qa.y, qa.z, 0, j), at(po, qa.y, qa.z, 1, j), fm, fo, fx);
      }
      best(fm, qa.w, t0, m_lane, m_w, m_chunk);
      best(fo, qa.w, t0, o_lane, o_w, o_chunk);
      best(fx, qa.w, t0, x_lane, x_w, x_chunk);
    }
#ifdef POA_PHASE_CYCLES
    // profiling builds: cycles waiting for the step's loads, cycles choosing
    // (in the row-path counters, unused by these builds) and steps
    if (w) {
      w->rows_g4 += ts1 - ts0;
      w->rows_generic += phase_clock() - ts1;
      w->far_preds += 1;
    }
#else
    (void)ts0;
    (void)ts1;
    (void)w;
#endif
    // moves to predecessor (lane l of chunk c): its descriptor becomes the
    // current row, its first two entries come from lane l's prefetch
    auto move_to = [&](int l, int c) {
      int4 qa = ea, qbd = eb;
      if (c != 0) {
        const int t = c + lane;
        qa = none;
        qbd = zero;
        if (t < pc) {
          qa = s.tb[2 * (pb + t)];
          qbd = s.tb[2 * (pb + t) + 1];
        }
      }
      i = __shfl_sync(FULL, qa.x, l);
      rs = __shfl_sync(FULL, qa.y, l);
      rl = __shfl_sync(FULL, qa.z, l);
      const int bx = __shfl_sync(FULL, qbd.x, l), by = __shfl_sync(FULL, qbd.y, l);
      pb = __shfl_sync(FULL, qbd.z, l);
      pc = __shfl_sync(FULL, qbd.w, l);
      ro = int64_t(uint64_t(uint32_t(bx)) | (uint64_t(uint32_t(by) & 0xffffu) << 32));
      rb = int((uint32_t(by) >> 16) & 0xffu);
      int4 na = none, nb = zero;
      if (c == 0) {
        const int4 a0 = make_int4(__shfl_sync(FULL, n0a.x, l), __shfl_sync(FULL, n0a.y, l),
                                  __shfl_sync(FULL, n0a.z, l), __shfl_sync(FULL, n0a.w, l));
        const int4 b0 = make_int4(__shfl_sync(FULL, n0b.x, l), __shfl_sync(FULL, n0b.y, l),
                                  __shfl_sync(FULL, n0b.z, l), __shfl_sync(FULL, n0b.w, l));
        if (lane == 0) {
          na = a0;
          nb = b0;
        }
        if (pc > 1) {
          const int4 a1 = make_int4(__shfl_sync(FULL, n1a.x, l), __shfl_sync(FULL, n1a.y, l),
                                    __shfl_sync(FULL, n1a.z, l), __shfl_sync(FULL, n1a.w, l));
          const int4 b1 = make_int4(__shfl_sync(FULL, n1b.x, l), __shfl_sync(FULL, n1b.y, l),
                                    __shfl_sync(FULL, n1b.z, l), __shfl_sync(FULL, n1b.w, l));
          if (lane == 1) {
            na = a1;
            nb = b1;
          }
        }
        if (lane >= 2 && lane < pc) {
          na = s.tb[2 * (pb + lane)];
          nb = s.tb[2 * (pb + lane) + 1];
        }
      } else if (lane < pc) {
        na = s.tb[2 * (pb + lane)];
        nb = s.tb[2 * (pb + lane) + 1];
      }
      ea = na;
      eb = nb;
    };
    const bool pref_ok = m_lane >= 0 &&
                         ((uint32_t(__shfl_sync(FULL, m_chunk == 0 ? eb.y : 0, m_lane)) >> 24) & 1u) != 0;
    bool pref = false;
    if ((op & OP_MATCH) && j > 0 && rb == qb && m_lane >= 0) {
      if (m_chunk == 0) {
        pref = pref_ok;
      } else {
        const int t = m_chunk + m_lane;
        pref = ((uint32_t(s.tb[2 * (pb + t) + 1].y) >> 24) & 1u) != 0;
      }
    }
    if (pref) {
      if (lane == 0) res[nres] = make_int4(i, j, KIND_DIAG, 0);
      ++nres;
      move_to(m_lane, m_chunk);
      j -= 1;
      op = OP_ALL;
      continue;
    }
    if ((op & OP_DELETE) && (op == OP_DELETE || Mij == Dij)) {
      if (o_lane >= 0) {
        move_to(o_lane, o_chunk);
        op = P.gap_open_raw == 0 ? OP_ALL : (OP_MATCH | OP_INSERT);
        continue;
      }
      if (x_lane >= 0) {
        move_to(x_lane, x_chunk);
        op = OP_DELETE;
        continue;
      }
    }
    if ((op & OP_INSERT) && j > 0 && j - 1 >= rs && (op == OP_INSERT || Mij == Iij)) {
      if (Iij == Mim + O) {
        if (lane == 0) res[nres] = make_int4(i, j, KIND_INS, 0);
        ++nres;
        j -= 1;
        op = P.gap_open_raw == 0 ? OP_ALL : (OP_MATCH | OP_DELETE);
        continue;
      }
      if (Iij == Iim + E) {
        if (lane == 0) res[nres] = make_int4(i, j, KIND_INS, 0);
        ++nres;
        j -= 1;
        op = OP_INSERT;
        continue;
      }
    }
    if ((op & OP_MATCH) && j > 0 && m_lane >= 0) {
      if (lane == 0) res[nres] = make_int4(i, j, KIND_DIAG, 0);
      ++nres;
      move_to(m_lane, m_chunk);
      j -= 1;
      op = OP_ALL;
      continue;
    }
    if (lane == 0) {
      J->err_i = i;
      J->err_j = j;
    }
    st = ST_TB_NO_PRED;
    break;
  }
  __syncwarp();
  if (st != ST_OK) return st;
  // resolve, reverse, drop the sink entry (pushed first) and prepend the
  // source: final[k] = resolve(pushed[nres - k]) for k = 1..nres-1
  auto resolve = [&](int4 r) -> int4 {
    const int qb = q8[r.y];
    if (r.z == KIND_INS || (r.x == n - 1 && r.y != m - 1)) return make_int4(-1, qb, -1, 0);
    const int node = J->rank_to_node[beg + r.x];
    const int nb = J->base[node];
    const int base = r.x == n - 1 ? P.unknown : nb;
    if (base == qb) return make_int4(node, nb, -1, 0);
    const int parent = J->parent[node];
    return make_int4(J->aligned[int64_t(parent) * P.sigma + qb], qb, parent, 0);
  };
  for (int q = 1 + lane; 2 * q <= nres; q += 32) {
    const int k = nres - q;
    const int4 a = res[q], b = res[k];
    res[k] = resolve(a);
    if (k != q) res[q] = resolve(b);
  }
  __syncwarp();
  if (nres > 0 && lane == 0) {
    const int src = J->rank_to_node[beg];
    res[0] = make_int4(src, J->base[src], -1, 0);
  }
  __syncwarp();
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

// Per-warp shared memory. The M and D states of the most recent rows live in
// a ring of RING_CAP entries per state: rows are packed back to back in row
// order, row r starting at entry (cumulative band length of rows < r) mod
// RING_CAP, so a predecessor's states are read from shared memory instead of
// L2/HBM while fewer than RING_CAP entries were written after it (about five
// rows of the widest bands kept here, ten of 256 columns). Also the scoring
// matrix, the guide-pass rings and the encoded query (one byte per column).
constexpr int RING_CAP = 2560;
constexpr int RING_MAX_LEN = 512;   // widest band computed by one striped tile (4 stripes)
constexpr int RING_WIDE_LEN = 2048; // widest band computed by striped tiles in segments
static_assert(RING_WIDE_LEN <= RING_CAP, "a ring row must fit the ring");
constexpr int SMEM_MATRIX = 512;   // sigma^2 entries kept in shared memory (sigma <= 22)
constexpr int SEQ_SMEM = 5632;     // padded query columns kept in shared memory
// Where a warp's ring lives: its own ring_m / ring_d by default; a warp
// running alone in its block may take the other warps' shared memory.
struct RingView {
  int32_t *m, *d;
  int cap;     // entries per state, a multiple of 8
  int pad[3];  // pad[0]: this warp leads cooperative rows (see CoopDesc)
};
struct WarpSmem {
  RingView rv;
  int32_t ring_m[RING_CAP];
  int32_t ring_d[RING_CAP];
  int32_t matrix[SMEM_MATRIX];
  int64_t gring_v[GRING];  // guide passes: head (forward) or tail (backward)
  int64_t gring_s[GRING];  // guide passes: support
  uint8_t seq8[SEQ_SMEM];
};

// Every kernel sets its warp's ring to the warp's own arrays first.
__device__ inline void ring_default(WarpSmem *sm) {
  if ((threadIdx.x & 31) == 0) {
    sm->rv.m = sm->ring_m;
    sm->rv.d = sm->ring_d;
    sm->rv.cap = RING_CAP;
    sm->rv.pad[0] = 0;  // no cooperative rows
    sm->rv.pad[1] = 0;
    sm->rv.pad[2] = 0;
  }
  __syncwarp();
}

// Ring entry of column j of a row whose band starts at `start` and whose
// first column sits at ring entry `pos`, in a ring of `cap` entries.
__device__ __forceinline__ int ring_at(int pos, int start, int j, int cap) {
  const int x = pos + (j - start);
  return x >= cap ? x - cap : x;
}

// One int32 DP row of at most 128*G columns (align.rs:751-828) in stripes:
// stripe g covers columns [start + 128g, start + 128g + 128) and lane l owns
// the 4 consecutive columns at 4l of each stripe, so every shared-memory and
// global access of a stripe is one contiguous 512-byte vector access. Bands
// start and end on multiples of 8, so a lane's 4 columns lie wholly inside or
// wholly outside any band. Predecessors (band, ring entry or arena row, held
// by the lanes of `vmask`) are folded into M and D; each lane scans its 4
// columns, a warp max-plus scan (shift 4E per lane) carries the insertion
// state across the lanes of a stripe, and the stripes chain their carries.
// All identities are exact in integers: I[j+1] = max(I[j] + E, md[j] + O)
// with I[start] = NEG32. The stripe loops are branch-free (loads go to a
// clamped, in-bounds column and the value is then selected) so the compiler
// can overlap the stripes' dependency chains.
// SEG: the tile is one segment of a row wider than 4 stripes, at column
// offset c0 of the row: its insertion state enters from `carry_io` (the
// state leaving the previous segment's last column) and leaves there, and
// the ring entries are written by the caller once every segment has read its
// predecessors.
template <int G, bool ADAPT, bool SEG = false>
__device__ __forceinline__ void dp_row_striped(int lane, int start, int len, int32_t *R, const uint8_t *seq8,
                                               const int32_t *mrow, int32_t E, int32_t O, unsigned vmask,
                                               int my_ps, int my_pl, int my_pos, const int32_t *my_g,
                                               int32_t *rm, int32_t *rd, int cap, int pos_i, int32_t &bestv,
                                               int &bestj, int c0 = 0, int32_t *carry_io = nullptr) {
  const int stop = start + len;
  const int cs = SEG ? start + c0 : start;  // first column of the tile
  int32_t Mx[G][4], Dx[G][4];
#pragma unroll
  for (int g = 0; g < G; ++g)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      Mx[g][k] = NEG32;
      Dx[g][k] = NEG32;
    }
  while (vmask) {
    const int t = __ffs(vmask) - 1;
    vmask &= vmask - 1;
    const int ps = __shfl_sync(FULL, my_ps, t);
    const int pl = __shfl_sync(FULL, my_pl, t);
    const int pos = __shfl_sync(FULL, my_pos, t);
    int4 m4[G], d4[G];
    int32_t prev[G];
    bool in[G];
    if (pos >= 0) {
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const int j0 = cs + 128 * g + 4 * lane;
        in[g] = j0 < stop && j0 >= ps && j0 < ps + pl;
        const int x = ring_at(pos, ps, in[g] ? j0 : ps, cap);
        m4[g] = *reinterpret_cast<const int4 *>(rm + x);
        d4[g] = *reinterpret_cast<const int4 *>(rd + x);
        prev[g] = rm[x == 0 ? cap - 1 : x - 1];
      }
    } else {
      // the predecessor row has left the ring: its arena row
      const int32_t *gp = reinterpret_cast<const int32_t *>(__shfl_sync(FULL, (long long)my_g, t));
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const int j0 = cs + 128 * g + 4 * lane;
        in[g] = j0 < stop && j0 >= ps && j0 < ps + pl;
        const int c = in[g] ? j0 - ps : 0;
        m4[g] = *reinterpret_cast<const int4 *>(gp + c);
        d4[g] = *reinterpret_cast<const int4 *>(gp + pl + c);
        prev[g] = gp[c > 0 ? c - 1 : 0];
      }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int j0 = cs + 128 * g + 4 * lane;
      const int32_t pv = j0 > ps ? prev[g] : NEG32;
      if (in[g]) {
        Mx[g][0] = maxs(Mx[g][0], pv);
        Mx[g][1] = maxs(Mx[g][1], m4[g].x);
        Mx[g][2] = maxs(Mx[g][2], m4[g].y);
        Mx[g][3] = maxs(Mx[g][3], m4[g].z);
        Dx[g][0] = __viaddmax_s32(d4[g].x, E, __viaddmax_s32(m4[g].x, O, Dx[g][0]));
        Dx[g][1] = __viaddmax_s32(d4[g].y, E, __viaddmax_s32(m4[g].y, O, Dx[g][1]));
        Dx[g][2] = __viaddmax_s32(d4[g].z, E, __viaddmax_s32(m4[g].z, O, Dx[g][2]));
        Dx[g][3] = __viaddmax_s32(d4[g].w, E, __viaddmax_s32(m4[g].w, O, Dx[g][3]));
      }
    }
  }
  // md, the in-lane scan x[k] = max over k' <= k of md[k'] + O + (k-k')E, and
  // per stripe the warp scan of the lane aggregates: pre[g] = the insertion
  // state entering the lane's first column from the lanes before it (without
  // the stripe's own carry; a value below every reachable state for lane 0).
  // Columns past the band read the band's last word and are never stored.
  constexpr int32_t BELOW = INT32_MIN / 2;
  int32_t X[G][4], pre[G];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const int j0 = cs + 128 * g + 4 * lane;
    const uint32_t bw = *reinterpret_cast<const uint32_t *>(seq8 + min(j0, stop - 4));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int32_t prof = mrow[(bw >> (8 * k)) & 0xff];
      Mx[g][k] = __viaddmax_s32(Mx[g][k], prof, Dx[g][k]);  // Mx now holds md
      X[g][k] = k == 0 ? Mx[g][k] + O : __viaddmax_s32(X[g][k - 1], E, Mx[g][k] + O);
    }
  }
  // (lanes below the shuffle distance get their own value back, and
  // y + d*4E <= y because gap penalties are never positive)
  int32_t T[G];  // the stripe's own insertion state leaving its last column
#pragma unroll
  for (int g = 0; g < G; ++g) {
    int32_t y = X[g][3];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) y = __viaddmax_s32(__shfl_up_sync(FULL, y, d), d * 4 * E, y);
    pre[g] = __shfl_up_sync(FULL, y, 1);
    if (lane == 0) pre[g] = BELOW;
    T[g] = __shfl_sync(FULL, y, 31);
  }
  // chain the stripes: carry = I at the stripe's first column (NEG32 at the
  // band start), carry[g+1] = max(carry[g] + 128E, T[g]); each lane's
  // carried-in state is max(pre, carry shifted). The T are independent, so
  // the chain is arithmetic only.
  int32_t cin[G];
  int32_t carry = SEG ? *carry_io : NEG32;
#pragma unroll
  for (int g = 0; g < G; ++g) {
    cin[g] = __viaddmax_s32(carry, 4 * lane * E, pre[g]);
    if (SEG || g + 1 < G) carry = __viaddmax_s32(carry, 128 * E, T[g]);
  }
  if (SEG) *carry_io = carry;
  __syncwarp();  // every predecessor read of the ring precedes this row's writes
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const int j0 = cs + 128 * g + 4 * lane;
    int32_t iv[4], mv[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      iv[k] = k == 0 ? cin[g] : __viaddmax_s32(cin[g], k * E, X[g][k - 1]);
      mv[k] = maxs(Mx[g][k], iv[k]);
    }
    if (j0 < stop) {
      if (ADAPT) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (mv[k] > bestv) {
            bestv = mv[k];
            bestj = j0 + k;
          }
      }
      const int o = j0 - start;
      if (!SEG) {
        const int x = ring_at(pos_i, start, j0, cap);
        *reinterpret_cast<int4 *>(rm + x) = make_int4(mv[0], mv[1], mv[2], mv[3]);
        *reinterpret_cast<int4 *>(rd + x) = make_int4(Dx[g][0], Dx[g][1], Dx[g][2], Dx[g][3]);
      }
      *reinterpret_cast<int4 *>(R + o) = make_int4(mv[0], mv[1], mv[2], mv[3]);
      *reinterpret_cast<int4 *>(R + len + o) = make_int4(Dx[g][0], Dx[g][1], Dx[g][2], Dx[g][3]);
      *reinterpret_cast<int4 *>(R + 2 * len + o) = make_int4(iv[0], iv[1], iv[2], iv[3]);
    }
  }
}

// A band wider than one tile (up to RING_WIDE_LEN): 512-column segments
// chained by their insertion carry, then the row into the ring (each lane
// copies the columns it wrote).
template <bool ADAPT>
__device__ __forceinline__ void dp_row_wide(int lane, int start, int len, int32_t *R, const uint8_t *seq8,
                                            const int32_t *mrow, int32_t E, int32_t O, unsigned vmask, int ps,
                                            int pl, int pos, const int32_t *g, int32_t *rm, int32_t *rd, int cap,
                                            int pos_i, int32_t &bv, int &bj) {
  int32_t carry = NEG32;
  int c0 = 0;
  for (; c0 + RING_MAX_LEN < len; c0 += RING_MAX_LEN)
    dp_row_striped<4, ADAPT, true>(lane, start, len, R, seq8, mrow, E, O, vmask, ps, pl, pos, g, rm, rd, cap, pos_i,
                                   bv, bj, c0, &carry);
  if (len - c0 <= 256)  // the last segment: two stripes when they cover it
    dp_row_striped<2, ADAPT, true>(lane, start, len, R, seq8, mrow, E, O, vmask, ps, pl, pos, g, rm, rd, cap, pos_i,
                                   bv, bj, c0, &carry);
  else
    dp_row_striped<4, ADAPT, true>(lane, start, len, R, seq8, mrow, E, O, vmask, ps, pl, pos, g, rm, rd, cap, pos_i,
                                   bv, bj, c0, &carry);
  __syncwarp();
  for (int o = 4 * lane; o < len; o += 128) {
    const int x = ring_at(pos_i, start, start + o, cap);
    *reinterpret_cast<int4 *>(rm + x) = *reinterpret_cast<const int4 *>(R + o);
    *reinterpret_cast<int4 *>(rd + x) = *reinterpret_cast<const int4 *>(R + len + o);
  }
}

// Dispatches one int32 row to the striped tile of the right width.
template <bool ADAPT, bool WIDE = false>
__device__ __forceinline__ void dp_row_fast(int lane, int start, int len, int32_t *R, const uint8_t *seq8,
                                            const int32_t *mrow, int32_t E, int32_t O, unsigned vmask, int ps,
                                            int pl, int pos, const int32_t *g, int32_t *rm, int32_t *rd, int cap,
                                            int pos_i, int32_t &bv, int &bj) {
  if (len <= 128)
    dp_row_striped<1, ADAPT>(lane, start, len, R, seq8, mrow, E, O, vmask, ps, pl, pos, g, rm, rd, cap, pos_i, bv, bj);
  else if (len <= 256)
    dp_row_striped<2, ADAPT>(lane, start, len, R, seq8, mrow, E, O, vmask, ps, pl, pos, g, rm, rd, cap, pos_i, bv, bj);
  else if (len <= 384)
    dp_row_striped<3, ADAPT>(lane, start, len, R, seq8, mrow, E, O, vmask, ps, pl, pos, g, rm, rd, cap, pos_i, bv, bj);
  else if (!WIDE || len <= RING_MAX_LEN)
    dp_row_striped<4, ADAPT>(lane, start, len, R, seq8, mrow, E, O, vmask, ps, pl, pos, g, rm, rd, cap, pos_i, bv, bj);
  else if constexpr (WIDE)
    dp_row_wide<ADAPT>(lane, start, len, R, seq8, mrow, E, O, vmask, ps, pl, pos, g, rm, rd, cap, pos_i, bv, bj);
}

// ---------------------------------------------------------------------------
// Cooperative rows. A warp running a giant job alone in its block (the other
// warps of the block would otherwise idle) has three of them compute its DP
// rows with it: stripe 0 of every row by the leader, stripes 1-3 by the
// helpers. The leader publishes
// each row in shared memory; the four warps meet at named barrier 1 three
// times per row (row published, stripe aggregates published, row written)
// and at barrier 2 at the start of every row loop and once when the job is
// done. The arithmetic is the single-warp striped row's: the stripe carries
// compose as carry[g+1] = max(aggregate[g], carry[g] + 128E).
constexpr int COOP_ROWS = 0, COOP_DONE = 1;  // phase modes
constexpr int COOP_GEN_MIN_LEN = 256;         // narrower int64 rows: the leader alone
constexpr int COOP_ROW = 0, COOP_STOP = 1, COOP_GEN = 2, COOP_SEG = 3;  // row operations
struct CoopDesc {
  int mode, op, start, len, pos_i, n_pred, cap, pad0;
  int32_t E, O, pad1, pad2;
  int32_t *R;
  const int32_t *mrow;
  const uint8_t *q8;
  int32_t *rm, *rd;
  int32_t agg[16];  // per 512-column segment (COOP_SEG: up to 4), per stripe
  int ps[32], pl[32], pos[32];
  const int32_t *g[32];
  // int64 rows (COOP_GEN): per read, the gaps, the arena and the plan arrays;
  // per row, its arena row and predecessor list; per warp, its segment's
  // insertion state leaving the segment
  int64_t E64, O64;
  const int64_t *gA;
  const int32_t *grs, *grl, *gseq;
  const int64_t *gro;
  int64_t *gR;
  const int2 *gpred;
  int64_t agg64[4];
};
static_assert(sizeof(CoopDesc) <= sizeof(int32_t) * RING_CAP, "CoopDesc must fit a ring array");
__device__ inline void coop_gen64(CoopDesc *c, int g);
__device__ inline void coop_seg(CoopDesc *c, int g);

__device__ __forceinline__ void coop_bar(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// Stripe g of the published row (every warp of the block calls this once per
// row, after barrier 1 has made the row visible).
__device__ inline void coop_stripe(CoopDesc *c, int g) {
  const int lane = threadIdx.x & 31;
  const int start = c->start, len = c->len, stop = start + len, cap = c->cap;
  const int32_t E = c->E, O = c->O;
  int32_t *rm = c->rm, *rd = c->rd;
  const int j0 = start + 128 * g + 4 * lane;
  int32_t Mx[4], Dx[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    Mx[k] = NEG32;
    Dx[k] = NEG32;
  }
  const int np = c->n_pred;
  for (int t = 0; t < np; ++t) {
    const int ps = c->ps[t], pl = c->pl[t], pos = c->pos[t];
    const int32_t *gp = c->g[t];
    const bool in = j0 < stop && j0 >= ps && j0 < ps + pl;
    int4 m4, d4;
    int32_t prev;
    if (pos >= 0) {
      const int x = ring_at(pos, ps, in ? j0 : ps, cap);
      m4 = *reinterpret_cast<const int4 *>(rm + x);
      d4 = *reinterpret_cast<const int4 *>(rd + x);
      prev = rm[x == 0 ? cap - 1 : x - 1];
    } else {
      const int c0 = in ? j0 - ps : 0;
      m4 = *reinterpret_cast<const int4 *>(gp + c0);
      d4 = *reinterpret_cast<const int4 *>(gp + pl + c0);
      prev = gp[c0 > 0 ? c0 - 1 : 0];
    }
    const int32_t pv = j0 > ps ? prev : NEG32;
    if (in) {
      Mx[0] = maxs(Mx[0], pv);
      Mx[1] = maxs(Mx[1], m4.x);
      Mx[2] = maxs(Mx[2], m4.y);
      Mx[3] = maxs(Mx[3], m4.z);
      Dx[0] = __viaddmax_s32(d4.x, E, __viaddmax_s32(m4.x, O, Dx[0]));
      Dx[1] = __viaddmax_s32(d4.y, E, __viaddmax_s32(m4.y, O, Dx[1]));
      Dx[2] = __viaddmax_s32(d4.z, E, __viaddmax_s32(m4.z, O, Dx[2]));
      Dx[3] = __viaddmax_s32(d4.w, E, __viaddmax_s32(m4.w, O, Dx[3]));
    }
  }
  constexpr int32_t BELOW = INT32_MIN / 2;
  int32_t X[4];
  const uint32_t bw = *reinterpret_cast<const uint32_t *>(c->q8 + min(j0, stop - 4));
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int32_t prof = c->mrow[(bw >> (8 * k)) & 0xff];
    Mx[k] = __viaddmax_s32(Mx[k], prof, Dx[k]);  // Mx now holds md
    X[k] = k == 0 ? Mx[k] + O : __viaddmax_s32(X[k - 1], E, Mx[k] + O);
  }
  int32_t y = X[3];
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) y = __viaddmax_s32(__shfl_up_sync(FULL, y, d), d * 4 * E, y);
  int32_t pre = __shfl_up_sync(FULL, y, 1);
  if (lane == 0) pre = BELOW;
  const int32_t y31 = __shfl_sync(FULL, y, 31);
  if (lane == 0) c->agg[g] = y31;
  coop_bar(1);
  int32_t carry = NEG32;
  for (int h = 0; h < g; ++h) carry = __viaddmax_s32(carry, 128 * E, c->agg[h]);
  const int32_t cin = __viaddmax_s32(carry, 4 * lane * E, pre);
  if (j0 < stop) {
    int32_t iv[4], mv[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      iv[k] = k == 0 ? cin : __viaddmax_s32(cin, k * E, X[k - 1]);
      mv[k] = maxs(Mx[k], iv[k]);
    }
    const int o = j0 - start;
    const int x = ring_at(c->pos_i, start, j0, cap);
    int32_t *R = c->R;
    *reinterpret_cast<int4 *>(rm + x) = make_int4(mv[0], mv[1], mv[2], mv[3]);
    *reinterpret_cast<int4 *>(rd + x) = make_int4(Dx[0], Dx[1], Dx[2], Dx[3]);
    *reinterpret_cast<int4 *>(R + o) = make_int4(mv[0], mv[1], mv[2], mv[3]);
    *reinterpret_cast<int4 *>(R + len + o) = make_int4(Dx[0], Dx[1], Dx[2], Dx[3]);
    *reinterpret_cast<int4 *>(R + 2 * len + o) = make_int4(iv[0], iv[1], iv[2], iv[3]);
  }
  coop_bar(1);
}

// Cooperative rows of 513-2048 columns (the wide kernel forms): the row's
// 512-column segments left to right, warp g computing stripe g of each (the
// stripe arithmetic of coop_stripe). After a segment's stripes publish their
// aggregates (barrier 1), each warp composes the insertion state entering
// its stripe from the state entering the segment and the stripes before it,
// and all warps carry the segment's four stripes into the next segment's
// entry state. The row enters the ring only after every segment has read
// its predecessors (each lane copies the columns it wrote; barrier 1 again
// once the row is written), since a wide row's later segments may read
// predecessor entries its earlier columns would overwrite.
__device__ inline void coop_seg(CoopDesc *c, int g) {
  const int lane = threadIdx.x & 31;
  const int start = c->start, len = c->len, stop = start + len, cap = c->cap;
  const int32_t E = c->E, O = c->O;
  int32_t *rm = c->rm, *rd = c->rd;
  int32_t *R = c->R;
  const int np = c->n_pred;
  const int nseg = (len + 511) / 512;
  constexpr int32_t BELOW = INT32_MIN / 2;
  int32_t entry = NEG32;  // insertion state entering the segment's first column
  for (int sg = 0; sg < nseg; ++sg) {
    const int j0 = start + 512 * sg + 128 * g + 4 * lane;
    int32_t Mx[4], Dx[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      Mx[k] = NEG32;
      Dx[k] = NEG32;
    }
    for (int t = 0; t < np; ++t) {
      const int ps = c->ps[t], pl = c->pl[t], pos = c->pos[t];
      const int32_t *gp = c->g[t];
      const bool in = j0 < stop && j0 >= ps && j0 < ps + pl;
      int4 m4, d4;
      int32_t prev;
      if (pos >= 0) {
        const int x = ring_at(pos, ps, in ? j0 : ps, cap);
        m4 = *reinterpret_cast<const int4 *>(rm + x);
        d4 = *reinterpret_cast<const int4 *>(rd + x);
        prev = rm[x == 0 ? cap - 1 : x - 1];
      } else {
        const int c0 = in ? j0 - ps : 0;
        m4 = *reinterpret_cast<const int4 *>(gp + c0);
        d4 = *reinterpret_cast<const int4 *>(gp + pl + c0);
        prev = gp[c0 > 0 ? c0 - 1 : 0];
      }
      const int32_t pv = j0 > ps ? prev : NEG32;
      if (in) {
        Mx[0] = maxs(Mx[0], pv);
        Mx[1] = maxs(Mx[1], m4.x);
        Mx[2] = maxs(Mx[2], m4.y);
        Mx[3] = maxs(Mx[3], m4.z);
        Dx[0] = __viaddmax_s32(d4.x, E, __viaddmax_s32(m4.x, O, Dx[0]));
        Dx[1] = __viaddmax_s32(d4.y, E, __viaddmax_s32(m4.y, O, Dx[1]));
        Dx[2] = __viaddmax_s32(d4.z, E, __viaddmax_s32(m4.z, O, Dx[2]));
        Dx[3] = __viaddmax_s32(d4.w, E, __viaddmax_s32(m4.w, O, Dx[3]));
      }
    }
    int32_t X[4];
    const uint32_t bw = *reinterpret_cast<const uint32_t *>(c->q8 + min(j0, stop - 4));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int32_t prof = c->mrow[(bw >> (8 * k)) & 0xff];
      Mx[k] = __viaddmax_s32(Mx[k], prof, Dx[k]);  // Mx now holds md
      X[k] = k == 0 ? Mx[k] + O : __viaddmax_s32(X[k - 1], E, Mx[k] + O);
    }
    int32_t y = X[3];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) y = __viaddmax_s32(__shfl_up_sync(FULL, y, d), d * 4 * E, y);
    int32_t pre = __shfl_up_sync(FULL, y, 1);
    if (lane == 0) pre = BELOW;
    const int32_t y31 = __shfl_sync(FULL, y, 31);
    if (lane == 0) c->agg[4 * sg + g] = y31;
    coop_bar(1);
    int32_t carry = entry;
    for (int h = 0; h < g; ++h) carry = __viaddmax_s32(carry, 128 * E, c->agg[4 * sg + h]);
    const int32_t cin = __viaddmax_s32(carry, 4 * lane * E, pre);
    if (j0 < stop) {
      int32_t iv[4], mv[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        iv[k] = k == 0 ? cin : __viaddmax_s32(cin, k * E, X[k - 1]);
        mv[k] = maxs(Mx[k], iv[k]);
      }
      const int o = j0 - start;
      *reinterpret_cast<int4 *>(R + o) = make_int4(mv[0], mv[1], mv[2], mv[3]);
      *reinterpret_cast<int4 *>(R + len + o) = make_int4(Dx[0], Dx[1], Dx[2], Dx[3]);
      *reinterpret_cast<int4 *>(R + 2 * len + o) = make_int4(iv[0], iv[1], iv[2], iv[3]);
    }
    for (int h = 0; h < 4; ++h) entry = __viaddmax_s32(entry, 128 * E, c->agg[4 * sg + h]);
  }
  for (int sg = 0; sg < nseg; ++sg) {
    const int j0 = start + 512 * sg + 128 * g + 4 * lane;
    if (j0 < stop) {
      const int o = j0 - start;
      const int x = ring_at(c->pos_i, start, j0, cap);
      *reinterpret_cast<int4 *>(rm + x) = *reinterpret_cast<const int4 *>(R + o);
      *reinterpret_cast<int4 *>(rd + x) = *reinterpret_cast<const int4 *>(R + len + o);
    }
  }
  coop_bar(1);
}

// The block-mates' side: rows of every row loop the leader opens, until the
// leader's job is done.
__device__ inline void coop_helper(CoopDesc *c, int g) {
  for (;;) {
    coop_bar(2);
    if (c->mode == COOP_DONE) {
      coop_bar(2);  // every helper has read the mode before the leader reuses the descriptor
      return;
    }
    for (;;) {
      coop_bar(1);
      if (c->op == COOP_STOP) break;
      if (c->op == COOP_GEN)
        coop_gen64(c, g);
      else if (c->op == COOP_SEG)
        coop_seg(c, g);
      else
        coop_stripe(c, g);
    }
  }
}

// Leader side of the release: the helpers leave coop_helper, and the
// leader's ring is its own slice again (the descriptor's memory included).
__device__ inline void coop_release(WarpSmem *sm) {
  if ((threadIdx.x & 31) == 0) reinterpret_cast<CoopDesc *>(sm->ring_m)->mode = COOP_DONE;
  coop_bar(2);
  coop_bar(2);
  ring_default(sm);
}

// Ring entry of a predecessor row's first column (arena offset `po`) while
// row `off` is computed, or -1 when the row's states are no longer (or were
// never) in the ring: intact while the rows written after it hold at most
// RING_CAP entries. Arena offsets are 3x the cumulative band length.
__device__ __forceinline__ int ring_pos(int64_t po, int64_t off, int64_t ring_floor, int cap) {
  if (po < ring_floor || off - po > 3 * int64_t(cap)) return -1;
  return int((po / 3) % cap);
}

// Copies row 0 (arena offset 0, computed serially) into the ring; returns the
// ring floor (1 when the row is too wide to enter it).
template <typename S>
__device__ inline int64_t ring_put_row0(int32_t *rm, int32_t *rd, const S *A, int len, int row_max) {
  const int lane = threadIdx.x & 31;
  if (len > row_max) return 1;
  for (int c = lane; c < len; c += 32) {
    rm[c] = int32_t(A[c]);
    rd[c] = int32_t(A[len + c]);
  }
  __syncwarp();
  return 0;
}

// One row by the generic interleaved loop (int64 kernel, rows wider than
// the kernel's ring row limit, or more than 32 predecessors): 32-column
// chunks, predecessor rows from the arena, a warp-shuffle scan per chunk with
// a serial carry. Several chunks are taken per step (two for int32, four for
// int64, whose rows are the widest), so the predecessor loads and the scans
// of all of them are in flight together (only the carry links them). With at most 32
// predecessors, lane t holds predecessor t's band and arena row for the
// whole row and the chunks take them by shuffle.
template <typename S>
__device__ __forceinline__ void dp_row_generic(int lane, int start, int len, S *R, const S *A, const Scratch &s,
                                               int pb, int pc, const int32_t *mrow, S E, S O, bool adapt, S &bestv,
                                               int &bestj) {
  constexpr S NEGV = ScoreTraits<S>::NEGV;
  constexpr int NCH = sizeof(S) == 8 ? 4 : 2;  // chunks per step
  const int stop = start + len;
  const bool held = pc <= 32;
  int my_ps = 0, my_pl = 0;
  const S *my_q = A;
  if (held && lane < pc) {
    const int p = s.pred[pb + lane].x;
    if (p >= 0) {
      my_ps = s.row_start[p];
      my_pl = s.row_len[p];
      my_q = A + s.row_off[p];
    }
  }
  const unsigned vmask = __ballot_sync(FULL, my_pl > 0);
  S carry = NEGV;
  for (int c0 = start; c0 < stop; c0 += 32 * NCH) {
    S M[NCH], D[NCH];
#pragma unroll
    for (int h = 0; h < NCH; ++h) {
      M[h] = NEGV;
      D[h] = NEGV;
    }
    if (held) {
      unsigned vm = vmask;
      while (vm) {
        const int t = __ffs(vm) - 1;
        vm &= vm - 1;
        const int ps = __shfl_sync(FULL, my_ps, t), pl = __shfl_sync(FULL, my_pl, t);
        const S *Q = reinterpret_cast<const S *>(__shfl_sync(FULL, (long long)my_q, t));
#pragma unroll
        for (int h = 0; h < NCH; ++h) {
          const int j = c0 + 32 * h + lane;
          if (j < stop && j >= ps && j < ps + pl) {
            const int k = j - ps;
            const S mp = Q[k], dp = Q[pl + k];
            const S dg = k > 0 ? Q[k - 1] : NEGV;
            M[h] = maxs(M[h], dg);
            D[h] = maxs(D[h], maxs<S>(dp + E, mp + O));
          }
        }
      }
    } else {
      for (int t = 0; t < pc; ++t) {
        const int p = s.pred[pb + t].x;
        if (p < 0) continue;
        const int ps = s.row_start[p], pl = s.row_len[p];
        const S *Q = A + s.row_off[p];
#pragma unroll
        for (int h = 0; h < NCH; ++h) {
          const int j = c0 + 32 * h + lane;
          if (j < stop && j >= ps && j < ps + pl) {
            const int k = j - ps;
            const S mp = Q[k], dp = Q[pl + k];
            const S dg = k > 0 ? Q[k - 1] : NEGV;
            M[h] = maxs(M[h], dg);
            D[h] = maxs(D[h], maxs<S>(dp + E, mp + O));
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < NCH; ++h) {
      if (c0 + 32 * h >= stop) break;  // (warp-uniform)
      const int j = c0 + 32 * h + lane;
      const bool valid = j < stop;
      const S prof = valid ? S(mrow[s.seq[j]]) : S(0);
      const S md = maxs<S>(M[h] + prof, D[h]);
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
        R[len + c] = D[h];
        R[2 * len + c] = I;
        if (adapt && Mf > bestv) {
          bestv = Mf;
          bestj = j;
        }
      }
      carry = shfl_s(x, 31);
    }
  }
}

// Cooperative int64 rows: a giant job's generic rows (at most 32
// predecessors) computed by its warp and three helpers, warp g taking the g-th
// quarter of the band (32-column aligned). Pass 1: each warp computes M and D
// from the predecessors, md and its segment's insertion scan as if the
// segment began the row (from a value below every state), storing md, D and
// that scan; the segments' last scan values are published (barrier 1). Pass
// 2: each warp composes the insertion state entering its segment from the
// segments before it, carry = max(last[h], carry + E x width[h]) from the
// row's initial NEGV, and finishes its columns: x = max(scan, carry + E x
// distance), I = the x of the column before, M = max(md, I). Max-plus
// addition distributes exactly over max in integers, so every stored state
// equals the one-warp generic row's (barrier 1 again once the row is written).
__device__ inline void coop_gen64(CoopDesc *c, int g) {
  using S = int64_t;
  constexpr S NEGV = NEG64;
  constexpr S BELOW = -(S(1) << 61);
  const int lane = threadIdx.x & 31;
  const int start = c->start, len = c->len, stop = start + len;
  const S E = c->E64, O = c->O64;
  const int seg = (len + 127) / 128 * 32;
  const int a = start + g * seg, b = min(stop, a + seg);
  S *R = c->gR;
  const S *A = c->gA;
  const int32_t *mrow = c->mrow;
  const int32_t *seq = c->gseq;
  const int pc = c->n_pred;
  int my_ps = 0, my_pl = 0;
  const S *my_q = A;
  if (lane < pc) {
    const int p = c->gpred[lane].x;
    if (p >= 0) {
      my_ps = c->grs[p];
      my_pl = c->grl[p];
      my_q = A + c->gro[p];
    }
  }
  const unsigned vmask = __ballot_sync(FULL, my_pl > 0);
  S lc = BELOW;
  for (int c0 = a; c0 < b; c0 += 32) {
    const int j = c0 + lane;
    const bool valid = j < stop;
    S M = NEGV, D = NEGV;
    unsigned vm = vmask;
    while (vm) {
      const int t = __ffs(vm) - 1;
      vm &= vm - 1;
      const int ps = __shfl_sync(FULL, my_ps, t), pl = __shfl_sync(FULL, my_pl, t);
      const S *Q = reinterpret_cast<const S *>(__shfl_sync(FULL, (long long)my_q, t));
      if (valid && j >= ps && j < ps + pl) {
        const int k = j - ps;
        const S mp = Q[k], dp = Q[pl + k];
        const S dg = k > 0 ? Q[k - 1] : NEGV;
        M = maxs(M, dg);
        D = maxs(D, maxs<S>(dp + E, mp + O));
      }
    }
    const S prof = valid ? S(mrow[seq[j]]) : S(0);
    const S md = maxs<S>(M + prof, D);
    S x = md + O;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const S y = shfl_up_s(x, d);
      if (lane >= d) x = maxs<S>(x, y + S(d) * E);
    }
    x = maxs<S>(x, lc + S(lane + 1) * E);
    if (valid) {
      const int cc = j - start;
      R[cc] = md;
      R[len + cc] = D;
      R[2 * len + cc] = x;
    }
    lc = shfl_s(x, 31);
  }
  if (lane == 0) c->agg64[g] = lc;
  coop_bar(1);
  S cin = NEGV;
  for (int h = 0; h < g; ++h) {
    const int ah = start + h * seg, bh = min(stop, ah + seg);
    if (bh > ah) cin = maxs<S>(c->agg64[h], cin + S(bh - ah) * E);
  }
  S prev = cin;  // x of the column before the chunk
  for (int c0 = a; c0 < b; c0 += 32) {
    const int j = c0 + lane;
    const bool valid = j < stop;
    const int cc = j - start;
    S xt = BELOW, md = NEGV;
    if (valid) {
      xt = R[2 * len + cc];
      md = R[cc];
    }
    xt = maxs<S>(xt, cin + S(j - a + 1) * E);
    S I = shfl_up_s(xt, 1);
    if (lane == 0) I = prev;
    if (valid) {
      R[cc] = maxs(md, I);
      R[2 * len + cc] = I;
    }
    prev = shfl_s(xt, 31);
  }
  coop_bar(1);
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

// A 16-byte load issued where it is written: the DP loop loads the next rows'
// plan while the current row computes, and a volatile load keeps the
// compiler from sinking it to its use.
__device__ __forceinline__ int4 ld_early(const int4 *p) {
  int4 v;
  asm volatile("ld.global.v4.s32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  return v;
}

// ---------------------------------------------------------------------------
// Row wavefront (static band, int32; align.rs:751-828 for every row at once).
// With a static band every row's band is known before the DP starts, so the
// rows need not run one after another: row i may compute its columns
// [8c, 8c + 8) ("chunk c") as soon as each predecessor has computed its own
// chunk c (the diagonal also needs the predecessor's column 8c - 1, which
// belongs to its chunk c - 1). Each lane owns one row at a time (rows
// 1 + lane, 33 + lane, ...) and walks it chunk by chunk with the serial
// recurrences in registers; the warp steps in lockstep, so about 32 rows are
// in flight, each a chunk or more behind the row before it. There is no
// cross-lane scan: the insertion state I is carried along the row by the
// lane that owns it.
//
// A chunk's M and D, with the M just left of it, go to a shared-memory slot
// of the lane that computed it (WAVE_KB slots per lane, indexed by chunk mod
// WAVE_KB) tagged (row << 13 | chunk), and its M, D and I go to the row's
// arena row as usual. A reader compares the slot's tag with the chunk it
// needs: equal, the states are there; smaller, the predecessor has not
// computed the chunk yet and the reader waits for a later step; larger, the
// slot was reused after the chunk was written, so the chunk is read from the
// predecessor's arena row. Every step reads first and writes second, with a
// warp barrier between, so a reader never sees a slot half-written.
//
// The arithmetic is the reference's int32 arithmetic term for term: per
// predecessor over the overlap of the two 8-aligned bands, M[j] gets
// Mp[j - 1] (NEG32 at the predecessor's first column) and D[j] gets
// max(Dp[j] + E, Mp[j] + O); then md = max(M + profile, D), I[start] =
// NEG32, I[j + 1] = max(I[j] + E, md[j] + O), M = max(md, I).
constexpr int WAVE_KB = 8;              // chunk slots per lane
constexpr int WAVE_SLOT = 20;           // int32 per slot: M[8], D[8], M left of the chunk, tag, 2 spare
constexpr int WAVE_TAG = 17;
constexpr int WAVE_MAX_ROWS = 1 << 18;  // tags hold the row in 18 bits ...
constexpr int WAVE_MAX_CHUNKS = 1 << 13;  // ... and the chunk in 13
static_assert(32 * WAVE_KB * WAVE_SLOT * 4 <= 2 * RING_CAP * 4, "wavefront slots must fit the ring arrays");

// Score of query code `code` (0..7) against a row's base, from the row's
// scores packed as signed bytes (lo: codes 0-3, hi: 4-7): prmt with the
// sign-replicate selector nibbles yields the sign-extended byte.
__device__ __forceinline__ int32_t prof_byte(uint32_t lo, uint32_t hi, uint32_t code) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(lo), "r"(hi), "r"(code * 0x1111u + 0x8880u));
  return int32_t(d);
}

// Whether a planned static-band read suits the row wavefront. Rows start
// about len/256 steps apart (8-column chunks, 32 lanes), so a predecessor d
// rows back was written about d * len / 256 steps before it is read, and the
// lane slots keep the last WAVE_KB chunks: predecessors further back than
// that are read from the arena, and in a lockstep warp one such read delays
// every lane. The wavefront is used when those reads are predicted for
// fewer than 0.3% of the predecessor chunk reads (graphs of few, shallow
// branches); otherwise the row-at-a-time loop runs.
__device__ inline bool wave_suits(const Scratch &s, int n, int64_t cells) {
  const int lane = threadIdx.x & 31;
  const int64_t avg = n > 1 ? cells / n : 0;
  uint64_t all = 0, far = 0;
  for (int i = 1 + lane; i < n; i += 32) {
    const int rs = s.row_start[i], rl = s.row_len[i];
    if (rl <= 0) continue;
    const int pb = s.pred_start[i], pc = s.pred_cnt[i];
    for (int t = 0; t < pc; ++t) {
      const int4 m = s.pmeta[pb + t];
      if (m.x < 0 || m.z <= 0) continue;
      const int lo = max(rs, m.y), hi = min(rs + rl, m.y + m.z);
      if (hi <= lo) continue;
      const uint64_t ch = uint64_t(hi - lo) >> 3;
      all += ch;
      if (int64_t(i - m.x) * avg > int64_t(WAVE_KB - 2) * 256) far += ch;
    }
  }
  for (int d = 16; d; d >>= 1) {
    all += __shfl_xor_sync(FULL, all, d);
    far += __shfl_xor_sync(FULL, far, d);
  }
  return far * 1000 < all * 3;
}

// Per row of a wavefront read, an 80-byte record (wrec, five int4):
// header (band start | band length << 16, arena offset, base | n << 8,
// pred_start) and the row's first eight predecessors with a non-empty band
// as (row, first chunk | chunks << 16). All n such predecessors are also
// listed compactly from pred_start on in `pent` (read as int2), where a lane
// finds the ninth and later ones.
constexpr int WAVE_REC = 20;  // int32 per row record
constexpr int WAVE_REC_PREDS = 8;
__device__ inline void plan_wave(Scratch &s, int n) {
  const int lane = threadIdx.x & 31;
  int2 *list = reinterpret_cast<int2 *>(s.pent);
  for (int i = lane; i < n; i += 32) {
    const int pb = s.pred_start[i], pc = s.pred_cnt[i];
    int32_t *rec = reinterpret_cast<int32_t *>(s.wrec) + WAVE_REC * i;
    int nv = 0;
    if (i > 0) {
      for (int t = 0; t < pc; ++t) {
        const int4 m = s.pmeta[pb + t];
        if (m.x < 0 || m.z <= 0) continue;
        const int2 e = make_int2(m.x, (m.y >> 3) | ((m.z >> 3) << 16));
        list[pb + nv] = e;
        if (nv < WAVE_REC_PREDS) reinterpret_cast<int2 *>(rec + 4)[nv] = e;
        ++nv;
      }
    }
    *reinterpret_cast<int4 *>(rec) =
        make_int4(s.row_start[i] | (s.row_len[i] << 16), int(s.row_off[i]), s.row_base[i] | (nv << 8), pb);
  }
  __syncwarp();
}

__device__ __forceinline__ int4 lds4(const int32_t *p) { return *reinterpret_cast<const int4 *>(p); }
__device__ __forceinline__ void st4(int32_t *p, int32_t a, int32_t b, int32_t c, int32_t d) {
  *reinterpret_cast<int4 *>(p) = make_int4(a, b, c, d);
}
// Asynchronous 16-byte global -> shared copy (cp.async), its commit and the
// wait for every copy this thread issued.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const uint32_t sa = uint32_t(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Shared memory of a wavefront beside the chunk slots (the query's shared
// byte copy is not used by it): per lane two row records (the current row's
// and the next row's, copied ahead with cp.async), then a 64-entry ring of
// (row, arena offset) of the rows begun most recently.
constexpr int WAVE_AUX_BYTES = 32 * 2 * WAVE_REC * 4 + 64 * 8;
static_assert(WAVE_AUX_BYTES <= SEQ_SMEM, "wavefront records must fit the query's shared bytes");

// Rows 1..n-1 of a planned static-band read (row 0 already in the arena).
// `slots` is the warp's 20 KB of chunk slots, `aux` its WAVE_AUX_BYTES of
// records, `q8` the query codes (one byte per column, global), `mat` the
// scoring matrix and, with BYTEPROF, `pk` each base's scores packed as bytes
// (two words per base). Returns the number of predecessor chunks read from
// the arena, or UINT32_MAX when a step found no lane able to advance (never
// expected: the lowest row in flight can always advance; the bound keeps a
// planning fault from spinning the warp).
template <bool BYTEPROF>
__device__ uint32_t dp_wave(const Scratch &s, int n, int32_t *A, const uint8_t *q8, const int32_t *mat, int sigma,
                            const uint32_t *pk, int32_t E, int32_t O, int32_t *slots, char *aux, Work *w) {
  const int lane = threadIdx.x & 31;
  for (int k = lane; k < 32 * WAVE_KB; k += 32) slots[k * WAVE_SLOT + WAVE_TAG] = -1;
  int2 *const offring = reinterpret_cast<int2 *>(aux + 32 * 2 * WAVE_REC * 4);
  for (int k = lane; k < 64; k += 32) offring[k] = make_int2(-1, 0);
  int32_t *const recs = reinterpret_cast<int32_t *>(aux) + lane * 2 * WAVE_REC;
  const int32_t *const wrec = reinterpret_cast<const int32_t *>(s.wrec);
  const int2 *const list = reinterpret_cast<const int2 *>(s.pent);
  int32_t *const mine = slots + lane * WAVE_KB * WAVE_SLOT;
  // copies row x's record into its buffer (rows alternate between the two)
  auto fetch = [&](int x) {
    int32_t *dst = recs + WAVE_REC * (((x - 1) >> 5) & 1);
    const int32_t *src = wrec + WAVE_REC * x;
#pragma unroll
    for (int k = 0; k < WAVE_REC / 4; ++k) cp_async16(dst + 4 * k, src + 4 * k);
    cp_async_commit();
  };
  int r = 1 + lane;
  if (r < n) fetch(r);
  int c = 0, cend = 0, start = 0, len = 0, nv = 0, pb = 0;
  const int32_t *ents = recs;
  int32_t *R = A;
  int32_t icarry = NEG32, mleft = NEG32;
  uint32_t plo = 0, phi = 0;
  const int32_t *mrow = mat;
  // takes the lane's next non-empty row (rows r, r + 32, ...): its record
  // arrived while the row before it ran; the next row's record is fetched
  auto begin_row = [&]() -> bool {
    while (r < n) {
      cp_async_wait_all();
      const int32_t *rec = recs + WAVE_REC * (((r - 1) >> 5) & 1);
      const int4 h = lds4(rec);
      if (r + 32 < n) fetch(r + 32);
      const uint32_t band = uint32_t(h.x);
      if ((band >> 16) > 0) {
        start = int(band & 0xffffu);
        len = int(band >> 16);
        R = A + h.y;
        nv = h.z >> 8;
        pb = h.w;
        ents = rec + 4;
        const int base = h.z & 0xff;
        c = start >> 3;
        cend = (start + len) >> 3;
        icarry = NEG32;
        mleft = NEG32;
        if (BYTEPROF) {
          plo = pk[2 * base];
          phi = pk[2 * base + 1];
        } else {
          mrow = mat + base * sigma;
        }
        offring[r & 63] = make_int2(r, h.y);
        return true;
      }
      r += 32;
    }
    return false;
  };
  bool have = begin_row();
  __syncwarp();
  uint32_t far = 0;
  for (;;) {
    if (!__any_sync(FULL, have)) break;
    const uint64_t tp0 = phase_clock();
    const uint32_t far_before = far;
    (void)far_before;
    int32_t Mx[8], Dx[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      Mx[k] = NEG32;
      Dx[k] = NEG32;
    }
    bool ready = have;
    if (have) {
      const int j0 = c << 3;
      for (int t = 0; t < nv; ++t) {
        const int2 e = t < WAVE_REC_PREDS ? *reinterpret_cast<const int2 *>(ents + 2 * t) : list[pb + t];
        const int p = e.x;
        const int p0 = e.y & 0xffff, p1 = p0 + (e.y >> 16);  // the predecessor's chunks [p0, p1)
        if (c < p0 || c >= p1) continue;
        int4 m0, m1, d0, d1;
        int32_t pv;
        bool got = false;
        if (p > 0) {
          const int32_t *sl = slots + (((p - 1) & 31) * WAVE_KB + (c & (WAVE_KB - 1))) * WAVE_SLOT;
          const int32_t tag = sl[WAVE_TAG], key = (p << 13) | c;
          if (tag < key) {
            ready = false;
            break;
          }
          if (tag == key) {
            m0 = lds4(sl);
            m1 = lds4(sl + 4);
            d0 = lds4(sl + 8);
            d1 = lds4(sl + 12);
            pv = sl[16];
            got = true;
          }
        }
        if (!got) {
          // the predecessor's arena row; its offset from the ring while the
          // row is among the last 64 begun
          const int2 oe = offring[p & 63];
          const int po = oe.x == p ? oe.y : wrec[WAVE_REC * p + 1];
          const int pl = (e.y >> 16) << 3;
          const int k = j0 - (p0 << 3);
          const int32_t *Q = A + po + k;
          m0 = lds4(Q);
          m1 = lds4(Q + 4);
          d0 = lds4(Q + pl);
          d1 = lds4(Q + pl + 4);
          pv = k > 0 ? Q[-1] : NEG32;
          ++far;
        }
        if (c == p0) pv = NEG32;
        const int32_t mp[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
        const int32_t dp[8] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
        Mx[0] = maxs(Mx[0], pv);
#pragma unroll
        for (int k2 = 1; k2 < 8; ++k2) Mx[k2] = maxs(Mx[k2], mp[k2 - 1]);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) Dx[k2] = __viaddmax_s32(dp[k2], E, __viaddmax_s32(mp[k2], O, Dx[k2]));
      }
    }
    if (!__any_sync(FULL, ready)) return UINT32_MAX;
    const uint64_t tp1 = phase_clock();
#ifdef POA_PHASE_CYCLES
    // profiling builds: gather cycles of steps without / with an arena read
    // (rows_g4 / rows_generic) and the number of steps with one (far_preds)
    {
      const bool anyfar = __any_sync(FULL, far != far_before);
      if (anyfar) {
        w->rows_generic += tp1 - tp0;
        w->far_preds += 1;
      } else {
        w->rows_g4 += tp1 - tp0;
      }
    }
#endif
    __syncwarp();
    if (ready) {
      const int j0 = c << 3;
      const uint2 qw = *reinterpret_cast<const uint2 *>(q8 + j0);
      int32_t Mo[8], Io[8];
      int32_t I = icarry;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t code = ((k < 4 ? qw.x : qw.y) >> (8 * (k & 3))) & 0xffu;
        const int32_t prof = BYTEPROF ? prof_byte(plo, phi, code) : mrow[code];
        const int32_t md = __viaddmax_s32(Mx[k], prof, Dx[k]);
        Io[k] = I;
        Mo[k] = maxs(md, I);
        I = __viaddmax_s32(I, E, md + O);
      }
      int32_t *sl = mine + (c & (WAVE_KB - 1)) * WAVE_SLOT;
      st4(sl, Mo[0], Mo[1], Mo[2], Mo[3]);
      st4(sl + 4, Mo[4], Mo[5], Mo[6], Mo[7]);
      st4(sl + 8, Dx[0], Dx[1], Dx[2], Dx[3]);
      st4(sl + 12, Dx[4], Dx[5], Dx[6], Dx[7]);
      sl[16] = mleft;
      sl[WAVE_TAG] = (r << 13) | c;
      const int o = j0 - start;
      st4(R + o, Mo[0], Mo[1], Mo[2], Mo[3]);
      st4(R + o + 4, Mo[4], Mo[5], Mo[6], Mo[7]);
      st4(R + len + o, Dx[0], Dx[1], Dx[2], Dx[3]);
      st4(R + len + o + 4, Dx[4], Dx[5], Dx[6], Dx[7]);
      st4(R + 2 * len + o, Io[0], Io[1], Io[2], Io[3]);
      st4(R + 2 * len + o + 4, Io[4], Io[5], Io[6], Io[7]);
      icarry = I;
      mleft = Mo[7];
      if (++c == cend) {
        r += 32;
        have = begin_row();
      }
    }
    __syncwarp();
    (void)tp0;
    (void)tp1;
  }
  cp_async_wait_all();  // no copy outlives the read (the records' memory is reused)
  return __reduce_add_sync(FULL, far);
}

// Static-band row plan (warp-wide), after fill_pmeta. Per row (planc):
// band start and length, predecessor list start and count, and the base
// code it scores with. Per predecessor entry (pent), where the predecessor's
// M and D states are: still in the ring (the predecessor and every row after
// it went through the ring, and at most RING_CAP entries were written since)
// as (ring entry of its first column, band start, band length, row), or in
// the arena as (-1 - cum_hi, band start, band length, cum_lo) with cum the
// predecessor's cumulative band length (its arena offset is 3 x cum); an
// entry whose predecessor is skipped has band length 0. A row goes through
// the ring when `ring` is set, its band is at most row_max and it has at
// most 32 predecessors (row 0: when its band fits). Counts the row kinds and
// the predecessors read from the arena into `w`.
__device__ inline void plan_rows(Scratch &s, int n, bool ring, int cap, Work *w, int row_max) {
  const int lane = threadIdx.x & 31;
  int carry = 0;  // rows before this block that did not go through the ring
  uint64_t g4 = 0, gen = 0, far = 0;
  for (int i0 = 0; i0 < n; i0 += 32) {
    const int i = i0 + lane;
    bool fast = true;
    if (i < n) {
      const int len = s.row_len[i], pc = s.pred_cnt[i];
      fast = ring && len <= row_max && (i == 0 || pc <= 32);
      if (i > 0 && len > 0) {
        g4 += fast && len > 384 ? 1 : 0;
        gen += fast ? 0 : 1;
      }
      s.planc[i] = make_int4(s.row_start[i], len, s.pred_start[i], int(uint32_t(pc) | (uint32_t(s.row_base[i]) << 24)));
    }
    const unsigned slow = __ballot_sync(FULL, i < n && !fast);
    if (i < n) s.nf[i] = carry + __popc(slow & ((1u << lane) - 1u));  // non-ring rows among 0..i-1
    carry += __popc(slow);
  }
  __syncwarp();
  for (int i = lane; i < n; i += 32) {
    const int pb = s.pred_start[i], pc = s.pred_cnt[i], nfi = s.nf[i];
    const int64_t off = s.row_off[i];
    for (int t = 0; t < pc; ++t) {
      const int4 m = s.pmeta[pb + t];
      const int64_t po = s.pmeta_off[pb + t];
      int4 e = make_int4(-1, 0, 0, 0);
      if (m.x >= 0 && m.z > 0) {
        if (s.nf[m.x] == nfi && off - po <= 3 * int64_t(cap)) {
          e = make_int4(int((po / 3) % cap), m.y, m.z, m.x);
        } else {
          const uint64_t cum = uint64_t(po / 3);
          e = make_int4(-1 - int(cum >> 31), m.y, m.z, int(cum & 0x7fffffffu));
          if (s.row_len[i] > 0 && s.row_len[i] <= row_max) ++far;
        }
      }
      s.pent[pb + t] = e;
    }
  }
  __syncwarp();
  for (int d = 16; d; d >>= 1) {
    g4 += __shfl_xor_sync(FULL, g4, d);
    gen += __shfl_xor_sync(FULL, gen, d);
    far += __shfl_xor_sync(FULL, far, d);
  }
#ifndef POA_PHASE_CYCLES
  w->rows_g4 += g4;
  w->rows_generic += gen;
  w->far_preds += far;
#endif
}

// Predecessor-cell updates of a planned read (after fill_pmeta): the sum
// over rows of each in-band predecessor's band overlap, which is the trip
// count of the reference's predecessor loop (align.rs:751-797).
__device__ inline uint64_t pred_overlap_cells(const Scratch &s, int n) {
  const int lane = threadIdx.x & 31;
  uint64_t tot = 0;
  for (int i = 1 + lane; i < n; i += 32) {
    const int rs = s.row_start[i], rl = s.row_len[i];
    if (rl <= 0) continue;
    const int pb = s.pred_start[i], pc = s.pred_cnt[i];
    for (int t = 0; t < pc; ++t) {
      const int4 m = s.pmeta[pb + t];
      if (m.x < 0 || m.z <= 0) continue;
      const int lo = max(rs, m.y), hi = min(rs + rl, m.y + m.z);
      if (hi > lo) tot += uint64_t(hi - lo);
    }
  }
  for (int d = 16; d; d >>= 1) tot += __shfl_xor_sync(FULL, tot, d);
  return tot;
}

// Per predecessor entry: (row, band start, band length, edge weight) and the
// row's arena offset, once every row's band is known (warp-wide).
__device__ inline void fill_pmeta(Scratch &s, int n) {
  const int lane = threadIdx.x & 31;
  const int etot = s.pred_start[n - 1] + s.pred_cnt[n - 1];
  for (int e = lane; e < etot; e += 32) {
    const int2 pr = s.pred[e];
    if (pr.x >= 0) {
      s.pmeta[e] = make_int4(pr.x, s.row_start[pr.x], s.row_len[pr.x], pr.y);
      s.pmeta_off[e] = s.row_off[pr.x];
    } else {
      s.pmeta[e] = make_int4(-1, 0, 0, 0);
      s.pmeta_off[e] = 0;
    }
  }
  __syncwarp();
}

// One DP kernel invocation (poa_simd_arena, align.rs:588-911, or
// poa_scalar_i64, align.rs:913-1162) by a whole warp.
// WIDE: bands up to RING_WIDE_LEN columns go through the striped tiles (in
// 512-column segments); otherwise bands above RING_MAX_LEN take the generic
// row. The batched kernel keeps the narrower form (its register budget), the
// seed-window kernels, whose bands are up to twice the window band, the wide.
template <typename S, bool WIDE = false>
__device__ int32_t poa_kernel(Job *J, const DevParams &P, char *arena, int64_t arena_bytes, int beg_id, int end_id,
                              const uint8_t *query, int qlen, bool adaptive_arg, uint64_t band_b, uint64_t f,
                              Scratch &s, int *n_items, Work *cells, WarpSmem *sm) {
  constexpr S NEGV = ScoreTraits<S>::NEGV;
  constexpr int kRowMax = WIDE ? RING_WIDE_LEN : RING_MAX_LEN;
  const int lane = threadIdx.x & 31;
  if (beg_id >= J->n_nodes || end_id >= J->n_nodes) return ST_ANCHOR_NOT_IN_GRAPH;
  const int beg = J->rank[beg_id], end = J->rank[end_id];
  if (end <= beg || end >= J->n_rank) return ST_ANCHORS_NOT_ORDERED;
  const int n = end - beg + 1;
  const int64_t m = int64_t(qlen) + 2;
  if (m > INT32_MAX) return ST_COORD_LIMITS;
  const int64_t padded = (m / 8 + 1) * 8;
  if (!carve_scratch(arena, arena_bytes, n, J->n_edges, padded, m + 1, s)) return ST_ARENA_FULL;
  // the byte copy the striped rows read: shared memory when it fits
  uint8_t *q8 = (sm && padded + 4 <= SEQ_SMEM) ? sm->seq8 : s.seq8;
  for (int64_t c = lane; c < padded + 4; c += 32) {
    const int code = (c == 0 || c > qlen) ? P.unknown : int(P.encode[query[c - 1]]);
    if (c < padded) s.seq[c] = code;
    q8[c] = uint8_t(code);
    if (q8 != s.seq8) s.seq8[c] = uint8_t(code);  // the row wavefront reads the global copy
  }
  const bool adaptive = adaptive_arg || P.adaptive;
  uint64_t bandu = band_b + (f == 0 ? 0 : uint64_t(m) / f);
  if (bandu < band_b) bandu = UINT64_MAX;
  const int64_t band = int64_t(bandu < uint64_t(INT32_MAX) ? bandu : uint64_t(INT32_MAX));
  const S E = S(P.gap_ext), O = S(P.gap_open);
  const S s00 = S(P.matrix[P.unknown * P.sigma + P.unknown]);
  __syncwarp();
  const uint64_t t_g0 = phase_clock();
  // the backward guide pass's ring borrows the DP ring's shared memory
  int32_t st = guides(J, s, beg, end, n, sm->gring_v, sm->gring_s, reinterpret_cast<int64_t *>(sm->ring_d), cells);
  const uint64_t t_g1 = phase_clock();
  cells->phase[0] += t_g1 - t_g0;
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
  // ring entries of rows before ring_floor (an arena offset) are not valid
  int64_t ring_floor = 0;
  int32_t *const rm = sm ? sm->rv.m : nullptr;
  int32_t *const rd = sm ? sm->rv.d : nullptr;
  const int rcap = sm ? sm->rv.cap : RING_CAP;
  if (sm) {
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
    fill_pmeta(s, n);
    const bool ring = kFastType && sm;
    if constexpr (kFastType) {
      // the row wavefront, unless this warp leads cooperative rows (its
      // helpers wait for rows) or the sizes exceed its tags
      const bool wave = ring && P.row_wave && sm->rv.pad[0] == 0 && n < WAVE_MAX_ROWS &&
                        (padded >> 3) < WAVE_MAX_CHUNKS && tot <= INT32_MAX &&
                        (P.row_wave == 2 || wave_suits(s, n, tot / 3));
      if (wave) {
        plan_wave(s, n);
        cells->pred_cells += pred_overlap_cells(s, n);
        if (s.row_len[0] > 0 && lane == 0) dp_row0<S>(A + s.row_off[0], s.row_len[0], s00, E, O);
        const int32_t *mat = smem_matrix ? sm->matrix : P.matrix;
        uint32_t far;
        if (P.byte_prof) {
          // each base's scores as signed bytes, two words per base
          uint32_t *pk = reinterpret_cast<uint32_t *>(sm->matrix) + (SMEM_MATRIX - 16);
          if (lane < 2 * P.sigma) {
            const int b = lane >> 1, k0 = 4 * (lane & 1);
            uint32_t w = 0;
            for (int k = 0; k < 4; ++k)
              if (k0 + k < P.sigma) w |= (uint32_t(P.matrix[b * P.sigma + k0 + k]) & 0xffu) << (8 * k);
            pk[lane] = w;
          }
          __syncwarp();
          far = dp_wave<true>(s, n, reinterpret_cast<int32_t *>(A), s.seq8, mat, P.sigma, pk, int32_t(E),
                              int32_t(O), sm->ring_m, reinterpret_cast<char *>(sm->seq8), cells);
        } else {
          __syncwarp();
          far = dp_wave<false>(s, n, reinterpret_cast<int32_t *>(A), s.seq8, mat, P.sigma, nullptr, int32_t(E),
                               int32_t(O), sm->ring_m, reinterpret_cast<char *>(sm->seq8), cells);
        }
        if (far == UINT32_MAX) return ST_WAVE_STALL;
        cells->wave = 1;
#ifndef POA_PHASE_CYCLES
        cells->far_preds += far;
#endif
        cells->cells += row_cells;
        cells->dp_bytes += row_cells * 3 * sizeof(S);
        const uint64_t t_w1 = phase_clock();
        cells->phase[1] += t_w1 - t_g1;
        // (the query's shared bytes held the wavefront's row records)
        st = traceback<S>(J, P, s, A, beg, n, m, smem_matrix ? sm->matrix : P.matrix, s.seq8, n_items, cells);
        cells->phase[2] += phase_clock() - t_w1;
        return st;
      }
    }
    plan_rows(s, n, ring, rcap, cells, kRowMax);
    cells->pred_cells += pred_overlap_cells(s, n);
    if (s.row_len[0] > 0 && lane == 0) dp_row0<S>(A + s.row_off[0], s.row_len[0], s00, E, O);
    __syncwarp();
    if (ring) ring_put_row0(rm, rd, A, s.row_len[0], kRowMax);
    // a lone giant's block-mates join the row loop (cooperative rows: the
    // striped int32 rows, or the int64 kernel's generic rows)
    const bool coop = sm && sm->rv.pad[0] != 0 && (ring || !kFastType);
    CoopDesc *cd = coop ? reinterpret_cast<CoopDesc *>(sm->ring_m) : nullptr;
    if (coop) cells->coop = 1;
    if (coop) {
      if (lane == 0) {
        cd->mode = COOP_ROWS;
        cd->E = int32_t(E);
        cd->O = int32_t(O);
        cd->q8 = q8;
        cd->rm = rm;
        cd->rd = rd;
        cd->cap = rcap;
        cd->E64 = int64_t(E);
        cd->O64 = int64_t(O);
        cd->gA = reinterpret_cast<const int64_t *>(A);
        cd->grs = s.row_start;
        cd->grl = s.row_len;
        cd->gseq = s.seq;
        cd->gro = s.row_off;
      }
      coop_bar(2);
    }
    // rows 1..n-1. The plans of a 64-row window sit in the lanes (rows
    // w0 + lane and w0 + 32 + lane), loaded 32 rows before they are needed;
    // each row's predecessor entries are loaded three rows ahead. A row's
    // arena offset and ring entry follow from the cumulative band length, so
    // no global load stands between one row and the next.
    const int4 zero = make_int4(0, 0, 0, 0), none = make_int4(-1, 0, 0, 0);
    int w0 = 0;
    int4 wc = lane < n ? ld_early(s.planc + lane) : zero;
    int4 wn = 32 + lane < n ? ld_early(s.planc + 32 + lane) : zero;
    auto pent_of = [&](int r) {  // r - w0 < 64
      if (r >= n) return none;
      const int d = r - w0;
      const int4 v = d < 32 ? wc : wn;
      const int pb = __shfl_sync(FULL, v.z, d & 31);
      const int pc = __shfl_sync(FULL, v.w, d & 31) & 0xffffff;
      return lane < pc ? ld_early(s.pent + pb + lane) : none;
    };
    int4 e1 = pent_of(1), e2 = pent_of(2), e3 = pent_of(3);
    int64_t cum = s.row_len[0];  // cumulative band length of the rows before row i
    int rpos = rcap > 0 ? int(cum % rcap) : 0;
    for (int i = 1; i < n; ++i) {
      if (i - w0 >= 32) {
        w0 += 32;
        wc = wn;
        wn = w0 + 32 + lane < n ? ld_early(s.planc + w0 + 32 + lane) : zero;
      }
      const int src = (i - w0) & 31;
      const int start = __shfl_sync(FULL, wc.x, src), len = __shfl_sync(FULL, wc.y, src);
      const int pb = __shfl_sync(FULL, wc.z, src);
      const uint32_t pcw = uint32_t(__shfl_sync(FULL, wc.w, src));
      const int pc = int(pcw & 0xffffffu), base = int(pcw >> 24);
      const int4 mt = e1;
      e1 = e2;
      e2 = e3;
      e3 = pent_of(i + 3);
      if (len == 0) continue;
      const int64_t off = 3 * cum;
      const int pos_i = rpos;
      cum += len;
      if (rcap > 0) {
        if (len < rcap) {
          rpos += len;
          if (rpos >= rcap) rpos -= rcap;
        } else {
          rpos = int(cum % rcap);
        }
      }
      S *R = A + off;
      if (ring && len <= kRowMax && pc <= 32) {
        const bool ok = mt.z > 0;
        const int64_t mcum = mt.x < 0 ? ((int64_t(-1 - mt.x) << 31) | int64_t(uint32_t(mt.w))) : 0;
        const int32_t *my_g = reinterpret_cast<const int32_t *>(A) + 3 * mcum;
        const unsigned vmask = __ballot_sync(FULL, ok);
        const int32_t *mrow = smem_matrix ? sm->matrix + base * P.sigma : P.matrix + base * P.sigma;
        if (coop) {
          const int slot = __popc(vmask & ((1u << lane) - 1u));
          if (ok) {
            cd->ps[slot] = mt.y;
            cd->pl[slot] = mt.z;
            cd->pos[slot] = mt.x < 0 ? -1 : mt.x;
            cd->g[slot] = my_g;
          }
          const bool seg = len > RING_MAX_LEN;  // (the wide forms only)
          if (lane == 0) {
            cd->op = seg ? COOP_SEG : COOP_ROW;
            cd->start = start;
            cd->len = len;
            cd->pos_i = pos_i;
            cd->n_pred = __popc(vmask);
            cd->R = reinterpret_cast<int32_t *>(R);
            cd->mrow = mrow;
          }
          coop_bar(1);
          if (seg)
            coop_seg(cd, 0);  // the leader computes stripe 0 of every segment
          else
            coop_stripe(cd, 0);  // the leader computes stripe 0
          continue;
        }
        int32_t bv = INT32_MIN;
        int bj = INT32_MAX;
        dp_row_fast<false, WIDE>(lane, start, len, reinterpret_cast<int32_t *>(R), q8, mrow, int32_t(E), int32_t(O), vmask,
                           mt.y, mt.z, (ok && mt.x >= 0) ? mt.x : -1, my_g, rm, rd, rcap, pos_i, bv, bj);
        __syncwarp();
        continue;
      }
      if constexpr (!kFastType) {
        if (coop && pc <= 32 && len >= COOP_GEN_MIN_LEN) {
          if (lane == 0) {
            cd->op = COOP_GEN;
            cd->start = start;
            cd->len = len;
            cd->n_pred = pc;
            cd->gR = reinterpret_cast<int64_t *>(R);
            cd->gpred = s.pred + pb;
            cd->mrow = P.matrix + base * P.sigma;
          }
          coop_bar(1);
          coop_gen64(cd, 0);  // the leader computes the first quarter
          continue;
        }
      }
      S bv = ScoreTraits<S>::LOWEST;
      int bj = INT32_MAX;
      dp_row_generic<S>(lane, start, len, R, A, s, pb, pc, P.matrix + base * P.sigma, E, O, false, bv, bj);
      __syncwarp();
    }
    if (coop) {  // the block-mates leave the row loop
      if (lane == 0) cd->op = COOP_STOP;
      coop_bar(1);
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
      if (lane == 0) s.row_base[i] = (i == n - 1) ? P.unknown : int(J->base[J->rank_to_node[beg + i]]);
      if (i == 0) {
        if (start != 0) {
          cells->cells += row_cells;
          cells->dp_bytes += row_cells * 3 * sizeof(S);
          return ST_BAND_EXCLUDES_SOURCE;
        }
        if (lane == 0) dp_row0<S>(R, len, s00, E, O);
        __syncwarp();
        if (kFastType && sm) ring_floor = ring_put_row0(rm, rd, A, len, kRowMax);
        continue;
      }
      const int node = J->rank_to_node[beg + i];
      const int base = (i == n - 1) ? P.unknown : int(J->base[node]);
      const int pb = s.pred_start[i], pc = s.pred_cnt[i];
      S bestv = ScoreTraits<S>::LOWEST;
      int bestj = INT32_MAX;
      if (kFastType && sm && len <= kRowMax && pc <= 32) {
        if (len > 384) cells->rows_g4 += 1;
        int my_ps = 0, my_pl = 0, my_pos = -1;
        const int32_t *my_g = nullptr;
        bool ok = false;
        if (lane < pc) {
          const int p = s.pred[pb + lane].x;
          if (p >= 0) {
            my_ps = s.row_start[p];
            my_pl = s.row_len[p];
            const int64_t po = s.row_off[p];
            my_g = reinterpret_cast<const int32_t *>(A) + po;
            ok = my_pl > 0;
            if (ok) my_pos = ring_pos(po, off, ring_floor, rcap);
          }
        }
        const unsigned vmask = __ballot_sync(FULL, ok);
        cells->far_preds += __popc(__ballot_sync(FULL, ok && my_pos < 0));
        const int32_t *mrow = smem_matrix ? sm->matrix + base * P.sigma : P.matrix + base * P.sigma;
        int32_t bv = INT32_MIN;
        int bj = INT32_MAX;
        dp_row_fast<true, WIDE>(lane, start, len, reinterpret_cast<int32_t *>(R), q8, mrow, int32_t(E), int32_t(O), vmask,
                          my_ps, my_pl, my_pos, my_g, rm, rd, rcap, int((off / 3) % rcap), bv, bj);
        bestv = S(bv);
        bestj = bj;
      } else {
        ring_floor = off + 1;  // this row does not enter the ring
        cells->rows_generic += 1;
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
  if (do_adapt) {
    __syncwarp();
    fill_pmeta(s, n);
    cells->pred_cells += pred_overlap_cells(s, n);
  }
  const uint64_t t_d1 = phase_clock();
  cells->phase[1] += t_d1 - t_g1;
  st = traceback<S>(J, P, s, A, beg, n, m, (sm && smem_matrix) ? sm->matrix : P.matrix, q8, n_items, cells);
  cells->phase[2] += phase_clock() - t_d1;
  return st;
}

// poa_inner (align.rs:531-545): score-guard dispatch.
template <bool WIDE = false>
__device__ inline int32_t poa_inner(Job *J, const DevParams &P, char *arena, int64_t bytes, int beg_id, int end_id,
                                    const uint8_t *q, int qlen, bool adaptive, uint64_t band_b, uint64_t f,
                                    Scratch &s, int *n_items, Work *cells, WarpSmem *sm) {
  const bool use32 = P.kernel == 1 || (P.kernel == 0 && i32_scores_safe(J, P, beg_id, end_id, qlen));
  if (use32)
    return poa_kernel<int32_t, WIDE>(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive, band_b, f, s, n_items, cells,
                               sm);
  return poa_kernel<int64_t, WIDE>(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive, band_b, f, s, n_items, cells,
                             sm);
}

// poa (align.rs:192-211): on an alignment error with f != 0, retry with the
// full matrix (f = 0, static band).
template <bool WIDE = false>
__device__ inline int32_t poa_retry(Job *J, const DevParams &P, char *arena, int64_t bytes, int beg_id, int end_id,
                                    const uint8_t *q, int qlen, bool adaptive, uint64_t band_b, Scratch &s,
                                    int *n_items, Work *cells, WarpSmem *sm) {
  int32_t st =
      poa_inner<WIDE>(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive, band_b, P.f, s, n_items, cells, sm);
  if (is_alignment_error(st) && P.f != 0)
    st = poa_inner<WIDE>(J, P, arena, bytes, beg_id, end_id, q, qlen, false, band_b, 0, s, n_items, cells, sm);
  return st;
}

// align::align (align.rs:81-98) for unseeded parameters; writes s.items.
template <bool WIDE = false>
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
  return poa_retry<WIDE>(J, P, arena, bytes, 0, 1, q, qlen, P.adaptive != 0, P.b, s, n_items, cells, sm);
}

// Re-sorts the rank windows of reorder_incremental (warp-wide). spans[k] =
// (u, v, old rank of u, -): path node u is followed on the path, after the new
// nodes spliced behind it (add[old rank of u] of them), by v of lower rank.
// Each window [rank(v), rank(u) + add] is merged with those it overlaps and
// re-sorted by Kahn's algorithm over the edges inside it. Returns false when a
// window holds a cycle.
__device__ inline bool repair_windows(Job *J, int4 *spans, int n_spans, const int32_t *add, int32_t *deg,
                                      int32_t *stack, int32_t *order) {
  const int lane = threadIdx.x & 31;
  // windows in new ranks, sorted by their first rank (lane 0; few per read)
  if (lane == 0) {
    for (int k = 0; k < n_spans; ++k) {
      const int4 sp = spans[k];
      spans[k] = make_int4(J->rank[sp.y], J->rank[sp.x] + add[sp.z], 0, 0);
    }
    for (int k = 1; k < n_spans; ++k) {
      const int4 x = spans[k];
      int q = k - 1;
      while (q >= 0 && spans[q].x > x.x) {
        spans[q + 1] = spans[q];
        --q;
      }
      spans[q + 1] = x;
    }
  }
  __syncwarp();
  bool ok = true;
  int k = 0;
  while (k < n_spans && ok) {
    const int lo = spans[k].x;
    int hi = spans[k].y;
    ++k;
    while (k < n_spans && spans[k].x <= hi) {
      hi = max(hi, spans[k].y);
      ++k;
    }
    const int w = hi - lo + 1;
    // in-degree from inside the window
    for (int q = lane; q < w; q += 32) {
      const int node = J->rank_to_node[lo + q];
      int d = 0;
      for_list(J, J->in_head, J->in_cnt, node, [&](int pred, int) {
        const int r = J->rank[pred];
        if (r >= lo && r <= hi) ++d;
      });
      deg[q] = d;
    }
    __syncwarp();
    int done = 0;
    if (lane == 0) {
      int sp = 0;
      for (int q = w - 1; q >= 0; --q)
        if (deg[q] == 0) stack[sp++] = q;
      while (sp > 0) {
        const int q = stack[--sp];
        const int node = J->rank_to_node[lo + q];
        order[done++] = node;
        for_list(J, J->out_head, J->out_cnt, node, [&](int succ, int) {
          const int r = J->rank[succ];
          if (r >= lo && r <= hi && --deg[r - lo] == 0) stack[sp++] = r - lo;
        });
      }
    }
    done = __shfl_sync(FULL, done, 0);
    __syncwarp();
    if (done != w) {
      ok = false;
      break;
    }
    for (int q = lane; q < w; q += 32) {
      const int node = order[q];
      J->rank[node] = lo + q;
      J->rank_to_node[lo + q] = node;
    }
    __syncwarp();
  }
  return ok;
}

// Splices a read's new nodes into the current topological order (warp-wide):
// each run of consecutive new nodes on the path is placed right after the
// pre-existing path node before it. Where two consecutive pre-existing path
// nodes are out of order (the path reached an existing column sibling placed
// after the node that follows it), the ranks between them, with the new nodes
// spliced there, form a window; overlapping windows are merged and each is
// re-sorted on its own by Kahn's algorithm over the edges inside it. Nodes
// outside the windows keep their relative order and every edge into or out of
// a window already points forward, so the result is a topological order. When
// a window holds a cycle (or scratch is short) nothing usable is produced and
// false is returned; the caller then runs the LIFO toposort of
// graph.rs:125-178, which reports the cycle. With a static band and no
// seeding the rank order does not change any alignment: band guides, DP
// states and traceback choices depend only on the predecessor / successor
// lists in insertion order.
__device__ inline bool reorder_incremental(Job *J, const int4 *items, int n_items, int n_old, char *buf,
                                           int64_t buf_bytes) {
  const int lane = threadIdx.x & 31;
  const int n_new = J->n_nodes;
  if (J->n_rank != n_old || n_items <= 0) return false;
  if (int64_t(4) * (2 * int64_t(n_old) + 4 * int64_t(n_new)) + int64_t(16) * (n_items + 2) > buf_bytes)
    return false;
  int32_t *add = reinterpret_cast<int32_t *>(buf);
  int32_t *first = add + n_old;
  int32_t *nr2n = first + n_old;
  int32_t *wdeg = nr2n + n_new;  // window scratch: degree, stack, order
  int32_t *wstack = wdeg + n_new;
  int32_t *worder = wstack + n_new;
  int4 *spans = reinterpret_cast<int4 *>(align_up(reinterpret_cast<int64_t>(worder + n_new), 16));
  for (int r = lane; r < n_old; r += 32) add[r] = 0;
  __syncwarp();
  long long carry = -1;  // last pre-existing path item as (index << 32 | rank)
  int n_spans = 0;
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
    bool out_of_order = false;
    int pt = 0, pr = 0;
    if (old && prev >= 0) {
      pt = int(prev >> 32);
      pr = int(prev & 0xffffffffLL);
      out_of_order = pr >= rk;
      if (t - pt - 1 > 0) {
        add[pr] = t - pt - 1;
        first[pr] = items[pt + 1].w;
      }
    }
    const unsigned om = __ballot_sync(FULL, out_of_order);
    if (out_of_order) spans[n_spans + __popc(om & ((1u << lane) - 1u))] = make_int4(items[pt].w, id, pr, 0);
    n_spans += __popc(om);
    const long long last = __shfl_sync(FULL, inc, 31);
    carry = last > carry ? last : carry;
  }
  if (carry < 0) return false;
  if (lane == 0) {
    const int pt = int(carry >> 32), pr = int(carry & 0xffffffffLL);
    if (n_items - pt - 1 > 0) {
      add[pr] = n_items - pt - 1;
      first[pr] = items[pt + 1].w;
    }
  }
  __syncwarp();
  // new ranks, four 32-row groups per step so their loads overlap
  constexpr int U = 4;
  int shift = 0;
  for (int r0 = 0; r0 < n_old; r0 += 32 * U) {
    int a[U], node[U], inc[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int r = r0 + 32 * u + lane;
      a[u] = r < n_old ? add[r] : 0;
      node[u] = r < n_old ? J->rank_to_node[r] : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      inc[u] = a[u];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(FULL, inc[u], d);
        if (lane >= d) inc[u] += v;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int r = r0 + 32 * u + lane;
      if (r < n_old) {
        const int nr = r + shift + inc[u] - a[u];
        nr2n[nr] = node[u];
        J->rank[node[u]] = nr;
        if (a[u] > 0) {
          const int f = first[r];
          for (int k = 0; k < a[u]; ++k) {
            nr2n[nr + 1 + k] = f + k;
            J->rank[f + k] = nr + 1 + k;
          }
        }
      }
      shift += __shfl_sync(FULL, inc[u], 31);
    }
  }
  __syncwarp();
  for (int r0 = 0; r0 < n_new; r0 += 32 * U) {
    int v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int r = r0 + 32 * u + lane;
      v[u] = r < n_new ? nr2n[r] : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int r = r0 + 32 * u + lane;
      if (r < n_new) J->rank_to_node[r] = v[u];
    }
  }
  __syncwarp();
  if (n_spans > 0 && !repair_windows(J, spans, n_spans, add, wdeg, wstack, worder)) return false;
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
template <bool WIDE = false>
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
  int32_t st = align_query<WIDE>(J, P, arena, bytes, q, qlen, s, &n_items, &cells, sm);
  if (st != ST_OK) return st;
  const uint64_t t_u0 = phase_clock();
  const int n_old = J->n_nodes;
  int32_t *mark = s.dp_bytes >= int64_t(n_old) * 4 ? reinterpret_cast<int32_t *>(s.dp) : nullptr;
  const int sid = J->read_id ? J->read_id[r] : J->seq_base + r;
  if (!add_path_warp(J, P, sid, s.items, n_items, &st, mark)) {
    if (lane == 0) st = add_path(J, P, sid, s.items, n_items);
    st = __shfl_sync(FULL, st, 0);
  }
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
      J->pred_cells += cells.pred_cells;
      J->far_preds += cells.far_preds;
      J->rows_g4 += cells.rows_g4;
      J->rows_generic += cells.rows_generic;
      J->coop |= cells.coop;
      J->wave_reads += cells.wave;
      cells.phase[3] += phase_clock() - t_u0;
      for (int k = 0; k < 4; ++k) J->phase[k] += cells.phase[k];
      J->next_read = r + 1;
    }
  }
  st = __shfl_sync(FULL, st, 0);
  __syncwarp();
  return st;
}

}  // namespace poa
