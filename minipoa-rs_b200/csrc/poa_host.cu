// Host runtime and C ABI of the B200 POA library: CUDA context, growable
// device-resident graphs, the batched scheduler, and output rendering.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <sys/stat.h>
#include <fstream>
#include <stdexcept>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/minipoa_b200.h"
#include "host_graph.h"
#include "poa_internal.h"
#include "gfa.h"
#include "poa_consensus.h"
#include "poa_pack.h"
#include "seed.h"

using namespace poa;

namespace {

struct CudaError {
  cudaError_t code;
  std::string where;
};

inline double now_steady() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) throw CudaError{e_, #call};             \
  } while (0)

struct AlignError {
  int code;  // POA_ERR_*
  std::string msg;
};

std::string status_message(int32_t st, int err_i, int err_j) {
  switch (st) {
    case ST_ANCHOR_NOT_IN_GRAPH: return "alignment anchor is not in graph";
    case ST_ANCHORS_NOT_ORDERED: return "alignment anchors are not topologically ordered";
    case ST_COORD_LIMITS: return "alignment exceeds coordinate limits";
    case ST_NO_PATH: return "no graph path connects alignment anchors";
    case ST_BAND_NO_INTERSECT: return "alignment band does not intersect graph path";
    case ST_BAND_EXCLUDES_SOURCE: return "alignment band excludes source";
    case ST_TB_NO_ADVANCE: return "alignment traceback failed to advance";
    case ST_TB_LEFT_BAND: return "alignment traceback left active band";
    case ST_TB_NO_PRED:
      return "alignment traceback has no predecessor at graph row " + std::to_string(err_i) + ", query column " +
             std::to_string(err_j);
    case ST_BASE_OUTSIDE: return "alignment base outside alphabet";
    case ST_UNKNOWN_NODE: return "alignment references an unknown node";
    case ST_CYCLE: return "graph contains a cycle (possibly between alignment columns)";
    case ST_COLUMN_DEPS: return "invalid graph column dependencies";
    case ST_ARENA_FULL: return "DP arena exhausted";
    case ST_GRAPH_FULL: return "graph capacity exhausted";
    case ST_OUT_TOO_SMALL: return "output buffer holds fewer items than the alignment path";
    case ST_SEEDING_UNSUPPORTED: return "seeded windows (-S) are not available in this build";
    case ST_WAVE_STALL: return "DP row wavefront made no progress (internal error)";
    default: return "unknown device status " + std::to_string(st);
  }
}

int status_code(int32_t st) {
  if (is_alignment_error(st)) return POA_ERR_ALIGN;
  if (st == ST_SEEDING_UNSUPPORTED) return POA_ERR_UNSUPPORTED;
  if (st == ST_OUT_TOO_SMALL) return POA_ERR_INVALID;
  if (st == ST_WAVE_STALL) return POA_ERR_TIMEOUT;
  return POA_ERR_ALLOC;
}

struct Caps {
  int32_t node_cap = 0, chunk_cap = 0, path_cap = 0, max_paths = 0;
  int sigma = 0;
};

// Assigns the graph arrays of one job inside `base` (nullptr: size only).
size_t layout(const Caps &c, char *base, Job *J) {
  size_t o = 0;
  auto take = [&](size_t bytes) -> char * {
    const size_t at = o;
    o = (o + bytes + 255) / 256 * 256;
    return base ? base + at : nullptr;
  };
  const size_t N = size_t(c.node_cap);
  J->base = (uint8_t *)take(N);
  J->parent = (int32_t *)take(N * 4);
  J->rank = (int32_t *)take(N * 4);
  J->coverage = (int32_t *)take(N * 4);
  J->in_head = (int32_t *)take(N * 4);
  J->in_tail = (int32_t *)take(N * 4);
  J->in_cnt = (int32_t *)take(N * 4);
  J->out_head = (int32_t *)take(N * 4);
  J->out_tail = (int32_t *)take(N * 4);
  J->out_cnt = (int32_t *)take(N * 4);
  J->rank_to_node = (int32_t *)take(N * 4);
  J->aligned = (int32_t *)take(N * size_t(c.sigma) * 4);
  J->chunk_id = (int32_t *)take(size_t(c.chunk_cap) * CHUNK * 4);
  J->chunk_w = (int32_t *)take(size_t(c.chunk_cap) * CHUNK * 4);
  J->chunk_next = (int32_t *)take(size_t(c.chunk_cap) * 4);
  J->path_items = (int32_t *)take(size_t(c.path_cap) * 4 + 4);
  J->path_off = (int32_t *)take(size_t(c.max_paths + 1) * 4);
  J->path_seq = (int32_t *)take(size_t(c.max_paths) * 4 + 4);
  J->node_cap = c.node_cap;
  J->chunk_cap = c.chunk_cap;
  J->path_cap = c.path_cap;
  J->max_paths = c.max_paths;
  return o;
}

// (pointer, bytes) of each array of a laid-out job, in a fixed order.
std::vector<std::pair<char *, size_t>> arrays(const Job &J, const Caps &c) {
  const size_t N = size_t(c.node_cap);
  return {{(char *)J.base, N},
          {(char *)J.parent, N * 4},
          {(char *)J.rank, N * 4},
          {(char *)J.coverage, N * 4},
          {(char *)J.in_head, N * 4},
          {(char *)J.in_tail, N * 4},
          {(char *)J.in_cnt, N * 4},
          {(char *)J.out_head, N * 4},
          {(char *)J.out_tail, N * 4},
          {(char *)J.out_cnt, N * 4},
          {(char *)J.rank_to_node, N * 4},
          {(char *)J.aligned, N * size_t(c.sigma) * 4},
          {(char *)J.chunk_id, size_t(c.chunk_cap) * CHUNK * 4},
          {(char *)J.chunk_w, size_t(c.chunk_cap) * CHUNK * 4},
          {(char *)J.chunk_next, size_t(c.chunk_cap) * 4},
          {(char *)J.path_items, size_t(c.path_cap) * 4 + 4},
          {(char *)J.path_off, size_t(c.max_paths + 1) * 4},
          {(char *)J.path_seq, size_t(c.max_paths) * 4 + 4}};
}

std::vector<uint8_t> encode_table(const HostParams &p) {
  std::vector<uint8_t> t(256);
  for (int c = 0; c < 256; ++c) t[size_t(c)] = uint8_t(p.encode(uint8_t(c)));
  return t;
}

thread_local std::string g_create_error;
// The message of the calling thread's last failed call: the server API is
// called from several threads at once (submit on one, wait on others).
thread_local std::string t_last_error;

char *dup_string(const std::string &s) {
  char *o = (char *)std::malloc(s.size() + 1);
  std::memcpy(o, s.data(), s.size());
  o[s.size()] = 0;
  return o;
}

}  // namespace

// ---------------------------------------------------------------------------

struct poa_batch;

struct poa_ctx {
  // live batches of this context: a batch that needs its DP arena pool while
  // others hold theirs takes their memory back (they re-allocate on their
  // next run)
  std::vector<poa_batch *> batches;
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  uint64_t budget = 0;
  uint64_t allocated = 0;
  char *arena = nullptr;
  int64_t arena_bytes = 0;
  uint8_t *qbuf = nullptr;
  size_t qbuf_bytes = 0;
  char *dlbuf = nullptr;  // graph downloads: packed records (grow-only, reused)
  size_t dlbuf_bytes = 0;
  int32_t *h_dl = nullptr;  // pinned host copy of the last graph download
  size_t h_dl_bytes = 0;
  int4 *items = nullptr;
  int32_t *n_items = nullptr;
  size_t items_cap = 0;
  int32_t *d_matrix = nullptr;
  uint8_t *d_encode = nullptr;
  size_t matrix_cap = 0;
  int window_launch = 0;  // seeded reads: 0 = one launch for all windows, 1 = one launch per window
  uint64_t seed_windows = 0, seed_launches = 0, seed_fallbacks = 0;

  void *dalloc(size_t bytes) {
    if (allocated + bytes > budget) throw AlignError{POA_ERR_ALLOC, "device memory budget exceeded"};
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw AlignError{POA_ERR_ALLOC, std::string("cudaMalloc failed: ") + cudaGetErrorString(e)};
    }
    allocated += bytes;
    return p;
  }
  void dfree(void *p, size_t bytes) {
    if (p) {
      const cudaError_t e = cudaFree(p);
      if (e != cudaSuccess) {
        cudaGetLastError();
        std::fprintf(stderr, "minipoa_b200: cudaFree failed: %s\n", cudaGetErrorString(e));
      }
      allocated -= std::min<uint64_t>(allocated, bytes);
    }
  }
  void ensure_arena(int64_t bytes) {
    if (arena_bytes >= bytes) return;
    dfree(arena, size_t(arena_bytes));
    arena = nullptr;
    arena_bytes = 0;
    arena = (char *)dalloc(size_t(bytes));
    arena_bytes = bytes;
  }
  void ensure_qbuf(size_t bytes) {
    if (qbuf_bytes >= bytes) return;
    dfree(qbuf, qbuf_bytes);
    qbuf = nullptr;
    qbuf_bytes = 0;
    qbuf = (uint8_t *)dalloc(bytes);
    qbuf_bytes = bytes;
  }
  // Graphs grow read by read: both download buffers grow by half again so
  // that a growing graph re-allocates them O(log n) times.
  void ensure_dlbuf(size_t bytes) {
    if (dlbuf_bytes >= bytes) return;
    size_t want = std::max(bytes, dlbuf_bytes + dlbuf_bytes / 2);
    dfree(dlbuf, dlbuf_bytes);
    dlbuf = nullptr;
    dlbuf_bytes = 0;
    if (allocated + want > budget) want = bytes;
    dlbuf = (char *)dalloc(want);
    dlbuf_bytes = want;
  }
  void ensure_h_dl(size_t bytes) {
    if (h_dl_bytes >= bytes) return;
    if (h_dl) cudaFreeHost(h_dl);
    h_dl = nullptr;
    const size_t grown = std::max(bytes, h_dl_bytes + h_dl_bytes / 2);
    h_dl_bytes = 0;
    CK(cudaHostAlloc(reinterpret_cast<void **>(&h_dl), grown, cudaHostAllocDefault));
    h_dl_bytes = grown;
  }
  void ensure_items(size_t n) {
    if (items_cap >= n) return;
    dfree(items, items_cap * sizeof(int4) + 16);
    items = nullptr;
    items_cap = 0;
    char *p = (char *)dalloc(n * sizeof(int4) + 16);
    items = (int4 *)p;
    n_items = (int32_t *)(p + n * sizeof(int4));
    items_cap = n;
  }
  DevParams params(const HostParams &hp) {
    const size_t need = hp.matrix.size();
    if (matrix_cap < need || !d_matrix) {
      dfree(d_matrix, matrix_cap * 4);
      d_matrix = nullptr;
      d_matrix = (int32_t *)dalloc(std::max<size_t>(need, 1) * 4);
      matrix_cap = std::max<size_t>(need, 1);
    }
    if (!d_encode) d_encode = (uint8_t *)dalloc(256);
    CK(cudaMemcpyAsync(d_matrix, hp.matrix.data(), need * 4, cudaMemcpyHostToDevice, stream));
    auto enc = encode_table(hp);
    CK(cudaMemcpyAsync(d_encode, enc.data(), 256, cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    return make_params(hp, d_matrix, d_encode);
  }
  static DevParams make_params(const HostParams &hp, const int32_t *m, const uint8_t *e) {
    DevParams P{};
    P.matrix = m;
    P.encode = e;
    P.sigma = int32_t(hp.alphabet.size());
    P.unknown = hp.encode('N');
    P.gap_open_raw = hp.gap_open;
    P.gap_ext = hp.gap_ext;
    P.gap_open = hp.gap_open + hp.gap_ext;
    P.adaptive = hp.adaptive ? 1 : 0;
    P.kernel = 0;
    P.seeding = hp.seeding ? 1 : 0;
    P.relaxed_order = 1;  // read loops finish with the exact LIFO order
    // static-band int32 rows: row at a time (0, the default: measured
    // fastest on the benchmark's mixed batch), as a wavefront where a read
    // suits it (MINIPOA_DP_ROWS=auto) or always (=wave)
    const char *rows_env = std::getenv("MINIPOA_DP_ROWS");
    P.row_wave = 0;
    if (rows_env && std::strcmp(rows_env, "auto") == 0) P.row_wave = 1;
    if (rows_env && std::strcmp(rows_env, "wave") == 0) P.row_wave = 2;
    // batched kernel form: bands up to 2048 columns as striped segments
    // (MINIPOA_WIDE_ROWS=1, or by default with the full matrix, f = 0, whose
    // bands are not bounded by the read length) or the form that keeps
    // rows above 512 columns on the generic row (=0)
    const char *wide_env = std::getenv("MINIPOA_WIDE_ROWS");
    P.wide_rows = hp.f == 0 ? 1 : 0;
    if (wide_env && std::strcmp(wide_env, "1") == 0) P.wide_rows = 1;
    if (wide_env && std::strcmp(wide_env, "0") == 0) P.wide_rows = 0;
    P.byte_prof = P.sigma <= 8 ? 1 : 0;
    for (int32_t v : hp.matrix)
      if (v < -128 || v > 127) P.byte_prof = 0;
    P.b = hp.b;
    P.f = hp.f;
    P.largest = hp.largest();
    return P;
  }
};

struct poa_graph {
  poa_ctx *ctx = nullptr;
  int sigma = 0, unknown = 0;
  Caps caps;
  char *storage = nullptr;
  size_t bytes = 0;
  Job *d_job = nullptr;
  Job h{};
  int64_t ub_nodes = 0, ub_chunks = 0, ub_path_used = 0, ub_paths = 0;

  ~poa_graph() {
    if (ctx) {
      ctx->dfree(storage, bytes);
      ctx->dfree(d_job, sizeof(Job));
    }
  }
  void sync() {
    CK(cudaMemcpyAsync(&h, d_job, sizeof(Job), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ub_nodes = h.n_nodes;
    ub_chunks = h.n_chunks;
    ub_path_used = h.path_used;
    ub_paths = h.n_paths;
  }
  void upload() {
    CK(cudaMemcpyAsync(d_job, &h, sizeof(Job), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  // Ensures room for a step that adds at most the given amounts.
  void reserve(int64_t nodes, int64_t chunks, int64_t path_items, int64_t paths) {
    if (ub_nodes + nodes <= caps.node_cap && ub_chunks + chunks <= caps.chunk_cap &&
        ub_path_used + path_items <= caps.path_cap && ub_paths + paths <= caps.max_paths) {
      ub_nodes += nodes;
      ub_chunks += chunks;
      ub_path_used += path_items;
      ub_paths += paths;
      return;
    }
    sync();
    Caps nc = caps;
    auto grow = [](int32_t cap, int64_t need) {
      int64_t c = cap;
      while (c < need) c = std::max<int64_t>(c * 2, 64);
      if (c > INT32_MAX / 2) c = INT32_MAX / 2;
      return int32_t(c);
    };
    nc.node_cap = grow(caps.node_cap, ub_nodes + nodes);
    nc.chunk_cap = grow(caps.chunk_cap, ub_chunks + chunks);
    nc.path_cap = grow(caps.path_cap, ub_path_used + path_items);
    nc.max_paths = grow(caps.max_paths, ub_paths + paths);
    if (nc.node_cap != caps.node_cap || nc.chunk_cap != caps.chunk_cap || nc.path_cap != caps.path_cap ||
        nc.max_paths != caps.max_paths) {
      Job nj = h;
      const size_t nbytes = layout(nc, nullptr, &nj);
      char *ns = (char *)ctx->dalloc(nbytes);
      layout(nc, ns, &nj);
      auto olda = arrays(h, caps);
      auto newa = arrays(nj, nc);
      for (size_t k = 0; k < olda.size(); ++k)
        CK(cudaMemcpyAsync(newa[k].first, olda[k].first, olda[k].second, cudaMemcpyDeviceToDevice, ctx->stream));
      nj.n_nodes = h.n_nodes;
      CK(cudaStreamSynchronize(ctx->stream));
      ctx->dfree(storage, bytes);
      storage = ns;
      bytes = nbytes;
      caps = nc;
      h = nj;
      upload();
    }
    ub_nodes += nodes;
    ub_chunks += chunks;
    ub_path_used += path_items;
    ub_paths += paths;
  }
  void check_status() {
    sync();
    if (h.status != ST_OK) {
      const int32_t st = h.status;
      h.status = ST_OK;
      upload();
      throw AlignError{status_code(st), status_message(st, h.err_i, h.err_j)};
    }
  }
  HostGraph download() {
    sync();
    const int64_t words = packed_words(h, sigma);
    // the context's download buffer (grown, never freed per call: a
    // cudaFree would synchronise the device on every download)
    // layout: per-block entry counts of the packing kernels, then the record
    constexpr size_t kRecAt = size_t(kPackOneMaxBlocks) * 16 + 256;
    ctx->ensure_dlbuf(size_t(words) * 4 + kRecAt);
    ctx->ensure_h_dl(size_t(words) * 4);
    int64_t *d_part = reinterpret_cast<int64_t *>(ctx->dlbuf);
    int32_t *d_out = reinterpret_cast<int32_t *>(ctx->dlbuf + kRecAt);
    CK(launch_pack_one(d_job, h.n_nodes, d_part, d_out, sigma, ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_dl, d_out, size_t(words) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return HostGraph::parse(ctx->h_dl);
  }
};

namespace {

poa_graph *new_graph(poa_ctx *ctx, const HostParams &hp, Caps caps) {
  auto g = std::make_unique<poa_graph>();
  g->ctx = ctx;
  g->sigma = int(hp.alphabet.size());
  g->unknown = hp.encode('N');
  caps.sigma = g->sigma;
  caps.node_cap = std::max(caps.node_cap, 64);
  caps.chunk_cap = std::max(caps.chunk_cap, 64);
  caps.path_cap = std::max(caps.path_cap, 64);
  caps.max_paths = std::max(caps.max_paths, 8);
  g->caps = caps;
  Job J{};
  g->bytes = layout(caps, nullptr, &J);
  g->storage = (char *)ctx->dalloc(g->bytes);
  layout(caps, g->storage, &J);
  g->d_job = (Job *)ctx->dalloc(sizeof(Job));
  g->h = J;
  g->upload();
  CK(launch_reset(g->d_job, 1, g->sigma, g->unknown, ctx->stream));
  g->sync();
  return g.release();
}

// Host images of a job's graph arrays for a host-built graph under `cc`,
// in the order of arrays(): edge lists as chunk chains in their insertion
// order. Ranks are written when `rank_of` / `order` are given (else 0).
struct GraphImage {
  std::vector<std::vector<char>> bufs;
  int32_t n_nodes = 0, n_chunks = 0, n_edges = 0, n_paths = 0, path_used = 0, n_rank = 0;
};

int64_t build_chunks(const BuildGraph &bg) {
  int64_t chunks = 0;
  for (int64_t i = 0; i < bg.n(); ++i)
    chunks += (int64_t(bg.in_id[size_t(i)].size()) + CHUNK - 1) / CHUNK +
              (int64_t(bg.out_id[size_t(i)].size()) + CHUNK - 1) / CHUNK;
  return chunks;
}

int64_t build_path_items(const BuildGraph &bg) {
  int64_t items = 0;
  for (auto &pth : bg.paths) items += int64_t(pth.size());
  return items;
}

GraphImage graph_image(const BuildGraph &bg, const Caps &cc, const std::vector<int32_t> *rank_of,
                       const std::vector<int32_t> *order) {
  const int64_t n = bg.n();
  const int sg = cc.sigma;
  const size_t N = size_t(cc.node_cap);
  std::vector<uint8_t> base(N, 0);
  std::vector<int32_t> parent(N, 0), rank(N, 0), cov(N, 0), ih(N, -1), it(N, -1), ic(N, 0), oh(N, -1), ot(N, -1),
      oc(N, 0), r2n(N, 0), al(N * size_t(sg), -1);
  std::vector<int32_t> cid(size_t(cc.chunk_cap) * CHUNK, 0), cw(size_t(cc.chunk_cap) * CHUNK, 0),
      cnext(size_t(cc.chunk_cap), -1);
  std::vector<int32_t> pit(size_t(cc.path_cap) + 1, 0), poff(size_t(cc.max_paths) + 1, 0),
      pseq(size_t(cc.max_paths) + 1, 0);
  int32_t nch = 0;
  auto put_list = [&](const std::vector<int32_t> &ids, const std::vector<int32_t> &ws, int32_t &head, int32_t &tail,
                      int32_t &cnt) {
    cnt = int32_t(ids.size());
    int32_t prev = -1;
    for (size_t k = 0; k < ids.size(); ++k) {
      if (k % CHUNK == 0) {
        const int32_t ch = nch++;
        if (prev < 0)
          head = ch;
        else
          cnext[size_t(prev)] = ch;
        prev = ch;
        tail = ch;
      }
      cid[size_t(prev) * CHUNK + k % CHUNK] = ids[k];
      cw[size_t(prev) * CHUNK + k % CHUNK] = ws[k];
    }
  };
  for (int64_t i = 0; i < n; ++i) {
    const size_t u = size_t(i);
    base[u] = uint8_t(bg.base[u]);
    parent[u] = bg.parent[u];
    cov[u] = bg.coverage[u];
    for (int k = 0; k < sg; ++k) al[u * size_t(sg) + size_t(k)] = bg.aligned[u * size_t(sg) + size_t(k)];
    put_list(bg.in_id[u], bg.in_w[u], ih[u], it[u], ic[u]);
    put_list(bg.out_id[u], bg.out_w[u], oh[u], ot[u], oc[u]);
    if (rank_of) rank[u] = (*rank_of)[u];
  }
  if (order)
    for (size_t r = 0; r < order->size(); ++r) r2n[r] = (*order)[r];
  int32_t used = 0;
  for (size_t k = 0; k < bg.paths.size(); ++k) {
    poff[k] = used;
    pseq[k] = bg.path_seq[k];
    for (int32_t id : bg.paths[k]) pit[size_t(used++)] = id;
  }
  poff[bg.paths.size()] = used;
  GraphImage img;
  auto add = [&](const void *p, size_t bytes) {
    img.bufs.emplace_back(reinterpret_cast<const char *>(p), reinterpret_cast<const char *>(p) + bytes);
  };
  add(base.data(), N);
  for (auto *v : {&parent, &rank, &cov, &ih, &it, &ic, &oh, &ot, &oc, &r2n}) add(v->data(), N * 4);
  add(al.data(), al.size() * 4);
  add(cid.data(), cid.size() * 4);
  add(cw.data(), cw.size() * 4);
  add(cnext.data(), cnext.size() * 4);
  add(pit.data(), size_t(cc.path_cap) * 4 + 4);
  add(poff.data(), size_t(cc.max_paths + 1) * 4);
  add(pseq.data(), size_t(cc.max_paths) * 4 + 4);
  img.n_nodes = int32_t(n);
  img.n_chunks = nch;
  img.n_edges = int32_t(bg.edges());
  img.n_paths = int32_t(bg.paths.size());
  img.path_used = used;
  img.n_rank = order ? int32_t(order->size()) : 0;
  return img;
}

// Copies a graph image into a laid-out job's arrays and sets its counts.
void put_image(const GraphImage &img, const Caps &cc, Job &J, cudaStream_t stream) {
  const auto dst = arrays(J, cc);
  for (size_t k = 0; k < dst.size(); ++k)
    CK(cudaMemcpyAsync(dst[k].first, img.bufs[k].data(), std::min(dst[k].second, img.bufs[k].size()),
                       cudaMemcpyHostToDevice, stream));
  J.n_nodes = img.n_nodes;
  J.n_chunks = img.n_chunks;
  J.n_edges = img.n_edges;
  J.n_paths = img.n_paths;
  J.path_used = img.path_used;
  J.n_rank = img.n_rank;
}

// A device graph from a host-built one (GFA input), ranked by the device's
// LIFO toposort (which rejects cycles). Room is left for `reserve` more
// nodes; the graph grows on demand when reads extend it.
poa_graph *import_graph(poa_ctx *ctx, const HostParams &hp, const BuildGraph &bg, int64_t reserve) {
  const int64_t n = bg.n(), chunks = build_chunks(bg), items = build_path_items(bg);
  if (n + reserve > INT32_MAX / 4 || 2 * chunks + reserve > INT32_MAX / 4)
    throw AlignError{POA_ERR_INVALID, "graph is too large"};
  Caps c;
  c.node_cap = int32_t(n + reserve + 8);
  c.chunk_cap = int32_t(chunks + 2 * reserve + 16);
  c.path_cap = int32_t(items + reserve + 8);
  c.max_paths = int32_t(bg.paths.size() + 8);
  std::unique_ptr<poa_graph> g(new_graph(ctx, hp, c));
  const GraphImage img = graph_image(bg, g->caps, nullptr, nullptr);
  put_image(img, g->caps, g->h, ctx->stream);
  g->h.status = ST_OK;
  g->upload();  // synchronises: the image is copied before it goes out of scope
  g->sync();
  ctx->ensure_arena(std::max<int64_t>(int64_t(g->h.n_nodes) * 8 + 64, int64_t(1) << 20));
  CK(launch_toposort(g->d_job, ctx->arena, ctx->arena_bytes, ctx->stream));
  g->check_status();
  return g.release();
}

template <class F>
int api(poa_ctx *ctx, F &&f) {
  (void)ctx;
  try {
    f();
    t_last_error.clear();
    return POA_OK;
  } catch (const AlignError &e) {
    t_last_error = e.msg;
    return e.code;
  } catch (const CudaError &e) {
    // a non-sticky error stays the runtime's "last error" until read; clear
    // it so the next call's launch check does not report it again
    cudaGetLastError();
    t_last_error = std::string(cudaGetErrorString(e.code)) + " (" + e.where + ")";
    return POA_ERR_CUDA;
  } catch (const std::bad_alloc &) {
    t_last_error = "host allocation failed";
    return POA_ERR_ALLOC;
  }
}

HostParams checked_params(const poa_params *p) {
  if (!p) throw AlignError{POA_ERR_INVALID, "null params"};
  HostParams hp = HostParams::from(p);
  std::string v = hp.validate();
  if (!v.empty()) throw AlignError{POA_ERR_INVALID, v};
  return hp;
}

// Runs the single-graph read loop reads[r0..r1) with arena growth on demand.
void extend_range(poa_ctx *ctx, const HostParams &hp, poa_graph *g, const std::vector<const uint8_t *> &seqs_in,
                  const std::vector<int64_t> &lens_in, int64_t r0) {
  const int64_t n = int64_t(seqs_in.size());
  if (r0 >= n) return;
  // progressive (-p, src/lib.rs:190-194): the reads go in guide order and
  // keep their own sequence ids
  std::vector<int64_t> order;
  if (hp.progressive && r0 == 0) order = guide_order(hp, seqs_in, lens_in);
  const bool ordered = !order.empty();
  std::vector<const uint8_t *> seqs(seqs_in);
  std::vector<int64_t> lens(lens_in);
  if (ordered)
    for (int64_t k = 0; k < n; ++k) {
      seqs[size_t(k)] = seqs_in[size_t(order[size_t(k)])];
      lens[size_t(k)] = lens_in[size_t(order[size_t(k)])];
    }
  int64_t total = 0, maxlen = 0;
  for (int64_t r = r0; r < n; ++r) {
    if (lens[r] > INT32_MAX / 4) throw AlignError{POA_ERR_INVALID, "sequence is too long"};
    total += lens[r];
    maxlen = std::max(maxlen, lens[r]);
  }
  g->reserve(total + 2 * (n - r0), 2 * (total + 3 * (n - r0)), total + (n - r0), n - r0);
  DevParams P = ctx->params(hp);
  // scheduler words of the one-job launch, then reads, offsets, lengths and
  // sequence ids, in one upload
  const size_t sched_bytes = ((4 + sched_words(1)) * 4 + 255) / 256 * 256;
  const size_t off_bytes = size_t(n) * 8, len_bytes = size_t(n) * 4, id_bytes = size_t(n) * 4;
  const size_t need = sched_bytes + off_bytes + len_bytes + id_bytes + size_t(std::max<int64_t>(total, 1)) + 64;
  ctx->ensure_qbuf(need);
  std::vector<uint8_t> host(need);
  int64_t *off = (int64_t *)(host.data() + sched_bytes);
  int32_t *ln = (int32_t *)(host.data() + sched_bytes + off_bytes);
  int32_t *ids = (int32_t *)(host.data() + sched_bytes + off_bytes + len_bytes);
  uint8_t *rd = host.data() + sched_bytes + off_bytes + len_bytes + id_bytes;
  int64_t at = 0;
  for (int64_t r = 0; r < n; ++r) {
    off[r] = at;
    ln[r] = int32_t(r >= r0 ? lens[r] : 0);
    ids[r] = int32_t(ordered ? order[size_t(r)] : r);
    if (r >= r0 && lens[r] > 0) std::memcpy(rd + at, seqs[r], size_t(lens[r]));
    if (r >= r0) at += lens[r];
  }
  CK(cudaMemcpyAsync(ctx->qbuf, host.data(), need, cudaMemcpyHostToDevice, ctx->stream));
  int32_t *d_sched = (int32_t *)ctx->qbuf;
  const int64_t *d_off = (const int64_t *)(ctx->qbuf + sched_bytes);
  const int32_t *d_len = (const int32_t *)(ctx->qbuf + sched_bytes + off_bytes);
  const int32_t *d_ids = (const int32_t *)(ctx->qbuf + sched_bytes + off_bytes + len_bytes);
  const uint8_t *d_rd = ctx->qbuf + sched_bytes + off_bytes + len_bytes + id_bytes;
  // The batched kernel runs the read loop as one job in a 4-warp block, the
  // job marked giant so the other three warps compute its DP rows with it;
  // the device advances next_read after each completed read. The job's
  // descriptor names its reads and its arena for the launch.
  g->sync();
  g->h.reads = d_rd;
  g->h.read_off = d_off;
  g->h.read_len = d_len;
  g->h.n_reads = int32_t(n);
  g->h.next_read = int32_t(r0);
  g->h.read_id = ordered ? d_ids : nullptr;
  g->h.giant = 1;
  g->h.done_flag = nullptr;
  // initial arena: scratch + a static-band estimate, grown on ARENA_FULL
  int64_t arena = std::max<int64_t>(int64_t(64) << 20, ctx->arena_bytes);
  auto detach = [&] {  // the descriptor as the other single-graph calls expect it
    g->h.status = ST_OK;
    g->h.arena = nullptr;
    g->h.arena_bytes = 0;
    g->h.read_id = nullptr;
    g->h.giant = 0;
    g->upload();
  };
  for (;;) {
    ctx->ensure_arena(arena);
    g->h.arena = ctx->arena;
    g->h.arena_bytes = ctx->arena_bytes;
    g->h.status = ST_OK;
    g->upload();
    CK(cudaMemsetAsync(d_sched, 0, sched_bytes, ctx->stream));
    CK(launch_single(g->d_job, d_sched, ctx->sm_count, P, ctx->stream));
    g->sync();
    const int32_t st = g->h.status;
    if (st == ST_OK) break;
    if (st == ST_ARENA_FULL) {
      if (arena >= int64_t(ctx->budget)) {
        detach();
        throw AlignError{POA_ERR_ALLOC, "DP arena exceeds the memory budget"};
      }
      arena = std::min<int64_t>(arena * 2, int64_t(ctx->budget - std::min(ctx->budget, ctx->allocated)) +
                                               ctx->arena_bytes);
      continue;
    }
    detach();
    throw AlignError{status_code(st), status_message(st, g->h.err_i, g->h.err_j)};
  }
  detach();
}

// align / poa on a graph without changing it.
std::vector<poa_aligned_base> align_path(poa_ctx *ctx, const HostParams &hp, poa_graph *g, const uint8_t *q,
                                         int64_t len, int mode, int64_t beg, int64_t end, int adaptive,
                                         uint64_t band_b, int kernel, int retry) {
  if (len < 0 || len > INT32_MAX / 4) throw AlignError{POA_ERR_INVALID, "sequence is too long"};
  DevParams P = ctx->params(hp);
  P.kernel = kernel;
  ctx->ensure_qbuf(size_t(len) + 16);
  if (len) CK(cudaMemcpyAsync(ctx->qbuf, q, size_t(len), cudaMemcpyHostToDevice, ctx->stream));
  ctx->ensure_items(size_t(len) + 4);
  g->sync();
  if (beg < 0 || end < 0 || beg >= g->h.n_nodes || end >= g->h.n_nodes) {
    if (mode == 1) throw AlignError{POA_ERR_ALIGN, "alignment anchor is not in graph"};
  }
  int64_t arena = std::max<int64_t>(int64_t(64) << 20, ctx->arena_bytes);
  for (;;) {
    ctx->ensure_arena(arena);
    CK(launch_align(g->d_job, P, ctx->arena, ctx->arena_bytes, ctx->qbuf, int(len), mode, int(beg), int(end),
                    adaptive, band_b, retry, ctx->items, ctx->n_items, ctx->stream));
    g->sync();
    const int32_t st = g->h.status;
    if (st == ST_OK) break;
    g->h.status = ST_OK;
    g->upload();
    if (st == ST_ARENA_FULL) {
      if (arena >= int64_t(ctx->budget)) throw AlignError{POA_ERR_ALLOC, "DP arena exceeds the memory budget"};
      arena *= 2;
      continue;
    }
    throw AlignError{status_code(st), status_message(st, g->h.err_i, g->h.err_j)};
  }
  int32_t n = 0;
  CK(cudaMemcpyAsync(&n, ctx->n_items, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  std::vector<int4> it(size_t(std::max(n, 0)));
  if (n > 0) CK(cudaMemcpyAsync(it.data(), ctx->items, size_t(n) * sizeof(int4), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  std::vector<poa_aligned_base> out(it.size());
  for (size_t k = 0; k < it.size(); ++k) out[k] = {it[k].x, it[k].y, it[k].z};
  return out;
}

// align::align with seeding (src/align.rs:99-164): the graph's consensus, the
// seed windows of the query against it (host), then one banded alignment per
// window between its anchor nodes (device) and the anchor nodes themselves,
// in window order. Anchors that are not usable as hard constraints, or no
// anchors at all, fall back to the whole graph with an adaptive band.
#ifdef POA_SEED_PROFILE
// profiling builds: host seconds of the seeded read loop's parts, printed
// when the process exits
struct SeedProfile {
  double download = 0, pack = 0, windows = 0, device = 0, fusion = 0;
  ~SeedProfile() {
    std::fprintf(stderr, "seed profile: download+order %.3f s (of it download %.3f s), consensus+windows %.3f s, "
                 "window DP %.3f s, add_path %.3f s\n", download, pack, windows, device, fusion);
  }
} g_seed_prof;
#define SEED_T(name) const double name = now_steady()
#define SEED_ADD(field, a, b) g_seed_prof.field += (b) - (a)
#else
#define SEED_T(name) (void)0
#define SEED_ADD(field, a, b) (void)0
#endif

std::vector<poa_aligned_base> seeded_align(poa_ctx *ctx, const HostParams &hp, poa_graph *g, const uint8_t *q,
                                           int64_t len, bool ranks_stale = false) {
  SEED_T(t0);
  g->sync();
  std::vector<poa_aligned_base> out;
  if (g->h.n_nodes <= 2) {
    out.push_back({0, hp.encode('N'), -1});
    for (int64_t c = 0; c < len; ++c) out.push_back({-1, hp.encode(q[c]), -1});
    return out;
  }
  SEED_T(tp0);
  HostGraph hg = g->download();
  SEED_T(tp1);
  SEED_ADD(pack, tp0, tp1);
  if (ranks_stale) {
    // the previous read's toposort (graph.rs:125-178), on the downloaded copy
    const int32_t st = hg.lifo_order();
    if (st != ST_OK) throw AlignError{status_code(st), status_message(st, 0, 0)};
    const size_t n = size_t(hg.n);
    CK(cudaMemcpyAsync(g->h.rank, hg.rank.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(g->h.rank_to_node, hg.rank_to_node.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream));
    g->sync();
    g->h.n_rank = hg.n_rank;
    g->h.order_exact = 1;
    g->upload();
  }
  SEED_T(t1);
  SEED_ADD(download, t0, t1);
  std::vector<uint8_t> cons;
  std::vector<int64_t> ids, cov;
  hg.consensus(hp, cons, ids, cov);
  const auto aw = anchor_windows(hp, q, len, cons.data(), int64_t(cons.size()));
  SEED_T(t2);
  SEED_ADD(windows, t1, t2);
  auto whole = [&] {
    ++ctx->seed_fallbacks;
    ++ctx->seed_launches;
    return align_path(ctx, hp, g, q, len, 1, 0, 1, 1, hp.b, 0, 1);
  };
  if (aw.first.empty()) return whole();
  struct Window {
    int64_t beg, end, qbeg, qend;
    bool adaptive;
    int64_t a0, a1;  // anchor node ids: ids[a0..a1)
  };
  std::vector<Window> windows;
  int64_t beg = 0, qbeg = 0, prev_t = -1;
  for (const Anchor &a : aw.first) {
    if (a.target_end + 1 < a.span) throw AlignError{POA_ERR_ALIGN, "invalid minimizer target span"};
    if (a.query_end + 1 < a.span) throw AlignError{POA_ERR_ALIGN, "invalid minimizer query span"};
    const int64_t ts = a.target_end + 1 - a.span, qs = a.query_end + 1 - a.span;
    bool valid = a.span > 0 && a.target_end < int64_t(ids.size()) && a.query_end < len && qs >= qbeg &&
                 (prev_t < 0 || ts > prev_t);
    for (int64_t o = 0; valid && o < a.span; ++o)
      valid = hp.encode(cons[size_t(ts + o)]) == hp.encode(q[qs + o]);
    if (!valid) return whole();
    windows.push_back({beg, ids[size_t(ts)], qbeg, qs, a.adaptive_before, ts, a.target_end});
    beg = ids[size_t(a.target_end)];
    qbeg = a.query_end + 1;
    prev_t = a.target_end;
  }
  windows.push_back({beg, 1, qbeg, len, aw.second, 0, 0});
  const int nw = int(windows.size());
  ctx->seed_windows += uint64_t(nw);
  std::vector<std::vector<poa_aligned_base>> parts(static_cast<size_t>(nw));
  std::vector<char> done(size_t(nw), 0);
  if (ctx->window_launch == 0 && nw > 1) {
    // all windows of the read in one launch, one warp each
    std::vector<int4> win(static_cast<size_t>(nw));
    std::vector<uint64_t> band(static_cast<size_t>(nw));
    std::vector<int64_t> item_off(size_t(nw) + 1, 0);
    for (int k = 0; k < nw; ++k) {
      const Window &w = windows[size_t(k)];
      const int64_t ql = w.qend - w.qbeg;
      win[size_t(k)] = make_int4(int(w.beg), int(w.end), int(w.qbeg), int(ql) | (w.adaptive ? int(0x80000000u) : 0));
      band[size_t(k)] = w.adaptive ? hp.b : hp.win_band;
      item_off[size_t(k) + 1] = item_off[size_t(k)] + ql + 8;
    }
    auto r256 = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t o_win = r256(size_t(len) + 16), o_band = o_win + r256(size_t(nw) * 16),
                 o_off = o_band + r256(size_t(nw) * 8), o_n = o_off + r256(size_t(nw + 1) * 8),
                 o_st = o_n + r256(size_t(nw) * 4), total = o_st + r256(size_t(nw) * 4);
    ctx->ensure_qbuf(total);
    ctx->ensure_items(size_t(item_off.back()) + 4);
    ctx->ensure_arena(std::max<int64_t>(ctx->arena_bytes, int64_t(nw) * (int64_t(32) << 20)));
    const int64_t slot = ctx->arena_bytes / nw / 256 * 256;
    uint8_t *qb = ctx->qbuf;
    if (len) CK(cudaMemcpyAsync(qb, q, size_t(len), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(qb + o_win, win.data(), size_t(nw) * 16, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(qb + o_band, band.data(), size_t(nw) * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(qb + o_off, item_off.data(), size_t(nw + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    const DevParams P = ctx->params(hp);
    ++ctx->seed_launches;
    CK(launch_windows(g->d_job, P, ctx->arena, slot, nw, reinterpret_cast<const int4 *>(qb + o_win),
                      reinterpret_cast<const uint64_t *>(qb + o_band), qb, ctx->items,
                      reinterpret_cast<const int64_t *>(qb + o_off), reinterpret_cast<int32_t *>(qb + o_n),
                      reinterpret_cast<int32_t *>(qb + o_st), ctx->stream));
    std::vector<int32_t> on(static_cast<size_t>(nw)), ost(static_cast<size_t>(nw));
    std::vector<int4> it(static_cast<size_t>(item_off.back()));
    CK(cudaMemcpyAsync(on.data(), qb + o_n, size_t(nw) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(ost.data(), qb + o_st, size_t(nw) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(it.data(), ctx->items, it.size() * sizeof(int4), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < nw; ++k) {
      const int32_t st = ost[size_t(k)];
      if (st == ST_ARENA_FULL) continue;  // aligned again below, with a growing arena
      if (st != ST_OK) {
        g->sync();
        throw AlignError{status_code(st), status_message(st, g->h.err_i, g->h.err_j)};
      }
      auto &pk = parts[size_t(k)];
      for (int32_t t = 0; t < on[size_t(k)]; ++t) {
        const int4 x = it[size_t(item_off[size_t(k)] + t)];
        pk.push_back({x.x, x.y, x.z});
      }
      done[size_t(k)] = 1;
    }
  }
  for (int k = 0; k < nw; ++k) {
    if (done[size_t(k)]) continue;
    const Window &w = windows[size_t(k)];
    ++ctx->seed_launches;
    parts[size_t(k)] = align_path(ctx, hp, g, q + w.qbeg, w.qend - w.qbeg, 1, w.beg, w.end, w.adaptive ? 1 : 0,
                                  w.adaptive ? hp.b : hp.win_band, 0, 1);
  }
  SEED_T(t3);
  SEED_ADD(device, t2, t3);
  for (int k = 0; k < nw; ++k) {
    const Window &w = windows[size_t(k)];
    out.insert(out.end(), parts[size_t(k)].begin(), parts[size_t(k)].end());
    for (int64_t t = w.a0; t < w.a1; ++t) out.push_back({ids[size_t(t)], hg.base[size_t(ids[size_t(t)])], -1});
  }
  return out;
}

// extend_graph (src/lib.rs:184-204) with seeding: per read, the seeded path,
// then add_path on the device; the LIFO toposort of each step runs on the
// host copy the next read downloads anyway (its consensus needs it), and on
// the device after the last read.
void seeded_extend(poa_ctx *ctx, const HostParams &hp, poa_graph *g, const std::vector<const uint8_t *> &seqs,
                   const std::vector<int64_t> &lens, int64_t r0) {
  const int64_t n = int64_t(seqs.size());
  // progressive (-p, src/lib.rs:190-194): reads in guide order, own ids
  std::vector<int64_t> order;
  if (hp.progressive && r0 == 0) order = guide_order(hp, seqs, lens);
  int64_t total = 0;
  for (int64_t r = r0; r < n; ++r) {
    if (lens[size_t(r)] > INT32_MAX / 4) throw AlignError{POA_ERR_INVALID, "sequence is too long"};
    total += lens[size_t(r)];
  }
  g->reserve(total + 2 * (n - r0), 2 * (total + 3 * (n - r0)), total + (n - r0), n - r0);
  const DevParams P = ctx->params(hp);
  bool stale = false;
  for (int64_t k = r0; k < n; ++k) {
    const int64_t r = order.empty() ? k : order[size_t(k)];
    auto path = seeded_align(ctx, hp, g, seqs[size_t(r)], lens[size_t(r)], stale);
    SEED_T(ta);
    std::vector<int4> it(path.size());
    for (size_t k = 0; k < path.size(); ++k)
      it[k] = make_int4(int(path[k].node), int(path[k].base), int(path[k].aligned), 0);
    ctx->ensure_items(it.size() + 4);
    if (!it.empty())
      CK(cudaMemcpyAsync(ctx->items, it.data(), it.size() * sizeof(int4), cudaMemcpyHostToDevice, ctx->stream));
    // scratch for add_path's node marks (n_nodes words)
    ctx->ensure_arena(std::max<int64_t>(int64_t(g->h.n_nodes) * 4 + 256, ctx->arena_bytes));
    CK(launch_add_path(g->d_job, P, int(r), ctx->items, int(it.size()), ctx->stream,
                       reinterpret_cast<int32_t *>(ctx->arena)));
    g->check_status();
    SEED_T(tb);
    SEED_ADD(fusion, ta, tb);
    stale = true;
  }
  if (stale) {
    ctx->ensure_arena(std::max<int64_t>(int64_t(g->h.n_nodes) * 8 + 64, int64_t(64) << 20));
    CK(launch_toposort(g->d_job, ctx->arena, ctx->arena_bytes, ctx->stream));
    g->check_status();
  }
}

std::vector<std::string> name_list(int64_t n, const char *const *names, const char *prefix) {
  std::vector<std::string> v(size_t(std::max<int64_t>(n, 0)));
  for (int64_t i = 0; i < n; ++i) v[size_t(i)] = names ? std::string(names[i]) : std::string(prefix) + std::to_string(i);
  return v;
}

}  // namespace

// ---------------------------------------------------------------------------
// Batch of independent read sets.

// Resident warps per SM of a batched run without a tuned setting: 5 of the
// kernel's 8 (the largest sets, which end the run, slow down when their SM
// also runs other jobs; the tuner picked 5 in most C3 runs, 3.16-3.21 s per
// step, against 3.5-3.65 s at 6 and 4.0-4.2 s at 8).
constexpr int kDefaultBatchWarpsPerSm = 5;

struct poa_batch {
  poa_ctx *ctx = nullptr;
  HostParams hp;
  DevParams P{};
  int64_t n_sets = 0;
  std::vector<int64_t> set_off;
  std::vector<int64_t> lens;
  int sigma = 0, unknown = 0;
  uint8_t *d_reads = nullptr;
  int64_t *d_read_off = nullptr;
  int32_t *d_read_len = nullptr;
  size_t reads_bytes = 0;
  int32_t *d_matrix = nullptr;
  uint8_t *d_encode = nullptr;
  char *storage = nullptr;
  size_t storage_bytes = 0;
  std::vector<Job> jobs;
  std::vector<Caps> caps;
  Job *d_jobs = nullptr;
  std::vector<int32_t> order;
  int32_t *d_order = nullptr;  // the pass's job order, then (at base_order()) the first pass's
  int32_t *d_queue = nullptr;
  char *arenas = nullptr;
  int64_t arena_pool = 0;
  int warps_per_sm = 0;
  uint64_t slot_bytes_override = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr, k0 = nullptr, k1 = nullptr;
  bool ran = false;
  uint64_t h2d_bytes = 0, d2h_bytes = 0;
  std::vector<double> est;     // estimated work per set (size order, giants, tuning bucket)
  double giant_factor = 1.5;   // giant: estimated work above this many per-warp shares
  int giant_alone = 0;         // a giant's SM runs only its team (see DevParams::giant_alone)
  std::string tune_key;        // autotuner cache key of the batch's size bucket
  // the first pass of a batched run (reset, queue set-up, persistent kernel)
  // captured once as a CUDA graph and replayed while its launch shape holds
  cudaGraphExec_t gexec = nullptr;
  int64_t g_slots = -1, g_slot_bytes = -1;
  int g_alone = -1;
  int g_team = -1;
  int graph_launches = 0;

  // d_order holds two orders: the running pass's, and at base_order() the
  // size order of the first pass, uploaded once so the captured first pass
  // copies it on the device
  size_t order_half() const { return (order.size() + 4) / 4 * 4; }
  size_t order_bytes() const { return 2 * order_half() * 4; }
  int32_t *base_order() const { return d_order + order_half(); }

  // Frees the DP arena pool (and the captured run that points into it).
  void drop_arenas() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
    g_slots = g_slot_bytes = -1;
    if (ctx) ctx->dfree(arenas, size_t(arena_pool));
    arenas = nullptr;
    arena_pool = 0;
  }

  ~poa_batch() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (!ctx) return;
    ctx->batches.erase(std::remove(ctx->batches.begin(), ctx->batches.end(), this), ctx->batches.end());
    ctx->dfree(d_read_off, reads_bytes);  // base of the reads allocation
    ctx->dfree(d_matrix, 0);
    ctx->dfree(d_encode, 0);
    ctx->dfree(storage, storage_bytes);
    ctx->dfree(d_jobs, jobs.size() * sizeof(Job));
    ctx->dfree(d_order, order_bytes());
    ctx->dfree(d_queue, sched_words(jobs.size()) * 4);
    ctx->dfree(arenas, size_t(arena_pool));
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (k0) cudaEventDestroy(k0);
    if (k1) cudaEventDestroy(k1);
  }

  // Giant jobs: well above the per-warp share of the whole batch, at most
  // one per SM (the largest ones, which start first, one per SM); none when
  // giant_factor is 0.
  void mark_giants() {
    const double share = std::accumulate(est.begin(), est.end(), 0.0) /
                         double(std::max(1, ctx->sm_count * batch_resident_warps_per_sm()));
    for (auto &J : jobs) J.giant = 0;
    if (giant_factor <= 0) return;
    for (int64_t k = 0; k < std::min<int64_t>(n_sets, ctx->sm_count); ++k) {
      const int32_t s = order[size_t(k)];
      jobs[size_t(s)].giant = est[size_t(s)] > giant_factor * share ? 1 : 0;
    }
  }

  void download_jobs() {
    CK(cudaMemcpyAsync(jobs.data(), d_jobs, jobs.size() * sizeof(Job), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  void upload_jobs() {
    CK(cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(Job), cudaMemcpyHostToDevice, ctx->stream));
  }

  // Consensus FASTA of every set, computed on the device (poa_consensus.cu):
  // only the consensus bases leave the GPU. A failed set gets its error line.
  std::vector<std::string> device_consensus() {
    download_jobs();
    const size_t nj = jobs.size();
    std::vector<int64_t> scr(nj + 1, 0), oo(nj + 1, 0);
    for (size_t s = 0; s < nj; ++s) {
      scr[s + 1] = scr[s] + consensus_scratch_bytes(jobs[s].n_nodes, jobs[s].n_edges);
      oo[s + 1] = oo[s] + (int64_t(jobs[s].n_nodes) + 15) / 16 * 16;
    }
    const size_t scr_bytes = size_t(scr.back()), out_bytes = size_t(oo.back());
    std::vector<uint8_t> dec(256, 'N');
    for (int c = 0; c < sigma; ++c) dec[size_t(c)] = hp.decode(c);
    // scratch: the DP arena pool when it holds it, else its own allocation
    const bool own = !(arenas && arena_pool >= int64_t(scr_bytes));
    char *d_scr = own ? (char *)ctx->dalloc(scr_bytes + 16) : arenas;
    uint8_t *d_out = nullptr, *d_dec = nullptr;
    int64_t *d_so = nullptr, *d_oo = nullptr;
    int32_t *d_len = nullptr;
    std::vector<int32_t> len(nj);
    std::vector<uint8_t> bytes(out_bytes + 1);
    auto release = [&] {
      if (own) ctx->dfree(d_scr, scr_bytes + 16);
      ctx->dfree(d_out, out_bytes + 16);
      ctx->dfree(d_dec, 256);
      ctx->dfree(d_so, (nj + 1) * 8);
      ctx->dfree(d_oo, (nj + 1) * 8);
      ctx->dfree(d_len, nj * 4 + 4);
    };
    try {
      d_out = (uint8_t *)ctx->dalloc(out_bytes + 16);
      d_dec = (uint8_t *)ctx->dalloc(256);
      d_so = (int64_t *)ctx->dalloc((nj + 1) * 8);
      d_oo = (int64_t *)ctx->dalloc((nj + 1) * 8);
      d_len = (int32_t *)ctx->dalloc(nj * 4 + 4);
      CK(cudaMemcpyAsync(d_dec, dec.data(), 256, cudaMemcpyHostToDevice, ctx->stream));
      CK(cudaMemcpyAsync(d_so, scr.data(), (nj + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
      CK(cudaMemcpyAsync(d_oo, oo.data(), (nj + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
      CK(launch_consensus(d_jobs, int(nj), d_dec, d_scr, d_so, d_out, d_oo, d_len, ctx->stream));
      CK(cudaMemcpyAsync(len.data(), d_len, nj * 4, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaMemcpyAsync(bytes.data(), d_out, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      d2h_bytes = out_bytes + nj * 4 + jobs.size() * sizeof(Job);
    } catch (...) {
      release();
      throw;
    }
    release();
    std::vector<std::string> parts(nj);
    for (size_t s = 0; s < nj; ++s) {
      const Job &J = jobs[s];
      if (J.status != ST_OK || len[s] < 0) {
        parts[s] = "!error " + status_message(J.status, J.err_i, J.err_j) + "\n";
        continue;
      }
      const char *b0 = reinterpret_cast<const char *>(bytes.data() + oo[s]);
      parts[s] = ">consensus sequence\n" + std::string(b0, b0 + len[s]) + "\n";
    }
    return parts;
  }

  // Packs the graphs of `ids` and parses them on the host.
  std::vector<HostGraph> graphs(const std::vector<int32_t> &ids) {
    download_jobs();
    std::vector<int64_t> off(ids.size() + 1, 0);
    for (size_t k = 0; k < ids.size(); ++k) off[k + 1] = off[k] + packed_words(jobs[size_t(ids[k])], sigma);
    const size_t words = size_t(off.back());
    // The DP arena pool takes what the budget leaves after a run; when the
    // packed graphs do not fit beside it, the pool is released (the next run
    // allocates it again).
    const uint64_t need = words * 4 + 16 + off.size() * 8 + ids.size() * 4 + 4 + 3 * 256;
    if (arenas && ctx->allocated + need > ctx->budget) {
      ctx->dfree(arenas, size_t(arena_pool));
      arenas = nullptr;
      arena_pool = 0;
    }
    int32_t *d_out = (int32_t *)ctx->dalloc(words * 4 + 16);
    int64_t *d_off = (int64_t *)ctx->dalloc(off.size() * 8);
    int32_t *d_ids = (int32_t *)ctx->dalloc(ids.size() * 4 + 4);
    std::vector<int32_t> rec(words + 1);
    auto release = [&] {
      ctx->dfree(d_out, words * 4 + 16);
      ctx->dfree(d_off, off.size() * 8);
      ctx->dfree(d_ids, ids.size() * 4 + 4);
    };
    try {
      CK(cudaMemcpyAsync(d_off, off.data(), off.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
      CK(cudaMemcpyAsync(d_ids, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
      CK(launch_pack(d_jobs, d_ids, int(ids.size()), d_off, d_out, sigma, ctx->stream));
      CK(cudaMemcpyAsync(rec.data(), d_out, words * 4, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      d2h_bytes = words * 4 + jobs.size() * sizeof(Job);
    } catch (...) {
      release();
      throw;
    }
    release();
    std::vector<HostGraph> out(ids.size());
    const int nt = std::max(1, std::min<int>(int(std::thread::hardware_concurrency()), 32));
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
      pool.emplace_back([&, t] {
        for (size_t k = size_t(t); k < ids.size(); k += size_t(nt)) out[k] = HostGraph::parse(rec.data() + off[k]);
      });
    for (auto &th : pool) th.join();
    return out;
  }
};

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

const char *poa_dp_backend(void) { return "cuda-sm100a (warp-per-job, i32 / guarded i64)"; }

int poa_ctx_create(int device, uint64_t mem_budget, poa_ctx **out) {
  *out = nullptr;
  auto ctx = std::make_unique<poa_ctx>();
  int rc = api(ctx.get(), [&] {
    int count = 0;
    CK(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) throw AlignError{POA_ERR_CUDA, "no such CUDA device"};
    CK(cudaSetDevice(device));
    cudaDeviceProp prop{};
    CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) throw AlignError{POA_ERR_CUDA, "this build targets sm_100a (B200)"};
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    ctx->budget = mem_budget ? std::min<uint64_t>(mem_budget, free_b) : uint64_t(double(free_b) * 0.9);
  });
  if (rc != POA_OK) {
    g_create_error = t_last_error;
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    return rc;
  }
  *out = ctx.release();
  return POA_OK;
}

void poa_ctx_destroy(poa_ctx *ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->dfree(ctx->arena, size_t(ctx->arena_bytes));
  ctx->dfree(ctx->qbuf, ctx->qbuf_bytes);
  ctx->dfree(ctx->dlbuf, ctx->dlbuf_bytes);
  if (ctx->h_dl) cudaFreeHost(ctx->h_dl);
  ctx->dfree(ctx->items, 0);
  ctx->dfree(ctx->d_matrix, 0);
  ctx->dfree(ctx->d_encode, 0);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

// The calling thread's last error; with a null context, that of its last
// failed poa_ctx_create.
const char *poa_last_error(const poa_ctx *ctx) { return ctx ? t_last_error.c_str() : g_create_error.c_str(); }
void poa_free(void *ptr) { std::free(ptr); }

int poa_ctx_tune_windows(poa_ctx *ctx, int32_t one_launch_per_window) {
  if (!ctx || one_launch_per_window < 0 || one_launch_per_window > 1) return POA_ERR_INVALID;
  ctx->window_launch = one_launch_per_window;
  return POA_OK;
}

int poa_ctx_window_stats(poa_ctx *ctx, uint64_t *windows, uint64_t *launches, uint64_t *fallbacks) {
  if (!ctx || !windows || !launches || !fallbacks) return POA_ERR_INVALID;
  *windows = ctx->seed_windows;
  *launches = ctx->seed_launches;
  *fallbacks = ctx->seed_fallbacks;
  return POA_OK;
}

int poa_params_validate(poa_ctx *ctx, const poa_params *params) {
  return api(ctx, [&] { checked_params(params); });
}

int poa_graph_new(poa_ctx *ctx, const poa_params *params, poa_graph **out) {
  *out = nullptr;
  return api(ctx, [&] {
    HostParams hp = checked_params(params);
    *out = new_graph(ctx, hp, Caps{});
  });
}

void poa_graph_free(poa_graph *graph) { delete graph; }

int poa_graph_read_gfa(poa_ctx *ctx, const poa_params *params, const char *text, int64_t len, poa_graph **out,
                       char **records, int64_t *records_len) {
  *out = nullptr;
  *records = nullptr;
  *records_len = 0;
  return api(ctx, [&] {
    HostParams hp = checked_params(params);
    if (len < 0 || (len > 0 && !text)) throw AlignError{POA_ERR_INVALID, "invalid GFA text"};
    std::vector<GfaRecord> recs;
    BuildGraph bg = [&] {
      try {
        return read_gfa(hp, text, size_t(len), recs);
      } catch (const std::runtime_error &e) {
        throw AlignError{POA_ERR_ALIGN, e.what()};
      }
    }();
    std::unique_ptr<poa_graph> g(import_graph(ctx, hp, bg, 1024));
    std::string r;
    for (auto &x : recs) r += x.name + "\t" + x.seq + "\n";
    *records = dup_string(r);
    *records_len = int64_t(r.size());
    *out = g.release();
  });
}

int poa_align_sequences(poa_ctx *ctx, const poa_params *params, int64_t n_seqs, const uint8_t *const *seqs,
                        const int64_t *lens, poa_graph **out) {
  *out = nullptr;
  return api(ctx, [&] {
    HostParams hp = checked_params(params);
    int64_t total = 0;
    for (int64_t r = 0; r < n_seqs; ++r) total += lens[r];
    Caps c;
    c.node_cap = int32_t(std::min<int64_t>(total + 2 * n_seqs + 4, INT32_MAX / 2));
    c.chunk_cap = int32_t(std::min<int64_t>(2 * (total + 3 * n_seqs) + 8, INT32_MAX / 2));
    c.path_cap = int32_t(std::min<int64_t>(total + n_seqs + 1, INT32_MAX / 2));
    c.max_paths = int32_t(n_seqs + 1);
    std::unique_ptr<poa_graph> g(new_graph(ctx, hp, c));
    std::vector<const uint8_t *> s(seqs, seqs + n_seqs);
    std::vector<int64_t> l(lens, lens + n_seqs);
    if (hp.seeding)
      seeded_extend(ctx, hp, g.get(), s, l, 0);
    else
      extend_range(ctx, hp, g.get(), s, l, 0);
    *out = g.release();
  });
}

int poa_extend_graph(poa_ctx *ctx, const poa_params *params, poa_graph *graph, int64_t n_seqs,
                     const uint8_t *const *seqs, const int64_t *lens, int64_t existing) {
  return api(ctx, [&] {
    HostParams hp = checked_params(params);
    HostParams ap = hp;
    if (existing > 0) ap.progressive = false;
    std::vector<const uint8_t *> s(seqs, seqs + n_seqs);
    std::vector<int64_t> l(lens, lens + n_seqs);
    if (ap.seeding)
      seeded_extend(ctx, ap, graph, s, l, existing);
    else
      extend_range(ctx, ap, graph, s, l, existing);
  });
}

int poa_align(poa_ctx *ctx, const poa_params *params, poa_graph *graph, const uint8_t *query, int64_t len,
              poa_aligned_base **out, int64_t *out_len) {
  *out = nullptr;
  *out_len = 0;
  return api(ctx, [&] {
    HostParams hp = checked_params(params);
    if (!graph || graph->ctx != ctx) throw AlignError{POA_ERR_INVALID, "the graph belongs to another context"};
    if (len < 0 || len > INT32_MAX / 4) throw AlignError{POA_ERR_INVALID, "sequence is too long"};
    auto v = hp.seeding ? seeded_align(ctx, hp, graph, query, len)
                        : align_path(ctx, hp, graph, query, len, 0, 0, 1, 0, hp.b, 0, 1);
    *out = (poa_aligned_base *)std::malloc(sizeof(poa_aligned_base) * (v.size() + 1));
    std::memcpy(*out, v.data(), v.size() * sizeof(poa_aligned_base));
    *out_len = int64_t(v.size());
  });
}

int poa_poa(poa_ctx *ctx, const poa_params *params, poa_graph *graph, int64_t beg_id, int64_t end_id,
            const uint8_t *query, int64_t len, int32_t adaptive, uint64_t band_b, int32_t kernel, int32_t retry,
            poa_aligned_base **out, int64_t *out_len) {
  *out = nullptr;
  *out_len = 0;
  return api(ctx, [&] {
    HostParams hp = checked_params(params);
    if (kernel < 0 || kernel > 2) throw AlignError{POA_ERR_INVALID, "kernel must be 0, 1 or 2"};
    auto v = align_path(ctx, hp, graph, query, len, 1, beg_id, end_id, adaptive, band_b, kernel, retry);
    *out = (poa_aligned_base *)std::malloc(sizeof(poa_aligned_base) * (v.size() + 1));
    std::memcpy(*out, v.data(), v.size() * sizeof(poa_aligned_base));
    *out_len = int64_t(v.size());
  });
}

int poa_graph_add_path(poa_ctx *ctx, poa_graph *graph, int64_t seq_id, const poa_aligned_base *items, int64_t n) {
  return api(ctx, [&] {
    if (n < 0 || n > INT32_MAX / 4) throw AlignError{POA_ERR_INVALID, "alignment is too long"};
    std::vector<int4> it(static_cast<size_t>(n));
    for (int64_t k = 0; k < n; ++k) {
      auto clamp = [](int64_t v) { return int32_t(v < -1 ? INT32_MAX : (v > INT32_MAX ? INT32_MAX : v)); };
      it[size_t(k)] = make_int4(clamp(items[k].node), items[k].base < 0 ? -1 : clamp(items[k].base),
                                clamp(items[k].aligned), 0);
    }
    graph->reserve(n, 2 * (n + 1), n, 1);
    ctx->ensure_items(size_t(n) + 4);
    if (n) CK(cudaMemcpyAsync(ctx->items, it.data(), size_t(n) * sizeof(int4), cudaMemcpyHostToDevice, ctx->stream));
    DevParams P{};
    P.sigma = graph->sigma;
    CK(launch_add_path(graph->d_job, P, int(seq_id), ctx->items, int(n), ctx->stream));
    graph->check_status();
  });
}

int poa_graph_add_node(poa_ctx *ctx, poa_graph *graph, int64_t base, int64_t *out_id) {
  return api(ctx, [&] {
    if (base < 0 || base >= graph->sigma) throw AlignError{POA_ERR_INVALID, "alignment base outside alphabet"};
    graph->reserve(1, 0, 0, 0);
    CK(launch_add_node(graph->d_job, graph->sigma, int(base), ctx->stream));
    graph->check_status();
    *out_id = graph->h.err_i;
  });
}

int poa_graph_add_edge(poa_ctx *ctx, poa_graph *graph, int64_t from, int64_t to) {
  return api(ctx, [&] {
    graph->sync();
    if (from < 0 || to < 0 || from >= graph->h.n_nodes || to >= graph->h.n_nodes)
      throw AlignError{POA_ERR_INVALID, "edge references an unknown node"};
    graph->reserve(0, 2, 0, 0);
    CK(launch_add_edge(graph->d_job, int(from), int(to), ctx->stream));
    graph->check_status();
  });
}

int poa_graph_toposort(poa_ctx *ctx, poa_graph *graph, int32_t grouped) {
  return api(ctx, [&] {
    if (grouped) {
      // Column-grouped ranks are computed on the host graph and written back.
      HostGraph hg = graph->download();
      std::vector<int32_t> node_rank, order;
      std::string err;
      if (!hg.grouped_ranks(node_rank, order, err)) throw AlignError{POA_ERR_ALIGN, err};
      if (!node_rank.empty())
        CK(cudaMemcpyAsync(graph->h.rank, node_rank.data(), node_rank.size() * 4, cudaMemcpyHostToDevice,
                           ctx->stream));
      if (!order.empty())
        CK(cudaMemcpyAsync(graph->h.rank_to_node, order.data(), order.size() * 4, cudaMemcpyHostToDevice,
                           ctx->stream));
      graph->h.n_rank = int32_t(order.size());
      graph->upload();
      return;
    }
    graph->sync();
    ctx->ensure_arena(std::max<int64_t>(int64_t(graph->h.n_nodes) * 8 + 64, int64_t(1) << 20));
    CK(launch_toposort(graph->d_job, ctx->arena, ctx->arena_bytes, ctx->stream));
    graph->check_status();
  });
}

int poa_graph_consensus(poa_ctx *ctx, const poa_params *params, poa_graph *graph, uint8_t **seq, int64_t **ids,
                        int64_t **coverage, int64_t *len) {
  *seq = nullptr;
  *ids = *coverage = nullptr;
  *len = 0;
  return api(ctx, [&] {
    HostParams hp = checked_params(params);
    HostGraph hg = graph->download();
    std::vector<uint8_t> s;
    std::vector<int64_t> id, cv;
    hg.consensus(hp, s, id, cv);
    *seq = (uint8_t *)std::malloc(s.size() + 1);
    std::memcpy(*seq, s.data(), s.size());
    (*seq)[s.size()] = 0;
    *ids = (int64_t *)std::malloc(id.size() * 8 + 8);
    *coverage = (int64_t *)std::malloc(cv.size() * 8 + 8);
    std::memcpy(*ids, id.data(), id.size() * 8);
    std::memcpy(*coverage, cv.data(), cv.size() * 8);
    *len = int64_t(s.size());
  });
}

int poa_graph_msa(poa_ctx *ctx, const poa_params *params, poa_graph *graph, int64_t n, const char *const *names,
                  const char *const *comments, char **out, int64_t *out_len) {
  *out = nullptr;
  *out_len = 0;
  return api(ctx, [&] {
    HostParams hp = checked_params(params);
    HostGraph hg = graph->download();
    auto nm = name_list(n, names, "read");
    std::vector<std::string> cm(size_t(std::max<int64_t>(n, 0)));
    for (int64_t i = 0; i < n && comments; ++i) cm[size_t(i)] = comments[i];
    std::string s, err;
    if (!hg.msa(hp, nm, cm, s, err)) throw AlignError{POA_ERR_ALIGN, err};
    *out = dup_string(s);
    *out_len = int64_t(s.size());
  });
}

int poa_graph_gfa(poa_ctx *ctx, const poa_params *params, poa_graph *graph, int64_t n, const char *const *names,
                  char **out, int64_t *out_len) {
  *out = nullptr;
  *out_len = 0;
  return api(ctx, [&] {
    HostParams hp = checked_params(params);
    HostGraph hg = graph->download();
    auto nm = name_list(n, names, "read");
    std::string s, err;
    if (!hg.gfa(hp, nm, s, err)) throw AlignError{POA_ERR_ALIGN, err};
    *out = dup_string(s);
    *out_len = int64_t(s.size());
  });
}

int poa_graph_sizes_get(poa_ctx *ctx, poa_graph *graph, poa_graph_sizes *out) {
  return api(ctx, [&] {
    graph->sync();
    out->n_nodes = graph->h.n_nodes;
    out->n_edges = graph->h.n_edges;
    out->n_paths = graph->h.n_paths;
    out->path_items = graph->h.path_used;
    out->alphabet = graph->sigma;
    out->n_rank = graph->h.n_rank;
  });
}

int poa_graph_export(poa_ctx *ctx, poa_graph *graph, int64_t *fields, int64_t *rank, int64_t *aligned,
                     int64_t *in_cnt, int64_t *out_cnt, int64_t *in_pairs, int64_t *out_pairs, int64_t *path_seq,
                     int64_t *path_len, int64_t *path_ids) {
  return api(ctx, [&] {
    HostGraph g = graph->download();
    for (int i = 0; i < g.n; ++i) {
      fields[4 * i] = g.base[i];
      fields[4 * i + 1] = g.parent[i];
      fields[4 * i + 2] = g.rank[i];
      fields[4 * i + 3] = g.coverage[i];
      in_cnt[i] = g.in_off[i + 1] - g.in_off[i];
      out_cnt[i] = g.out_off[i + 1] - g.out_off[i];
    }
    for (int i = 0; i < g.n_rank; ++i) rank[i] = g.rank_to_node[i];
    for (int64_t k = 0; k < int64_t(g.aligned.size()); ++k) aligned[k] = g.aligned[size_t(k)];
    for (size_t k = 0; k < g.in_id.size(); ++k) {
      in_pairs[2 * k] = g.in_id[k];
      in_pairs[2 * k + 1] = g.in_w[k];
    }
    for (size_t k = 0; k < g.out_id.size(); ++k) {
      out_pairs[2 * k] = g.out_id[k];
      out_pairs[2 * k + 1] = g.out_w[k];
    }
    for (size_t p = 0; p < g.path_seq.size(); ++p) {
      path_seq[p] = g.path_seq[p];
      path_len[p] = g.path_off[p + 1] - g.path_off[p];
    }
    for (size_t k = 0; k < g.path_items.size(); ++k) path_ids[k] = g.path_items[k];
  });
}

// ---- batch

// ---- batch autotuner cache

// Tuned launch settings per device and batch size bucket: one line
// "key<TAB>warps_per_sm<TAB>giant_factor<TAB>giant_alone" per bucket in the file named by
// MINIPOA_B200_TUNE_CACHE (default ~/.cache/minipoa_b200/tune.tsv).
std::string tune_path() {
  if (const char *p = std::getenv("MINIPOA_B200_TUNE_CACHE")) return p;
  const char *home = std::getenv("HOME");
  return std::string(home ? home : ".") + "/.cache/minipoa_b200/tune.tsv";
}

int log2_bucket(double x) {
  int b = 0;
  while (x >= 2.0 && b < 62) {
    x /= 2.0;
    ++b;
  }
  return b;
}

// Size bucket of a batch: device name, log2 of the set count, of the
// longest read and of the mean depth.
std::string tune_key(poa_ctx *ctx, int64_t n_sets, const int64_t *set_off, const int64_t *lens) {
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, ctx->device);
  int64_t mx = 0;
  for (int64_t r = 0; r < set_off[n_sets]; ++r) mx = std::max(mx, lens[r]);
  const double depth = n_sets ? double(set_off[n_sets]) / double(n_sets) : 0.0;
  return std::string(prop.name) + "|sets" + std::to_string(log2_bucket(double(n_sets))) + "|len" +
         std::to_string(log2_bucket(double(mx))) + "|depth" + std::to_string(log2_bucket(depth));
}

std::mutex g_tune_mu;

bool tune_lookup(const std::string &key, int *warps_per_sm, double *giant_factor, int *giant_alone) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  std::ifstream f(tune_path());
  std::string line;
  bool found = false;
  while (std::getline(f, line)) {
    const size_t a = line.find('\t'), b = a == std::string::npos ? a : line.find('\t', a + 1);
    if (b == std::string::npos || line.substr(0, a) != key) continue;
    const size_t c = line.find('\t', b + 1);
    *warps_per_sm = std::atoi(line.substr(a + 1, b - a - 1).c_str());
    *giant_factor = std::atof(line.substr(b + 1, c == std::string::npos ? std::string::npos : c - b - 1).c_str());
    *giant_alone = c == std::string::npos ? 0 : std::atoi(line.substr(c + 1).c_str());
    found = true;  // the last entry for a key wins
  }
  return found;
}

void tune_store(const std::string &key, int warps_per_sm, double giant_factor, int giant_alone) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  const std::string path = tune_path();
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) {
    std::string dir = path.substr(0, slash), cur;
    for (size_t i = 0; i <= dir.size(); ++i)
      if (i == dir.size() || dir[i] == '/') {
        cur = dir.substr(0, i);
        if (!cur.empty()) mkdir(cur.c_str(), 0755);
      }
  }
  std::ofstream f(path, std::ios::app);
  f << key << '\t' << warps_per_sm << '\t' << giant_factor << '\t' << giant_alone << '\n';
}

int poa_batch_create(poa_ctx *ctx, const poa_params *params, int64_t n_sets, const int64_t *set_off,
                     const uint8_t *const *seqs, const int64_t *lens, poa_batch **out) {
  *out = nullptr;
  return api(ctx, [&] {
    HostParams hp = checked_params(params);
    if (hp.seeding) throw AlignError{POA_ERR_UNSUPPORTED, "seeded windows (-S) are not available in this build"};
    auto b = std::make_unique<poa_batch>();
    b->ctx = ctx;
    b->hp = hp;
    b->n_sets = n_sets;
    b->set_off.assign(set_off, set_off + n_sets + 1);
    const int64_t n_reads = set_off[n_sets];
    b->lens.assign(lens, lens + n_reads);
    b->sigma = int(hp.alphabet.size());
    b->unknown = hp.encode('N');
    // reads: offsets, lengths, bytes
    int64_t total = 0;
    for (int64_t r = 0; r < n_reads; ++r) {
      if (lens[r] < 0 || lens[r] > INT32_MAX / 4) throw AlignError{POA_ERR_INVALID, "sequence is too long"};
      total += lens[r];
    }
    // progressive (-p, src/lib.rs:190-194): each set's reads are uploaded in
    // its guide order, with their own sequence ids beside them
    std::vector<int64_t> src(static_cast<size_t>(n_reads));
    std::vector<int32_t> rid(static_cast<size_t>(n_reads));
    for (int64_t st = 0; st < n_sets; ++st) {
      const int64_t a = set_off[st], k = set_off[st + 1] - a;
      std::vector<int64_t> order;
      if (hp.progressive)
        order = guide_order(hp, std::vector<const uint8_t *>(seqs + a, seqs + a + k),
                            std::vector<int64_t>(lens + a, lens + a + k));
      for (int64_t q = 0; q < k; ++q) {
        const int64_t o = order.empty() ? q : order[size_t(q)];
        src[size_t(a + q)] = a + o;
        rid[size_t(a + q)] = int32_t(o);
      }
    }
    const size_t off_bytes = size_t(n_reads) * 8 + 8, len_bytes = size_t(n_reads) * 4 + 4,
                 id_bytes = size_t(n_reads) * 4 + 4;
    b->reads_bytes = off_bytes + len_bytes + id_bytes + size_t(total) + 64;
    char *rb = (char *)ctx->dalloc(b->reads_bytes);
    b->d_read_off = (int64_t *)rb;
    b->d_read_len = (int32_t *)(rb + off_bytes);
    int32_t *d_read_id = (int32_t *)(rb + off_bytes + len_bytes);
    b->d_reads = (uint8_t *)(rb + off_bytes + len_bytes + id_bytes);
    {
      // (not value-initialised: every byte up to the reads' end is written)
      std::unique_ptr<char[]> host_buf(new char[b->reads_bytes]);
      char *const host_data = host_buf.get();
      std::memset(host_data + b->reads_bytes - 64, 0, 64);
      int64_t *off = (int64_t *)host_data;
      int32_t *ln = (int32_t *)(host_data + off_bytes);
      int32_t *ids = (int32_t *)(host_data + off_bytes + len_bytes);
      char *rd = host_data + off_bytes + len_bytes + id_bytes;
      int64_t at = 0;
      for (int64_t r = 0; r < n_reads; ++r) {
        const int64_t o = src[size_t(r)];
        off[r] = at;
        ln[r] = int32_t(lens[o]);
        ids[r] = rid[size_t(r)];
        if (lens[o]) std::memcpy(rd + at, seqs[o], size_t(lens[o]));
        at += lens[o];
      }
      off[n_reads] = at;
      ln[n_reads] = 0;
      ids[n_reads] = 0;
      CK(cudaMemcpyAsync(rb, host_data, b->reads_bytes, cudaMemcpyHostToDevice, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      b->h2d_bytes = b->reads_bytes;
    }
    b->d_matrix = (int32_t *)ctx->dalloc(hp.matrix.size() * 4 + 4);
    b->d_encode = (uint8_t *)ctx->dalloc(256);
    CK(cudaMemcpyAsync(b->d_matrix, hp.matrix.data(), hp.matrix.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    auto enc = encode_table(hp);
    CK(cudaMemcpyAsync(b->d_encode, enc.data(), 256, cudaMemcpyHostToDevice, ctx->stream));
    b->P = poa_ctx::make_params(hp, b->d_matrix, b->d_encode);
    // graph storage: exact worst case of each set
    b->jobs.resize(size_t(n_sets));
    b->caps.resize(size_t(n_sets));
    std::vector<size_t> at(size_t(n_sets) + 1, 0);
    for (int64_t s = 0; s < n_sets; ++s) {
      int64_t sum = 0;
      const int64_t k = set_off[s + 1] - set_off[s];
      for (int64_t r = set_off[s]; r < set_off[s + 1]; ++r) sum += lens[r];
      Caps c;
      c.sigma = b->sigma;
      c.node_cap = int32_t(std::min<int64_t>(sum + 2 * k + 8, INT32_MAX / 2));
      c.chunk_cap = int32_t(std::min<int64_t>(2 * (sum + 3 * k) + 16, INT32_MAX / 2));
      c.path_cap = int32_t(std::min<int64_t>(sum + k + 1, INT32_MAX / 2));
      c.max_paths = int32_t(k + 1);
      b->caps[size_t(s)] = c;
      Job J{};
      at[size_t(s) + 1] = at[size_t(s)] + layout(c, nullptr, &J);
    }
    b->storage_bytes = at.back();
    b->storage = (char *)ctx->dalloc(b->storage_bytes);
    for (int64_t s = 0; s < n_sets; ++s) {
      Job &J = b->jobs[size_t(s)];
      J = Job{};
      layout(b->caps[size_t(s)], b->storage + at[size_t(s)], &J);
      J.reads = b->d_reads;
      J.read_off = b->d_read_off + set_off[s];
      J.read_len = b->d_read_len + set_off[s];
      J.read_id = hp.progressive ? d_read_id + set_off[s] : nullptr;
      J.n_reads = int32_t(set_off[s + 1] - set_off[s]);
    }
    b->d_jobs = (Job *)ctx->dalloc(b->jobs.size() * sizeof(Job) + 16);
    b->upload_jobs();
    // size-ordered queue: largest estimated work first
    std::vector<double> est(size_t(n_sets), 0.0);
    for (int64_t s = 0; s < n_sets; ++s) {
      double mx = 0, sum = 0;
      for (int64_t r = set_off[s]; r < set_off[s + 1]; ++r) {
        mx = std::max(mx, double(lens[r]));
        sum += double(lens[r]);
      }
      const double w = 2.0 * (double(hp.b) + (hp.f ? mx / double(hp.f) : mx)) + 16.0;
      // rows grow with the reads already fused into the graph
      const double reads = double(set_off[s + 1] - set_off[s]);
      est[size_t(s)] = sum * std::min(w, mx + 16.0) * (1.0 + 0.03 * reads);
    }
    b->order.resize(size_t(n_sets));
    std::iota(b->order.begin(), b->order.end(), 0);
    std::stable_sort(b->order.begin(), b->order.end(), [&](int32_t a, int32_t c) { return est[a] > est[c]; });
    b->est = est;
    b->tune_key = tune_key(ctx, n_sets, set_off, lens);
    tune_lookup(b->tune_key, &b->warps_per_sm, &b->giant_factor, &b->giant_alone);
    b->mark_giants();
    b->upload_jobs();
    b->d_order = (int32_t *)ctx->dalloc(b->order_bytes());
    b->d_queue = (int32_t *)ctx->dalloc(sched_words(b->jobs.size()) * 4);
    CK(cudaMemcpyAsync(b->base_order(), b->order.data(), b->order.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaEventCreate(&b->e0));
    CK(cudaEventCreate(&b->e1));
    CK(cudaEventCreate(&b->k0));
    CK(cudaEventCreate(&b->k1));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->batches.push_back(b.get());
    *out = b.release();
  });
}

int poa_batch_autotune(poa_ctx *ctx, poa_batch *b, poa_batch_tuning *out) {
  return api(ctx, [&] {
    // candidate launch settings: resident warps per SM, the giant threshold
    // (0: no giant gets helper warps) and whether a giant's SM runs its team
    // alone; the first is the default
    struct Cand {
      int wps;
      double gf;
      int alone;
    };
    const Cand cand[] = {{kDefaultBatchWarpsPerSm, 1.5, 0}, {6, 1.5, 1}, {5, 1.5, 1}, {6, 1.0, 1}, {4, 1.5, 0},
                         {6, 1.5, 0}, {7, 1.5, 0}, {8, 1.5, 0}, {8, 1.5, 1}};
    double best_ms = 0;
    Cand best{b->warps_per_sm, b->giant_factor, b->giant_alone};
    int tried = 0;
    for (const Cand &c : cand) {
      b->warps_per_sm = c.wps;
      b->giant_factor = c.gf;
      b->giant_alone = c.alone;
      b->mark_giants();
      b->upload_jobs();
      poa_batch_stats st{};
      const int rc = poa_batch_run(ctx, b, 0, &st);
      if (rc != POA_OK) throw AlignError{rc, t_last_error};
      ++tried;
      if (tried == 1 || st.device_ms < best_ms) {
        best_ms = st.device_ms;
        best = c;
      }
    }
    b->warps_per_sm = best.wps;
    b->giant_factor = best.gf;
    b->giant_alone = best.alone;
    b->mark_giants();
    b->upload_jobs();
    tune_store(b->tune_key, best.wps, best.gf, best.alone);
    if (out) {
      out->warps_per_sm = best.wps;
      out->giant_alone = best.alone;
      out->giant_factor = best.gf;
      out->device_ms = best_ms;
      out->trials = tried;
    }
  });
}

int poa_batch_tuning_get(poa_ctx *ctx, poa_batch *b, poa_batch_tuning *out) {
  return api(ctx, [&] {
    out->warps_per_sm = b->warps_per_sm > 0 ? b->warps_per_sm : kDefaultBatchWarpsPerSm;
    out->giant_alone = b->giant_alone;
    out->giant_factor = b->giant_factor;
    out->device_ms = 0;
    out->trials = b->graph_launches;
  });
}

int poa_batch_tune(poa_ctx *ctx, poa_batch *batch, int32_t warps_per_sm, uint64_t arena_bytes_per_slot) {
  return api(ctx, [&] {
    if (warps_per_sm < 0) throw AlignError{POA_ERR_INVALID, "warps per SM must not be negative"};
    batch->warps_per_sm = warps_per_sm;
    batch->slot_bytes_override = arena_bytes_per_slot;
  });
}

int poa_batch_run(poa_ctx *ctx, poa_batch *b, int32_t mode, poa_batch_stats *stats) {
  return api(ctx, [&] {
    if (mode != 0 && mode != 1) throw AlignError{POA_ERR_INVALID, "mode must be 0 (batched) or 1 (plain)"};
    if (b->n_sets == 0) {  // nothing to align
      if (stats) *stats = poa_batch_stats{};
      b->ran = true;
      return;
    }
    // arena pool: the rest of the budget, allocated once
    if (!b->arenas) {
      // the other batches' pools are idle between their runs: take them back
      for (poa_batch *o : ctx->batches)
        if (o != b && o->arenas) o->drop_arenas();
      const uint64_t left = ctx->budget > ctx->allocated ? ctx->budget - ctx->allocated : 0;
      const int64_t pool = int64_t(left) - (int64_t(256) << 20);
      if (pool < (int64_t(64) << 20)) throw AlignError{POA_ERR_ALLOC, "no device memory left for DP arenas"};
      b->arenas = (char *)ctx->dalloc(size_t(pool));
      b->arena_pool = pool;
    }
    const int sms = ctx->sm_count;
    int wps = b->warps_per_sm > 0 ? b->warps_per_sm : kDefaultBatchWarpsPerSm;
    int passes = 0, launches = 0;
    double kernel_ms = 0;
    CK(cudaEventRecord(b->e0, ctx->stream));
    if (mode != 0) {
      CK(launch_reset(b->d_jobs, int(b->n_sets), b->sigma, b->unknown, ctx->stream));
      ++launches;
    }
    int slots_first = 0;
    if (mode == 0) {
      std::vector<int32_t> pending = b->order;
      int64_t slots = int64_t(sms) * wps;
      for (;;) {
        slots = std::max<int64_t>(1, std::min<int64_t>(slots, int64_t(pending.size())));
        // a small batch (at most one set per SM) runs as teams: one 4-warp
        // block per set, the set on warp 0 with three helper warps for its
        // DP rows, one arena per block (not with the row wavefront forced: a
        // warp leading helpers runs rows one at a time)
        const bool team = passes == 0 && !pending.empty() && b->giant_factor > 0 &&
                          int64_t(pending.size()) <= sms && b->P.row_wave != 2;
        if (team) slots = 4 * int64_t(pending.size());
        b->P.teams = team ? 1 : 0;
        int64_t slot_bytes = b->arena_pool / (team ? slots / 4 : slots) / 256 * 256;
        if (b->slot_bytes_override && passes == 0)
          slot_bytes = std::min<int64_t>(int64_t(b->slot_bytes_override), slot_bytes);
        if (passes == 0) {
          slots_first = int(slots);
          // the first pass as one CUDA graph (reset of every graph, queue
          // set-up, the persistent kernel), captured once per launch shape
          b->P.giant_alone = b->giant_alone;
          if (!b->gexec || b->g_slots != slots || b->g_slot_bytes != slot_bytes || b->g_alone != b->giant_alone ||
              b->g_team != int(team)) {
            if (b->gexec) cudaGraphExecDestroy(b->gexec);
            b->gexec = nullptr;
            CK(prepare_batch_kernel());
            cudaGraph_t graph = nullptr;
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t ce = launch_reset(b->d_jobs, int(b->n_sets), b->sigma, b->unknown, ctx->stream);
            if (ce == cudaSuccess)
              ce = cudaMemcpyAsync(b->d_order, b->base_order(), b->order.size() * 4, cudaMemcpyDeviceToDevice,
                                   ctx->stream);
            if (ce == cudaSuccess)
              ce = cudaMemsetAsync(b->d_queue, 0, sched_words(b->order.size()) * 4, ctx->stream);
            if (ce == cudaSuccess)
              ce = launch_batch(b->d_jobs, b->d_order, int(b->order.size()), b->d_queue, ctx->sm_count, b->P,
                                b->arenas, slot_bytes, int(slots), ctx->stream);
            const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &graph);
            if (ce == cudaSuccess) ce = ee;
            if (ce == cudaSuccess) ce = cudaGraphInstantiate(&b->gexec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            CK(ce);
            b->g_slots = slots;
            b->g_slot_bytes = slot_bytes;
            b->g_alone = b->giant_alone;
            b->g_team = int(team);
          }
          // timing events stay outside the graph: an event recorded during
          // capture becomes a dependency marker, not a timestamp
          CK(cudaEventRecord(b->k0, ctx->stream));
          CK(cudaGraphLaunch(b->gexec, ctx->stream));
          CK(cudaEventRecord(b->k1, ctx->stream));
          ++b->graph_launches;
          launches += 2;
        } else {
          CK(cudaMemcpyAsync(b->d_order, pending.data(), pending.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
          CK(cudaMemsetAsync(b->d_queue, 0, sched_words(pending.size()) * 4, ctx->stream));
          CK(cudaEventRecord(b->k0, ctx->stream));
          CK(launch_batch(b->d_jobs, b->d_order, int(pending.size()), b->d_queue, ctx->sm_count, b->P, b->arenas,
                          slot_bytes, int(slots), ctx->stream));
          CK(cudaEventRecord(b->k1, ctx->stream));
          ++launches;
        }
        ++passes;
        b->download_jobs();
        float kms = 0;
        CK(cudaEventElapsedTime(&kms, b->k0, b->k1));
        kernel_ms += kms;
        std::vector<int32_t> parked;
        for (int32_t s : pending)
          if (b->jobs[size_t(s)].status == ST_ARENA_FULL) parked.push_back(s);
        if (parked.empty()) break;
        if (slots == 1) throw AlignError{POA_ERR_ALLOC, "a read set needs more DP arena than the memory budget"};
        for (int32_t s : parked) b->jobs[size_t(s)].status = ST_OK;
        b->upload_jobs();
        pending = parked;
        slots = std::max<int64_t>(1, slots / 8);
      }
    } else {
      // plain form: every read is its own launch, one warp, whole pool as arena
      const int64_t slot_bytes = b->arena_pool / 256 * 256;
      slots_first = 1;
      CK(cudaEventRecord(b->k0, ctx->stream));
      for (int64_t s = 0; s < b->n_sets; ++s) {
        const int64_t k = b->set_off[s + 1] - b->set_off[s];
        for (int64_t r = 0; r < k; ++r) {
          CK(launch_extend_step(b->d_jobs + s, b->P, b->arenas, slot_bytes, int(r), ctx->stream));
          ++launches;
        }
      }
      CK(cudaEventRecord(b->k1, ctx->stream));
      CK(cudaEventSynchronize(b->k1));
      float kms = 0;
      CK(cudaEventElapsedTime(&kms, b->k0, b->k1));
      kernel_ms += kms;
      passes = 1;
    }
    CK(cudaEventRecord(b->e1, ctx->stream));
    CK(cudaEventSynchronize(b->e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, b->e0, b->e1));
    b->download_jobs();
    b->ran = true;
    if (stats) {
      for (int k = 0; k < 4; ++k) stats->phase_cycles[k] = 0;
      uint64_t cells = 0, reads = 0, dpb = 0, pc = 0, far = 0, g4 = 0, gen = 0;
      int32_t coop = 0, wave = 0;
      for (auto &J : b->jobs) {
        cells += J.cells;
        dpb += J.dp_bytes;
        reads += uint64_t(J.next_read);
        pc += J.pred_cells;
        far += J.far_preds;
        g4 += J.rows_g4;
        gen += J.rows_generic;
        coop += J.coop;
        wave += J.wave_reads;
        for (int k = 0; k < 4; ++k) stats->phase_cycles[k] += J.phase[k];
      }
      stats->cells = cells;
      stats->dp_bytes = dpb;
      stats->pred_cells = pc;
      stats->far_preds = far;
      stats->rows_g4 = g4;
      stats->rows_generic = gen;
      stats->coop_jobs = coop;
      stats->wave_reads = wave;
      stats->kernel_ms = kernel_ms;
      stats->reads = reads;
      stats->device_ms = ms;
      stats->launches = launches;
      stats->relaunches = passes - 1;
      stats->slots = slots_first;
    }
  });
}

int poa_batch_status(poa_ctx *ctx, poa_batch *b, int64_t set, char **message) {
  *message = nullptr;
  int rc = POA_OK;
  int api_rc = api(ctx, [&] {
    if (set < 0 || set >= b->n_sets) throw AlignError{POA_ERR_INVALID, "set index out of range"};
    const Job &J = b->jobs[size_t(set)];
    if (J.status != ST_OK) {
      rc = status_code(J.status);
      *message = dup_string(status_message(J.status, J.err_i, J.err_j));
    }
  });
  return api_rc != POA_OK ? api_rc : rc;
}

int poa_batch_output(poa_ctx *ctx, poa_batch *b, int64_t set, int32_t result, const char *const *names,
                     const char *const *comments, char **out, int64_t *out_len) {
  *out = nullptr;
  *out_len = 0;
  return api(ctx, [&] {
    if (set < 0 || set >= b->n_sets) throw AlignError{POA_ERR_INVALID, "set index out of range"};
    const Job &J = b->jobs[size_t(set)];
    if (J.status != ST_OK) throw AlignError{status_code(J.status), status_message(J.status, J.err_i, J.err_j)};
    auto gs = b->graphs({int32_t(set)});
    const int64_t k = b->set_off[set + 1] - b->set_off[set];
    auto nm = name_list(k, names, "read");
    std::vector<std::string> cm(static_cast<size_t>(k));
    for (int64_t i = 0; i < k && comments; ++i) cm[size_t(i)] = comments[i];
    std::string s, err;
    if (result == 0) {
      std::vector<uint8_t> sq;
      std::vector<int64_t> ids, cv;
      gs[0].consensus(b->hp, sq, ids, cv);
      s = ">consensus sequence\n" + std::string(sq.begin(), sq.end()) + "\n";
    } else if (result == 1) {
      if (!gs[0].msa(b->hp, nm, cm, s, err)) throw AlignError{POA_ERR_ALIGN, err};
    } else if (result == 2) {
      if (!gs[0].gfa(b->hp, nm, s, err)) throw AlignError{POA_ERR_ALIGN, err};
    } else {
      throw AlignError{POA_ERR_INVALID, "result format and verbosity must be 0..2"};
    }
    *out = dup_string(s);
    *out_len = int64_t(s.size());
  });
}

int poa_batch_output_all(poa_ctx *ctx, poa_batch *b, int32_t result, char **out, int64_t *out_len) {
  *out = nullptr;
  *out_len = 0;
  return api(ctx, [&] {
    if (result != 0 && result != 2) throw AlignError{POA_ERR_INVALID, "batch output supports results 0 and 2"};
    if (result == 0) {  // consensus on the device: only the sequences come back
      auto parts = b->device_consensus();
      size_t total = 0;
      for (auto &p : parts) total += p.size();
      std::string all;
      all.reserve(total);
      for (auto &p : parts) all += p;
      *out = dup_string(all);
      *out_len = int64_t(all.size());
      return;
    }
    std::vector<int32_t> ids(static_cast<size_t>(b->n_sets));
    std::iota(ids.begin(), ids.end(), 0);
    auto gs = b->graphs(ids);
    std::vector<std::string> parts(ids.size());
    const int nt = std::max(1, std::min<int>(int(std::thread::hardware_concurrency()), 32));
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
      pool.emplace_back([&, t] {
        for (size_t s = size_t(t); s < ids.size(); s += size_t(nt)) {
          const Job &J = b->jobs[s];
          if (J.status != ST_OK) {
            parts[s] = "!error " + status_message(J.status, J.err_i, J.err_j) + "\n";
            continue;
          }
          if (result == 0) {
            std::vector<uint8_t> sq;
            std::vector<int64_t> idv, cv;
            gs[s].consensus(b->hp, sq, idv, cv);
            parts[s] = ">consensus sequence\n" + std::string(sq.begin(), sq.end()) + "\n";
          } else {
            const int64_t k = b->set_off[s + 1] - b->set_off[s];
            auto nm = name_list(k, nullptr, "read");
            std::string err;
            if (!gs[s].gfa(b->hp, nm, parts[s], err)) parts[s] = "!error " + err + "\n";
          }
        }
      });
    for (auto &th : pool) th.join();
    size_t total = 0;
    for (auto &p : parts) total += p.size();
    std::string all;
    all.reserve(total);
    for (auto &p : parts) all += p;
    *out = dup_string(all);
    *out_len = int64_t(all.size());
  });
}

int poa_batch_graph(poa_ctx *ctx, poa_batch *b, int64_t set, poa_graph **out) {
  *out = nullptr;
  return api(ctx, [&] {
    if (set < 0 || set >= b->n_sets) throw AlignError{POA_ERR_INVALID, "set index out of range"};
    b->download_jobs();
    const Job &src = b->jobs[size_t(set)];
    Caps c = b->caps[size_t(set)];
    std::unique_ptr<poa_graph> g(new_graph(ctx, b->hp, c));
    auto olda = arrays(src, c);
    auto newa = arrays(g->h, g->caps);
    for (size_t k = 0; k < olda.size(); ++k)
      CK(cudaMemcpyAsync(newa[k].first, olda[k].first, olda[k].second, cudaMemcpyDeviceToDevice, ctx->stream));
    Job nj = g->h;
    nj.n_nodes = src.n_nodes;
    nj.n_chunks = src.n_chunks;
    nj.n_edges = src.n_edges;
    nj.n_paths = src.n_paths;
    nj.path_used = src.path_used;
    nj.n_rank = src.n_rank;
    nj.status = ST_OK;
    nj.cells = src.cells;
    g->h = nj;
    g->upload();
    g->sync();
    *out = g.release();
  });
}

int poa_batch_transfer_bytes(poa_ctx *ctx, poa_batch *b, uint64_t *h2d, uint64_t *d2h) {
  return api(ctx, [&] {
    *h2d = b->h2d_bytes;
    *d2h = b->d2h_bytes;
  });
}

void poa_batch_free(poa_batch *batch) { delete batch; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Serving loop: continuous batching of independent jobs (read sets, optionally
// extending a graph built from earlier reads). A dispatcher thread admits
// jobs in arrival order while the server's device pool holds their graph
// storage, reads, DP arena and descriptor, and publishes them to the job
// queue of one persistent serving kernel (k_serve), whose warps take jobs as
// they free up; the kernel ends after its warps have been idle a while and
// is launched again when work arrives. Finished graphs stay resident until
// released.

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// First-fit allocator over one device pool, in 256-byte granules.
struct PoolAlloc {
  char *base = nullptr;
  uint64_t size = 0, used = 0;
  std::map<uint64_t, uint64_t> free_;  // offset -> bytes
  void init(char *b, uint64_t n) {
    base = b;
    size = n;
    used = 0;
    free_.clear();
    if (n) free_[0] = n;
  }
  static uint64_t round(uint64_t n) { return (n + 255) / 256 * 256; }
  char *take(uint64_t bytes) {
    bytes = round(std::max<uint64_t>(bytes, 1));
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const uint64_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > bytes) free_[off + bytes] = len - bytes;
      used += bytes;
      return base + off;
    }
    return nullptr;
  }
  void give(char *p, uint64_t bytes) {
    if (!p) return;
    bytes = round(std::max<uint64_t>(bytes, 1));
    used -= std::min(used, bytes);
    auto it = free_.emplace(uint64_t(p - base), bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct ServerJob {
  int64_t id = 0;
  std::vector<uint8_t> bytes;  // the reads, back to back (in guide order with -p)
  std::vector<int64_t> lens;
  std::vector<int32_t> ids;    // with -p, the sequence id of each read as stored
  // an initial graph to extend (GFA jobs): built and ranked on the host at
  // submission, copied into the job's storage at admission; the job's reads
  // get sequence ids after its `existing` path records
  std::unique_ptr<BuildGraph> init;
  std::vector<int32_t> init_rank, init_order;
  std::unique_ptr<GraphImage> image;  // the initial graph's device arrays, built by the submitting thread
  int32_t existing = 0;
  int skips = 0;  // admission rounds that passed this job over at the head of the queue
  Caps caps;
  uint64_t storage_bytes = 0, reads_bytes = 0, arena_bytes = 0;
  char *storage = nullptr, *reads = nullptr, *arena = nullptr;
  Job J{};  // host copy of the device descriptor
  Job *d_desc = nullptr;  // its device copy (in the pool) while it is admitted
  int done_slot = -1;     // host-mapped flag the kernel raises when the job leaves it
  bool fresh = true;
  int32_t state = POA_SERVER_QUEUED;
  std::string error;
  double t_submit = 0, t_start = 0, t_done = 0;
};

// Pinned staging of one admission round (reads, descriptors, queue entries
// and the new tail), reusable once the round's copies have completed.
struct Stage {
  char *p = nullptr;
  size_t cap = 0;
  cudaEvent_t ev = nullptr;
  bool used = false;
};

}  // namespace

struct poa_server {
  poa_ctx *ctx = nullptr;
  HostParams hp;
  DevParams P{};
  char *pool_mem = nullptr;
  uint64_t pool_bytes = 0;
  PoolAlloc pool;
  std::mutex mu;
  std::condition_variable cv;
  std::map<int64_t, std::unique_ptr<ServerJob>> jobs;
  std::deque<int64_t> pending;
  // the persistent serving kernel and its job queue (device memory, in the
  // pool); uploads and queue publication go in order on up_stream
  ServeQueue *d_q = nullptr;
  uint32_t tail = 0;            // queue entries published
  uint32_t head_seen = 0;       // entries claimed, as last read while no kernel ran
  cudaStream_t up_stream = nullptr, k_stream = nullptr;
  cudaEvent_t k_done = nullptr;
  bool k_live = false;          // a serving kernel was launched and has not been seen to end
  bool stopping = false;        // its stop flag is set (the server was idle)
  int64_t idle_ns = 50000000;   // the kernel ends after the server has been idle this long
  double last_busy = 0;         // when the server last had queued or running jobs
  std::vector<Stage> stages;
  cudaStream_t out_stream = nullptr;
  std::thread worker;
  bool stop = false;
  int64_t next_id = 0;
  int32_t *h_done = nullptr;  // host-mapped completion flags
  int32_t *d_done = nullptr;
  std::vector<int> free_done;
  std::vector<int64_t> running;  // jobs on the device
  std::string fatal;
  double arena_scale = 1.0;  // multiplies the first DP arena of each job
  // statistics of finished jobs
  uint64_t done_jobs = 0, done_cells = 0, rounds = 0, launches = 0;
  double first_submit = -1, last_done = 0;

  ~poa_server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv.notify_all();
    if (worker.joinable()) worker.join();
    // the worker leaves with the queue empty and every job done; a kernel
    // still polling sees stop and leaves
    if (d_q && up_stream) {
      static const uint32_t leave = 2;
      cudaMemcpyAsync(&d_q->stop, &leave, 4, cudaMemcpyHostToDevice, up_stream);
      cudaStreamSynchronize(up_stream);
    }
    if (k_done) {
      if (k_live) cudaEventSynchronize(k_done);
      cudaEventDestroy(k_done);
    }
    for (auto &st : stages) {
      if (st.ev) {
        cudaEventSynchronize(st.ev);
        cudaEventDestroy(st.ev);
      }
      if (st.p) cudaFreeHost(st.p);
    }
    if (up_stream) cudaStreamDestroy(up_stream);
    if (k_stream) cudaStreamDestroy(k_stream);
    if (out_stream) cudaStreamDestroy(out_stream);
    if (h_done) cudaFreeHost(h_done);
    if (ctx) ctx->dfree(pool_mem, pool_bytes);
  }

  // Bytes a job needs beyond its arena: graph storage and reads.
  static void size_job(ServerJob &sj, int sigma) {
    int64_t sum = 0;
    const int64_t k = int64_t(sj.lens.size());
    for (int64_t l : sj.lens) sum += l;
    Caps c;
    c.sigma = sigma;
    c.node_cap = int32_t(std::min<int64_t>(sum + 2 * k + 8, INT32_MAX / 2));
    c.chunk_cap = int32_t(std::min<int64_t>(2 * (sum + 3 * k) + 16, INT32_MAX / 2));
    c.path_cap = int32_t(std::min<int64_t>(sum + k + 1, INT32_MAX / 2));
    c.max_paths = int32_t(k + 1);
    if (sj.init) {
      c.node_cap = int32_t(std::min<int64_t>(int64_t(c.node_cap) + sj.init->n(), INT32_MAX / 2));
      c.chunk_cap = int32_t(std::min<int64_t>(int64_t(c.chunk_cap) + build_chunks(*sj.init), INT32_MAX / 2));
      c.path_cap = int32_t(std::min<int64_t>(int64_t(c.path_cap) + build_path_items(*sj.init), INT32_MAX / 2));
      c.max_paths = int32_t(std::min<int64_t>(int64_t(c.max_paths) + int64_t(sj.init->paths.size()), INT32_MAX / 2));
    }
    sj.caps = c;
    Job J{};
    sj.storage_bytes = layout(c, nullptr, &J) + 256;
    sj.reads_bytes = uint64_t(k) * 16 + uint64_t(sum) + 64;  // offsets, lengths, ids, bytes
  }
  // First DP arena of a job: band cells of its widest read over an estimate of
  // the rows the graph grows to, plus per-row scratch; a job that needs more
  // parks and comes back with twice the arena.
  uint64_t first_arena(const ServerJob &sj) const {
    int64_t mx = 0;
    for (int64_t l : sj.lens) mx = std::max(mx, l);
    const double band = std::min(2.0 * (double(hp.b) + (hp.f ? double(mx) / double(hp.f) : double(mx))) + 16.0,
                                 double(mx) + 16.0);
    const double rows = double(mx) * (1.0 + 0.1 * double(sj.lens.size())) + 16.0 + (sj.init ? sj.init->n() : 0);
    return uint64_t(arena_scale * rows * (band * 12.0 + 400.0)) + (uint64_t(1) << 20);
  }

  void run();
  bool finish_jobs();
  bool admit_jobs();
  bool keep_kernel();
  Stage &stage_for(size_t need);
};

// Jobs whose completion flag is up: their descriptor is read back, and their
// arena, reads and descriptor go back to the pool while the other jobs run.
// A parked job (arena too small) goes back to the head of the queue with
// twice the arena; its graph stays where it is.
bool poa_server::finish_jobs() {
  std::vector<int64_t> ready;
  {
    std::lock_guard<std::mutex> lk(mu);
    for (int64_t id : running) {
      const ServerJob &sj = *jobs.at(id);
      if (reinterpret_cast<volatile int32_t *>(h_done)[sj.done_slot] != 0) ready.push_back(id);
    }
  }
  if (ready.empty()) return false;
  for (int64_t id : ready) {
    Job hj{};
    Job *src = nullptr;
    {
      std::lock_guard<std::mutex> lk(mu);
      src = jobs.at(id)->d_desc;
    }
    CK(cudaMemcpyAsync(&hj, src, sizeof(Job), cudaMemcpyDeviceToHost, out_stream));
    CK(cudaStreamSynchronize(out_stream));
    const double t = now_s();
    std::lock_guard<std::mutex> lk(mu);
    ServerJob &sj = *jobs.at(id);
    running.erase(std::find(running.begin(), running.end(), id));
    free_done.push_back(sj.done_slot);
    sj.done_slot = -1;
    pool.give(reinterpret_cast<char *>(sj.d_desc), sizeof(Job));
    sj.d_desc = nullptr;
    sj.J = hj;
    pool.give(sj.arena, sj.arena_bytes);
    sj.arena = nullptr;
    if (hj.status == ST_ARENA_FULL) {
      sj.arena_bytes *= 2;
      sj.J.status = ST_OK;
      sj.fresh = false;
      sj.state = POA_SERVER_QUEUED;
      pending.push_front(sj.id);
      continue;
    }
    pool.give(sj.reads, sj.reads_bytes);
    sj.reads = nullptr;
    sj.t_done = t;
    if (hj.status == ST_OK) {
      sj.state = POA_SERVER_DONE;
      done_cells += hj.cells;
    } else {
      sj.state = POA_SERVER_FAILED;
      sj.error = status_message(hj.status, hj.err_i, hj.err_j);
    }
    ++done_jobs;
    last_done = t;
  }
  cv.notify_all();
  return true;
}

// A pinned staging buffer of at least `need` bytes whose earlier copies have
// completed (waiting for the oldest one when all are in flight).
Stage &poa_server::stage_for(size_t need) {
  for (;;) {
    Stage *pick = nullptr;
    for (auto &st : stages) {
      if (st.used) {
        const cudaError_t q = cudaEventQuery(st.ev);
        if (q == cudaErrorNotReady) {
          cudaGetLastError();  // not an error: the copies are still running
          continue;
        }
        CK(q);
      }
      pick = &st;
      break;
    }
    if (!pick) {
      CK(cudaEventSynchronize(stages.front().ev));
      std::rotate(stages.begin(), stages.begin() + 1, stages.end());
      continue;
    }
    if (pick->cap < need) {
      if (pick->p) CK(cudaFreeHost(pick->p));
      pick->p = nullptr;
      pick->cap = 0;
      const size_t cap = std::max<size_t>(need, size_t(1) << 20);
      CK(cudaHostAlloc(reinterpret_cast<void **>(&pick->p), cap, cudaHostAllocDefault));
      pick->cap = cap;
    }
    if (!pick->ev) CK(cudaEventCreateWithFlags(&pick->ev, cudaEventDisableTiming));
    pick->used = true;
    return *pick;
  }
}

// Admits queued jobs in arrival order while the pool holds their graph
// storage, reads, DP arena and descriptor, uploads them and publishes them
// to the serving kernel's queue; returns whether any job was admitted.
bool poa_server::admit_jobs() {
  std::vector<ServerJob *> adm;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (pending.empty()) return false;
    // Arrival order, looking past a job that does not fit into the free pool
    // for up to kLookahead later jobs that do; a head job passed over
    // kMaxSkips times holds back the jobs behind it, so a large job is not
    // starved by a stream of small ones.
    constexpr int kLookahead = 32, kMaxSkips = 8;
    int passed = 0;
    for (size_t pi = 0; pi < pending.size() && adm.size() < free_done.size() &&
                        running.size() + adm.size() + 1 < size_t(SERVE_QCAP);) {
      ServerJob &sj = *jobs.at(pending[pi]);
      char *st = sj.storage ? sj.storage : pool.take(sj.storage_bytes);
      char *rd = sj.reads ? sj.reads : (st ? pool.take(sj.reads_bytes) : nullptr);
      char *ar = (st && rd) ? pool.take(sj.arena_bytes) : nullptr;
      char *ds = ar ? pool.take(sizeof(Job)) : nullptr;
      if (!ds) {
        pool.give(ar, sj.arena_bytes);
        if (!sj.storage) pool.give(st, sj.storage_bytes);
        if (!sj.reads) pool.give(rd, sj.reads_bytes);
        // a job larger than the whole idle pool can never run
        if (running.empty() && adm.empty()) {
          pool.give(sj.storage, sj.storage_bytes);
          pool.give(sj.reads, sj.reads_bytes);
          sj.storage = sj.reads = nullptr;
          sj.state = POA_SERVER_FAILED;
          sj.error = "job needs more device memory than the server pool";
          sj.t_done = now_s();
          pending.erase(pending.begin() + long(pi));
          cv.notify_all();
          continue;
        }
        if (pi == 0 && ++sj.skips > kMaxSkips) break;
        if (++passed > kLookahead) break;
        ++pi;
        continue;
      }
      sj.storage = st;
      sj.reads = rd;
      sj.arena = ar;
      sj.d_desc = reinterpret_cast<Job *>(ds);
      pending.erase(pending.begin() + long(pi));
      adm.push_back(&sj);
    }
    if (adm.empty()) return false;
  }
  // fresh jobs are uploaded (reads; an initial graph is copied in), every
  // admitted job's descriptor goes to its place in the pool, then the queue
  // entries and the new tail: all in order on up_stream, from one pinned
  // staging buffer
  const double t = now_s();
  size_t need = adm.size() * (PoolAlloc::round(sizeof(Job)) + 8) + 64;
  for (ServerJob *j : adm)
    if (j->fresh) need += PoolAlloc::round(j->reads_bytes);
  Stage &stg = stage_for(need);
  char *staging = stg.p;
  size_t staged = 0;
  std::vector<unsigned long long> entries;
  entries.reserve(adm.size());
  for (ServerJob *jp : adm) {
    ServerJob &sj = *jp;
    bool reset = false;
    if (sj.fresh) {
      Job J{};
      layout(sj.caps, sj.storage, &J);
      if (sj.init) {
        // the initial graph, ranked in the reference's LIFO order; copies
        // from pageable memory return once the driver has staged the bytes,
        // so the image can go at once
        put_image(*sj.image, sj.caps, J, up_stream);
        sj.image.reset();
        J.order_exact = 1;
        J.seq_base = sj.existing;
      } else {
        reset = true;  // Graph::new on the device when a warp takes the job
      }
      const int64_t n = int64_t(sj.lens.size());
      J.read_off = reinterpret_cast<int64_t *>(sj.reads);
      J.read_len = reinterpret_cast<int32_t *>(sj.reads + n * 8);
      J.read_id = sj.ids.empty() ? nullptr : reinterpret_cast<int32_t *>(sj.reads + n * 12);
      J.reads = reinterpret_cast<uint8_t *>(sj.reads + n * 16);
      J.n_reads = int32_t(n);
      char *host = staging + staged;
      staged += PoolAlloc::round(sj.reads_bytes);
      std::memset(host, 0, sj.reads_bytes);
      int64_t at = 0;
      for (int64_t r = 0; r < n; ++r) {
        reinterpret_cast<int64_t *>(host)[r] = at;
        reinterpret_cast<int32_t *>(host + n * 8)[r] = int32_t(sj.lens[size_t(r)]);
        reinterpret_cast<int32_t *>(host + n * 12)[r] = sj.ids.empty() ? int32_t(r) : sj.ids[size_t(r)];
        at += sj.lens[size_t(r)];
      }
      if (!sj.bytes.empty()) std::memcpy(host + n * 16, sj.bytes.data(), sj.bytes.size());
      CK(cudaMemcpyAsync(sj.reads, host, sj.reads_bytes, cudaMemcpyHostToDevice, up_stream));
      sj.J = J;
      sj.t_start = t;
    }
    sj.J.arena = sj.arena;
    sj.J.arena_bytes = int64_t(sj.arena_bytes);
    sj.J.giant = 0;
    {
      std::lock_guard<std::mutex> lk(mu);
      sj.done_slot = free_done.back();
      free_done.pop_back();
    }
    h_done[sj.done_slot] = 0;
    sj.J.done_flag = d_done + sj.done_slot;
    sj.state = POA_SERVER_RUNNING;
    std::memcpy(staging + staged, &sj.J, sizeof(Job));
    CK(cudaMemcpyAsync(sj.d_desc, staging + staged, sizeof(Job), cudaMemcpyHostToDevice, up_stream));
    staged += PoolAlloc::round(sizeof(Job));
    entries.push_back(reinterpret_cast<unsigned long long>(sj.d_desc) | (reset ? 1ull : 0ull));
  }
  // queue entries (split where the ring wraps), then the tail
  unsigned long long *ent = reinterpret_cast<unsigned long long *>(staging + staged);
  std::memcpy(ent, entries.data(), entries.size() * 8);
  staged += entries.size() * 8;
  const uint32_t first = tail % SERVE_QCAP;
  const size_t n1 = std::min<size_t>(entries.size(), size_t(SERVE_QCAP - first));
  CK(cudaMemcpyAsync(&d_q->slot[first], ent, n1 * 8, cudaMemcpyHostToDevice, up_stream));
  if (n1 < entries.size())
    CK(cudaMemcpyAsync(&d_q->slot[0], ent + n1, (entries.size() - n1) * 8, cudaMemcpyHostToDevice, up_stream));
  uint32_t *new_tail = reinterpret_cast<uint32_t *>(staging + staged);
  *new_tail = tail + uint32_t(entries.size());
  CK(cudaMemcpyAsync(&d_q->tail, new_tail, 4, cudaMemcpyHostToDevice, up_stream));
  CK(cudaEventRecord(stg.ev, up_stream));
  tail += uint32_t(entries.size());
  std::lock_guard<std::mutex> lk(mu);
  for (ServerJob *jp : adm) running.push_back(jp->id);
  ++rounds;
  return true;
}

// Keeps the serving kernel running while the server has work, and ends it
// (stop = 1: its warps leave once the queue is empty) after idle_ns without
// any; a kernel that ended with entries still unclaimed (published as it
// stopped) is launched again, with stop cleared first.
bool poa_server::keep_kernel() {
  static const uint32_t kRun = 0, kStop = 1;
  const double t = now_s();
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!pending.empty() || !running.empty()) last_busy = t;
  }
  if (k_live) {
    const cudaError_t q = cudaEventQuery(k_done);
    if (q == cudaErrorNotReady) {
      cudaGetLastError();
      if (!stopping && t - last_busy > double(idle_ns) * 1e-9) {
        CK(cudaMemcpyAsync(&d_q->stop, &kStop, 4, cudaMemcpyHostToDevice, up_stream));
        stopping = true;
      }
      return false;
    }
    CK(q);
    k_live = false;
    stopping = false;
  }
  if (head_seen == tail) return false;  // no kernel runs, so head cannot have moved
  uint32_t head = 0;
  CK(cudaMemcpyAsync(&head, &d_q->head, 4, cudaMemcpyDeviceToHost, up_stream));
  CK(cudaStreamSynchronize(up_stream));
  head_seen = head;
  if (head == tail) return false;
  CK(cudaMemcpyAsync(&d_q->stop, &kRun, 4, cudaMemcpyHostToDevice, up_stream));
  CK(cudaStreamSynchronize(up_stream));
  CK(launch_serve(d_q, ctx->sm_count, P, k_stream));
  CK(cudaEventRecord(k_done, k_stream));
  k_live = true;
  ++launches;
  return true;
}

void poa_server::run() {
  cudaSetDevice(ctx->device);
  try {
    for (;;) {
      bool progress = false;
      if (finish_jobs()) progress = true;
      if (admit_jobs()) progress = true;
      if (keep_kernel()) progress = true;
      std::unique_lock<std::mutex> lk(mu);
      if (stop && pending.empty() && running.empty()) break;
      if (!progress) cv.wait_for(lk, std::chrono::microseconds(running.empty() ? 2000 : 50));
    }
  } catch (const CudaError &e) {
    std::lock_guard<std::mutex> lk(mu);
    fatal = std::string(cudaGetErrorString(e.code)) + " (" + e.where + ")";
    for (auto &kv : jobs)
      if (kv.second->state == POA_SERVER_QUEUED || kv.second->state == POA_SERVER_RUNNING) {
        kv.second->state = POA_SERVER_FAILED;
        kv.second->error = fatal;
      }
    pending.clear();
    cv.notify_all();
  }
}

extern "C" {

int poa_server_create(poa_ctx *ctx, const poa_params *params, uint64_t pool_bytes, int32_t idle_ms,
                      poa_server **out) {
  if (out) *out = nullptr;
  if (!ctx || !out) return POA_ERR_INVALID;
  std::unique_ptr<poa_server> sv(new poa_server());
  const int rc = api(ctx, [&] {
    sv->hp = checked_params(params);
    if (sv->hp.seeding) throw AlignError{POA_ERR_UNSUPPORTED, "seeded windows (-S) are not available in this build"};
    if (idle_ms > 0) sv->idle_ns = int64_t(idle_ms) * 1000000;
    // idle DP arena pools of the context's batches go back to the budget
    for (poa_batch *o : ctx->batches)
      if (o->arenas) o->drop_arenas();
    const uint64_t left = ctx->budget > ctx->allocated ? ctx->budget - ctx->allocated : 0;
    if (pool_bytes == 0) pool_bytes = left > (uint64_t(512) << 20) ? left - (uint64_t(512) << 20) : 0;
    pool_bytes = pool_bytes / 256 * 256;  // the scoring tables follow the pool, 256-byte aligned
    if (pool_bytes < (uint64_t(64) << 20)) throw AlignError{POA_ERR_ALLOC, "server pool below 64 MiB"};
    const size_t mat = (sv->hp.matrix.size() * 4 + 255) / 256 * 256 + 256;
    const size_t qbytes = (sizeof(ServeQueue) + 255) / 256 * 256;
    sv->pool_mem = (char *)ctx->dalloc(pool_bytes + mat + qbytes);
    sv->ctx = ctx;
    sv->pool_bytes = pool_bytes + mat + qbytes;
    sv->d_q = reinterpret_cast<ServeQueue *>(sv->pool_mem + pool_bytes + mat);
    CK(cudaMemset(sv->d_q, 0, sizeof(ServeQueue)));
    int32_t *d_matrix = reinterpret_cast<int32_t *>(sv->pool_mem + pool_bytes);
    uint8_t *d_encode = reinterpret_cast<uint8_t *>(sv->pool_mem + pool_bytes + (sv->hp.matrix.size() * 4 + 255) / 256 * 256);
    CK(cudaMemcpy(d_matrix, sv->hp.matrix.data(), sv->hp.matrix.size() * 4, cudaMemcpyHostToDevice));
    auto enc = encode_table(sv->hp);
    CK(cudaMemcpy(d_encode, enc.data(), 256, cudaMemcpyHostToDevice));
    sv->P = poa_ctx::make_params(sv->hp, d_matrix, d_encode);
    sv->pool.init(sv->pool_mem, pool_bytes);
    CK(cudaStreamCreateWithFlags(&sv->up_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&sv->k_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&sv->out_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&sv->k_done, cudaEventDisableTiming));
    sv->stages.resize(8);
    constexpr int kDoneSlots = 1 << 16;
    CK(cudaHostAlloc(reinterpret_cast<void **>(&sv->h_done), kDoneSlots * 4, cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&sv->d_done), sv->h_done, 0));
    for (int k = kDoneSlots - 1; k >= 0; --k) sv->free_done.push_back(k);
    poa_server *raw = sv.get();
    sv->worker = std::thread([raw] { raw->run(); });
  });
  if (rc == POA_OK) *out = sv.release();
  return rc;
}

void poa_server_destroy(poa_server *server) { delete server; }

int poa_server_submit(poa_ctx *ctx, poa_server *sv, int64_t n_seqs, const uint8_t *const *seqs, const int64_t *lens,
                      int64_t *job_id) {
  if (!ctx || !sv || !job_id || (n_seqs > 0 && (!seqs || !lens)) || n_seqs < 0) return POA_ERR_INVALID;
  return api(ctx, [&] {
    auto sj = std::make_unique<ServerJob>();
    int64_t total = 0;
    for (int64_t r = 0; r < n_seqs; ++r) {
      if (lens[r] < 0 || lens[r] > INT32_MAX / 4) throw AlignError{POA_ERR_INVALID, "sequence is too long"};
      total += lens[r];
    }
    // progressive (-p, src/lib.rs:190-194): the reads are stored in guide
    // order with their own sequence ids
    std::vector<int64_t> order;
    if (sv->hp.progressive)
      order = guide_order(sv->hp, std::vector<const uint8_t *>(seqs, seqs + n_seqs),
                          std::vector<int64_t>(lens, lens + n_seqs));
    sj->bytes.resize(size_t(total));
    sj->lens.resize(size_t(n_seqs));
    int64_t at = 0;
    for (int64_t q = 0; q < n_seqs; ++q) {
      const int64_t r = order.empty() ? q : order[size_t(q)];
      sj->lens[size_t(q)] = lens[r];
      if (!order.empty()) sj->ids.push_back(int32_t(r));
      if (lens[r]) std::memcpy(sj->bytes.data() + at, seqs[r], size_t(lens[r]));
      at += lens[r];
    }
    poa_server::size_job(*sj, int(sv->hp.alphabet.size()));
    sj->arena_bytes = sv->first_arena(*sj);
    sj->t_submit = now_s();
    std::lock_guard<std::mutex> lk(sv->mu);
    if (!sv->fatal.empty()) throw AlignError{POA_ERR_CUDA, sv->fatal};
    sj->id = sv->next_id++;
    *job_id = sj->id;
    if (sv->first_submit < 0) sv->first_submit = sj->t_submit;
    sv->pending.push_back(sj->id);
    sv->jobs[sj->id] = std::move(sj);
    sv->cv.notify_all();
  });
}

int poa_server_submit_gfa(poa_ctx *ctx, poa_server *sv, const char *gfa, int64_t gfa_len, int64_t n_seqs,
                          const uint8_t *const *seqs, const int64_t *lens, int64_t *job_id) {
  if (!ctx || !sv || !job_id || (n_seqs > 0 && (!seqs || !lens)) || n_seqs < 0 || gfa_len < 0 ||
      (gfa_len > 0 && !gfa))
    return POA_ERR_INVALID;
  return api(ctx, [&] {
    auto sj = std::make_unique<ServerJob>();
    std::vector<GfaRecord> recs;
    try {
      sj->init.reset(new BuildGraph(read_gfa(sv->hp, gfa, size_t(gfa_len), recs)));
      sj->init->toposort(sj->init_rank, sj->init_order);
    } catch (const std::runtime_error &e) {
      throw AlignError{POA_ERR_ALIGN, e.what()};
    }
    sj->existing = int32_t(recs.size());
    int64_t total = 0;
    for (int64_t r = 0; r < n_seqs; ++r) {
      if (lens[r] < 0 || lens[r] > INT32_MAX / 4) throw AlignError{POA_ERR_INVALID, "sequence is too long"};
      total += lens[r];
    }
    sj->bytes.resize(size_t(total));
    sj->lens.assign(lens, lens + n_seqs);
    int64_t at = 0;
    for (int64_t r = 0; r < n_seqs; ++r) {
      if (lens[r]) std::memcpy(sj->bytes.data() + at, seqs[r], size_t(lens[r]));
      at += lens[r];
    }
    poa_server::size_job(*sj, int(sv->hp.alphabet.size()));
    sj->arena_bytes = sv->first_arena(*sj);
    // the device image of the initial graph is built here, not by the
    // dispatcher thread, which admits every job
    sj->image.reset(new GraphImage(graph_image(*sj->init, sj->caps, &sj->init_rank, &sj->init_order)));
    sj->t_submit = now_s();
    std::lock_guard<std::mutex> lk(sv->mu);
    if (!sv->fatal.empty()) throw AlignError{POA_ERR_CUDA, sv->fatal};
    sj->id = sv->next_id++;
    *job_id = sj->id;
    if (sv->first_submit < 0) sv->first_submit = sj->t_submit;
    sv->pending.push_back(sj->id);
    sv->jobs[sj->id] = std::move(sj);
    sv->cv.notify_all();
  });
}

int poa_server_wait(poa_ctx *ctx, poa_server *sv, int64_t job, double timeout_ms, int32_t *state) {
  if (!ctx || !sv) return POA_ERR_INVALID;
  return api(ctx, [&] {
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(job);
    if (it == sv->jobs.end()) throw AlignError{POA_ERR_INVALID, "unknown job"};
    ServerJob &sj = *it->second;
    auto finished = [&] { return sj.state == POA_SERVER_DONE || sj.state == POA_SERVER_FAILED; };
    if (timeout_ms < 0)
      sv->cv.wait(lk, finished);
    else
      sv->cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), finished);
    if (state) *state = sj.state;
    if (!finished() && timeout_ms >= 0) throw AlignError{POA_ERR_TIMEOUT, "job not finished within the timeout"};
  });
}

int poa_server_job_info(poa_ctx *ctx, poa_server *sv, int64_t job, poa_server_job *out) {
  if (!ctx || !sv || !out) return POA_ERR_INVALID;
  return api(ctx, [&] {
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(job);
    if (it == sv->jobs.end()) throw AlignError{POA_ERR_INVALID, "unknown job"};
    const ServerJob &sj = *it->second;
    out->state = sj.state;
    out->reserved = 0;
    out->cells = sj.J.cells;
    out->queued_ms = (sj.t_start > 0 ? sj.t_start - sj.t_submit : 0) * 1e3;
    out->latency_ms = (sj.t_done > 0 ? sj.t_done - sj.t_submit : 0) * 1e3;
    if (sj.state == POA_SERVER_FAILED) throw AlignError{POA_ERR_ALIGN, sj.error};
  });
}

int poa_server_output(poa_ctx *ctx, poa_server *sv, int64_t job, int32_t result, const char *const *names,
                      const char *const *comments, char **out, int64_t *out_len) {
  if (out) *out = nullptr;
  if (out_len) *out_len = 0;
  if (!ctx || !sv || !out || !out_len) return POA_ERR_INVALID;
  return api(ctx, [&] {
    Job J{};
    int64_t k = 0;
    char *tmp = nullptr;
    uint64_t tmp_bytes = 0, words = 0;
    const int sigma = int(sv->hp.alphabet.size());
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      auto it = sv->jobs.find(job);
      if (it == sv->jobs.end()) throw AlignError{POA_ERR_INVALID, "unknown job"};
      ServerJob &sj = *it->second;
      if (sj.state == POA_SERVER_FAILED) throw AlignError{POA_ERR_ALIGN, sj.error};
      if (sj.state != POA_SERVER_DONE) throw AlignError{POA_ERR_INVALID, "job has not finished"};
      J = sj.J;
      // sequence ids: the imported graph's path records, then the new reads
      k = int64_t(sj.existing) + int64_t(sj.lens.size());
      words = uint64_t(packed_words(J, sigma));
      tmp_bytes = 1024 + words * 4 + 16;
      tmp = sv->pool.take(tmp_bytes);
      if (!tmp) throw AlignError{POA_ERR_ALLOC, "server pool has no room for the output"};
    }
    std::vector<int32_t> rec(words + 1);
    auto release = [&] {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->pool.give(tmp, tmp_bytes);
    };
    try {
      Job *d_job = reinterpret_cast<Job *>(tmp);
      int64_t *d_off = reinterpret_cast<int64_t *>(tmp + 512);
      int32_t *d_id = reinterpret_cast<int32_t *>(tmp + 768);
      int32_t *d_out = reinterpret_cast<int32_t *>(tmp + 1024);
      const int64_t offs[2] = {0, int64_t(words)};
      const int32_t id0 = 0;
      cudaStream_t st = sv->out_stream;
      CK(cudaMemcpyAsync(d_job, &J, sizeof(Job), cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(d_off, offs, sizeof(offs), cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(d_id, &id0, 4, cudaMemcpyHostToDevice, st));
      CK(launch_pack(d_job, d_id, 1, d_off, d_out, sigma, st));
      CK(cudaMemcpyAsync(rec.data(), d_out, words * 4, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    } catch (...) {
      release();
      throw;
    }
    release();
    HostGraph g = HostGraph::parse(rec.data());
    auto nm = name_list(k, names, "read");
    std::vector<std::string> cm(static_cast<size_t>(k));
    for (int64_t i = 0; i < k && comments; ++i) cm[size_t(i)] = comments[i];
    std::string s, err;
    if (result == 0) {
      std::vector<uint8_t> sq;
      std::vector<int64_t> ids, cv;
      g.consensus(sv->hp, sq, ids, cv);
      s = ">consensus sequence\n" + std::string(sq.begin(), sq.end()) + "\n";
    } else if (result == 1) {
      if (!g.msa(sv->hp, nm, cm, s, err)) throw AlignError{POA_ERR_ALIGN, err};
    } else if (result == 2) {
      if (!g.gfa(sv->hp, nm, s, err)) throw AlignError{POA_ERR_ALIGN, err};
    } else {
      throw AlignError{POA_ERR_INVALID, "result format and verbosity must be 0..2"};
    }
    *out = dup_string(s);
    *out_len = int64_t(s.size());
  });
}

int poa_server_release(poa_ctx *ctx, poa_server *sv, int64_t job) {
  if (!ctx || !sv) return POA_ERR_INVALID;
  return api(ctx, [&] {
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(job);
    if (it == sv->jobs.end()) throw AlignError{POA_ERR_INVALID, "unknown job"};
    ServerJob &sj = *it->second;
    if (sj.state != POA_SERVER_DONE && sj.state != POA_SERVER_FAILED)
      throw AlignError{POA_ERR_INVALID, "job has not finished"};
    sv->pool.give(sj.storage, sj.storage_bytes);
    sv->jobs.erase(it);
    sv->cv.notify_all();
  });
}

int poa_server_tune(poa_ctx *ctx, poa_server *sv, double arena_scale) {
  if (!ctx || !sv) return POA_ERR_INVALID;
  return api(ctx, [&] {
    if (!(arena_scale > 0.0) || arena_scale > 1e6) throw AlignError{POA_ERR_INVALID, "arena scale must be positive"};
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->arena_scale = arena_scale;
  });
}

int poa_server_stats_get(poa_ctx *ctx, poa_server *sv, poa_server_stats *out) {
  if (!ctx || !sv || !out) return POA_ERR_INVALID;
  return api(ctx, [&] {
    std::lock_guard<std::mutex> lk(sv->mu);
    out->done_jobs = sv->done_jobs;
    out->done_cells = sv->done_cells;
    out->waves = sv->rounds;
    out->queued = uint64_t(sv->pending.size());
    out->kernel_launches = sv->launches;
    out->pool_bytes = sv->pool.size;
    out->pool_used = sv->pool.used;
    out->busy_s = sv->first_submit >= 0 ? sv->last_done - sv->first_submit : 0;
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Accessors for entry points defined in other translation units.
namespace poa {

Job *graph_device_job(poa_graph *g) { return g->d_job; }
int graph_alphabet(const poa_graph *g) { return g->sigma; }
const poa_ctx *graph_context(const poa_graph *g) { return g->ctx; }
cudaStream_t ctx_stream(const poa_ctx *c) { return c->stream; }
int ctx_device(const poa_ctx *c) { return c->device; }
void ctx_set_error(poa_ctx *c, const std::string &msg) {
  (void)c;
  t_last_error = msg;
}
std::string describe_status(int32_t st, int err_i, int err_j) { return status_message(st, err_i, err_j); }
int status_to_code(int32_t st) { return status_code(st); }

// Copies the graph's device descriptor to *out (device-to-host copy, no
// allocation); false with *err set on a CUDA failure.
bool graph_read_job(poa_graph *g, Job *out, std::string *err) {
  try {
    g->sync();
    *out = g->h;
    return true;
  } catch (const CudaError &e) {
    *err = std::string(cudaGetErrorString(e.code)) + " (" + e.where + ")";
    return false;
  }
}

// Clears a device-side error status left on the graph descriptor.
bool graph_clear_status(poa_graph *g, std::string *err) {
  try {
    g->h.status = ST_OK;
    g->upload();
    return true;
  } catch (const CudaError &e) {
    *err = std::string(cudaGetErrorString(e.code)) + " (" + e.where + ")";
    return false;
  }
}

}  // namespace poa
