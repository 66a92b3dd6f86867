// Heaviest-path consensus of device-resident graphs (Graph::consensus,
// minipoa-rs src/graph.rs:181-237), one warp per graph, so a batch's
// consensus sequences leave the GPU instead of its whole graphs.
//
// The reference walks the graph in FIFO Kahn order from the source and gives
// each node the incoming edge of largest weight, ties to the predecessor of
// larger accumulated score, then to the earlier incoming index; it stops
// when the sink is dequeued. A node's choice reads only its predecessors'
// scores, which are final once those predecessors are dequeued, so any
// topological order yields the same choices, provided the same nodes take
// part: a node is visited iff it is the source or it has incoming edges and
// all its predecessors were visited (its in-degree reaches zero in the FIFO
// walk). The kernel therefore walks the graph's resident rank order (a
// topological order) and marks visited nodes, then follows the choices back
// from the sink.
#include "poa_consensus.h"

namespace poa {

namespace {

// Per-graph scratch, carved from `scratch`: score[n] (u64), prev[n] (i32),
// visited[n] (u8), list_off[n + 1] (i32), list[n_edges] (pred, weight).
__host__ __device__ inline int64_t scratch_bytes(int64_t n, int64_t e) {
  auto up = [](int64_t x) { return (x + 15) / 16 * 16; };
  return up(n * 8) + up(n * 4) + up(n) + up((n + 1) * 4) + up(e * 8);
}

__global__ void k_consensus(const Job *jobs, int n_jobs, const uint8_t *decode, char *scratch,
                            const int64_t *scr_off, uint8_t *out, const int64_t *out_off, int32_t *out_len) {
  const int lane = threadIdx.x & 31;
  const int w = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
  if (w >= n_jobs) return;
  const Job &J = jobs[w];
  if (J.status != ST_OK) {
    if (lane == 0) out_len[w] = -1;
    return;
  }
  const int n = J.n_nodes;
  auto up = [](int64_t x) { return (x + 15) / 16 * 16; };
  char *base = scratch + scr_off[w];
  uint64_t *score = reinterpret_cast<uint64_t *>(base);
  int32_t *prev = reinterpret_cast<int32_t *>(base + up(int64_t(n) * 8));
  uint8_t *visited = reinterpret_cast<uint8_t *>(base + up(int64_t(n) * 8) + up(int64_t(n) * 4));
  int32_t *loff = reinterpret_cast<int32_t *>(base + up(int64_t(n) * 8) + up(int64_t(n) * 4) + up(n));
  int2 *list = reinterpret_cast<int2 *>(base + up(int64_t(n) * 8) + up(int64_t(n) * 4) + up(n) +
                                        up((int64_t(n) + 1) * 4));
  // incoming lists in rank order, flattened (warp prefix sums over 32 ranks)
  int at = 0;
  for (int r0 = 0; r0 < J.n_rank; r0 += 32) {
    const int r = r0 + lane;
    int v = -1, cnt = 0;
    if (r < J.n_rank) {
      v = J.rank_to_node[r];
      cnt = J.in_cnt[v];
    }
    int inc = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int x = __shfl_up_sync(FULL, inc, d);
      if (lane >= d) inc += x;
    }
    if (r < J.n_rank) {
      const int o = at + inc - cnt;
      loff[r] = o;
      int k = 0;
      for (int ch = J.in_head[v]; k < cnt; ch = J.chunk_next[ch])
        for (int s = 0; s < CHUNK && k < cnt; ++s, ++k)
          list[o + k] = make_int2(J.chunk_id[int64_t(ch) * CHUNK + s], J.chunk_w[int64_t(ch) * CHUNK + s]);
    }
    at += __shfl_sync(FULL, inc, 31);
  }
  if (lane == 0) loff[J.n_rank] = at;
  for (int v = lane; v < n; v += 32) {
    visited[v] = 0;
    prev[v] = -1;
    score[v] = 0;
  }
  __syncwarp();
  if (lane == 0) {
    // the walk in rank order (src/graph.rs:182-210)
    for (int r = 0; r < J.n_rank; ++r) {
      const int v = J.rank_to_node[r];
      const int lo = loff[r], hi = loff[r + 1];
      if (v != 0) {
        if (hi == lo) continue;  // no incoming edge: never dequeued
        bool all = true;
        int best = -1, bw = 0;
        uint64_t bs = 0;
        for (int k = lo; k < hi; ++k) {
          const int2 pw = list[k];
          if (!visited[pw.x]) {
            all = false;
            break;
          }
          const uint64_t sk = score[pw.x];
          // strictly heavier, or equal weight and strictly higher score; the
          // earlier index keeps full ties
          if (best < 0 || pw.y > bw || (pw.y == bw && sk > bs)) {
            best = pw.x;
            bw = pw.y;
            bs = sk;
          }
        }
        if (!all) continue;
        prev[v] = best;
        score[v] = bs + uint64_t(bw);
      }
      visited[v] = 1;
      if (v == 1) break;
    }
    // back from the sink (src/graph.rs:211-219): ids reversed into out
    int len = 0;
    for (int cur = prev[1]; cur > 0; cur = prev[cur]) ++len;
    uint8_t *o = out + out_off[w];
    int k = len;
    for (int cur = prev[1]; cur > 0; cur = prev[cur]) o[--k] = decode[J.base[cur]];
    out_len[w] = len;
  }
}

}  // namespace

int64_t consensus_scratch_bytes(int64_t n_nodes, int64_t n_edges) { return scratch_bytes(n_nodes, n_edges); }

cudaError_t launch_consensus(const Job *jobs_dev, int n_jobs, const uint8_t *decode, char *scratch,
                             const int64_t *scr_off, uint8_t *out, const int64_t *out_off, int32_t *out_len,
                             cudaStream_t stream) {
  if (n_jobs <= 0) return cudaSuccess;
  const int threads = 128;
  const int blocks = int((int64_t(n_jobs) * 32 + threads - 1) / threads);
  k_consensus<<<blocks, threads, 0, stream>>>(jobs_dev, n_jobs, decode, scratch, scr_off, out, out_off, out_len);
  return cudaGetLastError();
}

}  // namespace poa
