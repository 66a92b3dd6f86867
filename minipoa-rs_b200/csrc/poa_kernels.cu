// Kernels of the B200 POA library: the persistent batched read-loop kernel,
// the plain one-read-per-launch kernel, and the single-graph operations behind
// the reference-shaped C ABI. One warp per job; blocks of WARPS_PER_BLOCK
// independent warps, each with its own slice of dynamic shared memory.
#define POA_BATCH_WIDE 0
#include "poa_batch.cuh"

namespace poa {

// Plain form: one launch aligns one read of one job.
__global__ void k_extend_step(Job *J, DevParams P, char *arena, int64_t bytes, int r) {
  if (J->status != ST_OK || J->next_read != r) return;
  ring_default(warp_smem());
  int32_t st = extend_one(J, P, arena, bytes, J->reads + J->read_off[r], J->read_len[r], r, warp_smem());
  if ((threadIdx.x & 31) == 0) {
    if ((st == ST_OK && r + 1 == J->n_reads) || is_alignment_error(st)) {
      const int32_t fs = finalize_order(J, arena, bytes);
      if (st == ST_OK) st = fs;
    }
    if (st != ST_OK) J->status = st;
  }
}

// extend_graph over reads r0..r1-1 held in a caller buffer.
__global__ void k_extend_range(Job *J, DevParams P, char *arena, int64_t bytes, const uint8_t *reads,
                               const int64_t *read_off, const int32_t *read_len, int r0, int r1) {
  int32_t st = ST_OK;
  ring_default(warp_smem());
  for (int r = r0; r < r1; ++r) {
    st = extend_one(J, P, arena, bytes, reads + read_off[r], read_len[r], r, warp_smem());
    if (st != ST_OK) break;
  }
  if ((threadIdx.x & 31) == 0) {
    if (st == ST_OK || is_alignment_error(st)) {
      const int32_t fs = finalize_order(J, arena, bytes);
      if (st == ST_OK) st = fs;
    }
    if (st != ST_OK) J->status = st;
  }
}

// align::align (mode 0) or align::poa / poa_inner (mode 1) without modifying
// the graph; the path is copied to `out`.
__global__ void k_align(Job *J, DevParams P, char *arena, int64_t bytes, const uint8_t *q, int qlen, int mode,
                        int beg_id, int end_id, int adaptive, uint64_t band_b, int retry, int4 *out,
                        int32_t *out_n) {
  const int lane = threadIdx.x & 31;
  Scratch s;
  int n_items = 0;
  Work cells{};
  int32_t st;
  ring_default(warp_smem());
  if (mode == 0) {
    st = align_query(J, P, arena, bytes, q, qlen, s, &n_items, &cells, warp_smem());
  } else if (retry) {
    st = poa_retry<true>(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive != 0, band_b, s, &n_items, &cells,
                   warp_smem());
  } else {
    st = poa_inner<true>(J, P, arena, bytes, beg_id, end_id, q, qlen, adaptive != 0, band_b, P.f, s, &n_items, &cells,
                   warp_smem());
  }
  if (st == ST_OK)
    for (int k = lane; k < n_items; k += 32) out[k] = s.items[k];
  if (lane == 0) {
    J->status = st;
    *out_n = st == ST_OK ? n_items : 0;
    if (st == ST_OK) {
      J->cells += cells.cells;
      J->dp_bytes += cells.dp_bytes;
    }
  }
}

// The seed windows of one read (align.rs:99-164), one 4-warp team per
// window: block w aligns query[qbeg, qbeg + qlen) between anchor nodes beg
// (included) and end (excluded) with the full-DP retry, in its own arena
// slice, and writes its path to items[item_off[w] ...]; warp 0 runs the
// alignment and warps 1-3 help with its DP rows (cooperative rows, their
// shared memory the ring). The graph is only read.
__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32, BLOCKS_PER_SM)
    k_windows(Job *J, DevParams P, char *arenas, int64_t slot_bytes, int n_win, const int4 *win,
              const uint64_t *band, const uint8_t *query, int4 *items, const int64_t *item_off, int32_t *out_n,
              int32_t *out_st) {
  const int lane = threadIdx.x & 31;
  const int64_t w = blockIdx.x;
  if (w >= n_win) return;
  WarpSmem *sm = warp_smem();
  ring_default(sm);
  const int me = int(threadIdx.x >> 5);
  if (me > 0) {  // a helper: rows of the window's row loops until released
    coop_helper(reinterpret_cast<CoopDesc *>((sm - me)->ring_m), me);
    return;
  }
  if (lane == 0) {
    const int cap = int(3 * sizeof(WarpSmem) / 8 / 8 * 8);
    sm->rv.m = reinterpret_cast<int32_t *>(sm + 1);
    sm->rv.d = reinterpret_cast<int32_t *>(sm + 1) + cap;
    sm->rv.cap = cap;
    sm->rv.pad[0] = 1;  // cooperative rows
  }
  __syncwarp();
  const int4 d = win[w];  // (beg, end, qbeg, qlen | adaptive << 31)
  const bool adaptive = (unsigned(d.w) >> 31) != 0;
  const int qlen = d.w & 0x7fffffff;
  Scratch s;
  int n_items = 0;
  Work cells{};
  const int32_t st = poa_retry<true>(J, P, arenas + w * slot_bytes, slot_bytes, d.x, d.y, query + d.z, qlen, adaptive,
                               band[w], s, &n_items, &cells, sm);
  coop_release(sm);  // the helpers leave
  if (st == ST_OK)
    for (int k = lane; k < n_items; k += 32) items[item_off[w] + k] = s.items[k];
  if (lane == 0) {
    out_n[w] = st == ST_OK ? n_items : 0;
    out_st[w] = st;
    if (st == ST_OK) {
      atomicAdd(reinterpret_cast<unsigned long long *>(&J->cells), (unsigned long long)cells.cells);
      atomicAdd(reinterpret_cast<unsigned long long *>(&J->dp_bytes), (unsigned long long)cells.dp_bytes);
    }
  }
}

__global__ void k_add_path(Job *J, DevParams P, int seq_id, int4 *items, int n, int32_t *mark) {
  int32_t st = ST_OK;
  if (!add_path_warp(J, P, seq_id, items, n, &st, mark) && threadIdx.x == 0) st = add_path(J, P, seq_id, items, n);
  if (threadIdx.x == 0) J->status = st;
}

__global__ void k_add_node(Job *J, int sigma, int base) {
  if (threadIdx.x == 0) {
    if (J->n_nodes + 1 > J->node_cap) {
      J->status = ST_GRAPH_FULL;
      return;
    }
    J->err_i = add_node(J, sigma, base);
    J->status = ST_OK;
  }
}

__global__ void k_add_edge(Job *J, int from, int to) {
  if (threadIdx.x == 0) {
    if (J->n_chunks + 2 > J->chunk_cap) {
      J->status = ST_GRAPH_FULL;
      return;
    }
    add_edge(J, from, to);
    J->status = ST_OK;
  }
}

__global__ void k_toposort(Job *J, char *arena, int64_t bytes) {
  if (threadIdx.x == 0) {
    if (int64_t(J->n_nodes) * 8 > bytes) {
      J->status = ST_ARENA_FULL;
      return;
    }
    int32_t *deg = reinterpret_cast<int32_t *>(arena);
    J->status = toposort(J, deg, deg + J->n_nodes);
    J->order_exact = 1;
  }
}

// Graph::new (graph.rs:30-40) for every job: source and sink, no edges, no
// rank, no paths; the read loop restarts at read 0.
__global__ void k_reset(Job *jobs, int n_jobs, int sigma, int unknown) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n_jobs) reset_job(jobs + j, sigma, unknown);
}

cudaError_t prepare_batch_kernel() {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(WARPS_PER_BLOCK * sizeof(WarpSmem)));
    if (e != cudaSuccess) return e;
    e = prepare_batch_wide(int(WARPS_PER_BLOCK * sizeof(WarpSmem)));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  return cudaSuccess;
}

namespace {
// The batched kernel in the form the parameters ask for.
void batch_kernel(const DevParams &P, dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Job *jobs,
                  const int32_t *order, int n_jobs, int32_t *sched, int num_sms, char *arenas, int64_t slot_bytes,
                  int slots, ServeQueue *serve) {
  if (P.wide_rows)
    launch_batch_wide(grid, block, smem, stream, jobs, order, n_jobs, sched, num_sms, P, arenas, slot_bytes, slots,
                      serve);
  else
    k_batch<<<grid, block, smem, stream>>>(jobs, order, n_jobs, sched, num_sms, P, arenas, slot_bytes, slots, serve);
}
}  // namespace

cudaError_t launch_batch(const Job *jobs_dev, const int32_t *order, int n_jobs, int32_t *sched, int num_sms,
                         const DevParams &P, char *arenas, int64_t slot_bytes, int slots, cudaStream_t stream) {
  // fewer slots than a full machine: narrower blocks, so that the warps
  // spread over all SMs instead of filling a few
  int wpb = WARPS_PER_BLOCK;
  if (num_sms > 0 && slots < num_sms * WARPS_PER_BLOCK) wpb = std::max(1, (slots + num_sms - 1) / num_sms);
  if (P.teams) wpb = 4;  // one block per job: the job and its three helpers
  const int blocks = (slots + wpb - 1) / wpb;
  const cudaError_t pe = prepare_batch_kernel();
  if (pe != cudaSuccess) return pe;
  batch_kernel(P, blocks, wpb * 32, wpb * sizeof(WarpSmem), stream, const_cast<Job *>(jobs_dev), order, n_jobs, sched,
               num_sms, arenas, slot_bytes, slots, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_single(Job *job_dev, int32_t *order_sched, int num_sms, const DevParams &P, cudaStream_t stream) {
  const cudaError_t pe = prepare_batch_kernel();
  if (pe != cudaSuccess) return pe;
  batch_kernel(P, 1, 4 * 32, 4 * sizeof(WarpSmem), stream, job_dev, order_sched, 1, order_sched + 4, num_sms,
               nullptr, 0, 4, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_serve(ServeQueue *q, int num_sms, const DevParams &P, cudaStream_t stream) {
  const cudaError_t pe = prepare_batch_kernel();
  if (pe != cudaSuccess) return pe;
  const int slots = num_sms * SERVE_WARPS_PER_SM;
  batch_kernel(P, num_sms, SERVE_WARPS_PER_SM * 32, SERVE_WARPS_PER_SM * sizeof(WarpSmem), stream, nullptr, nullptr, 0,
               nullptr, num_sms, nullptr, 0, slots, q);
  return cudaGetLastError();
}

cudaError_t launch_extend_step(Job *job_dev, const DevParams &P, char *arena, int64_t bytes, int read,
                               cudaStream_t stream) {
  k_extend_step<<<1, 32, sizeof(WarpSmem), stream>>>(job_dev, P, arena, bytes, read);
  return cudaGetLastError();
}

cudaError_t launch_extend_range(Job *job_dev, const DevParams &P, char *arena, int64_t bytes, const uint8_t *reads,
                                const int64_t *read_off, const int32_t *read_len, int r0, int r1,
                                cudaStream_t stream) {
  k_extend_range<<<1, 32, sizeof(WarpSmem), stream>>>(job_dev, P, arena, bytes, reads, read_off, read_len, r0, r1);
  return cudaGetLastError();
}

cudaError_t launch_align(Job *job_dev, const DevParams &P, char *arena, int64_t bytes, const uint8_t *q, int qlen,
                         int mode, int beg_id, int end_id, int adaptive, uint64_t band_b, int retry, int4 *out,
                         int32_t *out_n, cudaStream_t stream) {
  k_align<<<1, 32, sizeof(WarpSmem), stream>>>(job_dev, P, arena, bytes, q, qlen, mode, beg_id, end_id, adaptive,
                                               band_b, retry, out, out_n);
  return cudaGetLastError();
}

cudaError_t launch_windows(Job *job_dev, const DevParams &P, char *arenas, int64_t slot_bytes, int n_win,
                           const int4 *win, const uint64_t *band, const uint8_t *query, int4 *items,
                           const int64_t *item_off, int32_t *out_n, int32_t *out_st, cudaStream_t stream) {
  if (n_win <= 0) return cudaSuccess;
  // one 4-warp team per window (the window's warp and three helpers)
  static bool attr = false;
  if (!attr) {
    const cudaError_t e =
        cudaFuncSetAttribute(k_windows, cudaFuncAttributeMaxDynamicSharedMemorySize, int(4 * sizeof(WarpSmem)));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_windows<<<n_win, 4 * 32, 4 * sizeof(WarpSmem), stream>>>(job_dev, P, arenas, slot_bytes, n_win, win, band, query,
                                                             items, item_off, out_n, out_st);
  return cudaGetLastError();
}

cudaError_t launch_add_path(Job *job_dev, const DevParams &P, int seq_id, int4 *items, int n,
                            cudaStream_t stream, int32_t *mark) {
  k_add_path<<<1, 32, 0, stream>>>(job_dev, P, seq_id, items, n, mark);
  return cudaGetLastError();
}

cudaError_t launch_add_node(Job *job_dev, int sigma, int base, cudaStream_t stream) {
  k_add_node<<<1, 32, 0, stream>>>(job_dev, sigma, base);
  return cudaGetLastError();
}

cudaError_t launch_add_edge(Job *job_dev, int from, int to, cudaStream_t stream) {
  k_add_edge<<<1, 32, 0, stream>>>(job_dev, from, to);
  return cudaGetLastError();
}

cudaError_t launch_toposort(Job *job_dev, char *arena, int64_t bytes, cudaStream_t stream) {
  k_toposort<<<1, 32, 0, stream>>>(job_dev, arena, bytes);
  return cudaGetLastError();
}

cudaError_t launch_reset(Job *jobs_dev, int n_jobs, int sigma, int unknown, cudaStream_t stream) {
  if (n_jobs <= 0) return cudaSuccess;
  k_reset<<<(n_jobs + 127) / 128, 128, 0, stream>>>(jobs_dev, n_jobs, sigma, unknown);
  return cudaGetLastError();
}

int kernel_launches_per_batch() { return 1; }

int batch_resident_warps_per_sm() { return BLOCKS_PER_SM * WARPS_PER_BLOCK; }

}  // namespace poa
