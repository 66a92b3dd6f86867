// The persistent batched read-loop kernel and the device pieces shared with
// the other kernels: one warp per job, blocks of WARPS_PER_BLOCK independent
// warps, each with its own slice of dynamic shared memory. The kernel comes
// in two DP row forms, each defined by the translation unit that includes
// this header with POA_BATCH_WIDE set: 0 (poa_kernels.cu, k_batch: bands up
// to 512 columns through the striped tiles) or 1 (poa_batch_wide.cu,
// k_batch_wide: up to 2048 in 512-column segments). Each is a plain kernel
// alone with its read loop, which the compiler then inlines whole.
#pragma once
#include "poa_internal.h"

#ifndef POA_BATCH_WIDE
#error "define POA_BATCH_WIDE (0 or 1) before including poa_batch.cuh"
#endif
#if POA_BATCH_WIDE
#define POA_K_BATCH k_batch_wide
#else
#define POA_K_BATCH k_batch
#endif

namespace poa {

constexpr int WARPS_PER_BLOCK = 8;
// One 8-warp block of the batched kernel fills one SM's 228 KB of shared
// memory (1 KB of it is reserved per block), matching __launch_bounds__; a
// giant job alone on its SM then has the whole SM's shared memory as its ring
// and three block-mates as helpers.
constexpr int BLOCKS_PER_SM = 1;
static_assert(BLOCKS_PER_SM * (WARPS_PER_BLOCK * sizeof(WarpSmem) + 1024) <= 228 * 1024,
              "WarpSmem too large for the blocks per SM");

__device__ __forceinline__ WarpSmem *warp_smem() {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  return reinterpret_cast<WarpSmem *>(dyn_smem) + (threadIdx.x >> 5);
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Serving mode: lane 0 claims the next queue entry (0 when the warp is to
// leave). An idle warp keeps polling, sleeping between empty polls (1 us,
// doubling to 32 us), until the host sets stop, so a job published at any
// time finds a warp; the host ends the kernel that way once the server has
// been idle a while. Every wait is bounded: a warp also leaves after
// SERVE_IDLE_LIMIT_NS without a job or SERVE_MAX_POLLS empty polls.
__device__ inline unsigned long long serve_claim(ServeQueue *q) {
  unsigned long long entry = 0;
  if ((threadIdx.x & 31) == 0) {
    const uint64_t t0 = globaltimer_ns();
    unsigned sleep_ns = 1000;
    for (int polls = 0;; ++polls) {
      const uint32_t stop = *reinterpret_cast<volatile uint32_t *>(&q->stop);
      if (stop >= 2) break;
      const uint32_t h = *reinterpret_cast<volatile uint32_t *>(&q->head);
      const uint32_t t = *reinterpret_cast<volatile uint32_t *>(&q->tail);
      if (h != t) {
        if (atomicCAS(&q->head, h, h + 1) == h) {
          __threadfence();
          entry = *reinterpret_cast<volatile unsigned long long *>(&q->slot[h & (SERVE_QCAP - 1)]);
          break;
        }
        continue;
      }
      if (stop == 1 || polls >= SERVE_MAX_POLLS || globaltimer_ns() - t0 > SERVE_IDLE_LIMIT_NS) break;
      __nanosleep(sleep_ns);
      if (sleep_ns < 32000) sleep_ns *= 2;
    }
  }
  return __shfl_sync(FULL, entry, 0);
}

// Runs a job's remaining reads on the calling warp (read loop, then the
// exact rank order), stores its status and raises its completion flag. A job
// that outgrows its arena parks at its current read (graph untouched).
// (in an unnamed namespace: each translation unit has its own form)
namespace {
constexpr bool kBatchWide = POA_BATCH_WIDE != 0;

__device__ inline void run_job(Job *J, const DevParams &P, char *arena, int64_t slot_bytes, WarpSmem *sm) {
  const int lane = threadIdx.x & 31;
  const int n_reads = J->n_reads;
  char *ja = J->arena ? J->arena : arena;
  const int64_t jb = J->arena ? J->arena_bytes : slot_bytes;
  int32_t st = ST_OK;
  for (int r = J->next_read; r < n_reads; ++r) {
    st = extend_one<kBatchWide>(J, P, ja, jb, J->reads + J->read_off[r], J->read_len[r], r, sm);
    if (st != ST_OK) break;
  }
  // a finished (or failed) job ends with the reference's exact rank order;
  // a parked job keeps its order for the next pass
  if (lane == 0) {
    if (st == ST_OK || is_alignment_error(st)) {
      const int32_t fs = finalize_order(J, ja, jb);
      if (st == ST_OK) st = fs;
    }
    J->status = st;
    if (J->done_flag) {
      __threadfence_system();  // the descriptor before the flag the host polls
      *reinterpret_cast<volatile int32_t *>(J->done_flag) = 1;
    }
  }
  __syncwarp();
}

}  // namespace

// Graph::new for one job (graph.rs:27-40: source and sink) and its counters.
__device__ inline void reset_job(Job *J, int sigma, int unknown) {
  J->n_nodes = 0;
  J->n_chunks = 0;
  J->n_edges = 0;
  J->n_paths = 0;
  J->path_used = 0;
  J->n_rank = 0;
  J->path_off[0] = 0;
  add_node(J, sigma, unknown);
  add_node(J, sigma, unknown);
  J->next_read = 0;
  J->seq_base = 0;
  J->status = ST_OK;
  J->err_i = J->err_j = 0;
  J->n_items = 0;
  J->cells = 0;
  J->dp_bytes = 0;
  J->pred_cells = 0;
  J->far_preds = 0;
  J->rows_g4 = 0;
  J->rows_generic = 0;
  J->coop = 0;
  J->wave_reads = 0;
  for (int k = 0; k < 4; ++k) J->phase[k] = 0;
  J->order_exact = 1;
}

// Persistent batched kernel: each warp takes jobs from a size-ordered queue
// (largest first) and runs their remaining reads. A job that outgrows the
// warp's DP arena parks at its current read (graph untouched) for a later
// pass with larger arenas. The first job of every warp is placed so that the
// largest jobs land on different SMs: the k-th warp to start on an SM takes
// one of the positions [k * num_sms, (k + 1) * num_sms), in the order the SMs
// reach that level; every later job comes from the shared queue, and a claim
// flag per position makes each job run exactly once. A giant job (marked by
// the host: one of the largest, far above the average share, at most one per
// SM) takes three adjacent block-mates as helpers for its DP rows and their
// shared memory as its ring; the block's other warps keep taking jobs, and
// the helpers join them when the giant job is done.
__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32, BLOCKS_PER_SM)
    POA_K_BATCH(Job *jobs, const int32_t *order, int n_jobs, int32_t *sched, int num_sms, DevParams P, char *arenas,
            int64_t slot_bytes, int slots, ServeQueue *serve) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  // the grid is rounded up to whole blocks; warps past the last slot own no
  // arena (they leave after the block's start-up barrier)
  const bool active = warp < slots;
  // (teams: one arena per block, the job's warp 0 uses it)
  char *arena = arenas + (P.teams ? int64_t(blockIdx.x) : warp) * slot_bytes;
  WarpSmem *sm = warp_smem();
  int32_t *queue = sched;
  int32_t *sm_count = sched + 4;
  int32_t *level_count = sm_count + SCHED_SM_SLOTS;
  int32_t *claim = level_count + SCHED_LEVELS;
  unsigned smid = 0;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
  const bool sm_ok = smid < unsigned(SCHED_SM_SLOTS);
  __shared__ int block_giant, giant_warp, firsts[WARPS_PER_BLOCK];
  if (threadIdx.x == 0) {
    block_giant = 0;
    giant_warp = -1;
  }
  ring_default(sm);
  __syncthreads();
  int first = -1, first_giant = 0;
  if (P.teams) {
    // team launch (a small batch): block b is job b's team, the job on warp
    // 0 and the other three warps its helpers; no job comes from the queue
    if (!serve && active && lane == 0 && (threadIdx.x >> 5) == 0 && blockIdx.x < unsigned(n_jobs)) {
      first = int(blockIdx.x);
      first_giant = 1;
      atomicAdd(&block_giant, 1);
      giant_warp = 0;
    }
  } else if (!serve && active && lane == 0 && sm_ok) {
    const int level = atomicAdd(&sm_count[smid], 1);
    if (level < SCHED_LEVELS) {
      const int64_t p0 = int64_t(level) * num_sms + atomicAdd(&level_count[level], 1);
      if (p0 < n_jobs) {
        first = int(p0);
        first_giant = jobs[order[p0]].giant;
        if (first_giant) {
          atomicAdd(&block_giant, 1);
          giant_warp = int(threadIdx.x >> 5);
        }
      }
    }
  }
  if (lane == 0) firsts[threadIdx.x >> 5] = first;
  __syncthreads();
  // a giant gets three adjacent block-mates as helpers for its DP rows
  // (cooperative rows) and their slices of shared memory as its ring (M,
  // then D); every warp of the block sees the same block_giant and
  // giant_warp. Warps past the last slot serve as helpers too: a helper
  // needs no arena while it helps.
  const int me = int(threadIdx.x >> 5), wpb = int(blockDim.x >> 5);
  int lead = giant_warp;
  int h0 = giant_warp < 0 ? -1 : (giant_warp + 3 < wpb ? giant_warp + 1 : (giant_warp >= 3 ? giant_warp - 3 : -1));
  if (block_giant == 1 && wpb == 8 && int64_t(blockIdx.x) * wpb + 4 < slots) {
    // in a full 8-warp block the giant runs on warp 4 with warps 0-2 as
    // helpers: warps map to the SM's four sub-partitions by index mod 4, so
    // the giant shares its sub-partition with a helper, which is parked
    // while the giant runs its band guides and traceback. Warp 4 and the
    // giant's warp swap their first jobs.
    lead = 4;
    h0 = 0;
    if (me == 4 && giant_warp != 4) {
      first = firsts[giant_warp];
      first_giant = 1;
    } else if (me == giant_warp && giant_warp != 4) {
      first = firsts[4];
      first_giant = 0;
    }
  }
  if (block_giant == 1 && wpb == 4 && int64_t(blockIdx.x) * wpb < slots) {
    // a 4-warp block (a single job run with helpers): the giant runs on warp
    // 0 with warps 1-3 as helpers, whichever warp drew it
    lead = 0;
    h0 = 1;
    if (me == 0 && giant_warp != 0) {
      first = firsts[giant_warp];
      first_giant = 1;
    } else if (me == giant_warp && giant_warp != 0) {
      first = firsts[0];
      first_giant = 0;
    }
  }
  const bool coop_block = block_giant == 1 && h0 >= 0;
  if (coop_block && me >= h0 && me < h0 + 3) {
    WarpSmem *leader = reinterpret_cast<WarpSmem *>(sm) - me + lead;
    coop_helper(reinterpret_cast<CoopDesc *>(leader->ring_m), me - h0 + 1);
    // released: the slice is this warp's own again, and it takes jobs from
    // the shared queue (its start position went to the queue)
    if (!active) return;
    ring_default(sm);
    first = -1;
    first_giant = 0;
  } else if (!active) {
    return;
  }
  // giant_alone: the giant's SM keeps only its team (the giant and its
  // helpers, which take other jobs once it is done); the block's other warps
  // leave, and their first positions, left unclaimed, go to the shared queue
  if (P.giant_alone && coop_block && me != lead && !(me >= h0 && me < h0 + 3)) return;
  first = __shfl_sync(FULL, first, 0);
  first_giant = __shfl_sync(FULL, first_giant, 0);
  if (first_giant && coop_block) {
    WarpSmem *base = reinterpret_cast<WarpSmem *>(sm) - me + h0;
    const int cap = int(3 * sizeof(WarpSmem) / 8 / 8 * 8);
    if (lane == 0) {
      sm->rv.m = reinterpret_cast<int32_t *>(base);
      sm->rv.d = reinterpret_cast<int32_t *>(base) + cap;
      sm->rv.cap = cap;
      sm->rv.pad[0] = 1;  // cooperative rows for the first (giant) job
    }
    __syncwarp();
  }
  if (lane == 0 && first >= 0 && atomicExch(&claim[first], 1) != 0) first = -1;
  first = __shfl_sync(FULL, first, 0);
  for (;;) {
    Job *J = nullptr;
    if (serve) {
      // serving mode: the next job the host published (jobs carry their own
      // DP arena); bit 0 of the entry asks for Graph::new first
      const unsigned long long entry = serve_claim(serve);
      if (entry == 0) break;
      J = reinterpret_cast<Job *>(entry & ~1ull);
      if ((entry & 1ull) && lane == 0) reset_job(J, P.sigma, P.unknown);
      __syncwarp();
    } else {
      int q = first;
      first = -1;
      if (q < 0 && P.teams) break;  // a team runs its own job only
      if (q < 0) {
        if (lane == 0) {
          do {
            q = atomicAdd(queue, 1);
          } while (q < n_jobs && atomicExch(&claim[q], 1) != 0);
        }
        q = __shfl_sync(FULL, q, 0);
        if (q >= n_jobs) break;
      }
      J = jobs + order[q];
    }
    run_job(J, P, arena, slot_bytes, sm);
    // the giant job is done: the helpers go back to the queue
    if (sm->rv.pad[0]) coop_release(sm);
  }
  // no job at all (the first position was claimed elsewhere and the queue is
  // empty): the helpers still wait for their release
  if (sm->rv.pad[0]) coop_release(sm);
}

// The wide form, compiled in poa_batch_wide.cu: its shared-memory attribute
// and a launch with the batched kernel's arguments.
cudaError_t prepare_batch_wide(int smem_bytes);

void launch_batch_wide(dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Job *jobs, const int32_t *order,
                       int n_jobs, int32_t *sched, int num_sms, const DevParams &P, char *arenas, int64_t slot_bytes,
                       int slots, ServeQueue *serve);

}  // namespace poa
