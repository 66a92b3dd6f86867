// Internal interface between the host runtime and the device kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "poa_device.cuh"

namespace poa {

// Launchers (poa_kernels.cu). All are asynchronous on `stream`.
// `sched` holds sched_words(n_jobs) zeroed int32 words: the queue head, the
// per-SM and per-level counters that spread the first jobs over the SMs, and
// one claim flag per queue position.
constexpr int SCHED_SM_SLOTS = 512, SCHED_LEVELS = 64;
inline size_t sched_words(size_t n_jobs) { return 4 + SCHED_SM_SLOTS + SCHED_LEVELS + n_jobs; }
// Sets the batched kernel's launch attributes (once per process); launch_batch
// calls it, and a caller capturing a launch into a CUDA graph calls it first.
cudaError_t prepare_batch_kernel();
cudaError_t launch_batch(const Job *jobs_dev, const int32_t *order, int n_jobs, int32_t *sched, int num_sms,
                         const DevParams &P, char *arenas, int64_t slot_bytes, int slots, cudaStream_t stream);
cudaError_t launch_extend_step(Job *job_dev, const DevParams &P, char *arena, int64_t bytes, int read,
                               cudaStream_t stream);
// The read loop of one job (its remaining reads, then the exact rank order)
// by the batched kernel in one 4-warp block: a job marked giant gets the
// other three warps as helpers for its DP rows. `order_sched` holds
// 4 + sched_words(1) zeroed int32 words (the queue order [0], then the
// scheduler words); the job's descriptor names its reads and its arena.
cudaError_t launch_single(Job *job_dev, int32_t *order_sched, int num_sms, const DevParams &P, cudaStream_t stream);
cudaError_t launch_extend_range(Job *job_dev, const DevParams &P, char *arena, int64_t bytes, const uint8_t *reads,
                                const int64_t *read_off, const int32_t *read_len, int r0, int r1,
                                cudaStream_t stream);
cudaError_t launch_align(Job *job_dev, const DevParams &P, char *arena, int64_t bytes, const uint8_t *q, int qlen,
                         int mode, int beg_id, int end_id, int adaptive, uint64_t band_b, int retry, int4 *out,
                         int32_t *out_n, cudaStream_t stream);
// One warp per seed window of a read (win: beg, end, qbeg, qlen | adaptive << 31).
cudaError_t launch_windows(Job *job_dev, const DevParams &P, char *arenas, int64_t slot_bytes, int n_win,
                           const int4 *win, const uint64_t *band, const uint8_t *query, int4 *items,
                           const int64_t *item_off, int32_t *out_n, int32_t *out_st, cudaStream_t stream);
// mark: n_nodes words of scratch for the warp path's distinct-node check
// (nullptr: nodes must come in strictly increasing rank order, else the
// serial add_path runs)
cudaError_t launch_add_path(Job *job_dev, const DevParams &P, int seq_id, int4 *items, int n,
                            cudaStream_t stream, int32_t *mark = nullptr);
cudaError_t launch_add_node(Job *job_dev, int sigma, int base, cudaStream_t stream);
cudaError_t launch_add_edge(Job *job_dev, int from, int to, cudaStream_t stream);
cudaError_t launch_toposort(Job *job_dev, char *arena, int64_t bytes, cudaStream_t stream);
cudaError_t launch_reset(Job *jobs_dev, int n_jobs, int sigma, int unknown, cudaStream_t stream);

// Job queue of the serving kernel, in device memory. The host publishes a
// job by writing its descriptor's address into slot[tail % SERVE_QCAP] and
// then raising tail (two copies in order on one stream); a warp claims the
// entry at head with a compare-and-swap while head != tail. Bit 0 of a slot
// marks a job to be reset to Graph::new first (descriptors are 256-byte
// aligned). stop = 1: warps leave once the queue is empty; 2: at once.
constexpr uint32_t SERVE_QCAP = 1u << 16;
constexpr int SERVE_WARPS_PER_SM = 7;  // one warp's registers stay free on each SM for output kernels
struct ServeQueue {
  uint32_t head, tail, stop, pad;
  unsigned long long slot[SERVE_QCAP];
};
// The batched kernel in serving mode (persistent): SERVE_WARPS_PER_SM warps
// per SM claim jobs from the queue and run their reads until the host sets
// stop; as a bound, a warp also leaves after SERVE_IDLE_LIMIT_NS without a
// job or SERVE_MAX_POLLS empty polls.
constexpr uint64_t SERVE_IDLE_LIMIT_NS = 10000000000ull;
constexpr int SERVE_MAX_POLLS = 1 << 20;
cudaError_t launch_serve(ServeQueue *q, int num_sms, const DevParams &P, cudaStream_t stream);
int kernel_launches_per_batch();
// Warps of the batched kernel resident on one SM (its blocks per SM x warps per block).
int batch_resident_warps_per_sm();

}  // namespace poa
