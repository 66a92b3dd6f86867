// The batched read-loop kernel in its wide form (DP bands up to 2048 columns
// through striped 512-column segments), alone in its translation unit so
// that the compiler inlines the whole read loop into it as it does for the
// narrow form.
#define POA_BATCH_WIDE 1
#include "poa_batch.cuh"

namespace poa {

cudaError_t prepare_batch_wide(int smem_bytes) {
  return cudaFuncSetAttribute(k_batch_wide, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
}

void launch_batch_wide(dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Job *jobs, const int32_t *order,
                       int n_jobs, int32_t *sched, int num_sms, const DevParams &P, char *arenas, int64_t slot_bytes,
                       int slots, ServeQueue *serve) {
  k_batch_wide<<<grid, block, smem, stream>>>(jobs, order, n_jobs, sched, num_sms, P, arenas, slot_bytes, slots,
                                              serve);
}

}  // namespace poa
