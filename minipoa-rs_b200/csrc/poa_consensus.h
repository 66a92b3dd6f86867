// Device consensus of resident graphs (poa_consensus.cu).
#pragma once
#include <cuda_runtime.h>

#include "poa_device.cuh"

namespace poa {
// Scratch bytes one graph of n_nodes nodes and n_edges edges needs.
int64_t consensus_scratch_bytes(int64_t n_nodes, int64_t n_edges);
// One warp per job: the consensus bases of job w (decoded through `decode`,
// 256 entries) at out + out_off[w] (room for n_nodes bytes), their count in
// out_len[w] (-1 for a job whose status is not ok). scratch + scr_off[w]
// holds consensus_scratch_bytes of job w.
cudaError_t launch_consensus(const Job *jobs_dev, int n_jobs, const uint8_t *decode, char *scratch,
                             const int64_t *scr_off, uint8_t *out, const int64_t *out_off, int32_t *out_len,
                             cudaStream_t stream);
}  // namespace poa
