#pragma once
#include <cuda_runtime.h>

#include "poa_device.cuh"

namespace poa {
__host__ __device__ int64_t packed_words(const Job &J, int sigma);
cudaError_t launch_pack(const Job *jobs_dev, const int32_t *ids, int n_ids, const int64_t *offsets, int32_t *out,
                        int sigma, cudaStream_t stream);
// One large job packed by many blocks; part holds 2 int64 per block
// (at most kPackOneMaxBlocks blocks).
constexpr int kPackOneMaxBlocks = 4 * 148;
cudaError_t launch_pack_one(const Job *job_dev, int n_nodes, int64_t *part, int32_t *out, int sigma,
                            cudaStream_t stream);
}  // namespace poa
