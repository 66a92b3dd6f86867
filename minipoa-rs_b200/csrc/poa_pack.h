#pragma once
#include <cuda_runtime.h>

#include "poa_device.cuh"

namespace poa {
__host__ __device__ int64_t packed_words(const Job &J, int sigma);
cudaError_t launch_pack(const Job *jobs_dev, const int32_t *ids, int n_ids, const int64_t *offsets, int32_t *out,
                        int sigma, cudaStream_t stream);
}  // namespace poa
