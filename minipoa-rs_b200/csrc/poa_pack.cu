// Packs device-resident job graphs into flat int32 records for one
// device-to-host copy. Record layout (words):
//   [0] n_nodes [1] in entries [2] out entries [3] n_paths [4] path items
//   [5] n_rank  [6] sigma
//   base[n] parent[n] rank[n] coverage[n] aligned[n*sigma] rank_to_node[n_rank]
//   in_cnt[n] out_cnt[n] in pairs (id, w) out pairs (id, w)
//   path_seq[n_paths] path_off[n_paths + 1] path_items[path_used]
#include "poa_pack.h"

#include <algorithm>

namespace poa {

__host__ __device__ int64_t packed_words(const Job &J, int sigma) {
  const int64_t n = J.n_nodes;
  int64_t in_e = J.n_edges;
  int64_t out_e = J.n_edges;  // every distinct edge has one in and one out entry
  return 7 + n * (5 + sigma) + J.n_rank + 2 * n + 2 * (in_e + out_e) + J.n_paths * 2 + 1 + J.path_used;
}

// One warp per job.
__global__ void k_pack(const Job *jobs, const int32_t *ids, int n_ids, const int64_t *offsets, int32_t *out,
                       int sigma) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n_ids) return;
  const Job &J = jobs[ids[w]];
  int32_t *o = out + offsets[w];
  const int n = J.n_nodes;
  if (lane == 0) {
    o[0] = n;
    o[1] = J.n_edges;
    o[2] = J.n_edges;
    o[3] = J.n_paths;
    o[4] = J.path_used;
    o[5] = J.n_rank;
    o[6] = sigma;
  }
  int32_t *base = o + 7;
  int32_t *parent = base + n;
  int32_t *rank = parent + n;
  int32_t *cov = rank + n;
  int32_t *al = cov + n;
  int32_t *r2n = al + int64_t(n) * sigma;
  int32_t *icnt = r2n + J.n_rank;
  int32_t *ocnt = icnt + n;
  int32_t *ipairs = ocnt + n;
  int32_t *opairs = ipairs + 2 * int64_t(J.n_edges);
  int32_t *pseq = opairs + 2 * int64_t(J.n_edges);
  int32_t *poff = pseq + J.n_paths;
  int32_t *pit = poff + J.n_paths + 1;
  for (int i = lane; i < n; i += 32) {
    base[i] = J.base[i];
    parent[i] = J.parent[i];
    rank[i] = J.rank[i];
    cov[i] = J.coverage[i];
    icnt[i] = J.in_cnt[i];
    ocnt[i] = J.out_cnt[i];
  }
  for (int64_t i = lane; i < int64_t(n) * sigma; i += 32) al[i] = J.aligned[i];
  for (int i = lane; i < J.n_rank; i += 32) r2n[i] = J.rank_to_node[i];
  for (int i = lane; i < J.n_paths; i += 32) pseq[i] = J.path_seq[i];
  for (int i = lane; i <= J.n_paths; i += 32) poff[i] = J.path_off[i];
  for (int i = lane; i < J.path_used; i += 32) pit[i] = J.path_items[i];
  // edge pairs: warp prefix sums over 32-node groups give each node's offset
  int64_t in_base = 0, out_base = 0;
  for (int g = 0; g < n; g += 32) {
    const int i = g + lane;
    const int ic = i < n ? J.in_cnt[i] : 0;
    const int oc = i < n ? J.out_cnt[i] : 0;
    int is = ic, os = oc;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int a = __shfl_up_sync(FULL, is, d);
      const int b = __shfl_up_sync(FULL, os, d);
      if (lane >= d) {
        is += a;
        os += b;
      }
    }
    if (i < n) {
      int64_t at = in_base + is - ic;
      int ch = J.in_head[i];
      for (int k = 0; k < ic; ch = J.chunk_next[ch])
        for (int s = 0; s < CHUNK && k < ic; ++s, ++k) {
          ipairs[2 * (at + k)] = J.chunk_id[int64_t(ch) * CHUNK + s];
          ipairs[2 * (at + k) + 1] = J.chunk_w[int64_t(ch) * CHUNK + s];
        }
      at = out_base + os - oc;
      ch = J.out_head[i];
      for (int k = 0; k < oc; ch = J.chunk_next[ch])
        for (int s = 0; s < CHUNK && k < oc; ++s, ++k) {
          opairs[2 * (at + k)] = J.chunk_id[int64_t(ch) * CHUNK + s];
          opairs[2 * (at + k) + 1] = J.chunk_w[int64_t(ch) * CHUNK + s];
        }
    }
    in_base += __shfl_sync(FULL, is, 31);
    out_base += __shfl_sync(FULL, os, 31);
  }
}

// One job over many blocks (a single large graph): the first kernel sums
// each block's in/out entry counts, the second copies the node arrays with
// the whole grid and writes each block's edge pairs from the prefix of the
// block sums, scanning its nodes 256 at a time.
namespace {
constexpr int kPackThreads = 256;

__device__ void block_sum2(int64_t &a, int64_t &b, int64_t *sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int d = 16; d; d >>= 1) {
    a += __shfl_xor_sync(FULL, a, d);
    b += __shfl_xor_sync(FULL, b, d);
  }
  if (lane == 0) {
    sh[2 * wid] = a;
    sh[2 * wid + 1] = b;
  }
  __syncthreads();
  a = b = 0;
  for (int w = 0; w < kPackThreads / 32; ++w) {
    a += sh[2 * w];
    b += sh[2 * w + 1];
  }
  __syncthreads();
}
}  // namespace

__global__ void __launch_bounds__(kPackThreads) k_pack_count(const Job *job, int npb, int64_t *part) {
  __shared__ int64_t sh[2 * kPackThreads / 32];
  const Job &J = *job;
  const int lo = blockIdx.x * npb, hi = min(J.n_nodes, lo + npb);
  int64_t a = 0, b = 0;
  for (int i = lo + threadIdx.x; i < hi; i += kPackThreads) {
    a += J.in_cnt[i];
    b += J.out_cnt[i];
  }
  block_sum2(a, b, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = b;
  }
}

__global__ void __launch_bounds__(kPackThreads) k_pack_wide(const Job *job, int npb, const int64_t *part, int32_t *o,
                                                            int sigma) {
  __shared__ int64_t sh[2 * kPackThreads / 32];
  __shared__ int32_t tile[2 * kPackThreads / 32];
  const Job &J = *job;
  const int n = J.n_nodes;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (blockIdx.x == 0 && tid == 0) {
    o[0] = n;
    o[1] = J.n_edges;
    o[2] = J.n_edges;
    o[3] = J.n_paths;
    o[4] = J.path_used;
    o[5] = J.n_rank;
    o[6] = sigma;
  }
  int32_t *base = o + 7;
  int32_t *parent = base + n;
  int32_t *rank = parent + n;
  int32_t *cov = rank + n;
  int32_t *al = cov + n;
  int32_t *r2n = al + int64_t(n) * sigma;
  int32_t *icnt = r2n + J.n_rank;
  int32_t *ocnt = icnt + n;
  int32_t *ipairs = ocnt + n;
  int32_t *opairs = ipairs + 2 * int64_t(J.n_edges);
  int32_t *pseq = opairs + 2 * int64_t(J.n_edges);
  int32_t *poff = pseq + J.n_paths;
  int32_t *pit = poff + J.n_paths + 1;
  const int64_t g0 = int64_t(blockIdx.x) * kPackThreads + tid, gs = int64_t(gridDim.x) * kPackThreads;
  for (int64_t i = g0; i < n; i += gs) {
    base[i] = J.base[i];
    parent[i] = J.parent[i];
    rank[i] = J.rank[i];
    cov[i] = J.coverage[i];
    icnt[i] = J.in_cnt[i];
    ocnt[i] = J.out_cnt[i];
  }
  for (int64_t i = g0; i < int64_t(n) * sigma; i += gs) al[i] = J.aligned[i];
  for (int64_t i = g0; i < J.n_rank; i += gs) r2n[i] = J.rank_to_node[i];
  for (int64_t i = g0; i < J.n_paths; i += gs) pseq[i] = J.path_seq[i];
  for (int64_t i = g0; i <= J.n_paths; i += gs) poff[i] = J.path_off[i];
  for (int64_t i = g0; i < J.path_used; i += gs) pit[i] = J.path_items[i];
  // this block's first in/out entry: the sum of the earlier blocks' counts
  int64_t in_base = 0, out_base = 0;
  for (int k = tid; k < int(blockIdx.x); k += kPackThreads) {
    in_base += part[2 * k];
    out_base += part[2 * k + 1];
  }
  block_sum2(in_base, out_base, sh);
  const int lo = blockIdx.x * npb, hi = min(n, lo + npb);
  for (int t = lo; t < hi; t += kPackThreads) {
    const int i = t + tid;
    const int ic = i < hi ? J.in_cnt[i] : 0;
    const int oc = i < hi ? J.out_cnt[i] : 0;
    int is = ic, os = oc;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int a = __shfl_up_sync(FULL, is, d);
      const int b = __shfl_up_sync(FULL, os, d);
      if (lane >= d) {
        is += a;
        os += b;
      }
    }
    if (lane == 31) {
      tile[2 * wid] = is;
      tile[2 * wid + 1] = os;
    }
    __syncthreads();
    int ti = 0, to = 0, pi = 0, po = 0;
    for (int w = 0; w < kPackThreads / 32; ++w) {
      if (w == wid) {
        pi = ti;
        po = to;
      }
      ti += tile[2 * w];
      to += tile[2 * w + 1];
    }
    __syncthreads();
    if (i < hi) {
      int64_t at = in_base + pi + is - ic;
      int ch = J.in_head[i];
      for (int k = 0; k < ic; ch = J.chunk_next[ch])
        for (int s = 0; s < CHUNK && k < ic; ++s, ++k) {
          ipairs[2 * (at + k)] = J.chunk_id[int64_t(ch) * CHUNK + s];
          ipairs[2 * (at + k) + 1] = J.chunk_w[int64_t(ch) * CHUNK + s];
        }
      at = out_base + po + os - oc;
      ch = J.out_head[i];
      for (int k = 0; k < oc; ch = J.chunk_next[ch])
        for (int s = 0; s < CHUNK && k < oc; ++s, ++k) {
          opairs[2 * (at + k)] = J.chunk_id[int64_t(ch) * CHUNK + s];
          opairs[2 * (at + k) + 1] = J.chunk_w[int64_t(ch) * CHUNK + s];
        }
    }
    in_base += ti;
    out_base += to;
  }
}

cudaError_t launch_pack_one(const Job *job_dev, int n_nodes, int64_t *part, int32_t *out, int sigma,
                            cudaStream_t stream) {
  int blocks = std::max(1, std::min((n_nodes + 1023) / 1024, kPackOneMaxBlocks));
  int npb = (n_nodes + blocks - 1) / blocks;
  npb = std::max(kPackThreads, (npb + kPackThreads - 1) / kPackThreads * kPackThreads);
  blocks = std::max(1, (n_nodes + npb - 1) / npb);
  k_pack_count<<<blocks, kPackThreads, 0, stream>>>(job_dev, npb, part);
  k_pack_wide<<<blocks, kPackThreads, 0, stream>>>(job_dev, npb, part, out, sigma);
  return cudaGetLastError();
}

cudaError_t launch_pack(const Job *jobs_dev, const int32_t *ids, int n_ids, const int64_t *offsets, int32_t *out,
                        int sigma, cudaStream_t stream) {
  if (n_ids <= 0) return cudaSuccess;
  const int threads = 128;
  const int blocks = (n_ids * 32 + threads - 1) / threads;
  k_pack<<<blocks, threads, 0, stream>>>(jobs_dev, ids, n_ids, offsets, out, sigma);
  return cudaGetLastError();
}

}  // namespace poa
