// poa_align_noalloc: align::align for callers that must not allocate device
// memory.
//
// Some callers cannot call cudaMalloc at the moment they need an alignment:
// a serving loop whose device memory is already carved up by another
// allocator, code running under a strict device-memory budget, or a thread
// that must not trigger the implicit device-wide synchronisation a cudaMalloc
// or cudaFree can cause. This entry point gives them the same result as
// poa_align without allocating anything: the DP scratch and the scoring tables
// live in one fixed-size array in device global memory, declared below, which
// every GPU that loads this library holds until the process exits.
//
// The array is shared by all calls. Each call rewrites every byte of it that
// it reads, so nothing carries over from the previous call, but two calls
// whose work overlaps on the GPU (on different streams, or from different
// threads) use the same bytes at the same time and corrupt each other: the
// caller must serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/minipoa_b200.h"
#include "host_graph.h"
#include "poa_internal.h"

namespace poa {

// Defined in poa_host.cu.
Job *graph_device_job(poa_graph *g);
int graph_alphabet(const poa_graph *g);
const poa_ctx *graph_context(const poa_graph *g);
cudaStream_t ctx_stream(const poa_ctx *c);
int ctx_device(const poa_ctx *c);
void ctx_set_error(poa_ctx *c, const std::string &msg);
std::string describe_status(int32_t st, int err_i, int err_j);
int status_to_code(int32_t st);
bool graph_read_job(poa_graph *g, Job *out, std::string *err);
bool graph_clear_status(poa_graph *g, std::string *err);

namespace {

// Layout: [scoring matrix, up to 256 x 256 int32][encode table, 256 bytes]
// [DP arena: per-read scratch and DP states].
constexpr size_t kTablesBytes = size_t(256) * 256 * 4 + 256;
constexpr size_t kArenaOffset = (kTablesBytes + 255) / 256 * 256;
static_assert(kArenaOffset < POA_NOALLOC_SCRATCH_BYTES, "scratch smaller than its table header");

static __device__ __align__(256) unsigned char g_noalloc_scratch[POA_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on `dev` (which must be current). The
// host-side name g_noalloc_scratch is only a stand-in for the symbol, so the
// address comes from cudaGetSymbolAddress, once per device.
unsigned char *scratch_on(int dev, std::string *err) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (dev < 0 || dev >= kMaxDevices) {
    *err = "device index out of range for the no-allocation scratch";
    return nullptr;
  }
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      *err = std::string("cudaGetSymbolAddress failed for the no-allocation scratch: ") + cudaGetErrorString(e);
      return nullptr;
    }
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
  }
  return g_scratch_ptr[dev];
}

__device__ __forceinline__ WarpSmem *noalloc_warp_smem() {
  extern __shared__ __align__(16) unsigned char noalloc_smem[];
  return reinterpret_cast<WarpSmem *>(noalloc_smem);
}

// align::align (align.rs:81-188) of one query, one warp, scratch in `arena`;
// the path goes to the caller's device buffer as AlignedBase records.
// A path longer than the caller's buffer (out_cap items) is not written and
// ends the call with ST_OUT_TOO_SMALL.
__global__ void k_align_noalloc(Job *J, DevParams P, char *arena, int64_t bytes, const uint8_t *q, int qlen,
                                poa_aligned_base *out, int64_t out_cap, int64_t *out_n) {
  const int lane = threadIdx.x & 31;
  Scratch s;
  int n_items = 0;
  Work cells{};
  ring_default(noalloc_warp_smem());
  int32_t st = align_query(J, P, arena, bytes, q, qlen, s, &n_items, &cells, noalloc_warp_smem());
  if (st == ST_OK && int64_t(n_items) > out_cap) st = ST_OUT_TOO_SMALL;
  if (st == ST_OK) {
    for (int k = lane; k < n_items; k += 32) {
      const int4 it = s.items[k];
      out[k] = poa_aligned_base{it.x, it.y, it.z};
    }
  }
  if (lane == 0) {
    J->status = st;
    *out_n = st == ST_OK ? n_items : 0;
  }
}

// Scratch the kernel carves before the DP states (carve_scratch), for a
// graph of n rows and e edges and a query of qlen bases.
int64_t scratch_floor(int64_t n, int64_t e, int64_t qlen) {
  const int64_t padded = (qlen + 2) / 8 * 8 + 8;
  // per row: 13 int64 arrays, 8 int32 arrays, an int4 plan and an 80-byte
  // wavefront record; per edge entry:
  // pred, succ, pmeta, pmeta_off, two traceback descriptors, pent; the query
  // as int32 and as bytes; the result items; 128-byte alignment of 36 arrays
  return n * (13 * 8 + 8 * 4 + 16 + 80) + (e + 1) * (8 + 8 + 16 + 8 + 32 + 16) + (padded + 32) * 5 +
         (qlen + 4) * 16 + 37 * 128;
}

}  // namespace
}  // namespace poa

using namespace poa;

extern "C" int poa_align_noalloc(poa_ctx *ctx, const poa_params *params, poa_graph *graph, const uint8_t *d_query,
                                 int64_t len, poa_aligned_base *d_out, int64_t out_cap, int64_t *d_out_len) {
  if (!ctx) return POA_ERR_INVALID;
  auto fail = [&](int code, const std::string &msg) {
    ctx_set_error(ctx, msg);
    return code;
  };
  if (!params || !graph || !d_out || !d_out_len || (len > 0 && !d_query))
    return fail(POA_ERR_INVALID, "null argument");
  if (graph_context(graph) != ctx) return fail(POA_ERR_INVALID, "the graph belongs to another context");
  const HostParams hp = HostParams::from(params);
  const std::string bad = hp.validate();
  if (!bad.empty()) return fail(POA_ERR_INVALID, bad);
  if (hp.seeding) return fail(POA_ERR_UNSUPPORTED, "seeded windows (-S) are not available in this build");
  if (int(hp.alphabet.size()) != graph_alphabet(graph))
    return fail(POA_ERR_INVALID, "alphabet size differs from the graph's");
  if (len < 0 || len > INT32_MAX / 4) return fail(POA_ERR_INVALID, "sequence is too long");
  if (out_cap < len + 1) return fail(POA_ERR_INVALID, "output buffer holds fewer than len + 1 items");
  const int64_t arena_bytes = int64_t(POA_NOALLOC_SCRATCH_BYTES) - int64_t(kArenaOffset);
  std::string err;
  Job h{};
  if (!graph_read_job(graph, &h, &err)) return fail(POA_ERR_CUDA, err);
  // the per-read scratch plus at least one 8-column band per row must fit
  const int64_t floor = scratch_floor(h.n_nodes, h.n_edges, len) + int64_t(h.n_nodes) * 8 * 3 * 8;
  if (floor > arena_bytes)
    return fail(POA_ERR_ALLOC, "graph and query need more than the " +
                                   std::to_string(POA_NOALLOC_SCRATCH_BYTES >> 20) +
                                   " MiB no-allocation scratch; use poa_align");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(POA_ERR_CUDA, cudaGetErrorString(e));
  if (dev != ctx_device(ctx)) return fail(POA_ERR_INVALID, "the context's device is not the current device");
  unsigned char *base = scratch_on(dev, &err);
  if (!base) return fail(POA_ERR_CUDA, err);
  const cudaStream_t stream = ctx_stream(ctx);
  // scoring tables into the scratch header
  const size_t mbytes = hp.matrix.size() * 4;
  uint8_t enc[256];
  for (int c = 0; c < 256; ++c) enc[c] = uint8_t(hp.encode(uint8_t(c)));
  e = cudaMemcpyAsync(base, hp.matrix.data(), mbytes, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + size_t(256) * 256 * 4, enc, 256, cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return fail(POA_ERR_CUDA, cudaGetErrorString(e));
  DevParams P{};
  P.matrix = reinterpret_cast<const int32_t *>(base);
  P.encode = base + size_t(256) * 256 * 4;
  P.sigma = int32_t(hp.alphabet.size());
  P.unknown = hp.encode('N');
  P.gap_open_raw = hp.gap_open;
  P.gap_ext = hp.gap_ext;
  P.gap_open = hp.gap_open + hp.gap_ext;
  P.adaptive = hp.adaptive ? 1 : 0;
  P.kernel = 0;
  P.seeding = 0;
  P.relaxed_order = 0;
  P.b = hp.b;
  P.f = hp.f;
  P.largest = hp.largest();
  k_align_noalloc<<<1, 32, sizeof(WarpSmem), stream>>>(graph_device_job(graph), P,
                                                        reinterpret_cast<char *>(base + kArenaOffset), arena_bytes,
                                                        d_query, int(len), d_out, out_cap, d_out_len);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(POA_ERR_CUDA, cudaGetErrorString(e));
  if (!graph_read_job(graph, &h, &err)) return fail(POA_ERR_CUDA, err);
  if (h.status != ST_OK) {
    const int32_t st = h.status;
    if (!graph_clear_status(graph, &err)) return fail(POA_ERR_CUDA, err);
    if (st == ST_ARENA_FULL)
      return fail(POA_ERR_ALLOC, "alignment needs more than the " + std::to_string(POA_NOALLOC_SCRATCH_BYTES >> 20) +
                                     " MiB no-allocation scratch; use poa_align");
    return fail(status_to_code(st), describe_status(st, h.err_i, h.err_j));
  }
  ctx_set_error(ctx, std::string());
  return POA_OK;
}
