/*
 * minipoa_b200 -- C ABI of the B200 (sm_100a) partial-order-alignment library.
 *
 * Drop-in boundary for minipoa-rs's POA hot path: affine-gap sequence-to-DAG
 * alignment over toposorted ranks, weighted traceback, read-into-graph fusion
 * and re-toposort. The DP, traceback, fusion and toposort run on the GPU and
 * the graph stays resident in device memory between reads; consensus / MSA /
 * GFA text is rendered on the host from the downloaded graph.
 *
 * Each entry point names the reference item it replaces (paths inside the
 * minipoa-rs project). The reference is a Rust library with no FFI of its
 * own; a Rust FFI crate binds these declarations in an extern "C" block.
 *
 * Conventions: every call returns int status (POA_OK = 0); on failure
 * poa_last_error(ctx) gives the reference's error text (the calling thread's
 * last error, so several threads can share a context's server). Buffers passed in are
 * caller-owned; buffers returned through out-pointers are library-owned and
 * released with poa_free. No call takes torch or other framework types.
 */
#ifndef MINIPOA_B200_H
#define MINIPOA_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. Alignment errors carry the reference's messages
 * (src/align.rs, src/graph.rs); resource codes are this library's own. */
enum {
  POA_OK = 0,
  POA_ERR_ALIGN = 1,        /* an alignment / graph error (message in poa_last_error) */
  POA_ERR_INVALID = 2,      /* invalid parameters or arguments (Params::validate text) */
  POA_ERR_CUDA = 3,         /* CUDA runtime failure, or no CUDA device */
  POA_ERR_ALLOC = 4,        /* device memory could not be allocated within the budget */
  POA_ERR_UNSUPPORTED = 5,  /* feature not available in this build (message says which) */
  POA_ERR_TIMEOUT = 6       /* a bounded device wait gave up */
};

/* Params (src/lib.rs:47-71). Same field order as the reference struct;
 * alphabet/matrix point at caller memory (alphabet_len^2 matrix entries). */
typedef struct poa_params {
  int32_t match_score;
  int32_t mismatch;
  int32_t gap_open;
  int32_t gap_ext;
  uint64_t b;
  uint64_t f;
  int32_t adaptive;
  int32_t seeding;
  uint64_t k;
  uint64_t w;
  int32_t progressive;
  int32_t result;
  uint64_t threads;
  uint64_t win_band;
  uint64_t win_max;
  double mm_filter_ratio;
  uint64_t max_occ;
  uint64_t tr_dist;
  int32_t verbose;
  int32_t is_rna;
  int32_t alphabet_len;
  int32_t reserved;
  const uint8_t *alphabet;
  const int32_t *matrix;
} poa_params;

/* AlignedBase (src/lib.rs:140-145); -1 encodes None. */
typedef struct poa_aligned_base {
  int64_t node;
  int64_t base;
  int64_t aligned;
} poa_aligned_base;

typedef struct poa_ctx poa_ctx;
typedef struct poa_graph poa_graph;
typedef struct poa_batch poa_batch;

/* dp_backend() (src/lib.rs:15-37): the DP backend string. */
const char *poa_dp_backend(void);

/* Context: one CUDA device, one stream, a DP arena and a memory budget in
 * bytes (0 = 90% of free device memory). No reference counterpart (the
 * reference keeps a thread-local arena, src/align.rs:222-226). */
int poa_ctx_create(int device, uint64_t mem_budget, poa_ctx **out);
void poa_ctx_destroy(poa_ctx *ctx);
const char *poa_last_error(const poa_ctx *ctx);
void poa_free(void *ptr);

/* Seeded reads (params->seeding): the seed windows of a read are aligned in
 * one launch, one warp per window (0, default), or one launch per window (1).
 * Same results; the second form is the reference-shaped one. */
int poa_ctx_tune_windows(poa_ctx *ctx, int32_t one_launch_per_window);
/* Seeded reads so far on this context: windows aligned, kernel launches
 * for them, and reads that fell back to the whole graph (no usable anchors). */
int poa_ctx_window_stats(poa_ctx *ctx, uint64_t *windows, uint64_t *launches, uint64_t *fallbacks);

/* Params::validate (src/lib.rs:149-173). */
int poa_params_validate(poa_ctx *ctx, const poa_params *params);

/* Graph::new (src/graph.rs:30-40): source and sink nodes, both base N. */
int poa_graph_new(poa_ctx *ctx, const poa_params *params, poa_graph **out);
void poa_graph_free(poa_graph *graph);

/* align_sequences (src/lib.rs:177-182): validate, new graph, then the serial
 * read loop of extend_graph (src/lib.rs:184-204). */
int poa_align_sequences(poa_ctx *ctx, const poa_params *params, int64_t n_seqs, const uint8_t *const *seqs,
                        const int64_t *lens, poa_graph **out);

/* extend_graph (src/lib.rs:184-204) on an existing graph, reads
 * existing..n_seqs-1 (their index is the path's sequence id). */
int poa_extend_graph(poa_ctx *ctx, const poa_params *params, poa_graph *graph, int64_t n_seqs,
                     const uint8_t *const *seqs, const int64_t *lens, int64_t existing);

/* align::align (src/align.rs:81-188): the path of `query` against the graph
 * in its current toposort order, source first, sink excluded. The graph is
 * not modified. *out has *out_len items; release with poa_free. */
int poa_align(poa_ctx *ctx, const poa_params *params, poa_graph *graph, const uint8_t *query, int64_t len,
              poa_aligned_base **out, int64_t *out_len);

/* align::poa (src/align.rs:192-211): align between anchors beg_id (included)
 * and end_id (excluded) with the full-DP retry. retry = 0 gives poa_inner
 * (src/align.rs:531-545) without the retry; kernel: 0 = score-guard dispatch
 * (src/align.rs:493-529), 1 = i32 kernel only, 2 = i64 kernel only. */
int poa_poa(poa_ctx *ctx, const poa_params *params, poa_graph *graph, int64_t beg_id, int64_t end_id,
            const uint8_t *query, int64_t len, int32_t adaptive, uint64_t band_b, int32_t kernel, int32_t retry,
            poa_aligned_base **out, int64_t *out_len);

/* Graph::add_path (src/graph.rs:82-122). */
int poa_graph_add_path(poa_ctx *ctx, poa_graph *graph, int64_t seq_id, const poa_aligned_base *items, int64_t n);
/* Graph::add_node (src/graph.rs:42-59) and Graph::add_edge (src/graph.rs:62-79). */
int poa_graph_add_node(poa_ctx *ctx, poa_graph *graph, int64_t base, int64_t *out_id);
int poa_graph_add_edge(poa_ctx *ctx, poa_graph *graph, int64_t from, int64_t to);
/* Graph::toposort (src/graph.rs:125-178); grouped != 0 orders column groups. */
int poa_graph_toposort(poa_ctx *ctx, poa_graph *graph, int32_t grouped);

/* Graph::consensus (src/graph.rs:181-237): sequence (decoded bytes), node
 * ids and coverage, each *len long; release each with poa_free. */
int poa_graph_consensus(poa_ctx *ctx, const poa_params *params, poa_graph *graph, uint8_t **seq, int64_t **ids,
                        int64_t **coverage, int64_t *len);
/* Graph::msa (src/graph.rs:239-279): FASTA rows for sequences 0..n-1. */
int poa_graph_msa(poa_ctx *ctx, const poa_params *params, poa_graph *graph, int64_t n, const char *const *names,
                  const char *const *comments, char **out, int64_t *out_len);
/* Graph::gfa (src/graph.rs:281-331). */
int poa_graph_gfa(poa_ctx *ctx, const poa_params *params, poa_graph *graph, int64_t n, const char *const *names,
                  char **out, int64_t *out_len);

/* The graph's public fields (src/graph.rs:6-27), downloaded: node count,
 * path count and sizes of the variable parts. */
typedef struct poa_graph_sizes {
  int64_t n_nodes;
  int64_t n_edges;   /* total incoming entries */
  int64_t n_paths;
  int64_t path_items;
  int64_t alphabet;
  int64_t n_rank;    /* entries of Graph::rank */
} poa_graph_sizes;
int poa_graph_sizes_get(poa_ctx *ctx, poa_graph *graph, poa_graph_sizes *out);
/* Fills caller buffers (sizes from poa_graph_sizes_get):
 * fields: 4*n_nodes (base, parent, rank, coverage); rank: n_nodes;
 * aligned: n_nodes*alphabet (-1 = None); in_cnt/out_cnt: n_nodes;
 * in_pairs/out_pairs: 2*n_edges (id, weight) in insertion order;
 * path_seq/path_len: n_paths; path_ids: path_items. */
int poa_graph_export(poa_ctx *ctx, poa_graph *graph, int64_t *fields, int64_t *rank, int64_t *aligned,
                     int64_t *in_cnt, int64_t *out_cnt, int64_t *in_pairs, int64_t *out_pairs, int64_t *path_seq,
                     int64_t *path_len, int64_t *path_ids);

/* No counterpart in the reference. poa_align for callers that cannot
 * allocate device memory when they align (a serving loop whose device memory
 * belongs to another allocator, a strict memory budget, or a thread that must
 * not trigger the device-wide synchronisation of cudaMalloc/cudaFree). The
 * call allocates no device memory: its DP scratch and scoring tables sit in one
 * library-owned array of POA_NOALLOC_SCRATCH_BYTES in device memory, which
 * every GPU that loads the library keeps until the process exits. d_query
 * (len bytes), d_out (out_cap >= len + 1 items) and d_out_len are device
 * pointers owned by the caller; the graph must be toposorted, as for
 * poa_align. The result equals poa_align's. A graph and query whose scratch
 * would exceed the array are rejected with POA_ERR_ALLOC and a message (use
 * poa_align then). The first call on a device looks up the array's device
 * address; make that first call before any stream capture. Calls share the
 * array: calls whose GPU work overlaps race and must be serialised by the
 * caller. The context's device must be the current device. */
#define POA_NOALLOC_SCRATCH_BYTES (32u << 20)
int poa_align_noalloc(poa_ctx *ctx, const poa_params *params, poa_graph *graph, const uint8_t *d_query, int64_t len,
                      poa_aligned_base *d_out, int64_t out_cap, int64_t *d_out_len);

/* ---- seed windows for seeded alignment (-S), host only (no context).
 * Outputs are released with poa_free. Minimizer selection is this library's
 * (forward ntHash, leftmost minimum); the reference takes it from the
 * simd-minimizers crate, so the chosen k-mers can differ. Everything after
 * the sketch follows src/minimizer.rs. */
typedef struct poa_minimizer {
  uint64_t value;  /* exact packed k-mer: A0 C1 T2 G3, first base in the low bits */
  int64_t end;     /* inclusive position of its last base */
  int64_t span;
} poa_minimizer;
typedef struct poa_anchor {
  int64_t target_end;
  int64_t query_end;
  int64_t span;
  int32_t adaptive_before;
  int32_t reserved;
} poa_anchor;
/* sketch (src/minimizer.rs:39-75). */
int poa_seed_sketch(const uint8_t *seq, int64_t len, int64_t k, int64_t w, poa_minimizer **out, int64_t *n);
/* repeat_intervals (src/minimizer.rs:79-110): *n_out (start, end) pairs. */
int poa_seed_repeat_intervals(const poa_minimizer *mm, int64_t n, int64_t len, int64_t max_dist, int64_t **out_pairs,
                              int64_t *n_out);
/* collect_anchors (src/minimizer.rs:128-172). */
int poa_seed_collect_anchors(const poa_params *params, const uint8_t *query, int64_t qlen, const uint8_t *target,
                             int64_t tlen, poa_anchor **out, int64_t *n);
/* chain (src/minimizer.rs:199-366). */
int poa_seed_chain(const poa_anchor *anchors, int64_t n, int64_t k, poa_anchor **out, int64_t *n_out);
/* partition_windows (src/minimizer.rs:371-457). */
int poa_seed_partition_windows(const poa_anchor *chain, int64_t n, int64_t tlen, int64_t qlen, int64_t max_drift,
                               int64_t max_win, poa_anchor **out, int64_t *n_out, int32_t *tail_adaptive);
/* anchor_windows (src/minimizer.rs:466-479): the windows align::align uses
 * with seeding (src/align.rs:99-164), which poa_align, poa_align_sequences
 * and poa_extend_graph run when params->seeding is set. */
int poa_seed_anchor_windows(const poa_params *params, const uint8_t *query, int64_t qlen, const uint8_t *consensus,
                            int64_t clen, poa_anchor **out, int64_t *n_out, int32_t *tail_adaptive);
/* guide_order (src/minimizer.rs:505-578): the order in which progressive
 * alignment (params->progressive, -p; src/lib.rs:190-194) adds the n reads,
 * as n read indices. Minimizer similarity from this library's sketches (see
 * above). poa_align_sequences, poa_extend_graph (no existing records), the
 * batched sets and the serving jobs align in this order; paths keep each
 * read's own index. */
int poa_seed_guide_order(const poa_params *params, int64_t n, const uint8_t *const *seqs, const int64_t *lens,
                         int64_t **out_order);

/* ---- batched independent read sets (no reference counterpart: the
 * reference runs one set per process; each set here is one extend_graph). */
typedef struct poa_batch_stats {
  uint64_t cells;       /* 8-aligned band cells computed, retries included */
  uint64_t reads;       /* reads aligned */
  double device_ms;     /* device time of the last run (CUDA events) */
  int32_t launches;     /* kernel launches in the last run */
  int32_t relaunches;   /* extra passes for jobs that outgrew their DP arena */
  int32_t slots;        /* concurrent warp slots of the first pass (teams: 4 per set) */
  int32_t reserved;
  double kernel_ms;     /* device time inside the read-loop kernel launches */
  uint64_t dp_bytes;    /* DP state bytes stored (M, D, I per cell) */
  uint64_t pred_cells;  /* predecessor-cell updates: per row, the band overlap of each
                           in-band predecessor (align.rs:751-797 trip count) */
  uint64_t far_preds;   /* predecessor rows read from the arena, not the shared-memory ring */
  uint64_t rows_g4;     /* DP rows of more than 384 columns on the striped tiles (the wide
                           kernel form: up to 2048 columns, in 512-column segments) */
  uint64_t rows_generic;  /* DP rows of the generic row (wider than the striped tiles,
                             > 32 predecessors, i64) */
  int32_t coop_jobs;    /* jobs that ran cooperative rows (a giant with helper warps) */
  int32_t wave_reads;   /* reads whose static-band DP ran as a row wavefront (lane per row) */
  uint64_t phase_cycles[4]; /* profiling builds only (POA_PHASE_CYCLES), else 0: warp cycles
                               in band guides, DP rows, traceback, graph update */
} poa_batch_stats;

/* Uploads n_sets read sets (set i = reads set_off[i]..set_off[i+1]-1) and
 * sizes device storage for them. mode: 0 = persistent batched kernel over all
 * sets (size-ordered queue), 1 = plain form, one launch per read of each set. */
int poa_batch_create(poa_ctx *ctx, const poa_params *params, int64_t n_sets, const int64_t *set_off,
                     const uint8_t *const *seqs, const int64_t *lens, poa_batch **out);
/* Resets every set's graph to Graph::new and aligns all reads on the device.
 * Inputs already resident; returns after the device work completes. A batch
 * of at most one set per SM runs as teams (one 4-warp block per set: the set
 * and three helper warps on its DP rows); results are the same either way.
 * A batch of no sets does nothing. */
int poa_batch_run(poa_ctx *ctx, poa_batch *batch, int32_t mode, poa_batch_stats *stats);
/* Per-set status after a run (0 = ok, else POA_ERR_ALIGN with message in
 * poa_batch_error). */
int poa_batch_status(poa_ctx *ctx, poa_batch *batch, int64_t set, char **message);
/* Output of set `set`: result 0 consensus FASTA, 1 MSA, 2 GFA, rendered with
 * names "read{i}" / empty comments unless names are given. */
int poa_batch_output(poa_ctx *ctx, poa_batch *batch, int64_t set, int32_t result, const char *const *names,
                     const char *const *comments, char **out, int64_t *out_len);
/* Output of every set concatenated in set order (result 0 or 2), rendered
 * on host threads. */
int poa_batch_output_all(poa_ctx *ctx, poa_batch *batch, int32_t result, char **out, int64_t *out_len);
/* One set's graph as a standalone graph handle (copied). */
int poa_batch_graph(poa_ctx *ctx, poa_batch *batch, int64_t set, poa_graph **out);
/* Host<->device bytes moved by the last poa_batch_create (reads, offsets,
 * lengths) and by the last output call (packed graphs). */
int poa_batch_transfer_bytes(poa_ctx *ctx, poa_batch *batch, uint64_t *h2d, uint64_t *d2h);
void poa_batch_free(poa_batch *batch);

/* Integer-pipe throughput of `device` (no reference counterpart: the
 * roofline denominator of the DP kernels, whose recurrences are 32-bit adds
 * and maxes). Fills out_ops_per_s[3] with operations per second of a plain
 * add, a plain max and the DPX fused add-max (two operations each), each
 * over every SM. Allocates a small device buffer; about 0.1 s. */
int poa_probe_int_peak(int32_t device, double *out_ops_per_s);

/* io::read_gfa (called at src/lib.rs:214-218; its source file is absent from
 * the reference tree, so the behaviour follows tests/io_cli.rs:374-431,
 * 563-610): GFA text -> a device graph ranked by the LIFO toposort, and its
 * path records as library-owned "name\tsequence\n" lines (one per P line,
 * in file order). Segments become chains of single-base nodes; only forward
 * links with a 0M overlap are accepted; duplicate segments, unknown
 * references, reverse orientations, self links, cycles and paths revisiting
 * a node ("revisits") are POA_ERR_ALIGN with the reason. Extending the graph
 * with new reads is poa_extend_graph with existing = the record count. */
int poa_graph_read_gfa(poa_ctx *ctx, const poa_params *params, const char *text, int64_t len, poa_graph **out,
                       char **records, int64_t *records_len);

/* Autotuner (no reference counterpart). Launch settings of the batched
 * kernel: resident warps per SM, the giant threshold (a set whose estimated
 * work exceeds giant_factor per-warp shares gets three helper warps; 0 =
 * none) and giant_alone (1: a giant's SM runs only the giant and its helpers
 * until it is done). poa_batch_autotune runs the batch under each candidate
 * setting, keeps the fastest, applies it and appends it to the cache file
 * (MINIPOA_B200_TUNE_CACHE, default ~/.cache/minipoa_b200/tune.tsv) under the
 * batch's size bucket (device, log2 of set count, longest read and mean
 * depth); poa_batch_create applies a cached setting for its bucket. Results
 * are the same under every setting. poa_batch_tuning_get reports the current
 * setting (trials = runs replayed from the captured CUDA graph so far). */
typedef struct poa_batch_tuning {
  int32_t warps_per_sm;
  int32_t giant_alone;
  double giant_factor;
  double device_ms;  /* device time of the chosen setting's run */
  int32_t trials;
  int32_t reserved2;
} poa_batch_tuning;
int poa_batch_autotune(poa_ctx *ctx, poa_batch *batch, poa_batch_tuning *out);
int poa_batch_tuning_get(poa_ctx *ctx, poa_batch *batch, poa_batch_tuning *out);

/* Tuning: warp slots per SM for the batched kernel (0 = 6, the untuned
 * default; poa_batch_create applies a cached tuned setting first; up to 8
 * are resident at once, more only add slots that start when others leave)
 * and the DP arena bytes per slot (0 = auto from the budget). */
int poa_batch_tune(poa_ctx *ctx, poa_batch *batch, int32_t warps_per_sm, uint64_t arena_bytes_per_slot);

/* ---- serving loop (no reference counterpart: the reference is a CLI that
 * runs one job per process). Continuous batching: jobs (each one
 * extend_graph over its reads, src/lib.rs:184-204, on a new graph) are
 * submitted at any time; a dispatcher thread admits them in arrival order
 * while the server's device pool holds their graph storage, reads, DP arena
 * and descriptor, and publishes them to the device-side job queue of one
 * persistent serving kernel: each of its warps (7 per SM) takes the next job
 * as soon as it finishes its last, so jobs that arrive while others run start
 * at once on free warps. The kernel ends when its warps have waited idle_ms
 * without work and is launched again when jobs arrive. A job's completion is
 * seen as soon as its warp finishes (host-mapped flag). A job whose DP
 * outgrows its arena parks at its current read and is re-admitted with twice
 * the arena. Finished graphs stay resident until released. Results are
 * byte-identical to poa_align_sequences on the same reads, whatever else
 * runs alongside. */
typedef struct poa_server poa_server;
enum {
  POA_SERVER_QUEUED = 0,   /* waiting for admission */
  POA_SERVER_RUNNING = 1,  /* on the device */
  POA_SERVER_DONE = 2,     /* finished; output available until released */
  POA_SERVER_FAILED = 3,   /* finished with an error (poa_server_job_info gives it) */
  POA_SERVER_PARKED = 4    /* needs a larger DP arena; re-admitted with twice the arena */
};
typedef struct poa_server_job {
  int32_t state;
  int32_t reserved;
  uint64_t cells;      /* band cells computed for the job */
  double queued_ms;    /* submission to admission (published to the kernel's queue) */
  double latency_ms;   /* submission to completion (0 while unfinished) */
} poa_server_job;
typedef struct poa_server_stats {
  uint64_t done_jobs;
  uint64_t done_cells;
  uint64_t waves;          /* admission rounds published to the serving kernel's queue */
  uint64_t queued;         /* jobs waiting for admission */
  uint64_t kernel_launches; /* serving-kernel launches so far */
  uint64_t pool_bytes;
  uint64_t pool_used;
  double busy_s;           /* first submission to the last completion */
} poa_server_stats;
/* pool_bytes: device memory of the server (0 = what the context's budget
 * leaves, less 512 MiB); idle_ms: how long the serving kernel's warps wait
 * for a job before the kernel ends (0 = 50 ms). */
int poa_server_create(poa_ctx *ctx, const poa_params *params, uint64_t pool_bytes, int32_t idle_ms,
                      poa_server **out);
/* Queues one job (its reads in order); returns at once with its id. */
int poa_server_submit(poa_ctx *ctx, poa_server *server, int64_t n_seqs, const uint8_t *const *seqs,
                      const int64_t *lens, int64_t *job_id);
/* Queues one job that extends an initial graph given as GFA text (the
 * reference's -i workflow, src/lib.rs:214-231, with progressive ordering
 * off): the GFA is parsed and ranked at once (errors as poa_graph_read_gfa),
 * copied into device memory when the job is admitted, and the reads are
 * aligned into it; their sequence ids follow the GFA's path records. */
int poa_server_submit_gfa(poa_ctx *ctx, poa_server *server, const char *gfa, int64_t gfa_len, int64_t n_seqs,
                          const uint8_t *const *seqs, const int64_t *lens, int64_t *job_id);
/* Waits for a job to finish (timeout_ms < 0: no limit; POA_ERR_TIMEOUT when
 * it runs out). */
int poa_server_wait(poa_ctx *ctx, poa_server *server, int64_t job, double timeout_ms, int32_t *state);
/* State and timings of a job; a failed job returns its error. */
int poa_server_job_info(poa_ctx *ctx, poa_server *server, int64_t job, poa_server_job *out);
/* Output of a finished job: result 0 consensus FASTA, 1 MSA, 2 GFA (names
 * "read{i}" and empty comments unless given). */
int poa_server_output(poa_ctx *ctx, poa_server *server, int64_t job, int32_t result, const char *const *names,
                      const char *const *comments, char **out, int64_t *out_len);
/* Frees a finished job's graph. */
int poa_server_release(poa_ctx *ctx, poa_server *server, int64_t job);
/* Scales the DP arena a job is first admitted with (default 1: an estimate
 * of its widest band over the rows its graph grows to). Below 1 a job takes
 * less memory and parks more often; for memory-tight deployments. */
int poa_server_tune(poa_ctx *ctx, poa_server *server, double arena_scale);
int poa_server_stats_get(poa_ctx *ctx, poa_server *server, poa_server_stats *out);
/* Finishes the queued and running jobs, then frees the server. */
void poa_server_destroy(poa_server *server);

#ifdef __cplusplus
}
#endif
#endif
