/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * C ABI of the CPU restatement of minipoa-rs's partial-order-alignment path
 * (src/align.rs, src/graph.rs, src/lib.rs). It is the checker the GPU library
 * is compared against, and the CPU baseline timed beside it. Nothing in the
 * shipped library links, loads or calls it.
 *
 * Parity pinning: the reference crate cannot be built (its src/io.rs is
 * missing and no Rust toolchain is present), so this restatement is pinned by
 * the reference's own known-answer tests and property tests, restated in
 * tests/test_oracle_*.py.
 *
 * orc_params has the same field order and layout as poa_params in
 * include/minipoa_b200.h so one Python structure serves both.
 */
#ifndef MINIPOA_ORACLE_H
#define MINIPOA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
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
} orc_params;

/* DP kernel selection for the oracle.
 * ORC_AUTO_SERIAL: reference dispatch (i32 when i32_scores_safe, else i64),
 *                  i32 restated serially with the SIMD kernel's exact sentinels.
 * ORC_FORCE_I64:   the reference's `scalar-dp` feature (always i64).
 * ORC_AUTO_AVX2:   reference dispatch with an 8-lane AVX2 i32 kernel
 *                  (mirrors wide::i32x8); the timed CPU baseline.
 * ORC_I32_ONLY / ORC_I64_ONLY: call poa_simd_i32 / poa_scalar_i64 directly
 *                  (no guard), as align.rs's unit tests do. */
enum { ORC_AUTO_SERIAL = 0, ORC_FORCE_I64 = 1, ORC_AUTO_AVX2 = 2, ORC_I32_ONLY = 3, ORC_I64_ONLY = 4 };

typedef struct orc_item { int64_t node; int64_t base; int64_t aligned; } orc_item; /* -1 = None */

void *orc_graph_new(const orc_params *p);
void orc_graph_free(void *g);
void *orc_graph_clone(const void *g);
void orc_free(void *ptr);
const char *orc_last_error(void);

/* lib.rs:177 / lib.rs:184 */
int orc_align_sequences(const orc_params *p, int64_t n, const uint8_t *const *seqs, const int64_t *lens,
                        int kernel, void **out_graph);
/* align_sequences with progressive guide order: the reads in `order` */
int orc_align_sequences_in_order(const orc_params *p, int64_t n, const uint8_t *const *seqs, const int64_t *lens,
                                 const int64_t *order, int kernel, void **out_graph);
int orc_extend_graph(const orc_params *p, void *g, int64_t n, const uint8_t *const *seqs, const int64_t *lens,
                     int64_t existing, int kernel);
/* align.rs:81 */
int orc_align(const orc_params *p, const void *g, const uint8_t *q, int64_t len, int kernel, orc_item **out,
              int64_t *out_len);
/* align.rs:192 (retry=1) or poa_inner / a direct kernel (retry=0) */
int orc_poa(const orc_params *p, const void *g, int64_t beg_id, int64_t end_id, const uint8_t *q, int64_t len,
            int adaptive, uint64_t band_b, int kernel, int retry, orc_item **out, int64_t *out_len);
int orc_i32_scores_safe(const orc_params *p, const void *g, int64_t beg_id, int64_t end_id, int64_t qlen);
/* graph.rs */
int orc_add_path(const orc_params *p, void *g, int64_t seq_id, const orc_item *items, int64_t n);
int orc_toposort(void *g, int grouped);
/* graph.rs:42 / graph.rs:62 */
int64_t orc_add_node(void *g, int64_t base);
void orc_add_edge(void *g, int64_t from, int64_t to);
int orc_consensus(const orc_params *p, const void *g, uint8_t **seq, int64_t **ids, int64_t **coverage,
                  int64_t *len);
int orc_msa(const orc_params *p, void *g, int64_t n, const char *const *names, const char *const *comments,
            char **out, int64_t *out_len);
int orc_gfa(const orc_params *p, const void *g, int64_t n, const char *const *names, char **out, int64_t *out_len);
int orc_params_validate(const orc_params *p);
int64_t orc_encode(const orc_params *p, uint8_t c);

/* Graph inspection: node count, node fields, edges (for byte-exact comparison
 * with the GPU library's graph). */
int64_t orc_graph_nodes(const void *g);
int64_t orc_graph_paths(const void *g);
/* Writes per node: base, parent, rank, coverage (4 x n int64). */
void orc_graph_node_fields(const void *g, int64_t *out);
/* Edge lists flattened: for each node its incoming (id,weight) pairs then
 * outgoing pairs; counts in *_cnt arrays (n each). Buffers sized by caller
 * from orc_graph_edge_total. */
int64_t orc_graph_edge_total(const void *g);
void orc_graph_edges(const void *g, int64_t *in_cnt, int64_t *out_cnt, int64_t *in_pairs, int64_t *out_pairs);
void orc_graph_rank(const void *g, int64_t *out);
int64_t orc_graph_rank_len(const void *g);
/* aligned[] groups: n * alphabet entries, -1 = None */
void orc_graph_aligned(const void *g, int64_t *out);
/* paths: seq ids (n_paths), lengths (n_paths), then concatenated ids */
int64_t orc_graph_path_total(const void *g);
void orc_graph_path_data(const void *g, int64_t *seq_ids, int64_t *lens, int64_t *ids);

/* DP cell counter (8-aligned band cells of computed rows, retries included),
 * accumulated per calling thread since the last reset. */
uint64_t orc_cells(void);
void orc_reset_cells(void);

/* Independent read sets run on `threads` host threads, one whole set per
 * thread at a time (the reference's -t has no effect on unseeded runs, so
 * this is the multi-process throughput form). Each set: n_reads reads from
 * the flattened arrays. Output format: 0 consensus FASTA, 2 GFA, -1 none.
 * Returns total cells; per-set output strings are hashed (FNV-1a 64) into
 * hashes[set]. */
int orc_batch_run(const orc_params *p, int64_t n_sets, const int64_t *set_off, const uint8_t *const *seqs,
                  const int64_t *lens, int kernel, int threads, int out_format, uint64_t *hashes,
                  uint64_t *cells);

/* Test hooks for the AVX2 insertion-prefix scan (align.rs:459-491). */
int orc_avx2_available(void);
uint64_t orc_fnv1a(const uint8_t *data, int64_t len);
int orc_read_gfa(const orc_params *p, const char *text, int64_t len, void **out_graph, char **records,
                 int64_t *records_len);
void orc_avx2_prefix(const int32_t *md8, int32_t carry, int32_t open, int32_t ext, int32_t *out8);

#ifdef __cplusplus
}
#endif
#endif
