// Host-side view of a downloaded graph and the text outputs rendered from it:
// consensus (graph.rs:181-237), MSA (graph.rs:239-279, with the grouped
// toposort of graph.rs:125-178) and GFA (graph.rs:281-331). Also the
// product's Params handling (lib.rs:47-173).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/minipoa_b200.h"

namespace poa {

struct HostParams {
  int32_t match_score = 2, mismatch = -4, gap_open = -4, gap_ext = -2;
  uint64_t b = 100, f = 40;
  bool adaptive = false, seeding = false;
  uint64_t k = 19, w = 10;
  bool progressive = false;
  int32_t result = 0;
  uint64_t threads = 1, win_band = 500, win_max = 10000;
  double mm_filter_ratio = 0.25;
  uint64_t max_occ = 0, tr_dist = 1000;
  int32_t verbose = 0;
  bool is_rna = false;
  std::vector<uint8_t> alphabet;
  std::vector<int32_t> matrix;

  static HostParams from(const poa_params *p);
  int encode(uint8_t c) const;       // lib.rs:110-126
  uint8_t decode(int code) const;    // lib.rs:127-134
  std::string validate() const;      // lib.rs:149-173, empty when valid
  uint64_t largest() const;          // align.rs:515-525
};

struct HostGraph {
  int n = 0, sigma = 0, n_rank = 0;
  std::vector<int32_t> base, parent, rank, coverage, aligned, rank_to_node;
  std::vector<int64_t> in_off, out_off;
  std::vector<int32_t> in_id, in_w, out_id, out_w;
  std::vector<int32_t> path_seq, path_items;
  std::vector<int64_t> path_off;

  // Parses one packed record (poa_pack.cu layout).
  static HostGraph parse(const int32_t *rec);

  void consensus(const HostParams &p, std::vector<uint8_t> &seq, std::vector<int64_t> &ids,
                 std::vector<int64_t> &cov) const;
  // Returns false with *err set on failure.
  bool msa(const HostParams &p, const std::vector<std::string> &names, const std::vector<std::string> &comments,
           std::string &out, std::string &err) const;
  bool gfa(const HostParams &p, const std::vector<std::string> &names, std::string &out, std::string &err) const;
  // LIFO Kahn order (graph.rs:125-178 with grouped = false) into rank /
  // rank_to_node; 0 or the device status code of the failure (cycle, column
  // dependencies).
  int32_t lifo_order();
  // Column-grouped LIFO Kahn ranks (graph.rs:125-178 with grouped = true).
  bool grouped_ranks(std::vector<int32_t> &node_rank, std::vector<int32_t> &order, std::string &err) const;
};

}  // namespace poa
