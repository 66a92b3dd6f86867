// Seed windows for seeded alignment (-S): minimizer sketches, exact anchor
// matches, sparse chaining and the window partition of src/minimizer.rs.
// Host code: the windows of one read are computed on the CPU from the
// graph's consensus and the per-window alignments run on the device.
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

#include "host_graph.h"

namespace poa {

struct Minimizer {
  uint64_t value;  // exact forward 2-bit packed k-mer (A0 C1 T2 G3, first base lowest)
  int64_t end;     // inclusive position of the k-mer's last base
  int64_t span;
};

struct Anchor {
  int64_t target_end, query_end, span;
  bool adaptive_before;
  bool operator==(const Anchor &o) const {
    return target_end == o.target_end && query_end == o.query_end && span == o.span &&
           adaptive_before == o.adaptive_before;
  }
};

std::vector<Minimizer> sketch(const uint8_t *seq, int64_t len, int64_t k, int64_t w);
std::vector<std::pair<int64_t, int64_t>> repeat_intervals(const std::vector<Minimizer> &mm, int64_t len,
                                                          int64_t max_dist);
std::vector<Anchor> collect_anchors(const HostParams &p, const uint8_t *q, int64_t qlen, const uint8_t *t,
                                    int64_t tlen);
std::vector<Anchor> chain(const std::vector<Anchor> &anchors, int64_t k);
std::pair<std::vector<Anchor>, bool> partition_windows(const std::vector<Anchor> &chain, int64_t tlen, int64_t qlen,
                                                       int64_t max_drift, int64_t max_win);
std::pair<std::vector<Anchor>, bool> anchor_windows(const HostParams &p, const uint8_t *q, int64_t qlen,
                                                    const uint8_t *consensus, int64_t clen);
// Progressive guide order (-p, src/minimizer.rs:505-578): the order in which
// the reads are added to the graph. The identity unless progressive, with at
// least two reads and a nucleotide alphabet.
std::vector<int64_t> guide_order(const HostParams &p, const std::vector<const uint8_t *> &seqs,
                                 const std::vector<int64_t> &lens);

}  // namespace poa
