// GFA input for initial graphs (the reference's io::read_gfa, declared by
// minipoa-rs src/lib.rs:7 and called at lib.rs:214-218; its source file is
// absent from the reference tree, so the behaviour follows its tests).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "host_graph.h"

namespace poa {

// A graph under construction on the host with graph.rs's mutation rules
// (add_node, add_edge, add_path: src/graph.rs:42-122): per node its incoming
// and outgoing lists with weights in insertion order, coverage and column
// group; paths as (sequence id, node ids). Node 0 is the source, node 1 the
// sink. Ranks are assigned on the device after import.
struct BuildGraph {
  int sigma = 0;
  std::vector<int32_t> base, parent, coverage;
  std::vector<std::vector<int32_t>> in_id, in_w, out_id, out_w;
  std::vector<int32_t> aligned;  // [n * sigma], -1 = None
  std::vector<int32_t> path_seq;
  std::vector<std::vector<int32_t>> paths;

  explicit BuildGraph(const HostParams &p);
  int32_t add_node(int b);
  void add_edge(int32_t from, int32_t to);
  bool has_edge(int32_t from, int32_t to) const;
  // add_path with every item naming an existing node (the source first)
  void add_path_nodes(int32_t seq_id, const std::vector<int32_t> &ids);
  int32_t n() const { return int32_t(base.size()); }
  int64_t edges() const;
  // Graph::toposort(false) (src/graph.rs:125-178): the stable LIFO Kahn
  // order; rank_of[node] and order[rank]. Throws with the reference's message
  // on a cycle.
  void toposort(std::vector<int32_t> &rank_of, std::vector<int32_t> &order) const;
};

struct GfaRecord {
  std::string name, seq;
};

// Parses GFA text into a graph and its path records. Construction order:
// nodes per segment base in S-line order; each path in P-line order through
// add_path from the source; the segment-internal and L-line edges that no
// path created; edges from the source to every node without an incoming
// edge and from every node without an outgoing edge to the sink. Throws
// std::runtime_error with the reason on invalid input (duplicate segments,
// unknown references, reverse orientations, non-zero overlaps, self links,
// segments without sequence, a path revisiting a node: "revisits"). Cycles
// are found by the toposort that follows the import.
BuildGraph read_gfa(const HostParams &p, const char *text, size_t len, std::vector<GfaRecord> &records);

}  // namespace poa
