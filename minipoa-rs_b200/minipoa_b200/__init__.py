"""B200-native partial-order alignment (the minipoa-rs POA hot path).

Mirrors the reference library: Params, Sequence, AlignedBase (src/lib.rs),
align_sequences / extend_graph / run / dp_backend (src/lib.rs), align / poa
(src/align.rs) and Graph (src/graph.rs), over the C ABI of
include/minipoa_b200.h. Batch runs many independent read sets on the GPU;
Server admits read sets as they arrive (continuous batching).
"""
from .params import AlignedBase, CParams, Params, Sequence, default_matrix  # noqa: F401
from .api import (  # noqa: F401
    Anchor, Batch, Context, Graph, Minimizer, PoaError, Server, align, anchor_windows, chain, collect_anchors,
    partition_windows, repeat_intervals, sketch, guide_order, align_sequences, default_context, dp_backend, extend_graph, int_peak, poa, read_gfa, run,
)
