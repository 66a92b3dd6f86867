"""B200-native partial-order alignment (minipoa-rs hot path) -- host API."""
from .params import AlignedBase, CParams, Params, Sequence, default_matrix  # noqa: F401
