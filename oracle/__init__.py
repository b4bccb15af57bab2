"""ORACLE - test infrastructure only.

CPU restatements of the reference hot path, used as the checker by tests/,
by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product
package (orthoroute_b200) never imports this package.
"""
from .orsp_oracle import (  # noqa: F401
    build_oracle,
    dijkstra,
    roi_bfs,
    path_to_edges,
    batch_bbox,
    update_costs,
    update_present_ema,
    update_history,
    compute_overuse,
    via_edge_metadata,
    via_usage,
    via_present,
    via_penalties,
    via_hard_block,
)
