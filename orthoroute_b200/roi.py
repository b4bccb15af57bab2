"""Device ROI extraction with the reference ROIExtractor interface
(orthoroute/algorithms/manhattan/unified_pathfinder.py:1345-1780)."""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr
from .solver import DeviceGraph, _stream


def _coords(lattice, n):
    if hasattr(lattice, "idx_to_coord"):
        return lattice.idx_to_coord(int(n))
    x, y, z = lattice.coords(int(n))
    return int(x), int(y), int(z)


class DeviceROIExtractor:
    """``extract_roi`` / ``extract_roi_bfs`` on the GPU.  Results are returned
    as numpy arrays like the reference (``return_device=True`` keeps them as
    CUDA tensors)."""

    def __init__(self, graph, use_gpu: bool = True, lattice=None, return_device: bool = False):
        self.dg = graph if isinstance(graph, DeviceGraph) else graph.dg
        self.N = self.dg.N
        self.lattice = lattice
        self.return_device = return_device

    def extract_roi(self, src: int, dst: int, initial_radius: int = 40, stagnation_bonus: float = 0.0,
                    portal_seeds: list = None):
        """UPF:1619-1634: radius = max(60, int(0.75*manhattan + 2*bonus))."""
        if self.lattice is not None:
            sx, sy, _ = _coords(self.lattice, src)
            dx, dy, _ = _coords(self.lattice, dst)
            manhattan = abs(dx - sx) + abs(dy - sy)
            radius = max(60, int(manhattan * 0.75 + stagnation_bonus * 2.0))
        else:
            radius = initial_radius
        return self.extract_roi_bfs(src, dst, initial_radius=radius, stagnation_bonus=stagnation_bonus,
                                    portal_seeds=portal_seeds)

    def extract_roi_bfs(self, src: int, dst: int, initial_radius: int = 40, stagnation_bonus: float = 0.0,
                        portal_seeds: list = None):
        """UPF:1636-1734: bidirectional BFS, depth <= min(radius + 2*bonus, 150),
        at most max_roi_nodes (default 50 000) nodes."""
        if portal_seeds:
            raise NotImplementedError("portal seeds are not supported by the device ROI extractor")
        max_depth = min(int(initial_radius + stagnation_bonus * 2.0), 150)
        max_nodes = int(getattr(self, "max_roi_nodes", 50_000))
        roi, g2r = self.dg.roi_bfs(int(src), int(dst), max_depth, max_nodes)
        if self.return_device:
            return roi, g2r
        return roi.cpu().numpy(), g2r.cpu().numpy()

    def box_map(self, box) -> torch.Tensor:
        """global_to_roi of an inclusive box [x0,x1,y0,y1,z0,z1] (device)."""
        g2r = torch.empty(self.N, dtype=torch.int32, device=self.dg.device)
        b = np.ascontiguousarray(box, dtype=np.int32)
        check(_lib.load().orsp_roi_box_map(self.dg.handle, ptr(b), ptr(g2r), _stream()), "orsp_roi_box_map")
        return g2r
