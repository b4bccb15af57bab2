"""Device-resident edge accounting with the reference EdgeAccountant interface
(orthoroute/algorithms/manhattan/unified_pathfinder.py:799-1068).

Arrays are float32 torch CUDA tensors: ``present``, ``present_ema``,
``history``, ``capacity``, ``total_cost``.  The reference's ``canonical``
dict (edge -> committed count) is an int32 ``usage`` tensor; ``canonical``
is still available as a dict view for callers that read it.
"""
from __future__ import annotations

from typing import Dict, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr
from .solver import _require_cuda, _stream, as_device


def _f32(x: float) -> float:
    """Python float -> the float32 value numpy would use for a weak scalar."""
    return float(np.float32(x))


class DeviceEdgeAccountant:
    def __init__(self, num_edges: int, use_gpu: bool = True, device=None):
        _require_cuda()
        self.E = int(num_edges)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        z = lambda: torch.zeros(self.E, dtype=torch.float32, device=self.device)  # noqa: E731
        self.present = z()
        self.present_ema = z()
        self.history = z()
        self.capacity = torch.ones(self.E, dtype=torch.float32, device=self.device)
        self.usage = torch.zeros(self.E, dtype=torch.int32, device=self.device)
        self.total_cost = None
        self.use_gpu = True
        self._over2 = torch.zeros(2, dtype=torch.int64, device=self.device)
        self._over2_h = torch.zeros(2, dtype=torch.int64).pin_memory()

    # --- canonical store --------------------------------------------------
    @property
    def canonical(self) -> Dict[int, int]:
        u = self.usage.cpu().numpy()
        nz = np.nonzero(u)[0]
        return {int(i): int(u[i]) for i in nz}

    def refresh_from_canonical(self):
        """present = float(count) (UPF:814-819)."""
        check(_lib.load().orsp_present_from_usage(self.E, ptr(self.usage), ptr(self.present), _stream()),
              "orsp_present_from_usage")

    def _edges(self, edge_indices) -> torch.Tensor:
        return as_device(edge_indices, torch.int32, self.device)

    def commit_path(self, edge_indices):
        """count += 1, present += 1 per edge (UPF:821-826)."""
        e = self._edges(edge_indices)
        if e.numel():
            check(_lib.load().orsp_commit_edges(int(e.numel()), ptr(e), ptr(self.usage), ptr(self.present), 1,
                                                _stream()), "orsp_commit_edges")

    def clear_path(self, edge_indices):
        """count -= 1 (>= 0), present = max(0, present - 1) (UPF:828-836)."""
        e = self._edges(edge_indices)
        if e.numel():
            check(_lib.load().orsp_commit_edges(int(e.numel()), ptr(e), ptr(self.usage), ptr(self.present), -1,
                                                _stream()), "orsp_commit_edges")

    def verify_present_matches_canonical(self) -> bool:
        return bool(torch.sum(torch.abs(self.present - self.usage.float())).item() <= 0.01)

    # --- per-iteration updates -------------------------------------------
    def compute_overuse(self, router_instance=None) -> Tuple[int, int]:
        """(sum of overuse incl. via column/segment overuse, overused edge count)
        (UPF:838-876)."""
        check(_lib.load().orsp_overuse(self.E, ptr(self.present), ptr(self.capacity), ptr(self._over2),
                                       ptr(self._over2_h), _stream()), "orsp_overuse")
        s, c = (int(v) for v in self._over2_h.tolist())
        if router_instance is not None:
            for use, cap in (("via_col_use", "via_col_cap"), ("via_seg_use", "via_seg_cap")):
                if hasattr(router_instance, use) and hasattr(router_instance, cap):
                    u = getattr(router_instance, use)
                    k = getattr(router_instance, cap)
                    u = u.cpu().numpy() if isinstance(u, torch.Tensor) else np.asarray(u)
                    k = k.cpu().numpy() if isinstance(k, torch.Tensor) else np.asarray(k)
                    s += int(np.maximum(0, u - k).sum())
        return s, c

    def update_present_ema(self, beta: float = 0.60):
        """present_ema = beta*present + (1-beta)*present_ema (UPF:963-971)."""
        check(_lib.load().orsp_update_present_ema(self.E, ptr(self.present), ptr(self.present_ema), _f32(beta),
                                                  _f32(1.0 - beta), _stream()), "orsp_update_present_ema")

    def update_history(self, gain: float, base_costs=None, history_cap_multiplier: float = 10.0,
                       decay_factor: float = 0.98, use_raw_present: bool = False):
        """UPF:898-961."""
        base = None if base_costs is None else as_device(base_costs, torch.float32, self.device)
        pres = self.present if use_raw_present else self.present_ema
        check(_lib.load().orsp_update_history(self.E, ptr(self.history), ptr(pres), ptr(self.capacity), ptr(base),
                                              _f32(gain), _f32(history_cap_multiplier), _f32(decay_factor),
                                              _stream()), "orsp_update_history")

    def update_costs(self, base_costs, pres_fac: float, hist_weight: float = 1.0, add_jitter: bool = True,
                     via_cost_multiplier: float = 1.0, base_cost_weight: float = 0.01, *, edge_layer=None,
                     layer_bias_per_layer=None, edge_kind=None):
        """UPF:973-1043, written to ``total_cost``."""
        base = as_device(base_costs, torch.float32, self.device)
        use_bias = edge_layer is not None and layer_bias_per_layer is not None and edge_kind is not None
        el = as_device(edge_layer, torch.uint8, self.device) if use_bias else None
        ek = as_device(edge_kind, torch.uint8, self.device) if use_bias else None
        lb = as_device(layer_bias_per_layer, torch.float32, self.device) if use_bias else None
        if self.total_cost is None or self.total_cost.numel() != self.E:
            self.total_cost = torch.empty(self.E, dtype=torch.float32, device=self.device)
        check(_lib.load().orsp_update_costs(self.E, ptr(base), ptr(self.present_ema), ptr(self.capacity),
                                            ptr(self.history), ptr(el), ptr(ek), ptr(lb), _f32(pres_fac),
                                            _f32(hist_weight), _f32(via_cost_multiplier), _f32(base_cost_weight),
                                            1 if add_jitter else 0, ptr(self.total_cost), _stream()),
              "orsp_update_costs")
