"""B200-native PathFinder search for OrthoRoute (sm_100a CUDA behind a C ABI).

Public entry points mirror the reference router's hot-path interfaces:

* ``GpuSolver``            - router.solver.gpu_solver (CUDADijkstra interface)
* ``DeviceEdgeAccountant`` - router.accounting (EdgeAccountant interface)
* ``DeviceROIExtractor``   - router.roi_extractor (ROIExtractor interface)
* ``PathFinder``           - the negotiation loop on the device kernels
* ``install``              - wires the whole B200 path into a reference PathFinderRouter
                             (orthoroute_b200.dropin: solver, accountant, ROI, via steps)
"""
from .lattice import Lattice, Board, build_lattice  # noqa: F401


__all__ = ["Lattice", "Board", "build_lattice", "GpuSolver", "DeviceGraph", "DeviceEdgeAccountant",
           "DeviceROIExtractor", "PathFinder", "NegotiationConfig", "install"]


def __getattr__(name):
    # torch-dependent modules load lazily so that the lattice helpers import
    # without CUDA.
    if name in ("GpuSolver", "DeviceGraph"):
        from . import solver

        return getattr(solver, name)
    if name == "DeviceEdgeAccountant":
        from .accounting import DeviceEdgeAccountant

        return DeviceEdgeAccountant
    if name == "DeviceROIExtractor":
        from .roi import DeviceROIExtractor

        return DeviceROIExtractor
    if name == "install":
        from .dropin import install

        return install
    if name in ("PathFinder", "NegotiationConfig"):
        from . import negotiate

        return getattr(negotiate, name)
    raise AttributeError(name)
