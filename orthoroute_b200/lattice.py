"""Synthetic routing lattices and boards in the reference's data formats.

A lattice is the 3D grid graph of OrthoRoute's Manhattan router in CSR form
(int32 indptr/indices, float32 base costs, uint8 edge_layer/edge_kind), with
nodes numbered like KiCadGeometry.node_index
(orthoroute/algorithms/manhattan/pathfinder/kicad_geometry.py:63-66):
``node = z*Nx*Ny + y*Nx + x``.

Layer directions follow Lattice3D._assign_directions
(orthoroute/algorithms/manhattan/unified_pathfinder.py:1091-1106): F.Cu (z=0)
vertical, then z odd horizontal / z even vertical; a 2-layer board allows both
directions on both layers.  Two edge sets are supported:

* ``planar="all", vias="adjacent"`` - the benchmark lattice: planar edges on
  every layer and vias only between adjacent layers.
* ``planar="inner", vias="full"`` - the reference's own Lattice3D.build_graph
  (UPF:1195-1287): planar edges on inner layers only and blind/buried vias
  between every pair of routing layers plus F.Cu -> inner (cost
  via_cost*(1 + 0.15*(span-1))).  The reference emits each via pair twice
  (UPF:1264-1276); ``duplicate_vias=True`` reproduces that.

Within a node's CSR row the edges are ordered planar (-, +) then vias by
increasing target layer; the CSR is sorted by source like CSRGraph.finalize
(UPF:674-745).  Everything is vectorised; a 1000x1000x12 lattice builds in a
few seconds.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np


def layer_directions(nz: int) -> list:
    """'h', 'v' or 'hv' per layer (Lattice3D._assign_directions, UPF:1091-1106)."""
    if nz == 2:
        return ["hv", "hv"]
    return ["v" if z == 0 else ("h" if z % 2 == 1 else "v") for z in range(nz)]


@dataclass
class Lattice:
    nx: int
    ny: int
    nz: int
    indptr: np.ndarray  # int32[N+1]
    indices: np.ndarray  # int32[E]
    base_cost: np.ndarray  # float32[E]
    edge_layer: np.ndarray  # uint8[E] (source layer, CSRGraph.finalize UPF:750)
    edge_kind: np.ndarray  # uint8[E] (1 = via)
    pitch: float = 1.0
    meta: dict = field(default_factory=dict)

    @property
    def N(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def E(self) -> int:
        return int(self.indices.shape[0])

    @property
    def plane(self) -> int:
        return self.nx * self.ny

    def node(self, x, y, z):
        return (np.asarray(z) * self.ny + np.asarray(y)) * self.nx + np.asarray(x)

    def coords(self, n):
        n = np.asarray(n)
        z = n // self.plane
        r = n - z * self.plane
        return r % self.nx, r // self.nx, z

    def edge_src(self) -> np.ndarray:
        deg = np.diff(self.indptr)
        return np.repeat(np.arange(self.N, dtype=np.int32), deg)


def build_lattice(
    nx: int,
    ny: int,
    nz: int,
    *,
    planar: str = "all",
    vias: str = "adjacent",
    pitch: float = 1.0,
    via_cost: float = 3.0,
    duplicate_vias: bool = False,
) -> Lattice:
    """Builds the CSR lattice described in the module docstring.  Each node's
    out-edges are in slot order: -x, +x, -y, +y (those its layer has), then
    its vias by target layer (each twice with duplicate_vias).  The rows are
    written layer by layer: the via targets of a layer are the same for all
    its nodes, so a layer's via block is one scatter."""
    if planar not in ("all", "inner") or vias not in ("adjacent", "full"):
        raise ValueError("planar must be 'all'|'inner', vias 'adjacent'|'full'")
    N = nx * ny * nz
    if N >= 2**31:
        raise ValueError("lattice too large for int32 node ids")
    dirs = layer_directions(nz)
    if planar == "all" or nz <= 2:
        planar_layer = np.ones(nz, dtype=bool)
    else:
        planar_layer = np.zeros(nz, dtype=bool)
        planar_layer[1 : nz - 1] = True
    has_h = np.array([d in ("h", "hv") for d in dirs]) & planar_layer
    has_v = np.array([d in ("v", "hv") for d in dirs]) & planar_layer
    plane = nx * ny
    r = np.arange(plane, dtype=np.int64)
    xr = r % nx
    yr = r // nx

    # via targets of a node on layer zz, in slot order, and their costs
    if vias == "full":
        # Lattice3D.get_legal_via_pairs (UPF:1136-1172): routing layers 1..nz-2
        # pairwise, plus F.Cu (0) <-> every routing layer; 2 layers: (0,1).
        if nz == 2:
            legal = {(0, 1), (1, 0)}
        else:
            routing = range(1, nz - 1)
            legal = {(a, b) for a in routing for b in routing if a != b}
            legal |= {(0, b) for b in routing} | {(b, 0) for b in routing}
        reps = 2 if duplicate_vias else 1
    via_t, via_c = [], []
    for zz in range(nz):
        if vias == "adjacent":
            t = [zz + dz for dz in (-1, 1) if 0 <= zz + dz < nz]
            c = [np.float32(via_cost)] * len(t)
        else:
            t = [tz for tz in range(nz) if (zz, tz) in legal for _ in range(reps)]
            # cost grows by 15 % per layer spanned beyond the first
            c = [np.float32(via_cost * (1.0 + 0.15 * (abs(tz - zz) - 1))) for tz in t]
        via_t.append(np.asarray(t, dtype=np.int64))
        via_c.append(np.asarray(c, dtype=np.float32))

    def planar_slots(zz):
        out = []
        if has_h[zz]:
            out += [(xr > 0, -1), (xr < nx - 1, 1)]
        if has_v[zz]:
            out += [(yr > 0, -nx), (yr < ny - 1, nx)]
        return out

    deg = np.empty(N, dtype=np.int64)
    for zz in range(nz):
        d = np.full(plane, via_t[zz].size, dtype=np.int64)
        for m, _ in planar_slots(zz):
            d += m
        deg[zz * plane:(zz + 1) * plane] = d
    indptr = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(deg, out=indptr[1:])
    E = int(indptr[-1])
    if E >= 2**31:
        raise ValueError("too many edges for int32 CSR")
    indices = np.empty(E, dtype=np.int32)
    base_cost = np.empty(E, dtype=np.float32)
    edge_kind = np.zeros(E, dtype=np.uint8)
    edge_layer = np.empty(E, dtype=np.uint8)
    pitch32 = np.float32(pitch)
    for zz in range(nz):
        a = zz * plane
        start = indptr[a:a + plane]
        k = np.zeros(plane, dtype=np.int64)
        for m, step in planar_slots(zz):
            pos = start[m] + k[m]
            indices[pos] = a + r[m] + step
            base_cost[pos] = pitch32
            k += m
        nv = via_t[zz].size
        if nv:
            pos = (start + k)[:, None] + np.arange(nv, dtype=np.int64)[None, :]
            indices[pos] = via_t[zz][None, :] * plane + r[:, None]
            base_cost[pos] = via_c[zz][None, :]
            edge_kind[pos] = 1
        edge_layer[indptr[a]:indptr[a + plane]] = zz
    return Lattice(
        nx=nx,
        ny=ny,
        nz=nz,
        indptr=indptr.astype(np.int32),
        indices=indices,
        base_cost=base_cost,
        edge_layer=edge_layer,
        edge_kind=edge_kind,
        pitch=pitch,
        meta={"planar": planar, "vias": vias, "via_cost": via_cost, "duplicate_vias": duplicate_vias},
    )


def uniform_weights(lat: Lattice, seed: int, blocked_frac: float = 0.0, via_weight: float = 3.0) -> np.ndarray:
    """fp32 weights exactly uniform in [1, 2) on planar edges (1 + (u32 >> 9) * 2^-23),
    via_weight on vias, and +inf on a Bernoulli(blocked_frac) subset."""
    rng = np.random.default_rng(seed)
    u = rng.integers(0, 2**32, size=lat.E, dtype=np.uint64).astype(np.uint32)
    w = (np.uint32(0x3F800000) | (u >> np.uint32(9))).view(np.float32).copy()
    w[lat.edge_kind == 1] = np.float32(via_weight)
    if blocked_frac > 0:
        blocked = rng.random(lat.E) < blocked_frac
        w[blocked] = np.float32(np.inf)
    return w


@dataclass
class Board:
    lattice: Lattice
    src: np.ndarray  # int32[M] node ids
    dst: np.ndarray  # int32[M]
    names: list
    meta: dict = field(default_factory=dict)


def board_uniform_pins(nx: int, ny: int, nz: int, nets: int, seed: int, **lat_kw) -> Board:
    """Two-pin nets with pins uniform on the top layer, all pin cells distinct."""
    lat = build_lattice(nx, ny, nz, **lat_kw)
    rng = np.random.default_rng(seed)
    cells = rng.choice(nx * ny, size=2 * nets, replace=False).astype(np.int64)
    src = cells[:nets].astype(np.int32)
    dst = cells[nets:].astype(np.int32)
    names = [f"N{i}" for i in range(nets)]
    return Board(lat, src, dst, names, meta={"kind": "uniform_pins", "seed": seed})


def board_footprints(
    nx: int,
    ny: int,
    nz: int,
    nets: int,
    footprints: Optional[int],
    seed: int,
    rows: int = 2,
    cols: int = 50,
    **lat_kw,
) -> Board:
    """Nets between connector footprints of rows x cols pins at 1-cell pitch on
    the top layer.  Each net joins two different random footprints; every pin
    is used by at most one net (a pin shared by more nets than its 3 escape
    edges could never reach zero overuse).  footprints=None picks the smallest
    count with 10 % spare pins."""
    lat = build_lattice(nx, ny, nz, **lat_kw)
    rng = np.random.default_rng(seed)
    pins_per = rows * cols
    if footprints is None:
        # every net joins two different footprints, so at least two
        footprints = max(2, int(np.ceil(1.1 * 2 * nets / pins_per)))
    if footprints * pins_per < 2 * nets:
        raise ValueError("not enough pins for the nets")
    # non-overlapping placement with a 2-cell keep-out around each footprint
    occ = np.zeros((ny, nx), dtype=bool)
    origins = []
    tries = 0
    while len(origins) < footprints:
        tries += 1
        if tries > 200000:
            raise RuntimeError("could not place footprints")
        ox = int(rng.integers(2, nx - cols - 2))
        oy = int(rng.integers(2, ny - rows - 2))
        if occ[oy - 2 : oy + rows + 2, ox - 2 : ox + cols + 2].any():
            continue
        occ[oy - 2 : oy + rows + 2, ox - 2 : ox + cols + 2] = True
        origins.append((ox, oy))
    free = [list(rng.permutation(pins_per)) for _ in range(footprints)]
    nfree = np.full(footprints, pins_per, dtype=np.float64)
    src = np.empty(nets, dtype=np.int64)
    dst = np.empty(nets, dtype=np.int64)
    for i in range(nets):
        # footprints drawn in proportion to their free pins
        a = int(rng.choice(footprints, p=nfree / nfree.sum()))
        w = nfree.copy()
        w[a] = 0
        if w.sum() == 0:
            raise RuntimeError("ran out of free pins")
        b = int(rng.choice(footprints, p=w / w.sum()))
        pa, pb = free[a].pop(), free[b].pop()
        nfree[a] -= 1
        nfree[b] -= 1
        ax, ay = origins[a][0] + pa % cols, origins[a][1] + pa // cols
        bx, by = origins[b][0] + pb % cols, origins[b][1] + pb // cols
        src[i] = ay * nx + ax
        dst[i] = by * nx + bx
    names = [f"N{i}" for i in range(nets)]
    return Board(
        lat,
        src.astype(np.int32),
        dst.astype(np.int32),
        names,
        meta={"kind": "footprints", "seed": seed, "footprints": footprints, "origins": origins},
    )


def bbox_with_margin(lat: Lattice, src, dst, margin: int, z_all: bool = True) -> np.ndarray:
    """Inclusive boxes [x0,x1,y0,y1,z0,z1] per net: bounding box of the two
    pins plus `margin` cells, clipped to the lattice, all layers."""
    sx, sy, sz = lat.coords(np.asarray(src))
    dx, dy, dz = lat.coords(np.asarray(dst))
    x0 = np.clip(np.minimum(sx, dx) - margin, 0, lat.nx - 1)
    x1 = np.clip(np.maximum(sx, dx) + margin, 0, lat.nx - 1)
    y0 = np.clip(np.minimum(sy, dy) - margin, 0, lat.ny - 1)
    y1 = np.clip(np.maximum(sy, dy) + margin, 0, lat.ny - 1)
    if z_all:
        z0 = np.zeros_like(x0)
        z1 = np.full_like(x0, lat.nz - 1)
    else:
        z0 = np.clip(np.minimum(sz, dz) - margin, 0, lat.nz - 1)
        z1 = np.clip(np.maximum(sz, dz) + margin, 0, lat.nz - 1)
    return np.stack([x0, x1, y0, y1, z0, z1], axis=1).astype(np.int32)


def random_boxes(lat: Lattice, count: int, seed: int, lo=(20, 20, 4), hi=(400, 400, 16)):
    """Boxes with each side log-uniform in [lo, hi] (clipped to the lattice),
    placed uniformly, with source and target uniform inside each box."""
    rng = np.random.default_rng(seed)
    dims = []
    for a, b, n in zip(lo, hi, (lat.nx, lat.ny, lat.nz)):
        s = np.exp(rng.uniform(np.log(a), np.log(b), size=count)).astype(np.int64)
        dims.append(np.clip(s, 1, n))
    w, h, d = dims
    x0 = (rng.random(count) * (lat.nx - w + 1)).astype(np.int64)
    y0 = (rng.random(count) * (lat.ny - h + 1)).astype(np.int64)
    z0 = (rng.random(count) * (lat.nz - d + 1)).astype(np.int64)
    boxes = np.stack([x0, x0 + w - 1, y0, y0 + h - 1, z0, z0 + d - 1], axis=1).astype(np.int32)
    sx = x0 + (rng.random(count) * w).astype(np.int64)
    sy = y0 + (rng.random(count) * h).astype(np.int64)
    sz = z0 + (rng.random(count) * d).astype(np.int64)
    tx = x0 + (rng.random(count) * w).astype(np.int64)
    ty = y0 + (rng.random(count) * h).astype(np.int64)
    tz = z0 + (rng.random(count) * d).astype(np.int64)
    src = lat.node(sx, sy, sz).astype(np.int32)
    dst = lat.node(tx, ty, tz).astype(np.int32)
    return boxes, src, dst


def box_edge_count(lat: Lattice, boxes: np.ndarray) -> np.ndarray:
    """Directed edges with both ends inside each box (the graph a box-ROI
    search runs on), for lattices with adjacent-layer vias."""
    if lat.meta.get("vias", "adjacent") != "adjacent" or lat.meta.get("duplicate_vias", False):
        raise ValueError("box_edge_count: adjacent, single vias only")
    dirs = layer_directions(lat.nz)
    if lat.meta.get("planar", "all") == "inner":
        dirs = [d if 0 < z < lat.nz - 1 else "" for z, d in enumerate(dirs)]
    b = np.asarray(boxes, dtype=np.int64)
    bw, bh, bd = b[:, 1] - b[:, 0] + 1, b[:, 3] - b[:, 2] + 1, b[:, 5] - b[:, 4] + 1
    has_h = np.array(["h" in d for d in dirs], dtype=np.int64)
    has_v = np.array(["v" in d for d in dirs], dtype=np.int64)
    ch = np.concatenate([[0], np.cumsum(has_h)])
    cv = np.concatenate([[0], np.cumsum(has_v)])
    nh = ch[b[:, 5] + 1] - ch[b[:, 4]]
    nv = cv[b[:, 5] + 1] - cv[b[:, 4]]
    return 2 * (nh * (bw - 1) * bh + nv * bw * (bh - 1) + bw * bh * (bd - 1))
