"""build_lattice writes each node's CSR row layer by layer.  This checks it
against the dense construction it replaced (every slot of every node as an
[N, slots] table, masked in slot order), array for array, over the planar,
via and duplicate-via options and the 1-, 2- and many-layer cases."""
import numpy as np
import pytest

from orthoroute_b200.lattice import build_lattice, layer_directions


def _dense(nx, ny, nz, planar="all", vias="adjacent", pitch=1.0, via_cost=3.0, duplicate_vias=False):
    N = nx * ny * nz
    dirs = layer_directions(nz)
    z, y, x = (a.reshape(-1) for a in np.meshgrid(np.arange(nz, dtype=np.int64), np.arange(ny, dtype=np.int64),
                                                  np.arange(nx, dtype=np.int64), indexing="ij"))
    node = np.arange(N, dtype=np.int64)
    if planar == "all" or nz <= 2:
        pl = np.ones(nz, dtype=bool)
    else:
        pl = np.zeros(nz, dtype=bool)
        pl[1:nz - 1] = True
    has_h = np.array([d in ("h", "hv") for d in dirs]) & pl
    has_v = np.array([d in ("v", "hv") for d in dirs]) & pl
    tgt, cst = [], []
    hz, vz = has_h[z], has_v[z]
    for ok, step in ((hz & (x > 0), -1), (hz & (x < nx - 1), 1), (vz & (y > 0), -nx), (vz & (y < ny - 1), nx)):
        tgt.append(np.where(ok, node + step, -1))
        cst.append(np.full(N, np.float32(pitch), np.float32))
    plane = nx * ny
    if vias == "adjacent":
        for dz in (-1, 1):
            tz = z + dz
            tgt.append(np.where((tz >= 0) & (tz < nz), node + dz * plane, -1))
            cst.append(np.full(N, np.float32(via_cost), np.float32))
    else:
        if nz == 2:
            legal = {(0, 1), (1, 0)}
        else:
            rt = range(1, nz - 1)
            legal = {(a, b) for a in rt for b in rt if a != b} | {(0, b) for b in rt} | {(b, 0) for b in rt}
        for tz in range(nz):
            ok = np.array([(zz, tz) in legal for zz in range(nz)])[z]
            c = (via_cost * (1.0 + 0.15 * (np.abs(tz - z) - 1))).astype(np.float32)
            for _ in range(2 if duplicate_vias else 1):
                tgt.append(np.where(ok, node + (tz - z) * plane, -1))
                cst.append(c)
    t = np.stack(tgt, axis=1)
    c = np.stack(cst, axis=1)
    m = t >= 0
    deg = m.sum(axis=1)
    indptr = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(deg, out=indptr[1:])
    ind = t[m]
    src = np.repeat(node, deg)
    return (indptr.astype(np.int32), ind.astype(np.int32), c[m], (src // plane).astype(np.uint8),
            ((ind // plane) != (src // plane)).astype(np.uint8))


@pytest.mark.parametrize("shape,planar,vias,dup", [
    ((7, 5, 1), "all", "adjacent", False),
    ((6, 5, 2), "all", "full", False),
    ((6, 5, 2), "all", "adjacent", True),
    ((9, 6, 4), "inner", "full", True),
    ((10, 8, 6), "all", "full", False),
    ((8, 7, 3), "inner", "adjacent", False),
    ((11, 4, 7), "all", "adjacent", False),
    ((5, 9, 8), "inner", "full", False),
])
def test_build_lattice_matches_dense_construction(shape, planar, vias, dup):
    nx, ny, nz = shape
    lat = build_lattice(nx, ny, nz, planar=planar, vias=vias, duplicate_vias=dup, pitch=0.4, via_cost=2.5)
    ref = _dense(nx, ny, nz, planar, vias, 0.4, 2.5, dup)
    for got, want, name in zip((lat.indptr, lat.indices, lat.base_cost, lat.edge_layer, lat.edge_kind), ref,
                               ("indptr", "indices", "base_cost", "edge_layer", "edge_kind")):
        assert got.dtype == want.dtype and np.array_equal(got, want), name
