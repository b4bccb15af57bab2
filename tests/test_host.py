"""Host-side checks that need no GPU: the C ABI library loads and exports every
symbol the headers in include/ declare, index arithmetic, lattice generator."""
import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent.parent


def _header_symbols():
    text = "".join(p.read_text() for p in sorted((REPO / "include").glob("*.h")))
    return sorted(set(re.findall(r"ORSP_API\s+[\w\s\*]+?\b(orsp_\w+)\s*\(", text)))


def test_library_exports_header_symbols():
    from orthoroute_b200 import _lib
    from orthoroute_b200.build import build_library

    build_library()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    syms = _header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/ but not exported"
    assert set(syms) == set(_lib.exported_symbols()), "ctypes table and header disagree"
    L = _lib.load()
    assert L.orsp_abi_version() == 1
    assert L.orsp_status_string(-3) == b"device timeout"


def test_integration_guide_names_every_entry_point():
    """Every entry point the headers declare appears in the integration
    guide, which maps each to the reference interface it replaces."""
    guide = (REPO / "INTEGRATION.md").read_text()
    missing = [s for s in _header_symbols() if s not in guide]
    assert not missing, missing


def test_host_validation_without_gpu():
    """Argument checks run on the host before any CUDA call."""
    from orthoroute_b200 import _lib

    L = _lib.load()
    h = ctypes.c_void_p()
    ip = np.array([0, 1], dtype=np.int32)
    ix = np.array([5], dtype=np.int32)  # out of range
    rc = L.orsp_graph_create(1, 1, _lib.ptr(ip), _lib.ptr(ix), 0, 0, 0, 0, ctypes.byref(h))
    assert rc == _lib.ORSP_ERR_ARG
    assert b"out of range" in L.orsp_last_error()
    rc = L.orsp_update_costs(10, None, None, None, None, None, None, None, 1.0, 1.0, 1.0, 1.0, 1, None, 0)
    assert rc == _lib.ORSP_ERR_ARG
    # the snapshot routing loop: negative repair rounds, and no graph
    n = ctypes.c_int64(-1)
    rc = L.orsp_route_nets_snapshot(None, 1, None, None, None, 1, None, 0, None, -1, None, None, 16, None, None,
                                    None, None, None, None, None, 1.0, 1.0, 1.0, 1.0, 0, ctypes.byref(n), 0)
    assert rc == _lib.ORSP_ERR_ARG and b"repair_rounds" in L.orsp_last_error()
    rc = L.orsp_route_nets_snapshot(None, 1, None, None, None, 1, None, 0, None, 2, None, None, 16, None, None,
                                    None, None, None, None, None, 1.0, 1.0, 1.0, 1.0, 0, ctypes.byref(n), 0)
    assert rc == _lib.ORSP_ERR_ARG and n.value == 0


def test_fastdiv_exhaustive_samples(tmp_path):
    """The Granlund-Montgomery divider used by the batched kernel, compiled for
    the host from the same header."""
    src = tmp_path / "t.cpp"
    src.write_text(
        '#define __host__\n#define __device__\n#define __forceinline__ inline\n'
        f'#include "{REPO}/orthoroute_b200/csrc/fastdiv.cuh"\n'
        "#include <cstdio>\n#include <cstdint>\n"
        "int main(){ uint32_t ds[]={1,2,3,7,100,101,600,1000,360000,1000000,6480000,(1u<<31)-1,1u<<31};\n"
        " uint64_t x=88172645463325252ull; long bad=0;\n"
        " for(uint32_t d: ds){ FastDiv f; f.init(d);\n"
        "  for(int i=0;i<200000;++i){ x^=x<<13; x^=x>>7; x^=x<<17; uint32_t n=(uint32_t)x;\n"
        "   if(i<1000) n=i; if(i>=1000&&i<2000) n=0xffffffffu-(i-1000);\n"
        "   if(f.div(n)!=n/d) ++bad; }}\n"
        " printf(\"%ld\\n\",bad); return bad!=0; }\n"
    )
    exe = tmp_path / "t"
    subprocess.run(["g++", "-O2", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout


def test_lattice_shapes_and_directions():
    from orthoroute_b200.lattice import build_lattice

    lat = build_lattice(100, 100, 4)
    assert (lat.N, lat.E) == (40_000, 139_200)
    lat = build_lattice(600, 600, 18)
    assert lat.E == 25_178_400
    small = build_lattice(5, 4, 4)
    src = small.edge_src()
    x0, y0, z0 = small.coords(src)
    x1, y1, z1 = small.coords(small.indices)
    planar = z0 == z1
    # F.Cu and even layers vertical, odd layers horizontal
    assert np.all((x0 == x1)[planar & (z0 % 2 == 0)])
    assert np.all((y0 == y1)[planar & (z0 % 2 == 1)])
    assert np.all(np.abs(z1 - z0)[~planar] == 1)
    assert np.array_equal(small.edge_kind.astype(bool), ~planar)
    # CSR sorted by source and symmetric topology
    pairs = set(zip(src.tolist(), small.indices.tolist()))
    assert all((v, u) in pairs for u, v in pairs)


def test_reference_style_lattice_matches_reference_graph(golden):
    """planar='inner', vias='full' reproduces the reference Lattice3D edge set
    (as a multiset of (u, v, cost))."""
    from orthoroute_b200.lattice import build_lattice

    g = golden("golden_dijkstra.npz")
    nx, ny, nz = (int(v) for v in g["ref_dims"])
    ref_ip, ref_ix, ref_c = g["ref_indptr"], g["ref_indices"], g["ref_base"]
    lat = build_lattice(nx, ny, nz, planar="inner", vias="full", pitch=0.4, via_cost=0.7, duplicate_vias=True)
    ref_src = np.repeat(np.arange(len(ref_ip) - 1), np.diff(ref_ip))
    a = sorted(zip(ref_src.tolist(), ref_ix.tolist(), np.round(ref_c, 5).tolist()))
    b = sorted(zip(lat.edge_src().tolist(), lat.indices.tolist(), np.round(lat.base_cost, 5).tolist()))
    assert a == b
    assert np.array_equal(np.sort(g["ref_edge_kind"]), np.sort(lat.edge_kind))


def test_uniform_weights_distribution():
    from orthoroute_b200.lattice import build_lattice, uniform_weights

    lat = build_lattice(60, 50, 6)
    w = uniform_weights(lat, seed=3, blocked_frac=0.05)
    fin = np.isfinite(w)
    assert abs((~fin).mean() - 0.05) < 0.01
    pl = fin & (lat.edge_kind == 0)
    assert w[pl].min() >= 1.0 and w[pl].max() < 2.0
    assert np.all(w[fin & (lat.edge_kind == 1)] == 3.0)
