"""The C-ABI library on the CPU: it loads, exports every declared symbol, and its host-only
logic (pattern + element map) matches the oracle bit for bit.  No kernel is launched."""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import solid
from wnfea_b200 import _lib
from wnfea_b200.mesh import generate_c3d10_ibeam_structured, generate_c3d10_kuhn_block

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(wn_\w+)\s*\(", text, flags=re.M)
    return names


def test_header_declares_functions():
    assert len(header_functions()) >= 20


def test_library_exports_every_header_symbol():
    lib = _lib.lib()
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert sorted(set(header_functions())) == sorted(_lib.SIGNATURES)


def pattern_host(conn, n_nodes):
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    nnzb = C.c_int64()
    rp = np.empty(n_nodes + 1, dtype=np.int32)
    _lib.call("wn_bsr3_pattern_host", n_nodes, len(conn), _lib.ptr(conn), C.byref(nnzb), _lib.ptr(rp), None, None)
    ci = np.empty(nnzb.value, dtype=np.int32)
    emap = np.empty((len(conn), 100), dtype=np.int32)
    _lib.call("wn_bsr3_pattern_host", n_nodes, len(conn), _lib.ptr(conn), C.byref(nnzb), _lib.ptr(rp), _lib.ptr(ci),
              _lib.ptr(emap))
    return rp, ci, emap


@pytest.mark.parametrize("which", ["c1", "ibeam"])
def test_pattern_and_map_bit_exact_vs_oracle(which):
    if which == "c1":
        m, _ = generate_c3d10_kuhn_block()
    else:
        m, _ = generate_c3d10_ibeam_structured(n_slices=6, length=4.0 * 6 / 315, seed=5)
    rp, ci, emap = pattern_host(m.solid_elements, len(m.mesh_nodes))
    orp, oci, oemap = solid.bsr3_pattern_and_map(m.solid_elements, len(m.mesh_nodes))
    assert np.array_equal(rp, orp)
    assert np.array_equal(ci, oci)
    assert np.array_equal(emap, oemap)


def test_pattern_rejects_bad_node_index():
    m, _ = generate_c3d10_kuhn_block(nx=2, ny=1, nz=1)
    conn = m.solid_elements.copy()
    conn[0, 3] = len(m.mesh_nodes)  # out of range
    with pytest.raises(_lib.WnError) as e:
        pattern_host(conn, len(m.mesh_nodes))
    assert e.value.code == -3
