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


def assembly_plan_host(conn, n_nodes):
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    nt, nemax, nel = C.c_int64(), C.c_int(), C.c_int64()
    _lib.call("wn_assembly_plan_host", n_nodes, len(conn), _lib.ptr(conn), C.byref(nt), C.byref(nemax), C.byref(nel),
              None, None, None, None, None)
    tiles = np.empty((nt.value, 4), dtype=np.int32)
    el_ptr = np.empty(nt.value + 1, dtype=np.int32)
    el = np.empty(nel.value, dtype=np.int32)
    contrib = np.empty(len(conn) * 100, dtype=np.uint16)
    rp, ci, _ = pattern_host(conn, n_nodes)
    perm = np.empty(len(ci), dtype=np.uint16)
    _lib.call("wn_assembly_plan_host", n_nodes, len(conn), _lib.ptr(conn), C.byref(nt), C.byref(nemax), C.byref(nel),
              _lib.ptr(tiles), _lib.ptr(el_ptr), _lib.ptr(el), _lib.ptr(contrib), _lib.ptr(perm))
    return tiles, el_ptr, el, contrib, perm, nemax.value, rp, ci


@pytest.mark.parametrize("which", ["c1", "ibeam-shuffled"])
def test_assembly_plan_rebuilds_the_oracle_matrix(which):
    """The tile-owner assembly's plan: tiles cover every block row once and match the streamed
    engine's tiling; each tile lists exactly the elements incident to its rows; perm is a
    permutation of the tile's blocks by descending contribution count; and summing, per block in
    the plan's order, the oracle's element blocks named by (slot, a, b) reproduces the oracle's
    assembled K (no Dirichlet BCs), with blocks (i, j) and (j, i) exact transposes."""
    from oracle import c3d10

    from wnfea_b200.model import solid_element_props

    if which == "c1":
        m, _ = generate_c3d10_kuhn_block()
    else:
        m, _ = generate_c3d10_ibeam_structured(n_slices=5, length=4.0 * 5 / 315, seed=2)
        perm_nodes = np.random.default_rng(3).permutation(len(m.mesh_nodes))
        inv = np.empty_like(perm_nodes)
        inv[perm_nodes] = np.arange(len(perm_nodes))
        m.mesh_nodes = m.mesh_nodes[perm_nodes].copy()
        m.solid_elements = inv[m.solid_elements].astype(np.int32)
    conn = np.ascontiguousarray(m.solid_elements, dtype=np.int32)
    n = len(m.mesh_nodes)
    tiles, el_ptr, el, contrib, perm, nemax, rp, ci = assembly_plan_host(conn, n)
    assert len(tiles) > 1 and tiles[0, 0] == 0 and tiles[-1, 1] == n
    assert np.array_equal(tiles[1:, 0], tiles[:-1, 1]) and np.array_equal(tiles[:, 2], rp[tiles[:, 0]])
    assert np.array_equal(tiles[:, 3], rp[tiles[:, 1]])
    nt_stream = C.c_int64()
    _lib.call("wn_stream_tiles_host", n, _lib.ptr(rp), None, 0, C.byref(nt_stream))
    st = np.empty((nt_stream.value, 4), dtype=np.int32)
    _lib.call("wn_stream_tiles_host", n, _lib.ptr(rp), _lib.ptr(st), nt_stream.value, C.byref(nt_stream))
    assert np.array_equal(st, tiles)
    node_tile = np.repeat(np.arange(len(tiles)), tiles[:, 1] - tiles[:, 0])
    for t in range(len(tiles)):
        mine = np.flatnonzero((node_tile[conn] == t).any(axis=1))
        assert np.array_equal(el[el_ptr[t]:el_ptr[t + 1]], mine)
    assert nemax == np.diff(el_ptr).max()
    Ke = c3d10.element_stiffness_batch(m.mesh_nodes[conn], solid_element_props(m))
    gptr = np.concatenate([[0], np.cumsum(np.bincount(pattern_host(conn, n)[2].ravel(), minlength=len(ci)))])
    vals = np.zeros((len(ci), 3, 3))
    for t in range(len(tiles)):
        b0, b1 = tiles[t, 2], tiles[t, 3]
        assert np.array_equal(np.sort(perm[b0:b1]), np.arange(b1 - b0))
        counts = np.diff(gptr[b0:b1 + 1])[perm[b0:b1]]
        assert np.all(np.diff(counts) <= 0)
        els = el[el_ptr[t]:el_ptr[t + 1]]
        for b in range(b0, b1):
            last = -1
            for q in range(gptr[b], gptr[b + 1]):
                code = int(contrib[q])
                e, a, bb = els[code >> 8], (code >> 4) & 15, code & 15
                assert e > last  # element order
                last = e
                vals[b] += Ke[e, 3 * a:3 * a + 3, 3 * bb:3 * bb + 3]
    K = solid.bsr3_to_csr(rp, ci, vals)
    assert abs(K - K.T).max() == 0.0
    Ko, _, _ = solid.assemble(m.mesh_nodes, conn, solid_element_props(m), apply_bcs=False)
    D = (K - Ko).tocsr()
    assert np.abs(D.data).max(initial=0.0) <= 1e-14 * np.abs(Ko.data).max()


def assembly_chunks_host(conn, n_nodes, n_tiles):
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    C_len, max_codes, n_chunks = C.c_int(), C.c_int(), C.c_int64()
    _lib.call("wn_assembly_chunks_host", n_nodes, len(conn), _lib.ptr(conn), C.byref(C_len), C.byref(max_codes),
              C.byref(n_chunks), None, None, None)
    chunk_ptr = np.empty(n_tiles + 1, dtype=np.int32)
    chunks = np.empty(max(n_chunks.value, 1), dtype=np.uint32)
    n_split = np.empty(n_tiles, dtype=np.int32)
    _lib.call("wn_assembly_chunks_host", n_nodes, len(conn), _lib.ptr(conn), C.byref(C_len), C.byref(max_codes),
              C.byref(n_chunks), _lib.ptr(chunk_ptr), _lib.ptr(chunks), _lib.ptr(n_split))
    return C_len.value, max_codes.value, chunk_ptr, chunks[:n_chunks.value], n_split


@pytest.mark.parametrize("which", ["c1", "ibeam-shuffled", "ibeam60"])
def test_assembly_work_items_cover_every_block(which):
    """The assembly kernel's work items, replayed on the host with the kernel's own index
    arithmetic (256 threads, three rounds): every block of a tile is summed exactly once --
    unsplit blocks by one thread, split blocks (more than chunk_len contributions) as chunks
    of at most chunk_len consecutive contributions that tile the block's list, cut by its count
    alone (so blocks (i, j) and (j, i) alike) and combined from the first chunk's thread --
    the chunk slots stay below 32 and the contribution codes inside max_codes."""
    if which == "c1":
        m, _ = generate_c3d10_kuhn_block()
    elif which == "ibeam60":
        m, _ = generate_c3d10_ibeam_structured(n_slices=60, length=4.0 * 60 / 315, seed=0)
    else:
        m, _ = generate_c3d10_ibeam_structured(n_slices=5, length=4.0 * 5 / 315, seed=2)
        perm_nodes = np.random.default_rng(3).permutation(len(m.mesh_nodes))
        inv = np.empty_like(perm_nodes)
        inv[perm_nodes] = np.arange(len(perm_nodes))
        m.mesh_nodes = m.mesh_nodes[perm_nodes].copy()
        m.solid_elements = inv[m.solid_elements].astype(np.int32)
    conn = np.ascontiguousarray(m.solid_elements, dtype=np.int32)
    n = len(m.mesh_nodes)
    tiles, el_ptr, el, contrib, perm, nemax, rp, ci = assembly_plan_host(conn, n)
    clen, max_codes, chunk_ptr, chunks, n_split = assembly_chunks_host(conn, n, len(tiles))
    gptr = np.concatenate([[0], np.cumsum(np.bincount(pattern_host(conn, n)[2].ravel(), minlength=len(ci)))])
    count = np.diff(gptr)
    assert 1 <= clen <= 63 or clen == 1024
    T, x = 256, np.arange(256)
    n_split_blocks = 0
    for t in range(len(tiles)):
        b0, b1 = int(tiles[t, 2]), int(tiles[t, 3])
        nb = b1 - b0
        c0, NH, H = int(chunk_ptr[t]), int(chunk_ptr[t + 1] - chunk_ptr[t]), int(n_split[t])
        L = nb - H
        assert 0 <= H and NH <= 32 and (H == 0) == (NH == 0) and NH >= 2 * H
        assert gptr[b1] - gptr[b0] <= max_codes
        loc = perm[b0:b1].astype(np.int64)
        cnt = count[b0 + loc]
        assert np.all(cnt[:H] > clen) and np.all(cnt[H:] <= clen)
        n0 = min(L, T - NH)
        ranks = [x[NH:][x[NH:] - NH < L] - NH]
        k1 = n0 + (T - 1 - x)
        ranks.append(k1[k1 < L])
        k2 = n0 + T + x[:NH]
        ranks.append(k2[k2 < L])
        assert np.array_equal(np.sort(np.concatenate(ranks)), np.arange(L))
        ch = chunks[c0:c0 + NH].astype(np.int64)
        cj, off, ln, first = ch & 511, (ch >> 9) & 1023, (ch >> 19) & 63, (ch >> 25) & 1
        y = 0
        for i in range(H):
            j = int(loc[i])
            c = int(count[b0 + j])
            nchunk = -(-c // clen)
            want = [c // nchunk + (1 if mm < c % nchunk else 0) for mm in range(nchunk)]
            assert first[y] == 1 and np.all(cj[y:y + nchunk] == j) and np.all(first[y + 1:y + nchunk] == 0)
            assert list(ln[y:y + nchunk]) == want
            assert list(off[y:y + nchunk]) == list(np.concatenate([[0], np.cumsum(want)[:-1]]))
            y += nchunk
            n_split_blocks += 1
        assert y == NH
    if which == "ibeam60":
        assert n_split_blocks > 0 and clen == 6


def test_element_api_rejects_bad_shapes():
    import wnfea_b200 as wn

    with pytest.raises(ValueError):
        wn.element_stiffness_c3d10(np.zeros((9, 3)), 2e11, 0.3)
    with pytest.raises(ValueError):
        wn.element_internal_forces_c3d10(np.zeros((10, 3)), np.zeros(29), 2e11, 0.3)
    with pytest.raises(ValueError):
        wn.element_stresses_c3d10(np.zeros((2, 10, 3)), np.zeros(30), 2e11, 0.3)


def test_precision_presets_select_solver_modes():
    import wnfea_b200 as wn

    assert wn.MIXED_FP32.solver_precision == "mixed_fp32"
    assert wn.FULL_FP64.solver_precision == "fp64"
    assert wn.TRI_PRECISION.solver_precision == "mixed_fp16"  # the FP16 V-cycle (solve precision 3)
