"""Tile plan of the streamed fine-matrix kernels, on the CPU (no kernel launch).

The plan comes from the library's own host builder (``wn_stream_tiles_host``); the segment
sizes below restate the tile-major pack layout the streamed kernels copy with one bulk copy
per tile, and check that every copy is 128-byte aligned and sized, fits a stage buffer and the
mbarrier transaction range, and that the local row starts fit their uint16 slots.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from wnfea_b200 import _lib
from wnfea_b200.mesh import generate_c3d10_ibeam_structured, generate_c3d10_kuhn_block

CAP = 512       # WN_STREAM_TILE_BLOCKS
ROW_CAP = 120   # WN_STREAM_TILE_ROWS


def pattern(coords, conn):
    n = len(coords)
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    nnzb = C.c_int64()
    rp = np.empty(n + 1, dtype=np.int32)
    _lib.call("wn_bsr3_pattern_host", n, len(conn), _lib.ptr(conn), C.byref(nnzb), _lib.ptr(rp), None, None)
    return rp


def tiles_of(rp):
    n = len(rp) - 1
    rp = np.ascontiguousarray(rp, dtype=np.int32)
    cnt = C.c_int64()
    _lib.call("wn_stream_tiles_host", n, _lib.ptr(rp), None, 0, C.byref(cnt))
    t = np.zeros((max(cnt.value, 1), 4), dtype=np.int32)
    _lib.call("wn_stream_tiles_host", n, _lib.ptr(rp), _lib.ptr(t), cnt.value, C.byref(cnt))
    return t[: cnt.value]


def check_plan(rp, tiles):
    n = len(rp) - 1
    assert len(tiles) > 0
    assert tiles[0, 0] == 0 and tiles[-1, 1] == n
    assert np.all(tiles[1:, 0] == tiles[:-1, 1])  # contiguous, whole rows, in order
    assert np.all(tiles[:, 1] > tiles[:, 0])
    assert np.all(tiles[:, 1] - tiles[:, 0] <= ROW_CAP)
    assert np.all(tiles[:, 2] == rp[tiles[:, 0]]) and np.all(tiles[:, 3] == rp[tiles[:, 1]])
    assert np.all(tiles[:, 3] - tiles[:, 2] <= CAP)


def pack_bytes(cntp, nr, elem_bytes):
    """Size of a packed tile segment: 9 value components of cntp blocks, cntp column indices,
    nr + 1 uint16 local row starts (16-byte multiple), the whole rounded up to 128 bytes."""
    row_off = 9 * cntp * elem_bytes + 4 * cntp
    return (row_off + ((2 * (nr + 1) + 15) & ~15) + 127) & ~127


def check_offsets(rp, tiles, elem_bytes):
    """Packed segments of every tile: one bulk copy each, 128-byte aligned and sized, laid end
    to end, no larger than a stage buffer, with row starts that fit uint16 and every local
    block index a consumer reads inside the tile's cntp blocks."""
    stage = pack_bytes(CAP, ROW_CAP, elem_bytes)
    seg = 0
    for r0, r1, b0, b1 in tiles.astype(np.int64):
        cnt = b1 - b0
        cntp = (cnt + 3) & ~3
        nb = pack_bytes(cntp, r1 - r0, elem_bytes)
        assert nb % 128 == 0 and 0 < nb <= stage
        assert 9 * cntp * elem_bytes % 16 == 0 and (9 * cntp * elem_bytes + 4 * cntp) % 16 == 0
        local = rp[r0:r1 + 1].astype(np.int64) - b0
        assert local[0] == 0 and local[-1] == cnt and np.all(np.diff(local) >= 0) and cnt < 65536
        seg += nb
    assert seg // 128 < 2 ** 31  # 32-bit segment indices
    assert stage < (1 << 20)      # mbarrier transaction count range


@pytest.mark.parametrize("slices", [4, 21])
def test_ibeam_plan(slices):
    m, _ = generate_c3d10_ibeam_structured(n_slices=slices, seed=0)
    rp = pattern(m.mesh_nodes, m.solid_elements)
    tiles = tiles_of(rp)
    check_plan(rp, tiles)
    check_offsets(rp, tiles, 4)
    check_offsets(rp, tiles, 8)


def test_block_plan():
    m, _ = generate_c3d10_kuhn_block(nx=12, ny=5, nz=7)
    rp = pattern(m.mesh_nodes, m.solid_elements)
    tiles = tiles_of(rp)
    check_plan(rp, tiles)
    check_offsets(rp, tiles, 4)
    check_offsets(rp, tiles, 8)


def test_ragged_rows():
    # rows of 1 .. 500 blocks in a seeded order, and runs of single-block rows longer than a tile
    rng = np.random.default_rng(3)
    lens = np.concatenate([rng.integers(1, 501, size=300), np.ones(400, dtype=np.int64), [512, 3, 512]])
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    tiles = tiles_of(rp)
    check_plan(rp, tiles)
    check_offsets(rp, tiles, 4)
    check_offsets(rp, tiles, 8)


def test_row_over_capacity_gives_no_plan():
    rp = np.array([0, 10, 10 + CAP + 1, 10 + CAP + 5], dtype=np.int32)
    assert len(tiles_of(rp)) == 0


def test_tiles_host_rejects_small_capacity():
    rp = np.arange(0, 5 * 600 + 1, 5, dtype=np.int32)  # 600 rows of 5 blocks -> several tiles
    cnt = C.c_int64()
    _lib.call("wn_stream_tiles_host", 600, _lib.ptr(rp), None, 0, C.byref(cnt))
    assert cnt.value >= 5
    buf = np.zeros((1, 4), dtype=np.int32)
    with pytest.raises(_lib.WnError):
        _lib.call("wn_stream_tiles_host", 600, _lib.ptr(rp), _lib.ptr(buf), 1, C.byref(cnt))
