"""GPU parity of the streamed fine-matrix kernels (bulk async copies into shared memory).

``wn_spmv_solid_device`` runs the streamed SpMV for every C3D10 system with a tile plan; the
fine level of the AMG V-cycle and the PCG product of the solver run the same engine.  The
product is checked against the float64 oracle (scipy CSR of the same values) on meshes whose
block counts put the value components at every 16-byte misalignment, with a seeded random
node numbering (scattered gathers) and with long and short rows; the status word of the
bounded pipeline waits must stay clear, and repeated products must be bit-identical.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from wnfea_b200 import _lib
from wnfea_b200.mesh import generate_c3d10_ibeam_structured, generate_c3d10_kuhn_block
from wnfea_b200.model import solid_element_props
from wnfea_b200.system import SolidSystem

pytestmark = pytest.mark.gpu


def _shuffled(m, seed):
    n = len(m.mesh_nodes)
    perm = np.random.default_rng(seed).permutation(n)
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)
    m.mesh_nodes = m.mesh_nodes[perm].copy()
    m.solid_elements = inv[m.solid_elements].astype(np.int32)
    return m


def _trimmed_block(k):
    """The 9 x 4 x 5 block without its last k elements (unused nodes dropped): k = 2 and 4 give
    block counts of 0 and 2 mod 4, which a whole structured mesh (odd node count) never has."""
    m = generate_c3d10_kuhn_block(nx=9, ny=4, nz=5)[0]
    conn = m.solid_elements[: len(m.solid_elements) - k]
    used = np.unique(conn)
    remap = np.full(len(m.mesh_nodes), -1, dtype=np.int64)
    remap[used] = np.arange(len(used))
    m.mesh_nodes = m.mesh_nodes[used].copy()
    m.solid_elements = remap[conn].astype(np.int32)
    return m


def _meshes():
    out = [("block-2", _trimmed_block(2)), ("block-4", _trimmed_block(4))]
    for slices in (3, 7, 20):
        out.append(("ibeam%d" % slices, generate_c3d10_ibeam_structured(n_slices=slices, length=4.0 * slices / 315,
                                                                         seed=slices)[0]))
    out.append(("block", generate_c3d10_kuhn_block(nx=9, ny=4, nz=5)[0]))
    out.append(("ibeam12-shuffled", _shuffled(generate_c3d10_ibeam_structured(n_slices=12, length=0.2, seed=1)[0], 7)))
    return out


def _status(s):
    st = C.c_int(-100)
    _lib.call("wn_solid_stream_status", s.handle, 1, C.byref(st))
    return st.value


@pytest.mark.parametrize("name,m", _meshes(), ids=lambda v: v if isinstance(v, str) else "")
def test_streamed_spmv_matches_oracle(name, m):
    import torch

    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    s.assemble(solid_element_props(m), apply_bcs=False)
    rp, ci = s.pattern()
    Kc = sp.bsr_matrix((s.values(), ci, rp), shape=(3 * s.n_nodes,) * 2).tocsr()
    x = np.random.default_rng(11).standard_normal(3 * s.n_nodes)
    ref = Kc @ x
    scale = np.abs(Kc) @ np.abs(x)
    dx = torch.from_numpy(x).cuda()
    dy = torch.full_like(dx, np.nan)
    _lib.call("wn_spmv_solid_device", s.handle, 0, dx.data_ptr(), dy.data_ptr(), 0)
    y64 = dy.cpu().numpy()
    # rows of <= 81 blocks (243 terms): |error| <= 256 eps sum |K||x| in either precision
    assert np.all(np.abs(y64 - ref) <= 256 * np.finfo(np.float64).eps * scale)
    dy2 = torch.full_like(dx, np.nan)
    _lib.call("wn_spmv_solid_device", s.handle, 0, dx.data_ptr(), dy2.data_ptr(), 0)
    assert torch.equal(dy, dy2)  # deterministic
    dx32 = dx.float()
    dy32 = torch.full_like(dx32, np.nan)
    _lib.call("wn_spmv_solid_device", s.handle, 1, dx32.data_ptr(), dy32.data_ptr(), 0)
    ref32 = Kc.astype(np.float32).astype(np.float64) @ dx32.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(dy32.cpu().numpy().astype(np.float64) - ref32) <= 256 * np.finfo(np.float32).eps * scale)
    assert _status(s) == 0


def test_meshes_cover_every_component_alignment():
    # the value component k of block b0 starts at k * nnzb + b0: nnzb mod 4 decides the shifts
    mods = set()
    for _, m in _meshes():
        s = SolidSystem(m.mesh_nodes, m.solid_elements)
        mods.add(s.nnzb % 4)
    assert mods == {0, 1, 2, 3}, mods


def test_streamed_solve_modes_agree():
    """FP64 and mixed solves (both through the streamed fine level) meet the tolerance and agree."""
    from wnfea_b200.model import solid_fixed_dofs, solid_load_vector

    m, _ = generate_c3d10_ibeam_structured(n_slices=16, length=0.2, seed=2)
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    s.set_fixed(solid_fixed_dofs(m))
    s.assemble(solid_element_props(m), apply_bcs=True)
    F = solid_load_vector(m)
    s.amg_setup()
    u64, st64 = s.solve(F, rtol=1e-10, precision=0)
    u32, st32 = s.solve(F, rtol=1e-10, precision=1)
    assert st64["status"] == 0 and st32["status"] == 0
    assert st64["rel_res"] <= 1e-10 and st32["rel_res"] <= 1e-10
    np.testing.assert_allclose(u32, u64, rtol=0, atol=1e-8 * np.abs(u64).max())
    u64b, _ = s.solve(F, rtol=1e-10, precision=0)
    assert np.array_equal(u64, u64b)  # deterministic dots and products


def test_streamed_spmv_unaligned_vectors():
    """x and y one element past an aligned address: the paired gathers of a 3-DOF block fall
    back to scalar loads and the product is unchanged."""
    import torch

    m = _trimmed_block(2)
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    s.assemble(solid_element_props(m), apply_bcs=False)
    n = 3 * s.n_nodes
    x = np.random.default_rng(3).standard_normal(n)
    for dt, prec in ((torch.float64, 0), (torch.float32, 1)):
        base = torch.zeros(n + 1, dtype=dt, device="cuda")
        base[1:] = torch.from_numpy(x).to(dt)
        xa = base[1:].clone()
        ya, yu = torch.empty_like(xa), torch.zeros(n + 1, dtype=dt, device="cuda")
        _lib.call("wn_spmv_solid_device", s.handle, prec, xa.data_ptr(), ya.data_ptr(), 0)
        _lib.call("wn_spmv_solid_device", s.handle, prec, base[1:].data_ptr(), yu[1:].data_ptr(), 0)
        torch.cuda.synchronize()
        assert torch.equal(ya, yu[1:])
    assert _status(s) == 0


@pytest.mark.parametrize("precision", [0, 1])
def test_streamed_coarse_levels_match_register_kernels(precision):
    """Every AMG level matrix and transfer operator streamed from its pack (stream_min_mb = 0)
    against none streamed (stream_min_mb = -1): same iterations, same solution to rounding (the
    6x6 level products sum in the register kernels' order; the 3x6 prolongation uses 4 lanes
    per row instead of 8, which reorders its sums)."""
    from wnfea_b200.amg import AMGParams
    from wnfea_b200.model import solid_fixed_dofs, solid_load_vector

    m, _ = generate_c3d10_ibeam_structured(n_slices=24, length=0.3, seed=5)
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    s.set_fixed(solid_fixed_dofs(m))
    s.assemble(solid_element_props(m), apply_bcs=True)
    F = solid_load_vector(m)
    out = []
    for mb in (-1.0, 0.0):
        s.amg_setup(AMGParams(stream_min_mb=mb))
        u, st = s.solve(F, rtol=1e-9, precision=precision)
        assert st["status"] == 0 and st["rel_res"] <= 1e-9
        out.append((u, st["iterations"]))
    assert out[0][1] == out[1][1]
    np.testing.assert_allclose(out[1][0], out[0][0], rtol=0, atol=1e-9 * np.abs(out[0][0]).max())


@pytest.mark.parametrize("precision", [0, 1])
def test_register_fine_level_matches_streamed(precision):
    """Streaming switched off (the register row kernels, the path of meshes whose rows exceed
    the tile capacity) against the streamed fine level: same iterations, same solution to
    rounding; the SpMV of the register path against the oracle; streaming back on restores
    the streamed results bit for bit."""
    import torch
    from wnfea_b200.model import solid_fixed_dofs, solid_load_vector

    m, _ = generate_c3d10_ibeam_structured(n_slices=24, length=0.3, seed=6)
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    s.set_fixed(solid_fixed_dofs(m))
    s.assemble(solid_element_props(m), apply_bcs=True)
    F = solid_load_vector(m)
    s.amg_setup()
    u_on, st_on = s.solve(F, rtol=1e-9, precision=precision)
    s.set_streaming(False)
    u_off, st_off = s.solve(F, rtol=1e-9, precision=precision)
    assert st_off["status"] == 0 and st_off["rel_res"] <= 1e-9
    assert abs(st_off["iterations"] - st_on["iterations"]) <= 1
    np.testing.assert_allclose(u_off, u_on, rtol=0, atol=1e-9 * np.abs(u_on).max())
    rp, ci = s.pattern()
    Kc = sp.bsr_matrix((s.values(), ci, rp), shape=(3 * s.n_nodes,) * 2).tocsr()
    x = np.random.default_rng(1).standard_normal(3 * s.n_nodes)
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty_like(dx)
    _lib.call("wn_spmv_solid_device", s.handle, 0, dx.data_ptr(), dy.data_ptr(), 0)
    assert np.all(np.abs(dy.cpu().numpy() - Kc @ x) <= 256 * np.finfo(np.float64).eps * (np.abs(Kc) @ np.abs(x)))
    s.set_streaming(True)
    u_again, st_again = s.solve(F, rtol=1e-9, precision=precision)
    assert st_again["iterations"] == st_on["iterations"] and np.array_equal(u_again, u_on)


def test_stream_wait_runs_out_and_the_handle_recovers():
    """Failure detection of the streamed pipeline, with no fault: the test hook makes the
    producer withhold one tile's copy (nothing arms that stage), so the consumers' bounded wait
    for it must run out after the short limit.  The product and the solve must report
    WN_ETIMEOUT; every CTA waits for the copies it did issue before it exits, so the context stays
    usable, and once the hook is off the next product and solve on the same handle are
    bit-identical to clean ones."""
    import torch

    m = generate_c3d10_ibeam_structured(n_slices=20, length=4.0 * 20 / 315, seed=5)[0]
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    s.assemble(solid_element_props(m), apply_bcs=False)
    rp, _ = s.pattern()
    nt = C.c_int64(0)
    _lib.call("wn_stream_tiles_host", s.n_nodes, _lib.ptr(rp), None, 0, C.byref(nt))
    assert nt.value > 8
    x = torch.from_numpy(np.random.default_rng(3).standard_normal(3 * s.n_nodes)).cuda()
    y_ref, y = torch.empty_like(x), torch.empty_like(x)
    _lib.call("wn_spmv_solid_device", s.handle, 0, x.data_ptr(), y_ref.data_ptr(), 0)
    assert _status(s) == 0
    for tile in (0, nt.value // 2, nt.value - 1):
        _lib.call("wn_solid_stream_test_hook", s.handle, 200_000, tile)  # 0.2 ms stage waits
        for prec, xv, yv in ((0, x, y), (1, x.float(), torch.empty_like(x, dtype=torch.float32))):
            _lib.call("wn_spmv_solid_device", s.handle, prec, xv.data_ptr(), yv.data_ptr(), 0)
            assert _status(s) == -9, (tile, prec)  # WN_ETIMEOUT, status word reset by _status
    _lib.call("wn_solid_stream_test_hook", s.handle, 0, -1)
    _lib.call("wn_spmv_solid_device", s.handle, 0, x.data_ptr(), y.data_ptr(), 0)
    assert _status(s) == 0
    assert torch.equal(y, y_ref)

    # the solver: its fine-level kernels (V-cycle and PCG product) stream the same matrix
    from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof

    K, F, _ = assemble_c3d10_sparse_3dof(m)  # root clamped, tip shear
    sfix = K.system
    for precision in (0, 1):
        u_clean, st_clean = sfix.solve(F, rtol=1e-8, precision=precision)
        assert st_clean["status"] == 0
        _lib.call("wn_solid_stream_test_hook", sfix.handle, 200_000, nt.value // 3)
        _, st_bad = sfix.solve(F, rtol=1e-8, precision=precision)
        assert st_bad["status"] == -9, st_bad
        _lib.call("wn_solid_stream_test_hook", sfix.handle, 0, -1)
        u_again, st_again = sfix.solve(F, rtol=1e-8, precision=precision)
        assert st_again["status"] == 0 and np.array_equal(u_again, u_clean)
