"""The allocation-free element-stiffness entry point (collected last on purpose).

wn_c3d10_element_stiffness_noalloc serves callers that cannot let the library call
cudaMalloc / cudaFree -- their device memory belongs to another allocator or a fixed pool,
or they cannot pay cudaFree's device-wide synchronisation.  Its only scratch is a fixed
device array shared by all calls.  This test calls it through the C ABI twice in a row, on
two different meshes (so stale scratch contents from the first call would show), and
compares each result with the allocating entry point wn_c3d10_element_stiffness at the
tolerance the other element tests use; it checks the reference's golden element stiffness
through the same call, the size limit, and that a connectivity entry outside the node range
is reported as an argument error without any coordinate read out of bounds.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from wnfea_b200 import _lib
from wnfea_b200.mesh import generate_c3d10_ibeam_structured, generate_c3d10_kuhn_block
from wnfea_b200.model import solid_element_props

pytestmark = pytest.mark.gpu


def _allocating(nodes, conn, props):
    coords = np.ascontiguousarray(nodes[conn])
    Ke = np.empty((len(conn), 30, 30))
    _lib.call("wn_c3d10_element_stiffness", len(conn), _lib.ptr(coords), _lib.ptr(np.ascontiguousarray(props)),
              _lib.ptr(Ke))
    return Ke


def test_noalloc_matches_allocating_entry_point_twice():
    import torch

    m1, _ = generate_c3d10_kuhn_block()  # 480 elements
    m2, _ = generate_c3d10_ibeam_structured(n_slices=3, length=4.0 * 3 / 315, seed=9)  # 1908 elements
    p2 = solid_element_props(m2)
    p2[:, 0] *= np.exp(np.random.default_rng(4).uniform(-1.0, 1.0, len(p2)))
    cases = [(m1.mesh_nodes, m1.solid_elements, solid_element_props(m1)), (m2.mesh_nodes, m2.solid_elements, p2)]
    for nodes, conn, props in cases:
        ref = _allocating(nodes, conn, props)
        d_nodes = torch.from_numpy(np.ascontiguousarray(nodes)).cuda()
        d_conn = torch.from_numpy(np.ascontiguousarray(conn, dtype=np.int32)).cuda()
        d_props = torch.from_numpy(np.ascontiguousarray(props)).cuda()
        d_Ke = torch.full((len(conn), 30, 30), float("nan"), dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        _lib.call("wn_c3d10_element_stiffness_noalloc", len(conn), len(nodes), d_nodes.data_ptr(),
                  d_conn.data_ptr(), d_props.data_ptr(), d_Ke.data_ptr(), stream)
        torch.cuda.synchronize()
        got = d_Ke.cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-14 * np.abs(ref).max())


def test_noalloc_matches_reference_golden_ke(golden):
    import torch

    g = golden("c3d10_element.npz")
    nodes = np.ascontiguousarray(np.vstack([g["tet"], g["curved"]]))
    conn = np.arange(20, dtype=np.int32).reshape(2, 10)
    props = np.array([[2.1e11, 0.3], [1.8e11, 0.33]])
    d_nodes, d_conn, d_props = (torch.from_numpy(a).cuda() for a in (nodes, conn, props))
    d_Ke = torch.empty((2, 30, 30), dtype=torch.float64, device="cuda")
    _lib.call("wn_c3d10_element_stiffness_noalloc", 2, len(nodes), d_nodes.data_ptr(), d_conn.data_ptr(),
              d_props.data_ptr(), d_Ke.data_ptr(), 0)
    Ke = d_Ke.cpu().numpy()
    for k, ref in enumerate((g["Ke_tet"], g["Ke_curved"])):
        np.testing.assert_allclose(Ke[k], ref, rtol=0, atol=1e-14 * np.abs(ref).max())


def test_noalloc_rejects_out_of_range_connectivity():
    import torch

    m, _ = generate_c3d10_kuhn_block(nx=2, ny=1, nz=1)
    nodes = np.ascontiguousarray(m.mesh_nodes)
    conn = np.ascontiguousarray(m.solid_elements, dtype=np.int32).copy()
    conn[1, 4] = len(nodes)  # one past the last node
    props = np.ascontiguousarray(solid_element_props(m))
    d_nodes, d_conn, d_props = (torch.from_numpy(a).cuda() for a in (nodes, conn, props))
    d_Ke = torch.empty((len(conn), 30, 30), dtype=torch.float64, device="cuda")
    lib = _lib.lib()
    rc = lib.wn_c3d10_element_stiffness_noalloc(len(conn), len(nodes), d_nodes.data_ptr(), d_conn.data_ptr(),
                                                d_props.data_ptr(), d_Ke.data_ptr(), 0)
    assert rc == -1  # WN_EINVAL
    assert "n_nodes" in _lib.last_error()
    torch.cuda.synchronize()  # the context is intact: the kernel read nothing out of bounds
    assert np.all(d_Ke[1].cpu().numpy() == 0.0)


def test_noalloc_rejects_batches_beyond_its_capacity():
    import torch

    m, _ = generate_c3d10_kuhn_block(nx=2, ny=1, nz=1)
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    too_many = 2048 + 1
    lib = _lib.lib()
    rc = lib.wn_c3d10_element_stiffness_noalloc(too_many, 4, d.data_ptr(), d.data_ptr(), d.data_ptr(), d.data_ptr(),
                                                0)
    assert rc == -8  # WN_ETOOBIG, nothing launched
    assert "2048" in _lib.last_error()
