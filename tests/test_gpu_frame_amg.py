"""Linear beam-frame systems on the GPU (6x6 blocks): AMG over the 6 rigid-body modes of beam
nodes + PCG, against a direct solve of the same (exported) stiffness."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.sparse.linalg import spsolve

from wnfea_b200 import _lib
from wnfea_b200.amg import AMGParams
from wnfea_b200.beam import frame_linear_system, solve_frame_linear
from wnfea_b200.frames import generate_frame_grid, generate_space_frame

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,rtol,tol", [("fp64", 1e-10, 1e-8), ("mixed_fp32", 1e-8, 1e-6)])
def test_space_frame_matches_direct_solve(precision, rtol, tol):
    m = generate_space_frame(6, 5, 7, seed=3)
    frame, system, F = frame_linear_system(m)
    K = frame.tangent_bsr().tocsr()
    assert abs(K - K.T).max() <= 1e-9 * abs(K).max()  # the stiffness at U = 0 is symmetric
    # 1,260 DOFs: a coarse size below the default keeps a multi-level hierarchy in the test
    system.amg_setup(AMGParams(coarse_size=300))
    U, st = system.solve(F, rtol=rtol, precision=precision)
    assert st["status"] == 0 and st["rel_res"] <= rtol and st["n_levels"] >= 2
    Ur = spsolve(K.tocsc(), F)
    assert np.linalg.norm(U - Ur) <= tol * np.linalg.norm(Ur)
    assert st["iterations"] < 200


def test_planar_frame_and_c3d10_guards():
    m = generate_frame_grid()
    U, st = solve_frame_linear(m, rtol=1e-10, precision="fp64")
    frame, system, F = frame_linear_system(m)
    Ur = spsolve(frame.tangent_bsr().tocsc(), F)
    assert st["status"] == 0 and np.linalg.norm(U - Ur) <= 1e-8 * np.linalg.norm(Ur)
    # a 6x6 system is not a C3D10 system
    with pytest.raises(_lib.WnError):
        _lib.call("wn_fint_c3d10_device", system._h, 1, 1, 0)
