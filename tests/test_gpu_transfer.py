"""State transfer through the C ABI (q2d_gpu_upload_prim / q2d_gpu_download_prim): the interior
of the caller's ghosted array (the reference layout P(4, -1:ni+2, -1:nj+2)) is copied exactly,
in both directions, and the caller's ghost layers are never written."""
import ctypes as C

import numpy as np
import pytest

from q2d_b200 import _abi, cases, make_options
from q2d_b200.solver import Q2DSolver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_upload_download_round_trip(precision):
    cs = cases.ramp(70, 23, seed=2)
    s = Q2DSolver(make_options(cs, precision=precision), [cs])
    try:
        s.step(2)                                   # resident state, graphs built
        b = cs.blocks[0]
        bid = s.block_ids[0][0]
        rng = np.random.default_rng(1)
        interior = 1.0 + rng.random((b.nj, b.ni, 4))
        P = np.full((b.nj + 4, b.ni + 4, 4), -7.0)
        P[2:-2, 2:-2] = interior
        assert s.lib.q2d_gpu_upload_prim(s.ctx, bid, _abi.dptr(P)) == 0
        Q = np.full((b.nj + 4, b.ni + 4, 4), 5.0)
        assert s.lib.q2d_gpu_download_prim(s.ctx, bid, _abi.dptr(Q)) == 0
        assert np.array_equal(Q[2:-2, 2:-2], interior)
        ghosts = np.ones(Q.shape[:2], bool)
        ghosts[2:-2, 2:-2] = False
        assert np.all(Q[ghosts] == 5.0)
        # the uploaded state is what the next step advances (dt recomputed from it)
        info = s.step(1, check=False)[0]
        assert info["iter"] == 3
    finally:
        s.close()
