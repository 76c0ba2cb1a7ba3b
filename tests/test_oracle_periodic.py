"""The oracle's translational periodic seam (BC 201) on the CPU: ghost metrics of the donor
cells (BC_Connect_Metrics_Periodic, Lib_Metrics.f90:556-700), free-stream preservation, exact
conservation of mass, momentum and energy on a doubly periodic domain, and the rejection of a
seam that is not one rigid translation."""
import ctypes as C
import copy

import numpy as np
import pytest

from q2d_b200 import cases, make_options
from tests.conftest import cons


def _geometry(o, ni, nj):
    dl = np.zeros((nj + 4, ni + 4, 2))
    st = o.lib.q2d_oracle_get_geometry(o.ctx, o.block_ids[0][0], dl.ctypes.data_as(C.POINTER(C.c_double)),
                                       None, None, None)
    assert st == 0
    return dl


def test_periodic_ghost_lengths_are_the_donor_cells():
    from oracle import oracle
    cs = cases.periodic_box(24, 20)
    o = oracle.solver(make_options(cs), [cs])
    try:
        dl = _geometry(o, 24, 20)
    finally:
        o.close()
    # frame index = cell index + 1 (cells -1 .. ni+2); rows 1..nj are frame rows 2..nj+1
    rows, cols = slice(2, 22), slice(2, 26)
    np.testing.assert_allclose(dl[rows, 1], dl[rows, 25], rtol=1e-12)   # i = 0   <- i = ni
    np.testing.assert_allclose(dl[rows, 0], dl[rows, 24], rtol=1e-12)   # i = -1  <- i = ni - 1
    np.testing.assert_allclose(dl[rows, 26], dl[rows, 2], rtol=1e-12)   # i = ni+1 <- i = 1
    np.testing.assert_allclose(dl[1, cols], dl[21, cols], rtol=1e-12)   # j = 0   <- j = nj
    np.testing.assert_allclose(dl[22, cols], dl[2, cols], rtol=1e-12)   # j = nj+1 <- j = 1


def test_periodic_free_stream_and_conservation():
    from oracle import oracle
    cs = cases.periodic_box(32, 24)
    sur = cases.cell_areas(cs.blocks[0])
    # a uniform flow stays uniform on the curved periodic grid
    uni = copy.deepcopy(cs)
    uni.blocks[0].prim[...] = np.array([1.0, 0.4, -0.25, 1.0 / 1.4])
    o = oracle.solver(make_options(uni), [uni])
    try:
        o.step(10)
        p = o.prim(0, 0)
        assert np.abs(p - uni.blocks[0].prim).max() <= 1e-13
    finally:
        o.close()
    o = oracle.solver(make_options(cs), [cs])
    try:
        def totals():
            U = cons(o.prim(0, 0))
            return np.array([(U[..., k] * sur).sum() for k in range(4)]), \
                np.array([(np.abs(U[..., k]) * sur).sum() for k in range(4)])
        t0, m0 = totals()
        info = o.step(60)[0]
        t1, _ = totals()
        assert info["err"] == 0 and info["time"] > 0
        assert np.all(np.abs(t1 - t0) <= 1e-13 * m0), (t0, t1)
        assert np.abs(o.prim(0, 0) - cs.blocks[0].prim).max() > 1e-4   # the flow did move
    finally:
        o.close()


def test_periodic_seam_must_be_a_rigid_translation():
    from oracle import oracle
    from q2d_b200.solver import Q2DError
    cs = cases.periodic_box(16, 12)
    bad = copy.deepcopy(cs)
    bad.blocks[0].nodes[-1, :, 1] += 0.01 * np.linspace(0.0, 1.0, 17)   # top edge no longer a copy
    with pytest.raises(Q2DError) as e:
        o = oracle.solver(make_options(bad), [bad])   # commit builds the ghost metrics
        try:
            o.step(1)
        finally:
            o.close()
    assert e.value.status == 1
