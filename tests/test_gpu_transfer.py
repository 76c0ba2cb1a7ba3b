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


@pytest.mark.parametrize("precision", [0, 1])
def test_error_isolation_between_cases(precision):
    """A NaN state injected from the host into one case (host-side fault injection) stops that
    case with Q2D_ERR_NAN; every other case of the batch advances exactly as in a run where the
    injected case was given back its own state."""
    batch = cases.area_nozzle_batch(n=4, seed=21, nx_range=(40, 80), ny_range=(8, 12))

    def run(inject):
        s = Q2DSolver(make_options(batch[0], precision=precision), batch)
        try:
            s.step(2)
            b = batch[1].blocks[0]
            bid = s.block_ids[1][0]
            P = np.zeros((b.nj + 4, b.ni + 4, 4))
            assert s.lib.q2d_gpu_download_prim(s.ctx, bid, _abi.dptr(P)) == 0
            if inject:
                P[2 + b.nj // 2, 2 + b.ni // 2, 3] = np.nan
            assert s.lib.q2d_gpu_upload_prim(s.ctx, bid, _abi.dptr(P)) == 0
            infos = s.step(8, check=False)
            return infos, [s.prim(c, 0) for c in range(len(batch))]
        finally:
            s.close()

    ref_i, ref_s = run(False)
    bad_i, bad_s = run(True)
    assert bad_i[1]["err"] == _abi.ERR_NAN and bad_i[1]["todo"] != _abi.TODO_CONTINUE or bad_i[1]["err"] != 0
    assert bad_i[1]["iter"] < 10
    for c in (0, 2, 3):
        assert bad_i[c]["err"] == 0 and bad_i[c]["iter"] == 10 == ref_i[c]["iter"]
        assert np.array_equal(bad_s[c], ref_s[c])


def _ghosted(b, rng, fill):
    interior = 1.0 + rng.random((b.nj, b.ni, 4))
    P = np.full((b.nj + 4, b.ni + 4, 4), fill)
    P[2:-2, 2:-2] = interior
    return P, interior


@pytest.mark.parametrize("precision", [0, 1])
def test_many_block_round_trip(precision):
    """q2d_gpu_upload_prim_many / q2d_gpu_download_prim_many over every block of a batch with
    multi-block cases: each block gets exactly its own array, ghosts untouched, and the result
    equals the single-block transfers."""
    batch = [cases.nozzle_axi(96, 24, nblocks=3), cases.ramp(70, 23, seed=2), cases.closed_box(17, 9)]
    s = Q2DSolver(make_options(batch[0], precision=precision), batch)
    try:
        s.step(1)
        rng = np.random.default_rng(4)
        ids, ups, interiors = [], [], []
        for c, cs in enumerate(batch):
            for k, b in enumerate(cs.blocks):
                P, inner = _ghosted(b, rng, -3.0)
                ids.append(s.block_ids[c][k])
                ups.append(P)
                interiors.append(inner)
        n = len(ids)
        idv = (C.c_int * n)(*ids)
        pin = (C.POINTER(C.c_double) * n)(*[_abi.dptr(a) for a in ups])
        assert s.lib.q2d_gpu_upload_prim_many(s.ctx, n, idv, pin) == 0
        downs = [np.full_like(a, 9.0) for a in ups]
        pout = (C.POINTER(C.c_double) * n)(*[_abi.dptr(a) for a in downs])
        assert s.lib.q2d_gpu_download_prim_many(s.ctx, n, idv, pout) == 0
        for Q, inner in zip(downs, interiors):
            assert np.array_equal(Q[2:-2, 2:-2], inner)
            ghosts = np.ones(Q.shape[:2], bool)
            ghosts[2:-2, 2:-2] = False
            assert np.all(Q[ghosts] == 9.0)
        flat = [p for row in s.prims() for p in row]
        for got, inner in zip(flat, interiors):
            assert np.array_equal(got, inner)
        bad = (C.c_int * 1)(10 ** 6)
        assert s.lib.q2d_gpu_download_prim_many(s.ctx, 1, bad, pout) == _abi.ERR_BADARG
    finally:
        s.close()


def test_many_block_transfer_wraps_the_staging_ring():
    """More state than one staging ring (128 MiB of doubles): the transfer waits for the ring
    and reuses it, and every block still arrives intact."""
    batch = [cases.closed_box(1600, 1200, seed=s) for s in range(3)]    # 5.76M cells, 184 MB
    s = Q2DSolver(make_options(batch[0], precision=1), batch)
    try:
        s.step(1)
        rng = np.random.default_rng(5)
        ups, inners = zip(*[_ghosted(cs.blocks[0], rng, 0.0) for cs in batch])
        ids = (C.c_int * 3)(*[s.block_ids[c][0] for c in range(3)])
        pin = (C.POINTER(C.c_double) * 3)(*[_abi.dptr(a) for a in ups])
        assert s.lib.q2d_gpu_upload_prim_many(s.ctx, 3, ids, pin) == 0
        for got, inner in zip(s.prims(), inners):
            assert np.array_equal(got[0], inner)
    finally:
        s.close()
