"""CUDA path vs the CPU oracle (FP64 form): per-step parity at <= 1e-12 relative L-infinity
(|gpu - oracle| / max|oracle| per primitive variable), through the C ABI, on every boundary
type, limiter, Riemann solver, RK scheme and source on the path."""
import numpy as np
import pytest

from q2d_b200 import cases
from tests.conftest import rel_linf
from tests.helpers import run_pair

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-12


def check(gs, os_, tol, what):
    for c, (gb, ob) in enumerate(zip(gs, os_)):
        for b, (g, o) in enumerate(zip(gb, ob)):
            err = rel_linf(g, o)
            assert np.all(np.isfinite(g)), f"{what}: non-finite GPU state case {c} block {b}"
            assert err.max() <= tol, f"{what}: case {c} block {b} rel Linf {err} > {tol}"


@pytest.mark.parametrize("limiter", ["iord", "minmod", "vanleer", "vanalbada", "mc", "superbee", "LIMO3"])
def test_riemann1d_one_step_all_limiters(limiter):
    cs = cases.riemann_1d(ni=128, nj=4, seed=7)
    gs, os_, gi, oi = run_pair([cs], 1, limiter=limiter)
    check(gs, os_, TOL_STEP, f"riemann1d/{limiter}")
    assert gi[0]["iter"] == oi[0]["iter"] == 1
    assert abs(gi[0]["dtglobal"] - oi[0]["dtglobal"]) <= 1e-14 * oi[0]["dtglobal"]


@pytest.mark.parametrize("riemann", ["HLLC", "HLLE", "LLF"])
@pytest.mark.parametrize("n_rk", [1, 2, 3])
def test_ramp_one_step_solvers(riemann, n_rk):
    cs = cases.ramp(96, 40, seed=3)
    gs, os_, gi, oi = run_pair([cs], 1, riemann=riemann, n_rk=n_rk)
    check(gs, os_, TOL_STEP, f"ramp/{riemann}/rk{n_rk}")
    for k in range(4):
        assert abs(gi[0]["residual"][k] - oi[0]["residual"][k]) <= 1e-10 * max(oi[0]["residual"][k], 1e-300)


def test_ramp_many_steps():
    cs = cases.ramp(96, 40, seed=5)
    gs, os_, gi, oi = run_pair([cs], 40, chunks=4)
    check(gs, os_, 1e-10, "ramp/40 steps")
    assert gi[0]["iter"] == oi[0]["iter"] == 40


def test_axisymmetric_nozzle_connection_blocks():
    cs = cases.nozzle_axi(ni=48, nj=16, nblocks=3, seed=9)
    gs, os_, gi, oi = run_pair([cs], 1)
    check(gs, os_, TOL_STEP, "nozzle_axi/1 step")
    gs, os_, gi, oi = run_pair([cs], 20, chunks=2)
    check(gs, os_, 1e-10, "nozzle_axi/20 steps")


def test_area_nozzle_batch_cases():
    batch = cases.area_nozzle_batch(n=6, seed=11, nx_range=(24, 80), ny_range=(4, 12))
    gs, os_, gi, oi = run_pair(batch, 1)
    check(gs, os_, TOL_STEP, "area batch/1 step")
    gs, os_, gi, oi = run_pair(batch, 15, chunks=3)
    check(gs, os_, 1e-10, "area batch/15 steps")
    for a, b in zip(gi, oi):
        assert a["iter"] == b["iter"]


def test_time_accurate_to_end_time():
    cs = cases.riemann_1d(ni=64, nj=4, seed=3, t_end=0.05)
    gs, os_, gi, oi = run_pair([cs], 500, chunks=5)
    check(gs, os_, 1e-10, "riemann1d to t_end")
    assert gi[0]["todo"] == oi[0]["todo"] == 3
    assert gi[0]["iter"] == oi[0]["iter"]
    assert abs(gi[0]["time"] - oi[0]["time"]) <= 1e-12


@pytest.mark.parametrize("schedule", [0, 1, 2])
def test_halo_reaching_ghosts_of_untouched_edge(schedule):
    """ni = 129 and nj = 41 leave a last tile one cell wide / one row high for every tile
    shape, so the halo of the tile before it reaches the ghost layer of a block edge that
    none of its own cells touch."""
    from q2d_b200 import make_options
    from q2d_b200.solver import Q2DSolver
    from oracle import oracle
    cs = cases.ramp(129, 41, seed=8)
    opts = make_options(cs)
    g = Q2DSolver(opts, [cs])
    o = oracle.solver(opts, [cs])
    try:
        g.set_schedule(schedule)
        g.step(3)
        o.step(3)
        check([[g.prim(0, 0)]], [[o.prim(0, 0)]], 1e-11, f"ramp 129x41 schedule {schedule}")
    finally:
        g.close()
        o.close()
