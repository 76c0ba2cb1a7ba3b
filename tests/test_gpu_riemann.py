"""The Riemann solvers of Assign_Riemann_Solver (Mod_Riemann.f90:25-109) beside HLLC / HLLE /
LLF / SLAU / SLAU2 / HLLC+ / HLLE++: HLLEM, rotated HLLC, PLLF, exact, Hanel, AUSM+, AUSM+-up,
AUSM+-up2 (Lib_Riemann_HLL.f90:172-226, 355-434; Lib_Riemann_LF.f90:44-98;
Lib_Riemann_Godunov.f90:14-248; Lib_Riemann_AUSM.f90:18-321), one run-time selected
instantiation of each stage kernel.

* FP64 form against the CPU oracle: <= 1e-12 relative L-infinity after one step, <= 1e-10 after
  several, on the developed ramp-channel flow (one block and 2 x 2 blocks) and on Sod.
* FP32-flux form (these solvers take their flux in FP64 from the FP32 face states) against the
  FP64 form: <= 1e-6 relative L1 (2e-6 for the rotated HLLC, whose rotation follows the FP32
  velocity jump), on the FP32-flux kernel and on the FP32-slope tile kernel; the latter also for
  SLAU, which it runs the same way.
"""
import numpy as np
import pytest

from q2d_b200 import cases, make_options
from q2d_b200.solver import Q2DSolver
from tests.conftest import rel_l1
from tests.helpers import run_pair
from tests.test_gpu_sd import check, developed  # noqa: F401  (module fixture)

pytestmark = pytest.mark.gpu

REMAINING = ["HLLEM", "HLLC Rotated", "PLLF", "exact", "Hanel", "AUSM+", "AUSM+-up", "AUSM+-up2"]


def opts(riem, **kw):
    return dict(riemann=riem, riemann_minf=3.0, **kw) if "up" in riem else dict(riemann=riem, **kw)


@pytest.mark.parametrize("riem", REMAINING)
def test_remaining_solvers_ramp_vs_oracle(developed, riem):   # noqa: F811
    one, split = developed
    gs, os_, _, _ = run_pair([one], 1, **opts(riem))
    # the rotated HLLC splits each face along the direction of the velocity jump, which turns
    # ulp-level differences of the face states (the FP64 kernel's shared reciprocals) into
    # differences of a few 1e-12 where that jump is small
    check(gs, os_, 5e-12 if riem == "HLLC Rotated" else 1e-12, f"one block {riem} 1 step")
    gs, os_, _, _ = run_pair([split], 4, chunks=2, **opts(riem, shock_detector=0))
    check(gs, os_, 1e-10, f"split {riem} 4 steps")


def sod(ni=200):
    cs = cases.riemann_1d(ni=ni, nj=1, states=(1.0, 1.0, 0.125, 0.1), limiter="mc", t_end=0.2)
    for r in cs.bcs:
        r["type"] = 300
    return cs


@pytest.mark.parametrize("riem", REMAINING)
def test_remaining_solvers_sod_vs_oracle(riem):
    cfl = 0.2 if "up" in riem else 0.5
    kw = dict(riemann=riem, cfl=cfl, riemann_minf=0.1) if "up" in riem else dict(riemann=riem, cfl=cfl)
    gs, os_, gi, oi = run_pair([sod()], 1, **kw)
    check(gs, os_, 1e-12, f"sod {riem} 1 step")
    gs, os_, gi, oi = run_pair([sod()], 30, chunks=3, **kw)
    check(gs, os_, 1e-10, f"sod {riem} 30 steps")


@pytest.mark.parametrize("riem", REMAINING + ["SLAU", "SLAU2"])
def test_remaining_solvers_fp32flux_vs_fp64(developed, riem):   # noqa: F811
    one, _ = developed
    out = {}
    for prec, sch in ((0, 0), (1, 4), (1, 0)):
        # plain MUSCL: the FP32-slope tile kernel has no shock-sensor instantiation
        s = Q2DSolver(make_options(one, precision=prec, **opts(riem, shock_detector=0)), [one])
        try:
            s.set_schedule(sch)
            info = s.step(10)[0]
            assert info["err"] == 0, info
            out[(prec, sch)] = s.prims()[0][0]
        finally:
            s.close()
    # the rotated solver splits the face along the direction of the velocity jump, which the FP32
    # face states set only to their rounding where the jump is small: 2e-6 for it
    tol = 2e-6 if riem == "HLLC Rotated" else 1e-6
    for key in ((1, 4), (1, 0)):
        err = rel_l1(out[key], out[(0, 0)])
        assert err.max() <= tol, f"{riem} precision/schedule {key}: rel L1 {err}"


def test_ausm_up_needs_minf():
    cs = sod(40)
    for riem in ("AUSM+-up", "AUSM+-up2"):
        with pytest.raises(Exception):
            Q2DSolver(make_options(cs, riemann=riem), [cs])
    s = Q2DSolver(make_options(cs, riemann="AUSM+-up", riemann_minf=0.2), [cs])
    s.close()


ALL_SOLVERS = ["HLLC", "HLLE", "LLF", "SLAU", "SLAU2", "HLLC+", "HLLE++"] + REMAINING


@pytest.mark.parametrize("riem", ALL_SOLVERS)
def test_every_solver_is_the_same_on_every_fp64_tile(riem):
    """Each solver on the three FP64 tiles (and with MUSCL-SD) gives the same state to the bit
    (per-cell arithmetic does not depend on the tile), and the first tile equals the oracle to
    1e-11 after 3 steps (1e-9 for the rotated HLLC): the dispatch reaches the right solver from
    every tile and instantiation."""
    cs = cases.ramp(70, 21, seed=12)
    kw = opts(riem, limiter="mc")
    for sd in (0, 1):
        states = []
        for sch in (0, 1, 2):
            s = Q2DSolver(make_options(cs, shock_detector=sd, **kw), [cs])
            try:
                s.set_schedule(sch)
                assert s.step(3)[0]["err"] == 0
                states.append(s.prim())
            finally:
                s.close()
        assert np.array_equal(states[0], states[1]) and np.array_equal(states[0], states[2]), (riem, sd)
        gs, os_, _, _ = run_pair([cs], 3, schedule=0, shock_detector=sd, **kw)
        # the rotated solver's direction (the velocity jump) is ill-conditioned where the jump
        # is small, so rounding differences of the face states grow faster through it
        check(gs, os_, 1e-9 if riem == "HLLC Rotated" else 1e-11, f"{riem} sd {sd} 3 steps")
