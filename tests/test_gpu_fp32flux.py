"""FP32-flux / FP64-state form on the GPU.

* Accuracy against the plain FP64 GPU path on the same inputs and steps: relative L1 error of
  every primitive variable (mean |fp32flux - fp64| over the variable's scale) <= 1e-6, the
  form's accuracy target; relative L-infinity <= 1e-4.
* Conservation: on a closed domain (slip walls) both forms keep the totals of mass and energy
  (sum of U * cell area) to round-off (1e-12 relative) over many steps.
* Schedules: every tile shape of the FP32-flux kernel gives the same state within the form's
  bound, and each schedule is deterministic run to run (bitwise).
"""
import numpy as np
import pytest

from q2d_b200 import cases, make_options
from q2d_b200.solver import Q2DSolver
from tests.conftest import cons, rel_l1, rel_linf

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6
LINF_TOL = 1e-4
SCHED = ["fp32-flux tile 32x10", "fp32-flux tile 32x8", "fp32-flux tile 64x4", "tile 32x10",
         "fp32-flux difference tile 32x8"]


def run(cs_list, steps, schedule=None, **ov):
    s = Q2DSolver(make_options(cs_list[0], **ov), cs_list)
    try:
        if schedule is not None:
            s.set_schedule(schedule)
        infos = s.step(steps, check=False)
        states = [[s.prim(c, b) for b in range(len(cs.blocks))] for c, cs in enumerate(cs_list)]
        return states, infos
    finally:
        s.close()


def compare(a, b, what):
    worst = np.zeros(2)
    for ca, cb in zip(a, b):
        for xa, xb in zip(ca, cb):
            assert np.all(np.isfinite(xa)), what
            l1, li = rel_l1(xa, xb).max(), rel_linf(xa, xb).max()
            worst = np.maximum(worst, [l1, li])
    assert worst[0] <= L1_TOL and worst[1] <= LINF_TOL, f"{what}: rel L1 {worst[0]:.3e} Linf {worst[1]:.3e}"
    return worst


@pytest.mark.parametrize("schedule", SCHED)
def test_ramp_fp32flux_vs_fp64(schedule):
    cs = cases.ramp(192, 64, seed=4)
    s32, i32 = run([cs], 300, schedule=schedule, precision=1)
    s64, i64 = run([cs], 300, precision=0)
    assert i32[0]["err"] == 0 and i64[0]["err"] == 0
    compare(s32, s64, f"ramp/{schedule}")


@pytest.mark.parametrize("schedule", SCHED[:2])
def test_axisymmetric_nozzle_blocks_fp32flux_vs_fp64(schedule):
    cs = cases.nozzle_axi(ni=64, nj=16, nblocks=3, seed=9)
    s32, i32 = run([cs], 200, schedule=schedule, precision=1)
    s64, i64 = run([cs], 200, precision=0)
    assert i32[0]["err"] == 0 and i64[0]["err"] == 0
    compare(s32, s64, f"nozzle_axi/{schedule}")


def test_area_batch_fp32flux_vs_fp64():
    batch = cases.area_nozzle_batch(n=12, seed=13, nx_range=(40, 200), ny_range=(8, 24))
    s32, _ = run(batch, 300, precision=1)
    s64, _ = run(batch, 300, precision=0)
    compare(s32, s64, "area batch")


@pytest.mark.parametrize("riemann", ["HLLE", "LLF"])
@pytest.mark.parametrize("limiter", ["minmod", "vanalbada", "mc", "superbee", "LIMO3", "iord"])
def test_fp32flux_solvers_and_limiters(riemann, limiter):
    cs = cases.ramp(96, 40, seed=3)
    s32, _ = run([cs], 40, precision=1, riemann=riemann, limiter=limiter)
    s64, _ = run([cs], 40, precision=0, riemann=riemann, limiter=limiter)
    compare(s32, s64, f"ramp/{riemann}/{limiter}")


def test_riemann1d_time_accurate_fp32flux():
    cs = cases.riemann_1d(ni=256, nj=4, seed=5)
    s32, i32 = run([cs], 150, precision=1)
    s64, i64 = run([cs], 150, precision=0)
    compare(s32, s64, "riemann1d")
    assert abs(i32[0]["time"] - i64[0]["time"]) <= 1e-6 * i64[0]["time"]


@pytest.mark.parametrize("precision", [0, 1])
def test_conservation_closed_domain(precision):
    cs = cases.closed_box(48, 40, seed=3)
    sur = cases.cell_areas(cs.blocks[0])
    s = Q2DSolver(make_options(cs, precision=precision), [cs])
    try:
        def totals():
            U = cons(s.prim(0, 0))
            return np.array([(U[..., k] * sur).sum() for k in (0, 3)])
        t0 = totals()
        s.step(100)
        t1 = totals()
        assert np.all(np.abs(t1 - t0) <= 1e-12 * np.abs(t0)), (t0, t1)
    finally:
        s.close()


def test_fp32flux_state_independent_of_tile():
    """Every face flux and cell update reads the same inputs whatever the tile shape, but each
    tile shape is a kernel instantiation of its own in which the compiler may fuse FP32
    multiply-adds differently: the schedules agree within the form's accuracy bound, and each
    one repeats its own result bit for bit (no dependence on timing or on the CTA order)."""
    batch = cases.area_nozzle_batch(n=5, seed=17, nx_range=(40, 150), ny_range=(8, 20))
    ref, _ = run(batch, 30, schedule=SCHED[0], precision=1)
    again, _ = run(batch, 30, schedule=SCHED[0], precision=1)
    for ca, cb in zip(again, ref):
        for xa, xb in zip(ca, cb):
            assert np.array_equal(xa, xb)
    for sch in (SCHED[1], SCHED[2], "fp32-flux tile 32x16", "fp32-flux tile 64x8", SCHED[4]):
        got, _ = run(batch, 30, schedule=sch, precision=1)
        compare(got, ref, sch)


@pytest.mark.parametrize("variant", ["inflow", "reverse", "low_p0"])
def test_stagnation_inflow_paths(variant):
    """The FP32-flux kernel evaluates stagnation inflow faces (BC 401) in FP32 when the
    discriminant of the face state is clearly positive, applies the symmetry flux when the flow
    leaves through the inlet, and hands negative or marginal discriminants (the reference's p0
    relaxation) to the FP64 routine. Each path stays within the form's tolerance of the plain
    FP64 path: a normal inflow, a reversed initial velocity (outflow through the inlet), and a
    total pressure below the interior pressure (negative discriminant)."""
    import copy
    cs = copy.deepcopy(cases.area_nozzle(96, 12, 1.5, 0.45, 5e5, 400.0))
    if variant == "reverse":
        cs.blocks[0].prim[..., 1] *= -1.0
    elif variant == "low_p0":
        for r in cs.bcs:
            if r["type"] == 401:
                r["p0"] = 0.5 * r["p0"]
    s32, i32 = run([cs], 20, precision=1)
    s64, i64 = run([cs], 20, precision=0)
    assert i32[0]["err"] == 0 and i64[0]["err"] == 0
    compare(s32, s64, f"stagnation inflow {variant}")
