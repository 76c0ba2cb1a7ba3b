"""Boundary paths that no benchmark case reaches, on the GPU against the oracle.

* BC 406 (BC_Outflow, Lib_BC_Fluxes_Outflow.f90:36-165): a supersonic exit and one with
  pamb <= 0 take the extrapolation branch; a subsonic exit under a back pressure above the
  isentropic pstar takes the back-pressure branch (face pressure relaxed by rel_fac, face
  sound speed along the isentrope, normal velocity from the outgoing Riemann invariant); exit
  faces with reverse flow fall back to the symmetry flux (Mod_BC_Fluxes.f90:216-227). Plain
  FP64 against the oracle <= 1e-12 relative L-infinity after one step and <= 1e-10 after 20,
  on every FP64 schedule; the FP32-flux form within its bound of the FP64 path.
* Translational periodic seams (BC 201, Mod_BC_Fluxes.f90:99-102 through the connection
  handler): a doubly periodic curvilinear box. FP64 against the oracle as above, and in both
  forms the totals of mass, both momenta and energy (sum of U times the cell area) stay put
  to round-off, 1e-12 of sum |U| times the area, over 200 steps while the flow moves.
"""
import copy

import numpy as np
import pytest

from q2d_b200 import cases, make_options
from q2d_b200.solver import Q2DSolver
from tests.conftest import cons, rel_l1, rel_l1_cons, rel_linf
from tests.helpers import run_pair

pytestmark = pytest.mark.gpu

FP64_SCHEDULES = ["tile 32x10", "tile 32x8", "tile 64x4"]
FP32_SCHEDULES = ["fp32-flux tile 32x10", "fp32-flux tile 32x8", "fp32-flux tile 64x4",
                  "fp32-flux difference tile 32x8"]


def outflow_case(kind: str):
    """Area-variation nozzle 120 x 10 with BC 406 at the exit. 'supersonic': the isentropic
    start (supersonic after the throat), pamb = 0.5 of the exit pressure. 'pamb0': the same
    with pamb = 0. 'subsonic': the subsonic isentropic branch through an area 1.3 times the
    sonic one, pamb 1.03 of the exit pressure, rel_fac 0.5. 'reverse': the subsonic case with
    the flow reversed in the last two columns of the lower four rows."""
    cs = copy.deepcopy(cases.area_nozzle(120, 10, 1.5, 0.45, 4e5, 450.0))
    g, R = 1.4, 287.0
    b = cs.blocks[0]
    if kind in ("subsonic", "reverse"):
        xn = np.linspace(0.0, 1.0, b.ni + 1)
        xc = 0.5 * (xn[:-1] + xn[1:])
        M = cases.mach_of_area(1.3 * (1.0 + 1.5 * (xc - 0.45) ** 2), np.zeros(b.ni, bool), g)
        rho, u, p = cases.isentropic_state(M, 4e5, 450.0, R, g)
        b.prim[..., 0] = rho[None, :]
        b.prim[..., 1] = u[None, :]
        b.prim[..., 3] = p[None, :]
        if kind == "reverse":
            b.prim[:4, -2:, 1] *= -1.0
    pe = float(b.prim[0, -1, 3])
    pamb = {"supersonic": 0.5 * pe, "pamb0": 0.0, "subsonic": 1.03 * pe, "reverse": 1.03 * pe}[kind]
    rel = 0.5 if kind in ("subsonic", "reverse") else 1.0
    for r in cs.bcs:
        if r["f"] == 2:
            r["type"] = 406
            r["pamb"] = pamb
            r["rel_fac"] = rel
    return cs


def check64(gs, os_, tol, what):
    for gb, ob in zip(gs, os_):
        for g, o in zip(gb, ob):
            assert np.all(np.isfinite(g)), what
            err = rel_linf(g, o).max()
            assert err <= tol, f"{what}: rel Linf {err:.3e} > {tol}"


@pytest.mark.parametrize("schedule", FP64_SCHEDULES)
@pytest.mark.parametrize("kind", ["supersonic", "pamb0", "subsonic", "reverse"])
def test_outflow_406_fp64_vs_oracle(kind, schedule):
    cs = outflow_case(kind)
    gs, os_, gi, oi = run_pair([cs], 1, schedule=schedule)
    check64(gs, os_, 1e-12, f"406/{kind}/{schedule}/1 step")
    assert gi[0]["err"] == oi[0]["err"] == 0
    gs, os_, gi, oi = run_pair([cs], 20, chunks=2, schedule=schedule)
    check64(gs, os_, 1e-10, f"406/{kind}/{schedule}/20 steps")
    assert gi[0]["iter"] == oi[0]["iter"] == 20


def test_outflow_406_branches_differ():
    """The subsonic back pressure really changes the exit flux: the subsonic case under BC 406
    departs from the same case under plain extrapolation (BC 400) in the exit column."""
    cs = outflow_case("subsonic")
    ext = copy.deepcopy(cs)
    for r in ext.bcs:
        if r["f"] == 2:
            r["type"] = 400
    a, _, _, _ = run_pair([cs], 1)
    b, _, _, _ = run_pair([ext], 1)
    d = np.abs(a[0][0][:, -1, 3] - b[0][0][:, -1, 3]).max() / np.abs(b[0][0][..., 3]).max()
    assert d > 1e-6, d


@pytest.mark.parametrize("schedule", FP32_SCHEDULES)
@pytest.mark.parametrize("kind", ["supersonic", "subsonic", "reverse"])
def test_outflow_406_fp32flux_vs_fp64(kind, schedule):
    cs = outflow_case(kind)
    opts32 = make_options(cs, precision=1)
    opts64 = make_options(cs, precision=0)
    out = []
    for opts, sch in ((opts32, schedule), (opts64, None)):
        s = Q2DSolver(opts, [cs])
        try:
            if sch is not None:
                s.set_schedule(sch)
            info = s.step(50, check=False)[0]
            assert info["err"] == 0
            out.append(s.prim(0, 0))
        finally:
            s.close()
    l1 = rel_l1(out[0], out[1]).max()
    l1c = rel_l1_cons(out[0], out[1]).max()
    li = rel_linf(out[0], out[1]).max()
    assert l1c <= 1e-6 and l1 <= 1e-6 and li <= 1e-4, (kind, schedule, l1c, l1, li)


@pytest.mark.parametrize("schedule", FP64_SCHEDULES)
def test_periodic_fp64_vs_oracle(schedule):
    cs = cases.periodic_box(40, 28)
    gs, os_, gi, oi = run_pair([cs], 1, schedule=schedule)
    check64(gs, os_, 1e-12, f"periodic/{schedule}/1 step")
    gs, os_, gi, oi = run_pair([cs], 30, chunks=3, schedule=schedule)
    check64(gs, os_, 1e-10, f"periodic/{schedule}/30 steps")


@pytest.mark.parametrize("schedule", FP64_SCHEDULES + FP32_SCHEDULES)
def test_periodic_conservation(schedule):
    cs = cases.periodic_box(48, 36, seed=11)
    sur = cases.cell_areas(cs.blocks[0])
    prec = 1 if schedule.startswith("fp32") else 0
    s = Q2DSolver(make_options(cs, precision=prec), [cs])
    try:
        s.set_schedule(schedule)

        def totals():
            U = cons(s.prim(0, 0))
            return (np.array([(U[..., k] * sur).sum() for k in range(4)]),
                    np.array([(np.abs(U[..., k]) * sur).sum() for k in range(4)]))
        t0, m0 = totals()
        info = s.step(200, check=False)[0]
        t1, _ = totals()
        assert info["err"] == 0
        assert np.all(np.abs(t1 - t0) <= 1e-12 * m0), (schedule, (t1 - t0) / m0)
        assert np.abs(s.prim(0, 0) - cs.blocks[0].prim).max() > 1e-3
    finally:
        s.close()
