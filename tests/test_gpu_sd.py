"""MUSCL-SD (space-reconstruction = MUSCL-SD): the face slopes scaled by the Tramel pressure
sensor of the face's left / lower cell (Mod_Fluxes.f90:132-204, Lib_Shock_Detector.f90:14-38),
of the boundary cell on a block-interface face (Lib_BC_Fluxes_Connection.f90).

* FP64 form against the CPU oracle: <= 1e-12 relative L-infinity after one step, <= 1e-10 after
  several, on every FP64 tile (ragged tiles included: the reference's ramp-channel grid is
  95 x 100 cells), on a developed flow whose shocks cross the tile edges, and on the same flow
  cut into 2 x 2 blocks whose interfaces the shocks cross (the sensor of halo cells across a tile
  or block edge, the corner ghosts), with each Riemann solver and limiter family.
* FP32-flux form against the FP64 form: <= 1e-6 relative L1 on every FP32-flux tile.
* The reference's ramp-channel case run to its 10000 iterations on the GPU passes its check.py
  gates (oblique-shock theory, sensor localisation, residual below 1e-3) with the errors the
  reference binary records, through the API and through q2d_host from the reference's formats.
* The sensor-driven Riemann solvers HLLC+ and HLLE++ (Lib_Riemann_HLL.f90:437-533, 572-605),
  which run the sensor with either reconstruction, to the same bars, and the ramp-channel case
  with each of them to the case's gates.
"""
import dataclasses

import numpy as np
import pytest

from q2d_b200 import make_options
from q2d_b200.solver import Q2DSolver
from tests.conftest import rel_l1, rel_linf
from tests.helpers import (ramp_channel_case, ramp_channel_gates, run_pair, sensor_field,
                           split_case)

pytestmark = pytest.mark.gpu


def check(gs, os_, tol, what):
    for c, (gb, ob) in enumerate(zip(gs, os_)):
        for b, (g, o) in enumerate(zip(gb, ob)):
            assert np.all(np.isfinite(g)), f"{what}: non-finite state case {c} block {b}"
            err = rel_linf(g, o)
            assert err.max() <= tol, f"{what}: case {c} block {b} rel Linf {err} > {tol}"


@pytest.fixture(scope="module")
def developed():
    """The ramp-channel flow after 150 oracle iterations (the oblique shock and its reflection
    formed), as a single-block case and cut into 2 x 2 blocks at i = 40, j = 50."""
    from oracle import oracle
    cs = ramp_channel_case()
    o = oracle.solver(make_options(cs), [cs])
    try:
        o.step(150)
        prim = o.prim()
    finally:
        o.close()
    one = dataclasses.replace(cs, blocks=[dataclasses.replace(cs.blocks[0], prim=prim)])
    beta = sensor_field(one, [prim])[0]
    assert (beta[:, 36:44] < 0.5).any() and (beta[46:54, :] < 0.5).any()   # shocks at the cuts
    return one, split_case(one, icuts=(40,), jcuts=(50,))


@pytest.mark.parametrize("schedule", [0, 1, 2])
def test_sd_ramp_channel_start_vs_oracle(schedule):
    cs = ramp_channel_case()
    gs, os_, _, _ = run_pair([cs], 1, schedule=schedule)
    check(gs, os_, 1e-12, f"ramp-channel sd schedule {schedule} 1 step")


@pytest.mark.parametrize("schedule", [0, 1, 2])
def test_sd_developed_vs_oracle(developed, schedule):
    for cs in developed:
        gs, os_, _, _ = run_pair([cs], 1, schedule=schedule)
        check(gs, os_, 1e-12, f"{cs.name} sd schedule {schedule} 1 step")
        gs, os_, gi, oi = run_pair([cs], 8, chunks=2, schedule=schedule)
        check(gs, os_, 1e-10, f"{cs.name} sd schedule {schedule} 8 steps")
        assert gi[0]["residual"][0] == pytest.approx(oi[0]["residual"][0], rel=1e-9)


@pytest.mark.parametrize("riemann,limiter", [("HLLC", "mc"), ("LLF", "vanleer"), ("SLAU", "vanalbada"),
                                             ("SLAU2", "superbee"), ("HLLE", "LIMO3")])
def test_sd_solvers_limiters_vs_oracle(developed, riemann, limiter):
    one, split = developed
    gs, os_, _, _ = run_pair([split], 4, chunks=2, riemann=riemann, limiter=limiter, irs_beta=0.0, cfl=0.5)
    check(gs, os_, 1e-10, f"split sd {riemann} {limiter}")
    gs, os_, _, _ = run_pair([one], 1, riemann=riemann, limiter=limiter, irs_beta=0.0, n_rk=2, cfl=0.5)
    check(gs, os_, 1e-12, f"one block sd {riemann} {limiter} rk2")


@pytest.mark.parametrize("schedule", [3, 4, 5, 6, 7])
def test_sd_fp32flux_vs_fp64(developed, schedule):
    for cs in developed:
        out = []
        for prec, sch in ((0, 0), (1, schedule)):
            s = Q2DSolver(make_options(cs, precision=prec), [cs])
            try:
                s.set_schedule(sch)
                info = s.step(10)[0]
                assert info["err"] == 0, info
                out.append(s.prims()[0])
            finally:
                s.close()
        for b, (g32, g64) in enumerate(zip(*out)):
            err = rel_l1(g32, g64)
            assert err.max() <= 1e-6, f"{cs.name} block {b} schedule {schedule}: rel L1 {err}"


def test_sd_changes_the_trajectory(developed):
    one, _ = developed
    a, _, _, _ = run_pair([one], 3)
    b, _, _, _ = run_pair([one], 3, shock_detector=0)
    assert rel_linf(a[0][0], b[0][0]).max() > 1e-6


@pytest.mark.parametrize("precision", [0, 1])
def test_ramp_channel_reference_gates(precision):
    """The reference's ramp-channel case on the GPU, its 10000 iterations: density residual below
    1e-3, the oblique-shock and sensor gates of its check.py, and the post / pre-shock errors the
    reference binary records (p2/p1 -0.002 %, T2/T1 +0.95 %, rho2/rho1 -0.94 %, M2 -0.94 %) to
    the digits given."""
    cs = ramp_channel_case()
    s = Q2DSolver(make_options(cs, precision=precision), [cs])
    try:
        info = s.step(10000)[0]
        prim = s.prims()[0][0]
    finally:
        s.close()
    assert info["err"] == 0 and info["iter"] == 10000 and info["residual"][0] < 1e-3, info
    beta = sensor_field(cs, [prim])[0]
    errs = 100.0 * np.array(ramp_channel_gates(cs, prim, beta))
    assert abs(errs[0] - (-0.002)) < 0.005, errs
    assert np.all(np.abs(errs[1:] - np.array([0.95, -0.94, -0.94])) < 0.01), errs


def test_ramp_channel_reference_case_through_host(tmp_path):
    """The ramp-channel case written in the reference's formats (space-reconstruction = MUSCL-SD)
    and run by q2d_host to its iteration limit: the residual history it writes stays finite and
    ends below 1e-3, and the field it writes passes the case's gates."""
    from q2d_b200 import refio
    from tests.test_host_harness import host
    cs = ramp_channel_case()
    refio.write_case(cs, tmp_path)
    assert "space-reconstruction = MUSCL-SD" in (tmp_path / "input.ini").read_text()
    host(tmp_path, "--gamma", repr(cs.options["gas_gamma"]), "--steps-per-call", 1000, "--quiet")
    res = np.loadtxt(tmp_path / "OUTPUT" / "residuals.dat")
    assert np.all(np.isfinite(res[:, 3])) and res[-1, 0] == 10000 and res[-1, 3] < 1e-3
    prim = refio.read_field(tmp_path / "OUTPUT" / "field.tec")[0].prim
    ramp_channel_gates(cs, prim, sensor_field(cs, [prim])[0])


@pytest.mark.parametrize("riemann", ["HLLC+", "HLLE++"])
@pytest.mark.parametrize("sd", [1, 0])
def test_sensor_driven_solvers_vs_oracle(developed, riemann, sd):
    """HLLC+ / HLLE++ (the sensor runs whatever the reconstruction; the Riemann solver blends by
    it) with MUSCL-SD and with plain MUSCL, on the three FP64 tiles."""
    for cs in developed:
        for schedule in (0, 1, 2):
            gs, os_, _, _ = run_pair([cs], 1, schedule=schedule, riemann=riemann, shock_detector=sd)
            check(gs, os_, 1e-12, f"{cs.name} {riemann} sd {sd} schedule {schedule} 1 step")
        gs, os_, gi, oi = run_pair([cs], 6, chunks=2, riemann=riemann, shock_detector=sd)
        check(gs, os_, 1e-10, f"{cs.name} {riemann} sd {sd} 6 steps")


@pytest.mark.parametrize("riemann", ["HLLC+", "HLLE++"])
def test_sensor_driven_solvers_fp32flux_vs_fp64(developed, riemann):
    for cs in developed:
        for schedule in (3, 4, 5, 6, 7):
            out = []
            for prec, sch in ((0, 0), (1, schedule)):
                s = Q2DSolver(make_options(cs, precision=prec, riemann=riemann), [cs])
                try:
                    s.set_schedule(sch)
                    info = s.step(10)[0]
                    assert info["err"] == 0, info
                    out.append(s.prims()[0])
                finally:
                    s.close()
            for b, (g32, g64) in enumerate(zip(*out)):
                err = rel_l1(g32, g64)
                assert err.max() <= 1e-6, f"{cs.name} {riemann} block {b} schedule {schedule}: rel L1 {err}"


@pytest.mark.parametrize("riemann", ["HLLC+", "HLLE++"])
@pytest.mark.parametrize("precision", [0, 1])
def test_ramp_channel_sensor_driven_solvers(riemann, precision):
    """The ramp-channel case with HLLC+ / HLLE++ (the reference's solver sweep) to its 10000
    iterations: residual below 1e-3 and the oblique-shock and sensor gates of its check.py."""
    cs = ramp_channel_case()
    s = Q2DSolver(make_options(cs, precision=precision, riemann=riemann), [cs])
    try:
        info = s.step(10000)[0]
        prim = s.prims()[0][0]
    finally:
        s.close()
    assert info["err"] == 0 and info["residual"][0] < 1e-3, info
    ramp_channel_gates(cs, prim, sensor_field(cs, [prim])[0])


@pytest.mark.parametrize("riemann", ["HLLC", "HLLC+", "AUSM+"])
def test_sd_one_dimensional_time_accurate(riemann):
    """MUSCL-SD on a 1-D time-accurate case (nj = 1: the sensor's j-neighbours are the ghost
    rows of both walls), FP64 against the oracle and the FP32-flux form against FP64."""
    from q2d_b200 import cases
    cs = cases.riemann_1d(ni=160, nj=1, states=(1.0, 1.0, 0.125, 0.1), limiter="minmod", t_end=0.2)
    gs, os_, _, _ = run_pair([cs], 1, shock_detector=1, riemann=riemann)
    check(gs, os_, 1e-12, f"1-D sd {riemann} 1 step")
    gs, os_, _, _ = run_pair([cs], 30, chunks=3, shock_detector=1, riemann=riemann)
    check(gs, os_, 1e-10, f"1-D sd {riemann} 30 steps")
    out = []
    for prec in (0, 1):
        s = Q2DSolver(make_options(cs, precision=prec, shock_detector=1, riemann=riemann), [cs])
        try:
            assert s.step(30)[0]["err"] == 0
            out.append(s.prim())
        finally:
            s.close()
    assert rel_l1(out[1], out[0]).max() <= 1e-6


@pytest.mark.parametrize("riemann", ["HLLEM", "exact", "AUSM+-up"])
def test_sd_with_run_time_solvers_fp32flux(developed, riemann):
    """MUSCL-SD with the run-time selected solvers in the FP32-flux form (its shock-sensor
    instantiation of the generic solver group) against the FP64 form."""
    one, _ = developed
    out = []
    for prec, sch in ((0, 0), (1, 4)):
        s = Q2DSolver(make_options(one, precision=prec, riemann=riemann, riemann_minf=3.0), [one])
        try:
            s.set_schedule(sch)
            assert s.step(10)[0]["err"] == 0
            out.append(s.prims()[0][0])
        finally:
            s.close()
    assert rel_l1(out[1], out[0]).max() <= 1e-6
