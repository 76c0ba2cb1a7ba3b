"""Restart (newrun = false; Wrap_Setup.f90:114-149, Read_IC IO_Solution.f90:38-126) and the
reference's residual history (Wrap_Postprocess.f90:128-133, 248-253).

* Through the API: a time-accurate case stopped after N steps and resumed from its state and
  time (q2d_gpu_set_case_time) reaches, after M more steps, exactly the state of an N + M step
  run, on the GPU and on the oracle; GPU and oracle agree to 1e-10.
* Through q2d_host: the same from OUTPUT/field.tec with newrun = false (the field is written
  with 17 significant digits, so the resumed run is bitwise the continuous one); the residual
  history holds (I8,E20.10,4E20.10) lines every res-diter iterations, appended to on restart;
  a steady run writes SOLUTIONTIME = -iterations and a restart counts on from int() of it.
"""
import dataclasses

import numpy as np
import pytest

from q2d_b200 import cases, make_options, refio
from q2d_b200.solver import Q2DSolver
from tests.conftest import rel_linf
from tests.test_host_harness import host

pytestmark = pytest.mark.gpu


def sod():
    return cases.riemann_1d(ni=200, nj=2, states=(1.0, 1.0, 0.125, 0.1), limiter="vanleer", t_end=0.2)


def run(cs, steps, lib=None):
    from oracle import oracle
    s = oracle.solver(make_options(cs), [cs]) if lib == "oracle" else Q2DSolver(make_options(cs), [cs])
    try:
        info = s.step(steps)[0]
        return s.prim(), info
    finally:
        s.close()


def resumed(cs, prim, time):
    blk = dataclasses.replace(cs.blocks[0], prim=prim)
    return dataclasses.replace(cs, blocks=[blk], meta=dict(cs.meta, restart_time=time))


@pytest.mark.parametrize("lib", ["gpu", "oracle"])
def test_restart_through_the_api_is_the_continuous_run(lib):
    cs = sod()
    p40, i40 = run(cs, 40, lib)
    p70, i70 = run(cs, 70, lib)
    p, i = run(resumed(cs, p40, i40["time"]), 30, lib)
    assert np.array_equal(p, p70), rel_linf(p, p70)
    assert i["time"] == i70["time"] and i["iter"] == 30


def test_restart_gpu_matches_oracle():
    cs = sod()
    g40, gi = run(cs, 40)
    o40, oi = run(cs, 40, "oracle")
    g, _ = run(resumed(cs, g40, gi["time"]), 30)
    o, _ = run(resumed(cs, o40, oi["time"]), 30, "oracle")
    assert rel_linf(g, o).max() <= 1e-10


def read_history(path):
    rows = []
    for line in path.read_text().splitlines():
        assert len(line) == 108, repr(line)
        rows.append([int(line[:8])] + [float(line[8 + 20 * k:28 + 20 * k]) for k in range(5)])
    return np.array(rows)


def test_restart_through_the_host(tmp_path):
    cs = sod()
    a, b = tmp_path / "a", tmp_path / "b"
    for d in (a, b):
        refio.write_case(cs, d, res_diter=5)
    host(a, "--max-steps", 40, "--quiet")
    field40 = refio.read_field(a / "OUTPUT" / "field.tec")[0]
    text = (a / "input.ini").read_text()
    (a / "input.ini").write_text(text.replace("[Q2D-Parameters]\n", "[Q2D-Parameters]\nnewrun = false\n"))
    host(a, "--max-steps", 30, "--quiet")
    host(b, "--max-steps", 70, "--quiet")
    fa = refio.read_field(a / "OUTPUT" / "field.tec")[0]
    fb = refio.read_field(b / "OUTPUT" / "field.tec")[0]
    assert np.array_equal(fa.prim, fb.prim)
    ta = (a / "OUTPUT" / "field.tec").read_text().split("SOLUTIONTIME=")[1].split()[0]
    tb = (b / "OUTPUT" / "field.tec").read_text().split("SOLUTIONTIME=")[1].split()[0]
    assert ta == tb and float(ta) > 0.0
    assert not np.array_equal(field40.prim, fb.prim)
    ha, hb = read_history(a / "OUTPUT" / "residual-history.dat"), read_history(b / "OUTPUT" / "residual-history.dat")
    # 40 steps then 30 more (iteration counter from 0 again: time-accurate restart), every 5
    assert list(ha[:, 0]) == list(range(5, 45, 5)) + list(range(5, 35, 5))
    assert list(hb[:, 0]) == list(range(5, 75, 5))
    assert np.allclose(ha[-1, 1:], hb[-1, 1:], rtol=1e-9)   # E20.10: ten significant digits
    assert np.all(np.diff(hb[:, 1]) > 0)                   # physical time


def test_steady_solution_time_and_restart_count(tmp_path):
    cs = cases.ramp(48, 16, seed=4)
    refio.write_case(cs, tmp_path, res_diter=10)
    host(tmp_path, "--max-steps", 50, "--quiet")
    text = (tmp_path / "OUTPUT" / "field.tec").read_text()
    assert float(text.split("SOLUTIONTIME=")[1].split()[0]) == -50.0
    ini = (tmp_path / "input.ini").read_text()
    (tmp_path / "input.ini").write_text(ini.replace("[Q2D-Parameters]\n", "[Q2D-Parameters]\nnewrun = false\n"))
    host(tmp_path, "--max-steps", 30, "--quiet")
    h = read_history(tmp_path / "OUTPUT" / "residual-history.dat")
    # iter_general from int(-50) on, time -1 for steady runs (Wrap_Setup.f90:145-147)
    assert list(h[:, 0]) == [10, 20, 30, 40, 50, -40, -30, -20]
    assert np.all(h[:, 1] == -1.0)
    text = (tmp_path / "OUTPUT" / "field.tec").read_text()
    assert float(text.split("SOLUTIONTIME=")[1].split()[0]) == 20.0


def test_case_end_batch_vs_oracle():
    """A per-case end in a batch context (q2d_gpu_set_case_end before commit and between
    calls): the GPU and the oracle stop each case at the same iteration with the same state."""
    from oracle import oracle
    batch = [cases.ramp(60, 20, seed=2), cases.ramp(48, 16, seed=4)]
    opts = make_options(batch[0], itermax=100)
    batch[0].meta["iter_end"] = 9
    try:
        g, o = Q2DSolver(opts, batch), oracle.solver(opts, batch)
    finally:
        batch[0].meta.pop("iter_end")
    try:
        gi, oi = g.step(15), o.step(15)
        assert [x["iter"] for x in gi] == [x["iter"] for x in oi] == [9, 15]
        assert gi[0]["todo"] == oi[0]["todo"] == 3
        g.set_case_end(1, 18)
        o.set_case_end(1, 18)
        gi, oi = g.step(15), o.step(15)
        assert gi[1]["iter"] == oi[1]["iter"] == 18 and gi[1]["todo"] == 3
        for c in range(2):
            assert rel_linf(g.prim(c, 0), o.prim(c, 0)).max() <= 1e-12
    finally:
        g.close()
        o.close()
