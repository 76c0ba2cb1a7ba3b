"""The command-line host (q2d_b200/lib/q2d_host): reads a case directory in the reference's
formats (input.ini, INPUT/bc.txt, INPUT/ic.tec, INPUT/block<b>_area.dat, INPUT/phase.txt) and
runs it through the C ABI, as the Fortran host's Q2D_setup / Q2D_solve would.

CPU tests run its --check mode (inputs parsed, no GPU); GPU tests run cases end to end and
compare the written OUTPUT/field.tec with the same cases run through the Python binding, and
the Shu-Osher run with the reference binary's own output."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from q2d_b200 import _abi, cases, make_options, refio
from q2d_b200.solver import Q2DSolver

GOLD = Path(__file__).resolve().parent / "golden"
OPT_FIELDS = ["limiter", "riemann", "n_rk", "time_accurate", "source", "rampa_iter", "res_diter",
              "sol_diter", "itermax", "cfl", "res_threshold", "time_threshold", "sol_dtime", "gas_R", "irs_beta",
              "shock_detector", "riemann_minf"]


def host(*args, check=True):
    r = subprocess.run([str(refio.host_binary()), *map(str, args)], capture_output=True, text=True, timeout=600)
    if check and r.returncode != 0:
        raise AssertionError(f"q2d_host {args}: rc={r.returncode}\n{r.stdout}\n{r.stderr}")
    return r


def small_cases():
    return {
        "ramp": cases.ramp(40, 12, seed=5),
        "nozzle_axi": cases.nozzle_axi(48, 10, nblocks=3, seed=6),
        "area_nozzle": cases.area_nozzle_batch(n=2, seed=7, nx_range=(40, 60), ny_range=(8, 10))[0],
        "shuosher": cases.shuosher(ni=64),
        "riemann1d": cases.riemann_1d(ni=50, nj=4, seed=8),
    }


def rec_tuple(r):
    alpha = r.get("alpha", 0.0)
    t = r["type"]
    if t not in (401, 405):
        alpha = 0.0
    alpha = -1.0 if alpha >= 0.5 * _abi.NORMAL_DIR else alpha
    keep = {401: ("T0", "p0", "rel_fac"), 405: ("mach", "T0", "pamb", "rel_fac"), 406: ("pamb", "rel_fac")}.get(t, ())
    vals = [float(r[k]) if k in keep else (1.0 if k == "rel_fac" else 0.0)
            for k in ("T0", "p0", "pamb", "mach")] + [alpha, float(r.get("rel_fac", 1.0)) if "rel_fac" in keep else 1.0]
    ints = [r["b"], r["i"], r["j"], r["f"], t]
    conn = [r.get("bs", 0), r.get("is_", r.get("is", 0)), r.get("js", 0), r.get("fs", 0),
            r.get("d11", 0), r.get("d12", 0), r.get("d21", 0), r.get("d22", 0)] if t == 101 else [0] * 8
    return ints + conn + vals


@pytest.mark.parametrize("name", ["ramp", "nozzle_axi", "area_nozzle", "shuosher", "riemann1d"])
def test_check_mode_reads_what_was_written(tmp_path, name):
    cs = small_cases()[name]
    refio.write_case(cs, tmp_path)
    o = make_options(cs)
    d = json.loads(host(tmp_path, "--check", "--gamma", repr(o.gas_gamma)).stdout)
    for k in OPT_FIELDS:
        assert d[k] == pytest.approx(getattr(o, k), rel=1e-15), k
    assert d["gas_gamma"] == o.gas_gamma
    assert d["unsupported"] == []
    assert [(b["ni"], b["nj"]) for b in d["blocks"]] == [(b.ni, b.nj) for b in cs.blocks]
    for got, B in zip(d["blocks"], cs.blocks):
        assert got["prim_sum"] == pytest.approx(float(np.sum(B.prim[..., 0]) + np.sum(B.prim[..., 1]) +
                                                      np.sum(B.prim[..., 2]) + np.sum(B.prim[..., 3])), rel=1e-12)
        if B.area is not None:
            assert got["area_sum"] == pytest.approx(float(np.sum(B.area)), rel=1e-12)
    assert len(d["bcs"]) == len(cs.bcs)
    for got, r in zip(d["bcs"], cs.bcs):
        assert got[:13] == rec_tuple(r)[:13]
        assert got[13:] == pytest.approx(rec_tuple(r)[13:], rel=1e-15)


def test_check_mode_limiter_keywords(tmp_path):
    """Setup_Space_Scheme / Assign_Limiter (Mod_Space.f90:18-78): MUSCL with 'none' is van Leer,
    the keyword is case-sensitive (lower-case 'limo3' is first order), and the limiter applies
    whatever the reconstruction keyword says."""
    cs = cases.ramp(20, 8)
    refio.write_case(cs, tmp_path)
    ini = (tmp_path / "input.ini").read_text()
    base = ini.replace("space-reconstruction = MUSCL\n", "").replace("flux-limiter = vanleer\n", "")
    for recon, lim, want in [("MUSCL", "none", 2), ("MUSCL", "limo3", 0), ("MUSCL", "LIMO3", 6),
                             ("first-order", "minmod", 1), ("MUSCL", "", 0), ("MUSCL", "superbee", 5)]:
        extra = f"space-reconstruction = {recon}\n" + (f"flux-limiter = {lim}\n" if lim else "")
        (tmp_path / "input.ini").write_text(base.replace("[Q2D-Numerics]\n", "[Q2D-Numerics]\n" + extra))
        assert json.loads(host(tmp_path, "--check").stdout)["limiter"] == want, (recon, lim)
    # MUSCL-SD turns the shock sensor on (Mod_Space.f90:25-27); without MUSCL it stays off
    for recon, want in [("MUSCL-SD", 1), ("MUSCL", 0), ("first-order", 0), ("SD", 0)]:
        extra = f"space-reconstruction = {recon}\nflux-limiter = minmod\n"
        (tmp_path / "input.ini").write_text(base.replace("[Q2D-Numerics]\n", "[Q2D-Numerics]\n" + extra))
        d = json.loads(host(tmp_path, "--check").stdout)
        assert d["shock_detector"] == want and not d["unsupported"], (recon, d["unsupported"])


def test_inputs_outside_the_path_fail_loudly(tmp_path):
    cs = cases.ramp(20, 8)
    refio.write_case(cs, tmp_path)
    ini = (tmp_path / "input.ini").read_text()
    (tmp_path / "input.ini").write_text(ini.replace("integration-variables = cons", "integration-variables = prim")
                                        .replace("[Q2D-IO]\n", "[Q2D-IO]\nsol-format = tecplot binary\n"))
    d = json.loads(host(tmp_path, "--check").stdout)
    assert d["unsupported"] == ["[Q2D-Numerics] integration-variables = prim", "[Q2D-IO] sol-format = tecplot binary"]
    r = host(tmp_path, check=False)   # refused before any device call
    assert r.returncode == 2 and "not on the built path" in r.stderr
    # Assign_Riemann_Solver keywords (Mod_Riemann.f90:25-109) of the built solvers
    for name, want in [("HLLC", 0), ("HLLE", 1), ("LLF", 2), ("Rusanov", 2), ("SLAU", 3), ("SLAU2", 4),
                       ("HLLC+", 5), ("HLLE++", 6), ("HLLEM", 7), ("HLLC Rotated", 8), ("PLLF", 9), ("exact", 10),
                       ("Exact", 10), ("Hanel", 11), ("AUSM+", 12), ("Roe", 0), ("hllc", 0)]:   # default: HLLC
        (tmp_path / "input.ini").write_text(ini.replace("riemann-solver = HLLC", f"riemann-solver = {name}"))
        d = json.loads(host(tmp_path, "--check").stdout)
        assert d["riemann"] == want and not d["unsupported"], (name, d["unsupported"])
    for name, want in [("AUSM+-up", 13), ("AUSM+-up2", 14)]:   # Minf required (Assign_Setup.f90:108-112)
        text = ini.replace("riemann-solver = HLLC", f"riemann-solver = {name}")
        (tmp_path / "input.ini").write_text(text)
        r = host(tmp_path, "--check", check=False)
        assert r.returncode != 0 and "Minf" in r.stderr
        (tmp_path / "input.ini").write_text(text.replace("[Q2D-Numerics]\n", "[Q2D-Numerics]\nriemann-options-Minf = 0.3\n"))
        d = json.loads(host(tmp_path, "--check").stdout)
        assert d["riemann"] == want and d["riemann_minf"] == 0.3 and not d["unsupported"]
    (tmp_path / "input.ini").write_text(ini)
    bc = (tmp_path / "INPUT" / "bc.txt").read_text().splitlines()
    bc[0] = bc[0][:-8] + f"{410:8d}"
    (tmp_path / "INPUT" / "bc.txt").write_text("\n".join(bc) + "\n")
    r = host(tmp_path, "--check", check=False)
    assert r.returncode == 1 and "410" in r.stderr


def test_reads_list_directed_records_across_lines(tmp_path):
    """Read_BCfile uses list-directed READs: a record may span lines, commas separate values and
    anything after the needed values on a line is skipped."""
    cs = cases.ramp(6, 4)
    refio.write_case(cs, tmp_path)
    txt = (tmp_path / "INPUT" / "bc.txt").read_text().splitlines()
    out = []
    for line in txt:
        t = line.split()
        if len(t) == 5 and t[4] == "405":
            out += [f"{t[0]}, {t[1]}, {t[2]}", f"{t[3]} {t[4]}  ! trailing text"]
        else:
            out.append(line)
    (tmp_path / "INPUT" / "bc.txt").write_text("\n".join(out) + "\n")
    d = json.loads(host(tmp_path, "--check").stdout)
    assert len(d["bcs"]) == len(cs.bcs)
    assert [r[4] for r in d["bcs"]] == [r["type"] for r in cs.bcs]


def _python_run(cs, steps, precision, irs_beta=0.0):
    s = Q2DSolver(make_options(cs, precision=precision, irs_beta=irs_beta), [cs])
    try:
        s.step(steps, check=False)
        return [s.prim(0, b) for b in range(len(cs.blocks))], s.info(0)
    finally:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,precision,irs", [("ramp", "fp64", 0.0), ("nozzle_axi", "fp64", 0.0),
                                               ("area_nozzle", "fp32-flux", 0.0), ("nozzle_axi", "fp64", 0.5)])
def test_host_run_equals_library_run(tmp_path, name, precision, irs):
    cs = small_cases()[name]
    steps = 25
    refio.write_case(cs, tmp_path, itermax=steps, irs_beta=irs)
    o = make_options(cs)
    r = host(tmp_path, "--precision", precision, "--gamma", repr(o.gas_gamma), "--steps-per-call", 10)
    assert "converged/ended after 25 steps" in r.stdout
    got = refio.read_field(tmp_path / "OUTPUT" / "field.tec")
    want, info = _python_run(cs, steps, 0 if precision == "fp64" else 1, irs)
    assert info["iter"] == steps
    for g, w, B in zip(got, want, cs.blocks):
        assert np.array_equal(g.nodes, np.asarray(B.nodes))
        assert np.array_equal(g.prim, w)
    hist = np.loadtxt(tmp_path / "OUTPUT" / "residuals.dat")
    assert hist[-1, 0] == steps and hist[-1, 3] == pytest.approx(info["residual"][0], rel=1e-15)


@pytest.mark.gpu
def test_host_shuosher_matches_reference_binary(tmp_path):
    """End to end from the reference's formats: the Shu-Osher case directory (N=400, MC, HLLC,
    RK3, CFL 0.5, time-accurate to t=1.8) run by q2d_host on the GPU reproduces the density the
    reference binary wrote (test/1D/ShuOsher-LIMO3/reference/baseline_mc.dat) to <= 1e-8
    relative L1, the gate the oracle meets."""
    cs = cases.shuosher()
    refio.write_case(cs, tmp_path, limiter="mc")
    host(tmp_path, "--steps-per-call", 200, "--quiet")
    ref = np.loadtxt(GOLD / "shuosher_mc.txt")
    rho = refio.read_field(tmp_path / "OUTPUT" / "field.tec")[0].prim[0, :, 0]
    rel_l1 = np.abs(rho - ref[:, 1]).sum() / np.abs(ref[:, 1]).sum()
    assert rel_l1 <= 1e-8, rel_l1


def test_restart_input_selection(tmp_path):
    """newrun = false (Read_IC, IO_Solution.f90:78-96; Wrap_Setup.f90:132-149): the initial field
    is OUTPUT/field.tec, else the last of OUTPUT/field1.tec, field2.tec, ...; a time-accurate
    case resumes at its SOLUTIONTIME, a steady one counts iterations from int(SOLUTIONTIME); a
    new run ignores SOLUTIONTIME; no restart field is an error."""
    cs = cases.riemann_1d(ni=40, nj=2, seed=4)
    refio.write_case(cs, tmp_path)
    ini = (tmp_path / "input.ini").read_text()
    ic = (tmp_path / "INPUT" / "ic.tec").read_text()
    out = tmp_path / "OUTPUT"
    out.mkdir()
    stamped = ic.replace("SOLUTIONTIME=0.000000000000000E+000", "SOLUTIONTIME=1.25E-002")
    assert stamped != ic
    (tmp_path / "INPUT" / "ic.tec").write_text(stamped)
    d = json.loads(host(tmp_path, "--check").stdout)
    assert d["newrun"] == 1 and d["case_time"] == 0.0 and d["initial_field"].endswith("INPUT/ic.tec")
    restart = ini.replace("[Q2D-Parameters]\n", "[Q2D-Parameters]\nnewrun = false\n")
    (tmp_path / "input.ini").write_text(restart)
    r = host(tmp_path, "--check", check=False)
    assert r.returncode != 0 and "OUTPUT/field.tec" in r.stderr
    (out / "field1.tec").write_text(stamped)
    (out / "field2.tec").write_text(stamped.replace("1.25E-002", "2.5E-002"))
    d = json.loads(host(tmp_path, "--check").stdout)
    assert d["initial_field"].endswith("OUTPUT/field2.tec") and d["case_time"] == 0.025 and d["iter_base"] == 0
    (out / "field.tec").write_text(stamped.replace("1.25E-002", "-3.0E+002"))
    d = json.loads(host(tmp_path, "--check").stdout)
    assert d["initial_field"].endswith("OUTPUT/field.tec") and d["case_time"] == -300.0
    (tmp_path / "input.ini").write_text(restart.replace("time-accurate = true", "time-accurate = false"))
    d = json.loads(host(tmp_path, "--check").stdout)
    assert d["time_accurate"] == 0 and d["case_time"] == 0.0 and d["iter_base"] == -300


def test_gamma_from_the_constant_cp_table(tmp_path):
    """--gamma table: gamma = cp / (cp - R) from INPUT/thermo.dat when cp is the same on every row
    (the reference's Air table); a temperature-dependent cp selects the thermally perfect table
    (every row, knot 0 extrapolated); rows off the 1-K grid are refused."""
    cs = cases.ramp(20, 8)
    refio.write_case(cs, tmp_path)
    d = json.loads(host(tmp_path, "--check", "--gamma", "table").stdout)
    R = d["gas_R"]
    lines = (tmp_path / "INPUT" / "thermo.dat").read_text().splitlines()
    rows = [ln for ln in lines if ln.strip() and (ln.strip()[0].isdigit() or ln.strip()[0] == ".")]
    cp = float(rows[0].split()[1])
    assert d["gas_gamma"] == pytest.approx(cp / (cp - R), rel=1e-15)
    k = lines.index(rows[-1])
    t = rows[-1].split()
    t[1] = repr(cp * 1.01)
    lines[k] = " ".join(t)
    (tmp_path / "INPUT" / "thermo.dat").write_text("\n".join(lines) + "\n")
    d = json.loads(host(tmp_path, "--check", "--gamma", "table").stdout)
    assert d["thermo_knots"] == len(rows) + 1 and d["gas_gamma"] == pytest.approx(cp / (cp - R), rel=1e-15)
    t[0] = "7.5"
    lines[k] = " ".join(t)
    (tmp_path / "INPUT" / "thermo.dat").write_text("\n".join(lines) + "\n")
    r = host(tmp_path, "--check", "--gamma", "table", check=False)
    assert r.returncode != 0 and "rows must be at T = 1, 2" in r.stderr
