"""The CPU oracle against the reference's own golden data and known answers.

Pins (tests/golden, generated by tests/golden/make_golden.py from the reference tree):
  - ShuOsher-LIMO3 limiter baselines: density written by the reference binary at N=400,
    t=1.8, HLLC, RK3, CFL 0.5 (test/1D/ShuOsher-LIMO3/reference/baseline_*.dat);
  - Sod79 exact solution table (test/1D/Sod79/reference/exact.txt) with the gates of
    test/1D/Sod79/check.py (discretisation-error gates, shock position);
  - exact Riemann solutions of the seeded 1-D workloads from the reference's exact solver
    (test/common/pycheck/q2d_exact1d.py), and its Toro test-1 known answer.
"""
from pathlib import Path

import numpy as np
import pytest

from q2d_b200 import cases, make_options
from oracle import oracle

GOLD = Path(__file__).resolve().parent / "golden"


def run_oracle(cs, **kw):
    s = oracle.solver(make_options(cs, **kw), [cs])
    try:
        info = s.solve(steps_per_call=200)
        return s.prim(), info
    finally:
        s.close()


@pytest.mark.parametrize("lim", ["iord", "minmod", "vanleer", "mc"])
def test_shuosher_matches_reference_binary(lim):
    """The oracle reproduces the reference binary's Shu-Osher density to <= 1e-8 relative L1
    (the baselines are printed with 10 significant digits) and <= 2e-7 max abs."""
    ref = np.loadtxt(GOLD / f"shuosher_{lim}.txt")
    cs = cases.shuosher()
    P, info = run_oracle(cs, limiter=lim)
    rho = P[0, :, 0]
    assert np.allclose(cs.meta["xc"], ref[:, 0], atol=1e-9)
    rel_l1 = np.abs(rho - ref[:, 1]).sum() / np.abs(ref[:, 1]).sum()
    assert rel_l1 <= 1e-8, rel_l1
    assert np.abs(rho - ref[:, 1]).max() <= 2e-7
    assert info["todo"] == 3 and info["time"] >= 1.8


def test_shuosher_negative_control():
    """A perturbed closure (the table's gamma = cp/(cp-R) = 1.399996 instead of 1.4) must FAIL
    the 1e-8 gate: the pin discriminates at the 1e-6 level."""
    ref = np.loadtxt(GOLD / "shuosher_mc.txt")
    R = 8314.46 / 28.970418
    P, _ = run_oracle(cases.shuosher(gamma=1004.5 / (1004.5 - R)), limiter="mc")
    rel_l1 = np.abs(P[0, :, 0] - ref[:, 1]).sum() / np.abs(ref[:, 1]).sum()
    assert rel_l1 > 1e-7


def sod79(riemann):
    cs = cases.riemann_1d(ni=400, nj=1, states=(1.0, 1.0, 0.125, 0.1), limiter="mc", t_end=0.2)
    for r in cs.bcs:   # the Sod79 case has BC 300 on every face (closed tube)
        r["type"] = 300
    return cs


def sod79_l1(P):
    ex = np.loadtxt(GOLD / "sod79_exact.txt")
    xc = 0.5 * (np.linspace(0, 1, 401)[:-1] + np.linspace(0, 1, 401)[1:])
    rho, p = P[0, :, 0], P[0, :, 3]
    re = np.interp(xc, ex[:, 0], ex[:, 1])
    pe = np.interp(xc, ex[:, 0], ex[:, 3])
    return np.abs(rho - re).sum() / np.abs(re).sum(), np.abs(p - pe).sum() / np.abs(pe).sum()


def test_sod79_slau_matches_reference_calibration():
    """The reference's own Sod79 configuration (400 cells, MC + SLAU, RK3, CFL 0.9, t = 0.2,
    closed tube; test/1D/Sod79/input.ini): the relative L1 errors of rho and p against the
    exact solution equal the values the reference binary measured when the case's gates were
    calibrated (test/1D/Sod79/check.py:14-15: 2.94e-3 and 2.08e-3) to the three digits
    printed there."""
    P, info = run_oracle(sod79("SLAU"), cfl=0.9, riemann="SLAU")
    l1r, l1p = sod79_l1(P)
    assert round(l1r, 5) == 0.00294 and round(l1p, 5) == 0.00208, (l1r, l1p)
    assert info["todo"] == 3 and info["time"] >= 0.2


def test_sod79_exact_gates():
    """Sod (rho 1/0.125, p 1/0.1) at 400 cells to t=0.2 with MC + HLLC, RK3, CFL 0.9:
    relative L1 of rho and p against the reference's exact.txt within the check.py gates
    (5e-3 / 3.5e-3) and the shock within 3 cells of x = 0.85043."""
    ex = np.loadtxt(GOLD / "sod79_exact.txt")
    cs = cases.riemann_1d(ni=400, nj=1, states=(1.0, 1.0, 0.125, 0.1), limiter="mc", t_end=0.2)
    # the Sod79 case has BC 300 on every face (closed tube)
    for r in cs.bcs:
        r["type"] = 300
    P, info = run_oracle(cs, cfl=0.9)
    xc = 0.5 * (np.linspace(0, 1, 401)[:-1] + np.linspace(0, 1, 401)[1:])
    rho, p = P[0, :, 0], P[0, :, 3]
    re = np.interp(xc, ex[:, 0], ex[:, 1])
    pe = np.interp(xc, ex[:, 0], ex[:, 3])
    l1r = np.abs(rho - re).sum() / np.abs(re).sum()
    l1p = np.abs(p - pe).sum() / np.abs(pe).sum()
    assert l1r <= 5e-3 and l1p <= 3.5e-3, (l1r, l1p)
    k = int(np.argmax(np.abs(np.diff(p[300:])))) + 300   # steepest pressure face right of the contact
    assert abs(0.5 * (xc[k] + xc[k + 1]) - 0.85043) <= 3 * 0.0025


def test_exact_riemann_seeded_workload():
    """The seeded 1-D workload (1024 x 4, minmod + HLLC) against the reference's exact solver:
    density L1 error of a first/second-order scheme at 1024 cells is a few 1e-3."""
    d = np.load(GOLD / "riemann_exact.npz")
    st = d["cfg1_states"]
    rl, _, pl, rr, _, pr = st[:6]
    cs = cases.riemann_1d(ni=int(st[6]), nj=4, states=(rl, pl, rr, pr), t_end=float(st[8]))
    P, info = run_oracle(cs)
    rho = P[:, :, 0].mean(axis=0)
    l1 = np.abs(rho - d["cfg1_rho"]).mean() / np.abs(d["cfg1_rho"]).mean()
    assert l1 <= 6e-3, l1
    # the four rows of the quasi-1D block stay identical (symmetry walls)
    assert np.abs(P[:, :, 0] - P[0:1, :, 0]).max() <= 1e-12


def test_exact_solver_known_answer():
    pstar, ustar = np.load(GOLD / "riemann_exact.npz")["toro1_pstar_ustar"]
    assert abs(pstar - 0.30313) < 1e-5 and abs(ustar - 0.92745) < 1e-5


# ------------------------------------------------------------------------------------------
# known answers for the scalar kernels
# ------------------------------------------------------------------------------------------
LIM = {"iord": 0, "minmod": 1, "vanleer": 2, "vanalbada": 3, "mc": 4, "superbee": 5, "LIMO3": 6}


def lim(name, x, y):
    return oracle.load().q2d_oracle_limiter(LIM[name], x, y)


def test_limiter_known_answers():
    assert lim("iord", 1.0, 2.0) == 0.0
    assert lim("minmod", 1.0, 2.0) == 1.0 and lim("minmod", 2.0, 1.0) == 1.0
    assert lim("minmod", 1.0, -1.0) == 0.0 and lim("minmod", -3.0, -2.0) == -2.0
    assert lim("minmod", 1.0, 1.0) == 1.0   # ties keep x (Lib_Limiters.f90:43-44)
    assert abs(lim("vanleer", 1.0, 1.0) - 1.0) < 1e-15
    assert abs(lim("vanleer", 1.0, 3.0) - 1.5) < 1e-15      # 2xy/(x+y)
    assert lim("vanleer", 1.0, -1.0) == 0.0
    assert abs(lim("vanalbada", 1.0, 1.0) - 1.0) < 1e-15
    assert abs(lim("mc", 1.0, 3.0) - 2.0) < 1e-15           # min(2r, (1+r)/2, 2) * x
    assert abs(lim("mc", 1.0, 0.5) - 0.75) < 1e-15
    assert abs(lim("superbee", 1.0, 0.5) - 1.0) < 1e-15
    assert abs(lim("superbee", 1.0, 3.0) - 2.0) < 1e-15
    assert abs(lim("LIMO3", 1.0, 1.0) - 1.0) < 1e-15
    assert lim("LIMO3", 1.0, -0.5) > 0.0                     # third order: no clip at extrema


def riemann(kind, L, R, nx=1.0, ny=0.0):
    import ctypes as C
    lib = oracle.load()
    opt = make_options({})
    a = (C.c_double * 4)(*L)
    b = (C.c_double * 4)(*R)
    out = (C.c_double * 4)()
    lib.q2d_oracle_riemann(kind, C.byref(opt), a, b, nx, ny, out)
    return np.array(out[:])


def phys_flux(P, nx, ny, g=1.4):
    r, u, v, p = P
    un = u * nx + v * ny
    H = g / (g - 1) * p / r + 0.5 * (u * u + v * v)
    return np.array([r * un, r * un * u + p * nx, r * un * v + p * ny, r * un * H])


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_riemann_consistency(kind):
    """F(U, U) equals the physical flux for HLLC, HLLE and Rusanov, in any direction."""
    rng = np.random.default_rng(5)
    for _ in range(20):
        P = [rng.uniform(0.2, 3), rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(0.2, 5)]
        th = rng.uniform(0, 2 * np.pi)
        n = (np.cos(th), np.sin(th))
        F = riemann(kind, P, P, *n)
        assert np.allclose(F, phys_flux(P, *n), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_riemann_supersonic_upwinding(kind):
    """Supersonic flow along the normal: HLLC/HLLE return the left physical flux exactly."""
    L = [1.0, 5.0, 0.3, 1.0]
    R = [0.5, 4.0, -0.2, 0.7]
    F = riemann(kind, L, R)
    if kind in (0, 1):
        assert np.allclose(F, phys_flux(L, 1.0, 0.0), rtol=1e-13)


def test_conservation_closed_domain():
    """All-wall (BC 300) curvilinear box, random smooth state: the oracle conserves mass and
    energy to round-off per step (sum of U * sur)."""
    cs = cases.closed_box(24, 24, seed=3)
    sur = cases.cell_areas(cs.blocks[0])
    s = oracle.solver(make_options(cs), [cs])
    try:
        def totals(P):
            from tests.conftest import cons
            U = cons(P)
            return np.array([(U[..., k] * sur).sum() for k in (0, 3)])
        t0 = totals(s.prim())
        s.step(20)
        t1 = totals(s.prim())
        assert np.all(np.abs(t1 - t0) <= 1e-12 * np.abs(t0)), (t0, t1)
    finally:
        s.close()


def test_planar_nozzle_irs_matches_reference_binary():
    """The reference's planar-nozzle case (implicit residual smoothing beta 0.5, stagnation
    inflow, area-variation source) through the oracle: its density residual follows the
    reference binary's printed history (test/2D/euler/planar-nozzle/solve.log) within 5 % at
    every printed iteration over six decades of convergence, it meets res-threshold 1e-10
    within 5 iterations of the binary (3172), and the converged state passes the case's own
    area-law acceptance gates (check.py)."""
    from tests.helpers import planar_nozzle_gates
    hist = np.loadtxt(GOLD / "planar_nozzle_residuals.txt")
    cs = cases.planar_nozzle()
    opts = make_options(cs)
    s = oracle.solver(opts, [cs])
    try:
        done = 0
        for it, res in hist[:-1]:
            info = s.step(int(it) - done, check=False)[0]
            done = int(it)
            assert info["iter"] == it and info["err"] == 0
            assert abs(info["residual"][0] / res - 1.0) < 0.05, (it, info["residual"][0], res)
        info = s.solve(steps_per_call=1)
        assert abs(info["iter"] - hist[-1, 0]) <= 5 and info["residual"][0] <= 1e-10
        planar_nozzle_gates(s.prim(), cs.meta["xc"], opts.gas_gamma)
    finally:
        s.close()


def test_chang_nozzle_axisymmetric_matches_reference_data():
    """The reference's chang-nozzle case (axisymmetric source, IRS, stagnation inflow) through
    the oracle: it converges (density residual below the case's 1e-6 sentinel within its 5000
    iterations) and the Mach number along the wall and the axis passes the case's gates against
    Chang's data (mean relative error < 5e-2, maximum < 1e-1)."""
    from tests.helpers import chang_nozzle_case, chang_nozzle_gates
    cs = chang_nozzle_case()
    s = oracle.solver(make_options(cs), [cs])
    try:
        info = s.solve(steps_per_call=500)
        assert info["err"] == 0 and info["residual"][0] < 1e-6, info
        chang_nozzle_gates(cs, s.prim())
    finally:
        s.close()


def test_sd_tramel_known_answers():
    """SD_Tramel (Lib_Shock_Detector.f90:14-38): 1 on a uniform or linear pressure stencil, 0 at
    and above the switch max(kp1, kp2) = 1/20, 1 - tanh(10 (sw/20)^3) below it, symmetric in the
    two directions."""
    lib = oracle.load()
    sd = lib.q2d_oracle_sd_tramel
    assert sd(1.0, 1.0, 1.0, 1.0, 1.0) == 1.0
    assert sd(2.0, 1.0, 3.0, 2.0, 2.0) == 1.0          # linear in i: no second difference
    assert sd(1.0, 1.0, 2.0, 1.0, 1.0) == 0.0          # kp1 = 1/5
    assert sd(1.0, 1.0, 1.0, 1.0, 2.0) == 0.0          # kp2 = 1/5
    for p2 in (1.01, 1.1, 1.2):
        sw = (p2 - 1.0) / (p2 + 3.0)
        want = 1.0 - np.tanh(10.0 * (sw / 20.0) ** 3) if sw < 0.05 else 0.0
        assert sd(1.0, 1.0, p2, 1.0, 1.0) == pytest.approx(want, rel=0, abs=1e-16)
        assert sd(1.0, 1.0, 1.0, 1.0, p2) == sd(1.0, 1.0, p2, 1.0, 1.0)
    # the switch: sw = 1/20 exactly (p2 = 23/19 gives (p2 - 1) / (p2 + 3) = 4/80) is a shock
    assert sd(1.0, 1.0, 1.0 + 4.0 / 19.0 - 1e-12, 1.0, 1.0) > 0.999999
    assert sd(1.0, 1.0, 1.0 + 4.0 / 19.0 + 1e-12, 1.0, 1.0) == 0.0


def test_ramp_channel_matches_reference_calibration():
    """The reference's ramp-channel case (Mach 3 over a 30-degree ramp: MUSCL-SD with minmod,
    HLLE, IRS beta 0.5, CFL 0.9 after a 100-iteration ramp) through the oracle: after 1500 of its
    10000 iterations the density residual is below the case's 1e-3 gate, the oblique-shock gates
    of its check.py pass, the sensor field passes its localisation gates, and the post / pre-shock
    errors against the theory equal those check.py records for the reference binary (p2/p1
    -0.002 %, T2/T1 +0.95 %, rho2/rho1 -0.94 %, M2 -0.94 %) to the digits it gives."""
    from tests.helpers import ramp_channel_case, ramp_channel_gates, sensor_field
    cs = ramp_channel_case()
    s = oracle.solver(make_options(cs), [cs])
    try:
        info = s.step(1500)[0]
        prim = s.prim()
    finally:
        s.close()
    assert info["err"] == 0 and info["iter"] == 1500 and info["residual"][0] < 1e-3, info
    beta = sensor_field(cs, [prim])[0]
    errs = 100.0 * np.array(ramp_channel_gates(cs, prim, beta))
    assert abs(errs[0] - (-0.002)) < 0.005, errs
    assert np.all(np.abs(errs[1:] - np.array([0.95, -0.94, -0.94])) < 0.01), errs


def riemann_sd(kind, L, R, beta, nx=1.0, ny=0.0):
    import ctypes as C
    lib = oracle.load()
    opt = make_options({})
    a = (C.c_double * 4)(*L)
    b = (C.c_double * 4)(*R)
    out = (C.c_double * 4)()
    lib.q2d_oracle_riemann_sd(kind, C.byref(opt), a, b, beta, nx, ny, out)
    return np.array(out[:])


def test_sensor_driven_riemann_known_answers():
    """HLLC+ (riemann_HLLCSD, Lib_Riemann_HLL.f90:572-605) is HLLE where the sensor is 0, HLLC
    where it is 1 and their beta-weighted blend between. HLLE++ (riemann_HLLEpp, :437-533) is
    consistent (F(U, U) the physical flux) for every beta; with beta = 0 its eigenvalues are the
    HLLE ones written in Roe waves, so it equals HLLE; with beta = 1 it is Roe's flux, which keeps
    a stationary contact exactly (no mass flux), where HLLE diffuses it."""
    rng = np.random.default_rng(17)
    for _ in range(20):
        L = [rng.uniform(0.2, 3), rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(0.2, 5)]
        R = [rng.uniform(0.2, 3), rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(0.2, 5)]
        th = rng.uniform(0, 2 * np.pi)
        n = (np.cos(th), np.sin(th))
        hllc, hlle = riemann(0, L, R, *n), riemann(1, L, R, *n)
        assert np.array_equal(riemann_sd(5, L, R, 1.0, *n), hllc)
        assert np.array_equal(riemann_sd(5, L, R, 0.0, *n), hlle)
        b = rng.uniform(0.01, 0.99)
        assert np.allclose(riemann_sd(5, L, R, b, *n), b * hllc + (1 - b) * hlle, rtol=1e-13, atol=1e-13)
        scale = np.abs(hlle).max()
        assert np.allclose(riemann_sd(6, L, R, 0.0, *n), hlle, rtol=1e-11, atol=1e-11 * scale)
        for beta in (0.0, 0.3, 1.0):
            assert np.allclose(riemann_sd(6, L, L, beta, *n), phys_flux(L, *n), rtol=1e-12, atol=1e-12)
    L, R = [1.0, 0.0, 0.3, 1.0], [0.25, 0.0, 0.3, 1.0]      # stationary contact, tangential flow
    assert abs(riemann_sd(6, L, R, 1.0)[0]) < 1e-15
    assert abs(riemann_sd(5, L, R, 1.0)[0]) < 1e-15          # HLLC resolves it too
    assert riemann_sd(6, L, R, 0.0)[0] > 1e-3               # HLLE does not


@pytest.mark.parametrize("riem", ["HLLC+", "HLLE++"])
def test_ramp_channel_sensor_driven_solvers(riem):
    """The ramp-channel case with the sensor-driven solvers of the reference's solver sweep
    (ramp-channel/Q2D.sh: HLLE, HLLC, HLLC+, SLAU) in place of HLLE: after 1500 iterations the
    residual is below 1e-3 and the oblique-shock and sensor gates of its check.py pass."""
    from tests.helpers import ramp_channel_case, ramp_channel_gates, sensor_field
    cs = ramp_channel_case()
    s = oracle.solver(make_options(cs, riemann=riem), [cs])
    try:
        info = s.step(1500)[0]
        prim = s.prim()
    finally:
        s.close()
    assert info["err"] == 0 and info["residual"][0] < 1e-3, info
    ramp_channel_gates(cs, prim, sensor_field(cs, [prim])[0])


REMAINING = ["HLLEM", "HLLC Rotated", "PLLF", "exact", "Hanel", "AUSM+", "AUSM+-up", "AUSM+-up2"]


def riemann_kw(kind, L, R, nx=1.0, ny=0.0, minf=0.1):
    import ctypes as C
    lib = oracle.load()
    opt = make_options({}, riemann_minf=minf)
    a = (C.c_double * 4)(*L)
    b = (C.c_double * 4)(*R)
    out = (C.c_double * 4)()
    lib.q2d_oracle_riemann_sd(kind, C.byref(opt), a, b, 1.0, nx, ny, out)
    return np.array(out[:])


def test_remaining_riemann_known_answers():
    """The rest of Assign_Riemann_Solver's solvers (HLLEM, rotated HLLC, PLLF, exact, Hanel,
    AUSM+, AUSM+-up, AUSM+-up2): consistent (F(U, U) is the physical flux) in any direction;
    the exact solver keeps a stationary contact (no mass flux), and HLLEM's antidiffusion removes
    most of the mass flux HLLE puts across it (its weight a / (a + |S1 + S4| / 2) stays below 1
    when the wave speeds are not symmetric); the exact solver's Godunov flux for Sod (rho
    1/0.125, p 1/0.1, at rest; the left fan's tail u* - a*_L < 0, so x/t = 0 is in the left star
    region) is the flux of the left star state, p* and u* from the reference's own exact solver
    (test/common/pycheck/q2d_exact1d.py, riemann_exact.npz), rho*_L = rho_L (p* / p_L)^(1 /
    gamma)."""
    rng = np.random.default_rng(23)
    for kind in range(7, 15):
        for _ in range(20):
            P = [rng.uniform(0.2, 3), rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(0.2, 5)]
            th = rng.uniform(0, 2 * np.pi)
            n = (np.cos(th), np.sin(th))
            F = riemann_kw(kind, P, P, *n)
            assert np.allclose(F, phys_flux(P, *n), rtol=1e-10, atol=1e-10), (kind, F, phys_flux(P, *n))
    L, R = [1.0, 0.0, 0.3, 1.0], [0.25, 0.0, 0.3, 1.0]
    assert abs(riemann_kw(10, L, R)[0]) < 1e-15
    hlle, hllem = riemann(1, L, R)[0], riemann_kw(7, L, R)[0]
    assert 0.0 < hllem < 0.5 * hlle, (hllem, hlle)   # antidiffusion weight a / (a + |S1 + S4| / 2) < 1
    ps, us = np.load(GOLD / "riemann_exact.npz")["toro1_pstar_ustar"]
    F = riemann_kw(10, [1.0, 0.0, 0.0, 1.0], [0.125, 0.0, 0.0, 0.1])
    assert np.allclose(F, phys_flux([ps ** (1.0 / 1.4), us, 0.0, ps], 1.0, 0.0), rtol=1e-6, atol=0), F


@pytest.mark.parametrize("riem", REMAINING)
def test_sod79_remaining_solvers(riem):
    """Sod at 400 cells with MC and each remaining solver (CFL 0.5; 0.2 for AUSM+-up and
    AUSM+-up2, Minf 0.1) meets the Sod79 check.py error gates (relative L1 of rho < 5e-3, of
    p < 3.5e-3) against the reference's exact.txt."""
    kw = dict(cfl=0.2, riemann_minf=0.1) if "up" in riem else dict(cfl=0.5)
    P, info = run_oracle(sod79(riem), riemann=riem, **kw)
    l1r, l1p = sod79_l1(P)
    assert info["todo"] == 3 and l1r < 5e-3 and l1p < 3.5e-3, (l1r, l1p)


def test_ausm_up_needs_minf():
    """AUSM+-up / AUSM+-up2 without riemann-options-Minf are refused (Assign_Setup.f90:108-112)."""
    cs = sod79("AUSM+-up")
    for riem in ("AUSM+-up", "AUSM+-up2"):
        with pytest.raises(Exception):
            oracle.solver(make_options(cs, riemann=riem), [cs])
