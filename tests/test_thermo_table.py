"""Thermally perfect single-species gas on a table (q2d_gpu_set_thermo_table).

The reference takes h(T) and cp(T) from FLINT's tables, interpolated linearly at int(T)
(roe_averages, Lib_Riemann_HLL.f90:229-317; Compute_Prim_Residual, Lib_Newstate.f90:245-294),
with gamma(T) = cp / (cp - R), a = sqrt(gamma p / rho), e = h - R T (docs/theory/thermo.md:39-99).
FLINT is not part of the reference tree and no reference case uses a variable-cp table, so this
form is unpinned: it is checked against closed forms of its own.

* Known answers on the oracle: for cp = a + b T (h exact at the 1-K knots) and states at whole
  temperatures, the sound speeds, the Roe-averaged sound speed and total enthalpy and the HLLE
  flux equal their closed forms; rho E -> p inverts exactly from a guess 200 K off.
* A constant-cp table reproduces the calorically perfect closure (oracle and GPU).
* Variable cp changes the solution, conserves mass, momenta and energy on a periodic domain,
  and the GPU's plain FP64 form equals the oracle (<= 1e-12 after one step, <= 1e-10 after
  20) on a ramp (HLLC, BC 405 / 400 / 300), a nozzle with BC 401 and 406 and the area source
  (HLLE) and the periodic box (LLF).
* The table is refused outside the plain FP64 form with HLLC / HLLE / LLF.
"""
import copy
import ctypes as C

import numpy as np
import pytest

from q2d_b200 import _abi, cases, make_options
from q2d_b200.solver import Q2DError, Q2DSolver
from tests.conftest import cons, rel_linf
from tests.helpers import constant_cp_table, linear_cp_table, run_pair

R = 287.0
A_CP, B_CP = 1000.0, 0.2


def _oracle():
    from oracle import oracle
    return oracle


def closed_forms(L, Rs, nx, ny):
    """Closed forms for cp = A + B T, h = A T + B T^2 / 2 at the states' temperatures."""
    def thermo(P):
        T = P[3] / (P[0] * R)
        cp = A_CP + B_CP * T
        h = A_CP * T + 0.5 * B_CP * T * T
        return T, cp, h, np.sqrt(cp / (cp - R) * P[3] / P[0])
    Tl, cpl, hl, al = thermo(L)
    Tr, cpr, hr, ar = thermo(Rs)
    sl, sr = np.sqrt(L[0]), np.sqrt(Rs[0])
    w = lambda a, b: (sr * b + sl * a) / (sl + sr)
    u, v, T = w(L[1], Rs[1]), w(L[2], Rs[2]), w(Tl, Tr)
    h0l = hl + 0.5 * (L[1] ** 2 + L[2] ** 2)
    h0r = hr + 0.5 * (Rs[1] ** 2 + Rs[2] ** 2)
    h0 = w(h0l, h0r)
    cv = 0.5 * (cpl + cpr) - R
    ei = w(hl - R * Tl, hr - R * Tr)
    a_roe = np.sqrt(R / cv * (h0 - 0.5 * (u * u + v * v) + cv * T - ei))
    unl, unr, un = L[1] * nx + L[2] * ny, Rs[1] * nx + Rs[2] * ny, u * nx + v * ny
    S1 = min(0.0, unl - al, un - a_roe)
    S4 = max(0.0, unr + ar, un + a_roe)
    UL = np.array([L[0], L[0] * L[1], L[0] * L[2], L[0] * h0l - L[3]])
    UR = np.array([Rs[0], Rs[0] * Rs[1], Rs[0] * Rs[2], Rs[0] * h0r - Rs[3]])
    FL = np.array([L[0] * unl, L[0] * unl * L[1] + L[3] * nx, L[0] * unl * L[2] + L[3] * ny, L[0] * unl * h0l])
    FR = np.array([Rs[0] * unr, Rs[0] * unr * Rs[1] + Rs[3] * nx, Rs[0] * unr * Rs[2] + Rs[3] * ny,
                   Rs[0] * unr * h0r])
    F = (S4 * FL - S1 * FR + S1 * S4 * (UR - UL)) / (S4 - S1)
    return dict(al=al, ar=ar, a_roe=a_roe, h0_roe=h0, hlle=F, rhoE=UL[3])


def state(rho, u, v, T):
    return np.array([rho, u, v, rho * R * T])


@pytest.mark.parametrize("TL,TR", [(400.0, 700.0), (300.0, 1500.0), (2000.0, 250.0)])
def test_known_answers_linear_cp(TL, TR):
    o = _oracle().load()
    h, cp = linear_cp_table(A_CP, B_CP)
    opts = _abi.default_options(gas_R=R, gas_gamma=1.4)
    L, Rs = state(1.2, 120.0, 25.0, TL), state(0.8, -30.0, 5.0, TR)
    nx, ny = 0.8, 0.6
    out = np.zeros(10)
    st = o.q2d_oracle_thermo_tab(_abi.RIEMANN["HLLE"], C.byref(opts), len(h), _abi.dptr(h), _abi.dptr(cp),
                                 _abi.dptr(L), _abi.dptr(Rs), nx, ny, _abi.dptr(out))
    assert st == _abi.OK
    ref = closed_forms(L, Rs, nx, ny)
    np.testing.assert_allclose(out[4:6], [ref["al"], ref["ar"]], rtol=1e-14)
    np.testing.assert_allclose(out[6], ref["a_roe"], rtol=1e-13)
    np.testing.assert_allclose(out[7], ref["h0_roe"], rtol=1e-14)
    np.testing.assert_allclose(out[0:4], ref["hlle"], rtol=1e-12, atol=1e-9 * np.abs(ref["hlle"]).max())
    np.testing.assert_allclose(out[8], ref["rhoE"], rtol=1e-14)
    np.testing.assert_allclose(out[9], L[3], rtol=1e-13)   # the inversion walked 200 K of knots


def test_between_knots_lerp():
    """Off the knots h and cp are the linear interpolants at int(T), so e(T) is piecewise linear
    and the pressure from rho E comes back exactly; gamma uses the interpolated cp."""
    o = _oracle().load()
    h, cp = linear_cp_table(A_CP, B_CP)
    opts = _abi.default_options(gas_R=R, gas_gamma=1.4)
    T = 537.3
    L, Rs = state(1.1, 40.0, 0.0, T), state(1.1, 40.0, 0.0, T)
    out = np.zeros(10)
    o.q2d_oracle_thermo_tab(0, C.byref(opts), len(h), _abi.dptr(h), _abi.dptr(cp), _abi.dptr(L), _abi.dptr(Rs),
                            1.0, 0.0, _abi.dptr(out))
    k, d = 537, T - 537
    hT = h[k] + (h[k + 1] - h[k]) * d
    cpT = cp[k] + (cp[k + 1] - cp[k]) * d
    np.testing.assert_allclose(out[4], np.sqrt(cpT / (cpT - R) * L[3] / L[0]), rtol=1e-14)
    np.testing.assert_allclose(out[8], L[0] * (hT - R * T) + 0.5 * L[0] * 40.0 ** 2, rtol=1e-14)
    np.testing.assert_allclose(out[9], L[3], rtol=1e-13)


def warm_box(seed=11, **opts):
    """The periodic box at about 300 K and 1e5 Pa with velocities of a few tens of m/s."""
    cs = copy.deepcopy(cases.periodic_box(40, 30, seed=seed, gas_R=R, **opts))
    P = cs.blocks[0].prim
    P[..., 0] *= 1.16
    P[..., 1:3] *= 300.0
    P[..., 3] *= 1.0e5
    return cs


def nozzle_406():
    from tests.test_gpu_boundaries import outflow_case
    return outflow_case("subsonic")


def run_oracle(cs, steps, table=None, **ov):
    s = _oracle().solver(make_options(cs, **ov), [cs], thermo_table=table)
    try:
        info = s.step(steps, check=False)[0]
        return [s.prim(0, b) for b in range(len(cs.blocks))], info
    finally:
        s.close()


@pytest.mark.parametrize("case", ["ramp", "nozzle_406"])
def test_constant_cp_table_is_the_perfect_gas_oracle(case):
    cs = cases.ramp(48, 16, seed=3) if case == "ramp" else nozzle_406()
    a, ia = run_oracle(cs, 20)
    b, ib = run_oracle(cs, 20, constant_cp_table(1.4, R))
    assert ia["err"] == ib["err"] == 0
    for x, y in zip(a, b):
        assert rel_linf(y, x).max() <= 1e-11


def test_variable_cp_changes_the_flow_and_conserves_oracle():
    cs = warm_box(riemann="HLLC")
    sur = cases.cell_areas(cs.blocks[0])
    tab = linear_cp_table(A_CP, B_CP)
    s = _oracle().solver(make_options(cs), [cs], thermo_table=tab)
    try:
        ho = _oracle().load()

        def totals(P):
            out = np.zeros(10)
            U = cons(P)   # mass and momenta do not depend on the closure
            Es = np.zeros(P.shape[:2])
            for j in range(P.shape[0]):
                for i in range(P.shape[1]):
                    ho.q2d_oracle_thermo_tab(0, C.byref(s.options), len(tab[0]), _abi.dptr(tab[0]),
                                             _abi.dptr(tab[1]), _abi.dptr(P[j, i].copy()),
                                             _abi.dptr(P[j, i].copy()), 1.0, 0.0, _abi.dptr(out))
                    Es[j, i] = out[8]
            U[..., 3] = Es
            return np.array([(U[..., k] * sur).sum() for k in range(4)]), \
                np.array([(np.abs(U[..., k]) * sur).sum() for k in range(4)])
        t0, m0 = totals(s.prim(0, 0))
        info = s.step(50, check=False)[0]
        assert info["err"] == 0
        P = s.prim(0, 0)
        t1, _ = totals(P)
        assert np.all(np.abs(t1 - t0) <= 1e-12 * m0), (t1 - t0) / m0
    finally:
        s.close()
    perfect, _ = run_oracle(cs, 50)
    assert np.abs(P - perfect[0]).max() / np.abs(perfect[0]).max(axis=(0, 1)).min() > 1e-6


def test_table_validation_oracle():
    o = _oracle().load()
    cs = cases.ramp(16, 6, seed=3)
    h, cp = linear_cp_table()
    for bad in (dict(precision=_abi.PREC_FP32_FLUX), dict(riemann="SLAU")):
        with pytest.raises(Q2DError):
            _oracle().solver(make_options(cs, **bad), [cs], thermo_table=(h, cp))
    with pytest.raises(Q2DError):   # cp <= R
        _oracle().solver(make_options(cs), [cs], thermo_table=(h, np.full_like(cp, 200.0)))
    assert o is not None


# ---- GPU ----------------------------------------------------------------------------------

GPU_CASES = {
    "ramp/HLLC": lambda: (cases.ramp(64, 20, seed=3), {}),
    "nozzle_406/HLLE": lambda: (nozzle_406(), dict(riemann="HLLE")),
    "box/LLF": lambda: (warm_box(riemann="LLF"), {}),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(GPU_CASES))
@pytest.mark.parametrize("schedule", ["tile 32x10", "tile 32x8", "tile 64x4"])
def test_gpu_equals_oracle_linear_cp(name, schedule):
    cs, ov = GPU_CASES[name]()
    tab = linear_cp_table(A_CP, B_CP)
    gs, os_, gi, oi = run_pair([cs], 1, schedule=schedule, thermo_table=tab, **ov)
    for g, o in zip(gs[0], os_[0]):
        assert rel_linf(g, o).max() <= 1e-12, name
    gs, os_, gi, oi = run_pair([cs], 20, chunks=2, schedule=schedule, thermo_table=tab, **ov)
    assert gi[0]["err"] == oi[0]["err"] == 0 and gi[0]["iter"] == oi[0]["iter"] == 20
    for g, o in zip(gs[0], os_[0]):
        assert np.all(np.isfinite(g)) and rel_linf(g, o).max() <= 1e-10, name
    perfect, _ = run_oracle(cs, 20, **ov)
    assert max(np.abs(g - p).max() / np.abs(p).max() for g, p in zip(gs[0], perfect)) > 1e-7


@pytest.mark.gpu
def test_gpu_constant_cp_table_is_the_perfect_gas():
    cs = nozzle_406()
    a = Q2DSolver(make_options(cs), [cs])
    b = Q2DSolver(make_options(cs), [cs], thermo_table=constant_cp_table(1.4, R))
    try:
        a.step(30)
        b.step(30)
        assert rel_linf(b.prim(0, 0), a.prim(0, 0)).max() <= 1e-11
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_gpu_table_refused_outside_the_fp64_hll_forms():
    cs = cases.ramp(16, 6, seed=3)
    tab = linear_cp_table()
    for bad in (dict(precision=_abi.PREC_FP32_FLUX), dict(riemann="SLAU"), dict(riemann="HLLC+")):
        with pytest.raises(Q2DError) as e:
            Q2DSolver(make_options(cs, **bad), [cs], thermo_table=tab)
        assert e.value.status == _abi.ERR_BADARG


@pytest.mark.gpu
def test_host_runs_a_variable_cp_thermo_dat(tmp_path):
    """q2d_host --gamma table with a temperature-dependent INPUT/thermo.dat runs the thermally
    perfect gas: its field equals the library's with the same table (to the 17 digits written)."""
    from q2d_b200 import refio
    from tests.test_host_harness import host
    cs = cases.ramp(40, 14, seed=3)
    tab = linear_cp_table(A_CP, B_CP, 3000)
    refio.write_case(cs, tmp_path, itermax=25, thermo_table=tab)
    host(tmp_path, "--gamma", "table", "--steps-per-call", 10, "--quiet")
    got = refio.read_field(tmp_path / "OUTPUT" / "field.tec")[0].prim
    s = Q2DSolver(make_options(cs, itermax=25), [cs], thermo_table=tab)
    try:
        s.step(25)
        want = s.prim(0, 0)
    finally:
        s.close()
    assert rel_linf(got, want).max() <= 1e-15
