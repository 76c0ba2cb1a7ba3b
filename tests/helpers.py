"""Drivers shared by the parity tests: run the same cases through the CUDA library and the
oracle and return their primitive states."""
from __future__ import annotations

import numpy as np

from q2d_b200 import make_options
from q2d_b200.solver import Q2DSolver


def run_pair(cases, steps: int, chunks: int = 1, schedule=None, thermo_table=None, **opt_overrides):
    """Advances the cases `steps` steps on both implementations (in `chunks` calls; the CUDA
    library on `schedule` when given; both on the thermally perfect gas of thermo_table when
    given) and returns (gpu_states, oracle_states, gpu_infos, oracle_infos); states are lists over
    cases of lists over blocks of (nj, ni, 4) arrays."""
    from oracle import oracle
    opts = make_options(cases[0], **opt_overrides)
    g = Q2DSolver(opts, cases, thermo_table=thermo_table)
    if schedule is not None:
        g.set_schedule(schedule)
    o = oracle.solver(opts, cases, thermo_table=thermo_table)
    try:
        per = max(1, steps // chunks)
        done = 0
        gi = oi = None
        while done < steps:
            n = min(per, steps - done)
            gi = g.step(n, check=False)
            oi = o.step(n, check=False)
            done += n
        gs = [[g.prim(c, b) for b in range(len(cs.blocks))] for c, cs in enumerate(cases)]
        os_ = [[o.prim(c, b) for b in range(len(cs.blocks))] for c, cs in enumerate(cases)]
        return gs, os_, gi, oi
    finally:
        g.close()
        o.close()


def planar_nozzle_gates(prim, xc, gamma):
    """The acceptance gates of the reference's planar-nozzle case (test/2D/euler/planar-nozzle/
    check.py): the column-averaged Mach number of the converged state against the quasi-1D
    isentropic area law, exit cell within 2e-3, cells more than 0.05 from the throat within
    5e-3, every cell but the two at each end within 1.5e-2 (relative); positive rho and p.
    Returns (exit, smooth, whole) relative errors."""
    from q2d_b200 import cases
    assert np.all(prim[..., 0] > 0) and np.all(prim[..., 3] > 0) and np.all(np.isfinite(prim))
    rho, u, p = prim[..., 0].mean(axis=0), prim[..., 1].mean(axis=0), prim[..., 3].mean(axis=0)
    mach = u / np.sqrt(gamma * p / rho)
    exact = cases.mach_of_area(cases.planar_nozzle_area(xc), xc > 0.4, gamma)
    rel = np.abs(mach - exact) / exact
    n = len(xc)
    interior = (xc > 2.0 / n) & (xc < 1.0 - 2.0 / n)
    smooth = interior & (np.abs(xc - 0.4) > 0.05)
    errs = (float(rel[-1]), float(rel[smooth].max()), float(rel[interior].max()))
    assert errs[0] < 2e-3 and errs[1] < 5e-3 and errs[2] < 1.5e-2, errs
    return errs


def chang_nozzle_case():
    """The reference's chang-nozzle case (test/2D/euler/chang-nozzle: input.ini, INPUT/) from the
    committed fixture: axisymmetric converging-diverging nozzle, 190 x 40 cells, stagnation
    inflow (BC 401), extrapolation outflow (400), axis and wall symmetry (300), MC + HLLC,
    SSP-RK3, CFL 0.8, IRS beta 0.5, local time steps, at most 5000 iterations; the air of its
    phase.txt (W = 28.970418) with gamma 1.4."""
    from pathlib import Path
    from q2d_b200 import cases
    from q2d_b200.cases import BlockSpec, CaseSpec, edge_records, stagnation_props
    f = np.load(Path(__file__).resolve().parent / "golden" / "chang_nozzle.npz")
    nodes, prim = f["nodes"], f["prim"]
    nj, ni = prim.shape[:2]
    T0, p0 = (float(v) for v in f["T0_p0"])
    blk = BlockSpec(ni, nj, nodes, prim)
    bcs = edge_records(1, ni, nj, {1: (401, stagnation_props(T0, p0)), 2: (400, {}), 3: (300, {}), 4: (300, {})})
    opts = dict(limiter="mc", riemann="HLLC", n_rk=3, cfl=0.8, time_accurate=0, irs_beta=0.5,
                source="axisymmetric", itermax=5000, gas_R=8314.46 / 28.970418, gas_gamma=1.4)
    return CaseSpec("chang_nozzle", [blk], bcs, opts, {"axis": f["axis_mach"], "wall": f["wall_mach"]})


def chang_nozzle_gates(cs, prim):
    """The chang-nozzle acceptance gates (test/2D/euler/chang-nozzle/check.py): Mach number in
    the wall row and in the axis row of cells, at the x of each column's first node, against
    Chang's (1996) data: mean relative error below 5e-2 and maximum below 1e-1 on both; positive
    density and pressure. Returns the four errors."""
    assert np.all(prim[..., 0] > 0) and np.all(prim[..., 3] > 0) and np.all(np.isfinite(prim))
    g = cs.options["gas_gamma"]
    mach = np.sqrt(prim[..., 1] ** 2 + prim[..., 2] ** 2) / np.sqrt(g * prim[..., 3] / prim[..., 0])
    ni = prim.shape[1]
    nodes = cs.blocks[0].nodes
    out = []
    for row, xrow, ref in ((-1, nodes[-1, :ni, 0], cs.meta["wall"]), (0, nodes[0, :ni, 0], cs.meta["axis"])):
        r = np.interp(xrow, ref[:, 0], ref[:, 1])
        eps = np.abs(mach[row] - r) / np.maximum(np.abs(r), 1e-3)
        out += [float(eps.mean()), float(eps.max())]
    assert out[0] < 5e-2 and out[2] < 5e-2 and out[1] < 1e-1 and out[3] < 1e-1, out
    return out


def ramp_channel_case():
    """The reference's ramp-channel case (test/2D/euler/ramp-channel: input.ini, INPUT/) from the
    committed fixture: Mach 3 flow over a 30-degree ramp in a channel, 95 x 100 cells, supersonic
    inflow (BC 405: M 3, T 1, p 1), extrapolation outflow (400), symmetry walls (300), MUSCL-SD
    with minmod + HLLE, SSP-RK3, CFL 0.9 reached over 100 iterations, IRS beta 0.5, local time
    steps, 10000 iterations; the air of its phase.txt (W = 28.970418) with gamma 1.4."""
    from pathlib import Path
    from q2d_b200.cases import BlockSpec, CaseSpec, edge_records, supersonic_props
    f = np.load(Path(__file__).resolve().parent / "golden" / "ramp_channel.npz")
    nodes, prim = f["nodes"], f["prim"]
    nj, ni = prim.shape[:2]
    mach, T, p = (float(v) for v in f["mach_T_p"])
    blk = BlockSpec(ni, nj, nodes, prim)
    bcs = edge_records(1, ni, nj, {1: (405, supersonic_props(mach, T, p)), 2: (400, {}), 3: (300, {}),
                                   4: (300, {})})
    opts = dict(limiter="minmod", riemann="HLLE", n_rk=3, cfl=0.9, rampa_iter=100, time_accurate=0,
                irs_beta=0.5, shock_detector=1, itermax=10000, gas_R=8314.46 / 28.970418, gas_gamma=1.4)
    return CaseSpec("ramp_channel", [blk], bcs, opts, {"mach": mach})


def prandtl_meyer_case():
    """The reference's prandtl-meyer case (test/2D/euler/prandtl-meyer: input.ini, INPUT/) from the
    committed fixture: Mach 2 flow turning round a convex corner, 50 x 50 cells, supersonic inflow
    (BC 405: M 2, T 1, p 1) on face 1, extrapolation (400) on faces 2 and 3, symmetry (300) on
    face 4; MUSCL van Leer + HLLE, SSP-RK3, CFL 1.0, IRS beta 0.5, local time steps, 2500
    iterations; the air of its phase.txt (W = 28.970418) with gamma 1.4."""
    from pathlib import Path
    from q2d_b200.cases import BlockSpec, CaseSpec, supersonic_props
    f = np.load(Path(__file__).resolve().parent / "golden" / "prandtl_meyer.npz")
    nodes, prim = f["nodes"], f["prim"]
    nj, ni = prim.shape[:2]
    bcs = []
    for row in f["bcs"]:
        b, i, j, fc, typ = (int(x) for x in row[:5])
        r = {"b": b, "i": i, "j": j, "f": fc, "type": typ}
        if typ == 405:
            r.update(supersonic_props(float(row[5]), float(row[6]), float(row[7])))
        bcs.append(r)
    opts = dict(limiter="vanleer", riemann="HLLE", n_rk=3, cfl=1.0, time_accurate=0, irs_beta=0.5,
                itermax=2500, gas_R=8314.46 / 28.970418, gas_gamma=1.4)
    return CaseSpec("prandtl_meyer", [BlockSpec(ni, nj, nodes, prim)], bcs, opts, {"mach": 2.0})


def prandtl_meyer_exit_mach(M1: float = 2.0, theta_deg: float = 34.971, g: float = 1.4) -> float:
    """The exit Mach number of the case's check.py: the Prandtl-Meyer expansion of M1 by
    theta (nu(M2) = nu(M1) + theta), by bisection."""
    import math

    def nu(M):
        return math.sqrt((g + 1) / (g - 1)) * math.atan(math.sqrt((g - 1) / (g + 1) * (M * M - 1))) - \
            math.atan(math.sqrt(M * M - 1))
    target = nu(M1) + math.radians(theta_deg)
    lo, hi = 1.01, 30.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if nu(mid) < target:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def oblique_shock(M1: float, delta: float, g: float):
    """Weak oblique-shock solution for a wedge of angle delta (radians): the theta-beta-Mach
    relation tan(delta) = 2 cot(b) (M1^2 sin^2 b - 1) / (M1^2 (g + cos 2b) + 2) solved for the
    smallest b above the Mach angle, then the normal-shock relations on M1 sin(b). Returns
    (M2, b, p2/p1, T2/T1, rho2/rho1)."""
    def tan_delta(b):
        return 2.0 / np.tan(b) * (M1 ** 2 * np.sin(b) ** 2 - 1.0) / (M1 ** 2 * (g + np.cos(2.0 * b)) + 2.0)
    mu = np.arcsin(1.0 / M1)
    bs = np.linspace(mu, 0.5 * np.pi, 20001)
    k = int(np.argmax(tan_delta(bs) >= np.tan(delta)))
    assert k > 0, "detached shock"
    lo, hi = bs[k - 1], bs[k]
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if tan_delta(mid) < np.tan(delta) else (lo, mid)
    b = 0.5 * (lo + hi)
    mn1 = M1 * np.sin(b)
    p21 = 1.0 + 2.0 * g / (g + 1.0) * (mn1 ** 2 - 1.0)
    r21 = (g + 1.0) * mn1 ** 2 / ((g - 1.0) * mn1 ** 2 + 2.0)
    mn2 = np.sqrt((mn1 ** 2 + 2.0 / (g - 1.0)) / (2.0 * g / (g - 1.0) * mn1 ** 2 - 1.0))
    return mn2 / np.sin(b - delta), b, p21, p21 / r21, r21


def ramp_channel_gates(cs, prim, beta=None):
    """The ramp-channel acceptance gates (test/2D/euler/ramp-channel/check.py), with the grid
    indices of its probes: (1) post / pre-shock ratios against the weak oblique-shock theory for
    the ramp angle measured from wall nodes 20..50 (pre-shock probe cells i 5:15, j 70:90; post-
    shock plateau cells i 36:48, j 0:12): p2/p1 within 1 %, T2/T1, rho2/rho1 and M2 within 2 %;
    (2) with the sensor field beta: it differentiates, >= 1 % of the cells below 0.99, >= 90 % of
    the cells below 0.5 downstream of the ramp tip, mean > 0.99 over cells i 2:12, j 40:60 and
    <= 2 % of the cells upstream of the tip below 0.5; (4) positive density and pressure. Returns
    the four signed relative errors of (1)."""
    assert np.all(np.isfinite(prim)) and np.all(prim[..., 0] > 0) and np.all(prim[..., 3] > 0)
    g, R = cs.options["gas_gamma"], cs.options["gas_R"]
    nodes = cs.blocks[0].nodes                       # (nj + 1, ni + 1, 2)
    delta = np.arctan2(nodes[0, 50, 1] - nodes[0, 20, 1], nodes[0, 50, 0] - nodes[0, 20, 0])
    m2_th, _, p21_th, t21_th, r21_th = oblique_shock(cs.meta["mach"], delta, g)
    pre, post = prim[70:90, 5:15], prim[0:12, 36:48]
    rho1, p1 = pre[..., 0].mean(), pre[..., 3].mean()
    T1 = (pre[..., 3] / (pre[..., 0] * R)).mean()
    rho2, p2 = post[..., 0].mean(), post[..., 3].mean()
    T2 = (post[..., 3] / (post[..., 0] * R)).mean()
    u2, v2 = post[..., 1].mean(), post[..., 2].mean()
    m2 = np.hypot(u2, v2) / np.sqrt(g * R * T2)
    errs = [p2 / p1 / p21_th - 1.0, T2 / T1 / t21_th - 1.0, rho2 / rho1 / r21_th - 1.0, m2 / m2_th - 1.0]
    assert abs(errs[0]) < 0.01 and max(map(abs, errs[1:])) < 0.02, errs
    if beta is not None:
        assert np.all(np.isfinite(beta)) and beta.max() > beta.min()
        assert (beta < 0.99).sum() >= beta.size // 100
        xc = 0.25 * (nodes[:-1, :-1, 0] + nodes[:-1, 1:, 0] + nodes[1:, :-1, 0] + nodes[1:, 1:, 0])
        x_tip = nodes[0, 20, 0]
        shock = beta < 0.5
        assert shock.any() and (xc[shock] > x_tip).mean() >= 0.90
        assert beta[40:60, 2:12].mean() > 0.99
        up = xc < x_tip
        assert (shock & up).sum() / max(up.sum(), 1) <= 0.02
    return errs


def sensor_field(cs, prims) -> list:
    """The shock sensor beta (SD_Tramel) of every block of a case for the given interior states
    ([block] -> (nj, ni, 4)), from the oracle's ghost fill: the field the reference writes as
    'beta' to its diagnostic output. Returns [block] -> (nj, ni)."""
    import ctypes as C
    import dataclasses
    from oracle import oracle
    blocks = [dataclasses.replace(b, prim=np.ascontiguousarray(p)) for b, p in zip(cs.blocks, prims)]
    cs2 = dataclasses.replace(cs, blocks=blocks)
    o = oracle.solver(make_options(cs2), [cs2])
    try:
        out = []
        for k, b in enumerate(blocks):
            beta = np.empty((b.nj, b.ni))
            st = o.lib.q2d_oracle_shock_sensor(o.ctx, o.block_ids[0][k], beta.ctypes.data_as(C.POINTER(C.c_double)))
            assert st == 0, st
            out.append(beta)
        return out
    finally:
        o.close()


def split_case(cs, icuts=(), jcuts=()):
    """A single-block case cut into a grid of blocks stitched by block-interface records (BC 101,
    identity orientation) at the interior node lines icuts (i) and jcuts (j); the original edge
    records go to the blocks that own their cells."""
    import dataclasses
    from q2d_b200.cases import BlockSpec
    (b0,) = cs.blocks
    ib = [0, *icuts, b0.ni]
    jb = [0, *jcuts, b0.nj]
    nI, nJ = len(ib) - 1, len(jb) - 1
    bid = lambda I, J: J * nI + I + 1   # noqa: E731
    blocks, bcs = [], []
    for J in range(nJ):
        for I in range(nI):
            i0, i1, j0, j1 = ib[I], ib[I + 1], jb[J], jb[J + 1]
            blocks.append(BlockSpec(i1 - i0, j1 - j0, b0.nodes[j0:j1 + 1, i0:i1 + 1].copy(),
                                    b0.prim[j0:j1, i0:i1].copy()))
    for r in cs.bcs:   # edge records of the original block, in face order
        i, j = r["i"] - 1, r["j"] - 1
        I = max(k for k in range(nI) if ib[k] <= i)
        J = max(k for k in range(nJ) if jb[k] <= j)
        rr = dict(r, b=bid(I, J), i=i - ib[I] + 1, j=j - jb[J] + 1)
        bcs.append(rr)
    conn = dict(d11=1, d12=0, d21=0, d22=1)
    for J in range(nJ):
        for I in range(nI):
            ni, nj = ib[I + 1] - ib[I], jb[J + 1] - jb[J]
            if I > 0:
                nl = ib[I] - ib[I - 1]
                bcs += [dict(b=bid(I, J), i=1, j=k, f=1, type=101, bs=bid(I - 1, J), is_=nl, js=k, fs=2, **conn)
                        for k in range(1, nj + 1)]
            if I < nI - 1:
                bcs += [dict(b=bid(I, J), i=ni, j=k, f=2, type=101, bs=bid(I + 1, J), is_=1, js=k, fs=1, **conn)
                        for k in range(1, nj + 1)]
            if J > 0:
                nl = jb[J] - jb[J - 1]
                bcs += [dict(b=bid(I, J), i=k, j=1, f=3, type=101, bs=bid(I, J - 1), is_=k, js=nl, fs=4, **conn)
                        for k in range(1, ni + 1)]
            if J < nJ - 1:
                bcs += [dict(b=bid(I, J), i=k, j=nj, f=4, type=101, bs=bid(I, J + 1), is_=k, js=1, fs=3, **conn)
                        for k in range(1, ni + 1)]
    bcs.sort(key=lambda r: (r["b"], r["f"], r["j"] if r["f"] <= 2 else r["i"]))
    return dataclasses.replace(cs, name=cs.name + "_split", blocks=blocks, bcs=bcs)


def linear_cp_table(a: float = 1000.0, b: float = 0.2, ntab: int = 5000):
    """A thermally perfect gas with cp(T) = a + b T [J/(kg K)]: the table of cp and of
    h(T) = a T + b T^2 / 2 on the knots T = 0, 1, .. ntab-1 K (h exact at the knots)."""
    T = np.arange(ntab, dtype=np.float64)
    return a * T + 0.5 * b * T * T, a + b * T


def constant_cp_table(gamma: float = 1.4, R: float = 287.0, ntab: int = 5000):
    """The calorically perfect gas written as a table: cp = gamma R / (gamma - 1), h = cp T."""
    cp = gamma * R / (gamma - 1.0)
    T = np.arange(ntab, dtype=np.float64)
    return cp * T, np.full(ntab, cp)
