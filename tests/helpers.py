"""Drivers shared by the parity tests: run the same cases through the CUDA library and the
oracle and return their primitive states."""
from __future__ import annotations

import numpy as np

from q2d_b200 import make_options
from q2d_b200.solver import Q2DSolver


def run_pair(cases, steps: int, chunks: int = 1, **opt_overrides):
    """Advances the cases `steps` steps on both implementations (in `chunks` calls) and returns
    (gpu_states, oracle_states, gpu_infos, oracle_infos); states are lists over cases of lists
    over blocks of (nj, ni, 4) arrays."""
    from oracle import oracle
    opts = make_options(cases[0], **opt_overrides)
    g = Q2DSolver(opts, cases)
    o = oracle.solver(opts, cases)
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
