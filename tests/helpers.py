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
