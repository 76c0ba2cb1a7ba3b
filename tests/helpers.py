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
