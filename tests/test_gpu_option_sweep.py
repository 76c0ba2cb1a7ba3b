"""Seeded sweep over the option space of the FP64 form against the oracle: for 24 drawn
combinations of limiter, Riemann solver, MUSCL-SD, implicit residual smoothing, RK scheme and
schedule, on the developed ramp-channel flow cut into 2 x 2 blocks (shocks across the block and
tile edges) or on a multi-block axisymmetric nozzle, two steps agree with the oracle to 1e-10
relative L-infinity; 16 more draws in the FP32-flux form on its five tiles against the FP64 form
to 1e-6 relative L1. A draw whose flow leaves the physical states (both implementations report
it) is skipped in favour of the next."""
import numpy as np
import pytest

from q2d_b200 import cases
from tests.helpers import run_pair
from tests.test_gpu_sd import check, developed  # noqa: F401  (module fixture)

pytestmark = pytest.mark.gpu

LIMITERS = ["iord", "minmod", "vanleer", "vanalbada", "mc", "superbee", "LIMO3"]
SOLVERS = ["HLLC", "HLLE", "LLF", "SLAU", "SLAU2", "HLLC+", "HLLE++", "HLLEM", "HLLC Rotated", "PLLF",
           "exact", "Hanel", "AUSM+", "AUSM+-up", "AUSM+-up2"]


def draws(n, seed=20261204):
    rng = np.random.default_rng(seed)
    for _ in range(n):
        yield dict(limiter=str(rng.choice(LIMITERS)), riemann=str(rng.choice(SOLVERS)),
                   shock_detector=int(rng.integers(0, 2)), irs_beta=float(rng.choice([0.0, 0.3, 0.5])),
                   n_rk=int(rng.integers(1, 4)), cfl=0.4, schedule=int(rng.integers(0, 3)),
                   case=int(rng.integers(0, 2)))


@pytest.mark.parametrize("k,d", list(enumerate(draws(24))))
def test_option_sweep_vs_oracle(developed, k, d):   # noqa: F811
    d = dict(d)
    case = d.pop("case")
    cs = developed[1] if case == 0 else cases.nozzle_axi(ni=36, nj=10, nblocks=2, seed=30 + k)
    if "up" in d["riemann"]:
        d["riemann_minf"] = 3.0 if case == 0 else 0.3
    gs, os_, gi, oi = run_pair([cs], 2, **d)
    if gi[0]["err"] or oi[0]["err"]:
        assert gi[0]["err"] == oi[0]["err"], (d, gi[0]["err"], oi[0]["err"])
        pytest.skip(f"non-physical state in both implementations: {d}")
    check(gs, os_, 1e-9 if d["riemann"] == "HLLC Rotated" else 1e-10, f"draw {k} {d}")


@pytest.mark.parametrize("k,d", list(enumerate(draws(16, seed=4821))))
def test_option_sweep_fp32flux_vs_fp64(developed, k, d):   # noqa: F811
    """The same kind of draws in the FP32-flux form on the FP32-flux kernel's five tiles against
    the FP64 form: <= 1e-6 relative L1 after 4 steps (2e-6 for the rotated HLLC)."""
    from q2d_b200 import make_options
    from q2d_b200.solver import Q2DSolver
    from tests.conftest import rel_l1
    d = dict(d)
    case, sch = d.pop("case"), 3 + k % 5
    d.pop("schedule")
    cs = developed[1] if case == 0 else cases.nozzle_axi(ni=36, nj=10, nblocks=2, seed=60 + k)
    if "up" in d["riemann"]:
        d["riemann_minf"] = 3.0 if case == 0 else 0.3
    out = []
    for prec, s_ in ((0, 0), (1, sch)):
        s = Q2DSolver(make_options(cs, precision=prec, **d), [cs])
        try:
            s.set_schedule(s_)
            info = s.step(4, check=False)[0]
            out.append((info["err"], s.prims()[0]))
        finally:
            s.close()
    if out[0][0] or out[1][0]:
        assert out[0][0] == out[1][0], (d, out[0][0], out[1][0])
        pytest.skip(f"non-physical state in both forms: {d}")
    tol = 2e-6 if d["riemann"] == "HLLC Rotated" else 1e-6
    for b, (x32, x64) in enumerate(zip(out[1][1], out[0][1])):
        err = rel_l1(x32, x64)
        assert err.max() <= tol, f"draw {k} {d} schedule {sch} block {b}: rel L1 {err}"
